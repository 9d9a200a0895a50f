"""tti_snapshot_static: the snapshot entry point that allocates no device
memory, for callers whose GPU memory must not grow when they need a snapshot
(a host application under a fixed GPU memory budget, or code running while
another stream of the process is being captured into a CUDA graph). It packs
through a static device array instead of the handle's staging buffer. Its
output must equal what the regular snapshot path (tti_run's callback)
delivers for the same wavefield, bit for bit, on consecutive calls; after the
first call on a device (which loads the array) device memory must not grow;
snapshots larger than the static array are refused; a capture of another
stream survives the call, and a handle whose own stream is being captured is
refused. Kept in a file that pytest collects last."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu


def _shot(ttifd, **over):
    cfg = dict(variant="coordinate_rotation", nz=80, nx=96, nt=121, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0,
               ealThick=8, freesurface=0, stype=1, wsave=0, savew=0)
    cfg.update(over)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=9)
    h = ttifd.Modeling(**cfg)
    h.upload_model(*synthetic.padded(m, cfg["ealThick"]))
    h.set_source([cfg["nx"] // 2], [20], synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])[None, :])
    h.run()
    return h


def test_static_snapshot_matches_run_callback(gpu_lib):
    import ttifd

    # nt - 1 is a multiple of snap_sample, so the last callback sees the final state
    cfg = dict(variant="tensor_rotation", nz=90, nx=120, nt=201, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0,
               ealThick=10, freesurface=1, stype=1, wsave=3, snap_sample=100, savew=0)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=5)
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    snaps = {}
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*synthetic.padded(m, cfg["ealThick"]))
        h.set_source([60], [4], w[None, :])
        h.run(lambda it, kind, a: snaps.__setitem__((it, kind), a))
        last = max(it for it, _ in snaps)
        assert last == cfg["nt"] - 1
        # two calls in a row, different kinds, then the first kind again
        for kind in (3, 1, 3):
            got = h.snapshot_static(kind)
            ref = snaps[(last, kind)]
            assert got.shape == ref.shape
            assert np.array_equal(got.view(np.uint32), ref.view(np.uint32)), f"kind {kind}"
            assert np.abs(ref).max() > 0


def test_static_snapshot_padded_area(gpu_lib):
    import ttifd

    cfg = dict(variant="coordinate_rotation", nz=64, nx=80, nt=101, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0,
               ealThick=8, stype=1, wsave=1, snap_sample=50, savew=1)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=6)
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    snaps = {}
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*synthetic.padded(m, cfg["ealThick"]))
        h.set_source([40], [30], w[None, :])
        h.run(lambda it, kind, a: snaps.__setitem__((it, kind), a))
        for kind in (2, 2):
            got = h.snapshot_static(kind)
            assert got.shape == (h.Nx, h.Nz)
            assert np.array_equal(got.view(np.uint32), snaps[(100, kind)].view(np.uint32))


def test_static_snapshot_rejects_oversize(gpu_lib):
    import ttifd

    # 4200 x 4100 physical cells > 16 Mi floats: refused before any GPU work
    with ttifd.Modeling(nz=4200, nx=4100, nt=2, dx=10.0, dz=10.0, dt=0.0008, fpeak=10.0, ealThick=0) as h:
        with pytest.raises(ttifd.TTIError) as e:
            h.snapshot_static(3)
        assert e.value.code == ttifd.ERR_ARG and "static buffer" in str(e.value)


def test_static_snapshot_does_not_grow_device_memory(gpu_lib):
    """After the first call on a device (which loads the array), a call on a
    handle that never allocated a snapshot buffer leaves free device memory
    exactly as it was."""
    import torch

    import ttifd

    with _shot(ttifd) as a:
        a.snapshot_static(1)  # first call on this device: loads the static array
    with _shot(ttifd) as b:
        torch.cuda.synchronize()
        free0, _ = torch.cuda.mem_get_info(0)
        for kind in (1, 3):
            got = b.snapshot_static(kind)
        torch.cuda.synchronize()
        free1, _ = torch.cuda.mem_get_info(0)
        assert free1 == free0, f"device memory changed by {free0 - free1} bytes"
        E = b.E
        vx = b.fetch_field(ttifd.F_VX)[E:b.Nx - E, E:b.Nz - E]
        assert np.array_equal(b.snapshot_static(1).view(np.uint32), vx.view(np.uint32))
        assert got.shape == vx.shape


@pytest.mark.parametrize("mode", ["global", "thread_local", "relaxed"])
def test_static_snapshot_while_another_stream_captures(gpu_lib, mode):
    """A capture on another stream (any capture mode) survives the call, and
    the snapshot is the same as without the capture."""
    import torch

    import ttifd

    with _shot(ttifd) as h:
        ref = h.snapshot_static(1)
        x = torch.zeros(1024, device="cuda:0")
        s = torch.cuda.Stream(device=0)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(s):
            g.capture_begin(capture_error_mode=mode)
            x.add_(1.0)
            got = h.snapshot_static(1)
            g.capture_end()
        g.replay()
        torch.cuda.synchronize()
        assert float(x[0]) == 1.0  # the captured work is intact
        assert np.array_equal(got.view(np.uint32), ref.view(np.uint32))


def test_static_snapshot_refuses_capturing_stream(gpu_lib):
    """The handle's own stream under capture: refused with TTI_ERR_STATE, and
    that capture is left intact."""
    import torch

    import ttifd

    with _shot(ttifd) as h:
        ref = h.snapshot_static(1)
        x = torch.zeros(1024, device="cuda:0")
        hs = torch.cuda.ExternalStream(h.stream, device=0)
        g = torch.cuda.CUDAGraph()
        with torch.cuda.stream(hs):
            g.capture_begin(capture_error_mode="relaxed")
            x.add_(1.0)
            with pytest.raises(ttifd.TTIError) as e:
                h.snapshot_static(1)
            g.capture_end()
        assert e.value.code == ttifd.ERR_STATE and "captured" in str(e.value)
        g.replay()
        torch.cuda.synchronize()
        assert float(x[0]) == 1.0
        assert np.array_equal(h.snapshot_static(1).view(np.uint32), ref.view(np.uint32))
