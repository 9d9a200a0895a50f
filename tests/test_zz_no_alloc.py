"""tti_snapshot_static: the snapshot entry point that allocates no device
memory, for callers that cannot allocate when they need a snapshot (during a
stream capture, or under a fixed GPU memory budget). It packs through a static
device array instead of the handle's staging buffer. Its output must equal
what the regular snapshot path (tti_run's callback) delivers for the same
wavefield, bit for bit, on consecutive calls; snapshots larger than the
static array are refused. Kept in a file that pytest collects last."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu


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
