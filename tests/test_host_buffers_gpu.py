"""Page-locked host buffers (tti_host_alloc): uploads from them, trace fetches
into them and snapshots delivered into a caller's buffer
(tti_set_snapshot_buffer, copies overlapped with the time steps, callbacks
deferred to the next snapshot step or the end of the run) give exactly what
the staged paths from and into pageable memory give."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu

CFG = dict(variant="coordinate_rotation", nz=70, nx=90, nt=240, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0,
           ealThick=10, freesurface=1, stype=1, seistype=3, mt=2, wsave=3, savew=0, snap_sample=50)


def _shot(ttifd, pads, snapbuf=None, pinned_out=False, abort_at=None):
    snaps = []
    with ttifd.Modeling(**CFG) as h:
        h.upload_model(*pads)
        w = synthetic.ricker(CFG["nt"], CFG["dt"], CFG["fpeak"])[None, :]
        h.set_source([45], [3], w)
        gx = np.arange(CFG["nx"], dtype=np.int32)
        for k in (0, 1, 2):
            h.set_receivers(k, gx, 2)
        if snapbuf is not None:
            h.set_snapshot_buffer(snapbuf)

        def cb(it, kind, a):
            if abort_at is not None and it >= abort_at:
                raise RuntimeError("stop")
            snaps.append((it, kind, a))

        h.run(cb)
        outs = []
        for k in (0, 1, 2):
            out = ttifd.host_empty((CFG["nx"], h.nts)) if pinned_out else None
            outs.append(h.fetch_traces(k, out=out).copy())
        params = [h.fetch_param(n) for n in ("c11", "c13", "invrho", "coef1")]
    return snaps, outs, params


@pytest.fixture(scope="module")
def pads():
    m = synthetic.layered_model(CFG["nz"], CFG["nx"], seed=5)
    return [np.array(a, np.float32) for a in synthetic.padded(m, CFG["ealThick"])]


def test_pinned_paths_match_pageable(gpu_lib, pads):
    import ttifd

    ref_snaps, ref_tr, ref_par = _shot(ttifd, pads)
    pinned = [ttifd.host_empty(a.shape) for a in pads]
    for d, a in zip(pinned, pads):
        d[...] = a
    nzo, nxo = CFG["nz"], CFG["nx"]
    buf = ttifd.host_empty(3 * nzo * nxo)
    snaps, tr, par = _shot(ttifd, pinned, snapbuf=buf, pinned_out=True)
    assert [(it, k) for it, k, _ in snaps] == [(it, k) for it, k, _ in ref_snaps]
    assert len(snaps) == 3 * len(range(0, CFG["nt"], CFG["snap_sample"]))
    for (_, _, a), (_, _, b) in zip(snaps, ref_snaps):
        assert np.array_equal(a, b)
    for a, b in zip(tr, ref_tr):
        assert np.array_equal(a, b)
    for a, b in zip(par, ref_par):
        assert np.array_equal(a, b)


def test_pageable_snapshot_buffer(gpu_lib, pads):
    import ttifd

    ref_snaps, _, _ = _shot(ttifd, pads)
    buf = np.empty(3 * CFG["nz"] * CFG["nx"], np.float32)
    snaps, _, _ = _shot(ttifd, pads, snapbuf=buf)
    assert [(it, k) for it, k, _ in snaps] == [(it, k) for it, k, _ in ref_snaps]
    for (_, _, a), (_, _, b) in zip(snaps, ref_snaps):
        assert np.array_equal(a, b)


def test_snapshot_buffer_errors_and_abort(gpu_lib, pads):
    import ttifd

    with ttifd.Modeling(**CFG) as h:
        with pytest.raises(ttifd.TTIError) as e:
            h.set_snapshot_buffer(np.empty(3 * CFG["nz"] * CFG["nx"] - 1, np.float32))
        assert e.value.code == ttifd.ERR_ARG
    with ttifd.Modeling(**dict(CFG, wsave=0)) as h:
        with pytest.raises(ttifd.TTIError) as e:
            h.set_snapshot_buffer(np.empty(16, np.float32))
        assert e.value.code == ttifd.ERR_STATE
    pageable = np.empty(4, np.float32)
    assert ttifd.load().tti_host_free(pageable.ctypes.data) == ttifd.ERR_ARG
    # a callback that aborts a deferred delivery ends the run with ERR_CALLBACK
    buf = ttifd.host_empty(3 * CFG["nz"] * CFG["nx"])
    with pytest.raises(ttifd.TTIError) as e:
        _shot(ttifd, pads, snapbuf=buf, abort_at=100)
    assert e.value.code == ttifd.ERR_CALLBACK
    assert "it=100" in str(e.value)
