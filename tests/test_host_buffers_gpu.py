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


@pytest.mark.parametrize("variant,fs", [("coordinate_rotation", 1), ("tensor_rotation", 0), ("bond_transformation", 1)])
def test_physical_upload_matches_padded(gpu_lib, variant, fs):
    """tti_upload_model_physical (unpadded arrays, rims filled on the device)
    gives every precomputed parameter and every trace of tti_upload_model on
    the host-padded arrays bit for bit, from pageable and from page-locked
    arrays; a model whose edges vary along both axes, so every rim cell's
    source cell matters."""
    import ttifd

    cfg = dict(CFG, variant=variant, freesurface=fs, nt=120, wsave=0)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=9)
    m.theta[...] += np.linspace(-7.0, 9.0, cfg["nx"], dtype=np.float32)[:, None]  # varies along x too
    phys = [np.array(a, np.float32) for a in m.arrays()]
    pads = [np.array(a, np.float32) for a in synthetic.padded(m, cfg["ealThick"])]
    pinned = [ttifd.host_empty(a.shape) for a in phys]
    for d, a in zip(pinned, phys):
        d[...] = a
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(cfg["nx"], dtype=np.int32)

    def shot(upload):
        with ttifd.Modeling(**cfg) as h:
            upload(h)
            params = {}
            for name in ttifd.PARAMS:
                try:
                    params[name] = h.fetch_param(name)
                except ttifd.TTIError:
                    pass  # not used by this formulation
            h.set_source([45], [3], w)
            for k in (0, 1, 2):
                h.set_receivers(k, gx, 2)
            h.run()
            return params, [h.fetch_traces(k).copy() for k in (0, 1, 2)]

    ref_par, ref_tr = shot(lambda h: h.upload_model(*pads))
    assert {"vp", "coef1", "invrho", "c11"} <= set(ref_par)
    for arrays in (phys, pinned):
        par, tr = shot(lambda h: h.upload_model_physical(*arrays))
        assert sorted(par) == sorted(ref_par)
        for name in ref_par:
            assert np.array_equal(par[name], ref_par[name]), name
        for a, b in zip(tr, ref_tr):
            assert np.array_equal(a, b)
    with ttifd.Modeling(**cfg) as h:
        with pytest.raises(ValueError):
            h.upload_model_physical(*pads)  # padded arrays where physical ones are due
        null = ttifd.load().tti_upload_model_physical(h._h, None, None, None, None, None, None)
        assert null == ttifd.ERR_ARG
