"""Failure paths of the library, each made without a GPU fault:
non-finite values in an uploaded model trip the receiver watchdog
(TTI_ERR_NONFINITE); allocation requests above the device's memory fail
cleanly with TTI_ERR_NOMEM and leave the handle (and the process) usable; and a
TMA tile wait that gives up (its poll limit lowered to zero for the test, the
copies in flight still drained) is reported as TTI_ERR_CUDA with the timeout
bit, after which a new handle runs normally."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu

CFG = dict(variant="coordinate_rotation", nz=120, nx=160, nt=150, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0,
           ealThick=10, freesurface=0, stype=1, seistype=1, mt=1)


def _model(nz, nx, seed=21):
    return synthetic.layered_model(nz, nx, seed=seed)


def _shot(h, cfg):
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    h.set_source([cfg["nx"] // 2], [10], w[None, :])
    gx = np.arange(cfg["nx"], dtype=np.int32)
    for k in (0, 1):
        h.set_receivers(k, gx, 5)


def test_nonfinite_model_trips_watchdog(gpu_lib, monkeypatch):
    import ttifd

    monkeypatch.delenv("TTIFD_WAIT_LIMIT", raising=False)
    m = _model(CFG["nz"], CFG["nx"])
    pads = [np.array(a, copy=True) for a in synthetic.padded(m, CFG["ealThick"])]
    E = CFG["ealThick"] + 5
    pads[0][E + 70:E + 90, E:E + 30] = np.nan  # vp: a NaN block around the source
    with ttifd.Modeling(**CFG) as h:
        h.upload_model(*pads)
        _shot(h, CFG)
        with pytest.raises(ttifd.TTIError) as e:
            h.run()
        assert e.value.code == ttifd.ERR_NONFINITE
        # the same handle with a clean model runs and records finite traces
        h.upload_model(*synthetic.padded(m, CFG["ealThick"]))
        h.run()
        tr = h.fetch_traces(0)
        assert np.isfinite(tr).all() and np.abs(tr).max() > 0


def test_create_beyond_device_memory_is_nomem(gpu_lib, monkeypatch):
    import ttifd

    monkeypatch.delenv("TTIFD_WAIT_LIMIT", raising=False)
    # one wavefield of 300000 x 300000 cells is 360 GB: the first allocation fails
    with pytest.raises(ttifd.TTIError) as e:
        ttifd.Modeling(nz=300000, nx=300000, nt=2, dx=10.0, dz=10.0, dt=0.0008, fpeak=10.0, ealThick=0)
    assert e.value.code == ttifd.ERR_NOMEM
    with ttifd.Modeling(**CFG) as h:  # the process is still usable
        h.upload_model(*synthetic.padded(_model(CFG["nz"], CFG["nx"]), CFG["ealThick"]))
        _shot(h, CFG)
        h.run()
        assert np.isfinite(h.fetch_traces(1)).all()


def test_gradient_beyond_device_memory_is_nomem_then_runs(gpu_lib, monkeypatch):
    import ttifd

    monkeypatch.delenv("TTIFD_WAIT_LIMIT", raising=False)
    cfg = dict(CFG, nz=1400, nx=1400, nt=5000)
    m = _model(cfg["nz"], cfg["nx"])
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*synthetic.padded(m, cfg["ealThick"]))
        _shot(h, cfg)
        for k in (0, 1):
            h.grad_set_observed(k, np.zeros((cfg["nx"], h.nts), np.float32))
        h.grad_zero()
        # every step kept: 5000 steps x 8 fields x 8 MB = 330 GB
        with pytest.raises(ttifd.TTIError) as e:
            h.grad_run(1)
        assert e.value.code == ttifd.ERR_NOMEM
        J = h.grad_run(100)  # 50 steps per segment fits
        assert np.isfinite(J) and J > 0
        g = h.grad_fetch("vp")
        assert np.isfinite(g).all() and np.abs(g).max() > 0


def test_tma_wait_timeout_is_reported(gpu_lib, monkeypatch):
    import ttifd

    monkeypatch.setenv("TTIFD_KERNEL", "tiled")
    m = _model(CFG["nz"], CFG["nx"])
    monkeypatch.setenv("TTIFD_WAIT_LIMIT", "0")  # the first poll already gives up
    with ttifd.Modeling(**CFG) as h:
        h.upload_model(*synthetic.padded(m, CFG["ealThick"]))
        _shot(h, CFG)
        with pytest.raises(ttifd.TTIError) as e:
            h.run()
        assert e.value.code == ttifd.ERR_CUDA and "timed out" in str(e.value)
    monkeypatch.delenv("TTIFD_WAIT_LIMIT")
    with ttifd.Modeling(**CFG) as h:  # the context is intact
        h.upload_model(*synthetic.padded(m, CFG["ealThick"]))
        _shot(h, CFG)
        h.run()
        tr = h.fetch_traces(0)
        assert np.isfinite(tr).all() and np.abs(tr).max() > 0
