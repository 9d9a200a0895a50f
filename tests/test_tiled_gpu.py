"""Tiled half-step kernels, under both in-tile schedules (row and walk), vs the
one-thread-per-cell kernels on grids of several tiles. In the exact rounding
mode all paths perform the same operations in the same order, so the
wavefields, traces and snapshots must be bit-identical; the gradient's forward
passes, which also write what the adjoint keeps, likewise."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu


def _run(kernel, monkeypatch, variant, fs, stype, nz=300, nx=260, nt=160):
    import ttifd

    monkeypatch.setenv("TTIFD_EXACT", "1")
    # "row" / "walk": the tiled kernels with either in-tile schedule
    monkeypatch.setenv("TTIFD_SCHEDULE", "walk" if kernel == "walk" else "row")
    monkeypatch.setenv("TTIFD_KERNEL", "tiled" if kernel in ("row", "walk") else kernel)
    cfg = dict(variant=variant, nz=nz, nx=nx, nt=nt, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0, ealThick=12,
               freesurface=fs, stype=stype, seistype=3, mt=2, wsave=3, snap_sample=50)
    m = synthetic.salt_model(nz, nx, seed=11, nlayers=12)
    pads = synthetic.padded(m, cfg["ealThick"])
    w = synthetic.ricker(nt, cfg["dt"], cfg["fpeak"])
    snaps = {}
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*pads)
        # sources straddling a band boundary (padded row 128) and the surface
        h.set_source([40, 200], [128 - h.E - 1, 2], np.stack([w, 0.5 * w]))
        gx = np.arange(0, nx, 3)
        for k in (0, 1, 2):
            h.set_receivers(k, gx, (gx * 7) % nz)
        h.run(lambda it, kind, a: snaps.__setitem__((it, kind), a))
        out = {f"tr{k}": h.fetch_traces(k) for k in (0, 1, 2)}
        for f in range(8 if variant == "tensor_rotation" else 5):
            out[f"f{f}"] = h.fetch_field(f)
    out.update({f"s{k}": v for k, v in snaps.items()})
    return out


@pytest.mark.parametrize("path", ["row", "walk"])
@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
@pytest.mark.parametrize("fs,stype", [(0, 1), (1, 1), (1, 4), (0, 8)])
def test_tiled_equals_per_cell_path(path, variant, fs, stype, monkeypatch, gpu_lib):
    ref = _run("naive", monkeypatch, variant, fs, stype)
    got = _run(path, monkeypatch, variant, fs, stype)
    assert ref.keys() == got.keys()
    for k in ref:
        a, b = np.asarray(got[k]), np.asarray(ref[k])
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (
            f"{variant} fs={fs} stype={stype} {k}: max |diff| {np.max(np.abs(a - b))}")


def _gradient(schedule, monkeypatch, variant, fs):
    import ttifd

    monkeypatch.setenv("TTIFD_EXACT", "1")
    monkeypatch.setenv("TTIFD_SCHEDULE", schedule)
    monkeypatch.setenv("TTIFD_KERNEL", "tiled")
    nz, nx, nt = 260, 200, 120
    cfg = dict(variant=variant, nz=nz, nx=nx, nt=nt, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0, ealThick=12,
               freesurface=fs, stype=1, seistype=1, mt=1)
    m = synthetic.salt_model(nz, nx, seed=13, nlayers=10)
    w = synthetic.ricker(nt, cfg["dt"], cfg["fpeak"])
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*synthetic.padded(m, cfg["ealThick"]))
        h.set_source([nx // 2], [3], w[None, :])
        gx = np.arange(0, nx, 2)
        for k in (0, 1):
            h.set_receivers(k, gx, 4)
            h.grad_set_observed(k, np.zeros((len(gx), h.nts), np.float32))
        h.grad_zero()
        J = h.grad_run(3)
        return J, {n: h.grad_fetch(n) for n in ("vp", "eps", "delta", "theta")}


@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
@pytest.mark.parametrize("fs", [0, 1])
def test_walk_schedule_gradient_equals_row_schedule(variant, fs, monkeypatch, gpu_lib):
    """The gradient's forward passes keep what the forward kernels write (strain
    rates, stress derivative combinations, tau); with the walk schedule on a
    grid of several tiles the gradient must be the row schedule's, bit for bit."""
    J0, g0 = _gradient("row", monkeypatch, variant, fs)
    J1, g1 = _gradient("walk", monkeypatch, variant, fs)
    assert J1 == pytest.approx(J0, rel=1e-12)  # J is a double atomic sum: order-dependent last bit
    for n in g0:
        assert np.array_equal(g1[n].view(np.uint32), g0[n].view(np.uint32)), n
        assert np.abs(g0[n]).max() > 0
