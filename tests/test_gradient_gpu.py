"""Device adjoint-state gradient (tti_grad_*) against the double-precision CPU
reference (oracle/ttifd_adjoint.c, itself pinned by the dot-product test and
central finite differences): misfit, the four model gradients and the source
gradient, for the stress source and the velocity sources; independence of the
checkpoint count; shot accumulation; the dot-product test of the device
adjoint."""
import numpy as np
import pytest

import synthetic
from pyoracle import AdjointOracle

pytestmark = pytest.mark.gpu

CFG = dict(nz=36, nx=48, nt=220, dx=10.0, dz=10.0, dt=0.001, fpeak=15.0, ealThick=8, seistype=3, mt=1)
NAMES = ("vp", "eps", "delta", "theta")


def _case(fs, sx=24, variant="coordinate_rotation"):
    cfg = dict(CFG, freesurface=fs, variant=variant)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=5, nlayers=4)
    pads = synthetic.padded(m, cfg["ealThick"])
    E = cfg["ealThick"] + 5
    true = [np.array(a, dtype=np.float64) for a in pads]
    true[0][E + 20:E + 30, E + 12:E + 20] *= 1.04
    true[5][E + 20:E + 30, E + 12:E + 20] += 6.0
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    gx = np.arange(0, cfg["nx"], 3)
    return cfg, pads, true, w, gx


def _device(cfg, pads, w, gx, dobs, ncheck, sx=24, h=None, sz=3):
    import ttifd

    own = h is None
    if own:
        h = ttifd.Modeling(**dict({"variant": "coordinate_rotation", "stype": 1}, **cfg))
        h.upload_model(*pads)
        h.grad_zero()
    h.set_source([sx], [sz], w[None, :])
    for k in (0, 1, 2):
        h.set_receivers(k, gx, 2)
        h.grad_set_observed(k, dobs[k])
    J = h.grad_run(ncheck)
    return h, J


def _rel(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


@pytest.mark.parametrize("kernel", ["tiled", "naive"])
@pytest.mark.parametrize("fs,variant", [(0, "coordinate_rotation"), (1, "coordinate_rotation"),
                                        (0, "bond_transformation"), (1, "bond_transformation"),
                                        (0, "tensor_rotation"), (1, "tensor_rotation")])
def test_gradient_matches_cpu_reference(fs, variant, kernel, monkeypatch, gpu_lib):
    """Both adjoint paths: TMA-tiled (default) and one thread per cell (TTIFD_KERNEL=naive)."""
    if kernel == "naive":
        monkeypatch.setenv("TTIFD_KERNEL", "naive")
    else:
        monkeypatch.delenv("TTIFD_KERNEL", raising=False)
    cfg, pads, true, w, gx = _case(fs, variant=variant)
    with AdjointOracle(cfg, pads) as adj:
        adj.set_model(*true)
        adj.set_source([24], [3], w[None, :])
        for k in (0, 1, 2):
            adj.set_receivers(k, gx, 2)
        dobs = adj.forward()
        adj.set_model(*pads)
        J_ref, g_ref, gs_ref = adj.gradient(dobs)
    h, J = _device(cfg, pads, w, gx, [d.astype(np.float32) for d in dobs], ncheck=9)
    with h:
        assert J == pytest.approx(J_ref, rel=1e-4)
        for name in NAMES:
            err = _rel(h.grad_fetch(name), g_ref[name])
            assert err <= 1e-3, (name, err)
        assert _rel(h.grad_fetch_source(1), gs_ref) <= 1e-4


def test_checkpoint_count_does_not_change_the_gradient(gpu_lib):
    cfg, pads, true, w, gx = _case(1)
    dobs = [np.zeros((gx.size, cfg["nt"]), np.float32) for _ in range(3)]
    out = []
    for ncheck in (1, 7, cfg["nt"]):
        h, J = _device(cfg, pads, w, gx, dobs, ncheck)
        with h:
            out.append((J, [h.grad_fetch(n) for n in NAMES]))
    for J, g in out[1:]:
        assert J == pytest.approx(out[0][0], rel=1e-12)  # a double atomic sum: order-dependent last bit
        for a, b in zip(g, out[0][1]):
            assert np.array_equal(a, b)


@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
def test_binomial_schedule_equals_uniform(variant, gpu_lib):
    """Binomial (Revolve) checkpointing, with slots from none to plenty and
    macro-steps of 1 to 40 steps, gives the uniform schedule's gradient bit
    for bit (the same forward steps and adjoint steps in the same order)."""
    import ttifd

    cfg, pads, true, w, gx = _case(1, variant=variant)
    dobs = [np.zeros((gx.size, cfg["nt"]), np.float32) for _ in range(3)]
    h, J0 = _device(cfg, pads, w, gx, dobs, 1)
    with h:
        ref = [h.grad_fetch(n) for n in NAMES]
        for snapshots, keep in ((3, 1), (0, 40), (2, 17), (30, 7), (5, 220)):
            h.grad_zero()
            J = h.grad_run_binomial(snapshots, keep)
            assert J == pytest.approx(J0, rel=1e-12)
            for a, b, n in zip([h.grad_fetch(n) for n in NAMES], ref, NAMES):
                assert np.array_equal(a, b), (snapshots, keep, n)
    assert ttifd.schedule_cost(220, 3) > 220  # (3, 1) recomputes steps more than once


def test_shots_accumulate(gpu_lib):
    cfg, pads, true, w, gx = _case(0)
    rng = np.random.default_rng(2)
    dobs = [1e-9 * rng.standard_normal((gx.size, cfg["nt"])).astype(np.float32) for _ in range(3)]
    singles = []
    for sx in (12, 30):
        h, _ = _device(cfg, pads, w, gx, dobs, 5, sx=sx)
        with h:
            singles.append(h.grad_fetch("vp"))
    h, _ = _device(cfg, pads, w, gx, dobs, 5, sx=12)
    with h:
        _device(cfg, pads, w, gx, dobs, 5, sx=30, h=h)
        both = h.grad_fetch("vp")
    assert _rel(both, singles[0] + singles[1]) <= 1e-6


def test_device_dot_product(gpu_lib):
    """<L w, r> = <w, L^T r> with the device forward and adjoint (float)."""
    import ttifd

    cfg, pads, true, w, gx = _case(1)
    with ttifd.Modeling(stype=1, **cfg) as h:
        h.upload_model(*pads)
        h.set_source([24], [3], w[None, :])
        for k in (0, 1, 2):
            h.set_receivers(k, gx, 2)
        h.run()
        d = [h.fetch_traces(k).astype(np.float64) for k in (0, 1, 2)]
    rng = np.random.default_rng(4)
    scale = max(np.abs(x).max() for x in d)
    r = [scale * rng.standard_normal(x.shape) for x in d]
    h, _ = _device(cfg, pads, w, gx, [(a - b).astype(np.float32) for a, b in zip(d, r)], ncheck=4)
    with h:
        gsrc = h.grad_fetch_source(1).astype(np.float64)
    lhs = sum(float(np.sum(a * b)) for a, b in zip(d, r))
    rhs = float(np.sum(gsrc[0] * w))
    assert abs(lhs - rhs) <= 2e-4 * abs(lhs), (lhs, rhs)


VSRC = [(s, 1, "coordinate_rotation", "tiled") for s in range(2, 9)] + \
    [(4, 0, "coordinate_rotation", "tiled"), (2, 1, "coordinate_rotation", "naive"),
     (8, 1, "coordinate_rotation", "naive"), (5, 1, "tensor_rotation", "tiled"), (7, 0, "bond_transformation", "tiled")]


@pytest.mark.parametrize("stype,fs,variant,kernel", VSRC)
def test_velocity_source_gradient_matches_cpu_reference(stype, fs, variant, kernel, monkeypatch, gpu_lib):
    """Velocity sources (stype 2-8): the model gradient (same adjoint kernels,
    forward replay with the velocity source) and the source gradient (read from
    lambda_v between the adjoint halves; one row below the free surface the
    window reaches the image rows, stype 8 sits on the surface row). The
    observed traces are the true model's at half amplitude, so the residual is
    of the size of the data: with the true model's own traces the residual is
    a small difference of two close wavefields, and the float forward's
    rounding (1e-5 of the traces) grows to 4e-4 of J for stype 8, which would
    measure the residual's conditioning rather than the adjoint."""
    if kernel == "naive":
        monkeypatch.setenv("TTIFD_KERNEL", "naive")
    else:
        monkeypatch.delenv("TTIFD_KERNEL", raising=False)
    cfg, pads, true, w, gx = _case(fs, variant=variant)
    cfg = dict(cfg, stype=stype)
    sz = 0 if stype == 8 else 1
    with AdjointOracle(cfg, pads) as adj:
        adj.set_model(*true)
        adj.set_source([24], [sz], w[None, :])
        for k in (0, 1, 2):
            adj.set_receivers(k, gx, 2)
        dobs = [0.5 * d for d in adj.forward()]
        adj.set_model(*pads)
        J_ref, g_ref, gs_ref = adj.gradient(dobs)
    h, J = _device(cfg, pads, w, gx, [d.astype(np.float32) for d in dobs], ncheck=9, sz=sz)
    with h:  # measured on B200: J 1e-7..1e-6, gradients 4e-7..1.4e-6, source gradient 5e-7..5e-6
        assert J == pytest.approx(J_ref, rel=1e-5)
        for name in NAMES:
            err = _rel(h.grad_fetch(name), g_ref[name])
            assert err <= 2e-5, (name, err)
        assert _rel(h.grad_fetch_source(1), gs_ref) <= 5e-5


@pytest.mark.parametrize("stype", [3, 8])
def test_device_dot_product_velocity_sources(stype, gpu_lib):
    """<L w, r> = <w, L^T r> for a velocity source whose cells reach the image
    rows above the free surface."""
    import ttifd

    cfg, pads, true, w, gx = _case(1)
    cfg = dict(cfg, stype=stype)
    sz = 0 if stype == 8 else 1
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*pads)
        h.set_source([24], [sz], w[None, :])
        for k in (0, 1, 2):
            h.set_receivers(k, gx, 2)
        h.run()
        d = [h.fetch_traces(k).astype(np.float64) for k in (0, 1, 2)]
    rng = np.random.default_rng(4)
    scale = max(np.abs(x).max() for x in d)
    r = [scale * rng.standard_normal(x.shape) for x in d]
    h, _ = _device(cfg, pads, w, gx, [(a - b).astype(np.float32) for a, b in zip(d, r)], ncheck=4, sz=sz)
    with h:
        gsrc = h.grad_fetch_source(1).astype(np.float64)
    lhs = sum(float(np.sum(a * b)) for a, b in zip(d, r))
    rhs = float(np.sum(gsrc[0] * w))
    assert abs(lhs - rhs) <= 2e-4 * abs(lhs), (lhs, rhs)


def test_gradient_sums_are_device_views(gpu_lib):
    """shots.gradient_sums wraps the library's device sums without a copy (what
    reduce_gradient all-reduces over NCCL): scaling them through torch scales
    the fetched gradient."""
    import torch

    import shots

    cfg, pads, true, w, gx = _case(0)
    rng = np.random.default_rng(6)
    dobs = [1e-9 * rng.standard_normal((gx.size, cfg["nt"])).astype(np.float32) for _ in range(3)]
    h, _ = _device(cfg, pads, w, gx, dobs, 5)
    with h:
        before = {n: h.grad_fetch(n) for n in NAMES}
        sums = shots.gradient_sums(h)
        assert len(sums) == 7 and all(t.is_cuda and t.dtype == torch.float32 for t in sums)
        for t in sums:
            t.mul_(2.0)
        torch.cuda.synchronize()
        for n in NAMES:
            np.testing.assert_allclose(h.grad_fetch(n), 2.0 * before[n], rtol=1e-6)


@pytest.mark.parametrize("mt,seistype,variant", [(3, 3, "coordinate_rotation"), (2, 1, "tensor_rotation"),
                                                 (4, 2, "bond_transformation")])
def test_gradient_sampling_and_components(mt, seistype, variant, gpu_lib):
    """Traces every mt-th step and only the components seistype records: the
    device adjoint injects the residuals at those steps and components, as the
    CPU reference does."""
    import ttifd

    fs = 0 if variant == "bond_transformation" else 1
    cfg, pads, true, w, gx = _case(fs, variant=variant)
    cfg = dict(cfg, mt=mt, seistype=seistype)
    with AdjointOracle(cfg, pads) as adj:
        adj.set_model(*true)
        adj.set_source([24], [3], w[None, :])
        for k in (0, 1, 2):
            adj.set_receivers(k, gx, 2)
        dobs = [0.5 * d for d in adj.forward()]
        adj.set_model(*pads)
        J_ref, g_ref, gs_ref = adj.gradient(dobs)
    with ttifd.Modeling(**dict({"stype": 1}, **cfg)) as h:
        h.upload_model(*pads)
        h.grad_zero()
        h.set_source([24], [3], w[None, :])
        on = [seistype in (1, 3), seistype in (1, 3), seistype in (2, 3)]
        for k in (0, 1, 2):
            h.set_receivers(k, gx, 2)
            if on[k]:
                h.grad_set_observed(k, dobs[k].astype(np.float32))
        J = h.grad_run(5)
        assert J == pytest.approx(J_ref, rel=1e-5)
        for name in NAMES:
            err = _rel(h.grad_fetch(name), g_ref[name])
            assert err <= 2e-5, (name, err)
        assert _rel(h.grad_fetch_source(1), gs_ref) <= 5e-5


def test_gradient_plan_fits_budget_and_runs(gpu_lib):
    """tti_grad_plan: the schedule for a memory budget fits it, more memory never
    costs more forward steps, and the planned run gives the gradient of the
    schedule that keeps every step."""
    cfg, pads, true, w, gx = _case(0)
    dobs = [np.zeros((gx.size, cfg["nt"]), np.float32) for _ in range(3)]
    h, _ = _device(cfg, pads, w, gx, dobs, 1)
    with h:
        ref = [h.grad_fetch(n) for n in NAMES]
        cell = h.grad_plan(1e15)  # unbounded: every step kept, no recomputation
        assert cell == {"snapshots": 0, "keep_steps": cfg["nt"], "forward_steps": cfg["nt"]}
        state = 5 * h.Nx * ((h.Nz + 31) // 32 * 32) * 4.0
        prev = None
        for budget in (3 * state, 12 * state, 60 * state):
            p = h.grad_plan(budget)
            kept = 8 * state / 5
            assert p["snapshots"] * state + p["keep_steps"] * kept <= budget
            if prev is not None:
                assert p["forward_steps"] <= prev
            prev = p["forward_steps"]
            h.grad_zero()
            h.grad_run_binomial(p["snapshots"], p["keep_steps"])
            for a, b in zip([h.grad_fetch(n) for n in NAMES], ref):
                assert np.array_equal(a, b)
