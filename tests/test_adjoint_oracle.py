"""The double-precision CPU reference of the adjoint-state gradient
(oracle/ttifd_adjoint.c), pinned the two ways an adjoint can be checked
without a reference implementation: the dot-product test <L s, r> = <s, L^T r>
of the source-to-trace map (the adjoint propagation, free surface and
receivers), and central finite differences of the misfit at seeded cells for
each of vp, epsilon, delta and theta (the stiffness chain rule)."""
import numpy as np
import pytest

import synthetic
from pyoracle import AdjointOracle

CFG = dict(nz=36, nx=48, nt=220, dx=10.0, dz=10.0, dt=0.001, fpeak=15.0, ealThick=8, seistype=3, mt=1)


def _setup(fs, seed=5, variant="coordinate_rotation"):
    cfg = dict(CFG, freesurface=fs, variant=variant)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=seed, nlayers=4)
    pads = synthetic.padded(m, cfg["ealThick"])
    adj = AdjointOracle(cfg, pads)
    adj.set_model(*pads)
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    adj.set_source([24], [3], w[None, :])
    gx = np.arange(0, cfg["nx"], 3)
    for k in (0, 1, 2):
        adj.set_receivers(k, gx, 2)
    return cfg, adj, pads, w


CASES = [(0, "coordinate_rotation"), (1, "coordinate_rotation"), (0, "bond_transformation"),
         (1, "bond_transformation"), (0, "tensor_rotation"), (1, "tensor_rotation")]


@pytest.mark.parametrize("fs,variant", CASES)
def test_dot_product(fs, variant):
    cfg, adj, pads, w = _setup(fs, variant=variant)
    with adj:
        d = adj.forward()
        rng = np.random.default_rng(1)
        r = [rng.standard_normal(a.shape) for a in d]
        J, g, gsrc = adj.gradient([a - b for a, b in zip(d, r)])
        lhs = sum(float(np.sum(a * b)) for a, b in zip(d, r))
        rhs = float(np.sum(gsrc[0] * w))
        assert J == pytest.approx(0.5 * sum(float(np.sum(b * b)) for b in r), rel=1e-12)
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


def _misfit(adj, model, dobs):
    adj.set_model(*model)
    d = adj.forward()
    return 0.5 * sum(float(np.sum((a - b) ** 2)) for a, b in zip(d, dobs))


@pytest.mark.parametrize("fs,variant", CASES)
def test_gradient_matches_central_differences(fs, variant):
    cfg, adj, pads, w = _setup(fs, variant=variant)
    E = cfg["ealThick"] + 5
    with adj:
        # observed data from a model with a perturbed patch; gradient at the start model
        true = [np.array(a, dtype=np.float64) for a in pads]
        true[0][E + 20:E + 30, E + 12:E + 20] *= 1.04
        true[5][E + 20:E + 30, E + 12:E + 20] += 6.0
        adj.set_model(*true)
        dobs = adj.forward()
        start = [np.array(a, dtype=np.float64) for a in pads]
        adj.set_model(*start)
        J0, g, _ = adj.gradient(dobs)
        assert J0 > 0
        rng = np.random.default_rng(3)
        checks = []
        for name, idx, h in (("vp", 0, 1e-3), ("eps", 3, 1e-3), ("delta", 4, 1e-3), ("theta", 5, 1e-2)):
            for _ in range(3):
                ix = E + 6 + int(rng.integers(0, cfg["nx"] - 12))
                iz = E + 6 + int(rng.integers(0, cfg["nz"] - 12))
                step = h * (start[0][ix, iz] if name == "vp" else 1.0)
                mp = [a.copy() for a in start]
                mm = [a.copy() for a in start]
                mp[idx][ix, iz] += step
                mm[idx][ix, iz] -= step
                fd = (_misfit(adj, mp, dobs) - _misfit(adj, mm, dobs)) / (2 * step)
                checks.append((name, ix, iz, fd, g[name][ix, iz]))
        scale = {n: max(abs(c[4]) for c in checks if c[0] == n) for n in ("vp", "eps", "delta", "theta")}
        for name, ix, iz, fd, an in checks:
            assert abs(fd - an) <= 1e-3 * max(abs(an), 1e-2 * scale[name]), (name, ix, iz, fd, an)


def test_bond_free_surface_row_gradient():
    """On the free-surface row the Bond moduli are replaced by an effective c11
    (bond:543-568); the gradient there goes through that rewrite."""
    cfg, adj, pads, w = _setup(1, variant="bond_transformation")
    E = cfg["ealThick"] + 5
    with adj:
        true = [np.array(a, dtype=np.float64) for a in pads]
        true[0][E + 10:E + 30, E:E + 6] *= 1.05
        true[5][E + 10:E + 30, E:E + 6] += 8.0
        adj.set_model(*true)
        dobs = adj.forward()
        start = [np.array(a, dtype=np.float64) for a in pads]
        adj.set_model(*start)
        _, g, _ = adj.gradient(dobs)
        for name, idx, h in (("vp", 0, 1e-3), ("eps", 3, 1e-3), ("theta", 5, 1e-2)):
            for ix in (E + 18, E + 27):
                step = h * (start[0][ix, E] if name == "vp" else 1.0)
                mp = [a.copy() for a in start]
                mm = [a.copy() for a in start]
                mp[idx][ix, E] += step
                mm[idx][ix, E] -= step
                fd = (_misfit(adj, mp, dobs) - _misfit(adj, mm, dobs)) / (2 * step)
                an = g[name][ix, E]
                assert abs(fd - an) <= 1e-3 * abs(an) and abs(an) > 0, (name, ix, fd, an)


def _setup_vsrc(stype, fs, variant="coordinate_rotation", seed=5):
    """A velocity source one row below the surface (stype 8: on it), so that
    with a free surface its cells reach the image rows the velocity update
    never writes."""
    cfg = dict(CFG, freesurface=fs, variant=variant, stype=stype)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=seed, nlayers=4)
    pads = synthetic.padded(m, cfg["ealThick"])
    adj = AdjointOracle(cfg, pads)
    adj.set_model(*pads)
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    sz = 0 if stype == 8 else 1
    adj.set_source([24], [sz], w[None, :])
    gx = np.arange(0, cfg["nx"], 3)
    for k in (0, 1, 2):
        adj.set_receivers(k, gx, 2)
    return cfg, adj, pads, w, sz


VSRC_CASES = [(s, fs, "coordinate_rotation") for s in range(2, 9) for fs in (0, 1)] + \
    [(2, 1, "tensor_rotation"), (5, 1, "tensor_rotation"), (3, 0, "bond_transformation"),
     (7, 0, "bond_transformation")]


@pytest.mark.parametrize("stype,fs,variant", [(1, 1, "coordinate_rotation")] + VSRC_CASES)
def test_forward_matches_float_restatement(stype, fs, variant):
    """The double forward of the adjoint reference against the float CPU
    restatement of the reference (oracle/ttifd_oracle.c) on the same inputs:
    same sources, stencils, free surface and receivers."""
    from pyoracle import Oracle

    cfg, adj, pads, w, sz = _setup_vsrc(stype, fs, variant)
    gx = np.arange(0, cfg["nx"], 3)
    with adj:
        d = adj.forward()
    with Oracle(**dict(cfg, wsave=0, energy=0)) as o:
        o.upload_model(*pads)
        o.set_source([24], [sz], w[None, :].astype(np.float32))
        for k in (0, 1, 2):
            o.set_receivers(k, gx, 2)
        o.run()
        ref = [o.fetch_traces(k).astype(np.float64) for k in (0, 1, 2)]
    for a, b in zip(d, ref):
        assert np.linalg.norm(a - b) <= 1e-4 * np.linalg.norm(b), np.linalg.norm(a - b) / np.linalg.norm(b)


@pytest.mark.parametrize("stype,fs,variant", VSRC_CASES)
def test_dot_product_velocity_sources(stype, fs, variant):
    """<L s, r> = <s, L^T r> with the velocity sources: the source gradient is
    read from lambda_v between the two adjoint halves, including the cells
    outside the velocity update."""
    cfg, adj, pads, w, _ = _setup_vsrc(stype, fs, variant)
    with adj:
        d = adj.forward()
        rng = np.random.default_rng(1)
        r = [rng.standard_normal(a.shape) for a in d]
        _, _, gsrc = adj.gradient([a - b for a, b in zip(d, r)])
        lhs = sum(float(np.sum(a * b)) for a, b in zip(d, r))
        rhs = float(np.sum(gsrc[0] * w))
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)


@pytest.mark.parametrize("stype,variant", [(2, "coordinate_rotation"), (6, "tensor_rotation"),
                                           (8, "bond_transformation")])
def test_velocity_source_gradient_matches_central_differences(stype, variant):
    cfg, adj, pads, w, _ = _setup_vsrc(stype, 1 if variant != "bond_transformation" else 0, variant)
    E = cfg["ealThick"] + 5
    with adj:
        true = [np.array(a, dtype=np.float64) for a in pads]
        true[0][E + 20:E + 30, E + 12:E + 20] *= 1.04
        true[5][E + 20:E + 30, E + 12:E + 20] += 6.0
        adj.set_model(*true)
        dobs = adj.forward()
        start = [np.array(a, dtype=np.float64) for a in pads]
        adj.set_model(*start)
        J0, g, _ = adj.gradient(dobs)
        assert J0 > 0
        rng = np.random.default_rng(7)
        for name, idx, h in (("vp", 0, 1e-3), ("eps", 3, 1e-3), ("delta", 4, 1e-3), ("theta", 5, 1e-2)):
            for _ in range(2):
                ix = E + 6 + int(rng.integers(0, cfg["nx"] - 12))
                iz = E + 6 + int(rng.integers(0, cfg["nz"] - 12))
                step = h * (start[0][ix, iz] if name == "vp" else 1.0)
                mp = [a.copy() for a in start]
                mm = [a.copy() for a in start]
                mp[idx][ix, iz] += step
                mm[idx][ix, iz] -= step
                fd = (_misfit(adj, mp, dobs) - _misfit(adj, mm, dobs)) / (2 * step)
                an = g[name][ix, iz]
                assert abs(fd - an) <= 1e-3 * max(abs(an), 1e-2 * np.abs(g[name]).max()), (name, ix, iz, fd, an)


@pytest.mark.parametrize("mt,seistype,variant", [(3, 3, "coordinate_rotation"), (2, 1, "tensor_rotation"),
                                                 (4, 2, "bond_transformation")])
def test_dot_product_sampling_and_components(mt, seistype, variant):
    """Traces every mt-th step, and only the components seistype records
    (1: vx vz, 2: p): the adjoint injects the residual at those steps only."""
    cfg = dict(CFG, freesurface=1 if variant != "bond_transformation" else 0, variant=variant, mt=mt,
               seistype=seistype)
    m = synthetic.layered_model(cfg["nz"], cfg["nx"], seed=5, nlayers=4)
    pads = synthetic.padded(m, cfg["ealThick"])
    with AdjointOracle(cfg, pads) as adj:
        adj.set_model(*pads)
        w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
        adj.set_source([24], [3], w[None, :])
        gx = np.arange(0, cfg["nx"], 3)
        for k in (0, 1, 2):
            adj.set_receivers(k, gx, 2)
        d = adj.forward()
        want = [seistype in (1, 3), seistype in (1, 3), seistype in (2, 3)]
        for x, on in zip(d, want):  # components not recorded stay zero
            assert x.shape[1] == (cfg["nt"] - 1) // mt + 1
            assert (np.abs(x).max() > 0) == on
        rng = np.random.default_rng(2)
        r = [rng.standard_normal(x.shape) if x is not None else None for x in d]
        _, _, gsrc = adj.gradient([a - b if a is not None else None for a, b in zip(d, r)])
        lhs = sum(float(np.sum(a * b)) for a, b in zip(d, r) if a is not None)
        rhs = float(np.sum(gsrc[0] * w))
        assert abs(lhs - rhs) <= 1e-10 * abs(lhs), (lhs, rhs)
