"""The device gradient against central finite differences of the device's own
misfit: at 50 seeded centres in the illuminated part of the interior (at
least 6 cells from the physical edges, outside the absorbing rims, so the
frozen MEAL arrays are the model's own), one of vp, epsilon, delta, theta is
perturbed by m <- m +- h s b with s the parameter's largest magnitude over
the physical model (epsilon and delta are small numbers, theta is in degrees),
h = 1e-3 for vp and epsilon and 1e-2 for delta and theta (whose misfit is
far less sensitive, so a smaller step would sink into rounding noise; the
central difference's own error, O(h^2), stays near 1e-4 even there), and b a
Gaussian bump (sigma 4 cells) of unit peak centred there, and
    (J(m + h s b) - J(m - h s b)) / 2   against   sum_cells g (h s b)
(vs and rho held fixed, as the gradient assumes). Bumps of about a hundred
cells where the waves pass, rather than single cells, keep the FP32 forward's
rounding noise (independent between the two runs) far below the measured
difference. Tolerance 1e-3 relative to the parameter's largest directional
derivative."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu

NZ, NX, NT, EAL = 90, 150, 700, 10
NAMES = {"vp": 0, "eps": 3, "delta": 4, "theta": 5}  # gradient name -> index in the padded model list
HREL = {"vp": 1e-3, "eps": 1e-3, "delta": 1e-2, "theta": 1e-2}
SIGMA = 4.0


def _setup(variant):
    import ttifd

    true = synthetic.layered_model(NZ, NX, seed=31, nlayers=4)
    start = synthetic.layered_model(NZ, NX, seed=31, nlayers=4)
    # start: true model with a smooth anomaly of every parameter removed
    z, x = np.meshgrid(np.arange(NZ), np.arange(NX))
    blob = np.exp(-((x - 75) ** 2 + (z - 28) ** 2) / (2 * 12.0 ** 2)).astype(np.float32)
    true.vp[...] = true.vp * (1 + 0.08 * blob)
    true.epsilon[...] = true.epsilon + 0.05 * blob
    true.delta[...] = true.delta + 0.03 * blob
    true.theta[...] = true.theta + 10.0 * blob
    cfg = dict(variant=variant, nz=NZ, nx=NX, nt=NT, dx=10.0, dz=10.0, dt=0.0008, fpeak=18.0, ealThick=EAL,
               freesurface=0, stype=1, seistype=1, mt=1)
    w = synthetic.ricker(NT, cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(0, NX, dtype=np.int32)
    pt = [np.array(a, np.float32) for a in synthetic.padded(true, EAL)]
    ps = [np.array(a, np.float32) for a in synthetic.padded(start, EAL)]
    ps[1], ps[2] = pt[1], pt[2]  # vs and rho as in the true model, held fixed
    h = ttifd.Modeling(**cfg)

    def traces(pads):
        h.upload_model(*pads)
        h.set_source([NX // 2], [3], w)
        for k in (0, 1):
            h.set_receivers(k, gx, 5)
        h.run()
        return [h.fetch_traces(k).astype(np.float64) for k in (0, 1)]

    dobs = traces(pt)
    return h, traces, dobs, ps


def _J(d, dobs):
    return 0.5 * sum(float(np.sum((a - b) ** 2)) for a, b in zip(d, dobs))


@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
def test_device_gradient_matches_central_differences(variant, gpu_lib):
    h, traces, dobs, ps = _setup(variant)
    with h:
        E = h.E
        h.upload_model(*ps)
        for k in (0, 1):
            h.grad_set_observed(k, dobs[k].astype(np.float32))
        h.grad_zero()
        h.grad_run(1)
        grads = {n: h.grad_fetch(n).astype(np.float64) for n in NAMES}
        rng = np.random.default_rng(50)
        # 50 centres at least 6 cells from the physical edges, in the upper half
        # that the surface shot and the receivers illuminate
        cz = rng.integers(6, NZ // 2, 50) + E
        cx = rng.integers(6, NX - 6, 50) + E
        scale = {n: float(np.max(np.abs(ps[i][E:-E, E:-E]))) for n, i in NAMES.items()}
        names = [list(NAMES)[i % 4] for i in range(50)]
        zz, xx = np.meshgrid(np.arange(h.Nz), np.arange(h.Nx))  # [Nx][Nz]
        res = {n: [] for n in NAMES}
        for z0, x0, name in zip(cz, cx, names):
            b = np.exp(-((xx - x0) ** 2 + (zz - z0) ** 2) / (2 * SIGMA ** 2))
            b[b < 1e-4] = 0.0
            i = NAMES[name]
            base = ps[i].astype(np.float64)
            step = HREL[name] * scale[name] * b
            Jpm = []
            for sgn in (1.0, -1.0):
                p = list(ps)
                p[i] = (base + sgn * step).astype(np.float32)
                Jpm.append(_J(traces(p), dobs))
            fd = (Jpm[0] - Jpm[1]) / 2.0
            # the perturbation the float arrays actually carry
            dm = ((base + step).astype(np.float32).astype(np.float64)
                  - (base - step).astype(np.float32).astype(np.float64)) / 2.0
            ad = float(np.sum(grads[name] * dm))
            res[name].append((fd, ad))
        errs = {}
        for name, pairs in res.items():
            fd = np.array([p[0] for p in pairs])
            ad = np.array([p[1] for p in pairs])
            peak = np.abs(fd).max()
            assert peak > 0, name
            errs[name] = float(np.abs(ad - fd).max() / peak)
        assert max(errs.values()) <= 1e-3, (variant, errs)
