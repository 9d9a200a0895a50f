"""The device gradient of the 16-shot gradient workload at its full size against
central finite differences of the device's own misfit (a record, like
parity_configs.py; the -m gpu test test_gradient_fd_gpu.py does the same on a
reduced grid).

Configuration: the layered 600 x 1200 model (seed 3) as the true model; the
start model its Gaussian blur (sigma 15 cells) in vp, epsilon, delta, theta,
with vs = vp / 1.8 and rho = 310 vp^0.25 of the blurred vp held fixed; 16
surface shots evenly spaced (sdepth 2), receivers on every column at z = 5,
12 Hz, dt 0.8 ms, nt 3000, ealThick 40, no free surface. The gradient of
J = 1/2 sum over shots and samples (d - dobs)^2 comes from the 16 shots at
once with 30 checkpoints (tti_batch_grad_run: 29 slots and a kept segment of
100 steps).

Finite differences: at 50 seeded centres (12 cells or more from the physical
edges, depth above nz / 2) one of vp, epsilon, delta, theta is perturbed by
m +- h s b, s the parameter's largest magnitude over the physical model, h =
1e-3 for vp and epsilon and 1e-2 for delta and theta, b a Gaussian bump
(sigma 4 cells, unit peak) on the physical cells only; (J+ - J-) / 2 is set
against sum g dm (dm as the float arrays carry it), and each parameter's
worst difference is given relative to its largest directional derivative.
At each parameter's worst centre the difference is then taken again with h
halved, doubled and quadrupled: an error that falls as h grows is the FP32
forward's rounding noise in J+ - J-, one that grows as h^2 is truncation.

    python tests/fd_gradient_16shots.py [--json out.json] [--nt 3000] [--centres 50]
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, ROOT)
import bench  # noqa: E402  (the gradient workload and its models)
import synthetic  # noqa: E402

NAMES = {"vp": 0, "eps": 3, "delta": 4, "theta": 5}  # gradient name -> index in the model list
HREL = {"vp": 1e-3, "eps": 1e-3, "delta": 1e-2, "theta": 1e-2}
SIGMA = 4.0


def run(nt=3000, centres=50, shots=16, study_factors=(0.5, 2.0, 4.0), log=print):
    import ttifd

    gw = bench.GRAD_WORKLOAD
    nz, nx, E0 = gw["nz"], gw["nx"], gw["ealThick"]
    cfg = dict(gw, variant="coordinate_rotation", nt=nt)
    true, start = bench.grad_models()
    wav = synthetic.ricker(nt, cfg["dt"], cfg["fpeak"])[None, :]
    gx = np.arange(nx, dtype=np.int32)
    sxs = [int(round((i + 0.5) * nx / shots)) for i in range(shots)]
    t0 = time.perf_counter()
    with ttifd.Batch([cfg], [0] * shots) as b:
        for i, sx in enumerate(sxs):
            b.instances[i].set_source([sx], [2], wav)
            for k in (0, 1):
                b.instances[i].set_receivers(k, gx, 5)

        def traces(pads):
            b.upload_model(0, *pads)
            b.run()
            return [[b.instances[i].fetch_traces(k).astype(np.float64) for k in (0, 1)] for i in range(shots)]

        dobs = traces(synthetic.padded(true, E0))
        ps = [np.array(a, np.float32) for a in synthetic.padded(start, E0)]

        def J(pads):
            d = traces(pads)
            return 0.5 * sum(float(np.sum((a - o) ** 2)) for di, oi in zip(d, dobs) for a, o in zip(di, oi))

        b.upload_model(0, *ps)
        for i in range(shots):
            inst = b.instances[i]
            for k in (0, 1):
                inst.grad_set_observed(k, dobs[i][k].astype(np.float32))
            inst.grad_zero()
        seg = -(-nt // 30)
        Js = b.grad_run(29, seg)
        g_ms = b.elapsed_ms
        h0 = b.instances[0]
        E = h0.E
        grads = {n: h0.grad_fetch(n).astype(np.float64) for n in NAMES}
        rng = np.random.default_rng(50)
        cz = rng.integers(12, nz // 2, centres) + E
        cx = rng.integers(12, nx - 12, centres) + E
        names = [list(NAMES)[i % 4] for i in range(centres)]
        phys = np.zeros((h0.Nx, h0.Nz), bool)
        phys[E:E + nx, E:E + nz] = True
        scale = {n: float(np.max(np.abs(ps[i][E:E + nx, E:E + nz]))) for n, i in NAMES.items()}
        zz, xx = np.meshgrid(np.arange(h0.Nz), np.arange(h0.Nx))

        def fd_at(z0, x0, name, hrel):
            """(J+ - J-) / 2 and sum g dm for the bump at padded (z0, x0)."""
            bump = np.exp(-((xx - x0) ** 2 + (zz - z0) ** 2) / (2 * SIGMA ** 2)) * phys
            bump[bump < 1e-4] = 0.0
            i = NAMES[name]
            base = ps[i].astype(np.float64)
            step = hrel * scale[name] * bump
            Jpm = []
            for sgn in (1.0, -1.0):
                p = list(ps)
                p[i] = (base + sgn * step).astype(np.float32)
                Jpm.append(J(p))
            dm = ((base + step).astype(np.float32).astype(np.float64)
                  - (base - step).astype(np.float32).astype(np.float64)) / 2.0
            return (Jpm[0] - Jpm[1]) / 2.0, float(np.sum(grads[name] * dm))

        res = {n: [] for n in NAMES}
        for z0, x0, name in zip(cz, cx, names):
            fd, ad = fd_at(z0, x0, name, HREL[name])
            res[name].append((int(z0 - E), int(x0 - E), fd, ad))
        # step-size study at each parameter's worst centre: an error that falls as
        # h grows is the FP32 forward's rounding noise in J+ - J-, one that grows
        # as h^2 is the central difference's truncation
        study = {}
        for name, rows in res.items():
            worst = max(rows, key=lambda r: abs(r[3] - r[2]))
            study[name] = {"z": worst[0], "x": worst[1], "steps": []}
            for f in study_factors:
                fd, ad = fd_at(worst[0] + E, worst[1] + E, name, f * HREL[name])
                study[name]["steps"].append({"h": f * HREL[name], "fd": fd, "g_dm": ad,
                                             "rel": abs(ad - fd) / abs(fd) if fd else float("inf")})
    wall = time.perf_counter() - t0
    out = {"nt": nt, "shots": shots, "centres": centres, "gradient_ms": g_ms, "misfit": float(sum(Js)),
           "wall_s": wall, "parameters": {}, "step_study": study}
    for name, rows in res.items():
        fd = np.array([r[2] for r in rows])
        ad = np.array([r[3] for r in rows])
        peak = float(np.abs(fd).max())
        err = float(np.abs(ad - fd).max() / peak) if peak > 0 else float("inf")
        out["parameters"][name] = {"cells": len(rows), "h": HREL[name], "worst_rel_to_largest": err,
                                   "median_rel": float(np.median(np.abs(ad - fd) / np.maximum(np.abs(fd), 1e-300))),
                                   "rows": rows}
        log(f"{name}: {len(rows)} centres, worst |g.dm - fd| / max|fd| = {err:.2e}; at its worst centre, "
            + ", ".join(f"h {s['h']:.1e}: {s['rel']:.2e}" for s in study[name]["steps"]))
    out["ok"] = all(p["worst_rel_to_largest"] <= 1e-3 for p in out["parameters"].values())
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--nt", type=int, default=3000)
    ap.add_argument("--centres", type=int, default=50)
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    r = run(nt=a.nt, centres=a.centres, log=lambda *x: print(*x, file=sys.stderr, flush=True))
    s = json.dumps(r, indent=1)
    if a.json:
        open(a.json, "w").write(s)
    print(json.dumps({k: v for k, v in r.items() if k != "parameters"}))
    sys.exit(0 if r["ok"] else 1)


if __name__ == "__main__":
    main()
