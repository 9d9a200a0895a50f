"""Trace and snapshot parity at the benchmark configurations, program against
program: the reference's own OpenMP build (oracle/_ref/strict, gcc -O2
-ffp-contract=off) and this library's drop-in programs
(tti-fdmodeling_b200/bin, GPU) run with the same getpar arguments on the same
input files, and every output file is compared:

  SU traces     240-byte headers byte-identical; samples rel-L2 <= 1e-5 and
                max |diff| <= 1e-4 of the component's peak;
  snapshots     the same two bounds per file;
  setup dumps   (D_, Beta_, coef*, invrho_, c*_) within 2 float ulp.

Configurations (seeded synthetic inputs with the benchmark's shapes; the
reference's demo files are not available):

  layered_200x400
      coordinate rotation, nz=200 nx=400 dx=dz=10 m, nt=1501, dt=0.8 ms, 5
      flat layers (seed 0), vs = vp/1.8, rho = 310 vp^0.25, one 15 Hz Ricker
      at (z=20, x=200), 400 receivers on z=5, ealThick=40, no free surface.
      Two runs: seistype=1 (vx, vz); seistype=2 with wsave=2 and
      snap_sample=750 (p snapshots at 0, 600 and 1200 ms).
  salt_1126x7872
      the three formulations on the salt-like 1126 x 7872 model (seed 1),
      nt=5001, dt=0.8 ms, one 12 Hz Ricker at the surface centre (sdepth 2,
      sx 3936), 7872 receivers on z=2, ealThick=60, free surface, seistype=3,
      wsave=2, snap_sample=1250 (p at 0, 1000, ..., 4000 ms).
  shots64_1126x3000, models48_uneven
      batched (run_batched below): 64 shots on a 1126 x 3000 crop of the
      salt-like model, and 48 layered models of seeded sizes.

Usage (from the repository root, after `make -C oracle REF=...` built
oracle/_ref and `make -C tti-fdmodeling_b200` the programs):

    python tests/parity_configs.py layered_200x400 [--json out.json]
    python tests/parity_configs.py salt_1126x7872 [--nt 5001] [--variants coordinate_rotation ...]

The -m gpu tests call run_config at full size for layered_200x400 and with a
short nt for salt_1126x7872.
"""
from __future__ import annotations

import argparse
import json
import os
import shutil
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tti-fdmodeling_b200"))
import synthetic  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "strict")
OURS = os.path.join(ROOT, "tti-fdmodeling_b200", "bin")
VARIANTS = ("coordinate_rotation", "tensor_rotation", "bond_transformation")
TRACE_RTOL, TRACE_PEAK = 1e-5, 1e-4
DUMPS = ("D_", "Beta_", "coef1_", "coef2_", "invrho_", "c11_", "c13_", "c15_", "c33_", "c35_", "c55_")

CONFIGS = {
    "layered_200x400": dict(model=("layered", 200, 400, 0), nt=1501, dx=10, dz=10, dt=0.0008, fpeak=15, ealThick=40,
                    freesurface=0, source=(200, 20), rec_z=5, variants=("coordinate_rotation",),
                    runs=[dict(seistype=1, wsave=0), dict(seistype=2, wsave=2, snap_sample=750)]),
    "salt_1126x7872": dict(model=("salt", 1126, 7872, 1), nt=5001, dx=10, dz=10, dt=0.0008, fpeak=12, ealThick=60,
                    freesurface=1, source=(3936, 2), rec_z=2, variants=VARIANTS,
                    runs=[dict(seistype=3, wsave=2, snap_sample=1250)]),
}


def available() -> bool:
    return all(os.path.exists(os.path.join(d, f"sufdmod2dTTIelastic_{v}")) for d in (REF, OURS) for v in VARIANTS)


def _model(kind, nz, nx, seed):
    return synthetic.layered_model(nz, nx, seed=seed) if kind == "layered" else synthetic.salt_model(nz, nx, seed=seed)


def _su(path):
    """(headers as bytes per trace, data [ntr][ns]) of an SU file."""
    raw = open(path, "rb").read()
    ns = int(np.frombuffer(raw[114:116], "<u2")[0])
    rec = 240 + 4 * ns
    ntr = len(raw) // rec
    a = np.frombuffer(raw[: ntr * rec], np.uint8).reshape(ntr, rec)
    return a[:, :240].tobytes(), a[:, 240:].copy().view("<f4").reshape(ntr, ns)


def _metrics(a, b):
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den, peak = np.linalg.norm(b), np.max(np.abs(b))
    d = a - b
    return (float(np.linalg.norm(d) / den) if den > 0 else float(np.linalg.norm(d)),
            float(np.max(np.abs(d)) / peak) if peak > 0 else float(np.max(np.abs(d))))


def compare_dirs(ref_dir, our_dir, skip):
    """Compares every output file of the reference run with ours."""
    res = []
    for fn in sorted(os.listdir(ref_dir)):
        if fn in skip or fn.endswith(".txt"):
            continue
        r = {"file": fn}
        ours = os.path.join(our_dir, fn)
        if not os.path.exists(ours):
            r.update(ok=False, why="missing in our output")
            res.append(r)
            continue
        if fn.endswith(".su"):
            hr, dr = _su(os.path.join(ref_dir, fn))
            ho, do = _su(ours)
            rel, mx = _metrics(do, dr) if do.shape == dr.shape else (np.inf, np.inf)
            r.update(kind="traces", headers_equal=hr == ho, rel_l2=rel, max_over_peak=mx,
                     ok=hr == ho and rel <= TRACE_RTOL and mx <= TRACE_PEAK)
        elif fn.startswith(DUMPS):
            a = np.fromfile(ours, np.float32).view(np.int32).astype(np.int64)
            b = np.fromfile(os.path.join(ref_dir, fn), np.float32).view(np.int32).astype(np.int64)
            ulp = int(np.abs(a - b).max()) if a.size == b.size else 1 << 30
            r.update(kind="setup dump", max_ulp=ulp, ok=ulp <= 2)
        else:
            a = np.fromfile(ours, np.float32)
            b = np.fromfile(os.path.join(ref_dir, fn), np.float32)
            rel, mx = _metrics(a, b) if a.size == b.size else (np.inf, np.inf)
            r.update(kind="snapshot" if "snap" in fn else "binary", rel_l2=rel, max_over_peak=mx,
                     ok=rel <= TRACE_RTOL and mx <= TRACE_PEAK)
        res.append(r)
    return res


def run_config(name, nt=None, variants=None, threads=None, log=print):
    """Runs one configuration through both programs; returns a list of
    per-run records with the per-file comparison and the programs' timings."""
    c = CONFIGS[name]
    nt = nt or c["nt"]
    kind, nz, nx, seed = c["model"]
    m = _model(kind, nz, nx, seed)
    work = tempfile.mkdtemp(prefix=f"parity_{name}_")
    out = []
    try:
        files = synthetic.write_model(work, m)
        sx, sd = c["source"]
        wav = synthetic.ricker(nt, c["dt"], c["fpeak"])
        synthetic.write_su_source(os.path.join(work, "src.su"), wav[None, :], [sx], [sd], c["dt"])
        synthetic.write_su_receivers(os.path.join(work, "rec.su"), np.arange(nx), np.full(nx, c["rec_z"]))
        env = dict(os.environ, OMP_NUM_THREADS=str(threads or os.cpu_count() or 1), OMP_PROC_BIND="close",
                   OMP_PLACES="cores", SUSHIM_QUIET="1")
        for variant in variants or c["variants"]:
            for run in c["runs"]:
                p = dict(nz=nz, nx=nx, nt=nt, dx=c["dx"], dz=c["dz"], dt=c["dt"], fpeak=c["fpeak"],
                         ealThick=c["ealThick"], freesurface=c["freesurface"], stype=1, mt=1, savew=0, shotID=1,
                         snap_sample=1)
                p.update(run)
                args = [f"{k}={v}" for k, v in p.items()]
                args += [f"{k}file={files[k]}" for k in ("vp", "vs", "rho", "epsilon", "delta", "theta")]
                args += [f"sourcefile={work}/src.su", f"recposfile={work}/rec.su", "snap_prefix=snap",
                         "trace_prefix=traces"]
                rec = {"config": name, "variant": variant, "nt": nt, "run": run, "files": None}
                dirs = {}
                for side, d in (("reference", REF), ("ours", OURS)):
                    wd = os.path.join(work, f"{variant}_{side}_{len(out)}")
                    os.makedirs(wd)
                    t0 = time.perf_counter()
                    r = subprocess.run([os.path.join(d, f"sufdmod2dTTIelastic_{variant}")] + args, cwd=wd, env=env,
                                       capture_output=True, text=True)
                    rec[f"{side}_wall_s"] = time.perf_counter() - t0
                    if r.returncode != 0:
                        raise RuntimeError(f"{side} {variant} failed ({r.returncode}): {r.stderr[-800:]}")
                    for line in r.stdout.splitlines():
                        if "Finite difference modeling takes" in line:
                            rec[f"{side}_loop_s"] = float(line.split("takes")[1].split()[0])
                    dirs[side] = wd
                rec["files"] = compare_dirs(dirs["reference"], dirs["ours"], skip=set())
                rec["ok"] = all(f["ok"] for f in rec["files"]) and len(rec["files"]) > 0
                out.append(rec)
                worst = max((f.get("rel_l2", 0.0) for f in rec["files"]), default=0.0)
                log(f"{name} {variant} {run}: {'ok' if rec['ok'] else 'FAIL'}; {len(rec['files'])} files, "
                    f"worst rel-L2 {worst:.2e}; loop {rec.get('reference_loop_s')} s (reference) vs "
                    f"{rec.get('ours_loop_s')} s (ours)")
                for d in dirs.values():
                    shutil.rmtree(d, ignore_errors=True)
    finally:
        shutil.rmtree(work, ignore_errors=True)
    return out


BATCHED = ("shots64_1126x3000", "models48_uneven")


def batched_setup(name, nt=None):
    """The instances of a batched configuration: (list of batch model configs,
    model_of, per model: the physical model, per instance: (model, sx, sz,
    nt, receiver x positions))."""
    if name == "shots64_1126x3000":
        # 64 shots 120 m apart on the nx=3000 crop (columns 2436..5435) of the salt-like 1126 x 7872 model
        nt = nt or 4000
        m = synthetic.crop(synthetic.salt_model(1126, 7872, seed=1), 2436, 3000)
        cfg = dict(variant="coordinate_rotation", nz=1126, nx=3000, nt=nt, dx=10.0, dz=10.0, dt=0.0008, fpeak=10.0,
                   ealThick=50, freesurface=1, stype=1, seistype=1, mt=1)
        inst = [(0, 1122 + 12 * i, 2, nt, np.arange(3000)) for i in range(64)]
        return [cfg], [0] * 64, [m], inst
    # models48_uneven: 48 layered models of seeded sizes, one centred shot each (as bench.py's uneven batch)
    rng = np.random.default_rng(4)
    sizes = [(int(rng.integers(256, 1127)), int(rng.integers(256, 4097)), int(rng.integers(1000, 4001)))
             for _ in range(48)]
    cfgs = [dict(variant="coordinate_rotation", nz=nz, nx=nx, nt=nt or t, dx=10.0, dz=10.0, dt=0.0008, fpeak=15.0,
                 ealThick=40, freesurface=0, stype=1, seistype=1, mt=1) for nz, nx, t in sizes]
    models = [synthetic.layered_model(nz, nx, seed=100 + k) for k, (nz, nx, _) in enumerate(sizes)]
    inst = [(k, c["nx"] // 2, 2, c["nt"], np.arange(c["nx"])) for k, c in enumerate(cfgs)]
    return cfgs, list(range(48)), models, inst


def run_batched(name, pick=None, nt=None, threads=None, log=print):
    """Every instance of a batched configuration in one batch on the GPU
    (ttifd.Batch: one launch per half-step for all of them), against the
    reference program run alone for the instances `pick` (default: shots64_1126x3000
    shots 0, 31, 63; models48_uneven the three smallest models); vx and vz traces
    compared with the bounds of the plain runs."""
    import ttifd

    cfgs, model_of, models, inst = batched_setup(name, nt)
    if pick is None:
        pick = [0, 31, 63] if name == "shots64_1126x3000" else sorted(
            range(len(inst)), key=lambda i: cfgs[model_of[i]]["nz"] * cfgs[model_of[i]]["nx"])[:3]
    t0 = time.perf_counter()
    ours = {}
    with ttifd.Batch(cfgs, model_of) as b:
        for k, m in enumerate(models):
            b.upload_model(k, *synthetic.padded(m, cfgs[k]["ealThick"]))
        for i, (k, sx, sz, t, gx) in enumerate(inst):
            c = cfgs[k]
            h = b.instances[i]
            h.set_source([sx], [sz], synthetic.ricker(t, c["dt"], c["fpeak"])[None, :])
            for comp in (0, 1):
                h.set_receivers(comp, gx, 2)
        b.run()
        for i in pick:
            ours[i] = [b.instances[i].fetch_traces(comp) for comp in (0, 1)]
    ours_wall = time.perf_counter() - t0
    env = dict(os.environ, OMP_NUM_THREADS=str(threads or os.cpu_count() or 1), OMP_PROC_BIND="close",
               OMP_PLACES="cores", SUSHIM_QUIET="1")
    out = []
    for i in pick:
        k, sx, sz, t, gx = inst[i]
        c = cfgs[k]
        work = tempfile.mkdtemp(prefix=f"parity_{name}_{i}_")
        try:
            files = synthetic.write_model(work, models[k])
            synthetic.write_su_source(os.path.join(work, "src.su"), synthetic.ricker(t, c["dt"], c["fpeak"])[None, :],
                                      [sx], [sz], c["dt"])
            synthetic.write_su_receivers(os.path.join(work, "rec.su"), gx, np.full(gx.size, 2))
            p = dict(nz=c["nz"], nx=c["nx"], nt=t, dx=c["dx"], dz=c["dz"], dt=c["dt"], fpeak=c["fpeak"],
                     ealThick=c["ealThick"], freesurface=c["freesurface"], stype=1, seistype=1, mt=1, wsave=0,
                     savew=0, shotID=1, snap_sample=1)
            args = [f"{a}={v}" for a, v in p.items()]
            args += [f"{a}file={files[a]}" for a in ("vp", "vs", "rho", "epsilon", "delta", "theta")]
            args += [f"sourcefile={work}/src.su", f"recposfile={work}/rec.su", "trace_prefix=traces"]
            r = subprocess.run([os.path.join(REF, "sufdmod2dTTIelastic_coordinate_rotation")] + args, cwd=work,
                               env=env, capture_output=True, text=True)
            if r.returncode != 0:
                raise RuntimeError(f"reference instance {i} failed ({r.returncode}): {r.stderr[-800:]}")
            rec = {"config": name, "instance": i, "nz": c["nz"], "nx": c["nx"], "nt": t, "sx": sx, "files": []}
            for line in r.stdout.splitlines():
                if "Finite difference modeling takes" in line:
                    rec["reference_loop_s"] = float(line.split("takes")[1].split()[0])
            for comp, tag in ((0, "vx"), (1, "vz")):
                fn = [f for f in os.listdir(work) if f.startswith(f"traces_{tag}_") and f.endswith(".su")]
                _, dr = _su(os.path.join(work, fn[0]))
                do = ours[i][comp]
                rel, mx = _metrics(do, dr) if do.shape == dr.shape else (np.inf, np.inf)
                rec["files"].append({"file": fn[0], "kind": "traces", "rel_l2": rel, "max_over_peak": mx,
                                     "ok": rel <= TRACE_RTOL and mx <= TRACE_PEAK})
            rec["ok"] = all(f["ok"] for f in rec["files"])
            out.append(rec)
            log(f"{name} instance {i} ({c['nz']}x{c['nx']}, nt {t}, sx {sx}): {'ok' if rec['ok'] else 'FAIL'}; "
                f"worst rel-L2 {max(f['rel_l2'] for f in rec['files']):.2e}; reference loop "
                f"{rec.get('reference_loop_s')} s")
        finally:
            shutil.rmtree(work, ignore_errors=True)
    for rec in out:
        rec["batch_wall_s"] = ours_wall  # the whole batch, every instance, upload to fetch
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("config", choices=sorted(CONFIGS) + list(BATCHED))
    ap.add_argument("--nt", type=int, default=None)
    ap.add_argument("--variants", nargs="*", default=None)
    ap.add_argument("--instances", type=int, nargs="*", default=None, help="batched configs: instances to check")
    ap.add_argument("--json", default=None)
    a = ap.parse_args()
    if not available():
        sys.exit("build oracle/_ref (make -C oracle REF=...) and the drop-in programs first")
    lg = lambda *x: print(*x, file=sys.stderr, flush=True)  # noqa: E731
    if a.config in BATCHED:
        recs = run_batched(a.config, pick=a.instances, nt=a.nt, log=lg)
    else:
        recs = run_config(a.config, nt=a.nt, variants=a.variants, log=lg)
    s = json.dumps({"cores": os.cpu_count(), "runs": recs}, indent=1)
    if a.json:
        open(a.json, "w").write(s)
    print(s)
    sys.exit(0 if all(r["ok"] for r in recs) else 1)


if __name__ == "__main__":
    main()
