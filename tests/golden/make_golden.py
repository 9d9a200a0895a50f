"""Generates the golden fixtures in tests/golden/*.npz by running the
reference's own programs, built unmodified from the reference sources by
oracle/Makefile (oracle/_ref/strict/), on small seeded cases.

Each fixture holds the case's getpar arguments, its inputs (physical model
arrays, SU source and receiver files as bytes) and every file the reference
wrote (SU traces, raw snapshots, setup dumps, energy text files), keyed by
file name. Run from the repository root:

    make -C oracle REF=<reference checkout> && python tests/golden/make_golden.py

Needs the reference tree (read-only) only through the built programs.
"""
from __future__ import annotations

import json
import os
import shutil
import subprocess
import sys
import tempfile

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
sys.path.insert(0, os.path.join(ROOT, "tti-fdmodeling_b200"))
import synthetic  # noqa: E402

REF = os.path.join(ROOT, "oracle", "_ref", "strict")
OUT = os.path.dirname(os.path.abspath(__file__))

BASE = dict(nz=40, nx=64, nt=300, dx=10, dz=10, dt=0.0008, fpeak=15, ealThick=10, freesurface=0, stype=1,
            seistype=3, mt=1, wsave=3, savew=0, snap_sample=100, mode=1, scalar=1, energy=0, shotID=1)

# name -> (variant, overrides, model kind, source (sx, sdepth) list, receivers (dtr, gdel))
CASES = {
    "coord_basic": ("coordinate_rotation", dict(energy=1), "layered", [(32, 12)], (2, 3)),
    "tensor_basic": ("tensor_rotation", dict(energy=1), "layered", [(32, 12)], (2, 3)),
    "bond_basic": ("bond_transformation", dict(energy=1), "layered", [(32, 12)], (2, 3)),
    "coord_fs": ("coordinate_rotation", dict(freesurface=1), "salt", [(30, 2)], (2, 1)),
    "tensor_fs": ("tensor_rotation", dict(freesurface=1), "salt", [(30, 2)], (2, 1)),
    "bond_fs": ("bond_transformation", dict(freesurface=1), "salt", [(30, 2)], (2, 1)),
    "coord_stype2": ("coordinate_rotation", dict(stype=2, seistype=1, wsave=1), "layered", [(20, 15)], (3, 4)),
    "coord_stype3": ("coordinate_rotation", dict(stype=3, seistype=1, wsave=0), "layered", [(20, 15)], (3, 4)),
    "coord_stype4": ("coordinate_rotation", dict(stype=4, seistype=3, wsave=2), "salt", [(40, 10)], (3, 4)),
    "tensor_stype5": ("tensor_rotation", dict(stype=5, seistype=1, wsave=4), "layered", [(20, 15)], (3, 4)),
    "tensor_stype6": ("tensor_rotation", dict(stype=6, seistype=2, wsave=5), "layered", [(20, 15)], (3, 4)),
    "bond_stype7": ("bond_transformation", dict(stype=7, seistype=1, wsave=1, freesurface=1), "salt",
                    [(25, 6)], (2, 0)),
    "bond_stype8": ("bond_transformation", dict(stype=8, seistype=3, wsave=0), "layered", [(30, 20)], (2, 5)),
    # two sources with overlapping windows, dx != dz (coord:633 uses invdx), mode 2, mt 2, savew 1
    "coord_multi_dxdz": ("coordinate_rotation", dict(dx=12, dz=8, mode=2, mt=2, savew=1, wsave=1,
                                                     snap_sample=75, seistype=3), "layered",
                         [(30, 14), (33, 16)], (1, 6)),
    # no vs/rho files: vp2vs / Gardner defaults (water cells vp <= 1500 -> vs = 0)
    "tensor_defaults": ("tensor_rotation", dict(wsave=2, snap_sample=150, scalar=-1), "layered_water",
                        [(32, 8)], (4, 2)),
    # thin absorbing rim (E = 7): the source window reaches the padded edge
    "bond_thin_rim": ("bond_transformation", dict(ealThick=2, eal_alpha=1.7, seistype=2, wsave=0), "salt",
                      [(0, 0)], (5, 0)),
    # Grids of several 128-row x 16-column kernel tiles (padded 310 x 210: 3 tile rows, 13 tile
    # columns, tile edges at padded row 128 and columns 5 + 16 k). The source windows straddle a
    # tile corner or a column edge; the receiver rows lie on a tile edge (padded row 128) or just
    # above it. Traces and the final p snapshot only (no setup dumps, to keep the files small).
    "coord_tiles": ("coordinate_rotation", dict(nz=280, nx=180, nt=400, seistype=3, wsave=2, snap_sample=399),
                    "salt", [(43, 113)], (1, 113)),
    "tensor_tiles_fs": ("tensor_rotation", dict(nz=280, nx=180, nt=400, freesurface=1, seistype=3, wsave=2,
                                                snap_sample=399), "salt", [(43, 108)], (1, 112)),
    "bond_tiles": ("bond_transformation", dict(nz=280, nx=180, nt=400, seistype=3, wsave=2, snap_sample=399),
                   "salt", [(59, 113)], (2, 112)),
}
# cases whose setup dumps (D_, Beta_, coef*, invrho_, c*_, vs_, rho_) are not kept in the fixture
NO_DUMPS = {"coord_tiles", "tensor_tiles_fs", "bond_tiles"}
DUMP_PREFIXES = ("D_", "Beta_", "coef1_", "coef2_", "invrho_", "c11_", "c13_", "c15_", "c33_", "c35_", "c55_",
                 "vs_", "rho_")


def make_model(kind: str, nz: int, nx: int, seed: int):
    if kind == "layered":
        return synthetic.layered_model(nz, nx, seed=seed)
    if kind == "layered_water":
        m = synthetic.layered_model(nz, nx, seed=seed)
        m.vp[:, : nz // 5] = 1500.0  # a water layer: vp2vs gives vs = 0 there
        return m
    return synthetic.salt_model(nz, nx, seed=seed, nlayers=8)


def run_case(name: str, seed: int) -> dict:
    variant, over, kind, sources, (dtr, gdel) = CASES[name]
    p = dict(BASE)
    p.update(over)
    work = tempfile.mkdtemp(prefix=f"golden_{name}_")
    try:
        m = make_model(kind, p["nz"], p["nx"], seed)
        files = synthetic.write_model(work, m)
        args = [f"{k}={p[k]}" for k in ("nz", "nx", "nt", "dx", "dz", "dt", "fpeak", "ealThick", "freesurface",
                                        "stype", "seistype", "mt", "wsave", "savew", "snap_sample", "mode",
                                        "scalar", "energy", "shotID")]
        if "eal_alpha" in p:
            args.append(f"eal_alpha={p['eal_alpha']}")
        for key in ("vp", "epsilon", "delta", "theta") + (() if kind == "layered_water" else ("vs", "rho")):
            args.append(f"{key}file={files[key]}")
        # source: the reference's own sumksrc2d for one source, SU writer for several
        src_path = os.path.join(work, "src.su")
        if len(sources) == 1:
            sx, sd = sources[0]
            with open(src_path, "wb") as f:
                subprocess.run([os.path.join(REF, "sumksrc2d"), f"sdepth={sd}", f"sx={sx}", f"dt={p['dt']}",
                                f"nt={p['nt']}", f"fpeak={p['fpeak']}", "A=1"], stdout=f, check=True,
                               stderr=subprocess.DEVNULL)
        else:
            w = np.stack([synthetic.ricker(p["nt"], p["dt"], p["fpeak"], amp=1.0 + 0.5 * k)
                          for k in range(len(sources))])
            synthetic.write_su_source(src_path, w, [s[0] for s in sources], [s[1] for s in sources], p["dt"])
        rec_path = os.path.join(work, "rec.su")
        with open(rec_path, "wb") as f:
            subprocess.run([os.path.join(REF, "sumkrcev2d"), f"sx={p['nx'] // 2}", f"gdel={gdel}", "offsetmin=0",
                            f"dtr={dtr}", f"offsetmax={p['nx']}", f"nx={p['nx']}"], stdout=f, check=True,
                           stderr=subprocess.DEVNULL)
        args += [f"sourcefile={src_path}", f"recposfile={rec_path}", "snap_prefix=snap", "trace_prefix=traces"]
        prog = os.path.join(REF, f"sufdmod2dTTIelastic_{variant}")
        env = dict(os.environ, OMP_NUM_THREADS="2", SUSHIM_QUIET="1")
        r = subprocess.run([prog] + args, cwd=work, env=env, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"{name}: reference failed: {r.stderr[-2000:]}")
        out = {}
        for fn in sorted(os.listdir(work)):
            full = os.path.join(work, fn)
            if fn in ("src.su", "rec.su") or fn in {os.path.basename(v) for v in files.values()}:
                continue
            if name in NO_DUMPS and fn.startswith(DUMP_PREFIXES):
                continue
            out["out/" + fn] = np.frombuffer(open(full, "rb").read(), dtype=np.uint8)
        rec = {
            "meta": np.frombuffer(json.dumps(dict(variant=variant, params=p, args=args, kind=kind,
                                                  sources=sources, seed=seed)).encode(), dtype=np.uint8),
            "in/src.su": np.frombuffer(open(src_path, "rb").read(), dtype=np.uint8),
            "in/rec.su": np.frombuffer(open(rec_path, "rb").read(), dtype=np.uint8),
        }
        for k, a in zip(("vp", "vs", "rho", "epsilon", "delta", "theta"), m.arrays()):
            rec["in/" + k] = a
        rec.update(out)
        return rec
    finally:
        shutil.rmtree(work, ignore_errors=True)


def main():
    if not os.path.exists(os.path.join(REF, "sufdmod2dTTIelastic_coordinate_rotation")):
        sys.exit("build the reference first: make -C oracle REF=<reference checkout>")
    only = set(sys.argv[1:])  # case names to (re)generate; none: all of them
    for k, name in enumerate(CASES):
        if only and name not in only:
            continue
        rec = run_case(name, seed=100 + k)
        path = os.path.join(OUT, f"{name}.npz")
        np.savez_compressed(path, **rec)
        print(f"{name}: {len(rec)} entries, {os.path.getsize(path) / 1024:.0f} KiB")


if __name__ == "__main__":
    main()
