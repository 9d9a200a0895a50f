"""Test-side host logic: turns a golden case (getpar arguments + input files)
into calls on either the CUDA library (ttifd.Modeling) or the oracle
(pyoracle.Oracle), and names the outputs like the reference's files so they
compare key by key with the fixtures."""
from __future__ import annotations

import io
import json
import math
import os

import numpy as np

import synthetic

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
PARAM_DUMPS = ["D", "Beta", "coef1", "coef2", "invrho", "c11", "c13", "c15", "c33", "c35", "c55"]


def golden_names():
    return sorted(f[:-4] for f in os.listdir(GOLDEN) if f.endswith(".npz"))


def load_golden(name: str) -> dict:
    z = np.load(os.path.join(GOLDEN, name + ".npz"))
    d = {k: z[k] for k in z.files}
    d["meta"] = json.loads(bytes(d["meta"]).decode())
    return d


def head_scalar_read(key: float, scalar: int) -> int:
    """src/lib/supro/head.c:37-51"""
    temp = int((-1.0 if scalar < 0 else 1.0) * math.log10(abs(scalar)))
    return int(float(np.float32(key)) * 10.0 ** temp)


def read_su_bytes(b: bytes):
    path = io.BytesIO(b)
    import tempfile

    with tempfile.NamedTemporaryFile(suffix=".su", delete=False) as f:
        f.write(b)
        name = f.name
    try:
        return synthetic.read_su(name)
    finally:
        os.unlink(name)


def geometry(case: dict):
    """read2dsource / read2dreceiver (obsinfo.c:34-87, 175-230) on the fixture's files."""
    p = case["meta"]["params"]
    hs, data = read_su_bytes(bytes(case["in/src.su"]))
    sx = [head_scalar_read(h["sx"], h["scalco"]) for h in hs]
    sz = [head_scalar_read(h["sdepth"], h["scalel"]) for h in hs]
    nt = p["nt"]
    src = np.zeros((len(hs), nt), np.float32)
    n = min(nt, data.shape[1])
    src[:, :n] = data[:, :n]
    hr, rd = read_su_bytes(bytes(case["in/rec.su"]))
    gx = rd[0].astype(np.int32)
    gz = rd[1].astype(np.int32)
    return np.array(sx, np.int32), np.array(sz, np.int32), src, gx, gz


def model_inputs(case: dict, E: int):
    p = case["meta"]["params"]
    vp = case["in/vp"]
    if case["meta"]["kind"] == "layered_water":
        vs = np.where(vp <= 1500.0, 0.0, 0.577350269189626 * vp.astype(np.float64)).astype(np.float32)
        rho = np.where(vp <= 1500.0, 1000.0, 1741.0 * np.power(vp.astype(np.float64) / 1000.0, 0.25))
        rho = rho.astype(np.float32)
    else:
        vs, rho = case["in/vs"], case["in/rho"]
    arrs = [vp, vs, rho, case["in/epsilon"], case["in/delta"], case["in/theta"]]
    assert vp.shape == (p["nx"], p["nz"])
    return [synthetic.pad(a, E) for a in arrs]


def config_of(case: dict) -> dict:
    p = case["meta"]["params"]
    cfg = {k: p[k] for k in ("nz", "nx", "nt", "dx", "dz", "dt", "fpeak", "ealThick", "freesurface", "stype",
                             "seistype", "mt", "wsave", "savew", "snap_sample", "mode", "scalar", "energy")}
    cfg["eal_alpha"] = p.get("eal_alpha", -1.0)
    cfg["variant"] = case["meta"]["variant"]
    return cfg


SNAP_NAMES = {1: "vx", 2: "vz", 3: "p", 4: "vxp", 5: "vzp", 6: "vxs", 7: "vzs"}


def run_backend(make, case: dict) -> dict:
    """Runs one golden case through a backend; returns {reference file name: array}."""
    cfg = config_of(case)
    p = case["meta"]["params"]
    out = {}
    with make(**cfg) as m:
        inputs = model_inputs(case, m.E)
        m.upload_model(*inputs)
        for name in PARAM_DUMPS:
            try:
                out[f"{name}_{m.Nz:05d}_{m.Nx:05d}.bin"] = m.fetch_param(name)
            except Exception:
                pass
        sx, sz, src, gx, gz = geometry(case)
        m.set_source(sx, sz, src)
        st = p["seistype"]
        if st in (1, 3):
            m.set_receivers(0, gx, gz)
            m.set_receivers(1, gx, gz)
        if st in (2, 3):
            m.set_receivers(2, gx, gz)
        nzo, nxo = (p["nz"], p["nx"]) if p["savew"] == 0 else (m.Nz, m.Nx)

        def snap(it, kind, arr):
            ms = int(np.float32(1000 * it) * np.float32(p["dt"]))
            out[f"snap_{SNAP_NAMES[kind]}_{nzo:05d}_{nxo:05d}_{ms:05d}ms.bin"] = arr

        m.run(snap)
        dtms = np.float32(p["dt"] * p["mt"]) * np.float32(1000.0)
        for kind, comp in ((0, "vx"), (1, "vz"), (2, "p")):
            if (kind < 2 and st in (1, 3)) or (kind == 2 and st in (2, 3)):
                tr = m.fetch_traces(kind)
                out[f"traces_{comp}_{p['shotID']:04d}_{m.nts:05d}_{tr.shape[0]:05d}_{dtms:05.2f}ms.su"] = tr
        if p["energy"] == 1:
            ek, ep = m.fetch_energy()
            out["Ek.txt"], out["Ep.txt"] = ek, ep
    return out


def golden_arrays(case: dict) -> dict:
    """The fixture's output files decoded to arrays (SU -> trace data)."""
    res = {}
    for k, v in case.items():
        if not k.startswith("out/"):
            continue
        fn = k[4:]
        b = bytes(v)
        if fn.endswith(".su"):
            res[fn] = read_su_bytes(b)[1]
        elif fn.endswith(".bin"):
            res[fn] = np.frombuffer(b, dtype=np.float32)
        elif fn.endswith(".txt"):
            res[fn] = np.array([float(x) for x in b.decode().split()], dtype=np.float64)
    return res


def rel_l2(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    den = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / den) if den > 0 else float(np.linalg.norm(a - b))


def max_abs_over_peak(a, b) -> float:
    a = np.asarray(a, np.float64).ravel()
    b = np.asarray(b, np.float64).ravel()
    peak = np.max(np.abs(b))
    return float(np.max(np.abs(a - b)) / peak) if peak > 0 else float(np.max(np.abs(a - b)))
