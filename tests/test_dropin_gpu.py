"""The drop-in programs (bin/sufdmod2dTTIelastic_*) run with the golden
cases' own getpar arguments and write the same files as the reference: same
names, SU headers byte for byte, raw vs_/rho_ defaults bit for bit, data
within the trace tolerance. Also checks the reference's error exits."""
import os
import subprocess

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tti-fdmodeling_b200", "bin")


def _programs():
    if not os.path.exists(os.path.join(BIN, "sufdmod2dTTIelastic_coordinate_rotation")):
        subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tti-fdmodeling_b200")], check=True)


def _stage(case, work):
    meta = case["meta"]
    args = []
    for a in meta["args"]:
        k, v = a.split("=", 1)
        if k.endswith("file"):
            v = os.path.join(work, os.path.basename(v))
        args.append(f"{k}={v}")
    for k in ("vp", "vs", "rho", "epsilon", "delta", "theta"):
        if "in/" + k in case:
            case["in/" + k].astype(np.float32).tofile(os.path.join(work, f"{k}.bin"))
    open(os.path.join(work, "src.su"), "wb").write(bytes(case["in/src.su"]))
    open(os.path.join(work, "rec.su"), "wb").write(bytes(case["in/rec.su"]))
    return args


@pytest.mark.parametrize("name", ["coord_basic", "tensor_fs", "bond_fs", "coord_multi_dxdz", "tensor_defaults",
                                  "bond_stype8", "tensor_stype6"])
def test_dropin_writes_reference_files(name, tmp_path, gpu_lib):
    _programs()
    case = helpers.load_golden(name)
    work = str(tmp_path)
    args = _stage(case, work)
    prog = os.path.join(BIN, f"sufdmod2dTTIelastic_{case['meta']['variant']}")
    r = subprocess.run([prog] + args, cwd=work, capture_output=True, text=True, env=dict(os.environ, TTIFD_QUIET="1"))
    assert r.returncode == 0, r.stderr[-2000:]
    assert "Finite difference modeling takes" in r.stdout and "Total time takes" in r.stdout
    for key, val in case.items():
        if not key.startswith("out/"):
            continue
        fn = key[4:]
        path = os.path.join(work, fn)
        assert os.path.exists(path), f"{name}: {fn} not written"
        got, ref = open(path, "rb").read(), bytes(val)
        assert len(got) == len(ref), f"{name}/{fn}: size {len(got)} != {len(ref)}"
        if fn.endswith(".su"):
            gh, gd = helpers.read_su_bytes(got)
            rh, rd = helpers.read_su_bytes(ref)
            n = len(gh)
            for t in range(n):
                off = t * (240 + 4 * gh[t]["ns"])
                assert got[off:off + 240] == ref[off:off + 240], f"{name}/{fn}: header of trace {t} differs"
            assert helpers.rel_l2(gd, rd) <= 1e-5 and helpers.max_abs_over_peak(gd, rd) <= 1e-4, f"{name}/{fn}"
        elif fn.startswith(("vs_", "rho_", "src.txt")):
            assert got == ref, f"{name}/{fn}: not identical"
        elif fn.endswith(".txt"):
            a = np.array([float(x) for x in got.split()])
            b = np.array([float(x) for x in ref.split()])
            fin = np.isfinite(b)
            np.testing.assert_allclose(a[fin], b[fin], rtol=5e-4)
        elif fn.startswith(tuple(d + "_" for d in helpers.PARAM_DUMPS)):
            a = np.frombuffer(got, np.int32).astype(np.int64)
            b = np.frombuffer(ref, np.int32).astype(np.int64)
            assert np.abs(a - b).max() <= 2, f"{name}/{fn}"
        else:  # snapshots
            a = np.frombuffer(got, np.float32)
            b = np.frombuffer(ref, np.float32)
            assert helpers.rel_l2(a, b) <= 1e-5 and helpers.max_abs_over_peak(a, b) <= 1e-4, f"{name}/{fn}"


def test_dropin_error_exits(tmp_path, gpu_lib):
    """Missing required key, unstable dt and an out-of-range source exit with 1."""
    _programs()
    case = helpers.load_golden("coord_basic")
    work = str(tmp_path)
    args = _stage(case, work)
    prog = os.path.join(BIN, "sufdmod2dTTIelastic_coordinate_rotation")

    def run(a):
        return subprocess.run([prog] + a, cwd=work, capture_output=True, text=True,
                              env=dict(os.environ, TTIFD_QUIET="1"))

    r = run([a for a in args if not a.startswith("fpeak=")])
    assert r.returncode == 1 and "peak frequency" in r.stderr
    r = run(args + ["dt=0.01"])
    assert r.returncode == 1 and "unstable" in r.stderr
    import synthetic

    synthetic.write_su_source(os.path.join(work, "bad.su"), np.zeros((1, 300), np.float32), [65], [3], 0.0008)
    r = run([a if not a.startswith("sourcefile=") else f"sourcefile={work}/bad.su" for a in args])
    assert r.returncode == 1 and "2nd dimension (65)" in r.stderr
