"""Input utilities (sumksrc2d, sumkrcev2d, cutbin2d) against the reference's
own builds of them: byte for byte on the files stored in the golden fixtures
(made by the reference programs), and on more argument sets when the
reference build (oracle/_ref/strict) is present."""
import os
import subprocess

import numpy as np
import pytest

import helpers

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
BIN = os.path.join(ROOT, "tti-fdmodeling_b200", "bin")
REF = os.path.join(ROOT, "oracle", "_ref", "strict")


@pytest.fixture(scope="module", autouse=True)
def utilities():
    subprocess.run(["make", "-s", "-C", os.path.join(ROOT, "tti-fdmodeling_b200"), "utils"], check=True)


def run(prog, args, stdin=None, ref=False):
    exe = os.path.join(REF if ref else BIN, prog)
    r = subprocess.run([exe] + args, input=stdin, capture_output=True, env=dict(os.environ, TTIFD_QUIET="1",
                                                                                 SUSHIM_QUIET="1"))
    assert r.returncode == 0, r.stderr.decode()[-500:]
    return r.stdout


@pytest.mark.parametrize("name", [n for n in helpers.golden_names()
                                  if len(helpers.load_golden(n)["meta"]["sources"]) == 1])
def test_source_and_receiver_files_match_fixtures(name):
    case = helpers.load_golden(name)
    meta = case["meta"]
    p = meta["params"]
    sx, sd = meta["sources"][0]
    src = run("sumksrc2d", [f"sdepth={sd}", f"sx={sx}", f"dt={p['dt']}", f"nt={p['nt']}", f"fpeak={p['fpeak']}",
                            "A=1"])
    assert src == bytes(case["in/src.su"])
    rec = bytes(case["in/rec.su"])
    hs, data = helpers.read_su_bytes(rec)
    gdel = int(data[1][0]) if data.shape[1] else 0
    dtr = int(hs[0]["d1"])
    got = run("sumkrcev2d", [f"sx={p['nx'] // 2}", f"gdel={gdel}", "offsetmin=0", f"dtr={dtr}",
                             f"offsetmax={p['nx']}", f"nx={p['nx']}"])
    assert got == rec


needs_ref = pytest.mark.skipif(not os.path.exists(os.path.join(REF, "sumksrc2d")),
                               reason="reference build not present")


@needs_ref
@pytest.mark.parametrize("wtype", [1, 2, 3, 4])
def test_wavelet_types_match_reference(wtype):
    args = ["sdepth=7", "sx=31", "dt=0.0005", "nt=777", "fpeak=23", "A=2.5", f"wtype={wtype}", "delay=0.05"]
    assert run("sumksrc2d", args) == run("sumksrc2d", args, ref=True)


@needs_ref
@pytest.mark.parametrize("mode,offmin,offmax,dtr,sx", [(0, 0, 50, 3, 40), (0, 5, 30, 2, 40), (1, 0, 25, 1, 10),
                                                      (2, 3, 100, 4, 77), (0, 0, 1000, 1, 0)])
def test_receiver_modes_match_reference(mode, offmin, offmax, dtr, sx):
    args = [f"sx={sx}", "gdel=3", f"offsetmin={offmin}", f"dtr={dtr}", f"offsetmax={offmax}", "nx=90",
            f"mode={mode}"]
    assert run("sumkrcev2d", args) == run("sumkrcev2d", args, ref=True)


def test_cutbin2d_matches_slicing():
    a = np.random.default_rng(0).standard_normal((37, 53)).astype(np.float32)  # n2=37 records of n1=53
    out = run("cutbin2d", ["n1=53", "n2=37", "fx1=4", "fx2=9", "nx1=20", "nx2=11"], stdin=a.tobytes())
    np.testing.assert_array_equal(np.frombuffer(out, np.float32).reshape(11, 20), a[9:20, 4:24])


@needs_ref
def test_cutbin2d_matches_reference():
    a = np.random.default_rng(1).standard_normal((41, 29)).astype(np.float32)
    args = ["n1=29", "n2=41", "fx1=3", "fx2=6", "nx1=17", "nx2=30"]
    assert run("cutbin2d", args, stdin=a.tobytes()) == run("cutbin2d", args, stdin=a.tobytes(), ref=True)
