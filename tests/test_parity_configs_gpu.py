"""Parity at the benchmark configurations with the default arithmetic, after
the full number of steps: traces and snapshots within rel-L2 <= 1e-5 and
max |diff| <= 1e-4 of the peak, SU headers byte-identical.

* program against program (tests/parity_configs.py): the reference's own
  OpenMP build and this library's drop-in programs on the same files,
  layered_200x400 in full (nt=1501, both runs) and salt_1126x7872 (all three
  formulations) over its first 301 steps. The full salt_1126x7872 (nt=5001)
  runs through the same script; its record is kept with the profiles.
* batched against the reference program: the 64-shot batch shots64_1126x3000
  and the 48-model uneven batch models48_uneven in one batch each on the GPU,
  over their first 301 steps, with two instances of each run alone through
  the reference build. The full-length record (nt 4000 and 1000-4000) is
  kept with the profiles.
* library against the CPU restatement (the oracle, itself bit-identical to
  the reference build on every golden case): layered_200x400's second run
  through the C ABI, so the check stands where the reference build is not at
  hand.
"""
import os
import sys

import numpy as np
import pytest

import synthetic

sys.path.insert(0, os.path.dirname(os.path.abspath(__file__)))
import parity_configs  # noqa: E402

pytestmark = pytest.mark.gpu

need_programs = pytest.mark.skipif(not parity_configs.available(),
                                   reason="oracle/_ref or the drop-in programs are not built")


def _check(recs):
    assert recs
    for r in recs:
        bad = [f for f in r["files"] if not f["ok"]]
        assert r["ok"] and not bad, (r["variant"], r["run"], bad)


@need_programs
def test_layered_200x400_full_programs(gpu_lib):
    recs = parity_configs.run_config("layered_200x400")
    _check(recs)
    names = {f["file"] for r in recs for f in r["files"]}
    assert any(n.startswith("snap_p_00200_00400_01200ms") for n in names)  # the 1200 ms snapshot
    assert any(n.startswith("traces_vx_0001_01501") for n in names)


@need_programs
@pytest.mark.parametrize("variant", parity_configs.VARIANTS)
def test_salt_1126x7872_first_steps_programs(variant, gpu_lib):
    _check(parity_configs.run_config("salt_1126x7872", nt=301, variants=[variant]))


def test_layered_200x400_library_against_restatement(gpu_lib, monkeypatch):
    import pyoracle
    import ttifd

    monkeypatch.delenv("TTIFD_EXACT", raising=False)
    c = parity_configs.CONFIGS["layered_200x400"]
    _, nz, nx, seed = c["model"]
    cfg = dict(variant="coordinate_rotation", nz=nz, nx=nx, nt=c["nt"], dx=10.0, dz=10.0, dt=c["dt"],
               fpeak=float(c["fpeak"]), ealThick=c["ealThick"], freesurface=0, stype=1, seistype=2, mt=1, wsave=2,
               snap_sample=750)
    m = synthetic.layered_model(nz, nx, seed=seed)
    pads = synthetic.padded(m, cfg["ealThick"])
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])
    out = {}
    for name, make in (("gpu", ttifd.Modeling), ("oracle", pyoracle.Oracle)):
        snaps = {}
        with make(**cfg) as h:
            h.upload_model(*pads)
            h.set_source([c["source"][0]], [c["source"][1]], w[None, :])
            h.set_receivers(2, np.arange(nx), c["rec_z"])
            h.run(lambda it, kind, a: snaps.__setitem__(it, np.array(a, copy=True)))
            out[name] = (h.fetch_traces(2), snaps)
    (tg, sg), (to, so) = out["gpu"], out["oracle"]
    assert sorted(sg) == sorted(so) == [0, 750, 1500]
    for a, b in [(tg, to)] + [(sg[k], so[k]) for k in (750, 1500)]:
        rel, mx = parity_configs._metrics(a, b)
        assert rel <= parity_configs.TRACE_RTOL and mx <= parity_configs.TRACE_PEAK, (rel, mx)


@need_programs
@pytest.mark.parametrize("name,pick", [("shots64_1126x3000", [0, 63]), ("models48_uneven", [5, 17])])
def test_batched_configs_first_steps(name, pick, gpu_lib):
    recs = parity_configs.run_batched(name, pick=pick, nt=301)
    assert [r["instance"] for r in recs] == pick
    for r in recs:
        assert r["ok"], r
