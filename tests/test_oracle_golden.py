"""Pins the oracle (CPU restatement) to the reference's own build: every
golden case, every output file. The restatement keeps the reference's
expression order, so traces, snapshots and setup dumps match bit for bit
(energy is summed in double here, in float by the reference)."""
import numpy as np
import pytest

import helpers


@pytest.mark.parametrize("name", helpers.golden_names())
def test_oracle_matches_reference_build(name, oracle_lib):
    case = helpers.load_golden(name)
    gold = helpers.golden_arrays(case)
    got = helpers.run_backend(oracle_lib.Oracle, case)
    compared = 0
    for fn, ref in gold.items():
        if fn in ("src.txt", "Eng.txt") or fn.startswith(("vs_", "rho_")):
            continue
        assert fn in got, f"{name}: no output for reference file {fn}"
        a = np.asarray(got[fn]).ravel()
        b = np.asarray(ref).ravel()
        assert a.size == b.size, f"{name}/{fn}: size {a.size} != {b.size}"
        if fn in ("Ek.txt", "Ep.txt"):
            fin = np.isfinite(b)
            np.testing.assert_allclose(a[fin], b[fin], rtol=2e-4, atol=1e-30, err_msg=f"{name}/{fn}")
        else:
            assert np.array_equal(a.view(np.uint32), b.astype(np.float32).view(np.uint32)), (
                f"{name}/{fn}: not bit-identical, max |diff| = {np.max(np.abs(a - b))}")
        compared += 1
    assert compared >= 3


def test_every_reference_output_is_covered():
    """Each fixture contains traces or snapshots, and at least one case exercises
    each formulation, the free surface and every stype."""
    seen = set()
    for name in helpers.golden_names():
        meta = helpers.load_golden(name)["meta"]
        p = meta["params"]
        seen.add(("variant", meta["variant"]))
        seen.add(("stype", p["stype"]))
        seen.add(("fs", p["freesurface"]))
        seen.add(("mode", p["mode"]))
    for v in ("coordinate_rotation", "tensor_rotation", "bond_transformation"):
        assert ("variant", v) in seen
    for s in range(1, 9):
        assert ("stype", s) in seen
    assert ("fs", 1) in seen and ("mode", 2) in seen
