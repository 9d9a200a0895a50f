"""GPU parity through the C ABI against the reference build's golden outputs.

Tolerances (the trace tolerance the project targets): traces and snapshots
rel-L2 <= 1e-5 and max |diff| <= 1e-4 of the peak; setup dumps within
2 float ulp (CUDA's double sin/cos may differ from the host libm in the last
place). With TTIFD_EXACT=1 the stencils round like a gcc -ffp-contract=off
build of the reference, and the wavefields then match to <= 1e-6."""
import os

import numpy as np
import pytest

import helpers

pytestmark = pytest.mark.gpu

TRACE_RTOL = 1e-5
TRACE_PEAK = 1e-4


def _compare(name, got, gold, rtol, peak):
    compared = 0
    for fn, ref in gold.items():
        if fn in ("src.txt", "Eng.txt") or fn.startswith(("vs_", "rho_")):
            continue
        assert fn in got, f"{name}: missing {fn}"
        a = np.asarray(got[fn], np.float32).ravel()
        b = np.asarray(ref, np.float32).ravel()
        assert a.size == b.size, f"{name}/{fn}: size"
        if fn.endswith(".txt"):
            fin = np.isfinite(b)
            np.testing.assert_allclose(a[fin], b[fin], rtol=5e-4, atol=1e-30)
        elif fn.startswith(tuple(d + "_" for d in helpers.PARAM_DUMPS)):
            ulp = np.abs(a.view(np.int32).astype(np.int64) - b.view(np.int32).astype(np.int64))
            assert ulp.max() <= 2, f"{name}/{fn}: {ulp.max()} ulp"
        else:
            r = helpers.rel_l2(a, b)
            m = helpers.max_abs_over_peak(a, b)
            assert r <= rtol and m <= peak, f"{name}/{fn}: rel-L2 {r:.3e} max/peak {m:.3e}"
        compared += 1
    assert compared >= 3


@pytest.mark.parametrize("arith", ["reference", "fma"])
@pytest.mark.parametrize("name", helpers.golden_names())
def test_gpu_matches_reference_build(name, arith, gpu_lib, monkeypatch):
    """The default arithmetic (the reference's rounding) and the FMA opt-in
    (TTIFD_EXACT=0) against the reference build's outputs."""
    import ttifd

    monkeypatch.setenv("TTIFD_EXACT", "1" if arith == "reference" else "0")
    case = helpers.load_golden(name)
    got = helpers.run_backend(ttifd.Modeling, case)
    _compare(name, got, helpers.golden_arrays(case), TRACE_RTOL, TRACE_PEAK)


@pytest.mark.parametrize("name", ["coord_basic", "tensor_fs", "bond_fs", "coord_multi_dxdz", "bond_stype8"])
def test_gpu_exact_rounding_mode(name, gpu_lib, monkeypatch):
    import ttifd

    monkeypatch.setenv("TTIFD_EXACT", "1")
    case = helpers.load_golden(name)
    got = helpers.run_backend(ttifd.Modeling, case)
    _compare(name, got, helpers.golden_arrays(case), 1e-6, 1e-6)


@pytest.mark.parametrize("name", ["coord_fs", "tensor_basic", "bond_thin_rim", "coord_stype4", "bond_stype7"])
def test_gpu_one_thread_per_cell_path(name, gpu_lib, monkeypatch):
    """The one-thread-per-cell path (TTIFD_KERNEL=naive, the cross-check of the
    tiled kernels) against the same golden outputs."""
    import ttifd

    monkeypatch.setenv("TTIFD_KERNEL", "naive")
    case = helpers.load_golden(name)
    got = helpers.run_backend(ttifd.Modeling, case)
    _compare(name, got, helpers.golden_arrays(case), TRACE_RTOL, TRACE_PEAK)


