"""The C-ABI library loads on a CPU-only host and exports every entry point
include/ttifd.h declares (no compute calls: there may be no GPU here)."""
import ctypes
import os
import re

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    names = set()
    for fn in os.listdir(os.path.join(ROOT, "include")):
        if fn.endswith(".h"):
            src = open(os.path.join(ROOT, "include", fn)).read()
            src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
            names.update(re.findall(r"\b(tti_\w+)\s*\(", src))
    return sorted(names)


def test_header_declares_the_boundary():
    names = declared_symbols()
    for must in ("tti_create", "tti_upload_model", "tti_set_source", "tti_set_receivers", "tti_run",
                 "tti_fetch_traces", "tti_destroy", "tti_last_error"):
        assert must in names


def test_library_exports_every_declared_symbol(gpu_lib):
    lib = gpu_lib
    missing = [n for n in declared_symbols() if not hasattr(lib, n)]
    assert not missing, f"not exported: {missing}"


def test_python_binding_covers_the_header():
    import ttifd

    names = set(declared_symbols())
    assert set(ttifd.EXPORTS) <= names


def test_create_without_gpu_fails_cleanly(gpu_lib):
    """On a host without a GPU tti_create must return an error, not crash."""
    import torch

    if torch.cuda.is_available():
        pytest.skip("a GPU is present")
    import ttifd

    with pytest.raises(ttifd.TTIError) as e:
        ttifd.Modeling(nz=10, nx=10, nt=10, dx=10, dz=10, dt=0.001, fpeak=10)
    assert e.value.code == ttifd.ERR_CUDA


@pytest.mark.parametrize("models,model_of,what", [
    ([dict(wsave=2)], [0], "traces only"),
    ([dict(energy=1)], [0], "traces only"),
    ([dict(), dict(variant=1)], [0, 1], "same formulation"),
    ([dict()], [0, 1], "out of range"),
    ([dict(), dict()], [0, 0], "has no instance"),
])
def test_batch_argument_checks(models, model_of, what, gpu_lib):
    """tti_batch_create validates its arguments on the host, before any device work."""
    import ttifd

    base = dict(nz=20, nx=30, nt=10, dx=10, dz=10, dt=0.001, fpeak=10)
    with pytest.raises(ttifd.TTIError) as e:
        ttifd.Batch([dict(base, **m) for m in models], model_of)
    assert e.value.code == ttifd.ERR_ARG
    assert what in str(e.value)


@pytest.mark.parametrize("shape", [(3, 5), (7, 1126), (2400, 1126), (7872, 1126)])
def test_snapshot_copy_is_exact(shape):
    """The wrapper hands each snapshot to the callback as a copy of the library's
    buffer; large ones are copied in row blocks from several threads."""
    import ttifd

    a = np.random.default_rng(1).standard_normal(shape).astype(np.float32)
    b = ttifd._copy(a)
    assert b is not a and b.shape == a.shape and b.dtype == a.dtype
    assert np.array_equal(a, b)
