"""The padding rule of tti_upload_model_physical: k_expand_physical gives every
padded cell the value of the physical cell at its clamped column and row. It
is checked here (CPU) against padModel2d's own two passes (padmod.c:33-59,
restated loop by loop on a padded array whose interior holds the model) and
against synthetic.pad, the host padding the GPU test compares the device
result with (tests/test_host_buffers_gpu.py)."""
import numpy as np
import pytest

import synthetic


def pad_model_2d(mod: np.ndarray, E: int) -> np.ndarray:
    """padmod.c:33-59 in place on a (Nx, Nz) array: the top and bottom rims of
    the physical columns first, then the left and right rims at full height."""
    Nx, Nz = mod.shape
    for ix in range(E, Nx - E):
        for layer in range(1, E + 1):
            mod[ix, E - layer] = mod[ix, E]
            mod[ix, Nz - E - 1 + layer] = mod[ix, Nz - E - 1]
    for layer in range(1, E + 1):
        for iz in range(Nz):
            mod[E - layer, iz] = mod[E, iz]
            mod[Nx - E - 1 + layer, iz] = mod[Nx - E - 1, iz]
    return mod


def clamped_gather(a: np.ndarray, E: int) -> np.ndarray:
    """What k_expand_physical writes: padded cell (ix, iz) takes physical cell
    (clamp(ix - E, 0, nx - 1), clamp(iz - E, 0, nz - 1))."""
    nx, nz = a.shape
    ix = np.clip(np.arange(nx + 2 * E) - E, 0, nx - 1)
    iz = np.clip(np.arange(nz + 2 * E) - E, 0, nz - 1)
    return a[np.ix_(ix, iz)]


@pytest.mark.parametrize("nx,nz,E", [(1, 1, 1), (3, 7, 5), (40, 64, 15), (13, 2, 7), (9, 30, 45)])
def test_clamped_gather_is_pad_model_2d(nx, nz, E):
    rng = np.random.default_rng(1000 * nx + nz)
    a = rng.standard_normal((nx, nz)).astype(np.float32)
    mod = np.zeros((nx + 2 * E, nz + 2 * E), np.float32)
    mod[E:E + nx, E:E + nz] = a
    ref = pad_model_2d(mod, E)
    assert np.array_equal(clamped_gather(a, E), ref)
    assert np.array_equal(synthetic.pad(a, E), ref)
