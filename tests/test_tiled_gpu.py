"""Tiled half-step kernels vs the one-thread-per-cell kernels on grids of
several tiles. In the exact rounding mode both paths perform the same
operations in the same order, so the wavefields, traces and snapshots must be
bit-identical."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu


def _run(kernel, monkeypatch, variant, fs, stype, nz=300, nx=260, nt=160):
    import ttifd

    monkeypatch.setenv("TTIFD_EXACT", "1")
    monkeypatch.setenv("TTIFD_KERNEL", kernel)
    cfg = dict(variant=variant, nz=nz, nx=nx, nt=nt, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0, ealThick=12,
               freesurface=fs, stype=stype, seistype=3, mt=2, wsave=3, snap_sample=50)
    m = synthetic.salt_model(nz, nx, seed=11, nlayers=12)
    pads = synthetic.padded(m, cfg["ealThick"])
    w = synthetic.ricker(nt, cfg["dt"], cfg["fpeak"])
    snaps = {}
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*pads)
        # sources straddling a band boundary (padded row 128) and the surface
        h.set_source([40, 200], [128 - h.E - 1, 2], np.stack([w, 0.5 * w]))
        gx = np.arange(0, nx, 3)
        for k in (0, 1, 2):
            h.set_receivers(k, gx, (gx * 7) % nz)
        h.run(lambda it, kind, a: snaps.__setitem__((it, kind), a))
        out = {f"tr{k}": h.fetch_traces(k) for k in (0, 1, 2)}
        for f in range(8 if variant == "tensor_rotation" else 5):
            out[f"f{f}"] = h.fetch_field(f)
    out.update({f"s{k}": v for k, v in snaps.items()})
    return out


@pytest.mark.parametrize("path", ["tiled"])
@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
@pytest.mark.parametrize("fs,stype", [(0, 1), (1, 1), (1, 4), (0, 8)])
def test_tiled_equals_per_cell_path(path, variant, fs, stype, monkeypatch, gpu_lib):
    ref = _run("naive", monkeypatch, variant, fs, stype)
    got = _run(path, monkeypatch, variant, fs, stype)
    assert ref.keys() == got.keys()
    for k in ref:
        a, b = np.asarray(got[k]), np.asarray(ref[k])
        assert np.array_equal(a.view(np.uint32), b.view(np.uint32)), (
            f"{variant} fs={fs} stype={stype} {k}: max |diff| {np.max(np.abs(a - b))}")

