"""Batched execution (tti_batch_*) against one-shot-at-a-time runs of the same
instances. The batched launches run the same per-tile code as the single-shot
tiled kernels, so in the exact rounding mode every trace must be bit-identical,
whatever the work order, the graph length, and the mix of models of different
sizes, step counts, free-surface settings and source types."""
import numpy as np
import pytest

import synthetic

pytestmark = pytest.mark.gpu

DT, FPEAK = 0.0008, 20.0


def _model_cfg(nz, nx, nt, fs, stype, variant="coordinate_rotation", ealThick=12, mode=1, seistype=3):
    return dict(variant=variant, nz=nz, nx=nx, nt=nt, dx=10.0, dz=10.0, dt=DT, fpeak=FPEAK, ealThick=ealThick,
                freesurface=fs, stype=stype, seistype=seistype, mt=2, mode=mode)


def _geometry(cfg, k):
    """Source and receivers of shot k on model cfg."""
    nz, nx, nt = cfg["nz"], cfg["nx"], cfg["nt"]
    w = synthetic.ricker(nt, DT, FPEAK)
    sx = [int((k * 37 + 11) % nx)]
    sz = [2 + (k % 3)]
    gx = np.arange(0, nx, 2)
    gz = (gx * 3 + k) % nz
    return sx, sz, w[None, :], gx, gz


def _single(cfg, model, k):
    import ttifd

    sx, sz, w, gx, gz = _geometry(cfg, k)
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*model)
        h.set_source(sx, sz, w)
        for c in (0, 1, 2):
            h.set_receivers(c, gx, gz)
        h.run()
        return [h.fetch_traces(c) for c in (0, 1, 2)]


def _batch(cfgs, models, model_of, group=0, graph_steps=20, grid="per-tile"):
    import ttifd

    out = []
    with ttifd.Batch(cfgs, model_of) as b:
        for m, model in enumerate(models):
            b.upload_model(m, *model)
        b.set_order(group, graph_steps)
        b.set_schedule(grid)
        for i, m in enumerate(model_of):
            sx, sz, w, gx, gz = _geometry(cfgs[m], i)
            inst = b.instances[i]
            inst.set_source(sx, sz, w)
            for c in (0, 1, 2):
                inst.set_receivers(c, gx, gz)
        b.run()
        for i in range(len(model_of)):
            out.append([b.instances[i].fetch_traces(c) for c in (0, 1, 2)])
        launches = b.kernel_launches
    return out, launches


def _models(cfgs):
    out = []
    for j, c in enumerate(cfgs):
        m = synthetic.salt_model(c["nz"], c["nx"], seed=20 + j, nlayers=8)
        out.append(synthetic.padded(m, c["ealThick"]))
    return out


@pytest.mark.parametrize("variant", ["coordinate_rotation", "tensor_rotation", "bond_transformation"])
def test_batch_equals_single_shots(variant, monkeypatch, gpu_lib):
    monkeypatch.setenv("TTIFD_EXACT", "1")
    monkeypatch.delenv("TTIFD_KERNEL", raising=False)
    cfgs = [_model_cfg(150, 260, 120, 1, 1, variant), _model_cfg(90, 140, 90, 0, 4, variant, ealThick=8)]
    models = _models(cfgs)
    model_of = [0, 1, 0, 0]
    got, launches = _batch(cfgs, models, model_of, graph_steps=16)
    assert launches >= 120 * 4
    for i, m in enumerate(model_of):
        ref = _single(cfgs[m], models[m], i)
        for c in range(3):
            assert np.array_equal(got[i][c].view(np.uint32), ref[c].view(np.uint32)), (
                f"{variant} instance {i} component {c}: max |diff| {np.max(np.abs(got[i][c] - ref[c]))}")


@pytest.mark.parametrize("group,graph_steps", [(1, 0), (0, 7), (2, 120)])
def test_batch_schedules_agree(group, graph_steps, monkeypatch, gpu_lib):
    monkeypatch.delenv("TTIFD_EXACT", raising=False)
    cfgs = [_model_cfg(130, 200, 100, 1, 1), _model_cfg(100, 160, 70, 1, 8, mode=2)]
    models = _models(cfgs)
    model_of = [0, 0, 1, 0, 1]
    ref, _ = _batch(cfgs, models, model_of, group=0, graph_steps=20)
    got, _ = _batch(cfgs, models, model_of, group=group, graph_steps=graph_steps)
    for i in range(len(model_of)):
        for c in range(3):
            assert np.array_equal(got[i][c].view(np.uint32), ref[i][c].view(np.uint32))


@pytest.mark.parametrize("graph_steps", [0, 20])
def test_batch_persistent_grid_agrees(graph_steps, monkeypatch, gpu_lib):
    """The persistent grid (one wave of CTAs walking the work table) gives the
    per-tile grid's traces bit for bit, with uneven models and mode 2."""
    monkeypatch.delenv("TTIFD_EXACT", raising=False)
    cfgs = [_model_cfg(130, 200, 100, 1, 1), _model_cfg(100, 160, 70, 1, 8, mode=2)]
    models = _models(cfgs)
    model_of = [0, 0, 1, 0, 1]
    ref, _ = _batch(cfgs, models, model_of, group=0, graph_steps=graph_steps)
    got, _ = _batch(cfgs, models, model_of, group=0, graph_steps=graph_steps, grid="persistent")
    for i in range(len(model_of)):
        for c in range(3):
            assert np.array_equal(got[i][c].view(np.uint32), ref[i][c].view(np.uint32)), (graph_steps, i, c)


def test_batch_fma_mode_matches_single_shot(monkeypatch, gpu_lib):
    monkeypatch.setenv("TTIFD_EXACT", "0")  # the FMA opt-in
    monkeypatch.delenv("TTIFD_KERNEL", raising=False)
    cfgs = [_model_cfg(140, 220, 150, 1, 1)]
    models = _models(cfgs)
    got, _ = _batch(cfgs, models, [0, 0, 0])
    for i in range(3):
        ref = _single(cfgs[0], models[0], i)
        for c in range(3):
            err = np.linalg.norm(got[i][c] - ref[c]) / max(np.linalg.norm(ref[c]), 1e-30)
            assert err <= 1e-6, (i, c, err)


def test_batch_autotune_keeps_results(monkeypatch, gpu_lib):
    """The autotuner only changes the schedule: a run after it gives the same traces."""
    import ttifd

    monkeypatch.delenv("TTIFD_EXACT", raising=False)
    cfgs = [_model_cfg(120, 180, 60, 1, 1)]
    models = _models(cfgs)
    ref, _ = _batch(cfgs, models, [0, 0, 0])
    with ttifd.Batch(cfgs, [0, 0, 0]) as b:
        b.upload_model(0, *models[0])
        for i in range(3):
            sx, sz, w, gx, gz = _geometry(cfgs[0], i)
            b.instances[i].set_source(sx, sz, w)
            for c in (0, 1, 2):
                b.instances[i].set_receivers(c, gx, gz)
        choice = b.autotune(12)
        assert choice["group"] in (0, 1, 2) and choice["graph_steps"] in (0, 20) and choice["ms_per_step"] > 0
        b.run()
        for i in range(3):
            for c in range(3):
                assert np.array_equal(b.instances[i].fetch_traces(c).view(np.uint32), ref[i][c].view(np.uint32))


@pytest.mark.parametrize("variant", ["coordinate_rotation", "bond_transformation"])
def test_batch_gradient_equals_sum_of_single_shots(variant, monkeypatch, gpu_lib):
    """tti_batch_grad_run (the shots' gradients at once, one stream each) against
    the same shots run one after another on one handle, whose sums accumulate."""
    import ttifd

    monkeypatch.delenv("TTIFD_EXACT", raising=False)
    cfg = _model_cfg(120, 160, 140, 1, 1, variant)
    cfg = dict(cfg, seistype=1)
    models = _models([cfg])
    shots = [(30, 2), (80, 2), (130, 3)]
    gx = np.arange(0, cfg["nx"], 2, dtype=np.int32)
    w = synthetic.ricker(cfg["nt"], cfg["dt"], cfg["fpeak"])[None, :]
    dobs = np.zeros((gx.size, (cfg["nt"] - 1) // cfg["mt"] + 1), np.float32)
    with ttifd.Batch([cfg], [0] * len(shots)) as b:
        b.upload_model(0, *models[0])
        for i, (sx, sz) in enumerate(shots):
            inst = b.instances[i]
            inst.set_source([sx], [sz], w)
            for k in (0, 1):
                inst.set_receivers(k, gx, 4)
                inst.grad_set_observed(k, dobs)
        Jb = b.grad_run(4, 10)
        got = {n: b.instances[0].grad_fetch(n) for n in ("vp", "eps", "delta", "theta")}
    with ttifd.Modeling(**cfg) as h:
        h.upload_model(*models[0])
        h.grad_zero()
        Js = []
        for sx, sz in shots:
            h.set_source([sx], [sz], w)
            for k in (0, 1):
                h.set_receivers(k, gx, 4)
                h.grad_set_observed(k, dobs)
            Js.append(h.grad_run_binomial(4, 10))
        ref = {n: h.grad_fetch(n) for n in got}
    assert Jb == pytest.approx(Js, rel=1e-12)
    for n in got:
        err = np.linalg.norm(got[n].astype(np.float64) - ref[n]) / np.linalg.norm(ref[n].astype(np.float64))
        assert err <= 1e-6, (n, err)
