"""Shot sharding across ranks, world_size 2 over gloo on CPU: every shot is
computed exactly once, per-rank results gathered on rank 0 equal a
single-process run, and the max-over-ranks timing reduction is right. The
per-shot computation here is the oracle (CPU); on GPUs each rank runs the
CUDA library the same way."""
import os
import pickle
import socket
import subprocess
import sys

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
sys.path.insert(0, os.path.join(ROOT, "tti-fdmodeling_b200"))
import shots  # noqa: E402

WORKER = r'''
import os, sys, pickle
sys.path.insert(0, os.path.join(sys.argv[1], "tti-fdmodeling_b200"))
sys.path.insert(0, os.path.join(sys.argv[1], "oracle"))
import numpy as np
import shots, synthetic, pyoracle
g = shots.Group(backend="gloo", timeout_s=60)
cfg = dict(variant="bond_transformation", nz=40, nx=60, nt=120, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0,
           ealThick=8, freesurface=1, seistype=2)
m = synthetic.salt_model(40, 60, seed=2, nlayers=6)
pads = synthetic.padded(m, 8)
w = synthetic.ricker(120, 0.0008, 20.0)
mine = {}
for s in shots.assign(5, g.rank, g.world):
    with pyoracle.Oracle(**cfg) as h:
        h.upload_model(*pads)
        h.set_source([8 + 10 * s], [2], w[None, :])
        h.set_receivers(2, np.arange(60), 1)
        h.run()
        mine[s] = h.fetch_traces(2)
t_max = g.max(1.0 + g.rank)
t_sum = g.sum(1.0 + g.rank)
allres = g.gather(mine)
if g.rank == 0:
    merged = {}
    for d in allres:
        for k, v in d.items():
            assert k not in merged
            merged[k] = v
    pickle.dump(dict(traces=merged, t_max=t_max, t_sum=t_sum), open(sys.argv[2], "wb"))
g.close()
'''


def test_assign_covers_every_shot_once():
    for n in (0, 1, 5, 64, 65):
        for world in (1, 2, 3, 8):
            got = sorted(s for r in range(world) for s in shots.assign(n, r, world))
            assert got == list(range(n))
            sizes = [len(shots.assign(n, r, world)) for r in range(world)]
            assert max(sizes) - min(sizes) <= 1


def test_two_ranks_gloo(tmp_path, oracle_lib):
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    script = tmp_path / "worker.py"
    script.write_text(WORKER)
    out = tmp_path / "res.pkl"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", OMP_NUM_THREADS="2")
    procs = [subprocess.Popen([sys.executable, str(script), ROOT, str(out)],
                              env=dict(env, RANK=str(r), LOCAL_RANK=str(r)),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE) for r in range(2)]
    for p in procs:
        _, err = p.communicate(timeout=240)
        assert p.returncode == 0, err.decode()[-2000:]
    res = pickle.load(open(out, "rb"))
    assert res["t_max"] == 2.0 and res["t_sum"] == 3.0
    assert sorted(res["traces"]) == list(range(5))
    # single-process reference of the same shots
    import pyoracle
    import synthetic

    cfg = dict(variant="bond_transformation", nz=40, nx=60, nt=120, dx=10.0, dz=10.0, dt=0.0008, fpeak=20.0,
               ealThick=8, freesurface=1, seistype=2)
    m = synthetic.salt_model(40, 60, seed=2, nlayers=6)
    pads = synthetic.padded(m, 8)
    w = synthetic.ricker(120, 0.0008, 20.0)
    for s in range(5):
        with pyoracle.Oracle(**cfg) as h:
            h.upload_model(*pads)
            h.set_source([8 + 10 * s], [2], w[None, :])
            h.set_receivers(2, np.arange(60), 1)
            h.run()
            np.testing.assert_array_equal(res["traces"][s], h.fetch_traces(2))


GRAD_WORKER = r'''
import os, sys, pickle
sys.path.insert(0, os.path.join(sys.argv[1], "tti-fdmodeling_b200"))
sys.path.insert(0, os.path.join(sys.argv[1], "oracle"))
import numpy as np
import shots, synthetic, pyoracle


class HostSums:
    # host-memory stand-in for a handle's 7 device gradient sums (same interface)
    device = "cpu"

    def __init__(self, n):
        self.arrays = [np.zeros(n, np.float32) for _ in range(7)]

    def grad_accumulators(self):
        return [a.ctypes.data for a in self.arrays], self.arrays[0].size, 0


g = shots.Group(backend="gloo", timeout_s=60)
cfg = dict(nz=30, nx=40, nt=150, dx=10.0, dz=10.0, dt=0.001, fpeak=15.0, ealThick=6, seistype=1, mt=1)
m = synthetic.layered_model(30, 40, seed=7, nlayers=3)
pads = synthetic.padded(m, 6)
w = synthetic.ricker(150, 0.001, 15.0)
hs = HostSums(pads[0].size)
with pyoracle.AdjointOracle(cfg, pads) as adj:
    adj.set_model(*pads)
    for k in (0, 1):
        adj.set_receivers(k, np.arange(0, 40, 2), 2)
    for s in shots.assign(3, g.rank, g.world):
        adj.set_source([6 + 12 * s], [2], w[None, :])
        dobs = [np.zeros((20, 150)), np.zeros((20, 150)), None]
        J, grad, _ = adj.gradient(dobs)
        for i, name in enumerate(("vp", "eps", "delta", "theta")):
            hs.arrays[i] += grad[name].ravel().astype(np.float32)
        hs.arrays[4][s] += np.float32(J)
views = shots.gradient_sums(hs)
assert all(v.data_ptr() == a.ctypes.data for v, a in zip(views, hs.arrays))  # views, not copies
shots.reduce_gradient(g, hs)
if g.rank == 0:
    pickle.dump(np.stack(hs.arrays), open(sys.argv[2], "wb"))
g.close()
'''


def test_gradient_sum_over_two_ranks_gloo(tmp_path, oracle_lib):
    """Each rank adds the gradients of its shots into its handle's sums;
    shots.reduce_gradient (through shots.gradient_sums, the zero-copy views it
    all-reduces in place) gives every rank the sums of all shots. The sums here
    are a host-memory stand-in with the handle's grad_accumulators interface,
    filled with oracle gradients; on GPUs the same two functions act on the
    library's device arrays over NCCL."""
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    script = tmp_path / "gworker.py"
    script.write_text(GRAD_WORKER)
    out = tmp_path / "grad.pkl"
    env = dict(os.environ, MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port), WORLD_SIZE="2", OMP_NUM_THREADS="2")
    procs = [subprocess.Popen([sys.executable, str(script), ROOT, str(out)],
                              env=dict(env, RANK=str(r), LOCAL_RANK=str(r)),
                              stdout=subprocess.PIPE, stderr=subprocess.PIPE) for r in range(2)]
    for p in procs:
        _, err = p.communicate(timeout=240)
        assert p.returncode == 0, err.decode()[-2000:]
    got = pickle.load(open(out, "rb"))
    import pyoracle
    import synthetic

    cfg = dict(nz=30, nx=40, nt=150, dx=10.0, dz=10.0, dt=0.001, fpeak=15.0, ealThick=6, seistype=1, mt=1)
    m = synthetic.layered_model(30, 40, seed=7, nlayers=3)
    pads = synthetic.padded(m, 6)
    w = synthetic.ricker(150, 0.001, 15.0)
    ref = np.zeros((7, pads[0].size))
    with pyoracle.AdjointOracle(cfg, pads) as adj:
        adj.set_model(*pads)
        for k in (0, 1):
            adj.set_receivers(k, np.arange(0, 40, 2), 2)
        for s in range(3):
            adj.set_source([6 + 12 * s], [2], w[None, :])
            J, grad, _ = adj.gradient([np.zeros((20, 150)), np.zeros((20, 150)), None])
            for i, name in enumerate(("vp", "eps", "delta", "theta")):
                ref[i] += grad[name].ravel().astype(np.float32)
            ref[4][s] += np.float32(J)
    assert np.abs(got[:4]).max() > 0
    np.testing.assert_allclose(got, ref, rtol=1e-6, atol=1e-30 + 1e-6 * np.abs(ref).max())
