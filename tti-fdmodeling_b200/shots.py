"""Shot sharding across ranks (one process per GPU).

Shots are independent in forward modelling (no exchange during propagation),
so a multi-GPU run gives each rank its own shots and needs no collective on
the data path. The collectives here are host-side plumbing over
torch.distributed: a barrier, the max over ranks of a timing, the sum of a
per-rank quantity, and gathering per-shot results on rank 0. The one exchange
of real data is the gradient: each rank adds its shots' adjoint-state
gradients into the sums held by its handle, and reduce_gradient sums those
device arrays over ranks in place (NCCL over NVLink; no host copy).
"""
from __future__ import annotations

import datetime
import os


def assign(n_shots: int, rank: int, world: int) -> list[int]:
    """Contiguous block of shot indices for `rank` (sizes differ by at most one)."""
    if world < 1 or not 0 <= rank < world:
        raise ValueError("bad rank/world")
    base, extra = divmod(n_shots, world)
    start = rank * base + min(rank, extra)
    return list(range(start, start + base + (1 if rank < extra else 0)))


class Group:
    """torch.distributed process group (or a single process when WORLD_SIZE is 1)."""

    def __init__(self, backend: str | None = None, timeout_s: int = 300):
        self.world = int(os.environ.get("WORLD_SIZE", "1"))
        self.rank = int(os.environ.get("RANK", "0"))
        self.local_rank = int(os.environ.get("LOCAL_RANK", "0"))
        self.dist = None
        self.device = "cpu"
        if self.world > 1:
            import torch
            import torch.distributed as dist

            if backend is None:
                backend = "nccl" if torch.cuda.is_available() else "gloo"
            if backend == "nccl":
                torch.cuda.set_device(self.local_rank)
                self.device = f"cuda:{self.local_rank}"
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=timeout_s))
            self.dist = dist

    def barrier(self) -> None:
        if self.dist is not None:
            self.dist.barrier()

    def _reduce(self, x: float, op) -> float:
        import torch

        t = torch.tensor([float(x)], dtype=torch.float64, device=self.device)
        self.dist.all_reduce(t, op=op)
        return float(t.item())

    def max(self, x: float) -> float:
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.MAX)

    def sum(self, x: float) -> float:
        return x if self.dist is None else self._reduce(x, self.dist.ReduceOp.SUM)

    def allreduce_(self, tensors) -> None:
        """Sums torch tensors over ranks in place (GPU tensors over NCCL)."""
        if self.dist is None:
            return
        for t in tensors:
            self.dist.all_reduce(t, op=self.dist.ReduceOp.SUM)

    def gather(self, obj):
        """List of every rank's `obj` on rank 0 (None elsewhere)."""
        if self.dist is None:
            return [obj]
        out = [None] * self.world if self.rank == 0 else None
        self.dist.gather_object(obj, out, dst=0)
        return out

    def close(self) -> None:
        if self.dist is not None:
            self.dist.destroy_process_group()
            self.dist = None


class _DeviceArray:
    """A float32 device buffer of the library, exposed to torch without a copy."""

    def __init__(self, ptr: int, n: int):
        self.__cuda_array_interface__ = {"shape": (n,), "typestr": "<f4", "data": (int(ptr), False), "version": 3,
                                         "strides": None}


def gradient_sums(h):
    """The 7 gradient sums of handle `h` as torch views of its memory, without a
    copy: device arrays for a library handle (ttifd.Modeling), host arrays for
    a handle whose `device` is "cpu" (a host-memory stand-in with the same
    grad_accumulators() interface, as the CPU tests use)."""
    import torch

    ptrs, n, _ = h.grad_accumulators()
    if getattr(h, "device", 0) == "cpu":
        import ctypes

        import numpy as np

        fp = ctypes.POINTER(ctypes.c_float)
        return [torch.from_numpy(np.ctypeslib.as_array(ctypes.cast(p, fp), shape=(n,))) for p in ptrs]
    return [torch.as_tensor(_DeviceArray(p, n), device=f"cuda:{h.device}") for p in ptrs]


def reduce_gradient(group: Group, h) -> None:
    """Sums the gradient of every rank's shots in place; afterwards tti_grad_fetch
    on any rank returns the gradient of all shots (the chain rule is linear in the sums)."""
    if group.dist is None:
        return
    import torch

    on_gpu = getattr(h, "device", 0) != "cpu"
    if on_gpu:
        torch.cuda.synchronize(h.device)
    group.allreduce_(gradient_sums(h))
    if on_gpu:
        torch.cuda.synchronize(h.device)
