"""ctypes binding of the C ABI in include/ttifd.h (libttifd.so).

The product path is C host code calling the CUDA library through the C ABI;
this module exposes the same calls to Python for the tests and the benchmark.
It never computes anything itself: when the shared library is missing the
import of :func:`load` raises, there is no fallback.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "lib", "libttifd.so")

# status codes
OK, ERR_ARG, ERR_UNSTABLE, ERR_RANGE, ERR_CUDA, ERR_NOMEM, ERR_NONFINITE, ERR_STATE, ERR_CALLBACK = range(9)
COORDINATE, TENSOR, BOND = 0, 1, 2
VARIANTS = {"coordinate_rotation": COORDINATE, "tensor_rotation": TENSOR, "bond_transformation": BOND}
REC_VX, REC_VZ, REC_P = 0, 1, 2
F_VX, F_VZ, F_SXX, F_SZZ, F_SXZ, F_TXX, F_TZZ, F_TXZ = range(8)
PARAMS = ["D", "Beta", "coef1", "coef2", "invrho", "c11", "c13", "c15", "c33", "c35", "c55", "sin", "cos",
          "sin_v", "cos_v", "sin2", "cos2", "sin_2theta", "vp", "vs", "rho"]
P = {name: i for i, name in enumerate(PARAMS)}


_COPY_POOL = None


def _copy(src: np.ndarray) -> np.ndarray:
    """A new array with the contents of `src`. Large arrays are copied in row
    blocks from a few threads (numpy releases the GIL while it copies), so the
    page faults of the fresh destination are taken in parallel: a 35 MB
    snapshot copies in about a third of the single-threaded time."""
    global _COPY_POOL
    out = np.empty_like(src)
    nth = min(8, os.cpu_count() or 1, src.shape[0])
    if src.nbytes < (8 << 20) or nth < 2:
        np.copyto(out, src)
        return out
    if _COPY_POOL is None:
        from concurrent.futures import ThreadPoolExecutor
        _COPY_POOL = ThreadPoolExecutor(max_workers=8, thread_name_prefix="ttifd-copy")
    step = -(-src.shape[0] // nth)
    blocks = [slice(b, min(b + step, src.shape[0])) for b in range(0, src.shape[0], step)]
    for f in [_COPY_POOL.submit(np.copyto, out[b], src[b]) for b in blocks]:
        f.result()
    return out


class TTIError(RuntimeError):
    def __init__(self, code: int, msg: str):
        super().__init__(f"[{code}] {msg}")
        self.code = code


class Config(C.Structure):
    """tti_config: the getpar keys of the reference drivers."""

    _fields_ = [("variant", C.c_int), ("nz", C.c_int), ("nx", C.c_int), ("nt", C.c_int), ("dx", C.c_float),
                ("dz", C.c_float), ("dt", C.c_float), ("ealThick", C.c_int), ("eal_alpha", C.c_float),
                ("freesurface", C.c_int), ("fpeak", C.c_float), ("scalar", C.c_float), ("stype", C.c_int),
                ("seistype", C.c_int), ("mt", C.c_int), ("wsave", C.c_int), ("savew", C.c_int),
                ("snap_sample", C.c_int), ("mode", C.c_int), ("energy", C.c_int)]

    DEFAULTS = dict(variant=0, ealThick=30, eal_alpha=-1.0, freesurface=0, scalar=1.0, stype=1, seistype=0, mt=1,
                    wsave=0, savew=0, snap_sample=1, mode=1, energy=0)

    @classmethod
    def make(cls, **kw) -> "Config":
        d = dict(cls.DEFAULTS)
        d.update(kw)
        if isinstance(d["variant"], str):
            d["variant"] = VARIANTS[d["variant"]]
        return cls(**{k: d[k] for k, _ in cls._fields_})


SNAP_FN = C.CFUNCTYPE(C.c_int, C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_float), C.c_int, C.c_int)

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_SIGNATURES = {
    "create": (C.c_int, [C.POINTER(C.c_void_p), C.POINTER(Config), C.c_int]),
    "destroy": (C.c_int, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "grid": (C.c_int, [C.c_void_p, _IP, _IP, _IP]),
    "upload_model": (C.c_int, [C.c_void_p] + [_FP] * 6),
    "upload_model_physical": (C.c_int, [C.c_void_p] + [_FP] * 6),
    "fetch_param": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "set_source": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP, _FP]),
    "set_receivers": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _IP, _IP]),
    "run": (C.c_int, [C.c_void_p, SNAP_FN, C.c_void_p]),
    "reset": (C.c_int, [C.c_void_p]),
    "step": (C.c_int, [C.c_void_p, C.c_int]),
    "elapsed_ms": (C.c_int, [C.c_void_p, _FP]),
    "fetch_traces": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "fetch_field": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "fetch_energy": (C.c_int, [C.c_void_p, _FP, _FP]),
    "profile_steps": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "kernel_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "snapshot_static": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "get_stream": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p)]),
    "host_alloc": (C.c_int, [C.c_size_t, C.POINTER(C.c_void_p)]),
    "host_free": (C.c_int, [C.c_void_p]),
    "set_snapshot_buffer": (C.c_int, [C.c_void_p, _FP, C.c_size_t]),
    "grad_set_observed": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "grad_zero": (C.c_int, [C.c_void_p]),
    "grad_run": (C.c_int, [C.c_void_p, C.c_int, C.POINTER(C.c_double)]),
    "grad_run_binomial": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
    "grad_schedule_cost": (C.c_longlong, [C.c_int, C.c_int]),
    "grad_plan": (C.c_int, [C.c_void_p, C.c_double, _IP, _IP, C.POINTER(C.c_longlong)]),
    "grad_fetch": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "grad_fetch_source": (C.c_int, [C.c_void_p, _FP]),
    "grad_accumulators": (C.c_int, [C.c_void_p, C.POINTER(C.c_void_p), C.POINTER(C.c_size_t),
                                    C.POINTER(C.c_size_t)]),
}
GRADS = {"vp": 0, "eps": 1, "delta": 2, "theta": 3}

_BATCH_SIGNATURES = {
    "batch_create": (C.c_int, [C.POINTER(C.c_void_p), C.c_int, C.POINTER(Config), C.c_int, _IP, C.c_int]),
    "batch_destroy": (C.c_int, [C.c_void_p]),
    "batch_last_error": (C.c_char_p, [C.c_void_p]),
    "batch_instance": (C.c_void_p, [C.c_void_p, C.c_int]),
    "batch_upload_model": (C.c_int, [C.c_void_p, C.c_int] + [_FP] * 6),
    "batch_set_order": (C.c_int, [C.c_void_p, C.c_int, C.c_int]),
    "batch_set_schedule": (C.c_int, [C.c_void_p, C.c_int]),
    "batch_get_schedule": (C.c_int, [C.c_void_p, _IP, _IP, _IP]),
    "batch_autotune": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP, _FP]),
    "batch_reset": (C.c_int, [C.c_void_p]),
    "batch_step": (C.c_int, [C.c_void_p, C.c_int]),
    "batch_run": (C.c_int, [C.c_void_p]),
    "batch_elapsed_ms": (C.c_int, [C.c_void_p, _FP]),
    "batch_kernel_launches": (C.c_int, [C.c_void_p, C.POINTER(C.c_longlong)]),
    "batch_grad_run": (C.c_int, [C.c_void_p, C.c_int, C.c_int, C.POINTER(C.c_double)]),
}
_SIGNATURES.update(_BATCH_SIGNATURES)
EXPORTS = ["tti_" + k for k in _SIGNATURES]

_lib = None


def load(path: str | None = None) -> C.CDLL:
    """Loads libttifd.so (raises OSError when it has not been built)."""
    global _lib
    if _lib is not None and path is None:
        return _lib
    lib = C.CDLL(path or LIB_PATH)
    for name, (res, args) in _SIGNATURES.items():
        fn = getattr(lib, "tti_" + name)
        fn.restype, fn.argtypes = res, args
    if path is None:
        _lib = lib
    return lib


def schedule_cost(macro_steps: int, snapshots: int) -> int:
    """Macro-steps advanced by the binomial schedule (tti_grad_schedule_cost; host only)."""
    return int(load().tti_grad_schedule_cost(macro_steps, snapshots))


def host_empty(shape, dtype=np.float32) -> np.ndarray:
    """An uninitialised array in page-locked host memory (tti_host_alloc),
    released when the array and its views are gone. Uploads from such arrays,
    trace fetches into them and snapshots delivered into them
    (Modeling.set_snapshot_buffer) skip the library's staging copies.
    Page-locking costs about 0.4 ms per MB: allocate once, reuse."""
    import weakref

    lib = load()
    dt = np.dtype(dtype)
    n = int(np.prod(shape, dtype=np.int64)) * dt.itemsize
    p = C.c_void_p()
    rc = lib.tti_host_alloc(max(n, 1), C.byref(p))
    if rc != OK:
        raise TTIError(rc, f"tti_host_alloc of {n} bytes failed")
    raw = (C.c_char * max(n, 1)).from_address(p.value)
    weakref.finalize(raw, lib.tti_host_free, C.c_void_p(p.value))
    return np.frombuffer(raw, dtype=dt, count=n // dt.itemsize).reshape(shape)


def _f(a: np.ndarray):
    return a.ctypes.data_as(_FP)


def _i(a: np.ndarray):
    return a.ctypes.data_as(_IP)


class Modeling:
    """One shot on one GPU: the object behind a tti_handle."""

    prefix = "tti_"

    def __init__(self, device: int = 0, lib: C.CDLL | None = None, **cfg):
        self.lib = lib or load()
        self.cfg = Config.make(**cfg)
        self.device = device
        self._h = C.c_void_p()
        self._call("create", C.byref(self._h), C.byref(self.cfg), device, handle=False)
        nz, nx, e = C.c_int(), C.c_int(), C.c_int()
        self._call("grid", self._h, C.byref(nz), C.byref(nx), C.byref(e))
        self.Nz, self.Nx, self.E = nz.value, nx.value, e.value
        self.nts = (self.cfg.nt - 1) // self.cfg.mt + 1
        self._nrec = {}
        self._snapbuf = None

    # -- plumbing
    def _fn(self, name):
        return getattr(self.lib, self.prefix + name)

    def _call(self, name, *args, handle=True):
        rc = self._fn(name)(*args)
        if rc != OK:
            msg = self._fn("last_error")(self._h if handle else None)
            raise TTIError(rc, (msg or b"").decode(errors="replace"))
        return rc

    def close(self):
        if self._h:
            self._fn("destroy")(self._h)
            self._h = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    # -- API
    def upload_model(self, vp, vs, rho, epsilon, delta, theta):
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho, epsilon, delta, theta)]
        for a in arrs:
            if a.shape != (self.Nx, self.Nz):
                raise ValueError(f"model arrays must be padded (Nx, Nz) = {(self.Nx, self.Nz)}, got {a.shape}")
        self._call("upload_model", self._h, *[_f(a) for a in arrs])

    def upload_model_physical(self, vp, vs, rho, epsilon, delta, theta):
        """The unpadded model, (nx, nz) arrays; the rims are filled on the
        device as padModel2d fills them (tti_upload_model_physical)."""
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho, epsilon, delta, theta)]
        want = (self.cfg.nx, self.cfg.nz)
        for a in arrs:
            if a.shape != want:
                raise ValueError(f"model arrays must be physical (nx, nz) = {want}, got {a.shape}")
        self._call("upload_model_physical", self._h, *[_f(a) for a in arrs])

    def fetch_param(self, name) -> np.ndarray:
        out = np.empty((self.Nx, self.Nz), np.float32)
        self._call("fetch_param", self._h, P[name] if isinstance(name, str) else name, _f(out))
        return out

    def set_source(self, posx, posz, wavelets):
        w = np.ascontiguousarray(np.atleast_2d(wavelets), dtype=np.float32)
        x = np.ascontiguousarray(np.atleast_1d(posx), dtype=np.int32)
        z = np.ascontiguousarray(np.atleast_1d(posz), dtype=np.int32)
        if w.shape != (x.size, self.cfg.nt):
            raise ValueError("wavelets must be [ntrace][nt]")
        self._call("set_source", self._h, x.size, _i(x), _i(z), _f(w))

    def set_receivers(self, kind, posx, posz):
        x = np.ascontiguousarray(posx, dtype=np.int32)
        z = np.ascontiguousarray(np.broadcast_to(posz, x.shape), dtype=np.int32)
        self._call("set_receivers", self._h, kind, x.size, _i(x), _i(z))
        self._nrec[kind] = x.size

    def run(self, snapshot=None, copy=True):
        """snapshot(it, kind, array[nx_out, nz_out]) -> None, or None. With
        copy=False the array is a view of the library's host buffer, valid only
        during the call (as for a C callback: write it out or copy it there)."""
        if snapshot is None:
            cb = SNAP_FN()
        else:
            def _cb(user, it, kind, data, nzo, nxo):
                try:
                    view = np.ctypeslib.as_array(data, shape=(nxo, nzo))
                    arr = _copy(view) if copy else view
                    snapshot(it, kind, arr)
                    return 0
                except Exception:  # abort the run
                    return 1
            cb = SNAP_FN(_cb)
        self._call("run", self._h, cb, None)

    def set_snapshot_buffer(self, buf):
        """Host buffer (float32, C-contiguous; None: the library's own) into
        which run() delivers snapshots (tti_set_snapshot_buffer). From
        host_empty, the copies overlap the time steps and each snapshot's
        callback runs at the next snapshot step or at the end of the run."""
        if buf is None:
            self._call("set_snapshot_buffer", self._h, None, 0)
            self._snapbuf = None
            return
        if buf.dtype != np.float32 or not buf.flags.c_contiguous:
            raise ValueError("snapshot buffer must be a C-contiguous float32 array")
        self._call("set_snapshot_buffer", self._h, _f(buf), buf.size)
        self._snapbuf = buf  # kept alive while the library holds its address

    def reset(self):
        self._call("reset", self._h)

    def step(self, n=1):
        self._call("step", self._h, n)

    @property
    def elapsed_ms(self) -> float:
        v = C.c_float()
        self._call("elapsed_ms", self._h, C.byref(v))
        return v.value

    def profile_steps(self, n):
        """Advances n steps; returns total device ms (velocity, stress, other)."""
        ms = np.zeros(3, np.float32)
        self._call("profile_steps", self._h, n, _f(ms))
        return tuple(float(x) for x in ms)

    @property
    def kernel_launches(self) -> int:
        v = C.c_longlong()
        self._call("kernel_launches", self._h, C.byref(v))
        return v.value

    def snapshot_static(self, kind) -> np.ndarray:
        """Snapshot through tti_snapshot_static (no device allocation)."""
        if self.cfg.savew == 0:
            shape = (self.Nx - 2 * self.E, self.Nz - 2 * self.E)
        else:
            shape = (self.Nx, self.Nz)
        out = np.empty(shape, np.float32)
        self._call("snapshot_static", self._h, kind, _f(out))
        return out

    @property
    def stream(self) -> int:
        """The handle's CUDA stream (cudaStream_t) as an integer."""
        s = C.c_void_p()
        self._call("get_stream", self._h, C.byref(s))
        return s.value or 0

    def fetch_traces(self, kind, out=None) -> np.ndarray:
        """[ntrace][nts] traces of one component; into `out` when given (a
        C-contiguous float32 array of that shape, e.g. from host_empty)."""
        shape = (self._nrec.get(kind, 0), self.nts)
        if out is None:
            out = np.empty(shape, np.float32)
        elif out.shape != shape or out.dtype != np.float32 or not out.flags.c_contiguous:
            raise ValueError(f"out must be a C-contiguous float32 array of shape {shape}")
        self._call("fetch_traces", self._h, kind, _f(out))
        return out

    def fetch_field(self, which) -> np.ndarray:
        out = np.empty((self.Nx, self.Nz), np.float32)
        self._call("fetch_field", self._h, which, _f(out))
        return out

    # -- adjoint-state gradient (three formulations, every source type)
    def grad_set_observed(self, kind, dobs):
        d = np.ascontiguousarray(dobs, dtype=np.float32)
        if d.shape != (self._nrec.get(kind, 0), self.nts):
            raise ValueError(f"observed traces must be [ntrace][nts] = {(self._nrec.get(kind, 0), self.nts)}")
        self._call("grad_set_observed", self._h, kind, _f(d))

    def grad_zero(self):
        self._call("grad_zero", self._h)

    def grad_run(self, ncheck: int) -> float:
        """Adds this shot's gradient to the sums; returns its misfit J."""
        J = C.c_double()
        self._call("grad_run", self._h, ncheck, C.byref(J))
        return J.value

    def grad_run_binomial(self, snapshots: int, keep_steps: int) -> float:
        """Binomial (Revolve) checkpointing: `snapshots` state slots, macro-steps of `keep_steps` steps."""
        J = C.c_double()
        self._call("grad_run_binomial", self._h, snapshots, keep_steps, C.byref(J))
        return J.value

    def grad_plan(self, budget_bytes: float) -> dict:
        """Binomial schedule that fits `budget_bytes` of checkpoints and kept steps (tti_grad_plan)."""
        s, k, f = C.c_int(), C.c_int(), C.c_longlong()
        self._call("grad_plan", self._h, float(budget_bytes), C.byref(s), C.byref(k), C.byref(f))
        return {"snapshots": s.value, "keep_steps": k.value, "forward_steps": f.value}

    def grad_fetch(self, name) -> np.ndarray:
        out = np.empty((self.Nx, self.Nz), np.float32)
        self._call("grad_fetch", self._h, GRADS[name] if isinstance(name, str) else name, _f(out))
        return out

    def grad_fetch_source(self, nsrc: int) -> np.ndarray:
        out = np.empty((nsrc, self.cfg.nt), np.float32)
        self._call("grad_fetch_source", self._h, _f(out))
        return out

    def grad_accumulators(self):
        """(7 device pointers, floats per array, pitch): the sums a multi-GPU run all-reduces."""
        ptrs = (C.c_void_p * 7)()
        n, pitch = C.c_size_t(), C.c_size_t()
        self._call("grad_accumulators", self._h, ptrs, C.byref(n), C.byref(pitch))
        return [p for p in ptrs], n.value, pitch.value

    def fetch_energy(self):
        ek = np.empty(self.cfg.nt, np.float32)
        ep = np.empty(self.cfg.nt, np.float32)
        self._call("fetch_energy", self._h, _f(ek), _f(ep))
        return ek, ep


class Instance(Modeling):
    """A shot of a batch: the batch's own handle, wrapped without ownership
    (set_source, set_receivers and fetch_traces act on it as on a single shot)."""

    def __init__(self, batch: "Batch", index: int, cfg: Config):
        self.lib = batch.lib
        self.cfg = cfg
        self.device = batch.device
        self._batch = batch  # keeps the batch (and the handle) alive
        self._h = C.c_void_p(self.lib.tti_batch_instance(batch._b, index))
        if not self._h:
            raise TTIError(ERR_ARG, f"no instance {index}")
        nz, nx, e = C.c_int(), C.c_int(), C.c_int()
        self._call("grid", self._h, C.byref(nz), C.byref(nx), C.byref(e))
        self.Nz, self.Nx, self.E = nz.value, nx.value, e.value
        self.nts = (self.cfg.nt - 1) // self.cfg.mt + 1
        self._nrec = {}

    def close(self):
        self._h = C.c_void_p()


class Batch:
    """Many instances (shots of one or more models) advanced together
    (tti_batch_*). `models` is a list of config dicts; `model_of[i]` is the
    model of instance i."""

    def __init__(self, models, model_of, device: int = 0, lib: C.CDLL | None = None):
        self.lib = lib or load()
        self.device = device
        self.cfgs = [Config.make(**m) for m in models]
        arr = (Config * len(self.cfgs))(*self.cfgs)
        mo = np.ascontiguousarray(model_of, dtype=np.int32)
        self._b = C.c_void_p()
        self._call("batch_create", C.byref(self._b), len(self.cfgs), arr, mo.size, _i(mo), device, handle=False)
        self.model_of = [int(m) for m in mo]
        self.instances = [Instance(self, i, self.cfgs[m]) for i, m in enumerate(self.model_of)]

    def _call(self, name, *args, handle=True):
        rc = getattr(self.lib, "tti_" + name)(*args)
        if rc != OK:
            msg = self.lib.tti_batch_last_error(self._b if handle else None)
            raise TTIError(rc, (msg or b"").decode(errors="replace"))
        return rc

    def close(self):
        if self._b:
            for inst in getattr(self, "instances", []):
                inst.close()
            self.lib.tti_batch_destroy(self._b)
            self._b = C.c_void_p()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def upload_model(self, m, vp, vs, rho, epsilon, delta, theta):
        inst = self.instances[self.model_of.index(m)]
        arrs = [np.ascontiguousarray(a, dtype=np.float32) for a in (vp, vs, rho, epsilon, delta, theta)]
        for a in arrs:
            if a.shape != (inst.Nx, inst.Nz):
                raise ValueError(f"model arrays must be padded (Nx, Nz) = {(inst.Nx, inst.Nz)}, got {a.shape}")
        self._call("batch_upload_model", self._b, m, *[_f(a) for a in arrs])

    def set_order(self, group: int, graph_steps: int):
        """Shots interleaved per tile in groups of `group` (0: all); graph of `graph_steps` steps (0: none)."""
        self._call("batch_set_order", self._b, group, graph_steps)

    GRIDS = ["per-tile", "persistent"]

    def set_schedule(self, grid):
        """Grid of the half-step launches: "per-tile" (0) or "persistent" (1)."""
        self._call("batch_set_schedule", self._b, self.GRIDS.index(grid) if isinstance(grid, str) else grid)

    def schedule(self) -> dict:
        g, gs, p = C.c_int(), C.c_int(), C.c_int()
        self._call("batch_get_schedule", self._b, C.byref(g), C.byref(gs), C.byref(p))
        return {"group": g.value, "graph_steps": gs.value, "grid": self.GRIDS[p.value]}

    def autotune(self, nsteps: int) -> dict:
        """Times the schedules on nsteps steps, keeps the fastest, resets the batch."""
        g, gs, ms = C.c_int(), C.c_int(), C.c_float()
        self._call("batch_autotune", self._b, nsteps, C.byref(g), C.byref(gs), C.byref(ms))
        return dict(self.schedule(), ms_per_step=ms.value)

    def reset(self):
        self._call("batch_reset", self._b)

    def step(self, n: int):
        self._call("batch_step", self._b, n)

    def run(self):
        self._call("batch_run", self._b)

    def grad_run(self, snapshots: int, keep_steps: int) -> list:
        """All instances' gradients at once (tti_batch_grad_run); returns each instance's J."""
        J = (C.c_double * len(self.instances))()
        self._call("batch_grad_run", self._b, snapshots, keep_steps, J)
        return list(J)

    @property
    def elapsed_ms(self) -> float:
        v = C.c_float()
        self._call("batch_elapsed_ms", self._b, C.byref(v))
        return v.value

    @property
    def kernel_launches(self) -> int:
        v = C.c_longlong()
        self._call("batch_kernel_launches", self._b, C.byref(v))
        return v.value
