"""ctypes wrapper of the CPU restatement (oracle/ttifd_oracle.c).

TEST INFRASTRUCTURE ONLY: imported by tests/, __graft_entry__.smoke() and the
CPU-baseline leg of bench.py, as the checker. Same method names as the
product binding (ttifd.Modeling) so parity tests drive both identically.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
sys.path.insert(0, os.path.join(ROOT, "tti-fdmodeling_b200"))
import ttifd  # noqa: E402  (tti_config layout and constants)

LIB_PATH = os.path.join(HERE, "_build", "libttifd_oracle.so")
REF_DIR = os.path.join(HERE, "_ref")

_FP = C.POINTER(C.c_float)
_IP = C.POINTER(C.c_int)
_SIG = {
    "create": (C.c_void_p, [C.POINTER(ttifd.Config)]),
    "destroy": (None, [C.c_void_p]),
    "last_error": (C.c_char_p, [C.c_void_p]),
    "grid": (C.c_int, [C.c_void_p, _IP, _IP, _IP]),
    "upload_model": (C.c_int, [C.c_void_p] + [_FP] * 6),
    "fetch_param": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "set_source": (C.c_int, [C.c_void_p, C.c_int, _IP, _IP, _FP]),
    "set_receivers": (C.c_int, [C.c_void_p, C.c_int, C.c_int, _IP, _IP]),
    "reset": (C.c_int, [C.c_void_p]),
    "step": (C.c_int, [C.c_void_p, C.c_int]),
    "current_it": (C.c_int, [C.c_void_p]),
    "fetch_traces": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "fetch_field": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "fetch_energy": (C.c_int, [C.c_void_p, _FP, _FP]),
    "snapshot": (C.c_int, [C.c_void_p, C.c_int, _FP]),
    "pad_model": (None, [_FP, C.c_int, C.c_int, C.c_int]),
    "vp2vs": (None, [_FP, _FP, C.c_int]),
    "vp2rho_gardner": (None, [_FP, _FP, C.c_int]),
    "dt_max": (C.c_double, [_FP, C.c_int, C.c_int, C.c_float, C.c_float]),
    "ricker": (None, [_FP, C.c_float, C.c_float, C.c_float, C.c_float, C.c_int]),
}

_lib = None


def build() -> None:
    """Builds the restatement (and the reference build when the tree is present)."""
    subprocess.run(["make", "-s", "-C", HERE], check=True)


def load() -> C.CDLL:
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build()
        lib = C.CDLL(LIB_PATH)
        for k, (res, args) in _SIG.items():
            fn = getattr(lib, "orc_" + k)
            fn.restype, fn.argtypes = res, args
        _lib = lib
    return _lib


def _f(a):
    return a.ctypes.data_as(_FP)


def _i(a):
    return a.ctypes.data_as(_IP)


class Oracle(ttifd.Modeling):
    """CPU restatement with the ttifd.Modeling interface."""

    prefix = "orc_"

    def __init__(self, **cfg):  # noqa: D107 (no device)
        self.lib = load()
        self.cfg = ttifd.Config.make(**cfg)
        self._h = C.c_void_p(self.lib.orc_create(C.byref(self.cfg)))
        nz, nx, e = C.c_int(), C.c_int(), C.c_int()
        self.lib.orc_grid(self._h, C.byref(nz), C.byref(nx), C.byref(e))
        self.Nz, self.Nx, self.E = nz.value, nx.value, e.value
        self.nts = (self.cfg.nt - 1) // self.cfg.mt + 1
        self._nrec = {}

    def run(self, snapshot=None):
        """Whole loop with snapshots, as tti_run does."""
        self.reset()
        kinds = {1: (1, 2), 2: (3,), 3: (1, 2, 3), 4: (4, 5), 5: (6, 7)}.get(self.cfg.wsave, ())
        for _ in range(self.cfg.nt):
            it = self.lib.orc_current_it(self._h)
            self.step(1)
            if snapshot is not None and self.cfg.wsave > 0 and it % self.cfg.snap_sample == 0:
                for k in kinds:
                    snapshot(it, k, self.snapshot(k))

    def snapshot(self, kind) -> np.ndarray:
        if self.cfg.savew == 0:
            shape = (self.Nx - 2 * self.E, self.Nz - 2 * self.E)
        else:
            shape = (self.Nx, self.Nz)
        out = np.empty(shape, np.float32)
        self.lib.orc_snapshot(self._h, kind, _f(out))
        return out

    @property
    def elapsed_ms(self):
        return float("nan")

    def close(self):
        if self._h:
            self.lib.orc_destroy(self._h)
            self._h = C.c_void_p()


def dt_max(vp_padded: np.ndarray, dx: float, dz: float) -> float:
    a = np.ascontiguousarray(vp_padded, dtype=np.float32)
    return load().orc_dt_max(_f(a), a.shape[0], a.shape[1], dx, dz)


def ricker(nt, dt, fpeak, amp=1.0, delay=None) -> np.ndarray:
    out = np.empty(nt, np.float32)
    if delay is None:
        delay = np.float32(1.5) / np.float32(fpeak)
    load().orc_ricker(_f(out), amp, fpeak, delay, dt, nt)
    return out


def pad_model(a: np.ndarray, E: int) -> np.ndarray:
    """padModel2d restated: (nx, nz) physical -> (nx+2E, nz+2E)."""
    nx, nz = a.shape
    out = np.zeros((nx + 2 * E, nz + 2 * E), np.float32)
    out[E:E + nx, E:E + nz] = a
    load().orc_pad_model(_f(out), out.shape[0], out.shape[1], E)
    return out


def ref_binary(variant: str, strict: bool = True) -> str | None:
    """Path of the reference program built from the reference's sources, or None."""
    p = os.path.join(REF_DIR, "strict" if strict else "bin", f"sufdmod2dTTIelastic_{variant}")
    return p if os.path.exists(p) else None


# ---------------------------------------------------------------- adjoint (double precision)
_DP = C.POINTER(C.c_double)
_ADJ_SIG = {
    "adj_create": (C.c_void_p, [C.c_int, C.c_int, C.c_int, C.c_double, C.c_double, C.c_double, C.c_int, C.c_int,
                                C.c_int, C.c_int, C.c_double]),
    "adj_destroy": (None, [C.c_void_p]),
    "adj_grid": (None, [C.c_void_p, _IP, _IP, _IP]),
    "adj_set_formulation": (None, [C.c_void_p, C.c_int]),
    "adj_set_stype": (None, [C.c_void_p, C.c_int]),
    "adj_set_meal": (None, [C.c_void_p, _FP, _FP, _FP]),
    "adj_set_model": (None, [C.c_void_p] + [_DP] * 6),
    "adj_set_source": (None, [C.c_void_p, C.c_int, _IP, _IP, _DP]),
    "adj_set_receivers": (None, [C.c_void_p, C.c_int, C.c_int, _IP, _IP]),
    "adj_forward": (None, [C.c_void_p, C.POINTER(_DP)]),
    "adj_gradient": (C.c_double, [C.c_void_p, C.POINTER(_DP), _DP, _DP, _DP, _DP, _DP]),
}


def _d(a):
    return a.ctypes.data_as(_DP)


class AdjointOracle:
    """Double-precision forward and adjoint-state gradient of the three
    formulations (cfg variant; oracle/ttifd_adjoint.c) with the stress source
    or a velocity source (cfg stype, default 1). MEAL coef1, coef2
    and Beta are frozen from the float setup of `meal_model` (padded arrays);
    vs and rho stay fixed; the model (vp, eps, delta, theta) can be changed
    with set_model for finite differences."""

    def __init__(self, cfg: dict, meal_model):
        lib = load()
        for name, (res, args) in _ADJ_SIG.items():
            fn = getattr(lib, name)
            fn.restype, fn.argtypes = res, args
        self.lib = lib
        self.cfg = dict(cfg)
        c = self.cfg
        self._c = lib.adj_create(c["nz"], c["nx"], c["nt"], c["dx"], c["dz"], c["dt"], c["ealThick"],
                                 c.get("freesurface", 0), c.get("mt", 1), c["seistype"], c.get("scalar", 1.0))
        variant = c.get("variant", 0)
        variant = ttifd.VARIANTS[variant] if isinstance(variant, str) else int(variant)
        lib.adj_set_formulation(self._c, variant)
        lib.adj_set_stype(self._c, int(c.get("stype", 1)))
        nz, nx, nts = C.c_int(), C.c_int(), C.c_int()
        lib.adj_grid(self._c, C.byref(nz), C.byref(nx), C.byref(nts))
        self.Nz, self.Nx, self.nts = nz.value, nx.value, nts.value
        with Oracle(**dict(c, variant="coordinate_rotation", stype=1, wsave=0, energy=0)) as o:
            o.upload_model(*meal_model)
            meal = [np.ascontiguousarray(o.fetch_param(p)) for p in ("coef1", "coef2", "Beta")]
        lib.adj_set_meal(self._c, *[_f(a) for a in meal])
        self._nrec = {}
        self.nsrc = 0

    def close(self):
        if self._c:
            self.lib.adj_destroy(self._c)
            self._c = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def set_model(self, vp, vs, rho, eps, delta, theta):
        arrs = [np.ascontiguousarray(a, dtype=np.float64) for a in (vp, vs, rho, eps, delta, theta)]
        for a in arrs:
            assert a.shape == (self.Nx, self.Nz)
        self._model = arrs
        self.lib.adj_set_model(self._c, *[_d(a) for a in arrs])

    def set_source(self, sx, sz, w):
        w = np.ascontiguousarray(np.atleast_2d(w), dtype=np.float64)
        x = np.ascontiguousarray(np.atleast_1d(sx), dtype=np.int32)
        z = np.ascontiguousarray(np.atleast_1d(sz), dtype=np.int32)
        self._src = w
        self.nsrc = x.size
        self.lib.adj_set_source(self._c, x.size, _i(x), _i(z), _d(w))

    def set_receivers(self, kind, gx, gz):
        x = np.ascontiguousarray(gx, dtype=np.int32)
        z = np.ascontiguousarray(np.broadcast_to(gz, x.shape), dtype=np.int32)
        self._nrec[kind] = x.size
        self.lib.adj_set_receivers(self._c, kind, x.size, _i(x), _i(z))

    def _rec_arrays(self):
        out = [np.zeros((self._nrec.get(k, 0), self.nts)) if self._nrec.get(k) else None for k in range(3)]
        ptrs = (_DP * 3)(*[_d(a) if a is not None else _DP() for a in out])
        return out, ptrs

    def forward(self):
        """Traces per component ([ntrace][nts] or None)."""
        out, ptrs = self._rec_arrays()
        self.lib.adj_forward(self._c, ptrs)
        return out

    def gradient(self, dobs):
        """(J, {vp, eps, delta, theta: [Nx][Nz]}, g_src[nsrc][nt])."""
        obs = [np.ascontiguousarray(d, dtype=np.float64) if d is not None else None for d in dobs]
        ptrs = (_DP * 3)(*[_d(a) if a is not None else _DP() for a in obs])
        g = {k: np.zeros((self.Nx, self.Nz)) for k in ("vp", "eps", "delta", "theta")}
        gs = np.zeros((max(self.nsrc, 1), self.cfg["nt"]))
        J = self.lib.adj_gradient(self._c, ptrs, _d(g["vp"]), _d(g["eps"]), _d(g["delta"]), _d(g["theta"]), _d(gs))
        return J, g, gs[:self.nsrc]
