"""Seeded synthetic TTI models and SU geometry files.

The reference's demo model (BP 2007 TTI, ``demo/file/*_bp_1126_7872_10m.bin``)
is not available, so benchmarks and tests run on seeded synthetic models with
the demo's shapes and value ranges:

* :func:`layered_model` -- flat layers (vp 1500..4500 m/s, epsilon, delta per
  layer, theta a smooth random field), the small CPU-runnable case.
* :func:`salt_model` -- 40 dipping layers with vp rising 1480..4800 m/s with
  depth, an elliptical 4500 m/s isotropic body, epsilon/delta ranges of the
  BP model and theta following the local layer dip; the demo's 1126 x 7872 size.

vs = vp / 1.8 and rho = 310 vp^0.25 (kg/m^3) are always written explicitly, so
the reference's water defaults (vp <= 1500, modparconvert.c:42-58, 128-141) are
not exercised by the benchmark inputs.

Files follow the reference's formats: raw FP32 models of nx records of nz
samples (z fastest, read by coord:349-454); SU source files as written by
``sumksrc2d`` (src/main/wavelet/sumksrc2d.c: one trace, sdepth/sx scaled by
scalel = scalco = -1000, dt in microseconds); SU receiver files as written by
``sumkrcev2d`` (trace 1 = gx in cells, trace 2 = gz in cells, ns = number of
receivers).
"""
from __future__ import annotations

import os
from dataclasses import dataclass

import numpy as np

# SU trace header: 240 bytes (SEG-Y rev.0 positions + SU extension).
SU_HDR = 240
_OFF = {  # byte offsets of the header fields used here
    "tracl": (0, "<i4"), "tracr": (4, "<i4"), "fldr": (8, "<i4"), "cdp": (20, "<i4"),
    "trid": (28, "<i2"), "offset": (36, "<i4"), "sdepth": (48, "<i4"), "gdel": (52, "<i4"),
    "sdel": (56, "<i4"), "scalel": (68, "<i2"), "scalco": (70, "<i2"), "sx": (72, "<i4"),
    "gx": (80, "<i4"), "ns": (114, "<u2"), "dt": (116, "<u2"), "d1": (180, "<f4"),
    "f1": (184, "<f4"), "ntr": (204, "<i4"),
}


@dataclass
class Model:
    """Physical-grid model arrays, each float32 of shape (nx, nz) (z fastest)."""

    vp: np.ndarray
    vs: np.ndarray
    rho: np.ndarray
    epsilon: np.ndarray
    delta: np.ndarray
    theta: np.ndarray  # degrees

    @property
    def nx(self) -> int:
        return self.vp.shape[0]

    @property
    def nz(self) -> int:
        return self.vp.shape[1]

    def arrays(self):
        return self.vp, self.vs, self.rho, self.epsilon, self.delta, self.theta


def _smooth(field: np.ndarray, sigma: float) -> np.ndarray:
    """Gaussian smoothing by FFT (periodic; fine for random fields)."""
    nx, nz = field.shape
    kx = np.fft.fftfreq(nx)[:, None]
    kz = np.fft.rfftfreq(nz)[None, :]
    g = np.exp(-2.0 * (np.pi * sigma) ** 2 * (kx * kx + kz * kz))
    return np.fft.irfft2(np.fft.rfft2(field) * g, s=field.shape)


def _derived(vp: np.ndarray):
    vs = (vp / 1.8).astype(np.float32)
    rho = (310.0 * np.power(vp.astype(np.float64), 0.25)).astype(np.float32)
    return vs, rho


def layered_model(nz: int = 200, nx: int = 400, seed: int = 0, nlayers: int = 5,
                  theta_max: float = 40.0) -> Model:
    """Flat layers with vp 1500..4500 m/s; epsilon U[0,0.25], delta U[0,min(eps,0.12)]
    per layer; theta a Gaussian-smoothed random field rescaled to +-theta_max deg."""
    rng = np.random.default_rng(seed)
    depths = np.sort(rng.uniform(0.08, 0.95, size=nlayers - 1)) * nz
    vps = np.linspace(1500.0, 4500.0, nlayers)
    eps_l = rng.uniform(0.0, 0.25, size=nlayers)
    del_l = np.array([rng.uniform(0.0, min(e, 0.12)) for e in eps_l])
    iz = np.arange(nz)
    layer = np.searchsorted(depths, iz, side="right")
    vp = np.broadcast_to(vps[layer][None, :], (nx, nz)).astype(np.float32)
    eps = np.broadcast_to(eps_l[layer][None, :], (nx, nz)).astype(np.float32)
    dlt = np.broadcast_to(del_l[layer][None, :], (nx, nz)).astype(np.float32)
    th = _smooth(rng.standard_normal((nx, nz)), sigma=max(4.0, min(nx, nz) / 10.0))
    th = th - th.min()
    th = (2.0 * th / max(th.max(), 1e-12) - 1.0) * theta_max
    vs, rho = _derived(vp)
    return Model(np.ascontiguousarray(vp), vs, rho, np.ascontiguousarray(eps),
                 np.ascontiguousarray(dlt), th.astype(np.float32))


def salt_model(nz: int = 1126, nx: int = 7872, seed: int = 1, nlayers: int = 40,
               theta_max: float = 60.0) -> Model:
    """Dipping layered model with an elliptical isotropic 4500 m/s body."""
    rng = np.random.default_rng(seed)
    x = np.arange(nx, dtype=np.float64)[:, None]
    z = np.arange(nz, dtype=np.float64)[None, :]
    base = np.sort(rng.uniform(0.0, 1.0, size=nlayers - 1)) * nz
    # each interface: depth(x) = base + slope*x + amplitude*sin(...)
    slope = rng.uniform(-0.06, 0.06, size=nlayers - 1)
    amp = rng.uniform(0.0, 0.03 * nz, size=nlayers - 1)
    wl = rng.uniform(0.3, 1.5, size=nlayers - 1) * nx
    ph = rng.uniform(0.0, 2 * np.pi, size=nlayers - 1)
    xc = x[:, 0]
    idx = np.zeros((nx, nz), dtype=np.int32)
    dip = np.zeros((nx, nz), dtype=np.float64)
    for k in range(nlayers - 1):
        h = base[k] + slope[k] * (xc - nx / 2) + amp[k] * np.sin(2 * np.pi * xc / wl[k] + ph[k])
        dh = slope[k] + amp[k] * 2 * np.pi / wl[k] * np.cos(2 * np.pi * xc / wl[k] + ph[k])
        below = z >= h[:, None]
        idx += below
        dip = np.where(below, np.degrees(np.arctan(dh))[:, None], dip)
    vtop = np.linspace(1480.0, 4800.0, nlayers)
    vp = vtop[idx] + rng.normal(0.0, 40.0, size=nlayers)[idx]
    vp = np.clip(vp, 1480.0, 4800.0)
    eps_l = rng.uniform(0.0, 0.3, size=nlayers)
    del_l = rng.uniform(0.0, 0.15, size=nlayers)
    eps = eps_l[idx]
    dlt = np.minimum(del_l[idx], eps)
    th = np.clip(dip, -theta_max, theta_max)
    # elliptical isotropic body
    cx, cz = nx * rng.uniform(0.35, 0.65), nz * rng.uniform(0.45, 0.65)
    ax, az = nx * 0.12, nz * 0.15
    body = ((x - cx) / ax) ** 2 + ((z - cz) / az) ** 2 <= 1.0
    vp = np.where(body, 4500.0, vp)
    eps = np.where(body, 0.0, eps)
    dlt = np.where(body, 0.0, dlt)
    th = np.where(body, 0.0, th)
    vp = vp.astype(np.float32)
    vs, rho = _derived(vp)
    return Model(vp, vs, rho, eps.astype(np.float32), dlt.astype(np.float32), th.astype(np.float32))


def crop(m: Model, x0: int, nx: int) -> Model:
    """Columns x0..x0+nx-1 (cutbin2d semantics along the slow axis)."""
    return Model(*(np.ascontiguousarray(a[x0:x0 + nx]) for a in m.arrays()))


def ricker(nt: int, dt: float, fpeak: float, amp: float = 1.0, delay: float | None = None) -> np.ndarray:
    """Ricker wavelet with riker_wlt's conventions (src/lib/wavelet/wavelet.c:81-99):
    delay 1.5/fpeak, zero for t > delay after the shift, first sample zero."""
    f32 = np.float32
    if delay is None:
        delay = f32(1.5) / f32(fpeak)
    it = np.arange(nt, dtype=f32)
    t = it * f32(dt) - f32(delay)
    a = (f32(3.141592654) * f32(fpeak) * t) ** 2
    w = (f32(amp) * (f32(1.0) - f32(2.0) * a) * np.exp(-a)).astype(f32)
    w[t > delay] = 0.0
    if nt:
        w[0] = 0.0
    return w


# ---------------------------------------------------------------- SU files
def _header(**fields) -> bytearray:
    h = bytearray(SU_HDR)
    for k, v in fields.items():
        off, fmt = _OFF[k]
        h[off:off + np.dtype(fmt).itemsize] = np.array([v], dtype=fmt).tobytes()
    return h


def write_su_source(path: str, wavelets: np.ndarray, sx, sdepth, dt: float) -> None:
    """Source file as sumksrc2d writes it; several traces give several sources
    (read2dsource reads tr.ntr traces, obsinfo.c:34-87)."""
    w = np.atleast_2d(np.asarray(wavelets, dtype=np.float32))
    sx = np.atleast_1d(sx)
    sdepth = np.atleast_1d(sdepth)
    with open(path, "wb") as f:
        for k in range(w.shape[0]):
            f.write(_header(tracl=1, trid=1, scalel=-1000, scalco=-1000, sdepth=int(sdepth[k]) * 1000,
                            sx=int(sx[k]) * 1000, ns=w.shape[1], dt=int(round(dt * 1e6)), f1=0.0,
                            d1=float(dt), ntr=w.shape[0]))
            f.write(w[k].tobytes())


def write_su_receivers(path: str, gx, gz) -> None:
    """Receiver-position file as sumkrcev2d writes it (trace 1 gx, trace 2 gz)."""
    gx = np.asarray(gx, dtype=np.float32)
    gz = np.broadcast_to(np.asarray(gz, dtype=np.float32), gx.shape)
    with open(path, "wb") as f:
        for data in (gx, gz):
            f.write(_header(tracl=1, trid=1, scalel=-1000, scalco=-1000, ns=gx.size, ntr=2, f1=0.0, d1=1.0))
            f.write(np.ascontiguousarray(data, dtype=np.float32).tobytes())


def read_su(path: str):
    """Returns (headers: list of dict, data: float32 array [ntr, ns])."""
    raw = open(path, "rb").read()
    pos, hdrs, rows = 0, [], []
    while pos + SU_HDR <= len(raw):
        h = raw[pos:pos + SU_HDR]
        hd = {k: np.frombuffer(h[o:o + np.dtype(t).itemsize], dtype=t)[0].item() for k, (o, t) in _OFF.items()}
        ns = hd["ns"]
        rows.append(np.frombuffer(raw[pos + SU_HDR:pos + SU_HDR + 4 * ns], dtype=np.float32))
        hdrs.append(hd)
        pos += SU_HDR + 4 * ns
    return hdrs, (np.stack(rows) if rows else np.zeros((0, 0), np.float32))


def write_model(directory: str, m: Model, prefix: str = "") -> dict:
    """Writes vp/vs/rho/epsilon/delta/theta as raw FP32 files; returns paths."""
    os.makedirs(directory, exist_ok=True)
    out = {}
    for name, a in zip(("vp", "vs", "rho", "epsilon", "delta", "theta"), m.arrays()):
        p = os.path.join(directory, f"{prefix}{name}.bin")
        np.ascontiguousarray(a, dtype=np.float32).tofile(p)
        out[name] = p
    return out


# ---------------------------------------------------------------- padding
def pad(a: np.ndarray, E: int) -> np.ndarray:
    """padModel2d (src/lib/absorbc/padmod.c:33-59) on a (nx, nz) array -> (nx+2E, nz+2E):
    edge replication, top/bottom first then left/right full height."""
    nx, nz = a.shape
    out = np.zeros((nx + 2 * E, nz + 2 * E), dtype=np.float32)
    out[E:E + nx, E:E + nz] = a
    out[E:E + nx, :E] = a[:, :1]
    out[E:E + nx, E + nz:] = a[:, -1:]
    out[:E, :] = out[E:E + 1, :]
    out[E + nx:, :] = out[E + nx - 1:E + nx, :]
    return out


def padded(m: Model, ealThick: int):
    """The six padded arrays the C ABI takes (E = ealThick + 5)."""
    E = ealThick + 5
    return tuple(pad(a, E) for a in m.arrays())
