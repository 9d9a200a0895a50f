// C ABI of the B200 TTI RSG library (include/ttifd.h).
#include <cfloat>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <future>
#include <vector>

#include <algorithm>
#include <numeric>

#include "tiled.cuh"

using namespace ttifd;

namespace {

thread_local std::string g_create_error;

int set_err(tti_handle *h, int code, const char *fmt, ...)
{
  char buf[1024];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof buf, fmt, ap);
  va_end(ap);
  if (h) h->err = buf;
  else g_create_error = buf;
  return code;
}

// On failure the runtime's last error is cleared too, so that a refused
// allocation is not found again by a later launch check.
#define CK(h, call)                                                                                     \
  do {                                                                                                  \
    cudaError_t e_ = (call);                                                                            \
    if (e_ != cudaSuccess) {                                                                            \
      cudaGetLastError();                                                                               \
      return set_err((h), e_ == cudaErrorMemoryAllocation ? TTI_ERR_NOMEM : TTI_ERR_CUDA, "%s: %s (%s:%d)", \
                     #call, cudaGetErrorString(e_), __FILE__, __LINE__);                                \
    }                                                                                                   \
  } while (0)

// Arrays each formulation needs on the device (beyond D/Beta/coef/vp/vs/rho
// which every formulation keeps for the setup dumps).
bool param_used(int variant, int p)
{
  switch (p) {
  case TTI_P_C15:
  case TTI_P_C35:
    return variant == TTI_BOND;
  case TTI_P_SIN:
  case TTI_P_COS:
  case TTI_P_SIN_V:
  case TTI_P_COS_V:
    return variant == TTI_COORDINATE;
  case TTI_P_SIN2:
  case TTI_P_COS2:
  case TTI_P_SIN_2T:
    return variant == TTI_TENSOR;
  default:
    return true;
  }
}

int nfields(int variant) { return variant == TTI_TENSOR ? 8 : 5; }

StepArgs step_args(const tti_handle *h)
{
  StepArgs a;
  a.g = h->g;
  a.f = Fields{h->fld[0], h->fld[1], h->fld[2], h->fld[3], h->fld[4], h->fld[5], h->fld[6], h->fld[7]};
  const float *const *P = h->par;
  a.p = Params{P[TTI_P_COEF1], P[TTI_P_COEF2], P[TTI_P_INVRHO], P[TTI_P_C11], P[TTI_P_C13], P[TTI_P_C15],
               P[TTI_P_C33],   P[TTI_P_C35],   P[TTI_P_C55],    P[TTI_P_SIN], P[TTI_P_COS], P[TTI_P_SIN_V],
               P[TTI_P_COS_V], P[TTI_P_SIN2],  P[TTI_P_COS2],   P[TTI_P_SIN_2T]};
  a.invdx = h->invdx;
  a.invdz = h->invdz;
  a.variant = h->cfg.variant;
  a.exact = h->exact;
  return a;
}

// Host precompute of the source weight tables in the reference's float
// expression order (coord:607, 684-691, 711-713, 733-734, 775-777, 880-882).
void source_tables(const tti_handle *h, SourceTables *t)
{
  const float dx = h->cfg.dx, dz = h->cfg.dz, dt = h->cfg.dt;
  const float alpha = logf(0.8f) / (dx * dx + dz * dz);
  for (int a = 0; a < 11; ++a)
    for (int b = 0; b < 11; ++b) {
      const float rx = (a - NH) * dx, rz = (b - NH) * dz;
      const float w = expf(alpha * (rx * rx + rz * rz)) * h->invdx * h->invdz * dt;
      const int k = a * 11 + b;
      t->k1[k] = 0.5f * w;
      t->kx[k] = 2.0f * alpha * rx * w;
      t->kz[k] = 2.0f * alpha * rz * w;
      t->k5[k] = w;
      t->k7[k] = 0.5f * sqrtf(2.0f) * w;
    }
  t->q8 = 0.125f * sqrtf(2.0f);
}

int check_cfg(const tti_config *c)
{
  if (c->variant < 0 || c->variant > 2) return set_err(nullptr, TTI_ERR_ARG, "variant must be 0, 1 or 2");
  if (c->nz <= 0 || c->nx <= 0 || c->nt <= 0) return set_err(nullptr, TTI_ERR_ARG, "nz, nx, nt must be positive");
  if (!(c->dx > 0) || !(c->dz > 0) || !(c->dt > 0)) return set_err(nullptr, TTI_ERR_ARG, "dx, dz, dt must be positive");
  if (c->ealThick < 0) return set_err(nullptr, TTI_ERR_ARG, "ealThick must be >= 0");
  if (!(c->fpeak > 0)) return set_err(nullptr, TTI_ERR_ARG, "fpeak must be positive");
  if (c->freesurface != 0 && c->freesurface != 1) return set_err(nullptr, TTI_ERR_ARG, "freesurface must be 0 or 1");
  if (c->stype < 1 || c->stype > 8) return set_err(nullptr, TTI_ERR_ARG, "stype must be 1..8");
  if (c->seistype < 0 || c->seistype > 3) return set_err(nullptr, TTI_ERR_ARG, "seistype must be 0..3");
  if (c->mt < 1) return set_err(nullptr, TTI_ERR_ARG, "mt must be >= 1");
  if (c->wsave < 0 || c->wsave > 5) return set_err(nullptr, TTI_ERR_ARG, "wsave must be 0..5");
  if (c->savew != 0 && c->savew != 1) return set_err(nullptr, TTI_ERR_ARG, "savew must be 0 or 1");
  if (c->wsave > 0 && c->snap_sample < 1) return set_err(nullptr, TTI_ERR_ARG, "snap_sample must be >= 1");
  if (c->mode != 1 && c->mode != 2) return set_err(nullptr, TTI_ERR_ARG, "mode must be 1 or 2");
  return TTI_OK;
}

int current_it(const tti_handle *h) { return h->cfg.mode == 2 ? h->cfg.nt - 1 - h->step_index : h->step_index; }

// Launches one time step (coord:611-926 body). With `ev` (5 events) the
// phases are bracketed for tti_profile_steps: ev[0] | velocity | ev[1] |
// velocity sources | ev[2] | stress | ev[3] | the rest | ev[4]. With `keep`
// (5 device arrays, the gradient's recompute pass) vx, vz, sxx, szz, sxz are
// copied there between the velocity sources and the stress update.
int launch_one_step(tti_handle *h, const SourceTables &tab, cudaEvent_t *ev = nullptr, float *const *keep = nullptr)
{
  const tti_config &c = h->cfg;
  const int it = current_it(h);
  StepArgs a = step_args(h);
  SourceSet s{h->nsrc, h->d_sx, h->d_sz, h->d_src, c.nt};
  const bool vsrc = s.n > 0 && c.stype >= 2, ssrc = s.n > 0 && c.stype == 1;
  tiled::HalfArgs ha{};
  // What the gradient keeps of this step (keep_fields). Tiled kernels: the
  // stress kernel writes the strain rates vxx vxz vzx vzz (keep[0..3]) and for
  // the tensor rotation the tau it starts from (keep[4..6]); the coordinate
  // velocity kernel writes the stress derivative combinations P Q R S
  // (keep[4..7]). Per-cell kernels: a copy of vx vz and sxx szz sxz (tensor:
  // txx tzz txz) after the sources, from whose stencils the adjoint works.
  const bool keep_tiled = keep && h->use_tiled;
  if (h->use_tiled) {
    const CUtensorMap *tm = static_cast<const CUtensorMap *>(h->tmaps);
    ha.g = h->g;
    ha.f = a.f;
    ha.p = a.p;
    ha.pk = packed::Packed{h->pk_cf, h->pk_vsc, h->pk_sc, h->pk_c4};
    ha.invdx = h->invdx;
    ha.invdz = h->invdz;
    ha.dt = c.dt;
    ha.x_base = NH;
    ha.undamped_ok = h->undamped_ok;
    ha.freesurface = c.freesurface;
    tiled::set_square(ha, h->exact);
    ha.wait_limit = h->wait_limit;
    ha.err = h->d_flag;
    ha.map[0] = tm[2];  // sxx szz sxz for the velocity update
    ha.map[1] = tm[3];
    ha.map[2] = tm[4];
    if (keep_tiled && c.variant == TTI_COORDINATE)
      for (int k = 0; k < 4; ++k) ha.kd[k] = keep[4 + k];
  }
  if (ev) CK(h, cudaEventRecord(ev[0], h->stream));
  if (h->use_tiled) CK(h, tiled::launch_velocity(ha, c.variant, h->exact, h->stream));
  else launch_velocity(a, h->stream);
  if (ev) CK(h, cudaEventRecord(ev[1], h->stream));
  if (vsrc) launch_sources(a, s, &tab, c.stype, 0, it, h->stream);
  if (keep && !keep_tiled) {  // v after the sources, and sigma or tau
    const bool t = c.variant == TTI_TENSOR;
    float *const src[5] = {h->fld[0], h->fld[1], h->fld[t ? 5 : 2], h->fld[t ? 6 : 3], h->fld[t ? 7 : 4]};
    launch_copy5(src, keep, 5, h->g.n, h->stream);
    h->launches++;
  }
  if (ev) CK(h, cudaEventRecord(ev[2], h->stream));
  if (h->use_tiled) {
    const CUtensorMap *tm = static_cast<const CUtensorMap *>(h->tmaps);
    ha.map[0] = tm[0];  // vx vz for the stress update
    ha.map[1] = tm[1];
    for (int k = 0; k < 4; ++k) ha.kd[k] = keep_tiled ? keep[k] : nullptr;
    for (int k = 0; k < 3; ++k) ha.kt[k] = keep_tiled && c.variant == TTI_TENSOR ? keep[4 + k] : nullptr;
    CK(h, tiled::launch_stress(ha, c.variant, h->exact, h->stream));
  } else {
    launch_stress(a, h->stream);
  }
  if (ev) CK(h, cudaEventRecord(ev[3], h->stream));
  h->launches += 2 + vsrc;
  // free surface, stress source and receivers: one column-parallel launch
  const bool rec_now = c.seistype > 0 && it % c.mt == 0 && h->nrec[0] + h->nrec[1] + h->nrec[2] > 0;
  if (c.freesurface == 1 || ssrc || rec_now) {
    PostArgs pa;
    pa.freesurface = c.freesurface;
    pa.stype = ssrc ? 1 : 0;
    pa.tensor = c.variant == TTI_TENSOR;
    pa.it = it;
    pa.irec = rec_now ? it / c.mt : -1;
    pa.src = s;
    memcpy(pa.k1, tab.k1, sizeof pa.k1);
    const bool want_v = c.seistype == 1 || c.seistype == 3, want_p = c.seistype == 2 || c.seistype == 3;
    for (int k = 0; k < 3; ++k) {
      const bool on = (k < 2 ? want_v : want_p) && h->nrec[k] > 0;
      pa.colptr[k] = on ? h->d_rcol[k] : nullptr;
      pa.rz[k] = h->d_rzs[k];
      pa.rid[k] = h->d_rid[k];
      pa.rec[k] = h->d_rec[k];
      pa.nrec[k] = h->nrec[k];
    }
    pa.flag = h->d_flag;
    launch_post(a, pa, h->stream);
    h->launches++;
  }
  if (c.energy == 1) {
    launch_energy(a, c.nz, c.nx, h->d_energy + 2 * (size_t)it, h->stream);
    h->launches++;
  }
  if (ev) CK(h, cudaEventRecord(ev[4], h->stream));
  CK(h, cudaGetLastError());
  h->step_index++;
  return TTI_OK;
}

int snapshot_kinds(int wsave, int *kinds)
{
  switch (wsave) {
  case 1: kinds[0] = 1; kinds[1] = 2; return 2;
  case 2: kinds[0] = 3; return 1;
  case 3: kinds[0] = 1; kinds[1] = 2; kinds[2] = 3; return 3;
  case 4: kinds[0] = 4; kinds[1] = 5; return 2;
  case 5: kinds[0] = 6; kinds[1] = 7; return 2;
  default: return 0;
  }
}

// Copies `bytes` from device memory into a host buffer whose pages are
// resident, ordered after the work already on h's stream; returns once the
// data are in place. Above one chunk, through two page-locked chunks: the DMA
// of chunk c runs while host threads copy chunk c - 1 out (the driver's own
// staging of a pageable destination is slower); otherwise directly.
int download(tti_handle *h, void *dst, const void *src, size_t bytes)
{
  constexpr size_t CH = PIN_CHUNK * sizeof(float);
  float *pin[2] = {nullptr, nullptr};
  if (bytes > CH) {
    pin[0] = pinned_chunk();
    pin[1] = pinned_chunk();
  }
  for (int b = 0; b < 2 && pin[0] && pin[1]; ++b)
    if (!h->pev[5 + b] && cudaEventCreateWithFlags(&h->pev[5 + b], cudaEventDisableTiming) != cudaSuccess)
      pinned_release(pin[b]), pin[b] = nullptr;
  if (!pin[0] || !pin[1]) {
    pinned_release(pin[0]);
    pinned_release(pin[1]);
    CK(h, cudaMemcpyAsync(dst, src, bytes, cudaMemcpyDeviceToHost, h->stream));
    CK(h, cudaStreamSynchronize(h->stream));
    return TTI_OK;
  }
  const size_t nchunk = (bytes + CH - 1) / CH;
  cudaError_t e = cudaSuccess;
  for (size_t c = 0; c <= nchunk && e == cudaSuccess; ++c) {
    if (c < nchunk) {
      const size_t off = c * CH, nb = std::min(CH, bytes - off);
      e = cudaMemcpyAsync(pin[c & 1], static_cast<const char *>(src) + off, nb, cudaMemcpyDeviceToHost, h->stream);
      if (e == cudaSuccess) e = cudaEventRecord(h->pev[5 + (c & 1)], h->stream);
    }
    if (c > 0 && e == cudaSuccess) {
      const size_t p = c - 1, off = p * CH, nb = std::min(CH, bytes - off);
      e = cudaEventSynchronize(h->pev[5 + (p & 1)]);
      if (e == cudaSuccess) parallel_copy(static_cast<char *>(dst) + off, pin[p & 1], nb, 8);
    }
  }
  // wait on the error path too before the chunks go back to the shared list
  const cudaError_t es = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = es;
  pinned_release(pin[0]);
  pinned_release(pin[1]);
  CK(h, e);
  return TTI_OK;
}

// Output size of one snapshot kind (savew = 0: the physical area).
void snapshot_dims(const tti_handle *h, int *nzo, int *nxo)
{
  const Grid &g = h->g;
  *nzo = h->cfg.savew == 0 ? g.Nz - 2 * g.E : g.Nz;
  *nxo = h->cfg.savew == 0 ? g.Nx - 2 * g.E : g.Nx;
}

// The snapshot of step h->snap_it whose copy into the caller's page-locked
// buffer is in flight on copy_stream: waits for the copy, then (deliver) runs
// the callbacks of its kinds in order. Error paths drop it once the copy is
// done, so that no transfer into the caller's buffer outlives tti_run.
int finish_snapshot(tti_handle *h, bool deliver)
{
  if (!h->snap_pending) return TTI_OK;
  h->snap_pending = false;
  const cudaError_t e = cudaEventSynchronize(h->snap_done);
  if (!deliver) return TTI_OK;
  CK(h, e);
  int nzo, nxo, kinds[3];
  snapshot_dims(h, &nzo, &nxo);
  const size_t n = (size_t)nzo * nxo;
  const int nk = snapshot_kinds(h->cfg.wsave, kinds);
  for (int q = 0; q < nk; ++q)
    if (h->snap_fn(h->snap_arg, h->snap_it, kinds[q], h->snap_user + q * n, nzo, nxo) != 0)
      return set_err(h, TTI_ERR_CALLBACK, "snapshot callback aborted the run at it=%d", h->snap_it);
  return TTI_OK;
}

int do_snapshot(tti_handle *h, tti_snapshot_fn fn, void *user, int it)
{
  int nzo, nxo, kinds[3];
  snapshot_dims(h, &nzo, &nxo);
  const size_t n = (size_t)nzo * nxo;
  const int nk = snapshot_kinds(h->cfg.wsave, kinds);
  // Into the caller's page-locked buffer: every kind packed on the device, one
  // copy on copy_stream that overlaps the next time steps on h->stream.
  const bool overlap = h->snap_user && h->snap_user_pinned;
  const size_t dev = overlap ? nk * n : n;
  if (overlap) {
    const int rc = finish_snapshot(h, true);  // the previous one, and d_snap is free again
    if (rc) return rc;
  }
  if (h->snap_cap < dev) {
    pool_free(h->d_snap, h->stream);
    h->d_snap = nullptr;
    h->snap_cap = 0;
    CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_snap), dev * sizeof(float), h->stream));
    h->snap_cap = dev;
  }
  StepArgs a = step_args(h);
  if (overlap) {
    if (!h->copy_stream) CK(h, cudaStreamCreateWithFlags(&h->copy_stream, cudaStreamNonBlocking));
    if (!h->snap_packed) CK(h, cudaEventCreateWithFlags(&h->snap_packed, cudaEventDisableTiming));
    if (!h->snap_done) CK(h, cudaEventCreateWithFlags(&h->snap_done, cudaEventDisableTiming));
    for (int q = 0; q < nk; ++q) {
      launch_snapshot(a, kinds[q], h->cfg.savew, h->d_snap + q * n, h->stream);
      h->launches++;
    }
    CK(h, cudaEventRecord(h->snap_packed, h->stream));
    CK(h, cudaStreamWaitEvent(h->copy_stream, h->snap_packed, 0));
    CK(h, cudaMemcpyAsync(h->snap_user, h->d_snap, nk * n * sizeof(float), cudaMemcpyDeviceToHost, h->copy_stream));
    CK(h, cudaEventRecord(h->snap_done, h->copy_stream));
    h->snap_pending = true;
    h->snap_it = it;
    h->snap_fn = fn;
    h->snap_arg = user;
    return TTI_OK;
  }
  float *host = h->snap_user;  // a pageable caller's buffer: kind q at q * n
  if (!host && h->h_snap_cap < n) {
    free(h->h_snap);
    h->h_snap_cap = 0;
    h->h_snap = static_cast<float *>(malloc(n * sizeof(float)));
    if (!h->h_snap) return set_err(h, TTI_ERR_NOMEM, "host allocation of the snapshot buffer failed");
    prefault(h->h_snap, n * sizeof(float));
    h->h_snap_cap = n;
  }
  for (int q = 0; q < nk; ++q) {
    float *dst = host ? host + q * n : h->h_snap;
    launch_snapshot(a, kinds[q], h->cfg.savew, h->d_snap, h->stream);
    h->launches++;
    const int rc = download(h, dst, h->d_snap, n * sizeof(float));
    if (rc) return rc;
    if (fn(user, it, kinds[q], dst, nzo, nxo) != 0)
      return set_err(h, TTI_ERR_CALLBACK, "snapshot callback aborted the run at it=%d", it);
  }
  return TTI_OK;
}

// The time loop of tti_run after the reset; device time between events
// ev0 and ev1. A snapshot of the last snapshot step may still be in flight.
int run_steps(tti_handle *h, const SourceTables &tab, tti_snapshot_fn snap, void *user)
{
  const tti_config &c = h->cfg;
  CK(h, cudaEventRecord(h->ev0, h->stream));
  for (int n = 0; n < c.nt; ++n) {
    const int it = current_it(h);
    int rc = launch_one_step(h, tab);
    if (rc == TTI_OK && snap && c.wsave > 0 && it % c.snap_sample == 0) rc = do_snapshot(h, snap, user, it);
    if (rc) return rc;
  }
  CK(h, cudaEventRecord(h->ev1, h->stream));
  CK(h, cudaEventSynchronize(h->ev1));
  CK(h, cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  return TTI_OK;
}

int check_flag(tti_handle *h)
{
  int flag = 0;
  CK(h, cudaMemcpyAsync(&flag, h->d_flag, sizeof(int), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  if (flag & 4) return set_err(h, TTI_ERR_CUDA, "a TMA tile wait timed out in a tiled half-step kernel");
  if (flag) return set_err(h, TTI_ERR_NONFINITE, "non-finite value recorded at a receiver (unstable run?)");
  return TTI_OK;
}

// Copies na host arrays [Nx][Nz] into dense device arrays [Nx][Nz] on h's
// stream (dense, not pitched: a contiguous host-to-device copy runs about 1.5x
// faster than a pitched one of the same bytes; the setup kernel re-pitches).
// From page-locked arrays (tti_host_alloc) one copy each, at the link's rate.
// Otherwise through two page-locked chunks, column blocks at a time: host threads copy
// block c into one chunk while the DMA engine moves block c - 1 from the other
// (TTIFD_UPLOAD=pageable: straight from the caller's pageable arrays, which
// the driver stages itself, about 10.5 GB/s on B200 hosts).
// `na` dense host arrays of `ncol` columns of `sl` floats each into dense
// device arrays (the padded model: Nx columns of Nz; the physical one: nx of nz).
int upload_arrays(tti_handle *h, const float *const *src, float *const *dst, int na, int sl, int ncol)
{
  const size_t col = (size_t)sl * sizeof(float);
  auto copy = [&](int k, int x0, const float *from, int nx) {
    return cudaMemcpyAsync(dst[k] + (size_t)x0 * sl, from, col * nx, cudaMemcpyHostToDevice, h->stream);
  };
  bool pinned = true;  // all from page-locked memory: straight to the device
  for (int k = 0; k < na; ++k) pinned = pinned && is_pinned(src[k]);
  if (pinned) {
    for (int k = 0; k < na; ++k) CK(h, copy(k, 0, src[k], ncol));
    return TTI_OK;
  }
  const char *mode = getenv("TTIFD_UPLOAD");
  const bool pageable = mode && strcmp(mode, "pageable") == 0;
  const int per = (int)std::min<size_t>(ncol, PIN_CHUNK / sl);  // columns per chunk
  float *pin[2] = {nullptr, nullptr};
  if (!pageable && per > 0) {
    pin[0] = pinned_chunk();
    pin[1] = pinned_chunk();
  }
  for (int b = 0; b < 2 && pin[0] && pin[1]; ++b)
    if (!h->pev[5 + b] && cudaEventCreateWithFlags(&h->pev[5 + b], cudaEventDisableTiming) != cudaSuccess)
      pinned_release(pin[b]), pin[b] = nullptr;
  if (!pin[0] || !pin[1]) {
    pinned_release(pin[0]);
    pinned_release(pin[1]);
    for (int k = 0; k < na; ++k) CK(h, copy(k, 0, src[k], ncol));
    return TTI_OK;
  }
  cudaError_t e = cudaSuccess;
  bool pending[2] = {false, false};
  int c = 0;
  for (int k = 0; k < na && e == cudaSuccess; ++k)
    for (int x0 = 0; x0 < ncol && e == cudaSuccess; x0 += per, ++c) {
      const int nx = std::min(per, ncol - x0), b = c & 1;
      if (pending[b]) e = cudaEventSynchronize(h->pev[5 + b]);  // chunk b's previous DMA has drained
      if (e != cudaSuccess) break;
      parallel_copy(pin[b], src[k] + (size_t)x0 * sl, col * nx, 8);
      e = copy(k, x0, pin[b], nx);
      if (e == cudaSuccess) e = cudaEventRecord(h->pev[5 + b], h->stream);
      pending[b] = true;
    }
  // the chunks go back to the shared free list only once their copies are done
  const cudaError_t es = cudaStreamSynchronize(h->stream);
  if (e == cudaSuccess) e = es;
  pinned_release(pin[0]);
  pinned_release(pin[1]);
  CK(h, e);
  return TTI_OK;
}

int copy_out_pitched(tti_handle *h, const float *src, float *out)
{
  const Grid &g = h->g;
  CK(h, cudaMemcpy2DAsync(out, (size_t)g.Nz * sizeof(float), src, (size_t)g.ldz * sizeof(float),
                          (size_t)g.Nz * sizeof(float), g.Nx, cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  return TTI_OK;
}

}  // namespace

namespace ttifd {
int keep_fields(const tti_handle *h)
{
  if (!h->use_tiled) return 5;
  return h->cfg.variant == TTI_COORDINATE ? 8 : h->cfg.variant == TTI_TENSOR ? 7 : 4;
}
StepArgs handle_step_args(const tti_handle *h) { return step_args(h); }
void handle_source_tables(const tti_handle *h, SourceTables *t) { source_tables(h, t); }
int handle_step(tti_handle *h, const SourceTables &tab, float *const *keep)
{
  return launch_one_step(h, tab, nullptr, keep);
}
int handle_check_flag(tti_handle *h) { return check_flag(h); }
int handle_error(tti_handle *h, int code, const char *msg) { return set_err(h, code, "%s", msg); }
}  // namespace ttifd

extern "C" {

const char *tti_last_error(const tti_handle *h) { return h ? h->err.c_str() : g_create_error.c_str(); }

int tti_create(tti_handle **out, const tti_config *cfg, int device)
{
  return ttifd::create_handle(out, cfg, device, nullptr, false);
}

}  // extern "C"

namespace ttifd {

// tti_create with two options for batched execution: `share` (its parameter
// arrays are used, not allocated; cfg must describe the same grid) and
// `force_tiled` (the tiled kernels whatever TTIFD_KERNEL says).
int create_handle(tti_handle **out, const tti_config *cfg, int device, const tti_handle *share, bool force_tiled)
{
  if (!out || !cfg) return set_err(nullptr, TTI_ERR_ARG, "null argument");
  *out = nullptr;
  int rc = check_cfg(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
    return set_err(nullptr, TTI_ERR_CUDA, "no CUDA device available");
  if (device < 0 || device >= ndev) return set_err(nullptr, TTI_ERR_ARG, "device %d out of range", device);
  tti_handle *h = new tti_handle();
  h->cfg = *cfg;
  h->device = device;
  // Default arithmetic: every product and sum rounded separately in the
  // reference's expression order (the results of a -ffp-contract=off build of
  // the reference, bit for bit); TTIFD_EXACT=0 lets the compiler contract into
  // FMA (about 3 % faster on the full workload, within 1e-5 of it otherwise).
  const char *ex = getenv("TTIFD_EXACT");
  h->exact = !(ex && ex[0] == '0');
  // test hook: polls of the first TMA wait of the tiled kernels (the timeout path)
  const char *wl = getenv("TTIFD_WAIT_LIMIT");
  h->wait_limit = wl && *wl ? (unsigned)strtoul(wl, nullptr, 10) : tiled::tma::WAIT_LIMIT;
  Grid &g = h->g;
  g.E = cfg->ealThick + NH;
  g.Nz = cfg->nz + 2 * g.E;
  g.Nx = cfg->nx + 2 * g.E;
  g.ldz = (g.Nz + 31) / 32 * 32;
  g.izStart = cfg->freesurface == 0 ? NH : g.E;
  g.n = (size_t)g.ldz * g.Nx;
  h->invdx = (float)(1.0 / cfg->dx);
  h->invdz = (float)(1.0 / cfg->dz);
  h->nts = (cfg->nt - 1) / cfg->mt + 1;
  auto fail = [&](int code) {
    std::string msg = h->err;
    tti_destroy(h);
    set_err(nullptr, code, "%s", msg.c_str());
    return code;
  };
  if (cudaSetDevice(device) != cudaSuccess) {
    set_err(h, TTI_ERR_CUDA, "cudaSetDevice(%d) failed", device);
    return fail(TTI_ERR_CUDA);
  }
  auto alloc = [&](float **p) -> int {
    cudaError_t e = pool_alloc(reinterpret_cast<void **>(p), g.n * sizeof(float), h->stream);
    if (e != cudaSuccess)
      return set_err(h, TTI_ERR_NOMEM, "device allocation of %zu bytes failed: %s", g.n * sizeof(float),
                     cudaGetErrorString(e));
    e = cudaMemsetAsync(*p, 0, g.n * sizeof(float), h->stream);
    if (e != cudaSuccess) return set_err(h, TTI_ERR_CUDA, "cudaMemset failed: %s", cudaGetErrorString(e));
    return TTI_OK;
  };
  if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess ||
      cudaEventCreate(&h->ev0) != cudaSuccess || cudaEventCreate(&h->ev1) != cudaSuccess) {
    set_err(h, TTI_ERR_CUDA, "stream/event creation failed");
    return fail(TTI_ERR_CUDA);
  }
  {
    // default: the tiled half-step kernels; TTIFD_KERNEL=naive selects the
    // one-thread-per-cell kernels (the cross-check path)
    const char *kern = getenv("TTIFD_KERNEL");
    const bool naive = kern && strcmp(kern, "naive") == 0;
    h->use_tiled = force_tiled || !naive;
  }
  for (int f = 0; f < nfields(cfg->variant); ++f)
    if ((rc = alloc(&h->fld[f]))) return fail(rc);
  if (h->use_tiled) {
    void *mem = nullptr;
    if (posix_memalign(&mem, 64, 5 * sizeof(CUtensorMap)) != 0) {
      set_err(h, TTI_ERR_NOMEM, "host allocation failed");
      return fail(TTI_ERR_NOMEM);
    }
    h->tmaps = mem;
    CUtensorMap *tm = static_cast<CUtensorMap *>(mem);
    for (int k = 0; k < 5; ++k)
      if (!tiled::encode_map(tm + k, g, h->fld[k])) {
        set_err(h, TTI_ERR_CUDA, "cuTensorMapEncodeTiled failed");
        return fail(TTI_ERR_CUDA);
      }
  }
  if (share) {
    h->owner = share;
    for (int p = 0; p < TTI_P_COUNT; ++p) h->par[p] = share->par[p];
    h->pk_cf = share->pk_cf;
    h->pk_vsc = share->pk_vsc;
    h->pk_sc = share->pk_sc;
    h->pk_c4 = share->pk_c4;
  } else if (h->use_tiled) {
    auto palloc = [&](void *p, size_t bytes) {
      return pool_alloc(static_cast<void **>(p), bytes, h->stream) == cudaSuccess;
    };
    bool okp = palloc(&h->pk_cf, g.n * sizeof(float2)) && palloc(&h->pk_sc, g.n * sizeof(float2)) &&
               palloc(&h->pk_c4, g.n * sizeof(float4)) &&
               (cfg->variant != TTI_COORDINATE || palloc(&h->pk_vsc, g.n * sizeof(float2)));
    if (!okp) {
      set_err(h, TTI_ERR_NOMEM, "device allocation of the packed parameters failed");
      return fail(TTI_ERR_NOMEM);
    }
  }
  for (int p = 0; p < TTI_P_COUNT && !share; ++p)
    if (param_used(cfg->variant, p) && (rc = alloc(&h->par[p]))) return fail(rc);
  if (pool_alloc(reinterpret_cast<void **>(&h->d_flag), sizeof(int), h->stream) != cudaSuccess ||
      pool_alloc(reinterpret_cast<void **>(&h->d_energy), sizeof(double) * 2 * (size_t)cfg->nt, h->stream) !=
          cudaSuccess) {
    set_err(h, TTI_ERR_NOMEM, "device allocation failed");
    return fail(TTI_ERR_NOMEM);
  }
  cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream);
  cudaMemsetAsync(h->d_energy, 0, sizeof(double) * 2 * (size_t)cfg->nt, h->stream);
  if (cudaStreamSynchronize(h->stream) != cudaSuccess) {
    set_err(h, TTI_ERR_CUDA, "initialisation failed");
    return fail(TTI_ERR_CUDA);
  }
  *out = h;
  return TTI_OK;
}

}  // namespace ttifd

extern "C" {

int tti_destroy(tti_handle *h)
{
  if (!h) return TTI_OK;
  cudaSetDevice(h->device);
  if (h->stream) cudaStreamSynchronize(h->stream);
  cudaStream_t fs = h->stream;  // pool blocks are released in stream order
  for (auto &p : h->fld) pool_free(p, fs);
  if (!h->owner) {
    for (auto &p : h->par) pool_free(p, fs);
    pool_free(h->pk_cf, fs);
    pool_free(h->pk_vsc, fs);
    pool_free(h->pk_sc, fs);
    pool_free(h->pk_c4, fs);
  }
  for (int k = 0; k < 3; ++k) {
    pool_free(h->d_rz[k], fs);  // with d_rzs, d_rid, d_rcol (one block)
    pool_free(h->d_rec[k], fs);
  }
  pool_free(h->d_sx, fs);
  pool_free(h->d_sz, fs);
  pool_free(h->d_src, fs);
  pool_free(h->d_energy, fs);
  pool_free(h->d_flag, fs);
  if (!h->owner) {  // a batch instance borrows its model's copies
    pool_free(h->m_eps, fs);
    pool_free(h->m_delta, fs);
    pool_free(h->m_theta, fs);
  }
  pool_free(h->d_snap, fs);
  pool_free(h->d_stage, fs);
  if (fs) cudaStreamSynchronize(fs);
  grad_release(h);
  free(h->h_snap);
  if (h->ev0) cudaEventDestroy(h->ev0);
  if (h->ev1) cudaEventDestroy(h->ev1);
  free(h->tmaps);
  for (auto e : h->pev)
    if (e) cudaEventDestroy(e);
  if (h->snap_packed) cudaEventDestroy(h->snap_packed);
  if (h->snap_done) cudaEventDestroy(h->snap_done);
  if (h->copy_stream) cudaStreamDestroy(h->copy_stream);
  if (h->stream) cudaStreamDestroy(h->stream);
  delete h;
  return TTI_OK;
}

int tti_grid(const tti_handle *h, int *Nz, int *Nx, int *E)
{
  if (!h) return TTI_ERR_ARG;
  if (Nz) *Nz = h->g.Nz;
  if (Nx) *Nx = h->g.Nx;
  if (E) *E = h->g.E;
  return TTI_OK;
}

// tti_upload_model (padded arrays) and tti_upload_model_physical (physical
// arrays, the rims filled on the device) from here on are one path.
static int upload_model(tti_handle *h, const float *const *src, bool physical)
{
  for (int k = 0; k < 6; ++k)
    if (!src[k]) return set_err(h, TTI_ERR_ARG, "null model array");
  if (h->owner) return set_err(h, TTI_ERR_STATE, "this handle shares the parameters of another; upload through it");
  CK(h, cudaSetDevice(h->device));
  const tti_config &c = h->cfg;
  const Grid &g = h->g;
  const size_t np = (size_t)g.Nz * g.Nx;
  // Stability check on the unscaled padded vp (stable.c:217-246; the rims
  // repeat physical values, so the physical maximum is the padded one). Its
  // host maximum runs on other threads while the arrays travel to the
  // device; nothing is computed from them on the device before it has passed.
  const float *vp = src[0];
  const size_t nv = physical ? (size_t)c.nz * c.nx : np;
  auto vmax_f = std::async(std::launch::async, [vp, nv] { return host_max(vp, nv, FLT_MIN); });
  // raw model on the device (dense [Nx][Nz], one block of six arrays), freed
  // after the precompute; a physical model first lands densely after it (one
  // contiguous copy per array: a pitched copy into the padded layout ran
  // slower than the padded bytes it saves) and is expanded on the device
  float *raw[6] = {}, *phys[6] = {};
  float *d_w = nullptr, *raw_block = nullptr;
  int rc = TTI_OK;
  {
    const size_t extra = physical ? 6 * nv : 0;
    cudaError_t e = pool_alloc(reinterpret_cast<void **>(&raw_block), (6 * np + extra) * sizeof(float), h->stream);
    if (e != cudaSuccess) rc = set_err(h, TTI_ERR_NOMEM, "device allocation failed: %s", cudaGetErrorString(e));
  }
  for (int k = 0; k < 6; ++k) {
    raw[k] = raw_block + (size_t)k * np;
    phys[k] = raw_block + 6 * np + (size_t)k * nv;
  }
  if (rc == TTI_OK)
    rc = physical ? upload_arrays(h, src, phys, 6, c.nz, c.nx)
                  : upload_arrays(h, src, raw, 6, g.Nz, g.Nx);
  if (rc == TTI_OK && physical) {
    launch_expand_physical(phys[0], raw_block, 6, c.nz, c.nx, g.E, h->stream);
    if (cudaGetLastError() != cudaSuccess) rc = set_err(h, TTI_ERR_CUDA, "model expansion kernel failed to launch");
  }
  {
    const double vmax = vmax_f.get();
    const double csum = (double)rsg(0) + (double)rsg(2) + (double)rsg(4);
    const double dtmax = 1.0f / (vmax * sqrt((1.0 / (c.dx * c.dx) + 1.0 / (c.dz * c.dz)) * csum));
    if (rc == TTI_OK && c.dt > dtmax) {
      cudaStreamSynchronize(h->stream);
      pool_free(raw_block, h->stream);
      return set_err(h, TTI_ERR_UNSTABLE,
                     "the finite differenct scheme is unstable! the time step size must smaller than %5.5f!", dtmax);
    }
  }
  if (rc == TTI_OK) {
    // MEAL scalars evaluated with the host libm, as meal.c:23-29, 62-66 do
    const int nl = g.E;
    const float pd = 2;
    const float Rcoef = powf(10.0f, -1.0f * ((log10f((float)nl) - 1.0f) / (log10f(2.0f))) - 3.0f - 0.5f * pd);
    const float alpha = c.eal_alpha == -1.0f ? 2.5f : c.eal_alpha;
    std::vector<float> w(nl + 1, 0.0f);
    for (int l = 1; l <= nl; ++l) {
      const float d = (0.1f * l) / (0.1f * nl);
      w[l] = expf(logf(2.0f) * powf(d, alpha)) - 1.0f;
    }
    cudaError_t e = pool_alloc(reinterpret_cast<void **>(&d_w), sizeof(float) * (nl + 1), h->stream);
    if (e == cudaSuccess)
      e = cudaMemcpyAsync(d_w, w.data(), sizeof(float) * (nl + 1), cudaMemcpyHostToDevice, h->stream);
    if (e != cudaSuccess) rc = set_err(h, TTI_ERR_CUDA, "MEAL table upload: %s", cudaGetErrorString(e));
    MealConst mc;
    mc.w = d_w;
    mc.logR = logf(Rcoef);
    const float thx = nl * c.dx, thz = nl * c.dz;
    mc.two_thx = 2.0f * thx;
    mc.two_thz = 2.0f * thz;
    mc.dx_fpeak = c.dx * c.fpeak;
    mc.dz_fpeak = c.dz * c.fpeak;
    mc.sqrt3 = sqrtf(3.0f);
    mc.dt = c.dt;
    float **P = h->par;
    SetupIn in{raw[0], raw[1], raw[2], raw[3], raw[4], raw[5], g.Nz};
    SetupOut o{P[TTI_P_D],   P[TTI_P_BETA],  P[TTI_P_COEF1], P[TTI_P_COEF2], P[TTI_P_VP],    P[TTI_P_VS],
               P[TTI_P_RHO], P[TTI_P_INVRHO], P[TTI_P_C11],  P[TTI_P_C13],   P[TTI_P_C15],   P[TTI_P_C33],
               P[TTI_P_C35], P[TTI_P_C55],   P[TTI_P_SIN],   P[TTI_P_COS],   P[TTI_P_SIN_V], P[TTI_P_COS_V],
               P[TTI_P_SIN2], P[TTI_P_COS2], P[TTI_P_SIN_2T]};
    if (rc == TTI_OK) {
      launch_setup(g, in, o, mc, c.variant, c.scalar, c.freesurface, h->stream);
      e = cudaGetLastError();
      if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
      if (e != cudaSuccess) rc = set_err(h, TTI_ERR_CUDA, "setup kernels: %s", cudaGetErrorString(e));
    }
  }
  cudaStreamSynchronize(h->stream);
  // the gradient's chain rule needs epsilon and delta as given (and theta for Bond)
  if (rc == TTI_OK) {
    for (int k = 0; k < (c.variant == TTI_BOND ? 3 : 2); ++k) {
      float *&dst = k == 0 ? h->m_eps : k == 1 ? h->m_delta : h->m_theta;
      if (!dst && pool_alloc(reinterpret_cast<void **>(&dst), g.n * sizeof(float), h->stream) != cudaSuccess) {
        rc = set_err(h, TTI_ERR_NOMEM, "device allocation failed");
        break;
      }
      cudaMemsetAsync(dst, 0, g.n * sizeof(float), h->stream);
      cudaMemcpy2DAsync(dst, (size_t)g.ldz * sizeof(float), raw[3 + k], (size_t)g.Nz * sizeof(float),
                        (size_t)g.Nz * sizeof(float), g.Nx, cudaMemcpyDeviceToDevice, h->stream);
    }
    cudaStreamSynchronize(h->stream);
  }
  pool_free(raw_block, h->stream);
  pool_free(d_w, h->stream);
  if (rc == TTI_OK && h->use_tiled) {
    packed::launch_pack(g, step_args(h).p, packed::Packed{h->pk_cf, h->pk_vsc, h->pk_sc, h->pk_c4}, c.variant,
                       h->stream);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) rc = set_err(h, TTI_ERR_CUDA, "packing parameters: %s", cudaGetErrorString(e));
  }
  if (rc == TTI_OK && h->use_tiled) {
    // the tiled kernels skip coef1/coef2 loads where they are exactly 1 and
    // dt; verify that on the device instead of assuming the MEAL rim geometry
    int *cnt = nullptr;
    int bad = -1;
    if (pool_alloc(reinterpret_cast<void **>(&cnt), sizeof(int), h->stream) == cudaSuccess) {
      cudaMemsetAsync(cnt, 0, sizeof(int), h->stream);
      packed::launch_check_undamped(g, h->par[TTI_P_COEF1], h->par[TTI_P_COEF2], c.dt, c.freesurface ? 0 : g.E, cnt,
                                   h->stream);
      cudaMemcpyAsync(&bad, cnt, sizeof(int), cudaMemcpyDeviceToHost, h->stream);
      pool_free(cnt, h->stream);
      cudaStreamSynchronize(h->stream);
    }
    h->undamped_ok = bad == 0;
  }
  if (rc == TTI_OK) h->have_model = true;
  return rc;
}

int tti_upload_model(tti_handle *h, const float *vp, const float *vs, const float *rho, const float *epsilon,
                     const float *delta, const float *theta)
{
  if (!h) return set_err(h, TTI_ERR_ARG, "null handle");
  const float *src[6] = {vp, vs, rho, epsilon, delta, theta};
  return upload_model(h, src, false);
}

int tti_upload_model_physical(tti_handle *h, const float *vp, const float *vs, const float *rho,
                              const float *epsilon, const float *delta, const float *theta)
{
  if (!h) return set_err(h, TTI_ERR_ARG, "null handle");
  const float *src[6] = {vp, vs, rho, epsilon, delta, theta};
  return upload_model(h, src, true);
}

int tti_fetch_param(tti_handle *h, int which, float *out)
{
  if (!h || !out) return TTI_ERR_ARG;
  if (which < 0 || which >= TTI_P_COUNT || !h->par[which])
    return set_err(h, TTI_ERR_ARG, "parameter %d is not used by this formulation", which);
  if (!h->have_model) return set_err(h, TTI_ERR_STATE, "model not uploaded");
  CK(h, cudaSetDevice(h->device));
  return copy_out_pitched(h, h->par[which], out);
}

int tti_set_source(tti_handle *h, int ntrace, const int *posx, const int *posz, const float *src)
{
  if (!h || ntrace < 0 || (ntrace > 0 && (!posx || !posz || !src))) return set_err(h, TTI_ERR_ARG, "bad source");
  const tti_config &c = h->cfg;
  for (int i = 0; i < ntrace; ++i) {
    if (posz[i] < 0 || posz[i] > c.nz)
      return set_err(h, TTI_ERR_RANGE, "the position of source in 1st dimension (%d) must be between 0 and %d!",
                     posz[i], c.nz);
    if (posx[i] < 0 || posx[i] > c.nx)
      return set_err(h, TTI_ERR_RANGE, "the position of source in 2nd dimension (%d) must be between 0 and %d!",
                     posx[i], c.nx);
  }
  CK(h, cudaSetDevice(h->device));
  pool_free(h->d_sx, h->stream);
  pool_free(h->d_sz, h->stream);
  pool_free(h->d_src, h->stream);
  h->d_sx = h->d_sz = nullptr;
  h->d_src = nullptr;
  h->nsrc = 0;
  if (ntrace == 0) return TTI_OK;
  std::vector<int> x(ntrace), z(ntrace);
  for (int i = 0; i < ntrace; ++i) {
    x[i] = posx[i] + h->g.E;
    z[i] = posz[i] + h->g.E;
  }
  CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_sx), sizeof(int) * ntrace, h->stream));
  CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_sz), sizeof(int) * ntrace, h->stream));
  CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_src), sizeof(float) * (size_t)ntrace * c.nt, h->stream));
  CK(h, cudaMemcpyAsync(h->d_sx, x.data(), sizeof(int) * ntrace, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->d_sz, z.data(), sizeof(int) * ntrace, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemcpyAsync(h->d_src, src, sizeof(float) * (size_t)ntrace * c.nt, cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  h->nsrc = ntrace;
  return TTI_OK;
}

int tti_set_receivers(tti_handle *h, int kind, int ntrace, const int *posx, const int *posz)
{
  if (!h || kind < 0 || kind > 2 || ntrace < 0 || (ntrace > 0 && (!posx || !posz)))
    return set_err(h, TTI_ERR_ARG, "bad receiver arguments");
  const tti_config &c = h->cfg;
  for (int i = 0; i < ntrace; ++i) {
    if (posz[i] < 0 || posz[i] > c.nz)
      return set_err(h, TTI_ERR_RANGE, "the position of receiver in 1st dimension (%d) must be between 0 and %d!",
                     posz[i], c.nz);
    if (posx[i] < 0 || posx[i] > c.nx)
      return set_err(h, TTI_ERR_RANGE, "the position of receiver in 2nd dimension (%d) must be between 0 and %d!",
                     posx[i], c.nx);
  }
  CK(h, cudaSetDevice(h->device));
  // One device block per component holds its receiver rows in the caller's
  // order (d_rz, owner of the block), then, grouped by padded-grid column for
  // the column pass (k_post), the rows (d_rzs), the receiver ids (d_rid) and
  // the column offsets (d_rcol): one copy and one synchronisation per call.
  pool_free(h->d_rz[kind], h->stream);
  pool_free(h->d_rec[kind], h->stream);
  h->d_rz[kind] = h->d_rzs[kind] = h->d_rid[kind] = h->d_rcol[kind] = nullptr;
  h->d_rec[kind] = nullptr;
  h->nrec[kind] = 0;
  if (ntrace == 0) return TTI_OK;
  const int Nx = h->g.Nx;
  std::vector<int> blk(3 * (size_t)ntrace + Nx + 1, 0), x(ntrace), order(ntrace);
  int *z = blk.data(), *zs = z + ntrace, *ids = zs + ntrace, *colptr = ids + ntrace;
  for (int i = 0; i < ntrace; ++i) {
    x[i] = posx[i] + h->g.E;
    z[i] = posz[i] + h->g.E;
  }
  std::iota(order.begin(), order.end(), 0);
  std::stable_sort(order.begin(), order.end(), [&](int a, int b) { return x[a] < x[b]; });
  for (int i = 0; i < ntrace; ++i) colptr[x[i] + 1]++;
  for (int c = 0; c < Nx; ++c) colptr[c + 1] += colptr[c];
  for (int i = 0; i < ntrace; ++i) {
    zs[i] = z[order[i]];
    ids[i] = order[i];
  }
  int *d = nullptr;
  CK(h, pool_alloc(reinterpret_cast<void **>(&d), sizeof(int) * blk.size(), h->stream));
  h->d_rz[kind] = d;
  h->d_rzs[kind] = d + ntrace;
  h->d_rid[kind] = d + 2 * (size_t)ntrace;
  h->d_rcol[kind] = d + 3 * (size_t)ntrace;
  // the traces (ntrace x nts floats, the largest of these) from the handle's pool
  CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_rec[kind]), sizeof(float) * (size_t)ntrace * h->nts, h->stream));
  CK(h, cudaMemcpyAsync(d, blk.data(), sizeof(int) * blk.size(), cudaMemcpyHostToDevice, h->stream));
  CK(h, cudaMemsetAsync(h->d_rec[kind], 0, sizeof(float) * (size_t)ntrace * h->nts, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));  // the host block goes out of scope
  h->nrec[kind] = ntrace;
  return TTI_OK;
}

int tti_reset(tti_handle *h)
{
  if (!h) return TTI_ERR_ARG;
  CK(h, cudaSetDevice(h->device));
  for (auto p : h->fld)
    if (p) CK(h, cudaMemsetAsync(p, 0, h->g.n * sizeof(float), h->stream));
  for (int k = 0; k < 3; ++k)
    if (h->d_rec[k]) CK(h, cudaMemsetAsync(h->d_rec[k], 0, sizeof(float) * (size_t)h->nrec[k] * h->nts, h->stream));
  CK(h, cudaMemsetAsync(h->d_energy, 0, sizeof(double) * 2 * (size_t)h->cfg.nt, h->stream));
  CK(h, cudaMemsetAsync(h->d_flag, 0, sizeof(int), h->stream));
  h->step_index = 0;
  return TTI_OK;
}

int tti_step(tti_handle *h, int nsteps)
{
  if (!h || nsteps < 0) return TTI_ERR_ARG;
  if (!h->have_model) return set_err(h, TTI_ERR_STATE, "model not uploaded");
  if (h->step_index + nsteps > h->cfg.nt) return set_err(h, TTI_ERR_STATE, "step past nt");
  CK(h, cudaSetDevice(h->device));
  SourceTables tab;
  source_tables(h, &tab);
  CK(h, cudaEventRecord(h->ev0, h->stream));
  for (int n = 0; n < nsteps; ++n) {
    int rc = launch_one_step(h, tab);
    if (rc) return rc;
  }
  CK(h, cudaEventRecord(h->ev1, h->stream));
  CK(h, cudaEventSynchronize(h->ev1));
  CK(h, cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  return check_flag(h);
}

int tti_set_snapshot_buffer(tti_handle *h, float *host, size_t floats)
{
  if (!h) return TTI_ERR_ARG;
  if (host) {
    int nzo, nxo, kinds[3];
    snapshot_dims(h, &nzo, &nxo);
    const size_t need = (size_t)snapshot_kinds(h->cfg.wsave, kinds) * nzo * nxo;
    if (need == 0) return set_err(h, TTI_ERR_STATE, "wsave = %d writes no snapshots", h->cfg.wsave);
    if (floats < need)
      return set_err(h, TTI_ERR_ARG, "snapshot buffer of %zu floats, wsave = %d needs %zu", floats, h->cfg.wsave,
                     need);
  }
  h->snap_user = host;
  h->snap_user_pinned = host && is_pinned(host);
  return TTI_OK;
}

int tti_run(tti_handle *h, tti_snapshot_fn snap, void *user)
{
  if (!h) return TTI_ERR_ARG;
  if (!h->have_model) return set_err(h, TTI_ERR_STATE, "model not uploaded");
  int rc = tti_reset(h);
  if (rc) return rc;
  SourceTables tab;
  source_tables(h, &tab);
  rc = run_steps(h, tab, snap, user);
  if (rc) {
    finish_snapshot(h, false);
    return rc;
  }
  if ((rc = finish_snapshot(h, true))) return rc;
  return check_flag(h);
}

int tti_profile_steps(tti_handle *h, int nsteps, float ms[3])
{
  if (!h || !ms || nsteps < 0) return TTI_ERR_ARG;
  if (!h->have_model) return set_err(h, TTI_ERR_STATE, "model not uploaded");
  if (h->step_index + nsteps > h->cfg.nt) return set_err(h, TTI_ERR_STATE, "step past nt");
  CK(h, cudaSetDevice(h->device));
  for (int k = 0; k < 5; ++k)
    if (!h->pev[k]) CK(h, cudaEventCreate(&h->pev[k]));
  SourceTables tab;
  source_tables(h, &tab);
  ms[0] = ms[1] = ms[2] = 0.0f;
  for (int n = 0; n < nsteps; ++n) {
    int rc = launch_one_step(h, tab, h->pev);
    if (rc) return rc;
    CK(h, cudaEventSynchronize(h->pev[4]));
    float t01, t12, t23, t34;
    CK(h, cudaEventElapsedTime(&t01, h->pev[0], h->pev[1]));
    CK(h, cudaEventElapsedTime(&t12, h->pev[1], h->pev[2]));
    CK(h, cudaEventElapsedTime(&t23, h->pev[2], h->pev[3]));
    CK(h, cudaEventElapsedTime(&t34, h->pev[3], h->pev[4]));
    ms[0] += t01;
    ms[1] += t23;
    ms[2] += t12 + t34;
  }
  return check_flag(h);
}

int tti_kernel_launches(const tti_handle *h, long long *n)
{
  if (!h || !n) return TTI_ERR_ARG;
  *n = h->launches;
  return TTI_OK;
}

int tti_get_stream(const tti_handle *h, void **stream)
{
  if (!h || !stream) return TTI_ERR_ARG;
  *stream = static_cast<void *>(h->stream);
  return TTI_OK;
}

int tti_elapsed_ms(const tti_handle *h, float *ms)
{
  if (!h || !ms) return TTI_ERR_ARG;
  *ms = h->last_ms;
  return TTI_OK;
}

int tti_fetch_traces(tti_handle *h, int kind, float *out)
{
  if (!h || !out || kind < 0 || kind > 2) return TTI_ERR_ARG;
  if (!h->d_rec[kind]) return set_err(h, TTI_ERR_ARG, "no receivers of kind %d", kind);
  CK(h, cudaSetDevice(h->device));
  const int n = h->nrec[kind], nts = h->nts;
  // Chunks of receivers transposed on the device (time-major to the caller's
  // [ntrace][nts]) into a staging buffer, then to the caller's block.
  constexpr size_t STAGE = PIN_CHUNK;  // floats per chunk
  if (!h->d_stage) CK(h, pool_alloc(reinterpret_cast<void **>(&h->d_stage), STAGE * sizeof(float), h->stream));
  if ((size_t)nts > STAGE || nts > 65535 * 32)
    return set_err(h, TTI_ERR_ARG, "trace of %d samples is longer than the fetch supports", nts);
  const int per = (int)std::max<size_t>(1, STAGE / (size_t)nts);  // receivers per chunk
  const int nchunk = (n + per - 1) / per;
  if (is_pinned(out)) {
    // page-locked destination: each chunk's copy runs asynchronously, and the
    // next transpose into the staging buffer waits for it in stream order
    for (int r0 = 0; r0 < n; r0 += per) {
      const int nr = std::min(per, n - r0);
      launch_transpose(h->d_rec[kind], h->d_stage, nts, n, r0, nr, h->stream);
      h->launches++;
      CK(h, cudaMemcpyAsync(out + (size_t)r0 * nts, h->d_stage, sizeof(float) * (size_t)nr * nts,
                            cudaMemcpyDeviceToHost, h->stream));
    }
    CK(h, cudaStreamSynchronize(h->stream));
    return TTI_OK;
  }
  // A fetch of one chunk goes straight to the caller's block: staging would
  // not overlap anything, and the first staged fetch of a process pays for
  // page-locking the chunks (about 13 ms for two).
  float *pin[2] = {nullptr, nullptr};
  if (nchunk > 1) {
    pin[0] = pinned_chunk();
    pin[1] = pinned_chunk();
  }
  for (int b = 0; b < 2 && pin[0] && pin[1]; ++b)
    if (!h->pev[5 + b] && cudaEventCreateWithFlags(&h->pev[5 + b], cudaEventDisableTiming) != cudaSuccess)
      pinned_release(pin[b]), pin[b] = nullptr;
  if (pin[0] && pin[1]) {
    // Through two page-locked chunks: the copy of chunk c to the host runs
    // while the host threads copy chunk c - 1 into the caller's block (taking
    // its page faults in parallel).
    cudaError_t e = cudaSuccess;
    for (int c = 0; c <= nchunk && e == cudaSuccess; ++c) {
      if (c < nchunk) {
        const int r0 = c * per, nr = std::min(per, n - r0), b = c & 1;
        launch_transpose(h->d_rec[kind], h->d_stage, nts, n, r0, nr, h->stream);
        h->launches++;
        e = cudaMemcpyAsync(pin[b], h->d_stage, sizeof(float) * (size_t)nr * nts, cudaMemcpyDeviceToHost, h->stream);
        if (e == cudaSuccess) e = cudaEventRecord(h->pev[5 + b], h->stream);
      }
      if (c > 0 && e == cudaSuccess) {
        const int p = c - 1, r0 = p * per, nr = std::min(per, n - r0), b = p & 1;
        e = cudaEventSynchronize(h->pev[5 + b]);
        if (e == cudaSuccess) parallel_copy(out + (size_t)r0 * nts, pin[b], sizeof(float) * (size_t)nr * nts);
      }
    }
    // wait for the stream on the error path too: a device-to-host copy into a
    // chunk may still be in flight, and a released chunk can go to another
    // handle at once
    const cudaError_t es = cudaStreamSynchronize(h->stream);
    if (e == cudaSuccess) e = es;
    pinned_release(pin[0]);
    pinned_release(pin[1]);
    CK(h, e);
    return TTI_OK;
  }
  pinned_release(pin[0]);
  pinned_release(pin[1]);
  // no page-locked memory: straight into the caller's block, its pages
  // faulted in first from several host threads
  prefault(out, sizeof(float) * (size_t)n * nts);
  for (int r0 = 0; r0 < n; r0 += per) {
    const int nr = std::min(per, n - r0);
    launch_transpose(h->d_rec[kind], h->d_stage, nts, n, r0, nr, h->stream);
    h->launches++;
    // pageable destination: returns once the copy is complete, so the next
    // chunk may overwrite the staging buffer
    CK(h, cudaMemcpyAsync(out + (size_t)r0 * nts, h->d_stage, sizeof(float) * (size_t)nr * nts,
                          cudaMemcpyDeviceToHost, h->stream));
  }
  CK(h, cudaStreamSynchronize(h->stream));
  return TTI_OK;
}

int tti_fetch_field(tti_handle *h, int which, float *out)
{
  if (!h || !out || which < 0 || which >= 8) return TTI_ERR_ARG;
  if (!h->fld[which]) return set_err(h, TTI_ERR_ARG, "field %d is not used by this formulation", which);
  CK(h, cudaSetDevice(h->device));
  return copy_out_pitched(h, h->fld[which], out);
}

int tti_fetch_energy(tti_handle *h, float *ek, float *ep)
{
  if (!h || !ek || !ep) return TTI_ERR_ARG;
  CK(h, cudaSetDevice(h->device));
  const int nt = h->cfg.nt;
  std::vector<double> e(2 * (size_t)nt);
  CK(h, cudaMemcpyAsync(e.data(), h->d_energy, sizeof(double) * e.size(), cudaMemcpyDeviceToHost, h->stream));
  CK(h, cudaStreamSynchronize(h->stream));
  for (int it = 0; it < nt; ++it) {
    ek[it] = 0.5f * (float)e[2 * (size_t)it] * h->cfg.dx * h->cfg.dz;
    ep[it] = 0.5f * (float)e[2 * (size_t)it + 1] * h->cfg.dx * h->cfg.dz;
  }
  return TTI_OK;
}

}  // extern "C"
