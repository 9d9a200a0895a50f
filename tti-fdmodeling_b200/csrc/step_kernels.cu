// Per-step kernels of the RSG time loop: velocity and stress updates along
// the two grid diagonals, free surface, sources, receivers, energy, snapshot
// packing.
#include <algorithm>

#include "launch.cuh"

namespace ttifd {

namespace {

// Velocity node (ix+1/2, iz+1/2) from a stress field, coord:621-630:
//   d1 = sum_k C_k (a[x+k][z+k]   - a[x-k+1][z-k+1])
//   d2 = sum_k C_k (a[x+k][z-k+1] - a[x-k+1][z+k])
template <bool X>
__device__ __forceinline__ void diag_v(const float *__restrict__ q, int L, float &d1, float &d2)
{
  using A = Ar<X>;
  float s1 = A::mul(rsg(0), A::sub(__ldg(q + L + 1), __ldg(q)));
  float s2 = A::mul(rsg(0), A::sub(__ldg(q + L), __ldg(q + 1)));
#pragma unroll
  for (int k = 2; k <= NH; ++k) {
    s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(__ldg(q + k * (L + 1)), __ldg(q - (k - 1) * (L + 1)))));
    s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(__ldg(q + k * L - (k - 1)), __ldg(q - (k - 1) * L + k))));
  }
  d1 = s1;
  d2 = s2;
}

// Stress node (ix, iz) from a velocity field, coord:811-816:
//   d1 = sum_k C_k (a[x+k-1][z+k-1] - a[x-k][z-k])
//   d2 = sum_k C_k (a[x+k-1][z-k]   - a[x-k][z+k-1])
template <bool X>
__device__ __forceinline__ void diag_s(const float *__restrict__ q, int L, float &d1, float &d2)
{
  using A = Ar<X>;
  float s1 = A::mul(rsg(0), A::sub(__ldg(q), __ldg(q - L - 1)));
  float s2 = A::mul(rsg(0), A::sub(__ldg(q - 1), __ldg(q - L)));
#pragma unroll
  for (int k = 2; k <= NH; ++k) {
    s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(__ldg(q + (k - 1) * (L + 1)), __ldg(q - k * (L + 1)))));
    s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(__ldg(q + (k - 1) * L - k), __ldg(q - k * L + (k - 1)))));
  }
  d1 = s1;
  d2 = s2;
}

constexpr int BZ = 32, BX = 8;

// coord:614-672, tensor:617-666, bond:654-703
template <int V, bool X>
__global__ void __launch_bounds__(BZ *BX) k_velocity(Grid g, Fields f, Params p, float invdx, float invdz)
{
  using A = Ar<X>;
  const int iz = g.izStart + blockIdx.x * BZ + threadIdx.x;
  const int ix = NH + blockIdx.y * BX + threadIdx.y;
  if (iz >= g.Nz - NH || ix >= g.Nx - NH) return;
  const int L = g.ldz;
  const size_t i = (size_t)ix * L + iz;
  float d1, d2;
  diag_v<X>(f.sxx + i, L, d1, d2);
  const float sxx_x = A::mul(A::mul(0.5f, A::add(d1, d2)), invdx);
  const float sxx_z = A::mul(A::mul(0.5f, A::sub(d1, d2)), invdx);  // invdx as in coord:633
  diag_v<X>(f.szz + i, L, d1, d2);
  const float szz_x = A::mul(A::mul(0.5f, A::add(d1, d2)), invdx);
  const float szz_z = A::mul(A::mul(0.5f, A::sub(d1, d2)), invdz);
  diag_v<X>(f.sxz + i, L, d1, d2);
  const float sxz_x = A::mul(A::mul(0.5f, A::add(d1, d2)), invdx);
  const float sxz_z = A::mul(A::mul(0.5f, A::sub(d1, d2)), invdz);
  const float a = p.coef1[i], br = A::mul(p.coef2[i], p.invrho[i]);
  float fx, fz;
  if (V == TTI_COORDINATE) {
    const float cv = p.csv[i], sv = p.snv[i];
    fx = A::add(A::add(A::sub(A::mul(cv, sxx_x), A::mul(sv, sxx_z)), A::mul(sv, sxz_x)), A::mul(cv, sxz_z));
    fz = A::add(A::add(A::sub(A::mul(cv, sxz_x), A::mul(sv, sxz_z)), A::mul(sv, szz_x)), A::mul(cv, szz_z));
  } else {
    fx = A::add(sxx_x, sxz_z);
    fz = A::add(sxz_x, szz_z);
  }
  f.vx[i] = A::add(A::mul(a, f.vx[i]), A::mul(br, fx));
  f.vz[i] = A::add(A::mul(a, f.vz[i]), A::mul(br, fz));
}

// coord:804-845, tensor:799-851 (tau update and sigma = R tau fused: the
// sigma pass reads only the same cell's tau), bond:836-873
template <int V, bool X>
__global__ void __launch_bounds__(BZ *BX) k_stress(Grid g, Fields f, Params p, float invdx, float invdz)
{
  using A = Ar<X>;
  const int iz = g.izStart + blockIdx.x * BZ + threadIdx.x;
  const int ix = NH + blockIdx.y * BX + threadIdx.y;
  if (iz >= g.Nz - NH || ix >= g.Nx - NH) return;
  const int L = g.ldz;
  const size_t i = (size_t)ix * L + iz;
  float d1, d2;
  diag_s<X>(f.vx + i, L, d1, d2);
  float vxx = A::mul(A::mul(0.5f, A::add(d1, d2)), invdx);
  float vxz = A::mul(A::mul(0.5f, A::sub(d1, d2)), invdz);
  diag_s<X>(f.vz + i, L, d1, d2);
  float vzx = A::mul(A::mul(0.5f, A::add(d1, d2)), invdx);
  float vzz = A::mul(A::mul(0.5f, A::sub(d1, d2)), invdz);
  const float a = p.coef1[i], b = p.coef2[i];
  const float c11 = p.c11[i], c13 = p.c13[i], c33 = p.c33[i], c55 = p.c55[i];
  if (V == TTI_COORDINATE) {
    const float s = p.sn[i], c = p.cs[i];
    float r = A::add(A::mul(s, vxx), A::mul(c, vxz));
    vxx = A::sub(A::mul(c, vxx), A::mul(s, vxz));
    vxz = r;
    r = A::add(A::mul(s, vzx), A::mul(c, vzz));
    vzx = A::sub(A::mul(c, vzx), A::mul(s, vzz));
    vzz = r;
    f.sxx[i] = A::add(A::mul(a, f.sxx[i]), A::mul(b, A::add(A::mul(c11, vxx), A::mul(c13, vzz))));
    f.szz[i] = A::add(A::mul(a, f.szz[i]), A::mul(b, A::add(A::mul(c13, vxx), A::mul(c33, vzz))));
    f.sxz[i] = A::add(A::mul(a, f.sxz[i]), A::mul(A::mul(b, c55), A::add(vzx, vxz)));
  } else if (V == TTI_TENSOR) {
    const float s2 = p.s2[i], c2 = p.c2[i], st = p.s2t[i];
    const float sh = A::add(vxz, vzx);
    const float exx = A::sub(A::add(A::mul(c2, vxx), A::mul(s2, vzz)), A::mul(A::mul(0.5f, st), sh));
    const float ezz = A::add(A::add(A::mul(s2, vxx), A::mul(c2, vzz)), A::mul(A::mul(0.5f, st), sh));
    const float exz = A::add(A::mul(st, A::sub(vxx, vzz)), A::mul(A::sub(c2, s2), sh));
    const float txx = A::add(A::mul(a, f.txx[i]), A::mul(b, A::add(A::mul(c11, exx), A::mul(c13, ezz))));
    const float tzz = A::add(A::mul(a, f.tzz[i]), A::mul(b, A::add(A::mul(c13, exx), A::mul(c33, ezz))));
    const float txz = A::add(A::mul(a, f.txz[i]), A::mul(A::mul(b, c55), exz));
    f.txx[i] = txx;
    f.tzz[i] = tzz;
    f.txz[i] = txz;
    f.sxx[i] = A::add(A::add(A::mul(c2, txx), A::mul(s2, tzz)), A::mul(st, txz));
    f.szz[i] = A::sub(A::add(A::mul(s2, txx), A::mul(c2, tzz)), A::mul(st, txz));
    f.sxz[i] = A::add(A::mul(A::mul(-0.5f, st), A::sub(txx, tzz)), A::mul(A::sub(c2, s2), txz));
  } else {
    const float c15 = p.c15[i], c35 = p.c35[i];
    const float sh = A::add(vzx, vxz);
    f.sxx[i] = A::add(A::mul(a, f.sxx[i]),
                      A::mul(b, A::add(A::add(A::mul(c11, vxx), A::mul(c13, vzz)), A::mul(c15, sh))));
    f.szz[i] = A::add(A::mul(a, f.szz[i]),
                      A::mul(b, A::add(A::add(A::mul(c13, vxx), A::mul(c33, vzz)), A::mul(c35, sh))));
    f.sxz[i] = A::add(A::mul(a, f.sxz[i]),
                      A::mul(b, A::add(A::add(A::mul(c15, vxx), A::mul(c35, vzz)), A::mul(c55, sh))));
  }
}

// coord:847-863: stress image about row s = izStart
__global__ void k_free_surface(Grid g, Fields f)
{
  const int ix = NH + blockIdx.x * blockDim.x + threadIdx.x;
  if (ix >= g.Nx - NH) return;
  const size_t c = (size_t)ix * g.ldz + g.izStart;
  f.sxz[c] = 0.0f;
  f.szz[c] = 0.0f;
  const float sxx0 = f.sxx[c];
#pragma unroll
  for (int k = 1; k <= NH; ++k) {
    f.sxx[c - k] = __fsub_rn(__fmul_rn(2.0f, sxx0), f.sxx[c + k]);
    f.szz[c - k] = -f.szz[c + k];
    f.sxz[c - k] = -f.sxz[c + k];
  }
}

__device__ __forceinline__ void acc(float *p, float k, float a) { *p = __fadd_rn(*p, __fmul_rn(k, a)); }
__device__ __forceinline__ void dec(float *p, float k, float a) { *p = __fsub_rn(*p, __fmul_rn(k, a)); }

// Sources over their 11 x 11 windows, one thread per window cell. Sources are
// applied one after another (a barrier between them) so overlapping windows
// accumulate in the reference's order; stype 8 runs on one thread.
__device__ void sources_block(const Grid &g, const Fields &f, const SourceSet &s, const SourceTables &t, int variant,
                              int stype, int stage, int it)
{
  const int tid = threadIdx.x;
  if (stage == 0 && stype == 8) {
    if (tid != 0) return;
    for (int n = 0; n < s.n; ++n) {
      const size_t c = (size_t)s.x[n] * g.ldz + s.z[n];
      const float a = s.w[(size_t)n * s.nt + it];
      const size_t L = g.ldz;
      dec(f.vx + c, t.q8, a);
      acc(f.vz + c, t.q8, a);
      dec(f.vx + c - L, t.q8, a);
      dec(f.vz + c - L, t.q8, a);
      acc(f.vx + c - L - 1, t.q8, a);
      dec(f.vz + c - L - 1, t.q8, a);
      acc(f.vx + c - 1, t.q8, a);
      acc(f.vz + c - 1, t.q8, a);
    }
    return;
  }
  int passes[2], np = 0;
  if (stage == 0) {
    if (stype == 2 || stype == 4) passes[np++] = 2;
    if (stype == 3 || stype == 4) passes[np++] = 3;
    if (stype >= 5 && stype <= 7) passes[np++] = stype;
  } else if (stype == 1) {
    passes[np++] = 1;
  }
  const int oa = tid / 11, ob = tid % 11;
  for (int pidx = 0; pidx < np; ++pidx) {
    const int kind = passes[pidx];
    for (int n = 0; n < s.n; ++n) {
      if (tid < 121) {
        const int ix = s.x[n] + oa - NH, iz = s.z[n] + ob - NH;
        if (ix >= 0 && ix < g.Nx && iz >= 0 && iz < g.Nz) {
          const size_t c = (size_t)ix * g.ldz + iz;
          const float a = s.w[(size_t)n * s.nt + it];
          switch (kind) {
          case 1:
            acc(f.sxx + c, t.k1[tid], a);
            acc(f.szz + c, t.k1[tid], a);
            if (variant == TTI_TENSOR) {
              acc(f.txx + c, t.k1[tid], a);
              acc(f.tzz + c, t.k1[tid], a);
            }
            break;
          case 2:
            acc(f.vx + c, t.kx[tid], a);
            acc(f.vz + c, t.kz[tid], a);
            break;
          case 3:
            dec(f.vx + c, t.kz[tid], a);
            acc(f.vz + c, t.kx[tid], a);
            break;
          case 5:
            acc(f.vx + c, t.k5[tid], a);
            break;
          case 6:
            acc(f.vz + c, t.k5[tid], a);
            break;
          case 7:
            acc(f.vx + c, t.k7[tid], a);
            acc(f.vz + c, t.k7[tid], a);
            break;
          }
        }
      }
      __syncthreads();
    }
  }
}

__global__ void k_sources(Grid g, Fields f, SourceSet s, SourceTables t, int variant, int stype, int stage, int it)
{
  sources_block(g, f, s, t, variant, stype, stage, it);
}

// Batched velocity sources: one block per instance, time index from the step counter.
__global__ void k_sources_batch(const BatchSrc *bs, const int *step)
{
  const BatchSrc &b = bs[blockIdx.x];
  const int n = *step;
  if (n >= b.nt || b.s.n == 0) return;
  sources_block(b.g, b.f, b.s, *b.tab, b.variant, b.stype, 0, b.mode2 ? b.nt - 1 - n : n);
}

__global__ void k_advance(int *step) { ++*step; }

// isoelastic.c:103-144; recorded time-major on the device ([irec][trace]).
__global__ void k_receivers(Grid g, Fields f, ReceiverSet r, int want_v, int want_p, int irec, int *flag)
{
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const int k = blockIdx.y;
  if (t >= r.n[k]) return;
  if ((k < 2 && !want_v) || (k == 2 && !want_p)) return;
  const size_t c = (size_t)r.x[k][t] * g.ldz + r.z[k][t];
  float v;
  if (k == TTI_REC_VX) v = f.vx[c];
  else if (k == TTI_REC_VZ) v = f.vz[c];
  else v = __fmul_rn(0.5f, __fadd_rn(f.sxx[c], f.szz[c]));
  r.rec[k][(size_t)irec * r.n[k] + t] = v;
  if (!isfinite(v)) atomicOr(flag, 1);
}

// coord:898-924, accumulated in double per step
__global__ void k_energy(Grid g, Fields f, Params p, int nz, int nx, double *out2)
{
  double ek = 0.0, ep = 0.0;
  const size_t n = (size_t)nz * nx;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const int ix = (int)(q / nz) + g.E, iz = (int)(q % nz) + g.E;
    const size_t i = (size_t)ix * g.ldz + iz;
    const float r = p.invrho[i], c11 = p.c11[i], c55 = p.c55[i];
    const float vx = f.vx[i], vz = f.vz[i], sx = f.sxx[i], sz = f.szz[i], sq = f.sxz[i];
    ek += (double)(__fdiv_rn(__fmul_rn(vx, vx), r) + __fdiv_rn(__fmul_rn(vz, vz), r));
    const float c1 = __fadd_rn(c11, __fmul_rn(2.0f, c55));
    const float num = __fadd_rn(__fmul_rn(__fsub_rn(__fmul_rn(c1, sx), __fmul_rn(c11, sz)), sx),
                                __fmul_rn(__fsub_rn(__fmul_rn(c11, sx), __fmul_rn(c1, sz)), sz));
    ep += (double)(__fdiv_rn(__fmul_rn(0.25f, num), __fmul_rn(c55, __fadd_rn(c11, c55))) +
                   __fdiv_rn(__fmul_rn(sq, sq), c55));
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    ek += __shfl_down_sync(0xffffffffu, ek, o);
    ep += __shfl_down_sync(0xffffffffu, ep, o);
  }
  if ((threadIdx.x & 31) == 0) {
    atomicAdd(out2, ek);
    atomicAdd(out2 + 1, ep);
  }
}

// After the stress update, one warp per padded-grid column applies, in the
// reference's order for that column: the free-surface image (coord:847-863;
// lanes 1-5 take the mirrored rows), the stress source stype 1 of each source
// in turn (coord:865-886, tensor:871-895 also adds to tau; lanes over the 11
// rows of the window), and the receiver samples (isoelastic.c:103-144; lanes
// over the column's receivers). Columns do not interact, so one launch
// replaces three; the warp makes each phase one memory round trip.
// PDL: the warp reads the column's receiver geometry (static since the
// receivers were set) before waiting for the previous kernel, so those loads
// overlap its tail.
__device__ void post_column(const Grid &g, const Fields &f, const PostArgs &p, int ix, int it, int irec,
                            bool pdl = false)
{
  const int lane = threadIdx.x & 31;
  const size_t col = (size_t)ix * g.ldz;
  // the first 32 receivers of each component in this column, one per lane
  int rb[3] = {0, 0, 0}, re[3] = {0, 0, 0}, rzl[3] = {0, 0, 0}, ridl[3] = {0, 0, 0};
  if (irec >= 0) {
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (p.colptr[k]) {
        rb[k] = p.colptr[k][ix];
        re[k] = p.colptr[k][ix + 1];
      }
#pragma unroll
    for (int k = 0; k < 3; ++k)
      if (rb[k] + lane < re[k]) {
        rzl[k] = p.rz[k][rb[k] + lane];
        ridl[k] = p.rid[k][rb[k] + lane];
      }
  }
  if (pdl) pdl_sync();
  if (p.freesurface && ix >= NH && ix < g.Nx - NH) {
    const size_t c = col + g.izStart;
    const float sxx0 = f.sxx[c];
    float xx = 0.0f, zz = 0.0f, xz = 0.0f;
    if (lane >= 1 && lane <= NH) {
      xx = f.sxx[c + lane];
      zz = f.szz[c + lane];
      xz = f.sxz[c + lane];
    }
    __syncwarp();
    if (lane >= 1 && lane <= NH) {
      f.sxx[c - lane] = __fsub_rn(__fmul_rn(2.0f, sxx0), xx);
      f.szz[c - lane] = -zz;
      f.sxz[c - lane] = -xz;
    } else if (lane == 0) {
      f.sxz[c] = 0.0f;
      f.szz[c] = 0.0f;
    }
    __syncwarp();
  }
  if (p.stype == 1) {
    for (int n = 0; n < p.src.n; ++n) {
      const int dx = ix - p.src.x[n];
      if (dx < -NH || dx > NH) continue;
      const int iz = p.src.z[n] + lane - NH;
      if (lane <= 2 * NH && iz >= 0 && iz < g.Nz) {
        const float a = p.src.w[(size_t)n * p.src.nt + it];
        const float ws = __fmul_rn(p.k1[(dx + NH) * 11 + lane], a);
        const size_t c = col + iz;
        f.sxx[c] = __fadd_rn(f.sxx[c], ws);
        f.szz[c] = __fadd_rn(f.szz[c], ws);
        if (p.tensor) {
          f.txx[c] = __fadd_rn(f.txx[c], ws);
          f.tzz[c] = __fadd_rn(f.tzz[c], ws);
        }
      }
      __syncwarp();
    }
  }
  if (irec >= 0) {
    // all three components' samples loaded before any is stored
    float v[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (rb[k] + lane >= re[k]) continue;
      const size_t c = col + rzl[k];
      if (k == TTI_REC_VX) v[k] = f.vx[c];
      else if (k == TTI_REC_VZ) v[k] = f.vz[c];
      else v[k] = __fmul_rn(0.5f, __fadd_rn(f.sxx[c], f.szz[c]));
    }
#pragma unroll
    for (int k = 0; k < 3; ++k) {
      if (rb[k] + lane >= re[k]) continue;
      p.rec[k][(size_t)irec * p.nrec[k] + ridl[k]] = v[k];
      if (!isfinite(v[k])) atomicOr(p.flag, 1);
    }
    // columns with more than 32 receivers of a component
    for (int k = 0; k < 3; ++k)
      for (int j = rb[k] + 32 + lane; j < re[k]; j += 32) {
        const size_t c = col + p.rz[k][j];
        float w;
        if (k == TTI_REC_VX) w = f.vx[c];
        else if (k == TTI_REC_VZ) w = f.vz[c];
        else w = __fmul_rn(0.5f, __fadd_rn(f.sxx[c], f.szz[c]));
        p.rec[k][(size_t)irec * p.nrec[k] + p.rid[k][j]] = w;
        if (!isfinite(w)) atomicOr(p.flag, 1);
      }
  }
}

__global__ void k_post(Grid g, Fields f, PostArgs p)
{
  const int ix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ix >= g.Nx) {
    pdl_sync();
    return;
  }
  post_column(g, f, p, ix, p.it, p.irec, true);
}

// Batched: blockIdx.y = instance; time index and receiver slot from the step counter.
__global__ void k_post_batch(const BatchPost *bp, const int *step)
{
  const BatchPost &b = bp[blockIdx.y];
  const int n = *step;
  if (n >= b.nt) return;
  const int it = b.mode2 ? b.nt - 1 - n : n;
  const int irec = b.rec_on && it % b.mt == 0 ? it / b.mt : -1;
  if (!b.p.freesurface && b.p.stype != 1 && irec < 0) return;
  const int ix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ix >= b.g.Nx) return;
  post_column(b.g, b.f, b.p, ix, it, irec);
}

__global__ void k_snapshot(Grid g, Fields f, int kind, int x0, int z0, int nzo, int nxo, float *dst)
{
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = blockIdx.y;
  if (iz >= nzo || ix >= nxo) return;
  const size_t c = (size_t)(ix + x0) * g.ldz + (iz + z0);
  float v;
  if (kind == 3) v = __fmul_rn(0.5f, __fadd_rn(f.sxx[c], f.szz[c]));
  else if (kind == 1 || kind == 4 || kind == 6) v = f.vx[c];
  else v = f.vz[c];
  dst[(size_t)ix * nzo + iz] = v;
}

}  // namespace

static dim3 interior_grid(const Grid &g)
{
  const int nz = g.Nz - NH - g.izStart, nx = g.Nx - 2 * NH;
  return dim3((nz + BZ - 1) / BZ, (nx + BX - 1) / BX);
}

#define TTI_DISPATCH(KERNEL, a, st)                                                                        \
  do {                                                                                                     \
    const dim3 grd = interior_grid(a.g), blk(BZ, BX);                                                       \
    if (grd.x == 0 || grd.y == 0) break;                                                                   \
    if (a.exact) {                                                                                         \
      if (a.variant == TTI_COORDINATE) KERNEL<TTI_COORDINATE, true><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz); \
      else if (a.variant == TTI_TENSOR) KERNEL<TTI_TENSOR, true><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz); \
      else KERNEL<TTI_BOND, true><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz);                     \
    } else {                                                                                               \
      if (a.variant == TTI_COORDINATE) KERNEL<TTI_COORDINATE, false><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz); \
      else if (a.variant == TTI_TENSOR) KERNEL<TTI_TENSOR, false><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz); \
      else KERNEL<TTI_BOND, false><<<grd, blk, 0, st>>>(a.g, a.f, a.p, a.invdx, a.invdz);                    \
    }                                                                                                      \
  } while (0)

void launch_velocity(const StepArgs &a, cudaStream_t st) { TTI_DISPATCH(k_velocity, a, st); }
void launch_stress(const StepArgs &a, cudaStream_t st) { TTI_DISPATCH(k_stress, a, st); }

void launch_free_surface(const StepArgs &a, cudaStream_t st)
{
  const int n = a.g.Nx - 2 * NH;
  if (n <= 0) return;
  k_free_surface<<<(n + 127) / 128, 128, 0, st>>>(a.g, a.f);
}

void launch_sources(const StepArgs &a, const SourceSet &s, const SourceTables *tab, int stype, int stage, int it,
                    cudaStream_t st)
{
  if (s.n <= 0) return;
  if (stage == 0 && (stype < 2 || stype > 8)) return;
  if (stage == 1 && stype != 1) return;
  k_sources<<<1, 128, 0, st>>>(a.g, a.f, s, *tab, a.variant, stype, stage, it);
}

void launch_receivers(const StepArgs &a, const ReceiverSet &r, int seistype, int irec, int *flag, cudaStream_t st)
{
  const int want_v = seistype == 1 || seistype == 3, want_p = seistype == 2 || seistype == 3;
  int nmax = 0;
  for (int k = 0; k < 3; ++k) nmax = r.n[k] > nmax ? r.n[k] : nmax;
  if (nmax == 0) return;
  k_receivers<<<dim3((nmax + 127) / 128, 3), 128, 0, st>>>(a.g, a.f, r, want_v, want_p, irec, flag);
}

void launch_energy(const StepArgs &a, int nz, int nx, double *out2, cudaStream_t st)
{
  k_energy<<<296, 256, 0, st>>>(a.g, a.f, a.p, nz, nx, out2);
}

void launch_post(const StepArgs &a, const PostArgs &p, cudaStream_t st)
{
  launch_pdl(k_post, dim3((a.g.Nx + 3) / 4), dim3(128), 0, st, a.g, a.f, p);  // 4 columns (warps) per block
}

void launch_post_batch(const BatchPost *d, int n, int maxNx, const int *step, cudaStream_t st)
{
  if (n > 0) k_post_batch<<<dim3((maxNx + 3) / 4, n), 128, 0, st>>>(d, step);
}

void launch_sources_batch(const BatchSrc *d, int n, const int *step, cudaStream_t st)
{
  if (n > 0) k_sources_batch<<<n, 128, 0, st>>>(d, step);
}

// up to five state arrays copied in one launch (the gradient's kept states)
struct Copy5 {
  const float4 *src[5];
  float4 *dst[5];
  int nf;
};
__global__ void k_copy5(Copy5 c, size_t n4)
{
  pdl_sync();
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n4; q += (size_t)gridDim.x * blockDim.x) {
#pragma unroll
    for (int f = 0; f < 5; ++f)
      if (f < c.nf) c.dst[f][q] = c.src[f][q];
  }
}

void launch_copy5(float *const *src, float *const *dst, int nf, size_t n, cudaStream_t st)
{
  Copy5 c;
  c.nf = std::min(nf, 5);
  for (int f = 0; f < 5; ++f) {
    c.src[f] = f < c.nf ? reinterpret_cast<const float4 *>(src[f]) : nullptr;
    c.dst[f] = f < c.nf ? reinterpret_cast<float4 *>(dst[f]) : nullptr;
  }
  const size_t n4 = n / 4;
  launch_pdl(k_copy5, dim3((unsigned)std::min<size_t>((n4 + 255) / 256, 148 * 16)), dim3(256), 0, st, c, n4);
}

// Receivers r0 .. r0 + nr - 1 of the time-major [nts][n] block, transposed to
// [nr][nts] (the Receiver2D.recv layout), through 32 x 32 shared tiles.
__global__ void k_transpose(const float *in, float *out, int nts, int n, int r0, int nr)
{
  __shared__ float t[32][33];
  const int ra = blockIdx.x * 32, t0 = blockIdx.y * 32;
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int tt = t0 + k, r = ra + threadIdx.x;
    if (tt < nts && r < nr) t[k][threadIdx.x] = in[(size_t)tt * n + r0 + r];
  }
  __syncthreads();
  for (int k = threadIdx.y; k < 32; k += blockDim.y) {
    const int r = ra + k, tt = t0 + threadIdx.x;
    if (tt < nts && r < nr) out[(size_t)r * nts + tt] = t[threadIdx.x][k];
  }
}

void launch_transpose(const float *in, float *out, int nts, int n, int r0, int nr, cudaStream_t st)
{
  k_transpose<<<dim3((nr + 31) / 32, (nts + 31) / 32), dim3(32, 8), 0, st>>>(in, out, nts, n, r0, nr);
}

void launch_advance(int *step, cudaStream_t st) { k_advance<<<1, 1, 0, st>>>(step); }

void launch_snapshot(const StepArgs &a, int kind, int savew, float *dst, cudaStream_t st)
{
  const Grid &g = a.g;
  const int x0 = savew == 0 ? g.E : 0, z0 = savew == 0 ? g.E : 0;
  const int nxo = savew == 0 ? g.Nx - 2 * g.E : g.Nx, nzo = savew == 0 ? g.Nz - 2 * g.E : g.Nz;
  k_snapshot<<<dim3((nzo + 127) / 128, nxo), 128, 0, st>>>(g, a.f, kind, x0, z0, nzo, nxo, dst);
}

}  // namespace ttifd
