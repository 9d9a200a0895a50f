// Adjoint-state gradient (tti_grad_*) of the three formulations, stated
// here for the coordinate rotation (the tensor and Bond branches differ in
// the stress-half adjoint and the chain rule only).
//
// Misfit J = 1/2 sum over the recorded samples of (d - dobs)^2. The forward
// step (coord:611-926) is, per time step n:
//   v'  = coef1 v + coef2 invrho R(theta_v) D_sigma sigma      velocity half (:614-672)
//         + velocity sources, stype 2-8 (:674-802)
//   s'  = coef1 s + coef2 H(c11, c13, c33, c55, theta) D_v v'   stress half (:804-845)
//   s'' = P_fs s' (free surface, :847-863), + stress source, record (isoelastic.c:103-144)
// Its discrete adjoint, run backwards from n = nt-1, is per step:
//   inject the residual at the receivers; P_fs^T; stress-half adjoint
//   (gradient terms of c11..c55 and theta at the stress node, then the
//   transposed stress stencils, which are minus the velocity-node stencils,
//   into lambda_v); velocity-half adjoint (gradient terms of sin/cos theta_v,
//   then the transposed velocity stencils, minus the stress-node stencils,
//   into lambda_sigma). Each adjoint step needs the forward v after the
//   velocity half and sigma before the stress half of the same step: the loop
//   is cut into ncheck segments; the first pass saves the full state at the
//   start of each segment but the last and keeps the last segment's states,
//   and the reverse pass recomputes each earlier segment from its checkpoint
//   (ncheck = 1 keeps every state and recomputes nothing).
// The chain rule maps the stiffness and angle sums to vp, epsilon, delta and
// theta (degrees) with vs and rho fixed and MEAL coef1, coef2, Beta frozen:
// c11 = rho' vp'^2 (1 + 2 eps), c13 = rho' (vp'^2 sqrt(f (f + 2 delta)) - vs'^2),
// c33 = rho' vp'^2, f = 1 - (vs'/vp')^2, vp' = vp / Beta (coord:497-515,
// meal.c:450-490).
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "tiled.cuh"

using namespace ttifd;

struct GradState {
  int ncheck = 0, seg = 0;  // checkpoints, steps per segment
  float *lam[8] = {};       // adjoint vx vz sxx szz sxz (+ txx tzz txz: tensor rotation)
  float *T[4] = {};         // stress-half adjoint strain terms (read by the transposed stress stencils)
  float *TV[6] = {};        // velocity-half adjoint derivative terms (read by the transposed velocity stencils)
  float *acc[7] = {};       // sums. coordinate: c11 c13 c33 (c55 kept zero) theta(stress node) sin_v cos_v;
                            // Bond: c11 c13 c33 c55 c15 c35 (the rotated moduli)
  float *out[4] = {};       // vp eps delta theta
  float *ckpt = nullptr;    // (ncheck - 1) x the formulation's fields (5, tensor 8)
  float *keep = nullptr;    // seg x nkeep fields per kept step (keep_fields: v, then P Q R S, sigma or tau)
  int nkeep = 0;
  float *obs[3] = {};       // observed traces, time-major [nts][ntrace]
  float *res[3] = {};       // residuals, time-major
  float *gsrc = nullptr;    // [nsrc][nt]
  int gsrc_n = 0;
  double *d_J = nullptr;
  bool have_obs[3] = {};
  CUtensorMap *maps = nullptr;  // host copies, 64-byte aligned: T0..T3, TV0..TV5
  // velocity sources (stype 2-8): per source vm cells (ix, iz, index in the
  // rim list or -1; ix < 0: off the grid) with weights (wx, wz),
  // v[cell] += w src(t); the cells of all windows outside the velocity update,
  // each once, with their accumulated transposed stencils (x, z) in double
  int4 *vcell = nullptr;
  float2 *vw = nullptr;
  int2 *vrim = nullptr;
  double *vrim_acc = nullptr;
  int vm = 0, vrim_n = 0;
  int surf_zorg = -1;  // row origin of the stress-half adjoint that folds in the column work; -1: a separate launch
  int surf_zend = 0;   // rows at or below this hold no column work
};

namespace {

constexpr int BZ = 32, BX = 8;

struct AdjArgs {
  Grid g;
  Params p;
  packed::Packed pk;  // packed parameters (null on the per-cell path)
  float *lam[8];
  float *T[4];
  float *TV[6];
  float *acc[7];
  const float *keep[8];  // this step's kept fields (keep_fields), null past them
  float hx, hz, dt;
  int z_lo;         // first row of the transposed velocity stencils
  int undamped_ok;  // coef1 == 1, coef2 == dt on [E, Nx - E) x [und_z0, Nz - E) (checked at upload)
  int und_z0;
};

__device__ __forceinline__ bool cell_undamped(const AdjArgs &a, int ix, int iz)
{
  const Grid &g = a.g;
  return a.undamped_ok && ix >= g.E && ix < g.Nx - g.E && iz >= a.und_z0 && iz < g.Nz - g.E;
}

// Stress-node parameters of one cell: coef1, coef2 (the constants 1 and dt in
// the undamped interior), c11 c13 c33 c55, and the formulation's pair
// (coordinate: sin, cos theta; tensor: sin^2, cos^2; Bond: c15, c35), from the
// packed arrays (PK) or the plain ones.
struct SParams {
  float c1, b, c11, c13, c33, c55, p, q;
};
template <bool PK, int V>
__device__ __forceinline__ SParams stress_params(const AdjArgs &a, size_t i, bool und)
{
  SParams s;
  if (und) {
    s.c1 = 1.0f;
    s.b = a.dt;
  } else if (PK) {
    const float2 cf = __ldg(a.pk.cf + i);
    s.c1 = cf.x;
    s.b = cf.y;
  } else {
    s.c1 = a.p.coef1[i];
    s.b = a.p.coef2[i];
  }
  if (PK) {
    const float4 c4 = __ldg(a.pk.c4 + i);
    const float2 sc = __ldg(a.pk.sc + i);
    s.c11 = c4.x;
    s.c13 = c4.y;
    s.c33 = c4.z;
    s.c55 = c4.w;
    s.p = sc.x;
    s.q = sc.y;
  } else {
    s.c11 = a.p.c11[i];
    s.c13 = a.p.c13[i];
    s.c33 = a.p.c33[i];
    s.c55 = a.p.c55[i];
    s.p = V == TTI_BOND ? a.p.c15[i] : V == TTI_TENSOR ? a.p.s2[i] : a.p.sn[i];
    s.q = V == TTI_BOND ? a.p.c35[i] : V == TTI_TENSOR ? a.p.c2[i] : a.p.cs[i];
  }
  return s;
}

__device__ __forceinline__ void pair_v(const float *a, size_t L, int ix, int iz, float &d1, float &d2)
{
  float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
  for (int k = 1; k <= NH; ++k) {
    s1 += rsg(k - 1) * (a[(size_t)(ix + k) * L + iz + k] - a[(size_t)(ix - k + 1) * L + iz - k + 1]);
    s2 += rsg(k - 1) * (a[(size_t)(ix + k) * L + iz - k + 1] - a[(size_t)(ix - k + 1) * L + iz + k]);
  }
  d1 = s1;
  d2 = s2;
}

__device__ __forceinline__ void pair_s(const float *a, size_t L, int ix, int iz, float &d1, float &d2)
{
  float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
  for (int k = 1; k <= NH; ++k) {
    s1 += rsg(k - 1) * (a[(size_t)(ix + k - 1) * L + iz + k - 1] - a[(size_t)(ix - k) * L + iz - k]);
    s2 += rsg(k - 1) * (a[(size_t)(ix + k - 1) * L + iz - k] - a[(size_t)(ix - k) * L + iz + k - 1]);
  }
  d1 = s1;
  d2 = s2;
}

__device__ __forceinline__ bool interior(const Grid &g, int ix, int iz)
{
  return ix >= NH && ix < g.Nx - NH && iz >= g.izStart && iz < g.Nz - NH;
}

// the stress-source weights 0.5 w over the 11 x 11 window
struct K1 {
  float k1[121];
};
// The column work of a reverse step, one warp per padded-grid column, in the
// order the step needs it: residual injection at the column's receivers (the
// adjoint of isoelastic.c:103-144), this column's part of dJ/d(source sample)
// (the adjoint of the stress source, read before the free surface as the
// source is added after it), then the adjoint of the free-surface image.
struct SurfaceArgs {
  Grid g;
  float *lam[8];
  const int *colptr[3], *rzs[3], *rid[3];  // receivers by column
  const float *res[3];                     // this step's residual rows (null: nothing to inject)
  int nrec[3];
  SourceSet src;
  K1 k1;
  float *gsrc;  // [nsrc][nt], summed over columns
  int it, fs, tensor;
};

// The column work for rows [r0, r1) of column ix, one warp.
__device__ __forceinline__ void surface_warp(const SurfaceArgs &a, int ix, int r0, int r1, int lane)
{
  const Grid &g = a.g;
  const size_t col = (size_t)ix * g.ldz;
  for (int k = 0; k < 3; ++k) {
    if (!a.res[k]) continue;
    for (int j = a.colptr[k][ix] + lane; j < a.colptr[k][ix + 1]; j += 32) {
      const int rz = a.rzs[k][j];
      if (rz < r0 || rz >= r1) continue;
      const size_t c = col + rz;
      const float r = a.res[k][a.rid[k][j]];
      if (k == TTI_REC_VX) atomicAdd(a.lam[0] + c, r);
      else if (k == TTI_REC_VZ) atomicAdd(a.lam[1] + c, r);
      else {
        atomicAdd(a.lam[2] + c, 0.5f * r);
        atomicAdd(a.lam[3] + c, 0.5f * r);
      }
    }
  }
  __syncwarp();
  for (int n = 0; n < a.src.n; ++n) {
    const int dx = ix - a.src.x[n];
    if (dx < -NH || dx > NH) continue;
    const int iz = a.src.z[n] + lane - NH;
    float v = 0.0f;
    if (lane <= 2 * NH && iz >= 0 && iz < g.Nz && iz >= r0 && iz < r1) {
      const size_t c = col + iz;
      float l = a.lam[2][c] + a.lam[3][c];
      if (a.tensor) l += a.lam[5][c] + a.lam[6][c];  // the source also adds to tau
      v = a.k1.k1[(dx + NH) * 11 + lane] * l;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0 && v != 0.0f) atomicAdd(a.gsrc + (size_t)n * a.src.nt + a.it, v);
  }
  __syncwarp();
  if (a.fs && ix >= NH && ix < g.Nx - NH && g.izStart - NH >= r0 && g.izStart + NH < r1) {
    // lane k moves image row izStart - k onto row izStart + k (distinct cells
    // for each k); lane 0 then adds the sxx images onto the surface row in
    // the order k = 1..5
    const size_t c = col + g.izStart;
    float *xx = a.lam[2], *zz = a.lam[3], *xz = a.lam[4];
    float img = 0.0f;
    if (lane >= 1 && lane <= NH) {
      const size_t m = c - lane, p = c + lane;
      img = xx[m];
      xx[p] -= img;
      zz[p] -= zz[m];
      xz[p] -= xz[m];
      xx[m] = 0.0f;
      zz[m] = 0.0f;
      xz[m] = 0.0f;
    }
    float add[NH];
#pragma unroll
    for (int k = 1; k <= NH; ++k) add[k - 1] = __shfl_sync(0xffffffffu, img, k);
    if (lane == 0) {
      float t = xx[c];
#pragma unroll
      for (int k = 0; k < NH; ++k) t += 2.0f * add[k];
      xx[c] = t;
      xz[c] = 0.0f;
      zz[c] = 0.0f;
    }
  }
  __syncwarp();
}

__global__ void k_adj_surface(SurfaceArgs a)
{
  pdl_sync();
  const int ix = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  if (ix >= a.g.Nx) return;
  surface_warp(a, ix, 0, a.g.Nz, threadIdx.x & 31);
}

// Adjoint of the velocity sources (coord:674-802), between the stress-half
// adjoint (T0..T3 written) and the velocity-half adjoint (lambda_v not yet
// updated). The source adds w src(t) to v after the velocity update, so
// dJ/d src(t) = sum over its cells of w . lambda_v with lambda_v already
// holding the transposed stress stencils of T. Cells outside the velocity
// update (image rows above a free surface, the rim) are never written by the
// forward step except by the source; their lambda_v only accumulates those
// stencils (a running sum over the whole reverse pass, kept in double beside
// lambda_v, which there holds only the injected residuals), which this kernel
// applies first, once per cell. One block: the rim update must finish before
// any source reads it.
struct VSrcArgs {
  Grid g;
  const float *lam0, *lam1;
  const float *T[4];
  const int4 *cell;
  const float2 *w;
  const int2 *rim;
  double *rim_acc;  // [nrim][2]
  int m, nsrc, nrim;
  float hx, hz;
  float *gsrc;  // [nsrc][nt]
  int nt, it;
};

__device__ __forceinline__ float t_at(const float *a, const Grid &g, int ix, int iz)
{
  return ix < 0 || ix >= g.Nx || iz < 0 || iz >= g.Nz ? 0.0f : a[(size_t)ix * g.ldz + iz];
}

// the transposed stress stencils at one velocity cell, T read as zero off the grid
__device__ float2 vsrc_dT(const VSrcArgs &a, int ix, int iz)
{
  float d[4][2];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    float s1 = 0.0f, s2 = 0.0f;
#pragma unroll
    for (int k = 1; k <= NH; ++k) {
      s1 += rsg(k - 1) * (t_at(a.T[f], a.g, ix + k, iz + k) - t_at(a.T[f], a.g, ix - k + 1, iz - k + 1));
      s2 += rsg(k - 1) * (t_at(a.T[f], a.g, ix + k, iz - k + 1) - t_at(a.T[f], a.g, ix - k + 1, iz + k));
    }
    d[f][0] = s1;
    d[f][1] = s2;
  }
  return make_float2(d[0][0] + d[1][1], d[2][0] + d[3][1]);  // T holds the combinations of store_T
}

constexpr int VSRC_THREADS = 256;

__global__ void __launch_bounds__(VSRC_THREADS) k_adj_vsource(VSrcArgs a)
{
  pdl_sync();
  const Grid &g = a.g;
  for (int q = threadIdx.x; q < a.nrim; q += blockDim.x) {
    const int2 c = a.rim[q];
    const float2 d = vsrc_dT(a, c.x, c.y);
    a.rim_acc[2 * q] -= d.x;
    a.rim_acc[2 * q + 1] -= d.y;
  }
  __syncthreads();
  __shared__ double part[VSRC_THREADS / 32];
  for (int n = 0; n < a.nsrc; ++n) {
    double v = 0.0;
    for (int q = threadIdx.x; q < a.m; q += blockDim.x) {
      const int4 c = a.cell[(size_t)n * a.m + q];
      if (c.x < 0) continue;
      const size_t i = (size_t)c.x * g.ldz + c.y;
      double lx = a.lam0[i], lz = a.lam1[i];
      if (c.z >= 0) {  // outside the velocity update: plus the accumulated stencils
        lx += a.rim_acc[2 * c.z];
        lz += a.rim_acc[2 * c.z + 1];
      } else {  // the velocity-half adjoint has not yet applied T here
        const float2 d = vsrc_dT(a, c.x, c.y);
        lx -= d.x;
        lz -= d.y;
      }
      const float2 w = a.w[(size_t)n * a.m + q];
      v += w.x * lx + w.y * lz;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int k = 0; k < (int)(blockDim.x >> 5); ++k) t += part[k];
      a.gsrc[(size_t)n * a.nt + a.it] = (float)t;
    }
    __syncthreads();
  }
}

// The transposed stress stencils are minus the velocity-node pairs; with
// t0..t3 the strain-rate adjoints (d/d vxx, vxz, vzx, vzz) they add to lambda_v
//   x: hx (d1 + d2)(t0) + hz (d1 - d2)(t1) = d1(hx t0 + hz t1) + d2(hx t0 - hz t1)
//   z: the same with t2, t3.
// The stencils are linear, so T holds those four combinations and each needs
// only one diagonal of the pair (40 taps a cell instead of 80).
__device__ __forceinline__ void store_T(const AdjArgs &a, size_t i, float t0, float t1, float t2, float t3)
{
  a.T[0][i] = a.hx * t0 + a.hz * t1;
  a.T[1][i] = a.hx * t0 - a.hz * t1;
  a.T[2][i] = a.hx * t2 + a.hz * t3;
  a.T[3][i] = a.hx * t2 - a.hz * t3;
}

// stress-half adjoint, local part: gradient sums, T0..T3, lambda_sigma *= coef1.
// PK (tiled path): packed parameters, and the strain rates the forward stress
// kernel kept (keep[0..3], tensor tau keep[4..6]); otherwise the stencils of
// the kept v (keep[0..1], tensor tau keep[2..4]). Block rows start at z_org.
// SURF: each warp (one column, 32 rows) first does the column work of its
// rows (surface_warp): the residual injection, the source gradient and, in the
// block whose rows hold izStart - 5 .. izStart + 5, the free-surface adjoint.
// That is all of it when z_org is at or above every receiver row, source
// window row and image row; the host checks this. Blocks from row z_end down
// have no column work and skip it.
template <int V, bool PK, bool SURF>
__global__ void __launch_bounds__(BZ *BX) k_adj_stress_local(AdjArgs a, SurfaceArgs sa, int z_org, int z_end)
{
  pdl_sync();
  const Grid &g = a.g;
  const int r0 = z_org + blockIdx.x * BZ;
  const int iz = r0 + threadIdx.x, ix = blockIdx.y * BX + threadIdx.y;
  if (SURF && ix < g.Nx && r0 < z_end) surface_warp(sa, ix, r0, r0 + BZ, threadIdx.x);
  if (!interior(g, ix, iz)) return;
  const size_t L = g.ldz, i = (size_t)ix * L + iz;
  const SParams m = stress_params<PK, V>(a, i, cell_undamped(a, ix, iz));
  const float la = a.lam[2][i], lb = a.lam[3][i], le = a.lam[4][i], b = m.b, c1 = m.c1;
  const float c11 = m.c11, c13 = m.c13, c33 = m.c33, c55 = m.c55;
  float vxx, vxz, vzx, vzz;
  if (PK) {
    vxx = a.keep[0][i];
    vxz = a.keep[1][i];
    vzx = a.keep[2][i];
    vzz = a.keep[3][i];
  } else {
    float a1, a2, b1, b2;
    pair_s(a.keep[0], L, ix, iz, a1, a2);
    pair_s(a.keep[1], L, ix, iz, b1, b2);
    vxx = a.hx * (a1 + a2);
    vxz = a.hz * (a1 - a2);
    vzx = a.hx * (b1 + b2);
    vzz = a.hz * (b1 - b2);
  }
  const float *const *tau = a.keep + (PK ? 4 : 2);
  if (V == TTI_BOND) {  // sigma += coef2 H (vxx, vzz, vzx + vxz), H symmetric with c15, c35 (bond:836-873)
    const float c15 = m.p, c35 = m.q, sh = vzx + vxz;
    a.acc[0][i] += b * la * vxx;
    a.acc[1][i] += b * (la * vzz + lb * vxx);
    a.acc[2][i] += b * lb * vzz;
    a.acc[3][i] += b * le * sh;
    a.acc[4][i] += b * (la * sh + le * vxx);
    a.acc[5][i] += b * (lb * sh + le * vzz);
    const float Lsh = b * (c15 * la + c35 * lb + c55 * le);
    store_T(a, i, b * (c11 * la + c13 * lb + c15 * le), Lsh, Lsh, b * (c13 * la + c33 * lb + c35 * le));
    a.lam[2][i] = c1 * la;
    a.lam[3][i] = c1 * lb;
    a.lam[4][i] = c1 * le;
    return;
  }
  if (V == TTI_TENSOR) {
    // forward (tensor:826-851): n = coef1 tau + coef2 H e(theta, v); tau' = n; sigma' = R(theta) n,
    // with tau the kept one from before the stress half.
    const float s2 = m.p, c2 = m.q, st = a.p.s2t[i], cd = c2 - s2, sh = vxz + vzx;
    const float exx = c2 * vxx + s2 * vzz - 0.5f * st * sh, ezz = s2 * vxx + c2 * vzz + 0.5f * st * sh;
    const float exz = st * (vxx - vzz) + cd * sh;
    const float nxx = c1 * tau[0][i] + b * (c11 * exx + c13 * ezz);
    const float nzz = c1 * tau[1][i] + b * (c13 * exx + c33 * ezz);
    const float nxz = c1 * tau[2][i] + b * c55 * exz;
    // lambda_n = lambda_tau' + R^T lambda_sigma'
    const float lxx = a.lam[5][i] + c2 * la + s2 * lb - 0.5f * st * le;
    const float lzz = a.lam[6][i] + s2 * la + c2 * lb + 0.5f * st * le;
    const float lxz = a.lam[7][i] + st * la - st * lb + cd * le;
    a.acc[0][i] += b * lxx * exx;
    a.acc[1][i] += b * (lxx * ezz + lzz * exx);
    a.acc[2][i] += b * lzz * ezz;
    a.acc[3][i] += b * lxz * exz;
    // theta: through the strain rotation (d s2 = st, d c2 = -st, d st = 2 cd) and through R
    const float dexx = st * (vzz - vxx) - cd * sh, dexz = 2.0f * cd * (vxx - vzz) - 2.0f * st * sh;
    const float rxx_ = -st * nxx + st * nzz + 2.0f * cd * nxz, rxz_ = -cd * (nxx - nzz) - 2.0f * st * nxz;
    a.acc[4][i] += lxx * b * (c11 - c13) * dexx + lzz * b * (c13 - c33) * dexx + lxz * b * c55 * dexz +
                   (la - lb) * rxx_ + le * rxz_;
    const float Lexx = b * (c11 * lxx + c13 * lzz), Lezz = b * (c13 * lxx + c33 * lzz), Lexz = b * c55 * lxz;
    const float Lsh = 0.5f * st * (Lezz - Lexx) + cd * Lexz;
    store_T(a, i, c2 * Lexx + s2 * Lezz + st * Lexz, Lsh, Lsh, s2 * Lexx + c2 * Lezz - st * Lexz);
    a.lam[5][i] = c1 * lxx;
    a.lam[6][i] = c1 * lzz;
    a.lam[7][i] = c1 * lxz;
    a.lam[2][i] = a.lam[3][i] = a.lam[4][i] = 0.0f;  // sigma is overwritten by R tau
    return;
  }
  const float s = m.p, co = m.q;
  const float rxx = co * vxx - s * vxz, rxz = s * vxx + co * vxz;
  const float rzx = co * vzx - s * vzz, rzz = s * vzx + co * vzz;
  a.acc[0][i] += b * la * rxx;
  a.acc[1][i] += b * (la * rzz + lb * rxx);
  a.acc[2][i] += b * lb * rzz;
  a.acc[4][i] += b * (la * (c13 * rzx - c11 * rxz) + lb * (c33 * rzx - c13 * rxz) + le * c55 * (rxx - rzz));
  const float Lxx = b * (c11 * la + c13 * lb), Lzz = b * (c13 * la + c33 * lb), Lq = b * c55 * le;
  store_T(a, i, co * Lxx + s * Lq, co * Lq - s * Lxx, co * Lq + s * Lzz, co * Lzz - s * Lq);
  a.lam[2][i] = c1 * la;
  a.lam[3][i] = c1 * lb;
  a.lam[4][i] = c1 * le;
}

// Transposed stress stencils into lambda_v (minus the velocity-node pairs),
// then the velocity-half adjoint at the same cell: sin/cos theta_v sums,
// TV0..TV5, lambda_v *= coef1. Both act on one cell's lambda_v, so one pass.
template <int V>
__global__ void __launch_bounds__(BZ *BX) k_adj_velocity(AdjArgs a)
{
  const Grid &g = a.g;
  const int iz = blockIdx.x * BZ + threadIdx.x, ix = blockIdx.y * BX + threadIdx.y;
  if (!interior(g, ix, iz)) return;
  const size_t L = g.ldz, i = (size_t)ix * L + iz;
  const float hx = a.hx, hz = a.hz;
  float lx, lz;
  {
    float p1, q2, r1, s2, u;
    pair_v(a.T[0], L, ix, iz, p1, u);
    pair_v(a.T[1], L, ix, iz, u, q2);
    pair_v(a.T[2], L, ix, iz, r1, u);
    pair_v(a.T[3], L, ix, iz, u, s2);
    lx = a.lam[0][i] - (p1 + q2);
    lz = a.lam[1][i] - (r1 + s2);
  }
  const float br = a.p.coef2[i] * a.p.invrho[i];
  const float Fx = br * lx, Fz = br * lz;
  // coordinate: rotation by theta_v; Bond: fx = sxx_x + sxz_z, fz = sxz_x + szz_z
  const float cv = V != TTI_COORDINATE ? 1.0f : a.p.csv[i], sv = V != TTI_COORDINATE ? 0.0f : a.p.snv[i];
  if (V == TTI_COORDINATE) {  // theta_v terms from the stencils of the kept sigma
    float a1, a2, b1, b2, e1, e2;
    pair_v(a.keep[2], L, ix, iz, a1, a2);
    pair_v(a.keep[3], L, ix, iz, b1, b2);
    pair_v(a.keep[4], L, ix, iz, e1, e2);
    const float sxx_x = hx * (a1 + a2), sxx_z = hx * (a1 - a2);  // 1/dx for both, as coord:633
    const float szz_x = hx * (b1 + b2), szz_z = hz * (b1 - b2);
    const float sxz_x = hx * (e1 + e2), sxz_z = hz * (e1 - e2);
    a.acc[5][i] += Fx * (sxz_x - sxx_z) + Fz * (szz_x - sxz_z);
    a.acc[6][i] += Fx * (sxx_x + sxz_z) + Fz * (sxz_x + szz_z);
  }
  const float Axx_x = cv * Fx, Axx_z = -sv * Fx;
  const float Axz_x = sv * Fx + cv * Fz, Axz_z = cv * Fx - sv * Fz;
  const float Azz_x = sv * Fz, Azz_z = cv * Fz;
  a.TV[0][i] = hx * (Axx_x + Axx_z);
  a.TV[1][i] = hx * (Axx_x - Axx_z);
  a.TV[2][i] = hx * Azz_x + hz * Azz_z;
  a.TV[3][i] = hx * Azz_x - hz * Azz_z;
  a.TV[4][i] = hx * Axz_x + hz * Axz_z;
  a.TV[5][i] = hx * Axz_x - hz * Axz_z;
  const float c1 = a.p.coef1[i];
  a.lam[0][i] = c1 * lx;
  a.lam[1][i] = c1 * lz;
}

// transposed velocity stencils into lambda_sigma (minus the stress-node pairs);
// with a free surface also the image rows above izStart
__global__ void __launch_bounds__(BZ *BX) k_adj_velocity_stencil(AdjArgs a)
{
  const Grid &g = a.g;
  const int iz = blockIdx.x * BZ + threadIdx.x, ix = blockIdx.y * BX + threadIdx.y;
  if (ix < NH || ix >= g.Nx - NH || iz < a.z_lo || iz >= g.Nz - NH) return;
  const size_t L = g.ldz, i = (size_t)ix * L + iz;
  float p1, p2, q1, q2, r1, r2, u;
  pair_s(a.TV[0], L, ix, iz, p1, u);
  pair_s(a.TV[1], L, ix, iz, u, p2);
  pair_s(a.TV[2], L, ix, iz, q1, u);
  pair_s(a.TV[3], L, ix, iz, u, q2);
  pair_s(a.TV[4], L, ix, iz, r1, u);
  pair_s(a.TV[5], L, ix, iz, u, r2);
  a.lam[2][i] -= p1 + p2;
  a.lam[3][i] -= q1 + q2;
  a.lam[4][i] -= r1 + r2;
}

// ---------------------------------------------------------------- tiled adjoint
// The two stencil passes of the adjoint on the forward path's 128 x 16 tiles:
// every stencil tap comes from a TMA halo box in shared memory (one 2D copy per
// field, the box origin rounded down to a 16-byte boundary, zeros outside the
// array), per-cell parameters from the packed arrays.
struct alignas(64) AdjTile {
  CUtensorMap map[6];  // velocity pass: T0..T3; stress-node pass: TV0..TV5
  AdjArgs a;
  packed::Packed pk;
  int z_base;  // first tile row (multiple of 4)
  int *err;    // bit 4: a TMA wait timed out
};

struct TileCells {
  int x0, z0, xc, z;
};
__device__ __forceinline__ TileCells tile_cells(int z_base)
{
  TileCells c;
  c.z0 = z_base + blockIdx.x * tiled::TZ;
  c.x0 = NH + blockIdx.y * tiled::TX;
  c.xc = c.x0 + (tiled::TX / 4) * (threadIdx.x >> 7);
  c.z = c.z0 + (threadIdx.x & 127);
  return c;
}

// stress-node pair of shared field q centred on (x, z): q[m * BZ + n] = value at (x + m, z + n)
__device__ __forceinline__ void spair(const float *q, float &d1, float &d2)
{
  constexpr int B = tiled::BZ;
  float s1 = rsg(0) * (q[0] - q[-B - 1]), s2 = rsg(0) * (q[-1] - q[-B]);
#pragma unroll
  for (int k = 2; k <= NH; ++k) {
    s1 += rsg(k - 1) * (q[(k - 1) * B + k - 1] - q[-k * B - k]);
    s2 += rsg(k - 1) * (q[(k - 1) * B - k] - q[-k * B + k - 1]);
  }
  d1 = s1;
  d2 = s2;
}

// one diagonal of the velocity-node pair of shared field q centred on (x, z)
__device__ __forceinline__ float vdiag1(const float *q)
{
  constexpr int B = tiled::BZ;
  float s = rsg(0) * (q[B + 1] - q[0]);
#pragma unroll
  for (int k = 2; k <= NH; ++k) s += rsg(k - 1) * (q[k * B + k] - q[(1 - k) * B + 1 - k]);
  return s;
}
__device__ __forceinline__ float vdiag2(const float *q)
{
  constexpr int B = tiled::BZ;
  float s = rsg(0) * (q[B] - q[1]);
#pragma unroll
  for (int k = 2; k <= NH; ++k) s += rsg(k - 1) * (q[k * B + 1 - k] - q[(1 - k) * B + k]);
  return s;
}

// While the halo boxes are in flight, the lanes of each warp ask L2 for the
// per-cell lines the velocity-half adjoint reads after the wait (coef1/coef2,
// invrho; coordinate also sin/cos theta_v, the kept P Q R S and the two theta_v
// sums): one 128-byte line per column and array, two for the float2 arrays.
template <int V>
__device__ __forceinline__ void prefetch_adj_velocity(const AdjTile &at, const TileCells &c)
{
  constexpr int SLOTS = V == TTI_COORDINATE ? 11 : 3;
  const AdjArgs &a = at.a;
  const int lane = threadIdx.x & 31, z = c.z - lane;  // the warp's first row
  if (z >= a.g.Nz - NH) return;
  for (int q = lane; q < (tiled::TX / 4) * SLOTS; q += 32) {
    const int col = q / SLOTS, k = q % SLOTS, x = c.xc + col;
    if (x >= a.g.Nx - NH) continue;
    const size_t i = (size_t)x * a.g.ldz + z;
    const void *p;
    if (k < 2) p = at.pk.cf + i + 16 * k;
    else if (k == 2) p = a.p.invrho + i;
    else if (k < 5) p = at.pk.vsc + i + 16 * (k - 3);
    else if (k < 9) p = a.keep[4 + (k - 5)] + i;
    else p = a.acc[5 + (k - 9)] + i;
    asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

// transposed stress stencils into lambda_v, then the velocity-half adjoint
// (maps: T0..T3; coordinate: the theta_v terms from the kept stress
// derivative combinations P Q R S that the forward velocity kernel wrote)
template <int V>
__global__ void __launch_bounds__(tiled::NT, 3) k_adj_velocity_tiled(const __grid_constant__ AdjTile at)
{
  pdl_sync();
  constexpr int F = tiled::FIELD, B = tiled::BZ;
  extern __shared__ __align__(128) float sm[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + 4 * F);
  const AdjArgs &a = at.a;
  const Grid &g = a.g;
  const TileCells c = tile_cells(at.z_base);
  tiled::tma::issue_tiles(at.map, sm, bar, 4, c.z0, c.x0, 4);
  const int z = c.z;
  const bool zin = z >= g.izStart && z < g.Nz - NH;
  // this row's lambda_v, loaded while the halo boxes are in flight
  constexpr int NJ = tiled::TX / 4;
  float l[NJ][2];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int x = c.xc + j;
    const size_t i = (size_t)x * g.ldz + z;
    const bool on = zin && x < g.Nx - NH;
    l[j][0] = on ? a.lam[0][i] : 0.0f;
    l[j][1] = on ? a.lam[1][i] : 0.0f;
  }
  prefetch_adj_velocity<V>(at, c);
  if (!tiled::tma::wait_tiles(at.err, bar)) return;
  if (!zin) return;
  const float hx = a.hx, hz = a.hz;
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int x = c.xc + j;
    if (x >= g.Nx - NH) break;
    const size_t i = (size_t)x * g.ldz + z;
    // the cell's inputs are requested before its stencil (the kept fields are
    // read-only here, so their loads need not wait behind the previous
    // column's stores)
    const float2 cf = cell_undamped(a, x, z) ? make_float2(1.0f, a.dt) : __ldg(at.pk.cf + i);
    const float ir = __ldg(a.p.invrho + i);
    float sv = 0.0f, cv = 1.0f;  // tensor and Bond: fx = sxx_x + sxz_z, fz = sxz_x + szz_z
    float kp = 0.0f, kq = 0.0f, kr = 0.0f, ks = 0.0f, a5 = 0.0f, a6 = 0.0f;
    if (V == TTI_COORDINATE) {
      const float2 vsc = __ldg(at.pk.vsc + i);
      sv = vsc.x;
      cv = vsc.y;
      kp = __ldg(a.keep[4] + i);
      kq = __ldg(a.keep[5] + i);
      kr = __ldg(a.keep[6] + i);
      ks = __ldg(a.keep[7] + i);
      a5 = a.acc[5][i];
      a6 = a.acc[6][i];
    }
    const float *q = sm + (x - c.x0 + 4) * B + (z - c.z0 + 8);
    const float lx = l[j][0] - (vdiag1(q) + vdiag2(q + F));
    const float lz = l[j][1] - (vdiag1(q + 2 * F) + vdiag2(q + 3 * F));
    const float br = cf.y * ir;
    const float Fx = br * lx, Fz = br * lz;
    if (V == TTI_COORDINATE) {
      // P = sxz_x - sxx_z, Q = szz_x - sxz_z, R = sxx_x + sxz_z, S = sxz_x + szz_z
      a.acc[5][i] = a5 + (Fx * kp + Fz * kq);
      a.acc[6][i] = a6 + (Fx * kr + Fz * ks);
    }
    const float Axx_x = cv * Fx, Axx_z = -sv * Fx;
    const float Axz_x = sv * Fx + cv * Fz, Axz_z = cv * Fx - sv * Fz;
    const float Azz_x = sv * Fz, Azz_z = cv * Fz;
    a.TV[0][i] = hx * (Axx_x + Axx_z);
    a.TV[1][i] = hx * (Axx_x - Axx_z);
    a.TV[2][i] = hx * Azz_x + hz * Azz_z;
    a.TV[3][i] = hx * Azz_x - hz * Azz_z;
    a.TV[4][i] = hx * Axz_x + hz * Axz_z;
    a.TV[5][i] = hx * Axz_x - hz * Axz_z;
    a.lam[0][i] = cf.x * lx;
    a.lam[1][i] = cf.x * lz;
  }
}

// TMA boxes of the TV pair p (components sxx, szz, sxz) into shared buffers
// 2b, 2b + 1, completing on barrier p; called by one thread.
__device__ __forceinline__ void issue_tv_pair(const AdjTile &at, float *sm, unsigned long long *bar, int p, int b,
                                              const TileCells &c)
{
  constexpr unsigned BOX_BYTES = tiled::BX * tiled::BZ * 4;
  tiled::tma::mbar_arrive_expect_tx(bar + p, 2 * BOX_BYTES);
  for (int k = 0; k < 2; ++k)
    tiled::tma::tma_load_2d(sm + (2 * b + k) * tiled::FIELD, at.map + 2 * p + k, c.z0 - 8, c.x0 - 5, bar + p);
}

// transposed velocity stencils into lambda_sigma (maps: TV0..TV5), rows from
// z_lo. The boxes come in three pairs (sxx: TV0 TV1, szz: TV2 TV3, sxz: TV4
// TV5) through two pair buffers: pairs 0 and 1 are in flight from the start,
// and pair 2 goes into pair 0's buffer once every thread is done with it. Four
// boxes (58 KB) instead of six let three CTAs share an SM.
__global__ void __launch_bounds__(tiled::NT, 3) k_adj_vstencil_tiled(const __grid_constant__ AdjTile at)
{
  pdl_sync();
  constexpr int F = tiled::FIELD, B = tiled::BZ;
  extern __shared__ __align__(128) float sm[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + 4 * F);
  const AdjArgs &a = at.a;
  const Grid &g = a.g;
  const TileCells c = tile_cells(at.z_base);
  if (threadIdx.x == 0) {
    for (int q = 0; q < 3; ++q) tiled::tma::mbar_init(bar + q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    issue_tv_pair(at, sm, bar, 0, 0, c);
    issue_tv_pair(at, sm, bar, 1, 1, c);
  }
  const int z = c.z;
  const bool zin = z >= a.z_lo && z < g.Nz - NH;
  // this row's lambda_sigma, loaded while the halo boxes are in flight
  constexpr int NJ = tiled::TX / 4;
  float l[NJ][3];
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int x = c.xc + j;
    const size_t i = (size_t)x * g.ldz + z;
    const bool on = zin && x < g.Nx - NH;
    l[j][0] = on ? a.lam[2][i] : 0.0f;
    l[j][1] = on ? a.lam[3][i] : 0.0f;
    l[j][2] = on ? a.lam[4][i] : 0.0f;
  }
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    if (q == 1) {
      // every thread is done with pair 0's buffer: pair 2 goes there while pair 1 is used
      __syncthreads();
      if (threadIdx.x == 0) {
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        issue_tv_pair(at, sm, bar, 2, 0, c);
      }
    }
    // on a timeout the pairs still in flight get a bounded drain: q .. 1 before pair 2 is issued, q .. 2 after
    if (!tiled::tma::wait_group(at.err, bar, q, q == 0 ? 2 : 3)) return;
    if (zin) {
#pragma unroll
      for (int j = 0; j < NJ; ++j) {
        const float *p = sm + (c.xc + j - c.x0 + 5) * B + (z - c.z0 + 8) + 2 * (q & 1) * F;
        float d1, d2, u;
        spair(p, d1, u);
        spair(p + F, u, d2);
        l[j][q] -= d1 + d2;
      }
    }
  }
  if (!zin) return;
#pragma unroll
  for (int j = 0; j < NJ; ++j) {
    const int x = c.xc + j;
    if (x >= g.Nx - NH) break;
    const size_t i = (size_t)x * g.ldz + z;
    a.lam[2][i] = l[j][0];
    a.lam[3][i] = l[j][1];
    a.lam[4][i] = l[j][2];
  }
}

template <typename K>
cudaError_t launch_adj_tile(K kernel, const AdjTile &at, int nfields, int z_first, const Grid &g, cudaStream_t st)
{
  const size_t bytes = (size_t)nfields * tiled::FIELD * sizeof(float) + 64;  // + up to 8 barriers
  static std::mutex mu;
  static const void *done[8];
  static int ndone = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    bool seen = false;
    for (int k = 0; k < ndone; ++k) seen = seen || done[k] == (const void *)kernel;
    if (!seen) {
      cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout, cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return e;
      if (ndone < 8) done[ndone++] = (const void *)kernel;
    }
  }
  AdjTile b = at;
  b.z_base = z_first & ~31;  // 32-row aligned: a warp's rows are one 128-byte line
  const int nz = g.Nz - NH - b.z_base, nx = g.Nx - 2 * NH;
  if (nz <= 0 || nx <= 0) return cudaSuccess;
  return launch_pdl(kernel, dim3((nz + tiled::TZ - 1) / tiled::TZ, (nx + tiled::TX - 1) / tiled::TX), dim3(tiled::NT),
                    bytes, st, b);
}

// residuals d - dobs (time-major) and J
__global__ void k_residual(const float *rec, const float *obs, float *res, size_t n, double *J)
{
  double acc = 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    const float r = rec[q] - obs[q];
    res[q] = r;
    acc += 0.5 * (double)r * (double)r;
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(J, acc);
}

// Bond rotation of the VTI moduli (bond:492-541): derivatives of c11 c13 c15
// c33 c35 c55 with respect to C11, C13, C33 and theta (d[0..3][0..5])
__device__ void bond_moduli_grad(double C11, double C13, double C33, double C55, double th, double d[4][6])
{
  const double sn = sin(th), cs = cos(th);
  const double s2 = sn * sn, c2 = cs * cs, s4 = s2 * s2, c4 = c2 * c2;
  const double s2t = sin(2.0 * th), c2t = cos(2.0 * th), s22 = s2t * s2t;
  const double ds2 = s2t, dc2 = -s2t, ds4 = 2.0 * s2 * s2t, dc4 = -2.0 * c2 * s2t;
  const double ds2t = 2.0 * c2t, dc2t = -2.0 * s2t, ds22 = 4.0 * s2t * c2t, dc22 = -ds22;
  const double A = C13 + 2.0 * C55;
  const double rows[4][6] = {
      {c4, 0.25 * s22, -0.5 * c2 * s2t, s4, -0.5 * s2 * s2t, 0.25 * s22},
      {0.5 * s22, s4 + c4, 0.5 * c2t * s2t, 0.5 * s22, -0.5 * c2t * s2t, -0.5 * s22},
      {s4, 0.25 * s22, 0.5 * s2 * s2t, c4, 0.5 * c2 * s2t, 0.25 * s22},
      {C11 * dc4 + C33 * ds4 + (0.5 * C13 + C55) * ds22, (0.25 * (C11 + C33) - C55) * ds22 + C13 * (ds4 + dc4),
       0.5 * ((-C11 * dc2 + C33 * ds2 + A * dc2t) * s2t + (-C11 * c2 + C33 * s2 + A * c2t) * ds2t),
       C11 * ds4 + C33 * dc4 + (0.5 * C13 + C55) * ds22,
       0.5 * ((-C11 * ds2 + C33 * dc2 - A * dc2t) * s2t + (-C11 * s2 + C33 * c2 - A * c2t) * ds2t),
       0.25 * (C11 + C33 - 2.0 * C13) * ds22 + C55 * dc22}};
  for (int m = 0; m < 4; ++m)
    for (int k = 0; k < 6; ++k) d[m][k] = rows[m][k];
}

// Bond free-surface row (bond:543-568): the moduli a = (c11 c13 c15 c33 c35 c55)
// act only through the effective c11' = a11 - a13 n35 + a15 n55; dc[k] = dc11'/da[k].
__device__ void bond_fs_c11_grad(const double a[6], double dc[6])
{
  const double a13 = a[1], a15 = a[2], a33 = a[3], a35 = a[4], a55 = a[5];
  const double N = a13 * a55 - a15 * a35, D = a33 * a55 - a35 * a35;
  double n35 = -N / D;
  const bool fallback = !isfinite(n35);
  if (fallback) n35 = -a13 / a33;
  if (!isfinite(n35)) n35 = 0.0;
  const double M = a13 * n35 - a15 * a33, Q = a33 * a55 - n35 * n35, n55 = M / Q;
  for (int v = 0; v < 6; ++v) {  // one-hot forward derivatives
    const double d11 = v == 0, d13 = v == 1, d15 = v == 2, d33 = v == 3, d35 = v == 4, d55 = v == 5;
    double dn35;
    if (!fallback) {
      const double dN = d13 * a55 + a13 * d55 - d15 * a35 - a15 * d35, dD = d33 * a55 + a33 * d55 - 2.0 * a35 * d35;
      dn35 = -(dN * D - N * dD) / (D * D);
    } else {
      dn35 = isfinite(-a13 / a33) ? -(d13 * a33 - a13 * d33) / (a33 * a33) : 0.0;
    }
    const double dM = d13 * n35 + a13 * dn35 - d15 * a33 - a15 * d33;
    const double dQ = d33 * a55 + a33 * d55 - 2.0 * n35 * dn35;
    dc[v] = d11 - d13 * n35 - a13 * dn35 + d15 * n55 + a15 * (dM * Q - M * dQ) / (Q * Q);
  }
}

// chain rule to vp, epsilon, delta, theta (degrees), every cell
template <int V>
__global__ void k_chain(Grid g, Params p, const float *vp, const float *vs, const float *rho, const float *beta,
                        const float *eps, const float *delta, const float *theta, GradState gs, float scalar,
                        int freesurface)
{
  const float rad = (float)(scalar * M_PI / 180.0);
  const int iz = blockIdx.x * BZ + threadIdx.x, ix = blockIdx.y * BX + threadIdx.y;
  if (iz >= g.Nz || ix >= g.Nx) return;
  const size_t L = g.ldz, i = (size_t)ix * L + iz;
  const double B = beta[i], P = vp[i], S = vs[i], R = rho[i];  // vp/Beta, vs/Beta, rho*Beta
  const double f = 1.0 - (S / P) * (S / P), e = eps[i], d = delta[i];
  const double q = sqrt(f * (f + 2.0 * d));
  const double dc11 = 2.0 * R * P * (1.0 + 2.0 * e), dc33 = 2.0 * R * P;
  const double dc13 = q > 0.0 ? R * (2.0 * P * q + (f + d) / q * 2.0 * S * S / P) : 0.0;
  double g11 = gs.acc[0][i], g13 = gs.acc[1][i], g33 = gs.acc[2][i];  // VTI moduli (coordinate)
  if (V == TTI_BOND) {  // through the Bond rotation: sums of c11 c13 c33 c55 c15 c35
    const double C11 = R * P * P * (1.0 + 2.0 * e), C13 = R * (P * P * q - S * S), C33 = R * P * P, C55 = R * S * S;
    double dm[4][6];
    const double th = scalar * (double)theta[i] / 180.0 * M_PI;
    bond_moduli_grad(C11, C13, C33, C55, th, dm);
    double gm[6] = {gs.acc[0][i], gs.acc[1][i], gs.acc[4][i], gs.acc[2][i], gs.acc[5][i], gs.acc[3][i]};
    if (freesurface && iz == g.E) {  // only the effective c11 acts on the free-surface row
      const double s2 = sin(th) * sin(th), c2 = cos(th) * cos(th), s4 = s2 * s2, c4 = c2 * c2;
      const double s2t = sin(2.0 * th), c2t = cos(2.0 * th), s22 = s2t * s2t, c22 = c2t * c2t;
      const double m[6] = {C11 * c4 + C33 * s4 + (0.5 * C13 + C55) * s22,
                           (0.25 * (C11 + C33) - C55) * s22 + C13 * (s4 + c4),
                           0.5 * (-C11 * c2 + C33 * s2 + (C13 + 2.0 * C55) * c2t) * s2t,
                           C11 * s4 + C33 * c4 + (0.5 * C13 + C55) * s22,
                           0.5 * (-C11 * s2 + C33 * c2 - (C13 + 2.0 * C55) * c2t) * s2t,
                           0.25 * (C11 + C33 - 2.0 * C13) * s22 + C55 * c22};
      double dc[6];
      bond_fs_c11_grad(m, dc);
      const double g11_ = gm[0];
      for (int k = 0; k < 6; ++k) gm[k] = g11_ * dc[k];
    }
    g11 = g13 = g33 = 0.0;
    double gt = 0.0;
    for (int k = 0; k < 6; ++k) {
      g11 += gm[k] * dm[0][k];
      g13 += gm[k] * dm[1][k];
      g33 += gm[k] * dm[2][k];
      gt += gm[k] * dm[3][k];
    }
    gs.out[3][i] = (float)(gt * rad);
  }
  gs.out[0][i] = (float)((g11 * dc11 + g13 * dc13 + g33 * dc33) / B);
  gs.out[1][i] = (float)(g11 * 2.0 * R * P * P);
  gs.out[2][i] = (float)(q > 0.0 ? g13 * R * P * P * f / q : 0.0);
  if (V == TTI_TENSOR) gs.out[3][i] = (float)(gs.acc[4][i] * rad);  // no rotation at the velocity node
  if (V != TTI_COORDINATE) return;
  double gt = gs.acc[4][i];
  const double sn = p.sn[i], cs = p.cs[i];
  for (int a = 0; a <= 1; ++a)
    for (int b = 0; b <= 1; ++b) {
      const int vx = ix - a, vz = iz - b;
      if (vx < 0 || vz < 0) continue;
      const bool inner = vx < g.Nx - 1 && vz < g.Nz - 1;
      if (!inner && (a || b)) continue;
      const size_t j = (size_t)vx * L + vz;
      gt += (inner ? 0.25 : 1.0) * (gs.acc[5][j] * cs - gs.acc[6][j] * sn);
    }
  gs.out[3][i] = (float)(gt * rad);
}

int gerr(tti_handle *h, int code, const char *msg) { return handle_error(h, code, msg); }

// On failure the runtime's last error is cleared as well: a refused
// allocation must not be found again by a later launch check.
#define GCK(h, call)                                                                    \
  do {                                                                                  \
    cudaError_t e_ = (call);                                                            \
    if (e_ != cudaSuccess) {                                                            \
      cudaGetLastError();                                                               \
      return gerr((h), e_ == cudaErrorMemoryAllocation ? TTI_ERR_NOMEM : TTI_ERR_CUDA, \
                  cudaGetErrorString(e_));                                              \
    }                                                                                   \
  } while (0)

int grad_check(tti_handle *h)
{
  if (!h->have_model || !h->m_eps) return gerr(h, TTI_ERR_STATE, "model not uploaded");
  return TTI_OK;
}

int grad_alloc(tti_handle *h)
{
  if (h->grad) return TTI_OK;
  GradState *s = new GradState();
  h->grad = s;
  const size_t n = h->g.n;
  auto al = [&](float **p) {
    if (cudaMalloc(p, n * sizeof(float)) != cudaSuccess) return false;
    return cudaMemsetAsync(*p, 0, n * sizeof(float), h->stream) == cudaSuccess;
  };
  bool ok = true;
  for (int k = 0; k < (h->cfg.variant == TTI_TENSOR ? 8 : 5); ++k) ok = ok && al(&s->lam[k]);
  for (auto &p : s->T) ok = ok && al(&p);
  for (auto &p : s->TV) ok = ok && al(&p);
  for (auto &p : s->acc) ok = ok && al(&p);
  for (auto &p : s->out) ok = ok && al(&p);
  ok = ok && cudaMalloc(&s->d_J, sizeof(double)) == cudaSuccess;
  if (!ok) {
    cudaGetLastError();
    return gerr(h, TTI_ERR_NOMEM, "device allocation of the gradient buffers failed");
  }
  if (h->use_tiled) {
    void *mem = nullptr;
    if (posix_memalign(&mem, 64, 10 * sizeof(CUtensorMap)) != 0)
      return gerr(h, TTI_ERR_NOMEM, "host allocation failed");
    s->maps = static_cast<CUtensorMap *>(mem);
    for (int k = 0; k < 10; ++k)
      if (!tiled::encode_map(s->maps + k, h->g, k < 4 ? s->T[k] : s->TV[k - 4]))
        return gerr(h, TTI_ERR_CUDA, "cuTensorMapEncodeTiled failed");
  }
  GCK(h, cudaStreamSynchronize(h->stream));
  return TTI_OK;
}

AdjArgs adj_args(tti_handle *h, int slot)
{
  GradState *s = h->grad;
  AdjArgs a;
  a.g = h->g;
  a.p = handle_step_args(h).p;
  for (int k = 0; k < 8; ++k) a.lam[k] = s->lam[k];
  for (int k = 0; k < 4; ++k) a.T[k] = s->T[k];
  for (int k = 0; k < 6; ++k) a.TV[k] = s->TV[k];
  for (int k = 0; k < 7; ++k) a.acc[k] = s->acc[k];
  for (int k = 0; k < 8; ++k) a.keep[k] = k < s->nkeep ? s->keep + ((size_t)slot * s->nkeep + k) * h->g.n : nullptr;
  a.hx = 0.5f * h->invdx;
  a.hz = 0.5f * h->invdz;
  a.dt = h->cfg.dt;
  a.pk = packed::Packed{h->pk_cf, h->pk_vsc, h->pk_sc, h->pk_c4};
  a.undamped_ok = h->use_tiled && h->undamped_ok;
  a.und_z0 = h->cfg.freesurface ? 0 : h->g.E;
  a.z_lo = h->cfg.freesurface ? std::max(NH, h->g.izStart - NH) : h->g.izStart;
  return a;
}

// Cells and weights of the velocity sources from the forward step's own
// tables (the same float weights sources_block adds with), and the cells of
// all windows outside the velocity update.
int vsource_tables(tti_handle *h, const SourceTables &tab)
{
  GradState *s = h->grad;
  cudaFree(s->vcell);
  cudaFree(s->vw);
  cudaFree(s->vrim);
  cudaFree(s->vrim_acc);
  s->vcell = nullptr;
  s->vw = nullptr;
  s->vrim = nullptr;
  s->vrim_acc = nullptr;
  s->vm = s->vrim_n = 0;
  const int stype = h->cfg.stype, ns = h->nsrc;
  if (stype < 2 || ns <= 0) return TTI_OK;
  const Grid &g = h->g;
  std::vector<int> sx(ns), sz(ns);
  GCK(h, cudaMemcpyAsync(sx.data(), h->d_sx, sizeof(int) * ns, cudaMemcpyDeviceToHost, h->stream));
  GCK(h, cudaMemcpyAsync(sz.data(), h->d_sz, sizeof(int) * ns, cudaMemcpyDeviceToHost, h->stream));
  GCK(h, cudaStreamSynchronize(h->stream));
  const int m = stype == 8 ? 4 : 121;
  std::vector<int4> cell((size_t)ns * m);
  std::vector<float2> w((size_t)ns * m);
  std::vector<int2> rim;
  for (int n = 0; n < ns; ++n)
    for (int q = 0; q < m; ++q) {
      int ix, iz;
      float wx = 0.0f, wz = 0.0f;
      if (stype == 8) {  // coord:782-801: four cells, +-sqrt(2)/8
        static const int ox[4] = {0, -1, -1, 0}, oz[4] = {0, 0, -1, -1};
        static const float gx[4] = {-1.0f, -1.0f, 1.0f, 1.0f}, gz[4] = {1.0f, -1.0f, -1.0f, 1.0f};
        ix = sx[n] + ox[q];
        iz = sz[n] + oz[q];
        wx = gx[q] * tab.q8;
        wz = gz[q] * tab.q8;
      } else {  // the 11 x 11 window, cell q = (x offset + 5) * 11 + (z offset + 5)
        ix = sx[n] + q / 11 - NH;
        iz = sz[n] + q % 11 - NH;
        if (stype == 2 || stype == 4) {
          wx += tab.kx[q];
          wz += tab.kz[q];
        }
        if (stype == 3 || stype == 4) {
          wx -= tab.kz[q];
          wz += tab.kx[q];
        }
        if (stype == 5) wx = tab.k5[q];
        if (stype == 6) wz = tab.k5[q];
        if (stype == 7) wx = wz = tab.k7[q];
      }
      const bool on = ix >= 0 && ix < g.Nx && iz >= 0 && iz < g.Nz;
      cell[(size_t)n * m + q] = on ? make_int4(ix, iz, -1, 0) : make_int4(-1, -1, -1, 0);
      w[(size_t)n * m + q] = make_float2(wx, wz);
      const bool upd = ix >= NH && ix < g.Nx - NH && iz >= g.izStart && iz < g.Nz - NH;
      if (on && !upd) rim.push_back(make_int2(ix, iz));
    }
  const auto less = [](int2 a, int2 b) { return a.x != b.x ? a.x < b.x : a.y < b.y; };
  std::sort(rim.begin(), rim.end(), less);
  rim.erase(std::unique(rim.begin(), rim.end(), [](int2 a, int2 b) { return a.x == b.x && a.y == b.y; }),
            rim.end());
  for (auto &c : cell)
    if (c.x >= 0) {
      const auto it = std::lower_bound(rim.begin(), rim.end(), make_int2(c.x, c.y), less);
      if (it != rim.end() && it->x == c.x && it->y == c.y) c.z = (int)(it - rim.begin());
    }
  GCK(h, cudaMalloc(&s->vcell, sizeof(int4) * cell.size()));
  GCK(h, cudaMalloc(&s->vw, sizeof(float2) * w.size()));
  GCK(h, cudaMemcpyAsync(s->vcell, cell.data(), sizeof(int4) * cell.size(), cudaMemcpyHostToDevice, h->stream));
  GCK(h, cudaMemcpyAsync(s->vw, w.data(), sizeof(float2) * w.size(), cudaMemcpyHostToDevice, h->stream));
  if (!rim.empty()) {
    GCK(h, cudaMalloc(&s->vrim, sizeof(int2) * rim.size()));
    GCK(h, cudaMalloc(&s->vrim_acc, sizeof(double) * 2 * rim.size()));
    GCK(h, cudaMemcpyAsync(s->vrim, rim.data(), sizeof(int2) * rim.size(), cudaMemcpyHostToDevice, h->stream));
    GCK(h, cudaMemsetAsync(s->vrim_acc, 0, sizeof(double) * 2 * rim.size(), h->stream));
  }
  GCK(h, cudaStreamSynchronize(h->stream));  // the host vectors go out of scope
  s->vm = m;
  s->vrim_n = (int)rim.size();
  return TTI_OK;
}

// Row origin for the stress-half adjoint with the column work folded in: the
// highest of the image rows (free surface), the receiver rows and the stress
// source's window rows, so that every warp's rows hold all the column work
// below them; -1 when the free-surface rows would not fall in one warp.
int surface_origin(tti_handle *h, int *z_org, int *z_end)
{
  const Grid &g = h->g;
  const tti_config &c = h->cfg;
  int z = c.freesurface == 1 ? g.izStart - NH : g.izStart;
  int e = c.freesurface == 1 ? g.izStart + NH + 1 : 0;
  std::vector<int> rows;
  for (int k = 0; k < 3; ++k) {
    if (h->nrec[k] <= 0) continue;
    rows.resize(h->nrec[k]);
    GCK(h, cudaMemcpyAsync(rows.data(), h->d_rz[k], sizeof(int) * rows.size(), cudaMemcpyDeviceToHost, h->stream));
    GCK(h, cudaStreamSynchronize(h->stream));
    for (int r : rows) {
      z = std::min(z, r);
      e = std::max(e, r + 1);
    }
  }
  if (c.stype == 1 && h->nsrc > 0) {
    rows.resize(h->nsrc);
    GCK(h, cudaMemcpyAsync(rows.data(), h->d_sz, sizeof(int) * rows.size(), cudaMemcpyDeviceToHost, h->stream));
    GCK(h, cudaStreamSynchronize(h->stream));
    for (int r : rows) {
      z = std::min(z, std::max(0, r - NH));
      e = std::max(e, std::min(g.Nz, r + NH + 1));
    }
  }
  z = std::max(z, 0);
  *z_end = e;
  // the free-surface adjoint needs rows izStart - 5 .. izStart + 5 in the first warp's 32 rows
  *z_org = c.freesurface == 1 && z < g.izStart + NH + 1 - BZ ? -1 : z;
  return TTI_OK;
}

int launch_vsource(tti_handle *h, const AdjArgs &a, int it)
{
  GradState *s = h->grad;
  if (s->vm == 0) return TTI_OK;
  VSrcArgs v;
  v.g = h->g;
  v.lam0 = a.lam[0];
  v.lam1 = a.lam[1];
  for (int k = 0; k < 4; ++k) v.T[k] = a.T[k];
  v.cell = s->vcell;
  v.w = s->vw;
  v.rim = s->vrim;
  v.rim_acc = s->vrim_acc;
  v.m = s->vm;
  v.nsrc = h->nsrc;
  v.nrim = s->vrim_n;
  v.hx = a.hx;
  v.hz = a.hz;
  v.gsrc = s->gsrc;
  v.nt = h->cfg.nt;
  v.it = it;
  GCK(h, launch_pdl(k_adj_vsource, dim3(1), dim3(VSRC_THREADS), 0, h->stream, v));
  h->launches++;
  return TTI_OK;
}

// adjoint of forward step index n (time index it), segment slot `slot`
int adjoint_step(tti_handle *h, int n, int slot, const SourceTables &tab)
{
  const tti_config &c = h->cfg;
  GradState *s = h->grad;
  const int it = c.mode == 2 ? c.nt - 1 - n : n;
  const AdjArgs a = adj_args(h, slot);
  const Grid &g = h->g;
  // injection, source gradient and free-surface adjoint: folded into the
  // stress-half adjoint on the tiled path where its row origin covers them,
  // else one column-parallel launch before it
  SurfaceArgs sa;
  memset(&sa, 0, sizeof sa);
  sa.g = g;
  for (int k = 0; k < 8; ++k) sa.lam[k] = a.lam[k];
  const bool inject = c.seistype > 0 && it % c.mt == 0;
  bool any = false;
  for (int k = 0; k < 3; ++k) {
    const bool on = inject && s->res[k] && h->nrec[k] > 0;
    sa.colptr[k] = h->d_rcol[k];
    sa.rzs[k] = h->d_rzs[k];
    sa.rid[k] = h->d_rid[k];
    sa.res[k] = on ? s->res[k] + (size_t)(it / c.mt) * h->nrec[k] : nullptr;
    any = any || on;
  }
  const bool ssrc = h->nsrc > 0 && c.stype == 1;
  sa.src = SourceSet{ssrc ? h->nsrc : 0, h->d_sx, h->d_sz, h->d_src, c.nt};
  memcpy(sa.k1.k1, tab.k1, sizeof sa.k1.k1);
  sa.gsrc = s->gsrc;
  sa.it = it;
  sa.fs = c.freesurface == 1;
  sa.tensor = c.variant == TTI_TENSOR;
  const bool merged = h->use_tiled && s->surf_zorg >= 0;
  if ((any || ssrc || sa.fs) && !merged) {
    GCK(h, launch_pdl(k_adj_surface, dim3((g.Nx + 3) / 4), dim3(128), 0, h->stream, sa));
    h->launches++;
  }
  h->launches += 3;
  if (h->use_tiled) {  // TMA halo tiles (the per-cell kernels below serve TTIFD_KERNEL=naive)
    // the stress-half adjoint stays one thread per cell: with the kept strain
    // rates it has no stencil, only per-cell reads and writes
    const int z0 = merged ? s->surf_zorg : 0;
    const dim3 blk(BZ, BX), grd((g.Nz - z0 + BZ - 1) / BZ, (g.Nx + BX - 1) / BX);
    if (merged) {
      if (c.variant == TTI_BOND)
        GCK(h, launch_pdl(k_adj_stress_local<TTI_BOND, true, true>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
      else if (c.variant == TTI_TENSOR)
        GCK(h, launch_pdl(k_adj_stress_local<TTI_TENSOR, true, true>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
      else
        GCK(h, launch_pdl(k_adj_stress_local<TTI_COORDINATE, true, true>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
    } else {
      if (c.variant == TTI_BOND)
        GCK(h, launch_pdl(k_adj_stress_local<TTI_BOND, true, false>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
      else if (c.variant == TTI_TENSOR)
        GCK(h, launch_pdl(k_adj_stress_local<TTI_TENSOR, true, false>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
      else
        GCK(h, launch_pdl(k_adj_stress_local<TTI_COORDINATE, true, false>, grd, blk, 0, h->stream, a, sa, z0, s->surf_zend));
    }
    if (int rc = launch_vsource(h, a, it)) return rc;
    AdjTile at;
    memset(&at, 0, sizeof at);
    at.a = a;
    at.pk = packed::Packed{h->pk_cf, h->pk_vsc, h->pk_sc, h->pk_c4};
    at.err = h->d_flag;
    for (int k = 0; k < 4; ++k) at.map[k] = s->maps[k];
    if (c.variant == TTI_COORDINATE)
      GCK(h, launch_adj_tile(k_adj_velocity_tiled<TTI_COORDINATE>, at, 4, g.izStart, g, h->stream));
    else  // tensor and Bond: no rotation at the velocity node
      GCK(h, launch_adj_tile(k_adj_velocity_tiled<TTI_BOND>, at, 4, g.izStart, g, h->stream));
    for (int k = 0; k < 6; ++k) at.map[k] = s->maps[4 + k];
    GCK(h, launch_adj_tile(k_adj_vstencil_tiled, at, 4, a.z_lo, g, h->stream));
    return TTI_OK;
  }
  const dim3 blk(BZ, BX), grd((g.Nz + BZ - 1) / BZ, (g.Nx + BX - 1) / BX);
  if (c.variant == TTI_BOND) k_adj_stress_local<TTI_BOND, false, false><<<grd, blk, 0, h->stream>>>(a, sa, 0, 0);
  else if (c.variant == TTI_TENSOR) k_adj_stress_local<TTI_TENSOR, false, false><<<grd, blk, 0, h->stream>>>(a, sa, 0, 0);
  else k_adj_stress_local<TTI_COORDINATE, false, false><<<grd, blk, 0, h->stream>>>(a, sa, 0, 0);
  if (int rc = launch_vsource(h, a, it)) return rc;
  if (c.variant == TTI_COORDINATE) k_adj_velocity<TTI_COORDINATE><<<grd, blk, 0, h->stream>>>(a);
  else k_adj_velocity<TTI_BOND><<<grd, blk, 0, h->stream>>>(a);  // tensor and Bond: no rotation at the velocity node
  k_adj_velocity_stencil<<<grd, blk, 0, h->stream>>>(a);
  GCK(h, cudaGetLastError());
  return TTI_OK;
}

}  // namespace

namespace ttifd {
void grad_release(tti_handle *h)
{
  GradState *s = h->grad;
  if (!s) return;
  for (auto p : s->lam) cudaFree(p);
  for (auto p : s->T) cudaFree(p);
  for (auto p : s->TV) cudaFree(p);
  for (auto p : s->acc) cudaFree(p);
  for (auto p : s->out) cudaFree(p);
  for (auto p : s->obs) cudaFree(p);
  for (auto p : s->res) cudaFree(p);
  cudaFree(s->ckpt);
  cudaFree(s->keep);
  cudaFree(s->gsrc);
  cudaFree(s->vcell);
  cudaFree(s->vw);
  cudaFree(s->vrim);
  cudaFree(s->vrim_acc);
  cudaFree(s->d_J);
  free(s->maps);
  delete s;
  h->grad = nullptr;
}
}  // namespace ttifd

extern "C" {

int tti_grad_set_observed(tti_handle *h, int kind, const float *dobs)
{
  if (!h || kind < 0 || kind > 2 || !dobs) return TTI_ERR_ARG;
  int rc = grad_check(h);
  if (rc) return rc;
  if (h->nrec[kind] <= 0) return gerr(h, TTI_ERR_STATE, "set the receivers of this component first");
  GCK(h, cudaSetDevice(h->device));
  if ((rc = grad_alloc(h))) return rc;
  GradState *s = h->grad;
  const int n = h->nrec[kind], nts = h->nts;
  cudaFree(s->obs[kind]);
  cudaFree(s->res[kind]);
  s->obs[kind] = s->res[kind] = nullptr;
  GCK(h, cudaMalloc(&s->obs[kind], sizeof(float) * (size_t)n * nts));
  GCK(h, cudaMalloc(&s->res[kind], sizeof(float) * (size_t)n * nts));
  std::vector<float> tm((size_t)n * nts);  // [ntrace][nts] -> time-major
  for (int r = 0; r < n; ++r)
    for (int t = 0; t < nts; ++t) tm[(size_t)t * n + r] = dobs[(size_t)r * nts + t];
  GCK(h, cudaMemcpy(s->obs[kind], tm.data(), sizeof(float) * tm.size(), cudaMemcpyHostToDevice));
  s->have_obs[kind] = true;
  return TTI_OK;
}

int tti_grad_zero(tti_handle *h)
{
  if (!h) return TTI_ERR_ARG;
  int rc = grad_check(h);
  if (rc) return rc;
  GCK(h, cudaSetDevice(h->device));
  if ((rc = grad_alloc(h))) return rc;
  for (auto p : h->grad->acc) GCK(h, cudaMemsetAsync(p, 0, h->g.n * sizeof(float), h->stream));
  GCK(h, cudaStreamSynchronize(h->stream));
  return TTI_OK;
}

}  // extern "C"

namespace {

// Buffers and tables of a gradient run: `slots` full-state checkpoints and a
// kept segment of `seg` steps (keep_fields each); the source tables in *tab.
int grad_prepare(tti_handle *h, int slots, int seg, SourceTables *tab)
{
  int rc = grad_check(h);
  if (rc) return rc;
  GCK(h, cudaSetDevice(h->device));
  if ((rc = grad_alloc(h))) return rc;
  GradState *s = h->grad;
  const tti_config &c = h->cfg;
  const bool want_v = c.seistype == 1 || c.seistype == 3, want_p = c.seistype == 2 || c.seistype == 3;
  for (int k = 0; k < 3; ++k) {
    const bool rec = (k < 2 ? want_v : want_p) && h->nrec[k] > 0;
    if (rec && !s->have_obs[k]) return gerr(h, TTI_ERR_STATE, "observed traces missing for a recorded component");
  }
  const int nf = h->cfg.variant == TTI_TENSOR ? 8 : 5;  // fields of a full state (checkpoints)
  const int nk = keep_fields(h);                       // fields of a kept step
  const size_t n = h->g.n;
  if (s->ncheck != slots + 1 || s->seg != seg || s->nkeep != nk) {
    cudaFree(s->ckpt);
    cudaFree(s->keep);
    s->ckpt = s->keep = nullptr;
    if (cudaMalloc(&s->ckpt, sizeof(float) * nf * n * std::max(1, slots)) != cudaSuccess ||
        cudaMalloc(&s->keep, sizeof(float) * nk * n * seg) != cudaSuccess) {
      cudaGetLastError();
      cudaFree(s->ckpt);  // nothing half-allocated stays behind; the handle stays usable
      cudaFree(s->keep);
      s->ckpt = s->keep = nullptr;
      s->ncheck = s->seg = s->nkeep = 0;
      return gerr(h, TTI_ERR_NOMEM, "device allocation of the checkpoints failed (use fewer steps per segment)");
    }
    s->ncheck = slots + 1;
    s->seg = seg;
    s->nkeep = nk;
  }
  const int nt = c.nt;
  if (s->gsrc_n != h->nsrc * nt) {
    cudaFree(s->gsrc);
    s->gsrc = nullptr;
    s->gsrc_n = 0;
    if (h->nsrc > 0) GCK(h, cudaMalloc(&s->gsrc, sizeof(float) * (size_t)h->nsrc * nt));
    s->gsrc_n = h->nsrc * nt;
  }
  handle_source_tables(h, tab);
  if ((rc = vsource_tables(h, *tab))) return rc;
  return surface_origin(h, &s->surf_zorg, &s->surf_zend);
}

// Residuals d - dobs of every recorded component and J (read back into *J at
// the end of the run), then the adjoint state zeroed.
int grad_start_adjoint(tti_handle *h, double *J)
{
  GradState *s = h->grad;
  const tti_config &c = h->cfg;
  const bool want_v = c.seistype == 1 || c.seistype == 3, want_p = c.seistype == 2 || c.seistype == 3;
  const size_t n = h->g.n;
  GCK(h, cudaMemsetAsync(s->d_J, 0, sizeof(double), h->stream));
  for (int k = 0; k < 3; ++k) {
    const bool rec = (k < 2 ? want_v : want_p) && h->nrec[k] > 0;
    if (!rec) continue;
    const size_t m = (size_t)h->nrec[k] * h->nts;
    k_residual<<<std::min<size_t>(1024, (m + 255) / 256), 256, 0, h->stream>>>(h->d_rec[k], s->obs[k], s->res[k], m,
                                                                               s->d_J);
  }
  GCK(h, cudaMemcpyAsync(J, s->d_J, sizeof(double), cudaMemcpyDeviceToHost, h->stream));
  for (auto p : s->lam)
    if (p) GCK(h, cudaMemsetAsync(p, 0, n * sizeof(float), h->stream));
  for (auto p : s->T) GCK(h, cudaMemsetAsync(p, 0, n * sizeof(float), h->stream));
  if (s->gsrc) GCK(h, cudaMemsetAsync(s->gsrc, 0, sizeof(float) * (size_t)s->gsrc_n, h->stream));
  for (auto p : s->TV) GCK(h, cudaMemsetAsync(p, 0, n * sizeof(float), h->stream));
  return TTI_OK;
}

// forward steps k0 .. k1-1 from the current state; `record`: what the adjoint
// needs of each step goes to the kept segment (slot k - k0)
int forward_steps(tti_handle *h, int k0, int k1, bool record, const SourceTables &tab)
{
  GradState *s = h->grad;
  const int nk = s->nkeep;
  for (int k = k0; k < k1; ++k) {
    float *keep[8] = {};
    if (record)
      for (int f = 0; f < nk; ++f) keep[f] = s->keep + ((size_t)(k - k0) * nk + f) * h->g.n;
    const int rc = handle_step(h, tab, record ? keep : nullptr);
    if (rc) return rc;
  }
  return TTI_OK;
}

int adjoint_steps(tti_handle *h, int k0, int k1, const SourceTables &tab)
{
  for (int k = k1 - 1; k >= k0; --k) {
    const int rc = adjoint_step(h, k, k - k0, tab);
    if (rc) return rc;
  }
  return TTI_OK;
}

int nfull(const tti_handle *h) { return h->cfg.variant == TTI_TENSOR ? 8 : 5; }

int store_state(tti_handle *h, int slot)
{
  const size_t n = h->g.n;
  for (int f = 0; f < nfull(h); ++f)
    GCK(h, cudaMemcpyAsync(h->grad->ckpt + ((size_t)slot * nfull(h) + f) * n, h->fld[f], n * sizeof(float),
                           cudaMemcpyDeviceToDevice, h->stream));
  return TTI_OK;
}

// the state of step `step` from checkpoint `slot` (slot < 0: the zero state of step 0)
int restore_state(tti_handle *h, int slot, int step)
{
  const size_t n = h->g.n;
  for (int f = 0; f < nfull(h); ++f) {
    if (slot < 0) GCK(h, cudaMemsetAsync(h->fld[f], 0, n * sizeof(float), h->stream));
    else
      GCK(h, cudaMemcpyAsync(h->fld[f], h->grad->ckpt + ((size_t)slot * nfull(h) + f) * n, n * sizeof(float),
                             cudaMemcpyDeviceToDevice, h->stream));
  }
  h->step_index = step;
  return TTI_OK;
}

int grad_finish(tti_handle *h, const double &J, double *misfit)
{
  GCK(h, cudaEventRecord(h->ev1, h->stream));
  GCK(h, cudaEventSynchronize(h->ev1));
  GCK(h, cudaEventElapsedTime(&h->last_ms, h->ev0, h->ev1));
  h->step_index = h->cfg.nt;
  if (misfit) *misfit = J;
  return handle_check_flag(h);
}

}  // namespace

namespace ttifd {

// One step of a gradient run's checkpoint schedule (macro-steps a .. b-1).
struct Action {
  enum Kind { ADVANCE, STORE, RESTORE, RECORD, START_ADJOINT, ADJOINT } kind;
  int a, b, slot;
};

struct BinomialPlan {
  int M, S;
  std::vector<long long> T;  // T(l, c) at [c][l]
  std::vector<int> D;        // best first split at [c][l]
  BinomialPlan(int M_, int S_);
  long long &t(int c, int l) { return T[(size_t)c * (M + 1) + l]; }
  int &d(int c, int l) { return D[(size_t)c * (M + 1) + l]; }
  int dd(int c, int l) const { return D[(size_t)c * (M + 1) + l]; }
  void actions(std::vector<Action> &out) const;
};

// Binomial checkpointing (Griewank and Walther's Revolve, ACM TOMS 26(1), 2000),
// stated here as its recursion. M macro-steps are reversed with S checkpoint
// slots; the state at macro-step a is held (in a slot, or the zero state at
// a = 0). reverse(a, b, c): if b - a = 1, restore x_a, record the macro-step
// (forward keeping what its adjoint needs) and run its adjoint; if c = 0,
// the same for each i = b-1 .. a after advancing from x_a to x_i; otherwise
// advance to a + d, store that state in a free slot, reverse(a + d, b, c - 1),
// release the slot and reverse(a, a + d, c). With T(l, c) the macro-steps
// advanced (recording excluded) to reverse l of them with c free slots,
//   T(l, 0) = l (l - 1) / 2,   T(1, c) = 0,
//   T(l, c) = min_d  d + T(l - d, c - 1) + T(d, c),
// an objective convex in d, so the best split is where its forward difference
// turns non-negative (a binary search). The table costs O(M S log M) time.
BinomialPlan::BinomialPlan(int M_, int S_) : M(M_), S(std::max(0, S_))
{
  T.assign((size_t)(S + 1) * (M + 1), 0);
  D.assign((size_t)(S + 1) * (M + 1), 0);
  for (int l = 1; l <= M; ++l) t(0, l) = (long long)l * (l - 1) / 2;
  for (int c = 1; c <= S; ++c) {
    t(c, 1) = 0;
    for (int l = 2; l <= M; ++l) {
      auto f = [&](int d) { return d + t(c - 1, l - d) + t(c, d); };
      int lo = 1, hi = l - 1;  // smallest d with f(d + 1) >= f(d)
      while (lo < hi) {
        const int mid = (lo + hi) / 2;
        if (f(mid + 1) >= f(mid)) hi = mid;
        else lo = mid + 1;
      }
      t(c, l) = f(lo);
      d(c, l) = lo;
    }
  }
}

void BinomialPlan::actions(std::vector<Action> &out) const
{
  struct Rec {
    const BinomialPlan &p;
    std::vector<Action> &out;
    std::vector<char> used;
    int cur = -1;  // macro-step whose start state is in the wavefields (-1: unknown)
    bool first = true;
    void emit(Action::Kind k, int a = 0, int b = 0, int slot = -1) { out.push_back(Action{k, a, b, slot}); }
    void go(int a, int b, int c, int slot_a)
    {
      const int l = b - a;
      if (l == 1 || c == 0) {
        for (int i = b - 1; i >= a; --i) {
          if (cur != i) {
            if (cur != a) emit(Action::RESTORE, a, 0, slot_a);
            if (i > a) emit(Action::ADVANCE, a, i);
          }
          emit(Action::RECORD, i, i + 1);
          if (first) {
            emit(Action::START_ADJOINT);
            first = false;
          }
          emit(Action::ADJOINT, i, i + 1);
          cur = i + 1;  // the recording left the state of macro-step i + 1
        }
        return;
      }
      const int m = a + p.dd(c, l);
      if (cur != a) emit(Action::RESTORE, a, 0, slot_a);
      emit(Action::ADVANCE, a, m);
      int k = 0;
      while (used[k]) ++k;
      used[k] = 1;
      emit(Action::STORE, m, 0, k);
      cur = m;
      go(m, b, c - 1, k);
      used[k] = 0;
      go(a, m, c, slot_a);
    }
  } r{*this, out, std::vector<char>(S + 1, 0)};
  r.cur = 0;  // the run starts from the zero state of step 0
  if (M > 0) r.go(0, M, S, -1);
}

}  // namespace ttifd

extern "C" {

long long tti_grad_schedule_cost(int macro_steps, int snapshots)
{
  if (macro_steps < 1 || snapshots < 0) return -1;
  const ttifd::BinomialPlan p(macro_steps, snapshots);
  std::vector<ttifd::Action> acts;
  p.actions(acts);
  long long adv = 0;
  for (const auto &a : acts)
    if (a.kind == ttifd::Action::ADVANCE) adv += a.b - a.a;
  return adv;
}

int tti_grad_plan(const tti_handle *h, double budget_bytes, int *snapshots, int *keep_steps, long long *forward_steps)
{
  if (!h || !snapshots || !keep_steps) return TTI_ERR_ARG;
  const int nt = h->cfg.nt;
  const double state = (double)(h->cfg.variant == TTI_TENSOR ? 8 : 5) * h->g.n * sizeof(float);
  const double kept = (double)keep_fields(h) * h->g.n * sizeof(float);
  // macro-step lengths on a geometric grid; the slots left over for each
  long long best = -1;
  int bs = 0, bl = 0;
  // (the last candidate is nt itself: one macro-step, every step kept)
  for (int L = 1; L <= nt; L = L == nt ? nt + 1 : std::min(nt, std::max(L + 1, (int)(L * 1.25)))) {
    const int M = (nt + L - 1) / L;
    if (M > 4000) continue;  // keeps the cost table small; longer macro-steps come next
    const double left = budget_bytes - L * kept;
    if (left < 0) break;  // longer macro-steps need still more memory
    int s = (int)std::min<double>(M - 1, std::floor(left / state));
    long long adv;
    if (s >= M - 1) {
      adv = M - 1;  // every macro-step start stored in one sweep
    } else {
      s = std::min(s, 256);  // beyond that, more slots save little (and the table grows)
      adv = ttifd::BinomialPlan(M, s).t(s, M);
    }
    const long long cost = adv * L + nt;  // advances plus one recording pass
    if (best < 0 || cost < best) {
      best = cost;
      bs = s;
      bl = L;
    }
  }
  if (best < 0)
    return gerr(const_cast<tti_handle *>(h), TTI_ERR_NOMEM,
                "the memory budget holds no kept step: no checkpoint schedule fits");
  *snapshots = bs;
  *keep_steps = bl;
  if (forward_steps) *forward_steps = best;
  return TTI_OK;
}

int tti_grad_run(tti_handle *h, int ncheck, double *misfit)
{
  if (!h || ncheck < 1) return TTI_ERR_ARG;
  const int nt = h->cfg.nt;
  ncheck = std::min(ncheck, nt);
  const int seg = (nt + ncheck - 1) / ncheck, nseg = (nt + seg - 1) / seg;
  SourceTables tab;
  int rc = grad_prepare(h, nseg - 1, seg, &tab);
  if (rc) return rc;
  // pass 1: forward with a checkpoint at every segment start but the last,
  // whose states are kept directly (ncheck = 1: all states, no recomputation)
  if ((rc = tti_reset(h))) return rc;
  GCK(h, cudaEventRecord(h->ev0, h->stream));
  for (int q = 0; q < nseg; ++q) {
    const bool last = q == nseg - 1;
    if (!last && (rc = store_state(h, q))) return rc;
    if ((rc = forward_steps(h, q * seg, std::min(nt, (q + 1) * seg), last, tab))) return rc;
  }
  double J = 0.0;
  if ((rc = grad_start_adjoint(h, &J))) return rc;
  // adjoint, segment by segment from the last
  for (int q = nseg - 1; q >= 0; --q) {
    const int k0 = q * seg, k1 = std::min(nt, (q + 1) * seg);
    if (q < nseg - 1) {  // recompute the segment from its checkpoint
      if ((rc = restore_state(h, q, k0))) return rc;
      if ((rc = forward_steps(h, k0, k1, true, tab))) return rc;
    }
    if ((rc = adjoint_steps(h, k0, k1, tab))) return rc;
  }
  return grad_finish(h, J, misfit);
}

int tti_grad_run_binomial(tti_handle *h, int snapshots, int keep_steps, double *misfit)
{
  if (!h || snapshots < 0 || keep_steps < 1) return TTI_ERR_ARG;
  const int nt = h->cfg.nt;
  keep_steps = std::min(keep_steps, nt);
  const int M = (nt + keep_steps - 1) / keep_steps;
  snapshots = std::min(snapshots, M - 1);
  SourceTables tab;
  int rc = grad_prepare(h, snapshots, keep_steps, &tab);
  if (rc) return rc;
  const BinomialPlan plan(M, snapshots);
  std::vector<Action> acts;
  plan.actions(acts);
  auto step_of = [&](int macro) { return std::min(nt, macro * keep_steps); };
  if ((rc = tti_reset(h))) return rc;
  GCK(h, cudaEventRecord(h->ev0, h->stream));
  double J = 0.0;
  for (const Action &a : acts) {
    switch (a.kind) {
    case Action::ADVANCE: rc = forward_steps(h, step_of(a.a), step_of(a.b), false, tab); break;
    case Action::STORE: rc = store_state(h, a.slot); break;
    case Action::RESTORE: rc = restore_state(h, a.slot, step_of(a.a)); break;
    case Action::RECORD: rc = forward_steps(h, step_of(a.a), step_of(a.b), true, tab); break;
    case Action::START_ADJOINT: rc = grad_start_adjoint(h, &J); break;
    case Action::ADJOINT: rc = adjoint_steps(h, step_of(a.a), step_of(a.b), tab); break;
    }
    if (rc) return rc;
  }
  return grad_finish(h, J, misfit);
}

int tti_grad_fetch(tti_handle *h, int which, float *out)
{
  if (!h || !out || which < 0 || which > 3) return TTI_ERR_ARG;
  if (!h->grad) return gerr(h, TTI_ERR_STATE, "no gradient computed");
  GCK(h, cudaSetDevice(h->device));
  GradState *s = h->grad;
  const Grid &g = h->g;
  const dim3 blk(BZ, BX), grd((g.Nz + BZ - 1) / BZ, (g.Nx + BX - 1) / BX);
  const float *th = h->m_theta;
  if (h->cfg.variant == TTI_TENSOR)
    k_chain<TTI_TENSOR><<<grd, blk, 0, h->stream>>>(g, handle_step_args(h).p, h->par[TTI_P_VP], h->par[TTI_P_VS],
                                                    h->par[TTI_P_RHO], h->par[TTI_P_BETA], h->m_eps, h->m_delta, th,
                                                    *s, h->cfg.scalar, h->cfg.freesurface);
  else if (h->cfg.variant == TTI_BOND)
    k_chain<TTI_BOND><<<grd, blk, 0, h->stream>>>(g, handle_step_args(h).p, h->par[TTI_P_VP], h->par[TTI_P_VS],
                                                  h->par[TTI_P_RHO], h->par[TTI_P_BETA], h->m_eps, h->m_delta, th,
                                                  *s, h->cfg.scalar, h->cfg.freesurface);
  else
    k_chain<TTI_COORDINATE><<<grd, blk, 0, h->stream>>>(g, handle_step_args(h).p, h->par[TTI_P_VP],
                                                        h->par[TTI_P_VS], h->par[TTI_P_RHO], h->par[TTI_P_BETA],
                                                        h->m_eps, h->m_delta, th, *s, h->cfg.scalar, h->cfg.freesurface);
  h->launches++;
  GCK(h, cudaGetLastError());
  GCK(h, cudaMemcpy2DAsync(out, (size_t)g.Nz * sizeof(float), s->out[which], (size_t)g.ldz * sizeof(float),
                           (size_t)g.Nz * sizeof(float), g.Nx, cudaMemcpyDeviceToHost, h->stream));
  GCK(h, cudaStreamSynchronize(h->stream));
  return TTI_OK;
}

int tti_grad_fetch_source(tti_handle *h, float *out)
{
  if (!h || !out) return TTI_ERR_ARG;
  if (!h->grad || !h->grad->gsrc) return gerr(h, TTI_ERR_STATE, "no source gradient computed");
  GCK(h, cudaSetDevice(h->device));
  GCK(h, cudaMemcpy(out, h->grad->gsrc, sizeof(float) * (size_t)h->grad->gsrc_n, cudaMemcpyDeviceToHost));
  return TTI_OK;
}

int tti_grad_accumulators(tti_handle *h, float **dev, size_t *count, size_t *pitch)
{
  if (!h || !dev) return TTI_ERR_ARG;
  if (!h->grad) return gerr(h, TTI_ERR_STATE, "no gradient buffers");
  for (int k = 0; k < 7; ++k) dev[k] = h->grad->acc[k];
  if (count) *count = h->g.n;
  if (pitch) *pitch = h->g.ldz;
  return TTI_OK;
}

}  // extern "C"
