// Tiled half-step kernels: the velocity update (coord:614-672, tensor:617-666,
// bond:654-703) and the stress update (coord:804-845, tensor:799-851 with the
// sigma = R tau pass fused, bond:836-873), each in place.
//
// A CTA owns a tile of TZ = 128 rows and TX = 16 columns. One elected thread
// loads the tile plus the stencil halo of every input field with a 2D TMA copy
// (cp.async.bulk.tensor, completion on an mbarrier, bounded wait); the box
// starts at row z0 - 8 so its innermost coordinate stays 16-byte aligned, and
// coordinates outside the array read zeros. Every stencil tap is then a
// shared-memory load at a compile-time offset from the thread's own cell.
// Each thread updates one row of TX / 4 columns (a warp's shared loads touch 32
// consecutive words); per-cell parameters are plain coalesced loads whose
// latency is hidden by 64 resident warps per SM (32 registers per thread).
// The velocity kernel reads only stress and the stress kernel only velocity
// from the tiles, so in-place updates are race-free.
#include <cudaTypedefs.h>

#include <algorithm>
#include <cstring>
#include <mutex>

#include "tiled.cuh"

namespace ttifd {
namespace tiled {

namespace {

// tile cells handled by a thread: row zr, columns xc .. xc + TX/4 - 1
struct Cells {
  int x0, z0, xc, zr;
};
__device__ __forceinline__ Cells cells_of(const HalfArgs &a, int tz, int tx)
{
  const int t = threadIdx.x;
  Cells c;
  c.z0 = a.z_base + tz * TZ;
  c.x0 = a.x_base + tx * TX;
  c.xc = c.x0 + (TX / 4) * (t >> 7);
  c.zr = c.z0 + (t & 127);
  return c;
}

// true when every cell of the tile lies where coef1 = 1 and coef2 = dt
__device__ __forceinline__ bool tile_undamped(const HalfArgs &a, const Cells &c)
{
  const Grid &g = a.g;
  return a.undamped_ok && c.x0 >= g.E && c.x0 + TX <= g.Nx - g.E && c.z0 >= (a.freesurface ? 0 : g.E) &&
         c.z0 + TZ <= g.Nz - g.E;
}

// Velocity update of tile (tz, tx); `map` holds the tensor maps of sxx, szz, sxz.
// Q (FMA mode, dx == dz): the coefficients carry h = 0.5 / dx, so a derivative
// is d1 + d2 or d1 - d2 without a product.
template <bool Q>
__device__ __forceinline__ float coef(const HalfArgs &a, int k)
{
  return Q ? a.hc[k] : rsg(k);
}

// While the halo boxes are in flight, lanes of each warp ask L2 for the
// per-cell lines the velocity update reads after the wait (vx, vz, invrho,
// coef1/coef2 outside the undamped interior, sin/cos theta_v for the
// coordinate rotation): the warp's 32 rows are one 128-byte line per column
// and array (two for the float2 arrays).
template <bool ROT>
__device__ __forceinline__ void prefetch_cells(const HalfArgs &a, const Cells &c, bool und)
{
  const int lane = threadIdx.x & 31, col = lane >> 3, k = lane & 7;
  const int x = c.xc + col, z = c.zr - lane;  // the warp's first row
  if (col >= TX / 4 || x >= a.g.Nx - NH || z >= a.g.Nz - NH) return;
  const size_t gi = (size_t)x * a.g.ldz + z;
  const void *p = nullptr;
  switch (k) {
  case 0: p = a.f.vx + gi; break;
  case 1: p = a.f.vz + gi; break;
  case 2: p = a.p.invrho + gi; break;
  case 3: p = und ? nullptr : (const void *)(a.pk.cf + gi); break;
  case 4: p = und ? nullptr : (const void *)(a.pk.cf + gi + 16); break;
  case 5: p = ROT ? (const void *)(a.pk.vsc + gi) : nullptr; break;
  case 6: p = ROT ? (const void *)(a.pk.vsc + gi + 16) : nullptr; break;
  default: break;
  }
  if (p) asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
}

// per-cell inputs of the velocity update
struct VCell {
  float vx0, vz0, c1, c2, ir;
};

__device__ __forceinline__ void load_vcell(const HalfArgs &a, bool und, size_t gi, VCell &o)
{
  o.vx0 = a.f.vx[gi];
  o.vz0 = a.f.vz[gi];
  o.c1 = 1.0f;
  o.c2 = a.dt;
  if (!und) {
    const float2 cf = __ldg(a.pk.cf + gi);
    o.c1 = cf.x;
    o.c2 = cf.y;
  }
  o.ir = __ldg(a.p.invrho + gi);
}

// The velocity update of one cell from its stencil sums d[f] = (d1, d2) of
// sxx, szz, sxz (coord:614-672, tensor:617-666, bond:654-703).
template <int V, bool X, bool Q, bool K>
__device__ __forceinline__ void velocity_store(const HalfArgs &a, size_t gi, const float (&d)[3][2], const VCell &p)
{
  using A = Ar<X>;
  const float invdx = a.invdx, invdz = a.invdz;
  // x and z derivatives 0.5 (d1 +- d2) / dx, / dz (already scaled when Q)
  auto dx_ = [&](int f) { return Q ? d[f][0] + d[f][1] : A::mul(A::mul(0.5f, A::add(d[f][0], d[f][1])), invdx); };
  auto dz_ = [&](int f, float inv) {
    return Q ? d[f][0] - d[f][1] : A::mul(A::mul(0.5f, A::sub(d[f][0], d[f][1])), inv);
  };
  const float sxx_x = dx_(0);
  const float szz_z = dz_(1, invdz);
  const float sxz_x = dx_(2);
  const float sxz_z = dz_(2, invdz);
  const float br = A::mul(p.c2, p.ir);
  float fx, fz;
  if (V == TTI_COORDINATE) {
    const float2 sc = __ldg(a.pk.vsc + gi);
    const float sv = sc.x, cv = sc.y;
    const float sxx_z = dz_(0, invdx);  // invdx as coord:633
    const float szz_x = dx_(1);
    fx = A::add(A::add(A::sub(A::mul(cv, sxx_x), A::mul(sv, sxx_z)), A::mul(sv, sxz_x)), A::mul(cv, sxz_z));
    fz = A::add(A::add(A::sub(A::mul(cv, sxz_x), A::mul(sv, sxz_z)), A::mul(sv, szz_x)), A::mul(cv, szz_z));
    if (K) {
      a.kd[0][gi] = sxz_x - sxx_z;
      a.kd[1][gi] = szz_x - sxz_z;
      a.kd[2][gi] = sxx_x + sxz_z;
      a.kd[3][gi] = sxz_x + szz_z;
    }
  } else {
    fx = A::add(sxx_x, sxz_z);
    fz = A::add(sxz_x, szz_z);
  }
  a.f.vx[gi] = A::add(A::mul(p.c1, p.vx0), A::mul(br, fx));
  a.f.vz[gi] = A::add(A::mul(p.c1, p.vz0), A::mul(br, fz));
}

// PB (a CTA that runs tile after tile): the boxes complete phase ph of the
// CTA's barrier pbar, initialised once; otherwise the tile initialises its own
// barrier after the boxes.
template <int V, bool X, bool Q, bool K = false, bool PB = false>
__device__ __forceinline__ void velocity_tile(const HalfArgs &a, const CUtensorMap *map, float *sm, int tz, int tx,
                                              unsigned long long *pbar = nullptr, int ph = 0)
{
  using A = Ar<X>;
  unsigned long long *bar = PB ? pbar : reinterpret_cast<unsigned long long *>(sm + 3 * FIELD);
  const Grid &g = a.g;
  const Cells c = cells_of(a, tz, tx);
  tma::issue_tiles(map, sm, bar, 3, c.z0, c.x0, 4, PB ? ph : -1);
  const int L = g.ldz;
  const bool und = tile_undamped(a, c);
  const int z = c.zr;
  const bool zin = z >= g.izStart && z < g.Nz - NH;
  prefetch_cells<V == TTI_COORDINATE>(a, c, und);
  if (!tma::wait_tiles(a.err, bar, a.wait_limit, PB ? (unsigned)ph : 0u)) return;
  if (!zin) return;
#pragma unroll
  for (int i = 0; i < TX / 4; ++i) {
    const int x = c.xc + i;
    if (x >= g.Nx - NH) break;
    const size_t gi = (size_t)x * L + z;
    VCell p;
    load_vcell(a, und, gi, p);
    // stress value at column x+m, row z+n: s[f * FIELD + m * BZ + n]
    const float *s = sm + (x - c.x0 + 4) * BZ + (z - c.z0 + 8);
    float d[3][2];
#pragma unroll
    for (int f = 0; f < 3; ++f) {
      const float *q = s + f * FIELD;
      // d1 = sum C_k (s[x+k][z+k] - s[x-k+1][z-k+1]); d2 = sum C_k (s[x+k][z-k+1] - s[x-k+1][z+k])
      float s1 = A::mul(coef<Q>(a, 0), A::sub(q[BZ + 1], q[0]));
      float s2 = A::mul(coef<Q>(a, 0), A::sub(q[BZ], q[1]));
#pragma unroll
      for (int k = 2; k <= NH; ++k) {
        s1 = A::add(s1, A::mul(coef<Q>(a, k - 1), A::sub(q[k * BZ + k], q[(1 - k) * BZ + 1 - k])));
        s2 = A::add(s2, A::mul(coef<Q>(a, k - 1), A::sub(q[k * BZ + 1 - k], q[(1 - k) * BZ + k])));
      }
      d[f][0] = s1;
      d[f][1] = s2;
    }
    velocity_store<V, X, Q, K>(a, gi, d, p);
  }
}

// per-cell inputs of the stress update
struct SCell {
  float c1, c2, s2t, o0, o1, o2;  // o*: sigma (coordinate, Bond) or tau (tensor)
  float4 c4;
  float2 sc;
};

template <int V>
__device__ __forceinline__ void load_scell(const HalfArgs &a, bool und, size_t gi, SCell &o)
{
  if (und) {
    o.c1 = 1.0f;
    o.c2 = a.dt;
  } else {
    const float2 cf = __ldg(a.pk.cf + gi);
    o.c1 = cf.x;
    o.c2 = cf.y;
  }
  o.c4 = __ldg(a.pk.c4 + gi);
  o.sc = __ldg(a.pk.sc + gi);
  if (V == TTI_TENSOR) {
    o.s2t = __ldg(a.p.s2t + gi);
    o.o0 = a.f.txx[gi];
    o.o1 = a.f.tzz[gi];
    o.o2 = a.f.txz[gi];
  } else {
    o.o0 = a.f.sxx[gi];
    o.o1 = a.f.szz[gi];
    o.o2 = a.f.sxz[gi];
  }
}

template <int V, bool X>
__device__ __forceinline__ void stress_store(const HalfArgs &a, size_t gi, float vxx, float vxz, float vzx, float vzz,
                                             const SCell &p)
{
  using A = Ar<X>;
  const float c1 = p.c1, c2 = p.c2;
  const float c11 = p.c4.x, c13 = p.c4.y, c33 = p.c4.z, c55 = p.c4.w;
  if (V == TTI_COORDINATE) {
    const float sn = p.sc.x, cs = p.sc.y;
    float q = A::add(A::mul(sn, vxx), A::mul(cs, vxz));
    vxx = A::sub(A::mul(cs, vxx), A::mul(sn, vxz));
    vxz = q;
    q = A::add(A::mul(sn, vzx), A::mul(cs, vzz));
    vzx = A::sub(A::mul(cs, vzx), A::mul(sn, vzz));
    vzz = q;
    a.f.sxx[gi] = A::add(A::mul(c1, p.o0), A::mul(c2, A::add(A::mul(c11, vxx), A::mul(c13, vzz))));
    a.f.szz[gi] = A::add(A::mul(c1, p.o1), A::mul(c2, A::add(A::mul(c13, vxx), A::mul(c33, vzz))));
    a.f.sxz[gi] = A::add(A::mul(c1, p.o2), A::mul(A::mul(c2, c55), A::add(vzx, vxz)));
  } else if (V == TTI_TENSOR) {
    const float s2 = p.sc.x, cc2 = p.sc.y, s2t = p.s2t;
    const float sh = A::add(vxz, vzx);
    const float exx = A::sub(A::add(A::mul(cc2, vxx), A::mul(s2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
    const float ezz = A::add(A::add(A::mul(s2, vxx), A::mul(cc2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
    const float exz = A::add(A::mul(s2t, A::sub(vxx, vzz)), A::mul(A::sub(cc2, s2), sh));
    const float ntx = A::add(A::mul(c1, p.o0), A::mul(c2, A::add(A::mul(c11, exx), A::mul(c13, ezz))));
    const float ntz = A::add(A::mul(c1, p.o1), A::mul(c2, A::add(A::mul(c13, exx), A::mul(c33, ezz))));
    const float ntq = A::add(A::mul(c1, p.o2), A::mul(A::mul(c2, c55), exz));
    a.f.txx[gi] = ntx;
    a.f.tzz[gi] = ntz;
    a.f.txz[gi] = ntq;
    a.f.sxx[gi] = A::add(A::add(A::mul(cc2, ntx), A::mul(s2, ntz)), A::mul(s2t, ntq));
    a.f.szz[gi] = A::sub(A::add(A::mul(s2, ntx), A::mul(cc2, ntz)), A::mul(s2t, ntq));
    a.f.sxz[gi] = A::add(A::mul(A::mul(-0.5f, s2t), A::sub(ntx, ntz)), A::mul(A::sub(cc2, s2), ntq));
  } else {
    const float c15 = p.sc.x, c35 = p.sc.y;
    const float sh = A::add(vzx, vxz);
    a.f.sxx[gi] =
        A::add(A::mul(c1, p.o0), A::mul(c2, A::add(A::add(A::mul(c11, vxx), A::mul(c13, vzz)), A::mul(c15, sh))));
    a.f.szz[gi] =
        A::add(A::mul(c1, p.o1), A::mul(c2, A::add(A::add(A::mul(c13, vxx), A::mul(c33, vzz)), A::mul(c35, sh))));
    a.f.sxz[gi] =
        A::add(A::mul(c1, p.o2), A::mul(c2, A::add(A::add(A::mul(c15, vxx), A::mul(c35, vzz)), A::mul(c55, sh))));
  }
}

// The stress update of one cell from its stencil sums d[f] = (d1, d2) of vx,
// vz: the strain rates, what the gradient keeps of them, then stress_store.
template <int V, bool X, bool Q, bool K>
__device__ __forceinline__ void stress_finish(const HalfArgs &a, size_t gi, const float (&d)[2][2], const SCell &p)
{
  using A = Ar<X>;
  const float invdx = a.invdx, invdz = a.invdz;
  const float vxx = Q ? d[0][0] + d[0][1] : A::mul(A::mul(0.5f, A::add(d[0][0], d[0][1])), invdx);
  const float vxz = Q ? d[0][0] - d[0][1] : A::mul(A::mul(0.5f, A::sub(d[0][0], d[0][1])), invdz);
  const float vzx = Q ? d[1][0] + d[1][1] : A::mul(A::mul(0.5f, A::add(d[1][0], d[1][1])), invdx);
  const float vzz = Q ? d[1][0] - d[1][1] : A::mul(A::mul(0.5f, A::sub(d[1][0], d[1][1])), invdz);
  if (K) {
    a.kd[0][gi] = vxx;
    a.kd[1][gi] = vxz;
    a.kd[2][gi] = vzx;
    a.kd[3][gi] = vzz;
    if (V == TTI_TENSOR) {
      a.kt[0][gi] = p.o0;
      a.kt[1][gi] = p.o1;
      a.kt[2][gi] = p.o2;
    }
  }
  stress_store<V, X>(a, gi, vxx, vxz, vzx, vzz, p);
}

// Stress update of tile (tz, tx); `map` holds the tensor maps of vx, vz.
// The same for the stress update: sigma (tensor: tau), coef1/coef2 outside the
// undamped interior, c11 c13 c33 c55 (four lines), the formulation's pair
// (two lines) and, for the tensor rotation, sin 2 theta.
template <int V>
__device__ __forceinline__ void prefetch_scells(const HalfArgs &a, const Cells &c, bool und)
{
  constexpr int SLOTS = V == TTI_TENSOR ? 12 : 11;
  const int lane = threadIdx.x & 31, z = c.zr - lane;
  if (z >= a.g.Nz - NH) return;
  for (int q = lane; q < (TX / 4) * SLOTS; q += 32) {
    const int col = q / SLOTS, k = q % SLOTS, x = c.xc + col;
    if (x >= a.g.Nx - NH) continue;
    const size_t gi = (size_t)x * a.g.ldz + z;
    const void *p = nullptr;
    if (k < 3) {
      const float *o = V == TTI_TENSOR ? (k == 0 ? a.f.txx : k == 1 ? a.f.tzz : a.f.txz)
                                       : (k == 0 ? a.f.sxx : k == 1 ? a.f.szz : a.f.sxz);
      p = o + gi;
    } else if (k < 5) {
      p = und ? nullptr : (const void *)(a.pk.cf + gi + 16 * (k - 3));
    } else if (k < 9) {
      p = a.pk.c4 + gi + 8 * (k - 5);
    } else if (k < 11) {
      p = a.pk.sc + gi + 16 * (k - 9);
    } else {
      p = a.p.s2t + gi;
    }
    if (p) asm volatile("prefetch.global.L2 [%0];" ::"l"(p));
  }
}

template <int V, bool X, bool Q, bool K = false, bool PB = false>
__device__ __forceinline__ void stress_tile(const HalfArgs &a, const CUtensorMap *map, float *sm, int tz, int tx,
                                            unsigned long long *pbar = nullptr, int ph = 0)
{
  using A = Ar<X>;
  unsigned long long *bar = PB ? pbar : reinterpret_cast<unsigned long long *>(sm + 2 * FIELD);
  const Grid &g = a.g;
  const Cells c = cells_of(a, tz, tx);
  tma::issue_tiles(map, sm, bar, 2, c.z0, c.x0, 5, PB ? ph : -1);
  const bool und = tile_undamped(a, c);
  const int z = c.zr;
  const bool zin = z >= g.izStart && z < g.Nz - NH;
  prefetch_scells<V>(a, c, und);
  if (!tma::wait_tiles(a.err, bar, a.wait_limit, PB ? (unsigned)ph : 0u)) return;
  if (!zin) return;
#pragma unroll
  for (int i = 0; i < TX / 4; ++i) {
    const int x = c.xc + i;
    if (x >= g.Nx - NH) break;
    const size_t gi = (size_t)x * g.ldz + z;
    SCell p;
    load_scell<V>(a, und, gi, p);
    // velocity value at column x+m, row z+n: s[f * FIELD + m * BZ + n]
    const float *s = sm + (x - c.x0 + 5) * BZ + (z - c.z0 + 8);
    float d[2][2];
#pragma unroll
    for (int f = 0; f < 2; ++f) {
      const float *q = s + f * FIELD;
      // d1 = sum C_k (v[x+k-1][z+k-1] - v[x-k][z-k]); d2 = sum C_k (v[x+k-1][z-k] - v[x-k][z+k-1])
      float s1 = A::mul(coef<Q>(a, 0), A::sub(q[0], q[-BZ - 1]));
      float s2 = A::mul(coef<Q>(a, 0), A::sub(q[-1], q[-BZ]));
#pragma unroll
      for (int k = 2; k <= NH; ++k) {
        s1 = A::add(s1, A::mul(coef<Q>(a, k - 1), A::sub(q[(k - 1) * BZ + k - 1], q[-k * BZ - k])));
        s2 = A::add(s2, A::mul(coef<Q>(a, k - 1), A::sub(q[(k - 1) * BZ - k], q[-k * BZ + k - 1])));
      }
      d[f][0] = s1;
      d[f][1] = s2;
    }
    stress_finish<V, X, Q, K>(a, gi, d, p);
  }
}

// Batched launches copy the instance's arguments (less the tensor maps, which
// TMA reads from global memory) into shared memory once per CTA: the fields are
// then uniform shared loads that the in-place global stores cannot alias.
constexpr int ARGS_OFF = 3 * FIELD + 16;  // floats: after the largest field set and its barrier
constexpr size_t ARGS_BYTES = sizeof(HalfArgs);
static_assert(ARGS_OFF % 16 == 0, "argument copy must be 16-byte aligned");
static_assert(ARGS_BYTES % 16 == 0, "HalfArgs must be a whole number of 16-byte words");

__device__ __forceinline__ const HalfArgs *stage_args(const HalfArgs *src, float *sm, size_t off = ARGS_OFF)
{
  HalfArgs *dst = reinterpret_cast<HalfArgs *>(sm + off);
  const int4 *s4 = reinterpret_cast<const int4 *>(src);
  int4 *d4 = reinterpret_cast<int4 *>(dst);
  for (int i = threadIdx.x; i < (int)(ARGS_BYTES / 16); i += blockDim.x) d4[i] = s4[i];
  __syncthreads();
  return dst;
}

// K (the gradient's forward pass also writes what the adjoint keeps): three
// CTAs per SM, so the extra live values fit in registers without spilling
template <int V, bool X, bool Q, bool K = false>
__global__ void __launch_bounds__(NT, K ? 3 : 4) k_velocity_tiled(const __grid_constant__ HalfArgs a)
{
  extern __shared__ __align__(128) float sm[];
  pdl_sync();
  velocity_tile<V, X, Q, K>(a, a.map, sm, blockIdx.x, blockIdx.y);
}

template <int V, bool X, bool Q, bool K = false>
__global__ void __launch_bounds__(NT, K ? 3 : 4) k_stress_tiled(const __grid_constant__ HalfArgs a)
{
  extern __shared__ __align__(128) float sm[];
  pdl_sync();
  stress_tile<V, X, Q, K>(a, a.map, sm, blockIdx.x, blockIdx.y);
}

// Work items blockIdx.x, blockIdx.x + gridDim.x, ... of the table: one item
// per CTA when the grid covers the table, several when a persistent grid of
// one resident wave walks it. The tile's shared memory (boxes, barrier,
// staged arguments) is reused by the next item only after every thread of
// the CTA is done with it.
template <typename F>
__device__ __forceinline__ void for_work(const HalfArgs *inst, const Work *work, int nwork, const int *step, F f)
{
  for (int i = blockIdx.x; i < nwork; i += gridDim.x) {
    const Work w = work[i];
    const HalfArgs *src = inst + w.inst;
    if (*step >= src->nt) continue;  // uniform over the CTA
    f(src, w);
    __syncthreads();
  }
}

template <int V, bool X, bool Q>
__global__ void __launch_bounds__(NT, 4) k_velocity_batch(const HalfArgs *__restrict__ inst,
                                                          const Work *__restrict__ work, int nwork, const int *step)
{
  extern __shared__ __align__(128) float sm[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + 3 * FIELD);
  if (threadIdx.x == 0) {  // one barrier for all the CTA's tiles (ordered by stage_args' barrier)
    tma::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int ph = 0;
  for_work(inst, work, nwork, step, [&](const HalfArgs *src, const Work &w) {
    const HalfArgs *a = stage_args(src, sm);
    velocity_tile<V, X, Q, false, true>(*a, src->map, sm, w.tile % a->tiles_z, w.tile / a->tiles_z, bar, ph);
    ph ^= 1;
  });
}

template <int V, bool X, bool Q>
__global__ void __launch_bounds__(NT, 4) k_stress_batch(const HalfArgs *__restrict__ inst,
                                                        const Work *__restrict__ work, int nwork, const int *step)
{
  extern __shared__ __align__(128) float sm[];
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(sm + 2 * FIELD);
  if (threadIdx.x == 0) {  // one barrier for all the CTA's tiles (ordered by stage_args' barrier)
    tma::mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  int ph = 0;
  for_work(inst, work, nwork, step, [&](const HalfArgs *src, const Work &w) {
    const HalfArgs *a = stage_args(src, sm);
    stress_tile<V, X, Q, false, true>(*a, src->map, sm, w.tile % a->tiles_z, w.tile / a->tiles_z, bar, ph);
    ph ^= 1;
  });
}

template <typename K>
cudaError_t set_attr(K kernel, size_t bytes)
{
  static std::mutex mu;
  static const void *done[128];
  static int ndone = 0;
  {
    std::lock_guard<std::mutex> lock(mu);
    bool seen = false;
    for (int i = 0; i < ndone; ++i) seen = seen || done[i] == (const void *)kernel;
    if (!seen) {
      cudaError_t e = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
      if (e == cudaSuccess)
        e = cudaFuncSetAttribute(kernel, cudaFuncAttributePreferredSharedMemoryCarveout,
                                 cudaSharedmemCarveoutMaxShared);
      if (e != cudaSuccess) return e;
      if (ndone < 128) done[ndone++] = (const void *)kernel;
    }
  }
  return cudaSuccess;
}

template <typename K>
cudaError_t launch_k(K kernel, const HalfArgs &a, int nfields, cudaStream_t st)
{
  const size_t bytes = (size_t)nfields * FIELD * sizeof(float) + 16;
  cudaError_t e = set_attr(kernel, bytes);
  if (e != cudaSuccess) return e;
  HalfArgs b = a;
  const dim3 gr = grid(a.g, &b.z_base);
  if (gr.x == 0 || gr.y == 0) return cudaSuccess;
  return launch_pdl(kernel, gr, dim3(NT), bytes, st, b);
}

}  // namespace


dim3 grid(const Grid &g, int *z_base)
{
  // izStart rounded down to 32 rows, so that a warp's 32 consecutive rows are
  // one 128-byte line of every per-cell array
  *z_base = g.izStart & ~31;
  const int nz = g.Nz - NH - *z_base, nx = g.Nx - 2 * NH;
  if (nz <= 0 || nx <= 0) return dim3(0, 0);
  return dim3((nz + TZ - 1) / TZ, (nx + TX - 1) / TX);
}

bool encode_map(CUtensorMap *map, const Grid &g, float *field)
{
  static PFN_cuTensorMapEncodeTiled_v12000 encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void *fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return false;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(fn);
  }
  const cuuint64_t dims[2] = {(cuuint64_t)g.ldz, (cuuint64_t)g.Nx};
  const cuuint64_t strides[1] = {(cuuint64_t)g.ldz * sizeof(float)};
  const cuuint32_t box[2] = {(cuuint32_t)BZ, (cuuint32_t)BX};
  const cuuint32_t estr[2] = {1, 1};
  return encode(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, field, dims, strides, box, estr,
                CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_128B,
                CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

template <bool X, bool Q>
cudaError_t velocity_xq(const HalfArgs &a, int variant, cudaStream_t st)
{
  if (variant == TTI_COORDINATE && a.kd[0]) return launch_k(k_velocity_tiled<TTI_COORDINATE, X, Q, true>, a, 3, st);
  if (variant == TTI_COORDINATE) return launch_k(k_velocity_tiled<TTI_COORDINATE, X, Q>, a, 3, st);
  if (variant == TTI_TENSOR) return launch_k(k_velocity_tiled<TTI_TENSOR, X, Q>, a, 3, st);
  return launch_k(k_velocity_tiled<TTI_BOND, X, Q>, a, 3, st);
}

template <bool X, bool Q>
cudaError_t stress_xq(const HalfArgs &a, int variant, cudaStream_t st)
{
  const bool k = a.kd[0] != nullptr;
  if (variant == TTI_COORDINATE)
    return k ? launch_k(k_stress_tiled<TTI_COORDINATE, X, Q, true>, a, 2, st)
             : launch_k(k_stress_tiled<TTI_COORDINATE, X, Q>, a, 2, st);
  if (variant == TTI_TENSOR)
    return k ? launch_k(k_stress_tiled<TTI_TENSOR, X, Q, true>, a, 2, st)
             : launch_k(k_stress_tiled<TTI_TENSOR, X, Q>, a, 2, st);
  return k ? launch_k(k_stress_tiled<TTI_BOND, X, Q, true>, a, 2, st) : launch_k(k_stress_tiled<TTI_BOND, X, Q>, a, 2, st);
}

cudaError_t launch_velocity(const HalfArgs &a, int variant, bool exact, cudaStream_t st)
{
  if (exact) return velocity_xq<true, false>(a, variant, st);
  return a.square ? velocity_xq<false, true>(a, variant, st) : velocity_xq<false, false>(a, variant, st);
}

cudaError_t launch_stress(const HalfArgs &a, int variant, bool exact, cudaStream_t st)
{
  if (exact) return stress_xq<true, false>(a, variant, st);
  return a.square ? stress_xq<false, true>(a, variant, st) : stress_xq<false, false>(a, variant, st);
}

constexpr size_t BATCH_SMEM = (size_t)ARGS_OFF * sizeof(float) + ARGS_BYTES;

// One CTA per work item, or (persistent) one resident wave of CTAs that walks
// the table: the SM count times the kernel's CTAs per SM at its shared memory.
template <typename K>
cudaError_t launch_batch_k(K kernel, const BatchLaunch &l, cudaStream_t st, size_t smem = BATCH_SMEM,
                           int threads = NT)
{
  cudaError_t e = set_attr(kernel, smem);
  if (e != cudaSuccess || l.nwork == 0) return e;
  int grid = l.nwork;
  if (l.persistent) {
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem)) != cudaSuccess) return e;
    grid = std::min(l.nwork, std::max(1, per_sm) * sms);
  }
  kernel<<<grid, threads, smem, st>>>(l.inst, l.work, l.nwork, l.step);
  return cudaGetLastError();
}

template <bool X, bool Q>
cudaError_t velocity_batch_x(const BatchLaunch &l, cudaStream_t st)
{
  if (l.variant == TTI_COORDINATE) return launch_batch_k(k_velocity_batch<TTI_COORDINATE, X, Q>, l, st);
  if (l.variant == TTI_TENSOR) return launch_batch_k(k_velocity_batch<TTI_TENSOR, X, Q>, l, st);
  return launch_batch_k(k_velocity_batch<TTI_BOND, X, Q>, l, st);
}

template <bool X, bool Q>
cudaError_t stress_batch_x(const BatchLaunch &l, cudaStream_t st)
{
  if (l.variant == TTI_COORDINATE) return launch_batch_k(k_stress_batch<TTI_COORDINATE, X, Q>, l, st);
  if (l.variant == TTI_TENSOR) return launch_batch_k(k_stress_batch<TTI_TENSOR, X, Q>, l, st);
  return launch_batch_k(k_stress_batch<TTI_BOND, X, Q>, l, st);
}

cudaError_t launch_velocity_batch(const BatchLaunch &l, cudaStream_t st)
{
  if (l.exact) return velocity_batch_x<true, false>(l, st);
  return l.square ? velocity_batch_x<false, true>(l, st) : velocity_batch_x<false, false>(l, st);
}

cudaError_t launch_stress_batch(const BatchLaunch &l, cudaStream_t st)
{
  if (l.exact) return stress_batch_x<true, false>(l, st);
  return l.square ? stress_batch_x<false, true>(l, st) : stress_batch_x<false, false>(l, st);
}

cudaError_t prepare_batch(BatchLaunch l)
{
  // a launch over zero CTAs only sets the attributes
  l.nwork = 0;
  cudaError_t e = launch_velocity_batch(l, nullptr);
  if (e == cudaSuccess) e = launch_stress_batch(l, nullptr);
  return e;
}

}  // namespace tiled
}  // namespace ttifd
