// One kernel per time step: velocity half-step, velocity sources, stress
// half-step, free surface and stress source fused (receivers are sampled by a
// small kernel afterwards).
//
// Work decomposition: a CTA of NT = 192 threads owns a band of at most
// BZ = 182 rows (z, the contiguous axis) and a segment of columns [x0, x1),
// and marches along x. At iteration j it
//   1. computes v_new for column xv = x0 - 5 + j over rows [z0-5, z0+bz+5)
//      (one row per thread: its band plus the 5-row halo the stress stencil
//      needs) from the stress columns xv-4 .. xv+5 held in a shared ring,
//   2. computes sigma_new for column xs = xv - 4 over its own rows from the
//      v_new columns xs-5 .. xs+4 held in a second shared ring.
// Stress columns arrive by cp.async.bulk (one elected thread; completion on a
// per-column mbarrier that every thread tests before use) P columns ahead;
// per-cell parameters (packed for 64/128-bit loads) and v_old, read once
// each, are loaded into registers one iteration ahead. One CTA barrier per
// column: the stress ring has R = P + 10 slots and the velocity ring NV >= 11,
// so a slot is refilled only after the barrier that follows its last read;
// both sizes are powers of two so a slot is one AND of a warp-uniform
// counter. Stencils are evaluated by all
// threads (every shared-memory read stays inside the rings) and the results
// kept only where the reference updates, which avoids divergent branches.
// State is double buffered (old -> new): halo rows and columns read by a CTA
// are never written during the step.
//
// Per-cell arithmetic is the reference's (coord:614-886, tensor:617-895,
// bond:654-913) under the same rounding policy as the per-kernel path.
#include "fused.cuh"

namespace ttifd {
namespace fused {

namespace {

__device__ __forceinline__ unsigned smem_u32(const void *p)
{
  return static_cast<unsigned>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(unsigned long long *bar, unsigned count)
{
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_arrive_expect_tx(unsigned long long *bar, unsigned bytes)
{
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
               : "memory");
}

// Bounded wait on an mbarrier phase: returns false after `limit` polls
// (about a second), so a copy that never lands cannot hang the GPU.
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit = 1u << 20)
{
  const unsigned a = smem_u32(bar);
  for (unsigned n = 0; n < limit; ++n) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(a), "r"(parity)
        : "memory");
    if (ok) return true;
  }
  return false;
}

__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, unsigned bytes, unsigned long long *bar)
{
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}

__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

constexpr int COLS = 3 * SR;    // floats per stress column (sxx, szz, sxz)
constexpr int COLV = 2 * VSTR;  // floats per velocity column (vx, vz)
constexpr int VOFF = R * COLS;  // start of the velocity ring
constexpr int SMEM_FLOATS = VOFF + NV * COLV + 32 + 2 * MAXSRC;
constexpr size_t SMEM_BYTES = SMEM_FLOATS * sizeof(float) + R * sizeof(unsigned long long);
static_assert(SMEM_FLOATS % 2 == 0, "mbarriers need 8-byte alignment");
static_assert(BZ + 25 <= SR, "stress ring rows");
static_assert(NV >= 11, "velocity ring must outlive one column");
static_assert((R & (R - 1)) == 0 && (NV & (NV - 1)) == 0, "ring sizes are powers of two");
static_assert(VSTR >= NT + 9 && SR >= NT + 12, "halo reads stay inside the rings");

// velocity sources (stype 2..8) on one cell, in the reference's order
__device__ __forceinline__ void vsource_cell(const FusedArgs &a, const int *sxz, int x, int z, float &vx, float &vz)
{
  const int st = a.stype;
  if (st == 8) {
    const float q = a.tab.q8;
    for (int n = 0; n < a.src.n; ++n) {
      const int dx = x - sxz[2 * n], dz = z - sxz[2 * n + 1];
      if (dx < -1 || dx > 0 || dz < -1 || dz > 0) continue;
      const float qs = __fmul_rn(q, __ldg(a.src.w + (size_t)n * a.src.nt + a.it));
      if (dx == 0 && dz == 0) {
        vx = __fsub_rn(vx, qs);
        vz = __fadd_rn(vz, qs);
      } else if (dx == -1 && dz == 0) {
        vx = __fsub_rn(vx, qs);
        vz = __fsub_rn(vz, qs);
      } else if (dx == -1 && dz == -1) {
        vx = __fadd_rn(vx, qs);
        vz = __fsub_rn(vz, qs);
      } else {
        vx = __fadd_rn(vx, qs);
        vz = __fadd_rn(vz, qs);
      }
    }
    return;
  }
  // divergence pass over all sources, then the curl pass (stype 4), or the force
  for (int pass = 0; pass < 2; ++pass) {
    int kind;
    if (pass == 0) kind = (st == 2 || st == 4) ? 2 : (st == 3 ? 3 : (st >= 5 ? st : 0));
    else kind = st == 4 ? 3 : 0;
    if (kind == 0) continue;
    for (int n = 0; n < a.src.n; ++n) {
      const int dx = x - sxz[2 * n], dz = z - sxz[2 * n + 1];
      if (dx < -NH || dx > NH || dz < -NH || dz > NH) continue;
      const int k = (dx + NH) * 11 + (dz + NH);
      const float s = __ldg(a.src.w + (size_t)n * a.src.nt + a.it);
      switch (kind) {
      case 2:
        vx = __fadd_rn(vx, __fmul_rn(a.tab.kx[k], s));
        vz = __fadd_rn(vz, __fmul_rn(a.tab.kz[k], s));
        break;
      case 3:
        vx = __fsub_rn(vx, __fmul_rn(a.tab.kz[k], s));
        vz = __fadd_rn(vz, __fmul_rn(a.tab.kx[k], s));
        break;
      case 5:
        vx = __fadd_rn(vx, __fmul_rn(a.tab.k5[k], s));
        break;
      case 6:
        vz = __fadd_rn(vz, __fmul_rn(a.tab.k5[k], s));
        break;
      case 7:
        vx = __fadd_rn(vx, __fmul_rn(a.tab.k7[k], s));
        vz = __fadd_rn(vz, __fmul_rn(a.tab.k7[k], s));
        break;
      }
    }
  }
}

// per-cell inputs read once, prefetched one iteration ahead
struct VIn {
  float vx, vz, c1, c2, ir, sv, cv;
};
struct SIn {
  float c1, c2;
  float4 c4;   // c11 c13 c33 c55
  float2 sc;   // see Packed
  float s2t;   // tensor
  float tau[3];
};

// Loads are issued by every thread; an invalid cell reads element 0 instead
// (the value is never used), which keeps the loop free of divergent branches.
template <int V>
__device__ __forceinline__ void load_v(const FusedArgs &a, bool ok, bool und, size_t i, VIn &o)
{
  i = ok ? i : 0;
  o.vx = __ldg(a.old.vx + i);
  o.vz = __ldg(a.old.vz + i);
  if (und) {
    o.c1 = 1.0f;
    o.c2 = a.dt;
  } else {
    const float2 cf = __ldg(a.pk.cf + i);
    o.c1 = cf.x;
    o.c2 = cf.y;
  }
  o.ir = __ldg(a.p.invrho + i);
  if (V == TTI_COORDINATE) {
    const float2 sc = __ldg(a.pk.vsc + i);
    o.sv = sc.x;
    o.cv = sc.y;
  }
}

template <int V>
__device__ __forceinline__ void load_s(const FusedArgs &a, bool ok, bool und, size_t i, SIn &o)
{
  i = ok ? i : 0;
  if (und) {
    o.c1 = 1.0f;
    o.c2 = a.dt;
  } else {
    const float2 cf = __ldg(a.pk.cf + i);
    o.c1 = cf.x;
    o.c2 = cf.y;
  }
  o.c4 = __ldg(a.pk.c4 + i);
  o.sc = __ldg(a.pk.sc + i);
  if (V == TTI_TENSOR) {
    o.s2t = __ldg(a.p.s2t + i);
    o.tau[0] = __ldg(a.old.txx + i);
    o.tau[1] = __ldg(a.old.tzz + i);
    o.tau[2] = __ldg(a.old.txz + i);
  }
}

template <int V, bool X>
__global__ void __maxnreg__(112) k_fused(const __grid_constant__ FusedArgs a)
{
  using A = Ar<X>;
  // shared memory: stress ring [R][3][SR] (row s at s - sbase), velocity ring
  // [NV][2][VSTR] (row r at r - (z0 - 5)), free-surface exchange, source
  // positions, R mbarriers
  extern __shared__ __align__(128) float smem[];
  float *fsbuf = smem + VOFF + NV * COLV;
  int *ssrc = reinterpret_cast<int *>(fsbuf + 32);
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(smem + SMEM_FLOATS);

  const Grid &g = a.g;
  const int t = threadIdx.x;
  const int bz = a.bz;  // rows owned by this CTA's band (<= BZ)
  const int z0 = blockIdx.y * bz;
  const int x0 = blockIdx.x * a.seg, x1 = min(x0 + a.seg, g.Nx);
  const int L = g.ldz;
  const int Nx = g.Nx;
  const int niter = (x1 - x0) + 9;  // xv = x0-5 .. x1+3
  const int ncol = niter + 9;       // stress columns x0-9 .. x1+8
  const int sbase = (z0 - 9) & ~3;  // first staged stress row (16-byte aligned)
  const int s_lo = max(sbase, 0), s_hi = min((z0 + bz + 10 + 3) & ~3, L);
  // Undamped CTA: every coefficient it reads is outside the MEAL rims, where
  // D = 0 makes coef1 = 1 and coef2 = dt exactly (meal.c:486-487).
  const bool und = a.undamped_ok && (x0 - 5 >= g.E) && (x1 + 3 < Nx - g.E) &&
                   (z0 - 5 >= (a.freesurface ? 0 : g.E)) && (z0 + bz + 5 < g.Nz - g.E);
  const bool fs_band = a.freesurface && z0 == 0;
  const int nsrc = a.src.n;  // <= MAXSRC (the host uses the per-kernel path otherwise)

  // stress column q (x = x0 - 9 + q) into ring slot q % R, mbarrier q % R
  auto issue_col = [&](int q) {
    unsigned long long *b = bar + (q % R);
    const int c = x0 - 9 + q;
    if (c < 0 || c >= Nx || s_hi <= s_lo) {
      mbar_arrive_expect_tx(b, 0);
      return;
    }
    const unsigned sb = (s_hi - s_lo) * 4u;
    mbar_arrive_expect_tx(b, 3 * sb);
    float *dst = smem + (q % R) * COLS + (s_lo - sbase);
    const size_t off = (size_t)c * L + s_lo;
    bulk_g2s(dst, a.old.sxx + off, sb, b);
    bulk_g2s(dst + SR, a.old.szz + off, sb, b);
    bulk_g2s(dst + 2 * SR, a.old.sxz + off, sb, b);
  };
  // each thread tests the column's mbarrier itself (a single poll once the
  // copy has landed); a timeout is voted at the next CTA barrier
  auto wait_col = [&](int q) -> bool { return mbar_wait(bar + (q % R), (q / R) & 1); };
  // on a timed-out wait: flag it, give copies in flight a bounded time, leave
  auto bail = [&](int first) {
    if (t == 0) {
      atomicOr(a.err, 2);
      for (int q = first; q < first + R && q < ncol; ++q) mbar_wait(bar + (q % R), (q / R) & 1, 1u << 14);
    }
  };

  if (t == 0) {
    for (int k = 0; k < R; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  for (int n = t; n < nsrc; n += NT) {
    ssrc[2 * n] = a.src.x[n];
    ssrc[2 * n + 1] = a.src.z[n];
  }
  __syncthreads();
  if (t == 0)
    for (int q = 0; q < P + 9 && q < ncol; ++q) issue_col(q);

  // thread roles
  const int r = z0 - 5 + t;  // velocity row
  const bool r_ok = t < bz + 10 && r >= 0 && r < g.Nz;
  const bool r_in = r_ok && r >= g.izStart && r < g.Nz - NH;
  const bool r_own = t >= 5 && t < bz + 5 && r < g.Nz;
  const int z = z0 + t;  // stress row (t < bz)
  const bool z_ok = t < bz && z < g.Nz;
  const bool z_in = z_ok && z >= g.izStart && z < g.Nz - NH;
  const int srow = r - sbase;       // this thread's velocity row in the stress ring
  const int zrow = z - sbase;       // this thread's stress row in the stress ring
  float *const sr_t = smem + srow;  // stress ring at this thread's velocity row
  float *const vr_t = smem + VOFF + t;

  VIn va{}, vb{};
  SIn sa{}, sb{};
  {
    const int xv = x0 - 5, xs = xv - 4;
    load_v<V>(a, r_ok && xv >= 0 && xv < Nx, und, (size_t)xv * L + r, va);
    load_s<V>(a, z_ok && xs >= x0 && xs < x1, und, (size_t)xs * L + z, sa);
  }
  {
    bool ok = true;
    for (int q = 0; q < 9 && q < ncol; ++q) ok = wait_col(q) && ok;
    if (__syncthreads_or(!ok)) {
      bail(0);
      return;
    }
  }

  // One march iteration. `vin/sin_` hold this iteration's inputs, `vnx/snx`
  // receive the next one's (two register sets alternate: no copies).
  auto body = [&](int j, const VIn &vin, const SIn &sin_, VIn &vnx, SIn &snx) -> bool {
    const int U = j;  // ring slots are taken modulo the power-of-two ring sizes
    const int xv = x0 - 5 + j, xs = xv - 4;
    load_v<V>(a, r_ok && xv + 1 < Nx && xv + 1 >= 0 && j + 1 < niter, und, (size_t)(xv + 1) * L + r, vnx);
    load_s<V>(a, z_ok && xs + 1 >= x0 && xs + 1 < x1, und, (size_t)(xs + 1) * L + z, snx);
    const bool ok = wait_col(j + 9);

    // ---------------- velocity half-step at column xv, row r
    const bool xv_ok = xv >= 0 && xv < Nx;
    if (xv_ok) {
      float vx = vin.vx, vz = vin.vz;
      if (xv >= NH && xv < Nx - NH) {
        // stress column xv+m (m = -4..5) sits in ring slot (U + m + 4) % R
        float d[3][2];
#pragma unroll
        for (int f = 0; f < 3; ++f) {
          const float *c = sr_t + f * SR;
#define SC(m) (c + (((U + (m) + 4) & (R - 1)) * COLS))
          // d1 = sum C_k (s[x+k][z+k] - s[x-k+1][z-k+1]); d2 = sum C_k (s[x+k][z-k+1] - s[x-k+1][z+k])
          float s1 = A::mul(rsg(0), A::sub(SC(1)[1], SC(0)[0]));
          float s2 = A::mul(rsg(0), A::sub(SC(1)[0], SC(0)[1]));
#pragma unroll
          for (int k = 2; k <= NH; ++k) {
            s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(SC(k)[k], SC(1 - k)[1 - k])));
            s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(SC(k)[1 - k], SC(1 - k)[k])));
          }
#undef SC
          d[f][0] = s1;
          d[f][1] = s2;
        }
        const float invdx = a.invdx, invdz = a.invdz;
        const float sxx_x = A::mul(A::mul(0.5f, A::add(d[0][0], d[0][1])), invdx);
        const float szz_z = A::mul(A::mul(0.5f, A::sub(d[1][0], d[1][1])), invdz);
        const float sxz_x = A::mul(A::mul(0.5f, A::add(d[2][0], d[2][1])), invdx);
        const float sxz_z = A::mul(A::mul(0.5f, A::sub(d[2][0], d[2][1])), invdz);
        const float br = A::mul(vin.c2, vin.ir);
        float fx, fz;
        if (V == TTI_COORDINATE) {
          const float sxx_z = A::mul(A::mul(0.5f, A::sub(d[0][0], d[0][1])), invdx);  // invdx as coord:633
          const float szz_x = A::mul(A::mul(0.5f, A::add(d[1][0], d[1][1])), invdx);
          const float sv = vin.sv, cv = vin.cv;
          fx = A::add(A::add(A::sub(A::mul(cv, sxx_x), A::mul(sv, sxx_z)), A::mul(sv, sxz_x)), A::mul(cv, sxz_z));
          fz = A::add(A::add(A::sub(A::mul(cv, sxz_x), A::mul(sv, sxz_z)), A::mul(sv, szz_x)), A::mul(cv, szz_z));
        } else {
          fx = A::add(sxx_x, sxz_z);
          fz = A::add(sxz_x, szz_z);
        }
        const float nvx = A::add(A::mul(vin.c1, vx), A::mul(br, fx));
        const float nvz = A::add(A::mul(vin.c1, vz), A::mul(br, fz));
        vx = r_in ? nvx : vx;
        vz = r_in ? nvz : vz;
      }
      if (a.stype >= 2 && nsrc > 0) vsource_cell(a, ssrc, xv, r, vx, vz);
      vr_t[(U & (NV - 1)) * COLV] = vx;
      vr_t[(U & (NV - 1)) * COLV + VSTR] = vz;
      if (r_own && xv >= x0 && xv < x1) {
        const size_t gi = (size_t)xv * L + r;
        a.nw.vx[gi] = vx;
        a.nw.vz[gi] = vz;
      }
    }
    // the one CTA barrier per column: v_new of column xv visible; every read
    // of stress column xs - 1 (previous column) is done, so its slot refills
    if (__syncthreads_or(!ok)) {
      bail(j + 9);
      return false;
    }
    if (t == 0 && j + 9 + P < ncol) {
      fence_proxy_async();
      issue_col(j + 9 + P);  // slot of column q = j - 1
    }

    // ---------------- stress half-step at column xs, row z
    const bool do_s = xs >= x0 && xs < x1;
    float sxx = 0.f, szz = 0.f, sxz = 0.f, txx = 0.f, tzz = 0.f, txz = 0.f;
    if (do_s) {
      const float *so = smem + (U & (R - 1)) * COLS + zrow;  // stress column xs = xv - 4
      sxx = so[0];
      szz = so[SR];
      sxz = so[2 * SR];
      if (V == TTI_TENSOR) {
        txx = sin_.tau[0];
        tzz = sin_.tau[1];
        txz = sin_.tau[2];
      }
      if (xs >= NH && xs < Nx - NH) {
        // velocity column xs+m (m = -5..4) was written at iteration j - 4 + m: slot (j - 4 + m) % NV;
        // row z sits at t + 5
        float d[2][2];
#pragma unroll
        for (int f = 0; f < 2; ++f) {
          const float *c = vr_t + 5 + f * VSTR;
#define VC(m) (c + (((U - 4 + (m)) & (NV - 1)) * COLV))
          // d1 = sum C_k (v[x+k-1][z+k-1] - v[x-k][z-k]); d2 = sum C_k (v[x+k-1][z-k] - v[x-k][z+k-1])
          float s1 = A::mul(rsg(0), A::sub(VC(0)[0], VC(-1)[-1]));
          float s2 = A::mul(rsg(0), A::sub(VC(0)[-1], VC(-1)[0]));
#pragma unroll
          for (int k = 2; k <= NH; ++k) {
            s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(VC(k - 1)[k - 1], VC(-k)[-k])));
            s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(VC(k - 1)[-k], VC(-k)[k - 1])));
          }
#undef VC
          d[f][0] = s1;
          d[f][1] = s2;
        }
        const float invdx = a.invdx, invdz = a.invdz;
        float vxx = A::mul(A::mul(0.5f, A::add(d[0][0], d[0][1])), invdx);
        float vxz = A::mul(A::mul(0.5f, A::sub(d[0][0], d[0][1])), invdz);
        float vzx = A::mul(A::mul(0.5f, A::add(d[1][0], d[1][1])), invdx);
        float vzz = A::mul(A::mul(0.5f, A::sub(d[1][0], d[1][1])), invdz);
        const float c1 = sin_.c1, c2 = sin_.c2;
        const float c11 = sin_.c4.x, c13 = sin_.c4.y, c33 = sin_.c4.z, c55 = sin_.c4.w;
        float nxx, nzz, nxz, ntx = txx, ntz = tzz, ntq = txz;
        if (V == TTI_COORDINATE) {
          const float s = sin_.sc.x, c = sin_.sc.y;
          float q = A::add(A::mul(s, vxx), A::mul(c, vxz));
          vxx = A::sub(A::mul(c, vxx), A::mul(s, vxz));
          vxz = q;
          q = A::add(A::mul(s, vzx), A::mul(c, vzz));
          vzx = A::sub(A::mul(c, vzx), A::mul(s, vzz));
          vzz = q;
          nxx = A::add(A::mul(c1, sxx), A::mul(c2, A::add(A::mul(c11, vxx), A::mul(c13, vzz))));
          nzz = A::add(A::mul(c1, szz), A::mul(c2, A::add(A::mul(c13, vxx), A::mul(c33, vzz))));
          nxz = A::add(A::mul(c1, sxz), A::mul(A::mul(c2, c55), A::add(vzx, vxz)));
        } else if (V == TTI_TENSOR) {
          const float s2 = sin_.sc.x, cc2 = sin_.sc.y, s2t = sin_.s2t;
          const float sh = A::add(vxz, vzx);
          const float exx = A::sub(A::add(A::mul(cc2, vxx), A::mul(s2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
          const float ezz = A::add(A::add(A::mul(s2, vxx), A::mul(cc2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
          const float exz = A::add(A::mul(s2t, A::sub(vxx, vzz)), A::mul(A::sub(cc2, s2), sh));
          ntx = A::add(A::mul(c1, txx), A::mul(c2, A::add(A::mul(c11, exx), A::mul(c13, ezz))));
          ntz = A::add(A::mul(c1, tzz), A::mul(c2, A::add(A::mul(c13, exx), A::mul(c33, ezz))));
          ntq = A::add(A::mul(c1, txz), A::mul(A::mul(c2, c55), exz));
          nxx = A::add(A::add(A::mul(cc2, ntx), A::mul(s2, ntz)), A::mul(s2t, ntq));
          nzz = A::sub(A::add(A::mul(s2, ntx), A::mul(cc2, ntz)), A::mul(s2t, ntq));
          nxz = A::add(A::mul(A::mul(-0.5f, s2t), A::sub(ntx, ntz)), A::mul(A::sub(cc2, s2), ntq));
        } else {
          const float c15 = sin_.sc.x, c35 = sin_.sc.y;
          const float sh = A::add(vzx, vxz);
          nxx = A::add(A::mul(c1, sxx), A::mul(c2, A::add(A::add(A::mul(c11, vxx), A::mul(c13, vzz)), A::mul(c15, sh))));
          nzz = A::add(A::mul(c1, szz), A::mul(c2, A::add(A::add(A::mul(c13, vxx), A::mul(c33, vzz)), A::mul(c35, sh))));
          nxz = A::add(A::mul(c1, sxz), A::mul(c2, A::add(A::add(A::mul(c15, vxx), A::mul(c35, vzz)), A::mul(c55, sh))));
        }
        sxx = z_in ? nxx : sxx;
        szz = z_in ? nzz : szz;
        sxz = z_in ? nxz : sxz;
        if (V == TTI_TENSOR) {
          txx = z_in ? ntx : txx;
          tzz = z_in ? ntz : tzz;
          txz = z_in ? ntq : txz;
        }
      }
    }
    // free surface: stress image about row E for interior columns (coord:847-863)
    if (fs_band) {
      const int E = g.izStart;
      const bool col_fs = do_s && xs >= NH && xs < Nx - NH;
      if (col_fs && z_ok && z >= E && z <= E + NH) {
        fsbuf[z - E] = sxx;
        fsbuf[8 + z - E] = szz;
        fsbuf[16 + z - E] = sxz;
      }
      __syncthreads();
      if (col_fs && z_ok) {
        if (z == E) {
          szz = 0.0f;
          sxz = 0.0f;
        } else if (z >= E - NH && z < E) {
          const int k = E - z;
          sxx = __fsub_rn(__fmul_rn(2.0f, fsbuf[0]), fsbuf[k]);
          szz = -fsbuf[8 + k];
          sxz = -fsbuf[16 + k];
        }
      }
    }
    if (do_s) {
      if (a.stype == 1) {
        // stress source after the free surface (coord:865-886)
        for (int n = 0; n < nsrc; ++n) {
          const int dx = xs - ssrc[2 * n];
          if (dx < -NH || dx > NH) continue;  // uniform over the CTA
          const int dz = z - ssrc[2 * n + 1];
          const float s = __ldg(a.src.w + (size_t)n * a.src.nt + a.it);
          if (dz >= -NH && dz <= NH && z_ok) {
            const float ws = __fmul_rn(a.tab.k1[(dx + NH) * 11 + (dz + NH)], s);
            sxx = __fadd_rn(sxx, ws);
            szz = __fadd_rn(szz, ws);
            if (V == TTI_TENSOR) {
              txx = __fadd_rn(txx, ws);
              tzz = __fadd_rn(tzz, ws);
            }
          }
        }
      }
      if (z_ok) {
        const size_t gi = (size_t)xs * L + z;
        a.nw.sxx[gi] = sxx;
        a.nw.szz[gi] = szz;
        a.nw.sxz[gi] = sxz;
        if (V == TTI_TENSOR) {
          a.nw.txx[gi] = txx;
          a.nw.tzz[gi] = tzz;
          a.nw.txz[gi] = txz;
        }
      }
    }
    return true;
  };

  for (int j = 0; j < niter; j += 2) {
    if (!body(j, va, sa, vb, sb)) return;
    if (j + 1 < niter && !body(j + 1, vb, sb, va, sa)) return;
  }
}

__global__ void k_pack(Grid g, Params p, Packed pk, int variant)
{
  const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
  if (i >= g.n) return;
  pk.cf[i] = make_float2(p.coef1[i], p.coef2[i]);
  pk.c4[i] = make_float4(p.c11[i], p.c13[i], p.c33[i], p.c55[i]);
  if (variant == TTI_COORDINATE) {
    pk.vsc[i] = make_float2(p.snv[i], p.csv[i]);
    pk.sc[i] = make_float2(p.sn[i], p.cs[i]);
  } else if (variant == TTI_TENSOR) {
    pk.sc[i] = make_float2(p.s2[i], p.c2[i]);
  } else {
    pk.sc[i] = make_float2(p.c15[i], p.c35[i]);
  }
}

__global__ void k_check_undamped(Grid g, const float *__restrict__ c1, const float *__restrict__ c2, float dt,
                                 int zD, int *count)
{
  const int ix = g.E + blockIdx.y;
  int bad = 0;
  for (int iz = zD + (int)threadIdx.x; iz < g.Nz - g.E; iz += blockDim.x) {
    const size_t i = (size_t)ix * g.ldz + iz;
    bad += (c1[i] != 1.0f) | (c2[i] != dt);
  }
  bad = __syncthreads_count(bad > 0);
  if (threadIdx.x == 0 && bad) atomicAdd(count, bad);
}

}  // namespace

void launch_pack(const Grid &g, const Params &p, const Packed &pk, int variant, cudaStream_t st)
{
  k_pack<<<(unsigned)((g.n + 255) / 256), 256, 0, st>>>(g, p, pk, variant);
}

void launch_check_undamped(const Grid &g, const float *coef1, const float *coef2, float dt, int zD, int *count,
                           cudaStream_t st)
{
  const int nx = g.Nx - 2 * g.E;
  if (nx <= 0) return;
  k_check_undamped<<<dim3(1, nx), 256, 0, st>>>(g, coef1, coef2, dt, zD, count);
}

size_t smem_bytes(int) { return SMEM_BYTES; }

template <int V, bool X>
static cudaError_t launch_t(const FusedArgs &a, cudaStream_t st)
{
  static bool configured = false;  // per template instance
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_fused<V, X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM_BYTES);
    if (e != cudaSuccess) return e;
    // all of the unified L1/shared capacity as shared memory: 3 CTAs per SM
    e = cudaFuncSetAttribute(k_fused<V, X>, cudaFuncAttributePreferredSharedMemoryCarveout,
                             cudaSharedmemCarveoutMaxShared);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const dim3 grid((a.g.Nx + a.seg - 1) / a.seg, (a.g.Nz + a.bz - 1) / a.bz);
  k_fused<V, X><<<grid, NT, SMEM_BYTES, st>>>(a);
  return cudaGetLastError();
}

cudaError_t launch_fused(const FusedArgs &a, int variant, bool exact, cudaStream_t st)
{
  if (exact) {
    if (variant == TTI_COORDINATE) return launch_t<TTI_COORDINATE, true>(a, st);
    if (variant == TTI_TENSOR) return launch_t<TTI_TENSOR, true>(a, st);
    return launch_t<TTI_BOND, true>(a, st);
  }
  if (variant == TTI_COORDINATE) return launch_t<TTI_COORDINATE, false>(a, st);
  if (variant == TTI_TENSOR) return launch_t<TTI_TENSOR, false>(a, st);
  return launch_t<TTI_BOND, false>(a, st);
}

}  // namespace fused
}  // namespace ttifd
