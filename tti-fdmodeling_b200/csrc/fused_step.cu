// One kernel per time step: velocity half-step, velocity sources, stress
// half-step, free surface, stress source and receiver sampling fused.
//
// Work decomposition: a CTA owns a band of BZ rows (z, the contiguous axis)
// and a segment of columns [x0, x1) and marches along x. At iteration j it
//   1. computes v_new for column xv = x0 - 5 + j over rows [z0-5, z0+BZ+5)
//      (its band plus the 5-row halo the stress stencil needs) from the
//      stress columns xv-4 .. xv+5 held in a shared-memory ring,
//   2. computes sigma_new for column xs = xv - 4 over its own rows from the
//      v_new columns xs-5 .. xs+4 held in a second ring.
// Stress columns, v_old and the per-cell parameters of the columns in use
// arrive through cp.async.bulk copies (one elected thread, completion on an
// mbarrier per stage) issued P iterations ahead. State is double buffered
// (old -> new) so halo rows and columns read by one CTA are never written by
// another during the step.
//
// Per-cell arithmetic is the reference's (coord:614-886, tensor:617-895,
// bond:654-913) with the same policy as the one-thread-per-cell kernels.
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

template <int V>
struct Lay {
  static constexpr int NVP = V == TTI_COORDINATE ? 5 : 3;  // coef1 coef2 invrho [sinv cosv]
  static constexpr int NSP = V == TTI_TENSOR ? 9 : 8;      // coef1 coef2 + moduli / angles
  static constexpr int NTAU = V == TTI_TENSOR ? 3 : 0;
  static constexpr int STAGE = 2 * VR + NVP * VR + NSP * BZ + NTAU * BZ;  // floats
  static constexpr int SRING = R * 3 * SR;
  static constexpr int VRING = NV * 2 * VR;
  static constexpr int FLOATS = SRING + VRING + P * STAGE + 32;
  static constexpr size_t BYTES = FLOATS * sizeof(float) + (P + 1) * sizeof(unsigned long long);
};

// source table and receiver lookup (kernel parameters)
__device__ __forceinline__ void vsource_cell(const FusedArgs &a, int x, int z, float &vx, float &vz)
{
  const int st = a.stype;
  if (st < 2 || a.src.n == 0) return;
  if (st == 8) {
    const float q = a.tab.q8;
    for (int n = 0; n < a.src.n; ++n) {
      const int dx = x - a.src.x[n], dz = z - a.src.z[n];
      if (dx < -1 || dx > 0 || dz < -1 || dz > 0) continue;
      const float s = __ldg(a.src.w + (size_t)n * a.src.nt + a.it);
      const float qs = __fmul_rn(q, s);
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
  // passes in the reference's block order: divergence, then curl, then forces
  for (int pass = 0; pass < 2; ++pass) {
    int kind;
    if (pass == 0) kind = (st == 2 || st == 4) ? 2 : (st == 3 ? 3 : (st >= 5 ? st : 0));
    else kind = st == 4 ? 3 : 0;
    if (kind == 0) continue;
    for (int n = 0; n < a.src.n; ++n) {
      const int dx = x - a.src.x[n], dz = z - a.src.z[n];
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

__device__ __forceinline__ void record(const FusedArgs &a, int kind, int x, int z, float v)
{
  const RecLookup &L = a.rec[kind];
  if (L.colptr == nullptr) return;
  const int b = __ldg(L.colptr + x), e = __ldg(L.colptr + x + 1);
  for (int j = b; j < e; ++j)
    if (__ldg(L.z + j) == z) L.out[(size_t)a.irec * L.n + __ldg(L.id + j)] = v;
}

template <int V, bool X>
__global__ void __launch_bounds__(BZ, 3) k_fused(const __grid_constant__ FusedArgs a)
{
  using A = Ar<X>;
  using Ly = Lay<V>;
  // shared memory: stress ring [R][3][SR] (row z at z - (z0 - 12)), velocity
  // ring [NV][2][VR] (row z at z - (z0 - 8)), P copy stages, the free-surface
  // exchange rows, then P + 1 mbarriers (stages, prologue)
  extern __shared__ __align__(128) float smem[];
  float *sring = smem;
  float *vring = sring + Ly::SRING;
  float *stage = vring + Ly::VRING;
  float *fsbuf = stage + P * Ly::STAGE;
  unsigned long long *bar = reinterpret_cast<unsigned long long *>(smem + Ly::FLOATS);

  const Grid &g = a.g;
  const int t = threadIdx.x;
  const int z0 = blockIdx.y * BZ;
  const int x0 = blockIdx.x * a.seg, x1 = min(x0 + a.seg, g.Nx);
  const int L = g.ldz;
  const int niter = (x1 - x0) + 9;  // xv = x0-5 .. x1+3
  const int xbeg = x0 - 5;
  // Undamped CTA: every cell it touches has D = 0, so coef1 = 1 and
  // coef2 = dt exactly (meal.c:486-487 with D = 0); those loads are skipped.
  const bool und = a.undamped_ok && (xbeg - 4 >= g.E) && (x1 + 3 + 5 < g.Nx - g.E) &&
                   (z0 - 9 >= (a.freesurface ? 0 : g.E)) && (z0 + BZ + 9 < g.Nz - g.E);
  const bool fs_band = a.freesurface && z0 == 0;

  // row ranges (clamped, 16-byte aligned) of the three kinds of column loads
  const int s_lo = max(z0 - 12, 0), s_hi = min(z0 + BZ + 12, L);
  const int v_lo = max(z0 - 8, 0), v_hi = min(z0 + BZ + 8, L);
  const int p_lo = z0, p_hi = min(z0 + BZ, L);

  auto ring_slot = [](int c, int n) { return (c + n * 4096) % n; };

  // one elected thread issues the copies of iteration j into stage j % P
  auto issue = [&](int j) {
    unsigned long long *b = bar + (j % P);
    float *st = stage + (j % P) * Ly::STAGE;
    const int xv = xbeg + j, cs = xv + 5, xs = xv - 4;
    unsigned bytes = 0;
    // pass 1: byte count (expect_tx must precede the copies)
    const bool has_s = cs >= 0 && cs < g.Nx;
    const bool has_v = xv >= 0 && xv < g.Nx;
    const bool has_p = xs >= x0 && xs < x1;
    const unsigned sb = (s_hi - s_lo) * 4u, vb = (v_hi - v_lo) * 4u, pb = (p_hi - p_lo) * 4u;
    if (has_s) bytes += 3 * sb;
    if (has_v) bytes += (2 + Ly::NVP - (und ? 2 : 0)) * vb;
    if (has_p) bytes += (Ly::NSP - (und ? 2 : 0) + Ly::NTAU) * pb;
    mbar_arrive_expect_tx(b, bytes);
    if (has_s) {
      float *dst = sring + ring_slot(cs, R) * 3 * SR + (s_lo - (z0 - 12));
      const size_t off = (size_t)cs * L + s_lo;
      bulk_g2s(dst, a.old.sxx + off, sb, b);
      bulk_g2s(dst + SR, a.old.szz + off, sb, b);
      bulk_g2s(dst + 2 * SR, a.old.sxz + off, sb, b);
    }
    if (has_v) {
      const size_t off = (size_t)xv * L + v_lo;
      float *dst = st + (v_lo - (z0 - 8));
      bulk_g2s(dst, a.old.vx + off, vb, b);
      bulk_g2s(dst + VR, a.old.vz + off, vb, b);
      float *pv = dst + 2 * VR;
      if (!und) {
        bulk_g2s(pv, a.p.coef1 + off, vb, b);
        bulk_g2s(pv + VR, a.p.coef2 + off, vb, b);
      }
      bulk_g2s(pv + 2 * VR, a.p.invrho + off, vb, b);
      if (V == TTI_COORDINATE) {
        bulk_g2s(pv + 3 * VR, a.p.snv + off, vb, b);
        bulk_g2s(pv + 4 * VR, a.p.csv + off, vb, b);
      }
    }
    if (has_p) {
      const size_t off = (size_t)xs * L + p_lo;
      float *dst = st + (2 + Ly::NVP) * VR + (p_lo - z0);
      const float *src[12];
      int n = 0;
      src[n++] = a.p.coef1;
      src[n++] = a.p.coef2;
      src[n++] = a.p.c11;
      src[n++] = a.p.c13;
      if (V == TTI_BOND) src[n++] = a.p.c15;
      src[n++] = a.p.c33;
      if (V == TTI_BOND) src[n++] = a.p.c35;
      src[n++] = a.p.c55;
      if (V == TTI_COORDINATE) {
        src[n++] = a.p.sn;
        src[n++] = a.p.cs;
      }
      if (V == TTI_TENSOR) {
        src[n++] = a.p.s2;
        src[n++] = a.p.c2;
        src[n++] = a.p.s2t;
        src[n++] = a.old.txx;
        src[n++] = a.old.tzz;
        src[n++] = a.old.txz;
      }
      for (int k = und ? 2 : 0; k < n; ++k) bulk_g2s(dst + k * BZ, src[k] + off, pb, b);
    }
  };

  if (t == 0) {
    for (int k = 0; k <= P; ++k) mbar_init(bar + k, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (t == 0) {
    // prologue: stress columns x0-9 .. x0-1 (read by the first stencils)
    unsigned long long *b = bar + P;
    const unsigned sb = (s_hi - s_lo) * 4u;
    unsigned bytes = 0;
    for (int c = x0 - 9; c < x0; ++c)
      if (c >= 0 && c < g.Nx) bytes += 3 * sb;
    mbar_arrive_expect_tx(b, bytes);
    for (int c = x0 - 9; c < x0; ++c) {
      if (c < 0 || c >= g.Nx) continue;
      float *dst = sring + ring_slot(c, R) * 3 * SR + (s_lo - (z0 - 12));
      const size_t off = (size_t)c * L + s_lo;
      bulk_g2s(dst, a.old.sxx + off, sb, b);
      bulk_g2s(dst + SR, a.old.szz + off, sb, b);
      bulk_g2s(dst + 2 * SR, a.old.sxz + off, sb, b);
    }
    for (int j = 0; j < P && j < niter; ++j) issue(j);
  }
  // On a timed-out wait: flag it, give the copies still in flight a bounded
  // time to land, and leave.
  auto bail = [&](int first_pending) {
    if (t == 0) {
      atomicOr(a.err, 2);
      for (int j = first_pending; j < first_pending + P && j < niter; ++j)
        mbar_wait(bar + (j % P), (j / P) & 1, 1u << 16);
    }
  };
  bool ok = mbar_wait(bar + P, 0);
  if (__syncthreads_or(!ok)) {
    bail(0);
    return;
  }

  const float dt = a.dt;
  for (int j = 0; j < niter; ++j) {
    ok = mbar_wait(bar + (j % P), (j / P) & 1);
    if (__syncthreads_or(!ok)) {
      bail(j);
      return;
    }
    const float *st = stage + (j % P) * Ly::STAGE;
    const int xv = xbeg + j, xs = xv - 4;

    // ---------------- velocity half-step at column xv
    if (xv >= 0 && xv < g.Nx) {
      const bool xin = xv >= NH && xv < g.Nx - NH;
      const bool own_x = xv >= x0 && xv < x1;
      float *vr = vring + ring_slot(xv, NV) * 2 * VR;
      const float *sbase[10];
#pragma unroll
      for (int k = 0; k < 10; ++k) sbase[k] = sring + ring_slot(xv - 4 + k, R) * 3 * SR;
      for (int pass = 0; pass < 2; ++pass) {
        int r;
        if (pass == 0) r = z0 + t;
        else if (t < 5) r = z0 - 5 + t;
        else if (t < 10) r = z0 + BZ + (t - 5);
        else break;
        if (r < 0 || r >= g.Nz) continue;
        const int iv = r - (z0 - 8);  // index in v rows
        float vx = st[iv], vz = st[VR + iv];
        if (xin && r >= g.izStart && r < g.Nz - NH) {
          const int is = r - (z0 - 12);  // index in sigma rows
          // d1 = sum C_k (s[x+k][z+k] - s[x-k+1][z-k+1]), d2 = sum C_k (s[x+k][z-k+1] - s[x-k+1][z+k]);
          // column xv+m lives in sbase[m+4]
          float d[3][2];
#pragma unroll
          for (int f = 0; f < 3; ++f) {
            float s1 = A::mul(rsg(0), A::sub(sbase[5][f * SR + is + 1], sbase[4][f * SR + is]));
            float s2 = A::mul(rsg(0), A::sub(sbase[5][f * SR + is], sbase[4][f * SR + is + 1]));
#pragma unroll
            for (int k = 2; k <= NH; ++k) {
              s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(sbase[4 + k][f * SR + is + k],
                                                         sbase[5 - k][f * SR + is - k + 1])));
              s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(sbase[4 + k][f * SR + is - k + 1],
                                                         sbase[5 - k][f * SR + is + k])));
            }
            d[f][0] = s1;
            d[f][1] = s2;
          }
          const float *pv = st + 2 * VR;
          const float c1 = und ? 1.0f : pv[iv], c2 = und ? dt : pv[VR + iv], ir = pv[2 * VR + iv];
          const float invdx = a.invdx, invdz = a.invdz;
          const float sxx_x = A::mul(A::mul(0.5f, A::add(d[0][0], d[0][1])), invdx);
          const float szz_z = A::mul(A::mul(0.5f, A::sub(d[1][0], d[1][1])), invdz);
          const float sxz_x = A::mul(A::mul(0.5f, A::add(d[2][0], d[2][1])), invdx);
          const float sxz_z = A::mul(A::mul(0.5f, A::sub(d[2][0], d[2][1])), invdz);
          const float br = A::mul(c2, ir);
          float fx, fz;
          if (V == TTI_COORDINATE) {
            const float sxx_z = A::mul(A::mul(0.5f, A::sub(d[0][0], d[0][1])), invdx);  // coord:633
            const float szz_x = A::mul(A::mul(0.5f, A::add(d[1][0], d[1][1])), invdx);
            const float sv = pv[3 * VR + iv], cv = pv[4 * VR + iv];
            fx = A::add(A::add(A::sub(A::mul(cv, sxx_x), A::mul(sv, sxx_z)), A::mul(sv, sxz_x)), A::mul(cv, sxz_z));
            fz = A::add(A::add(A::sub(A::mul(cv, sxz_x), A::mul(sv, sxz_z)), A::mul(sv, szz_x)), A::mul(cv, szz_z));
          } else {
            fx = A::add(sxx_x, sxz_z);
            fz = A::add(sxz_x, szz_z);
          }
          vx = A::add(A::mul(c1, vx), A::mul(br, fx));
          vz = A::add(A::mul(c1, vz), A::mul(br, fz));
        }
        vsource_cell(a, xv, r, vx, vz);
        vr[iv] = vx;
        vr[VR + iv] = vz;
        if (own_x && pass == 0) {
          const size_t gi = (size_t)xv * L + r;
          a.nw.vx[gi] = vx;
          a.nw.vz[gi] = vz;
          if (a.irec >= 0) {
            record(a, TTI_REC_VX, xv, r, vx);
            record(a, TTI_REC_VZ, xv, r, vz);
          }
        }
      }
    }
    __syncthreads();

    // ---------------- stress half-step at column xs
    const bool do_s = xs >= x0 && xs < x1;
    const int z = z0 + t;
    float sxx = 0.f, szz = 0.f, sxz = 0.f, txx = 0.f, tzz = 0.f, txz = 0.f;
    const bool row_ok = z < g.Nz;
    const bool sin_ = do_s && row_ok && xs >= NH && xs < g.Nx - NH && z >= g.izStart && z < g.Nz - NH;
    if (do_s && row_ok) {
      const float *so = sring + ring_slot(xs, R) * 3 * SR + (z - (z0 - 12));
      sxx = so[0];
      szz = so[SR];
      sxz = so[2 * SR];
      const float *sp = st + (2 + Ly::NVP) * VR + t;
      if (V == TTI_TENSOR) {
        txx = sp[(Ly::NSP + 0) * BZ];
        tzz = sp[(Ly::NSP + 1) * BZ];
        txz = sp[(Ly::NSP + 2) * BZ];
      }
      if (sin_) {
        const float *vb[10];
#pragma unroll
        for (int k = 0; k < 10; ++k) vb[k] = vring + ring_slot(xs - 5 + k, NV) * 2 * VR;
        // column xs+m lives in vb[m+5]; row z at index iv
        const int iv = z - (z0 - 8);
        float d[2][2];
#pragma unroll
        for (int f = 0; f < 2; ++f) {
          // d1 = sum C_k (v[x+k-1][z+k-1] - v[x-k][z-k]), d2 = sum C_k (v[x+k-1][z-k] - v[x-k][z+k-1])
          float s1 = A::mul(rsg(0), A::sub(vb[5][f * VR + iv], vb[4][f * VR + iv - 1]));
          float s2 = A::mul(rsg(0), A::sub(vb[5][f * VR + iv - 1], vb[4][f * VR + iv]));
#pragma unroll
          for (int k = 2; k <= NH; ++k) {
            s1 = A::add(s1, A::mul(rsg(k - 1), A::sub(vb[4 + k][f * VR + iv + k - 1], vb[5 - k][f * VR + iv - k])));
            s2 = A::add(s2, A::mul(rsg(k - 1), A::sub(vb[4 + k][f * VR + iv - k], vb[5 - k][f * VR + iv + k - 1])));
          }
          d[f][0] = s1;
          d[f][1] = s2;
        }
        const float invdx = a.invdx, invdz = a.invdz;
        float vxx = A::mul(A::mul(0.5f, A::add(d[0][0], d[0][1])), invdx);
        float vxz = A::mul(A::mul(0.5f, A::sub(d[0][0], d[0][1])), invdz);
        float vzx = A::mul(A::mul(0.5f, A::add(d[1][0], d[1][1])), invdx);
        float vzz = A::mul(A::mul(0.5f, A::sub(d[1][0], d[1][1])), invdz);
        const float c1 = und ? 1.0f : sp[0], c2 = und ? dt : sp[BZ];
        const float c11 = sp[2 * BZ], c13 = sp[3 * BZ];
        if (V == TTI_COORDINATE) {
          const float c33 = sp[4 * BZ], c55 = sp[5 * BZ], s = sp[6 * BZ], c = sp[7 * BZ];
          float r = A::add(A::mul(s, vxx), A::mul(c, vxz));
          vxx = A::sub(A::mul(c, vxx), A::mul(s, vxz));
          vxz = r;
          r = A::add(A::mul(s, vzx), A::mul(c, vzz));
          vzx = A::sub(A::mul(c, vzx), A::mul(s, vzz));
          vzz = r;
          sxx = A::add(A::mul(c1, sxx), A::mul(c2, A::add(A::mul(c11, vxx), A::mul(c13, vzz))));
          szz = A::add(A::mul(c1, szz), A::mul(c2, A::add(A::mul(c13, vxx), A::mul(c33, vzz))));
          sxz = A::add(A::mul(c1, sxz), A::mul(A::mul(c2, c55), A::add(vzx, vxz)));
        } else if (V == TTI_TENSOR) {
          const float c33 = sp[4 * BZ], c55 = sp[5 * BZ], s2 = sp[6 * BZ], cc2 = sp[7 * BZ], s2t = sp[8 * BZ];
          const float sh = A::add(vxz, vzx);
          const float exx = A::sub(A::add(A::mul(cc2, vxx), A::mul(s2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
          const float ezz = A::add(A::add(A::mul(s2, vxx), A::mul(cc2, vzz)), A::mul(A::mul(0.5f, s2t), sh));
          const float exz = A::add(A::mul(s2t, A::sub(vxx, vzz)), A::mul(A::sub(cc2, s2), sh));
          txx = A::add(A::mul(c1, txx), A::mul(c2, A::add(A::mul(c11, exx), A::mul(c13, ezz))));
          tzz = A::add(A::mul(c1, tzz), A::mul(c2, A::add(A::mul(c13, exx), A::mul(c33, ezz))));
          txz = A::add(A::mul(c1, txz), A::mul(A::mul(c2, c55), exz));
          sxx = A::add(A::add(A::mul(cc2, txx), A::mul(s2, tzz)), A::mul(s2t, txz));
          szz = A::sub(A::add(A::mul(s2, txx), A::mul(cc2, tzz)), A::mul(s2t, txz));
          sxz = A::add(A::mul(A::mul(-0.5f, s2t), A::sub(txx, tzz)), A::mul(A::sub(cc2, s2), txz));
        } else {
          const float c15 = sp[4 * BZ], c33 = sp[5 * BZ], c35 = sp[6 * BZ], c55 = sp[7 * BZ];
          const float sh = A::add(vzx, vxz);
          sxx = A::add(A::mul(c1, sxx), A::mul(c2, A::add(A::add(A::mul(c11, vxx), A::mul(c13, vzz)), A::mul(c15, sh))));
          szz = A::add(A::mul(c1, szz), A::mul(c2, A::add(A::add(A::mul(c13, vxx), A::mul(c33, vzz)), A::mul(c35, sh))));
          sxz = A::add(A::mul(c1, sxz), A::mul(c2, A::add(A::add(A::mul(c15, vxx), A::mul(c35, vzz)), A::mul(c55, sh))));
        }
      }
    }
    // free surface: stress image about row E (coord:847-863) for interior columns
    if (fs_band) {
      const int E = g.izStart;
      const bool col_fs = do_s && xs >= NH && xs < g.Nx - NH;
      if (col_fs && z >= E && z <= E + NH) {
        fsbuf[z - E] = sxx;
        fsbuf[8 + z - E] = szz;
        fsbuf[16 + z - E] = sxz;
      }
      __syncthreads();
      if (col_fs) {
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
    if (do_s && row_ok) {
      // stress source (stype 1), after the free surface (coord:865-886)
      if (a.stype == 1) {
        for (int n = 0; n < a.src.n; ++n) {
          const int dx = xs - a.src.x[n], dz = z - a.src.z[n];
          if (dx < -NH || dx > NH || dz < -NH || dz > NH) continue;
          const float w = a.tab.k1[(dx + NH) * 11 + (dz + NH)];
          const float s = __ldg(a.src.w + (size_t)n * a.src.nt + a.it);
          const float ws = __fmul_rn(w, s);
          sxx = __fadd_rn(sxx, ws);
          szz = __fadd_rn(szz, ws);
          if (V == TTI_TENSOR) {
            txx = __fadd_rn(txx, ws);
            tzz = __fadd_rn(tzz, ws);
          }
        }
      }
      const size_t gi = (size_t)xs * L + z;
      a.nw.sxx[gi] = sxx;
      a.nw.szz[gi] = szz;
      a.nw.sxz[gi] = sxz;
      if (V == TTI_TENSOR) {
        // tau is only updated in the interior; elsewhere it keeps its value
        // plus the stype-1 source (tensor:871-895)
        a.nw.txx[gi] = txx;
        a.nw.tzz[gi] = tzz;
        a.nw.txz[gi] = txz;
      }
      if (a.irec >= 0) record(a, TTI_REC_P, xs, z, __fmul_rn(0.5f, __fadd_rn(sxx, szz)));
    }
    __syncthreads();
    if (t == 0 && j + P < niter) {
      fence_proxy_async();
      issue(j + P);
    }
  }
}

}  // namespace

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

void launch_check_undamped(const Grid &g, const float *coef1, const float *coef2, float dt, int zD, int *count,
                           cudaStream_t st)
{
  const int nx = g.Nx - 2 * g.E;
  if (nx <= 0) return;
  k_check_undamped<<<dim3(1, nx), 256, 0, st>>>(g, coef1, coef2, dt, zD, count);
}

size_t smem_bytes(int variant)
{
  switch (variant) {
  case TTI_COORDINATE: return Lay<TTI_COORDINATE>::BYTES;
  case TTI_TENSOR: return Lay<TTI_TENSOR>::BYTES;
  default: return Lay<TTI_BOND>::BYTES;
  }
}

template <int V, bool X>
static cudaError_t launch_t(const FusedArgs &a, cudaStream_t st)
{
  const size_t bytes = Lay<V>::BYTES;
  static bool configured = false;  // per template instance, per process
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_fused<V, X>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e != cudaSuccess) return e;
    configured = true;
  }
  const dim3 grid((a.g.Nx + a.seg - 1) / a.seg, (a.g.Nz + BZ - 1) / BZ);
  k_fused<V, X><<<grid, BZ, bytes, st>>>(a);
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
