// One-time device precompute: MEAL damping/scaling, MEAL FD coefficients,
// the per-cell stiffness of each formulation, the Bond free-surface rewrite
// and the velocity-node averages.
//
// Every product, sum and quotient is rounded separately (explicit _rn
// intrinsics) in the reference's expression order, and the scalar pieces that
// involve libm (MEAL weights w(l), log(Rcoef)) are evaluated on the host, so
// the arrays match the reference's setup dumps except where CUDA's double
// sin/cos differ from the host libm in the last place.
#include "launch.cuh"

namespace ttifd {

namespace {

__device__ __forceinline__ double dm(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double da(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double ds(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double dd(double a, double b) { return __ddiv_rn(a, b); }
__device__ __forceinline__ float f2(double a) { return __double2float_rn(a); }
__device__ __forceinline__ float fm(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float fa(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float fs(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float fd(float a, float b) { return __fdiv_rn(a, b); }

constexpr double kPi = 3.14159265358979323846;

// Per cell: MEAL profile (meal.c:51-201), MEAL FD coefficients with the
// vp/vs/rho/D rescale (meal.c:450-490), stiffness (coord:497-515,
// tensor:500-519, bond:493-526) and the Bond free-surface rewrite
// (bond:543-568, a same-cell operation on row iz = E).
__global__ void k_setup_cell(Grid g, SetupIn in, SetupOut out, MealConst mc, int variant, float scalar,
                             int freesurface)
{
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = blockIdx.y;
  if (iz >= g.Nz || ix >= g.Nx) return;
  const size_t i = (size_t)ix * g.ldz + iz;       // outputs
  const size_t ri = (size_t)ix * in.pitch + iz;  // the raw model
  const int nl = g.E;
  float vp = in.vp[ri], vs = in.vs[ri], rho = in.rho[ri];

  // ---- MEAL profile
  const float Vs = vs == 0.0f ? fd(vp, mc.sqrt3) : vs;
  float Dx = 0.0f, Dz = 0.0f, Bx = 1.0f, Bz = 1.0f;
  int lz = 0, lx = 0;
  if (freesurface == 0 && iz < nl) lz = nl - iz;
  if (iz >= g.Nz - nl) lz = iz - (g.Nz - nl - 1);
  const int izs = freesurface == 0 ? 0 : nl;
  if (iz >= izs && ix < nl) lx = nl - ix;
  if (iz >= izs && ix >= g.Nx - nl) lx = ix - (g.Nx - nl - 1);
  if (lz) {
    const float w = mc.w[lz];
    const float d0 = fd(fm(fm(-3.0f, vp), mc.logR), mc.two_thz);
    const float beta = fd(fm(2.0f, fd(Vs, mc.dz_fpeak)), 10.0f);
    Dz = fm(d0, w);
    Bz = fa(1.0f, fm(fs(beta, 1.0f), w));
  }
  if (lx) {
    const float w = mc.w[lx];
    const float d0 = fd(fm(fm(-3.0f, vp), mc.logR), mc.two_thx);
    const float beta = fd(fm(2.0f, fd(Vs, mc.dx_fpeak)), 10.0f);
    Dx = fm(d0, w);
    Bx = fa(1.0f, fm(fs(beta, 1.0f), w));
  }
  float D = __fsqrt_rn(fa(fm(Dx, Dx), fm(Dz, Dz)));
  const float Beta = fa(__fsqrt_rn(fa(fm(fs(Bx, 1.0f), fs(Bx, 1.0f)), fm(fs(Bz, 1.0f), fs(Bz, 1.0f)))), 1.0f);

  // ---- MEAL FD coefficients (order 1)
  vp = fd(vp, Beta);
  vs = fd(vs, Beta);
  rho = fm(rho, Beta);
  D = fd(D, Beta);
  const double hdD = dm(dm(0.5, (double)mc.dt), (double)D);
  out.D[i] = D;
  out.Beta[i] = Beta;
  out.coef1[i] = f2(dd(ds(1.0, hdD), da(1.0, hdD)));
  out.coef2[i] = f2(dd((double)mc.dt, da(1.0, hdD)));
  out.vp[i] = vp;
  out.vs[i] = vs;
  out.rho[i] = rho;

  // ---- stiffness
  const float q = fd(vs, vp);
  const double f = ds(1.0, dm((double)q, (double)q));
  const float rvv = fm(fm(rho, vp), vp);
  const double C11 = dm((double)rvv, da(1.0, dm(2.0, (double)in.eps[ri])));
  const double C13 =
      dm((double)rho, ds(dm((double)fm(vp, vp), __dsqrt_rn(dm(f, da(f, dm(2.0, (double)in.delta[ri]))))),
                         (double)fm(vs, vs)));
  const float c33f = rvv;
  const float c55f = fm(fm(rho, vs), vs);
  const float th = f2(dm(dd((double)fm(scalar, in.theta[ri]), 180.0), kPi));
  const double thd = (double)th;
  if (variant == TTI_BOND) {
    const double C33 = (double)c33f, C55 = (double)c55f;
    const double sn = sin(thd), cs = cos(thd);
    const double s2 = dm(sn, sn), c2 = dm(cs, cs);
    const double s4 = dm(s2, s2), c4 = dm(c2, c2);
    const double s2t = sin(dm(2.0, thd)), c2t = cos(dm(2.0, thd));
    const double s22 = dm(s2t, s2t), c22 = dm(c2t, c2t);
    const double hc = da(dm(0.5, C13), C55);
    const double C13p2C55 = da(C13, dm(2.0, C55));
    float c11 = f2(da(da(dm(C11, c4), dm(C33, s4)), dm(hc, s22)));
    float c13 = f2(da(dm(ds(dm(0.25, da(C11, C33)), C55), s22), dm(C13, da(s4, c4))));
    float c15 = f2(dm(dm(0.5, da(da(dm(dm(-1.0, C11), c2), dm(C33, s2)), dm(C13p2C55, c2t))), s2t));
    float c33 = f2(da(da(dm(C11, s4), dm(C33, c4)), dm(hc, s22)));
    float c35 = f2(dm(dm(0.5, ds(da(dm(dm(-1.0, C11), s2), dm(C33, c2)), dm(C13p2C55, c2t))), s2t));
    float c55 = f2(da(dm(dm(0.25, ds(da(C11, C33), dm(2.0, C13))), s22), dm(C55, c22)));
    if (freesurface == 1 && iz == nl) {
      float n35 = -fd(fs(fm(c13, c55), fm(c15, c35)), fs(fm(c33, c55), fm(c35, c35)));
      const float n55 = fd(fs(fm(c13, n35), fm(c15, c33)), fs(fm(c33, c55), fm(n35, n35)));
      if (isnan(n35) || isinf(n35)) n35 = -fd(c13, c33);
      if (isnan(n35) || isinf(n35)) n35 = 0.0f;
      c11 = fa(fs(c11, fm(c13, n35)), fm(c15, n55));
      c13 = c15 = c33 = c35 = c55 = 0.0f;
    }
    out.c11[i] = c11;
    out.c13[i] = c13;
    out.c15[i] = c15;
    out.c33[i] = c33;
    out.c35[i] = c35;
    out.c55[i] = c55;
  } else {
    out.c11[i] = f2(C11);
    out.c13[i] = f2(C13);
    out.c33[i] = c33f;
    out.c55[i] = c55f;
    if (variant == TTI_COORDINATE) {
      out.sn[i] = f2(sin(thd));
      out.cs[i] = f2(cos(thd));
    } else {
      const double sn = sin(thd), cs = cos(thd);
      out.s2[i] = f2(dm(sn, sn));
      out.c2[i] = f2(dm(cs, cs));
      out.s2t[i] = f2(sin(dm(2.0, thd)));
    }
  }
}

// Buoyancy (and for the coordinate formulation sin/cos theta) averaged over
// the four stress nodes around the velocity node (ix+1/2, iz+1/2); the last
// row and column keep the stress-node value (coord:516-537).
__global__ void k_setup_average(Grid g, const float *__restrict__ rho, const float *__restrict__ sn,
                                const float *__restrict__ cs, float *__restrict__ invrho, float *__restrict__ snv,
                                float *__restrict__ csv)
{
  const int iz = blockIdx.x * blockDim.x + threadIdx.x;
  const int ix = blockIdx.y;
  if (iz >= g.Nz || ix >= g.Nx) return;
  const int L = g.ldz;
  const size_t i = (size_t)ix * L + iz;
  const bool inner = ix < g.Nx - 1 && iz < g.Nz - 1;
  if (inner) {
    const float s = fa(fa(fa(rho[i], rho[i + L]), rho[i + 1]), rho[i + L + 1]);
    invrho[i] = f2(dd(4.0, (double)s));
  } else {
    invrho[i] = f2(dd(1.0, (double)rho[i]));
  }
  if (snv) {
    if (inner) {
      snv[i] = f2(dm(0.25, (double)fa(fa(fa(sn[i], sn[i + L]), sn[i + 1]), sn[i + L + 1])));
      csv[i] = f2(dm(0.25, (double)fa(fa(fa(cs[i], cs[i + L]), cs[i + 1]), cs[i + L + 1])));
    } else {
      snv[i] = sn[i];
      csv[i] = cs[i];
    }
  }
}

// `na` dense physical [nx][nz] arrays (phys, nz * nx floats apart) into dense
// padded [Nx][Nz] arrays (pad, Nz * Nx floats apart, Nz = nz + 2E), as
// padModel2d (padmod.c:33-59) pads them on the host: its first pass copies
// row E (Nz - E - 1) up (down) in every physical column, its second copies
// column E (Nx - E - 1) left (right) at full height, so every rim cell holds
// the value of the physical cell at its clamped column and row.
__global__ void k_expand_physical(const float *phys, float *pad, int na, int nz, int nx, int E)
{
  const int Nz = nz + 2 * E, Nx = nx + 2 * E;
  const int iz = blockIdx.x * blockDim.x + threadIdx.x, ix = blockIdx.y;
  if (iz >= Nz || ix >= Nx) return;
  const int sx = min(max(ix - E, 0), nx - 1), sz = min(max(iz - E, 0), nz - 1);
  const size_t np = (size_t)Nz * Nx, nq = (size_t)nz * nx;
  const size_t d = (size_t)ix * Nz + iz, s = (size_t)sx * nz + sz;
  for (int k = 0; k < na; ++k) pad[k * np + d] = phys[k * nq + s];
}

}  // namespace

void launch_setup(const Grid &g, const SetupIn &in, const SetupOut &out, const MealConst &mc, int variant,
                  float scalar, int freesurface, cudaStream_t st)
{
  dim3 blk(128), grd((g.Nz + 127) / 128, g.Nx);
  k_setup_cell<<<grd, blk, 0, st>>>(g, in, out, mc, variant, scalar, freesurface);
  k_setup_average<<<grd, blk, 0, st>>>(g, out.rho, out.sn, out.cs, out.invrho, out.snv, out.csv);
}

void launch_expand_physical(const float *phys, float *pad, int na, int nz, int nx, int E, cudaStream_t st)
{
  const int Nz = nz + 2 * E, Nx = nx + 2 * E;
  k_expand_physical<<<dim3((Nz + 127) / 128, Nx), 128, 0, st>>>(phys, pad, na, nz, nx, E);
}

}  // namespace ttifd
