// Packing of the per-cell parameters (pack.cuh) and the check that coef1 = 1,
// coef2 = dt hold outside the MEAL rims, which lets the tiled kernels skip
// those loads in undamped tiles.
#include "pack.cuh"

namespace ttifd {
namespace packed {
namespace {

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

// one block per interior column: counts the rows [zD, Nz - E) where the MEAL
// coefficients differ from the undamped values
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

}  // namespace packed
}  // namespace ttifd
