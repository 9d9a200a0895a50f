// Per-cell parameters packed for wide loads (pack.cu), built once per model
// upload and read by the tiled half-step kernels and the adjoint kernels.
#pragma once

#include "launch.cuh"

namespace ttifd {
namespace packed {

// One 8- or 16-byte load per cell instead of two to four:
//   cf  = (coef1, coef2)
//   vsc = (sin, cos) of theta at the velocity node      (coordinate)
//   c4  = (c11, c13, c33, c55)
//   sc  = (sin, cos) of theta                            (coordinate)
//         (sin^2, cos^2)                                 (tensor; sin 2theta stays scalar)
//         (c15, c35)                                     (Bond)
struct Packed {
  float2 *cf, *vsc, *sc;
  float4 *c4;
};

// fills the packed parameter arrays from the per-parameter arrays
void launch_pack(const Grid &g, const Params &p, const Packed &pk, int variant, cudaStream_t st);
// counts cells of [E, Nx-E) x [zD, Nz-E) with coef1 != 1 or coef2 != dt
void launch_check_undamped(const Grid &g, const float *coef1, const float *coef2, float dt, int zD, int *count,
                           cudaStream_t st);

}  // namespace packed
}  // namespace ttifd
