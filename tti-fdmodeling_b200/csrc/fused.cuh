// Fused single-kernel time step (fused_step.cu).
#pragma once

#include "launch.cuh"

namespace ttifd {
namespace fused {

constexpr int NT = 192;      // threads per CTA: one velocity row each
constexpr int BZ = NT - 10;  // rows owned by a CTA (velocity rows add a 5-row halo each side)
constexpr int SR = 208;      // stress rows staged: [floor4(z0-9), ceil4(z0+BZ+10)) <= BZ + 25
constexpr int R = 16;        // stress ring columns (power of two: slot = column & 15)
constexpr int P = R - 10;    // stress columns in flight ahead of use
constexpr int NV = 16;       // velocity ring columns (>= 11)
constexpr int VSTR = NT + 12;  // floats per velocity-ring row block (halo reads reach NT + 8)
constexpr int MAXSRC = 32;     // sources handled in the fused step (staged in shared memory)

// Per-cell parameters packed for wide loads (built once at upload):
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

struct FusedArgs {
  Grid g;
  Fields old, nw;
  Params p;
  Packed pk;
  float invdx, invdz, dt;
  int seg;  // columns per CTA
  int bz;   // rows per band (<= BZ; bands balanced over Nz)
  int stype;
  SourceSet src;  // padded-grid positions
  SourceTables tab;
  int it;
  int freesurface;
  int undamped_ok;  // coef1 == 1 and coef2 == dt verified outside the rims
  int *err;         // bit 2: a copy wait timed out
};

size_t smem_bytes(int variant);
// fills the packed parameter arrays from the per-parameter arrays
void launch_pack(const Grid &g, const Params &p, const Packed &pk, int variant, cudaStream_t st);
cudaError_t launch_fused(const FusedArgs &a, int variant, bool exact, cudaStream_t st);
// counts cells of [E, Nx-E) x [zD, Nz-E) with coef1 != 1 or coef2 != dt
void launch_check_undamped(const Grid &g, const float *coef1, const float *coef2, float dt, int zD, int *count,
                           cudaStream_t st);

}  // namespace fused
}  // namespace ttifd
