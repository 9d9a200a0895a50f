// Fused single-kernel time step (fused_step.cu).
#pragma once

#include "launch.cuh"

namespace ttifd {
namespace fused {

constexpr int NT = 224;      // threads per CTA: one velocity row each
constexpr int BZ = NT - 10;  // rows owned by a CTA (velocity rows add a 5-row halo each side)
constexpr int SR = 240;      // stress rows staged: [floor4(z0-9), ceil4(z0+BZ+10)) <= BZ + 25
constexpr int NV = 11;       // velocity ring columns (stencil width + 1: no end-of-column barrier)
constexpr int P = 4;         // stress columns in flight ahead of use
constexpr int R = P + 10;    // stress ring columns (stencil width + prefetch + 1)

struct FusedArgs {
  Grid g;
  Fields old, nw;
  Params p;
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
cudaError_t launch_fused(const FusedArgs &a, int variant, bool exact, cudaStream_t st);
// counts cells of [E, Nx-E) x [zD, Nz-E) with coef1 != 1 or coef2 != dt
void launch_check_undamped(const Grid &g, const float *coef1, const float *coef2, float dt, int zD, int *count,
                           cudaStream_t st);

}  // namespace fused
}  // namespace ttifd
