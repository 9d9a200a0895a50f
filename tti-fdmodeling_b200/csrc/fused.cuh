// Fused single-kernel time step (fused_step.cu).
#pragma once

#include "launch.cuh"

namespace ttifd {
namespace fused {

constexpr int BZ = 128;    // rows owned by a CTA (= threads per CTA)
constexpr int SR = BZ + 24;  // stress rows staged: [z0-12, z0+BZ+12)
constexpr int VR = BZ + 16;  // velocity rows staged/computed: [z0-8, z0+BZ+8)
constexpr int NV = 10;       // velocity ring columns (stencil width)
constexpr int P = 4;         // copy stages in flight
constexpr int R = P + 9;     // stress ring columns (stencil width + prefetch)

// Receivers of one component grouped by padded-grid column:
// entries colptr[x] .. colptr[x+1]-1 hold row z[] and trace index id[].
struct RecLookup {
  const int *colptr, *z, *id;
  float *out;  // time-major [irec][n]
  int n;
};

struct FusedArgs {
  Grid g;
  Fields old, nw;
  Params p;
  float invdx, invdz, dt;
  int seg;  // columns per CTA
  int stype;
  SourceSet src;  // padded-grid positions
  SourceTables tab;
  int it;
  int irec;  // receiver sample index of this step, -1 when not recording
  RecLookup rec[3];
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
