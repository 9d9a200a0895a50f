// Tiled half-step kernels (tiled_step.cu): velocity and stress updates in
// place, each CTA loading its halo tile with one 2D TMA copy per field.
#pragma once

#include <cuda.h>

#include "fused.cuh"

namespace ttifd {
namespace tiled {

constexpr int TX = 16;        // tile columns (x)
constexpr int TZ = 128;       // tile rows (z)
constexpr int BZ = TZ + 16;   // TMA box rows: [z0-8, z0+TZ+8), 16-byte aligned start
constexpr int BX = TX + 9;    // TMA box columns: the tile plus the 10-point stencil's halo
constexpr int NT = 512;       // threads per CTA: one row x TX/4 columns each (64 warps per SM at 4 CTAs)
// floats per field region in shared memory, 128-byte aligned
constexpr int FIELD = (BX * BZ * 4 + 127) / 128 * 128 / 4;

struct alignas(64) HalfArgs {
  CUtensorMap map[3];  // velocity kernel: sxx szz sxz; stress kernel: vx vz
  Grid g;
  Fields f;
  Params p;
  fused::Packed pk;
  float invdx, invdz, dt;
  int z_base;  // first tile row (multiple of 4, <= izStart)
  int x_base;  // first tile column (= 5)
  int undamped_ok;
  int freesurface;
  int *err;    // bit 4: a TMA wait timed out
  int nt;      // batched launches: time steps of this instance (its CTAs idle once the step counter reaches it)
  int tiles_z; // batched launches: tile rows of this instance's grid
};

// One CTA of a batched launch: instance `inst`, tile `tile` (row tile % tiles_z, column tile / tiles_z).
struct Work {
  int inst, tile;
};

// Encodes the 2D tensor map of one [Nx][ldz] field for the halo box.
bool encode_map(CUtensorMap *map, const Grid &g, float *field);
// Tile grid; *z_base receives the first tile row.
dim3 grid(const Grid &g, int *z_base);
cudaError_t launch_velocity(const HalfArgs &a, int variant, bool exact, cudaStream_t st);
cudaError_t launch_stress(const HalfArgs &a, int variant, bool exact, cudaStream_t st);
// Batched: one launch over all instances' tiles. `inst` (device) holds each
// instance's arguments (z_base set), `work` (device) the CTA -> (instance, tile)
// table; `step` (device) is the shared step counter.
cudaError_t launch_velocity_batch(const HalfArgs *inst, const Work *work, int nwork, const int *step, int variant,
                                  bool exact, cudaStream_t st);
cudaError_t launch_stress_batch(const HalfArgs *inst, const Work *work, int nwork, const int *step, int variant,
                                bool exact, cudaStream_t st);
// Sets the kernels' shared-memory attributes (call before a stream capture).
cudaError_t prepare_batch(int variant, bool exact);

}  // namespace tiled
}  // namespace ttifd
