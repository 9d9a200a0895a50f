// Tiled half-step kernels (tiled_step.cu): velocity and stress updates in
// place, each CTA loading its halo tile with one 2D TMA copy per field.
#pragma once

#include <cuda.h>

#include "pack.cuh"

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
  packed::Packed pk;
  float invdx, invdz, dt;
  int z_base;  // first tile row (multiple of 4, <= izStart)
  int x_base;  // first tile column (= 5)
  int undamped_ok;
  int freesurface;
  int *err;    // bit 4: a TMA wait timed out
  int nt;      // batched launches: time steps of this instance (its CTAs idle once the step counter reaches it)
  int tiles_z; // batched launches: tile rows of this instance's grid
  int square;  // FMA mode with dx == dz: stencil coefficients hc fold in h = 0.5 / dx
  unsigned wait_limit;  // polls of the first TMA wait before it gives up (tma::WAIT_LIMIT)
  float hc[5]; // h * C_k
  // Gradient forward pass (null: nothing kept). Velocity update, coordinate
  // rotation: per cell the stress derivative combinations the adjoint's
  // theta_v terms need (sxz_x - sxx_z, szz_x - sxz_z, sxx_x + sxz_z,
  // sxz_x + szz_z). Stress update: the strain rates vxx vxz vzx vzz (not
  // rotated), and for the tensor rotation the tau it starts from (kt).
  float *kd[4];
  float *kt[3];
};

// Sets square / hc for FMA-mode launches on grids with dx == dz.
inline void set_square(HalfArgs &a, bool exact)
{
  a.square = !exact && a.invdx == a.invdz;
  for (int k = 0; k < 5; ++k) a.hc[k] = 0.5f * a.invdx * rsg(k);
}

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
// Batched: one launch over all instances' tiles (each instance's arguments
// with z_base set), driven by the work table.
struct BatchLaunch {
  const HalfArgs *inst;  // device: each instance's arguments (velocity or stress maps)
  const Work *work;      // device: the CTA -> (instance, tile) table
  int nwork;
  const int *step;       // device: the shared step counter
  int variant;
  bool exact, square;    // square: every instance has folded coefficients (set_square)
  bool persistent;       // one resident wave of CTAs walks the table (else one CTA per item)
};
cudaError_t launch_velocity_batch(const BatchLaunch &l, cudaStream_t st);
cudaError_t launch_stress_batch(const BatchLaunch &l, cudaStream_t st);
// Sets the kernels' shared-memory attributes (call before a stream capture).
cudaError_t prepare_batch(BatchLaunch l);

// Device side of the TMA halo tiles, shared by the tiled forward and adjoint kernels.
namespace tma {

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

// Polls of a bounded TMA wait (about a second): a copy that never lands cannot
// hang the GPU. A handle may lower it (TTIFD_WAIT_LIMIT at tti_create) to run
// the timeout path without a fault.
constexpr unsigned WAIT_LIMIT = 1u << 20;

__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, unsigned parity, unsigned limit = WAIT_LIMIT)
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

__device__ __forceinline__ void tma_load_2d(float *dst, const CUtensorMap *map, int c_inner, int c_outer,
                                            unsigned long long *bar)
{
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<unsigned long long>(map)), "r"(c_inner), "r"(c_outer), "r"(smem_u32(bar))
      : "memory");
}

static_assert((BZ * 4) % 16 == 0, "TMA inner box extent must be a multiple of 16 bytes");

// Issues the TMA copies of the halo boxes of `n` fields (origin row z0 - 8,
// column x0 - xoff); waited for by wait_tiles. With ph < 0 the barrier is
// initialised here (a CTA that loads one tile); with ph >= 0 it is a barrier
// the CTA initialised once, whose phase ph these copies complete (a CTA that
// loads tile after tile: an mbarrier must not be initialised again while it
// is valid).
__device__ __forceinline__ void issue_tiles(const CUtensorMap *map, float *sm, unsigned long long *bar, int n, int z0,
                                            int x0, int xoff, int ph = -1)
{
  constexpr unsigned BOX_BYTES = BX * BZ * 4;
  const int t = threadIdx.x;
  if (t == 0 && ph < 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();  // also: every thread is done with the boxes these copies replace
  if (t == 0) {
    mbar_arrive_expect_tx(bar, n * BOX_BYTES);
    for (int f = 0; f < n; ++f) tma_load_2d(sm + f * FIELD, map + f, z0 - 8, x0 - xoff, bar);
  }
}

// returns false (all threads) after a timed-out wait
__device__ __forceinline__ bool wait_tiles(int *err, unsigned long long *bar, unsigned limit = WAIT_LIMIT,
                                           unsigned parity = 0)
{
  const bool ok = mbar_wait(bar, parity, limit);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicOr(err, 4);
      mbar_wait(bar, parity, 1u << 16);  // give the copies in flight a bounded time
    }
    return false;
  }
  return true;
}

// The halo boxes of ng groups of `per` fields each, one barrier per group
// (bars[0..ng)), so that a CTA can work on a group while the next is in flight.
__device__ __forceinline__ void issue_groups(const CUtensorMap *map, float *sm, unsigned long long *bars, int ng,
                                             int per, int z0, int x0, int xoff)
{
  constexpr unsigned BOX_BYTES = BX * BZ * 4;
  const int t = threadIdx.x;
  if (t == 0) {
    for (int q = 0; q < ng; ++q) mbar_init(bars + q, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (t == 0)
    for (int q = 0; q < ng; ++q) {
      mbar_arrive_expect_tx(bars + q, per * BOX_BYTES);
      for (int f = q * per; f < (q + 1) * per; ++f) tma_load_2d(sm + f * FIELD, map + f, z0 - 8, x0 - xoff, bars + q);
    }
}

// Waits for group q of issue_groups (every thread of the CTA calls it); after a
// timeout returns false to all threads, having given the groups from q on a
// bounded time to land.
__device__ __forceinline__ bool wait_group(int *err, unsigned long long *bars, int q, int ng)
{
  const bool ok = mbar_wait(bars + q, 0);
  if (__syncthreads_or(!ok)) {
    if (threadIdx.x == 0) {
      atomicOr(err, 4);
      for (int r = q; r < ng; ++r) mbar_wait(bars + r, 0, 1u << 16);
    }
    return false;
  }
  return true;
}

}  // namespace tma
}  // namespace tiled
}  // namespace ttifd
