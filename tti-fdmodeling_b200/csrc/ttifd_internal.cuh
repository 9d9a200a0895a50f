// Internal declarations of the B200 TTI RSG library (not part of the C ABI).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdlib.h>

#include <string>

#include "../../include/ttifd.h"

namespace ttifd {

constexpr int NH = 5;  // half length of the 10th-order RSG operator

// Least-squares RSG coefficients C1..C5 (coord:468-469).
__host__ __device__ __forceinline__ constexpr float rsg(int k)
{
  return k == 0   ? 1.24362739770907f
         : k == 1 ? -0.114021164233934f
         : k == 2 ? 0.0272965993810630f
         : k == 3 ? -0.00699199493927320f
                  : 0.00132022981661381f;
}

// Programmatic dependent launch. A kernel launched with launch_pdl may be
// scheduled while the kernel before it in the stream is still draining; it
// calls pdl_sync() before touching any memory, which signals that its own
// dependents may be scheduled and then waits until the previous kernel has
// completed and its writes are visible. Without the launch attribute both
// instructions do nothing. TTIFD_PDL=0 launches normally.
__device__ __forceinline__ void pdl_sync()
{
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
}

inline bool pdl_enabled()
{
  static const bool on = [] {
    const char *e = getenv("TTIFD_PDL");
    return !(e && e[0] == '0');
  }();
  return on;
}

template <typename... KArgs, typename... Args>
cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, Args... args)
{
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

// Device grid description. Arrays are column-major in x: element (ix, iz) at
// ix * ldz + iz, ldz = Nz rounded up to 32 floats so every column starts on a
// 128-byte boundary. Cells iz in [Nz, ldz) are padding and stay zero.
struct Grid {
  int Nz, Nx, ldz, E, izStart;
  size_t n;  // ldz * Nx
};

// Arithmetic policy. Exact<true> rounds every product and sum separately in
// the reference's expression order (no FMA contraction), which reproduces a
// gcc -ffp-contract=off build of the reference bit for bit. Exact<false> lets
// the compiler contract a*b+c into FMA (one rounding instead of two).
template <bool X>
struct Ar;
template <>
struct Ar<true> {
  static __device__ __forceinline__ float mul(float a, float b) { return __fmul_rn(a, b); }
  static __device__ __forceinline__ float add(float a, float b) { return __fadd_rn(a, b); }
  static __device__ __forceinline__ float sub(float a, float b) { return __fsub_rn(a, b); }
};
template <>
struct Ar<false> {
  static __device__ __forceinline__ float mul(float a, float b) { return a * b; }
  static __device__ __forceinline__ float add(float a, float b) { return a + b; }
  static __device__ __forceinline__ float sub(float a, float b) { return a - b; }
};

struct Fields {
  float *vx, *vz, *sxx, *szz, *sxz, *txx, *tzz, *txz;
};

struct Params {
  const float *coef1, *coef2, *invrho;
  const float *c11, *c13, *c15, *c33, *c35, *c55;
  const float *sn, *cs, *snv, *csv;   // coordinate: sin/cos theta (stress / velocity node)
  const float *s2, *c2, *s2t;         // tensor: sin^2, cos^2, sin 2theta
};

struct SourceSet {
  int n;
  const int *x, *z;  // padded-grid cell of each source
  const float *w;    // [n][nt]
  int nt;
};

// Bulk device arrays of a handle from the library's per-device pool
// (devmem.cu), ordered on stream st; the caller synchronises st before other
// streams use the memory.
cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t st);
void pool_free(void *p, cudaStream_t st);

// Host-memory helpers (hostmem.cu): fault in every page of a host range from
// several threads before a pageable device-to-host copy; the maximum of n
// floats (NaN entries ignored, as fmaxf does) from several threads.
void prefault(void *p, size_t bytes);
// true for page-locked host memory known to CUDA (cudaHostAlloc, cudaHostRegister)
bool is_pinned(const void *p);
float host_max(const float *a, size_t n, float init);
// memcpy from up to max_threads host threads (1 MiB or more each). Into fresh
// pageable memory 16 threads help (they take the page faults in parallel);
// from resident memory into page-locked chunks 8 measured faster than 16.
void parallel_copy(void *dst, const void *src, size_t bytes, int max_threads = 16);
// Page-locked staging chunks of PIN_CHUNK floats from a process-wide free list
// (allocated on first need, kept until exit); null when none can be had.
constexpr size_t PIN_CHUNK = (size_t)4 << 20;
float *pinned_chunk();
void pinned_release(float *p);

struct ReceiverSet {
  int n[3];
  const int *x[3], *z[3];  // padded-grid cells
  float *rec[3];           // time-major on the device: [nts][n]
};

}  // namespace ttifd

// Host-side handle (C ABI object).
struct tti_handle {
  tti_config cfg;
  int device = 0;
  cudaStream_t stream = nullptr;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  ttifd::Grid g{};
  float *fld[8] = {};      // wavefields, updated in place
  bool use_tiled = false;  // tiled half-step kernels with TMA halo tiles (in place)
  const tti_handle *owner = nullptr;  // set when the parameter arrays belong to another handle (batched shots)
  float *m_eps = nullptr, *m_delta = nullptr;  // epsilon, delta as uploaded (gradient chain rule)
  float *m_theta = nullptr;                    // theta (degrees) as uploaded (Bond gradient chain rule)
  struct GradState *grad = nullptr;            // adjoint-state gradient buffers (adjoint.cu)
  void *tmaps = nullptr;   // host copy of the 5 tensor maps (vx vz sxx szz sxz), 64-byte aligned
  int undamped_ok = 0;  // coef1 == 1, coef2 == dt outside the absorbing rims (checked at upload)
  int *d_rcol[3] = {}, *d_rzs[3] = {}, *d_rid[3] = {};  // receivers grouped by column
  float2 *pk_cf = nullptr, *pk_vsc = nullptr, *pk_sc = nullptr;  // packed parameters (pack.cuh)
  float4 *pk_c4 = nullptr;
  float *par[TTI_P_COUNT] = {};
  float invdx = 0, invdz = 0, alpha_src = 0;
  // geometry
  int nsrc = 0;
  int *d_sx = nullptr, *d_sz = nullptr;
  float *d_src = nullptr;
  int nrec[3] = {0, 0, 0};
  int *d_rz[3] = {};  // receiver rows in the caller's order; owns the block d_rzs, d_rid, d_rcol point into
  float *d_rec[3] = {};
  int nts = 0;
  double *d_energy = nullptr;  // [nt][2]
  int *d_flag = nullptr;       // nonfinite watchdog
  float *d_snap = nullptr;      // packed snapshot kinds of one step, snap_cap floats
  float *h_snap = nullptr;      // snapshot handed to the callback (pageable, faulted in once), h_snap_cap floats
  float *d_stage = nullptr;     // trace fetch: device chunk of transposed traces
  size_t snap_cap = 0, h_snap_cap = 0;
  // caller's snapshot buffer (tti_set_snapshot_buffer); when page-locked the
  // copy runs on copy_stream and the callbacks of snapshot step snap_it follow
  // at the next snapshot step or at the end of tti_run
  float *snap_user = nullptr;
  bool snap_user_pinned = false;
  cudaStream_t copy_stream = nullptr;
  cudaEvent_t snap_packed = nullptr, snap_done = nullptr;
  bool snap_pending = false;
  int snap_it = 0;
  tti_snapshot_fn snap_fn = nullptr;
  void *snap_arg = nullptr;
  bool have_model = false;
  int step_index = 0;
  float last_ms = 0.0f;
  long long launches = 0;
  cudaEvent_t pev[8] = {};  // phase events for tti_profile_steps
  bool exact = false;
  unsigned wait_limit = 0;  // polls of the tiled kernels' first TMA wait
  std::string err;
};
