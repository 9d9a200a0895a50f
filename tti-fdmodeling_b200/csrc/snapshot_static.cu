// tti_snapshot_static: a wavefield snapshot that allocates no device memory.
//
// The regular snapshot path (tti_run's callback) packs the requested field
// into a device staging buffer that the handle allocates on first use and
// copies it to pinned host memory it also allocates. Some callers cannot
// allocate at the point where they want a snapshot: code running while a
// stream is being captured (device allocation is not a capturable stream
// operation and is refused in global capture mode), or a host application
// whose GPU memory is budgeted by another framework's pool and must not grow.
// This entry point packs into a fixed array that lives in this file's device
// module instead, and copies straight into the caller's host buffer.
//
// Costs and rules of the static array:
//  - 16 Mi floats (64 MiB) per GPU, reserved when this module is first loaded
//    on a device and held until the process exits, whether or not the entry
//    point is ever called on that device again;
//  - snapshots larger than that are rejected with TTI_ERR_ARG;
//  - every call on a device shares the one array: calls whose GPU work
//    overlaps (two handles on different streams of the same GPU, or two host
//    threads) race and must be serialised by the caller. The pack kernel
//    writes every element a call copies out, so nothing is carried over from
//    the previous call's contents;
//  - the device address of the array is looked up with cudaGetSymbolAddress
//    by the first call on each device (with that device current); make that
//    first call before any stream capture starts.
#include <mutex>

#include "launch.cuh"

namespace {

constexpr size_t kStaticSnapshotFloats = size_t(16) << 20;  // 64 MiB

static __device__ __align__(256) float g_snapshot_scratch[kStaticSnapshotFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
float *g_scratch_ptr[kMaxDevices] = {};  // device address of g_snapshot_scratch, per device

}  // namespace

extern "C" int tti_snapshot_static(tti_handle *h, int kind, float *out)
{
  using namespace ttifd;
  if (!h || !out) return TTI_ERR_ARG;
  if (kind < 1 || kind > 7) return handle_error(h, TTI_ERR_ARG, "snapshot kind must be 1..7");
  const Grid &g = h->g;
  const bool whole = h->cfg.savew != 0;
  const size_t nzo = whole ? g.Nz : g.Nz - 2 * g.E, nxo = whole ? g.Nx : g.Nx - 2 * g.E;
  const size_t n = nzo * nxo;
  if (n > kStaticSnapshotFloats) {
    char msg[256];
    snprintf(msg, sizeof msg,
             "snapshot of %zu floats exceeds the %zu-float static buffer of tti_snapshot_static; use the snapshot "
             "callback of tti_run instead",
             n, kStaticSnapshotFloats);
    return handle_error(h, TTI_ERR_ARG, msg);
  }
  if (h->device < 0 || h->device >= kMaxDevices) return handle_error(h, TTI_ERR_ARG, "device index too large");
  if (cudaSetDevice(h->device) != cudaSuccess) return handle_error(h, TTI_ERR_CUDA, "cudaSetDevice failed");
  float *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[h->device]) {
      // set-up, once per device with that device current: the host-side name
      // of the array is not a device address
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_snapshot_scratch);
      if (e != cudaSuccess) {
        char msg[256];
        snprintf(msg, sizeof msg, "cudaGetSymbolAddress of the static snapshot buffer failed: %s",
                 cudaGetErrorString(e));
        return handle_error(h, TTI_ERR_CUDA, msg);
      }
      g_scratch_ptr[h->device] = static_cast<float *>(p);
    }
    scratch = g_scratch_ptr[h->device];
  }
  launch_snapshot(handle_step_args(h), kind, h->cfg.savew, scratch, h->stream);
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) {
    char msg[256];
    snprintf(msg, sizeof msg, "tti_snapshot_static: %s", cudaGetErrorString(e));
    return handle_error(h, TTI_ERR_CUDA, msg);
  }
  return TTI_OK;
}
