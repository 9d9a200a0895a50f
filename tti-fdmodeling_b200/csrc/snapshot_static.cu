// tti_snapshot_static: a wavefield snapshot that allocates no device memory.
//
// The regular snapshot path (tti_run's callback) packs the requested field
// into a device staging buffer that the handle allocates on first use. Some
// callers cannot let device memory grow at the point where they want a
// snapshot: a host application whose GPU memory is budgeted by another
// framework's pool and must not grow, or code that runs while another stream
// of the process is being captured into a CUDA graph (in the default global
// capture mode a device allocation from any thread is refused and invalidates
// that capture). This entry point packs into a fixed array that lives in this
// file's device module instead, and copies straight into the caller's host
// buffer.
//
// Costs and rules of the static array:
//  - 16 Mi floats (64 MiB) per GPU. With CUDA's lazy module loading (the
//    default) the array is committed when this file's device code is first
//    loaded on a device, which is the first tti_snapshot_static call there;
//    from then on it is held until the process exits and no later call grows
//    device memory. A caller under a fixed budget makes one call early, with
//    a small handle if need be, to pay that cost up front;
//  - snapshots larger than that are rejected with TTI_ERR_ARG;
//  - every call on a device shares the one array: calls whose GPU work
//    overlaps (two handles on different streams of the same GPU, or two host
//    threads) race and must be serialised by the caller. The pack kernel
//    writes every element a call copies out, so nothing is carried over from
//    the previous call's contents;
//  - the device address of the array is looked up with cudaGetSymbolAddress
//    by the first call on each device (with that device current); make that
//    first call before any stream capture starts;
//  - the call ends with a copy to pageable host memory and a synchronisation
//    of the handle's stream, neither of which can be captured. It therefore
//    refuses, with TTI_ERR_STATE, a handle whose stream is being captured. While
//    other streams are being captured (in any capture mode) it runs with this
//    thread's capture interaction mode set to relaxed, so that those captures
//    stay valid, and restores the thread's mode before it returns.
#include <mutex>

#include "launch.cuh"

namespace {

constexpr size_t kStaticSnapshotFloats = size_t(16) << 20;  // 64 MiB

static __device__ __align__(256) float g_snapshot_scratch[kStaticSnapshotFloats];

constexpr int kMaxDevices = 64;
std::mutex g_mutex;
float *g_scratch_ptr[kMaxDevices] = {};  // device address of g_snapshot_scratch, per device

// Sets this thread's stream-capture interaction mode to relaxed for the
// lifetime of the object and puts the previous mode back afterwards.
struct RelaxedCaptureMode {
  cudaStreamCaptureMode prev = cudaStreamCaptureModeRelaxed;
  bool ok;
  RelaxedCaptureMode() { ok = cudaThreadExchangeStreamCaptureMode(&prev) == cudaSuccess; }
  ~RelaxedCaptureMode()
  {
    if (ok) cudaThreadExchangeStreamCaptureMode(&prev);
  }
};

int fail(tti_handle *h, int code, const char *what, cudaError_t e)
{
  char msg[256];
  snprintf(msg, sizeof msg, "tti_snapshot_static: %s%s%s", what, e == cudaSuccess ? "" : ": ",
           e == cudaSuccess ? "" : cudaGetErrorString(e));
  return ttifd::handle_error(h, code, msg);
}

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
  RelaxedCaptureMode relaxed;
  if (!relaxed.ok) return fail(h, TTI_ERR_CUDA, "cudaThreadExchangeStreamCaptureMode failed", cudaSuccess);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  cudaError_t e = cudaStreamIsCapturing(h->stream, &cap);
  if (e != cudaSuccess) return fail(h, TTI_ERR_CUDA, "cudaStreamIsCapturing", e);
  if (cap != cudaStreamCaptureStatusNone)
    return fail(h, TTI_ERR_STATE,
                "the handle's stream is being captured; the snapshot copies to pageable host memory and "
                "synchronises that stream, which a capture cannot hold",
                cudaSuccess);
  if ((e = cudaSetDevice(h->device)) != cudaSuccess) return fail(h, TTI_ERR_CUDA, "cudaSetDevice", e);
  float *scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mutex);
    if (!g_scratch_ptr[h->device]) {
      // set-up, once per device with that device current: the host-side name
      // of the array is not a device address
      void *p = nullptr;
      e = cudaGetSymbolAddress(&p, g_snapshot_scratch);
      if (e != cudaSuccess) return fail(h, TTI_ERR_CUDA, "cudaGetSymbolAddress of the static snapshot buffer", e);
      g_scratch_ptr[h->device] = static_cast<float *>(p);
    }
    scratch = g_scratch_ptr[h->device];
  }
  launch_snapshot(handle_step_args(h), kind, h->cfg.savew, scratch, h->stream);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpyAsync(out, scratch, n * sizeof(float), cudaMemcpyDeviceToHost, h->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(h->stream);
  if (e != cudaSuccess) return fail(h, TTI_ERR_CUDA, "pack and copy", e);
  return TTI_OK;
}
