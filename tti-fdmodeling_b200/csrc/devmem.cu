// Device memory of the handles' bulk arrays (wavefields, parameters, packed
// parameters, the raw model during the upload): a library-private
// stream-ordered pool per device that keeps up to POOL_KEEP bytes of freed
// blocks. A process that creates handle after handle of the same grid (one
// per shot) then maps device memory once: mapping 1.4 GB of fresh memory for a
// 1126 x 7872 handle took between 9 and 74 ms on B200 hosts, a reused block
// none. Blocks beyond POOL_KEEP go back to the driver at the next
// synchronisation. Allocation and release are ordered on the handle's stream,
// and every entry point that allocates synchronises that stream before it
// returns, so other streams only ever see completed allocations.
#include <mutex>

#include "ttifd_internal.cuh"

namespace ttifd {
namespace {

constexpr unsigned long long POOL_KEEP = 8ull << 30;
constexpr int MAX_DEVICES = 64;

std::mutex g_pool_mu;
cudaMemPool_t g_pool[MAX_DEVICES] = {};

cudaError_t pool_of(cudaMemPool_t *out)
{
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_pool_mu);
  if (!g_pool[dev]) {
    cudaMemPoolProps props = {};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool = nullptr;
    if ((e = cudaMemPoolCreate(&pool, &props)) != cudaSuccess) return e;
    unsigned long long keep = POOL_KEEP;
    if ((e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep)) != cudaSuccess) {
      cudaMemPoolDestroy(pool);
      return e;
    }
    g_pool[dev] = pool;
  }
  *out = g_pool[dev];
  return cudaSuccess;
}

}  // namespace

cudaError_t pool_alloc(void **p, size_t bytes, cudaStream_t st)
{
  *p = nullptr;
  cudaMemPool_t pool = nullptr;
  cudaError_t e = pool_of(&pool);
  if (e != cudaSuccess) return e;
  e = cudaMallocFromPoolAsync(p, bytes, pool, st);
  // a refused request is reported here; it must not linger as the runtime's
  // last error, where a later launch check would find it
  if (e != cudaSuccess) cudaGetLastError();
  return e;
}

void pool_free(void *p, cudaStream_t st)
{
  if (p) cudaFreeAsync(p, st);
}

}  // namespace ttifd
