// Host-side helpers of the transfer paths (no device code).
//
// A device-to-host copy into pageable memory that was never touched stops on a
// page fault per 4 KiB page: on B200 hosts 2.2 GB/s for a fresh 95 MB buffer,
// and pinned staging with a single-threaded copy fares no better. Faulting the
// pages in from several threads first (16 threads: 2.6 ms for 95 MB, 1.7 ms
// with the huge-page hint), then copying straight from the device (about
// 9 GB/s), avoids both the faults on the copy path and the cost of pinning
// (13 ms to allocate and 4.7 ms to free 32 MB of page-locked memory) on
// every handle. Where page-locked chunks can be had once per process, staging
// a trace fetch through two of them with a multi-threaded host copy into the
// caller's fresh block is faster still (15.5 GB/s): pinned_chunk hands out
// 16 MB chunks from a process-wide free list and they stay allocated until
// exit.
#include <float.h>
#include <stdint.h>
#include <sys/mman.h>

#include <algorithm>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "ttifd_internal.cuh"

namespace ttifd {
namespace {

int workers(size_t bytes)
{
  const size_t hw = std::max(1u, std::thread::hardware_concurrency());
  const size_t by_size = std::max<size_t>(1, bytes >> 22);  // at least 4 MiB each
  return (int)std::min<size_t>(std::min<size_t>(16, hw), by_size);
}

// f(begin, end) over [0, n) cut into nth contiguous ranges; the caller's
// thread takes the last range
template <class F>
void split(size_t n, int nth, F f)
{
  std::vector<std::thread> th;
  const size_t per = (n + nth - 1) / nth;
  for (int t = 0; t < nth - 1; ++t) {
    const size_t b = t * per, e = std::min(n, b + per);
    if (b < e) th.emplace_back(f, b, e);
  }
  const size_t b = (size_t)(nth - 1) * per;
  if (b < n) f(b, n);
  for (auto &x : th) x.join();
}

std::mutex g_pin_mu;
std::vector<float *> g_pin_free;  // page-locked staging chunks not in use

// Persistent copy workers for parallel_copy: a staged transfer calls it once
// per 16 MB chunk, and starting fresh threads for every chunk (18 chunks x 8
// threads for a 1126 x 7872 model) cost several milliseconds of the upload.
// One job at a time (callers queue on job_mu); the caller takes a share too.
class CopyPool {
 public:
  static CopyPool &get()
  {
    static CopyPool *p = new CopyPool();  // never destroyed: workers may outlive static destructors
    return *p;
  }
  // f(i) for i in [0, n), on up to n threads (the caller's included)
  void run(int n, const std::function<void(int)> &f)
  {
    std::lock_guard<std::mutex> job(job_mu_);
    {
      std::lock_guard<std::mutex> lock(mu_);
      f_ = &f;
      n_ = n;
      next_ = 1;  // item 0 is the caller's
      left_ = n - 1;
      ++gen_;
    }
    cv_.notify_all();
    f(0);
    std::unique_lock<std::mutex> lock(mu_);
    for (;;) {  // the caller helps with items no worker has taken yet
      if (next_ < n_) {
        const int i = next_++;
        lock.unlock();
        f(i);
        lock.lock();
        --left_;
        continue;
      }
      if (left_ == 0) break;
      done_.wait(lock);
    }
    f_ = nullptr;
  }
  int size() const { return (int)th_.size() + 1; }

 private:
  CopyPool()
  {
    const int hw = (int)std::max(1u, std::thread::hardware_concurrency());
    for (int t = 0; t < std::min(15, hw - 1); ++t) th_.emplace_back([this] { loop(); });
    for (auto &x : th_) x.detach();
  }
  void loop()
  {
    unsigned long long seen = 0;
    std::unique_lock<std::mutex> lock(mu_);
    for (;;) {
      cv_.wait(lock, [&] { return gen_ != seen && f_ && next_ < n_; });
      seen = gen_;
      while (f_ && next_ < n_) {
        const int i = next_++;
        const std::function<void(int)> *f = f_;
        lock.unlock();
        (*f)(i);
        lock.lock();
        if (--left_ == 0) done_.notify_all();
      }
    }
  }
  std::mutex job_mu_, mu_;
  std::condition_variable cv_, done_;
  const std::function<void(int)> *f_ = nullptr;
  int n_ = 0, next_ = 0, left_ = 0;
  unsigned long long gen_ = 0;
  std::vector<std::thread> th_;
};

}  // namespace

void parallel_copy(void *dst, const void *src, size_t bytes, int max_threads)
{
  CopyPool &pool = CopyPool::get();
  const int nth = (int)std::min<size_t>(std::min<size_t>((size_t)std::max(1, max_threads), (size_t)pool.size()),
                                        std::max<size_t>(1, bytes >> 20));
  char *d = static_cast<char *>(dst);
  const char *q = static_cast<const char *>(src);
  if (nth <= 1) {
    memcpy(d, q, bytes);
    return;
  }
  const size_t per = (bytes + nth - 1) / nth;
  pool.run(nth, [&](int i) {
    const size_t b = (size_t)i * per, e = std::min(bytes, b + per);
    if (b < e) memcpy(d + b, q + b, e - b);
  });
}

float *pinned_chunk()
{
  {
    std::lock_guard<std::mutex> lock(g_pin_mu);
    if (!g_pin_free.empty()) {
      float *p = g_pin_free.back();
      g_pin_free.pop_back();
      return p;
    }
  }
  // portable: a chunk serves handles on any device of the process
  float *p = nullptr;
  if (cudaHostAlloc(reinterpret_cast<void **>(&p), PIN_CHUNK * sizeof(float), cudaHostAllocPortable) != cudaSuccess)
    return nullptr;
  return p;
}

void pinned_release(float *p)
{
  if (!p) return;
  std::lock_guard<std::mutex> lock(g_pin_mu);
  g_pin_free.push_back(p);
}

bool is_pinned(const void *p)
{
  cudaPointerAttributes at;
  if (!p || cudaPointerGetAttributes(&at, p) != cudaSuccess) {
    cudaGetLastError();  // a failed query leaves nothing behind
    return false;
  }
  return at.type == cudaMemoryTypeHost;
}

void prefault(void *p, size_t bytes)
{
  if (!p || bytes == 0) return;
  // 2 MiB pages where the kernel grants them (transparent huge pages in
  // madvise mode): 512 times fewer faults over the aligned middle of the range
  constexpr uintptr_t HP = (uintptr_t)2 << 20;
  const uintptr_t h0 = ((uintptr_t)p + HP - 1) & ~(HP - 1), h1 = ((uintptr_t)p + bytes) & ~(HP - 1);
  if (bytes >= 4 * HP && h1 > h0) madvise(reinterpret_cast<void *>(h0), h1 - h0, MADV_HUGEPAGE);
  volatile char *c = static_cast<volatile char *>(p);
  const size_t pages = (bytes + 4095) / 4096;
  split(pages, workers(bytes), [c, bytes](size_t b, size_t e) {
    for (size_t q = b; q < e; ++q) c[std::min(q * 4096, bytes - 1)] = 0;
  });
}

float host_max(const float *a, size_t n, float init)
{
  if (n == 0) return init;
  const int nth = workers(n * sizeof(float));
  std::vector<float> part(nth, init);
  const size_t per = (n + nth - 1) / nth;
  split(n, nth, [&](size_t b, size_t e) {
    // eight running maxima; (v > m ? v : m) keeps m for a NaN v, as fmaxf does
    float m[8];
    for (float &x : m) x = init;
    size_t i = b;
    for (; i + 8 <= e; i += 8)
      for (int k = 0; k < 8; ++k) m[k] = a[i + k] > m[k] ? a[i + k] : m[k];
    for (; i < e; ++i) m[0] = a[i] > m[0] ? a[i] : m[0];
    float r = init;
    for (float x : m) r = fmaxf(r, x);
    part[b / per] = r;
  });
  float r = init;
  for (float x : part) r = fmaxf(r, x);
  return r;
}

}  // namespace ttifd

extern "C" {

int tti_host_alloc(size_t bytes, void **ptr)
{
  if (!ptr) return TTI_ERR_ARG;
  *ptr = nullptr;
  if (bytes == 0) return TTI_ERR_ARG;
  // portable: the buffer serves handles on any device of the process
  if (cudaHostAlloc(ptr, bytes, cudaHostAllocPortable) != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    return TTI_ERR_NOMEM;
  }
  return TTI_OK;
}

int tti_host_free(void *ptr)
{
  if (!ptr) return TTI_OK;
  if (!ttifd::is_pinned(ptr)) return TTI_ERR_ARG;
  if (cudaFreeHost(ptr) != cudaSuccess) {
    cudaGetLastError();
    return TTI_ERR_CUDA;
  }
  return TTI_OK;
}

}  // extern "C"
