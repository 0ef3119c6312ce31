// Opt-in per-kernel-family timing with CUDA events recorded on the stream each
// kernel is launched on.  Used by bench.py to time the dominant kernel inside
// the timed region; off by default (no events recorded).
#include <mutex>
#include <vector>

#include "mb_common.cuh"

namespace {
struct Pending {
  int id;
  cudaEvent_t a, b;
};
std::mutex g_mu;
bool g_on = false;
std::vector<Pending> g_pending;
cudaEvent_t g_open[MB_KSTAT_IDS] = {nullptr};
}  // namespace

void mb_kstat_mark(int id, cudaStream_t s, bool begin) {
  if (!g_on || id < 0 || id >= MB_KSTAT_IDS) return;
  std::lock_guard<std::mutex> lk(g_mu);
  cudaEvent_t e;
  if (cudaEventCreate(&e) != cudaSuccess) return;
  cudaEventRecord(e, s);
  if (begin) {
    if (g_open[id]) cudaEventDestroy(g_open[id]);
    g_open[id] = e;
  } else if (g_open[id]) {
    g_pending.push_back({id, g_open[id], e});
    g_open[id] = nullptr;
  } else {
    cudaEventDestroy(e);
  }
}

extern "C" void mb_kstats_enable(int on) {
  std::lock_guard<std::mutex> lk(g_mu);
  g_on = on != 0;
}

extern "C" int mb_kstats_read(int id, long long* count, double* total_ms) {
  std::lock_guard<std::mutex> lk(g_mu);
  long long c = 0;
  double t = 0.0;
  std::vector<Pending> keep;
  for (auto& p : g_pending) {
    if (p.id != id) {
      keep.push_back(p);
      continue;
    }
    float ms = 0.f;
    if (cudaEventSynchronize(p.b) == cudaSuccess && cudaEventElapsedTime(&ms, p.a, p.b) == cudaSuccess) {
      t += ms;
      ++c;
    }
    cudaEventDestroy(p.a);
    cudaEventDestroy(p.b);
  }
  g_pending.swap(keep);
  if (count) *count = c;
  if (total_ms) *total_ms = t;
  return MB_OK;
}

cudaError_t mb_malloc_async(void** p, size_t bytes, cudaStream_t s) {
  static std::mutex mu;
  static bool kept[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64) {
    std::lock_guard<std::mutex> lk(mu);
    if (!kept[dev]) {
      cudaMemPool_t pool;
      if (cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
        unsigned long long thr = ~0ull;
        cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
      }
      kept[dev] = true;
    }
  }
  return cudaMallocAsync(p, bytes, s);
}
