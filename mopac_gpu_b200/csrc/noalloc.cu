// Allocation-free variant of the electronic-energy reduction (helect).
//
// mb_helect_dev obtains its 2*n-double workspace from the stream-ordered
// allocator on every call.  Some callers cannot allocate device memory at the
// point where they need the energy: a Fortran or C host whose device memory is
// all handed out up front by its own arena, code running while a CUDA stream
// is being captured into a graph (an allocation there either breaks the
// capture or becomes part of the graph), or a loop with a hard latency budget
// that must not touch the allocator.  mb_helect_noalloc serves them: its
// scratch is a fixed array in the library's own device memory.
//
// Limits and sharing rules:
//   * n <= MB_HELECT_NOALLOC_MAX_N (16384 orbitals); the array is
//     2 * 16384 doubles = 256 KiB and every GPU that loads the library keeps
//     it for the life of the process.  Larger n is rejected with MB_ERR_ARG.
//   * All calls share the one array and it keeps the previous call's values.
//     Nothing in it has to start at zero: every slot the reduction reads is
//     written earlier in the same call.  Two calls whose kernels overlap on the
//     GPU (different streams, or different host threads) race on the array and
//     give wrong energies; serialise them.
//   * The first call on each device looks up the array's device address
//     (cudaGetSymbolAddress) with that device current and caches it; make that
//     first call outside any stream capture.  The cache is never refreshed:
//     after a cudaDeviceReset (which destroys the primary context and the
//     array with it) the cached address is stale, so a caller that resets
//     the device must not use this entry point again in the same process.
#include <mutex>

#include "mb_common.cuh"

#define MB_HELECT_NOALLOC_MAX_N 16384

extern "C" int mb_helect_ws(int n, const double* p, const double* h, const double* f, double* out, double* ws,
                            cudaStream_t stream);

// File-scope scratch: the row sums occupy the first n doubles and the
// diagonal terms the next n.
static __device__ __align__(256) double g_helect_scratch[2 * MB_HELECT_NOALLOC_MAX_N];

namespace {

constexpr int kMaxDevices = 64;
std::mutex g_addr_mu;
double* g_addr[kMaxDevices] = {nullptr};

// Device address of g_helect_scratch on the current device.  In host code the
// symbol's own name is only a host-side handle, never a device pointer.
int scratch_address(double** out) {
  int dev = 0;
  MB_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) return mb_set_error(MB_ERR_ARG, "mb_helect_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_addr_mu);
  if (!g_addr[dev]) {
    void* ptr = nullptr;
    cudaError_t e = cudaGetSymbolAddress(&ptr, g_helect_scratch);
    if (e != cudaSuccess) return mb_set_cuda_error(e, "cudaGetSymbolAddress(g_helect_scratch)", __FILE__, __LINE__);
    g_addr[dev] = static_cast<double*>(ptr);
  }
  *out = g_addr[dev];
  return MB_OK;
}

}  // namespace

extern "C" int mb_helect_noalloc(int n, const double* p, const double* h, const double* f, double* out,
                                 cudaStream_t stream) {
  if (n <= 0) return mb_set_error(MB_ERR_ARG, "mb_helect_noalloc: n <= 0");
  if (n > MB_HELECT_NOALLOC_MAX_N)
    return mb_set_error(MB_ERR_ARG, "mb_helect_noalloc: n exceeds the 16384-orbital scratch; use mb_helect_dev");
  double* ws = nullptr;
  MB_TRY(scratch_address(&ws));
  // same two kernels as mb_helect_dev; rows go to ws[0, n), diagonal terms to
  // ws[n, 2n) -- both fully written before they are read
  return mb_helect_ws(n, p, h, f, out, ws, stream);
}
