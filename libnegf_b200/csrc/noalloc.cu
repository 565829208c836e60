// Batched Sancho-Rubio decimation that allocates no device memory.
//
// negf_b200_decimation_batched needs a caller-provided work buffer, and the
// context API grows its workspace with cudaMalloc.  Some callers cannot do
// either: a code whose device memory is owned by another allocator (a
// framework's caching pool, a Fortran host that hands over only the arrays
// it already owns) must not have a library call cudaMalloc behind its back,
// and a solver loop that must not stall cannot afford cudaMalloc/cudaFree,
// which synchronise the device.  This entry point takes the scratch from a
// fixed array compiled into the library instead.
//
// The array is a file-scope __device__ variable of kScratchBytes (64 MiB).
// Every GPU on which this library's code is loaded holds it until the
// process exits (at the latest from the first call on that GPU).  Its device
// address is resolved on the host with cudaGetSymbolAddress, once per
// device and CUDA context, by the first call made while that device is
// current; make that first call before any stream capture.  A device reset
// (cudaDeviceReset, or a primary context torn down and made again) loads the
// module afresh, so the address is keyed on the current context and
// resolved again when the context changes; a failed launch also drops it.
// All calls share the one array and
// it keeps whatever the previous call left in it: calls whose kernels can
// overlap on the GPU (different streams, different host threads) race on
// it, so serialise them.  The decimation writes every scratch element it
// reads before reading it, so nothing in the array has to start at zero.
#include <cstdio>
#include <mutex>

#include "../../include/negf_b200.h"
#include "engine.cuh"

namespace {

constexpr size_t kScratchBytes = size_t(64) << 20;
constexpr int kMaxDevices = 64;

__device__ __align__(256) unsigned char g_decimation_scratch[kScratchBytes];

std::mutex g_mu;
void* g_scratch_addr[kMaxDevices] = {nullptr};
void* g_scratch_ctx[kMaxDevices] = {nullptr};   // context the address belongs to

// The current CUDA context (CUcontext), through the runtime's driver entry
// point so that the library needs no link against the driver library; null
// if the driver does not provide it (then the address is kept per device).
void* current_context() {
  typedef int (*CtxGetCurrent)(void**);
  static CtxGetCurrent fn = nullptr;
  static bool looked = false;
  if (!looked) {
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<CtxGetCurrent>(p);
    else
      cudaGetLastError();
    looked = true;
  }
  void* ctx = nullptr;
  if (fn && fn(&ctx) != 0) ctx = nullptr;
  return ctx;
}

}  // namespace

extern "C" int negf_b200_decimation_noalloc(int32_t batch, int32_t n, const double* Ao, const double* Bo,
                                            const double* Co, double* Go, int32_t* ncyc, double tol,
                                            int32_t max_iter, void* stream) {
  if (batch < 0 || n < 0 || n > negf::kMaxOrder || tol <= 0.0 || max_iter < 1) return NEGF_B200_ERR_BAD_ARG;
  if (batch == 0 || n == 0) return NEGF_B200_OK;
  if (!Ao || !Bo || !Co || !Go) return NEGF_B200_ERR_BAD_ARG;
  const size_t need = (size_t)batch * negf::decimation_batched_work_elems(n) * 16;
  if (need > kScratchBytes) {
    std::fprintf(stderr,
                 "negf_b200_decimation_noalloc: batch %d of order %d needs %zu bytes of scratch, "
                 "the fixed array holds %zu (at most %zu problems of this order per call)\n",
                 batch, n, need, kScratchBytes,
                 kScratchBytes / (negf::decimation_batched_work_elems(n) * 16));
    return NEGF_B200_ERR_ADMISSION;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) {
    cudaGetLastError();
    return NEGF_B200_ERR_CUDA;
  }
  void* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_mu);
    // (before the first lookup no context may be current yet: the lookup
    // creates it, and the context stored is the one current after it)
    void* ctx = current_context();
    if (!g_scratch_addr[dev] || g_scratch_ctx[dev] != ctx) {
      void* p = nullptr;
      cudaError_t e = cudaGetSymbolAddress(&p, g_decimation_scratch);
      if (e != cudaSuccess || !p) {
        cudaGetLastError();
        g_scratch_addr[dev] = nullptr;
        return NEGF_B200_ERR_CUDA;
      }
      g_scratch_addr[dev] = p;
      g_scratch_ctx[dev] = current_context();
    }
    scratch = g_scratch_addr[dev];
  }
  cudaError_t e = negf::launch_decimation_batched(batch, n, (const double2*)Ao, (const double2*)Bo,
                                                  (const double2*)Co, (double2*)Go, ncyc, tol, max_iter,
                                                  (double2*)scratch, (cudaStream_t)stream);
  if (e != cudaSuccess) {
    std::lock_guard<std::mutex> lk(g_mu);
    g_scratch_addr[dev] = nullptr;   // resolve again on the next call
    return NEGF_B200_ERR_CUDA;
  }
  return NEGF_B200_OK;
}
