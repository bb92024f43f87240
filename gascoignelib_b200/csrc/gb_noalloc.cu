#include "gb_context.cuh"

extern "C" {

// ------------------------------------------------- allocation-free dot product
//
// Scratch of gb_dot_noalloc: one FP64 partial per block plus the last-block
// ticket, in file-scope device arrays. Host code may not pass these names to a
// kernel (on the host they are stand-ins, not device addresses); their device
// addresses are looked up once per device with cudaGetSymbolAddress.

namespace gb {
constexpr int kNoAllocBlocks = 4096;
constexpr int64_t kNoAllocMaxN = int64_t(kNoAllocBlocks) * kRedThreads * 8;
static __device__ __align__(256) double g_noalloc_partials[kNoAllocBlocks];
static __device__ __align__(256) unsigned g_noalloc_ticket[64];
struct NoAllocAddr
{
  double* partials = nullptr;
  unsigned* ticket = nullptr;
};
constexpr int kNoAllocMaxDevices = 64;
static NoAllocAddr g_noalloc_addr[kNoAllocMaxDevices];
static std::mutex g_noalloc_mutex;
} // namespace gb

int
gb_dot_noalloc(const double* a, const double* b, int64_t n, double* out, void* stream)
{
  using namespace gb;
  if (!a || !b || !out || n < 0) {
    fprintf(stderr, "gb_dot_noalloc: null pointer or negative length\n");
    return GB_EINVAL;
  }
  if (n > kNoAllocMaxN) {
    fprintf(stderr,
            "gb_dot_noalloc: n = %lld exceeds the maximum %lld (scratch of %d "
            "partial sums); use gb_vec_dot\n",
            (long long)n, (long long)kNoAllocMaxN, kNoAllocBlocks);
    return GB_EINVAL;
  }
  // an error the caller's own earlier work left pending is reported, not
  // consumed: cudaGetLastError after our launch would otherwise clear it
  if (cudaPeekAtLastError() != cudaSuccess) {
    fprintf(stderr, "gb_dot_noalloc: a CUDA error is already pending\n");
    return GB_ECUDA;
  }
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kNoAllocMaxDevices)
    return GB_ECUDA;
  // the address is looked up once per device ordinal and kept for the life of
  // the process (it does not survive cudaDeviceReset of that device)
  NoAllocAddr addr;
  {
    std::lock_guard<std::mutex> lk(g_noalloc_mutex);
    if (!g_noalloc_addr[dev].partials) {
      void* pp = nullptr;
      void* tp = nullptr;
      if (cudaGetSymbolAddress(&pp, g_noalloc_partials) != cudaSuccess ||
          cudaGetSymbolAddress(&tp, g_noalloc_ticket) != cudaSuccess || !pp || !tp) {
        fprintf(stderr, "gb_dot_noalloc: cudaGetSymbolAddress failed\n");
        return GB_ECUDA;
      }
      g_noalloc_addr[dev].partials = static_cast<double*>(pp);
      g_noalloc_addr[dev].ticket = static_cast<unsigned*>(tp);
    }
    addr = g_noalloc_addr[dev];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  // the ticket must start at 0 (an earlier failed call may have left it set)
  if (cudaMemsetAsync(addr.ticket, 0, sizeof(unsigned), st) != cudaSuccess)
    return GB_ECUDA;
  const int grid = static_cast<int>(
    std::max<int64_t>(1, (n + int64_t(kRedThreads) * 8 - 1) / (int64_t(kRedThreads) * 8)));
  k_dot<double, double><<<grid, kRedThreads, 0, st>>>(
    n, a, b, addr.partials, addr.ticket, RedOut{ out, nullptr, nullptr, 0 });
  if (cudaGetLastError() != cudaSuccess)
    return GB_ECUDA;
  return GB_OK;
}

} // extern "C"
