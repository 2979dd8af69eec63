// noalloc.cu — overlap_with_zero over caller-owned device buffers, with no allocation.
//
// Some callers cannot let a library call cudaMalloc.  Examples: a host framework that owns
// all device memory through its own pool (a caching allocator hands out every byte, and a
// foreign cudaMalloc can fail or fragment it), or a latency-critical loop where
// cudaMalloc/cudaFree would stall because those calls can synchronise the device.  For them,
// ppvm_overlap_with_zero_noalloc computes the same quantity as ppvm_overlap_with_zero on
// terms the caller already holds in device memory.  Its only working memory is the
// fixed-size array below, compiled into the library: every GPU that loads the library keeps
// that array until the process exits.
//
// The array is shared by every call on a device and keeps the last call's partial sums.
// Each call overwrites every slot it later reads, so nothing has to start at zero.  Calls
// whose kernels overlap on the GPU (for example, issued on two different streams without
// ordering between them) race on the array and can return wrong sums: order them.

#include <cuda_runtime.h>

#include <cstdint>
#include <string>

#include "../../include/ppvm_cuda.h"

namespace {

constexpr int kNaBlock = 256;                    // threads per block
constexpr int kNaItems = 16;                     // terms per thread
constexpr int kNaChunk = kNaBlock * kNaItems;    // terms per block (4096)
constexpr int kNaMaxBlocks = 4096;               // partial-sum slots in the static array
constexpr unsigned long long kNaMaxTerms = (unsigned long long)kNaChunk * kNaMaxBlocks;  // 16,777,216
constexpr int kNaMaxWords = 8;                   // 512 qubits

// The fixed working memory: one partial sum per block (32 KiB per device).
static __device__ __align__(256) double g_na_partials[kNaMaxBlocks];

}  // namespace

namespace ppvm {
void set_last_error(const std::string& msg);  // engine.cu: text of ppvm_last_error_string()
}

namespace {

ppvm_status na_fail(ppvm_status s, const std::string& msg) {
  ppvm::set_last_error(msg);
  return s;
}

// Block b sums the coefficients of terms [b*4096, (b+1)*4096) whose X plane is zero, in a
// fixed order (thread t owns terms t, t+256, ...; then a fixed tree), into partials[b].
__global__ void __launch_bounds__(kNaBlock)
k_owz_noalloc_partials(const uint64_t* __restrict__ x, unsigned long long stride, int nwords,
                       const double* __restrict__ c, unsigned long long n, double* partials) {
  __shared__ double s_red[kNaBlock / 32];
  const unsigned long long base = (unsigned long long)blockIdx.x * kNaChunk;
  double acc = 0.0;
#pragma unroll 4
  for (int k = 0; k < kNaItems; ++k) {
    const unsigned long long i = base + (unsigned long long)k * kNaBlock + threadIdx.x;
    if (i < n) {
      uint64_t any = 0;
      for (int w = 0; w < nwords; ++w) any |= x[(unsigned long long)w * stride + i];
      if (any == 0) acc = __dadd_rn(acc, c[i]);
    }
  }
#pragma unroll
  for (int o = 16; o; o >>= 1) acc = __dadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double b = 0.0;
    for (int w = 0; w < kNaBlock / 32; ++w) b = __dadd_rn(b, s_red[w]);
    partials[blockIdx.x] = b;
  }
}

// One block adds partials[0..nb) in a fixed order and writes the result.
__global__ void __launch_bounds__(kNaBlock)
k_owz_noalloc_final(const double* partials, int nb, double* out) {
  __shared__ double s_red[kNaBlock / 32];
  double acc = 0.0;
  for (int i = threadIdx.x; i < nb; i += kNaBlock) acc = __dadd_rn(acc, partials[i]);
#pragma unroll
  for (int o = 16; o; o >>= 1) acc = __dadd_rn(acc, __shfl_down_sync(0xffffffffu, acc, o));
  if ((threadIdx.x & 31) == 0) s_red[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x == 0) {
    double r = 0.0;
    for (int w = 0; w < kNaBlock / 32; ++w) r = __dadd_rn(r, s_red[w]);
    *out = r;
  }
}

// Device address of the static array on the current device.  Host code cannot use the
// array's name as a device pointer (it names a host-side stand-in), so the address comes from
// the runtime.  It is looked up on every call, not cached: the lookup allocates nothing, and
// an address kept from before a cudaDeviceReset (or from an earlier primary context) would
// point at freed memory.
ppvm_status na_scratch(double** out) {
  void* p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_na_partials);
  if (e != cudaSuccess)
    return na_fail(PPVM_ECUDA, std::string("cudaGetSymbolAddress failed: ") + cudaGetErrorString(e));
  *out = static_cast<double*>(p);
  return PPVM_OK;
}

}  // namespace

extern "C" {

ppvm_status ppvm_overlap_with_zero_noalloc(const uint64_t* d_x, size_t x_stride, uint32_t n_words,
                                           const double* d_c, size_t n_terms, double* d_out,
                                           void* cuda_stream) {
  if (!d_out) return na_fail(PPVM_EINVAL, "null output pointer");
  if (n_words == 0 || n_words > (uint32_t)kNaMaxWords)
    return na_fail(PPVM_EINVAL, "n_words must be in [1, 8]");
  if (n_terms > kNaMaxTerms)
    return na_fail(PPVM_EINVAL, "n_terms exceeds the no-allocation limit of 16777216 terms "
                                "(4096 blocks of 4096 terms in the library's fixed working array)");
  if (n_terms && (!d_x || !d_c)) return na_fail(PPVM_EINVAL, "null input pointer");
  if (n_terms && x_stride < n_terms) return na_fail(PPVM_EINVAL, "x_stride must be >= n_terms");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return na_fail(PPVM_ENODEV, std::string("no CUDA device: ") + cudaGetErrorString(e));
  double* partials = nullptr;
  const ppvm_status st = na_scratch(&partials);
  if (st != PPVM_OK) return st;
  cudaStream_t stream = static_cast<cudaStream_t>(cuda_stream);
  const int nb = (int)((n_terms + kNaChunk - 1) / kNaChunk);
  if (nb > 0)
    k_owz_noalloc_partials<<<nb, kNaBlock, 0, stream>>>(d_x, (unsigned long long)x_stride, (int)n_words, d_c,
                                                        (unsigned long long)n_terms, partials);
  k_owz_noalloc_final<<<1, kNaBlock, 0, stream>>>(partials, nb, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return na_fail(PPVM_ECUDA, std::string("kernel launch failed: ") + cudaGetErrorString(e));
  return PPVM_OK;
}

}  // extern "C"
