// Projections out[k] = A[k] . x without any device allocation.
//
// Some callers of this library cannot allocate device memory at the moment
// they need projections: a solver loop that is being recorded into a CUDA
// graph (cudaMalloc/cudaFree are not stream-ordered and cannot be captured),
// a latency-bound service loop that must never hit the implicit device
// synchronisation of cudaMalloc/cudaFree, or a host program whose whole GPU
// memory is already handed out by an admission budget or another allocator so
// that an extra allocation could fail mid-solve.  For them tci_dots_noalloc
// does the same deterministic two-pass reduction as tci_dots but keeps its
// partial sums in one fixed, file-scope device array instead of memory
// obtained from cudaMalloc.
//
// Limits and sharing: at most kMaxRows rows per call.  The array costs
// kMaxRows * kBlocks * 8 bytes (303 KB) on every GPU that loads the library and
// is held until the process exits.  All calls share it and it keeps the last
// call's partial sums; every call overwrites all the partial sums it reads, so
// nothing needs clearing, but two calls whose kernels overlap on a GPU (for
// instance on two streams without ordering between them) race on it.
#include <cuda_runtime.h>

#include <cstdint>
#include <mutex>
#include <string>

#include "../../include/tigerci_sigma.h"
#include "host/capi_internal.h"

namespace {

constexpr int kThreads = 256;
constexpr int kBlocks = 592;  // 4 blocks per SM on a 148-SM B200
constexpr int64_t kMaxRows = TCI_DOTS_NOALLOC_MAX_ROWS;

// Partial sums, row-major [kMaxRows][kBlocks].
static __device__ __align__(256) double g_noalloc_scratch[kMaxRows * kBlocks];

__global__ void __launch_bounds__(kThreads) noalloc_partial(const double* __restrict__ A, long long lda, int m,
                                                            const double* __restrict__ x, long long n,
                                                            double* __restrict__ partial) {
  __shared__ double red[kThreads / 32];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long i0 = (long long)blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  for (int k = 0; k < m; ++k) {
    const double* a = A + (long long)k * lda;
    double acc = 0.0;
    for (long long i = i0 + threadIdx.x; i < i1; i += kThreads) acc = fma(a[i], x[i], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
      double t = 0.0;
      for (int w = 0; w < kThreads / 32; ++w) t += red[w];
      partial[(long long)k * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

__global__ void noalloc_final(const double* __restrict__ partial, int m, int nblk, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double t = 0.0;
  for (int b = 0; b < nblk; ++b) t += partial[(long long)k * nblk + b];
  out[k] = t;
}

// Device address of the scratch array, looked up once per device with that
// device current (in host code the array's name is only a host-side shadow).
std::mutex g_mu;
constexpr int kMaxDevices = 64;
double* g_scratch[kMaxDevices] = {};

double* scratch_of_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw tci::Error(TCI_ERR_CUDA, std::string("cudaGetDevice failed: ") + cudaGetErrorString(e));
  std::lock_guard<std::mutex> lk(g_mu);
  if (dev >= 0 && dev < kMaxDevices && g_scratch[dev]) return g_scratch[dev];
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
  if (e != cudaSuccess || !p)
    throw tci::Error(TCI_ERR_CUDA, std::string("cudaGetSymbolAddress of the projection scratch failed: ") +
                                       cudaGetErrorString(e));
  if (dev >= 0 && dev < kMaxDevices) g_scratch[dev] = static_cast<double*>(p);
  return static_cast<double*>(p);
}

}  // namespace

extern "C" int tci_dots_noalloc(const double* d_A, int64_t lda, int64_t m, const double* d_x, int64_t n,
                                double* d_out, void* stream) {
  if (!d_A || !d_x || !d_out || n <= 0 || m <= 0 || (m > 1 && lda < n)) {
    tci::set_error("tci_dots_noalloc: null pointer or inconsistent sizes");
    return TCI_ERR_ARG;
  }
  if (m > kMaxRows) {
    tci::set_error("tci_dots_noalloc: " + std::to_string((long long)m) + " rows exceed the fixed scratch limit of " +
                   std::to_string((long long)kMaxRows) + " (split the call or use tci_dots)");
    return TCI_ERR_ARG;
  }
  try {
    double* scratch = scratch_of_current_device();
    cudaStream_t st = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    noalloc_partial<<<kBlocks, kThreads, 0, st>>>(d_A, lda, (int)m, d_x, n, scratch);
    noalloc_final<<<(unsigned)((m + 127) / 128), 128, 0, st>>>(scratch, (int)m, kBlocks, d_out);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) throw tci::Error(TCI_ERR_CUDA, std::string("launch failed: ") + cudaGetErrorString(e));
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}
