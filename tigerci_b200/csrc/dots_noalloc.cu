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

// Device address of the scratch array.  In host code the array's name is only
// a host-side shadow; the address is looked up with cudaGetSymbolAddress with
// the device current, and it is valid only in the CUDA context it was looked
// up in (a cudaDeviceReset, or a driver-API caller that makes another context
// current on the same device, gives the array a new address).  So each cached
// address is kept with the context it belongs to and looked up again when the
// current context differs.
using CtxGetCurrentFn = int (*)(void**);  // CUresult cuCtxGetCurrent(CUcontext*)

std::mutex g_mu;
constexpr int kMaxDevices = 64;
struct ScratchSlot {
  void* ctx = nullptr;
  double* ptr = nullptr;
};
ScratchSlot g_scratch[kMaxDevices];
CtxGetCurrentFn g_ctx_get_current = nullptr;
bool g_ctx_fn_resolved = false;

void* current_context() {  // caller holds g_mu
  if (!g_ctx_fn_resolved) {
    g_ctx_fn_resolved = true;
    void* p = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      g_ctx_get_current = reinterpret_cast<CtxGetCurrentFn>(p);
  }
  void* ctx = nullptr;
  if (!g_ctx_get_current) throw tci::Error(TCI_ERR_CUDA, "tci_dots_noalloc: cuCtxGetCurrent unavailable");
  if (g_ctx_get_current(&ctx) != 0) ctx = nullptr;
  return ctx;  // nullptr until the runtime has made a context current
}

double* scratch_of_current_device() {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) throw tci::Error(TCI_ERR_CUDA, std::string("cudaGetDevice failed: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) throw tci::Error(TCI_ERR_CUDA, "tci_dots_noalloc: device index out of range");
  std::lock_guard<std::mutex> lk(g_mu);
  void* ctx = current_context();
  ScratchSlot& slot = g_scratch[dev];
  if (ctx && slot.ptr && slot.ctx == ctx) return slot.ptr;
  void* p = nullptr;
  e = cudaGetSymbolAddress(&p, g_noalloc_scratch);  // also makes the primary context current if none is
  if (e != cudaSuccess || !p)
    throw tci::Error(TCI_ERR_CUDA, std::string("cudaGetSymbolAddress of the projection scratch failed: ") +
                                       cudaGetErrorString(e));
  ctx = current_context();
  if (!ctx) throw tci::Error(TCI_ERR_CUDA, "tci_dots_noalloc: no current CUDA context after the symbol lookup");
  slot.ctx = ctx;
  slot.ptr = static_cast<double*>(p);
  return slot.ptr;
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
