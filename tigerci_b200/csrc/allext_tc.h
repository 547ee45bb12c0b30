// Host interface of the tcgen05 all-external product (allext_tc.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

namespace tci_tc_host {

struct AllextTc {
  CUtensorMap u2;              // U as interleaved TF32-high / FP32-low rows (2 padded_rows x np, fp32)
  const float* w = nullptr;    // W as FP32 tiles (convert_w)
  int64_t np = 0, m = 0;
  int64_t bn = 64;             // CI blocks per group (m, at most 64)
  double* y = nullptr;         // m x np FP64 output (overwritten)
  int* status = nullptr;       // device status word (0 ok, else a bounded wait gave up)
  int64_t kblock = 256;        // k elements per FP64 promotion block
};

int64_t padded_ld(int64_t np);   // fp32 row pitch (multiple of 32 elements)
int64_t padded_rows(int64_t m);  // CI blocks of the split U (multiple of 64); it has twice as many rows
int64_t u2_floats(int64_t m, int64_t np);  // size of the split U
int64_t w32_floats(int64_t np);  // size of W's FP32 tile array
// FP64 W (np x np) -> the tile array the kernel streams (w32_floats(np) floats)
cudaError_t convert_w(const double* w64, int64_t np, float* w32, cudaStream_t st);
// The tiles of W+ (plus) or W- over n externals straight from the packed (ab|cd) matrix X (n(n+1)/2 squared,
// FP64), without an FP64 W: w32_floats(n + n(n-1)/2) or w32_floats(n(n-1)/2) floats.
cudaError_t convert_w_from_x(const double* x, int64_t n, bool plus, float* w32, cudaStream_t st);
cudaError_t split_u(const double* u, int64_t m, int64_t np, float* u2, cudaStream_t st);
bool prepare(AllextTc& t, const float* w32, int64_t np, const float* u2, int64_t m, double* y, int* status,
             int64_t kblock, std::string& err);
// Self-test of the bounded-wait abort path: a kernel whose wait (polls polls, the kernels' own helper)
// can never complete records its timeout code in *status and returns.
cudaError_t bounded_wait_selftest(int64_t polls, int* status, cudaStream_t st);
int64_t spin_limit();  // the polls of the kernels' bounded waits
// Self-test of the kind::tf32 MMA instruction rate (M = m, 64 or 128; N = n in 16..256 step 16 (8..256 step 8
// for M = 64); nacc independent accumulators, nacc * n <= 512): cycles[cta] for iters * nacc back-to-back
// MMAs, one CTA per SM, grid CTAs.
cudaError_t mma_rate_selftest(int64_t m, int64_t n, int64_t nacc, int64_t iters, int grid, long long* cycles,
                              int* status, cudaStream_t st);
// Both products in one launch (either may be null; they must share the status
// word and promotion block).  Persistent: at most one CTA per SM.
cudaError_t launch(const AllextTc* a, const AllextTc* b, cudaStream_t st);

}  // namespace tci_tc_host
