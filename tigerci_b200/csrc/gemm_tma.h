// Host interface of the TMA-fed two-external kernel (gemm_tma.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

// R_t = beta R_t + sum over segments alpha X D (all n x n), tiles of 128 x 64
struct TmaProblem {
  double* C;                    // R_t (row pitch n)
  long long tile_begin;
  double beta;
  long long seg_begin, seg_end;
};
struct TmaSeg {
  long long x_row;              // first row of X in the split integral rows
  long long d_row;              // first row of D in the split pair-matrix rows
  double alpha;                 // coefficient times the transposition sign of D
};

namespace tci_gtma_host {

struct TmaMaps {
  CUtensorMap xhi, xlo, dhi, dlo;
  int64_t n = 0;
};

int tile_m();
int tile_n();
int64_t pitch(int64_t n);  // FP32 row pitch of the split arrays (multiple of 32)
// rows x n FP64 (pitch n) -> hi / lo FP32 (pitch `pitch(n)`)
cudaError_t split(const double* src, int64_t rows, int64_t n, float* hi, float* lo, cudaStream_t st);
bool prepare(TmaMaps& m, const float* xhi, const float* xlo, int64_t xrows, const float* dhi, const float* dlo,
             int64_t drows, int64_t n, std::string& err);
cudaError_t launch(const TmaMaps& m, const TmaProblem* probs, int nprob, const TmaSeg* segs, long long ntiles,
                   int* status, cudaStream_t st);

}  // namespace tci_gtma_host
