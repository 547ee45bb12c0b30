// Host interface of the TMA-fed 3xTF32 grouped GEMM (gemm_tma.cu).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <cstdint>
#include <string>

// C (row pitch ldc) = beta C + sum over segments alpha A_rows B_rows^T, tiles of 128 x tile_n(wide)
struct TmaProblem {
  double* C;
  long long ldc, M, N, tiles_n, tile_begin;
  double beta;
  long long seg_begin, seg_end;
  long long trans_c;  // the tile computes C^T: element (r, c) is stored at C[c][r]
  float* c_hi;        // non-null: C is written instead as TF32 high / FP32 low parts (row pitch ldcs, beta 0)
  float* c_lo;
  long long ldcs;
};
struct TmaSeg {
  long long a_row, b_row;  // first rows of the segment in the A and B arrays
  long long k0, K;         // columns k0 .. k0+K-1 (k0 a multiple of 32; K ends on a multiple of 32 or the row end)
  double alpha;
};

namespace tci_gtma_host {

// TF32-high / FP32-low copies of two FP64 row arrays, and their tensor maps
struct TmaMaps {
  CUtensorMap ahi, alo, bhi, blo;
  bool wide = true;  // tile width 128 (else 64, for B operands of at most 64 rows per problem)
};

int tile_m();
int tile_n(bool wide);
int64_t pitch(int64_t cols);  // FP32 row pitch of a split array (multiple of 32)
// rows x cols FP64 (row pitch ld) -> hi / lo FP32 (row pitch pitch(cols), zero padded)
cudaError_t split(const double* src, int64_t rows, int64_t cols, int64_t ld, float* hi, float* lo, cudaStream_t st);
// nmat consecutive rows x cols FP64 matrices -> their transposes, split: cols x pitch(rows) each, stacked
cudaError_t split_transposed(const double* src, int64_t nmat, int64_t rows, int64_t cols, float* hi, float* lo,
                             cudaStream_t st);
// maps over split arrays of arows x acols and brows x bcols
bool prepare(TmaMaps& m, const float* ahi, const float* alo, int64_t arows, int64_t acols, const float* bhi,
             const float* blo, int64_t brows, int64_t bcols, bool wide, std::string& err);
// kblock: k elements per FP64 promotion block (multiple of 32)
// persistent: at most one CTA per SM walking the tiles in a fixed order (tiles of similar length);
// otherwise one CTA per tile
cudaError_t launch(const TmaMaps& m, const TmaProblem* probs, int nprob, const TmaSeg* segs, long long ntiles,
                   int kblock, int* status, cudaStream_t st, bool persistent = true);

}  // namespace tci_gtma_host
