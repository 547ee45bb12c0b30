// Device-side tables of a grouped GEMM plan step (8-byte fields), shared by
// the FP64 SIMT kernel (sigma_device.cu) and the tcgen05 kernel (gemm_tc.cu).
//
//   C (M x N, row pitch ldc) = beta C + sum over the problem's segments of
//   alpha A B, A M x K (K x M when tA), B K x N (N x K when tB), row major.
#pragma once

namespace tci_dev {

struct DGemmProblem {
  double* C;
  long long ldc, M, N, tiles_n, tile_begin;  // tiles_n, tile_begin: in the launching kernel's tile shape
  double beta;
  long long seg_begin, seg_end;
  long long trans_c;  // tensor-core tables only: M, N and the segments describe C^T = B^T A^T
};
struct DGemmSeg {
  const double* A;
  const double* B;
  long long lda, ldb, K;
  int tA, tB;
  double alpha;
};

}  // namespace tci_dev
