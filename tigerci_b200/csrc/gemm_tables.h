// Device-side tables of a grouped GEMM (8-byte fields), shared by the FP64
// SIMT kernel (sigma_device.cu) and the tcgen05 kernel (gemm_tc.cu), and the
// host helper that tiles a list of problems for either kernel.
//
//   C (M x N, row pitch ldc) = beta C + sum over the problem's segments of
//   alpha A B, A M x K (K x M when tA), B K x N (N x K when tB), row major.
#pragma once
#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

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

// One problem before tiling.
struct HostGemm {
  double* C;
  long long ldc, M, N;
  double beta;
  std::vector<DGemmSeg> segs;
};

// Tiles the problems with tm x tn tiles (problems with M or N <= 0 are dropped).
// With allow_transpose, a problem whose N fills the tm-row tiles better than its
// M is stored transposed (C^T = B^T A^T, trans_c = 1).  Returns the tile count.
inline long long tile_problems(const std::vector<HostGemm>& in, long long tm, long long tn, bool allow_transpose,
                               std::vector<DGemmProblem>& probs, std::vector<DGemmSeg>& segs) {
  auto fill = [&](long long M, long long N) {
    return (double)M * (double)N / ((double)((M + tm - 1) / tm * tm) * (double)((N + tn - 1) / tn * tn));
  };
  long long tiles = 0;
  for (const auto& g : in) {
    if (g.M <= 0 || g.N <= 0) continue;
    const bool tr = allow_transpose && fill(g.N, g.M) > fill(g.M, g.N);
    DGemmProblem p{g.C, g.ldc, tr ? g.N : g.M, tr ? g.M : g.N, 0, tiles, g.beta, (long long)segs.size(), 0,
                   tr ? 1 : 0};
    for (const auto& x : g.segs)
      segs.push_back(tr ? DGemmSeg{x.B, x.A, x.ldb, x.lda, x.K, x.tB ? 0 : 1, x.tA ? 0 : 1, x.alpha} : x);
    p.seg_end = (long long)segs.size();
    p.tiles_n = (p.N + tn - 1) / tn;
    tiles += ((p.M + tm - 1) / tm) * p.tiles_n;
    probs.push_back(p);
  }
  return tiles;
}

// FP64 SIMT grouped GEMM (sigma_device.cu); cfg 0: 64 x 128 tiles, 1: 128 x 64.
cudaError_t launch_gemm_f64(int cfg, const DGemmProblem* probs, int nprob, const DGemmSeg* segs, long long ntiles,
                            cudaStream_t st);
// The cp.async-staged FP64 kernel (64 x 128 tiles): A not transposed, B K x N, operands 16-byte aligned
// with even leading dimensions.
cudaError_t launch_gemm_cp_f64(const DGemmProblem* probs, int nprob, const DGemmSeg* segs, long long ntiles,
                               cudaStream_t st);
inline long long gemm_cp_tile_m() { return 64; }
inline long long gemm_cp_tile_n() { return 128; }
inline long long gemm_f64_tile_m(int cfg) { return cfg == 0 ? 64 : 128; }
inline long long gemm_f64_tile_n(int cfg) { return cfg == 0 ? 128 : 64; }

}  // namespace tci_dev
