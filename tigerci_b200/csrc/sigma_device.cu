// Device executor of the sigma plan (host/plan.h) and the device half of the C
// ABI.  Kernels here (FP64):
//   gemm_tiled_f64    C = beta*C + sum_seg alpha*op(A)op(B), one CTA per 64x128
//                     or 128x64 tile of every problem, segments summed in table
//                     order (split-K for few-tile, long-K steps)
//   gemm_skinny_f64   problems of at most 8 rows: a warp per output column
//   axpy_segments     one block per target chunk, sources summed in table order
//   dot_segments      one block per target scalar
//   unpack_pairs / pack_pairs   SCEP <-> dense external pair matrices
//                     (tiger_fortran/scepmaker_mod.f90:121-257, 633-800)
//   build_allext      W+ / W- from the packed external (ab|cd) block
//   Davidson kernels  projections, linear combinations, preconditioner
// The mixed form's tensor-core steps run on allext_tc.cu, gemm_tma.cu and
// gemm_tc.cu.  The plan is replayed in a fixed launch order on one stream, so
// every sigma build is bitwise reproducible.
#include <cuda_runtime.h>

#include <algorithm>
#include <thread>
#include <tuple>
#include <array>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <cstring>
#include <future>
#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "../../include/tigerci_sigma.h"
#include "allext_tc.h"
#include "device_info.h"
#include "gemm_tables.h"
#include "gemm_tc.h"
#include "gemm_tma.h"
#include "host/capi_internal.h"
#include "host/plan.h"

using namespace tci;

#define TCI_CUDA(call)                                                                       \
  do {                                                                                       \
    cudaError_t _e = (call);                                                                 \
    if (_e != cudaSuccess)                                                                   \
      throw Error(TCI_ERR_CUDA, std::string(#call) + " (sigma_device.cu:" + std::to_string(__LINE__) + \
                                    ") failed: " + cudaGetErrorString(_e));                            \
  } while (0)

namespace {

unsigned sm_count() { return tci_dev::device_sms(); }

// ----------------------------------------------------------------------------
// device-side table layouts (plain structs, 8-byte fields)
using tci_dev::DGemmProblem;
using tci_dev::DGemmSeg;
struct DAxpyTarget {
  double* dst;             // already offset by base
  long long base;          // offset of this chunk inside the target range (applied to sources)
  long long len, src_begin, src_end;
};
struct DAxpySource {
  const double* src;
  const double* scale;  // nullptr: 1
  double coef;
};
struct DDotTarget {
  double* dst;
  long long src_begin, src_end;
};
struct DDotSource {
  const double* a;
  const double* b;
  long long len;
  double coef;
};
struct DHead {
  long long off_ab, off_aa, nsf_ab, nsf_aa, nsing, nD, dk0;
};

constexpr int GT = 64;   // tile edge
constexpr int GK = 16;   // k step
constexpr int GTH = 256; // threads (16 x 16, 4 x 4 outputs each)

__global__ void __launch_bounds__(GTH) gemm_grouped_f64(const DGemmProblem* __restrict__ probs, int nprob,
                                                        const DGemmSeg* __restrict__ segs) {
  __shared__ double As[GK][GT + 1];
  __shared__ double Bs[GK][GT + 1];
  // locate problem of this tile
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DGemmProblem P = probs[lo];
  const long long t = tile - P.tile_begin;
  const long long m0 = (t / P.tiles_n) * GT, n0 = (t % P.tiles_n) * GT;
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  double acc[4][4];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j] = 0.0;
  for (long long s = P.seg_begin; s < P.seg_end; ++s) {
    const DGemmSeg S = segs[s];
    double acs[4][4];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acs[i][j] = 0.0;
    for (long long k0 = 0; k0 < S.K; k0 += GK) {
      // load A tile (GT rows x GK cols) into As[k][m]
      for (int e = threadIdx.x; e < GT * GK; e += GTH) {
        int mm, kk;
        if (S.tA) { mm = e % GT; kk = e / GT; }   // A stored K x M: contiguous in m
        else { kk = e % GK; mm = e / GK; }        // A stored M x K: contiguous in k
        const long long gm = m0 + mm, gk = k0 + kk;
        double v = 0.0;
        if (gm < P.M && gk < S.K) v = S.tA ? S.A[gk * S.lda + gm] : S.A[gm * S.lda + gk];
        As[kk][mm] = v;
      }
      for (int e = threadIdx.x; e < GT * GK; e += GTH) {
        int nn, kk;
        if (S.tB) { kk = e % GK; nn = e / GK; }   // B stored N x K
        else { nn = e % GT; kk = e / GT; }        // B stored K x N
        const long long gn = n0 + nn, gk = k0 + kk;
        double v = 0.0;
        if (gn < P.N && gk < S.K) v = S.tB ? S.B[gn * S.ldb + gk] : S.B[gk * S.ldb + gn];
        Bs[kk][nn] = v;
      }
      __syncthreads();
#pragma unroll
      for (int kk = 0; kk < GK; ++kk) {
        double a[4], b[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) a[i] = As[kk][ty + 16 * i];
#pragma unroll
        for (int j = 0; j < 4; ++j) b[j] = Bs[kk][tx + 16 * j];
#pragma unroll
        for (int i = 0; i < 4; ++i)
#pragma unroll
          for (int j = 0; j < 4; ++j) acs[i][j] = fma(a[i], b[j], acs[i][j]);
      }
      __syncthreads();
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) acc[i][j] = fma(S.alpha, acs[i][j], acc[i][j]);
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long gm = m0 + ty + 16 * i;
    if (gm >= P.M) continue;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const long long gn = n0 + tx + 16 * j;
      if (gn >= P.N) continue;
      double* c = P.C + gm * P.ldc + gn;
      *c = (P.beta == 0.0) ? acc[i][j] : fma(P.beta, *c, acc[i][j]);
    }
  }
}


// Register-blocked FP64 GEMM: CTA tile BM x BN, k-step 16, each of the 256
// threads owns a TM x TN block of C; the next k-tile is prefetched into
// registers while the current one is consumed from shared memory (double
// buffered).  Same problem/segment tables and summation order per element as
// gemm_grouped_f64: segments in table order, k ascending within a segment.
template <int BM, int BN, int TM, int TN>
__global__ void __launch_bounds__(256, 2) gemm_tiled_f64(const DGemmProblem* __restrict__ probs, int nprob,
                                                      const DGemmSeg* __restrict__ segs) {
  constexpr int BK = 8;
  constexpr int NTX = BN / TN;  // threads along n
  static_assert((BM / TM) * (BN / TN) == 256, "256 threads");
  constexpr int LA = BM * BK / 256, LB = BN * BK / 256;  // elements loaded per thread
  __shared__ double As[2][BK][BM + 2];
  __shared__ double Bs[2][BK][BN + 2];
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DGemmProblem P = probs[lo];
  const long long t = tile - P.tile_begin;
  const long long m0 = (t / P.tiles_n) * BM, n0 = (t % P.tiles_n) * BN;
  const int tid = threadIdx.x, tx = tid % NTX, ty = tid / NTX;
  double acc[TM][TN];
#pragma unroll
  for (int i = 0; i < TM; ++i)
#pragma unroll
    for (int j = 0; j < TN; ++j) acc[i][j] = 0.0;
  for (long long sgi = P.seg_begin; sgi < P.seg_end; ++sgi) {
    const DGemmSeg S = segs[sgi];
    double ra[LA], rb[LB];
    // the segment's alpha is folded into its B operand as it is loaded
    auto load = [&](long long k0) {
#pragma unroll
      for (int u = 0; u < LA; ++u) {
        const int e = tid + u * 256;
        int mm, kk;
        if (S.tA) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
        const long long gm = m0 + mm, gk = k0 + kk;
        ra[u] = (gm < P.M && gk < S.K) ? (S.tA ? S.A[gk * S.lda + gm] : S.A[gm * S.lda + gk]) : 0.0;
      }
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const int e = tid + u * 256;
        int nn, kk;
        if (S.tB) { kk = e % BK; nn = e / BK; } else { nn = e % BN; kk = e / BN; }
        const long long gn = n0 + nn, gk = k0 + kk;
        rb[u] = (gn < P.N && gk < S.K) ? S.alpha * (S.tB ? S.B[gn * S.ldb + gk] : S.B[gk * S.ldb + gn]) : 0.0;
      }
    };
    auto store = [&](int buf) {
#pragma unroll
      for (int u = 0; u < LA; ++u) {
        const int e = tid + u * 256;
        int mm, kk;
        if (S.tA) { mm = e % BM; kk = e / BM; } else { kk = e % BK; mm = e / BK; }
        As[buf][kk][mm] = ra[u];
      }
#pragma unroll
      for (int u = 0; u < LB; ++u) {
        const int e = tid + u * 256;
        int nn, kk;
        if (S.tB) { kk = e % BK; nn = e / BK; } else { nn = e % BN; kk = e / BN; }
        Bs[buf][kk][nn] = rb[u];
      }
    };
    __syncthreads();  // previous segment finished reading the buffers
    load(0);
    store(0);
    __syncthreads();
    int buf = 0;
    for (long long k0 = 0; k0 < S.K; k0 += BK) {
      const bool more = k0 + BK < S.K;
      if (more) load(k0 + BK);
#pragma unroll
      for (int kk = 0; kk < BK; ++kk) {
        double a[TM], b[TN];
#pragma unroll
        for (int i = 0; i < TM; ++i) a[i] = As[buf][kk][ty + (BM / TM) * i];
#pragma unroll
        for (int j = 0; j < TN; ++j) b[j] = Bs[buf][kk][tx + NTX * j];
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
          for (int j = 0; j < TN; ++j) acc[i][j] = fma(a[i], b[j], acc[i][j]);
      }
      if (more) store(buf ^ 1);
      __syncthreads();
      buf ^= 1;
    }
  }
#pragma unroll
  for (int i = 0; i < TM; ++i) {
    const long long gm = m0 + ty + (BM / TM) * i;
    if (gm >= P.M) continue;
#pragma unroll
    for (int j = 0; j < TN; ++j) {
      const long long gn = n0 + tx + NTX * j;
      if (gn >= P.N) continue;
      double* c = P.C + gm * P.ldc + gn;
      *c = (P.beta == 0.0) ? acc[i][j] : fma(P.beta, *c, acc[i][j]);
    }
  }
}

// Skinny grouped GEMM (M <= SKINNY_M, B given as N x K): one warp per output
// column n of a problem computes C[m][n] for every row m as dot products over
// the segments (lanes along k, fixed-order warp reductions).  Covers the
// one-row products that would fill 1/64 of a tile of the tiled kernel.  Warp
// numbers are laid out so that the 8 warps of a block share one problem: the
// block looks its problem up once, and its warps read the same A rows (L1).
constexpr int SKINNY_M = 8;
__global__ void __launch_bounds__(256) gemm_skinny_f64(const DGemmProblem* __restrict__ probs, int nprob,
                                                       const DGemmSeg* __restrict__ segs, long long nwarps) {
  __shared__ int prob_of_block;
  const long long w0 = (long long)blockIdx.x * 8;  // first warp of the block
  if (threadIdx.x == 0) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (probs[mid].tile_begin <= w0) lo = mid;
      else hi = mid - 1;
    }
    prob_of_block = lo;
  }
  __syncthreads();
  const long long w = w0 + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  const DGemmProblem P = probs[prob_of_block];
  const long long n = w - P.tile_begin;
  if (w >= nwarps || n >= P.N) return;
  // each lane keeps sum_q alpha_q (its part of A_m . b_q); one reduction per row at the end
  double acc[SKINNY_M];
#pragma unroll
  for (int m = 0; m < SKINNY_M; ++m) acc[m] = 0.0;
  for (long long q = P.seg_begin; q < P.seg_end; ++q) {
    const DGemmSeg S = segs[q];
    const double* b = S.B + n * S.ldb;
    // 16-byte loads when both rows start on 16 bytes and K is even
    const bool vec = ((reinterpret_cast<uintptr_t>(S.A) | reinterpret_cast<uintptr_t>(b)) & 15) == 0 &&
                     ((S.lda | S.K) & 1) == 0;
    if (vec && S.K <= 256) {  // the b row in registers once, every row of A against it
      const double2* b2 = reinterpret_cast<const double2*>(b);
      const long long h = S.K / 2;
      double2 y[4];
#pragma unroll
      for (int e = 0; e < 4; ++e) y[e] = lane + 32 * e < h ? __ldg(b2 + lane + 32 * e) : make_double2(0.0, 0.0);
#pragma unroll
      for (int m = 0; m < SKINNY_M; ++m) {
        if (m >= P.M) break;
        const double2* a2 = reinterpret_cast<const double2*>(S.A + m * S.lda);
        double2 x[4];
#pragma unroll
        for (int e = 0; e < 4; ++e) x[e] = lane + 32 * e < h ? __ldg(a2 + lane + 32 * e) : make_double2(0.0, 0.0);
        double d = 0.0;
#pragma unroll
        for (int e = 0; e < 4; ++e) {
          d = fma(x[e].x, y[e].x, d);
          d = fma(x[e].y, y[e].y, d);
        }
        acc[m] = fma(S.alpha, d, acc[m]);
      }
      continue;
    }
#pragma unroll
    for (int m = 0; m < SKINNY_M; ++m) {
      if (m >= P.M) break;
      const double* a = S.A + m * S.lda;
      double d = 0.0;
      if (vec) {
        const double2* a2 = reinterpret_cast<const double2*>(a);
        const double2* b2 = reinterpret_cast<const double2*>(b);
        for (long long k = lane; k < S.K / 2; k += 32) {
          const double2 x = __ldg(a2 + k), y = __ldg(b2 + k);
          d = fma(x.x, y.x, d);
          d = fma(x.y, y.y, d);
        }
      } else {
        for (long long k = lane; k < S.K; k += 32) d = fma(__ldg(a + k), __ldg(b + k), d);
      }
      acc[m] = fma(S.alpha, d, acc[m]);
    }
  }
#pragma unroll
  for (int m = 0; m < SKINNY_M; ++m)
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc[m] += __shfl_xor_sync(0xffffffffu, acc[m], o);
  if (lane == 0)
    for (int m = 0; m < SKINNY_M && m < P.M; ++m) {
      double* c = P.C + m * P.ldc + n;
      *c = (P.beta == 0.0 ? 0.0 : P.beta * *c) + acc[m];
    }
}

__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }
// 8-byte form (gathers of single elements); src_bytes 0 fills the destination with zeros
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes) : "memory");
}

// Domain-restricted two-external products of a local deck (pair domains) over the common virtuals, as the
// reference takes them (two_int_seg_com_lmo_res, three_and_four_seg_mod_2.f90:7137-8005, GEMMs at :7718-7751).
// Source head mu's pair matrix is zero outside D_mu x D_mu and the target head lambda needs only
// D_lambda x D_lambda, so a term reaches only the columns in both domains:
//   R_lambda[a][b] += alpha sum_{c in D_mu} X[a][c] D_mu[c][b]      (a in D_lambda, b in D_lambda and D_mu)
// m_lambda x |common| x m_mu per term instead of m_lambda x m_lambda x m_mu. The step works on compact squares:
// per sigma build the pair matrices of the local heads are gathered into m x m squares (com_gather_sq), the
// products accumulate into compact m x m accumulators (zeroed first) that are then added into the padded ones
// (com_scatter_sq); the integral operands X[D_lambda][D_mu] are constant and compacted once at set-up when the
// device has room (com_pack_a), else gathered from the n x n matrices. Each term carries its common columns as
// positions in the source's and in the target's domain. A block owns 64 rows of one target and walks all its
// (term, 32-column chunk, 16-deep k chunk) in table order, the operands copied by 8-byte cp.async
// COM_STG - 1 chunks ahead of the FMAs (one barrier per chunk); at the end of each column chunk it adds alpha
// times its 64 x 32 sums into the target's square. Every element is written by one block, its terms in table
// order, and the barrier between two column chunks orders the read-modify-writes of different threads: the sum
// stays in a fixed order.
struct DComProblem {
  double* C;         // the target's compact accumulator (m x m, row pitch `pitch`)
  const int* dom;    // the target's domain (rows of the gathered integral operand)
  int m, pitch;
  long long tile_begin, seg_begin, seg_end;
};
struct DComSeg {
  const double* A;   // the n x n integral operand (gathered when Ac is nullptr)
  const double* Ac;  // A[D_target][D_source], row pitch pitch_a, or nullptr
  const double* B;   // the source's compact pair matrix, row pitch pitch_b
  const int* dom;    // the source's domain (the k range)
  const int* cs;     // the common columns: positions in the source's domain ...
  const int* ct;     // ... and in the target's
  int m, ncol, pitch_a, pitch_b;
  double alpha;
};
// one compaction job: Ac[r][c] = A[rows[r]][cols[c]] (r < m, c < ms), row pitch `pitch`
struct DComPack {
  const double* A;
  double* Ac;
  const int* rows;
  const int* cols;
  int m, ms, pitch;
};
__global__ void __launch_bounds__(256) com_pack_a(const DComPack* __restrict__ jobs, long long ld) {
  const DComPack J = jobs[blockIdx.x];
  for (int e = threadIdx.x; e < J.m * J.ms; e += blockDim.x) {
    const int r = e / J.ms, c = e - r * J.ms;
    J.Ac[(long long)r * J.pitch + c] = J.A[(long long)J.rows[r] * ld + J.cols[c]];
  }
}
// a padded n x n matrix and its compact m x m square over a domain
struct DComSq {
  double* pad;
  double* sq;
  const int* dom;
  int m, pitch;
};
__global__ void __launch_bounds__(256) com_gather_sq(const DComSq* __restrict__ sq, long long ld) {
  const DComSq Q = sq[blockIdx.x];
  for (int e = threadIdx.x; e < Q.m * Q.m; e += blockDim.x) {
    const int r = e / Q.m, c = e - r * Q.m;
    Q.sq[(long long)r * Q.pitch + c] = Q.pad[(long long)Q.dom[r] * ld + Q.dom[c]];
  }
}
__global__ void __launch_bounds__(256) com_scatter_sq(const DComSq* __restrict__ sq, long long ld) {
  const DComSq Q = sq[blockIdx.x];
  for (int e = threadIdx.x; e < Q.m * Q.m; e += blockDim.x) {
    const int r = e / Q.m, c = e - r * Q.m;
    Q.pad[(long long)Q.dom[r] * ld + Q.dom[c]] += Q.sq[(long long)r * Q.pitch + c];
  }
}
constexpr int COM_R = 64, COM_C = 32, COM_K = 16, COM_THREADS = 128, COM_STG = 3;
// position in a block's (segment, column chunk, k chunk) sequence
struct ComCursor {
  long long s;
  int c, k;
};
__global__ void __launch_bounds__(COM_THREADS, 4) gemm_com_f64(const DComProblem* __restrict__ probs, int nprob,
                                                              const DComSeg* __restrict__ segs, long long ld) {
  __shared__ __align__(16) double As[COM_STG][COM_K][COM_R];
  __shared__ __align__(16) double Bs[COM_STG][COM_K][COM_C];
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DComProblem P = probs[lo];
  if (P.seg_begin >= P.seg_end) return;
  const int r0 = (int)(tile - P.tile_begin) * COM_R;
  // outputs: rows 8 ty .. 8 ty + 7, columns tx and tx + 16 of the chunk
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  // copy slots: A rows ia + 8 q at k = ka; B rows kb + 4 q at column jb
  const int ka = tid & 15, ia = tid >> 4, kb = tid >> 5, jb = tid & 31;
  auto advance = [&](ComCursor& x, const DComSeg& S) {
    x.k += COM_K;
    if (x.k < S.m) return;
    x.k = 0;
    x.c += COM_C;
    if (x.c < S.ncol) return;
    x.c = 0;
    ++x.s;
  };
  // the copies of one chunk into stage st (zeros past the domains, the rows or the common columns)
  auto issue = [&](const ComCursor& x, const DComSeg& S, int st) {
    const int k = x.k + ka;
    if (S.Ac) {  // compacted: 16 consecutive k of a row across the 16 threads of a row group
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int r = r0 + ia + 8 * q;
        const bool ok = r < P.m && k < S.m;
        cp_async8(&As[st][ka][ia + 8 * q], ok ? (const void*)(S.Ac + (long long)r * S.pitch_a + k) : (const void*)S.Ac,
                  ok ? 8 : 0);
      }
    } else {
      const long long col = k < S.m ? (long long)S.dom[k] : -1;
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        const int r = r0 + ia + 8 * q;
        const bool ok = r < P.m && col >= 0;
        cp_async8(&As[st][ka][ia + 8 * q], ok ? (const void*)(S.A + (long long)P.dom[r] * ld + col) : (const void*)S.A,
                  ok ? 8 : 0);
      }
    }
    const int bc = x.c + jb < S.ncol ? S.cs[x.c + jb] : -1;
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int kk = x.k + kb + 4 * q;
      const bool ok = kk < S.m && bc >= 0;
      cp_async8(&Bs[st][kb + 4 * q][jb], ok ? (const void*)(S.B + (long long)kk * S.pitch_b + bc) : (const void*)S.B,
                ok ? 8 : 0);
    }
  };
  // producer cursor: COM_STG - 1 chunks ahead of the consumer
  ComCursor pc{P.seg_begin, 0, 0};
  DComSeg PS = segs[pc.s];
  for (int st = 0; st < COM_STG - 1; ++st) {
    if (pc.s < P.seg_end) {
      issue(pc, PS, st);
      advance(pc, PS);
      if (pc.s < P.seg_end && pc.c == 0 && pc.k == 0) PS = segs[pc.s];
    }
    cp_async_commit();
  }
  ComCursor cc{P.seg_begin, 0, 0};
  DComSeg S = segs[cc.s];
  double acc[8][2];
#pragma unroll
  for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
  for (int it = 0;; ++it) {
    const int st = it % COM_STG;
    cp_async_wait<COM_STG - 2>();  // this thread's copies of the chunk have landed
    __syncthreads();               // everyone's have, and the stage refilled below is no longer read
#pragma unroll
    for (int k = 0; k < COM_K; ++k) {
      const double2* ap = reinterpret_cast<const double2*>(&As[st][k][8 * ty]);
      double a[8];
#pragma unroll
      for (int h = 0; h < 4; ++h) {
        const double2 v = ap[h];
        a[2 * h] = v.x;
        a[2 * h + 1] = v.y;
      }
      const double b0 = Bs[st][k][tx], b1 = Bs[st][k][tx + 16];
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        acc[r][0] = fma(a[r], b0, acc[r][0]);
        acc[r][1] = fma(a[r], b1, acc[r][1]);
      }
    }
    // the copies COM_STG - 1 chunks ahead, after the FMAs so that their index loads overlap them
    if (pc.s < P.seg_end) {
      issue(pc, PS, (it + COM_STG - 1) % COM_STG);
      advance(pc, PS);
      if (pc.s < P.seg_end && pc.c == 0 && pc.k == 0) PS = segs[pc.s];
    }
    cp_async_commit();
    const ComCursor prev = cc;
    advance(cc, S);
    if (cc.s != prev.s || cc.c != prev.c) {  // this column chunk is complete: add it into the target's square
      int ct[2];
#pragma unroll
      for (int c = 0; c < 2; ++c) {
        const int j = prev.c + tx + 16 * c;
        ct[c] = j < S.ncol ? S.ct[j] : -1;
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) {
        const int i = r0 + 8 * ty + r;
        if (i >= P.m) continue;
        double* row = P.C + (long long)i * P.pitch;
#pragma unroll
        for (int c = 0; c < 2; ++c)
          if (ct[c] >= 0) row[ct[c]] += S.alpha * acc[r][c];
      }
#pragma unroll
      for (int r = 0; r < 8; ++r) acc[r][0] = acc[r][1] = 0.0;
      if (cc.s >= P.seg_end) break;
      if (cc.s != prev.s) S = segs[cc.s];
    }
  }
  cp_async_wait<0>();
}

// Domain-restricted three-external products of a local deck (pair domains), on the padded pair matrices and
// the (iq|bs) banks V_i[b][q n + s] (the reference's local three-external gathers, iabc_sig_cho_big_res,
// three_and_four_seg_mod_1.f90:1099-1376). The pair matrices of an N-2 head lambda are zero outside
// D_lambda x D_lambda and only the rows b in D_mu of the N-1 head mu = lambda + e_i reach the local sigma, so
//   forward  Y_(i,dk)[b] = sum_{q,s in D_lambda} V_i[b][q n + s] D_dk[q][s]          (b in D_mu)
//   reverse  R_dk[q][s] += sum_i sum_{b in D_mu(i)} U_(i,dk)[b] V_i[b][q n + s]       (q, s in D_lambda)
// with Y_(i,dk) the row (i nD + dk) n of Y and U_(i,dk) that of U. The pair matrices of one head share its
// domain: a unit takes up to D3_K of them, so each V_i element it reads serves all. Sums in a fixed order.
constexpr int D3_K = 4;   // pair matrices (dk) of one head per unit
constexpr int D3_QC = 8;  // rows q of the D_dk staged in shared memory per pass (forward)
struct D3Fwd {
  long long i, dk0;
  const int* dl;  // D_lambda (sorted externals)
  const int* dm;  // D_mu
  int ml, mm, nk;
  int b0, b1;     // the rows [b0, b1) of D_mu this block takes
};
constexpr int D3_BCHUNK = 32;  // rows of D_mu per forward block
struct D3Rev {
  long long dk0, tile_begin;
  const int* dl;
  int ml, nk;
  long long e_begin, e_end;  // its (i, D_mu) entries
};
struct D3RevEntry {
  long long i;
  const int* dm;
  int mm;
};
constexpr int D3R_T = 256;  // outputs (q, s) per reverse tile
__global__ void __launch_bounds__(256) dom3_forward(const D3Fwd* __restrict__ units, const double* __restrict__ V,
                                                    const double* __restrict__ D, double* __restrict__ Y, long long n,
                                                    long long nD) {
  extern __shared__ double d3_smem[];
  const D3Fwd u = units[blockIdx.x];
  const int nb = u.b1 - u.b0;
  double* ds = d3_smem;                             // [D3_K][D3_QC][ml]
  double* yacc = d3_smem + D3_K * D3_QC * u.ml;     // [D3_K][nb]
  int* sdl = reinterpret_cast<int*>(yacc + D3_K * nb);  // [ml]: D_lambda
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nwarp = blockDim.x >> 5;
  const long long n2 = n * n;
  const double* Vi = V + u.i * n * n2;
  for (int e = threadIdx.x; e < D3_K * nb; e += blockDim.x) yacc[e] = 0.0;
  for (int e = threadIdx.x; e < u.ml; e += blockDim.x) sdl[e] = u.dl[e];
  for (int q0 = 0; q0 < u.ml; q0 += D3_QC) {
    const int nq = min(D3_QC, u.ml - q0);
    __syncthreads();  // sdl is written / the previous pass's reads of ds are done
    for (int e = threadIdx.x; e < u.nk * nq * u.ml; e += blockDim.x) {
      const int k = e / (nq * u.ml), r = e - k * (nq * u.ml);
      const int qq = r / u.ml, sidx = r - qq * u.ml;
      ds[(k * D3_QC + qq) * u.ml + sidx] = D[(u.dk0 + k) * n2 + (long long)sdl[q0 + qq] * n + sdl[sidx]];
    }
    __syncthreads();
    long long qoff[D3_QC];
#pragma unroll
    for (int qq = 0; qq < D3_QC; ++qq) qoff[qq] = qq < nq ? (long long)sdl[q0 + qq] * n : 0;
    for (int bl = warp; bl < nb; bl += nwarp) {
      const double* vrow = Vi + (long long)u.dm[u.b0 + bl] * n2;
      double part[D3_K] = {0.0, 0.0, 0.0, 0.0};
      for (int sidx = lane; sidx < u.ml; sidx += 32) {
        const int c = sdl[sidx];
        double v[D3_QC];
#pragma unroll
        for (int qq = 0; qq < D3_QC; ++qq) v[qq] = qq < nq ? vrow[qoff[qq] + c] : 0.0;  // D3_QC loads in flight
#pragma unroll
        for (int qq = 0; qq < D3_QC; ++qq) {
#pragma unroll
          for (int k = 0; k < D3_K; ++k)
            if (k < u.nk && qq < nq) part[k] = fma(v[qq], ds[(k * D3_QC + qq) * u.ml + sidx], part[k]);
        }
      }
#pragma unroll
      for (int k = 0; k < D3_K; ++k) {
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) part[k] += __shfl_xor_sync(0xffffffffu, part[k], o);
      }
      if (lane == 0) {
#pragma unroll
        for (int k = 0; k < D3_K; ++k)
          if (k < u.nk) yacc[k * nb + bl] += part[k];
      }
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < u.nk * nb; e += blockDim.x) {
    const int k = e / nb, bl = e - k * nb;
    Y[(u.i * nD + u.dk0 + k) * n + u.dm[u.b0 + bl]] = yacc[k * nb + bl];
  }
}
__global__ void __launch_bounds__(D3R_T) dom3_reverse(const D3Rev* __restrict__ units, int nunit,
                                                      const D3RevEntry* __restrict__ ent,
                                                      const double* __restrict__ V, const double* __restrict__ U,
                                                      double* __restrict__ R, long long n, long long nD) {
  int lo = 0, hi = nunit - 1;  // the unit of this tile: the last with tile_begin <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (units[mid].tile_begin <= (long long)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const D3Rev u = units[lo];
  const int e = (int)(((long long)blockIdx.x - u.tile_begin) * D3R_T) + threadIdx.x;
  if (e >= u.ml * u.ml) return;
  const long long n2 = n * n;
  const int q = e / u.ml, sidx = e - q * u.ml;
  const long long col = (long long)u.dl[q] * n + u.dl[sidx];
  double acc[D3_K] = {0.0, 0.0, 0.0, 0.0};
  for (long long p = u.e_begin; p < u.e_end; ++p) {
    const D3RevEntry E = ent[p];
    const double* vcol = V + E.i * n * n2 + col;
    const double* urow = U + (E.i * nD + u.dk0) * n;
#pragma unroll 4
    for (int b = 0; b < E.mm; ++b) {
      const int bb = E.dm[b];
      const double v = vcol[(long long)bb * n2];
#pragma unroll
      for (int k = 0; k < D3_K; ++k)
        if (k < u.nk) acc[k] = fma(urow[k * n + bb], v, acc[k]);
    }
  }
#pragma unroll
  for (int k = 0; k < D3_K; ++k)
    if (k < u.nk) R[(u.dk0 + k) * n2 + col] += acc[k];
}

// The N-2 <-> valence exchange term of a local deck on the domains (the reference's local dv loops,
// three_and_four_seg_mod_2.f90:8007-8165): only the entries (pq, dk) that the plan's couplings use, each over
// D_lambda x D_lambda of the head lambda of dk, with K_pq the row pq of the exchange bank (n^2 long)
//   forward  F[pq nD + dk] = sum_{q,s in D_lambda} K_pq[q n + s] D_dk[q][s]
//   reverse  R_dk[q][s] += sum_pq G[pq nD + dk] K_pq[q n + s]                 (q, s in D_lambda)
struct DvEntry {
  long long pq, dk;
  const int* dl;
  int ml;
};
struct DvTarget {
  long long dk, tile_begin;
  const int* dl;
  int ml;
  long long e_begin, e_end;  // its entries (pq) in the entry table
};
__global__ void __launch_bounds__(256) dom_dv_forward(const DvEntry* __restrict__ ent, long long nent,
                                                      const double* __restrict__ K, const double* __restrict__ D,
                                                      double* __restrict__ F, long long n, long long nD) {
  const long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
  const int lane = threadIdx.x & 31;
  if (w >= nent) return;
  const DvEntry E = ent[w];
  const long long n2 = n * n;
  const double* kp = K + E.pq * n2;
  const double* dp = D + E.dk * n2;
  double acc = 0.0;
  for (int q = 0; q < E.ml; ++q) {
    const long long r = (long long)E.dl[q] * n;
    for (int sidx = lane; sidx < E.ml; sidx += 32) {
      const int c = E.dl[sidx];
      acc = fma(kp[r + c], dp[r + c], acc);
    }
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
  if (lane == 0) F[E.pq * nD + E.dk] = acc;
}
__global__ void __launch_bounds__(256) dom_dv_reverse(const DvTarget* __restrict__ tg, int ntg,
                                                      const long long* __restrict__ pqs,
                                                      const double* __restrict__ K, const double* __restrict__ G,
                                                      double* __restrict__ R, long long n, long long nD) {
  int lo = 0, hi = ntg - 1;  // the target of this tile: the last with tile_begin <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tg[mid].tile_begin <= (long long)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const DvTarget T = tg[lo];
  const int e = (int)(((long long)blockIdx.x - T.tile_begin) * blockDim.x) + threadIdx.x;
  if (e >= T.ml * T.ml) return;
  const long long n2 = n * n;
  const int q = e / T.ml, sidx = e - q * T.ml;
  const long long col = (long long)T.dl[q] * n + T.dl[sidx];
  double acc = 0.0;
  for (long long p = T.e_begin; p < T.e_end; ++p) acc = fma(G[pqs[p] * nD + T.dk], K[pqs[p] * n2 + col], acc);
  R[T.dk * n2 + col] += acc;
}

// The zero-external step of a local deck on the common positions: a target row of an N-2 or N-1 head
// (padded: one row of pairs or of externals per spin function) receives coef x the source row of another head
// of its kind, and only the positions in both heads' domains carry terms (the source row is zero outside its
// domain, the target's are never read back outside its own): dst[rel[e]] += coef src[rel[e]] over the list of
// relative positions of the head pair. One block per target row, its sources in table order with a barrier
// between two (the same position may fall to different threads in two lists): a fixed order of sums.
struct ZcTarget {
  double* dst;
  long long src_begin, src_end;
};
struct ZcSource {
  const double* src;
  const int* rel;
  int nrel;
  double coef;
};
__global__ void __launch_bounds__(256) axpy_common(const ZcTarget* __restrict__ tg, const ZcSource* __restrict__ so) {
  const ZcTarget T = tg[blockIdx.x];
  for (long long q = T.src_begin; q < T.src_end; ++q) {
    const ZcSource S = so[q];
    for (int e = threadIdx.x; e < S.nrel; e += blockDim.x) {
      const int r = S.rel[e];
      T.dst[r] = fma(S.coef, S.src[r], T.dst[r]);
    }
    __syncthreads();
  }
}

// The one-external term of a local deck on the pair domains: a coupling row w_t (over the externals) meets
// the pair matrix D_dk of the N-2 head lambda, zero outside D_lambda x D_lambda, so
//   forward  Z_t[b] = sum_{q in D_lambda} w_t[q] D_dk[q][b]      (b in D_lambda; the rest of the row zero)
//   reverse  R_dk[q][b] += sum_t w_t[q] Cg_t[b]                   (q, b in D_lambda; t over the rows of dk)
// with Cg_t the gathered CI row of the row's N-1 CSF (the reference's local one-external loops restrict the
// same sums to the allowed virtuals, three_and_four_seg_mod_1.f90:1099-1376). One block per row (forward) or
// per 256 outputs of one pair matrix (reverse); sums in a fixed order.
struct D1Row {
  const double* w;
  const double* D;
  double* z;
  const int* dl;
  int ml;
};
struct D1Target {
  double* R;
  const double* w;   // the first coupling row of the pair matrix's group
  const double* cg;  // its first gathered CI row
  const int* dl;
  int ml, rows;
  long long tile_begin;
};
__global__ void __launch_bounds__(128) dom1_forward(const D1Row* __restrict__ rows, long long n) {
  const D1Row U = rows[blockIdx.x];
  for (long long b = threadIdx.x; b < n; b += blockDim.x) U.z[b] = 0.0;
  __syncthreads();
  for (int j = threadIdx.x; j < U.ml; j += blockDim.x) {
    const int b = U.dl[j];
    double acc = 0.0;
    for (int q = 0; q < U.ml; ++q) {
      const int qq = U.dl[q];
      acc = fma(U.w[qq], U.D[(long long)qq * n + b], acc);
    }
    U.z[b] = acc;
  }
}
__global__ void __launch_bounds__(256) dom1_reverse(const D1Target* __restrict__ tg, int ntg, long long n) {
  int lo = 0, hi = ntg - 1;  // the target of this tile: the last with tile_begin <= blockIdx.x
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (tg[mid].tile_begin <= (long long)blockIdx.x) lo = mid;
    else hi = mid - 1;
  }
  const D1Target T = tg[lo];
  const int e = (int)(((long long)blockIdx.x - T.tile_begin) * blockDim.x) + threadIdx.x;
  if (e >= T.ml * T.ml) return;
  const int q = T.dl[e / T.ml], b = T.dl[e % T.ml];
  double acc = 0.0;
  for (int t = 0; t < T.rows; ++t) acc = fma(T.w[(long long)t * n + q], T.cg[(long long)t * n + b], acc);
  T.R[(long long)q * n + b] += acc;
}

// Row-panel FP64 GEMM for problems with few rows and long rows of B (the all-external product Y = U W: a
// few dozen gathered CI rows against the np x np operator): C (M x N) = beta C + sum over the segments of
// alpha A B, A M x K and B K x N row major, M <= MT.  A block of 256 threads owns 128 columns of one problem
// (tile_begin counts these column blocks).  B streams through shared memory in PANEL_KS-deep k slices by
// 16-byte cp.async copies, PANEL_STG slices in flight (B is read from HBM exactly once, and enough bytes
// are in flight to cover its latency); A's slices come the same way from L2.  Warp w computes rows
// (w / 2) * MT/4 ... of the columns (w % 2) * 64 + 2 lane, +1: per pair of k a thread reads two 16-byte
// B pairs and MT/4 16-byte A pairs (the same address across the warp) for MT FMAs.  Operands must start
// on 16 bytes with even leading dimensions (checked when the step is lowered).  A segment's alpha scales
// its B values as they are read.  Sums: segments in table order, k ascending.
constexpr int PANEL_T = 256;
constexpr int PANEL_COLS = 128;
constexpr int PANEL_KS = 16;
constexpr int PANEL_STG = 4;


template <int MT>
__global__ void __launch_bounds__(PANEL_T, 2) gemm_panel_f64(const DGemmProblem* __restrict__ probs, int nprob,
                                                             const DGemmSeg* __restrict__ segs) {
  constexpr int R = MT / 4;  // rows per warp
  static_assert(MT % 8 == 0, "MT multiple of 8");
  extern __shared__ __align__(16) double panel_smem[];
  double* Ws = panel_smem;                                   // [PANEL_STG][PANEL_KS][PANEL_COLS]
  double* As = panel_smem + PANEL_STG * PANEL_KS * PANEL_COLS;  // [PANEL_STG][MT][PANEL_KS]
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DGemmProblem P = probs[lo];
  const long long n0 = (tile - P.tile_begin) * PANEL_COLS;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int r0 = (warp >> 1) * R;
  const int col = (warp & 1) * 64 + 2 * lane;  // this thread's two columns n0 + col, + 1
  double acc[R][2];
#pragma unroll
  for (int r = 0; r < R; ++r) acc[r][0] = acc[r][1] = 0.0;
  for (long long sgi = P.seg_begin; sgi < P.seg_end; ++sgi) {
    const DGemmSeg S = segs[sgi];
    const long long K = S.K;
    const long long nsl = (K + PANEL_KS - 1) / PANEL_KS;
    const bool scaled = S.alpha != 1.0;
    // one k slice of B (PANEL_KS x 128) and A (MT x PANEL_KS) into stage st, zero past the edges
    auto issue = [&](long long sl, int st) {
      const long long k0 = sl * PANEL_KS;
      double* w = Ws + (size_t)st * PANEL_KS * PANEL_COLS;
#pragma unroll
      for (int u = 0; u < (PANEL_KS * PANEL_COLS / 2) / PANEL_T; ++u) {
        const int e = tid + u * PANEL_T;               // 16-byte chunk
        const int kk = e / (PANEL_COLS / 2), cc = 2 * (e % (PANEL_COLS / 2));
        const long long gk = k0 + kk, gn = n0 + cc;
        const int bytes = (gk < K && gn < P.N) ? (gn + 1 < P.N ? 16 : 8) : 0;
        cp_async16(w + kk * PANEL_COLS + cc, bytes ? (const void*)(S.B + gk * S.ldb + gn) : (const void*)S.B, bytes);
      }
      double* a = As + (size_t)st * MT * PANEL_KS;
      for (int e = tid; e < MT * PANEL_KS / 2; e += PANEL_T) {
        const int m = e / (PANEL_KS / 2), kk = 2 * (e % (PANEL_KS / 2));
        const long long gk = k0 + kk;
        const int bytes = (m < P.M && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
        cp_async16(a + m * PANEL_KS + kk, bytes ? (const void*)(S.A + m * S.lda + gk) : (const void*)S.A, bytes);
      }
    };
    __syncthreads();  // the previous segment's stages have been read
#pragma unroll
    for (int st = 0; st < PANEL_STG - 1; ++st) {
      if (st < nsl) issue(st, st);
      cp_async_commit();
    }
    for (long long sl = 0; sl < nsl; ++sl) {
      cp_async_wait<PANEL_STG - 2>();  // this thread's copies of slice sl have landed
      __syncthreads();                 // everyone's have, and slice sl - 1 has been read
      if (sl + PANEL_STG - 1 < nsl) issue(sl + PANEL_STG - 1, (int)((sl + PANEL_STG - 1) % PANEL_STG));
      cp_async_commit();
      const int st = (int)(sl % PANEL_STG);
      const double* w = Ws + (size_t)st * PANEL_KS * PANEL_COLS + col;
      const double* a = As + (size_t)st * MT * PANEL_KS + r0 * PANEL_KS;
#pragma unroll
      for (int kp = 0; kp < PANEL_KS / 2; ++kp) {
        double2 w0 = *reinterpret_cast<const double2*>(w + (2 * kp) * PANEL_COLS);
        double2 w1 = *reinterpret_cast<const double2*>(w + (2 * kp + 1) * PANEL_COLS);
        if (scaled) {  // the segment's alpha on B, as gemm_tiled_f64 applies it
          w0.x *= S.alpha, w0.y *= S.alpha, w1.x *= S.alpha, w1.y *= S.alpha;
        }
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const double2 x = *reinterpret_cast<const double2*>(a + r * PANEL_KS + 2 * kp);
          acc[r][0] = fma(x.y, w1.x, fma(x.x, w0.x, acc[r][0]));
          acc[r][1] = fma(x.y, w1.y, fma(x.x, w0.y, acc[r][1]));
        }
      }
    }
    cp_async_wait<0>();
  }
  const long long n = n0 + col;
  if (n >= P.N) return;
#pragma unroll
  for (int r = 0; r < R; ++r) {
    const long long m = r0 + r;
    if (m >= P.M) break;
    double* c = P.C + m * P.ldc + n;
    c[0] = (P.beta == 0.0) ? acc[r][0] : fma(P.beta, c[0], acc[r][0]);
    if (n + 1 < P.N) c[1] = (P.beta == 0.0) ? acc[r][1] : fma(P.beta, c[1], acc[r][1]);
  }
}
template <int MT>
constexpr size_t panel_smem_bytes() {
  return sizeof(double) * (size_t)PANEL_STG * PANEL_KS * (PANEL_COLS + MT);
}

// Tiled FP64 GEMM with the operands staged by cp.async (the problem / segment tables and tile numbering
// of gemm_tiled_f64<64, 128>): 64 x 128 tiles, 16-deep k slices, CP_STG slices in flight, 256 threads with
// 4 x 8 outputs each (rows ty + 16 i, columns tx + 16 j).  A is M x K row major (tA = 0); B is K x N
// (TB = 0, staged [k][n]) or N x K (TB = 1, staged [n][k] with its 16-byte chunks XOR-swizzled by the row
// so that the column reads of a warp spread over the banks).  A segment's alpha scales its B values as
// they are read, as in gemm_tiled_f64; segments in table order, k ascending.  Operands must start on
// 16 bytes with even leading dimensions (checked when the step is lowered).
constexpr int CP_BM = 64, CP_BN = 128, CP_BK = 16, CP_STG = 4;
template <int TB>
constexpr size_t cp_smem_bytes() {
  return sizeof(double) * (size_t)CP_STG * (CP_BM * CP_BK + CP_BK * CP_BN);
}
template <int TB>
__global__ void __launch_bounds__(256, 2) gemm_cp_f64(const DGemmProblem* __restrict__ probs, int nprob,
                                                      const DGemmSeg* __restrict__ segs) {
  extern __shared__ __align__(16) double cp_smem[];
  double* As = cp_smem;                                  // [CP_STG][CP_BM][CP_BK]
  double* Bs = cp_smem + CP_STG * CP_BM * CP_BK;         // [CP_STG][CP_BK][CP_BN] or [CP_STG][CP_BN][CP_BK]
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DGemmProblem P = probs[lo];
  const long long t = tile - P.tile_begin;
  const long long m0 = (t / P.tiles_n) * CP_BM, n0 = (t % P.tiles_n) * CP_BN;
  const int tid = threadIdx.x, tx = tid & 15, ty = tid >> 4;
  double acc[4][8];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 8; ++j) acc[i][j] = 0.0;
  for (long long sgi = P.seg_begin; sgi < P.seg_end; ++sgi) {
    const DGemmSeg S = segs[sgi];
    const long long K = S.K;
    const long long nsl = (K + CP_BK - 1) / CP_BK;
    const double al = S.alpha;
    auto issue = [&](long long sl, int st) {
      const long long k0 = sl * CP_BK;
      double* a = As + (size_t)st * CP_BM * CP_BK;
      double* b = Bs + (size_t)st * CP_BK * CP_BN;
      // A: 64 rows x 8 chunks = 512 chunks, 2 per thread
#pragma unroll
      for (int u = 0; u < 2; ++u) {
        const int e = tid + u * 256;
        const int m = e >> 3, kc = 2 * (e & 7);
        const long long gm = m0 + m, gk = k0 + kc;
        const int bytes = (gm < P.M && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
        cp_async16(a + m * CP_BK + kc, bytes ? (const void*)(S.A + gm * S.lda + gk) : (const void*)S.A, bytes);
      }
      // B: 16 x 128 doubles = 1024 chunks, 4 per thread
#pragma unroll
      for (int u = 0; u < 4; ++u) {
        const int e = tid + u * 256;
        if (TB == 0) {
          const int kk = e >> 6, nc = 2 * (e & 63);
          const long long gk = k0 + kk, gn = n0 + nc;
          const int bytes = (gk < K && gn < P.N) ? (gn + 1 < P.N ? 16 : 8) : 0;
          cp_async16(b + kk * CP_BN + nc, bytes ? (const void*)(S.B + gk * S.ldb + gn) : (const void*)S.B, bytes);
        } else {
          const int nn = e >> 3, c = e & 7;  // row nn of B (a column of op(B)), chunk c of its 16 k
          const long long gn = n0 + nn, gk = k0 + 2 * c;
          const int bytes = (gn < P.N && gk < K) ? (gk + 1 < K ? 16 : 8) : 0;
          cp_async16(b + nn * CP_BK + 2 * (c ^ (nn & 7)), bytes ? (const void*)(S.B + gn * S.ldb + gk) : (const void*)S.B,
                     bytes);
        }
      }
    };
    __syncthreads();  // the previous segment's stages have been read
#pragma unroll
    for (int st = 0; st < CP_STG - 1; ++st) {
      if (st < nsl) issue(st, st);
      cp_async_commit();
    }
    for (long long sl = 0; sl < nsl; ++sl) {
      cp_async_wait<CP_STG - 2>();
      __syncthreads();
      if (sl + CP_STG - 1 < nsl) issue(sl + CP_STG - 1, (int)((sl + CP_STG - 1) % CP_STG));
      cp_async_commit();
      const int st = (int)(sl % CP_STG);
      const double* a = As + (size_t)st * CP_BM * CP_BK;
      const double* b = Bs + (size_t)st * CP_BK * CP_BN;
#pragma unroll
      for (int kp = 0; kp < CP_BK / 2; ++kp) {
        double2 x[4];
#pragma unroll
        for (int i = 0; i < 4; ++i) x[i] = *reinterpret_cast<const double2*>(a + (ty + 16 * i) * CP_BK + 2 * kp);
#pragma unroll
        for (int j = 0; j < 8; ++j) {
          double b0, b1;
          if (TB == 0) {
            b0 = al * b[(2 * kp) * CP_BN + tx + 16 * j];
            b1 = al * b[(2 * kp + 1) * CP_BN + tx + 16 * j];
          } else {
            const int nn = tx + 16 * j;
            const double2 v = *reinterpret_cast<const double2*>(b + nn * CP_BK + 2 * (kp ^ (nn & 7)));
            b0 = al * v.x;
            b1 = al * v.y;
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[i][j] = fma(x[i].y, b1, fma(x[i].x, b0, acc[i][j]));
        }
      }
    }
    cp_async_wait<0>();
  }
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long long gm = m0 + ty + 16 * i;
    if (gm >= P.M) continue;
#pragma unroll
    for (int j = 0; j < 8; ++j) {
      const long long gn = n0 + tx + 16 * j;
      if (gn >= P.N) continue;
      double* c = P.C + gm * P.ldc + gn;
      *c = (P.beta == 0.0) ? acc[i][j] : fma(P.beta, *c, acc[i][j]);
    }
  }
}

// Segmented AXPY: target chunk t (at most AXPY_CHUNK elements) gets
//   dst[i] += sum_s coef_s * scale_s * src_s[base + i].
// One block per chunk; warp w takes the sources w, w + 8, ... in table order,
// and the eight warps' partial sums are added in warp order, so the result is
// independent of timing.  A short target with many sources spreads the
// sources over all threads instead; a target with few sources (a gather or a
// scatter) gives each thread one element and all the sources in order.
constexpr int AXPY_CHUNK = 256;
constexpr int AXPY_DIRECT = 8;  // targets with at most this many sources: one thread per element
// PAIRS: two sources per pass in the general path (steps whose targets have many sources; more registers).
template <bool PAIRS>
__global__ void __launch_bounds__(256, PAIRS ? 4 : 0) axpy_segments(const DAxpyTarget* __restrict__ tg, long long ntg,
                                                     const DAxpySource* __restrict__ src) {
  __shared__ double part[8][AXPY_CHUNK];
  const long long t = blockIdx.x;
  if (t >= ntg) return;
  const DAxpyTarget T = tg[t];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (T.src_end - T.src_begin <= AXPY_DIRECT) {
    // few sources (gathers, scatters): a thread per element sums every source in table order
    for (long long i = threadIdx.x; i < T.len; i += blockDim.x) {
      double acc = 0.0;
      for (long long s = T.src_begin; s < T.src_end; ++s) {
        const DAxpySource S = src[s];
        const double c = S.scale ? S.coef * (*S.scale) : S.coef;
        acc = fma(c, S.src[T.base + i], acc);
      }
      T.dst[i] += acc;
    }
    return;
  }
  if (T.len < 8 && T.src_end - T.src_begin > 64) {
    for (long long i = 0; i < T.len; ++i) {
      double acc = 0.0;
      for (long long s = T.src_begin + threadIdx.x; s < T.src_end; s += 256) {
        const DAxpySource S = src[s];
        const double c = S.scale ? S.coef * (*S.scale) : S.coef;
        acc = fma(c, S.src[T.base + i], acc);
      }
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
      if (lane == 0) part[warp][0] = acc;
      __syncthreads();
      if (threadIdx.x == 0) {
        double v = 0.0;
        for (int w = 0; w < 8; ++w) v += part[w][0];
        T.dst[i] += v;
      }
      __syncthreads();
    }
    return;
  }
  double acc[AXPY_CHUNK / 32];
#pragma unroll
  for (int e = 0; e < AXPY_CHUNK / 32; ++e) acc[e] = 0.0;
  long long s = T.src_begin + warp;
  // two sources per pass: both rows' loads are in flight before the first product (same order of fmas)
  if constexpr (PAIRS) for (; s + 8 < T.src_end; s += 16) {
    const DAxpySource S0 = src[s], S1 = src[s + 8];
    const double c0 = S0.scale ? S0.coef * (*S0.scale) : S0.coef;
    const double c1 = S1.scale ? S1.coef * (*S1.scale) : S1.coef;
    const double* x0 = S0.src + T.base;
    const double* x1 = S1.src + T.base;
    double v0[AXPY_CHUNK / 32], v1[AXPY_CHUNK / 32];
#pragma unroll
    for (int e = 0; e < AXPY_CHUNK / 32; ++e) {
      const long long i = lane + 32 * e;
      v0[e] = i < T.len ? x0[i] : 0.0;
      v1[e] = i < T.len ? x1[i] : 0.0;
    }
#pragma unroll
    for (int e = 0; e < AXPY_CHUNK / 32; ++e) {
      const long long i = lane + 32 * e;
      if (i < T.len) {
        acc[e] = fma(c0, v0[e], acc[e]);
        acc[e] = fma(c1, v1[e], acc[e]);
      }
    }
  }
  for (long long r = s; r < T.src_end; r += 8) {
    const DAxpySource S = src[r];
    const double c = S.scale ? S.coef * (*S.scale) : S.coef;
    const double* x = S.src + T.base;
#pragma unroll
    for (int e = 0; e < AXPY_CHUNK / 32; ++e) {
      const long long i = lane + 32 * e;
      if (i < T.len) acc[e] = fma(c, x[i], acc[e]);
    }
  }
#pragma unroll
  for (int e = 0; e < AXPY_CHUNK / 32; ++e) part[warp][lane + 32 * e] = acc[e];
  __syncthreads();
  if (threadIdx.x < T.len) {
    double v = 0.0;
#pragma unroll
    for (int w = 0; w < 8; ++w) v += part[w][threadIdx.x];
    T.dst[threadIdx.x] += v;
  }
}

// Segmented dot products: *dst += sum_s coef_s (a_s . b_s).  One block per
// target; warp w takes the sources w, w + 8, ... and reduces across its lanes
// once; fixed-order reductions.
__global__ void __launch_bounds__(256) dot_segments(const DDotTarget* __restrict__ tg, long long ntg,
                                                    const DDotSource* __restrict__ src) {
  __shared__ double part[8];
  const long long t = blockIdx.x;
  if (t >= ntg) return;
  const DDotTarget T = tg[t];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  // each lane keeps sum_s coef_s sum_{its i} a_s[i] b_s[i] over the warp's sources; one reduction at the end
  double total = 0.0;
  long long s = T.src_begin + warp;
  // short rows (up to 256 elements, 16-byte aligned, even length), two sources per pass: every load of both
  // is issued before the first product; the fmas keep the order of the general loop below
  for (; s + 8 < T.src_end; s += 16) {
    const DDotSource S0 = src[s], S1 = src[s + 8];
    const bool fast = ((reinterpret_cast<uintptr_t>(S0.a) | reinterpret_cast<uintptr_t>(S0.b) |
                        reinterpret_cast<uintptr_t>(S1.a) | reinterpret_cast<uintptr_t>(S1.b)) & 15) == 0 &&
                      ((S0.len | S1.len) & 1) == 0 && S0.len <= 256 && S1.len <= 256;
    if (!fast) break;
    const double2* a0 = reinterpret_cast<const double2*>(S0.a);
    const double2* b0 = reinterpret_cast<const double2*>(S0.b);
    const double2* a1 = reinterpret_cast<const double2*>(S1.a);
    const double2* b1 = reinterpret_cast<const double2*>(S1.b);
    const long long h0 = S0.len / 2, h1 = S1.len / 2;
    double2 x0[4], y0[4], x1[4], y1[4];
#pragma unroll
    for (int e = 0; e < 4; ++e) {
      const long long i = lane + 32 * e;
      const double2 z = make_double2(0.0, 0.0);
      x0[e] = i < h0 ? __ldg(a0 + i) : z;
      y0[e] = i < h0 ? __ldg(b0 + i) : z;
      x1[e] = i < h1 ? __ldg(a1 + i) : z;
      y1[e] = i < h1 ? __ldg(b1 + i) : z;
    }
    double acc0 = 0.0, acc1 = 0.0;
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (lane + 32 * e < h0) {
        acc0 = fma(x0[e].x, y0[e].x, acc0);
        acc0 = fma(x0[e].y, y0[e].y, acc0);
      }
#pragma unroll
    for (int e = 0; e < 4; ++e)
      if (lane + 32 * e < h1) {
        acc1 = fma(x1[e].x, y1[e].x, acc1);
        acc1 = fma(x1[e].y, y1[e].y, acc1);
      }
    total = fma(S0.coef, acc0, total);
    total = fma(S1.coef, acc1, total);
  }
  for (; s < T.src_end; s += 8) {
    const DDotSource S = src[s];
    double acc = 0.0;
    if (((reinterpret_cast<uintptr_t>(S.a) | reinterpret_cast<uintptr_t>(S.b)) & 15) == 0 && (S.len & 1) == 0) {
      const double2* a2 = reinterpret_cast<const double2*>(S.a);
      const double2* b2 = reinterpret_cast<const double2*>(S.b);
      for (long long i = lane; i < S.len / 2; i += 32) {
        const double2 x = __ldg(a2 + i), y = __ldg(b2 + i);
        acc = fma(x.x, y.x, acc);
        acc = fma(x.y, y.y, acc);
      }
    } else {
      for (long long i = lane; i < S.len; i += 32) acc = fma(__ldg(S.a + i), __ldg(S.b + i), acc);
    }
    total = fma(S.coef, acc, total);
  }
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) total += __shfl_xor_sync(0xffffffffu, total, o);
  if (lane == 0) part[warp] = total;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < 8; ++w) v += part[w];
    *T.dst += v;
  }
}

__global__ void unpack_pairs(const DHead* __restrict__ heads, const int* __restrict__ dk_head, long long nD, long long n,
                             const double* __restrict__ c, double* __restrict__ D) {
  const long long dk = blockIdx.y;
  if (dk >= nD) return;
  const DHead H = heads[dk_head[dk]];
  const long long k = dk - H.dk0;
  const double p = (k < H.nsing) ? 1.0 : -1.0;
  const long long nab = n * (n - 1) / 2;
  double* Dk = D + dk * n * n;
  const bool ab = k < H.nsf_ab, aa = k < H.nsf_aa;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < n * n; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / n, s = e % n;
    double v = 0.0;
    if (r == s) {
      if (aa) v = 1.4142135623730951 * c[H.off_aa + k * n + r];
    } else if (ab) {
      const long long i = r > s ? r : s, j = r > s ? s : r;
      const double x = c[H.off_ab + k * nab + i * (i - 1) / 2 + j];
      v = (r < s) ? x : p * x;
    }
    Dk[e] = v;
  }
}

// sigma_ab[k][i(i-1)/2+j] += R(j,i) + p R(i,j); sigma_aa[k][a] += sqrt2 R(a,a)
__global__ void pack_pairs(const DHead* __restrict__ heads, const int* __restrict__ dk_head, long long nD, long long n,
                           const double* __restrict__ R, double* __restrict__ sigma) {
  const long long dk = blockIdx.y;
  if (dk >= nD) return;
  const DHead H = heads[dk_head[dk]];
  const long long k = dk - H.dk0;
  const double p = (k < H.nsing) ? 1.0 : -1.0;
  const long long nab = n * (n - 1) / 2;
  const double* Rk = R + dk * n * n;
  if (k < H.nsf_ab) {
    for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < nab; e += (long long)gridDim.x * blockDim.x) {
      // invert e = i(i-1)/2 + j, i > j >= 0
      long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
      while (i * (i - 1) / 2 > e) --i;
      while ((i + 1) * i / 2 <= e) ++i;
      const long long j = e - i * (i - 1) / 2;
      sigma[H.off_ab + k * nab + e] += Rk[j * n + i] + p * Rk[i * n + j];
    }
  }
  if (k < H.nsf_aa) {
    for (long long a = (long long)blockIdx.x * blockDim.x + threadIdx.x; a < n; a += (long long)gridDim.x * blockDim.x)
      sigma[H.off_aa + k * n + a] += 1.4142135623730951 * Rk[a * n + a];
  }
}

__global__ void accumulate_f64(double* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

__device__ __forceinline__ long long pk(long long a, long long b) {
  return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a;
}

// W+ (np x np, rows [aa (n); ab a>b]) and W- (nm x nm) from X[(ab)][(cd)] = (ab|cd)
// x = a(a-1)/2 + b with a > b (the reference's pair order idx = a(a-1)/2 + b)
__device__ __forceinline__ void unpair_idx(long long x, long long& a, long long& b) {
  long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)x)) * 0.5);
  while (i * (i - 1) / 2 > x) --i;
  while ((i + 1) * i / 2 <= x) ++i;
  a = i;
  b = x - i * (i - 1) / 2;
}

// One W row per block iteration (W+ rows, then W- rows), the threads along its columns.  The column pair
// (b, d), d the fast index, lands in X's column index in both terms (X = Lpk Lpk^T is symmetric, so the
// exchange term is read as X[(c b)][(a d)]): consecutive columns read consecutive X words for d <= c, a.
__global__ void build_allext(const double* __restrict__ X, long long n, double* __restrict__ W) {
  const long long nab = n * (n - 1) / 2, np = n + nab, nm = nab, npk = n * (n + 1) / 2;
  for (long long row = blockIdx.x; row < np + nm; row += gridDim.x) {
    const bool plus = row < np;
    const long long r = plus ? row : row - np, ncol = plus ? np : nm;
    double* __restrict__ w = W + (plus ? r * np : np * np + r * nm);
    long long a, cc;
    const bool rd = plus && r < n;
    if (rd) {
      a = r;
      cc = r;
    } else {
      unpair_idx(plus ? r - n : r, a, cc);
    }
    for (long long c = threadIdx.x; c < ncol; c += blockDim.x) {
      const bool cd = plus && c < n;
      long long b, d;
      if (cd) {
        b = c;
        d = c;
      } else {
        unpair_idx(plus ? c - n : c, b, d);
      }
      double v;
      if (plus) {
        if (rd && cd) v = X[pk(a, b) * npk + pk(a, b)];
        else if (rd) v = 1.4142135623730951 * X[pk(a, b) * npk + pk(a, d)];
        else if (cd) v = 1.4142135623730951 * X[pk(a, b) * npk + pk(cc, b)];
        else v = X[pk(a, b) * npk + pk(cc, d)] + X[pk(cc, b) * npk + pk(a, d)];
      } else {
        v = X[pk(a, b) * npk + pk(cc, d)] - X[pk(cc, b) * npk + pk(a, d)];
      }
      w[c] = v;
    }
  }
}


// ----------------------------------------------------------------------------
// diagonal H_ii from the plan's diagonal entries (plan.h DiagEntry)
struct DDiag {
  long long off, len, type;
  double beta;
  long long foff, singlet;
};

// All-external part of the diagonal from W (its diagonal elements), or, when the plan has no W (local pair
// domains), from XD = [(aa|cc); (ac|ca)] (two n x n arrays): W+((ac),(ac)) = (aa|cc) + (ac|ca),
// W-((ac),(ac)) = (aa|cc) - (ac|ca), W+((aa),(aa)) = (aa|aa).
__global__ void build_diag_kernel(const DDiag* __restrict__ ent, long long nent, long long n, long long np, long long nm,
                                  const double* __restrict__ F, const double* __restrict__ W,
                                  const double* __restrict__ XD, double* __restrict__ hd) {
  const long long e = blockIdx.x;
  if (e >= nent) return;
  const DDiag D = ent[e];
  for (long long t = threadIdx.x; t < D.len; t += blockDim.x) {
    double v = D.beta;
    if (D.type == 1) {
      if (D.foff >= 0) v += F[D.foff + t * (n + 1)];
    } else if (D.type == 2) {
      if (D.foff >= 0) v += 2.0 * F[D.foff + t * (n + 1)];
      v += W ? W[t * np + t] : XD[t * n + t];
    } else if (D.type == 3) {
      long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)t)) * 0.5);
      while (i * (i - 1) / 2 > t) --i;
      while ((i + 1) * i / 2 <= t) ++i;
      const long long j = t - i * (i - 1) / 2;
      if (D.foff >= 0) v += F[D.foff + i * (n + 1)] + F[D.foff + j * (n + 1)];
      if (W) v += D.singlet ? W[(n + t) * np + (n + t)] : W[np * np + t * nm + t];
      else v += XD[i * n + j] + (D.singlet ? 1.0 : -1.0) * XD[n * n + i * n + j];
    }
    hd[D.off + t] = v;
  }
}

// Local pair domains: the CI vector in the local layout (n_loc CSFs) and the plan's vectors in the non-local
// layout; map[i] is the non-local index of local CSF i (an injection: every block padded to all externals).
__global__ void scatter_local(const double* __restrict__ c_loc, const long long* __restrict__ map, long long n_loc,
                              double* __restrict__ c_nl) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_loc; i += (long long)gridDim.x * blockDim.x)
    c_nl[map[i]] = c_loc[i];
}
__global__ void gather_local(const double* __restrict__ s_nl, const long long* __restrict__ map, long long n_loc,
                             double* __restrict__ s_loc) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n_loc; i += (long long)gridDim.x * blockDim.x)
    s_loc[i] = s_nl[map[i]];
}

// Davidson vector kernels (FP64, deterministic two-pass reductions)
constexpr int RB = 256;     // threads per reduction block
constexpr int RBLK = 592;   // reduction blocks (4 x 148 SMs)
// default Davidson subspace budget: the reference's DAVIDSON HARD DRIVE SPACE default of 30 GB
constexpr double kDefaultSubspaceBytes = 30e9;
// Several contexts may live in one process, driven from different host threads
// (the request server).  A graph capture on one thread and a cudaFree (which
// synchronises the device) on another are kept apart by this lock.
std::mutex g_capture_free_mu;

// Device memory of the sigma contexts comes from one stream-ordered pool per device that keeps the pages
// it has mapped (release threshold unlimited): a context set up after another one was destroyed (the
// request server, repeated set-ups in one process) reuses them instead of mapping new memory, which made
// set-up and tear-down times vary by hundreds of milliseconds.  Allocations and frees are ordered on the
// context's stream.
cudaError_t dev_malloc_v(void** p, size_t bytes, cudaStream_t st) {
  static std::mutex mu;
  static cudaMemPool_t pools[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= 64) return cudaMallocAsync(p, bytes, st);
  cudaMemPool_t pool = nullptr;
  {
    std::lock_guard<std::mutex> lk(mu);
    if (!pools[dev]) {
      cudaMemPoolProps props = {};
      props.allocType = cudaMemAllocationTypePinned;
      props.location.type = cudaMemLocationTypeDevice;
      props.location.id = dev;
      e = cudaMemPoolCreate(&pools[dev], &props);
      if (e != cudaSuccess) {
        pools[dev] = nullptr;
        return e;
      }
      uint64_t keep = UINT64_MAX;
      e = cudaMemPoolSetAttribute(pools[dev], cudaMemPoolAttrReleaseThreshold, &keep);
      if (e != cudaSuccess) return e;
    }
    pool = pools[dev];
  }
  return cudaMallocFromPoolAsync(p, bytes, pool, st);
}
template <class T>
cudaError_t dev_malloc(T** p, size_t bytes, cudaStream_t st) {
  return dev_malloc_v(reinterpret_cast<void**>(p), bytes, st);
}
inline cudaError_t dev_free(void* p, cudaStream_t st) { return p ? cudaFreeAsync(p, st) : cudaSuccess; }

// partial[k * RBLK + b] = sum over block b's chunk of A[k][i] * x[i].  Four rows per pass share the loads
// of x (each row's products are still summed in the order of the one-row loop).
__global__ void __launch_bounds__(RB) multi_dot_partial(const double* __restrict__ A, long long lda, int m,
                                                        const double* __restrict__ x, long long n,
                                                        double* __restrict__ partial) {
  __shared__ double red[4][RB / 32];
  const long long chunk = (n + gridDim.x - 1) / gridDim.x;
  const long long i0 = (long long)blockIdx.x * chunk, i1 = min(n, i0 + chunk);
  for (int k0 = 0; k0 < m; k0 += 4) {
    const int nk = min(4, m - k0);
    const double* a0 = A + (long long)k0 * lda;
    const double* a1 = nk > 1 ? a0 + lda : a0;
    const double* a2 = nk > 2 ? a0 + 2 * lda : a0;
    const double* a3 = nk > 3 ? a0 + 3 * lda : a0;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (long long i = i0 + threadIdx.x; i < i1; i += RB) {
      const double xi = x[i];
      acc[0] = fma(a0[i], xi, acc[0]);
      acc[1] = fma(a1[i], xi, acc[1]);
      acc[2] = fma(a2[i], xi, acc[2]);
      acc[3] = fma(a3[i], xi, acc[3]);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
#pragma unroll
      for (int o = 16; o > 0; o >>= 1) acc[q] += __shfl_xor_sync(0xffffffffu, acc[q], o);
      if ((threadIdx.x & 31) == 0) red[q][threadIdx.x >> 5] = acc[q];
    }
    __syncthreads();
    if (threadIdx.x < nk) {
      double t = 0.0;
      for (int w = 0; w < RB / 32; ++w) t += red[threadIdx.x][w];
      partial[(long long)(k0 + threadIdx.x) * gridDim.x + blockIdx.x] = t;
    }
    __syncthreads();
  }
}

__global__ void multi_dot_final(const double* __restrict__ partial, int m, int nblk, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double t = 0.0;
  for (int b = 0; b < nblk; ++b) t += partial[(long long)k * nblk + b];
  out[k] = t;
}

// out[k] = -(sum of the partials of k): the coefficients of one classical Gram-Schmidt pass
__global__ void multi_dot_final_neg(const double* __restrict__ partial, int m, int nblk, double* __restrict__ out) {
  const int k = blockIdx.x * blockDim.x + threadIdx.x;
  if (k >= m) return;
  double t = 0.0;
  for (int b = 0; b < nblk; ++b) t += partial[(long long)k * nblk + b];
  out[k] = -t;
}

// out[i] = beta*out[i] + sum_k ca[k] A[k][i] + sum_k cb[k] B[k][i]
__global__ void lincomb_kernel(double* __restrict__ out, double beta, const double* __restrict__ A,
                               const double* __restrict__ ca, const double* __restrict__ B,
                               const double* __restrict__ cb, int m, long long lda, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    double v = (beta == 0.0) ? 0.0 : beta * out[i];
    for (int k = 0; k < m; ++k) {
      if (A) v = fma(ca[k], A[(long long)k * lda + i], v);
      if (B) v = fma(cb[k], B[(long long)k * lda + i], v);
    }
    out[i] = v;
  }
}

// r_i <- -r_i / (hd_i - E), 0 where hd_i == E (davidson.f90:609-631)
__global__ void precondition_kernel(double* __restrict__ r, const double* __restrict__ hd, double E, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const double p = hd[i] - E;
    r[i] = (p == 0.0) ? 0.0 : -r[i] / p;
  }
}

// Generalized (ACPF-type) solves run on G^-1/2 (H - shift) G^-1/2: x <- s x with s = G^-1/2 before the sigma
// build, out = s (H x - shift x) after it, and the diagonal s^2 (H_ii - shift).
__global__ void scale_by(double* __restrict__ x, const double* __restrict__ s, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    x[i] *= s[i];
}
__global__ void gen_sigma_out(double* __restrict__ out, const double* __restrict__ hx, const double* __restrict__ x,
                              const double* __restrict__ s, double shift, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = s[i] * (hx[i] - shift * x[i]);
}
__global__ void gen_diag(double* __restrict__ out, const double* __restrict__ hd, const double* __restrict__ s,
                         double shift, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = s[i] * s[i] * (hd[i] - shift);
}

// r scaled by 1/|r| (or zeroed when |r| < 1e-14)
__global__ void normalize_kernel(double* __restrict__ r, const double* __restrict__ nrm2, long long n) {
  const double nr = sqrt(*nrm2);
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    r[i] = (fabs(nr) < 1e-14) ? 0.0 : r[i] / nr;
}
// ----------------------------------------------------------------------------
struct DevStep {
  int kind = 0;
  std::string name;
  // GEMM
  DGemmProblem* probs = nullptr;
  DGemmSeg* segs = nullptr;
  int nprob = 0;
  long long ntiles = 0;
  int cfg = 0;  // 0: 64x128 tiles, 1: 128x64 tiles
  // the same problems tiled for the tensor-core kernel (mixed-precision form)
  DGemmProblem* probs_tc = nullptr;
  DGemmSeg* segs_tc = nullptr;
  long long ntiles_tc = 0;
  int nprob_tc = 0;
  // two-external step on the TMA-fed kernel (integrals x pair matrices); tables when the step qualifies
  TmaProblem* tma_probs = nullptr;
  TmaSeg* tma_segs = nullptr;
  int tma_nprob = 0;
  long long tma_ntiles = 0;
  // 1: two-external (integrals x pair matrices), 2: forward three-external (V_i x pair rows), 3: reverse
  // three-external (transposed V_i rows x gathered coefficient rows), 4: singles-singles two-external
  // (integral rows x gathered single-vector rows, computed transposed), 5: forward one-external
  // (coupling-vector rows x pair matrices), 6: dv forward (exchange-bank rows x pair-matrix rows), 7: dv
  // reverse (transposed exchange-bank rows x transposed gathered rows, transposed output)
  int tma_kind = 0;
  long long tma_aux = 0;   // kinds 3, 4: offset of the gathered coefficients in BUF_T0
  long long tma_rows = 0;  // kinds 4, 6, 7: rows of the gathered coefficients / of the exchange bank
  long long tma_aux2 = 0;  // kind 7: offset of the exchange bank in BUF_JK
  // FP64 form: problems with at most SKINNY_M rows and B given as N x K run on the skinny kernel
  // FP64 problems on the cp.async-staged tiled kernel, by orientation of B
  DGemmProblem* cp_probs[2] = {};
  int cp_nprob[2] = {};
  long long cp_ntiles[2] = {};
  // FP64 problems of few rows on the row-panel kernel, by row class (M <= 16, 24, ..., 64)
  DGemmProblem* panel_probs[7] = {};
  int panel_nprob[7] = {};
  long long panel_ntiles[7] = {};
  DGemmProblem* skinny_probs = nullptr;
  int skinny_nprob = 0;
  long long skinny_nwarps = 0;
  DGemmProblem* probs_f = nullptr;  // its FP64 part (same-head one-electron-like segments)
  DGemmSeg* segs_f = nullptr;
  long long ntiles_f = 0;
  int nprob_f = 0;
  bool tc_ok = false;  // worth the tensor cores: enough work and tiles mostly full
  // local decks: the two-external step on the heads' domains and common columns (gemm_com_f64)
  DComProblem* com_probs = nullptr;
  DComSeg* com_segs = nullptr;
  int com_nprob = 0;
  long long com_ntiles = 0;
  DComPack* com_pack = nullptr;  // compaction of its constant operands, run once after the set-up steps
  long long com_njobs = 0;
  DComSq* com_gather = nullptr;   // pair matrices -> compact squares
  long long com_ngather = 0;
  DComSq* com_scatter = nullptr;  // compact accumulators -> padded ones
  long long com_nscatter = 0;
  double* com_rsq = nullptr;      // the compact accumulators (zeroed per build)
  long long com_rsq_len = 0;
  bool com_step = false;
  // local decks: the zero-external rows of N-2 and N-1 heads on the common positions (axpy_common)
  ZcTarget* zc_tg = nullptr;
  ZcSource* zc_src = nullptr;
  long long zc_ntg = 0;
  // local decks: the three-external term on the domains (dom3_forward in place of the split-k sum,
  // dom3_reverse in place of the reverse GEMM); d3_skip marks a padded forward GEMM that a domain kernel
  // replaces (three-external or N-2 <-> valence)
  bool d3_skip = false;
  int d3 = 0;  // 1: dom3_forward, 2: dom3_reverse
  D3Fwd* d3f = nullptr;
  long long d3f_n = 0;
  size_t d3f_smem = 0;
  D3Rev* d3r = nullptr;
  D3RevEntry* d3e = nullptr;
  int d3r_n = 0;
  long long d3r_tiles = 0;
  double* d3_rows = nullptr;  // forward: Y (output); reverse: U (input)
  // local decks: the N-2 <-> valence term on the domains (dom_dv_forward in place of the split-k sum,
  // dom_dv_reverse in place of the reverse GEMM; the padded forward GEMM marked d3_skip)
  int d1 = 0;  // local decks, one-external term on the domains: 1 dom1_forward, 2 dom1_reverse
  D1Row* d1_rows = nullptr;
  long long d1_nrows = 0;
  D1Target* d1_tg = nullptr;
  int d1_ntg = 0;
  long long d1_tiles = 0;
  int dv = 0;  // 1: forward, 2: reverse
  DvEntry* dv_ent = nullptr;
  long long dv_nent = 0;
  DvTarget* dv_tg = nullptr;
  long long* dv_pq = nullptr;
  int dv_ntg = 0;
  long long dv_tiles = 0;
  double* dv_vals = nullptr;  // forward: F (output); reverse: G (input)
  double* dv_k = nullptr;     // the exchange bank
  // AXPY / DOT
  DAxpyTarget* at = nullptr;
  DAxpySource* as = nullptr;
  DDotTarget* dt = nullptr;
  DDotSource* ds = nullptr;
  long long ntg = 0;
  bool axpy_pairs = false;  // targets with many sources on average: the two-sources-per-pass kernel
  // ZERO
  double* zptr = nullptr;
  long long zlen = 0;
};

// Device copy of a host table, ordered on `st` before the kernels that read it.
// (A plain cudaMemcpy from pageable memory may return before its DMA lands, and
// runs on the legacy stream, which a non-blocking stream does not wait for.)
template <class T>
T* upload(const std::vector<T>& v, std::vector<void*>& owned, cudaStream_t st) {
  if (v.empty()) return nullptr;
  T* d = nullptr;
  TCI_CUDA(dev_malloc(&d, v.size() * sizeof(T), st));
  owned.push_back(d);
  TCI_CUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, st));
  return d;
}

}  // namespace

struct tci_ctx {
  int device = 0;
  cudaStream_t stream = nullptr;
  CsfSpace sp;
  Plan plan;
  double* buf[NUM_BUFS] = {};
  std::vector<void*> owned;  // table allocations
  std::vector<DevStep> init, sigma;
  DHead* dheads = nullptr;
  int* dk_head = nullptr;
  double bytes_held = 0;
  double init_seconds = 0;
  // set-up started from the operator part of the plan before the whole plan existed (ctx_begin_operator):
  // the leading set-up steps already run, and their names and table sizes for the check against the plan
  size_t early_init = 0;
  std::vector<std::string> early_names;
  std::vector<std::array<size_t, 4>> early_shapes;
  std::vector<i64> early_sizes;
  bool wv_uploaded = false;  // the coupling-vector rows went up while the host built the rest of the plan
  double last_sigma_ms = 0;
  long long sigma_count = 0;
  cudaEvent_t ev0 = nullptr, ev1 = nullptr;
  bool profiling = false;
  bool use_graph = true;                // replay the sigma steps as one CUDA graph
  int64_t precision = 0;                // 0 plain FP64; 1 all-external on tcgen05 (3xTF32, FP64 promotion)
  int64_t tc_kblock = 128;              // k elements per FP64 promotion block of the tensor-core product
  int64_t tc_mode = 0;                  // precision 1: other GEMM steps on the tensor cores by size (0), all (1), none (2)
  // precision 1: roots finished as FP64 Rayleigh quotients: 1 with a plain-FP64 sigma build (keeps the FP64 W),
  // 2 with every term FP64 but the all-external one, which stays on its tensor-core kernel (no FP64 W kept)
  int64_t refine = 2;
  bool allext_tc_in_fp64 = false;       // set during a refine-2 finish build
  // mixed form with an FP64 finish: the same-head one-electron-like products of the dd step run on the
  // tensor cores as well (the finish's FP64 sigma build carries them in FP64 for the reported roots)
  bool f_on_tc = false;
  // split operands of the TMA-fed steps: integrals and V_i once, the pair matrices every build
  float *jk_hi = nullptr, *jk_lo = nullptr, *d_hi = nullptr, *d_lo = nullptr;
  float *v_hi = nullptr, *v_lo = nullptr, *df_hi = nullptr, *df_lo = nullptr;
  float *vt_hi = nullptr, *vt_lo = nullptr, *u3_hi = nullptr, *u3_lo = nullptr;  // reverse three-external
  float *cg_hi = nullptr, *cg_lo = nullptr;                                        // singles-singles
  float *wv_hi = nullptr, *wv_lo = nullptr;                                        // one-external vectors
  float *kb_hi = nullptr, *kb_lo = nullptr;                                        // dv exchange bank
  float *kbt_hi = nullptr, *kbt_lo = nullptr, *g2t_hi = nullptr, *g2t_lo = nullptr;  // dv reverse
  tci_gtma_host::TmaMaps tma_dd, tma_t3, tma_t3r, tma_ss, tma_1x, tma_dv, tma_dvr;
  bool tma_dd_ready = false, tma_t3_ready = false, tma_t3r_ready = false, tma_ss_ready = false, tma_1x_ready = false,
       tma_dv_ready = false, tma_dvr_ready = false;
  float* w32p = nullptr;                // FP32 W+ / W- (precision 1)
  float* w32m = nullptr;
  float* u2s = nullptr;                 // split singlet CI blocks for the tensor-core product
  float* u2t = nullptr;                 // split triplet CI blocks
  int* tc_status = nullptr;
  tci_tc_host::AllextTc tc_sing, tc_trip;
  cudaGraph_t graph = nullptr, graph_prof = nullptr;
  cudaGraphExec_t graph_exec = nullptr, graph_exec_prof = nullptr;  // plain / with per-step event nodes
  double* hd = nullptr;          // diagonal H_ii (device), built on first use
  // Local pair domains (a deck with allowed-virtual lists): the CI vectors of the calls have the local layout
  // (n_loc CSFs); the plan runs on the non-local space of the same deck with every block padded to all
  // externals (zeros outside the domains): sigma = P^T H P c with P the padding, exact for every term, since
  // H restricted to the local space is P^T H P.  The all-external term runs on the local layout directly,
  // in the pair-domain Cholesky form (tci_local); the plan leaves it out.
  bool local = false;
  i64 n_loc = 0;
  long long* d_map = nullptr;    // local CSF -> non-local CSF (device)
  tci_local* loc_allext = nullptr;
  double* xdiag = nullptr;       // (aa|cc) and (ac|ca), n x n each: the all-external diagonal without W
  double *loc_c = nullptr, *loc_s = nullptr;  // local-layout scratch vectors of the sigma entry points
  i64 nvec() const { return local ? n_loc : plan.total_csfs; }
  // generalized solve (tci_davidson_gen): sigma and the diagonal of G^-1/2 (H - gen_shift) G^-1/2
  const double* gen_s = nullptr;  // G^-1/2 (device) while such a solve runs, else nullptr
  const double* gen_g = nullptr;  // G (device) in such a solve: the residual norm is taken in the metric of c
  double gen_shift = 0.0;
  bool gen_follow = false;        // root following in such a solve (root_following, davidson.f90:732)
  bool acpf_root_follow = true;   // the reference's default (its keyword NO ACPF ROOT FOLLOW clears it)
  bool last_converged = false;    // the last Davidson solve met its tolerances for every root
  std::vector<i64> lowest_diag;  // CSF indices of the lowest diagonal elements, ascending (initial guesses)
  double* dots = nullptr;        // reduction scratch: partial sums and results
  double* coefs = nullptr;       // small device coefficient arrays
  int scratch_cap = 0;           // vectors dots / coefs are sized for
  double* dotbuf = nullptr;      // tci_dots reduction scratch
  int64_t dotbuf_cap = 0;        // doubles
  std::vector<cudaEvent_t> step_ev;     // 2 per sigma step
  std::vector<double> step_ms;          // accumulated per sigma step
  long long profiled_builds = 0;
  long long launch_count = 0;    // kernels this context has launched (sigma builds, Davidson, projections)
  bool dav_phases = false;       // time the Davidson phases (stream synchronised at each boundary)
  // Davidson vectors, kept between solves (reallocated only when a solve needs more)
  double *dav_c = nullptr, *dav_hc = nullptr, *dav_r = nullptr, *dav_tc = nullptr, *dav_th = nullptr;
  int64_t dav_cap = 0, dav_keep = 0;
  double dav_ms[8] = {};         // setup, sigma, projection, subspace eigensolve, residual,
                                 // preconditioner + Gram-Schmidt, restart, finish

  ~tci_ctx() {
    if (loc_allext) tci_local_destroy(loc_allext);
    if (graph_exec) cudaGraphExecDestroy(graph_exec);
    if (graph) cudaGraphDestroy(graph);
    if (graph_exec_prof) cudaGraphExecDestroy(graph_exec_prof);
    if (graph_prof) cudaGraphDestroy(graph_prof);
    for (auto e : step_ev) cudaEventDestroy(e);
    if (device >= 0) cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    std::lock_guard<std::mutex> lk(g_capture_free_mu);
    dev_free(dotbuf, stream);
    for (double* p : {dav_c, dav_hc, dav_r, dav_tc, dav_th}) dev_free(p, stream);
    for (int b = 0; b < NUM_BUFS; ++b) dev_free(buf[b], stream);
    for (void* p : owned) dev_free(p, stream);
    if (stream) cudaStreamSynchronize(stream);
    if (ev0) cudaEventDestroy(ev0);
    if (ev1) cudaEventDestroy(ev1);
    if (stream) cudaStreamDestroy(stream);
  }

  double* ptr(int b, i64 off) {
    if (b < 0 || b >= NUM_BUFS || !buf[b]) throw Error(TCI_ERR_INTERNAL, "plan references an unallocated buffer");
    if (off < 0 || off > plan.buf_size[b]) throw Error(TCI_ERR_INTERNAL, "plan offset outside its buffer");
    return buf[b] + off;
  }

  // Tables of the TMA-fed kernel for the two-external step (every tensor-core segment an n x n integral
  // matrix of BUF_JK times an n x n pair matrix of BUF_D) and the forward three-external step (pair-matrix
  // rows times V_i rows, computed transposed); a step that does not fit keeps the producer-fed kernel.
  void lower_tma(const Step& s, DevStep& d, const std::vector<DGemmProblem>& pr) {
    const i64 n = plan.n, n2 = n * n;
    const i64 TM = tci_gtma_host::tile_m();
    i64 TN = tci_gtma_host::tile_n(true);
    std::vector<TmaProblem> tp;
    std::vector<TmaSeg> ts;
    long long tiles = 0;
    auto push = [&](TmaProblem q) {
      q.tiles_n = (q.N + TN - 1) / TN;
      q.tile_begin = tiles;
      tiles += ((q.M + TM - 1) / TM) * q.tiles_n;
      tp.push_back(q);
    };
    size_t gi = 0;
    if (s.name == "dd two-external") {
      TN = tci_gtma_host::tile_n(tma_wide(1));
      std::vector<double> psign((size_t)std::max<i64>(plan.nD, 1), 1.0);
      for (const auto& h : plan.dheads)
        for (i64 k = 0; k < h.nD; ++k) psign[(size_t)(h.dk0 + k)] = k < h.nsing ? 1.0 : -1.0;
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        if (g.M != n || g.N != n || g.ldc != n) return;
        TmaProblem q{dp.C, n, n, n, 0, 0, g.beta, (long long)ts.size(), 0, 0, nullptr, nullptr, 0};
        bool has_f = false;
        const i64 xrows = plan.buf_size[BUF_JK] / n;  // F rows follow the integral rows in the split array
        for (i64 k = g.seg_begin; k < g.seg_end; ++k) {
          const GemmSeg& x = s.gs[(size_t)k];
          if (x.a == BUF_F || x.b == BUF_F) {
            if (f_on_tc && x.a == BUF_F && x.b == BUF_D && x.K == n && x.lda == n && x.ldb == n && !x.tA && !x.tB &&
                x.offA % n == 0 && x.offB % n2 == 0) {
              ts.push_back(TmaSeg{xrows + x.offA / n, x.offB / n, 0, n, x.alpha * psign[(size_t)(x.offB / n2)]});
              continue;
            }
            if (f_on_tc) return;  // an F segment of another shape: leave the step on the older path
            has_f = true;
            continue;
          }
          if (x.a != BUF_JK || x.b != BUF_D || x.K != n || x.lda != n || x.ldb != n || x.tA || x.tB || x.offA % n ||
              x.offB % n2)
            return;
          ts.push_back(TmaSeg{x.offA / n, x.offB / n, 0, n, x.alpha * psign[(size_t)(x.offB / n2)]});
        }
        q.seg_end = (long long)ts.size();
        if (has_f) q.beta = 1.0;  // the FP64 part of the step runs first
        if (q.seg_end == q.seg_begin && has_f) continue;
        push(q);
      }
      d.tma_kind = 1;
    } else if (s.name == "three-external forward") {
      TN = tci_gtma_host::tile_n(tma_wide(2));
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        if (g.N != n || g.ldc != n || g.seg_end - g.seg_begin != 1) return;
        const GemmSeg& x = s.gs[(size_t)g.seg_begin];
        if (x.a != BUF_D || x.b != BUF_V || x.tA || !x.tB || x.lda != n2 || x.ldb != n2 || x.offA % 32 ||
            x.offB % n2 != x.offA || !((x.offA + x.K) % 32 == 0 || x.offA + x.K == n2) || g.M > plan.nD)
          return;
        // C^T (n x nD) = V_i rows (n x K) . pair rows (nD x K)^T
        TmaProblem q{dp.C, n, n, g.M, 0, 0, g.beta, (long long)ts.size(), 0, 1, nullptr, nullptr, 0};
        ts.push_back(TmaSeg{(x.offB - x.offA) / n2, 0, x.offA, x.K, x.alpha});  // first row of V_i: i n
        q.seg_end = (long long)ts.size();
        push(q);
      }
      d.tma_kind = 2;
    } else if (s.name == "three-external reverse") {
      TN = tci_gtma_host::tile_n(tma_wide(3));
      // R (nD x n^2) += sum_i U_i (nD x n) V_i (n x n^2), computed as R^T = sum_i V_i^T U_i^T: A = rows of
      // the transposed V_i (n^2 x n, K-major), B = rows of U_i; the output tile is stored transposed
      long long ubase = -1;
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        if (g.M != plan.nD || g.N != n2 || g.ldc != n2) return;
        TmaProblem q{dp.C, n2, n2, g.M, 0, 0, g.beta, (long long)ts.size(), 0, 1, nullptr, nullptr, 0};
        for (i64 k = g.seg_begin; k < g.seg_end; ++k) {
          const GemmSeg& x = s.gs[(size_t)k];
          if (x.a != BUF_T0 || x.b != BUF_V || x.tA || x.tB || x.lda != n || x.ldb != n2 || x.K != n ||
              x.offB % (n * n2))
            return;
          const i64 i = x.offB / (n * n2);
          const long long ub = x.offA - i * plan.nD * n;
          if (ubase < 0) ubase = ub;
          if (ub != ubase || i >= plan.nint) return;
          ts.push_back(TmaSeg{i * n2, i * plan.nD, 0, n, x.alpha});
        }
        q.seg_end = (long long)ts.size();
        push(q);
      }
      if (ubase < 0 || ubase + plan.nint * plan.nD * n > plan.buf_size[BUF_T0]) return;
      d.tma_aux = ubase;
      d.tma_kind = 3;
    } else if (s.name == "one-external forward") {
      // Z rows (M x n) = coupling-vector rows of BUF_WV (M x n) x D_d, D_d entering as the K-major operand
      // through its symmetry (D^T = p D, the sign folded into alpha)
      TN = tci_gtma_host::tile_n(tma_wide(5));
      std::vector<double> psign((size_t)std::max<i64>(plan.nD, 1), 1.0);
      for (const auto& h : plan.dheads)
        for (i64 k = 0; k < h.nD; ++k) psign[(size_t)(h.dk0 + k)] = k < h.nsing ? 1.0 : -1.0;
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        if (g.N != n || g.ldc != n || g.seg_end - g.seg_begin != 1) return;
        const GemmSeg& x = s.gs[(size_t)g.seg_begin];
        if (x.a != BUF_WV || x.b != BUF_D || x.tA || x.tB || x.lda != n || x.ldb != n || x.K != n || x.offA % n ||
            x.offB % n2)
          return;
        TmaProblem q{dp.C, n, g.M, n, 0, 0, g.beta, (long long)ts.size(), 0, 0, nullptr, nullptr, 0};
        ts.push_back(TmaSeg{x.offA / n, x.offB / n, 0, n, x.alpha * psign[(size_t)(x.offB / n2)]});
        q.seg_end = (long long)ts.size();
        push(q);
      }
      d.tma_kind = 5;
    } else if (s.name == "dv forward") {
      // F2 partials (nk x nD, one problem per 32-aligned chunk of the n^2 contraction) = rows of the
      // exchange bank (nk x n^2, in BUF_JK) x pair-matrix rows (nD x n^2)
      TN = tci_gtma_host::tile_n(tma_wide(6));
      long long kbase = -1, nk = -1;
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        if (g.N != plan.nD || g.ldc != plan.nD || g.seg_end - g.seg_begin != 1) return;
        const GemmSeg& x = s.gs[(size_t)g.seg_begin];
        if (x.a != BUF_JK || x.b != BUF_D || x.tA || !x.tB || x.lda != n2 || x.ldb != n2 || x.offB % 32 ||
            !((x.offB + x.K) % 32 == 0 || x.offB + x.K == n2) || x.offB + x.K > n2)
          return;
        if (kbase < 0) {
          kbase = x.offA - x.offB;
          nk = g.M;
        }
        if (x.offA - x.offB != kbase || g.M != nk) return;
        TmaProblem q{dp.C, plan.nD, g.M, plan.nD, 0, 0, g.beta, (long long)ts.size(), 0, 0, nullptr, nullptr, 0};
        ts.push_back(TmaSeg{0, 0, x.offB, x.K, x.alpha});
        q.seg_end = (long long)ts.size();
        push(q);
      }
      if (kbase < 0 || kbase + nk * n2 > plan.buf_size[BUF_JK]) return;
      d.tma_aux = kbase;
      d.tma_rows = nk;
      d.tma_kind = 6;
    } else if (s.name == "dv reverse") {
      // R (nD x n^2) += G2^T (nD x nk) Kbank (nk x n^2), computed as R^T = Kbank^T G2: A = rows of the
      // transposed exchange bank (split once), B = rows of the transposed gathered G2 (split every build)
      TN = tci_gtma_host::tile_n(tma_wide(7));
      if (s.gp.size() != 1) return;
      const GemmProblem& g = s.gp[0];
      const DGemmProblem& dp = pr[gi++];
      if (g.M != plan.nD || g.N != n2 || g.ldc != n2 || g.seg_end - g.seg_begin != 1) return;
      const GemmSeg& x = s.gs[(size_t)g.seg_begin];
      if (x.a != BUF_T0 || x.b != BUF_JK || !x.tA || x.tB || x.lda != plan.nD || x.ldb != n2 ||
          x.offB + x.K * n2 > plan.buf_size[BUF_JK] || x.offA + x.K * plan.nD > plan.buf_size[BUF_T0])
        return;
      TmaProblem q{dp.C, n2, n2, plan.nD, 0, 0, g.beta, (long long)ts.size(), 0, 1, nullptr, nullptr, 0};
      ts.push_back(TmaSeg{0, 0, 0, x.K, x.alpha});
      q.seg_end = (long long)ts.size();
      push(q);
      d.tma_aux = x.offA;    // G2 in BUF_T0 (K x nD)
      d.tma_rows = x.K;      // nk
      d.tma_aux2 = x.offB;   // the exchange bank in BUF_JK (K x n^2)
      d.tma_kind = 7;
    } else if (s.name == "ss two-external") {
      // Y rows (M x n) = gathered rows (M x n) X^T with X an n x n integral matrix of BUF_JK, computed as
      // Y^T = X Cg^T: A = rows of X, B = the gathered rows.  Problems of at most SKINNY_M rows (the
      // one-electron-like operators among them) stay on the skinny FP64 kernel.
      TN = tci_gtma_host::tile_n(tma_wide(4));
      long long lo = -1, hi = -1;
      for (const auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        const DGemmProblem& dp = pr[gi++];
        bool skinny = g.M <= SKINNY_M;
        for (i64 k = g.seg_begin; skinny && k < g.seg_end; ++k) skinny = s.gs[(size_t)k].tA == 0 && s.gs[(size_t)k].tB == 1;
        if (skinny) continue;
        if (g.N != n || g.ldc != n) return;
        TmaProblem q{dp.C, n, n, g.M, 0, 0, g.beta, (long long)ts.size(), 0, 1, nullptr, nullptr, 0};
        for (i64 k = g.seg_begin; k < g.seg_end; ++k) {
          const GemmSeg& x = s.gs[(size_t)k];
          if (x.a != BUF_T0 || x.b != BUF_JK || x.tA || !x.tB || x.lda != n || x.ldb != n || x.K != n || x.offB % n)
            return;
          lo = lo < 0 ? x.offA : std::min<long long>(lo, x.offA);
          hi = std::max<long long>(hi, x.offA + g.M * n);
          ts.push_back(TmaSeg{x.offB / n, x.offA, 0, n, x.alpha});  // b_row: offset for now, a row below
        }
        q.seg_end = (long long)ts.size();
        push(q);
      }
      if (lo < 0) return;
      for (auto& x : ts) {
        if ((x.b_row - lo) % n) return;  // the gathered rows are consecutive n-vectors from lo
        x.b_row = (x.b_row - lo) / n;
      }
      d.tma_aux = lo;
      d.tma_rows = (hi - lo) / n;
      d.tma_kind = 4;
    } else {
      return;
    }
    if (tp.empty()) {
      d.tma_kind = 0;
      return;
    }
    d.tma_probs = upload(tp, owned, stream);
    d.tma_segs = upload(ts, owned, stream);
    d.tma_nprob = (int)tp.size();
    d.tma_ntiles = tiles;
  }

  // The two-external step of a local deck's plan on the heads' domains: the same problems and segments
  // (target pair matrix, integral matrix x source pair matrix, alpha), each restricted to the target's domain
  // rows, the source's domain as k range and the columns common to both, on compact squares of the local
  // heads' pair matrices and accumulators; heads without local CSFs, and terms without common columns, drop out.
  DevStep lower_dom(const Step& s, const tci::LocalSetup& ls) {
    DevStep d;
    d.kind = s.kind;
    d.name = s.name;
    const i64 n = plan.n, n2 = n * n;
    if (ls.dh_len.size() != plan.dheads.size() || ls.dh_off.size() != plan.dheads.size())
      throw Error(TCI_ERR_INTERNAL, "local domains do not match the plan's heads");
    for (int x : ls.dh_dom)
      if (x < 0 || x >= n) throw Error(TCI_ERR_INTERNAL, "local domain entry outside the externals");
    for (size_t h = 0; h < ls.dh_len.size(); ++h) {
      if (ls.dh_len[h] < 0 || ls.dh_len[h] > n || ls.dh_off[h] + ls.dh_len[h] > (i64)ls.dh_dom.size())
        throw Error(TCI_ERR_INTERNAL, "local domain slice out of range");
      if (!std::is_sorted(ls.dh_dom.begin() + ls.dh_off[h], ls.dh_dom.begin() + ls.dh_off[h] + ls.dh_len[h]))
        throw Error(TCI_ERR_INTERNAL, "local domain not sorted");
    }
    std::vector<i64> dk2h((size_t)plan.nD, -1);
    for (size_t h = 0; h < plan.dheads.size(); ++h)
      for (i64 k = 0; k < plan.dheads[h].nD; ++k) dk2h[(size_t)(plan.dheads[h].dk0 + k)] = (i64)h;
    auto dk_of = [&](i64 off) {
      const i64 dk = off / n2;
      if (off % n2 || dk < 0 || dk >= plan.nD || dk2h[(size_t)dk] < 0)
        throw Error(TCI_ERR_INTERNAL, "two-external operand is not a pair matrix");
      return dk;
    };
    auto mh = [&](i64 h) { return ls.dh_len[(size_t)h]; };
    auto pitch_of = [](i64 m) { return m + (m & 1); };
    // compact squares: one per pair matrix of a head with local CSFs, for the sources and for the targets
    std::vector<i64> sq_off((size_t)plan.nD, -1);
    i64 sq_len = 0;
    for (i64 dk = 0; dk < plan.nD; ++dk) {
      const i64 m = mh(dk2h[(size_t)dk]);
      if (m == 0) continue;
      sq_off[(size_t)dk] = sq_len;
      sq_len += m * pitch_of(m);
    }
    // common columns of two heads as positions in each domain, computed once per head pair
    std::map<std::pair<i64, i64>, std::pair<i64, i64>> common;  // (target head, source head) -> (offset, count)
    std::vector<int> cpos_s, cpos_t;
    auto common_of = [&](i64 ht, i64 hs) {
      auto it = common.find({ht, hs});
      if (it != common.end()) return it->second;
      const int *a = ls.dh_dom.data() + ls.dh_off[(size_t)ht], *b = ls.dh_dom.data() + ls.dh_off[(size_t)hs];
      const i64 o = (i64)cpos_s.size();
      for (i64 x = 0, y = 0; x < mh(ht) && y < mh(hs);) {
        if (a[x] < b[y]) ++x;
        else if (b[y] < a[x]) ++y;
        else {
          cpos_t.push_back((int)x++);
          cpos_s.push_back((int)y++);
        }
      }
      return common[{ht, hs}] = {o, (i64)cpos_s.size() - o};
    };
    struct HostSeg {
      const double* A;
      i64 dks, hs, col_off, ncol;
      double alpha;
    };
    struct HostProb {
      i64 dk, head, m;
      std::vector<HostSeg> segs;
    };
    std::vector<HostProb> probs;
    std::vector<char> seen((size_t)plan.nD, 0);
    std::vector<char> src_used((size_t)plan.nD, 0);
    for (const auto& g : s.gp) {
      if (g.c != BUF_R || g.M != n || g.N != n || g.ldc != n)
        throw Error(TCI_ERR_INTERNAL, "unexpected two-external problem shape");
      const i64 dk = dk_of(g.offC), h = dk2h[(size_t)dk], m = mh(h);
      if (seen[(size_t)dk]++) throw Error(TCI_ERR_INTERNAL, "two-external target listed twice");
      if (m == 0) continue;
      std::vector<HostSeg> hsg;
      for (i64 q = g.seg_begin; q < g.seg_end; ++q) {
        const GemmSeg& x = s.gs[(size_t)q];
        if (x.b != BUF_D || x.lda != n || x.ldb != n || x.K != n || x.tA || x.tB)
          throw Error(TCI_ERR_INTERNAL, "unexpected two-external segment shape");
        const i64 dks = dk_of(x.offB), hs = dk2h[(size_t)dks];
        if (mh(hs) == 0) continue;
        const auto cm = common_of(h, hs);
        if (cm.second == 0) continue;
        check_range(x.a, x.offA, n2);
        hsg.push_back(HostSeg{ptr(x.a, x.offA), dks, hs, cm.first, cm.second, x.alpha});
        src_used[(size_t)dks] = 1;
      }
      if (hsg.empty()) continue;
      probs.push_back(HostProb{dk, h, m, std::move(hsg)});
    }
    check_range(BUF_D, 0, plan.nD * n2);
    check_range(BUF_R, 0, plan.nD * n2);
    auto dev_alloc = [&](double** p, i64 len) {
      TCI_CUDA(dev_malloc(p, (size_t)std::max<i64>(1, len) * sizeof(double), stream));
      owned.push_back(*p);
      bytes_held += (double)std::max<i64>(1, len) * sizeof(double);
    };
    double *dsq = nullptr, *rsq = nullptr;
    dev_alloc(&dsq, sq_len);
    dev_alloc(&rsq, sq_len);
    const int* ddom = upload(ls.dh_dom, owned, stream);
    const int* dcs = upload(cpos_s, owned, stream);
    const int* dct = upload(cpos_t, owned, stream);
    // the integral operands are constant: each distinct (operand, target head, source head) block compacted
    // once at set-up (row pitch even), when the device has room for them beside a margin
    std::map<std::tuple<const double*, i64, i64>, i64> apos;
    i64 abytes = 0;
    for (const auto& p : probs)
      for (const auto& x : p.segs) {
        auto key = std::make_tuple(x.A, p.head, x.hs);
        if (apos.count(key)) continue;
        apos[key] = abytes / 8;
        abytes += 8 * p.m * pitch_of(mh(x.hs));
      }
    double* abuf = nullptr;
    {
      size_t fr = 0, tot = 0;
      if (abytes > 0 && cudaMemGetInfo(&fr, &tot) == cudaSuccess && (double)abytes + 8e9 < (double)fr &&
          dev_malloc(&abuf, (size_t)abytes, stream) == cudaSuccess) {
        owned.push_back(abuf);
        bytes_held += (double)abytes;
      } else {
        cudaGetLastError();
        abuf = nullptr;
      }
    }
    std::vector<DComPack> jobs;
    if (abuf)
      for (const auto& kv : apos) {
        const i64 ht = std::get<1>(kv.first), hs = std::get<2>(kv.first);
        jobs.push_back(DComPack{std::get<0>(kv.first), abuf + kv.second, ddom + ls.dh_off[(size_t)ht],
                                ddom + ls.dh_off[(size_t)hs], (int)mh(ht), (int)mh(hs), (int)pitch_of(mh(hs))});
      }
    // the squares: gathered sources (those some term reads), zeroed and scattered targets
    std::vector<DComSq> gsq, ssq;
    for (i64 dk = 0; dk < plan.nD; ++dk) {
      if (sq_off[(size_t)dk] < 0) continue;
      const i64 h = dk2h[(size_t)dk];
      DComSq q{buf[BUF_D] + dk * n2, dsq + sq_off[(size_t)dk], ddom + ls.dh_off[(size_t)h], (int)mh(h),
               (int)pitch_of(mh(h))};
      if (src_used[(size_t)dk]) gsq.push_back(q);
    }
    std::vector<DComProblem> pr;
    std::vector<DComSeg> sg;
    long long tiles = 0;
    for (const auto& p : probs) {
      ssq.push_back(DComSq{buf[BUF_R] + p.dk * n2, rsq + sq_off[(size_t)p.dk], ddom + ls.dh_off[(size_t)p.head],
                           (int)p.m, (int)pitch_of(p.m)});
      DComProblem P{rsq + sq_off[(size_t)p.dk], ddom + ls.dh_off[(size_t)p.head], (int)p.m, (int)pitch_of(p.m),
                    tiles, (long long)sg.size(), 0};
      for (const auto& x : p.segs) {
        const i64 ms = mh(x.hs);
        const double* ac = abuf ? abuf + apos.at(std::make_tuple(x.A, p.head, x.hs)) : nullptr;
        sg.push_back(DComSeg{x.A, ac, dsq + sq_off[(size_t)x.dks], ddom + ls.dh_off[(size_t)x.hs], dcs + x.col_off,
                             dct + x.col_off, (int)ms, (int)x.ncol, (int)pitch_of(ms), (int)pitch_of(ms), x.alpha});
      }
      P.seg_end = (long long)sg.size();
      tiles += (p.m + COM_R - 1) / COM_R;
      pr.push_back(P);
    }
    d.com_probs = upload(pr, owned, stream);
    d.com_segs = upload(sg, owned, stream);
    d.com_nprob = (int)pr.size();
    d.com_ntiles = tiles;
    d.com_pack = upload(jobs, owned, stream);
    d.com_njobs = (long long)jobs.size();
    d.com_gather = upload(gsq, owned, stream);
    d.com_ngather = (long long)gsq.size();
    d.com_scatter = upload(ssq, owned, stream);
    d.com_nscatter = (long long)ssq.size();
    d.com_rsq = rsq;
    d.com_rsq_len = sq_len;
    d.com_step = true;
    return d;
  }

  // The three-external term of a local deck on the domains. Units come from the reverse gather step: each of
  // its targets is the row U_(i,dk) (one (i, dk) with a nonzero coupling), its sources the CSF rows of the N-1
  // head mu = lambda + e_i. The zero, scatter and gather steps stay as they are. Returns false (the padded
  // steps stay) when the plan has no three-external term or a domain is too wide for the staging.
  bool lower_dom3(const std::vector<Step>& steps, const tci::LocalSetup& ls, DevStep& fwd, DevStep& rev) {
    const i64 n = plan.n, n2 = n * n, nD = plan.nD, nint = plan.nint;
    const Step *zy = nullptr, *zu = nullptr, *ga = nullptr;
    for (const auto& s : steps) {
      if (s.name == "three-external zero") zy = &s;
      if (s.name == "three-external reverse zero") zu = &s;
      if (s.name == "three-external reverse gather") ga = &s;
    }
    if (!zy || !zu || !ga || nD == 0) return false;
    if (zy->buf != BUF_T0 || zu->buf != BUF_T0 || zy->len != nint * nD * n || zu->len != nint * nD * n)
      throw Error(TCI_ERR_INTERNAL, "unexpected three-external row buffers");
    const size_t nh1 = ls.s1_begin.size();
    if (ls.s1_end.size() != nh1 || ls.s1_off.size() != nh1 || ls.s1_len.size() != nh1 ||
        ls.dh_len.size() != plan.dheads.size())
      throw Error(TCI_ERR_INTERNAL, "local domains do not match the plan's heads");
    for (int x : ls.s1_dom)
      if (x < 0 || x >= n) throw Error(TCI_ERR_INTERNAL, "local domain entry outside the externals");
    for (size_t h = 0; h < nh1; ++h)
      if (ls.s1_len[h] < 0 || ls.s1_len[h] > n || ls.s1_off[h] + ls.s1_len[h] > (i64)ls.s1_dom.size())
        throw Error(TCI_ERR_INTERNAL, "local domain slice out of range");
    std::vector<std::pair<i64, size_t>> by_begin;  // N-1 heads by their first CSF row
    for (size_t h = 0; h < nh1; ++h) by_begin.push_back({ls.s1_begin[h], h});
    std::sort(by_begin.begin(), by_begin.end());
    auto mu_of = [&](i64 row) -> size_t {
      auto it = std::upper_bound(by_begin.begin(), by_begin.end(), std::make_pair(row, (size_t)-1));
      if (it == by_begin.begin()) throw Error(TCI_ERR_INTERNAL, "three-external row outside the N-1 heads");
      const size_t h = std::prev(it)->second;
      if (row >= ls.s1_end[h] || (row - ls.s1_begin[h]) % n) throw Error(TCI_ERR_INTERNAL, "three-external row outside the N-1 heads");
      return h;
    };
    std::vector<i64> dk2h((size_t)nD, -1);
    for (size_t h = 0; h < plan.dheads.size(); ++h)
      for (i64 k = 0; k < plan.dheads[h].nD; ++k) dk2h[(size_t)(plan.dheads[h].dk0 + k)] = (i64)h;
    std::map<std::pair<i64, i64>, size_t> mu;  // (lambda head, i) -> mu head
    for (const auto& t : ga->at) {
      const i64 rel = t.off - zu->off;
      if (t.dst != BUF_T0 || t.len != n || rel < 0 || rel % n || rel / n >= nint * nD)
        throw Error(TCI_ERR_INTERNAL, "unexpected three-external gather target");
      const i64 i = (rel / n) / nD, dk = (rel / n) % nD, h = dk2h[(size_t)dk];
      if (h < 0) throw Error(TCI_ERR_INTERNAL, "three-external row of no pair matrix");
      for (i64 q = t.src_begin; q < t.src_end; ++q) {
        const AxpySource& x = ga->as[(size_t)q];
        if (x.src != BUF_C || x.sbuf >= 0) throw Error(TCI_ERR_INTERNAL, "unexpected three-external gather source");
        const size_t m = mu_of(x.off);
        auto ins = mu.insert({{h, i}, m});
        if (ins.first->second != m) throw Error(TCI_ERR_INTERNAL, "three-external coupling of two N-1 heads");
      }
    }
    check_range(BUF_V, 0, nint * n * n2);
    check_range(BUF_D, 0, nD * n2);
    check_range(BUF_R, 0, nD * n2);
    const int* ddl = upload(ls.dh_dom, owned, stream);
    const int* ddm = upload(ls.s1_dom, owned, stream);
    std::vector<D3Fwd> fu;
    std::vector<D3Rev> ru;
    std::vector<D3RevEntry> re;
    i64 max_ml = 0, max_mm = 0, tiles = 0;
    for (auto it = mu.begin(); it != mu.end();) {
      const i64 h = it->first.first;
      const i64 ml = ls.dh_len[(size_t)h], dk0 = plan.dheads[(size_t)h].dk0, nh = plan.dheads[(size_t)h].nD;
      const long long e0 = (long long)re.size();
      for (; it != mu.end() && it->first.first == h; ++it) {
        const i64 i = it->first.second, mm = ls.s1_len[it->second];
        if (ml == 0 || mm == 0) continue;
        re.push_back(D3RevEntry{i, ddm + ls.s1_off[it->second], (int)mm});
        max_mm = std::max(max_mm, mm);
        for (i64 c = 0; c < nh; c += D3_K)
          for (i64 b0 = 0; b0 < mm; b0 += D3_BCHUNK)
            fu.push_back(D3Fwd{i, dk0 + c, ddl + ls.dh_off[(size_t)h], ddm + ls.s1_off[it->second], (int)ml, (int)mm,
                               (int)std::min<i64>(D3_K, nh - c), (int)b0, (int)std::min<i64>(mm, b0 + D3_BCHUNK)});
      }
      if ((long long)re.size() == e0) continue;
      max_ml = std::max(max_ml, ml);
      for (i64 c = 0; c < nh; c += D3_K) {
        ru.push_back(D3Rev{dk0 + c, tiles, ddl + ls.dh_off[(size_t)h], (int)ml, (int)std::min<i64>(D3_K, nh - c), e0,
                           (long long)re.size()});
        tiles += (ml * ml + D3R_T - 1) / D3R_T;
      }
    }
    const size_t smem = (size_t)(D3_K * D3_QC * max_ml + D3_K * std::min<i64>(max_mm, D3_BCHUNK)) * sizeof(double) +
                        (size_t)max_ml * sizeof(int);
    if (smem > 200 * 1024) return false;
    fwd.d3 = 1;
    fwd.kind = STEP_AXPY;
    fwd.name = "three-external split-k sum";
    fwd.d3f = upload(fu, owned, stream);
    fwd.d3f_n = (long long)fu.size();
    fwd.d3f_smem = smem;
    fwd.d3_rows = ptr(BUF_T0, zy->off);
    rev.d3 = 2;
    rev.kind = STEP_GEMM;
    rev.name = "three-external reverse";
    rev.d3r = upload(ru, owned, stream);
    rev.d3e = upload(re, owned, stream);
    rev.d3r_n = (int)ru.size();
    rev.d3r_tiles = tiles;
    rev.d3_rows = ptr(BUF_T0, zu->off);
    return true;
  }

  // The zero-external step of a local deck: the target rows of N-2 heads (ab and aa blocks) and of N-1 heads
  // whose sources are all rows of the same kind move to axpy_common over the positions common to the two
  // heads' domains; the rest (valence rows) stay on the padded AXPY.
  DevStep lower_zero_local(const Step& s, const tci::LocalSetup& ls) {
    const i64 n = plan.n, nab = n * (n - 1) / 2;
    // rows: (begin, end, kind 0 ab / 1 aa / 2 N-1, head slot into the local domain tables)
    struct Range {
      i64 begin, end;
      int kind;
      size_t h;
    };
    std::vector<Range> rg;
    if (ls.dh_len.size() != plan.dheads.size() || ls.s1_begin.size() != ls.s1_len.size())
      throw Error(TCI_ERR_INTERNAL, "local domains do not match the plan's heads");
    for (size_t h = 0; h < plan.dheads.size(); ++h) {
      const auto& d = plan.dheads[h];
      if (d.off_ab >= 0 && d.nsf_ab > 0) rg.push_back(Range{d.off_ab, d.off_ab + d.nsf_ab * nab, 0, h});
      if (d.off_aa >= 0 && d.nsf_aa > 0) rg.push_back(Range{d.off_aa, d.off_aa + d.nsf_aa * n, 1, h});
    }
    for (size_t h = 0; h < ls.s1_begin.size(); ++h) rg.push_back(Range{ls.s1_begin[h], ls.s1_end[h], 2, h});
    std::sort(rg.begin(), rg.end(), [](const Range& a, const Range& b) { return a.begin < b.begin; });
    auto row_of = [&](i64 off, i64 len) -> const Range* {
      auto it = std::upper_bound(rg.begin(), rg.end(), off, [](i64 v, const Range& r) { return v < r.begin; });
      if (it == rg.begin()) return nullptr;
      const Range& r = *std::prev(it);
      const i64 rl = r.kind == 0 ? nab : n;
      if (off >= r.end || len != rl || (off - r.begin) % rl) return nullptr;
      return &r;
    };
    auto dom_of = [&](const Range& r, const int*& p, i64& m) {
      if (r.kind == 2) {
        p = ls.s1_dom.data() + ls.s1_off[r.h];
        m = ls.s1_len[r.h];
      } else {
        p = ls.dh_dom.data() + ls.dh_off[r.h];
        m = ls.dh_len[r.h];
      }
    };
    // relative positions common to two heads of one kind, computed once per pair
    std::map<std::tuple<int, size_t, size_t>, std::pair<i64, i64>> lists;
    std::vector<int> rel;
    auto list_of = [&](const Range& t, const Range& u) {
      auto key = std::make_tuple(t.kind, t.h, u.h);
      auto it = lists.find(key);
      if (it != lists.end()) return it->second;
      const int *a, *b;
      i64 ma, mb;
      dom_of(t, a, ma);
      dom_of(u, b, mb);
      std::vector<int> c;
      std::set_intersection(a, a + ma, b, b + mb, std::back_inserter(c));
      const i64 o = (i64)rel.size();
      if (t.kind == 0) {
        for (size_t i = 1; i < c.size(); ++i)
          for (size_t j = 0; j < i; ++j) rel.push_back(c[i] * (c[i] - 1) / 2 + c[j]);  // c sorted: c[i] > c[j]
      } else {
        rel.insert(rel.end(), c.begin(), c.end());
      }
      return lists[key] = {o, (i64)rel.size() - o};
    };
    Step rest = s;
    rest.at.clear();
    rest.as.clear();
    struct HT {
      i64 off, len;
      std::vector<std::tuple<i64, i64, i64, double>> src;  // (source offset, list offset, list length, coef)
    };
    std::vector<HT> loc;
    for (const auto& t : s.at) {
      const Range* rt = t.dst == BUF_S ? row_of(t.off, t.len) : nullptr;
      bool ok = rt != nullptr;
      for (i64 q = t.src_begin; ok && q < t.src_end; ++q) {
        const AxpySource& x = s.as[(size_t)q];
        const Range* rs = x.src == BUF_C && x.sbuf < 0 ? row_of(x.off, t.len) : nullptr;
        ok = rs && rs->kind == rt->kind;
      }
      if (!ok) {  // stays on the padded AXPY
        AxpyTarget nt = t;
        nt.src_begin = (i64)rest.as.size();
        for (i64 q = t.src_begin; q < t.src_end; ++q) rest.as.push_back(s.as[(size_t)q]);
        nt.src_end = (i64)rest.as.size();
        rest.at.push_back(nt);
        continue;
      }
      const int* dp;
      i64 mt;
      dom_of(*rt, dp, mt);
      if (mt == 0) continue;  // a head without local CSFs: its sigma is never read back
      HT h{t.off, t.len, {}};
      for (i64 q = t.src_begin; q < t.src_end; ++q) {
        const AxpySource& x = s.as[(size_t)q];
        const auto l = list_of(*rt, *row_of(x.off, t.len));
        if (l.second > 0) h.src.emplace_back(x.off, l.first, l.second, x.coef);
      }
      if (!h.src.empty()) loc.push_back(std::move(h));
    }
    DevStep d = lower(rest);
    d.name = s.name;
    const int* drel = upload(rel, owned, stream);
    std::vector<ZcTarget> zt;
    std::vector<ZcSource> zs;
    for (const auto& h : loc) {
      check_range(BUF_S, h.off, h.len);
      ZcTarget T{ptr(BUF_S, h.off), (long long)zs.size(), 0};
      for (const auto& x : h.src) {
        check_range(BUF_C, std::get<0>(x), h.len);
        zs.push_back(ZcSource{ptr(BUF_C, std::get<0>(x)), drel + std::get<1>(x), (int)std::get<2>(x), std::get<3>(x)});
      }
      T.src_end = (long long)zs.size();
      zt.push_back(T);
    }
    d.zc_tg = upload(zt, owned, stream);
    d.zc_src = upload(zs, owned, stream);
    d.zc_ntg = (long long)zt.size();
    return d;
  }

  // The one-external term of a local deck on the pair domains: the forward and reverse GEMMs of the plan
  // (one problem per pair matrix: its coupling rows against D_dk, and their transposes against the gathered CI
  // rows) become dom1_forward / dom1_reverse over D_lambda; the gather and scatter steps stay. Returns false
  // (the padded GEMMs stay) when the plan has no one-external term.
  bool lower_dom1(const std::vector<Step>& steps, const tci::LocalSetup& ls, DevStep& fwd, DevStep& rev) {
    const i64 n = plan.n, n2 = n * n;
    const Step *gf = nullptr, *gr = nullptr;
    for (const auto& s : steps) {
      if (s.name == "one-external forward") gf = &s;
      if (s.name == "one-external reverse") gr = &s;
    }
    if (!gf || !gr || plan.nD == 0) return false;
    if (ls.dh_len.size() != plan.dheads.size()) throw Error(TCI_ERR_INTERNAL, "local domains do not match the plan's heads");
    std::vector<i64> dk2h((size_t)plan.nD, -1);
    for (size_t h = 0; h < plan.dheads.size(); ++h)
      for (i64 k = 0; k < plan.dheads[h].nD; ++k) dk2h[(size_t)(plan.dheads[h].dk0 + k)] = (i64)h;
    const int* ddl = upload(ls.dh_dom, owned, stream);
    auto dk_of = [&](i64 off) {
      const i64 dk = off / n2;
      if (off % n2 || dk < 0 || dk >= plan.nD || dk2h[(size_t)dk] < 0)
        throw Error(TCI_ERR_INTERNAL, "one-external operand is not a pair matrix");
      return dk;
    };
    std::vector<D1Row> rows;
    for (const auto& g : gf->gp) {
      if (g.seg_end - g.seg_begin != 1 || g.c != BUF_T0 || g.N != n || g.ldc != n)
        throw Error(TCI_ERR_INTERNAL, "unexpected one-external problem");
      const GemmSeg& x = gf->gs[(size_t)g.seg_begin];
      if (x.a != BUF_WV || x.b != BUF_D || x.tA || x.tB || x.lda != n || x.ldb != n || x.K != n || x.alpha != 1.0 ||
          g.beta != 0.0)
        throw Error(TCI_ERR_INTERNAL, "unexpected one-external segment");
      const i64 h = dk2h[(size_t)dk_of(x.offB)], ml = ls.dh_len[(size_t)h];
      check_range(BUF_WV, x.offA, g.M * n);
      check_range(BUF_T0, g.offC, g.M * n);
      check_range(BUF_D, x.offB, n2);
      for (i64 t = 0; t < g.M; ++t)
        rows.push_back(D1Row{ptr(BUF_WV, x.offA + t * n), ptr(BUF_D, x.offB), ptr(BUF_T0, g.offC + t * n),
                             ddl + ls.dh_off[(size_t)h], (int)ml});
    }
    std::vector<D1Target> tg;
    long long tiles = 0;
    for (const auto& g : gr->gp) {
      if (g.seg_end - g.seg_begin != 1 || g.c != BUF_R || g.M != n || g.N != n || g.ldc != n)
        throw Error(TCI_ERR_INTERNAL, "unexpected one-external reverse problem");
      const GemmSeg& x = gr->gs[(size_t)g.seg_begin];
      if (x.a != BUF_WV || x.b != BUF_T0 || !x.tA || x.tB || x.lda != n || x.ldb != n || x.alpha != 1.0 ||
          g.beta != 1.0)
        throw Error(TCI_ERR_INTERNAL, "unexpected one-external reverse segment");
      const i64 h = dk2h[(size_t)dk_of(g.offC)], ml = ls.dh_len[(size_t)h];
      if (ml == 0) continue;
      check_range(BUF_WV, x.offA, x.K * n);
      check_range(BUF_T0, x.offB, x.K * n);
      check_range(BUF_R, g.offC, n2);
      tg.push_back(D1Target{ptr(BUF_R, g.offC), ptr(BUF_WV, x.offA), ptr(BUF_T0, x.offB), ddl + ls.dh_off[(size_t)h],
                            (int)ml, (int)x.K, tiles});
      tiles += (ml * ml + 255) / 256;
    }
    fwd.d1 = 1;
    fwd.kind = STEP_GEMM;
    fwd.name = gf->name;
    fwd.d1_rows = upload(rows, owned, stream);
    fwd.d1_nrows = (long long)rows.size();
    rev.d1 = 2;
    rev.kind = STEP_GEMM;
    rev.name = gr->name;
    rev.d1_tg = upload(tg, owned, stream);
    rev.d1_ntg = (int)tg.size();
    rev.d1_tiles = tiles;
    return true;
  }

  // The N-2 <-> valence term of a local deck on the domains. Forward entries (pq, dk) come from the scatter
  // step's sources (F + pq nD + dk), reverse ones from the gather step's targets (G + pq nD + dk); the zero,
  // scatter and gather steps stay. Returns false (the padded steps stay) when the plan has no such term.
  bool lower_dom_dv(const std::vector<Step>& steps, const tci::LocalSetup& ls, DevStep& fwd, DevStep& rev) {
    const i64 n = plan.n, n2 = n * n, nD = plan.nD, nk = plan.nint * plan.nint;
    const Step *zf = nullptr, *zg = nullptr, *sc = nullptr, *ga = nullptr, *gr = nullptr;
    for (const auto& s : steps) {
      if (s.name == "dv forward zero") zf = &s;
      if (s.name == "dv reverse zero") zg = &s;
      if (s.name == "dv scatter") sc = &s;
      if (s.name == "dv reverse gather") ga = &s;
      if (s.name == "dv reverse") gr = &s;
    }
    if (!zf || !zg || !sc || !ga || !gr || nD == 0) return false;
    if (zf->buf != BUF_T0 || zg->buf != BUF_T0 || zf->len != nk * nD || zg->len != nk * nD || gr->gs.size() != 1 ||
        gr->gs[0].b != BUF_JK || gr->gs[0].a != BUF_T0 || gr->gs[0].offA != zg->off || gr->gs[0].K != nk)
      throw Error(TCI_ERR_INTERNAL, "unexpected N-2 <-> valence steps");
    const i64 offK = gr->gs[0].offB;
    check_range(BUF_JK, offK, nk * n2);
    check_range(BUF_D, 0, nD * n2);
    check_range(BUF_R, 0, nD * n2);
    std::vector<i64> dk2h((size_t)nD, -1);
    for (size_t h = 0; h < plan.dheads.size(); ++h)
      for (i64 k = 0; k < plan.dheads[h].nD; ++k) dk2h[(size_t)(plan.dheads[h].dk0 + k)] = (i64)h;
    if (ls.dh_len.size() != plan.dheads.size()) throw Error(TCI_ERR_INTERNAL, "local domains do not match the plan's heads");
    auto entry = [&](i64 rel) {
      if (rel < 0 || rel >= nk * nD) throw Error(TCI_ERR_INTERNAL, "N-2 <-> valence entry out of range");
      const i64 pq = rel / nD, dk = rel % nD;
      if (dk2h[(size_t)dk] < 0) throw Error(TCI_ERR_INTERNAL, "N-2 <-> valence entry of no pair matrix");
      return std::make_pair(pq, dk);
    };
    const int* ddl = upload(ls.dh_dom, owned, stream);
    std::vector<std::pair<i64, i64>> fe;  // forward entries (pq, dk), sorted and unique
    for (const auto& x : sc->as) {
      if (x.src != BUF_T0 || x.sbuf >= 0) throw Error(TCI_ERR_INTERNAL, "unexpected N-2 <-> valence scatter source");
      fe.push_back(entry(x.off - zf->off));
    }
    std::sort(fe.begin(), fe.end());
    fe.erase(std::unique(fe.begin(), fe.end()), fe.end());
    std::vector<DvEntry> fwe;
    for (const auto& e : fe) {
      const i64 h = dk2h[(size_t)e.second], ml = ls.dh_len[(size_t)h];
      if (ml > 0) fwe.push_back(DvEntry{e.first, e.second, ddl + ls.dh_off[(size_t)h], (int)ml});
    }
    std::map<i64, std::vector<i64>> by_dk;  // reverse: dk -> its pq, ascending
    for (const auto& t : ga->at) {
      if (t.dst != BUF_T0 || t.len != 1) throw Error(TCI_ERR_INTERNAL, "unexpected N-2 <-> valence gather target");
      const auto e = entry(t.off - zg->off);
      by_dk[e.second].push_back(e.first);
    }
    std::vector<DvTarget> rt;
    std::vector<long long> pqs;
    long long tiles = 0;
    for (auto& kv : by_dk) {
      const i64 h = dk2h[(size_t)kv.first], ml = ls.dh_len[(size_t)h];
      if (ml == 0) continue;
      std::sort(kv.second.begin(), kv.second.end());
      kv.second.erase(std::unique(kv.second.begin(), kv.second.end()), kv.second.end());
      const long long e0 = (long long)pqs.size();
      pqs.insert(pqs.end(), kv.second.begin(), kv.second.end());
      rt.push_back(DvTarget{kv.first, tiles, ddl + ls.dh_off[(size_t)h], (int)ml, e0, (long long)pqs.size()});
      tiles += (ml * ml + 255) / 256;
    }
    fwd.dv = 1;
    fwd.kind = STEP_AXPY;
    fwd.name = "dv split-k sum";
    fwd.dv_ent = upload(fwe, owned, stream);
    fwd.dv_nent = (long long)fwe.size();
    fwd.dv_vals = ptr(BUF_T0, zf->off);
    fwd.dv_k = ptr(BUF_JK, offK);
    rev.dv = 2;
    rev.kind = STEP_GEMM;
    rev.name = "dv reverse";
    rev.dv_tg = upload(rt, owned, stream);
    rev.dv_pq = upload(pqs, owned, stream);
    rev.dv_ntg = (int)rt.size();
    rev.dv_tiles = tiles;
    rev.dv_vals = ptr(BUF_T0, zg->off);
    rev.dv_k = ptr(BUF_JK, offK);
    return true;
  }

  // local decks: the padded positions of the local CSFs, sorted (empty otherwise)
  std::vector<long long> loc_pos;
  bool any_local(i64 off, i64 len) const {
    auto it = std::lower_bound(loc_pos.begin(), loc_pos.end(), (long long)off);
    return it != loc_pos.end() && *it < off + len;
  }

  DevStep lower(const Step& s) {
    DevStep d;
    d.kind = s.kind;
    d.name = s.name;
    if (s.kind == STEP_GEMM) {
      std::vector<DGemmProblem> pr;
      std::vector<DGemmSeg> sg;
      long long tiles = 0;
      // tile shape: wide in n when the problems are short in m (e.g. few CI blocks times an operator)
      double sm = 0, sn = 0;
      for (auto& g : s.gp) {
        sm += (double)g.M;
        sn += (double)g.N;
      }
      d.cfg = (sm <= sn) ? 0 : 1;
      const i64 BMh = d.cfg == 0 ? 64 : 128, BNh = d.cfg == 0 ? 128 : 64;
      for (auto& g : s.gp) {
        const i64 tm = (g.M + BMh - 1) / BMh, tn = (g.N + BNh - 1) / BNh;
        if (g.M <= 0 || g.N <= 0) continue;
        check_range(g.c, g.offC, (g.M - 1) * g.ldc + g.N);
        pr.push_back(DGemmProblem{ptr(g.c, g.offC), g.ldc, g.M, g.N, tn, tiles, g.beta, g.seg_begin, g.seg_end, 0});
        tiles += tm * tn;
      }
      for (auto& g : s.gs) sg.push_back(DGemmSeg{ptr(g.a, g.offA), ptr(g.b, g.offB), g.lda, g.ldb, g.K, g.tA, g.tB, g.alpha});
      // full operand extents: A is M x K (K x M if transposed), B is K x N (N x K)
      for (auto& g : s.gp) {
        if (g.M <= 0 || g.N <= 0) continue;
        for (i64 q = g.seg_begin; q < g.seg_end; ++q) {
          const GemmSeg& x = s.gs[q];
          if (x.K <= 0) throw Error(TCI_ERR_INTERNAL, "GEMM segment with empty K");
          const i64 ra = x.tA ? x.K : g.M, ca = x.tA ? g.M : x.K;
          const i64 rb = x.tB ? g.N : x.K, cb = x.tB ? x.K : g.N;
          if (ca > x.lda || cb > x.ldb) throw Error(TCI_ERR_INTERNAL, "GEMM leading dimension too small");
          check_range(x.a, x.offA, (ra - 1) * x.lda + ca);
          check_range(x.b, x.offB, (rb - 1) * x.ldb + cb);
        }
      }
      d.segs = upload(sg, owned, stream);
      {
        // FP64 form: skinny problems (one-row products) to the warp-per-column kernel, the rest tiled
        std::vector<DGemmProblem> reg, sk, pan[7], cpp[2];
        long long rt = 0, wk = 0, pt[7] = {0, 0, 0, 0, 0, 0, 0}, ct[2] = {0, 0};
        for (const auto& g : pr) {
          bool skinny = g.M <= SKINNY_M && s.name != "all-external";
          for (long long q = g.seg_begin; skinny && q < g.seg_end; ++q) skinny = sg[(size_t)q].tA == 0 && sg[(size_t)q].tB == 1;
          // few rows against long rows of B (the all-external product: a few dozen CI rows x the operator;
          // the reverse three-external product: the pair-matrix rows x the (iq|bs) banks) on the row-panel
          // kernel when the operands allow 16-byte copies
          bool panel = g.M <= 64 && g.N >= 1024 && !skinny;
          for (long long q = g.seg_begin; panel && q < g.seg_end; ++q) {
            const DGemmSeg& x = sg[(size_t)q];
            panel = x.tA == 0 && x.tB == 0 && ((x.lda | x.ldb) & 1) == 0 &&
                    ((reinterpret_cast<uintptr_t>(x.A) | reinterpret_cast<uintptr_t>(x.B)) & 15) == 0;
          }
          if (panel) {
            const int c = (int)((g.M + 7) / 8) - 1;  // MT = 8 (c + 1), classes 16 ... 64
            const int cls = std::max(1, c) - 1;       // 0: MT 16, 1: 24, ..., 6: 64
            DGemmProblem x = g;
            x.tile_begin = pt[cls];
            pt[cls] += (g.N + PANEL_COLS - 1) / PANEL_COLS;
            pan[cls].push_back(x);
          } else if (skinny) {
            DGemmProblem x = g;
            x.tile_begin = wk;  // first warp (one per output column); a block of 8 warps stays in one problem
            wk += (g.N + 7) / 8 * 8;
            sk.push_back(x);
          } else {
            // the cp.async-staged tiled kernel where the operands allow 16-byte copies (A not transposed,
            // one orientation of B per problem), else the register-staged one
            bool cpk = true;
            int tb = -1;
            for (long long q = g.seg_begin; cpk && q < g.seg_end; ++q) {
              const DGemmSeg& x = sg[(size_t)q];
              cpk = x.tA == 0 && (tb < 0 || tb == x.tB) && ((x.lda | x.ldb) & 1) == 0 &&
                    ((reinterpret_cast<uintptr_t>(x.A) | reinterpret_cast<uintptr_t>(x.B)) & 15) == 0;
              tb = x.tB;
            }
            DGemmProblem x = g;
            if (cpk && tb >= 0) {
              x.tiles_n = (g.N + CP_BN - 1) / CP_BN;
              x.tile_begin = ct[tb];
              ct[tb] += ((g.M + CP_BM - 1) / CP_BM) * x.tiles_n;
              cpp[tb].push_back(x);
            } else {
              x.tile_begin = rt;
              rt += ((g.M + BMh - 1) / BMh) * x.tiles_n;
              reg.push_back(x);
            }
          }
        }
        d.probs = upload(reg, owned, stream);
        d.nprob = (int)reg.size();
        d.ntiles = rt;
        for (int b = 0; b < 2; ++b) {
          d.cp_probs[b] = upload(cpp[b], owned, stream);
          d.cp_nprob[b] = (int)cpp[b].size();
          d.cp_ntiles[b] = ct[b];
        }
        d.skinny_probs = upload(sk, owned, stream);
        d.skinny_nprob = (int)sk.size();
        d.skinny_nwarps = wk;
        for (int c = 0; c < 7; ++c) {
          d.panel_probs[c] = upload(pan[c], owned, stream);
          d.panel_nprob[c] = (int)pan[c].size();
          d.panel_ntiles[c] = pt[c];
        }
      }
      if (s.name != "all-external" && !pr.empty()) {
        // Mixed form.  Segments whose operand is a same-head one-electron-like operator (BUF_F: h, J_ii,
        // K_ii combinations, orbital-energy magnitudes) stay on the FP64 kernel; the cross-head integral
        // segments go to the tensor cores (3xTF32), added after the FP64 part (beta 1 where both exist).
        // With f_on_tc the dd step's TMA lowering takes the F segments onto the tensor cores as well.
        // Problems of at most SKINNY_M rows stay whole on the skinny FP64 kernel (launched in this form too).
        std::vector<tci_dev::HostGemm> f64, tcp;
        for (const auto& g : pr) {
          bool skinny = g.M <= SKINNY_M;
          for (long long q = g.seg_begin; skinny && q < g.seg_end; ++q) skinny = sg[(size_t)q].tA == 0 && sg[(size_t)q].tB == 1;
          if (skinny) continue;
          tci_dev::HostGemm hf{g.C, g.ldc, g.M, g.N, g.beta, {}}, ht{g.C, g.ldc, g.M, g.N, g.beta, {}};
          for (long long q = g.seg_begin; q < g.seg_end; ++q) {
            const bool f = s.gs[(size_t)q].a == BUF_F || s.gs[(size_t)q].b == BUF_F;
            (f ? hf : ht).segs.push_back(sg[(size_t)q]);
          }
          if (!hf.segs.empty()) {
            f64.push_back(hf);
            ht.beta = 1.0;
          }
          if (!ht.segs.empty() || hf.segs.empty()) tcp.push_back(ht);
        }
        std::vector<DGemmProblem> pf, pt;
        std::vector<DGemmSeg> sf, st;
        d.ntiles_f = tci_dev::tile_problems(f64, tci_dev::gemm_f64_tile_m(d.cfg), tci_dev::gemm_f64_tile_n(d.cfg), false,
                                            pf, sf);
        // 128 x 64 tiles; a problem short in M is computed transposed
        d.ntiles_tc = tci_dev::tile_problems(tcp, tci_gtc_host::tile_m(), tci_gtc_host::tile_n(), true, pt, st);
        double flops = 0, useful = 0, issued = 0;
        const i64 TM = tci_gtc_host::tile_m(), TN = tci_gtc_host::tile_n();
        for (const auto& g : pt) {
          double k = 0;
          for (long long q = g.seg_begin; q < g.seg_end; ++q) k += (double)st[(size_t)q].K;
          flops += 2.0 * (double)g.M * (double)g.N * k;
          useful += (double)g.M * (double)g.N * k;
          issued += (double)((g.M + TM - 1) / TM * TM) * (double)((g.N + TN - 1) / TN * TN) * k;
        }
        d.probs_f = upload(pf, owned, stream);
        d.segs_f = upload(sf, owned, stream);
        d.nprob_f = (int)pf.size();
        d.probs_tc = upload(pt, owned, stream);
        d.segs_tc = upload(st, owned, stream);
        d.nprob_tc = (int)pt.size();
        d.tc_ok = flops >= 5e7 && useful >= 0.25 * issued;
        lower_tma(s, d, pr);
        if (d.tma_probs) d.tc_ok = flops >= 5e7;  // the TMA-fed tables tile the step well
      }
    } else if (s.kind == STEP_AXPY) {
      constexpr i64 kChunk = AXPY_CHUNK;  // elements per block: long rows are spread over many blocks
      // chunk counts first, then targets and sources converted (and range-checked) in parallel
      std::vector<i64> first(s.at.size() + 1, 0);
      for (size_t i = 0; i < s.at.size(); ++i) first[i + 1] = first[i] + (std::max<i64>(0, s.at[i].len) + kChunk - 1) / kChunk;
      std::vector<DAxpyTarget> t((size_t)first.back());
      std::vector<DAxpySource> so(s.as.size());
      int bad = 0;
#pragma omp parallel for schedule(static) reduction(| : bad)
      for (long long i = 0; i < (long long)s.at.size(); ++i) {
        const AxpyTarget& x = s.at[(size_t)i];
        if (!range_ok(x.dst, x.off, x.len) || x.src_begin < 0 || x.src_end > (i64)s.as.size()) {
          bad |= 1;
          continue;
        }
        for (i64 b = 0; b < x.len; b += kChunk) {
          // local decks: a chunk of sigma without local CSFs is never read back (gather_local): dropped
          const i64 len = std::min(kChunk, x.len - b);
          const bool keep = x.dst != BUF_S || loc_pos.empty() || any_local(x.off + b, len);
          t[(size_t)(first[(size_t)i] + b / kChunk)] =
              DAxpyTarget{buf[x.dst] + x.off + b, b, keep ? len : 0, x.src_begin, x.src_end};
        }
        // source length equals its target's length
        for (i64 q = x.src_begin; q < x.src_end; ++q)
          if (!range_ok(s.as[(size_t)q].src, s.as[(size_t)q].off, x.len)) bad |= 1;
      }
#pragma omp parallel for schedule(static) reduction(| : bad)
      for (long long q = 0; q < (long long)s.as.size(); ++q) {
        const AxpySource& x = s.as[(size_t)q];
        if (!range_ok(x.src, x.off, 0) || (x.sbuf >= 0 && !range_ok(x.sbuf, x.sidx, 0))) {
          bad |= 1;
          continue;
        }
        so[(size_t)q] = DAxpySource{buf[x.src] + x.off, x.sbuf >= 0 ? buf[x.sbuf] + x.sidx : nullptr, x.coef};
      }
      if (bad) throw Error(TCI_ERR_INTERNAL, "plan range outside its buffer (or an unallocated buffer)");
      if (!loc_pos.empty())
        t.erase(std::remove_if(t.begin(), t.end(), [](const DAxpyTarget& x) { return x.len == 0; }), t.end());
      d.at = upload(t, owned, stream);
      d.as = upload(so, owned, stream);
      d.ntg = (long long)t.size();
      // many sources per target, and no short targets (whose path the occupancy bound of that kernel slows)
      d.axpy_pairs = !s.at.empty() && s.as.size() >= 32 * s.at.size() &&
                     std::all_of(s.at.begin(), s.at.end(), [](const AxpyTarget& x) { return x.len >= 8; });
    } else if (s.kind == STEP_DOT) {
      std::vector<DDotTarget> t;
      std::vector<DDotSource> so;
      for (auto& x : s.dt) t.push_back(DDotTarget{ptr(x.dst, x.off), x.src_begin, x.src_end});
      for (auto& x : s.ds) {
        check_range(x.a, x.aoff, x.len);
        check_range(x.b, x.boff, x.len);
        so.push_back(DDotSource{ptr(x.a, x.aoff), ptr(x.b, x.boff), x.len, x.coef});
      }
      d.dt = upload(t, owned, stream);
      d.ds = upload(so, owned, stream);
      d.ntg = (long long)t.size();
    } else if (s.kind == STEP_ZERO) {
      check_range(s.buf, s.off, s.len);
      d.zptr = ptr(s.buf, s.off);
      d.zlen = s.len;
    }
    return d;
  }


  void ensure_diag() {
    if (hd) return;
    const i64 n = plan.total_csfs;
    double* full = nullptr;  // the non-local diagonal (local pair domains: gathered into hd afterwards)
    TCI_CUDA(dev_malloc(&full, n * sizeof(double), stream));
    TCI_CUDA(cudaMemsetAsync(full, 0, n * sizeof(double), stream));
    std::vector<DDiag> e;
    for (auto& d : plan.diag) e.push_back(DDiag{d.off, d.len, d.type, d.beta, d.foff, d.singlet});
    for (auto& d : plan.diag) check_range(BUF_S, d.off, d.len);
    DDiag* de = upload(e, owned, stream);
    if (!buf[BUF_W] && !xdiag && std::any_of(e.begin(), e.end(), [](const DDiag& x) { return x.type >= 2; }))
      throw Error(TCI_ERR_INTERNAL, "no all-external diagonal for the N-2 blocks");
    if (!e.empty())
      build_diag_kernel<<<(unsigned)e.size(), 256, 0, stream>>>(de, (long long)e.size(), plan.n, plan.np, plan.nm,
                                                                buf[BUF_F], buf[BUF_W], xdiag, full);
    TCI_CUDA(cudaGetLastError());
    if (local) {
      TCI_CUDA(dev_malloc(&hd, n_loc * sizeof(double), stream));
      gather_local<<<sm_count() * 8, 256, 0, stream>>>(full, d_map, n_loc, hd);
      TCI_CUDA(cudaGetLastError());
      TCI_CUDA(cudaStreamSynchronize(stream));
      std::lock_guard<std::mutex> lk(g_capture_free_mu);
      TCI_CUDA(dev_free(full, stream));
    } else {
      hd = full;
    }
    owned.push_back(hd);
    TCI_CUDA(cudaStreamSynchronize(stream));
  }

  // reduction scratch for projections of up to mmax vectors (grows when a solve needs more)
  void ensure_scratch(int mmax) {
    if (dots && mmax <= scratch_cap) return;
    if (dots) {
      TCI_CUDA(cudaStreamSynchronize(stream));
      std::lock_guard<std::mutex> lk(g_capture_free_mu);
      for (void* p : {(void*)dots, (void*)coefs}) {
        dev_free(p, stream);
        owned.erase(std::find(owned.begin(), owned.end(), p));
      }
      dots = coefs = nullptr;
      scratch_cap = 0;
    }
    TCI_CUDA(dev_malloc(&dots, ((size_t)mmax * (RBLK + 1) + 16) * sizeof(double), stream));
    owned.push_back(dots);
    TCI_CUDA(dev_malloc(&coefs, (size_t)4 * mmax * sizeof(double), stream));
    owned.push_back(coefs);
    scratch_cap = mmax;
  }

  // out[0..m) = A[k] . x  (host result), deterministic
  void multi_dot(const double* A, i64 lda, int m, const double* x, i64 n, double* host_out) {
    multi_dot_partial<<<RBLK, RB, 0, stream>>>(A, lda, m, x, n, dots);
    multi_dot_final<<<(m + 127) / 128, 128, 0, stream>>>(dots, m, RBLK, dots + (size_t)m * RBLK);
    launch_count += 2;
    TCI_CUDA(cudaGetLastError());
    TCI_CUDA(cudaMemcpyAsync(host_out, dots + (size_t)m * RBLK, m * sizeof(double), cudaMemcpyDeviceToHost, stream));
    TCI_CUDA(cudaStreamSynchronize(stream));
  }
  // device-resident single dot into dots[off]
  void dot_dev(const double* a, const double* x, i64 n, double* dev_out) {
    multi_dot_partial<<<RBLK, RB, 0, stream>>>(a, 0, 1, x, n, dots);
    multi_dot_final<<<1, 32, 0, stream>>>(dots, 1, RBLK, dev_out);
    launch_count += 2;
    TCI_CUDA(cudaGetLastError());
  }

  void sigma_of(const double* d_c, double* d_s) {
    const i64 n = plan.total_csfs;
    if (local) {
      local_in(d_c);
      run_sigma_steps();
      local_out(d_c, d_s);
      sigma_count++;
      return;
    }
    TCI_CUDA(cudaMemcpyAsync(buf[BUF_C], d_c, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    if (gen_s) scale_by<<<sm_count() * 8, 256, 0, stream>>>(buf[BUF_C], gen_s, n);
    TCI_CUDA(cudaMemsetAsync(buf[BUF_S], 0, n * sizeof(double), stream));
    run_sigma_steps();
    gen_out(d_s);
    sigma_count++;
  }
  // local layout: the padded input of the plan (zeros outside the domains) and an empty output
  void local_in(const double* d_c) {
    if (gen_s) throw Error(TCI_ERR_INPUT, "the generalized (ACPF-type) solve is not available under pair domains");
    const i64 n = plan.total_csfs;
    TCI_CUDA(cudaMemsetAsync(buf[BUF_C], 0, n * sizeof(double), stream));
    scatter_local<<<sm_count() * 8, 256, 0, stream>>>(d_c, d_map, n_loc, buf[BUF_C]);
    TCI_CUDA(cudaMemsetAsync(buf[BUF_S], 0, n * sizeof(double), stream));
    launch_count += 1;
    TCI_CUDA(cudaGetLastError());
  }
  // local layout: d_s = P^T (plan's sigma) + the all-external term of the local blocks
  void local_out(const double* d_c, double* d_s) {
    gather_local<<<sm_count() * 8, 256, 0, stream>>>(buf[BUF_S], d_map, n_loc, d_s);
    launch_count += 1;
    TCI_CUDA(cudaGetLastError());
    if (loc_allext) {
      const int rc = tci_local_apply(loc_allext, d_c, d_s, n_loc, stream);
      if (rc != TCI_OK) throw Error(rc, "pair-domain all-external term failed");
    }
  }
  // d_s = BUF_S, or in a generalized solve G^-1/2 (BUF_S - shift BUF_C)
  void gen_out(double* d_s) {
    const i64 n = plan.total_csfs;
    if (gen_s) {
      gen_sigma_out<<<sm_count() * 8, 256, 0, stream>>>(d_s, buf[BUF_S], buf[BUF_C], gen_s, gen_shift, n);
      TCI_CUDA(cudaGetLastError());
    } else {
      TCI_CUDA(cudaMemcpyAsync(d_s, buf[BUF_S], n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
    }
  }
  // TMA-fed kernel's tile width per step kind: 128 unless the B operand has at most 64 rows per problem
  bool tma_wide(int kind) const {
    return (kind == 1 || kind == 5) ? plan.n > 64 : kind == 4 ? false : plan.nD > 64;  // 2, 3, 6, 7: B has nD rows
  }
  bool tma_ok(const DevStep& s) const {
    return (s.tma_kind == 1 && tma_dd_ready) || (s.tma_kind == 2 && tma_t3_ready) || (s.tma_kind == 3 && tma_t3r_ready) ||
           (s.tma_kind == 4 && tma_ss_ready) || (s.tma_kind == 5 && tma_1x_ready) || (s.tma_kind == 6 && tma_dv_ready) ||
           (s.tma_kind == 7 && tma_dvr_ready);
  }
  template <int TB>
  void launch_cp(const DevStep& s) {
    if (s.cp_ntiles[TB] <= 0) return;
    constexpr size_t smem = cp_smem_bytes<TB>();
    static bool attr_set[64] = {};  // per device
    int dev = 0;
    TCI_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
      TCI_CUDA(cudaFuncSetAttribute(gemm_cp_f64<TB>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_set[dev] = true;
    }
    gemm_cp_f64<TB><<<(unsigned)s.cp_ntiles[TB], 256, smem, stream>>>(s.cp_probs[TB], s.cp_nprob[TB], s.segs);
  }
  template <int MT>
  void launch_panel(const DevStep& s, int c) {
    if (s.panel_ntiles[c] <= 0) return;
    constexpr size_t smem = panel_smem_bytes<MT>();
    static bool attr_set[64] = {};  // per device
    int dev = 0;
    TCI_CUDA(cudaGetDevice(&dev));
    if (dev >= 0 && dev < 64 && !attr_set[dev]) {
      TCI_CUDA(cudaFuncSetAttribute(gemm_panel_f64<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
      attr_set[dev] = true;
    }
    gemm_panel_f64<MT><<<(unsigned)s.panel_ntiles[c], PANEL_T, smem, stream>>>(s.panel_probs[c], s.panel_nprob[c],
                                                                               s.segs);
  }
  // the mixed form runs this GEMM step on the tensor cores
  bool uses_tc(const DevStep& s) const {
    return precision == 1 && s.probs_tc && (tc_mode == 1 || (tc_mode == 0 && s.tc_ok));
  }
  // kernels one sigma build launches (graph nodes included)
  long long sigma_launches() const {
    long long k = 0;
    for (const auto& s : sigma) {
      if (s.com_step) {
        k += (s.com_ngather > 0 ? 1 : 0) + (s.com_ntiles > 0 ? 1 : 0) + (s.com_nscatter > 0 ? 1 : 0);
        continue;
      }
      if (s.d3_skip) continue;
      if (s.d1) {
        k += (s.d1_nrows > 0 || s.d1_tiles > 0) ? 1 : 0;
        continue;
      }
      if (s.dv) {
        k += (s.dv_nent > 0 || s.dv_tiles > 0) ? 1 : 0;
        continue;
      }
      if (s.d3) {
        k += (s.d3f_n > 0 || s.d3r_tiles > 0) ? 1 : 0;
        continue;
      }
      const bool tc_allext = precision == 1 || allext_tc_in_fp64;
      if (tc_allext && (s.name == "all-external zero" || s.name == "all-external split-k sum")) continue;
      if (tc_allext && s.kind == STEP_GEMM && s.name == "all-external") {
        k += (has_sing() ? 1 : 0) + (has_trip() ? 1 : 0) + ((has_sing() || has_trip()) ? 1 : 0);
        continue;
      }
      if (s.kind == STEP_GEMM && uses_tc(s)) {
        const bool f_in_tma = f_on_tc && s.tma_kind == 1 && s.tma_probs && tma_ok(s);
        k += (s.skinny_nwarps > 0 ? 1 : 0) + ((s.ntiles_f > 0 && !f_in_tma) ? 1 : 0) +
             ((s.tma_probs && tma_ok(s)) ? 2 : (s.ntiles_tc > 0 ? 1 : 0));
        continue;
      }
      if (s.kind == STEP_GEMM && s.skinny_nwarps > 0) k += 1;
      if (s.kind == STEP_GEMM) {
        for (int c = 0; c < 7; ++c) k += s.panel_ntiles[c] > 0 ? 1 : 0;
        for (int b = 0; b < 2; ++b) k += s.cp_ntiles[b] > 0 ? 1 : 0;
      }
      if (s.zc_ntg > 0) k += 1;
      if ((s.kind == STEP_GEMM && s.ntiles > 0) || ((s.kind == STEP_AXPY || s.kind == STEP_DOT) && s.ntg > 0) ||
          ((s.kind == STEP_UNPACK || s.kind == STEP_PACK) && plan.nD > 0))
        k += 1;
    }
    return k;
  }

  void ensure_step_events() {
    if (step_ev.size() != 2 * sigma.size()) {
      step_ev.resize(2 * sigma.size());
      for (auto& e : step_ev) TCI_CUDA(cudaEventCreate(&e));
      step_ms.assign(sigma.size(), 0.0);
    }
  }

  void record_steps(bool with_events, bool capturing) {
    // inside a stream capture an event record becomes a graph node only when
    // it is marked external
    const unsigned fl = capturing ? cudaEventRecordExternal : cudaEventRecordDefault;
    for (size_t i = 0; i < sigma.size(); ++i) {
      if (with_events) TCI_CUDA(cudaEventRecordWithFlags(step_ev[2 * i], stream, fl));
      run(sigma[i]);
      if (with_events) TCI_CUDA(cudaEventRecordWithFlags(step_ev[2 * i + 1], stream, fl));
    }
  }

  // One sigma build.  With graphs on, the step sequence is captured once (a
  // second capture carries an event-record node around every step for the
  // profiler) and replayed with a single launch.
  void run_sigma_steps() {
    if (profiling) ensure_step_events();
    if (use_graph) {
      cudaGraph_t& g = profiling ? graph_prof : graph;
      cudaGraphExec_t& ge = profiling ? graph_exec_prof : graph_exec;
      if (!ge) {
        std::lock_guard<std::mutex> lk(g_capture_free_mu);
        TCI_CUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
        try {
          record_steps(profiling, true);
        } catch (...) {
          cudaGraph_t tmp = nullptr;
          cudaStreamEndCapture(stream, &tmp);
          if (tmp) cudaGraphDestroy(tmp);
          throw;
        }
        TCI_CUDA(cudaStreamEndCapture(stream, &g));
        TCI_CUDA(cudaGraphInstantiate(&ge, g, 0));
      }
      TCI_CUDA(cudaGraphLaunch(ge, stream));
    } else {
      record_steps(profiling, false);
    }
    launch_count += sigma_launches();
    if (profiling) {
      TCI_CUDA(cudaStreamSynchronize(stream));
      for (size_t i = 0; i < sigma.size(); ++i) {
        float ms = 0;
        TCI_CUDA(cudaEventElapsedTime(&ms, step_ev[2 * i], step_ev[2 * i + 1]));
        step_ms[i] += ms;
      }
      profiled_builds++;
    }
  }

  bool has_sing() const { return plan.n_sing > 0; }
  bool has_trip() const { return plan.n_trip > 0 && plan.nm > 0; }
  void run_allext_tc() {
    if (has_sing())
      TCI_CUDA(tci_tc_host::split_u(buf[BUF_T0] + plan.allext_us, plan.n_sing, plan.np, u2s, stream));
    if (has_trip())
      TCI_CUDA(tci_tc_host::split_u(buf[BUF_T0] + plan.allext_ut, plan.n_trip, plan.nm, u2t, stream));
    TCI_CUDA(tci_tc_host::launch(has_sing() ? &tc_sing : nullptr, has_trip() ? &tc_trip : nullptr, stream));
  }

  // X (M x M, FP64) = A A^T with A = M rows of K values in BUF_T0, on the TMA-fed 3xTF32 kernel (set-up).
  void exchange_product_tc(const GemmProblem& g, const GemmSeg& x, int64_t kblock) {
    const i64 M = g.M, K = x.K, ld = tci_gtma_host::pitch(K);
    check_range(BUF_T0, x.offA, (M - 1) * x.lda + K);
    check_range(g.c, g.offC, (M - 1) * g.ldc + M);
    float *ah = nullptr, *al = nullptr;
    int* st = nullptr;
    auto release = [&]() {
      cudaStreamSynchronize(stream);
      std::lock_guard<std::mutex> lk(g_capture_free_mu);
      for (void* p : {(void*)ah, (void*)al, (void*)st}) dev_free(p, stream);
      cudaStreamSynchronize(stream);
    };
    try {
      TCI_CUDA(dev_malloc(&ah, sizeof(float) * (size_t)(M * ld), stream));
      TCI_CUDA(dev_malloc(&al, sizeof(float) * (size_t)(M * ld), stream));
      TCI_CUDA(dev_malloc(&st, sizeof(int), stream));
      TCI_CUDA(cudaMemsetAsync(st, 0, sizeof(int), stream));
      TCI_CUDA(tci_gtma_host::split(buf[BUF_T0] + x.offA, M, K, x.lda, ah, al, stream));
      tci_gtma_host::TmaMaps m;
      std::string err;
      if (!tci_gtma_host::prepare(m, ah, al, M, K, ah, al, M, K, true, err)) throw Error(TCI_ERR_CUDA, err);
      const i64 TM = tci_gtma_host::tile_m(), TN = tci_gtma_host::tile_n(true);
      std::vector<TmaProblem> q{TmaProblem{ptr(g.c, g.offC), g.ldc, M, M, (M + TN - 1) / TN, 0, 0.0, 0, 1, 0, nullptr,
                                           nullptr, 0}};
      std::vector<TmaSeg> sg{TmaSeg{0, 0, 0, K, x.alpha}};
      TmaProblem* dq = upload(q, owned, stream);
      TmaSeg* ds = upload(sg, owned, stream);
      TCI_CUDA(tci_gtma_host::launch(m, dq, 1, ds, ((M + TM - 1) / TM) * q[0].tiles_n, (int)kblock, st, stream));
      int h = 0;
      TCI_CUDA(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, stream));
      TCI_CUDA(cudaStreamSynchronize(stream));
      if (h != 0) throw Error(TCI_ERR_TIMEOUT, "tensor-core exchange product: a bounded wait gave up");
    } catch (...) {
      release();
      throw;
    }
    release();
  }

  // Moves W+/W- to FP32 for the tensor-core product and releases the FP64 copy.
  // local decks: the constant operands of the domain steps compacted, once the set-up steps have built them
  void prepare_local() {
    for (const auto& st : sigma)
      if (st.com_njobs > 0) com_pack_a<<<(unsigned)st.com_njobs, 256, 0, stream>>>(st.com_pack, plan.n);
    TCI_CUDA(cudaGetLastError());
  }

  void setup_precision() {
    if (precision != 1) return;
    ensure_diag();  // the diagonal reads the FP64 W
    const i64 np = plan.np, nm = plan.nm;
    auto alloc_f = [&](float** p, size_t n) {
      if (dev_malloc(p, n * sizeof(float), stream) != cudaSuccess) {
        cudaGetLastError();
        throw Error(TCI_ERR_MEMORY, "device allocation failed (fp32 operators)");
      }
      owned.push_back(*p);
      bytes_held += (double)n * sizeof(float);
    };
    const bool allext = np > 0;  // the plan carries the all-external term (not under pair domains)
    if (allext) {
      alloc_f(&w32p, (size_t)tci_tc_host::w32_floats(np));
      if (nm > 0) alloc_f(&w32m, (size_t)tci_tc_host::w32_floats(nm));
      alloc_f(&u2s, (size_t)tci_tc_host::u2_floats(std::max<i64>(1, plan.n_sing), np));
      if (has_trip()) {
        alloc_f(&u2t, (size_t)tci_tc_host::u2_floats(plan.n_trip, nm));
      }
    }
    TCI_CUDA(dev_malloc(&tc_status, sizeof(int), stream));
    owned.push_back(tc_status);
    TCI_CUDA(tci_gtc_host::prepare());
    bool want_dd = false, want_t3 = false, want_t3r = false, want_ss = false, want_1x = false, want_dv = false;
    bool want_dvr = false;
    long long dv_base = 0, dv_rows = 0, dvr_base = 0, dvr_rows = 0;
    long long ss_rows = 0;
    for (const auto& st : sigma) {
      want_dd = want_dd || (st.tma_probs && st.tma_kind == 1);
      want_t3 = want_t3 || (st.tma_probs && st.tma_kind == 2);
      want_t3r = want_t3r || (st.tma_probs && st.tma_kind == 3);
      want_1x = want_1x || (st.tma_probs && st.tma_kind == 5);
      if (st.tma_probs && st.tma_kind == 7) {
        want_dvr = true;
        dvr_base = st.tma_aux2;
        dvr_rows = st.tma_rows;
      }
      if (st.tma_probs && st.tma_kind == 6) {
        want_dv = true;
        dv_base = st.tma_aux;
        dv_rows = st.tma_rows;
      }
      if (st.tma_probs && st.tma_kind == 4) {
        want_ss = true;
        ss_rows = std::max(ss_rows, st.tma_rows);
      }
    }
    const i64 n = plan.n, n2 = n * n;
    std::string err;
    const i64 xrows = plan.buf_size[BUF_JK] / std::max<i64>(1, n);
    // with f_on_tc the same-head operators (BUF_F) follow the integral matrices in the same split array
    const i64 frows = f_on_tc ? plan.buf_size[BUF_F] / std::max<i64>(1, n) : 0;
    if ((want_dd && plan.nD > 0) || (want_ss && xrows > 0)) {  // the integral matrices, split once
      const i64 ld = tci_gtma_host::pitch(n);
      alloc_f(&jk_hi, (size_t)((xrows + frows) * ld));
      alloc_f(&jk_lo, (size_t)((xrows + frows) * ld));
      TCI_CUDA(tci_gtma_host::split(buf[BUF_JK], xrows, n, n, jk_hi, jk_lo, stream));
      if (frows > 0)
        TCI_CUDA(tci_gtma_host::split(buf[BUF_F], frows, n, n, jk_hi + xrows * ld, jk_lo + xrows * ld, stream));
    }
    if ((want_dd || want_1x) && plan.nD > 0) {  // the pair matrices, split every build
      const i64 ld = tci_gtma_host::pitch(n), drows = plan.nD * n;
      alloc_f(&d_hi, (size_t)(drows * ld));
      alloc_f(&d_lo, (size_t)(drows * ld));
    }
    if (want_dd && plan.nD > 0) {
      const i64 drows = plan.nD * n;
      if (!tci_gtma_host::prepare(tma_dd, jk_hi, jk_lo, xrows + frows, n, d_hi, d_lo, drows, n, tma_wide(1), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_dd_ready = true;
    }
    const i64 wvrows = plan.buf_size[BUF_WV] / std::max<i64>(1, n);
    if (want_1x && plan.nD > 0 && wvrows > 0) {  // the one-external coupling vectors, split once
      const i64 ld = tci_gtma_host::pitch(n), drows = plan.nD * n;
      alloc_f(&wv_hi, (size_t)(wvrows * ld));
      alloc_f(&wv_lo, (size_t)(wvrows * ld));
      TCI_CUDA(tci_gtma_host::split(buf[BUF_WV], wvrows, n, n, wv_hi, wv_lo, stream));
      if (!tci_gtma_host::prepare(tma_1x, wv_hi, wv_lo, wvrows, n, d_hi, d_lo, drows, n, tma_wide(5), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_1x_ready = true;
    }
    if (want_ss && xrows > 0 && ss_rows > 0) {
      const i64 ld = tci_gtma_host::pitch(n);
      alloc_f(&cg_hi, (size_t)(ss_rows * ld));
      alloc_f(&cg_lo, (size_t)(ss_rows * ld));
      if (!tci_gtma_host::prepare(tma_ss, jk_hi, jk_lo, xrows, n, cg_hi, cg_lo, ss_rows, n, tma_wide(4), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_ss_ready = true;
    }
    if ((want_t3 || want_dv) && plan.nD > 0) {  // pair matrices as rows of n^2, split every build
      const i64 ld = tci_gtma_host::pitch(n2);
      alloc_f(&df_hi, (size_t)(plan.nD * ld));
      alloc_f(&df_lo, (size_t)(plan.nD * ld));
    }
    if (want_dv && plan.nD > 0 && dv_rows > 0) {  // the exchange bank of the dv step, split once
      const i64 ld = tci_gtma_host::pitch(n2);
      alloc_f(&kb_hi, (size_t)(dv_rows * ld));
      alloc_f(&kb_lo, (size_t)(dv_rows * ld));
      TCI_CUDA(tci_gtma_host::split(buf[BUF_JK] + dv_base, dv_rows, n2, n2, kb_hi, kb_lo, stream));
      if (!tci_gtma_host::prepare(tma_dv, kb_hi, kb_lo, dv_rows, n2, df_hi, df_lo, plan.nD, n2, tma_wide(6), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_dv_ready = true;
    }
    if (want_dvr && plan.nD > 0 && dvr_rows > 0) {  // transposed exchange bank, once; transposed G2 per build
      const i64 ld = tci_gtma_host::pitch(dvr_rows);
      alloc_f(&kbt_hi, (size_t)(n2 * ld));
      alloc_f(&kbt_lo, (size_t)(n2 * ld));
      alloc_f(&g2t_hi, (size_t)(plan.nD * ld));
      alloc_f(&g2t_lo, (size_t)(plan.nD * ld));
      TCI_CUDA(tci_gtma_host::split_transposed(buf[BUF_JK] + dvr_base, 1, dvr_rows, n2, kbt_hi, kbt_lo, stream));
      if (!tci_gtma_host::prepare(tma_dvr, kbt_hi, kbt_lo, n2, dvr_rows, g2t_hi, g2t_lo, plan.nD, dvr_rows,
                                  tma_wide(7), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_dvr_ready = true;
    }
    if (want_t3 && plan.nD > 0) {
      const i64 ld = tci_gtma_host::pitch(n2), vrows = plan.nint * n;
      alloc_f(&v_hi, (size_t)(vrows * ld));
      alloc_f(&v_lo, (size_t)(vrows * ld));
      TCI_CUDA(tci_gtma_host::split(buf[BUF_V], vrows, n2, n2, v_hi, v_lo, stream));
      if (!tci_gtma_host::prepare(tma_t3, v_hi, v_lo, vrows, n2, df_hi, df_lo, plan.nD, n2, tma_wide(2), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_t3_ready = true;
    }
    if (want_t3r && plan.nD > 0) {
      // V_i transposed once (static operator); the gathered coefficients are split every sigma build
      const i64 ld = tci_gtma_host::pitch(n), vtrows = plan.nint * n2, urows = plan.nint * plan.nD;
      alloc_f(&vt_hi, (size_t)(vtrows * ld));
      alloc_f(&vt_lo, (size_t)(vtrows * ld));
      alloc_f(&u3_hi, (size_t)(urows * ld));
      alloc_f(&u3_lo, (size_t)(urows * ld));
      TCI_CUDA(tci_gtma_host::split_transposed(buf[BUF_V], plan.nint, n, n2, vt_hi, vt_lo, stream));
      if (!tci_gtma_host::prepare(tma_t3r, vt_hi, vt_lo, vtrows, n, u3_hi, u3_lo, urows, n, tma_wide(3), err))
        throw Error(TCI_ERR_CUDA, err);
      tma_t3r_ready = true;
    }
    TCI_CUDA(cudaMemsetAsync(tc_status, 0, sizeof(int), stream));
    if (allext) {
      TCI_CUDA(tci_tc_host::convert_w(buf[BUF_W], np, w32p, stream));
      if (nm > 0) TCI_CUDA(tci_tc_host::convert_w(buf[BUF_W] + np * np, nm, w32m, stream));
    }
    TCI_CUDA(cudaStreamSynchronize(stream));
    if (plan.n_sing > 0 && !tci_tc_host::prepare(tc_sing, w32p, np, u2s, plan.n_sing, buf[BUF_T0] + plan.allext_ys, tc_status, tc_kblock, err))
      throw Error(TCI_ERR_CUDA, err);
    if (plan.n_trip > 0 && nm > 0 &&
        !tci_tc_host::prepare(tc_trip, w32m, nm, u2t, plan.n_trip, buf[BUF_T0] + plan.allext_yt, tc_status, tc_kblock, err))
      throw Error(TCI_ERR_CUDA, err);
    if (refine != 1 && buf[BUF_W]) {  // the FP64 W is only needed for the plain-FP64 finish of the roots
      std::lock_guard<std::mutex> lk(g_capture_free_mu);
      TCI_CUDA(dev_free(buf[BUF_W], stream));
      bytes_held -= (double)plan.buf_size[BUF_W] * sizeof(double);
      buf[BUF_W] = nullptr;
    }
  }

  // One plain-FP64 sigma build in a mixed-precision context (the steps launched
  // one by one, outside the context's graph): d_s = H d_c.
  void sigma_of_fp64(const double* d_c, double* d_s) {
    const i64 n = plan.total_csfs;
    const bool tc_allext = (refine == 2 || refine == 3) && precision == 1;
    if (!buf[BUF_W] && !tc_allext && !local)
      throw Error(TCI_ERR_INTERNAL, "the FP64 operators of this context were released");
    if (local) {
      local_in(d_c);
    } else {
      TCI_CUDA(cudaMemcpyAsync(buf[BUF_C], d_c, n * sizeof(double), cudaMemcpyDeviceToDevice, stream));
      if (gen_s) scale_by<<<sm_count() * 8, 256, 0, stream>>>(buf[BUF_C], gen_s, n);
      TCI_CUDA(cudaMemsetAsync(buf[BUF_S], 0, n * sizeof(double), stream));
    }
    const int64_t saved = precision;
    precision = 0;
    allext_tc_in_fp64 = tc_allext;
    try {
      record_steps(false, false);
    } catch (...) {
      precision = saved;
      allext_tc_in_fp64 = false;
      throw;
    }
    launch_count += sigma_launches();
    precision = saved;
    allext_tc_in_fp64 = false;
    if (local) local_out(d_c, d_s);
    else gen_out(d_s);
  }

  // Status word of the bounded waits inside the tensor-core kernel.
  void check_tc_status() {
    if (!tc_status) return;
    int st = 0;
    TCI_CUDA(cudaMemcpy(&st, tc_status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) throw Error(TCI_ERR_TIMEOUT, "tensor-core kernel: a bounded wait gave up (code " + std::to_string(st) + ")");
  }

  // the range lies in an allocated buffer (no throw: usable inside parallel loops)
  bool range_ok(int b, i64 off, i64 len) const {
    return b >= 0 && b < NUM_BUFS && buf[b] && off >= 0 && len >= 0 && off + len <= plan.buf_size[b];
  }
  void check_range(int b, i64 off, i64 len) const {
    if (b < 0 || b >= NUM_BUFS || off < 0 || len < 0 || off + len > plan.buf_size[b])
      throw Error(TCI_ERR_INTERNAL, "plan range outside its buffer");
  }

  void run(const DevStep& s) {
    try {
      run_step(s);
    } catch (const Error& e) {
      throw Error(e.code, "plan step '" + s.name + "': " + e.what());
    }
  }

  void run_step(const DevStep& s) {
    // the tensor-core form writes the all-external products directly
    const bool tc_allext = precision == 1 || allext_tc_in_fp64;
    if (tc_allext && (s.name == "all-external zero" || s.name == "all-external split-k sum")) return;
    if (s.d3_skip) return;
    if (s.d1 == 1) {  // local deck: the forward one-external term on the domains
      if (s.d1_nrows > 0) dom1_forward<<<(unsigned)s.d1_nrows, 128, 0, stream>>>(s.d1_rows, plan.n);
      return;
    }
    if (s.d1 == 2) {  // local deck: the reverse one-external term on the domains
      if (s.d1_tiles > 0) dom1_reverse<<<(unsigned)s.d1_tiles, 256, 0, stream>>>(s.d1_tg, s.d1_ntg, plan.n);
      return;
    }
    if (s.dv == 1) {  // local deck: the forward N-2 <-> valence term on the domains
      if (s.dv_nent > 0)
        dom_dv_forward<<<(unsigned)((s.dv_nent + 7) / 8), 256, 0, stream>>>(s.dv_ent, s.dv_nent, s.dv_k, buf[BUF_D],
                                                                            s.dv_vals, plan.n, plan.nD);
      return;
    }
    if (s.dv == 2) {  // local deck: the reverse N-2 <-> valence term on the domains
      if (s.dv_tiles > 0)
        dom_dv_reverse<<<(unsigned)s.dv_tiles, 256, 0, stream>>>(s.dv_tg, s.dv_ntg, s.dv_pq, s.dv_k, s.dv_vals,
                                                                  buf[BUF_R], plan.n, plan.nD);
      return;
    }
    if (s.d3 == 1) {  // local deck: the forward three-external term on the domains
      if (s.d3f_n > 0) {
        static bool attr_set[64] = {};
        int dev = 0;
        TCI_CUDA(cudaGetDevice(&dev));
        if (s.d3f_smem > 48 * 1024 && dev < 64 && !attr_set[dev]) {
          TCI_CUDA(cudaFuncSetAttribute(dom3_forward, cudaFuncAttributeMaxDynamicSharedMemorySize, 200 * 1024));
          attr_set[dev] = true;
        }
        dom3_forward<<<(unsigned)s.d3f_n, 256, s.d3f_smem, stream>>>(s.d3f, buf[BUF_V], buf[BUF_D], s.d3_rows, plan.n,
                                                                    plan.nD);
      }
      return;
    }
    if (s.d3 == 2) {  // local deck: the reverse three-external term on the domains
      if (s.d3r_tiles > 0)
        dom3_reverse<<<(unsigned)s.d3r_tiles, D3R_T, 0, stream>>>(s.d3r, s.d3r_n, s.d3e, buf[BUF_V], s.d3_rows,
                                                                  buf[BUF_R], plan.n, plan.nD);
      return;
    }
    switch (s.kind) {
      case STEP_GEMM:
        if (s.com_step) {  // local deck: the two-external step on the domains
          if (s.com_ngather > 0)
            com_gather_sq<<<(unsigned)s.com_ngather, 256, 0, stream>>>(s.com_gather, plan.n);
          if (s.com_ntiles > 0) {
            TCI_CUDA(cudaMemsetAsync(s.com_rsq, 0, (size_t)s.com_rsq_len * sizeof(double), stream));
            gemm_com_f64<<<(unsigned)s.com_ntiles, COM_THREADS, 0, stream>>>(s.com_probs, s.com_nprob, s.com_segs,
                                                                           plan.n);
          }
          if (s.com_nscatter > 0)
            com_scatter_sq<<<(unsigned)s.com_nscatter, 256, 0, stream>>>(s.com_scatter, plan.n);
          break;
        }
        if (tc_allext && s.name == "all-external") {
          run_allext_tc();
          break;
        }
        if (uses_tc(s) && s.skinny_nwarps > 0)
          gemm_skinny_f64<<<(unsigned)((s.skinny_nwarps + 7) / 8), 256, 0, stream>>>(s.skinny_probs, s.skinny_nprob,
                                                                                  s.segs, s.skinny_nwarps);
        // finish mode 3: the three-external contractions stay on the tensor cores too
        if ((uses_tc(s) || (allext_tc_in_fp64 && refine == 3 && (s.tma_kind == 2 || s.tma_kind == 3))) &&
            s.tma_probs && tma_ok(s)) {
          const i64 n = plan.n;
          if (s.tma_kind == 1) {
            if (!f_on_tc) TCI_CUDA(tci_dev::launch_gemm_f64(s.cfg, s.probs_f, s.nprob_f, s.segs_f, s.ntiles_f, stream));
            TCI_CUDA(tci_gtma_host::split(buf[BUF_D], plan.nD * n, n, n, d_hi, d_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_dd, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else if (s.tma_kind == 2) {
            TCI_CUDA(tci_gtma_host::split(buf[BUF_D], plan.nD, n * n, n * n, df_hi, df_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_t3, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else if (s.tma_kind == 7) {
            TCI_CUDA(tci_gtma_host::split_transposed(buf[BUF_T0] + s.tma_aux, 1, s.tma_rows, plan.nD, g2t_hi, g2t_lo,
                                                     stream));
            TCI_CUDA(tci_gtma_host::launch(tma_dvr, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else if (s.tma_kind == 6) {
            TCI_CUDA(tci_gtma_host::split(buf[BUF_D], plan.nD, n * n, n * n, df_hi, df_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_dv, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else if (s.tma_kind == 5) {
            TCI_CUDA(tci_gtma_host::split(buf[BUF_D], plan.nD * n, n, n, d_hi, d_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_1x, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else if (s.tma_kind == 4) {
            TCI_CUDA(tci_gtma_host::split(buf[BUF_T0] + s.tma_aux, s.tma_rows, n, n, cg_hi, cg_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_ss, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          } else {
            TCI_CUDA(tci_gtma_host::split(buf[BUF_T0] + s.tma_aux, plan.nint * plan.nD, n, n, u3_hi, u3_lo, stream));
            TCI_CUDA(tci_gtma_host::launch(tma_t3r, s.tma_probs, s.tma_nprob, s.tma_segs, s.tma_ntiles, (int)tc_kblock,
                                           tc_status, stream));
          }
          break;
        }
        if (uses_tc(s)) {
          TCI_CUDA(tci_dev::launch_gemm_f64(s.cfg, s.probs_f, s.nprob_f, s.segs_f, s.ntiles_f, stream));
          TCI_CUDA(tci_gtc_host::launch(s.probs_tc, s.nprob_tc, s.segs_tc, s.ntiles_tc, tc_status, (int)tc_kblock, stream));
          break;
        }
        if (s.skinny_nwarps > 0)
          gemm_skinny_f64<<<(unsigned)((s.skinny_nwarps + 7) / 8), 256, 0, stream>>>(s.skinny_probs, s.skinny_nprob,
                                                                                  s.segs, s.skinny_nwarps);
        launch_panel<16>(s, 0);
        launch_panel<24>(s, 1);
        launch_panel<32>(s, 2);
        launch_panel<40>(s, 3);
        launch_panel<48>(s, 4);
        launch_panel<56>(s, 5);
        launch_panel<64>(s, 6);
        launch_cp<0>(s);
        launch_cp<1>(s);
        if (s.ntiles > 0) {
          if (s.cfg == 0) gemm_tiled_f64<64, 128, 4, 8><<<(unsigned)s.ntiles, 256, 0, stream>>>(s.probs, s.nprob, s.segs);
          else gemm_tiled_f64<128, 64, 8, 4><<<(unsigned)s.ntiles, 256, 0, stream>>>(s.probs, s.nprob, s.segs);
        }
        break;
      case STEP_AXPY:
        if (s.ntg > 0) {
          if (s.axpy_pairs) axpy_segments<true><<<(unsigned)s.ntg, 256, 0, stream>>>(s.at, s.ntg, s.as);
          else axpy_segments<false><<<(unsigned)s.ntg, 256, 0, stream>>>(s.at, s.ntg, s.as);
        }
        if (s.zc_ntg > 0) axpy_common<<<(unsigned)s.zc_ntg, 256, 0, stream>>>(s.zc_tg, s.zc_src);
        break;
      case STEP_DOT:
        if (s.ntg > 0) dot_segments<<<(unsigned)s.ntg, 256, 0, stream>>>(s.dt, s.ntg, s.ds);
        break;
      case STEP_ZERO:
        if (s.zlen > 0) TCI_CUDA(cudaMemsetAsync(s.zptr, 0, s.zlen * sizeof(double), stream));
        break;
      case STEP_UNPACK:
        if (plan.nD > 65535) throw Error(TCI_ERR_INPUT, "too many dense pair matrices for one launch");
        if (plan.nD > 0) {
          dim3 g((unsigned)std::min<long long>(64, (plan.n * plan.n + 255) / 256), (unsigned)plan.nD);
          unpack_pairs<<<g, 256, 0, stream>>>(dheads, dk_head, plan.nD, plan.n, buf[BUF_C], buf[BUF_D]);
        }
        break;
      case STEP_PACK:
        if (plan.nD > 0) {
          dim3 g((unsigned)std::min<long long>(64, (plan.n * plan.n / 2 + 255) / 256 + 1), (unsigned)plan.nD);
          pack_pairs<<<g, 256, 0, stream>>>(dheads, dk_head, plan.nD, plan.n, buf[BUF_R], buf[BUF_S]);
        }
        break;
      case STEP_WBUILD:
        build_allext<<<sm_count() * 16, 256, 0, stream>>>(buf[BUF_X], plan.n, buf[BUF_W]);
        break;
    }
    TCI_CUDA(cudaGetLastError());
  }
};

namespace tci_dev {
cudaError_t launch_gemm_cp_f64(const DGemmProblem* probs, int nprob, const DGemmSeg* segs, long long ntiles,
                               cudaStream_t st) {
  if (ntiles <= 0 || nprob <= 0) return cudaSuccess;
  constexpr size_t smem = cp_smem_bytes<0>();
  static bool attr_set[64] = {};  // per device
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && !attr_set[dev]) {
    e = cudaFuncSetAttribute(gemm_cp_f64<0>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    attr_set[dev] = true;
  }
  gemm_cp_f64<0><<<(unsigned)ntiles, 256, smem, st>>>(probs, nprob, segs);
  return cudaGetLastError();
}

cudaError_t launch_gemm_f64(int cfg, const DGemmProblem* probs, int nprob, const DGemmSeg* segs, long long ntiles,
                            cudaStream_t st) {
  if (ntiles <= 0 || nprob <= 0) return cudaSuccess;
  if (cfg == 0) gemm_tiled_f64<64, 128, 4, 8><<<(unsigned)ntiles, 256, 0, st>>>(probs, nprob, segs);
  else gemm_tiled_f64<128, 64, 8, 4><<<(unsigned)ntiles, 256, 0, st>>>(probs, nprob, segs);
  return cudaGetLastError();
}
}  // namespace tci_dev

extern "C" {

static int init_impl(const tci_deck* deck, const tci_operator* op, int64_t device, int64_t precision, int64_t kblock,
                     tci_ctx** out, int64_t refine = 2);

int tci_sigma_init(const tci_deck* deck, const tci_operator* op, int64_t device, tci_ctx** out) {
  return init_impl(deck, op, device, 0, 128, out);
}

int tci_sigma_init_ex(const tci_deck* deck, const tci_operator* op, int64_t device, const int64_t* options,
                      int64_t n_options, tci_ctx** out) {
  int64_t precision = 0, kblock = 128, tc_mode = 0, refine = 2;
  if (options && n_options > 0) precision = options[0];
  if (options && n_options > 1 && options[1] > 0) kblock = options[1];
  if (options && n_options > 2) tc_mode = options[2];
  if (options && n_options > 3) refine = options[3];
  if (precision < 0 || precision > 1 || tc_mode < 0 || tc_mode > 2 || refine < 0 || refine > 3) {
    set_error("unknown precision mode, tensor-core GEMM selection or finish");
    return TCI_ERR_ARG;
  }
  const int rc = init_impl(deck, op, device, precision, kblock, out, refine);
  if (rc == TCI_OK) tci::ctx_set_tc_gemms(*out, tc_mode);
  return rc;
}

static int init_impl(const tci_deck* deck, const tci_operator* op, int64_t device, int64_t precision, int64_t kblock,
                     tci_ctx** out, int64_t refine) {
  if (!out) return TCI_ERR_ARG;
  *out = nullptr;
  try {
    auto t0 = std::chrono::steady_clock::now();
    CsfSpace sp;
    Plan plan;
    if (deck && (deck->nm1_domain_ptr || deck->nm2_domain_ptr)) {
      // local pair domains: the plan on the non-local space of the same deck, the local layout mapped onto it
      tci::LocalSetup ls;
      build_space_from_c(deck, ls.loc);
      tci_deck nl = *deck;
      nl.nm1_domain_ptr = nl.nm1_domain_idx = nl.nm2_domain_ptr = nl.nm2_domain_idx = nullptr;
      build_space_from_c(&nl, sp);
      Operator o;
      operator_from_c(op, sp, o);
      tci::build_local_setup(ls.loc, sp, o, ls);
      build_plan(sp, o, plan, false);
      const int rc = tci::ctx_from_plan(std::move(sp), std::move(plan), o.chol, device, precision, kblock, out, refine,
                                        &ls);
      if (rc == TCI_OK) (*out)->init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
      return rc;
    }
    build_space_from_c(deck, sp);
    Operator o;
    operator_from_c(op, sp, o);
    // The host builds the sigma tables on a second thread while the device builds the integral banks from the
    // operator part of the plan (the same leading set-up steps the whole plan starts with).
    // The coupling-vector rows are complete before the zero-external blocks (the last long phase): they go up
    // while the host builds those.
    Plan early;
    tci::build_plan_operator_part(sp, o, early);
    std::exception_ptr plan_error, wv_error;
    std::promise<std::pair<const double*, size_t>> wv_ready;
    std::future<std::pair<const double*, size_t>> wv_rows = wv_ready.get_future();
    std::thread planner([&]() {
      try {
        build_plan(sp, o, plan, true, [&](const Plan& P) { wv_ready.set_value({P.wv.data(), P.wv.size()}); });
      } catch (...) {
        plan_error = std::current_exception();
      }
      try {
        wv_ready.set_value({nullptr, 0});  // the plan failed before its rows were complete
      } catch (const std::future_error&) {
      }
    });
    tci_ctx* started = nullptr;
    const int rc0 = tci::ctx_begin_operator(early, o.chol, device, precision, kblock, refine, &started);
    const auto wv = wv_rows.get();
    if (rc0 == TCI_OK && started && wv.first && wv.second > 0) {
      try {
        tci::ctx_upload_wv(started, wv.first, wv.second);
      } catch (...) {
        wv_error = std::current_exception();
      }
    }
    planner.join();
    if (plan_error || wv_error || rc0 != TCI_OK) {
      if (started) tci_destroy(started);
      if (plan_error) std::rethrow_exception(plan_error);
      if (wv_error) std::rethrow_exception(wv_error);
      return rc0;
    }
    const int rc = tci::ctx_from_plan(std::move(sp), std::move(plan), o.chol, device, precision, kblock, out, refine,
                                      nullptr, started);
    if (rc == TCI_OK) (*out)->init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return rc;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

}  // extern "C"

namespace tci {

void ctx_device_bytes(const Plan& P, int64_t precision, double* peak, double* resident, int64_t refine) {
  double all = 0, init_only = 0;
  for (int b = 0; b < NUM_BUFS; ++b) {
    const double bytes = (double)std::max<i64>(0, P.buf_size[b]) * 8.0;
    all += bytes;
    if (b == BUF_X || b == BUF_L || b == BUF_LE || b == BUF_LI) init_only += bytes;
  }
  // tables (steps, heads) are small next to the buffers; the diagonal is built on first use
  const double diag = 8.0 * (double)P.total_csfs;
  double pk = all, res = all - init_only + diag;
  if (precision == 1) {
    const double f32 = 4.0 * ((double)tci_tc_host::w32_floats(P.np) +
                              (P.nm > 0 ? (double)tci_tc_host::w32_floats(P.nm) : 0.0) +
                              2.0 * (double)tci_tc_host::padded_rows(std::max<i64>(1, P.n_sing)) *
                                  tci_tc_host::padded_ld(P.np) +
                              (P.nm > 0 ? 2.0 * (double)tci_tc_host::padded_rows(std::max<i64>(1, P.n_trip)) *
                                              tci_tc_host::padded_ld(P.nm)
                                        : 0.0) +
                              // split integrals and pair matrices of the TMA-fed two-external step
                              2.0 * (double)tci_gtma_host::pitch(P.n) *
                                  (double)(P.buf_size[BUF_JK] / std::max<i64>(1, P.n) + P.nD * P.n) +
                              2.0 * (double)tci_gtma_host::pitch(P.n * P.n) * (double)(P.nint * P.n + P.nD) +
                              // transposed V_i and the gathered coefficients of the reverse three-external step
                              2.0 * (double)tci_gtma_host::pitch(P.n) * (double)(P.nint * P.n * P.n + P.nint * P.nD) +
                              // one-external coupling vectors
                              2.0 * (double)tci_gtma_host::pitch(P.n) *
                                  (double)(P.buf_size[BUF_WV] / std::max<i64>(1, P.n)));
    // the same-head operators beside the integrals in the split array (mixed form with a finish)
    const double f32_f =
        refine != 0 ? 4.0 * 2.0 * (double)tci_gtma_host::pitch(P.n) * (double)(P.buf_size[BUF_F] / std::max<i64>(1, P.n)) : 0.0;
    // gathered single-vector rows of the singles-singles step (problems above the skinny size)
    double ss_rows = 0, dv_rows = 0;
    for (const auto& st : P.sigma_steps) {
      if (st.name == "ss two-external")
        for (const auto& g : st.gp)
          if (g.M > SKINNY_M) ss_rows += (double)g.M;
      if (st.name == "dv forward" && !st.gp.empty()) dv_rows = (double)st.gp[0].M;  // the exchange bank's rows
    }
    const double f32_all = f32 + f32_f + 4.0 * 2.0 * (double)tci_gtma_host::pitch(P.n) * ss_rows +
                           4.0 * 2.0 * (double)tci_gtma_host::pitch(P.n * P.n) * dv_rows +
                           4.0 * 2.0 * (double)tci_gtma_host::pitch((i64)dv_rows) * (double)(P.n * P.n + P.nD);
    pk = std::max(pk, res + f32_all);  // FP64 and FP32 operators coexist until the FP64 copy is released
    res += f32_all - (refine == 1 ? 0.0 : 8.0 * (double)std::max<i64>(0, P.buf_size[BUF_W]));
  }
  *peak = std::max(pk, res);
  *resident = res;
}

void ctx_set_tc_gemms(tci_ctx* ctx, int64_t mode) {
  if (ctx) ctx->tc_mode = mode;
}

void build_local_setup(const CsfSpace& loc, const CsfSpace& nl, const Operator& op, LocalSetup& ls) {
  build_local_structure(loc, nl, ls);
  const i64 n = nl.n_ext, nint = nl.n_int, N = op.nchol;
  // (aa|cc) and (ac|ca) over the externals, for the all-external part of the diagonal
  ls.xdiag.assign((size_t)(2 * n * n), 0.0);
  auto row = [&](i64 p, i64 q) {
    const i64 P = nint + std::max(p, q), Q = nint + std::min(p, q);
    return op.chol + (P * (P + 1) / 2 + Q) * N;
  };
#pragma omp parallel for schedule(dynamic, 4)
  for (i64 a = 0; a < n; ++a)
    for (i64 c = 0; c < n; ++c) {
      const double *la = row(a, a), *lc = row(c, c), *lx = row(a, c);
      double s1 = 0.0, s2 = 0.0;
      for (i64 J = 0; J < N; ++J) s1 += la[J] * lc[J], s2 += lx[J] * lx[J];
      ls.xdiag[(size_t)(a * n + c)] = s1;
      ls.xdiag[(size_t)(n * n + a * n + c)] = s2;
    }
}

void build_local_structure(const CsfSpace& loc, const CsfSpace& nl, LocalSetup& ls) {
  const i64 n = nl.n_ext, nab = n * (n - 1) / 2, nint = nl.n_int;
  if (loc.n_ext != n || loc.n_int != nint) throw Error(TCI_ERR_INTERNAL, "local and non-local spaces differ in shape");
  ls.map.assign((size_t)loc.total_csfs, -1);
  for (int k = 0; k < 3; ++k) {
    if (loc.paths[k].size() != nl.paths[k].size()) throw Error(TCI_ERR_INTERNAL, "local and non-local heads differ");
    for (size_t p = 0; p < loc.paths[k].size(); ++p) {
      const Head &h = loc.paths[k][p], &g = nl.paths[k][p];
      if (h.occ != g.occ) throw Error(TCI_ERR_INTERNAL, "local and non-local heads differ");
      if (k == 0) {
        if (h.off >= 0)
          for (i64 f = 0; f < h.nsf; ++f) ls.map[(size_t)(h.off + f)] = g.off + f;
        continue;
      }
      if (h.domain < 0) continue;
      const std::vector<int>& D = loc.domains[(size_t)h.domain];
      const i64 m = (i64)D.size(), mab = m * (m - 1) / 2;
      if (k == 1) {
        if (h.off < 0 || m == 0) continue;
        if (g.off < 0 || g.nsf != h.nsf) throw Error(TCI_ERR_INTERNAL, "N-1 block missing in the non-local space");
        for (i64 f = 0; f < h.nsf; ++f)
          for (i64 a = 0; a < m; ++a) ls.map[(size_t)(h.off + f * m + a)] = g.off + f * n + D[(size_t)a];
        continue;
      }
      if (h.off >= 0 && mab > 0) {
        if (g.off < 0 || g.nsf != h.nsf) throw Error(TCI_ERR_INTERNAL, "N-2 block missing in the non-local space");
        for (i64 f = 0; f < h.nsf; ++f)
          for (i64 i = 1; i < m; ++i)
            for (i64 j = 0; j < i; ++j) {
              const i64 I = D[(size_t)i], J = D[(size_t)j];  // sorted: I > J
              ls.map[(size_t)(h.off + f * mab + i * (i - 1) / 2 + j)] = g.off + f * nab + I * (I - 1) / 2 + J;
            }
      }
      if (h.off_aa >= 0 && m > 0) {
        if (g.off_aa < 0 || g.nsf_aa != h.nsf_aa) throw Error(TCI_ERR_INTERNAL, "N-2 aa block missing");
        for (i64 f = 0; f < h.nsf_aa; ++f)
          for (i64 a = 0; a < m; ++a) ls.map[(size_t)(h.off_aa + f * m + a)] = g.off_aa + f * n + D[(size_t)a];
      }
      // the pair-domain all-external term of this head (tci_local heads: off_ab, off_aa, nsf_ab, nsf_aa,
      // nsing, dom_off, dom_len)
      const i64 nsf_ab = (h.off >= 0 && mab > 0) ? h.nsf : 0, nsf_aa = (h.off_aa >= 0 && m > 0) ? h.nsf_aa : 0;
      if (nsf_ab == 0 && nsf_aa == 0) continue;
      ls.heads7.insert(ls.heads7.end(), {nsf_ab ? h.off : 0, nsf_aa ? h.off_aa : 0, nsf_ab, nsf_aa,
                                         nsf_aa > 0 ? (i64)loc.fsn[(size_t)h.singles] : 0, (i64)ls.dom_idx.size(), m});
      ls.heads_lex.push_back(h.lex);
      for (int a : D) ls.dom_idx.push_back(a);
    }
  }
  for (i64 x : ls.map)
    if (x < 0) throw Error(TCI_ERR_INTERNAL, "a local CSF has no non-local counterpart");
  // domains of the N-1 heads by their CSF rows in the non-local space
  for (size_t p = 0; p < nl.paths[1].size(); ++p) {
    const Head& g = nl.paths[1][p];
    if (!g.kept || g.off < 0 || g.nsf <= 0) continue;
    const Head& h = loc.paths[1][p];
    ls.s1_begin.push_back(g.off);
    ls.s1_end.push_back(g.off + (i64)g.nsf * n);
    ls.s1_off.push_back((int64_t)ls.s1_dom.size());
    if (h.domain >= 0 && h.off >= 0)
      for (int a : loc.domains[(size_t)h.domain]) ls.s1_dom.push_back(a);
    ls.s1_len.push_back((int64_t)ls.s1_dom.size() - ls.s1_off.back());
  }
  // domains of the plan's N-2 heads, in the plan's head order (Builder::setup_heads: kept heads with a
  // pair matrix)
  for (size_t p = 0; p < nl.paths[2].size(); ++p) {
    const Head& g = nl.paths[2][p];
    if (!g.kept) continue;
    const i64 nab_f = g.off >= 0 ? g.nsf : 0, naa_f = g.off_aa >= 0 ? g.nsf_aa : 0;
    if (std::max(nab_f, naa_f) == 0) continue;
    const Head& h = loc.paths[2][p];
    ls.dh_off.push_back((int64_t)ls.dh_dom.size());
    if (h.domain >= 0 && (h.off >= 0 || h.off_aa >= 0)) {
      for (int a : loc.domains[(size_t)h.domain]) ls.dh_dom.push_back(a);
    }
    ls.dh_len.push_back((int64_t)ls.dh_dom.size() - ls.dh_off.back());
  }
}

namespace setup {
// TCI_INIT_TIMING=1 prints the device set-up phases (each ends with a stream synchronisation)
struct InitTimer {
  bool on = std::getenv("TCI_INIT_TIMING") != nullptr;
  std::chrono::steady_clock::time_point tp = std::chrono::steady_clock::now();
  void operator()(const char* what, cudaStream_t st) {
    if (!on) return;
    cudaStreamSynchronize(st);
    const auto now = std::chrono::steady_clock::now();
    std::fprintf(stderr, "init %-28s %.3f s\n", what, std::chrono::duration<double>(now - tp).count());
    tp = now;
  }
};

// A context with its device and stream, nothing allocated.
std::unique_ptr<tci_ctx> new_ctx(int64_t device) {
  std::unique_ptr<tci_ctx> ctx(new tci_ctx());
  int ndev = 0;
  TCI_CUDA(cudaGetDeviceCount(&ndev));
  if (device < 0 || device >= ndev) throw Error(TCI_ERR_CUDA, "requested device is not available");
  ctx->device = (int)device;
  TCI_CUDA(cudaSetDevice(ctx->device));
  TCI_CUDA(cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking));
  TCI_CUDA(cudaEventCreate(&ctx->ev0));
  TCI_CUDA(cudaEventCreate(&ctx->ev1));
  return ctx;
}

// Allocates (zeroed) every buffer of the context's plan that is not allocated yet.
void alloc_plan_buffers(tci_ctx* ctx) {
  const Plan& P = ctx->plan;
  for (int b = 0; b < NUM_BUFS; ++b) {
    if (P.buf_size[b] <= 0 || ctx->buf[b]) continue;
    cudaError_t e = dev_malloc(&ctx->buf[b], P.buf_size[b] * sizeof(double), ctx->stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      throw Error(TCI_ERR_MEMORY, std::string("device allocation failed: ") + cudaGetErrorString(e));
    }
    // plan steps accumulate into their targets: every buffer starts at zero
    TCI_CUDA(cudaMemsetAsync(ctx->buf[b], 0, P.buf_size[b] * sizeof(double), ctx->stream));
    ctx->bytes_held += (double)P.buf_size[b] * sizeof(double);
  }
}

// Lowers and runs the plan's set-up steps from index `first` on.  In the mixed form without the plain-FP64
// finish the exchange product X = Lpk Lpk^T of the all-external operators (the largest set-up GEMM,
// 2 npk^2 N flops) runs on the TMA-fed tensor-core kernel; its 3xTF32 error is of the order of W's own FP32
// rounding in that form.  The other banks stay FP64.
void run_init_steps(tci_ctx* ctx, size_t first, bool x_tc, int64_t kblock, InitTimer& phase) {
  const Plan& P = ctx->plan;
  GemmProblem xg{};
  GemmSeg xs{};
  bool have_x = false;
  size_t banks = (size_t)-1;
  const size_t lowered0 = ctx->init.size();
  for (size_t i = first; i < P.init_steps.size(); ++i) {
    const Step& s = P.init_steps[i];
    if (x_tc && s.kind == STEP_GEMM && s.name == "integral banks") {
      Step s2 = s;
      for (size_t g = 0; g < s2.gp.size(); ++g)
        if (s2.gp[g].c == BUF_X && s2.gp[g].seg_end - s2.gp[g].seg_begin == 1) {
          xg = s2.gp[g];
          xs = s2.gs[(size_t)xg.seg_begin];
          s2.gp.erase(s2.gp.begin() + (long)g);
          have_x = xs.a == BUF_T0 && xs.b == BUF_T0 && xs.offA == xs.offB && !xs.tA && xs.tB && xg.M == xg.N;
          if (!have_x) s2 = s;  // not the expected shape: leave it on the FP64 kernel
          break;
        }
      banks = ctx->init.size();
      ctx->init.push_back(ctx->lower(s2));
      continue;
    }
    ctx->init.push_back(ctx->lower(s));
  }
  phase("lowering (set-up steps)", ctx->stream);
  for (size_t i = lowered0; i < ctx->init.size(); ++i) {
    ctx->run(ctx->init[i]);
    phase(ctx->init[i].name.c_str(), ctx->stream);
    if (i == banks && have_x) {
      ctx->exchange_product_tc(xg, xs, kblock);
      phase("exchange product (tcgen05)", ctx->stream);
    }
  }
}
}  // namespace setup
using setup::InitTimer;

int ctx_begin_operator(const Plan& early, const double* chol, int64_t device, int64_t precision, int64_t kblock,
                       int64_t refine, tci_ctx** out) {
  if (!out || !chol) return TCI_ERR_ARG;
  *out = nullptr;
  try {
    InitTimer phase;
    std::unique_ptr<tci_ctx> ctx = setup::new_ctx(device);
    ctx->plan = early;
    setup::alloc_plan_buffers(ctx.get());
    TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_L], chol, early.buf_size[BUF_L] * sizeof(double), cudaMemcpyHostToDevice,
                             ctx->stream));
    phase("operator buffers and upload", ctx->stream);
    setup::run_init_steps(ctx.get(), 0, precision == 1 && refine != 1, kblock, phase);
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->early_init = early.init_steps.size();
    for (const auto& st : early.init_steps) {
      ctx->early_names.push_back(st.name);
      ctx->early_shapes.push_back({st.gp.size(), st.gs.size(), st.at.size(), st.as.size()});
    }
    ctx->early_sizes = early.buf_size;
    *out = ctx.release();
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

// The coupling-vector rows (plan.wv) of a started context, uploaded as soon as the host has them.
void ctx_upload_wv(tci_ctx* ctx, const double* wv, size_t n) {
  TCI_CUDA(cudaSetDevice(ctx->device));
  double* p = nullptr;
  cudaError_t e = dev_malloc(&p, n * sizeof(double), ctx->stream);
  if (e != cudaSuccess) {
    cudaGetLastError();
    throw Error(TCI_ERR_MEMORY, std::string("device allocation failed: ") + cudaGetErrorString(e));
  }
  ctx->buf[BUF_WV] = p;
  ctx->bytes_held += (double)n * sizeof(double);
  ctx->early_sizes[BUF_WV] = (i64)n;
  TCI_CUDA(cudaMemcpyAsync(p, wv, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
  TCI_CUDA(cudaStreamSynchronize(ctx->stream));
  ctx->wv_uploaded = true;
}

int ctx_from_plan(CsfSpace&& sp, Plan&& plan, const double* chol, int64_t device, int64_t precision, int64_t kblock,
                  tci_ctx** out, int64_t refine, LocalSetup* ls, tci_ctx* started) {
  std::unique_ptr<tci_ctx> ctx(started);
  if (!out || !chol) return TCI_ERR_ARG;
  *out = nullptr;
  if (precision < 0 || precision > 1) {
    set_error("unknown precision mode");
    return TCI_ERR_ARG;
  }
  try {
    auto t0 = std::chrono::steady_clock::now();
    InitTimer phase;
    const bool timing = phase.on;
    if (ctx) {
      // set-up started from the operator part: its steps must be the plan's leading ones, its buffers the
      // plan's (the scratch buffer grows when the sigma steps need more)
      if (ls || ctx->device != (int)device) throw Error(TCI_ERR_INTERNAL, "started context does not fit the plan");
      TCI_CUDA(cudaSetDevice(ctx->device));
      if (plan.init_steps.size() < ctx->early_init) throw Error(TCI_ERR_INTERNAL, "plan lacks the started steps");
      for (size_t i = 0; i < ctx->early_init; ++i) {
        const Step& st = plan.init_steps[i];
        const std::array<size_t, 4> sh{st.gp.size(), st.gs.size(), st.at.size(), st.as.size()};
        if (st.name != ctx->early_names[i] || sh != ctx->early_shapes[i])
          throw Error(TCI_ERR_INTERNAL, "started set-up steps differ from the plan's");
      }
      for (int b = 0; b < NUM_BUFS; ++b) {
        if (!ctx->buf[b]) continue;
        if (b == BUF_T0 && plan.buf_size[b] > ctx->early_sizes[b]) {
          std::lock_guard<std::mutex> lk(g_capture_free_mu);
          TCI_CUDA(dev_free(ctx->buf[b], ctx->stream));
          ctx->bytes_held -= (double)ctx->early_sizes[b] * sizeof(double);
          ctx->buf[b] = nullptr;
        } else if (plan.buf_size[b] != ctx->early_sizes[b] && b != BUF_T0) {
          throw Error(TCI_ERR_INTERNAL, "started buffer sizes differ from the plan's");
        }
      }
    } else {
      ctx = setup::new_ctx(device);
    }
    ctx->sp = std::move(sp);
    const size_t started_steps = ctx->early_init;
    if (started_steps) {
      // the plan's scratch size may be larger; every other size equals the started one
      const i64 t0size = std::max(plan.buf_size[BUF_T0], ctx->early_sizes[BUF_T0]);
      ctx->plan = std::move(plan);
      if (ctx->buf[BUF_T0]) ctx->plan.buf_size[BUF_T0] = t0size;
    } else {
      ctx->plan = std::move(plan);
    }
    Plan& P = ctx->plan;
    setup::alloc_plan_buffers(ctx.get());
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    if (!started_steps)
      TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_L], chol, P.buf_size[BUF_L] * sizeof(double), cudaMemcpyHostToDevice,
                               ctx->stream));
    TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_JK] + 2 * P.nint * P.nint * P.n * P.n, P.h_vv.data(),
                             P.h_vv.size() * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    if (!P.wv.empty() && !ctx->wv_uploaded)
      TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_WV], P.wv.data(), P.wv.size() * sizeof(double), cudaMemcpyHostToDevice,
                               ctx->stream));
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    std::vector<DHead> dh;
    std::vector<int> dkh;
    for (size_t h = 0; h < P.dheads.size(); ++h) {
      const auto& d = P.dheads[h];
      dh.push_back(DHead{d.off_ab, d.off_aa, d.nsf_ab, d.nsf_aa, d.nsing, d.nD, d.dk0});
      for (i64 k = 0; k < d.nD; ++k) dkh.push_back((int)h);
    }
    ctx->dheads = upload(dh, ctx->owned, ctx->stream);
    ctx->dk_head = upload(dkh, ctx->owned, ctx->stream);
    if (ls) {
      ctx->local = true;
      ctx->n_loc = ls->loc.total_csfs;
      ctx->loc_pos.assign(ls->map.begin(), ls->map.end());
      std::sort(ctx->loc_pos.begin(), ctx->loc_pos.end());
      ctx->d_map = upload(ls->map, ctx->owned, ctx->stream);
      ctx->xdiag = upload(ls->xdiag, ctx->owned, ctx->stream);
      for (double** p : {&ctx->loc_c, &ctx->loc_s}) {
        TCI_CUDA(dev_malloc(p, (size_t)std::max<i64>(1, ctx->n_loc) * sizeof(double), ctx->stream));
        ctx->owned.push_back(*p);
      }
      if (!ls->heads7.empty()) {
        const int64_t opts[4] = {precision, (int64_t)16e9, kblock, 1};
        const int rc = tci_local_create(P.nint, P.n, chol, P.nchol, (int64_t)(ls->heads7.size() / 7), ls->heads7.data(),
                                        ls->dom_idx.data(), ctx->n_loc, device, opts, 4, &ctx->loc_allext);
        if (rc != TCI_OK) throw Error(rc, "pair-domain all-external set-up failed");
      }
      TCI_CUDA(cudaSetDevice(ctx->device));
    }
    phase("buffers and uploads", ctx->stream);
    ctx->f_on_tc = precision == 1 && refine != 0;
    DevStep d3f, d3r;
    const bool dom3 = ls && ctx->lower_dom3(P.sigma_steps, *ls, d3f, d3r);
    DevStep dvf, dvr;
    const bool domdv = ls && ctx->lower_dom_dv(P.sigma_steps, *ls, dvf, dvr);
    DevStep d1f, d1r;
    const bool dom1 = ls && ctx->lower_dom1(P.sigma_steps, *ls, d1f, d1r);
    for (auto& s : P.sigma_steps) {
      if (ls && s.kind == STEP_GEMM && s.name == "dd two-external")
        ctx->sigma.push_back(ctx->lower_dom(s, *ls));
      else if (dom3 && s.name == "three-external forward") {
        DevStep d;
        d.kind = s.kind;
        d.name = s.name;
        d.d3_skip = true;
        ctx->sigma.push_back(d);
      } else if (dom3 && s.name == "three-external split-k sum")
        ctx->sigma.push_back(d3f);
      else if (dom3 && s.name == "three-external reverse")
        ctx->sigma.push_back(d3r);
      else if (dom1 && s.name == "one-external forward")
        ctx->sigma.push_back(d1f);
      else if (dom1 && s.name == "one-external reverse")
        ctx->sigma.push_back(d1r);
      else if (ls && s.kind == STEP_AXPY && s.name == "zero-external")
        ctx->sigma.push_back(ctx->lower_zero_local(s, *ls));
      else if (domdv && s.name == "dv forward") {
        DevStep d;
        d.kind = s.kind;
        d.name = s.name;
        d.d3_skip = true;
        ctx->sigma.push_back(d);
      } else if (domdv && s.name == "dv split-k sum")
        ctx->sigma.push_back(dvf);
      else if (domdv && s.name == "dv reverse")
        ctx->sigma.push_back(dvr);
      else
        ctx->sigma.push_back(ctx->lower(s));
      if (timing) {  // the σ steps whose tables take a noticeable time
        cudaStreamSynchronize(ctx->stream);
        const double dt = std::chrono::duration<double>(std::chrono::steady_clock::now() - phase.tp).count();
        if (dt > 0.002) phase(("  lowering " + s.name).c_str(), ctx->stream);
      }
    }
    phase("lowering (step tables)", ctx->stream);
    setup::run_init_steps(ctx.get(), started_steps, precision == 1 && refine != 1, kblock, phase);
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    // init-only buffers
    for (int b : {BUF_X, BUF_L, BUF_LE, BUF_LI}) {
      if (ctx->buf[b]) {
        std::lock_guard<std::mutex> lk(g_capture_free_mu);
        TCI_CUDA(dev_free(ctx->buf[b], ctx->stream));
        ctx->bytes_held -= (double)P.buf_size[b] * sizeof(double);
        ctx->buf[b] = nullptr;
      }
    }
    if (const char* g = std::getenv("TCI_NO_GRAPH")) ctx->use_graph = (g[0] == '0');
    ctx->precision = precision;
    ctx->tc_kblock = kblock;
    ctx->refine = refine;
    ctx->setup_precision();
    ctx->prepare_local();
    phase("precision set-up", ctx->stream);
    ctx->init_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = ctx.release();
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

}  // namespace tci

extern "C" {

int tci_sigma_device(tci_ctx* ctx, const double* d_c, double* d_sigma, int64_t n, void* stream) {
  if (!ctx || !d_c || !d_sigma) return TCI_ERR_ARG;
  try {
    if (n != ctx->nvec()) throw Error(TCI_ERR_ARG, "vector length differs from total_csfs");
    TCI_CUDA(cudaSetDevice(ctx->device));
    // NULL means the legacy default stream (what an unqualified caller and torch's default stream use)
    cudaStream_t user = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    TCI_CUDA(cudaEventRecord(ctx->ev0, user));
    TCI_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev0, 0));
    const double* s_out = ctx->buf[BUF_S];
    if (ctx->local) {  // padded into the plan's layout, the result back in the local layout
      ctx->local_in(d_c);
      TCI_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
      ctx->run_sigma_steps();
      ctx->local_out(d_c, ctx->loc_s);
      TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
      s_out = ctx->loc_s;
    } else {
      // the plan addresses BUF_C / BUF_S: copy in and accumulate out
      TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_C], d_c, n * sizeof(double), cudaMemcpyDeviceToDevice, ctx->stream));
      TCI_CUDA(cudaMemsetAsync(ctx->buf[BUF_S], 0, n * sizeof(double), ctx->stream));
      TCI_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
      ctx->run_sigma_steps();
      TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    }
    // sigma += S (the caller's sigma accumulates, like htimesc)
    accumulate_f64<<<(unsigned)std::min<int64_t>((n + 255) / 256, sm_count() * 8), 256, 0, ctx->stream>>>(d_sigma, s_out, n);
    ctx->launch_count++;
    TCI_CUDA(cudaGetLastError());
    TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    TCI_CUDA(cudaStreamWaitEvent(user, ctx->ev1, 0));
    ctx->sigma_count++;
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_sigma(tci_ctx* ctx, const double* c, double* sigma, int64_t n) {
  if (!ctx || !c || !sigma) return TCI_ERR_ARG;
  try {
    if (n != ctx->nvec()) throw Error(TCI_ERR_ARG, "vector length differs from total_csfs");
    TCI_CUDA(cudaSetDevice(ctx->device));
    const double* s_out = ctx->buf[BUF_S];
    if (ctx->local) {
      TCI_CUDA(cudaMemcpyAsync(ctx->loc_c, c, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      ctx->local_in(ctx->loc_c);
      TCI_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
      ctx->run_sigma_steps();
      ctx->local_out(ctx->loc_c, ctx->loc_s);
      TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
      s_out = ctx->loc_s;
    } else {
      TCI_CUDA(cudaMemcpyAsync(ctx->buf[BUF_C], c, n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
      TCI_CUDA(cudaMemsetAsync(ctx->buf[BUF_S], 0, n * sizeof(double), ctx->stream));
      TCI_CUDA(cudaEventRecord(ctx->ev0, ctx->stream));
      ctx->run_sigma_steps();
      TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    }
    std::vector<double> tmp(n);
    TCI_CUDA(cudaMemcpyAsync(tmp.data(), s_out, n * sizeof(double), cudaMemcpyDeviceToHost, ctx->stream));
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    float ms = 0;
    TCI_CUDA(cudaEventElapsedTime(&ms, ctx->ev0, ctx->ev1));
    ctx->last_sigma_ms = ms;
    ctx->check_tc_status();
    for (int64_t i = 0; i < n; ++i) sigma[i] += tmp[i];
    ctx->sigma_count++;
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_diag(tci_ctx* ctx, double* hdiag, int64_t n) {
  if (!ctx || !hdiag) return TCI_ERR_ARG;
  try {
    if (n != ctx->nvec()) throw Error(TCI_ERR_ARG, "vector length differs from total_csfs");
    TCI_CUDA(cudaSetDevice(ctx->device));
    ctx->ensure_diag();
    TCI_CUDA(cudaMemcpy(hdiag, ctx->hd, n * sizeof(double), cudaMemcpyDeviceToHost));
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

}  // extern "C"

namespace {

// Root following (root_following, tiger_fortran/davidson.f90:732-812): state q keeps the subspace
// eigenvector with the largest overlap with the q-th basis vector (its initial guess, or its Ritz vector
// after a restart), measured in the metric the basis is orthonormal in; the first nroots eigenpairs are
// replaced by the chosen ones, in state order (a vector chosen twice is used twice, as in the reference).
void follow_roots(std::vector<double>& w, std::vector<double>& V, int m, int nroots) {
  std::vector<double> w2(w);
  std::vector<double> V2(V);
  for (int q = 0; q < nroots && q < m; ++q) {
    int best = 0;
    double bo = -1.0;
    for (int j = 0; j < m; ++j) {
      const double o = std::fabs(V[(size_t)q * m + j]);
      if (o > bo) bo = o, best = j;
    }
    w2[(size_t)q] = w[(size_t)best];
    for (int k = 0; k < m; ++k) V2[(size_t)k * m + q] = V[(size_t)k * m + best];
  }
  w.swap(w2);
  V.swap(V2);
}

// Cyclic Jacobi eigensolver for the small symmetric subspace matrix (the role of
// dsyev in dsyev_wrapper, tiger_fortran/math_utils.f90:417-479).  A is m x m row
// major; on exit w holds ascending eigenvalues and V (m x m, columns) the vectors.
void jacobi_eigh(std::vector<double> A, int m, std::vector<double>& w, std::vector<double>& V) {
  V.assign((size_t)m * m, 0.0);
  for (int i = 0; i < m; ++i) V[(size_t)i * m + i] = 1.0;
  for (int sweep = 0; sweep < 100; ++sweep) {
    double off = 0.0, tot = 0.0;
    for (int i = 0; i < m; ++i)
      for (int j = 0; j < m; ++j) {
        const double a = A[(size_t)i * m + j] * A[(size_t)i * m + j];
        tot += a;
        if (i != j) off += a;
      }
    if (off <= 1e-30 * tot || off == 0.0) break;
    for (int p = 0; p < m - 1; ++p)
      for (int q = p + 1; q < m; ++q) {
        const double apq = A[(size_t)p * m + q];
        if (std::fabs(apq) < 1e-300) continue;
        const double app = A[(size_t)p * m + p], aqq = A[(size_t)q * m + q];
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0 ? 1.0 : -1.0) / (std::fabs(theta) + std::sqrt(theta * theta + 1.0));
        const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
        for (int k = 0; k < m; ++k) {
          const double akp = A[(size_t)k * m + p], akq = A[(size_t)k * m + q];
          A[(size_t)k * m + p] = c * akp - s * akq;
          A[(size_t)k * m + q] = s * akp + c * akq;
        }
        for (int k = 0; k < m; ++k) {
          const double apk = A[(size_t)p * m + k], aqk = A[(size_t)q * m + k];
          A[(size_t)p * m + k] = c * apk - s * aqk;
          A[(size_t)q * m + k] = s * apk + c * aqk;
        }
        for (int k = 0; k < m; ++k) {
          const double vkp = V[(size_t)k * m + p], vkq = V[(size_t)k * m + q];
          V[(size_t)k * m + p] = c * vkp - s * vkq;
          V[(size_t)k * m + q] = s * vkp + c * vkq;
        }
      }
  }
  std::vector<int> ord(m);
  for (int i = 0; i < m; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return A[(size_t)a * m + a] < A[(size_t)b * m + b]; });
  w.resize(m);
  std::vector<double> V2((size_t)m * m);
  for (int j = 0; j < m; ++j) {
    w[j] = A[(size_t)ord[j] * m + ord[j]];
    // fix the sign so that the largest component is positive (deterministic output)
    int big = 0;
    for (int k = 1; k < m; ++k)
      if (std::fabs(V[(size_t)k * m + ord[j]]) > std::fabs(V[(size_t)big * m + ord[j]])) big = k;
    const double sg = V[(size_t)big * m + ord[j]] < 0 ? -1.0 : 1.0;
    for (int k = 0; k < m; ++k) V2[(size_t)k * m + j] = sg * V[(size_t)k * m + ord[j]];
  }
  V.swap(V2);
}

}  // namespace

extern "C" {

int tci_davidson(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                 double* energies, double* vectors, int64_t* iterations) {
  return tci_davidson_ex(ctx, nroots, tol_residual, tol_energy, maxit, 0, nullptr, energies, vectors, iterations);
}

// davidson_liu_gen_eig (tiger_fortran/davidson.f90:253-469): (H - e_shift) c = lambda G c, G = diag(g), solved
// as the standard problem of G^-1/2 (H - e_shift) G^-1/2 by the device Davidson above (y = G^1/2 c).
int tci_davidson_gen(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                     const double* g, double e_shift, double* energies, double* vectors, int64_t* iterations) {
  if (!ctx || !g || !energies || nroots <= 0 || !std::isfinite(e_shift)) return TCI_ERR_ARG;
  if (ctx->gen_s) return TCI_ERR_ARG;  // one generalized solve at a time on a context
  double* ds = nullptr;
  double* dd = nullptr;
  double* dg = nullptr;
  double* saved_hd = nullptr;
  std::vector<i64> saved_low;
  auto restore = [&]() {
    if (saved_hd) {
      ctx->hd = saved_hd;
      ctx->lowest_diag = saved_low;
    }
    ctx->gen_s = nullptr;
    ctx->gen_g = nullptr;
    ctx->gen_follow = false;
    ctx->gen_shift = 0.0;
    cudaStreamSynchronize(ctx->stream);
    std::lock_guard<std::mutex> lk(g_capture_free_mu);
    dev_free(ds, ctx->stream);
    dev_free(dd, ctx->stream);
    dev_free(dg, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
  };
  try {
    TCI_CUDA(cudaSetDevice(ctx->device));
    const i64 n = ctx->nvec();
    std::vector<double> sh((size_t)n);
    for (i64 i = 0; i < n; ++i) {
      if (!(g[i] > 0.0) || !std::isfinite(g[i])) throw Error(TCI_ERR_ARG, "the metric must be positive and finite");
      sh[(size_t)i] = 1.0 / std::sqrt(g[i]);
    }
    ctx->ensure_diag();
    TCI_CUDA(dev_malloc(&ds, (size_t)n * sizeof(double), ctx->stream));
    TCI_CUDA(dev_malloc(&dd, (size_t)n * sizeof(double), ctx->stream));
    TCI_CUDA(dev_malloc(&dg, (size_t)n * sizeof(double), ctx->stream));
    TCI_CUDA(cudaMemcpyAsync(ds, sh.data(), (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    TCI_CUDA(cudaMemcpyAsync(dg, g, (size_t)n * sizeof(double), cudaMemcpyHostToDevice, ctx->stream));
    gen_diag<<<sm_count() * 8, 256, 0, ctx->stream>>>(dd, ctx->hd, ds, e_shift, n);
    TCI_CUDA(cudaGetLastError());
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    saved_hd = ctx->hd;
    saved_low = ctx->lowest_diag;
    ctx->hd = dd;
    ctx->lowest_diag.clear();  // the initial guess follows the transformed diagonal
    ctx->gen_s = ds;
    ctx->gen_g = dg;
    ctx->gen_follow = ctx->acpf_root_follow;
    ctx->gen_shift = e_shift;
    const int rc = tci_davidson_ex(ctx, nroots, tol_residual, tol_energy, maxit, 0, nullptr, energies, vectors,
                                   iterations);
    restore();
    if (rc != TCI_OK) return rc;
    for (i64 k = 0; k < nroots; ++k) energies[k] += e_shift;
    if (vectors)  // c = G^-1/2 y, unit norm
      for (i64 k = 0; k < nroots; ++k) {
        double* v = vectors + k * n;
        double nrm = 0.0;
        for (i64 i = 0; i < n; ++i) {
          v[i] *= sh[(size_t)i];
          nrm += v[i] * v[i];
        }
        nrm = std::sqrt(nrm);
        if (nrm > 0.0)
          for (i64 i = 0; i < n; ++i) v[i] /= nrm;
      }
    return TCI_OK;
  } catch (...) {
    restore();
    return guard_status(std::current_exception());
  }
}

int64_t tci_davidson_capacity(int64_t n, int64_t nroots, int64_t maxit, int64_t subspace_bytes) {
  if (n <= 0 || nroots <= 0) return 0;
  if (maxit <= 0) maxit = 50 * nroots;
  const double budget = subspace_bytes > 0 ? (double)subspace_bytes : kDefaultSubspaceBytes;
  // the restart test fires at the first size T with 2 * T * n * 8 >= budget (and T > 4 * nroots);
  // the expansion that follows a test adds at most nroots vectors
  const int64_t t = std::max<int64_t>(4 * nroots + 1, (int64_t)std::ceil(budget / (16.0 * (double)n)));
  return std::min<int64_t>({n, (maxit + 1) * nroots, t - 1 + nroots});
}

int64_t tci_davidson_bytes(int64_t n, int64_t nroots, int64_t maxit, int64_t subspace_bytes) {
  const int64_t cap = tci_davidson_capacity(n, nroots, maxit, subspace_bytes);
  // c and H c vectors, the residual, the collapse buffers (2 * 2 * nroots vectors) and the reduction scratch
  return 8 * (n * (2 * cap + 1 + 4 * nroots) + (cap + 4) * (RBLK + 1) + 16 + 4 * (cap + 4));
}

// Block Davidson-Liu with HBM-resident expansion and sigma vectors, restating
// davidson_liu (tiger_fortran/davidson.f90:47-239): per unconverged root one
// sigma build and subspace expansion; subspace eigensolve; wavefunction,
// residual, convergence test (is_converged :564-602), diagonal preconditioner
// (:609-631) and modified Gram-Schmidt with renormalisation after every
// projection (:702-723).  The initial guess is the unit vectors of the lowest
// diagonal elements (init_from_diag, initial_davidson_guess.f90:99-137).
// The subspace restarts like restart_davidson_subspace
// (davidson_restart.f90:26-139): when it holds more than 4 vectors per root and
// its c and H c vectors need at least subspace_bytes (the role of DAVIDSON HARD
// DRIVE SPACE), it collapses onto the current and the previous Ritz vector of
// every unconverged root (the current one only for converged roots).  The
// collapsed set is orthonormalised as a whole, so the subspace basis stays
// orthonormal.  A non-null cancel flag that becomes non-zero ends the solve
// with TCI_ERR_CANCELLED at the next iteration boundary.
int tci_davidson_ex(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                    int64_t subspace_bytes, const int32_t* cancel, double* energies, double* vectors,
                    int64_t* iterations) {
  if (!ctx || !energies || nroots <= 0 || subspace_bytes < 0) return TCI_ERR_ARG;
  try {
    TCI_CUDA(cudaSetDevice(ctx->device));
    const i64 n = ctx->nvec();
    if (nroots > n) throw Error(TCI_ERR_ARG, "more roots than CSFs");
    if (maxit <= 0) maxit = 50 * nroots;
    const double budget = subspace_bytes > 0 ? (double)subspace_bytes : kDefaultSubspaceBytes;
    const int cap = (int)tci_davidson_capacity(n, nroots, maxit, subspace_bytes);
    const int keep = (int)std::min<i64>(2 * nroots, n);  // vectors kept by a collapse
    ctx->ensure_diag();
    ctx->ensure_scratch(cap + 4);
    // phase timing (tci_profile bit 1): the stream is synchronised at every boundary
    auto tp = std::chrono::steady_clock::now();
    int cur_phase = 0;
    auto mark = [&](int ph) {
      if (!ctx->dav_phases) return;
      TCI_CUDA(cudaStreamSynchronize(ctx->stream));
      const auto t = std::chrono::steady_clock::now();
      ctx->dav_ms[cur_phase] += std::chrono::duration<double, std::milli>(t - tp).count();
      tp = t;
      cur_phase = ph;
    };
    // the subspace vectors stay allocated in the context between solves
    auto free_all = [&]() { cudaStreamSynchronize(ctx->stream); };
    if (ctx->dav_cap < cap || ctx->dav_keep < keep) {
      TCI_CUDA(cudaStreamSynchronize(ctx->stream));
      {
        std::lock_guard<std::mutex> lk(g_capture_free_mu);
        for (double** p : {&ctx->dav_c, &ctx->dav_hc, &ctx->dav_r, &ctx->dav_tc, &ctx->dav_th}) {
          dev_free(*p, ctx->stream);
          *p = nullptr;
        }
      }
      ctx->dav_cap = ctx->dav_keep = 0;
      cudaStream_t ds = ctx->stream;
      cudaError_t e1 = dev_malloc(&ctx->dav_c, (size_t)cap * n * sizeof(double), ds);
      cudaError_t e2 = dev_malloc(&ctx->dav_hc, (size_t)cap * n * sizeof(double), ds);
      cudaError_t e3 = dev_malloc(&ctx->dav_r, (size_t)(n + 8) * sizeof(double), ds);
      cudaError_t e4 = dev_malloc(&ctx->dav_tc, (size_t)keep * n * sizeof(double), ds);
      cudaError_t e5 = dev_malloc(&ctx->dav_th, (size_t)keep * n * sizeof(double), ds);
      if (e1 != cudaSuccess || e2 != cudaSuccess || e3 != cudaSuccess || e4 != cudaSuccess || e5 != cudaSuccess) {
        cudaGetLastError();
        std::lock_guard<std::mutex> lk(g_capture_free_mu);
        for (double** p : {&ctx->dav_c, &ctx->dav_hc, &ctx->dav_r, &ctx->dav_tc, &ctx->dav_th}) {
          dev_free(*p, ctx->stream);
          *p = nullptr;
        }
        cudaStreamSynchronize(ctx->stream);
        throw Error(TCI_ERR_MEMORY, "device allocation of the Davidson subspace failed");
      }
      ctx->dav_cap = cap;
      ctx->dav_keep = keep;
    }
    double *Cs = ctx->dav_c, *HCs = ctx->dav_hc, *r = ctx->dav_r, *tmpC = ctx->dav_tc, *tmpH = ctx->dav_th;
    bool ran_out = false;  // a root stopped at maxit without meeting either tolerance
    try {
      cudaStream_t st = ctx->stream;
      const unsigned G = sm_count() * 8, TB = 256;
      // initial guess: unit vectors at the lowest diagonal elements (the order is a property of the
      // operator: kept in the context for the next solve)
      if ((i64)ctx->lowest_diag.size() < nroots) {
        std::vector<double> hd(n);
        TCI_CUDA(cudaMemcpy(hd.data(), ctx->hd, n * sizeof(double), cudaMemcpyDeviceToHost));
        std::vector<i64> all(n);
        for (i64 i = 0; i < n; ++i) all[i] = i;
        std::partial_sort(all.begin(), all.begin() + nroots, all.end(),
                          [&](i64 a, i64 b) { return hd[a] < hd[b] || (hd[a] == hd[b] && a < b); });
        ctx->lowest_diag.assign(all.begin(), all.begin() + nroots);
      }
      const std::vector<i64>& idx = ctx->lowest_diag;
      TCI_CUDA(cudaMemsetAsync(Cs, 0, (size_t)nroots * n * sizeof(double), st));
      const double one = 1.0;
      for (i64 k = 0; k < nroots; ++k)
        TCI_CUDA(cudaMemcpyAsync(Cs + k * n + idx[k], &one, sizeof(double), cudaMemcpyHostToDevice, st));
      TCI_CUDA(cudaStreamSynchronize(st));
      int num_vec = (int)nroots;
      std::vector<int> root2index(nroots);
      for (int k = 0; k < nroots; ++k) root2index[k] = k;
      std::vector<char> conv(nroots, 0), restarted(maxit + 2, 0);
      std::vector<double> energy(nroots, 0.0), dE(nroots, 0.0), hsub((size_t)cap * cap, 0.0), w, V, Vprev, col(cap);
      int mprev = 0;  // subspace dimension of Vprev
      auto lincomb_into = [&](double* dst, const double* src, const std::vector<double>& coef, int m) {
        TCI_CUDA(cudaMemcpyAsync(ctx->coefs, coef.data(), m * sizeof(double), cudaMemcpyHostToDevice, st));
        lincomb_kernel<<<G, TB, 0, st>>>(dst, 0.0, src, ctx->coefs, nullptr, nullptr, m, n, n);
        ctx->launch_count++;
        TCI_CUDA(cudaGetLastError());
        // the coefficient array is reused by the next call
        TCI_CUDA(cudaStreamSynchronize(st));
      };
      i64 it = 0;
      for (it = 1; it <= maxit; ++it) {
        if (cancel && __atomic_load_n(cancel, __ATOMIC_ACQUIRE) != 0) throw Error(TCI_ERR_CANCELLED, "solve cancelled");
        for (int q = 0; q < nroots; ++q) {
          if (conv[q]) continue;
          const int index = root2index[q];
          mark(1);
          ctx->sigma_of(Cs + (size_t)index * n, HCs + (size_t)index * n);
          mark(2);
          ctx->multi_dot(Cs, n, index + 1, HCs + (size_t)index * n, n, col.data());
          for (int k = 0; k <= index; ++k) hsub[(size_t)k * cap + index] = hsub[(size_t)index * cap + k] = col[k];
        }
        std::vector<double> h((size_t)num_vec * num_vec);
        for (int a = 0; a < num_vec; ++a)
          for (int b = 0; b < num_vec; ++b) h[(size_t)a * num_vec + b] = hsub[(size_t)a * cap + b];
        if (!w.empty()) {
          Vprev = V;
          mprev = (int)w.size();
        }
        mark(3);
        jacobi_eigh(h, num_vec, w, V);
        if (ctx->gen_follow) follow_roots(w, V, num_vec, (int)nroots);
        for (int q = 0; q < nroots; ++q) {
          dE[q] = std::fabs(w[q] - energy[q]);
          energy[q] = w[q];
        }
        const bool over_budget = num_vec > 4 * nroots && 16.0 * (double)n * num_vec >= budget;
        if (over_budget || num_vec + nroots > cap) {
          // restart_davidson_subspace: new basis {current, previous} per unconverged root, {current} per
          // converged root, as coefficient vectors in the present (orthonormal) basis
          mark(6);
          restarted[it] = 1;
          // (the current vectors go first so that a full subspace never drops one of them)
          std::vector<std::vector<double>> B;
          for (int q = 0; q < nroots; ++q) {
            std::vector<double> cur(num_vec);
            for (int k = 0; k < num_vec; ++k) cur[k] = V[(size_t)k * num_vec + q];
            B.push_back(cur);
          }
          for (int q = 0; q < nroots; ++q) {
            if (conv[q] || mprev == 0) continue;
            std::vector<double> prev(num_vec, 0.0);
            for (int k = 0; k < mprev && k < num_vec; ++k) prev[k] = Vprev[(size_t)k * mprev + q];
            B.push_back(prev);
          }
          const int limit = std::max<int>((int)nroots, std::min<int>(keep, cap - (int)nroots));
          // modified Gram-Schmidt in coefficient space; nearly dependent vectors are dropped
          std::vector<std::vector<double>> Q;
          for (auto& b : B) {
            for (auto& qv : Q) {
              double d = 0;
              for (int k = 0; k < num_vec; ++k) d += qv[k] * b[k];
              for (int k = 0; k < num_vec; ++k) b[k] -= d * qv[k];
            }
            double nr = 0;
            for (int k = 0; k < num_vec; ++k) nr += b[k] * b[k];
            nr = std::sqrt(nr);
            if (nr < 1e-8 || (int)Q.size() >= limit) continue;
            for (int k = 0; k < num_vec; ++k) b[k] /= nr;
            Q.push_back(b);
          }
          const int m2 = (int)Q.size();
          for (int j = 0; j < m2; ++j) {
            lincomb_into(tmpC + (size_t)j * n, Cs, Q[j], num_vec);
            lincomb_into(tmpH + (size_t)j * n, HCs, Q[j], num_vec);
          }
          TCI_CUDA(cudaMemcpyAsync(Cs, tmpC, (size_t)m2 * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
          TCI_CUDA(cudaMemcpyAsync(HCs, tmpH, (size_t)m2 * n * sizeof(double), cudaMemcpyDeviceToDevice, st));
          TCI_CUDA(cudaStreamSynchronize(st));
          // H in the new basis: Q^T hsub Q
          std::vector<double> hq((size_t)num_vec * m2, 0.0), hn((size_t)m2 * m2, 0.0);
          for (int a = 0; a < num_vec; ++a)
            for (int j = 0; j < m2; ++j) {
              double t = 0;
              for (int b = 0; b < num_vec; ++b) t += hsub[(size_t)a * cap + b] * Q[j][b];
              hq[(size_t)a * m2 + j] = t;
            }
          for (int i = 0; i < m2; ++i)
            for (int j = 0; j < m2; ++j) {
              double t = 0;
              for (int a = 0; a < num_vec; ++a) t += Q[i][a] * hq[(size_t)a * m2 + j];
              hn[(size_t)i * m2 + j] = t;
            }
          for (int i = 0; i < m2; ++i)
            for (int j = 0; j < m2; ++j) hn[(size_t)i * m2 + j] = hn[(size_t)j * m2 + i] =
                0.5 * (hn[(size_t)i * m2 + j] + hn[(size_t)j * m2 + i]);
          std::fill(hsub.begin(), hsub.end(), 0.0);
          for (int i = 0; i < m2; ++i)
            for (int j = 0; j < m2; ++j) hsub[(size_t)i * cap + j] = hn[(size_t)i * m2 + j];
          num_vec = m2;
          jacobi_eigh(hn, num_vec, w, V);
          if (ctx->gen_follow) follow_roots(w, V, num_vec, (int)nroots);
          for (int q = 0; q < nroots; ++q) energy[q] = w[q];
          Vprev.clear();
          mprev = 0;
        }
        // the Ritz vectors live in the subspace of this iteration (subspace_size in
        // davidson.f90:140); vectors appended below for earlier roots are not part of it
        const int subspace_size = num_vec;
        for (int q = 0; q < nroots; ++q) {
          if (conv[q]) continue;
          mark(4);
          // residual r = sum_k a_k (Hc_k - E c_k)
          std::vector<double> ca(subspace_size), cb(subspace_size);
          for (int k = 0; k < subspace_size; ++k) {
            cb[k] = V[(size_t)k * subspace_size + q];
            ca[k] = -energy[q] * cb[k];
          }
          TCI_CUDA(cudaMemcpyAsync(ctx->coefs, ca.data(), subspace_size * sizeof(double), cudaMemcpyHostToDevice, st));
          TCI_CUDA(cudaMemcpyAsync(ctx->coefs + cap, cb.data(), subspace_size * sizeof(double), cudaMemcpyHostToDevice, st));
          lincomb_kernel<<<G, TB, 0, st>>>(r, 0.0, Cs, ctx->coefs, HCs, ctx->coefs + cap, subspace_size, n, n);
          ctx->launch_count++;
          TCI_CUDA(cudaGetLastError());
          double nrm2 = 0.0;
          if (ctx->gen_g) {
            // generalized solve: the residual of the reference, (H - E_ref) c - lambda G c = G^1/2 r_y
            // (build_residual_gen_eig, davidson.f90:535-553), c = G^-1/2 y of unit G-norm as dsygv gives
            // it: |G^1/2 r_y|^2 = sum_i g_i r_y,i^2
            TCI_CUDA(cudaMemcpyAsync(tmpC, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
            scale_by<<<G, TB, 0, st>>>(tmpC, ctx->gen_g, n);
            ctx->launch_count++;
            ctx->multi_dot(r, 0, 1, tmpC, n, &nrm2);
          } else {
            ctx->multi_dot(r, 0, 1, r, n, &nrm2);
          }
          const double norm = std::sqrt(nrm2);
          // is_converged: never right after a restart; residual norm, then energy change (i > 1), then maxit
          bool halt = false;
          if (!(restarted[it] || (it > 1 && restarted[it - 1]))) {
            if (norm < tol_residual) halt = true;
            else if (std::fabs(dE[q]) < tol_energy) halt = it > 1;
            else if (it == maxit) halt = true, ran_out = true;
          }
          if (halt) {
            conv[q] = 1;
            continue;
          }
          mark(5);
          precondition_kernel<<<G, TB, 0, st>>>(r, ctx->hd, energy[q], n);
          ctx->launch_count++;
          TCI_CUDA(cudaGetLastError());
          // Orthogonalise against the basis (the reference's davidson.f90 runs modified Gram-Schmidt,
          // normalising after each projection).  Here: normalise, then block classical Gram-Schmidt twice
          // (all projections of one pass from one multi-dot and one linear combination), then normalise
          // with the same 1e-14 zeroing rule: the same vector up to rounding, as stable as modified
          // Gram-Schmidt, and four passes over the basis instead of two per basis vector.
          double* dev_ov = ctx->dots + (size_t)(cap + 4) * RBLK;
          double* dev_coef = dev_ov + 2;  // num_vec <= cap coefficients fit the buffer's tail
          ctx->dot_dev(r, r, n, dev_ov + 1);
          normalize_kernel<<<G, TB, 0, st>>>(r, dev_ov + 1, n);
          ctx->launch_count++;
          for (int pass = 0; pass < 2 && num_vec > 0; ++pass) {
            multi_dot_partial<<<RBLK, RB, 0, st>>>(Cs, n, num_vec, r, n, ctx->dots);
            multi_dot_final_neg<<<(num_vec + 127) / 128, 128, 0, st>>>(ctx->dots, num_vec, RBLK, dev_coef);
            lincomb_kernel<<<G, TB, 0, st>>>(r, 1.0, Cs, dev_coef, nullptr, nullptr, num_vec, n, n);
            ctx->launch_count += 3;
          }
          ctx->dot_dev(r, r, n, dev_ov + 1);
          normalize_kernel<<<G, TB, 0, st>>>(r, dev_ov + 1, n);
          ctx->launch_count++;
          TCI_CUDA(cudaGetLastError());
          if (num_vec >= cap) throw Error(TCI_ERR_INTERNAL, "Davidson subspace capacity exceeded");
          TCI_CUDA(cudaMemcpyAsync(Cs + (size_t)num_vec * n, r, n * sizeof(double), cudaMemcpyDeviceToDevice, st));
          root2index[q] = num_vec;
          num_vec++;
        }
        TCI_CUDA(cudaStreamSynchronize(st));
        bool all = true;
        for (int q = 0; q < nroots; ++q) all = all && conv[q];
        if (all) break;
      }
      ctx->last_converged = !ran_out && std::all_of(conv.begin(), conv.end(), [](int x) { return x != 0; });
      mark(7);
      ctx->check_tc_status();
      if (ctx->precision == 1 && ctx->refine) {
        // FP64 finish: each root is reported as the Rayleigh quotient of its Ritz vector with the plain-FP64
        // sigma (refine 2: all terms FP64 but the all-external one).  Its error is second order in the
        // eigenvector error the mixed products leave.
        const int m = (int)w.size();
        for (int q = 0; q < nroots; ++q) {
          std::vector<double> cb(m);
          for (int k = 0; k < m; ++k) cb[k] = V[(size_t)k * m + q];
          lincomb_into(r, Cs, cb, m);
          ctx->sigma_of_fp64(r, tmpH);
          double rr = 0.0, rhr = 0.0;
          ctx->multi_dot(r, 0, 1, r, n, &rr);
          ctx->multi_dot(r, 0, 1, tmpH, n, &rhr);
          energy[q] = rhr / rr;
        }
      }
      for (int q = 0; q < nroots; ++q) energies[q] = energy[q];
      if (iterations) *iterations = std::min<i64>(it, maxit);
      if (vectors) {
        const int m = (int)w.size();  // dimension of the last subspace eigensolve
        for (int q = 0; q < nroots; ++q) {
          std::vector<double> cb(m);
          for (int k = 0; k < m; ++k) cb[k] = V[(size_t)k * m + q];
          lincomb_into(r, Cs, cb, m);
          double nrm2 = 0.0;
          ctx->multi_dot(r, 0, 1, r, n, &nrm2);
          std::vector<double> hv(n);
          TCI_CUDA(cudaMemcpy(hv.data(), r, n * sizeof(double), cudaMemcpyDeviceToHost));
          const double inv = 1.0 / std::sqrt(nrm2);
          for (i64 i = 0; i < n; ++i) vectors[(size_t)q * n + i] = hv[i] * inv;
        }
      }
    } catch (...) {
      free_all();
      throw;
    }
    free_all();
    mark(0);
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_ctx_stats(const tci_ctx* ctx, double* out, int64_t len) {
  if (!ctx || !out || len < 8) return TCI_ERR_ARG;
  if (len >= 9) out[8] = 1.0 + (double)ctx->sigma_launches();  // + the accumulation into the caller's sigma
  if (len >= 10) out[9] = (double)ctx->launch_count;
  if (len >= 11) out[10] = ctx->last_converged ? 1.0 : 0.0;
  out[0] = (double)ctx->nvec();
  out[1] = ctx->bytes_held;
  out[2] = ctx->init_seconds;
  out[3] = ctx->last_sigma_ms;
  out[4] = ctx->plan.flops_total;
  out[5] = ctx->plan.flops_allext;
  out[6] = ctx->plan.bytes_allext;
  out[7] = (double)ctx->sigma_count;
  return TCI_OK;
}

// Batched deterministic projections out[k] = sum_i A[k*lda + i] x[i], k < m, on
// device arrays (the dot products of expand_krylov_subspace and the MGS
// overlaps, tiger_fortran/davidson.f90:478-494, 702-723, for a caller that
// keeps its Davidson vectors in HBM).  Two-pass reduction in a fixed order:
// the result does not depend on timing.  Scratch (m * 593 doubles) is owned by
// the context and grows on demand.
int tci_dots(tci_ctx* ctx, const double* d_A, int64_t lda, int64_t m, const double* d_x, int64_t n, double* d_out,
             void* stream) {
  if (!ctx || !d_A || !d_x || !d_out || m <= 0 || n <= 0 || (m > 1 && lda < n)) return TCI_ERR_ARG;
  try {
    TCI_CUDA(cudaSetDevice(ctx->device));
    cudaStream_t user = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    const int64_t need = m * (RBLK + 1);
    if (need > ctx->dotbuf_cap) {
      TCI_CUDA(cudaStreamSynchronize(ctx->stream));
      if (ctx->dotbuf) {
        std::lock_guard<std::mutex> lk(g_capture_free_mu);
        TCI_CUDA(dev_free(ctx->dotbuf, ctx->stream));
      }
      ctx->dotbuf = nullptr;
      ctx->dotbuf_cap = 0;
      if (dev_malloc(&ctx->dotbuf, need * sizeof(double), ctx->stream) != cudaSuccess) {
        cudaGetLastError();
        throw Error(TCI_ERR_MEMORY, "device allocation of the projection scratch failed");
      }
      ctx->dotbuf_cap = need;
    }
    TCI_CUDA(cudaEventRecord(ctx->ev0, user));
    TCI_CUDA(cudaStreamWaitEvent(ctx->stream, ctx->ev0, 0));
    multi_dot_partial<<<RBLK, RB, 0, ctx->stream>>>(d_A, lda, (int)m, d_x, n, ctx->dotbuf);
    multi_dot_final<<<(unsigned)((m + 127) / 128), 128, 0, ctx->stream>>>(ctx->dotbuf, (int)m, RBLK, d_out);
    ctx->launch_count += 2;
    TCI_CUDA(cudaGetLastError());
    TCI_CUDA(cudaEventRecord(ctx->ev1, ctx->stream));
    TCI_CUDA(cudaStreamWaitEvent(user, ctx->ev1, 0));
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_check(tci_ctx* ctx) {
  if (!ctx) return TCI_ERR_ARG;
  try {
    TCI_CUDA(cudaSetDevice(ctx->device));
    TCI_CUDA(cudaStreamSynchronize(ctx->stream));
    ctx->check_tc_status();
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_profile(tci_ctx* ctx, int64_t on) {
  if (!ctx) return TCI_ERR_ARG;
  ctx->profiling = (on & 1) != 0;
  ctx->dav_phases = (on & 2) != 0;
  ctx->step_ms.assign(ctx->sigma.size(), 0.0);
  ctx->profiled_builds = 0;
  for (double& v : ctx->dav_ms) v = 0.0;
  return TCI_OK;
}

int tci_davidson_phase_times(const tci_ctx* ctx, double* ms, int64_t len) {
  if (!ctx || !ms || len < 8) return TCI_ERR_ARG;
  for (int i = 0; i < 8; ++i) ms[i] = ctx->dav_ms[i];
  return TCI_OK;
}

int tci_step_times(const tci_ctx* ctx, double* ms, int64_t len, int64_t* nsteps, int64_t* nbuilds) {
  if (!ctx || !nsteps) return TCI_ERR_ARG;
  *nsteps = (int64_t)ctx->sigma.size();
  if (nbuilds) *nbuilds = ctx->profiled_builds;
  for (int64_t i = 0; ms && i < len && i < (int64_t)ctx->step_ms.size(); ++i) ms[i] = ctx->step_ms[i];
  return TCI_OK;
}

int tci_step_name(const tci_ctx* ctx, int64_t i, char* buf, int64_t len) {
  if (!ctx || !buf || len <= 0 || i < 0 || i >= (int64_t)ctx->sigma.size()) return TCI_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", ctx->sigma[i].name.c_str());
  return TCI_OK;
}

void tci_destroy(tci_ctx* ctx) { delete ctx; }

int tci_selftest_bounded_wait(int64_t device, int64_t polls, int64_t* status_out, double* ms_out) {
  if (!status_out || polls < 0) return TCI_ERR_ARG;
  int* st = nullptr;
  cudaStream_t s = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  auto cleanup = [&]() {
    if (s) cudaStreamSynchronize(s);
    if (st) cudaFree(st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
  };
  try {
    int ndev = 0;
    TCI_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) throw Error(TCI_ERR_CUDA, "requested device is not available");
    TCI_CUDA(cudaSetDevice((int)device));
    TCI_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    TCI_CUDA(cudaEventCreate(&e0));
    TCI_CUDA(cudaEventCreate(&e1));
    TCI_CUDA(cudaMalloc(&st, sizeof(int)));
    TCI_CUDA(cudaMemsetAsync(st, 0, sizeof(int), s));
    TCI_CUDA(cudaEventRecord(e0, s));
    TCI_CUDA(tci_tc_host::bounded_wait_selftest(polls ? polls : tci_tc_host::spin_limit(), st, s));
    TCI_CUDA(cudaEventRecord(e1, s));
    int h = 0;
    TCI_CUDA(cudaMemcpyAsync(&h, st, sizeof(int), cudaMemcpyDeviceToHost, s));
    TCI_CUDA(cudaStreamSynchronize(s));
    float ms = 0;
    TCI_CUDA(cudaEventElapsedTime(&ms, e0, e1));
    *status_out = h;
    if (ms_out) *ms_out = ms;
    cleanup();
    if (h != 0) {
      set_error("self-test: the bounded wait gave up (code " + std::to_string(h) + ")");
      return TCI_ERR_TIMEOUT;
    }
    return TCI_OK;
  } catch (...) {
    cleanup();
    return guard_status(std::current_exception());
  }
}

int tci_selftest_mma_rate(int64_t device, int64_t m, int64_t n, int64_t nacc, int64_t iters, double* cycles_per_mma) {
  // M = 64 accumulators are given twice the TMEM columns of their N (the half-lane layouts use up to 2 N)
  if (!cycles_per_mma || (m != 64 && m != 128) || n > 256 || n < (m == 64 ? 8 : 16) || n % (m == 64 ? 8 : 16) ||
      nacc < 1 || nacc * n * (m == 64 ? 2 : 1) > 512 || iters < 1 || iters > (1 << 20))
    return TCI_ERR_ARG;
  int* st = nullptr;
  long long* cyc = nullptr;
  cudaStream_t s = nullptr;
  auto cleanup = [&]() {
    if (s) cudaStreamSynchronize(s);
    if (st) cudaFree(st);
    if (cyc) cudaFree(cyc);
    if (s) cudaStreamDestroy(s);
  };
  try {
    int ndev = 0;
    TCI_CUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) throw Error(TCI_ERR_CUDA, "requested device is not available");
    TCI_CUDA(cudaSetDevice((int)device));
    const int grid = sm_count();
    TCI_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    TCI_CUDA(cudaMalloc(&st, sizeof(int)));
    TCI_CUDA(cudaMalloc(&cyc, sizeof(long long) * (size_t)grid));
    TCI_CUDA(cudaMemsetAsync(st, 0, sizeof(int), s));
    std::vector<long long> h((size_t)grid);
    for (int rep = 0; rep < 2; ++rep)  // the first launch warms up; the second is read
      TCI_CUDA(tci_tc_host::mma_rate_selftest(m, n, nacc, iters, grid, cyc, st, s));
    int hs = 0;
    TCI_CUDA(cudaMemcpyAsync(h.data(), cyc, sizeof(long long) * (size_t)grid, cudaMemcpyDeviceToHost, s));
    TCI_CUDA(cudaMemcpyAsync(&hs, st, sizeof(int), cudaMemcpyDeviceToHost, s));
    TCI_CUDA(cudaStreamSynchronize(s));
    cleanup();
    if (hs != 0) {
      set_error("MMA rate self-test: the commit's bounded wait gave up");
      return TCI_ERR_TIMEOUT;
    }
    *cycles_per_mma = (double)*std::max_element(h.begin(), h.end()) / (double)(iters * nacc);
    return TCI_OK;
  } catch (...) {
    cleanup();
    return guard_status(std::current_exception());
  }
}

}  // extern "C"
