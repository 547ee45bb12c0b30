// Grouped GEMM steps of the sigma plan on the 5th-generation tensor cores, for
// the mixed-precision form (3xTF32 products, FP32 accumulation in TMEM, FP64
// promotion every few k-steps, FP64 output).
//
// Same problem and segment tables as the FP64 SIMT kernel (gemm_tables.h):
// every CTA owns one 128 x 64 tile of one problem's C and runs over all of
// that problem's K segments in table order.  A problem short in M is
// computed transposed (C^T = B^T A^T, trans_c set) so that its long dimension
// fills the 128-row MMA.  The operands are FP64 in HBM /
// L2 with arbitrary leading dimensions and either orientation, which TMA
// cannot convert, so four producer warps load them with coalesced FP64 loads,
// fold the segment's alpha into B, split every element into a TF32 high part
// and an FP32 low part (x = hi + lo), and store both into shared memory in the
// K-major 128-byte-swizzle layout that the MMA descriptors read.  One thread
// issues two kind::tf32 MMAs per 8-wide k slice (A_hi x [B_hi; B_lo], A_lo x B_hi) into
// a double-buffered TMEM accumulator; every KB_PER_BLOCK k-steps the four
// epilogue warps add the FP32 block sums into FP64 registers, and write
// C = beta C + acc once at the end.
//
// Warp roles (288 threads): 0-3 epilogue (TMEM lane quadrants 0-3), 4-7
// producers, 8 TMEM allocator + MMA issuer.  Every mbarrier wait is bounded;
// on timeout the kernel records a status code, waits (bounded) for its MMAs in
// flight, frees its TMEM and returns.
#include <cuda_runtime.h>

#include <cstdint>

#include "gemm_tables.h"
#include "gemm_tc.h"
#include "tc_common.cuh"

namespace tci_gtc {

using namespace tci_tcx;
using tci_dev::DGemmProblem;
using tci_dev::DGemmSeg;

constexpr int BM = 128;  // MMA M: rows of C per tile
constexpr int BN = 64;   // MMA N: columns of C per tile
constexpr int BK = 32;   // k elements per stage (one 128-byte swizzled row)
constexpr int STAGES = 4;
constexpr int NPROD = 4;  // producer warps
constexpr int NTHREADS = 32 * (4 + NPROD + 1);
constexpr int A_BYTES = BM * BK * 4;  // 16 KB
constexpr int B_BYTES = BN * BK * 4;  // 8 KB
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
// B's high rows are followed by its low rows in a stage: A_hi x [B_hi; B_lo] is one MMA of N = 2 BN and
// A_lo x B_hi a second one (two instructions per k slice instead of three)
constexpr uint32_t kIdescBoth = idesc_tf32(BM, 2 * BN), kIdescHi = idesc_tf32(BM, BN);
constexpr int ACC_COLS = 2 * BN;  // hi x hi + lo x hi, then hi x lo
static_assert(BM * BK == 32 * 32 * NPROD && BN * BK == 16 * 32 * NPROD && NPROD == 4 && BK == 32,
              "producer element maps");

enum : int { ST_TIMEOUT_EMPTY = 11, ST_TIMEOUT_FULL = 12, ST_TIMEOUT_D = 13, ST_TIMEOUT_DE = 14 };

// x = hi + lo: hi is the TF32 truncation of the FP32 rounding of x, lo the FP32
// rounding of the remainder (the tensor core reads its top 19 bits).
__device__ __forceinline__ void split_store(uint8_t* hi_tile, uint8_t* lo_tile, int row, int k, double x) {
  const uint32_t hb = __float_as_uint((float)x) & 0xFFFFE000u;
  const float lo = (float)(x - (double)__uint_as_float(hb));
  const uint32_t off = sw128_offset(row, k);
  *reinterpret_cast<uint32_t*>(hi_tile + off) = hb;
  *reinterpret_cast<float*>(lo_tile + off) = lo;
}

__device__ __forceinline__ int steps_of(long long K) { return (int)((K + BK - 1) / BK); }

__global__ void __launch_bounds__(NTHREADS, 1)
    gemm_tc_tf32x3(const DGemmProblem* __restrict__ probs, int nprob, const DGemmSeg* __restrict__ segs,
                   int* __restrict__ status, int kb_per_block) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* dfull = empty + STAGES;  // 2
  uint64_t* dempty = dfull + 2;      // 2
  uint64_t* mma_done = dempty + 2;   // 1
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  // the tile and its problem
  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const DGemmProblem P = probs[lo];
  const long long t = tile - P.tile_begin;
  const long long m0 = (t / P.tiles_n) * BM, n0 = (t % P.tiles_n) * BN;
  int nsteps = 0;
  for (long long q = P.seg_begin; q < P.seg_end; ++q) nsteps += steps_of(segs[q].K);
  const int KB = kb_per_block;
  const int nblocks = (nsteps + KB - 1) / KB;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], NPROD);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], 4);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 8) {  // TMEM: two accumulator buffers of ACC_COLS fp32 columns
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * ACC_COLS));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *tmem_slot;

  auto fail = [&](int code) {
    atomicCAS(status, 0, code);
    *(volatile int*)abort_flag = 1;
  };
  auto aborted = [&]() { return *(volatile int*)abort_flag != 0; };

  if (warp >= 4 && warp < 4 + NPROD) {
    // ---------------- producers: FP64 -> (TF32 hi, FP32 lo), swizzled K-major tiles ----------------
    const int pw = warp - 4;
    int step = 0;
    for (long long q = P.seg_begin; q < P.seg_end && !aborted(); ++q) {
      const DGemmSeg S = segs[q];
      const int nk = steps_of(S.K);
      for (int kk = 0; kk < nk; ++kk, ++step) {
        const int s = step % STAGES;
        if (step >= STAGES && !mbar_wait(&empty[s], ((step / STAGES) - 1) & 1)) {
          fail(ST_TIMEOUT_EMPTY);
          break;
        }
        if (aborted()) break;
        const long long k0 = (long long)kk * BK;
        uint8_t* ahi = base + s * STAGE_BYTES;
        uint8_t* alo = ahi + A_BYTES;
        uint8_t* bhi = ahi + 2 * A_BYTES;
        uint8_t* blo = bhi + B_BYTES;
        // Every load of the stage is issued before any conversion (48 FP64
        // loads in flight per thread): the operands come from L2 / HBM and the
        // producers are latency bound otherwise.
        double xa[BM * BK / (32 * NPROD)], xb[BN * BK / (32 * NPROD)];
        // A tile (BM x BK): element i of this thread is (row, k) below
        if (!S.tA) {  // A[m][k]: a warp reads rows, lane = k
          const long long gk = k0 + lane;
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const long long gm = m0 + pw + NPROD * i;
            xa[i] = (gm < P.M && gk < S.K) ? S.A[gm * S.lda + gk] : 0.0;
          }
        } else {  // A[k][m]: warp pw takes k in [8 pw, 8 pw + 8); an instruction reads 4 k rows x 8
                  // consecutive m (lane = 8 (k & 3) + (m & 7)), so its shared-memory stores hit 32 banks
#pragma unroll
          for (int i = 0; i < 32; ++i) {
            const long long gk = k0 + 8 * pw + 4 * (i >> 4) + (lane >> 3), gm = m0 + 8 * (i & 15) + (lane & 7);
            xa[i] = (gm < P.M && gk < S.K) ? S.A[gk * S.lda + gm] : 0.0;
          }
        }
        // B tile (BN x BK, stored as rows n)
        if (S.tB) {  // B[n][k]: lane = k
          const long long gk = k0 + lane;
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const long long gn = n0 + pw + NPROD * i;
            xb[i] = (gn < P.N && gk < S.K) ? S.B[gn * S.ldb + gk] : 0.0;
          }
        } else {  // B[k][n]: as the transposed A path, 4 k rows x 8 consecutive n per instruction
#pragma unroll
          for (int i = 0; i < 16; ++i) {
            const long long gk = k0 + 8 * pw + 4 * (i >> 3) + (lane >> 3), gn = n0 + 8 * (i & 7) + (lane & 7);
            xb[i] = (gn < P.N && gk < S.K) ? S.B[gk * S.ldb + gn] : 0.0;
          }
        }
        if (!S.tA) {
#pragma unroll
          for (int i = 0; i < 32; ++i) split_store(ahi, alo, pw + NPROD * i, lane, xa[i]);
        } else {
#pragma unroll
          for (int i = 0; i < 32; ++i)
            split_store(ahi, alo, 8 * (i & 15) + (lane & 7), 8 * pw + 4 * (i >> 4) + (lane >> 3), xa[i]);
        }
        // the segment's alpha is folded into B
        if (S.tB) {
#pragma unroll
          for (int i = 0; i < 16; ++i) split_store(bhi, blo, pw + NPROD * i, lane, S.alpha * xb[i]);
        } else {
#pragma unroll
          for (int i = 0; i < 16; ++i)
            split_store(bhi, blo, 8 * (i & 7) + (lane & 7), 8 * pw + 4 * (i >> 3) + (lane >> 3), S.alpha * xb[i]);
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0) mbar_arrive(&full[s]);
      }
    }
  } else if (warp == 8) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      for (int step = 0; step < nsteps && !aborted(); ++step) {
        const int s = step % STAGES;
        const int blk = step / KB, buf = blk & 1;
        const bool first = (step % KB) == 0;
        if (first && blk >= 2 && !mbar_wait(&dempty[buf], ((blk / 2) - 1) & 1)) {
          fail(ST_TIMEOUT_DE);
          break;
        }
        if (!mbar_wait(&full[s], (step / STAGES) & 1)) {
          fail(ST_TIMEOUT_FULL);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint8_t* st = base + s * STAGE_BYTES;
        const uint32_t d = tmem + (uint32_t)(buf * ACC_COLS);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {  // 8 tf32 = 32 bytes per MMA k slice
          const uint64_t ahi = smem_desc_sw128(st + kk * 32), alo = smem_desc_sw128(st + A_BYTES + kk * 32);
          const uint64_t b = smem_desc_sw128(st + 2 * A_BYTES + kk * 32);  // B hi rows, then B lo rows
          mma_tf32(d, ahi, b, kIdescBoth, (first && kk == 0) ? 0u : 1u);
          mma_tf32(d, alo, b, kIdescHi, 1u);
        }
        mma_commit(&empty[s]);
        if ((step % KB) == KB - 1 || step == nsteps - 1) mma_commit(&dfull[buf]);
      }
      if (aborted()) {
        mma_commit(mma_done);
        mbar_wait(mma_done, 0);
      }
    }
  } else {
    // ---------------- epilogue: FP32 block sums -> FP64 registers -> C ----------------
    const long long r = m0 + warp * 32 + lane;  // C row owned by this thread (TMEM lane)
    double acc[BN];
#pragma unroll
    for (int j = 0; j < BN; ++j) acc[j] = 0.0;
    for (int blk = 0; blk < nblocks && !aborted(); ++blk) {
      const int buf = blk & 1;
      if (!mbar_wait(&dfull[buf], (blk / 2) & 1)) {
        fail(ST_TIMEOUT_D);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int c = 0; c < BN / 16; ++c) {
        uint32_t v[16];
        const uint32_t tq = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * ACC_COLS + c * 16);
        tmem_ld16(tq, v);  // hi x hi + lo x hi
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c * 16 + j] += (double)__uint_as_float(v[j]);
        tmem_ld16(tq + BN, v);  // hi x lo
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c * 16 + j] += (double)__uint_as_float(v[j]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&dempty[buf]);
    }
    if (!aborted() && r < P.M) {
      if (!P.trans_c) {
        double* crow = P.C + r * P.ldc;
#pragma unroll
        for (int j = 0; j < BN; ++j) {
          const long long n = n0 + j;
          if (n < P.N) crow[n] = (P.beta == 0.0 ? 0.0 : P.beta * crow[n]) + acc[j];
        }
      } else {
        // the problem was computed transposed (C^T = B^T A^T): element (r, n) goes to C[n][r]; lanes
        // hold consecutive r, so these stores are coalesced
#pragma unroll
        for (int j = 0; j < BN; ++j) {
          const long long n = n0 + j;
          if (n < P.N) {
            double* c = P.C + n * P.ldc + r;
            *c = (P.beta == 0.0 ? 0.0 : P.beta * *c) + acc[j];
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 8) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ACC_COLS));
}

}  // namespace tci_gtc

namespace tci_gtc_host {

int tile_m() { return tci_gtc::BM; }
int tile_n() { return tci_gtc::BN; }

cudaError_t prepare() {
  static bool done = false;
  if (done) return cudaSuccess;
  cudaError_t e =
      cudaFuncSetAttribute(tci_gtc::gemm_tc_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize, tci_gtc::SMEM_BYTES);
  if (e == cudaSuccess) done = true;
  return e;
}

cudaError_t launch(const tci_dev::DGemmProblem* probs, int nprob, const tci_dev::DGemmSeg* segs, long long ntiles,
                   int* status, int kblock, cudaStream_t st) {
  if (ntiles <= 0 || nprob <= 0) return cudaSuccess;
  tci_gtc::gemm_tc_tf32x3<<<(unsigned)ntiles, tci_gtc::NTHREADS, tci_gtc::SMEM_BYTES, st>>>(
      probs, nprob, segs, status, kblock / tci_gtc::BK);
  return cudaGetLastError();
}

}  // namespace tci_gtc_host
