// Grouped 3xTF32 GEMM on tcgen05 fed entirely by TMA, for plan steps whose
// operands are rows of two fixed arrays (mixed form):
//
//   C_p = beta C_p + sum_s alpha_s A[a_row_s + m, k0_s + k] B[b_row_s + n, k0_s + k]
//
// Both arrays are kept as TF32 high / FP32 low parts in HBM (static operands
// split once at set-up, per-sigma operands split by a small kernel right after
// they are produced), so the kernel streams K-major tiles straight into the
// 128-byte-swizzle layout with no conversion in the loop.  Users: the
// two-external step (integral matrices x pair matrices; the pair matrix enters
// as the K-major B operand through its symmetry, D^T = p D, the sign folded
// into alpha) and the forward three-external step (V_i rows x pair-matrix rows,
// computed transposed).  A segment's k steps form FP32 accumulation blocks of
// at most kblock elements in a double-buffered TMEM accumulator; the epilogue
// adds alpha_s times each block into FP64 registers, so the coefficients never
// touch the operands, and writes C (or C^T) once, or, for a product that feeds
// the next one, its TF32 high / FP32 low parts.
//
// Tiles are 128 x 128 (or 128 x 64).  The kernel is persistent: one CTA per
// SM walks tiles blockIdx.x, blockIdx.x + gridDim.x, ..., with the stage ring
// and the two TMEM accumulator buffers carrying on from tile to tile, so a
// tile's epilogue overlaps the next tile's loads and MMAs (the steps with
// short K, such as the pair-domain products, are made of many small tiles).
// Warp roles (320 threads): 0-7 epilogue (two warps per TMEM lane quadrant,
// one per half of the tile's columns), 8 TMA producer, 9 TMEM allocator + MMA
// issuer.  Bounded waits; on an abort the kernel waits (bounded) for its
// copies and MMAs in flight, frees its TMEM and returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "device_info.h"
#include "gemm_tma.h"
#include "tc_common.cuh"

namespace tci_gtma {

using namespace tci_tcx;

constexpr int BM = 128, BK = 32;
constexpr int NTHREADS = 320;
constexpr int EPI_WARPS = 8;  // warps 0-3: first half of the tile's columns, 4-7: second half (TMEM quadrant = warp mod 4)
constexpr int A_BYTES = BM * BK * 4;
// Output staging: per epilogue warp 32 rows x 33 floats (or 32 x 16 doubles), so that rows leave the
// epilogue as coalesced 128-byte segments instead of one scattered word per row.
constexpr int STAGE_OUT_FLOATS = 32 * 33;
constexpr int SMEM_BYTES = 192 * 1024 + 1024 + 256 + 8 * STAGE_OUT_FLOATS * 4;  // 192 KB of stages
// Tile width BN = 128 (wide operands) or 64 (B with few rows).  B's high rows are followed by its low
// rows in a stage, so A_hi x [B_hi; B_lo] is one MMA of N = 2 BN and A_lo x B_hi a second one: two
// instructions per k slice (an MMA costs about the same time whatever its N, so wide tiles and few
// instructions are what count).
template <int BN>
struct Tile {
  static constexpr int B_BYTES = BN * BK * 4;
  static constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
  static constexpr int STAGES = (192 * 1024) / STAGE_BYTES;  // 3 (BN 128) or 4 (BN 64)
  static constexpr uint32_t kIdescBoth = idesc_tf32(BM, 2 * BN), kIdescHi = idesc_tf32(BM, BN);
  static constexpr int ACC_COLS = 2 * BN;  // hi x hi + lo x hi, then hi x lo
};

enum : int { ST_TIMEOUT_EMPTY = 21, ST_TIMEOUT_FULL = 22, ST_TIMEOUT_D = 23, ST_TIMEOUT_DE = 24 };

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

template <int BN>
__global__ void __launch_bounds__(NTHREADS, 1)
    gemm_tma_tf32x3(const __grid_constant__ CUtensorMap ahi_map, const __grid_constant__ CUtensorMap alo_map,
                    const __grid_constant__ CUtensorMap bhi_map, const __grid_constant__ CUtensorMap blo_map,
                    const TmaProblem* __restrict__ probs, int nprob, const TmaSeg* __restrict__ segs, long long ntiles,
                    int kbs, int* __restrict__ status) {
  using T = Tile<BN>;
  constexpr int STAGES = T::STAGES, STAGE_BYTES = T::STAGE_BYTES, B_BYTES = T::B_BYTES, ACC_COLS = T::ACC_COLS;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* dfull = empty + STAGES;
  uint64_t* dempty = dfull + 2;
  uint64_t* mma_done = dempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);
  float* stage_out = reinterpret_cast<float*>(base + STAGES * STAGE_BYTES + 256);  // EPI_WARPS x STAGE_OUT_FLOATS

  // persistent: tiles blockIdx.x, blockIdx.x + gridDim.x, ...; every role walks the same tiles in the same
  // order, the stage ring and the two TMEM accumulator buffers carry on from tile to tile
  struct TileAt {
    int prob, m0, n0;
  };
  auto tile_at = [&](long long tile) {
    int lo = 0, hi = nprob - 1;
    while (lo < hi) {
      const int mid = (lo + hi + 1) >> 1;
      if (probs[mid].tile_begin <= tile) lo = mid;
      else hi = mid - 1;
    }
    const long long t = tile - probs[lo].tile_begin;
    return TileAt{lo, (int)(t / probs[lo].tiles_n) * BM, (int)(t % probs[lo].tiles_n) * BN};
  };

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&empty[s], 1);
    }
    for (int b = 0; b < 2; ++b) {
      mbar_init(&dfull[b], 1);
      mbar_init(&dempty[b], EPI_WARPS);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 9) {
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

  if (warp == 8) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int step = 0, last = -1;
      for (long long tile = blockIdx.x; tile < ntiles && !aborted(); tile += gridDim.x) {
        const TileAt ta = tile_at(tile);
        const TmaProblem& P = probs[ta.prob];
        const int m0 = ta.m0, n0 = ta.n0;
        for (long long q = P.seg_begin; q < P.seg_end && !aborted(); ++q) {
          const TmaSeg S = segs[q];
          const int nk = (int)((S.K + BK - 1) / BK);
          for (int kk = 0; kk < nk && !aborted(); ++kk, ++step) {
            const int s = step % STAGES;
            if (step >= STAGES && !mbar_wait(&empty[s], ((step / STAGES) - 1) & 1)) {
              fail(ST_TIMEOUT_EMPTY);
              break;
            }
            const int x = (int)S.k0 + kk * BK;
            uint8_t* st = base + s * STAGE_BYTES;
            mbar_expect_tx(&full[s], 2 * A_BYTES + 2 * B_BYTES);
            tma_load_2d(st, &ahi_map, &full[s], x, (int)S.a_row + m0);
            tma_load_2d(st + A_BYTES, &alo_map, &full[s], x, (int)S.a_row + m0);
            tma_load_2d(st + 2 * A_BYTES, &bhi_map, &full[s], x, (int)S.b_row + n0);
            tma_load_2d(st + 2 * A_BYTES + B_BYTES, &blo_map, &full[s], x, (int)S.b_row + n0);
            last = step;
          }
        }
      }
      if (aborted())
        for (int st = (last - STAGES + 1 > 0 ? last - STAGES + 1 : 0); st <= last; ++st)
          mbar_wait(&full[st % STAGES], (st / STAGES) & 1);
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer: blocks of at most kbs k steps, never across segments ----------------
    if (lane == 0) {
      int step = 0, blk = 0;
      for (long long tile = blockIdx.x; tile < ntiles && !aborted(); tile += gridDim.x) {
        const TmaProblem& P = probs[tile_at(tile).prob];
        for (long long q = P.seg_begin; q < P.seg_end && !aborted(); ++q) {
          const int nk = (int)((segs[q].K + BK - 1) / BK);
          for (int kk = 0; kk < nk && !aborted(); ++kk, ++step) {
            const int s = step % STAGES, buf = blk & 1;
            const bool first = (kk % kbs) == 0;
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
            for (int k8 = 0; k8 < BK / 8; ++k8) {
              const uint64_t ahi = smem_desc_sw128(st + k8 * 32), alo = smem_desc_sw128(st + A_BYTES + k8 * 32);
              const uint64_t b = smem_desc_sw128(st + 2 * A_BYTES + k8 * 32);  // B hi rows, then B lo rows
              mma_tf32(d, ahi, b, T::kIdescBoth, (first && k8 == 0) ? 0u : 1u);
              mma_tf32(d, alo, b, T::kIdescHi, 1u);
            }
            mma_commit(&empty[s]);
            if ((kk % kbs) == kbs - 1 || kk == nk - 1) {
              mma_commit(&dfull[buf]);
              ++blk;
            }
          }
        }
      }
      if (aborted()) {
        mma_commit(mma_done);
        mbar_wait(mma_done, 0);
      }
    }
  } else {
    // ---------------- epilogue: alpha_s * block -> FP64 registers -> C ----------------
    constexpr int COLS = BN / 2;  // tile columns per epilogue warp
    const int quad = warp & 3, half = warp >> 2;  // TMEM lane quadrant (= warp mod 4), column half
    int blk = 0;
    for (long long tile = blockIdx.x; tile < ntiles && !aborted(); tile += gridDim.x) {
      const TileAt ta = tile_at(tile);
      const TmaProblem& P = probs[ta.prob];
      const long long r = ta.m0 + quad * 32 + lane;
      const int nc0 = ta.n0 + half * COLS;  // first output column of this warp
      double acc[COLS];
#pragma unroll
      for (int j = 0; j < COLS; ++j) acc[j] = 0.0;
      for (long long q = P.seg_begin; q < P.seg_end && !aborted(); ++q) {
        const double a = segs[q].alpha;
        const int nk = (int)((segs[q].K + BK - 1) / BK);
        const int nb = (nk + kbs - 1) / kbs;
        for (int b = 0; b < nb && !aborted(); ++b, ++blk) {
          const int buf = blk & 1;
          if (!mbar_wait(&dfull[buf], (blk / 2) & 1)) {
            fail(ST_TIMEOUT_D);
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
          for (int c = 0; c < COLS / 16; ++c) {
            uint32_t v[16];
            const uint32_t tq =
                tmem + ((uint32_t)(quad * 32) << 16) + (uint32_t)(buf * ACC_COLS + half * COLS + c * 16);
            tmem_ld16(tq, v);  // hi x hi + lo x hi
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[c * 16 + j] = fma(a, (double)__uint_as_float(v[j]), acc[c * 16 + j]);
            tmem_ld16(tq + BN, v);  // hi x lo
#pragma unroll
            for (int j = 0; j < 16; ++j) acc[c * 16 + j] = fma(a, (double)__uint_as_float(v[j]), acc[c * 16 + j]);
          }
          asm volatile("tcgen05.fence::before_thread_sync;");
          __syncwarp();
          if (lane == 0) mbar_arrive(&dempty[buf]);
        }
      }
      // warp-uniform abort test: the staged stores below are warp-wide
      const bool stop = __any_sync(0xffffffffu, aborted());
      const long long r0w = ta.m0 + quad * 32;  // the warp's first row
      float* sb = stage_out + warp * STAGE_OUT_FLOATS;
      if (!stop && P.c_hi) {
        // split output (the next product's operand, in the layout split_rows writes): 32 x 32 blocks through
        // shared memory, high parts then low parts, each row written as one 128-byte segment
#pragma unroll
        for (int c0 = 0; c0 < COLS; c0 += 32)
#pragma unroll 1
          for (int part = 0; part < 2; ++part) {
#pragma unroll
            for (int jj = 0; jj < 32; ++jj) {
              const double x = acc[c0 + jj];
              const float h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
              sb[lane * 33 + jj] = part == 0 ? h : (float)(x - (double)h);
            }
            __syncwarp();
            float* out = part == 0 ? P.c_hi : P.c_lo;
            const long long col = nc0 + c0 + lane;
            for (int i = 0; i < 32; ++i) {
              const long long row = r0w + i;
              if (row < P.M && col < P.N) out[row * P.ldcs + col] = sb[i * 33 + lane];
            }
            __syncwarp();
          }
      } else if (!stop && !P.trans_c) {
        // FP64 rows: 32 x 16 blocks through shared memory (XOR-swizzled columns), two rows per store
        double* db = reinterpret_cast<double*>(sb);
#pragma unroll
        for (int c0 = 0; c0 < COLS; c0 += 16) {
#pragma unroll
          for (int jj = 0; jj < 16; ++jj) db[lane * 16 + (jj ^ (lane & 15))] = acc[c0 + jj];
          __syncwarp();
          for (int ii = 0; ii < 16; ++ii) {
            const int i = 2 * ii + (lane >> 4), j = lane & 15;
            const double v = db[i * 16 + (j ^ (i & 15))];
            const long long row = r0w + i, col = nc0 + c0 + j;
            if (row < P.M && col < P.N) {
              double* y = P.C + row * P.ldc + col;
              *y = (P.beta == 0.0 ? 0.0 : P.beta * *y) + v;
            }
          }
          __syncwarp();
        }
      } else if (!stop && r < P.M) {  // C^T: element (r, c) goes to C[c][r]; lanes hold consecutive r (coalesced)
#pragma unroll
        for (int j = 0; j < COLS; ++j) {
          const long long c = nc0 + j;
          if (c < P.N) {
            double* y = P.C + c * P.ldc + r;
            *y = (P.beta == 0.0 ? 0.0 : P.beta * *y) + acc[j];
          }
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 9) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * ACC_COLS));
}

// rows x cols FP64 (row pitch ld) -> TF32 hi / FP32 lo with row pitch ldp (columns cols..ldp zero)
__global__ void split_rows(const double* __restrict__ src, long long rows, long long cols, long long ld, long long ldp,
                           float* __restrict__ hi, float* __restrict__ lo) {
  const long long total = rows * ldp;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ldp, c = e % ldp;
    float h = 0.0f, l = 0.0f;
    if (c < cols) {
      const double x = src[r * ld + c];
      h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
      l = (float)(x - (double)h);
    }
    hi[e] = h;
    lo[e] = l;
  }
}

// nmat matrices of rows x cols FP64 (row-major, consecutive) -> their transposes as TF32 hi / FP32 lo
// rows of pitch ldp: row mat cols + c holds column c of matrix mat (columns rows..ldp untouched).
// 32 x 32 tiles through shared memory; grid (ceil(cols/32), ceil(rows/32), nmat), block 32 x 8.
__global__ void split_transposed(const double* __restrict__ src, long long rows, long long cols, long long ldp,
                                 float* __restrict__ hi, float* __restrict__ lo) {
  __shared__ double t[32][33];
  const long long mat = blockIdx.z;
  const long long c0 = (long long)blockIdx.x * 32, r0 = (long long)blockIdx.y * 32;
  const double* m = src + mat * rows * cols;
  for (int y = threadIdx.y; y < 32; y += 8) {
    const long long r = r0 + y, c = c0 + threadIdx.x;
    if (r < rows && c < cols) t[y][threadIdx.x] = m[r * cols + c];
  }
  __syncthreads();
  for (int y = threadIdx.y; y < 32; y += 8) {
    const long long c = c0 + y, r = r0 + threadIdx.x;  // output row c, column r
    if (r < rows && c < cols) {
      const double x = t[threadIdx.x][y];
      const float h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
      const long long o = (mat * cols + c) * ldp + r;
      hi[o] = h;
      lo[o] = (float)(x - (double)h);
    }
  }
}

}  // namespace tci_gtma

namespace {

typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                  const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
  static EncodeTiledFn fn = nullptr;
  if (!fn) {
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
      return nullptr;
    fn = reinterpret_cast<EncodeTiledFn>(p);
  }
  return fn;
}

// rows x n FP32 matrix with row pitch ldp; box BK x box_rows; out-of-range reads are zero
bool make_map(CUtensorMap* map, const float* p, uint64_t rows, uint64_t n, uint64_t ldp, uint32_t box_rows,
              std::string& err) {
  auto fn = encode_fn();
  if (!fn) {
    err = "cuTensorMapEncodeTiled unavailable";
    return false;
  }
  if ((reinterpret_cast<uintptr_t>(p) & 15) || ((ldp * 4) & 15)) {
    err = "tensor map base / pitch not 16-byte aligned";
    return false;
  }
  const cuuint64_t dims[2] = {n, rows};
  const cuuint64_t strides[1] = {ldp * 4};
  const cuuint32_t box[2] = {(cuuint32_t)tci_gtma::BK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  const CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(p), dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

}  // namespace

namespace tci_gtma_host {

int tile_m() { return tci_gtma::BM; }
int tile_n(bool wide) { return wide ? 128 : 64; }
int64_t pitch(int64_t cols) { return (cols + 31) / 32 * 32; }

cudaError_t split(const double* src, int64_t rows, int64_t cols, int64_t ld, float* hi, float* lo, cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  tci_gtma::split_rows<<<tci_dev::device_sms() * 8, 256, 0, st>>>(src, rows, cols, ld, pitch(cols), hi, lo);
  return cudaGetLastError();
}

cudaError_t split_transposed(const double* src, int64_t nmat, int64_t rows, int64_t cols, float* hi, float* lo,
                             cudaStream_t st) {
  if (nmat <= 0 || rows <= 0 || cols <= 0) return cudaSuccess;
  const int64_t ldp = pitch(rows);
  // zero the padding columns once (every element below rows is written by the kernel)
  cudaError_t e = cudaMemsetAsync(hi, 0, sizeof(float) * (size_t)(nmat * cols * ldp), st);
  if (e == cudaSuccess) e = cudaMemsetAsync(lo, 0, sizeof(float) * (size_t)(nmat * cols * ldp), st);
  if (e != cudaSuccess) return e;
  dim3 grid((unsigned)((cols + 31) / 32), (unsigned)((rows + 31) / 32), (unsigned)nmat);
  tci_gtma::split_transposed<<<grid, dim3(32, 8), 0, st>>>(src, rows, cols, ldp, hi, lo);
  return cudaGetLastError();
}

bool prepare(TmaMaps& m, const float* ahi, const float* alo, int64_t arows, int64_t acols, const float* bhi,
             const float* blo, int64_t brows, int64_t bcols, bool wide, std::string& err) {
  m.wide = wide;
  const uint32_t bn = (uint32_t)tile_n(wide);
  if (!make_map(&m.ahi, ahi, arows, acols, pitch(acols), tci_gtma::BM, err) ||
      !make_map(&m.alo, alo, arows, acols, pitch(acols), tci_gtma::BM, err) ||
      !make_map(&m.bhi, bhi, brows, bcols, pitch(bcols), bn, err) ||
      !make_map(&m.blo, blo, brows, bcols, pitch(bcols), bn, err))
    return false;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(tci_gtma::gemm_tma_tf32x3<128>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tci_gtma::SMEM_BYTES) != cudaSuccess ||
        cudaFuncSetAttribute(tci_gtma::gemm_tma_tf32x3<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tci_gtma::SMEM_BYTES) != cudaSuccess) {
      err = "cannot raise the dynamic shared memory limit";
      return false;
    }
    attr = true;
  }
  return true;
}

cudaError_t launch(const TmaMaps& m, const TmaProblem* probs, int nprob, const TmaSeg* segs, long long ntiles,
                   int kblock, int* status, cudaStream_t st, bool persistent) {
  if (ntiles <= 0 || nprob <= 0) return cudaSuccess;
  // persistent: one CTA per SM (the stages take 192 KB of shared memory); otherwise a CTA per tile, which
  // the hardware schedules dynamically (better for few tiles of very uneven length)
  const long long sms = tci_dev::device_sms();
  const unsigned grid = (unsigned)(persistent ? std::min<long long>(ntiles, sms) : ntiles);
  if (m.wide)
    tci_gtma::gemm_tma_tf32x3<128><<<grid, tci_gtma::NTHREADS, tci_gtma::SMEM_BYTES, st>>>(
        m.ahi, m.alo, m.bhi, m.blo, probs, nprob, segs, ntiles, kblock / tci_gtma::BK, status);
  else
    tci_gtma::gemm_tma_tf32x3<64><<<grid, tci_gtma::NTHREADS, tci_gtma::SMEM_BYTES, st>>>(
        m.ahi, m.alo, m.bhi, m.blo, probs, nprob, segs, ntiles, kblock / tci_gtma::BK, status);
  return cudaGetLastError();
}

}  // namespace tci_gtma_host
