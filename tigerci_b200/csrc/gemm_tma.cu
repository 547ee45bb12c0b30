// Two-external (internal pair) step of the mixed form fed entirely by TMA:
//
//   R_t (n x n) = beta R_t + sum_s alpha_s X_s D_s
//
// X_s is a (ij|ab) or (ia|jb) integral matrix (static), D_s the dense pair
// matrix of a source CI block (rebuilt every sigma).  Both are kept as TF32
// high / FP32 low parts in HBM (integrals split once at set-up, the pair
// matrices split by a small kernel right after they are unpacked), so the
// kernel streams them with TMA into the 128-byte-swizzle K-major layout with
// no conversion in the loop.  D_s enters as the K-major B operand through its
// symmetry: a pair matrix of a singlet-coupled function is symmetric and of a
// triplet-coupled one antisymmetric, so D^T = p D and the sign p folds into
// alpha.  Each segment (K = n) is one FP32 accumulation block in TMEM; the
// epilogue adds alpha_s p_s times it into FP64 registers, so the segments'
// coefficients never touch the operands.
//
// Warp roles (192 threads): 0-3 epilogue, 4 TMA producer, 5 TMEM allocator +
// MMA issuer.  Bounded waits as in the other tcgen05 kernels; on an abort the
// kernel waits (bounded) for its copies and MMAs in flight, frees its TMEM and
// returns.
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <string>

#include "gemm_tma.h"
#include "tc_common.cuh"

namespace tci_gtma {

using namespace tci_tcx;

constexpr int BM = 128, BN = 64, BK = 32, STAGES = 4;
constexpr int NTHREADS = 192;
constexpr int A_BYTES = BM * BK * 4, B_BYTES = BN * BK * 4;
constexpr int STAGE_BYTES = 2 * A_BYTES + 2 * B_BYTES;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;
constexpr uint32_t kIdesc = idesc_tf32(BM, BN);

enum : int { ST_TIMEOUT_EMPTY = 21, ST_TIMEOUT_FULL = 22, ST_TIMEOUT_D = 23, ST_TIMEOUT_DE = 24 };

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

__global__ void __launch_bounds__(NTHREADS, 1)
    gemm_tma_tf32x3(const __grid_constant__ CUtensorMap xhi, const __grid_constant__ CUtensorMap xlo,
                    const __grid_constant__ CUtensorMap dhi, const __grid_constant__ CUtensorMap dlo,
                    const TmaProblem* __restrict__ probs, int nprob, const TmaSeg* __restrict__ segs, int n,
                    int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
  uint64_t* empty = full + STAGES;
  uint64_t* dfull = empty + STAGES;
  uint64_t* dempty = dfull + 2;
  uint64_t* mma_done = dempty + 2;
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const long long tile = blockIdx.x;
  int lo = 0, hi = nprob - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (probs[mid].tile_begin <= tile) lo = mid;
    else hi = mid - 1;
  }
  const TmaProblem P = probs[lo];
  const long long t = tile - P.tile_begin;
  const int tiles_n = (n + BN - 1) / BN;
  const int m0 = (int)(t / tiles_n) * BM, n0 = (int)(t % tiles_n) * BN;
  const int ksteps = (n + BK - 1) / BK;       // per segment: one FP32 accumulation block
  const int nseg = (int)(P.seg_end - P.seg_begin);
  const int nsteps = nseg * ksteps;

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
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
  if (warp == 5) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(2 * BN));
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

  if (warp == 4) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int last = -1;
      for (int step = 0; step < nsteps && !aborted(); ++step) {
        const int s = step % STAGES;
        if (step >= STAGES && !mbar_wait(&empty[s], ((step / STAGES) - 1) & 1)) {
          fail(ST_TIMEOUT_EMPTY);
          break;
        }
        const TmaSeg S = segs[P.seg_begin + step / ksteps];
        const int k0 = (step % ksteps) * BK;
        uint8_t* st = base + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], 2 * A_BYTES + 2 * B_BYTES);
        tma_load_2d(st, &xhi, &full[s], k0, (int)S.x_row + m0);
        tma_load_2d(st + A_BYTES, &xlo, &full[s], k0, (int)S.x_row + m0);
        tma_load_2d(st + 2 * A_BYTES, &dhi, &full[s], k0, (int)S.d_row + n0);
        tma_load_2d(st + 2 * A_BYTES + B_BYTES, &dlo, &full[s], k0, (int)S.d_row + n0);
        last = step;
      }
      if (aborted())
        for (int step = (last - STAGES + 1 > 0 ? last - STAGES + 1 : 0); step <= last; ++step)
          mbar_wait(&full[step % STAGES], (step / STAGES) & 1);
    }
  } else if (warp == 5) {
    // ---------------- MMA issuer: one TMEM block per segment ----------------
    if (lane == 0) {
      for (int step = 0; step < nsteps && !aborted(); ++step) {
        const int s = step % STAGES;
        const int blk = step / ksteps, buf = blk & 1;
        const bool first = (step % ksteps) == 0;
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
        const uint32_t d = tmem + (uint32_t)(buf * BN);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {
          const uint64_t ahi = smem_desc_sw128(st + kk * 32), alo = smem_desc_sw128(st + A_BYTES + kk * 32);
          const uint64_t bhi = smem_desc_sw128(st + 2 * A_BYTES + kk * 32);
          const uint64_t blo = smem_desc_sw128(st + 2 * A_BYTES + B_BYTES + kk * 32);
          mma_tf32(d, ahi, bhi, kIdesc, (first && kk == 0) ? 0u : 1u);
          mma_tf32(d, ahi, blo, kIdesc, 1u);
          mma_tf32(d, alo, bhi, kIdesc, 1u);
        }
        mma_commit(&empty[s]);
        if ((step % ksteps) == ksteps - 1) mma_commit(&dfull[buf]);
      }
      if (aborted()) {
        mma_commit(mma_done);
        mbar_wait(mma_done, 0);
      }
    }
  } else {
    // ---------------- epilogue: alpha_s * block -> FP64 registers -> R ----------------
    const int r = m0 + warp * 32 + lane;
    double acc[BN];
#pragma unroll
    for (int j = 0; j < BN; ++j) acc[j] = 0.0;
    for (int blk = 0; blk < nseg && !aborted(); ++blk) {
      const int buf = blk & 1;
      const double a = segs[P.seg_begin + blk].alpha;
      if (!mbar_wait(&dfull[buf], (blk / 2) & 1)) {
        fail(ST_TIMEOUT_D);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
#pragma unroll
      for (int c = 0; c < BN / 16; ++c) {
        uint32_t v[16];
        tmem_ld16(tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * BN + c * 16), v);
#pragma unroll
        for (int j = 0; j < 16; ++j) acc[c * 16 + j] = fma(a, (double)__uint_as_float(v[j]), acc[c * 16 + j]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&dempty[buf]);
    }
    if (!aborted() && r < n) {
      double* crow = P.C + (long long)r * n;
#pragma unroll
      for (int j = 0; j < BN; ++j) {
        const int c = n0 + j;
        if (c < n) crow[c] = (P.beta == 0.0 ? 0.0 : P.beta * crow[c]) + acc[j];
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 5) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
}

// rows x n FP64 (row pitch n) -> TF32 hi / FP32 lo with row pitch ldp (columns n..ldp zero)
__global__ void split_rows(const double* __restrict__ src, long long rows, int n, int ldp, float* __restrict__ hi,
                           float* __restrict__ lo) {
  const long long total = rows * ldp;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ldp;
    const int c = (int)(e % ldp);
    float h = 0.0f, l = 0.0f;
    if (c < n) {
      const double x = src[r * n + c];
      h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
      l = (float)(x - (double)h);
    }
    hi[e] = h;
    lo[e] = l;
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
int tile_n() { return tci_gtma::BN; }
int64_t pitch(int64_t n) { return (n + 31) / 32 * 32; }

cudaError_t split(const double* src, int64_t rows, int64_t n, float* hi, float* lo, cudaStream_t st) {
  if (rows <= 0) return cudaSuccess;
  tci_gtma::split_rows<<<148 * 8, 256, 0, st>>>(src, rows, (int)n, (int)pitch(n), hi, lo);
  return cudaGetLastError();
}

bool prepare(TmaMaps& m, const float* xhi, const float* xlo, int64_t xrows, const float* dhi, const float* dlo,
             int64_t drows, int64_t n, std::string& err) {
  m.n = n;
  const uint64_t ldp = (uint64_t)pitch(n);
  if (!make_map(&m.xhi, xhi, xrows, n, ldp, tci_gtma::BM, err) || !make_map(&m.xlo, xlo, xrows, n, ldp, tci_gtma::BM, err) ||
      !make_map(&m.dhi, dhi, drows, n, ldp, tci_gtma::BN, err) || !make_map(&m.dlo, dlo, drows, n, ldp, tci_gtma::BN, err))
    return false;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(tci_gtma::gemm_tma_tf32x3, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tci_gtma::SMEM_BYTES) != cudaSuccess) {
      err = "cannot raise the dynamic shared memory limit";
      return false;
    }
    attr = true;
  }
  return true;
}

cudaError_t launch(const TmaMaps& m, const TmaProblem* probs, int nprob, const TmaSeg* segs, long long ntiles,
                   int* status, cudaStream_t st) {
  if (ntiles <= 0 || nprob <= 0) return cudaSuccess;
  tci_gtma::gemm_tma_tf32x3<<<(unsigned)ntiles, tci_gtma::NTHREADS, tci_gtma::SMEM_BYTES, st>>>(
      m.xhi, m.xlo, m.dhi, m.dlo, probs, nprob, segs, (int)m.n, status);
  return cudaGetLastError();
}

}  // namespace tci_gtma_host
