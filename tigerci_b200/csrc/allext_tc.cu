// Mixed-precision all-external product on the 5th-generation tensor cores.
//
//   Y[j][r] = sum_k W[r][k] U[j][k]      (W symmetric np x np, U: m CI blocks)
//
// W (the packed all-external operator W+ or W-, see plan.cpp) is stored in HBM
// as FP32 and streamed once per sigma build by TMA (128-byte swizzle).  Each
// W tile is split in shared memory into TF32 hi/lo parts; U arrives pre-split.
// Three kind::tf32 MMAs per k-step (hi*hi + hi*lo + lo*hi) accumulate FP32 in
// TMEM; every KBLOCK elements of k the partial sums are read back with
// tcgen05.ld and added into FP64 accumulators held in registers (promotion
// keeps the FP32 accumulation error at the block length), which are written
// to the output once at the end.  The product is HBM bound: W is read exactly
// once.  One launch covers both operators (W+ with the singlet blocks, W-
// with the triplet blocks), so their tiles share the waves.
//
// Warp roles (320 threads): warps 0-3 epilogue (TMEM lane quadrants 0-3),
// warps 4-7 hi/lo split, warp 8 TMA producer, warp 9 TMEM allocator + MMA
// issuer.  Every mbarrier wait is bounded; on timeout the kernel records an
// error code, drains and returns (no trap).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>

#include "allext_tc.h"

namespace tci_tc {

constexpr int BM = 128;      // W rows per CTA tile (MMA M)
constexpr int BN = 64;       // CI blocks per tile (MMA N)
constexpr int BK = 32;       // fp32 k elements per stage (one 128-byte swizzle row)
constexpr int STAGES = 4;
// The FP64 promotion block (k elements summed in TMEM before the FP64 add) is
// a launch parameter: the tensor core's FP32 accumulation error grows with it.
constexpr int W_BYTES = BM * BK * 4;   // 16 KB
constexpr int U_BYTES = BN * BK * 4;   // 8 KB
constexpr int STAGE_BYTES = 2 * W_BYTES + 2 * U_BYTES;
constexpr int NTHREADS = 320;
constexpr long long SPIN_LIMIT = 1ll << 22;  // bounded mbarrier waits (~seconds)

struct Smem {
  // stage buffers start at a 1024-byte aligned base (128B swizzle atoms)
  uint8_t* base;
};

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}

__device__ __forceinline__ void mbar_init(uint64_t* bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t* bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}
// Bounded wait for the phase with the given parity; returns false on timeout.
__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t parity) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < SPIN_LIMIT; ++i) {
    uint32_t done;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(done)
        : "r"(a), "r"(parity)
        : "memory");
    if (done) return true;
  }
  return false;
}

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}

// tcgen05 shared-memory matrix descriptor: K-major, 128-byte swizzle,
// 8-row core matrices 1024 bytes apart (SBO), version 1.
__device__ __forceinline__ uint64_t smem_desc(const void* p) {
  const uint64_t addr = smem_u32(p);
  uint64_t d = 0;
  d |= (addr & 0x3FFFFull) >> 4;           // start address
  d |= (uint64_t)(16 >> 4) << 16;          // leading byte offset (unused for swizzled K-major)
  d |= (uint64_t)(1024 >> 4) << 32;        // stride byte offset
  d |= (uint64_t)1 << 46;                  // descriptor version
  d |= (uint64_t)2 << 61;                  // 128-byte swizzle
  return d;
}

// Instruction descriptor: D f32, A/B tf32, both K-major, M = 128, N = 64.
constexpr uint32_t kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((uint32_t)(BN >> 3) << 17) | ((uint32_t)(BM >> 4) << 24);

__device__ __forceinline__ void mma_tf32(uint32_t d_tmem, uint64_t a, uint64_t b, uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], %1, %2, %3, p;\n}\n" ::"r"(d_tmem),
      "l"(a), "l"(b), "r"(kIdesc), "r"(accumulate));
}
__device__ __forceinline__ void mma_commit(uint64_t* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(smem_u32(bar))
               : "memory");
}

// Error codes written to the kernel's status word.
enum : int { ST_OK = 0, ST_TIMEOUT_FULL = 1, ST_TIMEOUT_CONV = 2, ST_TIMEOUT_EMPTY = 3, ST_TIMEOUT_D = 4, ST_TIMEOUT_DE = 5 };

// One product of the launch: Y (m x np, row pitch ldy) = U W over `tiles`
// panels of BM W rows.
struct Product {
  int np, m, tiles;
  double* Y;
  long long ldy;
};

__global__ void __launch_bounds__(NTHREADS, 1)
    allext_tf32x3_kernel(const __grid_constant__ CUtensorMap wmap0, const __grid_constant__ CUtensorMap uhi_map0,
                         const __grid_constant__ CUtensorMap ulo_map0, const __grid_constant__ CUtensorMap wmap1,
                         const __grid_constant__ CUtensorMap uhi_map1, const __grid_constant__ CUtensorMap ulo_map1,
                         Product p0, Product p1, int* __restrict__ status, int kb_per_block, int ksplit) {
  const int KB_PER_BLOCK = kb_per_block;
  // CTA -> (tile, k split); which product the tile belongs to (uniform over the CTA: the early exit
  // precedes all set-up)
  const int tile = (int)blockIdx.x / ksplit, split = (int)blockIdx.x % ksplit;
  const bool second = tile >= p0.tiles;
  const Product P = second ? p1 : p0;
  const CUtensorMap* wmap = second ? &wmap1 : &wmap0;
  const CUtensorMap* uhi_map = second ? &uhi_map1 : &uhi_map0;
  const CUtensorMap* ulo_map = second ? &ulo_map1 : &ulo_map0;
  const int np = P.np, m = P.m;
  const int ublock = blockIdx.y;       // which group of BN CI blocks
  if (ublock * BN >= m) return;
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint64_t* full = reinterpret_cast<uint64_t*>(base + STAGES * STAGE_BYTES);
  uint64_t* conv = full + STAGES;
  uint64_t* empty = conv + STAGES;
  uint64_t* dfull = empty + STAGES;   // 2
  uint64_t* dempty = dfull + 2;       // 2
  uint64_t* mma_done = dempty + 2;    // 1: drain of the MMAs in flight after an abort
  uint32_t* tmem_slot = reinterpret_cast<uint32_t*>(mma_done + 1);
  int* abort_flag = reinterpret_cast<int*>(tmem_slot + 1);

  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int row0 = (second ? tile - p0.tiles : tile) * BM;
  // k steps of this split: [kbase, kbase + nk)
  const int nk_all = (np + BK - 1) / BK, per = (nk_all + ksplit - 1) / ksplit;
  const int kbase = split * per;
  const int nk = nk_all - kbase < per ? (nk_all - kbase > 0 ? nk_all - kbase : 0) : per;
  const int nblocks = (nk + KB_PER_BLOCK - 1) / KB_PER_BLOCK;

  if (threadIdx.x == 0) {
    for (int s = 0; s < STAGES; ++s) {
      mbar_init(&full[s], 1);
      mbar_init(&conv[s], 4);
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
  if (warp == 9) {  // TMEM: 2 accumulator buffers of BN fp32 columns
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

  if (warp == 8) {
    // ---------------- TMA producer ----------------
    if (lane == 0) {
      int last = -1;  // last k-step whose copies were issued
      for (int kb = 0; kb < nk && !aborted(); ++kb) {
        const int s = kb % STAGES;
        if (kb >= STAGES && !mbar_wait(&empty[s], ((kb / STAGES) - 1) & 1)) {
          fail(ST_TIMEOUT_EMPTY);
          break;
        }
        uint8_t* st = base + s * STAGE_BYTES;
        mbar_expect_tx(&full[s], W_BYTES + 2 * U_BYTES);
        tma_load_2d(st, wmap, &full[s], (kbase + kb) * BK, row0);
        tma_load_2d(st + 2 * W_BYTES, uhi_map, &full[s], (kbase + kb) * BK, ublock * BN);
        tma_load_2d(st + 2 * W_BYTES + U_BYTES, ulo_map, &full[s], (kbase + kb) * BK, ublock * BN);
        last = kb;
      }
      if (aborted()) {
        // the copies of the last STAGES issued k-steps may still be landing: wait (bounded) for them
        // before the shared memory is released
        for (int kb = (last - STAGES + 1 > 0 ? last - STAGES + 1 : 0); kb <= last; ++kb)
          mbar_wait(&full[kb % STAGES], (kb / STAGES) & 1);
      }
    }
  } else if (warp >= 4 && warp < 8) {
    // ---------------- TF32 hi/lo split of the W tile (in place + lo copy) ----------------
    const int cw = warp - 4;
    for (int kb = 0; kb < nk && !aborted(); ++kb) {
      const int s = kb % STAGES;
      if (!mbar_wait(&full[s], (kb / STAGES) & 1)) {
        fail(ST_TIMEOUT_FULL);
        break;
      }
      uint32_t* whi = reinterpret_cast<uint32_t*>(base + s * STAGE_BYTES);
      uint32_t* wlo = reinterpret_cast<uint32_t*>(base + s * STAGE_BYTES + W_BYTES);
      // a warp per 128-byte row: lane l holds element l (conflict free; the
      // swizzle permutes 16-byte chunks within the row, lo keeps the same layout).
      // Eight rows per batch: their loads are issued before any store, so the
      // shared-memory latency is paid once per batch.
#pragma unroll
      for (int r0 = cw; r0 < BM; r0 += 4 * 8) {
        uint32_t x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = whi[(r0 + 4 * i) * BK + lane];
#pragma unroll
        for (int i = 0; i < 8; ++i) {
          const uint32_t hi = x[i] & 0xFFFFE000u;
          const float lo = __uint_as_float(x[i]) - __uint_as_float(hi);
          whi[(r0 + 4 * i) * BK + lane] = hi;
          wlo[(r0 + 4 * i) * BK + lane] = __float_as_uint(lo);
        }
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer ----------------
    if (lane == 0) {
      for (int kb = 0; kb < nk && !aborted(); ++kb) {
        const int s = kb % STAGES;
        const int blk = kb / KB_PER_BLOCK, buf = blk & 1;
        const bool first = (kb % KB_PER_BLOCK) == 0;
        if (first && blk >= 2 && !mbar_wait(&dempty[buf], ((blk / 2) - 1) & 1)) {
          fail(ST_TIMEOUT_DE);
          break;
        }
        if (!mbar_wait(&conv[s], (kb / STAGES) & 1)) {
          fail(ST_TIMEOUT_CONV);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        uint8_t* st = base + s * STAGE_BYTES;
        const uint32_t d = tmem + (uint32_t)(buf * BN);
#pragma unroll
        for (int kk = 0; kk < BK / 8; ++kk) {  // 8 tf32 = 32 bytes per MMA step
          const uint64_t ahi = smem_desc(st + kk * 32), alo = smem_desc(st + W_BYTES + kk * 32);
          const uint64_t bhi = smem_desc(st + 2 * W_BYTES + kk * 32);
          const uint64_t blo = smem_desc(st + 2 * W_BYTES + U_BYTES + kk * 32);
          mma_tf32(d, ahi, bhi, (first && kk == 0) ? 0u : 1u);
          mma_tf32(d, ahi, blo, 1u);
          mma_tf32(d, alo, bhi, 1u);
        }
        mma_commit(&empty[s]);
        if ((kb % KB_PER_BLOCK) == KB_PER_BLOCK - 1 || kb == nk - 1) mma_commit(&dfull[buf]);
      }
      if (aborted()) {
        // MMAs issued before the abort may still be writing TMEM: wait (bounded) for all of them
        mma_commit(mma_done);
        mbar_wait(mma_done, 0);
      }
    }
  } else {
    // ---------------- epilogue: FP32 block sums -> FP64 register accumulators ----------------
    const int r = row0 + warp * 32 + lane;  // W row owned by this thread
    double acc[BN];
#pragma unroll
    for (int t = 0; t < BN; ++t) acc[t] = 0.0;
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
        const uint32_t taddr = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * BN + c * 16);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7]),
              "=r"(v[8]), "=r"(v[9]), "=r"(v[10]), "=r"(v[11]), "=r"(v[12]), "=r"(v[13]), "=r"(v[14]), "=r"(v[15])
            : "r"(taddr));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
        for (int t = 0; t < 16; ++t) acc[c * 16 + t] += (double)__uint_as_float(v[t]);
      }
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&dempty[buf]);
    }
    if (!aborted() && r < np) {
#pragma unroll
      for (int t = 0; t < BN; ++t) {
        const int j = ublock * BN + t;
        if (j < m) {
          // two splits add into the zeroed output: x + y rounds the same in either order, so the
          // result does not depend on which split finishes first
          if (ksplit == 1) P.Y[(long long)j * P.ldy + r] = acc[t];
          else atomicAdd(&P.Y[(long long)j * P.ldy + r], acc[t]);
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 9) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(2 * BN));
}

// FP64 -> FP32 copy with a padded leading dimension (W at init).
__global__ void to_f32_padded(const double* __restrict__ src, long long rows, long long cols, long long lds,
                              float* __restrict__ dst, long long ldd) {
  const long long total = rows * ldd;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long r = e / ldd, c = e % ldd;
    dst[e] = (c < cols) ? (float)src[r * lds + c] : 0.0f;
  }
}

// U (m x np, FP64) -> TF32 hi (masked) and lo parts, rows padded to a multiple of BN.
__global__ void split_u(const double* __restrict__ U, int m, int np, long long ldu, float* __restrict__ hi,
                        float* __restrict__ lo, int mpad, long long ldw) {
  const long long total = (long long)mpad * ldw;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long j = e / ldw, k = e % ldw;
    float h = 0.0f, l = 0.0f;
    if (j < m && k < np) {
      const double x = U[j * ldu + k];
      const float xf = (float)x;
      h = __uint_as_float(__float_as_uint(xf) & 0xFFFFE000u);
      l = (float)(x - (double)h);
    }
    hi[e] = h;
    lo[e] = l;
  }
}

}  // namespace tci_tc

// ---------------------------------------------------------------------------
namespace {

// signature of cuTensorMapEncodeTiled (driver API), resolved at run time
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

bool make_map(CUtensorMap* map, const float* base, uint64_t rows, uint64_t cols, uint64_t ld, uint32_t box_rows,
              std::string& err) {
  auto fn = encode_fn();
  if (!fn) {
    err = "cuTensorMapEncodeTiled unavailable";
    return false;
  }
  if ((reinterpret_cast<uintptr_t>(base) & 15) || ((ld * 4) & 15)) {
    err = "tensor map base / stride not 16-byte aligned";
    return false;
  }
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {ld * 4};
  const cuuint32_t box[2] = {(cuuint32_t)tci_tc::BK, box_rows};
  const cuuint32_t estr[2] = {1, 1};
  CUresult r = fn(map, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<float*>(base), dims, strides, box, estr,
                  CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                  CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) {
    err = "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")";
    return false;
  }
  return true;
}

}  // namespace

namespace tci_tc_host {

int64_t padded_ld(int64_t np) { return (np + 31) / 32 * 32; }
int64_t padded_rows(int64_t m) { return (m + tci_tc::BN - 1) / tci_tc::BN * tci_tc::BN; }

cudaError_t convert_w(const double* w64, int64_t np, float* w32, cudaStream_t st) {
  tci_tc::to_f32_padded<<<148 * 16, 256, 0, st>>>(w64, np, np, np, w32, padded_ld(np));
  return cudaGetLastError();
}

cudaError_t split_u(const double* u, int64_t m, int64_t np, float* hi, float* lo, cudaStream_t st) {
  tci_tc::split_u<<<148 * 4, 256, 0, st>>>(u, (int)m, (int)np, np, hi, lo, (int)padded_rows(m), padded_ld(np));
  return cudaGetLastError();
}

bool prepare(AllextTc& t, const float* w32, int64_t np, const float* uhi, const float* ulo, int64_t m, double* y,
             int* status, int64_t kblock, std::string& err) {
  if (kblock < tci_tc::BK || kblock % tci_tc::BK) {
    err = "promotion block must be a positive multiple of 32";
    return false;
  }
  t.kblock = kblock;
  t.np = np;
  t.m = m;
  t.y = y;
  t.status = status;
  const uint64_t ld = (uint64_t)padded_ld(np);
  if (!make_map(&t.wmap, w32, np, np, ld, tci_tc::BM, err)) return false;
  if (!make_map(&t.uhi, uhi, padded_rows(m), np, ld, tci_tc::BN, err)) return false;
  if (!make_map(&t.ulo, ulo, padded_rows(m), np, ld, tci_tc::BN, err)) return false;
  static bool attr = false;
  if (!attr) {
    const int smem = tci_tc::STAGES * tci_tc::STAGE_BYTES + 1024 + 256;
    if (cudaFuncSetAttribute(tci_tc::allext_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem) !=
        cudaSuccess) {
      err = "cannot raise the dynamic shared memory limit";
      return false;
    }
    attr = true;
  }
  return true;
}

// Two k splits when the tiles fill fewer than four waves of one CTA per SM: the
// last, partly filled wave then costs less (more than two splits would make
// the atomic accumulation order-dependent).
int ksplit(const AllextTc* a, const AllextTc* b) {
  if (!a) std::swap(a, b);
  if (!a) return 1;
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const int64_t ub = std::max(padded_rows(a->m), b ? padded_rows(b->m) : 0) / tci_tc::BN;
  const int64_t tiles = ((a->np + tci_tc::BM - 1) / tci_tc::BM + (b ? (b->np + tci_tc::BM - 1) / tci_tc::BM : 0)) * ub;
  return tiles < 4 * (int64_t)sms ? 2 : 1;
}

cudaError_t launch(const AllextTc* a, const AllextTc* b, cudaStream_t st) {
  if (!a && !b) return cudaSuccess;
  if (!a) std::swap(a, b);
  const int smem = tci_tc::STAGES * tci_tc::STAGE_BYTES + 1024 + 256;
  auto product = [](const AllextTc* t) {
    tci_tc::Product p{};
    if (!t) return p;
    p.np = (int)t->np;
    p.m = (int)t->m;
    p.tiles = (int)((t->np + tci_tc::BM - 1) / tci_tc::BM);
    p.Y = t->y;
    p.ldy = t->np;
    return p;
  };
  const tci_tc::Product p0 = product(a), p1 = product(b);
  const int64_t ub = std::max(padded_rows(a->m), b ? padded_rows(b->m) : 0) / tci_tc::BN;
  const int ks = ksplit(a, b);
  if (ks > 1) {  // the two splits accumulate into zeroed outputs
    cudaError_t e = cudaMemsetAsync(a->y, 0, sizeof(double) * (size_t)(a->m * a->np), st);
    if (e == cudaSuccess && b) e = cudaMemsetAsync(b->y, 0, sizeof(double) * (size_t)(b->m * b->np), st);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((p0.tiles + p1.tiles) * ks), (unsigned)ub);
  const AllextTc* c = b ? b : a;  // maps of the second product (unused when there is none)
  tci_tc::allext_tf32x3_kernel<<<grid, tci_tc::NTHREADS, smem, st>>>(
      a->wmap, a->uhi, a->ulo, c->wmap, c->uhi, c->ulo, p0, p1, a->status, (int)(a->kblock / tci_tc::BK), ks);
  return cudaGetLastError();
}

}  // namespace tci_tc_host
