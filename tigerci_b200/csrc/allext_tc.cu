// Mixed-precision all-external product on the 5th-generation tensor cores.
//
//   Y[j][r] = sum_k W[r][k] U[j][k]      (W symmetric np x np, U: m CI blocks)
//
// W (the packed all-external operator W+ or W-, see plan.cpp) is stored in HBM
// as FP32 tiles of 128 rows x 32 k, each a contiguous 16 KB block already in
// the 128-byte swizzle layout and ordered panel-major then k, so that a CTA's
// range of k-steps is one sequential stream of HBM, fetched by plain bulk
// copies and requested into L2 a few tiles ahead.  It is read once per sigma
// build.  Each
// W tile is split into TF32 hi/lo parts by converter warps that read it from
// shared memory a row per thread and store both parts into tensor memory,
// where the MMA takes its A operand: shared memory then carries W once (TMA
// write, converter read) instead of once per MMA, which is what bounded the
// shared-memory form at small N.  U arrives pre-split and is the B operand in
// shared memory, its high rows directly followed by its low rows.  Per 8-wide
// k slice two kind::tf32 MMAs (W_hi x [U_hi; U_lo] with N = 2 bn, then W_lo x
// U_hi with N = bn into the first bn columns) form the three 3xTF32 products:
// small MMAs cost nearly a fixed time each, so two instructions instead of
// three is what counts.  They accumulate FP32 in TMEM; every KBLOCK elements of k the partial sums are read back with
// tcgen05.ld and added into FP64 accumulators held in registers (promotion
// keeps the FP32 accumulation error at the block length).  The product is HBM
// bound: W is read exactly once.
//
// Work split (persistent, stream-K): one launch covers both operators (W+
// with the singlet blocks, W- with the triplet blocks).  Their k-steps form
// one linear sequence (operator, CI-block group, 128-row panel, k); each CTA
// (one per SM) takes an equal contiguous range of it, so the pipeline runs
// without refills from panel to panel and every SM streams the same number of
// W bytes.  A range is at least one panel long, so a panel is shared by at
// most two CTAs: both add their FP64 partial sums into the zeroed output, and
// a + b rounds the same in either order, so the result does not depend on
// which CTA finishes first.  The MMA's N is the operator's own CI-block count
// rounded up to 16 (at most 64), not a fixed 64.
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
#include "tc_common.cuh"

namespace tci_tc {

using namespace tci_tcx;

constexpr int BM = 128;      // W rows per panel (MMA M)
constexpr int BN = 64;       // largest CI-block group (MMA N)
constexpr int BK = 32;       // fp32 k elements per stage (one 128-byte swizzle row)
constexpr int STAGES = 4;
constexpr int PREFETCH = 8;  // W tiles requested into L2 ahead of the ring
constexpr int TILE_FLOATS = BM * BK;  // one W tile
// The FP64 promotion block (k elements summed in TMEM before the FP64 add) is
// a launch parameter: the tensor core's FP32 accumulation error grows with it.
constexpr int W_BYTES = BM * BK * 4;   // 16 KB
constexpr int U_BYTES = 2 * BN * BK * 4;   // 16 KB: U hi rows then U lo rows (room for the largest group)
constexpr int STAGE_BYTES = W_BYTES + U_BYTES;
// TMEM columns: two accumulator buffers of 2 BN (hi x [hi; lo] + lo x hi), then per stage the A
// operand's hi (BK columns) and lo (BK columns)
constexpr int ACC_COLS = 2 * BN;
constexpr int A_COL0 = 2 * ACC_COLS;
constexpr int TMEM_COLS = 512;
static_assert(A_COL0 + STAGES * 2 * BK <= TMEM_COLS, "TMEM columns");
constexpr int NTHREADS = 320;
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
      : "memory");
}
// D (tmem) += A (tmem: lane = row, one column per k) * B (shared memory descriptor)
__device__ __forceinline__ void mma_tf32_ta(uint32_t d_tmem, uint32_t a_tmem, uint64_t b, uint32_t idesc,
                                            uint32_t accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d_tmem),
      "r"(a_tmem), "l"(b), "r"(idesc), "r"(accumulate));
}
// 32 consecutive 32-bit TMEM columns of this warp's 32 lanes
__device__ __forceinline__ void tmem_st32(uint32_t taddr, const uint32_t (&v)[32]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x32.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16,"
      "%17,%18,%19,%20,%21,%22,%23,%24,%25,%26,%27,%28,%29,%30,%31,%32};" ::"r"(taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15]), "r"(v[16]), "r"(v[17]), "r"(v[18]),
      "r"(v[19]), "r"(v[20]), "r"(v[21]), "r"(v[22]), "r"(v[23]), "r"(v[24]), "r"(v[25]), "r"(v[26]), "r"(v[27]),
      "r"(v[28]), "r"(v[29]), "r"(v[30]), "r"(v[31])
      : "memory");
}

// Contiguous global -> shared copy completing on an mbarrier (addresses 16-byte aligned, size a multiple of 16).
__device__ __forceinline__ void bulk_load(void* dst, const void* src, uint32_t bytes, uint64_t* bar) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(reinterpret_cast<uint64_t>(src)), "r"(bytes), "r"(smem_u32(bar))
               : "memory");
}
// Hint: bring a contiguous range into L2 (no shared memory, no completion to wait for).
__device__ __forceinline__ void bulk_prefetch_l2(const void* src, uint32_t bytes) {
  asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(reinterpret_cast<uint64_t>(src)), "r"(bytes)
               : "memory");
}

// Error codes written to the kernel's status word.
enum : int { ST_OK = 0, ST_TIMEOUT_FULL = 1, ST_TIMEOUT_CONV = 2, ST_TIMEOUT_EMPTY = 3, ST_TIMEOUT_D = 4, ST_TIMEOUT_DE = 5 };

// One operator of the launch: Y (m x np, row pitch ldy) = U W, as groups of
// bn CI blocks x panels of BM W rows x nk k-steps.
struct Product {
  const float* W;   // tiles of TILE_FLOATS: tile (panel, k) at (panel nk + k) TILE_FLOATS
  int np, m, bn, groups, panels, nk;
  long long units;  // groups * panels * nk
  double* Y;
  long long ldy;
};

// A run of consecutive k-steps of one (operator, group, panel) inside a CTA's range.
struct Segment {
  int prod, group, panel, k0, k1;
};

// The segment starting at linear k-step position pos (pos < end).
__device__ __forceinline__ Segment segment_at(const Product& p0, const Product& p1, long long pos, long long end) {
  Segment g;
  g.prod = pos >= p0.units ? 1 : 0;
  const Product& P = g.prod ? p1 : p0;
  const long long u = g.prod ? pos - p0.units : pos;
  const long long per_group = (long long)P.panels * P.nk;
  g.group = (int)(u / per_group);
  const long long v = u - (long long)g.group * per_group;
  g.panel = (int)(v / P.nk);
  g.k0 = (int)(v - (long long)g.panel * P.nk);
  const long long left = end - pos;
  g.k1 = (long long)(P.nk - g.k0) < left ? P.nk : (int)(g.k0 + left);
  return g;
}

__global__ void __launch_bounds__(NTHREADS, 1)
    allext_tf32x3_kernel(const __grid_constant__ CUtensorMap uhi_map0, const __grid_constant__ CUtensorMap ulo_map0,
                         const __grid_constant__ CUtensorMap uhi_map1, const __grid_constant__ CUtensorMap ulo_map1,
                         Product p0, Product p1, int* __restrict__ status, int kb_per_block) {
  const int KB_PER_BLOCK = kb_per_block;
  const long long total = p0.units + p1.units;
  const long long begin = total * (long long)blockIdx.x / gridDim.x;
  const long long end = total * (long long)(blockIdx.x + 1) / gridDim.x;
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
  if (warp == 9) {  // TMEM: 2 accumulator buffers of BN fp32 columns + the A operand of every stage
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(tmem_slot)),
                 "r"(TMEM_COLS));
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
      int step = 0, last = -1;  // k-steps issued so far in this CTA; the last one
      for (long long pos = begin; pos < end && !aborted();) {
        const Segment g = segment_at(p0, p1, pos, end);
        const float* wt = (g.prod ? p1.W : p0.W) + (long long)g.panel * (g.prod ? p1.nk : p0.nk) * TILE_FLOATS;
        const CUtensorMap* uhi_map = g.prod ? &uhi_map1 : &uhi_map0;
        const CUtensorMap* ulo_map = g.prod ? &ulo_map1 : &ulo_map0;
        const int bn = g.prod ? p1.bn : p0.bn;
        const uint32_t bytes = (uint32_t)(W_BYTES + 2 * bn * BK * 4);
        for (int k = g.k0; k < g.k0 + PREFETCH && k < g.k1; ++k) bulk_prefetch_l2(wt + (long long)k * TILE_FLOATS, W_BYTES);
        for (int k = g.k0; k < g.k1 && !aborted(); ++k, ++step) {
          const int s = step % STAGES;
          if (step >= STAGES && !mbar_wait(&empty[s], ((step / STAGES) - 1) & 1)) {
            fail(ST_TIMEOUT_EMPTY);
            break;
          }
          if (k + PREFETCH < g.k1) bulk_prefetch_l2(wt + (long long)(k + PREFETCH) * TILE_FLOATS, W_BYTES);
          uint8_t* st = base + s * STAGE_BYTES;
          mbar_expect_tx(&full[s], bytes);
          bulk_load(st, wt + (long long)k * TILE_FLOATS, W_BYTES, &full[s]);
          tma_load_2d(st + W_BYTES, uhi_map, &full[s], k * BK, g.group * bn);
          tma_load_2d(st + W_BYTES + bn * BK * 4, ulo_map, &full[s], k * BK, g.group * bn);
          last = step;
        }
        pos += g.k1 - g.k0;
      }
      if (aborted()) {
        // the copies of the last STAGES issued k-steps may still be landing: wait (bounded) for them
        // before the shared memory is released
        for (int st = (last - STAGES + 1 > 0 ? last - STAGES + 1 : 0); st <= last; ++st)
          mbar_wait(&full[st % STAGES], (st / STAGES) & 1);
      }
    }
  } else if (warp >= 4 && warp < 8) {
    // ---------------- TF32 hi/lo split of the W tile into TMEM (A operand) ----------------
    // thread = W row 32 cw + lane = TMEM lane; the 128-byte swizzle puts the 16-byte chunks of
    // eight consecutive rows on distinct banks, so the row-per-thread reads are conflict free
    const int cw = warp - 4, row = cw * 32 + lane;
    const long long nsteps = end - begin;
    for (long long step = 0; step < nsteps && !aborted(); ++step) {
      const int s = (int)(step % STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((step / STAGES) & 1))) {
        fail(ST_TIMEOUT_FULL);
        break;
      }
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint8_t* w = base + s * STAGE_BYTES + row * 128;
      uint32_t hi[BK], lo[BK];
#pragma unroll
      for (int j = 0; j < BK / 4; ++j) {
        const uint4 q = *reinterpret_cast<const uint4*>(w + ((j ^ (row & 7)) << 4));
        hi[4 * j] = q.x;
        hi[4 * j + 1] = q.y;
        hi[4 * j + 2] = q.z;
        hi[4 * j + 3] = q.w;
      }
#pragma unroll
      for (int k = 0; k < BK; ++k) {
        const uint32_t h = hi[k] & 0xFFFFE000u;
        lo[k] = __float_as_uint(__uint_as_float(hi[k]) - __uint_as_float(h));
        hi[k] = h;
      }
      const uint32_t acol = tmem + ((uint32_t)(cw * 32) << 16) + (uint32_t)(A_COL0 + s * 2 * BK);
      tmem_st32(acol, hi);
      tmem_st32(acol + BK, lo);
      asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory");
      asm volatile("tcgen05.fence::before_thread_sync;");
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer: promotion blocks of KB_PER_BLOCK steps, never across segments ----------------
    if (lane == 0) {
      int step = 0, blk = 0;
      for (long long pos = begin; pos < end && !aborted();) {
        const Segment g = segment_at(p0, p1, pos, end);
        const int bn = g.prod ? p1.bn : p0.bn;
        const uint32_t idesc_both = idesc_tf32(BM, 2 * bn), idesc_hi = idesc_tf32(BM, bn);
        for (int k = g.k0; k < g.k1 && !aborted(); ++k, ++step) {
          const int kin = k - g.k0;
          const bool first = (kin % KB_PER_BLOCK) == 0;
          const int buf = blk & 1;
          if (first && blk >= 2 && !mbar_wait(&dempty[buf], ((blk / 2) - 1) & 1)) {
            fail(ST_TIMEOUT_DE);
            break;
          }
          const int s = step % STAGES;
          if (!mbar_wait(&conv[s], (step / STAGES) & 1)) {
            fail(ST_TIMEOUT_CONV);
            break;
          }
          asm volatile("tcgen05.fence::after_thread_sync;");
          uint8_t* st = base + s * STAGE_BYTES;
          const uint32_t d = tmem + (uint32_t)(buf * ACC_COLS);
          const uint32_t ahi = tmem + (uint32_t)(A_COL0 + s * 2 * BK), alo = ahi + BK;
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk) {  // 8 tf32 = 8 TMEM columns / 32 bytes of a B row per MMA step
            const uint64_t b = smem_desc_sw128(st + W_BYTES + kk * 32);  // U hi rows, then U lo rows
            mma_tf32_ta(d, ahi + kk * 8, b, idesc_both, (first && kk == 0) ? 0u : 1u);
            mma_tf32_ta(d, alo + kk * 8, b, idesc_hi, 1u);
          }
          mma_commit(&empty[s]);
          if ((kin % KB_PER_BLOCK) == KB_PER_BLOCK - 1 || k == g.k1 - 1) {
            mma_commit(&dfull[buf]);
            ++blk;
          }
        }
        pos += g.k1 - g.k0;
      }
      if (aborted()) {
        // MMAs issued before the abort may still be writing TMEM: wait (bounded) for all of them
        mma_commit(mma_done);
        mbar_wait(mma_done, 0);
      }
    }
  } else {
    // ---------------- epilogue: FP32 block sums -> FP64 register accumulators -> Y ----------------
    int blk = 0;
    for (long long pos = begin; pos < end && !aborted();) {
      const Segment g = segment_at(p0, p1, pos, end);
      const Product& P = g.prod ? p1 : p0;
      const int nblocks = (g.k1 - g.k0 + KB_PER_BLOCK - 1) / KB_PER_BLOCK;
      double acc[BN];
#pragma unroll
      for (int t = 0; t < BN; ++t) acc[t] = 0.0;
      for (int b = 0; b < nblocks && !aborted(); ++b, ++blk) {
        const int buf = blk & 1;
        if (!mbar_wait(&dfull[buf], (blk / 2) & 1)) {
          fail(ST_TIMEOUT_D);
          break;
        }
        asm volatile("tcgen05.fence::after_thread_sync;");
        const uint32_t dq = tmem + ((uint32_t)(warp * 32) << 16) + (uint32_t)(buf * ACC_COLS);
#pragma unroll
        for (int c = 0; c < BN / 16; ++c) {
          if (c * 16 < P.bn) {
            uint32_t v[16];
            tmem_ld16(dq + (uint32_t)(c * 16), v);  // hi x hi + lo x hi
#pragma unroll
            for (int t = 0; t < 16; ++t) acc[c * 16 + t] += (double)__uint_as_float(v[t]);
            tmem_ld16(dq + (uint32_t)(P.bn + c * 16), v);  // hi x lo
#pragma unroll
            for (int t = 0; t < 16; ++t) acc[c * 16 + t] += (double)__uint_as_float(v[t]);
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) mbar_arrive(&dempty[buf]);
      }
      const int r = g.panel * BM + warp * 32 + lane;  // W row owned by this thread
      if (!aborted() && r < P.np) {
#pragma unroll
        for (int t = 0; t < BN; ++t) {
          const int j = g.group * P.bn + t;
          // one or two CTAs add into the zeroed output (see the header)
          if (t < P.bn && j < P.m) atomicAdd(&P.Y[(long long)j * P.ldy + r], acc[t]);
        }
      }
      pos += g.k1 - g.k0;
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (warp == 9) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TMEM_COLS));
}

// FP64 W (np x np) -> FP32 tiles (W at init): tile (panel, k) holds rows panel BM .. +BM-1, columns
// k BK .. +BK-1 in the 128-byte swizzle layout (16-byte chunks of row r permuted by r mod 8), zero past np.
__global__ void to_f32_tiles(const double* __restrict__ src, long long np, int nk, float* __restrict__ dst,
                             long long total) {
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / TILE_FLOATS;
    const int i = (int)(e % TILE_FLOATS);  // element index within the tile: row i / BK, column i % BK
    const int r = i / BK, c = i % BK;
    const long long panel = t / nk, k = t % nk;
    const long long gr = panel * BM + r, gc = k * BK + c;
    const float v = (gr < np && gc < np) ? (float)src[gr * np + gc] : 0.0f;
    dst[t * TILE_FLOATS + (sw128_offset(r, c) >> 2)] = v;
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

int64_t w32_floats(int64_t np) {
  return (np + tci_tc::BM - 1) / tci_tc::BM * tci_tc::BM * ((np + tci_tc::BK - 1) / tci_tc::BK * tci_tc::BK);
}

cudaError_t convert_w(const double* w64, int64_t np, float* w32, cudaStream_t st) {
  tci_tc::to_f32_tiles<<<148 * 16, 256, 0, st>>>(w64, np, (int)((np + tci_tc::BK - 1) / tci_tc::BK), w32,
                                                  (long long)w32_floats(np));
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
  if (m <= 0 || np <= 0) {
    err = "empty all-external product";
    return false;
  }
  t.kblock = kblock;
  t.np = np;
  t.m = m;
  // MMA N: the CI blocks of one group, rounded up to 16 (groups of BN when there are more)
  t.bn = m >= tci_tc::BN ? tci_tc::BN : (m + 15) / 16 * 16;
  t.y = y;
  t.status = status;
  if (reinterpret_cast<uintptr_t>(w32) & 15) {
    err = "W tiles not 16-byte aligned";
    return false;
  }
  t.w = w32;
  const uint64_t ld = (uint64_t)padded_ld(np);
  if (!make_map(&t.uhi, uhi, padded_rows(m), np, ld, (uint32_t)t.bn, err)) return false;
  if (!make_map(&t.ulo, ulo, padded_rows(m), np, ld, (uint32_t)t.bn, err)) return false;
  static bool attr = false;
  if (!attr) {
    if (cudaFuncSetAttribute(tci_tc::allext_tf32x3_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             tci_tc::SMEM_BYTES) != cudaSuccess) {
      err = "cannot raise the dynamic shared memory limit";
      return false;
    }
    attr = true;
  }
  return true;
}

cudaError_t launch(const AllextTc* a, const AllextTc* b, cudaStream_t st) {
  if (!a && !b) return cudaSuccess;
  if (!a) std::swap(a, b);
  auto product = [](const AllextTc* t) {
    tci_tc::Product p{};
    if (!t) return p;
    p.W = t->w;
    p.np = (int)t->np;
    p.m = (int)t->m;
    p.bn = (int)t->bn;
    p.groups = (int)((t->m + t->bn - 1) / t->bn);
    p.panels = (int)((t->np + tci_tc::BM - 1) / tci_tc::BM);
    p.nk = (int)((t->np + tci_tc::BK - 1) / tci_tc::BK);
    p.units = (long long)p.groups * p.panels * p.nk;
    p.Y = t->y;
    p.ldy = t->np;
    return p;
  };
  const tci_tc::Product p0 = product(a), p1 = product(b);
  // one CTA per SM, each range at least one panel long (a panel then spans at most two ranges)
  int dev = 0, sms = 148;
  if (cudaGetDevice(&dev) == cudaSuccess) cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long total = p0.units + p1.units, nk_max = std::max(p0.nk, p1.nk);
  const long long grid = std::max<long long>(1, std::min<long long>(sms, total / nk_max));
  // the CTAs add into zeroed outputs
  cudaError_t e = cudaMemsetAsync(a->y, 0, sizeof(double) * (size_t)(a->m * a->np), st);
  if (e == cudaSuccess && b) e = cudaMemsetAsync(b->y, 0, sizeof(double) * (size_t)(b->m * b->np), st);
  if (e != cudaSuccess) return e;
  const AllextTc* c = b ? b : a;  // maps of the second product (unused when there is none)
  tci_tc::allext_tf32x3_kernel<<<(unsigned)grid, tci_tc::NTHREADS, tci_tc::SMEM_BYTES, st>>>(
      a->uhi, a->ulo, c->uhi, c->ulo, p0, p1, a->status, (int)(a->kblock / tci_tc::BK));
  return cudaGetLastError();
}

}  // namespace tci_tc_host
