// Mixed-precision all-external product on the 5th-generation tensor cores.
//
//   Y[j][r] = sum_k W[r][k] U[j][k]      (W symmetric np x np, U: m CI blocks)
//
// W (the packed all-external operator W+ or W-, see plan.cpp) is stored in HBM
// as FP32 tiles of 128 rows x 32 k, each a contiguous 16 KB block already in
// the 128-byte swizzle layout and ordered panel-major then k, so that a CTA's
// range of k-steps is one sequential stream of HBM, fetched by plain bulk
// copies and requested into L2 a few tiles ahead.  It is read once per sigma
// build.  U arrives split into TF32 high and FP32 low rows, interleaved
// (row 2j = hi U[j], row 2j+1 = lo U[j]).
//
// The 3xTF32 products hi*hi + hi*lo + lo*hi come from ONE kind::tf32 MMA per
// 8-wide k slice: A = the interleaved U rows of a group of bn <= 64 CI blocks
// (M = 128 TMEM lanes, 2 bn of them used), B = the W panel's 128 rows followed
// by their low parts (N = 256).  Lane 2j then holds U_hi[j] W_hi + U_hi[j] W_lo
// in its two column halves and lane 2j+1 holds U_lo[j] W_hi (its second half,
// lo x lo, is not used); the epilogue joins the lane pair with a shuffle.  On
// B200 an MMA into one accumulator costs about the same time whatever its M
// (64, 128) and N (64..256) (measured by mma_rate_selftest below: 188 cycles
// per kind::tf32 instruction; 150 on two alternating accumulators), so the
// instruction count is what bounds this product, and this arrangement needs a
// quarter of the MMAs of W-in-M with three products.  The tensor core reads a
// kind::tf32 operand's top 19 bits only (raw FP32 and masked operands gave
// bit-identical results on B200), so the W tile serves as its own high part as
// it lands; the converter warps write only the low parts.  The MMAs
// accumulate FP32 in TMEM; every KBLOCK elements of k the partial sums are
// read back with tcgen05.ld and added into FP64 accumulators held in registers
// (promotion keeps the FP32 accumulation error at the block length).
//
// Work split (persistent, stream-K): one launch covers both operators (W+
// with the singlet blocks, W- with the triplet blocks).  Their k-steps form
// one linear sequence (operator, CI-block group, 128-row panel, k); each CTA
// (one per SM) takes a contiguous range of it, so the pipeline runs without
// refills from panel to panel.  The CTAs are shared between the operators in
// proportion to their k-steps; with several CI-block groups the CTAs of an
// operator are dealt round the groups and the t-th CTA of every group takes
// the same share of its group's (panel, k) sequence, so the groups stream
// the same W tiles side by side and a tile leaves HBM once (cta_range).  A
// range is at least one panel long, so a panel is shared by at most two
// CTAs: both add their FP64 partial sums into the zeroed output, and a + b
// rounds the same in either order, so the result does not depend on which
// CTA finishes first.
//
// Warp roles (448 threads): warps 0-3 and 10-13 epilogue (two per TMEM lane
// quadrant), warps 4-7 low parts of the W tile, warp 8 producer (bulk copy +
// TMA), warp 9 TMEM allocator + MMA issuer.  Every mbarrier wait is bounded; on timeout
// the kernel records an error code, drains and returns (no trap).
#include <cuda.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdint>
#include <cstdio>
#include <string>

#include "allext_tc.h"
#include "device_info.h"
#include "tc_common.cuh"

namespace tci_tc {

using namespace tci_tcx;

constexpr int BM = 128;      // W rows per panel
constexpr int BN = 64;       // largest CI-block group (2 BN interleaved U rows = the MMA's M)
constexpr int BK = 32;       // fp32 k elements per stage (one 128-byte swizzle row)
constexpr int STAGES = 4;
constexpr int PREFETCH = 8;  // W tiles requested into L2 ahead of the ring
constexpr int TILE_FLOATS = BM * BK;  // one W tile
constexpr int MMA_N = 2 * BM;         // W rows, then their low parts
// The FP64 promotion block (k elements summed in TMEM before the FP64 add) is
// a launch parameter: the tensor core's FP32 accumulation error grows with it.
constexpr int W_BYTES = BM * BK * 4;        // 16 KB
constexpr int B_BYTES = 2 * W_BYTES;        // W tile (its own high part) + low parts
constexpr int A_BYTES = 2 * BN * BK * 4;    // 16 KB: interleaved U rows (room for the largest group)
constexpr int STAGE_BYTES = B_BYTES + A_BYTES;
constexpr int TMEM_COLS = 2 * MMA_N;        // two accumulator buffers
constexpr int NTHREADS = 448;
constexpr int EPI_WARPS = 8;  // warps 0-3 and 10-13: two per TMEM lane quadrant, each half of the panel
constexpr int SMEM_BYTES = STAGES * STAGE_BYTES + 1024 + 256;

__device__ __forceinline__ void tma_load_2d(void* dst, const CUtensorMap* map, uint64_t* bar, int x, int y) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4}], [%2];" ::"r"(
          smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(smem_u32(bar)), "r"(x), "r"(y)
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

// 8 consecutive 32-bit TMEM columns of this warp's 32 lanes (complete after tmem_wait_ld).
__device__ __forceinline__ void tmem_ld8(uint32_t taddr, uint32_t (&v)[8]) {
  asm volatile("tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0,%1,%2,%3,%4,%5,%6,%7}, [%8];"
               : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
               : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

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

// The CTA's range of the linear k-step sequence.  The CTAs are shared between the two operators in
// proportion to their k-steps; within an operator CTA i works on CI-block group i mod G (G groups), and the
// n_g CTAs of group g split that group's (panel, k) sequence into n_g equal shares, the t-th CTA of every
// group taking the t-th share.  CTAs with the same t stream the same W tiles at about the same time, so a
// tile comes from HBM once and from L2 for the other groups.  A share is at least one panel long (n_g is
// capped at the panel count; CTAs past it stay idle), so a panel is still shared by at most two CTAs.  With
// fewer CTAs than groups the operator's sequence is split into equal contiguous ranges.
__device__ __forceinline__ void cta_range(const Product& p0, const Product& p1, long long& begin, long long& end) {
  const int C = (int)gridDim.x, b = (int)blockIdx.x;
  const long long total = p0.units + p1.units;
  if (C == 1) {
    begin = 0;
    end = total;
    return;
  }
  int c0 = C;  // CTAs of operator 0
  if (p0.units == 0) {
    c0 = 0;
  } else if (p1.units > 0) {
    c0 = (int)llround((double)C * (double)p0.units / (double)total);
    c0 = c0 < 1 ? 1 : (c0 > C - 1 ? C - 1 : c0);
  }
  const bool second = b >= c0;
  const Product& P = second ? p1 : p0;
  const long long base = second ? p0.units : 0;
  const int i = second ? b - c0 : b, nc = second ? C - c0 : c0;
  if (nc < P.groups) {
    begin = base + P.units * i / nc;
    end = base + P.units * (i + 1) / nc;
    return;
  }
  const int g = i % P.groups, t = i / P.groups;
  int ng = nc / P.groups + (g < nc % P.groups ? 1 : 0);
  if (ng > P.panels) ng = P.panels;
  const long long per = (long long)P.panels * P.nk, gb = base + (long long)g * per;
  if (t >= ng) {
    begin = end = gb;
    return;
  }
  begin = gb + per * t / ng;
  end = gb + per * (t + 1) / ng;
}

__global__ void __launch_bounds__(NTHREADS, 1)
    allext_tf32x3_kernel(const __grid_constant__ CUtensorMap u_map0, const __grid_constant__ CUtensorMap u_map1,
                         Product p0, Product p1, int* __restrict__ status, int kb_per_block) {
  const int KB_PER_BLOCK = kb_per_block;
  long long begin, end;
  cta_range(p0, p1, begin, end);
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
      mbar_init(&dempty[b], EPI_WARPS);
    }
    mbar_init(mma_done, 1);
    *abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (warp == 9) {  // TMEM: 2 accumulator buffers of MMA_N fp32 columns
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
    // ---------------- producer: W tile by bulk copy (L2 lead), U rows by TMA ----------------
    if (lane == 0) {
      int step = 0, last = -1;  // k-steps issued so far in this CTA; the last one
      for (long long pos = begin; pos < end && !aborted();) {
        const Segment g = segment_at(p0, p1, pos, end);
        const float* wt = (g.prod ? p1.W : p0.W) + (long long)g.panel * (g.prod ? p1.nk : p0.nk) * TILE_FLOATS;
        const CUtensorMap* u_map = g.prod ? &u_map1 : &u_map0;
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
          tma_load_2d(st + B_BYTES, u_map, &full[s], k * BK, g.group * 2 * bn);
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
    // ---------------- low parts of the W tile: rows BM.. of the B operand ----------------
    const int cw = warp - 4;
    const long long nsteps = end - begin;
    for (long long step = 0; step < nsteps && !aborted(); ++step) {
      const int s = (int)(step % STAGES);
      if (!mbar_wait(&full[s], (uint32_t)((step / STAGES) & 1))) {
        fail(ST_TIMEOUT_FULL);
        break;
      }
      const uint32_t* w = reinterpret_cast<const uint32_t*>(base + s * STAGE_BYTES);
      float* wlo = reinterpret_cast<float*>(base + s * STAGE_BYTES + W_BYTES);
      // a warp per 128-byte row, lane l holds element l (conflict free); row r + BM has the same
      // swizzle permutation as row r, so the low part keeps the tile's layout.  Eight rows per
      // batch: their loads are issued before any store.
#pragma unroll
      for (int r0 = cw; r0 < BM; r0 += 4 * 8) {
        uint32_t x[8];
#pragma unroll
        for (int i = 0; i < 8; ++i) x[i] = w[(r0 + 4 * i) * BK + lane];
#pragma unroll
        for (int i = 0; i < 8; ++i)
          wlo[(r0 + 4 * i) * BK + lane] = __uint_as_float(x[i]) - __uint_as_float(x[i] & 0xFFFFE000u);
      }
      asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
      __syncwarp();
      if (lane == 0) mbar_arrive(&conv[s]);
    }
  } else if (warp == 9) {
    // ---------------- MMA issuer: promotion blocks of KB_PER_BLOCK steps, never across segments ----------------
    if (lane == 0) {
      const uint32_t idesc = idesc_tf32(2 * BN, MMA_N);
      int step = 0, blk = 0;
      for (long long pos = begin; pos < end && !aborted();) {
        const Segment g = segment_at(p0, p1, pos, end);
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
          const uint32_t d = tmem + (uint32_t)(buf * MMA_N);
#pragma unroll
          for (int kk = 0; kk < BK / 8; ++kk)  // 8 tf32 = 32 bytes of every row per MMA
            mma_tf32(d, smem_desc_sw128(st + B_BYTES + kk * 32), smem_desc_sw128(st + kk * 32), idesc,
                     (first && kk == 0) ? 0u : 1u);
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
  } else if (warp < 4 || warp >= 10) {
    // ---------------- epilogue: lane pairs joined, FP32 block sums -> FP64 registers -> Y ----------------
    // TMEM lane quadrant q = warp mod 4: lane l is U row 32 q + l = CI block 16 q + l / 2, high (even)
    // or low (odd) part; warps 0-3 take panel columns 0-63, warps 10-13 columns 64-127.  Per 8-column
    // chunk the even lane keeps columns 0-3 and the odd lane 4-7 after the pair exchange.
    const int q = warp & 3, half = warp >= 10 ? 1 : 0;
    const int odd = lane & 1;
    const int jl = 16 * q + (lane >> 1);  // CI block within the group
    constexpr int COLS = BM / 2;          // panel columns per warp
    int blk = 0;
    for (long long pos = begin; pos < end && !aborted();) {
      const Segment g = segment_at(p0, p1, pos, end);
      const Product& P = g.prod ? p1 : p0;
      const bool active = 32 * q < 2 * P.bn;  // warp-uniform: the quadrant holds used U rows
      const int nblocks = (g.k1 - g.k0 + KB_PER_BLOCK - 1) / KB_PER_BLOCK;
      double acc[COLS / 2];
#pragma unroll
      for (int t = 0; t < COLS / 2; ++t) acc[t] = 0.0;
      for (int b = 0; b < nblocks && !aborted(); ++b, ++blk) {
        const int buf = blk & 1;
        if (!mbar_wait(&dfull[buf], (blk / 2) & 1)) {
          fail(ST_TIMEOUT_D);
          break;
        }
        if (active) {
          asm volatile("tcgen05.fence::after_thread_sync;");
          const uint32_t dq = tmem + ((uint32_t)(q * 32) << 16) + (uint32_t)(buf * MMA_N + half * COLS);
#pragma unroll
          for (int c0 = 0; c0 < COLS / 8; c0 += 2) {  // two 8-column chunks per wait
            uint32_t vh[2][8], vl[2][8];
#pragma unroll
            for (int i = 0; i < 2; ++i) {
              tmem_ld8(dq + (uint32_t)((c0 + i) * 8), vh[i]);       // x W_hi
              tmem_ld8(dq + (uint32_t)(BM + (c0 + i) * 8), vl[i]);  // x W_lo
            }
            tmem_wait_ld();
#pragma unroll
            for (int i = 0; i < 2; ++i)
#pragma unroll
              for (int t = 0; t < 4; ++t) {
                // even lane: U_hi (W_hi + W_lo); odd lane: U_lo W_hi (both FP32 block sums)
                const float s0 = __uint_as_float(vh[i][t]) + (odd ? 0.0f : __uint_as_float(vl[i][t]));
                const float s1 = __uint_as_float(vh[i][4 + t]) + (odd ? 0.0f : __uint_as_float(vl[i][4 + t]));
                const float recv = __shfl_xor_sync(0xffffffffu, odd ? s0 : s1, 1);
                acc[(c0 + i) * 4 + t] += (double)((odd ? s1 : s0) + recv);
              }
          }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncwarp();
        if (lane == 0) mbar_arrive(&dempty[buf]);
      }
      const int j = g.group * P.bn + jl;
      if (!aborted() && active && jl < P.bn && j < P.m) {
#pragma unroll
        for (int c = 0; c < COLS / 8; ++c)
#pragma unroll
          for (int t = 0; t < 4; ++t) {
            const int r = g.panel * BM + half * COLS + c * 8 + (odd ? 4 : 0) + t;
            // one or two CTAs add into the zeroed output (see the header)
            if (r < P.np) atomicAdd(&P.Y[(long long)j * P.ldy + r], acc[c * 4 + t]);
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

// The same tiles built directly from the packed external (ab|cd) matrix X (npk x npk, npk = n(n+1)/2,
// row (ab) = a(a+1)/2 + b, a >= b) without an FP64 W: W+ (plus, np = n + n(n-1)/2 rows: the n pairs (aa),
// then (ac) a > c at n + a(a-1)/2 + c) or W- (nm = n(n-1)/2 rows (ac)), by the element formulas of the FP64
// build (sqrt2 on the (aa) rows / columns of W+; (ab|cd) +- (ad|cb) elsewhere).
__device__ __forceinline__ long long xpk(long long a, long long b) {
  return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a;
}
__device__ __forceinline__ void xunpair(long long x, long long& a, long long& b) {
  long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)x)) * 0.5);
  while (i * (i - 1) / 2 > x) --i;
  while ((i + 1) * i / 2 <= x) ++i;
  a = i;
  b = x - i * (i - 1) / 2;
}
__global__ void x_to_f32_tiles(const double* __restrict__ X, long long n, int plus, int nk, float* __restrict__ dst,
                               long long total) {
  const long long nab = n * (n - 1) / 2, np = plus ? n + nab : nab, npk = n * (n + 1) / 2;
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / TILE_FLOATS;
    const int i = (int)(e % TILE_FLOATS);
    const int r = i / BK, c = i % BK;
    const long long panel = t / nk, k = t % nk;
    const long long gr = panel * BM + r, gc = k * BK + c;
    float v = 0.0f;
    if (gr < np && gc < np) {
      long long a, cc, b, d;
      const bool rd = plus && gr < n, cd = plus && gc < n;
      if (rd) a = cc = gr;
      else xunpair(plus ? gr - n : gr, a, cc);
      if (cd) b = d = gc;
      else xunpair(plus ? gc - n : gc, b, d);
      double w;
      if (plus) {
        if (rd && cd) w = X[xpk(a, b) * npk + xpk(a, b)];
        else if (rd) w = 1.4142135623730951 * X[xpk(a, b) * npk + xpk(a, d)];
        else if (cd) w = 1.4142135623730951 * X[xpk(a, b) * npk + xpk(cc, b)];
        else w = X[xpk(a, b) * npk + xpk(cc, d)] + X[xpk(cc, b) * npk + xpk(a, d)];
      } else {
        w = X[xpk(a, b) * npk + xpk(cc, d)] - X[xpk(cc, b) * npk + xpk(a, d)];
      }
      v = (float)w;
    }
    dst[t * TILE_FLOATS + (sw128_offset(r, c) >> 2)] = v;
  }
}

// U (m x np, FP64) -> interleaved rows: 2j = TF32 high part of U[j] (masked), 2j+1 = FP32 low
// part; rows up to 2 mpad, zero past m and np.
__global__ void split_u(const double* __restrict__ U, int m, int np, long long ldu, float* __restrict__ u2,
                        int mpad, long long ldw) {
  const long long total = (long long)mpad * ldw;  // element pairs
  for (long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x; e < total; e += (long long)gridDim.x * blockDim.x) {
    const long long j = e / ldw, k = e % ldw;
    float h = 0.0f, l = 0.0f;
    if (j < m && k < np) {
      const double x = U[j * ldu + k];
      h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
      l = (float)(x - (double)h);
    }
    u2[(2 * j) * ldw + k] = h;
    u2[(2 * j + 1) * ldw + k] = l;
  }
}

// Self-test of the abort path: one CTA waits, with the kernels' own bounded wait, on an mbarrier that
// nothing arrives at, records the code the kernels record for a stalled operand (ST_TIMEOUT_FULL) and
// returns; the other warps wait for the abort flag as the kernels' consumers do.  polls: the wait's limit.
__global__ void bounded_wait_selftest(int* __restrict__ status, long long polls) {
  __shared__ uint64_t bar;
  __shared__ int abort_flag;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);
    abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    if (!mbar_wait(&bar, 0, polls)) {
      atomicCAS(status, 0, ST_TIMEOUT_FULL);
      *(volatile int*)&abort_flag = 1;
    }
  }
  __syncthreads();
}

// Self-test of the MMA instruction rate: one thread per CTA issues iters x nacc kind::tf32 MMAs (M = m, 64 or
// 128, N = n, K = 8, operands zero in shared memory) back to back into nacc independent TMEM accumulators of n
// columns, commits once and waits (bounded); cycles[cta] = clock64 span.  One CTA per SM (the shared memory
// request keeps a second one off the SM, so the 512-column TMEM allocation never waits on another CTA).
constexpr int RATE_SMEM = 120 * 1024;
__global__ void __launch_bounds__(128, 1) mma_rate_selftest(int m, int n, int nacc, int iters,
                                                           long long* __restrict__ cycles, int* __restrict__ status) {
  extern __shared__ uint8_t smem_raw[];
  uint8_t* base = reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
  uint8_t* A = base;          // 128 rows x 128 bytes
  uint8_t* B = base + 16384;  // 256 rows x 128 bytes
  uint64_t* bar = reinterpret_cast<uint64_t*>(base + 16384 + 32768);
  uint32_t* slot = reinterpret_cast<uint32_t*>(bar + 1);
  for (int i = threadIdx.x; i < (16384 + 32768) / 4; i += blockDim.x) reinterpret_cast<uint32_t*>(base)[i] = 0u;
  asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (threadIdx.x < 32) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(slot)), "r"(512));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = *slot;
  if (threadIdx.x == 0) {
    const uint64_t a = smem_desc_sw128(A), b = smem_desc_sw128(B);
    const uint32_t id = idesc_tf32(m, n);
    const long long t0 = clock64();
    for (int i = 0; i < iters; ++i)
      for (int q = 0; q < nacc; ++q) mma_tf32(tmem + (uint32_t)(q * n * (m == 64 ? 2 : 1)), a, b, id, i > 0 ? 1u : 0u);
    mma_commit(bar);
    bool ok = mbar_wait(bar, 0);
    if (!ok) ok = mbar_wait(bar, 0);
    cycles[blockIdx.x] = clock64() - t0;
    if (!ok) atomicCAS(status, 0, ST_TIMEOUT_D);
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (threadIdx.x < 32) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(512));
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
  tci_tc::to_f32_tiles<<<tci_dev::device_sms() * 16, 256, 0, st>>>(w64, np, (int)((np + tci_tc::BK - 1) / tci_tc::BK), w32,
                                                  (long long)w32_floats(np));
  return cudaGetLastError();
}

cudaError_t convert_w_from_x(const double* x, int64_t n, bool plus, float* w32, cudaStream_t st) {
  const int64_t np = plus ? n + n * (n - 1) / 2 : n * (n - 1) / 2;
  if (np <= 0) return cudaSuccess;
  tci_tc::x_to_f32_tiles<<<tci_dev::device_sms() * 16, 256, 0, st>>>(x, n, plus ? 1 : 0, (int)((np + tci_tc::BK - 1) / tci_tc::BK), w32,
                                                    (long long)w32_floats(np));
  return cudaGetLastError();
}

cudaError_t bounded_wait_selftest(int64_t polls, int* status, cudaStream_t st) {
  tci_tc::bounded_wait_selftest<<<1, 128, 0, st>>>(status, (long long)polls);
  return cudaGetLastError();
}
int64_t spin_limit() { return tci_tcx::SPIN_LIMIT; }

cudaError_t mma_rate_selftest(int64_t m, int64_t n, int64_t nacc, int64_t iters, int grid, long long* cycles,
                              int* status, cudaStream_t st) {
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(tci_tc::mma_rate_selftest, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         tci_tc::RATE_SMEM);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  tci_tc::mma_rate_selftest<<<grid, 128, tci_tc::RATE_SMEM, st>>>((int)m, (int)n, (int)nacc, (int)iters, cycles,
                                                                  status);
  return cudaGetLastError();
}

int64_t u2_floats(int64_t m, int64_t np) { return 2 * padded_rows(m) * padded_ld(np); }

cudaError_t split_u(const double* u, int64_t m, int64_t np, float* u2, cudaStream_t st) {
  tci_tc::split_u<<<tci_dev::device_sms() * 4, 256, 0, st>>>(u, (int)m, (int)np, np, u2, (int)padded_rows(m), padded_ld(np));
  return cudaGetLastError();
}

bool prepare(AllextTc& t, const float* w32, int64_t np, const float* u2, int64_t m, double* y, int* status,
             int64_t kblock, std::string& err) {
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
  // CI blocks per group (their 2 bn interleaved rows fill at most the MMA's 128 rows)
  t.bn = m >= tci_tc::BN ? tci_tc::BN : m;
  t.y = y;
  t.status = status;
  if (reinterpret_cast<uintptr_t>(w32) & 15) {
    err = "W tiles not 16-byte aligned";
    return false;
  }
  t.w = w32;
  const uint64_t ld = (uint64_t)padded_ld(np);
  if (!make_map(&t.u2, u2, 2 * padded_rows(m), np, ld, (uint32_t)(2 * t.bn), err)) return false;
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
  const long long sms = tci_dev::device_sms();
  const long long total = p0.units + p1.units, nk_max = std::max(p0.nk, p1.nk);
  const long long grid = std::max<long long>(1, std::min<long long>(sms, total / nk_max));
  // the CTAs add into zeroed outputs
  cudaError_t e = cudaMemsetAsync(a->y, 0, sizeof(double) * (size_t)(a->m * a->np), st);
  if (e == cudaSuccess && b) e = cudaMemsetAsync(b->y, 0, sizeof(double) * (size_t)(b->m * b->np), st);
  if (e != cudaSuccess) return e;
  const AllextTc* c = b ? b : a;  // map of the second product (unused when there is none)
  tci_tc::allext_tf32x3_kernel<<<(unsigned)grid, tci_tc::NTHREADS, tci_tc::SMEM_BYTES, st>>>(
      a->u2, c->u2, p0, p1, a->status, (int)(a->kblock / tci_tc::BK));
  return cudaGetLastError();
}

}  // namespace tci_tc_host
