// All-external term of a local MRSDCI space with pair domains, batched over
// heads of uneven size (tci_local_*).
//
// In TigerCI's local correlation treatment every N-2 head h (internal pair)
// keeps only the external orbitals of its own domain (virtual_truncation,
// tiger_fortran/locist_mod.f90:358-451), and the all-external loops
// (ext_3_4_seg_loops_vec_lmo_res_2, three_and_four_seg_mod_1.f90:3240-3518)
// run over those domains.  Here the term is applied in the Cholesky form
//
//   R_hk = 1/2 sum_J L^J_h D_hk L^J_h,   D_hk = SCEP matrix of the CI block
//   (h, spin function k), L^J_h = L^J restricted to domain(h) x domain(h),
//
// and sigma_hk += pack(R_hk), which equals the reference's integral form (the
// factor 1/2 compensates the two triangles of D).  The Cholesky vectors are
// processed in chunks of Jc: per chunk a gather kernel builds L^J_h for all
// heads (one launch), then two grouped GEMM launches cover every head and spin
// function at once, whatever their domain sizes:
//
//   T_hk (Jc n_h x n_h) = [L^J_h]_J (Jc n_h x n_h) D_hk
//   R_hk (n_h x n_h)   += 1/2 sum_J T_hkJ L^J_h       (Jc K-segments of n_h)
//
// on the FP64 SIMT kernel or, in the mixed form, on the TMA-fed tcgen05 3xTF32
// kernel: there L^J_h, D_hk and T_hk live as TF32-high / FP32-low rows (pitch a
// multiple of 32, zero past each domain), the first GEMM writes T_hk directly
// in that split form and the second accumulates R_hk in FP64.
// The chunk size and the FP64 tile shape of the second GEMM come from a small
// autotuner that times each candidate once at set-up.  One application
// (unpack, chunks, pack) is captured as one CUDA graph.
//
// In the mixed form a second, dense form competes with it: the packed
// integral form of the non-local all-external term (W+ over the pairs (aa)
// and (ac), W- over (ac), a > c, of ALL externals, as FP32 tiles built once
// from X = Lpk Lpk^T) applied to the local blocks placed at their pairs among
// all externals (zero elsewhere, rows of U+ for singlet-coupled and U- for
// triplet-coupled spin functions) on the tcgen05 all-external kernel
// (allext_tc.cu), the result read back at the domain's pairs.  Exact: the
// blocks are zero outside their domains, so (W U)_h restricted to domain(h)
// is the domain-restricted integral form.  It spends its flops on the zero
// columns of U (2 np^2 per block against 4 nchol n_h^3 in the Cholesky form)
// but runs them as one long stream of W tiles at the all-external kernel's
// rate, which beats the short uneven GEMMs of the Cholesky form when the
// domains are a sizeable part of the externals.  Both are timed at set-up
// (device memory permitting: X and the W tiles need 8 npv^2 + 4 np^2 + 4 nm^2
// bytes) and the faster one is kept.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/tigerci_sigma.h"
#include "allext_tc.h"
#include "device_info.h"
#include "gemm_tables.h"
#include "gemm_tma.h"
#include "host/capi_internal.h"

using namespace tci;
using tci_dev::DGemmProblem;
using tci_dev::DGemmSeg;
using tci_dev::HostGemm;

#define LCUDA(call)                                                                                      \
  do {                                                                                                   \
    cudaError_t _e = (call);                                                                             \
    if (_e != cudaSuccess)                                                                               \
      throw Error(TCI_ERR_CUDA, std::string(#call) + " (local_allext.cu:" + std::to_string(__LINE__) + \
                                    ") failed: " + cudaGetErrorString(_e));                              \
  } while (0)

namespace {

// one (head, spin function) block
struct DLocBlock {
  long long off_ab, off_aa;  // CI offsets of the head's ab / aa blocks (spin function 0)
  long long n, k;            // domain size, spin function
  long long ab, aa;          // spin function k has an ab block / an aa block
  double p;                  // +1 singlet-coupled, -1 triplet-coupled
  long long d_off;           // offset of D_hk / R_hk (n rows of pitch ld)
  long long head;            // index of the head
  long long t_off;           // offset of T_hk (jmax n x n) in the chunk buffer
  long long drow, trow;      // mixed form: first row of D_hk / T_hk in the split arrays
  long long urow;            // dense form: row of the block in U+ (p = +1) or U- (p = -1)
  long long ld;              // row pitch of the FP64 squares: n rounded up to even (16-byte aligned rows)
};
// one head for the gather
struct DLocHead {
  long long dom_off, n, lc_off;  // domain slice, offset of L^J_h (jmax x n x n) in the chunk buffer
  long long lrow;                // mixed form: first row of L^J_h (jmax n rows) in the split array
  long long ld;                  // row pitch of L^J_h (n rounded up to even)
};

__device__ __forceinline__ long long vpair(long long a, long long b) {
  return a >= b ? a * (a + 1) / 2 + b : b * (b + 1) / 2 + a;
}

// LT[J][vp] = L[vp][J] (32 x 32 tiles through shared memory)
__global__ void transpose_l(const double* __restrict__ L, long long npv, long long nchol, double* __restrict__ LT) {
  __shared__ double t[32][33];
  const long long r0 = (long long)blockIdx.y * 32, c0 = (long long)blockIdx.x * 32;
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const long long r = r0 + i, c = c0 + threadIdx.x;
    t[i][threadIdx.x] = (r < npv && c < nchol) ? L[r * nchol + c] : 0.0;
  }
  __syncthreads();
  for (int i = threadIdx.y; i < 32; i += blockDim.y) {
    const long long c = c0 + i, r = r0 + threadIdx.x;
    if (c < nchol && r < npv) LT[c * npv + r] = t[threadIdx.x][i];
  }
}

// Lc[lc_off + j n ld + a ld + c] = LT[J0 + j][vpair(dom[a], dom[c])]; blocks run
// head-fastest so that one row LT[J] serves every head from L2.
__global__ void gather_lc(const double* __restrict__ LT, long long npv, long long J0, const DLocHead* __restrict__ heads,
                          const long long* __restrict__ dom, double* __restrict__ Lc) {
  const DLocHead H = heads[blockIdx.x];
  const long long j = blockIdx.y;
  const double* row = LT + (J0 + j) * npv;
  const long long* d = dom + H.dom_off;
  double* out = Lc + H.lc_off + j * H.n * H.ld;
  for (long long e = threadIdx.x; e < H.n * H.n; e += blockDim.x) {
    const long long a = e / H.n, c = e % H.n;
    out[a * H.ld + c] = row[vpair(d[a], d[c])];
  }
}

__global__ void unpack_local(const DLocBlock* __restrict__ blk, const double* __restrict__ c, double* __restrict__ D) {
  const DLocBlock B = blk[blockIdx.x];
  const long long n = B.n, nab = n * (n - 1) / 2;
  double* Dk = D + B.d_off;
  for (long long e = threadIdx.x; e < n * n; e += blockDim.x) {
    const long long r = e / n, s = e % n;
    double v = 0.0;
    if (r == s) {
      if (B.aa) v = 1.4142135623730951 * c[B.off_aa + B.k * n + r];
    } else if (B.ab) {
      const long long i = r > s ? r : s, j = r > s ? s : r;
      const double x = c[B.off_ab + B.k * nab + i * (i - 1) / 2 + j];
      v = (r < s) ? x : B.p * x;
    }
    Dk[r * B.ld + s] = v;
  }
}

__global__ void pack_local(const DLocBlock* __restrict__ blk, const double* __restrict__ R, double* __restrict__ sigma) {
  const DLocBlock B = blk[blockIdx.x];
  const long long n = B.n, nab = n * (n - 1) / 2;
  const double* Rk = R + B.d_off;
  if (B.ab)
    for (long long e = threadIdx.x; e < nab; e += blockDim.x) {
      long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
      while (i * (i - 1) / 2 > e) --i;
      while ((i + 1) * i / 2 <= e) ++i;
      const long long j = e - i * (i - 1) / 2;
      sigma[B.off_ab + B.k * nab + e] += Rk[j * B.ld + i] + B.p * Rk[i * B.ld + j];
    }
  if (B.aa)
    for (long long a = threadIdx.x; a < n; a += blockDim.x)
      sigma[B.off_aa + B.k * n + a] += 1.4142135623730951 * Rk[a * B.ld + a];
}

// TF32 high part (low 13 mantissa bits cleared) and FP32 remainder, as the TMA-fed kernel reads them
__device__ __forceinline__ void split_put(float* hi, float* lo, long long i, double x) {
  const float h = __uint_as_float(__float_as_uint((float)x) & 0xFFFFE000u);
  hi[i] = h;
  lo[i] = (float)(x - (double)h);
}

// Mixed form: the gathered L^J_h as split rows of pitch ldp (row lrow + j n + a, column c)
__global__ void gather_lc_split(const double* __restrict__ LT, long long npv, long long J0,
                                const DLocHead* __restrict__ heads, const long long* __restrict__ dom,
                                float* __restrict__ hi, float* __restrict__ lo, long long ldp) {
  const DLocHead H = heads[blockIdx.x];
  const long long j = blockIdx.y;
  const double* row = LT + (J0 + j) * npv;
  const long long* d = dom + H.dom_off;
  const long long r0 = H.lrow + j * H.n;
  for (long long e = threadIdx.x; e < H.n * H.n; e += blockDim.x) {
    const long long a = e / H.n, c = e % H.n;
    split_put(hi, lo, (r0 + a) * ldp + c, row[vpair(d[a], d[c])]);
  }
}

// Mixed form: D_hk as split rows of pitch ldp (same matrix as unpack_local)
__global__ void unpack_local_split(const DLocBlock* __restrict__ blk, const double* __restrict__ c,
                                   float* __restrict__ hi, float* __restrict__ lo, long long ldp) {
  const DLocBlock B = blk[blockIdx.x];
  const long long n = B.n, nab = n * (n - 1) / 2;
  for (long long e = threadIdx.x; e < n * n; e += blockDim.x) {
    const long long r = e / n, s = e % n;
    double v = 0.0;
    if (r == s) {
      if (B.aa) v = 1.4142135623730951 * c[B.off_aa + B.k * n + r];
    } else if (B.ab) {
      const long long i = r > s ? r : s, j = r > s ? s : r;
      const double x = c[B.off_ab + B.k * nab + i * (i - 1) / 2 + j];
      v = (r < s) ? x : B.p * x;
    }
    split_put(hi, lo, (B.drow + r) * ldp + s, v);
  }
}

// Dense form: the block's entries at their places among all externals, as the interleaved TF32-high /
// FP32-low rows of U+ (singlet-coupled blocks: the n_ext pairs (aa), then the pairs (ac), a > c, at
// n_ext + a(a-1)/2 + c) or U- (triplet-coupled blocks: the pairs (ac) at a(a-1)/2 + c).  The rows are zero
// outside the domain (set before the launch).
__global__ void gather_dense(const DLocBlock* __restrict__ blk, const DLocHead* __restrict__ heads,
                             const long long* __restrict__ dom, const double* __restrict__ c, long long n_ext,
                             float* __restrict__ u2p, long long ldp_p, float* __restrict__ u2m, long long ldp_m) {
  const DLocBlock B = blk[blockIdx.x];
  const long long* d = dom + heads[B.head].dom_off;
  const long long n = B.n, nab = n * (n - 1) / 2;
  const bool plus = B.p > 0.0;
  const long long ld = plus ? ldp_p : ldp_m, base = plus ? n_ext : 0;
  float* hi = (plus ? u2p : u2m) + 2 * B.urow * ld;
  float* lo = hi + ld;
  if (B.ab)
    for (long long e = threadIdx.x; e < nab; e += blockDim.x) {
      long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
      while (i * (i - 1) / 2 > e) --i;
      while ((i + 1) * i / 2 <= e) ++i;
      const long long I = d[i], J = d[e - i * (i - 1) / 2];  // sorted domain: I > J
      split_put(hi, lo, base + I * (I - 1) / 2 + J, c[B.off_ab + B.k * nab + e]);
    }
  if (B.aa)
    for (long long a = threadIdx.x; a < n; a += blockDim.x) split_put(hi, lo, d[a], c[B.off_aa + B.k * n + a]);
}

// Dense form: the block's entries of Y+ (row pitch ldy_p) / Y- (ldy_m) into sigma (every entry of a block is
// written: sigma holds nothing else there)
__global__ void scatter_dense(const DLocBlock* __restrict__ blk, const DLocHead* __restrict__ heads,
                              const long long* __restrict__ dom, const double* __restrict__ yp, long long ldy_p,
                              const double* __restrict__ ym, long long ldy_m, long long n_ext,
                              double* __restrict__ sigma) {
  const DLocBlock B = blk[blockIdx.x];
  const long long* d = dom + heads[B.head].dom_off;
  const long long n = B.n, nab = n * (n - 1) / 2;
  const bool plus = B.p > 0.0;
  const double* y = plus ? yp + B.urow * ldy_p : ym + B.urow * ldy_m;
  const long long base = plus ? n_ext : 0;
  if (B.ab)
    for (long long e = threadIdx.x; e < nab; e += blockDim.x) {
      long long i = (long long)((1.0 + sqrt(1.0 + 8.0 * (double)e)) * 0.5);
      while (i * (i - 1) / 2 > e) --i;
      while ((i + 1) * i / 2 <= e) ++i;
      const long long I = d[i], J = d[e - i * (i - 1) / 2];
      sigma[B.off_ab + B.k * nab + e] = y[base + I * (I - 1) / 2 + J];
    }
  if (B.aa)
    for (long long a = threadIdx.x; a < n; a += blockDim.x) sigma[B.off_aa + B.k * n + a] = y[d[a]];
}

__global__ void add_into(double* __restrict__ dst, const double* __restrict__ src, long long n) {
  for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    dst[i] += src[i];
}

struct GemmLaunch {
  DGemmProblem* probs = nullptr;
  DGemmSeg* segs = nullptr;
  int nprob = 0;
  long long ntiles = 0;
  int cfg = 0;  // FP64 tile shape
};
struct TmaLaunch {
  TmaProblem* probs = nullptr;
  TmaSeg* segs = nullptr;
  int nprob = 0;
  long long ntiles = 0;
};

}  // namespace

struct tci_local {
  int device = 0;
  cudaStream_t stream = nullptr;
  int64_t nint = 0, nvirt = 0, nchol = 0, total = 0, precision = 0, kblock = 128;
  int64_t npv = 0;   // virtual pairs
  int64_t jmax = 0;  // largest chunk the buffers hold
  int64_t jc = 0;    // chunk in use
  int cfg2 = 0;      // FP64 tile shape of the second GEMM in use
  double flops = 0, lbytes = 0, dev_bytes = 0, last_ms = 0, tuned_ms = 0;
  int64_t candidates = 0;
  std::vector<void*> owned;
  std::unordered_map<void*, double> sizes;  // bytes of each alloc() buffer
  double *LT = nullptr, *Lc = nullptr, *T = nullptr, *D = nullptr, *R = nullptr, *Cb = nullptr, *Sb = nullptr;
  long long rlen = 0;
  DLocHead* dheads = nullptr;
  DLocBlock* dblocks = nullptr;
  long long* ddom = nullptr;
  std::vector<DLocBlock> blocks;
  std::vector<DLocHead> heads;
  int* status = nullptr;
  GemmLaunch g1, g2, g1r, g2r;  // full chunks and the shorter last chunk
  // mixed form: split arrays (row pitch ldp) and the TMA-fed tables
  long long ldp = 0, rows_l = 0, rows_d = 0, rows_t = 0;
  float *lc_hi = nullptr, *lc_lo = nullptr, *d_hi = nullptr, *d_lo = nullptr, *t_hi = nullptr, *t_lo = nullptr;
  tci_gtma_host::TmaMaps map1, map1n, map2;  // T = Lc D (128- or 64-wide tiles) ; R += 1/2 T Lc
  TmaLaunch m1, m2, m1r, m2r;
  // dense padded integral form (mixed precision): W+ / W- over all externals as FP32 tiles
  int form = 0;              // form in use: 0 Cholesky, 1 dense
  bool dense_ready = false;  // the dense operators are built
  int64_t np_d = 0, nm_d = 0, nsing_d = 0, ntrip_d = 0;
  float *w32p = nullptr, *w32m = nullptr, *u2p = nullptr, *u2m = nullptr;
  double *yp = nullptr, *ym = nullptr;
  tci_tc_host::AllextTc tcp, tcm;
  double dense_flops = 0, dense_ms = 0, dense_bytes = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  cudaEvent_t e0 = nullptr, e1 = nullptr;

  ~tci_local() {
    release_graph();
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (void* p : owned) cudaFree(p);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (stream) cudaStreamDestroy(stream);
  }
  void release_graph() {
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    exec = nullptr;
    graph = nullptr;
  }

  template <class T>
  T* upload(const std::vector<T>& v) {
    if (v.empty()) return nullptr;
    T* d = nullptr;
    if (cudaMalloc(&d, v.size() * sizeof(T)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(TCI_ERR_MEMORY, "device allocation failed (local all-external tables)");
    }
    owned.push_back(d);
    // stream-ordered before the kernels that read it (see sigma_device.cu upload)
    LCUDA(cudaMemcpyAsync(d, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice, stream));
    return d;
  }
  // frees an allocation made by alloc()
  template <class T>
  void release(T*& p) {
    if (!p) return;
    LCUDA(cudaStreamSynchronize(stream));
    auto it = std::find(owned.begin(), owned.end(), (void*)p);
    if (it != owned.end()) owned.erase(it);
    auto sz = sizes.find((void*)p);
    if (sz != sizes.end()) {
      dev_bytes -= sz->second;
      sizes.erase(sz);
    }
    LCUDA(cudaFree(p));
    p = nullptr;
  }
  float* alloc_f(size_t n) { return reinterpret_cast<float*>(alloc((n + 1) / 2)); }
  double* alloc(size_t n) {
    double* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(TCI_ERR_MEMORY, "device allocation failed (local all-external buffers)");
    }
    owned.push_back(p);
    dev_bytes += (double)n * sizeof(double);
    sizes[(void*)p] = (double)n * sizeof(double);
    return p;
  }

  // FP64 form: GEMM tables for chunks of j vectors (the chunk buffers are laid out for jmax)
  void make_gemms(int64_t j, int cfg_second, GemmLaunch& a, GemmLaunch& b) {
    std::vector<HostGemm> v1, v2;
    for (const auto& B : blocks) {
      const DLocHead& H = heads[B.head];
      const long long n = B.n, ld = B.ld;
      double* Tk = T + B.t_off;
      v1.push_back(HostGemm{Tk, ld, j * n, n, 0.0, {DGemmSeg{Lc + H.lc_off, D + B.d_off, ld, ld, n, 0, 0, 1.0}}});
      HostGemm y{R + B.d_off, ld, n, n, 1.0, {}};
      for (int64_t q = 0; q < j; ++q)
        y.segs.push_back(DGemmSeg{Tk + q * n * ld, Lc + H.lc_off + q * n * ld, ld, ld, n, 0, 0, 0.5});
      v2.push_back(std::move(y));
    }
    auto finish = [&](std::vector<HostGemm>& v, int cfg, GemmLaunch& g) {
      std::vector<DGemmProblem> pr;
      std::vector<DGemmSeg> sg;
      g.cfg = cfg;
      const long long tm = cfg == 2 ? tci_dev::gemm_cp_tile_m() : tci_dev::gemm_f64_tile_m(cfg);
      const long long tn = cfg == 2 ? tci_dev::gemm_cp_tile_n() : tci_dev::gemm_f64_tile_n(cfg);
      g.ntiles = tci_dev::tile_problems(v, tm, tn, false, pr, sg);
      g.probs = upload(pr);
      g.segs = upload(sg);
      g.nprob = (int)pr.size();
    };
    // cfg_second 0: both GEMMs on the cp.async-staged kernel (64 x 128 tiles; the even row pitches keep every
    // operand row 16-byte aligned); 1: the register-staged kernel, 128 x 64 tiles
    finish(v1, cfg_second == 0 ? 2 : 1, a);
    finish(v2, cfg_second == 0 ? 2 : 1, b);
  }

  // mixed form: TMA-fed tables for chunks of j vectors; narrow1: the first GEMM on 64-wide tiles
  void make_tma(int64_t j, bool narrow1, TmaLaunch& a, TmaLaunch& b) {
    const long long TM = tci_gtma_host::tile_m(), TN = tci_gtma_host::tile_n(map2.wide);
    const long long TN1 = tci_gtma_host::tile_n(narrow1 ? map1n.wide : map1.wide);
    std::vector<TmaProblem> p1, p2;
    std::vector<TmaSeg> s1, s2;
    long long t1 = 0, t2 = 0;
    for (const auto& B : blocks) {
      const DLocHead& H = heads[B.head];
      const long long n = B.n, tn = (n + TN - 1) / TN, tn1 = (n + TN1 - 1) / TN1;
      // T_hk (j n x n) = Lc_h D_hk, written split; D_hk enters as the K-major operand through D^T = p D
      TmaProblem q1{nullptr, 0, j * n, n, tn1, t1, 0.0, (long long)s1.size(), 0, 0,
                    t_hi + B.trow * ldp, t_lo + B.trow * ldp, ldp};
      s1.push_back(TmaSeg{H.lrow, B.drow, 0, n, B.p});
      q1.seg_end = (long long)s1.size();
      t1 += ((j * n + TM - 1) / TM) * tn1;
      p1.push_back(q1);
      // R_hk += 1/2 sum_J T_hkJ L^J_h (L^J_h symmetric: its rows are the K-major operand)
      TmaProblem q2{R + B.d_off, B.ld, n, n, tn, t2, 1.0, (long long)s2.size(), 0, 0, nullptr, nullptr, 0};
      for (int64_t q = 0; q < j; ++q) s2.push_back(TmaSeg{B.trow + q * n, H.lrow + q * n, 0, n, 0.5});
      q2.seg_end = (long long)s2.size();
      t2 += ((n + TM - 1) / TM) * tn;
      p2.push_back(q2);
    }
    a.probs = upload(p1);
    a.segs = upload(s1);
    a.nprob = (int)p1.size();
    a.ntiles = t1;
    b.probs = upload(p2);
    b.segs = upload(s2);
    b.nprob = (int)p2.size();
    b.ntiles = t2;
  }

  void launch_gemm(const GemmLaunch& g) {
    if (g.ntiles <= 0) return;
    if (g.cfg == 2) LCUDA(tci_dev::launch_gemm_cp_f64(g.probs, g.nprob, g.segs, g.ntiles, stream));
    else LCUDA(tci_dev::launch_gemm_f64(g.cfg, g.probs, g.nprob, g.segs, g.ntiles, stream));
  }

  // Dense form set-up from the virtual-virtual Cholesky rows lpk (npv x nchol, row-major, on the device):
  // the exchange product X = Lpk Lpk^T (npv x npv) on the TMA-fed 3xTF32 kernel, the W+ / W- tiles read
  // from it, X released.  Assigns each block its row of U+ / U-.
  void build_dense(const double* lpk) {
    const int64_t n = nvirt, nab = n * (n - 1) / 2;
    np_d = n + nab;
    nm_d = nab;
    nsing_d = ntrip_d = 0;
    for (auto& B : blocks) B.urow = B.p > 0.0 ? nsing_d++ : ntrip_d++;
    const int64_t ldk = tci_gtma_host::pitch(nchol);
    float* ah = alloc_f((size_t)(npv * ldk));
    float* al = alloc_f((size_t)(npv * ldk));
    double* X = alloc((size_t)(npv * npv));
    LCUDA(tci_gtma_host::split(lpk, npv, nchol, nchol, ah, al, stream));
    tci_gtma_host::TmaMaps m;
    std::string err;
    if (!tci_gtma_host::prepare(m, ah, al, npv, nchol, ah, al, npv, nchol, true, err)) throw Error(TCI_ERR_CUDA, err);
    const long long TM = tci_gtma_host::tile_m(), TN = tci_gtma_host::tile_n(true), tn = (npv + TN - 1) / TN;
    std::vector<TmaProblem> q{TmaProblem{X, npv, npv, npv, tn, 0, 0.0, 0, 1, 0, nullptr, nullptr, 0}};
    std::vector<TmaSeg> sg{TmaSeg{0, 0, 0, nchol, 1.0}};
    TmaProblem* dq = upload(q);
    TmaSeg* ds = upload(sg);
    LCUDA(tci_gtma_host::launch(m, dq, 1, ds, ((npv + TM - 1) / TM) * tn, (int)kblock, status, stream));
    LCUDA(cudaStreamSynchronize(stream));
    check_status();
    release(ah);
    release(al);
    w32p = alloc_f((size_t)tci_tc_host::w32_floats(np_d));
    LCUDA(tci_tc_host::convert_w_from_x(X, n, true, w32p, stream));
    if (nm_d > 0) {
      w32m = alloc_f((size_t)tci_tc_host::w32_floats(nm_d));
      LCUDA(tci_tc_host::convert_w_from_x(X, n, false, w32m, stream));
    }
    release(X);
    if (nsing_d > 0) {
      u2p = alloc_f((size_t)tci_tc_host::u2_floats(nsing_d, np_d));
      yp = alloc((size_t)(nsing_d * np_d));
      if (!tci_tc_host::prepare(tcp, w32p, np_d, u2p, nsing_d, yp, status, kblock, err)) throw Error(TCI_ERR_CUDA, err);
    }
    if (ntrip_d > 0) {
      u2m = alloc_f((size_t)tci_tc_host::u2_floats(ntrip_d, nm_d));
      ym = alloc((size_t)(ntrip_d * nm_d));
      if (!tci_tc_host::prepare(tcm, w32m, nm_d, u2m, ntrip_d, ym, status, kblock, err)) throw Error(TCI_ERR_CUDA, err);
    }
    dense_flops = 2.0 * (double)np_d * (double)np_d * (double)nsing_d + 2.0 * (double)nm_d * (double)nm_d * (double)ntrip_d;
    dense_bytes = 4.0 * ((double)tci_tc_host::w32_floats(np_d) + (nm_d > 0 ? (double)tci_tc_host::w32_floats(nm_d) : 0.0));
    dense_ready = true;
  }

  // Dense form, one application: Sb = [U+ W+ ; U- W-] gathered from and scattered to the local blocks.
  void record_dense() {
    const unsigned nb = (unsigned)blocks.size();
    LCUDA(cudaMemsetAsync(Sb, 0, sizeof(double) * (size_t)total, stream));
    if (nsing_d > 0)
      LCUDA(cudaMemsetAsync(u2p, 0, sizeof(float) * (size_t)tci_tc_host::u2_floats(nsing_d, np_d), stream));
    if (ntrip_d > 0)
      LCUDA(cudaMemsetAsync(u2m, 0, sizeof(float) * (size_t)tci_tc_host::u2_floats(ntrip_d, nm_d), stream));
    gather_dense<<<nb, 256, 0, stream>>>(dblocks, dheads, ddom, Cb, nvirt, u2p, tci_tc_host::padded_ld(np_d), u2m,
                                         tci_tc_host::padded_ld(std::max<int64_t>(1, nm_d)));
    LCUDA(cudaGetLastError());
    LCUDA(tci_tc_host::launch(nsing_d > 0 ? &tcp : nullptr, ntrip_d > 0 ? &tcm : nullptr, stream));
    scatter_dense<<<nb, 256, 0, stream>>>(dblocks, dheads, ddom, yp, np_d, ym, nm_d, nvirt, Sb);
    LCUDA(cudaGetLastError());
  }

  // One application on the internal buffers: Sb = A Cb.
  void record_apply() {
    const unsigned nb = (unsigned)blocks.size();
    if (form == 1) {
      record_dense();
      return;
    }
    if (precision == 1) {
      unpack_local_split<<<nb, 256, 0, stream>>>(dblocks, Cb, d_hi, d_lo, ldp);
      LCUDA(cudaGetLastError());
      LCUDA(cudaMemsetAsync(R, 0, sizeof(double) * (size_t)rlen, stream));
      LCUDA(cudaMemsetAsync(Sb, 0, sizeof(double) * (size_t)total, stream));
      for (int64_t J0 = 0; J0 < nchol; J0 += jc) {
        const int64_t jn = std::min<int64_t>(jc, nchol - J0);
        gather_lc_split<<<dim3((unsigned)heads.size(), (unsigned)jn), 256, 0, stream>>>(LT, npv, J0, dheads, ddom,
                                                                                       lc_hi, lc_lo, ldp);
        LCUDA(cudaGetLastError());
        const TmaLaunch& a = jn == jc ? m1 : m1r;
        const TmaLaunch& b = jn == jc ? m2 : m2r;
        LCUDA(tci_gtma_host::launch(cfg2 == 1 ? map1n : map1, a.probs, a.nprob, a.segs, a.ntiles, (int)kblock, status,
                                    stream));
        // second GEMM: few tiles with K = j n_h of very different length, left to the hardware scheduler
        LCUDA(tci_gtma_host::launch(map2, b.probs, b.nprob, b.segs, b.ntiles, (int)kblock, status, stream, false));
      }
      pack_local<<<nb, 256, 0, stream>>>(dblocks, R, Sb);
      LCUDA(cudaGetLastError());
      return;
    }
    unpack_local<<<nb, 256, 0, stream>>>(dblocks, Cb, D);
    LCUDA(cudaGetLastError());
    LCUDA(cudaMemsetAsync(R, 0, sizeof(double) * (size_t)rlen, stream));
    LCUDA(cudaMemsetAsync(Sb, 0, sizeof(double) * (size_t)total, stream));
    for (int64_t J0 = 0; J0 < nchol; J0 += jc) {
      const int64_t jn = std::min<int64_t>(jc, nchol - J0);
      gather_lc<<<dim3((unsigned)heads.size(), (unsigned)jn), 256, 0, stream>>>(LT, npv, J0, dheads, ddom, Lc);
      LCUDA(cudaGetLastError());
      launch_gemm(jn == jc ? g1 : g1r);
      launch_gemm(jn == jc ? g2 : g2r);
    }
    pack_local<<<nb, 256, 0, stream>>>(dblocks, R, Sb);
    LCUDA(cudaGetLastError());
  }

  // Tables and graph for chunk size j and second-GEMM tile shape cfg (Cholesky form).
  void configure(int64_t j, int cfg) {
    release_graph();
    form = 0;
    jc = j;
    cfg2 = cfg;
    const int64_t rem = nchol % jc;
    if (precision == 1) {
      make_tma(jc, cfg2 == 1, m1, m2);
      if (rem) make_tma(rem, cfg2 == 1, m1r, m2r);
    } else {
      make_gemms(jc, cfg2, g1, g2);
      if (rem) make_gemms(rem, cfg2, g1r, g2r);
    }
    capture();
  }
  // Graph of the dense form.
  void configure_dense() {
    release_graph();
    form = 1;
    capture();
  }
  // one application captured as the graph in use
  void capture() {
    LCUDA(cudaStreamBeginCapture(stream, cudaStreamCaptureModeThreadLocal));
    try {
      record_apply();
    } catch (...) {
      cudaGraph_t tmp = nullptr;
      cudaStreamEndCapture(stream, &tmp);
      if (tmp) cudaGraphDestroy(tmp);
      throw;
    }
    LCUDA(cudaStreamEndCapture(stream, &graph));
    LCUDA(cudaGraphInstantiate(&exec, graph, 0));
  }

  void run() {
    LCUDA(cudaEventRecord(e0, stream));
    LCUDA(cudaGraphLaunch(exec, stream));
    LCUDA(cudaEventRecord(e1, stream));
  }
  // one timed application of the graph in use (ms)
  float time_once() {
    run();
    LCUDA(cudaStreamSynchronize(stream));
    float ms = 0;
    LCUDA(cudaEventElapsedTime(&ms, e0, e1));
    return ms;
  }
  // buffers of the Cholesky form (after the dense form was chosen)
  void release_cholesky() {
    for (double** p : {&LT, &Lc, &T, &D, &R}) release(*p);
    for (float** p : {&lc_hi, &lc_lo, &d_hi, &d_lo, &t_hi, &t_lo}) release(*p);
  }
  // buffers of the dense form (after the Cholesky form was chosen)
  void release_dense() {
    for (float** p : {&w32p, &w32m, &u2p, &u2m}) release(*p);
    for (double** p : {&yp, &ym}) release(*p);
    dense_ready = false;
  }

  void check_status() {
    if (!status) return;
    int st = 0;
    LCUDA(cudaMemcpy(&st, status, sizeof(int), cudaMemcpyDeviceToHost));
    if (st != 0) throw Error(TCI_ERR_TIMEOUT, "tensor-core kernel: a bounded wait gave up (code " + std::to_string(st) + ")");
  }
};

extern "C" {

int tci_local_create(int64_t num_internal, int64_t num_external, const double* chol, int64_t nchol, int64_t n_heads,
                     const int64_t* heads, const int64_t* dom_idx, int64_t total_len, int64_t device,
                     const int64_t* options, int64_t n_options, tci_local** out) {
  if (!out || !chol || !heads || !dom_idx || n_heads <= 0 || nchol <= 0 || num_internal < 0 || num_external <= 0 ||
      total_len <= 0)
    return TCI_ERR_ARG;
  *out = nullptr;
  try {
    std::unique_ptr<tci_local> L(new tci_local());
    L->nint = num_internal;
    L->nvirt = num_external;
    L->nchol = nchol;
    L->total = total_len;
    L->precision = (options && n_options > 0) ? options[0] : 0;
    const double budget = (options && n_options > 1 && options[1] > 0) ? (double)options[1] : 16e9;
    if (options && n_options > 2 && options[2] > 0) L->kblock = options[2];
    const bool tune = !(options && n_options > 3 && options[3] == 0);
    const int64_t want_form = (options && n_options > 4) ? options[4] : 0;  // 0 faster, 1 Cholesky, 2 dense
    if (want_form < 0 || want_form > 2) throw Error(TCI_ERR_ARG, "unknown all-external form");
    if (L->precision < 0 || L->precision > 1 || L->kblock % 32) throw Error(TCI_ERR_ARG, "bad precision or promotion block");
    // heads and blocks (host checks: every index below is bounds-checked here, not on the device)
    long long dtot = 0, lc_per_j = 0, t_per_j = 0, dom_total = 0, lrows = 0, drows = 0, nmax = 0;
    for (int64_t h = 0; h < n_heads; ++h) {
      const int64_t* H = heads + 7 * h;
      const int64_t off_ab = H[0], off_aa = H[1], nsf_ab = H[2], nsf_aa = H[3], nsing = H[4], doff = H[5], n = H[6];
      if (n < 1 || doff < 0 || nsf_ab < 0 || nsf_aa < 0 || nsing < 0 || nsing > std::max(nsf_ab, nsf_aa))
        throw Error(TCI_ERR_INPUT, "inconsistent head record");
      dom_total = std::max<long long>(dom_total, doff + n);
      const long long nab = n * (n - 1) / 2;
      if ((nsf_ab > 0 && (off_ab < 0 || off_ab + nsf_ab * nab > total_len)) ||
          (nsf_aa > 0 && (off_aa < 0 || off_aa + nsf_aa * n > total_len)))
        throw Error(TCI_ERR_INPUT, "head block outside the CI vector");
      const long long nk = std::max(nsf_ab, nsf_aa);
      if (nk == 0) continue;
      const long long ld = n + (n & 1);
      // offsets per Cholesky vector, scaled by jmax below
      L->heads.push_back(DLocHead{doff, n, lc_per_j, lrows, ld});
      const long long hi = (long long)L->heads.size() - 1;
      for (long long k = 0; k < nk; ++k) {
        DLocBlock blk{off_ab, off_aa, n, k, k < nsf_ab ? 1 : 0, k < nsf_aa ? 1 : 0,
                      k < nsing ? 1.0 : -1.0, dtot, hi, t_per_j, drows, drows, 0, ld};
        L->blocks.push_back(blk);
        dtot += n * ld;
        drows += n;
        t_per_j += n * ld;
        L->flops += 4.0 * (double)nchol * (double)n * (double)n * (double)n;
      }
      lc_per_j += n * ld;
      lrows += n;
      nmax = std::max<long long>(nmax, n);
      L->lbytes += 8.0 * (double)nchol * (double)n * (double)n;
    }
    if (L->heads.empty()) throw Error(TCI_ERR_INPUT, "no head has a CI block");
    std::vector<long long> dom(dom_idx, dom_idx + dom_total);
    for (const auto& H : L->heads)
      for (long long a = 0; a < H.n; ++a) {
        const long long v = dom[H.dom_off + a];
        if (v < 0 || v >= num_external || (a > 0 && v <= dom[H.dom_off + a - 1]))
          throw Error(TCI_ERR_INPUT, "domains must be sorted, distinct external indices");
      }
    // chunk size: the gathered L^J_h and the T_hk of one chunk fit the budget
    // (mixed form: TF32-high / FP32-low rows of pitch ldp instead of FP64 squares)
    L->ldp = tci_gtma_host::pitch(nmax);
    const double per_j = L->precision == 1 ? 8.0 * (double)L->ldp * (double)(lrows + drows)
                                           : 8.0 * (double)(lc_per_j + t_per_j);
    L->jmax = std::max<int64_t>(1, std::min<int64_t>(nchol, (int64_t)(budget / per_j)));
    for (auto& H : L->heads) {
      H.lc_off *= L->jmax;
      H.lrow *= L->jmax;
    }
    for (auto& B : L->blocks) {
      B.t_off *= L->jmax;
      B.trow *= L->jmax;
    }
    L->rows_l = lrows * L->jmax;
    L->rows_d = drows;
    L->rows_t = drows * L->jmax;
    L->rlen = dtot;

    int ndev = 0;
    LCUDA(cudaGetDeviceCount(&ndev));
    if (device < 0 || device >= ndev) throw Error(TCI_ERR_CUDA, "requested device is not available");
    L->device = (int)device;
    LCUDA(cudaSetDevice(L->device));
    LCUDA(cudaStreamCreateWithFlags(&L->stream, cudaStreamNonBlocking));
    LCUDA(cudaEventCreate(&L->e0));
    LCUDA(cudaEventCreate(&L->e1));
    LCUDA(cudaMalloc(&L->status, sizeof(int)));
    L->owned.push_back(L->status);
    LCUDA(cudaMemsetAsync(L->status, 0, sizeof(int), L->stream));
    L->npv = num_external * (num_external + 1) / 2;
    // form: the dense padded integral form needs the mixed precision and every aa block singlet-coupled
    bool dense = L->precision == 1 && want_form != 1;
    for (const auto& B : L->blocks)
      if (B.aa && B.p < 0.0) dense = false;
    if (want_form == 2 && !dense)
      throw Error(TCI_ERR_INPUT, "the dense all-external form needs the mixed precision and singlet-coupled aa blocks");
    const bool chol_form = want_form != 2;
    if (dense) {
      // device bytes it needs at set-up (X, the split Cholesky rows, the W tiles, U and Y), with the
      // Cholesky form's buffers when both are timed, against what the device has free
      const int64_t n = num_external, nab = n * (n - 1) / 2, np = n + nab;
      int64_t ns = 0, nt = 0;
      for (const auto& B : L->blocks) (B.p > 0.0 ? ns : nt)++;
      double need = 8.0 * (double)L->npv * (double)L->npv + 8.0 * (double)L->npv * (double)tci_gtma_host::pitch(nchol) +
                    4.0 * ((double)tci_tc_host::w32_floats(np) + (nab > 0 ? (double)tci_tc_host::w32_floats(nab) : 0.0)) +
                    (ns > 0 ? 4.0 * (double)tci_tc_host::u2_floats(ns, np) + 8.0 * (double)(ns * np) : 0.0) +
                    (nt > 0 ? 4.0 * (double)tci_tc_host::u2_floats(nt, nab) + 8.0 * (double)(nt * nab) : 0.0) +
                    8.0 * (double)L->npv * (double)nchol + 2e9;
      if (chol_form) need += 8.0 * (double)L->npv * (double)nchol + per_j * (double)L->jmax + 8.0 * (double)dtot;
      size_t free_b = 0, total_b = 0;
      LCUDA(cudaMemGetInfo(&free_b, &total_b));
      if ((double)free_b < need) {
        if (want_form == 2) throw Error(TCI_ERR_MEMORY, "not enough device memory for the dense all-external form");
        dense = false;
      }
    }
    // virtual-virtual Cholesky rows (row-major on the device for the dense form's exchange product, J-major
    // for the Cholesky form)
    {
      std::vector<double> lvv((size_t)(L->npv * nchol));
      for (int64_t a = 0; a < num_external; ++a) {
        const int64_t p = num_internal + a;
        const int64_t row0 = p * (p + 1) / 2 + num_internal;  // pair (p, num_internal + b), b <= a
        std::memcpy(lvv.data() + (size_t)(a * (a + 1) / 2) * nchol, chol + (size_t)row0 * nchol,
                    sizeof(double) * (size_t)(a + 1) * nchol);
      }
      double* tmp = L->alloc(lvv.size());
      LCUDA(cudaMemcpyAsync(tmp, lvv.data(), lvv.size() * sizeof(double), cudaMemcpyHostToDevice, L->stream));
      if (dense) L->build_dense(tmp);
      if (chol_form) {
        L->LT = L->alloc(lvv.size());
        dim3 grid((unsigned)((nchol + 31) / 32), (unsigned)((L->npv + 31) / 32));
        transpose_l<<<grid, dim3(32, 8), 0, L->stream>>>(tmp, L->npv, nchol, L->LT);
        LCUDA(cudaGetLastError());
      }
      L->release(tmp);
    }
    if (chol_form && L->precision == 1) {
      // split arrays, zeroed once: the columns past each domain's n stay zero (the padding of the K tiles)
      auto falloc = [&](float** p, long long rows) {
        *p = L->alloc_f((size_t)(rows * L->ldp));
        LCUDA(cudaMemsetAsync(*p, 0, sizeof(float) * (size_t)(rows * L->ldp), L->stream));
      };
      falloc(&L->lc_hi, L->rows_l);
      falloc(&L->lc_lo, L->rows_l);
      falloc(&L->d_hi, L->rows_d);
      falloc(&L->d_lo, L->rows_d);
      falloc(&L->t_hi, L->rows_t);
      falloc(&L->t_lo, L->rows_t);
      std::string err;
      const bool wide = nmax > 64;  // tile width: the B operands have n_h rows per problem
      if (!tci_gtma_host::prepare(L->map1, L->lc_hi, L->lc_lo, L->rows_l, nmax, L->d_hi, L->d_lo, L->rows_d, nmax, wide,
                                  err) ||
          !tci_gtma_host::prepare(L->map1n, L->lc_hi, L->lc_lo, L->rows_l, nmax, L->d_hi, L->d_lo, L->rows_d, nmax,
                                  false, err) ||
          !tci_gtma_host::prepare(L->map2, L->t_hi, L->t_lo, L->rows_t, nmax, L->lc_hi, L->lc_lo, L->rows_l, nmax, wide,
                                  err))
        throw Error(TCI_ERR_CUDA, err);
    } else if (chol_form) {
      L->Lc = L->alloc((size_t)(lc_per_j * L->jmax));
      L->T = L->alloc((size_t)(t_per_j * L->jmax));
      L->D = L->alloc((size_t)dtot);
    }
    if (chol_form) L->R = L->alloc((size_t)dtot);
    L->Cb = L->alloc((size_t)total_len);
    L->Sb = L->alloc((size_t)total_len);
    LCUDA(cudaMemsetAsync(L->Cb, 0, sizeof(double) * (size_t)total_len, L->stream));
    LCUDA(cudaMemsetAsync(L->Sb, 0, sizeof(double) * (size_t)total_len, L->stream));
    L->dheads = L->upload(L->heads);
    L->dblocks = L->upload(L->blocks);
    L->ddom = L->upload(dom);

    // autotuner: chunk size (largest, half, quarter) x FP64 tile shape of the second GEMM (mixed form: tile
    // width of the first GEMM, 128 or 64); one timed run each.  Then the dense form, timed on its second
    // run; the faster form stays and the other's buffers are released.
    double best = 1e300;
    if (chol_form) {
      std::vector<std::pair<int64_t, int>> cand;
      for (int64_t j : {L->jmax, std::max<int64_t>(1, L->jmax / 2), std::max<int64_t>(1, L->jmax / 4)})
        for (int cfg : {0, 1}) {
          if (std::find(cand.begin(), cand.end(), std::make_pair(j, cfg)) == cand.end()) cand.push_back({j, cfg});
        }
      if (!tune) cand.resize(1);
      std::pair<int64_t, int> pick = cand[0];
      for (const auto& c : cand) {
        L->configure(c.first, c.second);
        const float ms = L->time_once();
        if (ms < best) {
          best = ms;
          pick = c;
        }
      }
      L->candidates = (int64_t)cand.size();
      L->tuned_ms = best;
      if (pick != std::make_pair(L->jc, L->cfg2)) L->configure(pick.first, pick.second);
    }
    if (L->dense_ready) {
      L->configure_dense();
      L->time_once();
      L->dense_ms = L->time_once();
      L->check_status();
      if (!chol_form || L->dense_ms < best) {
        L->release_cholesky();
      } else {
        L->release_dense();
        L->configure(L->jc, L->cfg2);
      }
    }
    L->check_status();
    *out = L.release();
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_local_apply(tci_local* L, const double* d_c, double* d_sigma, int64_t n, void* stream) {
  if (!L || !d_c || !d_sigma) return TCI_ERR_ARG;
  try {
    if (n != L->total) throw Error(TCI_ERR_ARG, "vector length differs from the heads' CI length");
    LCUDA(cudaSetDevice(L->device));
    cudaStream_t user = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    LCUDA(cudaEventRecord(L->e0, user));
    LCUDA(cudaStreamWaitEvent(L->stream, L->e0, 0));
    LCUDA(cudaMemcpyAsync(L->Cb, d_c, sizeof(double) * (size_t)n, cudaMemcpyDeviceToDevice, L->stream));
    L->run();
    add_into<<<(unsigned)std::min<int64_t>((n + 255) / 256, (int64_t)tci_dev::device_sms() * 8), 256, 0, L->stream>>>(d_sigma, L->Sb, n);
    LCUDA(cudaGetLastError());
    LCUDA(cudaEventRecord(L->e1, L->stream));  // after the accumulation into the caller's sigma
    LCUDA(cudaStreamWaitEvent(user, L->e1, 0));
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_local_apply_host(tci_local* L, const double* c, double* sigma, int64_t n) {
  if (!L || !c || !sigma) return TCI_ERR_ARG;
  try {
    if (n != L->total) throw Error(TCI_ERR_ARG, "vector length differs from the heads' CI length");
    LCUDA(cudaSetDevice(L->device));
    LCUDA(cudaMemcpyAsync(L->Cb, c, sizeof(double) * (size_t)n, cudaMemcpyHostToDevice, L->stream));
    L->run();
    std::vector<double> tmp((size_t)n);
    LCUDA(cudaMemcpyAsync(tmp.data(), L->Sb, sizeof(double) * (size_t)n, cudaMemcpyDeviceToHost, L->stream));
    LCUDA(cudaStreamSynchronize(L->stream));
    float ms = 0;
    LCUDA(cudaEventElapsedTime(&ms, L->e0, L->e1));
    L->last_ms = ms;
    L->check_status();
    for (int64_t i = 0; i < n; ++i) sigma[i] += tmp[(size_t)i];
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_local_stats(const tci_local* L, double* out, int64_t len) {
  if (!L || !out || len < 9) return TCI_ERR_ARG;
  const double v[13] = {L->flops,       L->lbytes,           L->dev_bytes,   (double)L->jc,    (double)L->cfg2,
                        L->tuned_ms,    (double)L->candidates, L->last_ms,   (double)L->blocks.size(),
                        (double)L->form, L->dense_ms,        L->dense_flops, L->dense_bytes};
  std::memcpy(out, v, sizeof(double) * (size_t)std::min<int64_t>(len, 13));
  return TCI_OK;
}

void tci_local_destroy(tci_local* L) { delete L; }

}  // extern "C"
