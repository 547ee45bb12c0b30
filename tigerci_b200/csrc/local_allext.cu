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
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include "../../include/tigerci_sigma.h"
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
  long long d_off;           // offset of D_hk / R_hk (n x n)
  long long head;            // index of the head
  long long t_off;           // offset of T_hk (jmax n x n) in the chunk buffer
  long long drow, trow;      // mixed form: first row of D_hk / T_hk in the split arrays
};
// one head for the gather
struct DLocHead {
  long long dom_off, n, lc_off;  // domain slice, offset of L^J_h (jmax x n x n) in the chunk buffer
  long long lrow;                // mixed form: first row of L^J_h (jmax n rows) in the split array
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

// Lc[lc_off + j n^2 + a n + c] = LT[J0 + j][vpair(dom[a], dom[c])]; blocks run
// head-fastest so that one row LT[J] serves every head from L2.
__global__ void gather_lc(const double* __restrict__ LT, long long npv, long long J0, const DLocHead* __restrict__ heads,
                          const long long* __restrict__ dom, double* __restrict__ Lc) {
  const DLocHead H = heads[blockIdx.x];
  const long long j = blockIdx.y;
  const double* row = LT + (J0 + j) * npv;
  const long long* d = dom + H.dom_off;
  double* out = Lc + H.lc_off + j * H.n * H.n;
  for (long long e = threadIdx.x; e < H.n * H.n; e += blockDim.x) {
    const long long a = e / H.n, c = e % H.n;
    out[e] = row[vpair(d[a], d[c])];
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
    Dk[e] = v;
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
      sigma[B.off_ab + B.k * nab + e] += Rk[j * n + i] + B.p * Rk[i * n + j];
    }
  if (B.aa)
    for (long long a = threadIdx.x; a < n; a += blockDim.x)
      sigma[B.off_aa + B.k * n + a] += 1.4142135623730951 * Rk[a * n + a];
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
  double* alloc(size_t n) {
    double* p = nullptr;
    if (cudaMalloc(&p, std::max<size_t>(1, n) * sizeof(double)) != cudaSuccess) {
      cudaGetLastError();
      throw Error(TCI_ERR_MEMORY, "device allocation failed (local all-external buffers)");
    }
    owned.push_back(p);
    dev_bytes += (double)n * sizeof(double);
    return p;
  }

  // FP64 form: GEMM tables for chunks of j vectors (the chunk buffers are laid out for jmax)
  void make_gemms(int64_t j, int cfg_second, GemmLaunch& a, GemmLaunch& b) {
    std::vector<HostGemm> v1, v2;
    for (const auto& B : blocks) {
      const DLocHead& H = heads[B.head];
      const long long n = B.n;
      double* Tk = T + B.t_off;
      v1.push_back(HostGemm{Tk, n, j * n, n, 0.0, {DGemmSeg{Lc + H.lc_off, D + B.d_off, n, n, n, 0, 0, 1.0}}});
      HostGemm y{R + B.d_off, n, n, n, 1.0, {}};
      for (int64_t q = 0; q < j; ++q)
        y.segs.push_back(DGemmSeg{Tk + q * n * n, Lc + H.lc_off + q * n * n, n, n, n, 0, 0, 0.5});
      v2.push_back(std::move(y));
    }
    auto finish = [&](std::vector<HostGemm>& v, int cfg, GemmLaunch& g) {
      std::vector<DGemmProblem> pr;
      std::vector<DGemmSeg> sg;
      g.cfg = cfg;
      g.ntiles = tci_dev::tile_problems(v, tci_dev::gemm_f64_tile_m(cfg), tci_dev::gemm_f64_tile_n(cfg), false, pr, sg);
      g.probs = upload(pr);
      g.segs = upload(sg);
      g.nprob = (int)pr.size();
    };
    finish(v1, 1, a);  // tall problems: 128 x 64 tiles
    finish(v2, cfg_second, b);
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
      TmaProblem q2{R + B.d_off, n, n, n, tn, t2, 1.0, (long long)s2.size(), 0, 0, nullptr, nullptr, 0};
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
    LCUDA(tci_dev::launch_gemm_f64(g.cfg, g.probs, g.nprob, g.segs, g.ntiles, stream));
  }

  // One application on the internal buffers: Sb = A Cb.
  void record_apply() {
    const unsigned nb = (unsigned)blocks.size();
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

  // Tables and graph for chunk size j and second-GEMM tile shape cfg.
  void configure(int64_t j, int cfg) {
    release_graph();
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
      L->heads.push_back(DLocHead{doff, n, lc_per_j, lrows});  // offsets per Cholesky vector, scaled by jmax below
      const long long hi = (long long)L->heads.size() - 1;
      for (long long k = 0; k < nk; ++k) {
        L->blocks.push_back(DLocBlock{off_ab, off_aa, n, k, k < nsf_ab ? 1 : 0, k < nsf_aa ? 1 : 0,
                                      k < nsing ? 1.0 : -1.0, dtot, hi, t_per_j, drows, drows});
        dtot += n * n;
        drows += n;
        t_per_j += n * n;
        L->flops += 4.0 * (double)nchol * (double)n * (double)n * (double)n;
      }
      lc_per_j += n * n;
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
    // virtual-virtual Cholesky rows, then J-major on the device
    L->npv = num_external * (num_external + 1) / 2;
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
      L->LT = L->alloc(lvv.size());
      dim3 grid((unsigned)((nchol + 31) / 32), (unsigned)((L->npv + 31) / 32));
      transpose_l<<<grid, dim3(32, 8), 0, L->stream>>>(tmp, L->npv, nchol, L->LT);
      LCUDA(cudaGetLastError());
      LCUDA(cudaStreamSynchronize(L->stream));
      LCUDA(cudaFree(tmp));
      L->owned.erase(std::find(L->owned.begin(), L->owned.end(), (void*)tmp));
      L->dev_bytes -= (double)lvv.size() * sizeof(double);
    }
    if (L->precision == 1) {
      // split arrays, zeroed once: the columns past each domain's n stay zero (the padding of the K tiles)
      auto falloc = [&](float** p, long long rows) {
        *p = reinterpret_cast<float*>(L->alloc((size_t)(rows * L->ldp + 1) / 2));
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
    } else {
      L->Lc = L->alloc((size_t)(lc_per_j * L->jmax));
      L->T = L->alloc((size_t)(t_per_j * L->jmax));
      L->D = L->alloc((size_t)dtot);
    }
    L->R = L->alloc((size_t)dtot);
    L->Cb = L->alloc((size_t)total_len);
    L->Sb = L->alloc((size_t)total_len);
    LCUDA(cudaMemsetAsync(L->Cb, 0, sizeof(double) * (size_t)total_len, L->stream));
    L->dheads = L->upload(L->heads);
    L->dblocks = L->upload(L->blocks);
    L->ddom = L->upload(dom);
    LCUDA(cudaMalloc(&L->status, sizeof(int)));
    L->owned.push_back(L->status);
    LCUDA(cudaMemsetAsync(L->status, 0, sizeof(int), L->stream));

    // autotuner: chunk size (largest, half, quarter) x FP64 tile shape of the second GEMM (mixed form: tile
    // width of the first GEMM, 128 or 64); one timed run each
    std::vector<std::pair<int64_t, int>> cand;
    for (int64_t j : {L->jmax, std::max<int64_t>(1, L->jmax / 2), std::max<int64_t>(1, L->jmax / 4)})
      for (int cfg : {0, 1}) {
        if (std::find(cand.begin(), cand.end(), std::make_pair(j, cfg)) == cand.end()) cand.push_back({j, cfg});
      }
    if (!tune) cand.resize(1);
    double best = 1e300;
    std::pair<int64_t, int> pick = cand[0];
    for (const auto& c : cand) {
      L->configure(c.first, c.second);
      L->run();
      LCUDA(cudaStreamSynchronize(L->stream));
      float ms = 0;
      LCUDA(cudaEventElapsedTime(&ms, L->e0, L->e1));
      if (ms < best) {
        best = ms;
        pick = c;
      }
    }
    L->candidates = (int64_t)cand.size();
    L->tuned_ms = best;
    if (pick != std::make_pair(L->jc, L->cfg2)) L->configure(pick.first, pick.second);
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
    add_into<<<(unsigned)std::min<int64_t>((n + 255) / 256, 148 * 8), 256, 0, L->stream>>>(d_sigma, L->Sb, n);
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
  const double v[9] = {L->flops,       L->lbytes,        L->dev_bytes, (double)L->jc, (double)L->cfg2,
                       L->tuned_ms,    (double)L->candidates, L->last_ms, (double)L->blocks.size()};
  std::memcpy(out, v, sizeof(v));
  return TCI_OK;
}

void tci_local_destroy(tci_local* L) { delete L; }

}  // extern "C"
