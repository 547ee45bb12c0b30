// The sigma plan: the complete sigma = H c of the MRSDCI space written as a
// short program over a handful of device buffers.  The host builds it once
// (this replaces the reference's iteration-1 "dry run" that enumerates loop
// records, e.g. three_and_four_seg_mod_1.f90:412-438, 695-776 and
// three_and_four_seg_mod_2.f90:1095-1195) and the device replays it on every
// sigma build.
//
// Step kinds:
//   GEMM   C(M x N) = beta*C + sum_seg alpha_seg * op(A_seg) op(B_seg)   (row major)
//   AXPY   dst[off:off+len] += sum_src coef * scale * src[soff:soff+len]
//   DOT    dst[off] += sum_src coef * <a[aoff:aoff+len], b[boff:boff+len]>
//   UNPACK CI vector -> dense external pair matrices of the N-2 heads (SCEP)
//   PACK   dense accumulators -> sigma (unSCEP), tiger_fortran/scepmaker_mod.f90
//   ZERO   buffer range
// Every target range is written by exactly one table entry per launch and the
// sources of an entry are summed in table order, so a sigma build is
// deterministic (same result alone or interleaved with other requests).
#pragma once
#include <sys/mman.h>

#include <cstdlib>
#include <functional>
#include <memory>
#include <new>
#include <type_traits>
#include <utility>
#include <vector>

#include "tci_host.h"

namespace tci {

// Allocator whose value-construction leaves the elements uninitialised: large arrays the plan builder fills
// in parallel right after sizing them (the first touch of each page then happens on the filling thread).
template <class T>
struct NoInitAlloc : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInitAlloc<U>;
  };
  NoInitAlloc() = default;
  template <class U>
  NoInitAlloc(const NoInitAlloc<U>&) noexcept {}
  template <class U>
  void construct(U* p) noexcept(std::is_nothrow_default_constructible<U>::value) {
    ::new ((void*)p) U;
  }
  template <class U, class... A>
  void construct(U* p, A&&... a) {
    ::new ((void*)p) U(std::forward<A>(a)...);
  }
  // large arrays (the coupling-vector rows: hundreds of MB) on 2 MB pages where the kernel allows it: the
  // threads that fill them fault in 2 MB at a time
  static constexpr std::size_t kLarge = std::size_t(64) << 20;
  T* allocate(std::size_t n) {
    const std::size_t bytes = n * sizeof(T);
    if (bytes < kLarge) return std::allocator<T>::allocate(n);
    void* p = nullptr;
    if (posix_memalign(&p, std::size_t(2) << 20, bytes) != 0) throw std::bad_alloc();
    madvise(p, bytes, MADV_HUGEPAGE);  // advice only: without it the pages stay 4 KB
    return static_cast<T*>(p);
  }
  void deallocate(T* p, std::size_t n) {
    if (n * sizeof(T) < kLarge) {
      std::allocator<T>::deallocate(p, n);
      return;
    }
    std::free(p);
  }
};

enum BufId : int {
  BUF_C = 0,   // input CI vector
  BUF_S,       // output sigma vector (accumulated)
  BUF_D,       // dense N-2 pair matrices, nD x n x n
  BUF_R,       // dense N-2 accumulators, nD x n x n
  BUF_T0,      // scratch
  BUF_T1,
  BUF_T2,
  BUF_T3,
  BUF_JK,      // (ij|ab) and (ia|jb) banks + h_ab: (2*nint^2 + 1) x n x n
  BUF_V,       // three-external banks, nint x n x n^2: V_i[b][q][s] = (iq|bs)
  BUF_W,       // all-external operators W+ (np x np) then W- (nm x nm)
  BUF_F,       // same-head combined one-external-electron operators, n x n each
  BUF_WV,      // precomputed vectors (one-external couplings), n each
  BUF_L,       // Cholesky vectors as given, npair_all x nchol
  BUF_LE,      // gathered L: internal-external rows, nint x n x nchol
  BUF_LV,      // gathered L: external-external rows, n*n x nchol
  BUF_LI,      // gathered L: internal-internal rows, nint*nint x nchol
  BUF_X,       // packed external (ab|cd), np x np (init only)
  NUM_BUFS
};

enum StepKind : int { STEP_GEMM = 0, STEP_AXPY, STEP_DOT, STEP_UNPACK, STEP_PACK, STEP_ZERO, STEP_WBUILD };

struct GemmProblem {
  int c;
  i64 offC, ldc, M, N;
  double beta;
  i64 seg_begin, seg_end;
};
struct GemmSeg {
  int a, b;
  i64 offA, lda, offB, ldb, K;
  int tA, tB;
  double alpha;
};
struct AxpyTarget {
  int dst;
  i64 off, len;
  i64 src_begin, src_end;
};
struct AxpySource {
  int src;
  i64 off;
  double coef;
  int sbuf;    // -1: no data-dependent scale
  i64 sidx;
};
struct DotTarget {
  int dst;
  i64 off;
  i64 src_begin, src_end;
};
struct DotSource {
  int a, b;
  i64 aoff, boff, len;
  double coef;
};

struct Step {
  int kind = 0;
  std::string name;
  std::vector<GemmProblem> gp;
  std::vector<GemmSeg> gs;
  std::vector<AxpyTarget> at;
  std::vector<AxpySource> as;
  std::vector<DotTarget> dt;
  std::vector<DotSource> ds;
  int buf = 0;          // ZERO
  i64 off = 0, len = 0; // ZERO
};

// One N-2 head as seen by UNPACK/PACK.
struct DHeadInfo {
  i64 off_ab, off_aa;  // CI-vector offsets (-1 if absent)
  i64 nsf_ab, nsf_aa;  // spin functions of each block
  i64 nsing;           // singlet-coupled functions (first nsing of the ab block)
  i64 nD;              // dense matrices of this head = max(nsf_ab, nsf_aa)
  i64 dk0;             // first dense matrix index
};

// One contiguous run of CSFs whose diagonal H_ii is assembled on the device:
//   type 0 valence:   beta
//   type 1 N-1 row:   beta + F(a,a)
//   type 2 N-2 aa:    beta + 2 F(a,a) + W+(a,a)
//   type 3 N-2 ab:    beta + F(i,i) + F(j,j) + W+-((ij),(ij))
// beta is the zero-external diagonal, F the same-head operator (BUF_F offset
// foff, -1 if none) and W the all-external operator.
struct DiagEntry {
  i64 off, len;
  i64 type;
  double beta;
  i64 foff;
  i64 singlet;
};

struct Plan {
  i64 nint = 0, n = 0, nchol = 0, total_csfs = 0, npair_all = 0;
  i64 nD = 0;                    // dense N-2 matrices
  std::vector<DHeadInfo> dheads;
  std::vector<double> dk_sign;   // +1 singlet-coupled, -1 triplet-coupled per dense matrix
  std::vector<i64> buf_size;     // doubles per buffer
  std::vector<double> h_vv;      // external one-electron block (n x n), uploaded into BUF_JK tail
  std::vector<double, NoInitAlloc<double>> wv;  // BUF_WV contents
  std::vector<Step> init_steps;  // run once after upload of L
  std::vector<Step> sigma_steps; // run per sigma build
  std::vector<DiagEntry> diag;   // diagonal H_ii assembly
  // algorithmic work per sigma build, for roofline reporting
  double flops_allext = 0, flops_total = 0, bytes_allext = 0;
  i64 np = 0, nm = 0;            // packed pair dimensions of W+ / W-
  i64 n_sing = 0, n_trip = 0;    // dense matrices per coupling type
  i64 allext_us = -1, allext_ys = -1, allext_ut = -1, allext_yt = -1;  // BUF_T0 offsets of U+/Y+/U-/Y-
};

struct Operator {
  const double* h = nullptr;     // n_orb x n_orb, row major, symmetric
  const double* chol = nullptr;  // [pair][J], pair = p(p+1)/2 + q, p >= q (0-based)
  i64 nchol = 0;
  double core_energy = 0.0;
};

// with_allext = false leaves the all-external term out (no X / W buffers, no WBUILD, no all-external steps;
// the diagonal entries of types 2 and 3 then need the all-external diagonal from elsewhere): the form used
// under local pair domains, whose all-external term runs in the pair-domain Cholesky form.
void build_plan(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext = true);
// The same, calling wv_done(plan) once the coupling-vector rows (plan.wv) are complete: the later phases
// (the zero-external blocks, the diagonal) leave plan.wv alone, so another thread may read it from then on.
void build_plan(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext,
                const std::function<void(const Plan&)>& wv_done);
// The leading set-up steps of build_plan's plan that need the orbital counts and the Cholesky rank only
// (gather cholesky rows, integral banks, all-external operators) and the sizes of their buffers.
void build_plan_operator_part(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext = true);

}  // namespace tci
