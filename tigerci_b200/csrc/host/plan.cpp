// Builds the sigma plan (plan.h) for a non-local MRSDCI space.
//
// Term classes (external electrons N-2 = "D", N-1 = "S", valence = "V"), with
// the reference routines they replace:
//   DD all-external (ab|cd) ........ three_and_four_seg_mod_1.f90:318-632, 3240-3627
//   DD two-external (ij|ab),(ia|jb)  three_and_four_seg_mod_2.f90:1000-1408, 7137-8005
//                                    two_seg_mod_3.f90:274-406, 2177-2795 (same head)
//   DS three-external (ia|bc) ...... three_and_four_seg_mod_1.f90:636-1756, 2867-3140
//   DS one-external (ij|ka), h_ia .. two_seg_mod_3.f90:617, 2797; mod_1.f90:1757-2216
//   DV two-external (ia|jb) ........ three_and_four_seg_mod_2.f90:7346-7408, 8007-8165
//   SS two-external ................ three_and_four_seg_mod_2.f90:7792-7956; two_seg_mod_3.f90
//   SV one-external ................ two_seg_mod_3.f90:617-883
//   zero-external / same config .... two_seg_mod_3.f90:884-1065; mod_2.f90:305-6233; diagtimesc.f90
// Coupling coefficients come from the CSF expansion of coupling.cpp applied to
// model configurations in which the external orbitals are replaced by three
// representative orbitals e0 < e1 < e2 placed after the internal ones (the
// coupling depends only on the relative order of the open shells).  Each
// coefficient is normalised against the dense-matrix form the device applies
// (UNPACK -> products -> PACK), so one canonical external pattern fixes it.
#include "plan.h"

#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <memory>
#include <tuple>
#include <unordered_map>

#include "coupling.h"

namespace tci {

namespace {

const double kSqrt2 = std::sqrt(2.0);
constexpr double kTiny = 1e-14;

// Open-addressing map from a packed occupation key (2 bits per internal orbital) to a head index, for the
// lookups of the zero-external enumeration (one per candidate excitation): linear probing in a power-of-two
// table at most half full.
struct KeyIndex {
  std::vector<uint64_t> keys;
  std::vector<i64> vals;
  uint64_t mask = 0;
  static constexpr uint64_t kEmpty = ~0ull;
  static uint64_t slot(uint64_t k) { return (k * 0x9E3779B97F4A7C15ull) >> 20; }
  void build(const std::vector<std::pair<uint64_t, i64>>& kv) {
    size_t cap = 16;
    while (cap < 2 * kv.size()) cap <<= 1;
    keys.assign(cap, kEmpty);
    vals.assign(cap, -1);
    mask = cap - 1;
    for (const auto& e : kv) {
      uint64_t h = slot(e.first) & mask;
      while (keys[h] != kEmpty && keys[h] != e.first) h = (h + 1) & mask;
      keys[h] = e.first;
      vals[h] = e.second;
    }
  }
  i64 find(uint64_t k) const {
    if (keys.empty()) return -1;
    for (uint64_t h = slot(k) & mask;; h = (h + 1) & mask) {
      if (keys[h] == k) return vals[h];
      if (keys[h] == kEmpty) return -1;
    }
  }
};

struct VecHash {
  size_t operator()(const std::vector<int8_t>& v) const {
    size_t h = 1469598103934665603ull;
    for (int8_t x : v) h = (h ^ (uint8_t)x) * 1099511628211ull;
    return h;
  }
};

inline int parity_below(Det d, int x) {
  Det m = d & ((((Det)1) << x) - 1);
  return (__builtin_popcountll((uint64_t)m) + __builtin_popcountll((uint64_t)(m >> 64))) & 1;
}

struct Ints {
  i64 norb = 0, nint = 0, n = 0, N = 0;
  const double* h = nullptr;
  const double* L = nullptr;
  std::vector<double> I4;  // (ij|kl), internal
  std::vector<double> I3;  // (iq|jk): [i][j][k][q]
  static i64 pair(i64 p, i64 q) { return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p; }
  double eri(i64 p, i64 q, i64 r, i64 s) const {
    const double* a = L + pair(p, q) * N;
    const double* b = L + pair(r, s) * N;
    double acc = 0;
    for (i64 J = 0; J < N; ++J) acc += a[J] * b[J];
    return acc;
  }
  double h1(i64 p, i64 q) const { return h[p * norb + q]; }
  double i4(i64 i, i64 j, i64 k, i64 l) const { return I4[((i * nint + j) * nint + k) * nint + l]; }
  const double* i3(i64 i, i64 j, i64 k) const { return I3.data() + ((i * nint + j) * nint + k) * n; }
  void build() {
    const i64 ni = nint;
    I4.assign(ni * ni * ni * ni, 0.0);
#pragma omp parallel for collapse(2) schedule(dynamic)
    for (i64 i = 0; i < ni; ++i)
      for (i64 j = 0; j < ni; ++j)
        for (i64 k = 0; k < ni; ++k)
          for (i64 l = 0; l < ni; ++l) I4[((i * ni + j) * ni + k) * ni + l] = eri(i, j, k, l);
    I3.assign(ni * ni * ni * n, 0.0);
    // (iq|jk) = L[pair(i, q)] . L[pair(j, k)]: the internal pair rows (the first ni(ni+1)/2 rows of L)
    // transposed once, then 4 rows L[pair(i, q)] x 4 internal pairs per register block, every dot still
    // summed in J order (the same value as eri())
    const i64 npr = ni * (ni + 1) / 2, npr8 = (npr + 3) / 4 * 4, nq4 = (n + 3) / 4;
    std::vector<double> Lt((size_t)(N * npr8), 0.0);
    std::vector<int> pj((size_t)npr), pk((size_t)npr);
    for (i64 j = 0; j < ni; ++j)
      for (i64 k = 0; k <= j; ++k) {
        pj[(size_t)pair(j, k)] = (int)j;
        pk[(size_t)pair(j, k)] = (int)k;
      }
    for (i64 pr = 0; pr < npr; ++pr)
      for (i64 J = 0; J < N; ++J) Lt[(size_t)(J * npr8 + pr)] = L[pr * N + J];
#pragma omp parallel for collapse(3) schedule(dynamic)
    for (i64 i = 0; i < ni; ++i)
      for (i64 qb = 0; qb < nq4; ++qb)
        for (i64 pb = 0; pb < npr8; pb += 4) {
          const double* a0 = L + pair(i, ni + std::min<i64>(qb * 4 + 0, n - 1)) * N;
          const double* a1 = L + pair(i, ni + std::min<i64>(qb * 4 + 1, n - 1)) * N;
          const double* a2 = L + pair(i, ni + std::min<i64>(qb * 4 + 2, n - 1)) * N;
          const double* a3 = L + pair(i, ni + std::min<i64>(qb * 4 + 3, n - 1)) * N;
          double c00 = 0, c01 = 0, c02 = 0, c03 = 0, c10 = 0, c11 = 0, c12 = 0, c13 = 0;
          double c20 = 0, c21 = 0, c22 = 0, c23 = 0, c30 = 0, c31 = 0, c32 = 0, c33 = 0;
          const double* lt = &Lt[(size_t)pb];
          for (i64 J = 0; J < N; ++J, lt += npr8) {
            const double l0 = lt[0], l1 = lt[1], l2 = lt[2], l3 = lt[3];
            const double x0 = a0[J], x1 = a1[J], x2 = a2[J], x3 = a3[J];
            c00 += x0 * l0; c01 += x0 * l1; c02 += x0 * l2; c03 += x0 * l3;
            c10 += x1 * l0; c11 += x1 * l1; c12 += x1 * l2; c13 += x1 * l3;
            c20 += x2 * l0; c21 += x2 * l1; c22 += x2 * l2; c23 += x2 * l3;
            c30 += x3 * l0; c31 += x3 * l1; c32 += x3 * l2; c33 += x3 * l3;
          }
          const double acc[4][4] = {{c00, c01, c02, c03}, {c10, c11, c12, c13}, {c20, c21, c22, c23}, {c30, c31, c32, c33}};
          for (int r = 0; r < 4; ++r) {
            const i64 q = qb * 4 + r;
            if (q >= n) break;
            for (int c = 0; c < 4 && pb + c < npr; ++c) {
              const i64 j = pj[(size_t)(pb + c)], k = pk[(size_t)(pb + c)];
              I3[(size_t)(((i * ni + j) * ni + k) * n + q)] = acc[r][c];
              I3[(size_t)(((i * ni + k) * ni + j) * n + q)] = acc[r][c];
            }
          }
        }
  }
};

// Bump allocator over one scratch buffer.
struct Scratch {
  i64 top = 0;
  i64 alloc(i64 len) {
    i64 o = top;
    top += (len + 31) / 32 * 32;
    return o;
  }
};

struct Builder {
  const CsfSpace& sp;
  const Operator& op;
  Plan& P;
  SpinTables tables;
  std::unique_ptr<CouplingEngine> eng;
  Ints I;
  i64 nint = 0, n = 0, n2 = 0, nab = 0, N = 0;
  int e0 = 0, e1 = 0, e2 = 0;
  std::unordered_map<std::vector<int8_t>, i64, VecHash> idx[3];
  // the same index keyed by the packed occupation (2 bits per internal orbital; nint <= 32)
  KeyIndex pidx[3];
  std::vector<i64> dk0, nDh;  // per N-2 path
  i64 nF = 0;                 // matrices used in BUF_F
  Scratch T;                  // BUF_T0 regions used per sigma build
  i64 init_scratch = 0;       // BUF_T0 doubles used during init
  i64 offJ = 0, offK = 0, offH = 0;
  // zero-external diagonal beta per (block, path, k) and same-head operator offsets per (kind, path, k)
  std::map<std::tuple<int, i64, i64>, double> beta_diag;
  std::map<std::tuple<int, i64, i64>, i64> fdiag;
  void build_diag();

  bool with_allext = true;     // false: no all-external term (no X, W, WBUILD or all-external steps)
  std::function<void(const Plan&)> wv_done;  // called once plan.wv is complete (after sv)

  Builder(const CsfSpace& s, const Operator& o, Plan& p) : sp(s), op(o), P(p) {}

  i64 Jof(i64 i, i64 j) const { return offJ + (i * nint + j) * n2; }
  i64 Kof(i64 p, i64 q) const { return offK + (p * nint + q) * n2; }

  std::vector<int8_t> ext(const Head& h, int x, int y) const {
    std::vector<int8_t> o(h.occ.begin(), h.occ.end());
    o.resize(nint + 3, 0);
    if (x >= 0) o[x] += 1;
    if (y >= 0) o[y] += 1;
    return o;
  }
  Config cfgV(const Head& h) const { return Config{ext(h, -1, -1)}; }
  Config cfgS(const Head& h, int x) const { return Config{ext(h, x, -1)}; }
  Config cfgD(const Head& h, int x, int y) const { return Config{ext(h, x, y)}; }
  const Head* find(int kind, const std::vector<int8_t>& occ) const {
    auto it = idx[kind].find(occ);
    if (it == idx[kind].end()) return nullptr;
    const Head& h = sp.paths[kind][it->second];
    return h.kept ? &h : nullptr;
  }
  std::vector<double> M(const Config& L, const Config& R, const Op& o) {
    std::vector<double> m;
    eng->matrix(L, R, o, m);
    return m;
  }
  double sgn(const Head& h, i64 k) const { return P.dk_sign[dk0[h.lex - 1] + k]; }
  i64 dk(const Head& h, i64 k) const { return dk0[h.lex - 1] + k; }
  i64 nD(const Head& h) const { return nDh[h.lex - 1]; }
  static bool has(const Head& h) { return h.kept && h.nsf > 0 && h.off >= 0; }

  void run();
  void run_operator_part();
  void setup_heads();
  void init_steps();
  void allext();
  void dd_x();
  void ds();
  void dv();
  void ss();
  void sv();
  void internal_blocks();
  static Step mkstep(int kind, const char* name) {
    Step s;
    s.kind = kind;
    s.name = name;
    return s;
  }
  // Returned references are invalidated by the next push onto the same list.
  Step& step(std::vector<Step>& v, int kind, const char* name) {
    v.push_back(Step());
    v.back().kind = kind;
    v.back().name = name;
    return v.back();
  }
  void zero_step(std::vector<Step>& v, int buf, i64 off, i64 len, const char* name) {
    Step& s = step(v, STEP_ZERO, name);
    s.buf = buf;
    s.off = off;
    s.len = len;
  }
};

void Builder::setup_heads() {
  for (int k = 0; k < 3; ++k) {
    std::vector<std::pair<uint64_t, i64>> kv;
    for (size_t p = 0; p < sp.paths[k].size(); ++p)
      if (sp.paths[k][p].kept) {
        idx[k][sp.paths[k][p].occ] = (i64)p;
        if (nint <= 32) {
          uint64_t key = 0;
          for (i64 q = 0; q < nint; ++q) key |= (uint64_t)sp.paths[k][p].occ[(size_t)q] << (2 * q);
          kv.push_back({key, (i64)p});
        }
      }
    pidx[k].build(kv);
  }
  const auto& D = sp.paths[2];
  dk0.assign(D.size(), -1);
  nDh.assign(D.size(), 0);
  for (size_t p = 0; p < D.size(); ++p) {
    const Head& h = D[p];
    if (!h.kept) continue;
    i64 nab_f = h.off >= 0 ? h.nsf : 0, naa_f = h.off_aa >= 0 ? h.nsf_aa : 0;
    i64 nd = std::max(nab_f, naa_f);
    if (nd == 0) continue;
    dk0[p] = P.nD;
    nDh[p] = nd;
    DHeadInfo di{h.off >= 0 ? h.off : -1, h.off_aa, nab_f, naa_f, naa_f > 0 ? (i64)sp.fsn[h.singles] : 0, nd, P.nD};
    P.dheads.push_back(di);
    for (i64 k = 0; k < nd; ++k) P.dk_sign.push_back(k < di.nsing ? 1.0 : -1.0);
    P.nD += nd;
  }
}

// ---------------------------------------------------------------------------
// Zero-external terms: all-internal Hamiltonian between configurations of one
// kind with spectator externals, by Slater rules on the CSF determinants.
void Builder::internal_blocks() {
  Step& st = step(P.sigma_steps, STEP_AXPY, "zero-external");
  struct TargetRows {
    std::vector<AxpySource> src;
    std::vector<AxpyTarget> rows;  // src_begin / src_end relative to src
  };
  std::vector<std::vector<TargetRows>> pattern_rows;  // per pattern, per head
  struct Pat {
    int kind, x, y, block;  // block: 0 valence, 1 N-1 row, 2 N-2 aa, 3 N-2 ab
  };
  const Pat pats[4] = {{0, -1, -1, 0}, {1, e0, -1, 1}, {2, e0, e0, 2}, {2, e0, e1, 3}};
  const int ni = (int)nint;
  bool bad_count = false;
  for (const Pat& pt : pats) {
    const auto& heads = sp.paths[pt.kind];
    auto nsf_of = [&](const Head& h) -> i64 {
      if (pt.block == 2) return h.off_aa >= 0 ? h.nsf_aa : 0;
      if (pt.block == 3) return h.off >= 0 ? h.nsf : 0;
      return h.off >= 0 ? h.nsf : 0;
    };
    auto off_of = [&](const Head& h) -> i64 { return pt.block == 2 ? h.off_aa : h.off; };
    const i64 len = pt.block == 0 ? 1 : pt.block == 3 ? nab : n;
    if (len == 0) continue;
    auto cfg = [&](const Head& h) {
      return pt.kind == 0 ? cfgV(h) : pt.kind == 1 ? cfgS(h, pt.x) : cfgD(h, pt.x, pt.y);
    };
    // Heads in parallel: every source head hs owns its blocks (by target, in target order), so the result
    // does not depend on the schedule.
    std::vector<std::vector<std::pair<i64, std::vector<double>>>> by_src(heads.size());
    const int nthr = omp_get_max_threads();
    std::vector<std::unique_ptr<CouplingEngine>> engines((size_t)nthr);
    for (auto& e : engines) e = std::make_unique<CouplingEngine>(tables);
    // per thread: the expansion of each head of this pattern, looked up once
    std::vector<std::vector<const CsfExpansion*>> hexp((size_t)omp_get_max_threads(),
                                                       std::vector<const CsfExpansion*>(heads.size(), nullptr));
    const bool packed = nint <= 32;
    const uint64_t mask2 = packed ? (nint == 32 ? ~0ull : ((1ull << (2 * nint)) - 1)) & 0x5555555555555555ull : 0;
    // per thread: the slot of each target head in the current source head's block list (-1: none yet)
    std::vector<std::vector<int>> slot((size_t)nthr, std::vector<int>(heads.size(), -1));
    // per thread: bit (p, q, r, s) set when removing electrons from spatial orbitals p <= q and adding them to
    // r <= s turns the current source head into a kept head of the pattern (the target of a double
    // excitation depends only on its spatial orbitals, so one lookup per spatial move serves every
    // determinant and spin assignment)
    const size_t nq = packed ? (size_t)ni * ni * ni * ni : 0;
    std::vector<std::vector<uint64_t>> dbits((size_t)nthr, std::vector<uint64_t>((nq + 63) / 64, 0));
    // and whether any such move starts with (p, q) or with (p, q, r): whole loop levels skipped
    std::vector<std::vector<uint8_t>> dany((size_t)nthr, std::vector<uint8_t>(packed ? (size_t)ni * ni * (ni + 1) : 0, 0));
    // Pair form, for patterns of up to 8192 heads: every target head within two electron moves of the source
    // (by internal occupation) and every determinant pair of the two heads that differs in at most four
    // internal spin orbitals (and not at all in the spectator externals) gives one Slater-rule element, the
    // same elements the excitation enumeration below reaches from the source determinants; no per-candidate
    // lookups. The expansions of the pattern's kept heads are made once up front.
    const bool pair_form = packed && heads.size() <= 8192;
    std::vector<const CsfExpansion*> pexp(pair_form ? heads.size() : 0, nullptr);
    if (pair_form) {
#pragma omp parallel for schedule(dynamic, 16)
      for (long long tl = 0; tl < (long long)heads.size(); ++tl) {
        const Head& Tg = heads[(size_t)tl];
        if (!Tg.kept || nsf_of(Tg) == 0) continue;
        const CsfExpansion& e = engines[(size_t)omp_get_thread_num()]->expand(cfg(Tg));
        if (e.nsf == nsf_of(Tg)) pexp[(size_t)tl] = &e;
      }
    }
    const uint64_t int_mask = packed ? (ni == 32 ? ~0ull : ((1ull << (2 * ni)) - 1)) : 0;
#pragma omp parallel for schedule(dynamic, 4)
    for (long long hsl = 0; hsl < (long long)heads.size(); ++hsl) {
      const size_t hs = (size_t)hsl;
      const int th = omp_get_thread_num();
      CouplingEngine& E = *engines[(size_t)th];  // per-thread expansion cache
      auto& hx = hexp[(size_t)th];
      auto& sl = slot[(size_t)th];
      auto& db = dbits[(size_t)th];
      uint8_t* any3 = dany[(size_t)th].data();             // (p, q, r)
      uint8_t* any2 = any3 + (packed ? (size_t)ni * ni * ni : 0);  // (p, q)
      // this source head's blocks by target
      auto& local = by_src[hs];
      const Head& S = heads[hs];
      if (!S.kept || nsf_of(S) == 0) continue;
      const CsfExpansion& eS = E.expand(cfg(S));
      if (eS.nsf != nsf_of(S)) {
        bad_count = true;
        continue;
      }
      auto kept_target = [&](i64 t) { return t >= 0 && heads[(size_t)t].kept && nsf_of(heads[(size_t)t]) != 0; };
      if (pair_form) {
        // target-major: this loop's head is the target T (eS / S name it here), the candidates the sources;
        // local collects T's blocks in source order
        auto orb = [](int x) { return x >> 1; };
        auto spn = [](int x) { return x & 1; };
        auto low_bit = [](uint64_t v) { return __builtin_ctzll(v); };
        const CsfExpansion& eT = eS;
        const Head& Tg = S;
        for (size_t t = 0; t < heads.size(); ++t) {
          const CsfExpansion* eSp = pexp[t];
          if (!eSp) continue;
          const CsfExpansion& eSrc = *eSp;
          int dist = 0;
          for (int p = 0; p < ni && dist <= 4; ++p)
            dist += std::abs((int)heads[t].occ[(size_t)p] - (int)Tg.occ[(size_t)p]);
          if (dist > 4) continue;
          std::vector<double>* blk = nullptr;
          for (size_t r = 0; r < eSrc.dets.size(); ++r) {
            const Det d0 = eSrc.dets[r];
            const double* thS = eSrc.basis->coeff.data() + r * eSrc.nsf;
            for (size_t q = 0; q < eT.dets.size(); ++q) {
              const Det dt = eT.dets[q];
              const Det x = d0 ^ dt;
              if ((uint64_t)(x >> 64) != 0 || ((uint64_t)x & ~int_mask) != 0) continue;  // externals must agree
              const uint64_t xl = (uint64_t)x;
              const int nb = __builtin_popcountll(xl);
              if (nb > 4) continue;
              const uint64_t dl = (uint64_t)d0 & int_mask;
              double val = 0.0;
              if (nb == 0) {  // diagonal
                for (uint64_t a = dl; a; a &= a - 1) {
                  const int xa = low_bit(a), pp = orb(xa);
                  val += I.h1(pp, pp);
                  for (uint64_t b = dl; b; b &= b - 1) {
                    const int xb = low_bit(b), qq = orb(xb);
                    val += 0.5 * I.i4(pp, pp, qq, qq);
                    if (spn(xa) == spn(xb)) val -= 0.5 * I.i4(pp, qq, qq, pp);
                  }
                }
              } else if (nb == 2) {  // single xa -> xb
                const int xa = low_bit(xl & dl), xb = low_bit(xl & ~dl);
                const int pp = orb(xb), qq = orb(xa);
                double v = I.h1(pp, qq);
                for (uint64_t c = dl & ~(1ull << xa); c; c &= c - 1) {
                  const int xc = low_bit(c), rr = orb(xc);
                  v += I.i4(pp, qq, rr, rr);
                  if (spn(xc) == spn(xa)) v -= I.i4(pp, rr, rr, qq);
                }
                Det d = d0;
                double ph = parity_below(d, xa) ? -1.0 : 1.0;
                d &= ~(((Det)1) << xa);
                if (parity_below(d, xb)) ph = -ph;
                val = ph * v;
              } else {  // double (xa, xb) -> (xc, xd), xa < xb, xc < xd
                const uint64_t hole = xl & dl, part = xl & ~dl;
                const int xa = low_bit(hole), xb = low_bit(hole & (hole - 1));
                const int xc = low_bit(part), xd = low_bit(part & (part - 1));
                double v = 0.0;
                if (spn(xc) == spn(xa) && spn(xd) == spn(xb)) v += I.i4(orb(xc), orb(xa), orb(xd), orb(xb));
                if (spn(xc) == spn(xb) && spn(xd) == spn(xa)) v -= I.i4(orb(xc), orb(xb), orb(xd), orb(xa));
                if (v != 0.0) {
                  Det d = d0;  // a+_c a+_d a_b a_a
                  double ph = 1.0;
                  if (parity_below(d, xa)) ph = -ph;
                  d &= ~(((Det)1) << xa);
                  if (parity_below(d, xb)) ph = -ph;
                  d &= ~(((Det)1) << xb);
                  if (parity_below(d, xd)) ph = -ph;
                  d |= ((Det)1) << xd;
                  if (parity_below(d, xc)) ph = -ph;
                  val = ph * v;
                }
              }
              if (val == 0.0) continue;
              if (!blk) {
                local.emplace_back((i64)t, std::vector<double>((size_t)eT.nsf * eSrc.nsf, 0.0));
                blk = &local.back().second;
              }
              const double* thT = eT.basis->coeff.data() + q * eT.nsf;
              const double f = val * eT.sign * eSrc.sign;
              for (int a = 0; a < eT.nsf; ++a) {
                if (thT[a] == 0.0) continue;
                for (int b = 0; b < eSrc.nsf; ++b) (*blk)[(size_t)a * eSrc.nsf + b] += f * thT[a] * thS[b];
              }
            }
          }
        }
        continue;  // local is in source order
      }
      if (packed) {  // the spatial double moves of this head that stay in the pattern's kept heads
        std::fill(db.begin(), db.end(), 0ull);
        std::fill(dany[(size_t)th].begin(), dany[(size_t)th].end(), (uint8_t)0);
        uint64_t key = 0;
        for (int p = 0; p < ni; ++p) key |= (uint64_t)S.occ[(size_t)p] << (2 * p);
        for (int p = 0; p < ni; ++p) {
          if (S.occ[(size_t)p] == 0) continue;
          for (int q = p; q < ni; ++q) {
            if (S.occ[(size_t)q] < (q == p ? 2 : 1)) continue;
            const uint64_t k2 = key - (1ull << (2 * p)) - (1ull << (2 * q));
            auto o = [&](int x) { return (int)((k2 >> (2 * x)) & 3); };
            for (int r = 0; r < ni; ++r) {
              if (o(r) == 2) continue;
              for (int t = r; t < ni; ++t) {
                if (o(t) > (t == r ? 0 : 1)) continue;
                if (!kept_target(pidx[pt.kind].find(k2 + (1ull << (2 * r)) + (1ull << (2 * t))))) continue;
                const size_t bit = (((size_t)p * ni + q) * ni + r) * ni + t;
                db[bit >> 6] |= 1ull << (bit & 63);
                any3[((size_t)p * ni + q) * ni + r] = 1;
                any2[(size_t)p * ni + q] = 1;
              }
            }
          }
        }
      }
      for (size_t r = 0; r < eS.dets.size(); ++r) {
        const double* thS = eS.basis->coeff.data() + r * eS.nsf;
        const Det d0 = eS.dets[r];
        int occ[128], vir[128], no = 0, nv = 0;
        for (int x = 0; x < 2 * ni; ++x) {
          if ((d0 >> x) & 1) occ[no++] = x;
          else vir[nv++] = x;
        }
        // the kept head of this pattern whose configuration is the determinant's (nullptr if none)
        auto target_of = [&](Det d) -> const Head* {
          const Head* Tg = nullptr;
          if (packed) {  // per-orbital electron counts of the determinant, 2 bits each
            const uint64_t lo = (uint64_t)d;
            const i64 t = pidx[pt.kind].find((lo & mask2) + ((lo >> 1) & mask2));
            if (t >= 0) Tg = &heads[(size_t)t];
          } else {
            std::vector<int8_t> o(ni);
            for (int p = 0; p < ni; ++p) o[p] = (int8_t)(((d >> (2 * p)) & 1) + ((d >> (2 * p + 1)) & 1));
            Tg = find(pt.kind, o);
          }
          return (Tg && Tg->kept && nsf_of(*Tg) != 0) ? Tg : nullptr;
        };
        auto emit_to = [&](const Head* Tg, Det d, double val) {
          if (val == 0.0 || !Tg) return;
          const size_t ti = (size_t)(Tg->lex - 1);
          if (!hx[ti]) hx[ti] = &E.expand(cfg(*Tg));
          const CsfExpansion& eT = *hx[ti];
          int row = -1;
          if (eT.dets.size() <= 32) {
            for (size_t x = 0; x < eT.dets.size(); ++x)
              if (eT.dets[x] == d) {
                row = (int)x;
                break;
              }
          } else {
            auto it = eT.index.find(d);
            if (it != eT.index.end()) row = it->second;
          }
          if (row < 0) return;
          const double* thT = eT.basis->coeff.data() + (size_t)row * eT.nsf;
          if (sl[ti] < 0) {
            sl[ti] = (int)local.size();
            local.emplace_back((i64)ti, std::vector<double>((size_t)eT.nsf * eS.nsf, 0.0));
          }
          auto& blk = local[(size_t)sl[ti]].second;
          const double f = val * eT.sign * eS.sign;
          for (int a = 0; a < eT.nsf; ++a) {
            if (thT[a] == 0.0) continue;
            for (int b = 0; b < eS.nsf; ++b) blk[(size_t)a * eS.nsf + b] += f * thT[a] * thS[b];
          }
        };
        auto emit = [&](Det d, double val) {
          if (val != 0.0) emit_to(target_of(d), d, val);
        };
        auto orb = [](int x) { return x >> 1; };
        auto spn = [](int x) { return x & 1; };
        {  // diagonal
          double e = 0;
          for (int a = 0; a < no; ++a) {
            const int p = orb(occ[a]);
            e += I.h1(p, p);
            for (int b = 0; b < no; ++b) {
              const int q = orb(occ[b]);
              e += 0.5 * I.i4(p, p, q, q);
              if (spn(occ[a]) == spn(occ[b])) e -= 0.5 * I.i4(p, q, q, p);
            }
          }
          emit(d0, e);
        }
        for (int a = 0; a < no; ++a)  // singles xa -> xb
          for (int b = 0; b < nv; ++b) {
            const int xa = occ[a], xb = vir[b];
            if (spn(xa) != spn(xb)) continue;
            const int p = orb(xb), q = orb(xa);
            double v = I.h1(p, q);
            for (int c = 0; c < no; ++c) {
              if (c == a) continue;
              const int r = orb(occ[c]);
              v += I.i4(p, q, r, r);
              if (spn(occ[c]) == spn(xa)) v -= I.i4(p, r, r, q);
            }
            Det d = d0;
            double ph = parity_below(d, xa) ? -1.0 : 1.0;
            d &= ~(((Det)1) << xa);
            if (parity_below(d, xb)) ph = -ph;
            d |= ((Det)1) << xb;
            emit(d, ph * v);
          }
        for (int a = 0; a < no; ++a)  // doubles (xa,xb) -> (xc,xd)
          for (int b = a + 1; b < no; ++b) {
            if (packed && !any2[(size_t)orb(occ[a]) * ni + orb(occ[b])]) continue;
            for (int c = 0; c < nv; ++c) {
              if (packed && !any3[((size_t)orb(occ[a]) * ni + orb(occ[b])) * ni + orb(vir[c])]) continue;
              for (int dd = c + 1; dd < nv; ++dd) {
                const int xa = occ[a], xb = occ[b], xc = vir[c], xd = vir[dd];
                if (spn(xa) + spn(xb) != spn(xc) + spn(xd)) continue;
                if (packed) {
                  const size_t bit = (((size_t)orb(xa) * ni + orb(xb)) * ni + orb(xc)) * ni + orb(xd);
                  if (!((db[bit >> 6] >> (bit & 63)) & 1)) continue;
                }
                // the target configuration first: most candidates leave the CI space
                const Det dt = d0 ^ ((((Det)1) << xa) | (((Det)1) << xb) | (((Det)1) << xc) | (((Det)1) << xd));
                const Head* Tg = target_of(dt);
                if (!Tg) continue;
                double v = 0;
                if (spn(xc) == spn(xa) && spn(xd) == spn(xb)) v += I.i4(orb(xc), orb(xa), orb(xd), orb(xb));
                if (spn(xc) == spn(xb) && spn(xd) == spn(xa)) v -= I.i4(orb(xc), orb(xb), orb(xd), orb(xa));
                if (v == 0.0) continue;
                Det d = d0;  // a+_c a+_d a_b a_a
                double ph = 1.0;
                if (parity_below(d, xa)) ph = -ph;
                d &= ~(((Det)1) << xa);
                if (parity_below(d, xb)) ph = -ph;
                d &= ~(((Det)1) << xb);
                if (parity_below(d, xd)) ph = -ph;
                d |= ((Det)1) << xd;
                if (parity_below(d, xc)) ph = -ph;
                d |= ((Det)1) << xc;
                emit_to(Tg, d, ph * v);
              }
            }
          }
      }
      for (const auto& kv : local) sl[(size_t)kv.first] = -1;
      std::sort(local.begin(), local.end(),
                [](const std::pair<i64, std::vector<double>>& x, const std::pair<i64, std::vector<double>>& y) {
                  return x.first < y.first;
                });
    }
    if (bad_count) throw Error(4, "spin-function count mismatch in zero-external block");
    // blocks by target, sources ascending (the pair form made them by target already)
    std::vector<std::vector<std::pair<i64, const std::vector<double>*>>> bytgt(heads.size());
    if (pair_form) {
#pragma omp parallel for schedule(dynamic, 16)
      for (long long tl = 0; tl < (long long)heads.size(); ++tl)
        for (const auto& sb : by_src[(size_t)tl]) bytgt[(size_t)tl].push_back({sb.first, &sb.second});
      for (size_t t = 0; t < heads.size(); ++t)
        for (const auto& sb : by_src[t])
          if (sb.first == (i64)t) {
            const i64 ns = nsf_of(heads[t]);
            for (i64 a = 0; a < ns; ++a) beta_diag[{pt.block, (i64)t, a}] = sb.second[(size_t)a * ns + a];
          }
    }
    for (size_t hs = 0; !pair_form && hs < heads.size(); ++hs)
      for (const auto& tb : by_src[hs]) {
        bytgt[(size_t)tb.first].push_back({(i64)hs, &tb.second});
        if (tb.first == (i64)hs) {
          const i64 ns = nsf_of(heads[hs]);
          for (i64 a = 0; a < ns; ++a) beta_diag[{pt.block, (i64)hs, a}] = tb.second[(size_t)a * ns + a];
        }
      }
    // the rows of every target (sources and row records), built per target in parallel; all patterns' rows
    // go into the step tables at the end, in pattern and target order
    auto& po = pattern_rows.emplace_back(heads.size());
#pragma omp parallel for schedule(dynamic, 16)
    for (long long tl = 0; tl < (long long)heads.size(); ++tl) {
      const auto& tv = bytgt[(size_t)tl];
      if (tv.empty()) continue;
      const Head& Tg = heads[(size_t)tl];
      const i64 nsfT = nsf_of(Tg);
      auto& out = po[(size_t)tl];
      for (i64 a = 0; a < nsfT; ++a) {
        const i64 begin = (i64)out.src.size();
        for (const auto& sv : tv) {
          const Head& S = heads[(size_t)sv.first];
          const i64 nsfS = nsf_of(S);
          for (i64 b = 0; b < nsfS; ++b) {
            const double v = (*sv.second)[(size_t)a * nsfS + b];
            if (std::fabs(v) < kTiny) continue;
            out.src.push_back(AxpySource{BUF_C, off_of(S) + b * len, v, -1, 0});
          }
        }
        const i64 end = (i64)out.src.size();
        if (end > begin) out.rows.push_back(AxpyTarget{BUF_S, off_of(Tg) + a * len, len, begin, end});
      }
    }
    // exact: integer-valued terms far below 2^53, so the sum does not depend on the order
    for (const auto& tr : po)
      for (const auto& r : tr.rows) P.flops_total += 2.0 * (double)len * (double)(r.src_end - r.src_begin);
  }
  // every target's place in the step tables, then the rows copied in parallel
  std::vector<std::pair<size_t, size_t>> order;  // (pattern, head) with rows
  std::vector<size_t> soff(1, 0), toff(1, 0);
  for (size_t q = 0; q < pattern_rows.size(); ++q)
    for (size_t t = 0; t < pattern_rows[q].size(); ++t) {
      const auto& tr = pattern_rows[q][t];
      if (tr.rows.empty()) continue;
      order.push_back({q, t});
      soff.push_back(soff.back() + tr.src.size());
      toff.push_back(toff.back() + tr.rows.size());
    }
  st.as.resize(soff.back());
  st.at.resize(toff.back());
#pragma omp parallel for schedule(dynamic, 16)
  for (long long ol = 0; ol < (long long)order.size(); ++ol) {
    auto& tr = pattern_rows[order[(size_t)ol].first][order[(size_t)ol].second];
    std::copy(tr.src.begin(), tr.src.end(), st.as.begin() + (std::ptrdiff_t)soff[(size_t)ol]);
    for (size_t j = 0; j < tr.rows.size(); ++j) {
      AxpyTarget x = tr.rows[j];
      x.src_begin += (i64)soff[(size_t)ol];
      x.src_end += (i64)soff[(size_t)ol];
      st.at[toff[(size_t)ol] + j] = x;
    }
    std::vector<AxpySource>().swap(tr.src);
  }
}

// ---------------------------------------------------------------------------
// One-electron-in-the-external-space operators X acting on one external
// electron: R[T,kt] += a * X * D[S,ks].  Returns a (nD(T) x nD(S)).
// op(x,z) creates external x and annihilates external z.
template <class MakeOp>
std::vector<double> alpha_dd(Builder& B, const Head& Tg, const Head& S, MakeOp make_op) {
  const i64 nT = B.nD(Tg), nS = B.nD(S);
  std::vector<double> a((size_t)nT * nS, 0.0);
  const bool Tab = Tg.off >= 0, Sab = S.off >= 0, Taa = Tg.off_aa >= 0, Saa = S.off_aa >= 0;
  if (Tab && Sab) {  // target (e0,e1) <- source (e2,e1): predicted p_s
    auto m = B.M(B.cfgD(Tg, B.e0, B.e1), B.cfgD(S, B.e2, B.e1), make_op(B.e0, B.e2));
    for (i64 kt = 0; kt < Tg.nsf; ++kt)
      for (i64 ks = 0; ks < S.nsf; ++ks) a[kt * nS + ks] = m[kt * S.nsf + ks] * B.sgn(S, ks);
  } else if (Tab && Saa) {  // target (e0,e2) <- source (e2,e2): predicted sqrt2
    auto m = B.M(B.cfgD(Tg, B.e0, B.e2), B.cfgD(S, B.e2, B.e2), make_op(B.e0, B.e2));
    for (i64 kt = 0; kt < Tg.nsf; ++kt)
      for (i64 ks = 0; ks < S.nsf_aa; ++ks) a[kt * nS + ks] = m[kt * S.nsf_aa + ks] / kSqrt2;
  } else if (Taa && Sab) {  // target (e0,e0) <- source (e2,e0): predicted sqrt2*p_s
    auto m = B.M(B.cfgD(Tg, B.e0, B.e0), B.cfgD(S, B.e2, B.e0), make_op(B.e0, B.e2));
    for (i64 kt = 0; kt < Tg.nsf_aa; ++kt)
      for (i64 ks = 0; ks < S.nsf; ++ks) a[kt * nS + ks] = m[kt * S.nsf + ks] / (kSqrt2 * B.sgn(S, ks));
  } else if (Taa && Saa) {  // target (e0,e0) <- source (e0,e0), x = z: predicted 2
    auto m = B.M(B.cfgD(Tg, B.e0, B.e0), B.cfgD(S, B.e0, B.e0), make_op(B.e0, B.e0));
    for (i64 kt = 0; kt < Tg.nsf_aa; ++kt)
      for (i64 ks = 0; ks < S.nsf_aa; ++ks) a[kt * nS + ks] = m[kt * S.nsf_aa + ks] / 2.0;
  }
  return a;
}

void Builder::dd_x() {
  Step& fcomb = step(P.init_steps, STEP_AXPY, "dd same-head operators");
  struct Term {
    i64 src_dk;
    int xbuf;
    i64 xoff;
    double a;
  };
  std::vector<std::vector<Term>> terms(P.nD);
  auto opJ = [](i64 i, i64 j) { return [=](int x, int z) { return Op{x, z, (int)i, (int)j}; }; };
  auto opK = [](i64 i, i64 j) { return [=](int x, int z) { return Op{x, (int)j, (int)i, z}; }; };
  auto opH = []() { return [](int x, int z) { return Op{x, z, -1, -1}; }; };
  for (size_t hs = 0; hs < sp.paths[2].size(); ++hs) {
    const Head& S = sp.paths[2][hs];
    if (!S.kept || nD(S) == 0) continue;
    const i64 nS = nD(S);
    {  // same head: F = a_h h + sum_i a_J J_ii + a_K K_ii
      std::vector<std::vector<std::pair<i64, double>>> comb((size_t)nS * nS);
      auto add = [&](const std::vector<double>& a, i64 xoff) {
        for (size_t t = 0; t < a.size(); ++t)
          if (std::fabs(a[t]) > kTiny) comb[t].push_back({xoff, a[t]});
      };
      add(alpha_dd(*this, S, S, opH()), offH);
      for (i64 i = 0; i < nint; ++i) {
        if (S.occ[i] == 0) continue;
        add(alpha_dd(*this, S, S, opJ(i, i)), Jof(i, i));
        add(alpha_dd(*this, S, S, opK(i, i)), Kof(i, i));
      }
      for (i64 kt = 0; kt < nS; ++kt)
        for (i64 ks = 0; ks < nS; ++ks) {
          auto& c = comb[kt * nS + ks];
          if (c.empty()) continue;
          AxpyTarget tg{BUF_F, nF * n2, n2, (i64)fcomb.as.size(), 0};
          for (auto& pr : c) fcomb.as.push_back(AxpySource{BUF_JK, pr.first, pr.second, -1, 0});
          tg.src_end = (i64)fcomb.as.size();
          fcomb.at.push_back(tg);
          terms[dk(S, kt)].push_back(Term{dk(S, ks), BUF_F, nF * n2, 1.0});
          if (kt == ks) fdiag[{2, (i64)hs, kt}] = nF * n2;
          ++nF;
        }
    }
    for (i64 j = 0; j < nint; ++j) {  // other heads: internal j -> i
      if (S.occ[j] == 0) continue;
      for (i64 i = 0; i < nint; ++i) {
        if (i == j || S.occ[i] == 2) continue;
        std::vector<int8_t> o(S.occ.begin(), S.occ.end());
        o[j] -= 1;
        o[i] += 1;
        const Head* Tg = find(2, o);
        if (!Tg || nD(*Tg) == 0) continue;
        auto aJ = alpha_dd(*this, *Tg, S, opJ(i, j));
        auto aK = alpha_dd(*this, *Tg, S, opK(i, j));
        const i64 nT = nD(*Tg);
        for (i64 kt = 0; kt < nT; ++kt)
          for (i64 ks = 0; ks < nS; ++ks) {
            const double vj = aJ[kt * nS + ks], vk = aK[kt * nS + ks];
            if (std::fabs(vj) > kTiny) terms[dk(*Tg, kt)].push_back(Term{dk(S, ks), BUF_JK, Jof(i, j), vj});
            if (std::fabs(vk) > kTiny) terms[dk(*Tg, kt)].push_back(Term{dk(S, ks), BUF_JK, Kof(j, i), vk});
          }
      }
    }
  }
  Step& st = step(P.sigma_steps, STEP_GEMM, "dd two-external");
  for (i64 d = 0; d < P.nD; ++d) {
    if (terms[d].empty()) continue;
    GemmProblem gp{BUF_R, d * n2, n, n, n, 1.0, (i64)st.gs.size(), 0};
    for (auto& t : terms[d]) st.gs.push_back(GemmSeg{t.xbuf, BUF_D, t.xoff, n, t.src_dk * n2, n, n, 0, 0, t.a});
    gp.seg_end = (i64)st.gs.size();
    st.gp.push_back(gp);
    P.flops_total += 2.0 * n * n * n * (double)terms[d].size();
  }
}

// ---------------------------------------------------------------------------
// DS: three-external (iq|bs) and one-external (iq|jk), h_iq.
void Builder::ds() {
  // ---- three-external: sigma_mu[b] += a * sum_{q,s} (iq|bs) D[q][s]
  struct T3 {
    i64 mu_row;  // CI offset of row (mu, k')
    i64 i, dkk;
    double a;
  };
  std::vector<T3> t3;
  // ---- one-external vectors: w(q) = sum a_op (iq|jk) (+ a h_iq), one per (mu k', dk)
  struct T1 {
    i64 mu_row, dkk;
    std::vector<double> w;
  };
  std::vector<T1> t1;
  // Source heads in parallel: every key (mu row, dk) of T1 and every T3 entry belongs to one source head (dk
  // is that head's), so per-head lists concatenated in head order give the serial loop's tables exactly.
  struct HeadOut {
    std::vector<T3> t3;
    std::vector<T1> t1;
  };
  const auto& heads2 = sp.paths[2];
  std::vector<HeadOut> hout(heads2.size());
  std::vector<std::unique_ptr<CouplingEngine>> engines((size_t)omp_get_max_threads());
  for (auto& e : engines) e = std::make_unique<CouplingEngine>(tables);
#pragma omp parallel for schedule(dynamic, 4)
  for (long long hsl = 0; hsl < (long long)heads2.size(); ++hsl) {
    const size_t hs = (size_t)hsl;
    CouplingEngine& E = *engines[(size_t)omp_get_thread_num()];  // per-thread expansion cache
    auto M = [&](const Config& L, const Config& R, const Op& o) {
      std::vector<double> m;
      E.matrix(L, R, o, m);
      return m;
    };
    auto& out = hout[hs];
    std::map<std::pair<i64, i64>, size_t> t1_index;  // this head's keys, in first-use order in out.t1
    auto w_of = [&](i64 mu_row, i64 dkk) -> std::vector<double>& {
      auto key = std::make_pair(mu_row, dkk);
      auto it = t1_index.find(key);
      if (it != t1_index.end()) return out.t1[it->second].w;
      t1_index[key] = out.t1.size();
      out.t1.push_back(T1{mu_row, dkk, std::vector<double>(n, 0.0)});
      return out.t1.back().w;
    };
    const Head& S = heads2[hs];
    if (!S.kept || nD(S) == 0) continue;
    const i64 nS = nD(S);
    const bool Sab = S.off >= 0;
    // three-external: mu = S + e_i
    for (i64 i = 0; i < nint; ++i) {
      if (S.occ[i] == 2) continue;
      std::vector<int8_t> o(S.occ.begin(), S.occ.end());
      o[i] += 1;
      const Head* Mu = find(1, o);
      if (!Mu || Mu->nsf == 0) continue;
      std::vector<double> a((size_t)Mu->nsf * nS, 0.0);
      if (Sab) {  // source (e1,e0), target (e2), op e_{i e0, e2 e1}: predicted 1
        auto m = M(cfgS(*Mu, e2), cfgD(S, e1, e0), Op{(int)i, e0, e2, e1});
        for (i64 kt = 0; kt < Mu->nsf; ++kt)
          for (i64 ks = 0; ks < S.nsf; ++ks) a[kt * nS + ks] = m[kt * S.nsf + ks];
      } else {  // source (e0,e0), target (e2), op e_{i e0, e2 e0}: predicted sqrt2
        auto m = M(cfgS(*Mu, e2), cfgD(S, e0, e0), Op{(int)i, e0, e2, e0});
        for (i64 kt = 0; kt < Mu->nsf; ++kt)
          for (i64 ks = 0; ks < S.nsf_aa; ++ks) a[kt * nS + ks] = m[kt * S.nsf_aa + ks] / kSqrt2;
      }
      for (i64 kt = 0; kt < Mu->nsf; ++kt)
        for (i64 ks = 0; ks < nS; ++ks)
          if (std::fabs(a[kt * nS + ks]) > kTiny) out.t3.push_back(T3{Mu->off + kt * n, i, dk(S, ks), a[kt * nS + ks]});
    }
    // one-external: ops e_{iq,jk} (a+_i a+_j a_k a_q) and E_iq
    auto add_op = [&](const Head* Mu, int i, int j, int k, bool one_el) {
      const i64 nT = Mu->nsf;
      std::vector<double> a((size_t)nT * nS, 0.0);
      if (Sab) {  // source (e1,e0) -> target (e0), annihilate q = e1: predicted p_s
        Op o = one_el ? Op{i, e1, -1, -1} : Op{i, e1, j, k};
        auto m = M(cfgS(*Mu, e0), cfgD(S, e1, e0), o);
        for (i64 kt = 0; kt < nT; ++kt)
          for (i64 ks = 0; ks < S.nsf; ++ks) a[kt * nS + ks] = m[kt * S.nsf + ks] * sgn(S, ks);
      } else {  // source (e0,e0) -> target (e0): predicted sqrt2
        Op o = one_el ? Op{i, e0, -1, -1} : Op{i, e0, j, k};
        auto m = M(cfgS(*Mu, e0), cfgD(S, e0, e0), o);
        for (i64 kt = 0; kt < nT; ++kt)
          for (i64 ks = 0; ks < S.nsf_aa; ++ks) a[kt * nS + ks] = m[kt * S.nsf_aa + ks] / kSqrt2;
      }
      for (i64 kt = 0; kt < nT; ++kt)
        for (i64 ks = 0; ks < nS; ++ks) {
          const double v = a[kt * nS + ks];
          if (std::fabs(v) <= kTiny) continue;
          auto& w = w_of(Mu->off + kt * n, dk(S, ks));
          if (one_el) {
            for (i64 q = 0; q < n; ++q) w[q] += v * I.h1(i, nint + q);
          } else {
            const double* iq = I.i3(i, j, k);
            for (i64 q = 0; q < n; ++q) w[q] += v * iq[q];
          }
        }
    };
    for (i64 i = 0; i < nint; ++i) {  // E_iq
      if (S.occ[i] == 2) continue;
      std::vector<int8_t> o(S.occ.begin(), S.occ.end());
      o[i] += 1;
      const Head* Mu = find(1, o);
      if (Mu && Mu->nsf > 0) add_op(Mu, (int)i, -1, -1, true);
    }
    for (i64 k = 0; k < nint; ++k) {
      if (S.occ[k] == 0) continue;
      for (i64 j = 0; j < nint; ++j) {
        std::vector<int8_t> o1(S.occ.begin(), S.occ.end());
        o1[k] -= 1;
        if (o1[j] == 2) continue;
        o1[j] += 1;
        for (i64 i = 0; i < nint; ++i) {
          if (o1[i] == 2) continue;
          std::vector<int8_t> o2 = o1;
          o2[i] += 1;
          const Head* Mu = find(1, o2);
          if (Mu && Mu->nsf > 0) add_op(Mu, (int)i, (int)j, (int)k, false);
        }
      }
    }
  }
  for (auto& ho : hout) {
    t3.insert(t3.end(), ho.t3.begin(), ho.t3.end());
    for (auto& x : ho.t1) t1.push_back(std::move(x));
  }

  // ---- device steps for the three-external term (V_i stored [b][(q,s)])
  if (!t3.empty()) {
    const i64 Y = T.alloc(nint * P.nD * n);  // Y[i][dk][b] = sum_{(q,s)} D[dk][(q,s)] V_i[b][(q,s)]
    std::vector<char> used(nint, 0);
    for (auto& t : t3) used[t.i] = 1;
    std::vector<std::pair<i64, i64>> outs;  // (offset into T0 of Y_i, i)
    for (i64 i = 0; i < nint; ++i)
      if (used[i]) outs.push_back({Y + i * P.nD * n, i});
    // split-K over (q,s): the output is only nD x n, the contraction n^2 long
    const i64 S = std::max<i64>(1, std::min<i64>(32, n2 / 2048));
    // chunks start on multiples of 32 columns (the tensor-core form loads 32-column tiles by TMA)
    const i64 kc = ((n2 + S - 1) / S + 31) / 32 * 32;
    const i64 Pt = T.alloc(S * (i64)outs.size() * P.nD * n);
    Step g = mkstep(STEP_GEMM, "three-external forward");
    for (size_t o = 0; o < outs.size(); ++o)
      for (i64 sidx = 0; sidx < S; ++sidx) {
        const i64 k0 = sidx * kc, kl = std::min(kc, n2 - k0);
        if (kl <= 0) continue;
        GemmProblem gp{BUF_T0, Pt + ((i64)o * S + sidx) * P.nD * n, n, P.nD, n, 0.0, (i64)g.gs.size(), 0};
        g.gs.push_back(GemmSeg{BUF_D, BUF_V, k0, n2, outs[o].second * n * n2 + k0, n2, kl, 0, 1, 1.0});
        gp.seg_end = (i64)g.gs.size();
        g.gp.push_back(gp);
      }
    P.sigma_steps.push_back(std::move(g));
    Step red = mkstep(STEP_AXPY, "three-external split-k sum");
    for (size_t o = 0; o < outs.size(); ++o) {
      AxpyTarget tg{BUF_T0, outs[o].first, P.nD * n, (i64)red.as.size(), 0};
      for (i64 sidx = 0; sidx < S; ++sidx)
        if (sidx * kc < n2) red.as.push_back(AxpySource{BUF_T0, Pt + ((i64)o * S + sidx) * P.nD * n, 1.0, -1, 0});
      tg.src_end = (i64)red.as.size();
      red.at.push_back(tg);
    }
    zero_step(P.sigma_steps, BUF_T0, Y, nint * P.nD * n, "three-external zero");
    P.sigma_steps.push_back(std::move(red));
    P.flops_total += 2.0 * P.nD * n * n2 * (double)outs.size();
    Step& sc = step(P.sigma_steps, STEP_AXPY, "three-external scatter");
    std::map<i64, std::vector<const T3*>> by_mu;
    for (auto& t : t3) by_mu[t.mu_row].push_back(&t);
    for (auto& kv : by_mu) {
      AxpyTarget tg{BUF_S, kv.first, n, (i64)sc.as.size(), 0};
      for (auto* t : kv.second) sc.as.push_back(AxpySource{BUF_T0, Y + (t->i * P.nD + t->dkk) * n, t->a, -1, 0});
      tg.src_end = (i64)sc.as.size();
      sc.at.push_back(tg);
    }
    // reverse: U[i][dk][b] = sum a c_mu ; R[dk][(q,s)] += sum_i U[i][dk][b] V_i[b][(q,s)]
    const i64 U = T.alloc(nint * P.nD * n);
    zero_step(P.sigma_steps, BUF_T0, U, nint * P.nD * n, "three-external reverse zero");
    Step& ga = step(P.sigma_steps, STEP_AXPY, "three-external reverse gather");
    std::map<std::pair<i64, i64>, std::vector<const T3*>> by_idk;
    for (auto& t : t3) by_idk[{t.i, t.dkk}].push_back(&t);
    for (auto& kv : by_idk) {
      AxpyTarget tg{BUF_T0, U + (kv.first.first * P.nD + kv.first.second) * n, n, (i64)ga.as.size(), 0};
      for (auto* t : kv.second) ga.as.push_back(AxpySource{BUF_C, t->mu_row, t->a, -1, 0});
      tg.src_end = (i64)ga.as.size();
      ga.at.push_back(tg);
    }
    Step& gr = step(P.sigma_steps, STEP_GEMM, "three-external reverse");
    GemmProblem gp{BUF_R, 0, n2, P.nD, n2, 1.0, (i64)gr.gs.size(), 0};
    for (i64 i = 0; i < nint; ++i)
      if (used[i]) gr.gs.push_back(GemmSeg{BUF_T0, BUF_V, U + i * P.nD * n, n, i * n * n2, n2, n, 0, 0, 1.0});
    gp.seg_end = (i64)gr.gs.size();
    if (gp.seg_end > gp.seg_begin) gr.gp.push_back(gp);
    for (i64 i = 0; i < nint; ++i)
      if (used[i]) P.flops_total += 2.0 * P.nD * n * n2;
  }

  // ---- device steps for the one-external term (vectors ordered by dk)
  if (!t1.empty()) {
    std::vector<size_t> order(t1.size());
    for (size_t t = 0; t < t1.size(); ++t) order[t] = t;
    std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) { return t1[x].dkk < t1[y].dkk; });
    const i64 wbase = (i64)P.wv.size() / std::max<i64>(n, 1);
    {
      const size_t w0 = P.wv.size();
      P.wv.resize(w0 + order.size() * (size_t)n);
#pragma omp parallel for schedule(static)
      for (long long r = 0; r < (long long)order.size(); ++r)
        std::copy(t1[order[(size_t)r]].w.begin(), t1[order[(size_t)r]].w.end(), P.wv.begin() + (std::ptrdiff_t)(w0 + (size_t)r * n));
    }
    const i64 m = (i64)order.size();
    const i64 Z = T.alloc(m * n), Cg = T.alloc(m * n);
    zero_step(P.sigma_steps, BUF_T0, Cg, m * n, "one-external gather zero");
    Step g = mkstep(STEP_GEMM, "one-external forward");
    Step ga = mkstep(STEP_AXPY, "one-external reverse gather");
    Step gr = mkstep(STEP_GEMM, "one-external reverse");
    Step sc = mkstep(STEP_AXPY, "one-external scatter");
    size_t r = 0;
    while (r < order.size()) {
      size_t e = r;
      const i64 d = t1[order[r]].dkk;
      while (e < order.size() && t1[order[e]].dkk == d) ++e;
      const i64 cnt = (i64)(e - r);
      // Z[r:e] = W[r:e] (cnt x n) * D[d] (n x n)
      GemmProblem gp{BUF_T0, Z + (i64)r * n, n, cnt, n, 0.0, (i64)g.gs.size(), 0};
      g.gs.push_back(GemmSeg{BUF_WV, BUF_D, (wbase + (i64)r) * n, n, d * n2, n, n, 0, 0, 1.0});
      gp.seg_end = (i64)g.gs.size();
      g.gp.push_back(gp);
      // R[d] += W[r:e]^T (n x cnt) * Cg[r:e] (cnt x n)
      GemmProblem gq{BUF_R, d * n2, n, n, n, 1.0, (i64)gr.gs.size(), 0};
      gr.gs.push_back(GemmSeg{BUF_WV, BUF_T0, (wbase + (i64)r) * n, n, Cg + (i64)r * n, n, cnt, 1, 0, 1.0});
      gq.seg_end = (i64)gr.gs.size();
      gr.gp.push_back(gq);
      P.flops_total += 4.0 * cnt * n * n;
      r = e;
    }
    for (size_t t = 0; t < order.size(); ++t) {
      AxpyTarget tg{BUF_T0, Cg + (i64)t * n, n, (i64)ga.as.size(), 0};
      ga.as.push_back(AxpySource{BUF_C, t1[order[t]].mu_row, 1.0, -1, 0});
      tg.src_end = (i64)ga.as.size();
      ga.at.push_back(tg);
    }
    std::map<i64, std::vector<i64>> by_mu;
    for (size_t t = 0; t < order.size(); ++t) by_mu[t1[order[t]].mu_row].push_back((i64)t);
    for (auto& kv : by_mu) {
      AxpyTarget tg{BUF_S, kv.first, n, (i64)sc.as.size(), 0};
      for (i64 t : kv.second) sc.as.push_back(AxpySource{BUF_T0, Z + t * n, 1.0, -1, 0});
      tg.src_end = (i64)sc.as.size();
      sc.at.push_back(tg);
    }
    P.sigma_steps.push_back(std::move(g));
    P.sigma_steps.push_back(std::move(ga));
    P.sigma_steps.push_back(std::move(gr));
    P.sigma_steps.push_back(std::move(sc));
  }
}

// ---------------------------------------------------------------------------
// DV: sigma_v += a <K^{ij}, D>; R += a c_v K^{ij}.  ops e_{iq,js}, i <= j.
void Builder::dv() {
  struct TV {
    i64 v_csf, pq, dkk;
    double a;
  };
  std::vector<TV> tv;
  for (size_t hs = 0; hs < sp.paths[2].size(); ++hs) {
    const Head& S = sp.paths[2][hs];
    if (!S.kept || nD(S) == 0) continue;
    const i64 nS = nD(S);
    for (i64 i = 0; i < nint; ++i)
      for (i64 j = i; j < nint; ++j) {
        std::vector<int8_t> o(S.occ.begin(), S.occ.end());
        o[i] += 1;
        o[j] += 1;
        if (o[i] > 2 || o[j] > 2) continue;
        const Head* V = find(0, o);
        if (!V || V->nsf == 0) continue;
        std::vector<double> a((size_t)V->nsf * nS, 0.0);
        if (S.off >= 0) {  // source (e1,e0): unit (i e0|j e1)
          auto m = M(cfgV(*V), cfgD(S, e1, e0), Op{(int)i, e0, (int)j, e1});
          const double div = (i == j) ? 2.0 : 1.0;
          for (i64 kt = 0; kt < V->nsf; ++kt)
            for (i64 ks = 0; ks < S.nsf; ++ks) a[kt * nS + ks] = m[kt * S.nsf + ks] / div;
        } else {  // source (e0,e0)
          auto m = M(cfgV(*V), cfgD(S, e0, e0), Op{(int)i, e0, (int)j, e0});
          const double f = (i == j) ? 0.5 / kSqrt2 : 1.0 / kSqrt2;
          for (i64 kt = 0; kt < V->nsf; ++kt)
            for (i64 ks = 0; ks < S.nsf_aa; ++ks) a[kt * nS + ks] = m[kt * S.nsf_aa + ks] * f;
        }
        for (i64 kt = 0; kt < V->nsf; ++kt)
          for (i64 ks = 0; ks < nS; ++ks)
            if (std::fabs(a[kt * nS + ks]) > kTiny) tv.push_back(TV{V->off + kt, i * nint + j, dk(S, ks), a[kt * nS + ks]});
      }
  }
  if (tv.empty()) return;
  const i64 nk = nint * nint;
  const i64 F2 = T.alloc(nk * P.nD), G2 = T.alloc(nk * P.nD);
  zero_step(P.sigma_steps, BUF_T0, F2, nk * P.nD, "dv forward zero");
  {  // F2 (nk x nD) = Kbank (nk x n^2) * D^T, split over the n^2 contraction
    const i64 S = std::max<i64>(1, std::min<i64>(64, n2 / 1024));
    // chunks start on multiples of 32 columns (the tensor-core form loads 32-column tiles by TMA)
    const i64 kc = ((n2 + S - 1) / S + 31) / 32 * 32;
    const i64 Pt = T.alloc(S * nk * P.nD);
    Step& g = step(P.sigma_steps, STEP_GEMM, "dv forward");
    for (i64 sidx = 0; sidx < S; ++sidx) {
      const i64 k0 = sidx * kc, kl = std::min(kc, n2 - k0);
      if (kl <= 0) continue;
      GemmProblem gp{BUF_T0, Pt + sidx * nk * P.nD, P.nD, nk, P.nD, 0.0, (i64)g.gs.size(), 0};
      g.gs.push_back(GemmSeg{BUF_JK, BUF_D, offK + k0, n2, k0, n2, kl, 0, 1, 1.0});
      gp.seg_end = (i64)g.gs.size();
      g.gp.push_back(gp);
    }
    Step& red = step(P.sigma_steps, STEP_AXPY, "dv split-k sum");
    AxpyTarget tg{BUF_T0, F2, nk * P.nD, 0, 0};
    for (i64 sidx = 0; sidx < S; ++sidx)
      if (sidx * kc < n2) red.as.push_back(AxpySource{BUF_T0, Pt + sidx * nk * P.nD, 1.0, -1, 0});
    tg.src_end = (i64)red.as.size();
    red.at.push_back(tg);
    P.flops_total += 2.0 * nk * P.nD * n2;
  }
  Step& sc = step(P.sigma_steps, STEP_AXPY, "dv scatter");
  std::map<i64, std::vector<const TV*>> by_v;
  for (auto& t : tv) by_v[t.v_csf].push_back(&t);
  for (auto& kv : by_v) {
    AxpyTarget tg{BUF_S, kv.first, 1, (i64)sc.as.size(), 0};
    for (auto* t : kv.second) sc.as.push_back(AxpySource{BUF_T0, F2 + t->pq * P.nD + t->dkk, t->a, -1, 0});
    tg.src_end = (i64)sc.as.size();
    sc.at.push_back(tg);
  }
  zero_step(P.sigma_steps, BUF_T0, G2, nk * P.nD, "dv reverse zero");
  Step& ga = step(P.sigma_steps, STEP_AXPY, "dv reverse gather");
  std::map<std::pair<i64, i64>, std::vector<const TV*>> by_g;
  for (auto& t : tv) by_g[{t.pq, t.dkk}].push_back(&t);
  for (auto& kv : by_g) {
    AxpyTarget tg{BUF_T0, G2 + kv.first.first * P.nD + kv.first.second, 1, (i64)ga.as.size(), 0};
    for (auto* t : kv.second) ga.as.push_back(AxpySource{BUF_C, t->v_csf, t->a, -1, 0});
    tg.src_end = (i64)ga.as.size();
    ga.at.push_back(tg);
  }
  Step& gr = step(P.sigma_steps, STEP_GEMM, "dv reverse");
  {  // R (nD x n^2) += G2^T (nD x nk) * Kbank (nk x n^2)
    GemmProblem gp{BUF_R, 0, n2, P.nD, n2, 1.0, (i64)gr.gs.size(), 0};
    gr.gs.push_back(GemmSeg{BUF_T0, BUF_JK, G2, P.nD, offK, n2, nk, 1, 0, 1.0});
    gp.seg_end = (i64)gr.gs.size();
    gr.gp.push_back(gp);
    P.flops_total += 2.0 * nk * P.nD * n2;
  }
}

// ---------------------------------------------------------------------------
// SS: sigma_mu'[k'] += a X c_mu[k] with X in {J_ij, K_ji, combined same-head}.
void Builder::ss() {
  Step& fcomb = step(P.init_steps, STEP_AXPY, "ss same-head operators");
  struct TS {
    i64 tgt_row, src_row;
    int xbuf;
    i64 xoff;
    double a;
  };
  std::vector<TS> ts;
  for (size_t hs = 0; hs < sp.paths[1].size(); ++hs) {
    const Head& S = sp.paths[1][hs];
    if (!has(S)) continue;
    const i64 nS = S.nsf;
    auto al = [&](const Head& Tg, Op o) {
      return M(cfgS(Tg, e0), cfgS(S, e1), o);  // predicted 1
    };
    {  // same head
      std::vector<std::vector<std::pair<i64, double>>> comb((size_t)nS * nS);
      auto add = [&](const std::vector<double>& a, i64 xoff) {
        for (size_t t = 0; t < a.size(); ++t)
          if (std::fabs(a[t]) > kTiny) comb[t].push_back({xoff, a[t]});
      };
      add(al(S, Op{e0, e1, -1, -1}), offH);
      for (i64 i = 0; i < nint; ++i) {
        if (S.occ[i] == 0) continue;
        add(al(S, Op{e0, e1, (int)i, (int)i}), Jof(i, i));
        add(al(S, Op{e0, (int)i, (int)i, e1}), Kof(i, i));
      }
      for (i64 kt = 0; kt < nS; ++kt)
        for (i64 ks = 0; ks < nS; ++ks) {
          auto& c = comb[kt * nS + ks];
          if (c.empty()) continue;
          AxpyTarget tg{BUF_F, nF * n2, n2, (i64)fcomb.as.size(), 0};
          for (auto& pr : c) fcomb.as.push_back(AxpySource{BUF_JK, pr.first, pr.second, -1, 0});
          tg.src_end = (i64)fcomb.as.size();
          fcomb.at.push_back(tg);
          ts.push_back(TS{S.off + kt * n, S.off + ks * n, BUF_F, nF * n2, 1.0});
          if (kt == ks) fdiag[{1, (i64)hs, kt}] = nF * n2;
          ++nF;
        }
    }
    for (i64 j = 0; j < nint; ++j) {
      if (S.occ[j] == 0) continue;
      for (i64 i = 0; i < nint; ++i) {
        if (i == j || S.occ[i] == 2) continue;
        std::vector<int8_t> o(S.occ.begin(), S.occ.end());
        o[j] -= 1;
        o[i] += 1;
        const Head* Tg = find(1, o);
        if (!Tg || !has(*Tg)) continue;
        auto aJ = al(*Tg, Op{e0, e1, (int)i, (int)j});
        auto aK = al(*Tg, Op{e0, (int)j, (int)i, e1});
        for (i64 kt = 0; kt < Tg->nsf; ++kt)
          for (i64 ks = 0; ks < nS; ++ks) {
            const double vj = aJ[kt * nS + ks], vk = aK[kt * nS + ks];
            if (std::fabs(vj) > kTiny) ts.push_back(TS{Tg->off + kt * n, S.off + ks * n, BUF_JK, Jof(i, j), vj});
            if (std::fabs(vk) > kTiny) ts.push_back(TS{Tg->off + kt * n, S.off + ks * n, BUF_JK, Kof(j, i), vk});
          }
      }
    }
  }
  if (ts.empty()) return;
  // group by operator: Y[rows] = Cg[rows] * X^T
  std::vector<size_t> order(ts.size());
  for (size_t t = 0; t < ts.size(); ++t) order[t] = t;
  std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
    return std::make_pair(ts[x].xbuf, ts[x].xoff) < std::make_pair(ts[y].xbuf, ts[y].xoff);
  });
  const i64 m = (i64)ts.size();
  const i64 Cg = T.alloc(m * n), Yr = T.alloc(m * n);
  zero_step(P.sigma_steps, BUF_T0, Cg, m * n, "ss gather zero");
  Step ga = mkstep(STEP_AXPY, "ss gather");
  Step g = mkstep(STEP_GEMM, "ss two-external");
  Step sc = mkstep(STEP_AXPY, "ss scatter");
  for (i64 r = 0; r < m; ++r) {
    AxpyTarget tg{BUF_T0, Cg + r * n, n, (i64)ga.as.size(), 0};
    ga.as.push_back(AxpySource{BUF_C, ts[order[r]].src_row, 1.0, -1, 0});
    tg.src_end = (i64)ga.as.size();
    ga.at.push_back(tg);
  }
  i64 r = 0;
  while (r < m) {
    i64 e = r;
    const auto key = std::make_pair(ts[order[r]].xbuf, ts[order[r]].xoff);
    while (e < m && std::make_pair(ts[order[e]].xbuf, ts[order[e]].xoff) == key) ++e;
    GemmProblem gp{BUF_T0, Yr + r * n, n, e - r, n, 0.0, (i64)g.gs.size(), 0};
    g.gs.push_back(GemmSeg{BUF_T0, key.first, Cg + r * n, n, key.second, n, n, 0, 1, 1.0});
    gp.seg_end = (i64)g.gs.size();
    g.gp.push_back(gp);
    P.flops_total += 2.0 * (e - r) * n * n;
    r = e;
  }
  std::map<i64, std::vector<i64>> by_t;
  for (i64 q = 0; q < m; ++q) by_t[ts[order[q]].tgt_row].push_back(q);
  for (auto& kv : by_t) {
    AxpyTarget tg{BUF_S, kv.first, n, (i64)sc.as.size(), 0};
    for (i64 q : kv.second) sc.as.push_back(AxpySource{BUF_T0, Yr + q * n, ts[order[q]].a, -1, 0});
    tg.src_end = (i64)sc.as.size();
    sc.at.push_back(tg);
  }
  P.sigma_steps.push_back(std::move(ga));
  P.sigma_steps.push_back(std::move(g));
  P.sigma_steps.push_back(std::move(sc));
}

// ---------------------------------------------------------------------------
// SV: sigma_mu[k'] += c_v[k] w ; sigma_v[k] += <w, c_mu[k']>.
// ops e_{xi,jk} = a+_x a+_j a_k a_i with (xi|jk), and E_xi with h_xi.
void Builder::sv() {
  // (mu row, v csf) -> w.  Two passes over the valence heads (in parallel, each head owning the keys of its
  // own CSFs): the first records every coupling (key, coefficient, integral vector) in loop order, the keys
  // are then placed in (mu row, v csf) order, and the second accumulates each head's couplings in the same
  // order directly into the W-vector array (no per-row buffers to copy).
  struct SvOp {
    std::pair<i64, i64> key;
    double a;
    const double* vec;  // nullptr: the one-electron column h(nint + x, hi) scaled by hs
    double hs;
    i64 hi;
  };
  const size_t nV = sp.paths[0].size();
  std::vector<std::vector<SvOp>> vops(nV);
  std::vector<std::vector<std::pair<i64, i64>>> vkeys(nV);  // each head's keys, sorted
  std::vector<std::unique_ptr<CouplingEngine>> engines((size_t)omp_get_max_threads());
  for (auto& e : engines) e = std::make_unique<CouplingEngine>(tables);
  // per thread: the expansion of each N-1 head (with the external electron), looked up once
  std::vector<std::vector<const CsfExpansion*>> hexp1((size_t)omp_get_max_threads(),
                                                      std::vector<const CsfExpansion*>(sp.paths[1].size(), nullptr));
#pragma omp parallel for schedule(dynamic, 4)
  for (long long hvl = 0; hvl < (long long)nV; ++hvl) {
    CouplingEngine& E = *engines[(size_t)omp_get_thread_num()];  // per-thread expansion cache
    const Head& V = sp.paths[0][(size_t)hvl];
    if (!has(V)) continue;
    const CsfExpansion& eV = E.expand(cfgV(V));
    auto& hx = hexp1[(size_t)omp_get_thread_num()];
    auto& ops = vops[(size_t)hvl];
    std::vector<double> m;
    auto add = [&](const Head* Mu, Op o, const double* vec, double hval_scale, i64 hi) {
      const size_t mi = (size_t)(Mu->lex - 1);
      if (!hx[mi]) hx[mi] = &E.expand(cfgS(*Mu, e0));
      E.matrix(*hx[mi], eV, o, m);  // predicted 1
      for (i64 kt = 0; kt < Mu->nsf; ++kt)
        for (i64 ks = 0; ks < V.nsf; ++ks) {
          const double a = m[kt * V.nsf + ks];
          if (std::fabs(a) <= kTiny) continue;
          ops.push_back(SvOp{{Mu->off + kt * n, V.off + ks}, a, vec, hval_scale, hi});
        }
    };
    // one working occupation, changed in place (no allocation per candidate)
    std::vector<int8_t> o(V.occ.begin(), V.occ.end());
    for (i64 i = 0; i < nint; ++i) {
      if (V.occ[i] == 0) continue;
      o[i] -= 1;
      if (const Head* Mu = find(1, o); Mu && has(*Mu)) add(Mu, Op{e0, (int)i, -1, -1}, nullptr, 1.0, i);
      for (i64 k = 0; k < nint; ++k) {
        if (o[k] == 0) continue;
        o[k] -= 1;
        for (i64 j = 0; j < nint; ++j) {
          if (o[j] == 2) continue;
          o[j] += 1;
          const Head* Mu = find(1, o);
          if (Mu && has(*Mu)) add(Mu, Op{e0, (int)i, (int)j, (int)k}, I.i3(i, j, k), 0.0, 0);  // (xi|jk) = I3[i][j][k][x]
          o[j] -= 1;
        }
        o[k] += 1;
      }
      o[i] += 1;
    }
    auto& ks = vkeys[(size_t)hvl];
    ks.reserve(ops.size());
    for (const auto& op : ops) ks.push_back(op.key);
    std::sort(ks.begin(), ks.end());
    ks.erase(std::unique(ks.begin(), ks.end()), ks.end());
  }
  // every key in (mu row, v csf) order; a row's place is its rank. The N-1 heads' rows are disjoint ranges
  // in lexical order, so the keys go into one bucket per N-1 head, each sorted on its own.
  const size_t nM = sp.paths[1].size();
  std::vector<i64> m_begin(nM, -1);
  for (size_t mi = 0; mi < nM; ++mi)
    if (has(sp.paths[1][mi])) m_begin[mi] = sp.paths[1][mi].off;
  std::vector<std::pair<i64, size_t>> starts;  // (first row, head) of the N-1 heads with CSFs, by row
  for (size_t mi = 0; mi < nM; ++mi)
    if (m_begin[mi] >= 0) starts.push_back({m_begin[mi], mi});
  std::sort(starts.begin(), starts.end());
  std::vector<std::vector<std::pair<std::pair<i64, i64>, i64>>> bucket(starts.size());
  for (size_t v = 0; v < nV; ++v)
    for (const auto& k : vkeys[v]) {
      const auto it = std::upper_bound(starts.begin(), starts.end(), std::make_pair(k.first, (size_t)-1));
      bucket[(size_t)(it - starts.begin()) - 1].push_back({k, (i64)v});
    }
#pragma omp parallel for schedule(dynamic, 8)
  for (long long b = 0; b < (long long)bucket.size(); ++b) std::sort(bucket[(size_t)b].begin(), bucket[(size_t)b].end());
  std::vector<std::pair<std::pair<i64, i64>, i64>> keys;  // (key, owning head)
  {
    size_t total = 0;
    for (const auto& b : bucket) total += b.size();
    keys.reserve(total);
    for (auto& b : bucket) {
      keys.insert(keys.end(), b.begin(), b.end());
      std::vector<std::pair<std::pair<i64, i64>, i64>>().swap(b);
    }
  }
  if (keys.empty()) return;
  const i64 wbase = (i64)P.wv.size() / std::max<i64>(n, 1);
  std::vector<std::pair<std::pair<i64, i64>, i64>> rows;
  rows.reserve(keys.size());
  std::vector<std::vector<i64>> vrow(nV);  // per head: the W rows of its sorted keys
  for (size_t v = 0; v < nV; ++v) vrow[v].reserve(vkeys[v].size());
  for (const auto& kv : keys) {
    vrow[(size_t)kv.second].push_back(wbase + (i64)rows.size());  // keys of one head arrive in its sorted order
    rows.push_back({kv.first, wbase + (i64)rows.size()});
  }
  // one allocation (hundreds of MB at the kernel-scale size), each head's rows zeroed and accumulated by
  // the thread that owns the head
  const size_t w0 = P.wv.size();
  P.wv.resize(w0 + keys.size() * (size_t)n);
  double* W = P.wv.data();
#pragma omp parallel for schedule(dynamic, 4)
  for (long long hvl = 0; hvl < (long long)nV; ++hvl) {
    const auto& ks = vkeys[(size_t)hvl];
    const auto& rs = vrow[(size_t)hvl];
    for (i64 r : rs) std::fill(W + (size_t)r * n, W + (size_t)(r + 1) * n, 0.0);
    for (const auto& op : vops[(size_t)hvl]) {
      const size_t at = (size_t)(std::lower_bound(ks.begin(), ks.end(), op.key) - ks.begin());
      double* w = W + (size_t)rs[at] * n;
      if (op.vec) {
        for (i64 x = 0; x < n; ++x) w[x] += op.a * op.vec[x];
      } else {
        for (i64 x = 0; x < n; ++x) w[x] += op.a * op.hs * I.h1(nint + x, op.hi);
      }
    }
    std::vector<SvOp>().swap(vops[(size_t)hvl]);
  }
  Step& fw = step(P.sigma_steps, STEP_AXPY, "sv forward");
  // rows are in (mu row, v csf) order: one target per run of equal mu rows
  fw.as.reserve(fw.as.size() + rows.size());
  for (size_t t = 0; t < rows.size();) {
    AxpyTarget tg{BUF_S, rows[t].first.first, n, (i64)fw.as.size(), 0};
    const i64 mu = rows[t].first.first;
    for (; t < rows.size() && rows[t].first.first == mu; ++t)
      fw.as.push_back(AxpySource{BUF_WV, rows[t].second * n, 1.0, BUF_C, rows[t].first.second});
    tg.src_end = (i64)fw.as.size();
    fw.at.push_back(tg);
  }
  Step& rv = step(P.sigma_steps, STEP_DOT, "sv reverse");
  // by v csf, the rows of one v in (mu row) order
  std::vector<size_t> byv(rows.size());
  for (size_t t = 0; t < rows.size(); ++t) byv[t] = t;
  std::stable_sort(byv.begin(), byv.end(),
                   [&](size_t x, size_t y) { return rows[x].first.second < rows[y].first.second; });
  rv.ds.reserve(rv.ds.size() + rows.size());
  for (size_t k = 0; k < byv.size();) {
    const i64 v = rows[byv[k]].first.second;
    DotTarget tg{BUF_S, v, (i64)rv.ds.size(), 0};
    for (; k < byv.size() && rows[byv[k]].first.second == v; ++k) {
      const size_t t = byv[k];
      rv.ds.push_back(DotSource{BUF_WV, BUF_C, rows[t].second * n, rows[t].first.first, n, 1.0});
    }
    tg.src_end = (i64)rv.ds.size();
    rv.dt.push_back(tg);
  }
  P.flops_total += 4.0 * n * rows.size();
}

// ---------------------------------------------------------------------------
// All-external term in packed integral form:
//   singlet: [s_aa; s_ab] += W+ [c_aa; c_ab]    triplet: s_ab += W- c_ab
// W+ rows/cols: n diagonal pairs then the n(n-1)/2 pairs a>b in the
// reference's order idx = a(a-1)/2 + b (scepmaker_mod.f90:60-90).
void Builder::allext() {
  const i64 np = n + nab, nm = nab;
  P.np = np;
  P.nm = nm;
  std::vector<std::pair<const DHeadInfo*, i64>> sing, trip;
  for (auto& d : P.dheads)
    for (i64 k = 0; k < d.nD; ++k) (k < d.nsing ? sing : trip).push_back({&d, k});
  P.n_sing = (i64)sing.size();
  P.n_trip = (i64)trip.size();
  const i64 Us = T.alloc(std::max<i64>(1, P.n_sing) * np), Ys = T.alloc(std::max<i64>(1, P.n_sing) * np);
  const i64 Ut = T.alloc(std::max<i64>(1, P.n_trip) * nm), Yt = T.alloc(std::max<i64>(1, P.n_trip) * nm);
  P.allext_us = Us;
  P.allext_ys = Ys;
  P.allext_ut = Ut;
  P.allext_yt = Yt;
  zero_step(P.sigma_steps, BUF_T0, Us, P.n_sing * np, "all-external gather zero");
  zero_step(P.sigma_steps, BUF_T0, Ut, P.n_trip * nm, "all-external gather zero");
  Step& ga = step(P.sigma_steps, STEP_AXPY, "all-external gather");
  auto gather = [&](i64 dst, i64 len, i64 src) {
    AxpyTarget tg{BUF_T0, dst, len, (i64)ga.as.size(), 0};
    ga.as.push_back(AxpySource{BUF_C, src, 1.0, -1, 0});
    tg.src_end = (i64)ga.as.size();
    ga.at.push_back(tg);
  };
  for (i64 r = 0; r < P.n_sing; ++r) {
    const DHeadInfo& d = *sing[r].first;
    const i64 k = sing[r].second;
    if (k < d.nsf_aa) gather(Us + r * np, n, d.off_aa + k * n);
    if (k < d.nsf_ab && nab > 0) gather(Us + r * np + n, nab, d.off_ab + k * nab);
  }
  for (i64 r = 0; r < P.n_trip; ++r) {
    const DHeadInfo& d = *trip[r].first;
    const i64 k = trip[r].second;
    if (nab > 0) gather(Ut + r * nm, nab, d.off_ab + k * nab);
  }
  // FP64 form: Y = U W with the contraction split in S slices (the product has
  // few output rows and a very long k); the slices are summed in order.  S gives
  // the row-panel kernel (128 columns per block) about eight blocks per SM; the
  // slices start on multiples of 32 columns of U (16-byte aligned operands).
  const i64 offWm = np * np;
  const i64 col_blocks = std::max<i64>(1, (np + 127) / 128);
  const i64 S = std::max<i64>(1, std::min<i64>({16, np / 512, (148 * 8 + col_blocks - 1) / col_blocks}));
  const i64 Ps = T.alloc(S * std::max<i64>(1, P.n_sing) * np), Pt = T.alloc(S * std::max<i64>(1, P.n_trip) * nm);
  Step& g = step(P.sigma_steps, STEP_GEMM, "all-external");
  auto add_split = [&](i64 m, i64 dim, i64 U, i64 woff, i64 part) {
    const i64 kc = ((dim + S - 1) / S + 31) / 32 * 32;
    for (i64 sidx = 0; sidx < S; ++sidx) {
      const i64 k0 = sidx * kc, kl = std::min(kc, dim - k0);
      if (kl <= 0) continue;
      GemmProblem gp{BUF_T0, part + sidx * m * dim, dim, m, dim, 0.0, (i64)g.gs.size(), 0};
      g.gs.push_back(GemmSeg{BUF_T0, BUF_W, U + k0, dim, woff + k0 * dim, dim, kl, 0, 0, 1.0});
      gp.seg_end = (i64)g.gs.size();
      g.gp.push_back(gp);
    }
  };
  if (P.n_sing > 0) add_split(P.n_sing, np, Us, 0, Ps);
  if (P.n_trip > 0 && nm > 0) add_split(P.n_trip, nm, Ut, offWm, Pt);
  Step red = mkstep(STEP_AXPY, "all-external split-k sum");
  auto add_sum = [&](i64 m, i64 dim, i64 Y, i64 part) {
    const i64 kc = ((dim + S - 1) / S + 31) / 32 * 32;
    AxpyTarget tg{BUF_T0, Y, m * dim, (i64)red.as.size(), 0};
    for (i64 sidx = 0; sidx < S; ++sidx)
      if (sidx * kc < dim) red.as.push_back(AxpySource{BUF_T0, part + sidx * m * dim, 1.0, -1, 0});
    tg.src_end = (i64)red.as.size();
    red.at.push_back(tg);
  };
  zero_step(P.sigma_steps, BUF_T0, Ys, std::max<i64>(1, P.n_sing) * np, "all-external zero");
  zero_step(P.sigma_steps, BUF_T0, Yt, std::max<i64>(1, P.n_trip) * nm, "all-external zero");
  if (P.n_sing > 0) add_sum(P.n_sing, np, Ys, Ps);
  if (P.n_trip > 0 && nm > 0) add_sum(P.n_trip, nm, Yt, Pt);
  P.sigma_steps.push_back(std::move(red));
  P.flops_allext = 2.0 * (double)np * np * P.n_sing + 2.0 * (double)nm * nm * P.n_trip;
  P.bytes_allext = 8.0 * ((double)np * np + (P.n_trip > 0 ? (double)nm * nm : 0.0)) +
                   16.0 * ((double)P.n_sing * np + (double)P.n_trip * nm);
  P.flops_total += P.flops_allext;
  Step& sc = step(P.sigma_steps, STEP_AXPY, "all-external scatter");
  auto scatter = [&](i64 dst, i64 len, i64 src) {
    AxpyTarget tg{BUF_S, dst, len, (i64)sc.as.size(), 0};
    sc.as.push_back(AxpySource{BUF_T0, src, 1.0, -1, 0});
    tg.src_end = (i64)sc.as.size();
    sc.at.push_back(tg);
  };
  for (i64 r = 0; r < P.n_sing; ++r) {
    const DHeadInfo& d = *sing[r].first;
    const i64 k = sing[r].second;
    if (k < d.nsf_aa) scatter(d.off_aa + k * n, n, Ys + r * np);
    if (k < d.nsf_ab && nab > 0) scatter(d.off_ab + k * nab, nab, Ys + r * np + n);
  }
  for (i64 r = 0; r < P.n_trip; ++r) {
    const DHeadInfo& d = *trip[r].first;
    if (nab > 0) scatter(d.off_ab + trip[r].second * nab, nab, Yt + r * nm);
  }
  P.buf_size[BUF_W] = np * np + nm * nm;
  P.buf_size[BUF_X] = (n * (n + 1) / 2) * (n * (n + 1) / 2);
}

// ---------------------------------------------------------------------------
void Builder::build_diag() {
  auto beta = [&](int block, i64 p, i64 k) {
    auto it = beta_diag.find({block, p, k});
    return it == beta_diag.end() ? 0.0 : it->second;
  };
  auto foff = [&](int kind, i64 p, i64 k) -> i64 {
    auto it = fdiag.find({kind, p, k});
    return it == fdiag.end() ? -1 : it->second;
  };
  for (size_t p = 0; p < sp.paths[0].size(); ++p) {
    const Head& h = sp.paths[0][p];
    if (!has(h)) continue;
    for (i64 k = 0; k < h.nsf; ++k) P.diag.push_back(DiagEntry{h.off + k, 1, 0, beta(0, (i64)p, k), -1, 1});
  }
  for (size_t p = 0; p < sp.paths[1].size(); ++p) {
    const Head& h = sp.paths[1][p];
    if (!has(h)) continue;
    for (i64 k = 0; k < h.nsf; ++k) P.diag.push_back(DiagEntry{h.off + k * n, n, 1, beta(1, (i64)p, k), foff(1, (i64)p, k), 1});
  }
  for (size_t p = 0; p < sp.paths[2].size(); ++p) {
    const Head& h = sp.paths[2][p];
    if (!h.kept || nDh[p] == 0) continue;
    if (h.off_aa >= 0)
      for (i64 k = 0; k < h.nsf_aa; ++k)
        P.diag.push_back(DiagEntry{h.off_aa + k * n, n, 2, beta(2, (i64)p, k), foff(2, (i64)p, k), 1});
    if (h.off >= 0 && nab > 0)
      for (i64 k = 0; k < h.nsf; ++k)
        P.diag.push_back(DiagEntry{h.off + k * nab, nab, 3, beta(3, (i64)p, k), foff(2, (i64)p, k),
                                   P.dk_sign[dk0[p] + k] > 0 ? 1 : 0});
  }
}

void Builder::init_steps() {
  // gather L rows into dense blocks
  Step& ga = step(P.init_steps, STEP_AXPY, "gather cholesky rows");
  auto g1 = [&](int dst, i64 doff, i64 len, i64 pair) {
    AxpyTarget tg{dst, doff, len, (i64)ga.as.size(), 0};
    ga.as.push_back(AxpySource{BUF_L, pair * N, 1.0, -1, 0});
    tg.src_end = (i64)ga.as.size();
    ga.at.push_back(tg);
  };
  for (i64 i = 0; i < nint; ++i)
    for (i64 q = 0; q < n; ++q) g1(BUF_LE, (i * n + q) * N, N, Ints::pair(i, nint + q));
  for (i64 a = 0; a < n; ++a)
    for (i64 b = 0; b < n; ++b) g1(BUF_LV, (a * n + b) * N, N, Ints::pair(nint + a, nint + b));
  for (i64 i = 0; i < nint; ++i)
    for (i64 j = 0; j < nint; ++j) g1(BUF_LI, (i * nint + j) * N, N, Ints::pair(i, j));
  // packed external pairs (a>=b): rows a(a+1)/2 + b, contiguous in L for each a
  const i64 npk = n * (n + 1) / 2;
  Scratch Ti;
  const i64 Lpk_off = with_allext ? Ti.alloc(npk * N) : 0;
  if (with_allext)
    for (i64 a = 0; a < n; ++a) g1(BUF_T0, Lpk_off + (a * (a + 1) / 2) * N, (a + 1) * N, Ints::pair(nint + a, nint));
  init_scratch = Ti.top;
  Step& gb = step(P.init_steps, STEP_GEMM, "integral banks");
  {  // J[(ij)][(ab)] = LI (nint^2 x N) * LV^T
    GemmProblem gp{BUF_JK, offJ, n2, nint * nint, n2, 0.0, (i64)gb.gs.size(), 0};
    gb.gs.push_back(GemmSeg{BUF_LI, BUF_LV, 0, N, 0, N, N, 0, 1, 1.0});
    gp.seg_end = (i64)gb.gs.size();
    gb.gp.push_back(gp);
  }
  for (i64 p = 0; p < nint; ++p)
    for (i64 q = 0; q < nint; ++q) {  // K[p][q] = LE[p] * LE[q]^T
      GemmProblem gp{BUF_JK, Kof(p, q), n, n, n, 0.0, (i64)gb.gs.size(), 0};
      gb.gs.push_back(GemmSeg{BUF_LE, BUF_LE, p * n * N, N, q * n * N, N, N, 0, 1, 1.0});
      gp.seg_end = (i64)gb.gs.size();
      gb.gp.push_back(gp);
    }
  for (i64 i = 0; i < nint; ++i)  // V_i[b][q][s] = (iq|bs) = LE[i] (n x N) * LV[b rows]^T (N x n)
    for (i64 b = 0; b < n; ++b) {
      GemmProblem gp{BUF_V, (i * n + b) * n2, n, n, n, 0.0, (i64)gb.gs.size(), 0};
      gb.gs.push_back(GemmSeg{BUF_LE, BUF_LV, i * n * N, N, b * n * N, N, N, 0, 1, 1.0});
      gp.seg_end = (i64)gb.gs.size();
      gb.gp.push_back(gp);
    }
  if (!with_allext) return;
  {  // X = Lpk Lpk^T
    GemmProblem gp{BUF_X, 0, npk, npk, npk, 0.0, (i64)gb.gs.size(), 0};
    gb.gs.push_back(GemmSeg{BUF_T0, BUF_T0, Lpk_off, N, Lpk_off, N, N, 0, 1, 1.0});
    gp.seg_end = (i64)gb.gs.size();
    gb.gp.push_back(gp);
  }
  step(P.init_steps, STEP_WBUILD, "all-external operators");
}

void Builder::run() {
  const Deck& d = sp.deck;
  nint = sp.n_int;
  n = sp.n_ext;
  n2 = n * n;
  nab = n * (n - 1) / 2;
  N = op.nchol;
  for (const auto& dm : sp.domains)
    if ((i64)dm.size() != n)
      throw Error(3, "the dense-operator plan is built on the non-local space (domains are mapped onto it)");
  if (nint + 3 > 64) throw Error(3, "at most 61 internal orbitals are supported");
  P.nint = nint;
  P.n = n;
  P.nchol = N;
  P.total_csfs = sp.total_csfs;
  P.npair_all = d.num_orbitals * (d.num_orbitals + 1) / 2;
  P.buf_size.assign(NUM_BUFS, 0);
  build_spin_tables((int)sp.open_shells, (int)d.spin_mult, tables);
  eng = std::make_unique<CouplingEngine>(tables);
  e0 = (int)nint;
  e1 = (int)nint + 1;
  e2 = (int)nint + 2;
  I.norb = d.num_orbitals;
  I.nint = nint;
  I.n = n;
  I.N = N;
  I.h = op.h;
  I.L = op.chol;
  // TCI_PLAN_TIMING=1 prints the wall time of every phase of the plan build to stderr
  const bool timing = std::getenv("TCI_PLAN_TIMING") != nullptr;
  auto t_last = std::chrono::steady_clock::now();
  auto tick = [&](const char* what) {
    if (!timing) return;
    const auto t = std::chrono::steady_clock::now();
    std::fprintf(stderr, "plan %-16s %8.3f s\n", what, std::chrono::duration<double>(t - t_last).count());
    t_last = t;
  };
  tick("spin tables");
  I.build();
  tick("integrals");
  offJ = 0;
  offK = nint * nint * n2;
  offH = 2 * nint * nint * n2;
  setup_heads();
  init_steps();
  tick("heads, init");
  zero_step(P.sigma_steps, BUF_R, 0, P.nD * n2, "zero accumulators");
  step(P.sigma_steps, STEP_UNPACK, "unpack");
  if (with_allext) allext();
  tick("all-external");
  dd_x();
  tick("dd");
  ds();
  tick("ds");
  dv();
  tick("dv");
  ss();
  tick("ss");
  sv();
  tick("sv");
  if (wv_done) wv_done(P);
  internal_blocks();
  tick("internal");
  step(P.sigma_steps, STEP_PACK, "pack");
  build_diag();
  tick("diagonal");
  P.h_vv.assign(n2, 0.0);
  for (i64 a = 0; a < n; ++a)
    for (i64 b = 0; b < n; ++b) P.h_vv[a * n + b] = I.h1(nint + a, nint + b);
  P.buf_size[BUF_C] = sp.total_csfs;
  P.buf_size[BUF_S] = sp.total_csfs;
  P.buf_size[BUF_D] = std::max<i64>(1, P.nD * n2);
  P.buf_size[BUF_R] = std::max<i64>(1, P.nD * n2);
  P.buf_size[BUF_T0] = std::max<i64>(T.top, init_scratch);
  P.buf_size[BUF_JK] = (2 * nint * nint + 1) * n2;
  P.buf_size[BUF_V] = nint * n * n2;
  P.buf_size[BUF_F] = std::max<i64>(1, nF * n2);
  P.buf_size[BUF_WV] = std::max<i64>(1, (i64)P.wv.size());
  P.buf_size[BUF_L] = P.npair_all * N;
  P.buf_size[BUF_LE] = nint * n * N;
  P.buf_size[BUF_LV] = n2 * N;
  P.buf_size[BUF_LI] = nint * nint * N;
}

// The operator part of the plan alone: the set-up steps that depend on the orbital counts and the Cholesky
// rank only (gather cholesky rows, integral banks, all-external operators), with the sizes of the buffers they
// use, exactly as run() makes them (run() emits them first).  The device can build the integral banks from
// these while the host builds the sigma tables.
void Builder::run_operator_part() {
  const Deck& d = sp.deck;
  nint = sp.n_int;
  n = sp.n_ext;
  n2 = n * n;
  nab = n * (n - 1) / 2;
  N = op.nchol;
  P.nint = nint;
  P.n = n;
  P.nchol = N;
  P.total_csfs = sp.total_csfs;
  P.npair_all = d.num_orbitals * (d.num_orbitals + 1) / 2;
  P.buf_size.assign(NUM_BUFS, 0);
  offJ = 0;
  offK = nint * nint * n2;
  offH = 2 * nint * nint * n2;
  init_steps();
  if (with_allext) {
    P.np = n + nab;
    P.nm = nab;
    P.buf_size[BUF_W] = P.np * P.np + P.nm * P.nm;
    P.buf_size[BUF_X] = (n * (n + 1) / 2) * (n * (n + 1) / 2);
  }
  P.buf_size[BUF_T0] = init_scratch;
  P.buf_size[BUF_JK] = (2 * nint * nint + 1) * n2;
  P.buf_size[BUF_V] = nint * n * n2;
  P.buf_size[BUF_L] = P.npair_all * N;
  P.buf_size[BUF_LE] = nint * n * N;
  P.buf_size[BUF_LV] = n2 * N;
  P.buf_size[BUF_LI] = nint * nint * N;
}

}  // namespace

void build_plan_operator_part(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext) {
  plan = Plan();
  Builder b(sp, op, plan);
  b.with_allext = with_allext;
  b.run_operator_part();
}

void build_plan(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext) {
  build_plan(sp, op, plan, with_allext, nullptr);
}

void build_plan(const CsfSpace& sp, const Operator& op, Plan& plan, bool with_allext,
                const std::function<void(const Plan&)>& wv_done) {
  plan = Plan();
  Builder b(sp, op, plan);
  b.with_allext = with_allext;
  b.wv_done = wv_done;
  b.run();
}

}  // namespace tci
