// Spin functions of the SGGA: branching diagram and SFT graph restated from
// tiger_fortran/spin_mod.f90:99-522, plus their explicit expansion over spin
// strings (genealogical Clebsch-Gordan coupling along the same paths).
//
// Arc convention (spin_mod.f90:282-330): vertex open_shells is the start of
// every path (multiplicity 1), vertex 0 its end (multiplicity spinM), and arc i
// joins vertex i to vertex i-1.  Open shell i of a configuration (ascending
// orbital order) sits on arc i, so the highest orbital is coupled first.  A
// configuration with s < open_shells open shells uses the first fsn(s) SFT
// functions, whose arcs s+1..open_shells are ground-level singlet pairs
// (spin_mod.f90:1004-1014).
#include "tci_host.h"

#include <cmath>
#include <tuple>
#include <memory>
#include <mutex>

namespace tci {

void build_spin_tables(int open_shells, int spinM, SpinTables& t) {
  t = SpinTables();
  t.open_shells = open_shells;
  t.spin_mult = spinM;
  // fsn for this multiplicity (graph_mod.f90:436-489) with wrong parities zeroed
  std::vector<i64> fsn3(open_shells + 3, 0);
  t.fsn_all.assign(open_shells + 1, 0);
  t.fsn_all[0] = (spinM == 1) ? 1 : 0;
  fsn3[0] = 1;
  fsn3[1] = 1;
  for (int i = 1; i <= open_shells; ++i) {
    for (int j = (i % 2) + 1; j <= i + 1; j += 2) {
      i64 nf = (j == 1) ? fsn3[2] : (j == i + 1 ? 1 : fsn3[j - 1] + fsn3[j + 1]);
      fsn3[j] = nf;
    }
    bool ok = (i >= spinM - 1) && ((i - (spinM - 1)) % 2 == 0);
    t.fsn_all[i] = ok ? (spinM < (int)fsn3.size() ? fsn3[spinM] : 0) : 0;
  }
  const int nsf = (int)t.fsn_all[open_shells];
  t.nsf_max = nsf;
  if (open_shells < 1 || nsf < 1) {
    t.spin_matrix.assign((open_shells + 1) * std::max(nsf, 1), 1);
    if (nsf >= 1) t.spin_matrix[0] = spinM;
    return;
  }

  // ---- branching_diagram (spin_mod.f90:99-228) -------------------------
  const int up = (open_shells + spinM - 1) / 2;
  const int down = open_shells - up;
  std::vector<i64> br((up + 2) * (down + 3), 0);
  auto B = [&](int a, int b) -> i64& { return br[a * (down + 3) + b]; };
  {
    int a = up, b = down + 1, amax = up, bmax = down + 1;
    for (;;) {
      if (a == up && b == down + 1) B(a, b) = 1;
      else if (b == down + 1 || a + 1 == b) B(a, b) = B(a + 1, b);
      else if (b == 1 && a < up) B(a, b) = B(a + 1, b) + B(a, b + 1);
      else if (a == up) B(a, b) = 1;
      else B(a, b) = B(a + 1, b) + B(a, b + 1);
      if (a == 1 && b == 1) break;
      if (b == down + 1 || a + 1 == b || a == b) {
        if (bmax > 1 && amax == up) {
          bmax -= 1;
          a = amax;
          b = bmax;
          continue;
        } else if (bmax == 1 && amax <= up) {
          amax -= 1;
          a = amax;
          b = bmax;
          continue;
        }
      } else {
        a -= 1;
        b += 1;
        continue;
      }
      throw Error(4, "branching diagram walk failed");
    }
  }

  // ---- sft_graph (spin_mod.f90:232-522) ---------------------------------
  t.sft.assign((open_shells - 1) * nsf, 0);
  t.spin_matrix.assign((open_shells + 1) * nsf, 0);
  auto SFT = [&](int i, int w) -> int& { return t.sft[(i - 1) * nsf + (w - 1)]; };
  auto SM = [&](int v, int w) -> int& { return t.spin_matrix[v * nsf + (w - 1)]; };
  std::vector<char> path(open_shells + 1, 0);
  std::vector<int> pa(open_shells + 1, 0), pb(open_shells + 1, 0);
  path[open_shells] = 1;
  int shells = open_shells - 1;
  pa[open_shells] = 0;
  pb[open_shells] = 1;
  pa[shells] = 1;
  pb[shells] = 1;
  i64 weight = 1;
  for (int w = 1; w <= nsf; ++w) {
    SM(0, w) = spinM;
    SM(open_shells, w) = 1;
  }
  for (;;) {
    for (;;) {  // get_spin_function
      if (pa[shells] == up && pb[shells] == down + 1 && shells == 0) break;
      if (pb[shells] == down + 1 || pb[shells] == pa[shells] + 1) {
        path[shells] = 1;
        shells -= 1;
        pa[shells] = pa[shells + 1] + 1;
        pb[shells] = pb[shells + 1];
      } else {
        path[shells] = 0;
        shells -= 1;
        pa[shells] = pa[shells + 1];
        pb[shells] = pb[shells + 1] + 1;
      }
    }
    if (weight < 1 || weight > nsf) throw Error(4, "SFT weight out of range");
    const int W = (int)weight;
    for (int i = open_shells - 1; i >= 1; --i) {
      const bool prev = path[i + 1], cur = path[i];
      const int a = pa[i], b = pb[i];
      SM(i, W) = prev ? SM(i + 1, W) + 1 : SM(i + 1, W) - 1;
      if (prev && !cur && a == b) {
        SFT(i, W) = W;
      } else if (prev && !cur) {
        i64 nw = weight - B(a - 1, b + 1);
        if (b + 2 <= down + 1) nw += B(a - 1, b + 2);
        SFT(i, W) = (int)nw;
      } else if (!prev && cur) {
        i64 nw = weight + B(a, b);
        if (b <= a && b < down + 1) nw -= B(a, b + 1);
        SFT(i, W) = (int)(-nw);
      } else {
        SFT(i, W) = 0;
      }
    }
    shells = 1;
    bool done = false;
    for (;;) {  // look_for_branch_point
      if (shells == open_shells) {
        done = true;
        break;
      } else if (!path[shells] && pa[shells] < up) {
        path[shells] = 1;
        weight += B(pa[shells], pb[shells] + 1);
        shells -= 1;
        pa[shells] = pa[shells + 1] + 1;
        pb[shells] = pb[shells + 1];
        break;
      } else {
        shells += 1;
        if (pb[shells] < down + 1 && pb[shells] <= pa[shells] && path[shells])
          weight -= B(pa[shells], pb[shells] + 1);
      }
    }
    if (done) break;
  }
}

namespace {

// <S, M - m; 1/2, m | S', M>, S' = S +- 1/2 (Condon-Shortley phases).
double cg_half(double S, double Sp, double M, double m) {
  const double den = 2.0 * S + 1.0;
  if (Sp > S) {
    return (m > 0) ? std::sqrt((S + M + 0.5) / den) : std::sqrt((S - M + 0.5) / den);
  }
  return (m > 0) ? -std::sqrt((S - M + 0.5) / den) : std::sqrt((S + M + 0.5) / den);
}

}  // namespace

const SpinBasis& spin_basis(const SpinTables& t, int s) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, int>, std::unique_ptr<SpinBasis>> cache;
  std::lock_guard<std::mutex> lk(mu);
  auto key = std::make_tuple(t.open_shells, t.spin_mult, s);
  auto it = cache.find(key);
  if (it != cache.end()) return *it->second;
  auto sb = std::make_unique<SpinBasis>();
  sb->s = s;
  const int spinM = t.spin_mult;
  const int nsf = (s <= t.open_shells && s >= 0) ? (int)t.fsn_all[s] : 0;
  sb->nsf = nsf;
  if (s > 30) throw Error(4, "spin basis too large");
  const double S_fin = 0.5 * (spinM - 1);
  // strings with M_S = S: number of beta spins = (s - (spinM-1)) / 2
  if (nsf > 0) {
    const int nbeta = (s - (spinM - 1)) / 2;
    for (uint32_t x = 0; x < (1u << s); ++x)
      if (__builtin_popcount(x) == nbeta) sb->strings.push_back(x);
    for (size_t i = 0; i < sb->strings.size(); ++i) sb->index[sb->strings[i]] = (int)i;
    sb->coeff.assign(sb->strings.size() * nsf, 0.0);
    for (int f = 0; f < nsf; ++f) {
      // padding check: arcs s+1..open_shells must be ground-level pairs
      if (t.mult(s, f) != 1) throw Error(4, "spin function ordering does not pad low open-shell counts");
      for (size_t r = 0; r < sb->strings.size(); ++r) {
        const uint32_t x = sb->strings[r];
        double c = 1.0, M = 0.0, S = 0.0;
        for (int arc = s; arc >= 1; --arc) {  // highest arc coupled first
          const double m = ((x >> (arc - 1)) & 1u) ? -0.5 : 0.5;
          const double Sp = 0.5 * (t.mult(arc - 1, f) - 1);
          const double Mp = M + m;
          if (std::fabs(Mp) > Sp + 1e-9) {
            c = 0.0;
            break;
          }
          c *= cg_half(S, Sp, Mp, m);
          S = Sp;
          M = Mp;
        }
        if (std::fabs(M - S_fin) > 1e-9) c = 0.0;
        sb->coeff[r * nsf + f] = c;
      }
    }
  }
  auto& ref = *sb;
  cache[key] = std::move(sb);
  return ref;
}

}  // namespace tci
