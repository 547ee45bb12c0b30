#include "coupling.h"

#include <memory>

namespace tci {

namespace {

inline int popc(Det x) {
  return __builtin_popcountll((uint64_t)x) + __builtin_popcountll((uint64_t)(x >> 64));
}
inline Det bit(int x) { return ((Det)1) << x; }
// phase of moving an operator past the occupied spin orbitals below x
inline int below(Det d, int x) { return popc(d & (bit(x) - 1)); }

// apply a_x; returns false if empty
inline bool annihilate(Det& d, int x, double& ph) {
  if (!(d & bit(x))) return false;
  if (below(d, x) & 1) ph = -ph;
  d &= ~bit(x);
  return true;
}
inline bool create(Det& d, int x, double& ph) {
  if (d & bit(x)) return false;
  if (below(d, x) & 1) ph = -ph;
  d |= bit(x);
  return true;
}

}  // namespace

const CsfExpansion& CouplingEngine::expand(const Config& c) {
  {
    std::lock_guard<std::mutex> lk(mu_);
    auto it = cache_.find(c.occ);
    if (it != cache_.end()) return *it->second;
  }
  auto e = std::make_unique<CsfExpansion>();
  const int n = (int)c.occ.size();
  if (2 * n > 128) throw Error(4, "coupling engine supports at most 64 orbitals");
  for (int p = 0; p < n; ++p)
    if (c.occ[p] == 1) e->open.push_back(p);
  e->s = (int)e->open.size();
  e->basis = &spin_basis(tables_, e->s);
  e->nsf = e->basis->nsf;
  e->sign = ((e->s * (e->s - 1) / 2) % 2) ? -1.0 : 1.0;
  Det closed = 0;
  for (int p = 0; p < n; ++p)
    if (c.occ[p] == 2) closed |= bit(2 * p) | bit(2 * p + 1);
  for (size_t r = 0; r < e->basis->strings.size(); ++r) {
    const uint32_t x = e->basis->strings[r];
    Det d = closed;
    for (int i = 0; i < e->s; ++i) d |= bit(2 * e->open[i] + (int)((x >> i) & 1u));
    e->dets.push_back(d);
    e->index[d] = (int)r;
  }
  std::lock_guard<std::mutex> lk(mu_);
  auto it = cache_.find(c.occ);
  if (it != cache_.end()) return *it->second;  // another thread expanded it meanwhile
  auto& ref = *e;
  cache_[c.occ] = std::move(e);
  return ref;
}

void CouplingEngine::matrix(const Config& L, const Config& R, const Op& op, std::vector<double>& out) {
  matrix(expand(L), expand(R), op, out);
}

void CouplingEngine::matrix(const CsfExpansion& eL, const CsfExpansion& eR, const Op& op, std::vector<double>& out) {
  out.assign((size_t)eL.nsf * eR.nsf, 0.0);
  accumulate(eL, eR, op, 1.0, out);
}

void CouplingEngine::accumulate(const Config& L, const Config& R, const Op& op, double coef,
                                std::vector<double>& out) {
  accumulate(expand(L), expand(R), op, coef, out);
}

void CouplingEngine::accumulate(const CsfExpansion& eL, const CsfExpansion& eR, const Op& op, double coef,
                                std::vector<double>& out) {
  const int nL = eL.nsf, nR = eR.nsf;
  if (nL == 0 || nR == 0) return;
  const double* TL = eL.basis->coeff.data();
  const double* TR = eR.basis->coeff.data();
  const bool two = op.r >= 0;
  std::vector<double> tmp(nL);
  for (size_t rr = 0; rr < eR.dets.size(); ++rr) {
    const double* thR = TR + rr * nR;
    bool any = false;
    for (int k = 0; k < nR; ++k) any |= (thR[k] != 0.0);
    if (!any) continue;
    for (int sg = 0; sg < 2; ++sg) {
      for (int tg = 0; tg < (two ? 2 : 1); ++tg) {
        Det d = eR.dets[rr];
        double ph = 1.0;
        if (two) {
          // a+_{p sg} a+_{r tg} a_{s tg} a_{q sg}
          if (!annihilate(d, 2 * op.q + sg, ph)) continue;
          if (!annihilate(d, 2 * op.s + tg, ph)) continue;
          if (!create(d, 2 * op.r + tg, ph)) continue;
          if (!create(d, 2 * op.p + sg, ph)) continue;
        } else {
          if (!annihilate(d, 2 * op.q + sg, ph)) continue;
          if (!create(d, 2 * op.p + sg, ph)) continue;
        }
        auto jt = eL.index.find(d);
        if (jt == eL.index.end()) continue;
        const double* thL = TL + (size_t)jt->second * nL;
        const double f = coef * ph * eL.sign * eR.sign;
        for (int kl = 0; kl < nL; ++kl) {
          if (thL[kl] == 0.0) continue;
          const double a = f * thL[kl];
          double* row = out.data() + (size_t)kl * nR;
          for (int k = 0; k < nR; ++k) row[k] += a * thR[k];
        }
      }
    }
  }
}

}  // namespace tci
