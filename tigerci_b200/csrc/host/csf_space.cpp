// CSF space: distinct-row table, internal tree search and CI-vector index
// vectors, restated from TigerCI's graph module.
//   graph_border ............ tiger_fortran/graph_mod.f90:101-259
//   drt_maker ............... tiger_fortran/graph_mod.f90:263-378
//   get_fsn ................. tiger_fortran/graph_mod.f90:381-491
//   tree_search_internal .... tiger_fortran/graph_mod.f90:572-1003
//   index_vector_internal ... tiger_fortran/graph_mod.f90:1007-1589
//   vertex/belong/add0/1/2 .. tiger_fortran/ci_utilities_mod.f90:49-124
//   allowed virtual lists ... tiger_fortran/allowed_virtuals_mod.f90:163-339
#include "tci_host.h"

#include <algorithm>
#include <cstdlib>

namespace tci {

bool CsfSpace::belong(i64 i, i64 j) const {
  if (i < 0 || j < 0 || i > deck.num_orbitals) return false;
  return j >= left_border[i] && j <= right_border[i];
}

namespace {

struct Graph {
  CsfSpace& g;
  explicit Graph(CsfSpace& s) : g(s) {}
  i64& Y0(i64 v) { return g.y0[v]; }
  bool add0(i64 i, i64 j) const {
    if (i < 0 || j < 0) return false;
    return g.belong(i, j) && g.y0[g.vertex(i, j)] > 0;
  }
  bool add1(i64 i, i64 j) const {
    if (i < 0 || j < 0) return false;
    return g.belong(i, j) && g.y1[g.vertex(i, j)] >= 0;
  }
  bool add2(i64 i, i64 j) const {
    if (i < 0 || j < 0) return false;
    return g.belong(i, j) && g.y2[g.vertex(i, j)] >= 0;
  }
};

// Number of spin functions per open-shell count (graph_mod.f90:381-491).  The
// entries of the wrong parity keep the stale value of the previous level, as
// in the reference; they are only read through the shellU sentinel logic.
void get_fsn(const Deck& d, i64& open_shells, std::vector<i64>& fsn) {
  open_shells = 0;
  const i64 nint = d.num_internal();
  for (i64 r = 0; r < d.num_ref; ++r) {
    i64 ref_singles = 0;
    for (i64 j = d.num_inactive; j < d.num_inactive + d.num_active; ++j)
      if (d.refs[r * nint + j] == 1) ++ref_singles;
    open_shells = std::max(ref_singles + 4, open_shells);
  }
  if (d.num_elec < open_shells) open_shells = d.num_elec;
  if (d.spin_mult % 2 == 0 && open_shells % 2 == 0) open_shells += 1;
  if (open_shells > kFsnSize) throw Error(3, "too many open shells");
  fsn.assign(kFsnSize + 1, 0);
  std::vector<i64> fsn3(open_shells + 3, 0);
  fsn[0] = 1;
  fsn3[0] = 1;
  fsn3[1] = 1;
  for (i64 i = 1; i <= open_shells; ++i) {
    for (i64 j = (i % 2) + 1; j <= i + 1; j += 2) {
      i64 nf;
      if (j == 1) nf = fsn3[2];
      else if (j == i + 1) nf = 1;
      else nf = fsn3[j - 1] + fsn3[j + 1];
      fsn3[j] = nf;
    }
    fsn[i] = (d.spin_mult < (i64)fsn3.size()) ? fsn3[d.spin_mult] : 0;
  }
}

}  // namespace

void build_csf_space(const Deck& d, const DomainSpec& dom, CsfSpace& g) {
  g = CsfSpace();
  g.deck = d;
  const i64 norb = d.num_orbitals, nint = d.num_internal(), nel = d.num_elec;
  g.n_int = nint;
  g.n_ext = norb - nint;
  if (nint < 2 || g.n_ext < 1) throw Error(3, "need >=2 internal and >=1 external orbitals");
  if ((i64)d.refs.size() != d.num_ref * nint) throw Error(3, "reference occupations size mismatch");
  if (d.spin_mult < 1 || d.num_elec < 2) throw Error(3, "bad spin multiplicity or electron count");
  for (i64 r = 0; r < d.num_ref; ++r) {
    i64 ne = 0;
    for (i64 j = 0; j < nint; ++j) ne += d.refs[r * nint + j];
    if (ne != nel) throw Error(3, "reference electron count differs from NUMBER OF ELECTRONS");
  }

  get_fsn(d, g.open_shells, g.fsn);

  // ---- graph_border (graph_mod.f90:101-259) ------------------------------
  const i64 min_singles = d.spin_mult - 1;
  const i64 right_singles = min_singles;
  const i64 right_doubly = (nel - right_singles) / 2;
  const i64 left_singles = std::max<i64>(0, min_singles);
  const i64 left_doubly = (nel - left_singles) / 2;
  const i64 left_unocc = norb - left_singles - left_doubly;
  g.left_border.assign(norb + 1, 0);
  g.right_border.assign(norb + 1, 0);
  for (i64 i = 1; i <= norb; ++i) {
    i64 add = (i <= left_unocc) ? 0 : (i <= left_unocc + left_singles ? 1 : 2);
    g.left_border[i] = (i == 1) ? add : g.left_border[i - 1] + add;
  }
  for (i64 i = 1; i <= norb; ++i) {
    i64 add = (i <= right_doubly) ? 2 : (i <= right_doubly + right_singles ? 1 : 0);
    g.right_border[i] = (i == 1) ? add : g.right_border[i - 1] + add;
  }
  auto ref_occ = [&](i64 orb1, i64 r) -> i64 {  // 1-based orbital, padded with zeros
    return orb1 <= nint ? d.refs[r * nint + orb1 - 1] : 0;
  };
  std::vector<i64> temp(d.num_ref);
  for (i64 r = 0; r < d.num_ref; ++r) temp[r] = ref_occ(1, r);
  for (i64 i = 2; i <= norb; ++i) {
    i64 min_elec = 2 * i, max_elec = 0;
    for (i64 r = 0; r < d.num_ref; ++r) {
      i64 cum = temp[r] + ref_occ(i, r);
      max_elec = std::max(max_elec, cum);
      min_elec = std::min(min_elec, cum);
      temp[r] = cum;
    }
    g.left_border[i] = std::max(min_elec - kExcitationLevel, g.left_border[i]);
    g.right_border[i] = std::min(max_elec + kExcitationLevel, g.right_border[i]);
  }
  g.auxiliary.assign(norb + 1, 0);
  g.num_vert = 1;
  g.auxiliary[0] = 1;
  for (i64 i = 1; i <= norb; ++i) {
    g.auxiliary[i] = g.num_vert + 1 - g.left_border[i];
    g.num_vert = g.right_border[i] + g.auxiliary[i];
  }

  // ---- drt_maker (graph_mod.f90:263-378) ---------------------------------
  g.y0.assign(g.num_vert + 2, 0);
  g.y1.assign(g.num_vert + 2, 0);
  g.y2.assign(g.num_vert + 2, 0);
  Graph G(g);
  g.y0[1] = g.belong(1, 0) ? 1 : -1;
  g.y1[1] = g.belong(1, 1) ? 0 : -1;
  g.y2[1] = g.belong(1, 2) ? 0 : -1;
  for (i64 i = 1; i <= norb; ++i) {
    for (i64 j = g.right_border[i]; j >= g.left_border[i]; --j) {
      const i64 va = g.vertex(i - 1, j);
      const i64 v = g.vertex(i, j);
      i64 w = 0;
      if (G.add0(i - 1, j)) w += std::llabs(g.y0[va]);
      if (G.add1(i - 1, j - 1)) w += std::llabs(g.y0[va - 1]);
      if (G.add2(i - 1, j - 2)) w += std::llabs(g.y0[va - 2]);
      g.y0[v] = g.belong(i + 1, j) ? w : -w;
      w = 0;
      if (!g.belong(i + 1, j + 1)) w = -1;
      else if (G.add0(i, j + 1)) w = std::llabs(g.y0[g.vertex(i, j + 1)]);
      g.y1[v] = w;
      w = 0;
      if (!g.belong(i + 1, j + 2)) {
        w = -1;
      } else {
        if (G.add1(i, j + 1)) w += std::llabs(g.y0[g.vertex(i, j + 1)]);
        if (G.add0(i, j + 2)) w += std::llabs(g.y0[g.vertex(i, j + 2)]);
      }
      g.y2[v] = w;
    }
  }
  g.total_configurations = std::llabs(g.y0[g.num_vert]);

  // ---- tree_search_internal (graph_mod.f90:572-1003) ---------------------
  for (int k = 0; k < 3; ++k) {
    if (!g.belong(nint, nel - k)) continue;
    i64 np = std::llabs(g.y0[g.vertex(nint, nel - k)]);
    g.paths[k].assign(np, Head());
    for (i64 p = 0; p < np; ++p) {
      g.paths[k][p].lex = p + 1;
      g.paths[k][p].kind = k;
    }
  }
  std::vector<int> singles_v[3];  // raw singles or kill per path (iv0/iv1/iv2 before indexing)
  std::vector<char> visited[3];
  for (int k = 0; k < 3; ++k) {
    singles_v[k].assign(g.paths[k].size(), 0);
    visited[k].assign(g.paths[k].size(), 0);
  }
  {
    std::vector<i64> change(norb + 1, 0), singles(nint + 1, 0), lex(nint + 1, 0);
    i64 vert = 1, orbital = 0, electrons = 0;
    change[0] = 2;
    lex[0] = 1;
    auto check_excitation = [&]() {
      i64 e = 0;
      for (i64 j = 0; j < nint; ++j) e += change[j];
      for (i64 r = 0; r < d.num_ref; ++r) {
        i64 diff = 0;
        for (i64 j = 0; j < nint; ++j) diff += std::llabs(change[j] - d.refs[r * nint + j]);
        diff += nel - e;
        if (diff <= 2 * kExcitationLevel) return true;
      }
      return false;
    };
    auto check_frozen = [&]() {
      for (i64 j = 0; j < d.num_frozen; ++j)
        if (change[j] != 2) return false;
      return true;
    };
    auto record = [&]() {
      int k = (int)(nel - electrons);
      if (k < 0 || k > 2) throw Error(4, "tree search left the internal/external border");
      i64 p = lex[orbital] - 1;
      Head& h = g.paths[k].at(p);
      h.singles = (int)singles[orbital];
      h.occ.assign(nint, 0);
      for (i64 j = 0; j < nint; ++j) h.occ[j] = (int8_t)change[j];
      visited[k][p] = 1;
      singles_v[k][p] = (check_excitation() && check_frozen()) ? (int)singles[orbital] : (int)kKillNumber;
    };
    for (;;) {
      i64 step = change[orbital];
      if (step == 2 || step == 1 || step == 0) {
        i64 arc = step == 2 ? g.y2[vert] : (step == 1 ? g.y1[vert] : g.y0[vert]);
        if (arc >= 0) {
          electrons += step;
          orbital += 1;
          vert = g.auxiliary[orbital] + electrons;
          singles[orbital] = singles[orbital - 1] + (step == 1 ? 1 : 0);
          lex[orbital] = lex[orbital - 1] + (step == 0 ? 0 : arc);
          if (orbital == nint) {
            record();
            orbital -= 1;
            change[orbital] -= 1;
            electrons -= step;
            vert = g.auxiliary[orbital] + electrons;
            continue;
          }
          change[orbital] = 2;
          continue;
        }
        if (step == 2) change[orbital] = 1;
        else if (step == 1) change[orbital] = 0;
        else change[orbital] = -1;
        continue;
      }
      // step == -1: ran out of steps at this level
      if (orbital != 0) {
        orbital -= 1;
        electrons -= change[orbital];
        change[orbital] -= 1;
        vert = g.auxiliary[orbital] + electrons;
      } else {
        break;
      }
    }
  }

  // ---- domains (allowed_virtuals_mod.f90:163-339) -------------------------
  auto add_domain = [&](std::vector<int> v) -> i64 {
    std::sort(v.begin(), v.end());
    for (size_t i = 0; i < g.domains.size(); ++i)
      if (g.domains[i] == v) return (i64)i;
    g.domains.push_back(v);
    return (i64)g.domains.size() - 1;
  };
  std::vector<int> all(g.n_ext);
  for (i64 a = 0; a < g.n_ext; ++a) all[a] = (int)a;
  for (int k = 1; k <= 2; ++k) {
    const auto& spec = (k == 1) ? dom.nm1 : dom.nm2;
    if (!spec.empty() && spec.size() != g.paths[k].size())
      throw Error(3, "domain list count differs from the number of internal paths");
    for (size_t p = 0; p < g.paths[k].size(); ++p) {
      if (spec.empty()) {
        g.paths[k][p].domain = add_domain(all);
      } else if (spec[p].size() == 1 && spec[p][0] < 0) {
        g.paths[k][p].domain = -1;
      } else {
        for (int a : spec[p])
          if (a < 0 || a >= g.n_ext) throw Error(3, "domain entry out of range");
        g.paths[k][p].domain = add_domain(spec[p]);
      }
    }
  }
  auto nvirt = [&](const Head& h) -> i64 {
    return h.domain < 0 ? 0 : (i64)g.domains[h.domain].size();
  };

  // ---- index_vector_internal (graph_mod.f90:1007-1589) -------------------
  std::vector<i64>& fsn = g.fsn;
  const i64 spinM = d.spin_mult, os = g.open_shells;
  const i64 shell1 = os % 2, shellU = shell1 + 1;
  std::vector<i64> tmp(std::max<i64>(kFsnSize, 2) + 3, 0);
  auto T = [&](i64 i) -> i64& { return tmp.at(i + 2); };  // allow index -2..

  // valence
  std::vector<i64> iv(g.paths[0].size());
  for (size_t p = 0; p < iv.size(); ++p) {
    i64 s = singles_v[0][p];
    if (s > kFsnSize) throw Error(3, "too many open shells in a valence path");
    if (s < spinM - 1 || s > os) s = shellU;
    iv[p] = s;
    T(s) += 1;
  }
  g.removed = T(shellU);
  i64 ncsf = 0;
  for (i64 i = spinM - 1; i <= os; i += 2) {
    ncsf += T(i) * fsn[i];
    if (T(i) > 0) g.cfg_count[0][(int)i] = T(i);
  }
  g.total_csfs = ncsf;
  g.num_valence = ncsf;
  T(shellU) = -1;
  fsn[shellU] = 0;
  ncsf = 1;
  for (i64 i = shell1; i <= os; i += 2) {
    i64 c = T(i);
    T(i) = ncsf;
    ncsf += c * fsn[i];
  }
  for (size_t p = 0; p < iv.size(); ++p) {
    i64 s = iv[p];
    Head& h = g.paths[0][p];
    if (s == shellU) {
      h.kept = false;
    } else {
      h.kept = true;
      h.off = T(s) - 1;
      h.nsf = (int)fsn[s];
      T(s) += fsn[s];
    }
  }

  // N-1
  std::fill(tmp.begin(), tmp.end(), 0);
  iv.assign(g.paths[1].size(), 0);
  for (size_t p = 0; p < iv.size(); ++p) {
    i64 s = singles_v[1][p];
    if (s + 1 > kFsnSize) throw Error(3, "too many open shells in an N-1 path");
    if (s + 1 < spinM - 1 || s + 1 > os) s = shellU - 1;
    iv[p] = s;
    T(s + 1) += nvirt(g.paths[1][p]);
  }
  g.removed += T(shellU);
  ncsf = 0;
  for (i64 i = spinM - 1; i <= os; i += 2) {
    ncsf += T(i) * fsn[i];
    if (T(i) > 0) g.cfg_count[1][(int)i] = T(i);
  }
  g.total_csfs += ncsf;
  T(shellU) = -1;
  fsn[shellU] = 0;
  i64 start = g.num_valence + 1;
  for (size_t p = 0; p < iv.size(); ++p) {
    i64 s = iv[p] + 1;
    Head& h = g.paths[1][p];
    if (s == shellU) {
      h.kept = false;
    } else {
      h.kept = true;
      h.off = start - 1;
      h.nsf = (int)fsn[s];
      start += fsn[s] * nvirt(h);
    }
  }
  g.num_nm1 = start - g.num_valence - 1;

  // N-2
  std::fill(tmp.begin(), tmp.end(), 0);
  std::vector<i64> iv2(g.paths[2].size()), iv3(g.paths[2].size());
  for (size_t p = 0; p < iv2.size(); ++p) {
    i64 s2 = singles_v[2][p], s3 = singles_v[2][p];
    if (s2 + 2 > kFsnSize || s3 > kFsnSize) throw Error(3, "too many open shells in an N-2 path");
    if (s2 + 2 < spinM - 1 || s2 + 2 > os) s2 = shellU - 2;
    i64 nv = nvirt(g.paths[2][p]);
    T(s2 + 2) += nv * (nv - 1) / 2;
    if (s3 < spinM - 1 || s3 > os) s3 = shellU;
    T(s3) += nv;
    iv2[p] = s2;
    iv3[p] = s3;
  }
  g.removed += T(shellU);
  ncsf = 0;
  for (i64 i = spinM - 1; i <= os; i += 2) {
    ncsf += T(i) * fsn[i];
    if (T(i) > 0) g.cfg_count[2][(int)i] = T(i);
  }
  g.total_csfs += ncsf;
  T(shellU) = -1;
  fsn[shellU] = 0;
  start = g.num_valence + g.num_nm1 + 1;
  for (size_t p = 0; p < iv2.size(); ++p) {
    Head& h = g.paths[2][p];
    i64 nv = nvirt(h);
    i64 s = iv3[p];
    if (s != shellU) {
      h.off_aa = start - 1;
      h.nsf_aa = (int)fsn[s];
      start += fsn[s] * nv;
    }
    s = iv2[p] + 2;
    if (s != shellU) {
      h.off = start - 1;
      h.nsf = (int)fsn[s];
      start += fsn[s] * (nv * (nv - 1) / 2);
    }
    h.kept = (h.off >= 0 || h.off_aa >= 0);
  }
  g.num_nm2 = start - g.num_valence - g.num_nm1 - 1;

  // final zeroing of the spin-function counts (graph_mod.f90:1545-1555)
  for (i64 i = 0; i <= spinM - 2 && i <= kFsnSize; ++i) fsn[i] = 0;
  for (i64 i = spinM; i <= os - 1; i += 2) fsn[i] = 0;
  for (i64 i = os + 1; i <= kFsnSize; ++i) fsn[i] = 0;
  // heads that were never reached by the tree search keep singles 0 like the
  // reference's zero-initialised index vectors; flag them so callers can tell
  for (int k = 0; k < 3; ++k)
    for (size_t p = 0; p < g.paths[k].size(); ++p)
      if (!visited[k][p]) g.paths[k][p].occ.assign(nint, -1);
}

}  // namespace tci
