// Host-only part of the C ABI (include/tigerci_sigma.h): error reporting, CSF
// space queries and plan construction / export.  No CUDA dependency.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <string>

#include "../../../include/tigerci_sigma.h"
#include "capi_internal.h"
#include "plan.h"

namespace tci {
thread_local std::string g_last_error;
void set_error(const std::string& m) { g_last_error = m; }
}  // namespace tci

using namespace tci;

struct tci_space {
  CsfSpace sp;
};
struct tci_plan {
  CsfSpace sp;
  Plan plan;
};

namespace tci {

int guard_status(const std::exception_ptr& ep) {
  try {
    std::rethrow_exception(ep);
  } catch (const Error& e) {
    set_error(e.what());
    return e.code;
  } catch (const std::bad_alloc&) {
    set_error("host allocation failed");
    return TCI_ERR_MEMORY;
  } catch (const std::exception& e) {
    set_error(e.what());
    return TCI_ERR_INTERNAL;
  } catch (...) {
    set_error("unknown failure");
    return TCI_ERR_INTERNAL;
  }
}

void deck_from_c(const tci_deck* d, Deck& out, DomainSpec& dom) {
  if (!d) throw Error(TCI_ERR_ARG, "deck is null");
  out.num_orbitals = d->num_orbitals;
  out.num_frozen = d->num_frozen;
  out.num_inactive = d->num_inactive;
  out.num_active = d->num_active;
  out.num_elec = d->num_elec;
  out.spin_mult = d->spin_mult;
  out.num_ref = d->num_ref;
  const i64 nint = out.num_internal();
  if (out.num_orbitals <= 0 || nint <= 0 || out.num_ref <= 0 || out.num_frozen < 0 ||
      out.num_frozen > out.num_inactive || nint >= out.num_orbitals)
    throw Error(TCI_ERR_INPUT, "inconsistent orbital counts in deck");
  if (!d->ref_occ) throw Error(TCI_ERR_ARG, "reference occupations are null");
  out.refs.resize(out.num_ref * nint);
  for (i64 i = 0; i < out.num_ref * nint; ++i) {
    const i64 v = d->ref_occ[i];
    if (v < 0 || v > 2) throw Error(TCI_ERR_INPUT, "reference occupation outside 0..2");
    out.refs[i] = (int)v;
  }
  auto csr = [&](const int64_t* ptr, const int64_t* idx, std::vector<std::vector<int>>& dst) {
    dst.clear();
    if (!ptr) return;
    if (!idx) throw Error(TCI_ERR_ARG, "domain index array is null");
    return;  // filled once the path counts are known (see expand_domains)
  };
  csr(d->nm1_domain_ptr, d->nm1_domain_idx, dom.nm1);
  csr(d->nm2_domain_ptr, d->nm2_domain_idx, dom.nm2);
}

void build_space_from_c(const tci_deck* d, CsfSpace& sp) {
  Deck deck;
  DomainSpec dom;
  deck_from_c(d, deck, dom);
  if (d->nm1_domain_ptr || d->nm2_domain_ptr) {
    // path counts are needed to read the CSR arrays: build once non-locally
    CsfSpace probe;
    build_csf_space(deck, DomainSpec(), probe);
    auto rd = [&](const int64_t* ptr, const int64_t* idx, size_t np, std::vector<std::vector<int>>& dst) {
      if (!ptr) return;
      dst.resize(np);
      for (size_t p = 0; p < np; ++p) {
        if (ptr[p + 1] < ptr[p]) throw Error(TCI_ERR_INPUT, "domain CSR pointers decrease");
        for (int64_t t = ptr[p]; t < ptr[p + 1]; ++t) dst[p].push_back((int)idx[t]);
      }
    };
    rd(d->nm1_domain_ptr, d->nm1_domain_idx, probe.paths[1].size(), dom.nm1);
    rd(d->nm2_domain_ptr, d->nm2_domain_idx, probe.paths[2].size(), dom.nm2);
  }
  build_csf_space(deck, dom, sp);
}

void operator_from_c(const tci_operator* op, const CsfSpace& sp, Operator& out) {
  if (!op || !op->h || !op->chol) throw Error(TCI_ERR_ARG, "operator or its arrays are null");
  if (op->nchol <= 0) throw Error(TCI_ERR_INPUT, "nchol must be positive");
  (void)sp;
  out.h = op->h;
  out.chol = op->chol;
  out.nchol = op->nchol;
  out.core_energy = op->core_energy;
}

}  // namespace tci

extern "C" {

int tci_last_error(char* buf, int64_t len) {
  if (!buf || len <= 0) return TCI_ERR_ARG;
  std::snprintf(buf, (size_t)len, "%s", g_last_error.c_str());
  return TCI_OK;
}

int tci_operator_from_records(int64_t num_orbitals, int64_t nchol, const int64_t* mo_ind_inv, const double* records,
                              int64_t n_records, double* chol_out) {
  if (num_orbitals <= 0 || nchol <= 0 || n_records < 0 || !mo_ind_inv || !chol_out || (n_records > 0 && !records)) {
    set_error("tci_operator_from_records: bad argument");
    return TCI_ERR_ARG;
  }
  const int64_t npair = num_orbitals * (num_orbitals + 1) / 2;
  for (int64_t pq = 0; pq < npair; ++pq)
    if (mo_ind_inv[pq] < 0 || mo_ind_inv[pq] > n_records) {
      set_error("mo_ind_inv entry " + std::to_string(pq) + " is outside 0.." + std::to_string(n_records));
      return TCI_ERR_INPUT;
    }
  for (int64_t pq = 0; pq < npair; ++pq) {
    double* dst = chol_out + pq * nchol;
    const int64_t r = mo_ind_inv[pq];
    if (r == 0)
      std::memset(dst, 0, sizeof(double) * (size_t)nchol);
    else
      std::memcpy(dst, records + (r - 1) * nchol, sizeof(double) * (size_t)nchol);
  }
  return TCI_OK;
}

int tci_space_create(const tci_deck* deck, tci_space** out) {
  if (!out) return TCI_ERR_ARG;
  *out = nullptr;
  try {
    auto* s = new tci_space();
    try {
      build_space_from_c(deck, s->sp);
    } catch (...) {
      delete s;
      throw;
    }
    *out = s;
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_space_counts(const tci_space* s, int64_t* out, int64_t len) {
  if (!s || !out || len < 12) return TCI_ERR_ARG;
  const CsfSpace& sp = s->sp;
  out[0] = sp.total_csfs;
  out[1] = sp.num_valence;
  out[2] = sp.num_nm1;
  out[3] = sp.num_nm2;
  out[4] = sp.total_configurations;
  out[5] = sp.removed;
  out[6] = sp.open_shells;
  out[7] = (int64_t)sp.paths[0].size();
  out[8] = (int64_t)sp.paths[1].size();
  out[9] = (int64_t)sp.paths[2].size();
  out[10] = sp.num_vert;
  out[11] = (int64_t)sp.domains.size();
  return TCI_OK;
}

int tci_space_index_vector(const tci_space* s, int64_t kind, int64_t* out, int64_t len) {
  if (!s || !out || kind < 0 || kind > 3) return TCI_ERR_ARG;
  const auto& P = s->sp.paths[kind == 3 ? 2 : kind];
  if (len != (int64_t)P.size()) {
    set_error("index vector length mismatch");
    return TCI_ERR_ARG;
  }
  for (size_t p = 0; p < P.size(); ++p) {
    const Head& h = P[p];
    i64 v = (kind == 3) ? h.off_aa : h.off;
    out[p] = v >= 0 ? v + 1 : kKillNumber;
  }
  return TCI_OK;
}

int tci_space_path(const tci_space* s, int64_t kind, int64_t lex, int64_t* occ, int64_t* info) {
  if (!s || kind < 0 || kind > 2 || !occ || !info) return TCI_ERR_ARG;
  const auto& P = s->sp.paths[kind];
  if (lex < 1 || lex > (int64_t)P.size()) return TCI_ERR_ARG;
  const Head& h = P[lex - 1];
  for (i64 j = 0; j < s->sp.n_int; ++j) occ[j] = h.occ.empty() ? -1 : h.occ[j];
  info[0] = h.lex;
  info[1] = h.singles;
  info[2] = h.kept ? 1 : 0;
  info[3] = h.nsf;
  info[4] = h.nsf_aa;
  info[5] = h.domain < 0 ? (kind == 0 ? 0 : 0) : (int64_t)s->sp.domains[h.domain].size();
  return TCI_OK;
}

int tci_acpf_gdiag(const tci_space* s, int64_t flag, double custom_g, double* g, int64_t* cls, int64_t n) {
  if (!s || !g || n != s->sp.total_csfs) return TCI_ERR_ARG;
  try {
    const CsfSpace& sp = s->sp;
    const Deck& d = sp.deck;
    // get_gvalues (gtimesc.f90:316-378)
    const double N = (double)(d.num_elec - 2 * d.num_frozen);
    double v[5];
    if (flag == 1) {
      v[0] = v[1] = 1.0;
      v[2] = v[3] = v[4] = 2.0 / N;
    } else if (flag == 2) {
      v[0] = v[1] = 1.0;
      v[2] = v[3] = (4.0 / N) * (1.0 - 1.0 / (2.0 * (N - 1.0)));
      v[4] = 2.0 / N;
    } else if (flag == 3) {
      v[0] = v[1] = 1.0;
      v[2] = v[3] = v[4] = (4.0 / N) * (1.0 - 1.0 / (2.0 * (N - 1.0)));
    } else if (flag == 4) {
      v[0] = v[1] = 1.0;
      v[2] = v[3] = custom_g;
      v[4] = 2.0 / N;
    } else if (flag == 9) {
      v[0] = v[1] = v[2] = v[3] = v[4] = 1.0;
    } else {
      throw Error(TCI_ERR_ARG, "unknown ACPF flag");
    }
    // build_g_diagonal (gtimesc.f90:106-201): N-1 CSFs g4, N-2 CSFs g5, valence CSFs by configuration
    std::vector<int64_t> c((size_t)n, 0);
    for (i64 i = sp.num_valence; i < sp.num_valence + sp.num_nm1; ++i) c[(size_t)i] = 4;
    for (i64 i = sp.num_valence + sp.num_nm1; i < n; ++i) c[(size_t)i] = 5;
    const i64 ni = d.num_internal();
    for (const Head& h : sp.paths[0]) {
      if (!h.kept || h.off < 0 || h.nsf <= 0) continue;
      i64 inact = 0;
      for (i64 j = 0; j < d.num_inactive; ++j) inact += h.occ[(size_t)j];
      int k = 3;  // an inactive hole (g_diag_no_external :262-272)
      if (inact == 2 * d.num_inactive) {
        bool ref = false;  // active occupations of a reference (:274-291)
        for (i64 r = 0; r < d.num_ref && !ref; ++r) {
          bool same = true;
          for (i64 j = d.num_inactive; j < ni; ++j) same = same && h.occ[(size_t)j] == d.refs[(size_t)(r * ni + j)];
          ref = same;
        }
        k = ref ? 1 : 2;
      }
      for (i64 t = 0; t < h.nsf; ++t) c[(size_t)(h.off + t)] = k;
    }
    for (i64 i = 0; i < n; ++i) {
      if (c[(size_t)i] == 0) throw Error(TCI_ERR_INTERNAL, "a CSF without an ACPF class");
      g[i] = v[c[(size_t)i] - 1];
      if (cls) cls[i] = c[(size_t)i];
    }
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_local_allext_records(const tci_deck* deck, int64_t* out, int64_t cap, int64_t* count) {
  try {
    if (!deck || !count || !(deck->nm1_domain_ptr || deck->nm2_domain_ptr)) return TCI_ERR_ARG;
    tci::LocalSetup ls;
    build_space_from_c(deck, ls.loc);
    tci_deck nl = *deck;
    nl.nm1_domain_ptr = nl.nm1_domain_idx = nl.nm2_domain_ptr = nl.nm2_domain_idx = nullptr;
    CsfSpace sp;
    build_space_from_c(&nl, sp);
    tci::build_local_structure(ls.loc, sp, ls);
    const i64 nint = ls.loc.n_int, nh = (i64)ls.heads7.size() / 7;
    i64 nrec = 0;
    for (i64 j = 0; j < nh; ++j) {
      const i64 m = ls.heads7[(size_t)(7 * j + 6)];
      nrec += m * (m + 1) / 2;
    }
    *count = nrec;
    if (!out) return TCI_OK;
    if (cap < 8 * nrec) return TCI_ERR_ARG;
    int64_t* r = out;
    for (i64 j = 0; j < nh; ++j) {
      const int64_t* h = ls.heads7.data() + 7 * j;
      const int64_t* dom = ls.dom_idx.data() + h[5];
      for (i64 ia = 0; ia < h[6]; ++ia)
        for (i64 ic = 0; ic <= ia; ++ic) {
          const i64 a = nint + 1 + dom[ia], c = nint + 1 + dom[ic];  // sorted domain: a >= c
          r[0] = a * (a - 1) / 2 + c;
          r[1] = ls.heads_lex[(size_t)j] - 1;
          r[2] = h[2] > 0 ? h[0] + 1 : 0;
          r[3] = h[3] > 0 ? h[1] + 1 : 0;
          r[4] = h[3];
          r[5] = h[2];
          r[6] = ia + 1;
          r[7] = ic + 1;
          r += 8;
        }
    }
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_reference_weight(const tci_space* s, const double* c, int64_t n, double* c0sq) {
  if (!s || !c || !c0sq || n != s->sp.total_csfs) return TCI_ERR_ARG;
  // calculate_ref_coeff_squared (aposteriori.f90:133-160): c^2 summed over the CSFs of the reference
  // configurations with no external electron, i.e. the metric's class 1
  std::vector<double> g((size_t)n);
  std::vector<int64_t> cls((size_t)n);
  const int rc = tci_acpf_gdiag(s, 9, 0.0, g.data(), cls.data(), n);
  if (rc != TCI_OK) return rc;
  double t = 0.0;
  for (int64_t i = 0; i < n; ++i)
    if (cls[(size_t)i] == 1) t += c[i] * c[i];
  *c0sq = t;
  return TCI_OK;
}

int tci_aposteriori(int64_t n_corr_elec, double c0sq, double e_corr, double* out, int64_t len) {
  if (!out || len < 5 || !std::isfinite(c0sq) || !std::isfinite(e_corr)) return TCI_ERR_ARG;
  if (n_corr_elec < 4 || c0sq <= 0.5 || c0sq > 1.0) {
    set_error("a posteriori corrections need at least 4 correlated electrons and 1/2 < c0^2 <= 1");
    return TCI_ERR_INPUT;
  }
  // the size-extensivity corrections of aposteriori.f90:162-221 (Davidson; renormalised Davidson;
  // Davidson-Silver; Meissner; Pople in the closed form of Duch and Diercksen, J. Chem. Phys. 101, 3018 (1994))
  const double q = 1.0 - c0sq, N = (double)n_corr_elec;
  out[0] = e_corr * q;
  out[1] = e_corr * q / c0sq;
  out[2] = e_corr * q / (2.0 * c0sq - 1.0);
  out[3] = e_corr * (q / c0sq) * ((N - 2.0) * (N - 3.0) / (N * (N - 1.0)));
  const double d = 2.0 * c0sq - 1.0;
  out[4] = e_corr * (2.0 * c0sq / (d * (1.0 + std::sqrt(1.0 + 8.0 * c0sq * q / (N * d * d)))) - 1.0);
  return TCI_OK;
}

int tci_space_block_counts(const tci_space* s, int64_t kind, int64_t* out, int64_t max_triples, int64_t* n_triples) {
  if (!s || kind < 0 || kind > 2 || !n_triples) return TCI_ERR_ARG;
  const auto& m = s->sp.cfg_count[kind];
  *n_triples = (int64_t)m.size();
  int64_t t = 0;
  for (auto& kv : m) {
    if (t >= max_triples || !out) break;
    out[3 * t + 0] = kv.first;
    // the reference prints fsn before its final zeroing; recompute it here
    SpinTables tb;
    build_spin_tables((int)s->sp.open_shells, (int)s->sp.deck.spin_mult, tb);
    out[3 * t + 1] = kv.first <= s->sp.open_shells ? tb.fsn_all[kv.first] : 0;
    out[3 * t + 2] = kv.second;
    ++t;
  }
  return TCI_OK;
}

void tci_space_destroy(tci_space* s) { delete s; }

int tci_plan_create(const tci_deck* deck, const tci_operator* op, tci_plan** out) {
  if (!out) return TCI_ERR_ARG;
  *out = nullptr;
  try {
    auto* p = new tci_plan();
    try {
      build_space_from_c(deck, p->sp);
      Operator o;
      operator_from_c(op, p->sp, o);
      build_plan(p->sp, o, p->plan);
    } catch (...) {
      delete p;
      throw;
    }
    *out = p;
    return TCI_OK;
  } catch (...) {
    return guard_status(std::current_exception());
  }
}

int tci_plan_export(const tci_plan* p, const char* path) {
  if (!p || !path) return TCI_ERR_ARG;
  FILE* f = std::fopen(path, "wb");
  if (!f) {
    set_error(std::string("cannot open ") + path);
    return TCI_ERR_ARG;
  }
  const Plan& P = p->plan;
  auto wi = [&](int64_t v) { std::fwrite(&v, 8, 1, f); };
  auto wd = [&](double v) { std::fwrite(&v, 8, 1, f); };
  std::fwrite("TCIPLAN1", 1, 8, f);
  const std::vector<Step>* lists[2] = {&P.init_steps, &P.sigma_steps};
  wi(P.nint); wi(P.n); wi(P.nchol); wi(P.total_csfs); wi(P.npair_all); wi(P.nD);
  wi((int64_t)P.dheads.size()); wi(NUM_BUFS); wi((int64_t)P.init_steps.size()); wi((int64_t)P.sigma_steps.size());
  wi((int64_t)P.h_vv.size()); wi((int64_t)P.wv.size()); wi(P.np); wi(P.nm); wi((int64_t)P.diag.size());
  for (int b = 0; b < NUM_BUFS; ++b) wi(P.buf_size[b]);
  for (auto& d : P.dheads) { wi(d.off_ab); wi(d.off_aa); wi(d.nsf_ab); wi(d.nsf_aa); wi(d.nsing); wi(d.nD); wi(d.dk0); }
  for (double v : P.dk_sign) wd(v);
  for (double v : P.h_vv) wd(v);
  for (double v : P.wv) wd(v);
  for (auto& d : P.diag) { wi(d.off); wi(d.len); wi(d.type); wd(d.beta); wi(d.foff); wi(d.singlet); }
  for (auto* L : lists)
    for (const Step& s : *L) {
      wi(s.kind);
      char name[64] = {0};
      std::snprintf(name, sizeof(name), "%s", s.name.c_str());
      std::fwrite(name, 1, 64, f);
      wi((int64_t)s.gp.size()); wi((int64_t)s.gs.size()); wi((int64_t)s.at.size());
      wi((int64_t)s.as.size()); wi((int64_t)s.dt.size()); wi((int64_t)s.ds.size());
      wi(s.buf); wi(s.off); wi(s.len);
      for (auto& g : s.gp) { wi(g.c); wi(g.offC); wi(g.ldc); wi(g.M); wi(g.N); wd(g.beta); wi(g.seg_begin); wi(g.seg_end); }
      for (auto& g : s.gs) { wi(g.a); wi(g.b); wi(g.offA); wi(g.lda); wi(g.offB); wi(g.ldb); wi(g.K); wi(g.tA); wi(g.tB); wd(g.alpha); }
      for (auto& t : s.at) { wi(t.dst); wi(t.off); wi(t.len); wi(t.src_begin); wi(t.src_end); }
      for (auto& t : s.as) { wi(t.src); wi(t.off); wd(t.coef); wi(t.sbuf); wi(t.sidx); }
      for (auto& t : s.dt) { wi(t.dst); wi(t.off); wi(t.src_begin); wi(t.src_end); }
      for (auto& t : s.ds) { wi(t.a); wi(t.b); wi(t.aoff); wi(t.boff); wi(t.len); wd(t.coef); }
    }
  std::fclose(f);
  return TCI_OK;
}

int tci_plan_stats(const tci_plan* p, double* out, int64_t len) {
  if (!p || !out || len < 8) return TCI_ERR_ARG;
  const Plan& P = p->plan;
  if (len >= 10) {
    // device bytes: peak during set-up (every plan buffer) and resident after it
    // (set-up-only buffers released); a Davidson subspace adds 2 * vectors * total_csfs * 8
    double peak = 0, resident = 0;
    for (int b = 0; b < NUM_BUFS; ++b) {
      const double bytes = (double)std::max<i64>(0, P.buf_size[b]) * 8.0;
      peak += bytes;
      if (b != BUF_X && b != BUF_L && b != BUF_LE && b != BUF_LI) resident += bytes;
    }
    out[8] = peak;
    out[9] = resident;
  }
  out[0] = (double)P.total_csfs;
  out[1] = (double)P.nD;
  out[2] = (double)P.n_sing;
  out[3] = (double)P.n_trip;
  out[4] = P.flops_allext;
  out[5] = P.flops_total;
  out[6] = P.bytes_allext;
  out[7] = (double)P.sigma_steps.size();
  return TCI_OK;
}

void tci_plan_destroy(tci_plan* p) { delete p; }

}  // extern "C"
