// Molecular front end: AO integrals over contracted Gaussians, the pivoted
// Cholesky decomposition of the AO two-electron integral matrix, a restricted
// Hartree-Fock solver on those Cholesky vectors, and the AO -> MO transform of
// the vectors into the cholesky_data layout the sigma build consumes.
//
// In the reference this is the set-up before Davidson:
//   tiger_cpp/main.cpp:270-361   cholesky(): decompose, then transfrom_to_MO_basis, then write L^J_ij (i >= j)
//   tiger_cpp/Cholesky.cpp:268-307 Cho_WholeMat::decompose: the (screened) AO ERI matrix factorised by LAPACK
//                                  dpstf2 with full diagonal pivoting, stopping when the largest remaining
//                                  diagonal is at most CD THRESHOLD
//   tiger_cpp/Cholesky.cpp:78-165  X^J_mu,i = sum_nu C_nu,i L^J_mu,nu ; L^J_ij = sum_mu C_mu,j X^J_mu,i
//   tiger_fortran/cholesky_transform.f90:379 (the same transform out of core)
// The reference computes the AO integrals with libint through Erkale and reads its orbitals from a Molden
// file (tiger_cpp/OrbitalParsers.cpp); it has no SCF.  Here the integrals follow the McMurchie-Davidson
// scheme (L. E. McMurchie and E. R. Davidson, J. Comput. Phys. 26, 218 (1978)): Hermite expansion
// coefficients of Gaussian products, Hermite Coulomb integrals from the Boys function.  The pivoted
// Cholesky decomposition computes the diagonal and only the columns it pivots on (by shell-pair blocks),
// with dpstf2's pivot rule (largest remaining diagonal, first on ties) and stopping rule, so it gives the
// vectors of the full-matrix factorisation without forming the matrix.  RHF (Roothaan-Hall with DIIS,
// P. Pulay, Chem. Phys. Lett. 73, 393 (1980)) supplies canonical orbitals where none are given.
//
// Basis conventions (Molden): primitives normalised, contracted functions renormalised to unit
// self-overlap per Cartesian component; p order x y z; Cartesian d order xx yy zz xy xz yz; pure d order
// d0 d+1 d-1 d+2 d-2 with d0 = zz - (xx + yy)/2, d+1 = xz, d-1 = yz, d+2 = sqrt(3)/2 (xx - yy), d-2 = xy
// in the normalised Cartesian components.
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../../include/tigerci_sigma.h"
#include "capi_internal.h"

namespace tci {
namespace {

constexpr int kMaxL = 2;                 // s, p, d
constexpr int kMaxLtot = 4 * kMaxL;      // (dd|dd)
constexpr int kRdim = kMaxLtot + 1;
constexpr double kPi = 3.14159265358979323846;

inline int ncart(int l) { return (l + 1) * (l + 2) / 2; }

const int kCart[3][6][3] = {{{0, 0, 0}},
                            {{1, 0, 0}, {0, 1, 0}, {0, 0, 1}},
                            {{2, 0, 0}, {0, 2, 0}, {0, 0, 2}, {1, 1, 0}, {1, 0, 1}, {0, 1, 1}}};

double dfact(int k) {  // (k)!! with (-1)!! = 1
  double r = 1.0;
  for (; k > 1; k -= 2) r *= k;
  return r;
}

struct Shell {
  int atom = 0, l = 0;
  double A[3] = {0, 0, 0};
  std::vector<double> exps;
  std::vector<double> coef[6];  // per Cartesian component: contraction coefficient x primitive norm x renorm
  int first = 0;                // first output function
  int nout = 0;                 // output functions (Cartesian or pure)
  bool pure = false;
};

// Boys function F_n(T), n = 0..nmax: series for F_nmax and downward recursion below T = 33, the closed
// form of F_0 and upward recursion above (F_{n+1} = ((2n+1) F_n - e^-T) / 2T).
void boys(int nmax, double T, double* F) {
  if (T < 1e-13) {
    for (int n = 0; n <= nmax; ++n) F[n] = 1.0 / (2 * n + 1) - T / (2 * n + 3);
    return;
  }
  const double e = std::exp(-T);
  if (T > 33.0) {
    F[0] = 0.5 * std::sqrt(kPi / T) * std::erf(std::sqrt(T));
    for (int n = 0; n < nmax; ++n) F[n + 1] = ((2 * n + 1) * F[n] - e) / (2.0 * T);
    return;
  }
  double term = 1.0 / (2 * nmax + 1), sum = term;
  for (int k = 1; k < 400; ++k) {
    term *= 2.0 * T / (2 * nmax + 2 * k + 1);
    sum += term;
    if (term < 1e-17 * sum) break;
  }
  F[nmax] = e * sum;
  for (int n = nmax - 1; n >= 0; --n) F[n] = (2.0 * T * F[n + 1] + e) / (2 * n + 1);
}

// Hermite expansion coefficients E^{ij}_t of a 1D Gaussian product, i <= la, j <= lb (lb up to kMaxL + 2
// for the kinetic energy), Xab = A - B.
struct ECube {
  double v[kMaxL + 1][kMaxL + 3][2 * kMaxL + 4];
  double at(int i, int j, int t) const { return (t < 0 || t > i + j) ? 0.0 : v[i][j][t]; }
};

void hermite_e(int la, int lb, double a, double b, double Xab, ECube& E) {
  const double p = a + b, mu = a * b / p;
  const double XPA = -b / p * Xab, XPB = a / p * Xab, i2p = 0.5 / p;
  std::memset(&E, 0, sizeof(E));
  E.v[0][0][0] = std::exp(-mu * Xab * Xab);
  for (int i = 0; i <= la; ++i)
    for (int j = 0; j <= lb; ++j) {
      if (i == 0 && j == 0) continue;
      for (int t = 0; t <= i + j; ++t) {
        if (j == 0)
          E.v[i][0][t] = i2p * E.at(i - 1, 0, t - 1) + XPA * E.at(i - 1, 0, t) + (t + 1) * E.at(i - 1, 0, t + 1);
        else
          E.v[i][j][t] = i2p * E.at(i, j - 1, t - 1) + XPB * E.at(i, j - 1, t) + (t + 1) * E.at(i, j - 1, t + 1);
      }
    }
}

// Hermite Coulomb integrals R_{tuv} = R^0_{tuv}(alpha, PC) for t + u + v <= L, written to R[(t*kRdim+u)*kRdim+v].
void hermite_r(int L, double alpha, double X, double Y, double Z, double* R) {
  double F[kMaxLtot + 1];
  boys(L, alpha * (X * X + Y * Y + Z * Z), F);
  const int d = L + 1;
  double W[kRdim * kRdim * kRdim * kRdim];
  auto ix = [d](int n, int t, int u, int v) { return ((n * d + t) * d + u) * d + v; };
  double pw = 1.0;
  for (int n = 0; n <= L; ++n) {
    W[ix(n, 0, 0, 0)] = pw * F[n];
    pw *= -2.0 * alpha;
  }
  for (int s = 1; s <= L; ++s)
    for (int n = 0; n + s <= L; ++n)
      for (int t = 0; t <= s; ++t)
        for (int u = 0; t + u <= s; ++u) {
          const int v = s - t - u;
          double val;
          if (t > 0)
            val = (t > 1 ? (t - 1) * W[ix(n + 1, t - 2, u, v)] : 0.0) + X * W[ix(n + 1, t - 1, u, v)];
          else if (u > 0)
            val = (u > 1 ? (u - 1) * W[ix(n + 1, t, u - 2, v)] : 0.0) + Y * W[ix(n + 1, t, u - 1, v)];
          else
            val = (v > 1 ? (v - 1) * W[ix(n + 1, t, u, v - 2)] : 0.0) + Z * W[ix(n + 1, t, u, v - 1)];
          W[ix(n, t, u, v)] = val;
        }
  for (int t = 0; t <= L; ++t)
    for (int u = 0; t + u <= L; ++u)
      for (int v = 0; t + u + v <= L; ++v) R[(t * kRdim + u) * kRdim + v] = W[ix(0, t, u, v)];
}

// Pure-d combination of the normalised Cartesian components (rows d0 d+1 d-1 d+2 d-2; columns xx yy zz xy xz yz).
const double kPureD[5][6] = {{-0.5, -0.5, 1.0, 0, 0, 0},
                             {0, 0, 0, 0, 1.0, 0},
                             {0, 0, 0, 0, 0, 1.0},
                             {0.86602540378443864676, -0.86602540378443864676, 0, 0, 0, 0},
                             {0, 0, 0, 1.0, 0, 0}};

// In-place transform of index `pos` (of 4, extents ext[]) of a block from Cartesian to pure d; ext[pos] becomes 5.
void block_to_pure(std::vector<double>& blk, int* ext, int pos) {
  int outer = 1, inner = 1;
  for (int k = 0; k < pos; ++k) outer *= ext[k];
  for (int k = pos + 1; k < 4; ++k) inner *= ext[k];
  std::vector<double> out((size_t)outer * 5 * inner, 0.0);
  for (int o = 0; o < outer; ++o)
    for (int r = 0; r < 5; ++r)
      for (int c = 0; c < 6; ++c) {
        const double w = kPureD[r][c];
        if (w == 0.0) continue;
        const double* src = &blk[((size_t)o * 6 + c) * inner];
        double* dst = &out[((size_t)o * 5 + r) * inner];
        for (int i = 0; i < inner; ++i) dst[i] += w * src[i];
      }
  blk.swap(out);
  ext[pos] = 5;
}

struct PrimPair {
  double p, P[3], pref;  // pref folds nothing; coefficients applied per component
  int ka, kb;
  ECube Ex, Ey, Ez;
};

}  // namespace

struct Integrals {
  std::vector<double> Z, xyz;  // atoms
  std::vector<Shell> shells;
  int nbf = 0;                 // output functions
  double e_nuc = 0.0;
  // pivoted Cholesky of the AO ERI matrix: chol[pq * nchol + J], pq = mu(mu+1)/2 + nu
  std::vector<double> chol;
  int64_t nchol = 0;
  double cd_threshold = 0.0, max_remaining = 0.0, seconds = 0.0;
  int64_t quartets = 0, pivot_blocks = 0;
  std::vector<int> func_shell;  // shell of each output function

  // (AB|CD) block in output functions, layout [a][b][c][d]
  void eri_block(int sa, int sb, int sc, int sd, std::vector<double>& out) const;
  void one_electron(std::vector<double>& S, std::vector<double>& T, std::vector<double>& V) const;
};

namespace {

void prim_pairs(const Shell& A, const Shell& B, int lb_extra, std::vector<PrimPair>& out) {
  out.clear();
  for (size_t ka = 0; ka < A.exps.size(); ++ka)
    for (size_t kb = 0; kb < B.exps.size(); ++kb) {
      PrimPair pp;
      const double a = A.exps[ka], b = B.exps[kb];
      pp.p = a + b;
      for (int k = 0; k < 3; ++k) pp.P[k] = (a * A.A[k] + b * B.A[k]) / pp.p;
      const double AB2 = (A.A[0] - B.A[0]) * (A.A[0] - B.A[0]) + (A.A[1] - B.A[1]) * (A.A[1] - B.A[1]) +
                         (A.A[2] - B.A[2]) * (A.A[2] - B.A[2]);
      if (a * b / pp.p * AB2 > 60.0) continue;  // e^-60: below any threshold of interest
      pp.ka = (int)ka;
      pp.kb = (int)kb;
      pp.pref = 1.0;
      hermite_e(A.l, B.l + lb_extra, a, b, A.A[0] - B.A[0], pp.Ex);
      hermite_e(A.l, B.l + lb_extra, a, b, A.A[1] - B.A[1], pp.Ey);
      hermite_e(A.l, B.l + lb_extra, a, b, A.A[2] - B.A[2], pp.Ez);
      out.push_back(pp);
    }
}

}  // namespace

void Integrals::eri_block(int sa, int sb, int sc, int sd, std::vector<double>& out) const {
  const Shell &A = shells[sa], &B = shells[sb], &Cs = shells[sc], &D = shells[sd];
  const int na = ncart(A.l), nb = ncart(B.l), nc = ncart(Cs.l), nd = ncart(D.l);
  const int Lb = A.l + B.l, Lk = Cs.l + D.l, Lt = Lb + Lk;
  // Hermite index lists
  int hb[35][3], hk[35][3];
  int nhb = 0, nhk = 0;
  for (int t = 0; t <= Lb; ++t)
    for (int u = 0; t + u <= Lb; ++u)
      for (int v = 0; t + u + v <= Lb; ++v) hb[nhb][0] = t, hb[nhb][1] = u, hb[nhb][2] = v, ++nhb;
  for (int t = 0; t <= Lk; ++t)
    for (int u = 0; t + u <= Lk; ++u)
      for (int v = 0; t + u + v <= Lk; ++v) hk[nhk][0] = t, hk[nhk][1] = u, hk[nhk][2] = v, ++nhk;
  std::vector<PrimPair> bra, ket;
  prim_pairs(A, B, 0, bra);
  prim_pairs(Cs, D, 0, ket);
  const int nab = na * nb, ncd = nc * nd;
  std::vector<double> cart((size_t)nab * ncd, 0.0);
  std::vector<double> Ebra((size_t)nab * nhb), Eket((size_t)ncd * nhk), G((size_t)nhb * ncd);
  std::vector<double> RR(kRdim * kRdim * kRdim);
  // ket Hermite coefficients per primitive pair (with the (-1)^(tau+nu+phi) sign), computed once
  std::vector<std::vector<double>> EketAll(ket.size());
  for (size_t q = 0; q < ket.size(); ++q) {
    const PrimPair& kp = ket[q];
    auto& Ek = EketAll[q];
    Ek.assign((size_t)ncd * nhk, 0.0);
    for (int c = 0; c < nc; ++c)
      for (int d = 0; d < nd; ++d) {
        const int* lc = kCart[Cs.l][c];
        const int* ld = kCart[D.l][d];
        const double cf = Cs.coef[c][kp.ka] * D.coef[d][kp.kb];
        for (int h = 0; h < nhk; ++h) {
          const int t = hk[h][0], u = hk[h][1], v = hk[h][2];
          const double sgn = ((t + u + v) & 1) ? -1.0 : 1.0;
          Ek[(size_t)(c * nd + d) * nhk + h] =
              sgn * cf * kp.Ex.at(lc[0], ld[0], t) * kp.Ey.at(lc[1], ld[1], u) * kp.Ez.at(lc[2], ld[2], v);
        }
      }
  }
  for (const PrimPair& bp : bra) {
    for (int a = 0; a < na; ++a)
      for (int b = 0; b < nb; ++b) {
        const int* la = kCart[A.l][a];
        const int* lb = kCart[B.l][b];
        const double cf = A.coef[a][bp.ka] * B.coef[b][bp.kb];
        for (int h = 0; h < nhb; ++h)
          Ebra[(size_t)(a * nb + b) * nhb + h] =
              cf * bp.Ex.at(la[0], lb[0], hb[h][0]) * bp.Ey.at(la[1], lb[1], hb[h][1]) * bp.Ez.at(la[2], lb[2], hb[h][2]);
      }
    std::fill(G.begin(), G.end(), 0.0);
    for (size_t q = 0; q < ket.size(); ++q) {
      const PrimPair& kp = ket[q];
      const double p = bp.p, qq = kp.p, alpha = p * qq / (p + qq);
      const double pref = 2.0 * std::pow(kPi, 2.5) / (p * qq * std::sqrt(p + qq));
      hermite_r(Lt, alpha, bp.P[0] - kp.P[0], bp.P[1] - kp.P[1], bp.P[2] - kp.P[2], RR.data());
      const auto& Ek = EketAll[q];
      for (int h = 0; h < nhb; ++h) {
        const int t = hb[h][0], u = hb[h][1], v = hb[h][2];
        double* g = &G[(size_t)h * ncd];
        for (int h2 = 0; h2 < nhk; ++h2) {
          const double r = pref * RR[((t + hk[h2][0]) * kRdim + u + hk[h2][1]) * kRdim + v + hk[h2][2]];
          for (int cd = 0; cd < ncd; ++cd) g[cd] += r * Ek[(size_t)cd * nhk + h2];
        }
      }
    }
    for (int ab = 0; ab < nab; ++ab) {
      const double* e = &Ebra[(size_t)ab * nhb];
      double* o = &cart[(size_t)ab * ncd];
      for (int h = 0; h < nhb; ++h) {
        const double w = e[h];
        if (w == 0.0) continue;
        const double* g = &G[(size_t)h * ncd];
        for (int cd = 0; cd < ncd; ++cd) o[cd] += w * g[cd];
      }
    }
  }
  int ext[4] = {na, nb, nc, nd};
  const Shell* sh[4] = {&A, &B, &Cs, &D};
  for (int k = 0; k < 4; ++k)
    if (sh[k]->pure && sh[k]->l == 2) block_to_pure(cart, ext, k);
  out.swap(cart);
}

void Integrals::one_electron(std::vector<double>& S, std::vector<double>& T, std::vector<double>& V) const {
  const int n = nbf;
  S.assign((size_t)n * n, 0.0);
  T.assign((size_t)n * n, 0.0);
  V.assign((size_t)n * n, 0.0);
  const int ns = (int)shells.size();
  const int natom = (int)Z.size();
#pragma omp parallel for schedule(dynamic)
  for (int sab = 0; sab < ns * ns; ++sab) {
    const int sa = sab / ns, sb = sab % ns;
    if (sb > sa) continue;
    const Shell &A = shells[sa], &B = shells[sb];
    const int na = ncart(A.l), nb = ncart(B.l);
    std::vector<double> s((size_t)na * nb, 0.0), t((size_t)na * nb, 0.0), v((size_t)na * nb, 0.0);
    std::vector<PrimPair> pp;
    prim_pairs(A, B, 2, pp);
    std::vector<double> RR(kRdim * kRdim * kRdim);
    for (const PrimPair& q : pp) {
      const double b = B.exps[q.kb], p = q.p;
      const double sq = std::sqrt(kPi / p);
      // nuclear-attraction Hermite integrals per atom
      std::vector<std::vector<double>> Rn(natom);
      for (int c = 0; c < natom; ++c) {
        Rn[c].resize(RR.size());
        hermite_r(A.l + B.l, p, q.P[0] - xyz[3 * c], q.P[1] - xyz[3 * c + 1], q.P[2] - xyz[3 * c + 2], Rn[c].data());
      }
      for (int ia = 0; ia < na; ++ia)
        for (int ib = 0; ib < nb; ++ib) {
          const int* la = kCart[A.l][ia];
          const int* lb = kCart[B.l][ib];
          const double cf = A.coef[ia][q.ka] * B.coef[ib][q.kb];
          const ECube* E[3] = {&q.Ex, &q.Ey, &q.Ez};
          double s1[3], t1[3];
          for (int k = 0; k < 3; ++k) {
            const int i = la[k], j = lb[k];
            auto S1 = [&](int jj) { return jj < 0 ? 0.0 : E[k]->at(i, jj, 0) * sq; };
            s1[k] = S1(j);
            t1[k] = -0.5 * (j * (j - 1) * S1(j - 2) - 2.0 * b * (2 * j + 1) * S1(j) + 4.0 * b * b * S1(j + 2));
          }
          s[ia * nb + ib] += cf * s1[0] * s1[1] * s1[2];
          t[ia * nb + ib] += cf * (t1[0] * s1[1] * s1[2] + s1[0] * t1[1] * s1[2] + s1[0] * s1[1] * t1[2]);
          double vv = 0.0;
          for (int tt = 0; tt <= la[0] + lb[0]; ++tt)
            for (int u = 0; u <= la[1] + lb[1]; ++u)
              for (int w = 0; w <= la[2] + lb[2]; ++w) {
                const double e = q.Ex.at(la[0], lb[0], tt) * q.Ey.at(la[1], lb[1], u) * q.Ez.at(la[2], lb[2], w);
                if (e == 0.0) continue;
                double r = 0.0;
                for (int c = 0; c < natom; ++c) r -= Z[c] * Rn[c][(tt * kRdim + u) * kRdim + w];
                vv += e * r;
              }
          v[ia * nb + ib] += cf * 2.0 * kPi / p * vv;
        }
    }
    // to output functions
    auto finish = [&](std::vector<double>& m, std::vector<double>& dst) {
      int ext[4] = {na, nb, 1, 1};
      if (A.pure && A.l == 2) block_to_pure(m, ext, 0);
      if (B.pure && B.l == 2) block_to_pure(m, ext, 1);
      for (int i = 0; i < ext[0]; ++i)
        for (int j = 0; j < ext[1]; ++j) {
          const double x = m[i * ext[1] + j];
          dst[(size_t)(A.first + i) * n + B.first + j] = x;
          dst[(size_t)(B.first + j) * n + A.first + i] = x;
        }
    };
    finish(s, S);
    finish(t, T);
    finish(v, V);
  }
}

namespace {

void build_molecule(const tci_molecule* m, Integrals& it) {
  if (!m || m->n_atoms <= 0 || !m->charges || !m->coords || m->n_shells <= 0 || !m->shell_atom || !m->shell_l ||
      !m->shell_nprim || !m->exponents || !m->coefficients)
    throw Error(TCI_ERR_ARG, "tci_molecule: missing fields");
  it.Z.assign(m->charges, m->charges + m->n_atoms);
  it.xyz.assign(m->coords, m->coords + 3 * m->n_atoms);
  for (int i = 0; i < m->n_atoms; ++i)
    for (int j = 0; j < i; ++j) {
      double r2 = 0;
      for (int k = 0; k < 3; ++k) r2 += (it.xyz[3 * i + k] - it.xyz[3 * j + k]) * (it.xyz[3 * i + k] - it.xyz[3 * j + k]);
      if (r2 < 1e-12) throw Error(TCI_ERR_INPUT, "tci_molecule: two atoms at the same position");
      it.e_nuc += it.Z[i] * it.Z[j] / std::sqrt(r2);
    }
  int64_t off = 0;
  int first = 0;
  for (int64_t s = 0; s < m->n_shells; ++s) {
    Shell sh;
    sh.atom = (int)m->shell_atom[s];
    sh.l = (int)m->shell_l[s];
    const int64_t np = m->shell_nprim[s];
    if (sh.atom < 0 || sh.atom >= m->n_atoms || sh.l < 0 || sh.l > kMaxL || np <= 0)
      throw Error(TCI_ERR_INPUT, "tci_molecule: shell " + std::to_string((long long)s) +
                                     " has a bad atom, angular momentum (s, p, d supported) or primitive count");
    for (int k = 0; k < 3; ++k) sh.A[k] = it.xyz[3 * sh.atom + k];
    sh.exps.assign(m->exponents + off, m->exponents + off + np);
    for (double e : sh.exps)
      if (!(e > 0.0)) throw Error(TCI_ERR_INPUT, "tci_molecule: non-positive exponent");
    const double* cf = m->coefficients + off;
    off += np;
    for (int c = 0; c < ncart(sh.l); ++c) {
      const int* lmn = kCart[sh.l][c];
      std::vector<double> w(np);
      for (int64_t k = 0; k < np; ++k) {
        const double a = sh.exps[k];
        w[k] = cf[k] * std::pow(2.0 * a / kPi, 0.75) * std::pow(4.0 * a, 0.5 * sh.l) /
               std::sqrt(dfact(2 * lmn[0] - 1) * dfact(2 * lmn[1] - 1) * dfact(2 * lmn[2] - 1));
      }
      // self-overlap of the contracted component
      double ss = 0.0;
      for (int64_t i = 0; i < np; ++i)
        for (int64_t j = 0; j < np; ++j) {
          const double p = sh.exps[i] + sh.exps[j];
          double v = std::pow(kPi / p, 1.5);
          for (int k = 0; k < 3; ++k) v *= dfact(2 * lmn[k] - 1) / std::pow(2.0 * p, lmn[k]);
          ss += w[i] * w[j] * v;
        }
      if (!(ss > 0.0)) throw Error(TCI_ERR_INPUT, "tci_molecule: contracted function with zero norm");
      for (auto& x : w) x /= std::sqrt(ss);
      sh.coef[c] = w;
    }
    sh.pure = (m->pure_d != 0) && sh.l == 2;
    sh.first = first;
    sh.nout = sh.pure ? 5 : ncart(sh.l);
    first += sh.nout;
    it.shells.push_back(std::move(sh));
  }
  it.nbf = first;
  it.func_shell.resize(it.nbf);
  for (int s = 0; s < (int)it.shells.size(); ++s)
    for (int k = 0; k < it.shells[s].nout; ++k) it.func_shell[it.shells[s].first + k] = s;
}

inline int64_t pidx(int64_t p, int64_t q) { return p >= q ? p * (p + 1) / 2 + q : q * (q + 1) / 2 + p; }

// Pivoted Cholesky of the AO ERI matrix over function pairs mu >= nu.
void decompose(Integrals& it, double thresh) {
  const int n = it.nbf, ns = (int)it.shells.size();
  const int64_t npair = (int64_t)n * (n + 1) / 2;
  // diagonal (mu nu|mu nu) from the (AB|AB) blocks
  std::vector<double> diag(npair, 0.0);
  int64_t quartets = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : quartets)
  for (int sab = 0; sab < ns * ns; ++sab) {
    const int sa = sab / ns, sb = sab % ns;
    if (sb > sa) continue;
    std::vector<double> blk;
    it.eri_block(sa, sb, sa, sb, blk);
    ++quartets;
    const Shell &A = it.shells[sa], &B = it.shells[sb];
    for (int a = 0; a < A.nout; ++a)
      for (int b = 0; b < B.nout; ++b) {
        const int mu = A.first + a, nu = B.first + b;
        if (nu > mu) continue;
        diag[pidx(mu, nu)] = blk[(((size_t)a * B.nout + b) * A.nout + a) * B.nout + b];
      }
  }
  // shell pair of every shell-pair block, and its function pairs
  std::unordered_map<int64_t, std::vector<double>> cache;  // pair index -> ERI column
  int64_t cap = std::max<int64_t>(64, std::min<int64_t>(npair, 4 * n));
  std::vector<double> L((size_t)npair * cap, 0.0);
  int64_t J = 0;
  std::vector<char> used(npair, 0);
  std::vector<double> col(npair);
  int64_t blocks = 0;
  while (J < npair) {
    int64_t piv = -1;
    double dmax = -1.0;
    for (int64_t k = 0; k < npair; ++k)
      if (!used[k] && diag[k] > dmax) dmax = diag[k], piv = k;
    if (piv < 0 || dmax <= thresh) {
      it.max_remaining = std::max(0.0, dmax);
      break;
    }
    auto f = cache.find(piv);
    if (f == cache.end()) {
      // columns of every function pair of the pivot's shell pair
      int64_t mu = (int64_t)((std::sqrt(8.0 * piv + 1.0) - 1.0) / 2.0);
      while (mu * (mu + 1) / 2 > piv) --mu;
      while ((mu + 1) * (mu + 2) / 2 <= piv) ++mu;
      const int64_t nu = piv - mu * (mu + 1) / 2;
      const int sc = it.func_shell[mu], sd = it.func_shell[nu];
      const Shell &Cs = it.shells[sc], &D = it.shells[sd];
      std::vector<std::pair<int64_t, std::vector<double>>> cols;
      for (int c = 0; c < Cs.nout; ++c)
        for (int d = 0; d < D.nout; ++d) {
          const int64_t g = Cs.first + c, h = D.first + d;
          if (h > g) continue;
          const int64_t pq = pidx(g, h);
          if (used[pq] || cache.count(pq)) continue;
          cols.emplace_back(pq, std::vector<double>(npair, 0.0));
        }
      std::unordered_map<int64_t, size_t> slot;
      for (size_t i = 0; i < cols.size(); ++i) slot[cols[i].first] = i;
      int64_t qn = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : qn)
      for (int sab = 0; sab < ns * ns; ++sab) {
        const int sa = sab / ns, sb = sab % ns;
        if (sb > sa) continue;
        std::vector<double> blk;
        it.eri_block(sa, sb, sc, sd, blk);
        ++qn;
        const Shell &A = it.shells[sa], &B = it.shells[sb];
        for (int a = 0; a < A.nout; ++a)
          for (int b = 0; b < B.nout; ++b) {
            const int64_t m1 = A.first + a, n1 = B.first + b;
            if (n1 > m1) continue;
            const int64_t row = pidx(m1, n1);
            for (int c = 0; c < Cs.nout; ++c)
              for (int d = 0; d < D.nout; ++d) {
                const int64_t g = Cs.first + c, h = D.first + d;
                if (h > g) continue;
                auto s = slot.find(pidx(g, h));
                if (s == slot.end()) continue;
                cols[s->second].second[row] = blk[(((size_t)a * B.nout + b) * Cs.nout + c) * D.nout + d];
              }
          }
      }
      quartets += qn;
      ++blocks;
      for (auto& c : cols) cache.emplace(c.first, std::move(c.second));
      f = cache.find(piv);
      if (f == cache.end()) throw Error(TCI_ERR_INTERNAL, "Cholesky: pivot column missing");
    }
    if (J == cap) {  // grow the vector store
      const int64_t ncap = std::min<int64_t>(npair, 2 * cap);
      std::vector<double> L2((size_t)npair * ncap, 0.0);
#pragma omp parallel for
      for (int64_t k = 0; k < npair; ++k) std::memcpy(&L2[(size_t)k * ncap], &L[(size_t)k * cap], sizeof(double) * J);
      L.swap(L2);
      cap = ncap;
    }
    const std::vector<double>& g = f->second;
    const double* lp = &L[(size_t)piv * cap];
    const double inv = 1.0 / std::sqrt(dmax);
#pragma omp parallel for schedule(static)
    for (int64_t k = 0; k < npair; ++k) {
      const double* lk = &L[(size_t)k * cap];
      double acc = g[k];
      for (int64_t K = 0; K < J; ++K) acc -= lk[K] * lp[K];
      const double v = used[k] ? 0.0 : acc * inv;
      L[(size_t)k * cap + J] = v;
      diag[k] -= v * v;
    }
    L[(size_t)piv * cap + J] = std::sqrt(dmax);  // exact on the pivot row
    used[piv] = 1;
    diag[piv] = 0.0;
    cache.erase(piv);
    ++J;
  }
  it.nchol = J;
  it.chol.assign((size_t)npair * J, 0.0);
  for (int64_t k = 0; k < npair; ++k) std::memcpy(&it.chol[(size_t)k * J], &L[(size_t)k * cap], sizeof(double) * J);
  it.quartets = quartets;
  it.pivot_blocks = blocks;
  it.cd_threshold = thresh;
}

// Eigen-decomposition of a symmetric matrix (row major n x n): Householder reduction to tridiagonal form
// (A = Q T Q^T, one reflector per column) and the implicit QL iteration with Wilkinson shifts on T
// (the Wilkinson-Reinsch procedures tred2 / tql2, Handbook for Automatic Computation II, 1971), the plane
// rotations accumulated into Q.  w ascending, eigenvectors as the columns of V.
void eigh_sym(int n, std::vector<double> A, std::vector<double>& w, std::vector<double>& V) {
  std::vector<double> Q((size_t)n * n, 0.0), v(n), pv(n), u(n);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  for (int k = 0; k + 2 < n; ++k) {
    double nrm = 0.0;
    for (int i = k + 1; i < n; ++i) nrm += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    nrm = std::sqrt(nrm);
    if (nrm < 1e-300) continue;
    const double x0 = A[(size_t)(k + 1) * n + k];
    const double alpha = x0 > 0 ? -nrm : nrm;
    std::fill(v.begin(), v.end(), 0.0);
    for (int i = k + 1; i < n; ++i) v[i] = A[(size_t)i * n + k];
    v[k + 1] -= alpha;
    double vn = 0.0;
    for (int i = k + 1; i < n; ++i) vn += v[i] * v[i];
    vn = std::sqrt(vn);
    if (vn < 1e-300) continue;
    for (int i = k + 1; i < n; ++i) v[i] /= vn;
    // H A H = A - 2 (v q^T + q v^T), p = A v, q = p - (v.p) v
    double K = 0.0;
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      const double* a = &A[(size_t)i * n];
      for (int j = k + 1; j < n; ++j) s += a[j] * v[j];
      pv[i] = s;
      K += v[i] * s;
    }
    for (int i = 0; i < n; ++i) pv[i] -= K * v[i];
    for (int i = 0; i < n; ++i) {
      double* a = &A[(size_t)i * n];
      const double vi = v[i], qi = pv[i];
      for (int j = 0; j < n; ++j) a[j] -= 2.0 * (vi * pv[j] + qi * v[j]);
    }
    // Q <- Q H
    for (int i = 0; i < n; ++i) {
      double s = 0.0;
      const double* q = &Q[(size_t)i * n];
      for (int j = k + 1; j < n; ++j) s += q[j] * v[j];
      u[i] = s;
    }
    for (int i = 0; i < n; ++i) {
      double* q = &Q[(size_t)i * n];
      const double ui = 2.0 * u[i];
      for (int j = k + 1; j < n; ++j) q[j] -= ui * v[j];
    }
  }
  std::vector<double> d(n), e(n, 0.0);
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = A[(size_t)(i + 1) * n + i];  // e[i] couples i and i + 1
  const double eps = 2.220446049250313e-16;
  for (int l = 0; l < n; ++l) {
    for (int iter = 0; iter < 200; ++iter) {
      int m = l;
      for (; m + 1 < n; ++m) {
        const double dd = std::fabs(d[m]) + std::fabs(d[m + 1]);
        if (std::fabs(e[m]) <= eps * dd) break;
      }
      if (m == l) break;
      // Wilkinson shift from the leading 2 x 2 block of the unreduced part
      double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
      double r = std::hypot(g, 1.0);
      g = d[m] - d[l] + e[l] / (g + (g >= 0 ? r : -r));
      double s = 1.0, c = 1.0, p = 0.0;
      int i = m - 1;
      bool deflated = false;
      for (; i >= l; --i) {
        const double f = s * e[i], b = c * e[i];
        r = std::hypot(f, g);
        e[i + 1] = r;
        if (r == 0.0) {  // underflow: split here
          d[i + 1] -= p;
          e[m] = 0.0;
          deflated = true;
          break;
        }
        s = f / r;
        c = g / r;
        g = d[i + 1] - p;
        r = (d[i] - g) * s + 2.0 * c * b;
        p = s * r;
        d[i + 1] = g + p;
        g = c * r - b;
        for (int k = 0; k < n; ++k) {
          double* q = &Q[(size_t)k * n];
          const double t = q[i + 1];
          q[i + 1] = s * q[i] + c * t;
          q[i] = c * q[i] - s * t;
        }
      }
      if (deflated) continue;
      d[l] -= p;
      e[l] = g;
      e[m] = 0.0;
    }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::stable_sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
  w.resize(n);
  V.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    w[j] = d[ord[j]];
    for (int i = 0; i < n; ++i) V[(size_t)i * n + j] = Q[(size_t)i * n + ord[j]];
  }
}

// C = A (m x k) * B (k x n), row major, plain blocked loops (small matrices).
void matmul(int m, int k, int n, const double* A, const double* B, double* C, bool transA = false) {
  std::fill(C, C + (size_t)m * n, 0.0);
  for (int i = 0; i < m; ++i)
    for (int l = 0; l < k; ++l) {
      const double a = transA ? A[(size_t)l * m + i] : A[(size_t)i * k + l];
      if (a == 0.0) continue;
      const double* b = B + (size_t)l * n;
      double* c = C + (size_t)i * n;
      for (int j = 0; j < n; ++j) c[j] += a * b[j];
    }
}

// Solves the DIIS equations (Pulay): minimise |sum c_i e_i| with sum c_i = 1, by Gaussian elimination with
// partial pivoting on the bordered Gram matrix.
bool diis_coefficients(const std::vector<std::vector<double>>& errs, std::vector<double>& c) {
  const int m = (int)errs.size(), d = m + 1;
  std::vector<double> M((size_t)d * d, 0.0), r(d, 0.0);
  for (int i = 0; i < m; ++i)
    for (int j = 0; j <= i; ++j) {
      double s = 0.0;
      for (size_t k = 0; k < errs[i].size(); ++k) s += errs[i][k] * errs[j][k];
      M[(size_t)i * d + j] = M[(size_t)j * d + i] = s;
    }
  for (int i = 0; i < m; ++i) M[(size_t)i * d + m] = M[(size_t)m * d + i] = -1.0;
  r[m] = -1.0;
  for (int col = 0; col < d; ++col) {
    int piv = col;
    for (int i = col + 1; i < d; ++i)
      if (std::fabs(M[(size_t)i * d + col]) > std::fabs(M[(size_t)piv * d + col])) piv = i;
    if (std::fabs(M[(size_t)piv * d + col]) < 1e-300) return false;
    if (piv != col) {
      for (int j = 0; j < d; ++j) std::swap(M[(size_t)col * d + j], M[(size_t)piv * d + j]);
      std::swap(r[col], r[piv]);
    }
    for (int i = col + 1; i < d; ++i) {
      const double f = M[(size_t)i * d + col] / M[(size_t)col * d + col];
      for (int j = col; j < d; ++j) M[(size_t)i * d + j] -= f * M[(size_t)col * d + j];
      r[i] -= f * r[col];
    }
  }
  std::vector<double> x(d);
  for (int i = d - 1; i >= 0; --i) {
    double s = r[i];
    for (int j = i + 1; j < d; ++j) s -= M[(size_t)i * d + j] * x[j];
    x[i] = s / M[(size_t)i * d + i];
  }
  c.assign(x.begin(), x.begin() + m);
  return true;
}

// Fock matrix F = h + J[D] - 1/2 K[D] of the closed-shell density D = 2 C_occ C_occ^T, from the AO Cholesky
// vectors: J_mn = sum_J L^J_mn gamma_J, gamma_J = sum_ls L^J_ls D_ls; K = 2 sum_J B_J B_J^T, B_J = L^J C_occ.
void fock(const Integrals& it, const std::vector<double>& h, const std::vector<double>& Cocc, int nocc,
          const std::vector<double>& D, std::vector<double>& F) {
  const int n = it.nbf;
  const int64_t npair = (int64_t)n * (n + 1) / 2, nc = it.nchol;
  std::vector<double> gamma(nc, 0.0);
  for (int64_t pq = 0; pq < npair; ++pq) {
    int64_t p = (int64_t)((std::sqrt(8.0 * pq + 1.0) - 1.0) / 2.0);
    while (p * (p + 1) / 2 > pq) --p;
    while ((p + 1) * (p + 2) / 2 <= pq) ++p;
    const int64_t q = pq - p * (p + 1) / 2;
    const double w = (p == q ? 1.0 : 2.0) * D[(size_t)p * n + q];
    const double* l = &it.chol[(size_t)pq * nc];
    for (int64_t J = 0; J < nc; ++J) gamma[J] += w * l[J];
  }
  F = h;
  int nthr = omp_get_max_threads();
  std::vector<std::vector<double>> Kt(nthr, std::vector<double>((size_t)n * n, 0.0));
#pragma omp parallel
  {
    std::vector<double> Lf((size_t)n * n), B((size_t)n * nocc);
    auto& K = Kt[omp_get_thread_num()];
#pragma omp for schedule(dynamic, 4)
    for (int64_t J = 0; J < nc; ++J) {
      for (int p = 0; p < n; ++p)
        for (int q = 0; q <= p; ++q) Lf[(size_t)p * n + q] = Lf[(size_t)q * n + p] = it.chol[(size_t)pidx(p, q) * nc + J];
      matmul(n, n, nocc, Lf.data(), Cocc.data(), B.data());
      for (int p = 0; p < n; ++p)
        for (int q = 0; q <= p; ++q) {
          double s = 0.0;
          for (int i = 0; i < nocc; ++i) s += B[(size_t)p * nocc + i] * B[(size_t)q * nocc + i];
          K[(size_t)p * n + q] += s;
        }
    }
  }
  for (int p = 0; p < n; ++p)
    for (int q = 0; q <= p; ++q) {
      double k = 0.0;
      for (int t = 0; t < nthr; ++t) k += Kt[t][(size_t)p * n + q];
      double j = 0.0;
      const double* l = &it.chol[(size_t)pidx(p, q) * nc];
      for (int64_t J = 0; J < nc; ++J) j += l[J] * gamma[J];
      // K[D] = 2 sum_J B B^T; F = h + J - K[D]/2
      F[(size_t)p * n + q] += j - k;
      if (p != q) F[(size_t)q * n + p] = F[(size_t)p * n + q];
    }
}

}  // namespace
}  // namespace tci

using tci::Error;

struct tci_integrals : tci::Integrals {};

extern "C" int tci_integrals_create(const tci_molecule* mol, double cd_threshold, tci_integrals** out) {
  try {
    if (!out) throw Error(TCI_ERR_ARG, "tci_integrals_create: null output");
    if (!(cd_threshold > 0.0)) throw Error(TCI_ERR_ARG, "tci_integrals_create: CD threshold must be positive");
    auto t0 = std::chrono::steady_clock::now();
    std::unique_ptr<tci_integrals> it(new tci_integrals());
    tci::build_molecule(mol, *it);
    tci::decompose(*it, cd_threshold);
    it->seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    *out = it.release();
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}

extern "C" int tci_integrals_info(const tci_integrals* it, double* out, int64_t len) {
  if (!it || !out || len < 1) {
    tci::set_error("tci_integrals_info: null argument");
    return TCI_ERR_ARG;
  }
  const double v[8] = {(double)it->nbf, (double)it->nchol, it->e_nuc, it->seconds, it->max_remaining,
                       (double)it->quartets, (double)it->pivot_blocks, (double)it->shells.size()};
  for (int64_t i = 0; i < len && i < 8; ++i) out[i] = v[i];
  return TCI_OK;
}

extern "C" int tci_integrals_one_electron(const tci_integrals* it, double* S, double* h, int64_t nbf) {
  try {
    if (!it || nbf != it->nbf) throw Error(TCI_ERR_ARG, "tci_integrals_one_electron: size mismatch");
    std::vector<double> s, t, v;
    it->one_electron(s, t, v);
    if (S) std::memcpy(S, s.data(), sizeof(double) * s.size());
    if (h)
      for (size_t i = 0; i < t.size(); ++i) h[i] = t[i] + v[i];
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}

extern "C" int tci_integrals_ao_cholesky(const tci_integrals* it, double* chol, int64_t npair, int64_t nchol) {
  if (!it || !chol || npair != (int64_t)it->nbf * (it->nbf + 1) / 2 || nchol != it->nchol) {
    tci::set_error("tci_integrals_ao_cholesky: size mismatch");
    return TCI_ERR_ARG;
  }
  std::memcpy(chol, it->chol.data(), sizeof(double) * it->chol.size());
  return TCI_OK;
}

extern "C" int tci_integrals_ao_eri(const tci_integrals* it, double* eri, int64_t nbf) {
  try {
    if (!it || !eri || nbf != it->nbf) throw Error(TCI_ERR_ARG, "tci_integrals_ao_eri: size mismatch");
    if (nbf > 200) throw Error(TCI_ERR_ARG, "tci_integrals_ao_eri: the full tensor is for small bases (<= 200)");
    const int ns = (int)it->shells.size();
    const size_t n = (size_t)nbf;
#pragma omp parallel for schedule(dynamic) collapse(2)
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) {
        std::vector<double> blk;
        for (int c = 0; c < ns; ++c)
          for (int d = 0; d < ns; ++d) {
            it->eri_block(a, b, c, d, blk);
            const auto &A = it->shells[a], &B = it->shells[b], &Cs = it->shells[c], &D = it->shells[d];
            for (int i = 0; i < A.nout; ++i)
              for (int j = 0; j < B.nout; ++j)
                for (int k = 0; k < Cs.nout; ++k)
                  for (int l = 0; l < D.nout; ++l)
                    eri[(((A.first + i) * n + B.first + j) * n + Cs.first + k) * n + D.first + l] =
                        blk[(((size_t)i * B.nout + j) * Cs.nout + k) * D.nout + l];
          }
      }
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}

extern "C" int tci_rhf(const tci_integrals* it, int64_t n_occ, int64_t maxit, double conv, double* C, double* eps,
                       double* info) {
  try {
    if (!it || !C || !eps) throw Error(TCI_ERR_ARG, "tci_rhf: null argument");
    const int n = it->nbf;
    if (n_occ <= 0 || n_occ > n) throw Error(TCI_ERR_ARG, "tci_rhf: bad number of doubly occupied orbitals");
    if (maxit <= 0) maxit = 100;
    if (!(conv > 0.0)) conv = 1e-10;
    const int nocc = (int)n_occ;
    std::vector<double> S, T, V;
    it->one_electron(S, T, V);
    std::vector<double> h((size_t)n * n);
    for (size_t i = 0; i < h.size(); ++i) h[i] = T[i] + V[i];
    // symmetric orthogonaliser X = S^-1/2
    std::vector<double> sw, sv;
    tci::eigh_sym(n, S, sw, sv);
    if (sw[0] < 1e-9) throw Error(TCI_ERR_INPUT, "tci_rhf: near-linearly-dependent basis (overlap eigenvalue < 1e-9)");
    std::vector<double> X((size_t)n * n, 0.0);
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        double s = 0.0;
        for (int k = 0; k < n; ++k) s += sv[(size_t)i * n + k] * sv[(size_t)j * n + k] / std::sqrt(sw[k]);
        X[(size_t)i * n + j] = s;
      }
    auto solve = [&](const std::vector<double>& F, std::vector<double>& Cout, std::vector<double>& e) {
      std::vector<double> t1((size_t)n * n), Fp((size_t)n * n), Cp;
      tci::matmul(n, n, n, X.data(), F.data(), t1.data(), true);  // X^T F (X symmetric)
      tci::matmul(n, n, n, t1.data(), X.data(), Fp.data());
      tci::eigh_sym(n, Fp, e, Cp);
      Cout.resize((size_t)n * n);
      tci::matmul(n, n, n, X.data(), Cp.data(), Cout.data());
    };
    std::vector<double> Cm, e;
    solve(h, Cm, e);
    std::vector<double> D((size_t)n * n), F, Cocc((size_t)n * nocc);
    std::vector<std::vector<double>> Fs, Es;
    double E = 0.0, Eold = 0.0, err = 1.0;
    int64_t iter = 0;
    bool done = false;
    for (iter = 1; iter <= maxit; ++iter) {
      for (int p = 0; p < n; ++p)
        for (int i = 0; i < nocc; ++i) Cocc[(size_t)p * nocc + i] = Cm[(size_t)p * n + i];
      for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) {
          double s = 0.0;
          for (int i = 0; i < nocc; ++i) s += Cocc[(size_t)p * nocc + i] * Cocc[(size_t)q * nocc + i];
          D[(size_t)p * n + q] = 2.0 * s;
        }
      tci::fock(*it, h, Cocc, nocc, D, F);
      E = it->e_nuc;
      for (size_t k = 0; k < D.size(); ++k) E += 0.5 * D[k] * (h[k] + F[k]);
      // DIIS error X^T (F D S - S D F) X
      std::vector<double> FD((size_t)n * n), FDS((size_t)n * n), ev((size_t)n * n), t1((size_t)n * n), eo((size_t)n * n);
      tci::matmul(n, n, n, F.data(), D.data(), FD.data());
      tci::matmul(n, n, n, FD.data(), S.data(), FDS.data());
      for (int p = 0; p < n; ++p)
        for (int q = 0; q < n; ++q) ev[(size_t)p * n + q] = FDS[(size_t)p * n + q] - FDS[(size_t)q * n + p];
      tci::matmul(n, n, n, X.data(), ev.data(), t1.data(), true);
      tci::matmul(n, n, n, t1.data(), X.data(), eo.data());
      err = 0.0;
      for (double x : eo) err = std::max(err, std::fabs(x));
      if (iter > 1 && std::fabs(E - Eold) < conv && err < std::sqrt(conv)) {
        done = true;
        break;
      }
      Eold = E;
      Fs.push_back(F);
      Es.push_back(eo);
      if (Fs.size() > 8) {
        Fs.erase(Fs.begin());
        Es.erase(Es.begin());
      }
      std::vector<double> Fx = F, cf;
      if (Fs.size() >= 2 && tci::diis_coefficients(Es, cf)) {
        std::fill(Fx.begin(), Fx.end(), 0.0);
        for (size_t k = 0; k < Fs.size(); ++k)
          for (size_t i = 0; i < Fx.size(); ++i) Fx[i] += cf[k] * Fs[k][i];
      }
      solve(Fx, Cm, e);
    }
    // canonical orbitals of the final Fock matrix
    solve(F, Cm, e);
    std::memcpy(C, Cm.data(), sizeof(double) * Cm.size());
    std::memcpy(eps, e.data(), sizeof(double) * n);
    if (info) {
      info[0] = E;
      info[1] = (double)std::min<int64_t>(iter, maxit);
      info[2] = done ? 1.0 : 0.0;
      info[3] = err;
    }
    if (!done) throw Error(TCI_ERR_INPUT, "tci_rhf: no convergence in " + std::to_string((long long)maxit) + " iterations");
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}

extern "C" int tci_mo_operator(const tci_integrals* it, const double* C, int64_t nmo, double* h, double* chol,
                               int64_t nchol) {
  try {
    if (!it || !C || !h || !chol) throw Error(TCI_ERR_ARG, "tci_mo_operator: null argument");
    const int n = it->nbf;
    if (nmo <= 0 || nmo > n || nchol != it->nchol) throw Error(TCI_ERR_ARG, "tci_mo_operator: size mismatch");
    const int m = (int)nmo;
    std::vector<double> S, T, V;
    it->one_electron(S, T, V);
    std::vector<double> hao((size_t)n * n), t1((size_t)m * n), hm((size_t)m * m);
    for (size_t i = 0; i < hao.size(); ++i) hao[i] = T[i] + V[i];
    // C is n x m row major: h_mo = C^T h C
    tci::matmul(m, n, n, C, hao.data(), t1.data(), true);
    tci::matmul(m, n, m, t1.data(), C, hm.data());
    std::memcpy(h, hm.data(), sizeof(double) * hm.size());
    const int64_t nc = it->nchol, mpair = (int64_t)m * (m + 1) / 2;
#pragma omp parallel
    {
      std::vector<double> Lf((size_t)n * n), Xj((size_t)m * n), Y((size_t)m * m);
#pragma omp for schedule(dynamic, 4)
      for (int64_t J = 0; J < nc; ++J) {
        for (int p = 0; p < n; ++p)
          for (int q = 0; q <= p; ++q)
            Lf[(size_t)p * n + q] = Lf[(size_t)q * n + p] = it->chol[(size_t)tci::pidx(p, q) * nc + J];
        tci::matmul(m, n, n, C, Lf.data(), Xj.data(), true);  // X = C^T L^J
        tci::matmul(m, n, m, Xj.data(), C, Y.data());         // Y = X C
        for (int p = 0; p < m; ++p)
          for (int q = 0; q <= p; ++q) chol[(size_t)tci::pidx(p, q) * nc + J] = Y[(size_t)p * m + q];
      }
    }
    (void)mpair;
    return TCI_OK;
  } catch (...) {
    return tci::guard_status(std::current_exception());
  }
}

extern "C" void tci_integrals_destroy(tci_integrals* it) { delete it; }
