/*
 * Oracle (test infrastructure only; never linked into the product).
 *
 * 1. Dense determinant Hamiltonian-vector product y = H x over an explicit list
 *    of Slater determinants (spin orbital 2p+sigma, at most 64 spin orbitals),
 *    by the Slater-Condon rules.  Used with the CSF <-> determinant map of
 *    oracle/dense.py to form sigma = H c in TigerCI's CSF basis for small cases.
 *
 * 2. The reference's all-external term in its integral-driven form
 *    (tiger_fortran/three_and_four_seg_mod_1.f90:318-632 and 3240-3518):
 *    for each external pair a >= c the (ab|cd) slab is formed from the
 *    Cholesky vectors (dgemm at mod_1:556) and every N-2 head whose domain
 *    holds a and c receives
 *      sigma_[ac] += sum_{b>d} C_[bd]((ab|cd) +- (ad|cb)) + sqrt2 sum_b C_bb (ab|cb)
 *      sigma_aa   += sqrt2 sum_{b>d} C_[bd](ab|ad) + sum_b C_bb (ab|ab)
 *    (singlet-coupled functions symmetric, triplet-coupled antisymmetric,
 *    mod_1:3354-3503).  Used as the CPU baseline of the all-external term.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

static inline int popc(uint64_t x) { return __builtin_popcountll(x); }
static inline int par_below(uint64_t d, int x) { return popc(d & ((x == 64) ? ~0ull : ((1ull << x) - 1))) & 1; }

/* eri[((p*n+q)*n+r)*n+s] = (pq|rs) */
static double sc_element(uint64_t di, uint64_t dj, int n, const double* h, const double* eri) {
  uint64_t diff = di ^ dj;
  int nd = popc(diff);
  if (nd > 4) return 0.0;
#define ERI(p, q, r, s) eri[(((int64_t)(p) * n + (q)) * n + (r)) * n + (s)]
  if (nd == 0) {
    double e = 0.0;
    for (int x = 0; x < 2 * n; ++x) {
      if (!((di >> x) & 1)) continue;
      int p = x >> 1;
      e += h[p * n + p];
      for (int y = 0; y < 2 * n; ++y) {
        if (!((di >> y) & 1)) continue;
        int q = y >> 1;
        e += 0.5 * ERI(p, p, q, q);
        if ((x & 1) == (y & 1)) e -= 0.5 * ERI(p, q, q, p);
      }
    }
    return e;
  }
  uint64_t ann = dj & diff; /* occupied in dj, empty in di */
  uint64_t cre = di & diff;
  if (nd == 2) {
    int a = __builtin_ctzll(ann), c = __builtin_ctzll(cre);
    if ((a & 1) != (c & 1)) return 0.0;
    int p = c >> 1, q = a >> 1;
    double v = h[p * n + q];
    for (int y = 0; y < 2 * n; ++y) {
      if (!((dj >> y) & 1) || y == a) continue;
      int r = y >> 1;
      v += ERI(p, q, r, r);
      if ((y & 1) == (a & 1)) v -= ERI(p, r, r, q);
    }
    /* phase of a+_c a_a on dj */
    uint64_t d = dj;
    int ph = par_below(d, a);
    d &= ~(1ull << a);
    ph ^= par_below(d, c);
    return ph ? -v : v;
  }
  /* double: a+_c a+_d a_b a_a with a<b (ann), c<d (cre) */
  int a = __builtin_ctzll(ann);
  int b = 63 - __builtin_clzll(ann);
  int c = __builtin_ctzll(cre);
  int dd = 63 - __builtin_clzll(cre);
  double v = 0.0;
  if ((c & 1) == (a & 1) && (dd & 1) == (b & 1)) v += ERI(c >> 1, a >> 1, dd >> 1, b >> 1);
  if ((c & 1) == (b & 1) && (dd & 1) == (a & 1)) v -= ERI(c >> 1, b >> 1, dd >> 1, a >> 1);
  if (v == 0.0) return 0.0;
  uint64_t d = dj;
  int ph = par_below(d, a);
  d &= ~(1ull << a);
  ph ^= par_below(d, b);
  d &= ~(1ull << b);
  ph ^= par_below(d, dd);
  d |= 1ull << dd;
  ph ^= par_below(d, c);
  return ph ? -v : v;
#undef ERI
}

/* y[i] += sum_j H[i][j] x[j] over the listed determinants */
void oracle_hdet_matvec(int64_t ndet, const uint64_t* dets, int n, const double* h, const double* eri,
                        const double* x, double* y) {
#pragma omp parallel for schedule(dynamic, 16)
  for (int64_t i = 0; i < ndet; ++i) {
    double acc = 0.0;
    for (int64_t j = 0; j < ndet; ++j) {
      if (x[j] == 0.0) continue;
      if (popc(dets[i] ^ dets[j]) > 4) continue;
      acc += sc_element(dets[i], dets[j], n, h, eri) * x[j];
    }
    y[i] += acc;
  }
}

/*
 * All-external sigma in the reference's integral-driven form for a non-local
 * space.  chol: [pair][J] with pair = p(p+1)/2+q (p>=q), external orbitals
 * nint..nint+n-1.  heads: nh records (off_ab, off_aa, nsf_ab, nsf_aa, nsing).
 * Loops over a (OpenMP, like mod_1:442-465) and c <= a, forms the slab
 * V[b][d] = (ab|cd) for all b, d, and applies it to every head.
 */
typedef void (*dgemm_fn)(const char*, const char*, const int*, const int*, const int*, const double*,
                         const double*, const int*, const double*, const int*, const double*, double*, const int*);
static dgemm_fn g_dgemm = 0;
/* Optional BLAS dgemm (Fortran ABI), e.g. scipy's bundled OpenBLAS, used for
 * the (ab|cd) slab like the reference's dgemm at mod_1:556. */
void oracle_set_dgemm(void* fn) { g_dgemm = (dgemm_fn)fn; }
dgemm_fn oracle_get_dgemm(void) { return g_dgemm; }

void oracle_allext_sigma(int64_t nint, int64_t n, int64_t nchol, const double* chol, int64_t nh,
                         const int64_t* heads, const double* c, double* sigma, int64_t a_begin, int64_t a_end) {
  const double s2 = sqrt(2.0);
  const int64_t nab = n * (n - 1) / 2;
#define PAIR(p, q) ((p) >= (q) ? (p) * ((p) + 1) / 2 + (q) : (q) * ((q) + 1) / 2 + (p))
#pragma omp parallel
  {
    double* Lab = (double*)malloc(sizeof(double) * n * nchol);
    double* Lcd = (double*)malloc(sizeof(double) * n * nchol);
    double* V = (double*)malloc(sizeof(double) * n * n);
    double* Vx = (double*)malloc(sizeof(double) * n * n);
#pragma omp for schedule(dynamic, 1)
    for (int64_t a = a_begin; a < a_end; ++a) {
      for (int64_t b = 0; b < n; ++b) memcpy(Lab + b * nchol, chol + PAIR(nint + a, nint + b) * nchol, sizeof(double) * nchol);
      for (int64_t cc = 0; cc <= a; ++cc) {
        for (int64_t d = 0; d < n; ++d) memcpy(Lcd + d * nchol, chol + PAIR(nint + cc, nint + d) * nchol, sizeof(double) * nchol);
        /* V[b][d] = (ab|cd) = sum_J Lab[b][J] Lcd[d][J]  (the dgemm of mod_1:556) */
        if (g_dgemm) {
          /* column-major view: V^T(d,b) = Lcd^T(d,J) Lab(J,b) */
          const int nn = (int)n, kk = (int)nchol;
          const double one = 1.0, zero = 0.0;
          g_dgemm("T", "N", &nn, &nn, &kk, &one, Lcd, &kk, Lab, &kk, &zero, V, &nn);
        } else {
          for (int64_t b = 0; b < n; ++b)
            for (int64_t d = 0; d < n; ++d) {
              const double* x = Lab + b * nchol;
              const double* y = Lcd + d * nchol;
              double acc = 0.0;
              for (int64_t J = 0; J < nchol; ++J) acc += x[J] * y[J];
              V[b * n + d] = acc;
            }
        }
        /* exchange slab (ad|cb) = V'[d][b] needs (ad|cb): for fixed a,c it is V transposed */
        for (int64_t b = 0; b < n; ++b)
          for (int64_t d = 0; d < n; ++d) Vx[b * n + d] = V[d * n + b];
        for (int64_t hh = 0; hh < nh; ++hh) {
          const int64_t* H = heads + 5 * hh;
          const int64_t off_ab = H[0], off_aa = H[1], nsf_ab = H[2], nsf_aa = H[3], nsing = H[4];
          const int64_t nk = nsf_ab > nsf_aa ? nsf_ab : nsf_aa;
          for (int64_t k = 0; k < nk; ++k) {
            const int singlet = k < nsing;
            const double* cab = (k < nsf_ab) ? c + off_ab + k * nab : NULL;
            const double* caa = (k < nsf_aa) ? c + off_aa + k * n : NULL;
            double acc = 0.0;
            if (a != cc) {
              if (!(k < nsf_ab)) continue;
              for (int64_t b = 1; b < n; ++b)
                for (int64_t d = 0; d < b; ++d) {
                  const double cv = cab[b * (b - 1) / 2 + d];
                  acc += cv * (singlet ? (V[b * n + d] + Vx[b * n + d]) : (V[b * n + d] - Vx[b * n + d]));
                }
              if (singlet && caa)
                for (int64_t b = 0; b < n; ++b) acc += s2 * caa[b] * V[b * n + b];
              /* sigma index of the pair (a, cc), a > cc; one writer per (a, cc) */
              sigma[off_ab + k * nab + a * (a - 1) / 2 + cc] += acc;
            } else {
              if (!singlet || !caa) continue;
              if (cab)
                for (int64_t b = 1; b < n; ++b)
                  for (int64_t d = 0; d < b; ++d) acc += s2 * cab[b * (b - 1) / 2 + d] * V[b * n + d];
              for (int64_t b = 0; b < n; ++b) acc += caa[b] * V[b * n + b];
              sigma[off_aa + k * n + a] += acc;
            }
          }
        }
      }
    }
    free(Lab);
    free(Lcd);
    free(V);
    free(Vx);
  }
#undef PAIR
}

/* Local (pair-domain) all-external sigma, integral form.  Same arithmetic as
 * oracle_allext_sigma, with every external index of head h restricted to its
 * domain dom[h] (sorted virtual indices; local index = position in the list),
 * as in ext_3_4_seg_loops_vec_lmo_res_2 (three_and_four_seg_mod_1.f90:3240-3518)
 * with virtual_truncation (locist_mod.f90:358-451).  heads: 7 int64 per head
 * (off_ab, off_aa, nsf_ab, nsf_aa, nsing, dom_off, dom_len); blocks of head h
 * have dom_len-sized external dimensions.  Heads [h_begin, h_end) only (a
 * sample).  The head loop is parallel: every head owns its sigma blocks. */
void oracle_allext_local_sigma(int64_t nint, int64_t nchol, const double* chol, int64_t nh, const int64_t* heads,
                               const int64_t* dom_idx, const double* c, double* sigma, int64_t h_begin,
                               int64_t h_end) {
  const double s2 = sqrt(2.0);
  int64_t nmax = 1;
  for (int64_t hh = 0; hh < nh; ++hh)
    if (heads[7 * hh + 6] > nmax) nmax = heads[7 * hh + 6];
#define PAIR(p, q) ((p) >= (q) ? (p) * ((p) + 1) / 2 + (q) : (q) * ((q) + 1) / 2 + (p))
#pragma omp parallel
  {
    double* Lab = (double*)malloc(sizeof(double) * nmax * nchol);
    double* Lcd = (double*)malloc(sizeof(double) * nmax * nchol);
    double* V = (double*)malloc(sizeof(double) * nmax * nmax);
    double* Vx = (double*)malloc(sizeof(double) * nmax * nmax);
#pragma omp for schedule(dynamic, 1)
    for (int64_t hh = h_begin; hh < h_end; ++hh) {
      const int64_t* H = heads + 7 * hh;
      const int64_t off_ab = H[0], off_aa = H[1], nsf_ab = H[2], nsf_aa = H[3], nsing = H[4];
      const int64_t* dom = dom_idx + H[5];
      const int64_t n = H[6], nab = n * (n - 1) / 2;
      const int64_t nk = nsf_ab > nsf_aa ? nsf_ab : nsf_aa;
      for (int64_t a = 0; a < n; ++a) {
        for (int64_t b = 0; b < n; ++b)
          memcpy(Lab + b * nchol, chol + PAIR(nint + dom[a], nint + dom[b]) * nchol, sizeof(double) * nchol);
        for (int64_t cc = 0; cc <= a; ++cc) {
          for (int64_t d = 0; d < n; ++d)
            memcpy(Lcd + d * nchol, chol + PAIR(nint + dom[cc], nint + dom[d]) * nchol, sizeof(double) * nchol);
          if (g_dgemm) {
            const int nn = (int)n, kk = (int)nchol;
            const double one = 1.0, zero = 0.0;
            g_dgemm("T", "N", &nn, &nn, &kk, &one, Lcd, &kk, Lab, &kk, &zero, V, &nn);
          } else {
            for (int64_t b = 0; b < n; ++b)
              for (int64_t d = 0; d < n; ++d) {
                const double* x = Lab + b * nchol;
                const double* y = Lcd + d * nchol;
                double acc = 0.0;
                for (int64_t J = 0; J < nchol; ++J) acc += x[J] * y[J];
                V[b * n + d] = acc;
              }
          }
          for (int64_t b = 0; b < n; ++b)
            for (int64_t d = 0; d < n; ++d) Vx[b * n + d] = V[d * n + b];
          for (int64_t k = 0; k < nk; ++k) {
            const int singlet = k < nsing;
            const double* cab = (k < nsf_ab) ? c + off_ab + k * nab : NULL;
            const double* caa = (k < nsf_aa) ? c + off_aa + k * n : NULL;
            double acc = 0.0;
            if (a != cc) {
              if (!(k < nsf_ab)) continue;
              for (int64_t b = 1; b < n; ++b)
                for (int64_t d = 0; d < b; ++d) {
                  const double cv = cab[b * (b - 1) / 2 + d];
                  acc += cv * (singlet ? (V[b * n + d] + Vx[b * n + d]) : (V[b * n + d] - Vx[b * n + d]));
                }
              if (singlet && caa)
                for (int64_t b = 0; b < n; ++b) acc += s2 * caa[b] * V[b * n + b];
              sigma[off_ab + k * nab + a * (a - 1) / 2 + cc] += acc;
            } else {
              if (!singlet || !caa) continue;
              if (cab)
                for (int64_t b = 1; b < n; ++b)
                  for (int64_t d = 0; d < b; ++d) acc += s2 * cab[b * (b - 1) / 2 + d] * V[b * n + d];
              for (int64_t b = 0; b < n; ++b) acc += caa[b] * V[b * n + b];
              sigma[off_aa + k * n + a] += acc;
            }
          }
        }
      }
    }
    free(Lab);
    free(Lcd);
    free(V);
    free(Vx);
  }
#undef PAIR
}

int oracle_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
