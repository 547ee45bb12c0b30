/*
 * Oracle (test and CPU-baseline infrastructure only; never linked into the
 * product).  A CPU sigma = H c of the whole MRSDCI space that follows the
 * reference's integral-direct cost structure, used as the timed CPU arm:
 *
 *  - every sigma build first forms its integrals from the Cholesky vectors,
 *    as the reference does for each htimesc call (tiger_fortran/htimesc.f90:
 *    46-147): the (ij|ab), (ia|jb) banks of the two-external loops
 *    (three_and_four_seg_mod_2.f90:1332-1336, dgemm/dgemv) and the (ia|bc)
 *    banks of the three-external loops (three_and_four_seg_mod_1.f90:
 *    1203-1288), by dgemm over the Cholesky rows;
 *  - the all-external term runs in the reference's loop form
 *    (oracle_allext_sigma in detci.c: one (ab|cd) slab per external pair a >= c
 *    formed by dgemm, mod_1:556, applied to every N-2 head, mod_1:3240-3518);
 *  - every other coupling (three-, two-, one- and zero-external loops,
 *    diagtimesc) is replayed from the loop records of an exported sigma plan
 *    (the records the reference enumerates in its iteration-1 dry run):
 *    dgemm for the integral-times-CI-block products, axpy / dot loops for the
 *    coupling-coefficient scatters and gathers, the SCEP unpack / pack of
 *    scepmaker_mod.f90:60-800.
 *
 * FP64 throughout; OpenMP over independent records (one writer per target
 * range), BLAS dgemm single-threaded inside each (scipy's bundled OpenBLAS,
 * set with oracle_set_dgemm).  The plan file layout is written by
 * tci_plan_export (tigerci_b200/plan_io.py documents it).
 */
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifdef _OPENMP
#include <omp.h>
#endif

typedef void (*dgemm_fn)(const char*, const char*, const int*, const int*, const int*, const double*,
                         const double*, const int*, const double*, const int*, const double*, double*, const int*);
extern void oracle_allext_sigma(int64_t nint, int64_t n, int64_t nchol, const double* chol, int64_t nh,
                                const int64_t* heads, const double* c, double* sigma, int64_t a_begin, int64_t a_end);
dgemm_fn oracle_get_dgemm(void);

enum { B_C = 0, B_S, B_D, B_R, B_T0, B_T1, B_T2, B_T3, B_JK, B_V, B_W, B_F, B_WV, B_L, B_LE, B_LV, B_LI, B_X, NB };
enum { K_GEMM = 0, K_AXPY, K_DOT, K_UNPACK, K_PACK, K_ZERO, K_WBUILD };

typedef struct { int64_t c, offC, ldc, M, N; double beta; int64_t s0, s1; } gp_t;
typedef struct { int64_t a, b, offA, lda, offB, ldb, K, tA, tB; double alpha; } gs_t;
typedef struct { int64_t dst, off, len, s0, s1; } at_t;
typedef struct { int64_t src, off; double coef; int64_t sbuf, sidx; } as_t;
typedef struct { int64_t dst, off, s0, s1; } dt_t;
typedef struct { int64_t a, b, aoff, boff, len; double coef; } ds_t;
typedef struct { int64_t off_ab, off_aa, nsf_ab, nsf_aa, nsing, nD, dk0; } dh_t;
typedef struct { int64_t off, len, type; double beta; int64_t foff, singlet; } dg_t;

typedef struct {
  int64_t kind;
  char name[64];
  int64_t ngp, ngs, nat, nas, ndt, nds, buf, off, len;
  gp_t* gp;
  gs_t* gs;
  at_t* at;
  as_t* as;
  dt_t* dt;
  ds_t* ds;
} step_t;

typedef struct {
  int64_t nint, n, nchol, total, npair, nD, ndh, ninit, nsig, nhvv, nwv, np, nm, ndiag;
  int64_t bufsz[NB];
  dh_t* dh;
  dg_t* dg;
  double* hvv;
  double* wv;
  step_t* init;
  step_t* sig;
  double* buf[NB];
  const double* chol;
  int64_t* heads5; /* off_ab, off_aa, nsf_ab, nsf_aa, nsing per head, for the loop-form all-external term */
  int64_t nheads5;
} plan_t;

static int rd(FILE* f, void* p, size_t n) { return fread(p, 1, n, f) == n ? 0 : -1; }

static int read_step(FILE* f, step_t* s) {
  if (rd(f, &s->kind, 8) || rd(f, s->name, 64)) return -1;
  int64_t h[9];
  if (rd(f, h, sizeof(h))) return -1;
  s->ngp = h[0], s->ngs = h[1], s->nat = h[2], s->nas = h[3], s->ndt = h[4], s->nds = h[5];
  s->buf = h[6], s->off = h[7], s->len = h[8];
#define RDARR(field, type, cnt)                                                  \
  s->field = (type*)malloc(sizeof(type) * ((cnt) > 0 ? (cnt) : 1));             \
  if ((cnt) > 0 && rd(f, s->field, sizeof(type) * (cnt))) return -1;
  RDARR(gp, gp_t, s->ngp)
  RDARR(gs, gs_t, s->ngs)
  RDARR(at, at_t, s->nat)
  RDARR(as, as_t, s->nas)
  RDARR(dt, dt_t, s->ndt)
  RDARR(ds, ds_t, s->nds)
#undef RDARR
  return 0;
}

static int is_allext(const step_t* s) { return strncmp(s->name, "all-external", 12) == 0; }

void plancpu_free(void* hp) {
  plan_t* p = (plan_t*)hp;
  if (!p) return;
  for (int b = 0; b < NB; ++b)
    if (b != B_L) free(p->buf[b]);
  step_t* lists[2] = {p->init, p->sig};
  int64_t counts[2] = {p->ninit, p->nsig};
  for (int l = 0; l < 2; ++l)
    for (int64_t i = 0; lists[l] && i < counts[l]; ++i) {
      step_t* s = &lists[l][i];
      free(s->gp), free(s->gs), free(s->at), free(s->as), free(s->dt), free(s->ds);
    }
  free(p->init), free(p->sig), free(p->dh), free(p->dg), free(p->hvv), free(p->wv), free(p->heads5);
  free(p);
}

/* Loads an exported plan and allocates its buffers, except the packed all-external operators (W, X), which
 * the loop-form all-external term does not use.  chol: the Cholesky vectors the plan was built for
 * ([pair][J]); kept by pointer.  Returns NULL on failure. */
void* plancpu_load(const char* path, const double* chol) {
  FILE* f = fopen(path, "rb");
  if (!f) return NULL;
  plan_t* p = (plan_t*)calloc(1, sizeof(plan_t));
  char magic[8];
  int64_t h[15];
  if (rd(f, magic, 8) || memcmp(magic, "TCIPLAN1", 8) || rd(f, h, sizeof(h))) goto fail;
  p->nint = h[0], p->n = h[1], p->nchol = h[2], p->total = h[3], p->npair = h[4], p->nD = h[5], p->ndh = h[6];
  if (h[7] != NB) goto fail;
  p->ninit = h[8], p->nsig = h[9], p->nhvv = h[10], p->nwv = h[11], p->np = h[12], p->nm = h[13], p->ndiag = h[14];
  if (rd(f, p->bufsz, sizeof(p->bufsz))) goto fail;
  p->dh = (dh_t*)malloc(sizeof(dh_t) * (p->ndh ? p->ndh : 1));
  if (p->ndh && rd(f, p->dh, sizeof(dh_t) * p->ndh)) goto fail;
  if (fseek(f, 8 * p->nD, SEEK_CUR)) goto fail; /* dk signs */
  p->hvv = (double*)malloc(8 * (p->nhvv ? p->nhvv : 1));
  p->wv = (double*)malloc(8 * (p->nwv ? p->nwv : 1));
  if ((p->nhvv && rd(f, p->hvv, 8 * p->nhvv)) || (p->nwv && rd(f, p->wv, 8 * p->nwv))) goto fail;
  p->dg = (dg_t*)malloc(sizeof(dg_t) * (p->ndiag ? p->ndiag : 1));
  if (p->ndiag && rd(f, p->dg, sizeof(dg_t) * p->ndiag)) goto fail;
  p->init = (step_t*)calloc(p->ninit ? p->ninit : 1, sizeof(step_t));
  p->sig = (step_t*)calloc(p->nsig ? p->nsig : 1, sizeof(step_t));
  for (int64_t i = 0; i < p->ninit; ++i)
    if (read_step(f, &p->init[i])) goto fail;
  for (int64_t i = 0; i < p->nsig; ++i)
    if (read_step(f, &p->sig[i])) goto fail;
  fclose(f);
  f = NULL;
  for (int b = 0; b < NB; ++b) {
    if (b == B_W || b == B_X || b == B_L) continue;
    const int64_t sz = p->bufsz[b] > 0 ? p->bufsz[b] : 1;
    p->buf[b] = (double*)calloc((size_t)sz, 8);
    if (!p->buf[b]) goto fail;
  }
  p->chol = chol;
  p->buf[B_L] = (double*)chol;
  p->heads5 = (int64_t*)malloc(sizeof(int64_t) * 5 * (p->ndh ? p->ndh : 1));
  for (int64_t i = 0; i < p->ndh; ++i) {
    const dh_t* d = &p->dh[i];
    int64_t* o = p->heads5 + 5 * p->nheads5;
    if (d->nsf_ab == 0 && d->nsf_aa == 0) continue;
    o[0] = d->nsf_ab ? d->off_ab : -1;
    o[1] = d->nsf_aa ? d->off_aa : -1;
    o[2] = d->nsf_ab, o[3] = d->nsf_aa, o[4] = d->nsing;
    ++p->nheads5;
  }
  return p;
fail:
  if (f) fclose(f);
  plancpu_free(p);
  return NULL;
}

/* Rows [i0, i1) of C (M x N, row major) = beta C + sum over segments alpha op(A) op(B), by column-major dgemm
 * on the transposes (C^T = op(B)^T op(A)^T). */
static void run_gemm_rows(plan_t* p, const step_t* s, const gp_t* g, int64_t i0, int64_t i1, dgemm_fn dg) {
  /* products into or out of the packed all-external operators (not allocated here: the loop form forms
   * its (ab|cd) slabs itself) are left out */
  if (!p->buf[g->c]) return;
  for (int64_t k = g->s0; k < g->s1; ++k)
    if (!p->buf[s->gs[k].a] || !p->buf[s->gs[k].b]) return;
  double* C = p->buf[g->c] + g->offC + i0 * g->ldc;
  const int64_t rows = i1 - i0;
  if (rows <= 0 || g->N == 0) return;
  if (g->beta == 0.0)
    for (int64_t i = 0; i < rows; ++i) memset(C + i * g->ldc, 0, 8 * (size_t)g->N);
  else if (g->beta != 1.0)
    for (int64_t i = 0; i < rows; ++i)
      for (int64_t j = 0; j < g->N; ++j) C[i * g->ldc + j] *= g->beta;
  for (int64_t k = g->s0; k < g->s1; ++k) {
    const gs_t* q = &s->gs[k];
    if (q->K == 0) continue;
    const double* A = p->buf[q->a] + q->offA + (q->tA ? i0 : i0 * q->lda);
    const double* B = p->buf[q->b] + q->offB;
    if (dg) {
      const int m = (int)g->N, n = (int)rows, kk = (int)q->K, lda = (int)q->lda, ldb = (int)q->ldb,
                ldc = (int)g->ldc;
      const double one = 1.0;
      dg(q->tB ? "T" : "N", q->tA ? "T" : "N", &m, &n, &kk, &q->alpha, B, &ldb, A, &lda, &one, C, &ldc);
    } else {
      for (int64_t i = 0; i < rows; ++i)
        for (int64_t j = 0; j < g->N; ++j) {
          double acc = 0.0;
          for (int64_t l = 0; l < q->K; ++l) {
            const double a = q->tA ? A[l * q->lda + i] : A[i * q->lda + l];
            const double b = q->tB ? B[j * q->ldb + l] : B[l * q->ldb + j];
            acc += a * b;
          }
          C[i * g->ldc + j] += q->alpha * acc;
        }
    }
  }
}

static void run_step(plan_t* p, const step_t* s, dgemm_fn dg) {
  const int64_t n = p->n, nab = n * (n - 1) / 2;
  const double s2 = sqrt(2.0);
  switch (s->kind) {
    case K_ZERO:
      if (p->buf[s->buf]) memset(p->buf[s->buf] + s->off, 0, 8 * (size_t)s->len);
      break;
    case K_GEMM: {
      /* few problems: split their rows so that every thread has work */
      int nthr = 1;
#ifdef _OPENMP
      nthr = omp_get_max_threads();
#endif
      int64_t split = 1;
      if (s->ngp < 4 * nthr) split = (4 * nthr + s->ngp - 1) / s->ngp;
      const int64_t ntask = s->ngp * split;
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t t = 0; t < ntask; ++t) {
        const gp_t* g = &s->gp[t / split];
        const int64_t part = t % split, chunk = (g->M + split - 1) / split;
        const int64_t i0 = part * chunk, i1 = (i0 + chunk < g->M) ? i0 + chunk : g->M;
        run_gemm_rows(p, s, g, i0, i1, dg);
      }
      break;
    }
    case K_AXPY:
#pragma omp parallel for schedule(dynamic, 16)
      for (int64_t t = 0; t < s->nat; ++t) {
        const at_t* T = &s->at[t];
        double* dst = p->buf[T->dst] + T->off;
        for (int64_t k = T->s0; k < T->s1; ++k) {
          const as_t* A = &s->as[k];
          const double c = A->coef * (A->sbuf >= 0 ? p->buf[A->sbuf][A->sidx] : 1.0);
          const double* src = p->buf[A->src] + A->off;
          for (int64_t i = 0; i < T->len; ++i) dst[i] += c * src[i];
        }
      }
      break;
    case K_DOT:
#pragma omp parallel for schedule(dynamic, 16)
      for (int64_t t = 0; t < s->ndt; ++t) {
        const dt_t* T = &s->dt[t];
        double tot = 0.0;
        for (int64_t k = T->s0; k < T->s1; ++k) {
          const ds_t* D = &s->ds[k];
          const double* a = p->buf[D->a] + D->aoff;
          const double* b = p->buf[D->b] + D->boff;
          double acc = 0.0;
          for (int64_t i = 0; i < D->len; ++i) acc += a[i] * b[i];
          tot += D->coef * acc;
        }
        p->buf[T->dst][T->off] += tot;
      }
      break;
    case K_UNPACK: {
      const double* c = p->buf[B_C];
      double* D = p->buf[B_D];
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t hh = 0; hh < p->ndh; ++hh) {
        const dh_t* h = &p->dh[hh];
        for (int64_t k = 0; k < h->nD; ++k) {
          double* M = D + (h->dk0 + k) * n * n;
          memset(M, 0, 8 * (size_t)(n * n));
          const double ph = k < h->nsing ? 1.0 : -1.0;
          if (k < h->nsf_ab) {
            const double* seg = c + h->off_ab + k * nab;
            for (int64_t i = 1; i < n; ++i)
              for (int64_t j = 0; j < i; ++j) {
                const double v = seg[i * (i - 1) / 2 + j];
                M[j * n + i] = v;
                M[i * n + j] = ph * v;
              }
          }
          if (k < h->nsf_aa)
            for (int64_t a = 0; a < n; ++a) M[a * n + a] = s2 * c[h->off_aa + k * n + a];
        }
      }
      break;
    }
    case K_PACK: {
      const double* R = p->buf[B_R];
      double* S = p->buf[B_S];
#pragma omp parallel for schedule(dynamic, 1)
      for (int64_t hh = 0; hh < p->ndh; ++hh) {
        const dh_t* h = &p->dh[hh];
        for (int64_t k = 0; k < h->nD; ++k) {
          const double* M = R + (h->dk0 + k) * n * n;
          const double ph = k < h->nsing ? 1.0 : -1.0;
          if (k < h->nsf_ab) {
            double* seg = S + h->off_ab + k * nab;
            for (int64_t i = 1; i < n; ++i)
              for (int64_t j = 0; j < i; ++j) seg[i * (i - 1) / 2 + j] += M[j * n + i] + ph * M[i * n + j];
          }
          if (k < h->nsf_aa)
            for (int64_t a = 0; a < n; ++a) S[h->off_aa + k * n + a] += s2 * M[a * n + a];
        }
      }
      break;
    }
    default:
      break;
  }
}

/* Forms the integral banks from the Cholesky vectors (the plan's set-up steps other than the packed
 * all-external operators), as the reference does at every sigma build. */
void plancpu_integrals(void* hp) {
  plan_t* p = (plan_t*)hp;
  dgemm_fn dg = oracle_get_dgemm();
  /* the set-up steps accumulate into their targets: start every derived buffer from zero */
  for (int b = 0; b < NB; ++b)
    if (b != B_L && b != B_C && b != B_S && p->buf[b] && p->bufsz[b] > 0) memset(p->buf[b], 0, 8 * (size_t)p->bufsz[b]);
  memcpy(p->buf[B_JK] + 2 * p->nint * p->nint * p->n * p->n, p->hvv, 8 * (size_t)p->nhvv);
  if (p->nwv) memcpy(p->buf[B_WV], p->wv, 8 * (size_t)p->nwv);
  for (int64_t i = 0; i < p->ninit; ++i)
    if (p->init[i].kind != K_WBUILD) run_step(p, &p->init[i], dg);
}

/* sigma += H c (host arrays of total_csfs).  integrals != 0 forms the integral banks first (one complete
 * integral-direct sigma build); the all-external term runs in the loop form. */
void plancpu_sigma(void* hp, const double* c, double* sigma, int integrals) {
  plan_t* p = (plan_t*)hp;
  dgemm_fn dg = oracle_get_dgemm();
  if (integrals) plancpu_integrals(hp);
  memcpy(p->buf[B_C], c, 8 * (size_t)p->total);
  memset(p->buf[B_S], 0, 8 * (size_t)p->total);
  for (int64_t i = 0; i < p->nsig; ++i)
    if (!is_allext(&p->sig[i])) run_step(p, &p->sig[i], dg);
  oracle_allext_sigma(p->nint, p->n, p->nchol, p->chol, p->nheads5, p->heads5, c, p->buf[B_S], 0, p->n);
  for (int64_t i = 0; i < p->total; ++i) sigma[i] += p->buf[B_S][i];
}

int64_t plancpu_total(void* hp) { return ((plan_t*)hp)->total; }

/* Diagonal H_ii (the preconditioner of Davidson, diag_element_mod_2.f90:83) from the plan's diagonal
 * entries: zero-external part beta plus the same-head operators F (formed by plancpu_integrals) and the
 * all-external diagonal (aa|aa), (aa|cc) +- (ac|ca) from the Cholesky vectors. */
void plancpu_diag(void* hp, double* out) {
  plan_t* p = (plan_t*)hp;
  const int64_t n = p->n, nint = p->nint, nc = p->nchol;
  const double* F = p->buf[B_F];
#define PIDX(x, y) ((x) >= (y) ? (x) * ((x) + 1) / 2 + (y) : (y) * ((y) + 1) / 2 + (x))
  double* aacc = (double*)malloc(sizeof(double) * n * n); /* (aa|cc) */
  double* acca = (double*)malloc(sizeof(double) * n * n); /* (ac|ca) */
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t a = 0; a < n; ++a)
    for (int64_t c = 0; c < n; ++c) {
      const double* la = p->chol + PIDX(nint + a, nint + a) * nc;
      const double* lc = p->chol + PIDX(nint + c, nint + c) * nc;
      const double* lx = p->chol + PIDX(nint + a, nint + c) * nc;
      double s1 = 0.0, s2 = 0.0;
      for (int64_t J = 0; J < nc; ++J) s1 += la[J] * lc[J], s2 += lx[J] * lx[J];
      aacc[a * n + c] = s1;
      acca[a * n + c] = s2;
    }
#undef PIDX
  for (int64_t k = 0; k < p->ndiag; ++k) {
    const dg_t* d = &p->dg[k];
    double* o = out + d->off;
#define FD(a) (d->foff >= 0 ? F[d->foff + (a) * (n + 1)] : 0.0)
    if (d->type == 0) {
      o[0] = d->beta;
    } else if (d->type == 1) {
      for (int64_t a = 0; a < n; ++a) o[a] = d->beta + FD(a);
    } else if (d->type == 2) {
      for (int64_t a = 0; a < n; ++a) o[a] = d->beta + 2.0 * FD(a) + aacc[a * n + a];
    } else {
      int64_t e = 0;
      for (int64_t i = 1; i < n; ++i)
        for (int64_t j = 0; j < i; ++j, ++e)
          o[e] = d->beta + FD(i) + FD(j) + aacc[i * n + j] + (d->singlet ? 1.0 : -1.0) * acca[i * n + j];
    }
#undef FD
  }
  free(aacc);
  free(acca);
}
