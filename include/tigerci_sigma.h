/*
 * tigerci_sigma.h - C ABI of the B200 sigma-vector build for TigerCI's
 * multireference singles-and-doubles CI (MRSDCI).
 *
 * All integers are int64_t (TigerCI is compiled with -fdefault-integer-8,
 * tiger_ci/CMakeLists.txt:39), all reals are double.  Every entry point that
 * returns int returns 0 on success and a non-zero TCI_ERR_* code otherwise; it
 * never aborts the process.  The message of the last failure on the calling
 * thread is available from tci_last_error().  Contexts are owned by the
 * library and are not thread-safe: use one context per stream / request.
 */
#ifndef TIGERCI_SIGMA_H
#define TIGERCI_SIGMA_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define TCI_OK 0
#define TCI_ERR_ARG 1      /* bad argument (null pointer, size mismatch)          */
#define TCI_ERR_CUDA 2     /* CUDA runtime failure or no usable device            */
#define TCI_ERR_INPUT 3    /* input deck / operator inconsistent or unsupported   */
#define TCI_ERR_INTERNAL 4 /* internal consistency check failed                   */
#define TCI_ERR_MEMORY 5   /* device or host allocation failed / over budget      */
#define TCI_ERR_TIMEOUT 6  /* a bounded device wait gave up                       */
#define TCI_ERR_CANCELLED 7 /* the caller cancelled the solve                     */

typedef struct tci_space tci_space;
typedef struct tci_plan tci_plan;
typedef struct tci_ctx tci_ctx;

/* Input keywords that define the CSF space (tc/InputReader.cpp:36-196):
 * NUMBER OF ORBITALS / FROZEN / INACTIVE / ACTIVE ORBITALS, NUMBER OF
 * ELECTRONS, SPIN MULTIPLICITY, NUMBER OF REFERENCES, REFERENCE OCCUPATIONS.
 * Optional local pair domains (allowed virtuals per internal path, the data of
 * tiger_fortran/allowed_virtuals_mod.f90) are given in CSR form over the N-1
 * and N-2 paths in lexical order, external indices 0-based and sorted; a path
 * whose list is the single entry -1 is removed.  NULL pointers mean non-local. */
typedef struct tci_deck {
  int64_t num_orbitals;
  int64_t num_frozen;
  int64_t num_inactive;
  int64_t num_active;
  int64_t num_elec;
  int64_t spin_mult;
  int64_t num_ref;
  const int64_t* ref_occ; /* num_ref x (num_inactive + num_active), row major */
  const int64_t* nm1_domain_ptr;
  const int64_t* nm1_domain_idx;
  const int64_t* nm2_domain_ptr;
  const int64_t* nm2_domain_idx;
} tci_deck;

/* Molecular-orbital Hamiltonian.  h is num_orbitals x num_orbitals (symmetric,
 * row major).  chol holds the Cholesky vectors in the layout of TigerCI's
 * cholesky_data%cho_vectors(numcho, npair) (tiger_fortran/cholesky_structs.f90:35-39):
 * element (J, pq) at chol[pq * nchol + J] with pq = p(p+1)/2 + q, p >= q,
 * 0-based orbitals, so that (pq|rs) = sum_J L^J_pq L^J_rs. */
typedef struct tci_operator {
  const double* h;
  const double* chol;
  int64_t nchol;
  double core_energy;
} tci_operator;

/* Thread-local message of the last failure (empty string if none). */
int tci_last_error(char* buf, int64_t len);

/* The tci_operator chol array from Cholesky records addressed through
 * TigerCI's cholesky_data%mo_ind_inv (tiger_fortran/cholesky_structs.f90;
 * read as cho_vectors(:, mo_ind_inv(pq)) with 0 meaning a zero vector, e.g.
 * three_and_four_seg_mod_1.f90:504-512, and restored from CD_restart by
 * cholesky_transform.f90:234-244): mo_ind_inv[pq] (pq = p(p+1)/2 + q,
 * 0-based, num_orbitals(num_orbitals+1)/2 entries) is the 1-based record of
 * pair pq in records (n_records x nchol, row major) or 0.  chol_out gets
 * npair x nchol.  TCI_ERR_INPUT for an entry outside 0..n_records.  Where
 * mo_ind_inv is the identity (the reference's transforms write it so) the
 * records are the chol array as they are. */
int tci_operator_from_records(int64_t num_orbitals, int64_t nchol, const int64_t* mo_ind_inv, const double* records,
                              int64_t n_records, double* chol_out);

/* ---- CSF space (host only; no GPU needed) --------------------------------
 * Replaces graph_driver (tiger_fortran/graph_mod.f90:48-99): distinct-row
 * table, tree search and CI-vector index vectors. */
int tci_space_create(const tci_deck* deck, tci_space** out);
/* out[0..11]: total_csfs, num_valence, num_nm1, num_nm2, total_configurations,
 * removed, open_shells, paths(N), paths(N-1), paths(N-2), num_vertices, n_domains */
int tci_space_counts(const tci_space* sp, int64_t* out, int64_t len);
/* Index vector of kind 0 (valence, internal_index_vector0), 1 (N-1, vector1),
 * 2 (N-2 "ab", vector2) or 3 (N-2 "aa", vector3): 1-based CSF offsets as in the
 * reference, kill_number (-1000000) for removed paths.  len = number of paths. */
int tci_space_index_vector(const tci_space* sp, int64_t kind, int64_t* out, int64_t len);
/* Occupation (num_internal entries) and info[0..5] = lex, singles, kept, nsf,
 * nsf_aa, n_virtuals of path lex (1-based) of kind 0/1/2. */
int tci_space_path(const tci_space* sp, int64_t kind, int64_t lex, int64_t* occ, int64_t* info);
/* Number of "For s singles there are f spinfunctions and c configurations"
 * entries of block kind (0 valence, 1 N-1, 2 N-2), written as (s, f, c) triples. */
int tci_space_block_counts(const tci_space* sp, int64_t kind, int64_t* out, int64_t max_triples, int64_t* n_triples);
void tci_space_destroy(tci_space* sp);
/* Diagonal metric G of the (MR)ACPF / ACPF-2 / (MR)AQCC functionals, replacing
 * build_compressed_g (tiger_fortran/gtimesc.f90:37-55): get_gvalues (:316-378)
 * for flag 1 ACPF, 2 ACPF-2, 3 AQCC, 4 custom (g3 = g4 = custom_g), 9 test
 * (all ones), and build_g_diagonal (:106-201) for the CSF classes: valence
 * CSFs of a reference configuration (g1), other valence CSFs with the inactive
 * orbitals full (g2), valence CSFs with an inactive hole (g3), N-1 (g4), N-2
 * (g5).  g gets n = total_csfs values; cls (may be NULL) the class 1..5. */
int tci_acpf_gdiag(const tci_space* sp, int64_t flag, double custom_g, double* g, int64_t* cls, int64_t n);

/* ---- Sigma plan (host only) ------------------------------------------------
 * Replaces the iteration-1 loop enumeration ("dry run") of the sigma build:
 * every coupling coefficient and task table, built once. */
int tci_plan_create(const tci_deck* deck, const tci_operator* op, tci_plan** out);
/* Writes the plan as a flat binary file (layout: tigerci_b200/plan_io.py). */
int tci_plan_export(const tci_plan* plan, const char* path);
/* out[0..7]: total_csfs, n_dense, n_singlet, n_triplet, flops_allext,
 * flops_total, bytes_allext, n_steps; when len >= 10 also out[8] = peak
 * device bytes of tci_sigma_init (FP64 form) and out[9] = device bytes held
 * after it.  Host only: used to admit requests against a memory budget. */
int tci_plan_stats(const tci_plan* plan, double* out, int64_t len);
void tci_plan_destroy(tci_plan* plan);

/* ---- Device sigma build ------------------------------------------------------
 * Replaces htimesc(civec, sigmavec, data) (tiger_fortran/htimesc.f90:46-147).
 * tci_sigma_init uploads the operator, builds the integral banks and the plan on
 * `device`.  tci_sigma accumulates sigma += H c exactly like htimesc (the caller
 * zeroes sigma, tiger_fortran/davidson.f90:126); c and sigma are host arrays of
 * length total_csfs.  tci_sigma_device does the same on device arrays, ordered
 * after prior work on the given cudaStream_t and before later work on it
 * (NULL = the legacy default stream). */
int tci_sigma_init(const tci_deck* deck, const tci_operator* op, int64_t device, tci_ctx** out);
/* As tci_sigma_init with options: options[0] = precision mode, 0 plain FP64
 * (default), 1 mixed (TCI_PRECISION_TF32X3): the integral contractions run on
 * the tcgen05 tensor cores as 3xTF32 split products with FP32 accumulation
 * promoted to FP64 every options[1] k elements (multiple of 32, default 128):
 * the all-external term with FP32 W operators, and the three-, two- and
 * one-external GEMM steps from their FP64 operands.  options[2] selects those
 * other GEMM steps: 0 by size (default), 1 all of them, 2 none.  The coupling-
 * coefficient products, same-head one-electron-like operators (on the
 * tensor cores in the two-external step when options[3] != 0), gathers,
 * scatters and reductions stay FP64.  options[3] picks how tci_davidson
 * reports the roots of the mixed form: 2 (default) as the Rayleigh quotient of
 * each Ritz vector with one sigma build in which every term is FP64 but the
 * all-external one, which stays on its tensor-core kernel (the FP64 W is
 * released after the diagonal is built); 1 the same with a plain-FP64 sigma
 * build (the FP64 W stays resident); 3 as 2 with the three-external
 * contractions on the tensor cores too; 0 the mixed Ritz values.  The finished
 * root's error is second order in the eigenvector error of the mixed products
 * plus, for 2 and 3, the first-order error of the terms left on the tensor
 * cores.  In modes 0, 2 and 3 the set-up exchange product of the all-external
 * operators runs on the tensor cores as well (3xTF32, FP64 promotion). */
#define TCI_PRECISION_FP64 0
#define TCI_PRECISION_TF32X3 1
int tci_sigma_init_ex(const tci_deck* deck, const tci_operator* op, int64_t device, const int64_t* options,
                      int64_t n_options, tci_ctx** out);
int tci_sigma(tci_ctx* ctx, const double* c, double* sigma, int64_t n);
int tci_sigma_device(tci_ctx* ctx, const double* d_c, double* d_sigma, int64_t n, void* stream);
/* Diagonal H_ii (tiger_fortran/diag_element_mod_2.f90:83) for the
 * preconditioner, host array of length total_csfs. */
int tci_diag(tci_ctx* ctx, double* hdiag, int64_t n);
/* Device-resident Davidson-Liu solve for the nroots lowest roots (replaces
 * davidson_liu, tiger_fortran/davidson.f90:47-239, with the expansion and
 * sigma vectors kept in HBM instead of on disk).  Converges a root when the
 * residual norm drops below tol_residual (RESIDUAL TOLERANCE) or the energy
 * change below tol_energy (ENERGY TOLERANCE); maxit <= 0 means 50 * nroots.
 * energies[nroots] receives the eigenvalues of H (without the core energy);
 * vectors (nroots x total_csfs, may be NULL) the normalised eigenvectors. */
int tci_davidson(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                 double* energies, double* vectors, int64_t* iterations);
/* tci_davidson with a subspace memory budget and cancellation.
 * subspace_bytes plays the role of DAVIDSON HARD DRIVE SPACE
 * (tiger_cpp/InputReader.cpp:76, 30 GB when 0): once the subspace holds more
 * than 4 vectors per root and its c and H c vectors need that many bytes, it
 * restarts from the current and previous Ritz vectors of each root
 * (restart_davidson_subspace, tiger_fortran/davidson_restart.f90:26-139).
 * cancel (may be NULL) is polled at every iteration; a non-zero value ends
 * the solve with TCI_ERR_CANCELLED.  tci_davidson_bytes gives the device bytes
 * such a solve allocates (host only), tci_davidson_capacity its vector count. */
int tci_davidson_ex(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                    int64_t subspace_bytes, const int32_t* cancel, double* energies, double* vectors,
                    int64_t* iterations);
int64_t tci_davidson_capacity(int64_t n, int64_t nroots, int64_t maxit, int64_t subspace_bytes);
/* Generalized eigenproblem of the ACPF-type functionals, replacing
 * davidson_liu_gen_eig (tiger_fortran/davidson.f90:253-469):
 * (H - e_shift) c = lambda G c with G = diag(g) (host array of total_csfs
 * positive values, e.g. from tci_acpf_gdiag) and e_shift the reference energy.
 * Solved as the standard problem of G^-1/2 (H - e_shift) G^-1/2 (y = G^1/2 c)
 * by the device Davidson of tci_davidson_ex (same budget, mixed form and
 * finish); the residual norm tested against tol_residual is the reference's,
 * |(H - e_shift) c - lambda G c| with c of unit G-norm (build_residual_gen_eig,
 * tiger_fortran/davidson.f90:535-553), and roots are followed by their
 * overlap with their initial guess (root_following, davidson.f90:732, on by
 * default in the reference: NO ACPF ROOT FOLLOW unset).  energies get lambda + e_shift; vectors (may be NULL) the
 * unit-norm c of each root.  For the length of the call the context's
 * diagonal and sigma build stand for the transformed operator, so no other
 * call may use the same context (from another thread) until it returns. */
int tci_davidson_gen(tci_ctx* ctx, int64_t nroots, double tol_residual, double tol_energy, int64_t maxit,
                     const double* g, double e_shift, double* energies, double* vectors, int64_t* iterations);
int64_t tci_davidson_bytes(int64_t n, int64_t nroots, int64_t maxit, int64_t subspace_bytes);
/* Batched projections for a caller-driven Davidson with device-resident vectors
 * (expand_krylov_subspace / orthonormalize_vector, tiger_fortran/davidson.f90:478,
 * 702): d_out[k] = sum_i d_A[k*lda + i] * d_x[i] for k < m, all device arrays,
 * ordered on `stream` (NULL = legacy default stream).  Deterministic
 * fixed-order reduction; scratch is owned by the context. */
int tci_dots(tci_ctx* ctx, const double* d_A, int64_t lda, int64_t m, const double* d_x, int64_t n, double* d_out,
             void* stream);
/* tci_dots without device allocation, for callers that cannot call cudaMalloc
 * when they need projections: a solver loop being recorded into a CUDA graph,
 * a latency-bound service loop that must avoid cudaMalloc/cudaFree's implicit
 * device synchronisation, or a program whose GPU memory is fully handed out
 * by an admission budget or another allocator.  No counterpart in the
 * reference (its projections run on the host, tiger_fortran/davidson.f90).
 * Needs no context.  At most TCI_DOTS_NOALLOC_MAX_ROWS rows per call (larger m
 * returns TCI_ERR_ARG).  The partial sums live in one fixed device array
 * (TCI_DOTS_NOALLOC_MAX_ROWS x 592 doubles, 303 KB) that each GPU loading the
 * library holds until exit.  Every call shares it and overwrites what it
 * reads, so calls whose kernels overlap on a GPU race.  The first call on a
 * device looks the array's address up (cudaGetSymbolAddress), so make it
 * before any stream capture.  The address belongs to the CUDA context current
 * at that call; a call under another context of the device (after a
 * cudaDeviceReset, or a driver-API context of the caller's) looks it up again. */
#define TCI_DOTS_NOALLOC_MAX_ROWS 64
int tci_dots_noalloc(const double* d_A, int64_t lda, int64_t m, const double* d_x, int64_t n, double* d_out,
                     void* stream);
/* out[0..10]: total_csfs, device bytes held, init seconds, last sigma ms,
 * flops per sigma, all-external flops, all-external bytes, sigma builds,
 * kernel launches per sigma build (out[8], when len >= 9), kernels launched
 * by this context so far (out[9], when len >= 10), 1 if the last Davidson
 * solve met its residual or energy tolerance for every root before maxit,
 * else 0 (out[10], when len >= 11) */
int tci_ctx_stats(const tci_ctx* ctx, double* out, int64_t len);
/* Per-step CUDA-event timing of the sigma plan (off by default).  When on,
 * every sigma build records an event pair around each plan step on the
 * context's stream; tci_step_times returns the accumulated milliseconds per
 * step and the number of profiled builds since tci_profile was called. */
/* Waits for the context's stream and reports a device-side failure recorded
 * by a bounded wait (TCI_ERR_TIMEOUT), else 0. */
int tci_check(tci_ctx* ctx);
/* on: bit 0 times the sigma plan steps (tci_step_times); bit 1 times the
 * phases of tci_davidson / tci_davidson_ex (synchronising the stream at each
 * phase boundary), read with tci_davidson_phase_times: ms[8] = set-up, sigma,
 * projections, subspace eigensolve, residual, preconditioner + Gram-Schmidt,
 * restart, finish.  Both reset the accumulated times. */
int tci_profile(tci_ctx* ctx, int64_t on);
int tci_davidson_phase_times(const tci_ctx* ctx, double* ms, int64_t len);
int tci_step_times(const tci_ctx* ctx, double* ms, int64_t len, int64_t* nsteps, int64_t* nbuilds);
int tci_step_name(const tci_ctx* ctx, int64_t i, char* buf, int64_t len);
void tci_destroy(tci_ctx* ctx);

/* Self-test of the tensor-core kernels' abort path: a one-CTA kernel waits,
 * with the kernels' own bounded mbarrier wait, on a barrier that nothing
 * arrives at; after `polls` polls (0: the kernels' own limit) it records the
 * stalled-operand code in its status word and returns, and the host reports
 * TCI_ERR_TIMEOUT with *status_out the code and *ms_out (may be NULL) the
 * kernel's duration.  The context stays usable. */
int tci_selftest_bounded_wait(int64_t device, int64_t polls, int64_t* status_out, double* ms_out);
/* Instruction rate of tcgen05.mma kind::tf32 (M = m: 64 or 128; N = n:
 * 16..256 in steps of 16, or 8..256 in steps of 8 for M = 64; K = 8) on this
 * device: one thread per SM issues iters x nacc MMAs back to back into nacc
 * independent TMEM accumulators (nacc x n <= 512 columns, nacc x 2 n for
 * M = 64) and commits once;
 * *cycles_per_mma = the slowest SM's clock64 span / (iters x nacc), from the
 * second of two launches. */
int tci_selftest_mma_rate(int64_t device, int64_t m, int64_t n, int64_t nacc, int64_t iters, double* cycles_per_mma);

/* ---- A posteriori corrections (calculate_a_posteriori_corrections,
 * tiger_fortran/aposteriori.f90:28-221, called after a one-root SDCI solve,
 * driver_sdci.f90:73).  tci_reference_weight: c0^2 = sum of c_i^2 over the
 * CSFs of the reference configurations (no external electron) of a
 * space-length vector.  tci_aposteriori: out[5] = the Davidson, renormalised
 * Davidson, Davidson-Silver, Meissner and Pople corrections for correlation
 * energy e_corr (total - reference energy), c0^2 and n_corr_elec correlated
 * electrons (num_elec - 2 num_frozen); TCI_ERR_INPUT below 4 electrons (the
 * reference prints none there) or outside 1/2 < c0^2 <= 1. */
int tci_reference_weight(const tci_space* s, const double* c, int64_t n, double* c0sq);
int tci_aposteriori(int64_t n_corr_elec, double c0sq, double e_corr, double* out, int64_t len);

/* ---- The loop records of the local all-external term (host only) ---------
 * The reference enumerates the local all-external loops in a dry run before
 * the first iteration (all_external_3_4_loops_cho_2's first pass,
 * tiger_fortran/three_and_four_seg_mod_1.f90:414-436, records written by
 * build_ext_34seg_dryrun, :3142-3238): for each external pair a >= c
 * (absolute orbital numbers from 1) and each N-2 internal path whose domain
 * holds both, one record.  tci_local_allext_records writes the records of
 * the heads and domains this library's pair-domain term applies (the heads
 * tci_sigma_init builds for a deck with domains), 8 int64 each:
 * icount = a (a - 1) / 2 + c, head weight (lexical index - 1), ab address and
 * aa address (1-based CI offsets of the head's blocks, 0 for an absent
 * block), aa and ab spin functions, and the positions of a and c in the
 * domain (from 1), heads in the library's order, pairs a >= c within each.
 * *count = the number of records; out (NULL: count only) takes 8 x *count
 * entries, TCI_ERR_ARG when cap is smaller or the deck has no domains. */
int tci_local_allext_records(const tci_deck* deck, int64_t* out, int64_t cap, int64_t* count);

/* ---- Local pair domains: the all-external term over uneven domains -----
 * Replaces the local all-external loops (ext_3_4_seg_loops_vec_lmo_res_2,
 * tiger_fortran/three_and_four_seg_mod_1.f90:3240-3518, over the domains of
 * virtual_truncation, tiger_fortran/locist_mod.f90:358-451) for a set of N-2
 * heads, each with its own sorted domain of external orbitals.  heads: 7
 * int64 per head: off_ab, off_aa (CI offsets of the head's ab and aa blocks),
 * nsf_ab, nsf_aa (spin functions with an ab / aa block), nsing (the first
 * nsing are singlet-coupled), dom_off, dom_len (its slice of dom_idx: sorted
 * external indices 0..num_external-1).  A block of a head has its domain's
 * size: ab n(n-1)/2 per spin function, pair index i(i-1)/2+j (i > j), aa n.
 * chol is the tci_operator Cholesky array over num_internal + num_external
 * orbitals.  Applied in the Cholesky form (two grouped GEMMs over all heads
 * per chunk of Cholesky vectors) or, in the mixed precision, in the dense
 * padded integral form (the blocks placed among all externals against FP32
 * W+ / W- tiles over all external pairs, on the tcgen05 all-external kernel),
 * whichever a timed run at set-up finds faster.  options: [0] precision
 * (TCI_PRECISION_*), [1] device bytes for the per-chunk buffers (default
 * 16e9), [2] promotion block, [3] 0 to skip the set-up autotuning of chunk
 * size and tile shape, [4] form: 0 the faster (default; the dense form only
 * where the device has room for X = Lpk Lpk^T and the W tiles), 1 Cholesky,
 * 2 dense (TCI_ERR_INPUT in FP64 or with a triplet-coupled aa block,
 * TCI_ERR_MEMORY without the room). */
typedef struct tci_local tci_local;
int tci_local_create(int64_t num_internal, int64_t num_external, const double* chol, int64_t nchol, int64_t n_heads,
                     const int64_t* heads, const int64_t* dom_idx, int64_t total_len, int64_t device,
                     const int64_t* options, int64_t n_options, tci_local** out);
/* sigma += A c on device arrays of length total_len, ordered on stream (NULL =
 * legacy default stream). */
int tci_local_apply(tci_local* loc, const double* d_c, double* d_sigma, int64_t n, void* stream);
/* The same with host arrays. */
int tci_local_apply_host(tci_local* loc, const double* c, double* sigma, int64_t n);
/* out[len], len >= 9, up to 13: flops per application (4 nchol sum n^3 over
 * head spin functions), gathered Cholesky bytes per application, device
 * bytes, chunk size, FP64 tile shape of the second GEMM, autotuned time (ms),
 * autotuner candidates, last host application (ms), head spin-function
 * blocks, form applied (0 Cholesky, 1 dense), the dense form's set-up time
 * (ms, 0 if not timed), its flops (2 np^2 per singlet-coupled and 2 nm^2 per
 * triplet-coupled block), its W tile bytes. */
int tci_local_stats(const tci_local* loc, double* out, int64_t len);
void tci_local_destroy(tci_local* loc);

/* ---- Molecular front end (host) -------------------------------------------
 * The set-up that produces the tci_operator of a molecule, replacing
 * cholesky() (tiger_cpp/main.cpp:270-361): the AO two-electron integral
 * matrix decomposed by pivoted Cholesky with the CD THRESHOLD as dpstf2's
 * tolerance (Cho_WholeMat::decompose, tiger_cpp/Cholesky.cpp:268-307), and
 * the vectors transformed to the MO basis (transfrom_to_MO_basis,
 * tiger_cpp/Cholesky.cpp:78-165; tiger_fortran/cholesky_transform.f90:379).
 * The reference takes its AO integrals from libint and its orbitals from a
 * Molden file; here the integrals are computed by the McMurchie-Davidson
 * scheme, and tci_rhf gives canonical RHF orbitals where no orbitals are
 * given.  Shells are s, p or d over normalised primitives (Molden [GTO]
 * convention); Cartesian components in Molden order (p: x y z; d: xx yy zz xy
 * xz yz), pure d in Molden [5D] order (d0 d+1 d-1 d+2 d-2). */
typedef struct tci_molecule {
  int64_t n_atoms;
  const double* charges;      /* nuclear charge of each atom                       */
  const double* coords;       /* n_atoms x 3, bohr                                 */
  int64_t n_shells;
  const int64_t* shell_atom;  /* 0-based atom of each shell                        */
  const int64_t* shell_l;     /* 0 s, 1 p, 2 d                                     */
  const int64_t* shell_nprim; /* primitives of each shell                          */
  const double* exponents;    /* concatenated over the shells                      */
  const double* coefficients; /* contraction coefficients of normalised primitives */
  int64_t pure_d;             /* 1: five pure d functions per d shell; 0: six Cartesian */
} tci_molecule;
typedef struct tci_integrals tci_integrals;
/* AO integrals and the pivoted Cholesky decomposition of (mu nu|lambda sigma)
 * down to cd_threshold (largest remaining diagonal). */
int tci_integrals_create(const tci_molecule* mol, double cd_threshold, tci_integrals** out);
/* out[0..7]: basis functions, Cholesky vectors, nuclear repulsion, seconds,
 * largest remaining diagonal, ERI shell quartets computed, pivot shell-pair
 * blocks, shells. */
int tci_integrals_info(const tci_integrals* it, double* out, int64_t len);
/* Overlap S and core Hamiltonian h = T + V (nbf x nbf, row major); either may be NULL. */
int tci_integrals_one_electron(const tci_integrals* it, double* S, double* h, int64_t nbf);
/* AO Cholesky vectors chol[pq * nchol + J], pq = mu(mu+1)/2 + nu (mu >= nu). */
int tci_integrals_ao_cholesky(const tci_integrals* it, double* chol, int64_t npair, int64_t nchol);
/* Exact AO ERI tensor eri[((mu*n + nu)*n + la)*n + si] (not from the
 * decomposition), for checking small bases (nbf <= 200). */
int tci_integrals_ao_eri(const tci_integrals* it, double* eri, int64_t nbf);
/* Closed-shell RHF on the Cholesky vectors (DIIS), n_occ doubly occupied
 * orbitals; C (nbf x nbf, row major: C[mu * nbf + p]) gets the canonical
 * orbitals in ascending order of eps.  info[4] (may be NULL): total energy
 * (nuclear repulsion included), iterations, converged (1/0), DIIS error.
 * TCI_ERR_INPUT when it does not converge within maxit (<= 0: 100). */
int tci_rhf(const tci_integrals* it, int64_t n_occ, int64_t maxit, double conv, double* C, double* eps, double* info);
/* The tci_operator arrays in the basis of the nmo orbitals C (nbf x nmo, row
 * major): h = C^T h_AO C (nmo x nmo) and chol[pq * nchol + J] = (C^T L^J C)_pq
 * with pq = p(p+1)/2 + q (p >= q), the cholesky_data layout. */
int tci_mo_operator(const tci_integrals* it, const double* C, int64_t nmo, double* h, double* chol, int64_t nchol);
void tci_integrals_destroy(tci_integrals* it);

/* ---- Serving: continuously batched CI solves on one GPU ----------------
 * No counterpart in the reference, which runs one solve per process
 * (tiger_fortran/tiger_ci.f90 -> davidson_liu).  Submitted solves are
 * planned on host threads, admitted in arrival order when a slot is free and
 * their device-memory estimate fits the HBM budget, and solved by
 * tci_davidson_ex on a context of their own (own CUDA stream), so the sigma
 * builds of the admitted requests overlap on the device.  A request's result
 * is the one a lone tci_davidson_ex call gives. */
typedef struct tci_server tci_server;
typedef struct {
  int64_t device;
  int64_t slots;                     /* solves on the GPU at once (1..64)            */
  int64_t planners;                  /* host threads building plans (1..64)          */
  int64_t hbm_budget_bytes;          /* device bytes all admitted solves may reserve */
  int64_t precision;                 /* TCI_PRECISION_*                              */
  int64_t subspace_vectors_per_root; /* Davidson c / H c vectors per root before a
                                        restart (0: 12)                              */
  int64_t schedule_only;             /* 1: no device work; an admitted request holds
                                        its slot and reservation schedule_only_ms and
                                        returns NaN energies (scheduling tests)      */
  double schedule_only_ms;
  int64_t inject_worker_exit_at;     /* host fault injection: the worker thread that
                                        makes this admission (1-based) dies; 0 off   */
  int64_t tc_gemms;                  /* tci_sigma_init_ex options[2] of every request */
} tci_server_config;
int tci_server_create(const tci_server_config* cfg, tci_server** out);
/* Copies the deck and operator (the caller may free them on return); rejects
 * non-finite operator values (TCI_ERR_INPUT).  *id identifies the request. */
int tci_server_submit(tci_server* s, const tci_deck* deck, const tci_operator* op, int64_t nroots, double tol_residual,
                      double tol_energy, int64_t maxit, int64_t* id);
/* Waits up to timeout_s seconds (< 0: no limit; TCI_ERR_TIMEOUT when it runs
 * out) and returns the request's status.  energies[len]; info[9] = status,
 * iterations, submit / planned / admitted / done times (s since the server
 * started), reserved device bytes, total_csfs, core energy. */
int tci_server_wait(tci_server* s, int64_t id, double timeout_s, double* energies, int64_t len, double* info);
/* Cancels a queued request at once, a running one at its next iteration
 * (its status becomes TCI_ERR_CANCELLED). */
int tci_server_cancel(tci_server* s, int64_t id);
/* out[13]: submitted, succeeded, failed, cancelled, queued, running, peak
 * running, peak reserved bytes, p50 and p99 time to solution (s), solves/s
 * (successes over first submission .. last success), worker restarts,
 * reserved bytes now. */
int tci_server_stats(tci_server* s, double* out, int64_t len);
/* Cancels what is running or queued and joins the server's threads. */
void tci_server_destroy(tci_server* s);

#ifdef __cplusplus
}
#endif

#endif /* TIGERCI_SIGMA_H */
