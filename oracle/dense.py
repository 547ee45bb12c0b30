"""Oracle (test infrastructure only): sigma = H c in TigerCI's CSF basis for
small cases, by expanding every CSF over Slater determinants and applying the
determinant Hamiltonian with the Slater-Condon rules (oracle/detci.c).

The CSF basis and CI-vector layout are restated from the reference:
  * CSF list and offsets: graph_mod.f90:1007-1589 (oracle/sgga.py build_space)
  * spin functions: SFT graph order, spin_mod.f90:232-522 (oracle/sgga.py)
  * N-1 block: spin-major, one virtual per entry (graph_mod.f90:1073-1083)
  * N-2 blocks: "aa" (one virtual doubly occupied) then "ab" with pair index
    i(i-1)/2 + j for i > j (graph_mod.f90:1084-1101, scepmaker_mod.f90:60-90)
Determinant convention: open-shell creators in coupling order (highest
orbital first) followed by the doubly occupied pairs, i.e. a phase
(-1)^{s(s-1)/2} relative to the canonical ascending spin-orbital order.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

from . import sgga

HERE = os.path.dirname(os.path.abspath(__file__))
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(BUILD, "liboracle.so")


def build_oracle(force=False):
    os.makedirs(BUILD, exist_ok=True)
    srcs = [os.path.join(HERE, "detci.c"), os.path.join(HERE, "plancpu.c")]
    if force or not os.path.exists(LIB) or any(os.path.getmtime(LIB) < os.path.getmtime(s) for s in srcs):
        subprocess.check_call(["gcc", "-O3", "-march=native", "-fopenmp", "-fPIC", "-shared", "-o", LIB, *srcs, "-lm"])
    return LIB


_lib = None


def lib():
    global _lib
    if _lib is None:
        build_oracle()
        L = C.CDLL(LIB)
        L.oracle_hdet_matvec.argtypes = [C.c_int64, C.c_void_p, C.c_int, C.c_void_p, C.c_void_p, C.c_void_p,
                                         C.c_void_p]
        L.oracle_allext_sigma.argtypes = [C.c_int64, C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p,
                                          C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
        L.oracle_allext_local_sigma.argtypes = [C.c_int64, C.c_int64, C.c_void_p, C.c_int64, C.c_void_p, C.c_void_p,
                                                C.c_void_p, C.c_void_p, C.c_int64, C.c_int64]
        L.oracle_set_dgemm.argtypes = [C.c_void_p]
        L.oracle_num_threads.restype = C.c_int
        L.plancpu_load.argtypes = [C.c_char_p, C.c_void_p]
        L.plancpu_load.restype = C.c_void_p
        L.plancpu_sigma.argtypes = [C.c_void_p, C.c_void_p, C.c_void_p, C.c_int]
        L.plancpu_integrals.argtypes = [C.c_void_p]
        L.plancpu_free.argtypes = [C.c_void_p]
        L.plancpu_diag.argtypes = [C.c_void_p, C.c_void_p]
        L.plancpu_total.argtypes = [C.c_void_p]
        L.plancpu_total.restype = C.c_int64
        _lib = L
    return _lib


def eri_from_chol(chol, norb):
    """(pq|rs) = sum_J L^J_pq L^J_rs, chol[p(p+1)/2+q, J]."""
    idx = np.zeros((norb, norb), dtype=np.int64)
    for p in range(norb):
        for q in range(p + 1):
            idx[p, q] = idx[q, p] = p * (p + 1) // 2 + q
    Lf = chol[idx.reshape(-1)]  # (norb*norb, nchol)
    return (Lf @ Lf.T).reshape(norb, norb, norb, norb)


class DenseSigma:
    """Builds the CSF -> determinant map for a (small) non-local MRSDCI space."""

    def __init__(self, deck: sgga.Deck):
        self.deck = deck
        self.space = sp = sgga.build_space(deck)
        nint, norb = deck.num_internal, deck.num_orbitals
        n = norb - nint
        self.n = n
        os_ = sp.open_shells
        fsn_all, sft, sm = sgga.spin_tables(os_, deck.spin_mult)
        self._exp = {}
        for s in range(0, os_ + 1):
            if fsn_all[s] > 0:
                self._exp[s] = sgga.yk_expansion(sm, s, fsn_all[s], deck.spin_mult)
        rows, cols, vals = [], [], []
        det_index = {}

        def add_csf(csf, occ):
            open_ = [p for p, o in enumerate(occ) if o == 1]
            s = len(open_)
            strings, theta = self._exp[s]
            k = csf[1]
            sign = -1.0 if (s * (s - 1) // 2) % 2 else 1.0
            closed = 0
            for p, o in enumerate(occ):
                if o == 2:
                    closed |= (1 << (2 * p)) | (1 << (2 * p + 1))
            for r, x in enumerate(strings):
                t = theta[r, k]
                if t == 0.0:
                    continue
                d = closed
                for i, p in enumerate(open_):
                    d |= 1 << (2 * p + ((x >> i) & 1))
                j = det_index.setdefault(d, len(det_index))
                rows.append(j)
                cols.append(csf[0])
                vals.append(sign * t)

        ncsf = sp.total_csfs
        seen = np.zeros(ncsf, dtype=bool)
        for h in sp.paths[0]:
            if h["off"] is None:
                continue
            for k in range(h["nsf"]):
                occ = list(h["occ"]) + [0] * n
                add_csf((h["off"] + k, k), occ)
                seen[h["off"] + k] = True
        for h in sp.paths[1]:
            if h["off"] is None:
                continue
            for k in range(h["nsf"]):
                for a in range(n):
                    occ = list(h["occ"]) + [0] * n
                    occ[nint + a] = 1
                    add_csf((h["off"] + k * n + a, k), occ)
                    seen[h["off"] + k * n + a] = True
        nab = n * (n - 1) // 2
        for h in sp.paths[2]:
            if h["off_aa"] is not None:
                for k in range(h["nsf_aa"]):
                    for a in range(n):
                        occ = list(h["occ"]) + [0] * n
                        occ[nint + a] = 2
                        add_csf((h["off_aa"] + k * n + a, k), occ)
                        seen[h["off_aa"] + k * n + a] = True
            if h["off"] is not None:
                for k in range(h["nsf"]):
                    for i in range(1, n):
                        for j in range(i):
                            occ = list(h["occ"]) + [0] * n
                            occ[nint + i] = 1
                            occ[nint + j] = 1
                            e = h["off"] + k * nab + i * (i - 1) // 2 + j
                            add_csf((e, k), occ)
                            seen[e] = True
        if not seen.all():
            raise RuntimeError("CSF list does not cover the CI vector")
        self.dets = np.zeros(len(det_index), dtype=np.uint64)
        for d, j in det_index.items():
            self.dets[j] = d
        import scipy.sparse as sps

        self.T = sps.csr_matrix((vals, (rows, cols)), shape=(len(det_index), ncsf))
        self.ncsf = ncsf

    def sigma(self, h, chol, c):
        norb = self.deck.num_orbitals
        if 2 * norb > 64:
            raise ValueError("dense oracle supports at most 32 orbitals")
        eri = np.ascontiguousarray(eri_from_chol(chol, norb))
        h = np.ascontiguousarray(h, dtype=np.float64)
        x = np.ascontiguousarray(self.T @ c, dtype=np.float64)
        y = np.zeros_like(x)
        lib().oracle_hdet_matvec(len(self.dets), self.dets.ctypes.data, norb, h.ctypes.data, eri.ctypes.data,
                                 x.ctypes.data, y.ctypes.data)
        return self.T.T @ y

    def hamiltonian(self, h, chol):
        """Dense CSF Hamiltonian (tiny cases only)."""
        H = np.zeros((self.ncsf, self.ncsf))
        for j in range(self.ncsf):
            e = np.zeros(self.ncsf)
            e[j] = 1.0
            H[:, j] = self.sigma(h, chol, e)
        return H


def use_blas():
    """Route the oracle's (ab|cd) slab through scipy's bundled OpenBLAS dgemm
    (the reference calls dgemm there).  Returns True when found."""
    import glob

    import scipy

    libs = glob.glob(os.path.join(os.path.dirname(scipy.__file__), "..", "scipy.libs", "libscipy_openblas*.so"))
    for p in libs:
        try:
            ob = C.CDLL(p)
            fn = getattr(ob, "scipy_dgemm_")
        except (OSError, AttributeError):
            continue
        # one BLAS thread per call: the oracle already runs one OpenMP thread per outer index
        try:
            ob.scipy_openblas_set_num_threads64_(1)
        except AttributeError:
            for name in ("openblas_set_num_threads", "scipy_openblas_set_num_threads"):
                if hasattr(ob, name):
                    getattr(ob, name)(1)
                    break
        lib().oracle_set_dgemm(C.cast(fn, C.c_void_p))
        return True
    return False


def allext_sigma(space, nint, n, chol, c, nthreads=None, a_range=None):
    """Reference integral-form all-external sigma (detci.c oracle_allext_sigma);
    a_range=(a0, a1) restricts the outer external index (a sample)."""
    heads = []
    for h in space.paths[2]:
        off_ab = -1 if h["off"] is None else h["off"]
        off_aa = -1 if h["off_aa"] is None else h["off_aa"]
        nsf_ab = 0 if h["off"] is None else h["nsf"]
        nsf_aa = 0 if h["off_aa"] is None else h["nsf_aa"]
        if nsf_ab == 0 and nsf_aa == 0:
            continue
        nsing = nsf_aa
        heads.append([off_ab, off_aa, nsf_ab, nsf_aa, nsing])
    heads = np.ascontiguousarray(np.array(heads, dtype=np.int64).reshape(-1, 5))
    chol = np.ascontiguousarray(chol, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    s = np.zeros_like(c)
    if nthreads:
        os.environ["OMP_NUM_THREADS"] = str(nthreads)
    a0, a1 = a_range if a_range else (0, n)
    lib().oracle_allext_sigma(nint, n, chol.shape[1], chol.ctypes.data, len(heads), heads.ctypes.data,
                              c.ctypes.data, s.ctypes.data, a0, a1)
    return s


def allext_local_sigma(nint, chol, heads, dom_idx, c, head_range=None):
    """Reference integral-form all-external sigma over pair domains (detci.c
    oracle_allext_local_sigma).  heads: int64 rows (off_ab, off_aa, nsf_ab,
    nsf_aa, nsing, dom_off, dom_len); dom_idx: concatenated sorted domains
    (external indices); head_range=(h0, h1) restricts the heads (a sample)."""
    heads = np.ascontiguousarray(np.asarray(heads, dtype=np.int64).reshape(-1, 7))
    dom_idx = np.ascontiguousarray(np.asarray(dom_idx, dtype=np.int64))
    chol = np.ascontiguousarray(chol, dtype=np.float64)
    c = np.ascontiguousarray(c, dtype=np.float64)
    s = np.zeros_like(c)
    h0, h1 = head_range if head_range else (0, len(heads))
    lib().oracle_allext_local_sigma(nint, chol.shape[1], chol.ctypes.data, len(heads), heads.ctypes.data,
                                    dom_idx.ctypes.data, c.ctypes.data, s.ctypes.data, h0, h1)
    return s


class PlanSigmaCPU:
    """Integral-direct CPU sigma build (plancpu.c): the integrals formed from the
    Cholesky vectors at every build, the all-external term in the reference's
    loop form, every other coupling replayed from the loop records of an
    exported plan (tci_plan_export).  Test and CPU-baseline use only."""

    def __init__(self, plan_path, chol):
        self._chol = np.ascontiguousarray(chol, dtype=np.float64)
        self._h = lib().plancpu_load(plan_path.encode(), self._chol.ctypes.data)
        if not self._h:
            raise RuntimeError(f"cannot load plan {plan_path}")
        self.n = int(lib().plancpu_total(self._h))

    def sigma(self, c, integrals=True):
        c = np.ascontiguousarray(c, dtype=np.float64)
        s = np.zeros_like(c)
        lib().plancpu_sigma(self._h, c.ctypes.data, s.ctypes.data, 1 if integrals else 0)
        return s

    def diag(self):
        """H_ii (forms the integral banks first)."""
        lib().plancpu_integrals(self._h)
        d = np.zeros(self.n)
        lib().plancpu_diag(self._h, d.ctypes.data)
        return d

    def close(self):
        if getattr(self, "_h", None):
            lib().plancpu_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
