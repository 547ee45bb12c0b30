"""Python host API over the C ABI, mirroring TigerCI's own interfaces.

* ``Deck`` holds the input keywords that define the CSF space
  (tc/InputReader.cpp:36-196; REFERENCE OCCUPATIONS as strings).
* ``CsfSpace`` replaces ``graph_driver`` (tiger_fortran/graph_mod.f90:48-99).
* ``Plan`` exposes the host-built sigma plan (replaces the iteration-1 dry run).
* ``SigmaBuilder.htimesc(civec, sigmavec)`` accumulates sigma += H c exactly
  like ``htimesc`` (tiger_fortran/htimesc.f90:46); the caller zeroes sigma.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Optional, Sequence

import numpy as np

from . import _lib
from ._lib import TciDeck, TciOperator, check, lib, ptr

KILL_NUMBER = -1000000


@dataclass
class Deck:
    num_orbitals: int
    num_inactive: int
    num_active: int
    num_elec: int
    spin_mult: int
    refs: Sequence[str]
    num_frozen: int = 0
    nm1_domains: Optional[Sequence[Sequence[int]]] = None
    nm2_domains: Optional[Sequence[Sequence[int]]] = None
    _keep: list = field(default_factory=list, repr=False)

    @property
    def num_internal(self):
        return self.num_inactive + self.num_active

    @property
    def num_external(self):
        return self.num_orbitals - self.num_internal

    def c_struct(self) -> TciDeck:
        nint = self.num_internal
        occ = np.array([[int(ch) for ch in str(r)[:nint]] for r in self.refs], dtype=np.int64)
        if occ.shape[1] != nint:
            raise ValueError("reference occupation strings must cover the internal orbitals")
        self._keep = [occ]
        d = TciDeck(self.num_orbitals, self.num_frozen, self.num_inactive, self.num_active, self.num_elec,
                    self.spin_mult, len(self.refs), ptr(occ), None, None, None, None)
        for name, doms in (("nm1", self.nm1_domains), ("nm2", self.nm2_domains)):
            if doms is None:
                continue
            p = np.zeros(len(doms) + 1, dtype=np.int64)
            for i, dm in enumerate(doms):
                p[i + 1] = p[i] + len(dm)
            idx = np.concatenate([np.asarray(dm, dtype=np.int64) for dm in doms]) if len(doms) else np.zeros(0, np.int64)
            idx = np.ascontiguousarray(idx, dtype=np.int64)
            self._keep += [p, idx]
            setattr(d, f"{name}_domain_ptr", ptr(p))
            setattr(d, f"{name}_domain_idx", ptr(idx))
        return d


class CsfSpace:
    """Distinct-row table, tree search and CI-vector index vectors."""

    def __init__(self, deck: Deck):
        self.deck = deck
        self._d = deck.c_struct()
        h = C.c_void_p()
        check(lib().tci_space_create(C.byref(self._d), C.byref(h)))
        self._h = h

    def acpf_gdiag(self, flag: int = 1, custom_g: float = 0.0):
        """Diagonal metric of the ACPF-type functionals (build_compressed_g): (g, class 1..5 per CSF)."""
        n = self.counts()["total_csfs"]
        g = np.zeros(n)
        cls = np.zeros(n, dtype=np.int64)
        check(lib().tci_acpf_gdiag(self._h, flag, custom_g, ptr(g), ptr(cls), n))
        return g, cls

    def reference_weight(self, c: np.ndarray) -> float:
        """c0^2: the squared coefficients of the reference configurations' CSFs summed (tci_reference_weight)."""
        c = np.ascontiguousarray(c, dtype=np.float64)
        out = C.c_double()
        check(lib().tci_reference_weight(self._h, ptr(c), c.size, C.byref(out)))
        return out.value

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tci_space_destroy(self._h)
            self._h = None

    def counts(self) -> dict:
        out = np.zeros(12, dtype=np.int64)
        check(lib().tci_space_counts(self._h, ptr(out), 12))
        keys = ["total_csfs", "num_valence", "num_nm1", "num_nm2", "total_configurations", "removed",
                "open_shells", "paths_v", "paths_nm1", "paths_nm2", "num_vertices", "n_domains"]
        return dict(zip(keys, (int(x) for x in out)))

    def index_vector(self, kind: int) -> np.ndarray:
        c = self.counts()
        n = [c["paths_v"], c["paths_nm1"], c["paths_nm2"], c["paths_nm2"]][kind]
        out = np.zeros(n, dtype=np.int64)
        check(lib().tci_space_index_vector(self._h, kind, ptr(out), n))
        return out

    def path(self, kind: int, lex: int):
        occ = np.zeros(self.deck.num_internal, dtype=np.int64)
        info = np.zeros(6, dtype=np.int64)
        check(lib().tci_space_path(self._h, kind, lex, ptr(occ), ptr(info)))
        return occ, dict(zip(["lex", "singles", "kept", "nsf", "nsf_aa", "n_virt"], (int(x) for x in info)))

    def block_counts(self, kind: int) -> dict:
        out = np.zeros(3 * 64, dtype=np.int64)
        nt = C.c_int64()
        check(lib().tci_space_block_counts(self._h, kind, ptr(out), 64, C.byref(nt)))
        return {int(out[3 * t]): (int(out[3 * t + 1]), int(out[3 * t + 2])) for t in range(nt.value)}


APOSTERIORI = ("davidson", "renormalized_davidson", "davidson_silver", "meissner", "pople")


def aposteriori(c0sq: float, e_corr: float, n_corr_elec: int) -> dict:
    """The reference's a posteriori corrections (tci_aposteriori): {name: correction (Eh)}."""
    out = np.zeros(5)
    check(lib().tci_aposteriori(int(n_corr_elec), float(c0sq), float(e_corr), ptr(out), 5))
    return dict(zip(APOSTERIORI, out.tolist()))


class Operator:
    """MO Hamiltonian: h (n_orb x n_orb) and Cholesky vectors in TigerCI's
    cho_vectors(numcho, npair) layout, i.e. chol[pair, J] with
    pair = p(p+1)/2 + q for p >= q (0-based)."""

    def __init__(self, h: np.ndarray, chol: np.ndarray, core_energy: float = 0.0):
        self.h = np.ascontiguousarray(h, dtype=np.float64)
        self.chol = np.ascontiguousarray(chol, dtype=np.float64)
        n = self.h.shape[0]
        if self.h.shape != (n, n) or self.chol.ndim != 2 or self.chol.shape[0] != n * (n + 1) // 2:
            raise ValueError("h must be n x n and chol n(n+1)/2 x nchol")
        self.core_energy = float(core_energy)

    @property
    def nchol(self):
        return self.chol.shape[1]

    @classmethod
    def from_records(cls, h: np.ndarray, records: np.ndarray, mo_ind_inv, core_energy: float = 0.0) -> "Operator":
        """The operator from Cholesky records addressed through the reference's mo_ind_inv (1-based record of
        each pair, 0 for a zero vector), by tci_operator_from_records."""
        h = np.ascontiguousarray(h, dtype=np.float64)
        n = h.shape[0]
        rec = np.ascontiguousarray(records, dtype=np.float64)
        if rec.ndim != 2:
            raise ValueError("records must be n_records x nchol")
        inv = np.ascontiguousarray(mo_ind_inv, dtype=np.int64)
        if inv.shape != (n * (n + 1) // 2,):
            raise ValueError("mo_ind_inv must have n(n+1)/2 entries")
        chol = np.empty((n * (n + 1) // 2, rec.shape[1]))
        check(lib().tci_operator_from_records(n, rec.shape[1], ptr(inv), ptr(rec) if rec.size else None,
                                              rec.shape[0], ptr(chol)))
        return cls(h, chol, core_energy)

    def c_struct(self) -> TciOperator:
        return TciOperator(ptr(self.h), ptr(self.chol), self.nchol, self.core_energy)


class Plan:
    """Host-built sigma plan (no GPU)."""

    def __init__(self, deck: Deck, op: Operator):
        self._d = deck.c_struct()
        self._o = op.c_struct()
        self._op = op
        h = C.c_void_p()
        check(lib().tci_plan_create(C.byref(self._d), C.byref(self._o), C.byref(h)))
        self._h = h

    def __del__(self):
        if getattr(self, "_h", None):
            lib().tci_plan_destroy(self._h)
            self._h = None

    def export(self, path: str):
        check(lib().tci_plan_export(self._h, path.encode()))

    def stats(self) -> dict:
        out = np.zeros(10, dtype=np.float64)
        check(lib().tci_plan_stats(self._h, ptr(out), 10))
        keys = ["total_csfs", "n_dense", "n_singlet", "n_triplet", "flops_allext", "flops_total", "bytes_allext",
                "n_steps", "device_bytes_peak", "device_bytes_resident"]
        return dict(zip(keys, out.tolist()))


class SigmaBuilder:
    """Device-resident sigma = H c on one GPU (the htimesc slot)."""

    PRECISIONS = {"fp64": 0, "tf32x3": 1}

    TC_GEMMS = {"by_size": 0, "all": 1, "none": 2}

    def __init__(self, deck: Deck, op: Operator, device: int = 0, precision: str = "fp64", promote_every: int = 128,
                 tc_gemms: str = "by_size", fp64_finish="no_allext"):
        """fp64_finish (mixed form): "no_allext" (default) reports each root as the Rayleigh quotient of its
        Ritz vector with a sigma build in which every term is FP64 but the all-external one, which stays on
        its tensor-core kernel (no FP64 W kept); "full" / True does the same with a plain-FP64 sigma build
        (the FP64 W stays resident); "no_allext_3ext" is "no_allext" with the three-external contractions on
        the tensor cores too; "none" / False reports the mixed Ritz values."""
        self._d = deck.c_struct()
        self._o = op.c_struct()
        self._op = op
        self.deck = deck
        self.precision = precision
        h = C.c_void_p()
        finish = {True: 1, False: 0, "full": 1, "none": 0, "no_allext": 2, "no_allext_3ext": 3}[fp64_finish]
        opts = np.array([self.PRECISIONS[precision], promote_every, self.TC_GEMMS[tc_gemms], finish], dtype=np.int64)
        check(lib().tci_sigma_init_ex(C.byref(self._d), C.byref(self._o), device, ptr(opts), 4, C.byref(h)))
        self._h = h
        self.n = int(self.stats()["total_csfs"])

    def close(self):
        if getattr(self, "_h", None):
            lib().tci_destroy(self._h)
            self._h = None

    def __del__(self):
        self.close()

    def htimesc(self, civec: np.ndarray, sigmavec: np.ndarray):
        """sigmavec += H civec (host float64 arrays of length total_csfs)."""
        if civec.dtype != np.float64 or sigmavec.dtype != np.float64:
            raise TypeError("float64 arrays required")
        if not (civec.flags.c_contiguous and sigmavec.flags.c_contiguous):
            raise ValueError("contiguous arrays required")
        check(lib().tci_sigma(self._h, ptr(civec), ptr(sigmavec), civec.size))

    def sigma(self, civec: np.ndarray) -> np.ndarray:
        s = np.zeros_like(civec, dtype=np.float64)
        self.htimesc(np.ascontiguousarray(civec, dtype=np.float64), s)
        return s

    def dots(self, A_ptr: int, lda: int, m: int, x_ptr: int, n: int, out_ptr: int, stream: int = 0):
        """out[k] = A[k] . x on device arrays (deterministic)."""
        check(lib().tci_dots(self._h, C.c_void_p(A_ptr), lda, m, C.c_void_p(x_ptr), n, C.c_void_p(out_ptr),
                             C.c_void_p(stream or None)))

    def check(self):
        """Synchronise and raise if a bounded device wait gave up."""
        check(lib().tci_check(self._h))

    def htimesc_device(self, c_ptr: int, s_ptr: int, n: int, stream: int = 0):
        """Device pointers (e.g. torch tensors' data_ptr()) on `stream`."""
        check(lib().tci_sigma_device(self._h, C.c_void_p(c_ptr), C.c_void_p(s_ptr), n, C.c_void_p(stream or None)))

    def diag(self) -> np.ndarray:
        """Diagonal H_ii (preconditioner input)."""
        out = np.zeros(self.n)
        check(lib().tci_diag(self._h, ptr(out), self.n))
        return out

    def davidson(self, nroots: int = 1, tol_residual: float = 1e-6, tol_energy: float = 1e-6, maxit: int = 0,
                 want_vectors: bool = False, subspace_bytes: int = 0, cancel=None):
        """Device-resident Davidson-Liu (davidson_liu); returns (energies, vectors|None, iterations).

        subspace_bytes bounds the c / H c subspace like DAVIDSON HARD DRIVE
        SPACE (0: 30 GB); cancel is an optional numpy int32 array of one
        element whose becoming non-zero ends the solve (TCI_ERR_CANCELLED)."""
        e = np.zeros(nroots)
        v = np.zeros((nroots, self.n)) if want_vectors else None
        it = C.c_int64()
        if cancel is not None and (cancel.dtype != np.int32 or cancel.size < 1):
            raise TypeError("cancel must be an int32 array")
        check(lib().tci_davidson_ex(self._h, nroots, tol_residual, tol_energy, maxit, int(subspace_bytes),
                                    ptr(cancel) if cancel is not None else None, ptr(e),
                                    ptr(v) if v is not None else None, C.byref(it)))
        return e, v, it.value

    def acpf(self, nroots: int = 1, flag: int = 1, custom_g: float = 0.0, tol_residual: float = 1e-6,
             tol_energy: float = 1e-6, maxit: int = 0, want_vectors: bool = False, e_ref=None):
        """(MR)ACPF / ACPF-2 / (MR)AQCC roots (acpf_driver + davidson_liu_gen_eig): (H - E_ref) c = lambda G c
        with G from CsfSpace.acpf_gdiag(flag).  E_ref defaults to the lowest eigenvalue of H in the space of
        the reference-configuration CSFs (class 1).  Returns (energies, vectors|None, iterations, E_ref);
        energies are electronic, like davidson()."""
        g, cls = CsfSpace(self.deck).acpf_gdiag(flag, custom_g)
        if e_ref is None:
            idx = np.nonzero(cls == 1)[0]
            if idx.size == 0:
                raise ValueError("no reference CSF in the space")
            Hr = np.zeros((idx.size, idx.size))
            for j, i in enumerate(idx):
                x = np.zeros(self.n)
                x[i] = 1.0
                Hr[:, j] = self.sigma(x)[idx]
            e_ref = float(np.linalg.eigvalsh(0.5 * (Hr + Hr.T))[0])
        e = np.zeros(nroots)
        v = np.zeros((nroots, self.n)) if want_vectors else None
        it = C.c_int64()
        check(lib().tci_davidson_gen(self._h, nroots, tol_residual, tol_energy, maxit, ptr(g), float(e_ref), ptr(e),
                                     ptr(v) if v is not None else None, C.byref(it)))
        return e, v, it.value, e_ref

    def profile(self, on: bool = True, davidson_phases: bool = False):
        """Per-step CUDA-event timing of subsequent sigma builds; with
        davidson_phases, wall time per Davidson phase (stream synchronised at
        each phase boundary)."""
        check(lib().tci_profile(self._h, (1 if on else 0) | (2 if davidson_phases else 0)))

    def davidson_phase_times(self) -> dict:
        ms = np.zeros(8)
        check(lib().tci_davidson_phase_times(self._h, ptr(ms), 8))
        keys = ["setup", "sigma", "projection", "subspace_eig", "residual", "precondition_mgs", "restart", "finish"]
        return dict(zip(keys, ms.tolist()))

    def step_times(self) -> list:
        """[(step name, accumulated ms)] and the number of profiled builds."""
        ns, nb = C.c_int64(), C.c_int64()
        check(lib().tci_step_times(self._h, None, 0, C.byref(ns), C.byref(nb)))
        ms = np.zeros(ns.value)
        check(lib().tci_step_times(self._h, ptr(ms), ns.value, C.byref(ns), C.byref(nb)))
        names = []
        buf = C.create_string_buffer(128)
        for i in range(ns.value):
            check(lib().tci_step_name(self._h, i, buf, 128))
            names.append(buf.value.decode())
        return list(zip(names, ms.tolist())), nb.value

    def stats(self) -> dict:
        out = np.zeros(11, dtype=np.float64)
        check(lib().tci_ctx_stats(self._h, ptr(out), 11))
        keys = ["total_csfs", "device_bytes", "init_seconds", "last_sigma_ms", "flops_per_sigma",
                "flops_allext", "bytes_allext", "sigma_count", "launches_per_sigma", "launches", "converged"]
        return dict(zip(keys, out.tolist()))
