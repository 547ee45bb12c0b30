"""Continuously batched CI solves on one GPU (tci_server_* in the C ABI).

`Server` submits solves to the library's request server: host threads build
each request's CSF space and sigma plan while others run, requests are
admitted in arrival order when a slot is free and their device-memory
estimate fits the HBM budget, and every admitted solve runs the device
Davidson on a context and CUDA stream of its own, so the sigma builds of the
requests in flight overlap on the GPU.

`hn_chain_stream` generates the serving workload: a seeded Poisson stream of
linear H_n chain solves (n even in 8..24, H-H spacing in [1.4, 3.0] bohr,
cc-pVDZ: 5 n orbitals, singlet, 1-4 roots).  `chain_problem` builds a
request's deck and MO operator through the molecular front end (RHF/cc-pVDZ
orbitals, Cholesky vectors); `request_problem` is a fast synthetic stand-in
with the same sizes for scheduling tests.
"""
from __future__ import annotations

import ctypes as C
import itertools
from dataclasses import dataclass

import numpy as np

from ._lib import TciError, check, last_error, lib, ptr
from .api import Deck, Operator
from .synthetic import synthetic_operator

PRECISIONS = {"fp64": 0, "tf32x3": 1}
STATUS_CANCELLED = 7


class TciServerConfig(C.Structure):
    _fields_ = [("device", C.c_int64), ("slots", C.c_int64), ("planners", C.c_int64),
                ("hbm_budget_bytes", C.c_int64), ("precision", C.c_int64),
                ("subspace_vectors_per_root", C.c_int64), ("schedule_only", C.c_int64),
                ("schedule_only_ms", C.c_double), ("inject_worker_exit_at", C.c_int64), ("tc_gemms", C.c_int64)]


def _bind():
    L = lib()
    if not getattr(L, "_server_bound", False):
        P, i64, dbl = C.c_void_p, C.c_int64, C.c_double
        L.tci_server_create.argtypes = [C.POINTER(TciServerConfig), C.POINTER(P)]
        L.tci_server_submit.argtypes = [P, P, P, i64, dbl, dbl, i64, C.POINTER(i64)]
        L.tci_server_wait.argtypes = [P, i64, dbl, P, i64, P]
        L.tci_server_cancel.argtypes = [P, i64]
        L.tci_server_stats.argtypes = [P, P, i64]
        L.tci_server_destroy.argtypes = [P]
        L.tci_server_destroy.restype = None
        L._server_bound = True
    return L


@dataclass
class Result:
    id: int
    status: int
    energies: np.ndarray
    iterations: int
    t_submit: float
    t_planned: float
    t_admitted: float
    t_done: float
    reserved_bytes: float
    total_csfs: int
    error: str = ""

    @property
    def time_to_solution(self) -> float:
        return self.t_done - self.t_submit


class Server:
    def __init__(self, device: int = 0, slots: int = 4, hbm_budget: float = 150e9, precision: str = "tf32x3",
                 planners: int = 2, subspace_vectors_per_root: int = 12, schedule_only: bool = False,
                 schedule_only_ms: float = 0.0, inject_worker_exit_at: int = 0, tc_gemms: str = "by_size"):
        self._L = _bind()
        cfg = TciServerConfig(device, slots, planners, int(hbm_budget), PRECISIONS[precision],
                              subspace_vectors_per_root, 1 if schedule_only else 0, float(schedule_only_ms),
                              inject_worker_exit_at, {"by_size": 0, "all": 1, "none": 2}[tc_gemms])
        h = C.c_void_p()
        check(self._L.tci_server_create(C.byref(cfg), C.byref(h)))
        self._h = h
        self._nroots = {}

    def submit(self, deck: Deck, op: Operator, nroots: int = 1, tol_residual: float = 1e-6,
               tol_energy: float = 1e-6, maxit: int = 0) -> int:
        d, o = deck.c_struct(), op.c_struct()
        rid = C.c_int64()
        check(self._L.tci_server_submit(self._h, C.byref(d), C.byref(o), nroots, tol_residual, tol_energy, maxit,
                                        C.byref(rid)))
        self._nroots[rid.value] = nroots
        return rid.value

    def wait(self, rid: int, timeout: float = -1.0) -> Result:
        """Blocks until the request finishes (raises TciError with code 6 when
        `timeout` seconds pass first); a failed request is returned with its
        status, not raised."""
        n = self._nroots[rid]
        e = np.zeros(n)
        info = np.full(9, -1.0)  # left untouched when the wait itself times out
        rc = self._L.tci_server_wait(self._h, rid, float(timeout), ptr(e), n, ptr(info))
        if rc == 6 and info[0] == -1.0:
            raise TciError(rc, last_error())
        return Result(rid, int(info[0]), e, int(info[1]), info[2], info[3], info[4], info[5], info[6], int(info[7]),
                      last_error() if rc != 0 else "")

    def cancel(self, rid: int):
        check(self._L.tci_server_cancel(self._h, rid))

    def stats(self) -> dict:
        out = np.zeros(13)
        check(self._L.tci_server_stats(self._h, ptr(out), 13))
        keys = ["submitted", "succeeded", "failed", "cancelled", "queued", "running", "peak_running",
                "peak_reserved_bytes", "p50_s", "p99_s", "solves_per_s", "worker_restarts", "reserved_bytes"]
        return dict(zip(keys, out.tolist()))

    def close(self):
        if getattr(self, "_h", None):
            self._L.tci_server_destroy(self._h)
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def __del__(self):
        self.close()


@dataclass
class RequestSpec:
    index: int
    arrival: float      # seconds after the stream starts
    n_atoms: int        # H_n chain length (even, 8..24)
    spacing: float      # H-H distance, bohr
    nroots: int


def hn_chain_stream(n_requests: int = 256, rate: float = 4.0, seed: int = 7):
    """Seeded Poisson arrivals (exponential gaps of mean 1/rate) of H_n chain
    solves: n uniform in {8, 10, ..., 24}, spacing uniform in [1.4, 3.0] bohr,
    roots uniform in {1..4}."""
    rng = np.random.default_rng(seed)
    t = 0.0
    out = []
    for i in range(n_requests):
        t += rng.exponential(1.0 / rate)
        out.append(RequestSpec(i, t, int(rng.choice(np.arange(8, 25, 2))), float(rng.uniform(1.4, 3.0)),
                               int(rng.integers(1, 5))))
    return out


def request_problem(spec: RequestSpec, seed: int = 7):
    """Deck and MO operator standing in for an H_n chain in cc-pVDZ.

    Sizes follow the chain: 5 n orbitals; n electrons; n/2 - 1 doubly
    occupied internal orbitals plus a 2-orbital active space (HOMO/LUMO)
    whose three singlet-compatible occupations (20, 11, 02) are the
    references; the other 5 n - n/2 - 1 orbitals are external; Cholesky rank
    4 x 5 n.  The integrals are a seeded synthetic operator at molecular
    magnitude whose coupling grows with the spacing (stretched chains are
    more strongly correlated).  A full CAS(n/2, n/2) reference list makes the
    MRCI space of the longer chains intractable for any solver, hence the
    2-orbital active space."""
    n = spec.n_atoms
    nbf = 5 * n
    nin, act = n // 2 - 1, 2
    refs = ["2" * nin + "".join(map(str, occ)) for occ in itertools.product((0, 1, 2), repeat=act)
            if sum(occ) == act]
    deck = Deck(num_orbitals=nbf, num_inactive=nin, num_active=act, num_elec=n, spin_mult=1, refs=refs)
    scale = 0.02 * (spec.spacing / 1.4) ** 0.5
    h, L = synthetic_operator(nbf, 4 * nbf, seed=seed * 100003 + spec.index, scale=scale, diag_range=(-2.0, 1.0),
                              offdiag_sigma=0.02)
    return deck, Operator(h, L)


def chain_problem(spec: RequestSpec, cd_threshold: float = 1e-6, n_active: int = 2):
    """Deck and MO operator of an H_n chain request through the molecular front end: cc-pVDZ (5 n functions),
    canonical RHF orbitals, Cholesky vectors of the AO integrals at cd_threshold transformed to them,
    nuclear repulsion as the core energy.  The references are the complete active space of the n_active
    orbitals around the Fermi level (n_active electrons: HOMO/LUMO, occupations 20, 11, 02 for the default
    2), the other occupied orbitals inactive.  A full CAS(n/2, n/2) reference list (tens of thousands of
    occupations for n = 24) makes the MRCI space of the longer chains intractable for any solver."""
    from .molecule import h_chain, mrsdci_problem

    sym, xyz = h_chain(spec.n_atoms, spec.spacing)
    deck, op, _ = mrsdci_problem(sym, xyz, "cc-pVDZ", pure_d=True, n_frozen=0, cas=(n_active, n_active),
                                 cd_threshold=cd_threshold)
    return deck, op
