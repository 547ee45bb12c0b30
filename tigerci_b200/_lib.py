"""ctypes binding of libtigerci_sigma.so (include/tigerci_sigma.h).

The library is built in-tree (tigerci_b200/libtigerci_sigma.so).  Loading
fails loudly if it is missing: there is no Python fallback for any entry
point.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "libtigerci_sigma.so")

i64 = C.c_int64
dbl = C.c_double
P = C.c_void_p

EXPORTS = [
    "tci_last_error",
    "tci_space_create",
    "tci_space_counts",
    "tci_space_index_vector",
    "tci_space_path",
    "tci_space_block_counts",
    "tci_space_destroy",
    "tci_plan_create",
    "tci_plan_export",
    "tci_plan_stats",
    "tci_plan_destroy",
    "tci_sigma_init",
    "tci_sigma_init_ex",
    "tci_check",
    "tci_sigma",
    "tci_sigma_device",
    "tci_diag",
    "tci_davidson",
    "tci_davidson_ex",
    "tci_davidson_gen",
    "tci_acpf_gdiag",
    "tci_davidson_capacity",
    "tci_davidson_bytes",
    "tci_local_create",
    "tci_local_apply",
    "tci_local_apply_host",
    "tci_local_stats",
    "tci_local_destroy",
    "tci_server_create",
    "tci_server_submit",
    "tci_server_wait",
    "tci_server_cancel",
    "tci_server_stats",
    "tci_server_destroy",
    "tci_dots",
    "tci_dots_noalloc",
    "tci_ctx_stats",
    "tci_profile",
    "tci_davidson_phase_times",
    "tci_step_times",
    "tci_step_name",
    "tci_destroy",
    "tci_selftest_bounded_wait",
    "tci_selftest_mma_rate",
    "tci_operator_from_records",
    "tci_reference_weight",
    "tci_aposteriori",
    "tci_local_allext_records",
    "tci_integrals_create",
    "tci_integrals_info",
    "tci_integrals_one_electron",
    "tci_integrals_ao_cholesky",
    "tci_integrals_ao_eri",
    "tci_rhf",
    "tci_mo_operator",
    "tci_integrals_destroy",
]


class TciDeck(C.Structure):
    _fields_ = [
        ("num_orbitals", i64),
        ("num_frozen", i64),
        ("num_inactive", i64),
        ("num_active", i64),
        ("num_elec", i64),
        ("spin_mult", i64),
        ("num_ref", i64),
        ("ref_occ", P),
        ("nm1_domain_ptr", P),
        ("nm1_domain_idx", P),
        ("nm2_domain_ptr", P),
        ("nm2_domain_idx", P),
    ]


class TciOperator(C.Structure):
    _fields_ = [("h", P), ("chol", P), ("nchol", i64), ("core_energy", dbl)]


class TciMolecule(C.Structure):
    _fields_ = [
        ("n_atoms", i64),
        ("charges", P),
        ("coords", P),
        ("n_shells", i64),
        ("shell_atom", P),
        ("shell_l", P),
        ("shell_nprim", P),
        ("exponents", P),
        ("coefficients", P),
        ("pure_d", i64),
    ]


class TciError(RuntimeError):
    def __init__(self, code, msg):
        super().__init__(f"[{code}] {msg}")
        self.code = code


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise ImportError(f"{LIB_PATH} is missing: run `python -m tigerci_b200.build` first")
        L = C.CDLL(LIB_PATH)
        for name in EXPORTS:
            getattr(L, name)  # raises if the symbol is absent
        L.tci_last_error.argtypes = [C.c_char_p, i64]
        L.tci_space_create.argtypes = [C.POINTER(TciDeck), C.POINTER(P)]
        L.tci_space_counts.argtypes = [P, P, i64]
        L.tci_space_index_vector.argtypes = [P, i64, P, i64]
        L.tci_space_path.argtypes = [P, i64, i64, P, P]
        L.tci_space_block_counts.argtypes = [P, i64, P, i64, P]
        L.tci_space_destroy.argtypes = [P]
        L.tci_space_destroy.restype = None
        L.tci_plan_create.argtypes = [C.POINTER(TciDeck), C.POINTER(TciOperator), C.POINTER(P)]
        L.tci_plan_export.argtypes = [P, C.c_char_p]
        L.tci_plan_stats.argtypes = [P, P, i64]
        L.tci_plan_destroy.argtypes = [P]
        L.tci_plan_destroy.restype = None
        L.tci_sigma_init.argtypes = [C.POINTER(TciDeck), C.POINTER(TciOperator), i64, C.POINTER(P)]
        L.tci_sigma_init_ex.argtypes = [C.POINTER(TciDeck), C.POINTER(TciOperator), i64, P, i64, C.POINTER(P)]
        L.tci_check.argtypes = [P]
        L.tci_sigma.argtypes = [P, P, P, i64]
        L.tci_sigma_device.argtypes = [P, P, P, i64, P]
        L.tci_diag.argtypes = [P, P, i64]
        L.tci_davidson.argtypes = [P, i64, dbl, dbl, i64, P, P, P]
        L.tci_davidson_ex.argtypes = [P, i64, dbl, dbl, i64, i64, P, P, P, P]
        L.tci_davidson_gen.argtypes = [P, i64, dbl, dbl, i64, P, dbl, P, P, P]
        L.tci_acpf_gdiag.argtypes = [P, i64, dbl, P, P, i64]
        L.tci_davidson_capacity.argtypes = [i64, i64, i64, i64]
        L.tci_davidson_capacity.restype = i64
        L.tci_davidson_bytes.argtypes = [i64, i64, i64, i64]
        L.tci_davidson_bytes.restype = i64
        L.tci_dots.argtypes = [P, P, i64, i64, P, i64, P, P]
        L.tci_dots_noalloc.argtypes = [P, i64, i64, P, i64, P, P]
        L.tci_ctx_stats.argtypes = [P, P, i64]
        L.tci_profile.argtypes = [P, i64]
        L.tci_davidson_phase_times.argtypes = [P, P, i64]
        L.tci_step_times.argtypes = [P, P, i64, P, P]
        L.tci_step_name.argtypes = [P, i64, C.c_char_p, i64]
        L.tci_destroy.argtypes = [P]
        L.tci_destroy.restype = None
        L.tci_selftest_bounded_wait.argtypes = [i64, i64, P, P]
        L.tci_selftest_mma_rate.argtypes = [i64, i64, i64, i64, i64, P]
        L.tci_operator_from_records.argtypes = [i64, i64, P, P, i64, P]
        L.tci_reference_weight.argtypes = [P, P, i64, P]
        L.tci_aposteriori.argtypes = [i64, dbl, dbl, P, i64]
        L.tci_local_allext_records.argtypes = [C.POINTER(TciDeck), P, i64, P]
        L.tci_integrals_create.argtypes = [C.POINTER(TciMolecule), dbl, C.POINTER(P)]
        L.tci_integrals_info.argtypes = [P, P, i64]
        L.tci_integrals_one_electron.argtypes = [P, P, P, i64]
        L.tci_integrals_ao_cholesky.argtypes = [P, P, i64, i64]
        L.tci_integrals_ao_eri.argtypes = [P, P, i64]
        L.tci_rhf.argtypes = [P, i64, i64, dbl, P, P, P]
        L.tci_mo_operator.argtypes = [P, P, i64, P, P, i64]
        L.tci_integrals_destroy.argtypes = [P]
        L.tci_integrals_destroy.restype = None
        _lib = L
    return _lib


def last_error() -> str:
    buf = C.create_string_buffer(1024)
    lib().tci_last_error(buf, 1024)
    return buf.value.decode(errors="replace")


def check(code):
    if code != 0:
        raise TciError(code, last_error())


def ptr(a: np.ndarray):
    return a.ctypes.data_as(P) if a is not None else None
