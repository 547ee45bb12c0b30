"""The C-ABI library loads without a GPU and exports every entry point
declared in include/*.h; host-only entry points work on CPU."""
import ctypes
import glob
import os
import re

import numpy as np
import pytest

import tigerci_b200 as T
from tigerci_b200 import _lib

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared_symbols():
    syms = set()
    for hdr in glob.glob(os.path.join(ROOT, "include", "*.h")):
        txt = open(hdr).read()
        txt = re.sub(r"/\*.*?\*/", "", txt, flags=re.S)
        for m in re.finditer(r"^\s*(?:int|int64_t|void|const char\s*\*)\s+(tci_\w+)\s*\(", txt, flags=re.M):
            syms.add(m.group(1))
    return syms


def test_library_exports_every_declared_symbol():
    lib = ctypes.CDLL(_lib.LIB_PATH)
    syms = declared_symbols()
    assert len(syms) >= 15
    for s in sorted(syms):
        assert hasattr(lib, s), s
    assert set(_lib.EXPORTS) <= syms


def test_library_is_in_tree():
    assert os.path.dirname(_lib.LIB_PATH) == os.path.join(ROOT, "tigerci_b200")


def test_null_arguments_return_error_codes():
    lib = _lib.lib()
    assert lib.tci_space_create(None, None) != 0
    assert lib.tci_space_counts(None, None, 0) != 0
    assert lib.tci_plan_create(None, None, None) != 0
    assert lib.tci_sigma(None, None, None, 0) != 0
    assert lib.tci_plan_stats(None, None, 0) != 0


def test_plan_stats_on_cpu():
    deck = T.Deck(10, 2, 2, 6, 1, ["2220", "2202"])
    from tigerci_b200.synthetic import synthetic_operator

    h, L = synthetic_operator(10, 8, seed=3, scale=0.3)
    st = T.Plan(deck, T.Operator(h, L)).stats()
    assert st["total_csfs"] == T.CsfSpace(deck).counts()["total_csfs"]
    assert st["flops_allext"] > 0 and st["n_steps"] > 5


def test_operator_from_records_follows_mo_ind_inv():
    """Records addressed through the reference's mo_ind_inv: a permutation with zero (skipped) pairs, the
    identity, and an entry out of range."""
    import tigerci_b200 as T

    rng = np.random.default_rng(4)
    n, nchol = 5, 7
    npair = n * (n + 1) // 2
    full = rng.standard_normal((npair, nchol))
    keep = np.sort(rng.choice(npair, size=11, replace=False))
    full[np.setdiff1d(np.arange(npair), keep)] = 0.0
    order = rng.permutation(len(keep))
    records = full[keep[order]]
    inv = np.zeros(npair, dtype=np.int64)
    inv[keep[order]] = np.arange(1, len(keep) + 1)
    h = np.eye(n)
    op = T.Operator.from_records(h, records, inv)
    assert np.array_equal(op.chol, full)
    ident = T.Operator.from_records(h, full, np.arange(1, npair + 1))
    assert np.array_equal(ident.chol, full)
    bad = inv.copy()
    bad[3] = len(keep) + 1
    with pytest.raises(Exception):
        T.Operator.from_records(h, records, bad)
