"""The host-built sigma plan (coupling coefficients, task tables, dense
pair-matrix algebra) replayed by a numpy interpreter equals sigma = H c of
the dense oracle in the reference's CSF basis, for every term class."""
import numpy as np
import pytest

import tigerci_b200 as T
from cases import SMALL_CASES, case_id, oracle_deck, product_deck
from oracle import dense
from plan_exec import PlanInterpreter
from tigerci_b200.synthetic import random_civec, synthetic_operator


def _setup(c, tmp_path, nchol=10, seed=11):
    h, L = synthetic_operator(c["no"], nchol, seed=seed, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    plan = T.Plan(product_deck(c), T.Operator(h, L))
    p = str(tmp_path / "plan.bin")
    plan.export(p)
    return h, L, PlanInterpreter(p, h, L), dense.DenseSigma(oracle_deck(c))


@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_plan_sigma_equals_dense_oracle(c, tmp_path):
    h, L, pi, od = _setup(c, tmp_path)
    for seed in (1, 2):
        x = random_civec(od.ncsf, seed)
        ref = od.sigma(h, L, x)
        got = pi.sigma(x)
        assert np.abs(got - ref).max() <= 1e-12 * np.abs(ref).max()


@pytest.mark.parametrize("c", SMALL_CASES[:3], ids=case_id)
def test_plan_block_classes(c, tmp_path):
    """Each source block (valence / N-1 / N-2) into each target block."""
    h, L, pi, od = _setup(c, tmp_path, seed=3)
    sp = od.space
    nv, n1 = sp.num_valence, sp.num_nm1
    blocks = [slice(0, nv), slice(nv, nv + n1), slice(nv + n1, od.ncsf)]
    for sb in blocks:
        x = np.zeros(od.ncsf)
        x[sb] = random_civec(od.ncsf, 4)[sb]
        ref = od.sigma(h, L, x)
        got = pi.sigma(x)
        assert np.abs(got - ref).max() <= 1e-12 * max(1.0, np.abs(ref).max())


def test_one_electron_only_operator(tmp_path):
    """Zero Cholesky vectors isolate the one-electron couplings of every class."""
    c = SMALL_CASES[2]
    h, L = synthetic_operator(c["no"], 4, seed=2, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.2)
    L[:] = 0.0
    plan = T.Plan(product_deck(c), T.Operator(h, L))
    p = str(tmp_path / "p.bin")
    plan.export(p)
    pi = PlanInterpreter(p, h, L)
    od = dense.DenseSigma(oracle_deck(c))
    x = random_civec(od.ncsf, 9)
    ref = od.sigma(h, L, x)
    assert np.abs(pi.sigma(x) - ref).max() <= 1e-12 * np.abs(ref).max()


def test_plan_is_deterministic(tmp_path):
    c = SMALL_CASES[5]
    h, L, pi, od = _setup(c, tmp_path)
    x = random_civec(od.ncsf, 3)
    assert np.array_equal(pi.sigma(x), pi.sigma(x))


@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_plan_diagonal_equals_dense_diagonal(c, tmp_path):
    """H_ii assembled from zero-external betas, same-head operator diagonals
    and the W diagonals (replaces diag_element, diag_element_mod_2.f90:83)."""
    h, L, pi, od = _setup(c, tmp_path)
    if od.ncsf > 800:
        pytest.skip("dense diagonal too large")
    H = od.hamiltonian(h, L)
    assert np.abs(pi.diagonal() - np.diag(H)).max() <= 1e-12 * np.abs(np.diag(H)).max()


_EXPORT = r"""
import sys
sys.path.insert(0, {root!r})
import tigerci_b200 as T
from tigerci_b200.synthetic import synthetic_operator
deck = T.Deck(26, 4, 2, 10, 1, ["222220", "222202"])
h, L = synthetic_operator(26, 40, seed=21, scale=0.25, diag_range=(-6, 1), offdiag_sigma=0.05)
T.Plan(deck, T.Operator(h, L)).export({path!r})
"""


def test_plan_bytes_do_not_depend_on_thread_count(tmp_path):
    """The plan builder runs heads in parallel (zero-external blocks, three-/one-external
    couplings, sv rows, the (iq|jk) table); the exported plan is the same byte for byte
    with one thread and with four."""
    import os
    import subprocess
    import sys

    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    out = []
    for threads in ("1", "4"):
        path = str(tmp_path / f"plan_{threads}.bin")
        env = dict(os.environ, OMP_NUM_THREADS=threads)
        subprocess.run([sys.executable, "-c", _EXPORT.format(root=root, path=path)], env=env, check=True,
                       timeout=300)
        out.append(open(path, "rb").read())
    assert len(out[0]) > 0 and out[0] == out[1]
