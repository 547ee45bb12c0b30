"""Davidson-Liu: the CPU restatement (oracle) converges to the exact lowest
eigenvalues of the dense oracle Hamiltonian, and the device-resident solver
(tci_davidson) reproduces the oracle's energies."""
import numpy as np
import pytest

import tigerci_b200 as T
from cases import SMALL_CASES, case_id, oracle_deck, product_deck
from oracle import davidson as odav
from oracle import dense
from tigerci_b200.synthetic import synthetic_operator


def _op(c):
    return synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)


@pytest.mark.parametrize("c", SMALL_CASES[:5], ids=case_id)
def test_oracle_davidson_converges_to_exact_roots(c):
    h, L = _op(c)
    od = dense.DenseSigma(oracle_deck(c))
    H = od.hamiltonian(h, L)
    e_exact = np.linalg.eigvalsh(H)[:2]
    e, v, it = odav.davidson_liu(lambda x: H @ x, np.diag(H).copy(), roots=2, tol_residual=1e-8, tol_energy=1e-12)
    assert np.abs(e - e_exact).max() < 1e-9
    for q in range(2):
        assert np.linalg.norm(H @ v[q] - e[q] * v[q]) < 1e-6


@pytest.mark.gpu
@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_device_davidson_matches_oracle(c, need_gpu):
    h, L = _op(c)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    od = dense.DenseSigma(oracle_deck(c))
    H = od.hamiltonian(h, L) if od.ncsf <= 800 else None
    hd = sb.diag()
    if H is not None:
        assert np.abs(hd - np.diag(H)).max() <= 1e-12 * np.abs(np.diag(H)).max()
    roots = 2 if sb.n > 4 else 1
    e_dev, v_dev, it_dev = sb.davidson(roots, 1e-8, 1e-12, want_vectors=True)
    e_or, v_or, it_or = odav.davidson_liu(lambda x: od.sigma(h, L, x), hd, roots=roots, tol_residual=1e-8,
                                          tol_energy=1e-12)
    assert np.abs(e_dev - e_or).max() < 1e-8
    if H is not None:
        assert np.abs(e_dev - np.linalg.eigvalsh(H)[:roots]).max() < 1e-8
    # a root may stop on the energy-change criterion (is_converged, davidson.f90:564-602)
    # before its residual reaches tol_residual; its residual is then still small
    for q in range(roots):
        r = sb.sigma(v_dev[q]) - e_dev[q] * v_dev[q]
        assert np.linalg.norm(r) < 1e-5
    sb.close()


@pytest.mark.gpu
def test_contexts_do_not_share_state(need_gpu):
    """A second context created after another one frees memory gives the same
    sigma as a fresh one (device buffers start zeroed)."""
    from tigerci_b200.synthetic import random_civec

    c = SMALL_CASES[8]
    h, L = _op(c)
    a = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    x = random_civec(a.n, 2)
    ref = a.sigma(x)
    h2, L2 = synthetic_operator(c["no"], 10, seed=12, scale=0.3)
    b = T.SigmaBuilder(product_deck(c), T.Operator(h2, L2), device=0)
    _ = b.sigma(x)
    b.close()
    c2 = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    assert np.array_equal(c2.sigma(x), ref)
    a.close()
    c2.close()


@pytest.mark.gpu
def test_projection_entry_point_matches_host_dots(need_gpu):
    import torch

    c = SMALL_CASES[8]
    h, L = _op(c)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    rng = np.random.default_rng(4)
    n, m = 100003, 7
    A = torch.from_numpy(rng.standard_normal((m, n))).cuda()
    x = torch.from_numpy(rng.standard_normal(n)).cuda()
    out = torch.zeros(m, dtype=torch.float64, device="cuda")
    sb.dots(A.data_ptr(), n, m, x.data_ptr(), n, out.data_ptr())
    torch.cuda.synchronize()
    ref = A.cpu().numpy() @ x.cpu().numpy()
    assert np.abs(out.cpu().numpy() - ref).max() <= 1e-12 * np.abs(ref).max() + 1e-12
    out2 = torch.zeros_like(out)
    sb.dots(A.data_ptr(), n, m, x.data_ptr(), n, out2.data_ptr())
    torch.cuda.synchronize()
    assert torch.equal(out, out2)
    sb.close()


@pytest.mark.parametrize("roots", [1, 2])
def test_oracle_restart_under_a_disk_budget_reaches_the_same_roots(roots):
    """need_to_restart_subspace / restart_davidson_subspace (davidson_restart.f90:26-139):
    with room for only a few vectors the solver collapses onto current + previous
    Ritz vectors and still converges to the exact roots."""
    c = SMALL_CASES[3]
    h, L = _op(c)
    od = dense.DenseSigma(oracle_deck(c))
    H = od.hamiltonian(h, L)
    n = H.shape[0]
    exact = np.linalg.eigvalsh(H)[:roots]
    budget = 16 * n * (4 * roots + 2)
    e, v, it = odav.davidson_liu(lambda x: H @ x, np.diag(H).copy(), roots=roots, tol_residual=1e-9,
                                 tol_energy=1e-13, disk_space=budget)
    assert np.abs(e - exact).max() < 1e-9


def test_subspace_capacity_follows_the_budget():
    from tigerci_b200 import _lib

    L = _lib.lib()
    n = 1000
    # default budget (30 GB) leaves the reference's maxit-bound subspace
    assert L.tci_davidson_capacity(n, 1, 0, 0) == 51
    assert L.tci_davidson_capacity(n, 2, 0, 0) == 2 * 101
    # a budget for 12 vectors: restart at 12 (> 4 roots), room for the expansion after the test
    assert L.tci_davidson_capacity(n, 2, 0, 16 * n * 12) == 11 + 2
    # never below 4 vectors per root + 1 before a restart can fire
    assert L.tci_davidson_capacity(n, 2, 0, 16) == 8 + 2
    b = L.tci_davidson_bytes(n, 2, 0, 16 * n * 12)
    assert b >= 8 * n * (2 * 13 + 1)


@pytest.mark.gpu
def test_device_restart_under_a_subspace_budget(need_gpu):
    c = SMALL_CASES[3]
    h, L = _op(c)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    od = dense.DenseSigma(oracle_deck(c))
    H = od.hamiltonian(h, L)
    exact = np.linalg.eigvalsh(H)[:2]
    n = sb.n
    e_free, _, it_free = sb.davidson(2, 1e-9, 1e-13)
    e_rs, _, it_rs = sb.davidson(2, 1e-9, 1e-13, subspace_bytes=16 * n * 10)
    assert np.abs(e_free - exact).max() < 1e-8
    assert np.abs(e_rs - exact).max() < 1e-8
    assert it_rs > 5  # the capacity (11 vectors) forces restarts before convergence
    sb.close()


@pytest.mark.gpu
def test_device_solve_can_be_cancelled(need_gpu):
    c = SMALL_CASES[3]
    h, L = _op(c)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    flag = np.ones(1, dtype=np.int32)
    from tigerci_b200 import _lib

    with pytest.raises(_lib.TciError) as ei:
        sb.davidson(1, 1e-9, 1e-13, cancel=flag)
    assert ei.value.code == 7
    flag[0] = 0
    e, _, _ = sb.davidson(1, 1e-9, 1e-13, cancel=flag)  # the context stays usable
    assert np.isfinite(e).all()
    sb.close()


@pytest.mark.gpu
def test_context_reused_for_more_roots(need_gpu):
    """A context that solved for one root solves for three (larger subspace and
    reduction scratch) exactly as a fresh context does."""
    c = SMALL_CASES[8]
    h, L = _op(c)
    a = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    a.davidson(1, 1e-8, 1e-12)
    e3, _, _ = a.davidson(3, 1e-8, 1e-12)
    b = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    f3, _, _ = b.davidson(3, 1e-8, 1e-12)
    assert np.array_equal(e3, f3)
    a.close()
    b.close()
