"""Device sigma build (through the C ABI) against the oracle."""
import numpy as np
import pytest

import tigerci_b200 as T
from cases import SMALL_CASES, case_id, oracle_deck, product_deck
from oracle import dense
from tigerci_b200.synthetic import random_civec, synthetic_operator

pytestmark = pytest.mark.gpu

# plain-FP64 sigma must agree with the oracle within 1e-10 relative
RTOL = 1e-10


@pytest.mark.parametrize("c", SMALL_CASES, ids=case_id)
def test_device_sigma_equals_dense_oracle(c, need_gpu):
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    od = dense.DenseSigma(oracle_deck(c))
    for seed in (1, 2):
        x = random_civec(od.ncsf, seed)
        ref = od.sigma(h, L, x)
        got = sb.sigma(x)
        assert np.abs(got - ref).max() <= RTOL * np.abs(ref).max()
    sb.close()


def test_htimesc_accumulates_and_is_deterministic(need_gpu):
    c = SMALL_CASES[8]
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    x = random_civec(sb.n, 3)
    s1 = sb.sigma(x)
    s2 = sb.sigma(x)
    assert np.array_equal(s1, s2)  # bitwise reproducible
    acc = np.ones(sb.n)
    sb.htimesc(x, acc)
    assert np.array_equal(acc - 1.0, s1) or np.abs(acc - 1.0 - s1).max() < 1e-15 * np.abs(s1).max() + 1e-15


def _medium():
    # 6 internal (4 inactive, 2 active), 20 externals, two references
    deck = T.Deck(26, 4, 2, 10, 1, ["222220", "222202"])
    h, L = synthetic_operator(26, 40, seed=21, scale=0.25, diag_range=(-6, 1), offdiag_sigma=0.05)
    return deck, h, L


def test_medium_case_against_plan_interpreter_and_reference_allext(need_gpu, tmp_path):
    from plan_exec import PlanInterpreter
    from oracle import sgga

    deck, h, L = _medium()
    op = T.Operator(h, L)
    sb = T.SigmaBuilder(deck, op, device=0)
    plan = T.Plan(deck, op)
    p = str(tmp_path / "p.bin")
    plan.export(p)
    pi = PlanInterpreter(p, h, L)
    x = random_civec(sb.n, 5)
    got = sb.sigma(x)
    ref = pi.sigma(x)
    assert np.abs(got - ref).max() <= RTOL * np.abs(ref).max()
    # the all-external part alone against the reference-form loop (mod_1:3240-3518)
    osp = sgga.build_space(sgga.Deck(26, 4, 2, 10, 1, ["222220", "222202"]))
    nv, n1 = osp.num_valence, osp.num_nm1
    xd = np.zeros(sb.n)
    xd[nv + n1:] = x[nv + n1:]
    Lz = L.copy()
    hz = np.zeros_like(h)
    # isolate the (ab|cd) term: only external-external Cholesky rows survive
    nint = 6
    for p_ in range(26):
        for q_ in range(p_ + 1):
            if p_ < nint or q_ < nint:
                Lz[p_ * (p_ + 1) // 2 + q_] = 0.0
    sbz = T.SigmaBuilder(deck, T.Operator(hz, Lz), device=0)
    s_allext = sbz.sigma(xd)[nv + n1:]
    s_ref = dense.allext_sigma(osp, nint, 20, Lz, xd)[nv + n1:]
    assert np.abs(s_allext - s_ref).max() <= RTOL * np.abs(s_ref).max()


def test_hermiticity_and_linearity_at_size(need_gpu):
    """Size-independent properties on a larger space: <x|Hy> = <y|Hx>, and
    H(ax + by) = aHx + bHy."""
    deck = T.Deck(16 + 60, 8, 8, 16, 1, ["2" * 8 + "0" * 8])
    h, L = synthetic_operator(76, 200, seed=1234)
    sb = T.SigmaBuilder(deck, T.Operator(h, L), device=0)
    x = random_civec(sb.n, 1)
    y = random_civec(sb.n, 2)
    hx, hy = sb.sigma(x), sb.sigma(y)
    assert abs(x @ hy - y @ hx) <= 1e-11 * abs(x @ hy)
    hz = sb.sigma(2.0 * x - 3.0 * y)
    assert np.abs(hz - (2.0 * hx - 3.0 * hy)).max() <= 1e-11 * np.abs(hz).max()


def test_error_codes(need_gpu):
    c = SMALL_CASES[0]
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    with pytest.raises(T._lib.TciError if hasattr(T, "_lib") else Exception):
        sb.htimesc(np.zeros(sb.n + 1), np.zeros(sb.n + 1))
    with pytest.raises(Exception):
        T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=99)


def test_device_pointer_entry_point(need_gpu):
    import torch

    c = SMALL_CASES[2]
    h, L = synthetic_operator(c["no"], 10, seed=11, scale=0.3, diag_range=(-3, 1), offdiag_sigma=0.1)
    sb = T.SigmaBuilder(product_deck(c), T.Operator(h, L), device=0)
    x = random_civec(sb.n, 4)
    ref = sb.sigma(x)
    xc = torch.from_numpy(x).cuda()
    sc = torch.full_like(xc, 0.5)
    s = torch.cuda.current_stream()
    sb.htimesc_device(xc.data_ptr(), sc.data_ptr(), sb.n, s.cuda_stream)
    torch.cuda.synchronize()
    assert np.abs(sc.cpu().numpy() - 0.5 - ref).max() <= 1e-14 * np.abs(ref).max() + 1e-15
