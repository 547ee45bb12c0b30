"""All-external term over pair domains (tci_local_*): the oracle's integral
form over domains against the Cholesky form it is applied in, and the device
(FP64 and mixed) against the oracle."""
import numpy as np
import pytest

from oracle import dense
from tigerci_b200 import local
from tigerci_b200.synthetic import synthetic_operator


def _problem(n_pairs=12, n_int=5, n_virt=30, dmin=3, dmax=14, nchol=40, seed=3):
    heads, dom, total = local.pair_domain_problem(n_pairs, n_int, n_virt, dmin, dmax, seed=seed)
    h, L = synthetic_operator(n_int + n_virt, nchol, seed=seed + 1, scale=0.5)
    c = np.random.default_rng(seed + 2).standard_normal(total)
    return heads, dom, total, L, c


def _pair(p, q):
    return p * (p + 1) // 2 + q if p >= q else q * (q + 1) // 2 + p


def _cholesky_form(n_int, L, heads, dom, c):
    """sigma_hk = pack(1/2 sum_J L^J_h D_hk L^J_h) in numpy (the device's formulation)."""
    s = np.zeros_like(c)
    for off_ab, off_aa, nsf_ab, nsf_aa, nsing, doff, n in heads:
        d = dom[doff:doff + n]
        idx = np.array([[_pair(n_int + a, n_int + b) for b in d] for a in d])
        Lh = np.moveaxis(L[idx], 2, 0)  # (J, n, n)
        nab = n * (n - 1) // 2
        iu, ju = np.tril_indices(n, -1)  # i > j, pair index i(i-1)/2 + j in this order
        for k in range(max(nsf_ab, nsf_aa)):
            p = 1.0 if k < nsing else -1.0
            D = np.zeros((n, n))
            if k < nsf_aa:
                D[np.arange(n), np.arange(n)] = np.sqrt(2) * c[off_aa + k * n:off_aa + (k + 1) * n]
            if k < nsf_ab:
                x = c[off_ab + k * nab:off_ab + (k + 1) * nab]
                D[ju, iu] = x
                D[iu, ju] = p * x
            R = 0.5 * np.einsum("Jac,cd,Jdb->ab", Lh, D, Lh)
            if k < nsf_ab:
                s[off_ab + k * nab:off_ab + (k + 1) * nab] += R[ju, iu] + p * R[iu, ju]
            if k < nsf_aa:
                s[off_aa + k * n:off_aa + (k + 1) * n] += np.sqrt(2) * np.diag(R)
    return s


def test_oracle_integral_form_equals_cholesky_form():
    heads, dom, total, L, c = _problem()
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    sc = _cholesky_form(5, L, heads, dom, c)
    assert np.abs(so - sc).max() <= 1e-12 * np.abs(so).max()


def test_oracle_local_equals_non_local_when_every_domain_is_everything():
    """With every domain the full external space the local oracle is the
    non-local all-external oracle restricted to these heads."""
    heads, dom, total = local.pair_domain_problem(6, 4, 9, 9, 9, seed=5)
    assert all(h[6] == 9 for h in heads)
    h, L = synthetic_operator(13, 20, seed=6, scale=0.5)
    c = np.random.default_rng(1).standard_normal(total)
    so = dense.allext_local_sigma(4, L, heads, dom, c)
    sc = _cholesky_form(4, L, heads, dom, c)
    assert np.abs(so - sc).max() <= 1e-12 * np.abs(so).max()


def test_pair_domain_problem_shapes():
    heads, dom, total = local.pair_domain_problem(600, 35, 400, 20, 180, seed=99)
    assert len(heads) == 600
    n = heads[:, 6]
    assert n.min() >= 20 and n.max() <= 180
    assert ((heads[:, 2] == 1) | (heads[:, 2] == 2)).all()
    # domains sorted and within the external space
    for off_ab, off_aa, nsf_ab, nsf_aa, nsing, doff, m in heads[:20]:
        d = dom[doff:doff + m]
        assert (np.diff(d) > 0).all() and d.min() >= 0 and d.max() < 400
    last = heads[-1]
    assert total == last[0] + last[2] * last[6] * (last[6] - 1) // 2


@pytest.mark.gpu
@pytest.mark.parametrize("chunk_bytes", [16e9, 3e5])
def test_device_fp64_matches_oracle(chunk_bytes, need_gpu):
    heads, dom, total, L, c = _problem()
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    op = local.LocalAllExternal(5, 30, L, heads, dom, total, device=0, precision="fp64", chunk_bytes=chunk_bytes)
    sd = op.apply(c)
    st = op.stats()
    if chunk_bytes < 1e6:
        assert st["chunk"] < 40  # several chunks and a shorter last one
    assert np.abs(sd - so).max() <= 1e-10 * np.abs(so).max()
    assert np.array_equal(sd, op.apply(c))  # deterministic
    op.close()


@pytest.mark.gpu
def test_device_mixed_matches_oracle(need_gpu):
    heads, dom, total, L, c = _problem(n_pairs=15, n_virt=60, dmin=10, dmax=50, nchol=64)
    so = dense.allext_local_sigma(5, L, heads, dom, c)
    op = local.LocalAllExternal(5, 60, L, heads, dom, total, device=0, precision="tf32x3")
    sd = op.apply(c)
    assert np.linalg.norm(sd - so) <= 2e-5 * np.linalg.norm(so)
    assert np.array_equal(sd, op.apply(c))
    op.close()


@pytest.mark.gpu
def test_device_apply_accumulates_on_a_stream(need_gpu):
    import torch

    heads, dom, total, L, c = _problem()
    op = local.LocalAllExternal(5, 30, L, heads, dom, total, device=0)
    ref = op.apply(c)
    ct = torch.from_numpy(c).cuda()
    st = torch.ones(total, dtype=torch.float64, device="cuda")
    s = torch.cuda.Stream()
    with torch.cuda.stream(s):
        op.apply_device(ct.data_ptr(), st.data_ptr(), s.cuda_stream)
    torch.cuda.synchronize()
    assert np.abs(st.cpu().numpy() - 1.0 - ref).max() <= 1e-12 * np.abs(ref).max()
    op.close()
