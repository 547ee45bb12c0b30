"""Spin functions: the genealogical (Clebsch-Gordan) expansion used by the
product reproduces the transposition matrices of the reference's SFT-graph
algorithm (spin_mod.f90:526-830, restated in oracle/sgga.py), with the
reference's (-1)^P convention: T_ref(i,j) = -<theta|P(i,j)|theta>."""
import numpy as np
import pytest

from oracle import sgga


@pytest.mark.parametrize("os_,mult", [(2, 1), (4, 1), (6, 1), (8, 1), (3, 2), (5, 2), (7, 2), (4, 3), (6, 3), (6, 5),
                                      (7, 4), (10, 1)])
def test_transpositions_match_reference(os_, mult):
    fsn_all, sft, sm = sgga.spin_tables(os_, mult)
    nsf = fsn_all[os_]
    cyc = sgga.make_cycles(os_, nsf, sft, sm)
    tr = sgga.make_transpositions(os_, nsf, cyc)
    strings, th = sgga.yk_expansion(sm, os_, nsf, mult)
    assert np.allclose(th.T @ th, np.eye(nsf), atol=1e-13)
    idx = {x: i for i, x in enumerate(strings)}
    for (i, j), T in tr.items():
        P = np.zeros((len(strings), len(strings)))
        for r, x in enumerate(strings):
            bi, bj = (x >> (i - 1)) & 1, (x >> (j - 1)) & 1
            y = x & ~((1 << (i - 1)) | (1 << (j - 1))) | (bj << (i - 1)) | (bi << (j - 1))
            P[idx[y], r] = 1
        assert np.allclose(T, -(th.T @ P @ th), atol=1e-12), (i, j)


@pytest.mark.parametrize("os_,mult", [(6, 1), (7, 2), (8, 3)])
def test_lower_open_shell_functions_are_padded_prefixes(os_, mult):
    """Functions for s < open_shells are the first fsn(s) SFT functions with
    ground-level singlet pairs on the arcs above s (spin_mod.f90:1004-1014)."""
    fsn_all, sft, sm = sgga.spin_tables(os_, mult)
    for s in range(mult - 1, os_ + 1, 2):
        for f in range(fsn_all[s]):
            assert sm[s, f] == 1
            assert all(sm[v, f] in (1, 2) for v in range(s, os_ + 1))


def test_fsn_counts():
    # number of spin functions = number of branching-diagram paths
    fsn_all, _, _ = sgga.spin_tables(10, 1)
    assert [fsn_all[s] for s in range(0, 11, 2)] == [1, 1, 2, 5, 14, 42]
    fsn_all, _, _ = sgga.spin_tables(9, 2)
    assert [fsn_all[s] for s in range(1, 10, 2)] == [1, 2, 5, 14, 42]
