"""Molecular workloads through the front end: H2O / cc-pVDZ (24 functions), O 1s
frozen, CAS(4,4) references (19) on canonical RHF orbitals, CD THRESHOLD
1e-6, singlet, one root, Davidson stopped by the residual (1e-6).

The host part (front end, deck) runs on CPU; the GPU test solves it on the
device in FP64 and in the mixed form and compares with the oracle: its
Davidson (davidson.f90 restated) over the integral-direct CPU sigma
(plancpu.c), 1e-8 Eh for FP64 and 1 uEh for the mixed form."""
import numpy as np
import pytest

import tigerci_b200 as T
from oracle import davidson, dense
from tigerci_b200 import molecule as M


def test_water_problem_shapes():
    deck, op, info = M.water_c1()
    assert info["nbf"] == 24 and deck.num_orbitals == 24
    assert (deck.num_frozen, deck.num_inactive, deck.num_active, deck.num_external) == (1, 3, 4, 17)
    assert len(deck.refs) == 19 and all(r.startswith("222") for r in deck.refs)
    assert deck.num_elec == 10
    assert abs(info["e_scf"] - (-76.0268)) < 1e-3  # RHF/cc-pVDZ of water near its experimental geometry
    assert T.CsfSpace(deck).counts()["total_csfs"] == 40539


def test_cas_references():
    import json
    import os

    assert len(M.cas_references(0, 4, 4, 1)) == 19
    assert M.cas_references(1, 2, 2, 1) == ["220", "211", "202"]
    # the reference's Ethylene triplet deck lists exactly the triplet CAS(4,4) occupations
    runs = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "reference_runs.json")))["runs"]
    eth = next(r for r in runs if r["run"] == "Ethylene_HighSpin")
    assert set(M.cas_references(6, 4, 4, 3)) == set(eth["deck"]["refs"])


def _oracle_energy(deck, op, tmp_path):
    p = str(tmp_path / "c1.plan")
    T.Plan(deck, op).export(p)
    dense.use_blas()
    pc = dense.PlanSigmaCPU(p, op.chol)
    d = pc.diag()
    e, _, it = davidson.davidson_liu(lambda x: pc.sigma(x, integrals=False), d, 1, 1e-6, 1e-10)
    pc.close()
    return float(e[0]) + op.core_energy


@pytest.mark.gpu
def test_water_mrsdci_on_device_against_oracle(need_gpu, tmp_path):
    deck, op, info = M.water_c1()
    e_oracle = _oracle_energy(deck, op, tmp_path)
    for form, tol in (("fp64", 1e-8), ("tf32x3", 1e-6)):
        sb = T.SigmaBuilder(deck, op, device=0, precision=form)
        e, _, it = sb.davidson(1, 1e-6, 1e-10)
        sb.close()
        assert abs(e[0] + op.core_energy - e_oracle) <= tol, (form, e[0] + op.core_energy, e_oracle)
