"""A posteriori corrections (calculate_a_posteriori_corrections, aposteriori.f90:28-221) against the
blocks the reference printed after its one-root runs (tests/golden/reference_runs.json, written by
tests/golden/make_reference_runs.py): from the printed c0^2 and the printed energies the five corrections
must come out as printed (to the print's eight digits), for both printed definitions of c0^2."""
import json
import os

import numpy as np
import pytest

import tigerci_b200 as T

HERE = os.path.dirname(os.path.abspath(__file__))
RUNS = [r for r in json.load(open(os.path.join(HERE, "golden", "reference_runs.json")))["runs"]
        if r["printed"].get("aposteriori")]


@pytest.mark.parametrize("r", RUNS, ids=[r["run"] for r in RUNS])
def test_corrections_from_the_printed_weight_match_the_printed_ones(r):
    p = r["printed"]
    d = r["deck"]
    e_corr = p["roots"][-1] - p["reference_energy"]
    n_corr = d["num_elec"] - 2 * d["num_frozen"]
    for block in p["aposteriori"]:
        got = T.aposteriori(block["c0sq"], e_corr, n_corr)
        for name, v in got.items():
            # c0^2 is printed to 8 digits: 1 - c0^2 carries its rounding (5e-9) relative to its own size
            tol = abs(block[name]) * (1e-7 + 6e-9 / (1.0 - block["c0sq"])) + 1e-12
            assert abs(v - block[name]) <= tol, (name, v, block[name])


def test_corrections_refused_where_the_reference_prints_none():
    with pytest.raises(Exception):
        T.aposteriori(0.95, -0.1, 2)  # fewer than 4 correlated electrons
    with pytest.raises(Exception):
        T.aposteriori(0.4, -0.1, 10)  # c0^2 <= 1/2: the Davidson-Silver and Pople forms are singular


def test_reference_weight_sums_the_reference_configurations():
    deck = T.Deck(8, 2, 2, 6, 1, ["2220", "2202"])
    sp = T.CsfSpace(deck)
    n = sp.counts()["total_csfs"]
    g, cls = sp.acpf_gdiag(1)
    c = np.random.default_rng(3).standard_normal(n)
    assert abs(sp.reference_weight(c) - float((c[cls == 1] ** 2).sum())) <= 1e-12 * float((c ** 2).sum())
