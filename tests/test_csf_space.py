"""CSF space (graph, tree search, index vectors) against the known-answer
counts printed by the reference's own regression runs
(tests/golden/csf_counts.json, see tests/golden/make_golden.py)."""
import json
import os

import pytest

import tigerci_b200 as T
from oracle import sgga

GOLD = json.load(open(os.path.join(os.path.dirname(__file__), "golden", "csf_counts.json")))


def _id(r):
    return r["source"].split("/")[2] + ("" if r["nonlocal"] else "-valence")


@pytest.mark.parametrize("r", GOLD, ids=[_id(r) for r in GOLD])
def test_oracle_matches_reference_outputs(r):
    deck = sgga.Deck(r["num_orbitals"], r["num_inactive"], r["num_active"], r["num_elec"], r["spin_mult"], r["refs"],
                     r["num_frozen"])
    sp = sgga.build_space(deck)
    assert sp.total_configurations == r["total_configurations"]
    assert sp.open_shells == r["open_shells"]
    assert sp.num_valence == r["num_valence"]
    assert {str(k): v for k, v in sp.counts[0].items()} == {k: v[1] for k, v in r["counts"]["valence"].items()}
    if r["nonlocal"]:
        assert (sp.num_nm1, sp.num_nm2, sp.total_csfs) == (r["num_nm1"], r["num_nm2"], r["total_csfs"])
        assert sp.total_configurations - sp.removed == r["kept"]
        assert {str(k): v for k, v in sp.counts[1].items()} == {k: v[1] for k, v in r["counts"]["nm1"].items()}
        assert {str(k): v for k, v in sp.counts[2].items()} == {k: v[1] for k, v in r["counts"]["nm2"].items()}


@pytest.mark.parametrize("r", GOLD, ids=[_id(r) for r in GOLD])
def test_product_matches_reference_outputs(r):
    deck = T.Deck(r["num_orbitals"], r["num_inactive"], r["num_active"], r["num_elec"], r["spin_mult"], r["refs"],
                  num_frozen=r["num_frozen"])
    sp = T.CsfSpace(deck)
    c = sp.counts()
    assert c["total_configurations"] == r["total_configurations"]
    assert c["open_shells"] == r["open_shells"]
    assert c["num_valence"] == r["num_valence"]
    assert sp.block_counts(0) == {int(k): tuple(v) for k, v in r["counts"]["valence"].items()}
    if r["nonlocal"]:
        assert (c["num_nm1"], c["num_nm2"], c["total_csfs"]) == (r["num_nm1"], r["num_nm2"], r["total_csfs"])
        assert c["total_configurations"] - c["removed"] == r["kept"]
        assert sp.block_counts(1) == {int(k): tuple(v) for k, v in r["counts"]["nm1"].items()}
        assert sp.block_counts(2) == {int(k): tuple(v) for k, v in r["counts"]["nm2"].items()}


@pytest.mark.parametrize("r", [g for g in GOLD if g["total_configurations"] < 200000], ids=lambda r: _id(r))
def test_index_vectors_bit_exact_vs_oracle(r):
    """Every index-vector entry (1-based offsets / kill_number) and every path
    occupation agrees between product and oracle."""
    deck = T.Deck(r["num_orbitals"], r["num_inactive"], r["num_active"], r["num_elec"], r["spin_mult"], r["refs"],
                  num_frozen=r["num_frozen"])
    sp = T.CsfSpace(deck)
    osp = sgga.build_space(sgga.Deck(r["num_orbitals"], r["num_inactive"], r["num_active"], r["num_elec"],
                                     r["spin_mult"], r["refs"], r["num_frozen"]))
    for kind, key in ((0, "off"), (1, "off"), (2, "off"), (3, "off_aa")):
        iv = sp.index_vector(kind)
        paths = osp.paths[2 if kind == 3 else kind]
        ref = [(p[key] + 1) if p[key] is not None else T.KILL_NUMBER for p in paths]
        assert iv.tolist() == ref
    for kind in range(3):
        for p in osp.paths[kind][:200]:
            occ, info = sp.path(kind, p["lex"])
            assert occ.tolist() == p["occ"]
            assert info["singles"] == p["singles"]


def test_removed_paths_and_errors():
    # references inconsistent with the electron count are rejected with a status code
    with pytest.raises(Exception) as e:
        T.CsfSpace(T.Deck(6, 2, 1, 4, 1, ["221"]))
    assert "electron" in str(e.value)
    # a frozen orbital removes every path that excites out of it
    a = T.CsfSpace(T.Deck(8, 3, 1, 8, 1, ["2222"])).counts()
    b = T.CsfSpace(T.Deck(8, 3, 1, 8, 1, ["2222"], num_frozen=1)).counts()
    assert b["total_csfs"] < a["total_csfs"]
    osp = sgga.build_space(sgga.Deck(8, 3, 1, 8, 1, ["2222"], 1))
    assert osp.total_csfs == b["total_csfs"]
