"""The request server (tci_server_*): admission against the HBM budget, arrival
order, cancellation, host-side fault injection (a worker thread that dies,
corrupted input) and the serving workload generator.  The scheduling tests run
the server without device work (schedule_only) on CPU; the GPU test checks that
a solve gives the same roots alone and in a mix of concurrent solves."""
import time

import numpy as np
import pytest

from tigerci_b200 import serve
from tigerci_b200._lib import TciError


def small_problem(i, n_atoms=8):
    return serve.request_problem(serve.RequestSpec(i, 0.0, n_atoms, 1.4 + 0.1 * i, 1 + i % 3))


def test_stream_is_seeded_and_has_the_workload_distribution():
    a = serve.hn_chain_stream(256, rate=4.0, seed=7)
    b = serve.hn_chain_stream(256, rate=4.0, seed=7)
    assert a == b
    arr = np.array([s.arrival for s in a])
    assert (np.diff(arr) > 0).all()
    assert abs(np.mean(np.diff(arr)) - 0.25) < 0.05  # Poisson at 4 requests/s
    ns = {s.n_atoms for s in a}
    assert ns <= set(range(8, 25, 2)) and len(ns) == 9
    assert all(1.4 <= s.spacing <= 3.0 for s in a)
    assert {s.nroots for s in a} == {1, 2, 3, 4}


@pytest.mark.parametrize("n", [8, 16, 24])
def test_request_problem_has_the_chain_sizes(n):
    deck, op = serve.request_problem(serve.RequestSpec(0, 0.0, n, 2.0, 1))
    assert deck.num_orbitals == 5 * n
    assert deck.num_internal == n // 2 + 1
    assert deck.num_external == 5 * n - n // 2 - 1
    assert deck.num_elec == n and len(deck.refs) == 3
    assert op.nchol == 20 * n


def test_admission_respects_the_budget_and_rejects_oversized_requests():
    probs = [small_problem(i, n) for i, n in enumerate([8, 10, 12, 8, 10, 12, 8, 14])]
    budget = 0.3e9
    with serve.Server(slots=4, hbm_budget=budget, schedule_only=True, schedule_only_ms=40, precision="fp64",
                      planners=2) as srv:
        ids = [srv.submit(d, o, nroots=1 + k % 3) for k, (d, o) in enumerate(probs)]
        res = [srv.wait(i, timeout=60) for i in ids]
        st = srv.stats()
    assert st["peak_reserved_bytes"] <= budget
    assert st["reserved_bytes"] == 0
    over = [r for r in res if r.reserved_bytes > budget]
    assert over, "the largest request should not fit this budget"
    for r in res:
        if r.reserved_bytes > budget:
            assert r.status == 5 and r.t_admitted < 0
        else:
            assert r.status == 0 and r.t_admitted >= r.t_planned >= r.t_submit
    assert st["succeeded"] + st["failed"] == len(probs)


def test_one_slot_admits_in_arrival_order():
    """Planned requests are admitted in arrival order (with several planners a
    request whose plan is still being built does not hold back later ones)."""
    probs = [small_problem(i) for i in range(6)]
    with serve.Server(slots=1, hbm_budget=100e9, schedule_only=True, schedule_only_ms=30, precision="fp64",
                      planners=1) as srv:
        ids = [srv.submit(d, o) for d, o in probs]
        res = [srv.wait(i, timeout=60) for i in ids]
        st = srv.stats()
    adm = [r.t_admitted for r in res]
    assert adm == sorted(adm)
    assert st["peak_running"] == 1
    # continuous batching: later requests were planned while earlier ones held the slot
    assert max(r.t_planned for r in res) < res[-1].t_admitted


def test_several_slots_overlap():
    probs = [small_problem(i) for i in range(8)]
    with serve.Server(slots=4, hbm_budget=100e9, schedule_only=True, schedule_only_ms=200, precision="fp64") as srv:
        ids = [srv.submit(d, o) for d, o in probs]
        for i in ids:
            srv.wait(i, timeout=60)
        st = srv.stats()
    assert st["peak_running"] >= 2
    assert st["p50_s"] > 0 and st["p99_s"] >= st["p50_s"] and st["solves_per_s"] > 0


def test_cancel_queued_and_running_requests():
    probs = [small_problem(i) for i in range(3)]
    with serve.Server(slots=1, hbm_budget=100e9, schedule_only=True, schedule_only_ms=5000, precision="fp64") as srv:
        ids = [srv.submit(d, o) for d, o in probs]
        t = time.time()
        while srv.stats()["running"] < 1 and time.time() - t < 30:
            time.sleep(0.01)
        srv.cancel(ids[2])  # still queued
        srv.cancel(ids[0])  # running
        r0, r2 = srv.wait(ids[0], timeout=30), srv.wait(ids[2], timeout=30)
        assert r0.status == serve.STATUS_CANCELLED and r2.status == serve.STATUS_CANCELLED
        assert time.time() - t < 5  # the running one stopped early
        srv.cancel(ids[1])
        assert srv.wait(ids[1], timeout=30).status == serve.STATUS_CANCELLED
        assert srv.stats()["cancelled"] == 3


def test_a_dead_worker_is_replaced_and_its_request_requeued():
    probs = [small_problem(i) for i in range(5)]
    with serve.Server(slots=2, hbm_budget=100e9, schedule_only=True, schedule_only_ms=30, precision="fp64",
                      inject_worker_exit_at=2) as srv:
        ids = [srv.submit(d, o) for d, o in probs]
        res = [srv.wait(i, timeout=60) for i in ids]
        st = srv.stats()
    assert all(r.status == 0 for r in res)
    assert st["worker_restarts"] == 1 and st["succeeded"] == 5 and st["reserved_bytes"] == 0


def test_corrupted_input_is_rejected_on_the_host():
    deck, op = small_problem(0)
    op.chol[3, 2] = np.nan
    with serve.Server(slots=1, hbm_budget=100e9, schedule_only=True, precision="fp64") as srv:
        with pytest.raises(TciError) as ei:
            srv.submit(deck, op)
        assert ei.value.code == 3


def test_wait_times_out_without_losing_the_request():
    deck, op = small_problem(0)
    with serve.Server(slots=1, hbm_budget=100e9, schedule_only=True, schedule_only_ms=300, precision="fp64") as srv:
        rid = srv.submit(deck, op)
        with pytest.raises(TciError) as ei:
            srv.wait(rid, timeout=0.001)
        assert ei.value.code == 6
        assert srv.wait(rid, timeout=30).status == 0


@pytest.mark.gpu
def test_results_are_the_same_alone_and_in_the_mix(need_gpu):
    """Each request's roots do not depend on what runs beside it (deterministic
    kernels, one context and stream per request)."""
    specs = [serve.RequestSpec(i, 0.0, n, 1.4 + 0.2 * i, r) for i, (n, r) in enumerate([(8, 2), (10, 1), (8, 3),
                                                                                        (12, 2), (10, 2), (8, 1)])]
    probs = [serve.request_problem(s) for s in specs]
    by_form = {}
    for precision in ("fp64", "tf32x3"):
        alone = []
        with serve.Server(slots=1, hbm_budget=50e9, precision=precision) as srv:
            for s, (d, o) in zip(specs, probs):
                r = srv.wait(srv.submit(d, o, s.nroots, 1e-6, 1e-9), timeout=600)
                assert r.status == 0, r.error
                alone.append(r.energies)
        with serve.Server(slots=4, hbm_budget=50e9, precision=precision) as srv:
            ids = [srv.submit(d, o, s.nroots, 1e-6, 1e-9) for s, (d, o) in zip(specs, probs)]
            mixed = [srv.wait(i, timeout=600) for i in ids]
            st = srv.stats()
        assert st["peak_running"] >= 2
        for a, m in zip(alone, mixed):
            assert m.status == 0, m.error
            assert np.abs(a - m.energies).max() <= 1e-10
        by_form[precision] = alone
    # the mixed-precision served form lands within 1 uEh of the FP64 form
    for a64, a32 in zip(by_form["fp64"], by_form["tf32x3"]):
        assert np.abs(a64 - a32).max() <= 1e-6
