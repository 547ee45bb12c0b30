"""Benchmark of the Davidson sigma = H c path on the kernel-scale synthetic
MRSDCI problem: 16 internal orbitals (8 doubly occupied + 8 active), 240
virtuals, Cholesky rank 1600, 16 electrons, singlet, one closed-shell
reference (1,971,105 CSFs).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

One step = one Davidson solve (1 root, RESIDUAL TOLERANCE 1e-6, ENERGY
TOLERANCE 1e-8) of that problem, with the operator scaled to molecular
magnitude (L x 0.02, h diagonal in [-2, 1], off-diagonal N(0, 0.02)) so that
1 uEh is a meaningful agreement bound.

value    : Davidson solves/s of the fastest form whose root lies within
           1 uEh of the plain-FP64 GPU form (the mixed tf32x3 form when it
           does), contexts resident in HBM.
e2e      : the same solve through the public C ABI from host buffers:
           tci_sigma_init (deck + operator uploaded from pinned host memory),
           tci_davidson, eigenvector read back, tci_destroy.
sigma    : 100-build style sigma throughput on the operator exactly as the
           kernel-scale configuration specifies (L ~ N(0,1)...), FP64 and
           tf32x3, with the per-step profile and the all-external roofline.
latency  : p50 / p99 time-to-solution of the timed solves.
cpu_baseline / --impl reference: whole sigma builds of the same problem on the
           host cores by the oracle's integral-direct CPU sigma
           (oracle/plancpu.c: integrals formed from the Cholesky vectors at
           every build as the reference does, the all-external term in the
           reference's loop form, every other coupling replayed from the loop
           records, OpenMP + OpenBLAS dgemm).  A step of the reference arm is
           one such sigma build (a bounded sample of a solve); solves/s is the
           measured sigma rate over the sigma builds a solve takes (the FP64
           solve's iteration count, measured on the GPU).  The reference
           (Fortran + IO_buffer submodule) cannot be compiled here, so this
           port is its CPU arm.
N > 1 runs independent replicas (no collective).
"""
from __future__ import annotations

import argparse
import json
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

N_INT_INACTIVE, N_INT_ACTIVE, N_VIRT, N_CHOL, N_ELEC = 8, 8, 240, 1600, 16
if "--virt" in sys.argv:  # smaller case for profiler captures
    N_VIRT = int(sys.argv[sys.argv.index("--virt") + 1])
WORKLOAD = f"kernel-scale synthetic MRSDCI sigma build: 16 internal (8 inactive + 8 active), {N_VIRT} virtuals, Cholesky rank 1600, 16 electrons, singlet, 1 reference"
METRIC = "Davidson solves/s at 1 \u00b5Eh vs plain FP64 GPU form; \u03c3-build TFLOP/s; p50/p99 lat"
SOLVE_WORKLOAD = WORKLOAD.replace("sigma build", "Davidson solve (1 root)") + "; operator scaled to molecular magnitude"
TOL_RESIDUAL, TOL_ENERGY = 1e-6, 1e-8
# sigma builds one FP64 solve of the molecular-magnitude problem takes: the iterations of the FP64 GPU solve
# of this operator (one sigma build per iteration at one root), measured on a B200 (27) and re-measured by
# every run of this benchmark's own arm (solves.fp64.iterations); the reference arm has no GPU to count them
SIGMA_BUILDS_PER_SOLVE = 27
# ncu DRAM bytes (read + write) of one launch over its algorithmic bytes (the W operators): FP64 split-K
# all-external at 120 virtuals 845.1 MB / 829.5 MB; tcgen05 all-external at 140 virtuals 809.9 MB / 773.4 MB
TRAFFIC_RATIO = {"fp64": 845.142 / 829.498, "tf32x3": (800.509 + 9.346) / 773.381}
TRAFFIC_SOURCE = {"fp64": "ncu dram read+write ratio at 120 virtuals x full-size bytes",
                  "tf32x3": "ncu dram read+write ratio at 140 virtuals x full-size bytes"}


def deck_and_operator(molecular=False):
    import tigerci_b200 as T
    from tigerci_b200.synthetic import synthetic_operator

    nint = N_INT_INACTIVE + N_INT_ACTIVE
    deck = T.Deck(nint + N_VIRT, N_INT_INACTIVE, N_INT_ACTIVE, N_ELEC, 1, ["2" * N_INT_INACTIVE + "0" * N_INT_ACTIVE])
    if molecular:
        h, L = synthetic_operator(nint + N_VIRT, N_CHOL, seed=1234, scale=0.02, diag_range=(-2.0, 1.0),
                                  offdiag_sigma=0.02)
    else:
        h, L = synthetic_operator(nint + N_VIRT, N_CHOL, seed=1234)
    return deck, T.Operator(h, L)


def reduce_max(t, dist=None, device=None):
    """The largest of t over the ranks of the process group (t itself without one): every timed quantity
    of a multi-GPU run is the slowest rank's."""
    if not dist:
        return t
    import torch

    tt = torch.tensor([t], dtype=torch.float64, device=device or "cpu")
    dist.all_reduce(tt, op=dist.ReduceOp.MAX)
    return float(tt.item())


def replica_rate(world, units_per_rank, t_max):
    """Whole-job rate of N independent replicas: the units all ranks processed over the slowest rank's time."""
    return world * units_per_rank / t_max


def _np_default(o):
    if isinstance(o, np.generic):
        return o.item()
    if isinstance(o, np.ndarray):
        return o.tolist()
    raise TypeError(f"{type(o).__name__} is not JSON serializable")


def dumps(obj) -> str:
    """json.dumps that takes numpy scalars and arrays."""
    return json.dumps(obj, default=_np_default)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


def fp64_gemm_peak(device):
    """cuBLAS FP64 GEMM throughput on this GPU (torch.matmul, 8192^3 float64, best of 5 after 2 warm-ups,
    CUDA events): the compute roof of the FP64 form, which the measured peaks file does not carry."""
    import torch

    n = 8192
    g = torch.Generator(device=device).manual_seed(0)
    a = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    b = torch.randn(n, n, dtype=torch.float64, device=device, generator=g)
    for _ in range(2):
        torch.matmul(a, b)
    best = float("inf")
    for _ in range(5):
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record()
        torch.matmul(a, b)
        e1.record()
        torch.cuda.synchronize()
        best = min(best, e0.elapsed_time(e1) / 1e3)
    del a, b
    torch.cuda.empty_cache()
    return 2.0 * n ** 3 / best / 1e12


class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index, period_ms=100):
        self.index = index
        self.period_ms = period_ms
        self.rows = []
        self._p = None
        self._t = None

    def _read(self):
        # one nvidia-smi process sampling every period_ms for the whole region (a new process per sample
        # took ~0.3 s, too few samples for a region of a second)
        try:
            for line in self._p.stdout:
                line = line.strip()
                if line:
                    self.rows.append([x.strip() for x in line.split(",")])
        except Exception:
            pass

    def __enter__(self):
        try:
            self._p = subprocess.Popen(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                        "--format=csv,noheader,nounits", "-lms", str(self.period_ms)],
                                       stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
        except Exception:
            self._p = None
            return self
        self._t = threading.Thread(target=self._read, daemon=True)
        self._t.start()
        time.sleep(0.3)  # the first sample is taken before the timed work starts
        return self

    def __exit__(self, *a):
        if self._p is None:
            return
        self._p.terminate()
        try:
            self._p.wait(timeout=5)
        except Exception:
            self._p.kill()
            self._p.wait(timeout=5)
        self._t.join(timeout=5)
        if not self.rows:  # nothing came through the pipe: one sample now rather than none
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_sigma_arm(molecular=True, steps=1, warmup=0, c_host=None):
    """Times whole sigma builds of the benchmark problem with the oracle's
    integral-direct CPU sigma (oracle/plancpu.c) on all host cores: the plan's
    loop records exported once, then warmup + steps builds, each forming its
    integrals from the Cholesky vectors and running every term.  Returns the
    per-build times, the last sigma and the thread count."""
    import tempfile

    import tigerci_b200 as T
    from oracle import dense

    deck, op = deck_and_operator(molecular=molecular)
    blas = dense.use_blas()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "plan.bin")
        T.Plan(deck, op).export(path)
        pc = dense.PlanSigmaCPU(path, op.chol)
    if c_host is None:
        c_host = np.random.default_rng(3).standard_normal(pc.n)
        c_host /= np.linalg.norm(c_host)
    times, sigma = [], None
    for i in range(warmup + steps):
        t = time.perf_counter()
        sigma = pc.sigma(c_host, integrals=True)
        dt = time.perf_counter() - t
        if i >= warmup:
            times.append(dt)
    pc.close()
    return dict(times=times, sigma=sigma, cores=int(dense.lib().oracle_num_threads()), blas=blas, n=pc.n)


CPU_SAMPLE = ("one whole sigma build per step (integrals formed from the Cholesky vectors, all-external term in "
              "the reference's loop form, every other coupling from the loop records; OpenMP + OpenBLAS dgemm); "
              "solves/s = 1 / (sigma time x sigma builds per FP64 solve)")


def solve_config(n_csf):
    return {"workload": SOLVE_WORKLOAD, "total_csfs": n_csf, "roots": 1, "tol_residual": TOL_RESIDUAL,
            "tol_energy": TOL_ENERGY, "parallelism": "single",
            "l2": "a solve streams the W operators (13.3 GB FP64 / 6.7 GB FP32) > L2 every sigma; "
                  "256 MB write between timed solves"}


def run_reference(args, rank, world):
    if rank != 0:
        return
    r = cpu_sigma_arm(molecular=True, steps=args.steps, warmup=args.warmup)
    t_sigma = float(np.mean(r["times"]))
    v = 1.0 / (t_sigma * SIGMA_BUILDS_PER_SOLVE)
    sample = CPU_SAMPLE + f"; {SIGMA_BUILDS_PER_SOLVE} sigma builds per FP64 solve"
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "solves/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t_sigma,
            "step": "one whole CPU sigma build (a bounded sample of a solve)",
            "sigma_builds_per_solve": SIGMA_BUILDS_PER_SOLVE,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded operators of the benchmark shape)",
            "config": dict(solve_config(r["n"]), parallelism="replicas" if world > 1 else "single"),
            "latency_ms": {"p50": 1e3 * float(np.percentile(r["times"], 50)),
                           "p99": 1e3 * float(np.percentile(r["times"], 99)), "what": "per CPU sigma build"},
            "cpu_baseline": {"value": v, "unit": "solves/s", "cores": r["cores"], "kind": "port", "sample": sample},
            "e2e": {"value": v, "unit": "solves/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(dumps(line), flush=True)


def serve_measure(n_requests, slots, device, serial_per_n=2, planners=4):
    """The serving configuration: the seeded stream of H_n chain solves (Poisson, 4 requests/s), every
    request's deck and MO operator built through the molecular front end first (RHF/cc-pVDZ, Cholesky
    vectors; CAS(2,2) references).  Two passes through the request server in the mixed form: the stream
    replayed in real time (arrival-bound), and all requests submitted at once (capacity).  Against them the
    plain FP64 form solving requests one after another: serial_per_n requests of every chain length timed
    (context set-up included), the stream's serial time estimated from the mean time of each length."""
    import torch

    import tigerci_b200 as T
    from tigerci_b200 import serve

    specs = serve.hn_chain_stream(n_requests, rate=4.0, seed=7)
    t0 = time.perf_counter()
    problems = [serve.chain_problem(s) for s in specs]
    t_front = time.perf_counter() - t0

    def one_pass(arrivals):
        with serve.Server(device=device, slots=slots, hbm_budget=150e9, precision="tf32x3", planners=planners) as srv:
            t0 = time.perf_counter()
            ids = []
            for s, (d, o), a in zip(specs, problems, arrivals):
                delay = a - (time.perf_counter() - t0)
                if delay > 0:
                    time.sleep(delay)
                ids.append(srv.submit(d, o, s.nroots, TOL_RESIDUAL, TOL_ENERGY))
            res = [srv.wait(i) for i in ids]
            st = srv.stats()
        bad = [r.error for r in res if r.status != 0]
        return res, {"solves_per_s": st["solves_per_s"], "p50_s": st["p50_s"], "p99_s": st["p99_s"],
                     "peak_running": st["peak_running"], "peak_reserved_gb": st["peak_reserved_bytes"] / 1e9,
                     "median_phase_s": {"plan": float(np.median([r.t_planned - r.t_submit for r in res])),
                                        "wait_admission": float(np.median([r.t_admitted - r.t_planned for r in res])),
                                        "run": float(np.median([r.t_done - r.t_admitted for r in res]))},
                     "failed": bad[:3]}

    res_rt, rt = one_pass([s.arrival for s in specs])
    res_sat, sat = one_pass([0.0] * len(specs))
    torch.cuda.synchronize()
    by_n = {}
    for i, s in enumerate(specs):
        by_n.setdefault(s.n_atoms, []).append(i)
    sample = [i for n in sorted(by_n) for i in by_n[n][:serial_per_n]]
    t_of = {}
    dmax, matched, flipped = 0.0, 0, 0
    for i in sample:
        (d, o), s = problems[i], specs[i]
        t = time.perf_counter()
        sb = T.SigmaBuilder(d, o, device=device, precision="fp64")
        # the server's subspace budget (12 vectors per root, restarting), so both forms take the same path
        e, _, _ = sb.davidson(s.nroots, TOL_RESIDUAL, TOL_ENERGY, subspace_bytes=16 * sb.n * 12 * s.nroots)
        sb.close()
        t_of.setdefault(s.n_atoms, []).append(time.perf_counter() - t)
        for r in (res_rt[i], res_sat[i]):
            if r.status != 0:
                continue
            for a, b in zip(r.energies, e):
                # a root more than 1e-4 Eh away is another state of the space (the diagonal initial guess
                # can leave a symmetry sector unexplored, and rounding decides whether it is found), not a
                # precision error of the same state
                if abs(a - b) < 1e-4:
                    matched += 1
                    dmax = max(dmax, abs(a - b))
                else:
                    flipped += 1
    t_serial = sum(float(np.mean(t_of[s.n_atoms])) for s in specs)
    fp64_rate = n_requests / t_serial
    return {"requests": n_requests, "arrivals": "Poisson 4/s, seed 7", "slots": slots, "planners": planners,
            "hbm_budget_gb": 150, "form": "tf32x3",
            "problems": "H_n chains through the molecular front end: cc-pVDZ, RHF orbitals, Cholesky vectors "
                        "(1e-6), CAS(2,2) references (HOMO/LUMO) in place of CAS(n/2,n/2)",
            "front_end_s_total": t_front,
            "realtime": rt, "saturated": sat,
            "solves_per_s": sat["solves_per_s"], "p50_s": rt["p50_s"], "p99_s": rt["p99_s"],
            "fp64_serial_solves_per_s": fp64_rate,
            "fp64_serial_sample": f"{serial_per_n} requests per chain length ({len(sample)} of {n_requests}) solved "
                                  "one after another, stream time estimated from each length's mean",
            "vs_fp64_serial": sat["solves_per_s"] / fp64_rate,
            "max_abs_root_diff_vs_fp64": dmax, "all_within_1uEh": dmax <= 1e-6,
            "roots_compared": matched, "roots_on_another_state": flipped,
            "total_csfs_range": [min(r.total_csfs for r in res_sat), max(r.total_csfs for r in res_sat)]}


def molecular_measure(device, steps=3, warmup=1):
    """Water through the molecular front end (the CPU-runnable configuration): RHF/cc-pVDZ orbitals, O 1s
    frozen, CAS(4,4) references, Cholesky threshold 1e-6; Davidson solves on the device in both forms
    (CUDA-event time to solution), and end to end: front end + plan + device set-up + solve."""
    import torch

    import tigerci_b200 as T
    from tigerci_b200 import molecule as M

    t0 = time.perf_counter()
    deck, op, info = M.water_c1()
    t_front = time.perf_counter() - t0
    out = {"workload": "H2O (R(O-H) 0.9572 A, HOH 104.52 deg), cc-pVDZ (24 functions), O 1s frozen, CAS(4,4) "
                       "(19 references) on canonical RHF orbitals, CD threshold 1e-6, singlet, 1 root, "
                       "residual 1e-6 (energy tolerance 1e-10)",
           "nchol": info["nchol"], "e_scf": info["e_scf"], "front_end_s": t_front, "front_end_phases_s": info["seconds"]}
    for form in ("fp64", "tf32x3"):
        t = time.perf_counter()
        sb = T.SigmaBuilder(deck, op, device=device, precision=form)
        init_s = time.perf_counter() - t
        for _ in range(warmup):
            sb.davidson(1, 1e-6, 1e-10)
        times, e, it = [], None, 0
        for _ in range(steps):
            torch.cuda.synchronize()
            a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
            a.record()
            e, _, it = sb.davidson(1, 1e-6, 1e-10)
            b.record()
            torch.cuda.synchronize()
            times.append(a.elapsed_time(b) / 1e3)
        out["total_csfs"] = sb.n
        sb.close()
        out[form] = {"energy": float(e[0]) + op.core_energy, "iterations": int(it),
                     "ms_per_solve": 1e3 * float(np.mean(times)), "solves_per_s": 1.0 / float(np.mean(times)),
                     "init_s": init_s}
    out["mixed_minus_fp64"] = out["tf32x3"]["energy"] - out["fp64"]["energy"]
    torch.cuda.synchronize()
    t = time.perf_counter()
    d2, o2, _ = M.water_c1()
    sb = T.SigmaBuilder(d2, o2, device=device, precision="fp64")
    e, v, _ = sb.davidson(1, 1e-6, 1e-10, want_vectors=True)
    sb.close()
    out["e2e_s"] = time.perf_counter() - t
    out["e2e_what"] = "front end (integrals, Cholesky, RHF, AO->MO) + plan + device set-up + FP64 solve + vector read-back"
    out["_deck_op"] = (deck, op)
    return out


def local_solve_measure(device, nchol=2400, n_int=35, n_virt=400, dmax=180):
    """The batching configuration as a Davidson solve: 35 doubly occupied internal orbitals (630 internal
    pairs), 400 externals, every pair and single-hole path with a random domain of 20..180 externals (seed
    99), Cholesky rank 2400, operator at molecular magnitude; 1 root, residual 1e-6.  The all-external term
    runs on the pair-domain operator (the faster of its Cholesky and dense forms), the two-external N-2 step
    on the domains, every other term on the non-local plan with the blocks padded to all externals; FP64 and
    mixed forms.  n_int / n_virt / dmax shrink it (profiler captures)."""
    import torch

    import tigerci_b200 as T
    from tigerci_b200 import local
    from tigerci_b200.synthetic import synthetic_operator

    deck = local.pair_domain_deck(n_int=n_int, n_virt=n_virt, dmax=dmax)
    h, L = synthetic_operator(deck.num_orbitals, nchol, seed=1234, scale=0.02, diag_range=(-2.0, 1.0),
                              offdiag_sigma=0.02)
    op = T.Operator(h, L)
    out = {"workload": f"local MRSDCI: {n_int} doubly occupied internal orbitals ({n_int * (n_int + 1) // 2} pair "
                       f"paths), {n_virt} externals, domains U{{20..{dmax}}} per pair and single-hole path (seed 99), "
                       f"Cholesky rank {nchol}, molecular magnitude; 1 root, residual 1e-6, energy tolerance 1e-8"}
    for form in ("tf32x3", "fp64"):
        t = time.perf_counter()
        sb = T.SigmaBuilder(deck, op, device=device, precision=form)
        init_s = time.perf_counter() - t
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        e, _, it = sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY)
        b.record()
        torch.cuda.synchronize()
        st = sb.stats()
        out["total_csfs"] = sb.n
        sb.profile(False, davidson_phases=True)
        sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY)
        phases = {k: round(v, 1) for k, v in sb.davidson_phase_times().items()}
        # one sigma build with the plan's steps timed (the padded non-local plan; the pair-domain
        # all-external term runs after it and is timed by the local leg)
        sb.profile(True)
        x = np.random.default_rng(3).standard_normal(sb.n)
        t1 = time.perf_counter()
        sb.sigma(x)
        sigma_ms = 1e3 * (time.perf_counter() - t1)
        steps, nb = sb.step_times()
        sb.profile(False)
        sb.close()
        top = sorted(steps, key=lambda kv: -kv[1])[:10]
        out[form] = {"energy": float(e[0]), "iterations": int(it), "ms_per_solve": a.elapsed_time(b),
                     "solves_per_s": 1e3 / a.elapsed_time(b), "init_s": init_s, "phase_ms": phases,
                     "device_gb": st["device_bytes"] / 1e9, "sigma_host_ms": round(sigma_ms, 1),
                     "plan_step_ms": {k: round(v / max(nb, 1), 2) for k, v in top}}
    out["mixed_minus_fp64"] = out["tf32x3"]["energy"] - out["fp64"]["energy"]
    out["within_1uEh"] = abs(out["mixed_minus_fp64"]) <= 1e-6
    out["vs_fp64_form"] = out["fp64"]["ms_per_solve"] / out["tf32x3"]["ms_per_solve"]
    return out


def octane_measure(device, nroots=3):
    """The precision configuration: all-trans n-octane / cc-pVDZ (202 functions), 8 C 1s frozen, CAS(8,8)
    active space on RHF orbitals with the references of tigerci_b200.molecule.OCTANE_REFS, 3 roots; the mixed
    form (3xTF32 contractions, FP64 Davidson, FP64 finish) against the plain FP64 GPU form."""
    import torch

    import tigerci_b200 as T
    from tigerci_b200 import molecule as M

    t0 = time.perf_counter()
    deck, op, info = M.octane_c3()
    out = {"workload": "n-octane (all-trans, staggered), cc-pVDZ (202 functions), 8 C 1s frozen, CAS(8,8) active "
                       f"space, references {list(M.OCTANE_REFS)} over it, singlet, {nroots} roots, CD 1e-6, residual "
                       "1e-6 (energy tolerance 1e-10)",
           "front_end_s": time.perf_counter() - t0, "nchol": info["nchol"], "e_scf": info["e_scf"]}
    for form in ("fp64", "tf32x3"):
        t = time.perf_counter()
        sb = T.SigmaBuilder(deck, op, device=device, precision=form)
        init_s = time.perf_counter() - t
        torch.cuda.synchronize()
        a, b = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        a.record()
        e, _, it = sb.davidson(nroots, 1e-6, 1e-10)
        b.record()
        torch.cuda.synchronize()
        out["total_csfs"] = sb.n
        st = sb.stats()
        sb.close()
        out[form] = {"energies": [float(x) + op.core_energy for x in e], "iterations": int(it),
                     "ms_per_solve": a.elapsed_time(b), "init_s": init_s, "sigma_flops": st["flops_per_sigma"]}
    out["mixed_minus_fp64"] = [x - y for x, y in zip(out["tf32x3"]["energies"], out["fp64"]["energies"])]
    out["max_abs_diff_uEh"] = 1e6 * max(abs(x) for x in out["mixed_minus_fp64"])
    out["vs_fp64_form"] = out["fp64"]["ms_per_solve"] / out["tf32x3"]["ms_per_solve"]
    return out


def molecular_cpu(mol):
    """The oracle on the same water problem: its Davidson over the integral-direct CPU sigma (integrals formed
    at every build), timed, and the device FP64 root's distance from it."""
    import tempfile

    import tigerci_b200 as T
    from oracle import davidson, dense

    deck, op = mol.pop("_deck_op")
    dense.use_blas()
    with tempfile.TemporaryDirectory() as tmp:
        path = os.path.join(tmp, "plan.bin")
        T.Plan(deck, op).export(path)
        pc = dense.PlanSigmaCPU(path, op.chol)
    t = time.perf_counter()
    d = pc.diag()
    e, _, it = davidson.davidson_liu(lambda x: pc.sigma(x, integrals=True), d, 1, 1e-6, 1e-10)
    dt = time.perf_counter() - t
    pc.close()
    e_or = float(e[0]) + op.core_energy
    return {"energy": e_or, "iterations": int(it), "seconds_per_solve": dt, "cores": int(dense.lib().oracle_num_threads()),
            "fp64_minus_oracle": mol["fp64"]["energy"] - e_or, "mixed_minus_oracle": mol["tf32x3"]["energy"] - e_or,
            "gpu_fp64_speedup": dt / (mol["fp64"]["ms_per_solve"] / 1e3),
            "what": "oracle Davidson (davidson.f90 restated) over the integral-direct CPU sigma"}


def local_measure(n_pairs, device, hbm, bf16, steps=3, warmup=3, nchol=2400, forms=("tf32x3", "fp64"), n_virt=400):
    """All-external term over uneven pair domains: n_pairs internal pairs (35
    doubly occupied internal orbitals), domains of 20..180 of 400 external
    orbitals (seed 99), Cholesky rank 2400 as in the kernel-scale operator.
    Times tci_local_apply (one CUDA graph per application) in both forms."""
    import torch

    from tigerci_b200 import local
    from tigerci_b200.synthetic import synthetic_operator

    n_int = 35
    heads, dom, total = local.pair_domain_problem(n_pairs, n_int, n_virt, 20, min(180, n_virt), seed=99)
    _, L = synthetic_operator(n_int + n_virt, nchol, seed=1234)
    rng = np.random.default_rng(7)
    c_host = rng.standard_normal(total)
    c = torch.from_numpy(c_host).cuda(device)
    out = {"workload": f"{len(heads)} internal pairs, domains U{{20..{min(180, n_virt)}}} of {n_virt} externals (seed 99), "
                       f"Cholesky rank {nchol}; CI length {total}",
           "heads": int(len(heads))}
    sig = {}
    for form, n_steps in [(f, steps if f == "tf32x3" else 1) for f in forms]:
        t0 = time.perf_counter()
        op = local.LocalAllExternal(n_int, n_virt, L, heads, dom, total, device=device, precision=form)
        init_s = time.perf_counter() - t0
        st = op.stats()
        s = torch.zeros_like(c)
        for _ in range(warmup if form == "tf32x3" else 1):
            op.apply_device(c.data_ptr(), s.data_ptr())
        torch.cuda.synchronize()
        ev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
        for i in range(n_steps):
            s.zero_()
            ev[i][0].record()
            op.apply_device(c.data_ptr(), s.data_ptr())
            ev[i][1].record()
        torch.cuda.synchronize()
        t = sum(a.elapsed_time(b) for a, b in ev) / 1e3 / n_steps
        sig[form] = s.cpu().numpy()
        # 3xTF32 issues three MMAs per product: its FP32-accurate peak is a third of the TF32 peak
        # (half the measured dense BF16 figure)
        peak = bf16 / 2 / 3 if form == "tf32x3" else None
        # the form applied: the Cholesky form's flops are the useful work; the dense form does its own
        # (padded) flops on the all-external kernel, and those set its tensor roofline
        fl = st["dense_flops"] if st["form"] == "dense" else st["flops"]
        kern = ("allext_tf32x3_kernel (dense padded W+/W- over all external pairs, tcgen05 kind::tf32, 3xTF32)"
                if st["form"] == "dense" else
                "tma_gemm (grouped 3xTF32, pair-domain Cholesky form)" if form == "tf32x3" else
                "gemm_f64 grouped (pair-domain Cholesky form, FP64)")
        out[form] = {"ms_per_apply": 1e3 * t, "form": st["form"], "useful_tflops": st["flops"] / t / 1e12,
                     "flops_per_apply": fl, "cholesky_form_flops": st["flops"],
                     "cholesky_form_setup_ms": st["tuned_ms"], "dense_form_setup_ms": st["dense_ms"] or None,
                     "chunk": int(st["chunk"]), "tile_cfg": int(st["tile_cfg"]),
                     "autotune_candidates": int(st["candidates"]), "device_gb": st["device_bytes"] / 1e9,
                     "init_s": init_s,
                     "roofline": {"kernel": kern, "bound": "tensor", "achieved": fl / t / 1e12, "peak": peak,
                                  "unit": "TFLOP/s", "frac": (fl / t / 1e12 / peak) if peak else None,
                                  "peak_kind": "3xTF32: measured dense BF16 / 2 / 3" if peak else None}}
        if st["form"] == "dense":
            # the W tiles are streamed once per group of 64 CI blocks of each operator
            out[form]["w_gb"] = st["dense_w_bytes"] / 1e9
        op.close()
    if "tf32x3" in sig and "fp64" in sig:
        a, b = sig["tf32x3"], sig["fp64"]
        out["mixed_rel_err_vs_fp64"] = float(np.linalg.norm(a - b) / np.linalg.norm(b))
    return out


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5, help="timed Davidson solves per form")
    ap.add_argument("--warmup", type=int, default=3, help="untimed Davidson solves per form")
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--virt", type=int, default=N_VIRT, help="virtual orbitals (default: the benchmark's 240)")
    ap.add_argument("--forms", default="fp64,tf32x3", help="precision forms to measure")
    ap.add_argument("--sigma-builds", type=int, default=20, help="timed sigma builds per form")
    ap.add_argument("--e2e-steps", type=int, default=2, help="end-to-end solves through the C ABI")
    ap.add_argument("--sigma-only", action="store_true", help="sigma builds only (profiler launch lists)")
    ap.add_argument("--serve-requests", type=int, default=256, help="requests of the serving stream to replay")
    ap.add_argument("--serve-slots", type=int, default=6)
    ap.add_argument("--serve-planners", type=int, default=4, help="host threads building plans for the server")
    ap.add_argument("--local-nchol", type=int, default=2400, help="Cholesky rank of the pair-domain workload")
    ap.add_argument("--local-forms", default="tf32x3,fp64", help="forms of the pair-domain measurement")
    ap.add_argument("--serve-only", action="store_true", help="only the serving measurement")
    ap.add_argument("--local-pairs", type=int, default=600, help="pairs of the pair-domain workload (0: skip)")
    ap.add_argument("--acpf-solves", type=int, default=3, help="timed ACPF solves on the solve operator (0: skip)")
    ap.add_argument("--local-only", action="store_true", help="only the pair-domain measurement")
    ap.add_argument("--no-molecular", action="store_true", help="skip the water (front end) measurement")
    ap.add_argument("--octane-only", action="store_true", help="only the n-octane precision measurement")
    ap.add_argument("--local-solve-only", action="store_true", help="only the pair-domain Davidson solve")
    ap.add_argument("--local-virt", type=int, default=400, help="externals of the pair-domain workloads")
    ap.add_argument("--local-int", type=int, default=35, help="internal orbitals of the pair-domain solve")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return
    if args.warmup < 3 and not args.sigma_only:
        ap.error("at least 3 warm-up steps")

    import torch

    import tigerci_b200 as T

    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist

        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=600))
    torch.cuda.set_device(local)
    dev = f"cuda:{local}"
    forms = [f for f in args.forms.split(",") if f]
    hbm, bf16, peak_kind = measured_peaks()
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def max_over_ranks(t):
        return reduce_max(t, dist, dev)

    if args.serve_only:
        if rank == 0:
            print(dumps({"serving": serve_measure(args.serve_requests, args.serve_slots, local, planners=args.serve_planners)}), flush=True)
        return
    if args.local_solve_only:
        if rank == 0:
            print(dumps({"local_solve": local_solve_measure(local, n_int=args.local_int, n_virt=args.local_virt,
                                                            dmax=min(180, args.local_virt))}), flush=True)
        return
    if args.octane_only:
        if rank == 0:
            print(dumps({"octane_c3": octane_measure(local)}), flush=True)
        return
    if args.local_only:
        if rank == 0:
            print(dumps({"local_pairs": local_measure(args.local_pairs, local, hbm, bf16, nchol=args.local_nchol,
                                                    forms=tuple(f for f in args.local_forms.split(",") if f),
                                                    n_virt=args.local_virt)}), flush=True)
        return

    # ---- sigma builds on the operator exactly as the kernel-scale configuration specifies
    deck, op = deck_and_operator()

    def sigma_measure(precision, n_steps):
        """Warm-up, timed sigma builds (graph replay), then a profiled pass with
        event nodes around every plan step (roofline of the all-external kernel)."""
        t0 = time.perf_counter()
        sb = T.SigmaBuilder(deck, op, device=local, precision=precision)
        init_s = time.perf_counter() - t0
        n = sb.n
        rng = np.random.default_rng(7 + rank)
        c_host = rng.standard_normal(n)
        c_host /= np.linalg.norm(c_host)
        c = torch.from_numpy(c_host).to(dev)
        s = torch.zeros_like(c)
        with torch.cuda.stream(stream):
            for _ in range(3):
                sb.htimesc_device(c.data_ptr(), s.data_ptr(), n, stream.cuda_stream)
        torch.cuda.synchronize()

        def timed(profile):
            sb.profile(profile)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
            launches0 = sb.stats()["launches"]
            with ClockSampler(local) as clk, torch.cuda.stream(stream):
                torch.cuda.synchronize()
                for i in range(n_steps):
                    flush.fill_(float(i))  # write 256 MB > L2 between timed builds
                    s.zero_()
                    evs[i][0].record(stream)
                    sb.htimesc_device(c.data_ptr(), s.data_ptr(), n, stream.cuda_stream)
                    evs[i][1].record(stream)
                torch.cuda.synchronize()
            launches = sb.stats()["launches"] - launches0
            prof = sb.step_times() if profile else None
            sb.profile(False)
            return sum(a.elapsed_time(b) for a, b in evs) / 1e3, clk, prof, launches

        if dist:
            dist.barrier()
        t_total, clk, _, launches = timed(False)
        t_total = max_over_ranks(t_total)
        t_prof, _, (steps_prof, nb), _ = timed(True)
        sb.check()
        sigma = s.cpu().numpy().copy()
        st = sb.stats()
        prof = {name: ms / max(nb, 1) for name, ms in steps_prof}
        out = dict(n=n, c_host=c_host, t_total=t_total, clk=clk, prof=prof, t_prof=t_prof, stats=st,
                   init_s=init_s, sigma=sigma, launches=launches, sb=sb)
        return out

    sig = {}
    for f in forms:
        try:
            sig[f] = sigma_measure(f, args.sigma_builds)
        except Exception as exc:  # one form failing leaves the other's line
            sig[f] = {"error": str(exc)[:300]}
    if "fp64" in sig and "error" not in sig["fp64"]:
        for f in sig:
            if f != "fp64" and "error" not in sig[f]:
                a, b = sig[f]["sigma"], sig["fp64"]["sigma"]
                sig[f]["sigma_rel_err_vs_fp64"] = float(np.abs(a - b).max() / np.abs(b).max())
    for f in sig:
        if "sb" in sig[f]:
            sig[f].pop("sb").close()

    try:
        fp64_peak = fp64_gemm_peak(dev) if "fp64" in forms else None
    except Exception:  # the FP64 roof is a side figure
        fp64_peak = None

    def sigma_summary(f, m):
        if "error" in m:
            return m
        st = m["stats"]
        if f == "fp64":
            t_dom = (m["prof"]["all-external"] + m["prof"].get("all-external split-k sum", 0.0)) / 1e3
            kernel, bytes_ = "gemm_panel_f64 split-k (all-external W+/W- product, FP64 FMA)", st["bytes_allext"]
        else:
            t_dom = m["prof"]["all-external"] / 1e3
            kernel = "allext_tf32x3_kernel (tcgen05 kind::tf32, TMA, 3xTF32, FP64 promotion)"
            bytes_ = st["bytes_allext"] / 2.0  # FP32 W: half of the FP64 bytes (padding aside)
        d = {"sigma_builds_per_s": world * args.sigma_builds / m["t_total"],
             "ms_per_build": 1e3 * m["t_total"] / args.sigma_builds,
             "sigma_tflops": st["flops_per_sigma"] * args.sigma_builds * world / m["t_total"] / 1e12,
             "roofline": {"kernel": kernel, "bound": "hbm", "achieved": bytes_ / t_dom / 1e9, "peak": hbm,
                          "unit": "GB/s", "frac": bytes_ / t_dom / 1e9 / hbm,
                          "traffic": TRAFFIC_RATIO[f] * bytes_, "algorithmic_bytes": bytes_,
                          "traffic_source": TRAFFIC_SOURCE[f],
                          "peak_kind": peak_kind, "ms": 1e3 * t_dom},
             "launches_per_build": m["launches"] / args.sigma_builds,
             "step_ms": {k: round(v, 4) for k, v in sorted(m["prof"].items(), key=lambda kv: -kv[1])[:12]},
             "profiled_ms_per_build": 1e3 * m["t_prof"] / args.sigma_builds, "init_s": m["init_s"],
             "clocks": m["clk"].summary()}
        if f == "fp64" and fp64_peak:
            # a few dozen CI rows against W: 2 m flops per 8-byte W element, above the FP64 ridge (peak / HBM
            # bandwidth) for m >= 32, so the FP64 compute rate bounds it
            d["roofline_fp64"] = {"kernel": kernel, "bound": "fp64", "achieved": st["flops_allext"] / t_dom / 1e12,
                                  "peak": fp64_peak, "unit": "TFLOP/s",
                                  "frac": st["flops_allext"] / t_dom / 1e12 / fp64_peak,
                                  "peak_kind": "cuBLAS FP64 GEMM measured in this run (8192^3)",
                                  "flops": st["flops_allext"], "ms": 1e3 * t_dom}
        if "sigma_rel_err_vs_fp64" in m:
            d["sigma_rel_err_vs_fp64"] = m["sigma_rel_err_vs_fp64"]
        return d

    sigma_lines = {f: sigma_summary(f, m) for f, m in sig.items()}
    n_csf = next((m["n"] for m in sig.values() if "n" in m), None)
    if args.sigma_only:
        if rank == 0:
            print(dumps({"sigma_only": True, "config": {"workload": WORKLOAD, "total_csfs": n_csf},
                              "sigma": sigma_lines}), flush=True)
        if dist:
            dist.barrier()
            dist.destroy_process_group()
        return

    # ---- Davidson solves on the molecular-magnitude operator (same shapes)
    deck_m, op_m = deck_and_operator(molecular=True)

    def solve_measure(precision):
        t0 = time.perf_counter()
        sb = T.SigmaBuilder(deck_m, op_m, device=local, precision=precision)
        init_s = time.perf_counter() - t0
        for _ in range(args.warmup):
            sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY)
        times, energies, iters = [], [], []
        launches0 = sb.stats()["launches"]
        if dist:
            dist.barrier()
        with ClockSampler(local) as clk:
            for i in range(args.steps):
                flush.fill_(float(i))
                torch.cuda.synchronize()
                ev0, ev1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
                ev0.record()
                e, _, it = sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY)
                ev1.record()
                torch.cuda.synchronize()
                times.append(ev0.elapsed_time(ev1) / 1e3)
                energies.append(float(e[0]))
                iters.append(int(it))
        launches = sb.stats()["launches"] - launches0
        # one more (untimed) solve with the phases timed (the stream is synchronised at each boundary)
        sb.profile(False, davidson_phases=True)
        sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY)
        phases = {k: round(v, 2) for k, v in sb.davidson_phase_times().items()}
        sb.profile(False)
        sb.check()
        sb.close()
        t_total = max_over_ranks(sum(times))
        return dict(times=times, t_total=t_total, energy=energies[-1], energies=energies, iterations=iters,
                    launches=launches, clk=clk, init_s=init_s, phases=phases)

    def acpf_measure(nsolves, form):
        """MR-ACPF (flag 1) on the water problem of the molecular leg (cc-pVDZ, CAS(4,4) references, RHF
        orbitals): the FP64 form once for its energy, `form` timed (host wall clock around SigmaBuilder.acpf,
        the metric build included).  The synthetic solve operator is no ACPF case: its internal space holds
        CSFs within a few mEh of the reference energy outside the reference space, so the lowest root of
        (H - E_ref) c = lambda G c is an intruder with a small reference weight."""
        from tigerci_b200 import molecule as M

        deck_w, op_w, _ = M.water_c1()
        out = {"flag": 1, "what": "(H - E_ref) c = lambda G c, generalized device Davidson, residual in the c "
                                  "metric, root following",
               "workload": "H2O cc-pVDZ, O 1s frozen, CAS(4,4) references (19), singlet, 1 root"}
        for f in dict.fromkeys(("fp64", form)):
            sb = T.SigmaBuilder(deck_w, op_w, device=local, precision=f)
            e, _, it, e_ref = sb.acpf(1, flag=1, tol_residual=TOL_RESIDUAL, tol_energy=TOL_ENERGY)
            ts = []
            for _ in range(nsolves if f == form else 0):
                torch.cuda.synchronize()
                t = time.perf_counter()
                e, _, it, _ = sb.acpf(1, flag=1, tol_residual=TOL_RESIDUAL, tol_energy=TOL_ENERGY, e_ref=e_ref)
                torch.cuda.synchronize()
                ts.append(time.perf_counter() - t)
            conv = bool(sb.stats()["converged"])
            sb.close()
            out[f] = {"energy": float(e[0]) + op_w.core_energy, "iterations": int(it), "converged": conv,
                      "e_ref": float(e_ref) + op_w.core_energy}
            if ts and conv:
                out[f].update({"solves_per_s": len(ts) / sum(ts), "ms_per_solve": 1e3 * sum(ts) / len(ts)})
            elif ts:  # a solve that ran to maxit has no solve rate: its time per iteration
                out[f]["ms_per_iteration"] = 1e3 * sum(ts) / len(ts) / max(1, int(it))
        if form != "fp64":
            out[form]["energy_minus_fp64"] = out[form]["energy"] - out["fp64"]["energy"]
        return out

    solves = {}
    for f in forms:
        try:
            solves[f] = solve_measure(f)
        except Exception as exc:
            solves[f] = {"error": str(exc)[:300]}
    ok = {f: m for f, m in solves.items() if "error" not in m}
    e64 = ok["fp64"]["energy"] if "fp64" in ok else None
    meets = {f: (e64 is not None and abs(m["energy"] - e64) <= 1e-6) for f, m in ok.items()}
    # the fastest form whose root is within 1 uEh of the FP64 form's
    cand = [f for f in ok if meets[f]]
    best = min(cand, key=lambda f: ok[f]["t_total"]) if cand else (next(iter(ok)) if ok else None)
    if best is None:
        raise RuntimeError(f"no Davidson form ran: {solves}")
    bm = ok[best]
    value = replica_rate(world, args.steps, bm["t_total"])
    lat = np.array(bm["times"]) * 1e3

    # ---- end to end through the public C ABI: init from pinned host operator, solve, vector read-back
    L_pin = torch.from_numpy(op_m.chol).pin_memory()
    h_pin = torch.from_numpy(op_m.h).pin_memory()
    op_pin = T.Operator(h_pin.numpy(), L_pin.numpy())
    e2e_t = []
    for i in range(args.e2e_steps):
        torch.cuda.synchronize()
        t = time.perf_counter()
        sb = T.SigmaBuilder(deck_m, op_pin, device=local, precision=best)
        e, v, _ = sb.davidson(1, TOL_RESIDUAL, TOL_ENERGY, want_vectors=True)
        sb.close()
        e2e_t.append(time.perf_counter() - t)
    e2e = world / max_over_ranks(float(np.mean(e2e_t)))
    h2d = int(op_m.chol.nbytes + op_m.h.nbytes)
    d2h = int(8 * n_csf + 8)

    def solve_summary(f):
        m = solves[f]
        if "error" in m:
            return m
        return {"solves_per_s": world * args.steps / m["t_total"], "ms_per_solve": 1e3 * m["t_total"] / args.steps,
                "iterations": m["iterations"][-1], "energy": m["energy"],
                "energy_minus_fp64": (m["energy"] - e64) if e64 is not None else None,
                "within_1uEh_of_fp64": meets.get(f), "init_s": m["init_s"],
                "launches_per_solve": m["launches"] / args.steps, "phase_ms": m["phases"]}

    line = {"metric": METRIC, "value": value, "unit": "solves/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * bm["t_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64" if best == "fp64" else "f64+tf32x3",
            "data": "synthetic (seeded operators of the benchmark shape)",
            "config": dict(solve_config(n_csf), parallelism="replicas" if world > 1 else "single"),
            "form": best,
            "vs_fp64_form": (ok["fp64"]["t_total"] / bm["t_total"]) if "fp64" in ok else None,
            "latency_ms": {"p50": float(np.percentile(lat, 50)), "p99": float(np.percentile(lat, 99)),
                           "what": "time to solution of the timed solves"},
            "sigma_tflops": sigma_lines.get(best, {}).get("sigma_tflops"),
            "e2e": {"value": e2e, "unit": "solves/s", "h2d_bytes_per_step": h2d, "d2h_bytes_per_step": d2h,
                    "what": "tci_sigma_init from pinned host operator + tci_davidson + eigenvector read-back"},
            "gpu_launches": int(bm["launches"]),
            "roofline": sigma_lines.get(best, {}).get("roofline"),
            "clocks": bm["clk"].summary(),
            "solves": {f: solve_summary(f) for f in solves},
            "sigma": sigma_lines}
    if args.serve_requests > 0:
        try:
            line["serving"] = serve_measure(args.serve_requests, args.serve_slots, local, planners=args.serve_planners)
        except Exception as exc:
            line["serving"] = {"error": str(exc)[:300]}
    if args.acpf_solves > 0:
        try:
            line["acpf"] = acpf_measure(args.acpf_solves, best)
        except Exception as exc:
            line["acpf"] = {"error": str(exc)[:300]}
    mol = None
    if not args.no_molecular:
        try:
            mol = molecular_measure(local)
            line["molecular_c1"] = {k: v for k, v in mol.items() if not k.startswith("_")}
        except Exception as exc:
            line["molecular_c1"] = {"error": str(exc)[:300]}
    if args.local_pairs > 0:
        try:
            line["local_pairs"] = local_measure(args.local_pairs, local, hbm, bf16, nchol=args.local_nchol,
                                                    forms=tuple(f for f in args.local_forms.split(",") if f))
        except Exception as exc:
            line["local_pairs"] = {"error": str(exc)[:300]}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        # one whole CPU sigma build of the kernel-scale operator, on the CI vector of the device FP64 sigma
        # builds above: its time gives the CPU solve rate (x the FP64 solve's measured iteration count), its
        # result the full-size parity of the device FP64 sigma
        n_sig = ok["fp64"]["iterations"][-1] if "fp64" in ok else SIGMA_BUILDS_PER_SOLVE
        have = "fp64" in sig and "sigma" in sig["fp64"]
        cb = cpu_sigma_arm(molecular=False, steps=1, warmup=0, c_host=sig["fp64"]["c_host"] if have else None)
        t_sigma = cb["times"][0]
        line["cpu_baseline"] = {"value": 1.0 / (t_sigma * n_sig), "unit": "solves/s", "cores": cb["cores"],
                                "kind": "port", "sample": CPU_SAMPLE + f"; {n_sig} sigma builds per FP64 solve "
                                f"(this run's FP64 GPU solve); one build, {t_sigma:.1f} s"}
        if have:
            ref = cb["sigma"]
            line["parity"] = {"what": "device FP64 sigma vs the oracle's integral-direct CPU sigma, kernel-scale "
                                      "operator, full size, same CI vector (max abs diff / max abs)",
                              "rel_err": float(np.abs(sig["fp64"]["sigma"] - ref).max() / np.abs(ref).max()),
                              "tolerance": 1e-10}
            if "tf32x3" in sig and "sigma" in sig["tf32x3"]:
                line["parity"]["mixed_rel_err"] = float(np.abs(sig["tf32x3"]["sigma"] - ref).max() / np.abs(ref).max())
        line["sigma_builds_per_solve_fp64"] = {"measured": n_sig, "reference_arm_uses": SIGMA_BUILDS_PER_SOLVE}
        if mol is not None and "fp64" in mol:
            try:
                line["molecular_c1"]["oracle"] = molecular_cpu(mol)
            except Exception as exc:
                line["molecular_c1"]["oracle"] = {"error": str(exc)[:300]}
    if rank == 0:
        print(dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
