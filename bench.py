"""Benchmark: plain-FP64 sigma = H c of the kernel-scale synthetic MRSDCI
operator (16 internal orbitals: 8 doubly occupied + 8 active, 240 virtuals,
Cholesky rank 1600, 16 electrons, singlet, one closed-shell reference;
1,971,105 CSFs).  One step = one sigma build.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

value  : sigma builds/s with c and sigma resident in HBM (tci_sigma_device).
e2e    : the same metric through tci_sigma with host buffers (H2D of c and
         D2H of sigma inside every timed step).
roofline: the dominant plan step, timed with CUDA events on the library's
         stream inside the timed region.
cpu_baseline / --impl reference: the reference's integral-driven all-external
         loop restated in C (oracle, OpenMP + OpenBLAS dgemm like the
         reference), on a bounded sample of external indices, extrapolated
         to a full sigma build.  The reference (Fortran + IO_buffer
         submodule) cannot be compiled here, so this port is its CPU arm.
N > 1 runs independent replicas (one sigma per GPU, no collective).
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
METRIC = "sigma builds/s (plain FP64 sigma = H c)"


def deck_and_operator():
    import tigerci_b200 as T
    from tigerci_b200.synthetic import synthetic_operator

    nint = N_INT_INACTIVE + N_INT_ACTIVE
    deck = T.Deck(nint + N_VIRT, N_INT_INACTIVE, N_INT_ACTIVE, N_ELEC, 1, ["2" * N_INT_INACTIVE + "0" * N_INT_ACTIVE])
    h, L = synthetic_operator(nint + N_VIRT, N_CHOL, seed=1234)
    return deck, T.Operator(h, L)


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return d.get("hbm_gbs", 6650.0), d.get("bf16_tflops", 1590.0), "measured"
    return 6650.0, 1590.0, "fallback"


class ClockSampler:
    FIELDS = "clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap"

    def __init__(self, index):
        self.index = index
        self.rows = []
        self._stop = threading.Event()
        self._t = None

    def _run(self):
        while not self._stop.is_set():
            try:
                out = subprocess.run(["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                                      "--format=csv,noheader,nounits"], capture_output=True, text=True, timeout=5)
                for line in out.stdout.strip().splitlines():
                    self.rows.append([x.strip() for x in line.split(",")])
            except Exception:
                pass
            self._stop.wait(0.2)

    def __enter__(self):
        self._t = threading.Thread(target=self._run, daemon=True)
        self._t.start()
        return self

    def __exit__(self, *a):
        self._stop.set()
        self._t.join(timeout=10)

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        sm = [float(r[0]) for r in self.rows if r[0].replace(".", "").isdigit()]
        mx = [float(r[1]) for r in self.rows if r[1].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in self.rows for i in range(4) if len(r) > 3 + i and r[3 + i] == "Active"})
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": reasons, "samples": len(self.rows)}


def cpu_sample(budget_s=12.0):
    """Time the oracle's reference-form all-external loop on a bounded set of
    external indices a (each a covers the pairs c <= a) and extrapolate."""
    from oracle import dense, sgga
    import tigerci_b200 as T  # noqa: F401  (deck/operator helpers only)

    deck, op = deck_and_operator()
    osp = sgga.build_space(sgga.Deck(deck.num_orbitals, deck.num_inactive, deck.num_active, deck.num_elec, 1,
                                     list(deck.refs)))
    blas = dense.use_blas()
    nint = N_INT_INACTIVE + N_INT_ACTIVE
    rng = np.random.default_rng(3)
    c = rng.standard_normal(osp.total_csfs)
    # grow the sample until it takes ~budget_s
    a1 = N_VIRT
    a0 = N_VIRT - 4
    while True:
        t = time.perf_counter()
        dense.allext_sigma(osp, nint, N_VIRT, op.chol, c, a_range=(a0, a1))
        dt = time.perf_counter() - t
        if dt > budget_s / 4 or a0 == 0:
            break
        a0 = max(0, a1 - int((a1 - a0) * max(2.0, budget_s / max(dt, 1e-3) / 2)))
    pairs = sum(a + 1 for a in range(a0, a1))
    total_pairs = N_VIRT * (N_VIRT + 1) // 2
    t_sigma = dt * total_pairs / pairs
    threads = dense.lib().oracle_num_threads()
    return dict(t_sigma=t_sigma, sample=f"all-external term only (the reference spends ~78% of sigma there), "
                f"external index a in [{a0},{a1}) = {pairs} of {total_pairs} (a,c) pairs, {dt:.1f} s, "
                f"extrapolated by pair count; OpenBLAS dgemm={'yes' if blas else 'no'}", cores=threads)


def run_reference(args, rank, world):
    if rank != 0:
        return
    from oracle import dense

    times = []
    info = None
    for i in range(args.warmup + args.steps):
        info = cpu_sample(budget_s=8.0)
        if i >= args.warmup:
            times.append(info["t_sigma"])
    v = 1.0 / float(np.mean(times))
    line = {"impl": "reference", "metric": METRIC, "value": v, "unit": "builds/s", "n_gpus": args.gpus,
            "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded operator of the benchmark shape)",
            "config": {"workload": WORKLOAD},
            "cpu_baseline": {"value": v, "unit": "builds/s", "cores": info["cores"], "kind": "port",
                             "sample": info["sample"]},
            "e2e": {"value": v, "unit": "builds/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--virt", type=int, default=N_VIRT, help="virtual orbitals (default: the benchmark's 240)")
    args = ap.parse_args()
    rank = int(os.environ.get("RANK", "0"))
    world = int(os.environ.get("WORLD_SIZE", "1"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if args.impl == "reference":
        run_reference(args, rank, world)
        return

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
    deck, op = deck_and_operator()
    hbm, bf16, peak_kind = measured_peaks()
    stream = torch.cuda.Stream(device=dev)
    flush = torch.empty(256 * 1024 * 1024 // 4, dtype=torch.float32, device=dev)

    def measure(precision, n_steps):
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
            for _ in range(args.warmup):
                sb.htimesc_device(c.data_ptr(), s.data_ptr(), n, stream.cuda_stream)
        torch.cuda.synchronize()

        def timed(profile):
            sb.profile(profile)
            evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(n_steps)]
            with ClockSampler(local) as clk, torch.cuda.stream(stream):
                torch.cuda.synchronize()
                for i in range(n_steps):
                    flush.fill_(float(i))  # write 256 MB > L2 between timed builds
                    s.zero_()
                    evs[i][0].record(stream)
                    sb.htimesc_device(c.data_ptr(), s.data_ptr(), n, stream.cuda_stream)
                    evs[i][1].record(stream)
                torch.cuda.synchronize()
            prof = sb.step_times() if profile else None
            sb.profile(False)
            return sum(a.elapsed_time(b) for a, b in evs) / 1e3, clk, prof

        if dist:
            dist.barrier()
        t_total, clk, _ = timed(False)
        if dist:
            tt = torch.tensor([t_total], device=dev)
            dist.all_reduce(tt, op=dist.ReduceOp.MAX)
            t_total = float(tt.item())
        t_prof, _, (steps_prof, nb) = timed(True)
        sb.check()
        sigma = s.cpu().numpy().copy()
        st = sb.stats()
        prof = {name: ms / max(nb, 1) for name, ms in steps_prof}
        return dict(sb=sb, n=n, c_host=c_host, t_total=t_total, clk=clk, prof=prof, t_prof=t_prof, stats=st,
                    init_s=init_s, sigma=sigma)

    m64 = measure("fp64", args.steps)
    sb = m64["sb"]
    n = m64["n"]
    value = world * args.steps / m64["t_total"]
    # e2e through the C ABI with host buffers (H2D of c and D2H of sigma per step)
    pin_c = torch.from_numpy(m64["c_host"]).pin_memory().numpy()
    sig = np.zeros(n)
    e2e_times = []
    for i in range(max(2, min(args.steps, 5))):
        sig[:] = 0
        torch.cuda.synchronize()
        t = time.perf_counter()
        sb.htimesc(pin_c, sig)
        e2e_times.append(time.perf_counter() - t)
    e2e = 1.0 / float(np.mean(e2e_times))
    st = m64["stats"]
    t_dom = m64["prof"]["all-external"] / 1e3 + m64["prof"].get("all-external split-k sum", 0.0) / 1e3
    roof = {"kernel": "gemm_tiled_f64 split-k (all-external W+/W- product, FP64)", "bound": "hbm",
            "achieved": st["bytes_allext"] / t_dom / 1e9, "peak": hbm, "unit": "GB/s",
            "frac": st["bytes_allext"] / t_dom / 1e9 / hbm, "traffic": None, "peak_kind": peak_kind}
    # Davidson solves at the reference's default tolerances (RESIDUAL/ENERGY TOLERANCE 1e-6)
    def solves(b, k):
        ts, es, its = [], None, None
        for _ in range(k):
            torch.cuda.synchronize()
            t = time.perf_counter()
            es, _, its = b.davidson(1, 1e-6, 1e-6)
            ts.append(time.perf_counter() - t)
        return 1.0 / float(np.mean(ts)), es, its

    dav64 = solves(sb, 2)
    sb.close()
    mixed = {}
    try:
        mx = measure("tf32x3", args.steps)
        sbx = mx["sb"]
        stx = mx["stats"]
        t_tc = mx["prof"]["all-external"] / 1e3
        np_, nm_ = None, None
        dav_x = solves(sbx, 2)
        w32_bytes = stx["bytes_allext"] / 2.0  # FP32 W: half of the FP64 bytes (padding aside)
        mixed = {"sigma_builds_per_s": world * args.steps / mx["t_total"],
                 "ms_per_step": 1e3 * mx["t_total"] / args.steps,
                 "sigma_rel_err_vs_fp64": float(np.abs(mx["sigma"] - m64["sigma"]).max() / np.abs(m64["sigma"]).max()),
                 "roofline": {"kernel": "allext_tf32x3_kernel (tcgen05 kind::tf32, TMA, 3xTF32, FP64 promotion)",
                              "bound": "hbm", "achieved": w32_bytes / t_tc / 1e9, "peak": hbm, "unit": "GB/s",
                              "frac": w32_bytes / t_tc / 1e9 / hbm, "traffic": None, "peak_kind": peak_kind},
                 "davidson_solves_per_s": dav_x[0], "davidson_iterations": int(dav_x[2]),
                 "energy": float(dav_x[1][0]), "step_ms": {k: round(v, 4) for k, v in sorted(mx["prof"].items(), key=lambda kv: -kv[1])[:8]},
                 "init_s": mx["init_s"]}
        sbx.close()
    except Exception as exc:  # the FP64 line stands on its own
        mixed = {"error": str(exc)[:300]}
    line = {"metric": METRIC, "value": value, "unit": "builds/s", "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": 1e3 * m64["t_total"] / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f64",
            "data": "synthetic (seeded operator of the benchmark shape)",
            "config": {"workload": WORKLOAD, "total_csfs": n, "parallelism": "replicas" if world > 1 else "single",
                       "l2": "flushed by a 256 MB write between timed builds; W operators (13.3 GB) exceed L2"},
            "sigma_tflops": st["flops_per_sigma"] * args.steps * world / m64["t_total"] / 1e12,
            "e2e": {"value": e2e, "unit": "builds/s", "h2d_bytes_per_step": 8 * n, "d2h_bytes_per_step": 8 * n},
            "gpu_launches": int(st["launches_per_sigma"]) * args.steps,
            "roofline": roof,
            "davidson": {"fp64_solves_per_s": dav64[0], "fp64_iterations": int(dav64[2]), "fp64_energy": float(dav64[1][0]),
                         "tf32x3_solves_per_s": mixed.get("davidson_solves_per_s"),
                         "tf32x3_energy_minus_fp64": (mixed["energy"] - float(dav64[1][0])) if "energy" in mixed else None},
            "mixed_tf32x3": mixed,
            "step_ms": {k: round(v, 4) for k, v in sorted(m64["prof"].items(), key=lambda kv: -kv[1])},
            "profiled_ms_per_step": 1e3 * m64["t_prof"] / args.steps,
            "init_s": m64["init_s"], "clocks": m64["clk"].summary()}
    if rank == 0 and world == 1 and not args.no_cpu_baseline:
        cb = cpu_sample()
        line["cpu_baseline"] = {"value": 1.0 / cb["t_sigma"], "unit": "builds/s", "cores": cb["cores"],
                                "kind": "port", "sample": cb["sample"]}
    if rank == 0:
        print(json.dumps(line), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
