#!/usr/bin/env python
"""Spin-flip attempts/s of the B200 simulated-annealing sampler.

Workload: the uneven batch -- 512 independent random-regular Ising problems,
n ~ U[64, 4096], degree ~ U{3..16}, J ~ N(0,1), h ~ N(0,0.1), reads ~ U[32,1024],
sweeps ~ U[256,2048], geometric beta 0.1 -> 5.0, Metropolis, sequential order,
seeded synthetic data.  One step = one anneal of the whole batch (every read of
every problem).  The persistent kernel (one launch, device work queue) is the
headline; the plain one-launch-per-problem kernel is timed beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

Under torchrun each rank anneals its own full batch (weak scaling, no
collective on the data path); timing is the max over ranks.
"""
from __future__ import annotations

import argparse
import copy
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
for _p in (os.path.join(ROOT, "dwave-samplers_b200"), os.path.join(ROOT, "oracle")):
    if _p not in sys.path:
        sys.path.insert(0, _p)

from b200sa import workloads  # noqa: E402

METRIC = "spin-flip attempts/s, 1 B200: batched vs plain (bit-exact); BM grad steps/s"
UNIT = "attempts/s"
FALLBACK_HBM_GBS = 6650.0
# DRAM bytes (dram__bytes_read.sum + dram__bytes_write.sum) per attempt of the
# n ~ 4000 bucket launch with delta energies in per-read global slots, from one
# ncu capture of the full uneven batch with every schedule cut to 5% of its
# sweeps: 695.7 GB over 2.26e10 attempts (0.12 bytes read, 30.7 written).  The
# traffic is per attempt (the schedule length repeats the same sweeps), so a
# full launch's traffic is this figure times its attempts.
L2_SLOT_DRAM_BYTES_PER_ATTEMPT = 30.8


def parse_args():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=3)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["ours", "reference"], default="ours")
    ap.add_argument("--problems", type=int, default=512)
    ap.add_argument("--plain-steps", type=int, default=1)
    ap.add_argument("--e2e-steps", type=int, default=1)
    ap.add_argument("--cpu-budget", type=float, default=15.0,
                    help="seconds of CPU baseline sampling on rank 0")
    ap.add_argument("--no-plain", action="store_true")
    ap.add_argument("--sweep-scale", type=float, default=1.0,
                    help="scale every schedule's length (profiling captures only; "
                         "1.0 is the benchmark workload)")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--n-range", type=int, nargs=2, default=None,
                    help="problem sizes (profiling captures only; default 64 4096)")
    ap.add_argument("--reads-range", type=int, nargs=2, default=None,
                    help="reads per problem (profiling captures only; default 32 1024)")
    ap.add_argument("--no-tune", action="store_true",
                    help="skip the autotuner (occupancy rule per bucket)")
    ap.add_argument("--mode", choices=["graph", "persistent"], default="graph",
                    help="batched runs: persistent launches replayed as a CUDA graph, or issued "
                         "one by one")
    ap.add_argument("--bm-steps", type=int, default=2,
                    help="timed Boltzmann-machine gradient steps (after one untimed step)")
    ap.add_argument("--bm-target-reads", type=int, default=8192,
                    help="reads behind the BM target correlations (outside the timed steps)")
    ap.add_argument("--descent-samples", type=int, default=16384,
                    help="steepest-descent leg: samples (0 skips it)")
    ap.add_argument("--rotor-samples", type=int, default=32768,
                    help="rotor-model (SQA) annealing leg: samples (0 skips it)")
    ap.add_argument("--pimc-samples", type=int, default=65536,
                    help="path-integral (SQA) annealing leg: samples (0 skips it)")
    ap.add_argument("--dense-reads", type=int, default=1000,
                    help="dense n=100 leg (1000 geometric sweeps): reads (0 skips it)")
    ap.add_argument("--lattice-reads", type=int, default=256,
                    help="3D lattice L=32 leg (4096 linear sweeps): reads (0 skips it)")
    ap.add_argument("--k16-reads", type=int, default=4096,
                    help="complete graph K16 leg (fixed beta 1, 10000 Gibbs sweeps): reads "
                         "(0 skips it)")
    return ap.parse_args()


def max_over_ranks(x: float, world: int, device=None) -> float:
    """Max of a per-rank scalar over all ranks (timings: the slowest rank)."""
    if world == 1:
        return x
    import torch
    import torch.distributed as dist
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def workload(args, rank=0):
    kw = {}
    if getattr(args, "n_range", None):
        kw["n_range"] = tuple(args.n_range)
    if getattr(args, "reads_range", None):
        kw["reads_range"] = tuple(args.reads_range)
    probs = workloads.uneven_batch(num_problems=args.problems, **kw)
    if args.sweep_scale != 1.0:
        for p in probs:
            k = max(1, int(round(len(p.betas) * args.sweep_scale)))
            p.betas = np.geomspace(0.1, 5.0, k)
    if rank:  # weak scaling: same shapes, rank-specific read seeds
        for p in probs:
            p.seeds = p.seeds + np.uint64(rank * (1 << 32))
    return probs


def workload_config(args, probs):
    return {
        "workload": f"uneven batch: {len(probs)} random-regular Ising problems, n~U[64,4096], "
                    "degree~U{3..16}, J~N(0,1), h~N(0,0.1), reads~U[32,1024], "
                    "sweeps~U[256,2048], geometric beta 0.1->5.0, Metropolis, sequential",
        "problems": len(probs),
        "reads": int(sum(p.num_reads for p in probs)),
        "attempts_per_step": int(sum(p.attempts for p in probs)),
        "max_n": int(max(p.n for p in probs)),
        "l2": "inputs larger than L2 (packed problems + states exceed 126 MB)",
        "seeds": "per read: base_seed + r",
    }


# ---------------------------------------------------------------- CPU side --

def cpu_threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def cpu_sample(probs, budget_s, threads=None, max_reads=None, gpu_out=None):
    """Time the reference's own CPU implementation (the extension built from
    its sources) -- or the C restatement when that build is absent -- on a
    bounded sample of reads of the same workload, all host threads, one read
    per call (num_samples=1, seed = that read's seed).

    ``gpu_out`` = (states, energies, state_offsets, read_offsets) of the GPU
    run of the same batch: every sampled read's reference result is then
    compared with the GPU's, bit for bit (``checked_reads`` / ``mismatches``)."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    threads = threads or cpu_threads()
    ref = oracle.reference_module()
    kind = "reference" if ref is not None else "port"
    rng = np.random.default_rng(99)
    order = [(int(p), 0) for p in rng.permutation(len(probs))]
    lists = {}

    results = {}

    def one(item):
        p, r = item
        P = probs[p]
        if ref is not None:
            if p not in lists:
                lists[p] = (list(map(float, P.h)), list(map(int, P.u)), list(map(int, P.v)),
                            list(map(float, P.J)))
            h, u, v, J = lists[p]
            s, e = ref.simulated_annealing(1, h, u, v, J, P.sweeps_per_beta, P.betas,
                                           int(P.seeds[r]), P.states[r:r + 1].copy())
        else:
            s, e = oracle.run(P.h, P.u, P.v, P.J, P.states[r:r + 1], P.sweeps_per_beta, P.betas,
                              P.seeds[r:r + 1])
        results[(p, r)] = (np.asarray(s)[0].copy(), float(np.asarray(e)[0]))
        return P.sweeps_per_beta * len(P.betas) * P.n

    # Python-list conversion outside the timed region.
    if ref is not None:
        for p, _ in order[: 4 * threads]:
            P = probs[p]
            lists[p] = (list(map(float, P.h)), list(map(int, P.u)), list(map(int, P.v)),
                        list(map(float, P.J)))
    attempts = 0
    reads = 0
    i = 0
    t0 = time.perf_counter()
    with ThreadPoolExecutor(max_workers=threads) as ex:
        while i < len(order):
            if max_reads is not None and reads >= max_reads:
                break
            chunk = order[i:i + threads]
            i += len(chunk)
            attempts += sum(ex.map(one, chunk))
            reads += len(chunk)
            if max_reads is None and time.perf_counter() - t0 >= budget_s:
                break
    dt = time.perf_counter() - t0
    out = {"value": attempts / dt, "unit": UNIT, "cores": threads, "kind": kind,
           "sample": f"{reads} reads (read 0 of randomly chosen problems of the same batch, "
                     f"full schedules), {attempts:.3e} attempts in {dt:.1f} s",
           "seconds": dt, "attempts": attempts}
    if gpu_out is not None:
        states, energies, so, ro = gpu_out
        bad = 0
        for (p, r), (s_ref, e_ref) in results.items():
            P = probs[p]
            s_gpu = states[so[p] + r * P.n: so[p] + (r + 1) * P.n]
            e_gpu = energies[ro[p] + r]
            if not (np.array_equal(s_gpu, s_ref)
                    and np.float64(e_gpu).view(np.uint64) == np.float64(e_ref).view(np.uint64)):
                bad += 1
        out["checked_reads"] = len(results)
        out["mismatches"] = bad
    return out


# ------------------------------------------------------------- GPU helpers --

def gpu_selector(device):
    """nvidia-smi -i argument for a torch device: its UUID when available
    (the visible device need not be physical GPU `device`)."""
    try:
        import torch
        uuid = str(torch.cuda.get_device_properties(device).uuid)
        if uuid:
            return uuid if uuid.startswith("GPU-") else "GPU-" + uuid
    except Exception:
        pass
    vis = os.environ.get("CUDA_VISIBLE_DEVICES")
    if vis:
        return vis.split(",")[device].strip()
    return str(device)


class Clocks:
    """Samples SM clock and throttle reasons with nvidia-smi while running."""
    FIELDS = ("clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.index = gpu_selector(device)
        self.proc = None
        self.lines = []

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(
                ["nvidia-smi", "-i", str(self.index), f"--query-gpu={self.FIELDS}",
                 "--format=csv,noheader,nounits", "-lms", "200"],
                stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.thread = threading.Thread(target=self._read, daemon=True)
            self.thread.start()
        except OSError:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.lines.append(line.strip())

    def __exit__(self, *exc):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except subprocess.TimeoutExpired:
                self.proc.kill()

    def summary(self):
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 8:
                continue
            try:
                sm.append(float(f[0]))
                mx = float(f[1])
            except ValueError:
                continue
            for name, val in zip(names, f[4:8]):
                if val.lower().startswith("active"):
                    reasons.add(name)
        if not sm:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": [], "samples": 0}
        load = [x for x in sm if mx and x > 0.3 * mx] or sm
        return {"sm_mhz": statistics.median(load), "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def measured_hbm_peak():
    path = os.path.join(ROOT, "MEASURED_PEAKS.json")
    try:
        with open(path) as f:
            return float(json.load(f)["hbm_gbs"]), "measured"
    except (OSError, KeyError, ValueError):
        return FALLBACK_HBM_GBS, "fallback"


def algorithmic_bytes(probs, flips):
    """Bytes the sweep must touch per launch (per-read state model):
    initial delta energies n*(8 + 13*d), per attempt 9 (delta energy 8 + spin 1),
    per flip 29*d + 9 (d x (index 4 + coupling 8 + neighbour spin 1 + delta
    energy read-modify-write 16) + own spin and delta energy), and the final
    energy 9n + 14m."""
    fixed = 0.0
    deg_w = 0.0
    att = 0.0
    for p in probs:
        n, m, R = p.n, p.J.shape[0], p.num_reads
        d = 2.0 * m / max(n, 1)
        a = p.attempts
        fixed += R * (n * (8 + 13 * d) + 9 * n + 14 * m) + 9 * a
        deg_w += d * a
        att += a
    dbar = deg_w / max(att, 1)
    return fixed + flips * (29 * dbar + 9)


def h2d_d2h_bytes(probs):
    bi = bo = 0
    for p in probs:
        n, m, R, nb = p.n, p.J.shape[0], p.num_reads, len(p.betas)
        # packed arena (row, col, w, h, vinfo, COO, betas, thresholds), seeds,
        # work items and initial states
        bi += 4 * (n + 1) + 24 * m + 8 * n + n + 16 * m + 16 * nb + 8 * R + 16 * R + n * R
        bo += n * R + 8 * R
    return bi, bo


# ------------------------------------------------------------------ arms ----

def bench_descent(args, local, world, rank):
    """Steepest descent (b200sa_steepest_descent, host buffers in and out,
    linear-search solver) from uniform random states on a random 6-regular
    Ising problem, n = 2048, J~N(0,1), h~N(0,0.1); one untimed call, then two
    timed calls (host clock, max over ranks).  Rank 0 also times the
    reference's own descent extension on all host threads over a bounded
    sample of the same samples."""
    import oracle
    from b200sa.greedy import steepest_gradient_descent
    rng = np.random.default_rng(17)
    n, u, v = workloads.random_regular(2048, 6, rng, graph_seed=17)
    J = rng.normal(0, 1, u.shape[0])
    h = rng.normal(0, 0.1, n)
    R = args.descent_samples
    init = (2 * rng.integers(0, 2, (R, n)) - 1).astype(np.int8)
    steepest_gradient_descent(R, h, u, v, J, init.copy(), False, device=local)
    times, steps = [], 0
    for _ in range(2):
        st = init.copy()
        t0 = time.perf_counter()
        _, _, k = steepest_gradient_descent(R, h, u, v, J, st, False, device=local)
        times.append(max_over_ranks(time.perf_counter() - t0, world, "cuda"))
        steps = int(k.sum())
    sec = statistics.median(times)
    out = {"workload": "random 6-regular Ising, n=2048, J~N(0,1), h~N(0,0.1), uniform random "
                       "initial states, linear-search solver",
           "samples": R, "samples_per_s": world * R / sec, "flips_per_s": world * steps / sec,
           "seconds": sec, "flips_per_sample": steps / R,
           "note": "host buffers in and out (the call as a user makes it)"}
    ref = oracle.reference_descent_module() if (rank == 0 and not args.no_cpu) else None
    if ref is not None:
        from concurrent.futures import ThreadPoolExecutor
        threads = cpu_threads()
        chunk = 8
        sample = min(R, threads * chunk * 2)
        hl, ul, vl, Jl = list(map(float, h)), list(map(int, u)), list(map(int, v)), list(map(float, J))

        def one(i):  # the binding releases the GIL while descending (descent.pyx:102)
            part = init[i:i + chunk].copy()
            ref.steepest_gradient_descent(part.shape[0], hl, ul, vl, Jl, part, False)

        with ThreadPoolExecutor(threads) as ex:
            t0 = time.perf_counter()
            list(ex.map(one, range(0, sample, chunk)))
            cpu = time.perf_counter() - t0
        out["cpu_reference"] = {"samples_per_s": sample / cpu, "cores": threads,
                                "sample": f"{sample} of the same samples"}
        out["gpu_over_cpu"] = out["samples_per_s"] / out["cpu_reference"]["samples_per_s"]
    return out


def bench_rotor(args, local, world, rank):
    """Rotor-model (SQA) annealing (b200sa_rotor_anneal, host buffers,
    MetropolisNonErgodic, sequential order, per-sample seeds) on a random
    6-regular problem, n = 512, J~N(0,1), h~N(0,0.1), transverse fields
    U[0.5, 1.5], 64 sweeps of geometric schedules (problem 0.1 -> 5,
    driver 5 -> 0.05), uniform random angles; one untimed call, then two
    timed calls.  Rank 0 also times the reference's own extension (one call
    per sample, seed + r) on all host threads over a bounded sample."""
    import oracle
    from b200sa.sqa import simulated_annealing as rotor
    rng = np.random.default_rng(29)
    n, u, v = workloads.random_regular(512, 6, rng, graph_seed=29)
    J = rng.normal(0, 1, u.shape[0])
    h = rng.normal(0, 0.1, n)
    tf = rng.uniform(0.5, 1.5, n)
    hp = np.geomspace(0.1, 5.0, 64)
    hd = np.geomspace(5.0, 0.05, 64)
    R = args.rotor_samples
    init = rng.integers(0, 256, (R, n)).astype(np.uint8)
    call = lambda st: rotor(R, h, u, v, J, tf, 1, hp, hd, 1234, st, False,
                            "MetropolisNonErgodic", 0, device=local)
    call(init.copy())
    times = []
    for _ in range(2):
        st = init.copy()
        t0 = time.perf_counter()
        call(st)
        times.append(max_over_ranks(time.perf_counter() - t0, world, "cuda"))
    sec = statistics.median(times)
    attempts = R * n * len(hp)
    out = {"workload": "rotor model, random 6-regular n=512, J~N(0,1), h~N(0,0.1), transverse "
                       "fields U[0.5,1.5], 64 sweeps, MetropolisNonErgodic, sequential order",
           "samples": R, "attempts_per_s": world * attempts / sec, "seconds": sec,
           "note": "host buffers in and out (the call as a user makes it)"}
    ref = oracle.reference_rotormc_module() if (rank == 0 and not args.no_cpu) else None
    if ref is not None:
        from concurrent.futures import ThreadPoolExecutor
        threads = cpu_threads()
        sample = min(R, threads * 4)
        args_ref = (list(map(float, h)), list(map(int, u)), list(map(int, v)),
                    list(map(float, J)), list(map(float, tf)), 1, hp, hd)

        def one(r):  # one call per sample, seed + r; the binding releases the GIL
            ref.simulated_annealing(1, *args_ref, 1234 + r, init[r:r + 1].copy(), False,
                                    "MetropolisNonErgodic", 0)

        with ThreadPoolExecutor(threads) as ex:
            t0 = time.perf_counter()
            list(ex.map(one, range(sample)))
            cpu = time.perf_counter() - t0
        out["cpu_reference"] = {"attempts_per_s": sample * n * len(hp) / cpu, "cores": threads,
                                "sample": f"{sample} of the same samples"}
        out["gpu_over_cpu"] = out["attempts_per_s"] / out["cpu_reference"]["attempts_per_s"]
    return out


def bench_pimc(args, local, world, rank):
    """Path-integral Monte Carlo (SQA) annealing (b200sa_path_anneal, host
    buffers, single-qubit updates, per-sample seeds) on a random 6-regular
    problem, n = 512, J~N(0,1), h~N(0,0.1), 16 schedule steps of one sweep
    (invTemp 0.1 -> 5, transverse field 5 -> 0.05, geometric), uniform random
    initial states; one untimed call, then two timed calls.  Rank 0 also times
    the reference's own extension (one call per sample, seed + r) on all host
    threads over a bounded sample."""
    import oracle
    from b200sa.sqa import path_annealing
    rng = np.random.default_rng(31)
    n, u, v = workloads.random_regular(512, 6, rng, graph_seed=31)
    J = rng.normal(0, 1, u.shape[0])
    h = rng.normal(0, 0.1, n)
    hp = np.geomspace(0.1, 5.0, 16)
    hd = np.geomspace(5.0, 0.05, 16)
    R = args.pimc_samples
    init = (2 * rng.integers(0, 2, (R, n)) - 1).astype(np.int8)
    nb = np.zeros((R, n), np.intc)
    none = np.zeros(1, np.intc)
    call = lambda st: path_annealing(R, h, u, v, J, 1, hp, hd, 1.0, 1.0, 1, 1, 4321, st, True,
                                     True, nb, none, none, 0, device=local)
    call(init.copy())
    times = []
    for _ in range(2):
        st = init.copy()
        t0 = time.perf_counter()
        call(st)
        times.append(max_over_ranks(time.perf_counter() - t0, world, "cuda"))
    sec = statistics.median(times)
    updates = R * n * len(hp)
    out = {"workload": "path-integral annealing, random 6-regular n=512, J~N(0,1), h~N(0,0.1), "
                       "16 steps x 1 sweep, invTemp 0.1->5, Gamma 5->0.05, single-qubit updates",
           "samples": R, "updates_per_s": world * updates / sec, "seconds": sec,
           "note": "host buffers in and out (the call as a user makes it)"}
    ref = oracle.reference_pimc_module() if (rank == 0 and not args.no_cpu) else None
    if ref is not None:
        from concurrent.futures import ThreadPoolExecutor
        threads = cpu_threads()
        sample = min(R, threads * 32)
        args_ref = (list(map(float, h)), list(map(int, u)), list(map(int, v)),
                    list(map(float, J)), 1, hp, hd, 1.0, 1.0, 1, 1)

        def one(r):  # one call per sample, seed + r; the binding releases the GIL
            ref.simulated_annealing(1, *args_ref, 4321 + r, init[r:r + 1].copy(), True, True,
                                    np.zeros((1, n), np.intc), np.zeros(1, np.intc),
                                    np.zeros(1, np.intc), 0)

        with ThreadPoolExecutor(threads) as ex:
            t0 = time.perf_counter()
            list(ex.map(one, range(sample)))
            cpu = time.perf_counter() - t0
        out["cpu_reference"] = {"updates_per_s": sample * n * len(hp) / cpu, "cores": threads,
                                "sample": f"{sample} of the same samples"}
        out["gpu_over_cpu"] = out["updates_per_s"] / out["cpu_reference"]["updates_per_s"]
    return out


def bench_single(args, local, world, rank, inst, label, calls, cpu_reads):
    """One problem through simulated_annealing (the drop-in binding: host
    buffers in and out), per-read seeds.  `value` = attempts / device time of
    the sweep launches (CUDA events inside the call); `e2e` = attempts / wall
    time of the whole call.  Median of `calls` calls.  Rank 0 also times the
    reference's own extension (one read per call, all host threads) on
    `cpu_reads` of the same reads and compares them with the GPU's."""
    import oracle
    from concurrent.futures import ThreadPoolExecutor
    from b200sa import simulated_annealing
    gibbs = inst.proposal.lower() == "gibbs"
    kern, wall, stats = [], [], {}
    s = e = None
    for _ in range(calls):
        st = inst.states.copy()
        stats = {}
        t0 = time.perf_counter()
        s, e = simulated_annealing(inst.num_reads, inst.h, inst.u, inst.v, inst.J,
                                   inst.sweeps_per_beta, inst.betas, 0, st, inst.randomize_order,
                                   inst.proposal, seeds=inst.seeds, device=local, stats=stats)
        wall.append(max_over_ranks(time.perf_counter() - t0, world, "cuda"))
        kern.append(max_over_ranks(stats["kernel_ms"] / 1000.0, world, "cuda"))
    A = inst.attempts
    out = {"workload": label, "reads": inst.num_reads, "attempts_per_call": A,
           "value": world * A / statistics.median(kern), "unit": UNIT,
           "e2e": world * A / statistics.median(wall),
           "kernel_seconds": statistics.median(kern), "call_seconds": statistics.median(wall),
           "calls": calls, "attempts_per_pass": A / max(stats["passes"], 1),
           "flips": stats["flips"], "near_ties": stats["near_ties"]}
    ref = oracle.reference_module() if (rank == 0 and not args.no_cpu) else None
    if ref is not None and cpu_reads > 0:
        threads = cpu_threads()
        hl, ul, vl, Jl = (list(map(float, inst.h)), list(map(int, inst.u)),
                          list(map(int, inst.v)), list(map(float, inst.J)))
        crit = "Gibbs" if gibbs else "Metropolis"

        def one(r):  # num_samples=1, that read's seed; the binding releases the GIL
            rs, re_ = ref.simulated_annealing(1, hl, ul, vl, Jl, inst.sweeps_per_beta, inst.betas,
                                              int(inst.seeds[r]), inst.states[r:r + 1].copy(),
                                              inst.randomize_order, crit)
            return (np.array_equal(rs[0], s[r])
                    and np.float64(re_[0]).view(np.uint64) == np.float64(e[r]).view(np.uint64))

        rows = list(range(min(cpu_reads, inst.num_reads)))
        with ThreadPoolExecutor(threads) as ex:
            t0 = time.perf_counter()
            same = list(ex.map(one, rows))
            cpu = time.perf_counter() - t0
        per_read = inst.attempts // inst.num_reads
        out["cpu_reference"] = {"value": len(rows) * per_read / cpu, "unit": UNIT,
                                "cores": threads, "kind": "reference",
                                "sample": f"{len(rows)} of the same reads, one read per call"}
        out["checked_reads"] = len(rows)
        out["mismatches"] = int(len(rows) - sum(same))
        out["gpu_over_cpu"] = out["value"] / out["cpu_reference"]["value"]
        out["e2e_over_cpu"] = out["e2e"] / out["cpu_reference"]["value"]
    return out


def bench_bm(args, local, world):
    """Batched Boltzmann-machine learning: 64 six-regular models, n~U[256,2048],
    ground truth J*~N(0,0.5), h*=0, targets from 8192 reads; per gradient step
    1024 fixed-beta (beta=1) Gibbs reads x 2000 sweeps of every model in one
    persistent batch (autotuned launch shapes, weights written on the device),
    the moments kernel backward and an Adam update (lr 1e-2).  One untimed
    step (it includes the autotuner), then `bm_steps` timed steps (host clock
    around each synchronized step, max over ranks)."""
    import torch
    from b200sa import bm
    truth = workloads.bm_models(num_models=64, n_range=(256, 2048), d=6, J_sigma=0.5, seed=5)
    reads, sweeps = 1024, 2000
    res = bm.fit(truth, beta=1.0, steps=1 + args.bm_steps, reads=reads, sweeps=sweeps, lr=1e-2,
                 target_reads=args.bm_target_reads, target_sweeps=sweeps, seed=3, device=local)
    timed = [max_over_ranks(t, world, "cuda") for t in res.step_seconds[1:]]
    sec = sum(timed) / len(timed)
    attempts = reads * sweeps * sum(len(h) for h, *_ in truth)
    return {"grad_steps_per_s": world / sec, "seconds_per_step": sec, "steps_timed": len(timed),
            "attempts_per_step": attempts, "attempts_per_s": world * attempts / sec,
            "models": len(truth), "reads": reads, "sweeps": sweeps, "beta": 1.0,
            "target_reads": args.bm_target_reads, "target_seconds": res.target_seconds,
            "corr_error": [res.corr_error[0], res.corr_error[-1]],
            "note": "each rank fits its own 64 models (weak scaling); targets from "
                    f"{args.bm_target_reads} reads, outside the timed steps"}


def run_reference(args):
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return 0
    probs = workload(args)
    threads = cpu_threads()
    per_step = max(threads, 2 * threads)
    for _ in range(args.warmup):
        cpu_sample(probs, 0, threads, max_reads=threads)
    t_att = 0
    t_sec = 0.0
    last = None
    for k in range(args.steps):
        r = cpu_sample(probs[k % 2::2] if k % 2 else probs, 0, threads, max_reads=per_step)
        t_att += r["attempts"]
        t_sec += r["seconds"]
        last = r
    value = t_att / t_sec
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT,
        "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup,
        "ms_per_step": 1000.0 * t_sec / args.steps, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, probs),
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": threads, "kind": last["kind"],
                         "sample": f"each step: {per_step} reads of the batch, one read per call "
                                   "(num_samples=1, that read's seed), all host threads"},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line))
    return 0


def run_ours(args):
    import torch
    import torch.distributed as dist
    from b200sa import Plan, sample_batch

    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    if world > 1:
        from datetime import timedelta
        torch.cuda.set_device(local)
        dist.init_process_group("nccl", timeout=timedelta(seconds=600),
                                device_id=torch.device("cuda", local))
    else:
        torch.cuda.set_device(local)

    def barrier():
        if world > 1:
            dist.barrier()

    probs = workload(args, rank)
    attempts = int(sum(p.attempts for p in probs))
    plan = Plan(probs, device=local)
    tune = None
    if not args.no_tune:
        import tempfile
        cache = os.path.join(tempfile.gettempdir(), f"b200sa_tune_{os.getpid()}.txt")
        t0 = time.perf_counter()
        entries = plan.autotune(cache, force=True)
        tune = {"seconds": time.perf_counter() - t0, "buckets": [
            {k: e[k] for k in ("max_n", "items", "staging", "warps_per_cta", "ctas_per_sm",
                               "registers", "candidates")} for e in entries]}
        os.environ["B200SA_TUNE_CACHE"] = cache  # the e2e call reuses these choices
    host_states = np.concatenate([p.states.ravel() for p in probs])
    sin = torch.from_numpy(host_states).cuda()
    sout = torch.empty_like(sin)
    en = torch.empty(plan.total_reads, dtype=torch.float64, device="cuda")
    stream = torch.cuda.Stream()

    run_stats = {}

    def timed(mode, warmup, steps):
        for k in range(warmup):
            last = k == warmup - 1
            st = plan.run(sin, sout, en, mode=mode, stream=stream, sync=last)
            if last:
                run_stats[mode] = st
        torch.cuda.synchronize()
        barrier()
        torch.cuda.synchronize()
        e0 = torch.cuda.Event(enable_timing=True)
        e1 = torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        for _ in range(steps):
            plan.run(sin, sout, en, mode=mode, stream=stream, sync=False)
        e1.record(stream)
        torch.cuda.synchronize()
        barrier()
        return e0.elapsed_time(e1)

    with Clocks(local) as clk:
        total_ms = timed(args.mode, args.warmup, args.steps)
    total_ms = max_over_ranks(total_ms, world, "cuda")
    ms_step = total_ms / args.steps
    value = world * attempts / (ms_step / 1000.0)

    # Per-bucket device times of the last timed step (events around each
    # bucket's launch, captured into the graph) and their counters.
    buckets = plan.bucket_report()
    gpu_out = (sout.cpu().numpy(), en.cpu().numpy(), plan.state_offsets, plan.read_offsets)

    # Counters of the last warm-up run (deterministic for these inputs).
    if args.mode not in run_stats:
        run_stats[args.mode] = plan.run(sin, sout, en, mode=args.mode, stream=stream, sync=True)
    stats = run_stats[args.mode]
    flips = stats["flips"]
    if stats["attempts"] != attempts:
        raise RuntimeError(f"attempt count mismatch: {stats['attempts']} != {attempts}")

    line = {
        "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms_step, "higher_is_better": True,
        "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": workload_config(args, probs) | {
            "parallelism": f"independent batch per GPU x{world}",
            "batched_runs": ("persistent launches replayed as one CUDA graph" if args.mode == "graph"
                             else "persistent launches"),
            "autotune": tune},
    }
    peak, peak_src = measured_hbm_peak()
    # The dominant kernel: the bucket launch with the most work (attempts);
    # buckets run side by side, so the launch that spans the step is not
    # necessarily the one doing most of it.
    timed_b = [b for b in buckets if b["ms"] > 0]
    dom = max(timed_b, key=lambda b: b["attempts"]) if timed_b else None
    if dom is not None:
        achieved = dom["model_bytes"] / (dom["ms"] / 1000.0) / 1e9
        scaled = dom["staging"] == 2 and dom["max_n"] > 2048
        line["roofline"] = {
            "bound": "hbm", "achieved": achieved, "peak": peak, "unit": "GB/s",
            "frac": achieved / peak,
            "traffic": L2_SLOT_DRAM_BYTES_PER_ATTEMPT * dom["attempts"] if scaled else None,
            "traffic_source": ("ncu DRAM bytes per attempt of this bucket's launch (schedules cut "
                               "to 5%), times this launch's attempts" if scaled else
                               "no capture for this launch's state location"),
            "peak_source": peak_src,
            "kernel": f"sweep launch of the n<={dom['max_n']} bucket (state location "
                      f"{dom['staging']}, {dom['registers']} registers, {dom['warps_per_cta']} "
                      f"warps per CTA, grid {dom['grid']})",
            "algorithmic_bytes_per_launch": dom["model_bytes"], "launch_ms": dom["ms"],
            "note": "algorithmic bytes = the sweep's state accesses (delta energies, spins, "
                    "adjacency), mostly served from shared memory, L1 and L2; the sweep is a "
                    "latency-bound sequential chain per read, not HBM-bound",
            "step_achieved_gbs": algorithmic_bytes(probs, flips) / (ms_step / 1000.0) / 1e9}
    line["buckets"] = [{k: b[k] for k in ("max_n", "kind", "reads", "attempts", "ms", "staging",
                                          "warps_per_cta", "registers")}
                       | {"attempts_per_pass": b["attempts"] / max(b["passes"], 1)}
                       for b in buckets]
    line["clocks"] = clk.summary()
    line["gpu_launches"] = args.steps * int(stats["launches"])
    line["counters"] = {"flips": flips, "near_ties": stats["near_ties"],
                        "attempts_per_pass": attempts / max(stats["passes"], 1),
                        "check_run_kernel_ms": stats["kernel_ms"]}

    if not args.no_plain:
        # One launch per problem, problems in order.  "plain" gives every launch
        # the autotuned shape of its size bucket (so the ratio measures the
        # batching alone); "plain_untuned" uses the occupancy rule.
        plain_ms = max_over_ranks(timed("plain_tuned", 0, args.plain_steps), world,
                                  "cuda") / args.plain_steps
        line["plain"] = {"value": world * attempts / (plain_ms / 1000.0), "ms_per_step": plain_ms,
                         "launches_per_step": len(probs),
                         "shapes": "autotuned per size bucket, as the batched run"}
        line["batched_over_plain"] = plain_ms / ms_step
        if not args.no_tune:
            pu_ms = max_over_ranks(timed("plain", 0, args.plain_steps), world,
                                   "cuda") / args.plain_steps
            line["plain_untuned"] = {"value": world * attempts / (pu_ms / 1000.0),
                                     "ms_per_step": pu_ms, "launches_per_step": len(probs),
                                     "shapes": "occupancy rule (no autotuning)"}
            line["batched_over_plain_untuned"] = pu_ms / ms_step

    # End to end through the C ABI with host buffers (pack + H2D + anneal + D2H).
    # The states (inputs and outputs) live in pinned host memory, as a caller
    # feeding the sampler from a pinned staging buffer would keep them.
    bi, bo = h2d_d2h_bytes(probs)
    e2e_times = []
    pinned = torch.empty(sum(p.states.size for p in probs), dtype=torch.int8,
                         pin_memory=torch.cuda.is_available())
    for _ in range(args.e2e_steps):
        work = [copy.copy(p) for p in probs]
        off = 0
        for w in work:
            view = pinned[off:off + w.states.size].numpy().reshape(w.states.shape)
            view[...] = w.states
            w.states = view
            off += w.states.size
        torch.cuda.synchronize()
        barrier()
        t0 = time.perf_counter()
        sample_batch(work, mode=args.mode, device=local)
        dt = time.perf_counter() - t0
        e2e_times.append(max_over_ranks(dt, world, "cuda"))
    if e2e_times:
        e2e = statistics.median(e2e_times)
        line["e2e"] = {"value": world * attempts / e2e, "unit": UNIT, "h2d_bytes_per_step": bi,
                       "d2h_bytes_per_step": bo, "seconds_per_step": e2e}

    plan.close()
    del sin, sout, en
    if args.dense_reads > 0:
        inst = workloads.dense_ising(reads=args.dense_reads)
        lab = ("dense n=100, edge p=0.5, J,h~U[-1,1], {} reads x 1000 geometric sweeps 0.1->4.2, "
               "Metropolis, {} order")
        line["dense100"] = bench_single(args, local, world, rank, inst,
                                        lab.format(args.dense_reads, "sequential"), 3,
                                        args.dense_reads)
        inst.randomize_order = True
        line["dense100_random"] = bench_single(args, local, world, rank, inst,
                                               lab.format(args.dense_reads, "random"), 3,
                                               args.dense_reads)
    if args.lattice_reads > 0:
        inst = workloads.cubic_lattice(reads=args.lattice_reads)
        line["lattice32"] = bench_single(
            args, local, world, rank, inst,
            f"3D periodic cubic lattice L=32 (32768 spins), J=+-1, h=0, {args.lattice_reads} reads "
            "x 4096 linear sweeps 0.1->3.0, Metropolis, sequential order", 1, cpu_threads())
    if args.k16_reads > 0:
        inst = workloads.complete_graph(reads=args.k16_reads)
        line["k16_gibbs"] = bench_single(
            args, local, world, rank, inst,
            f"complete graph K16, J~N(0,0.3), h~N(0,0.1), {args.k16_reads} reads x 10000 sweeps "
            "at fixed beta 1, Gibbs, sequential order", 3, args.k16_reads)
    if args.bm_steps > 0:
        line["bm"] = bench_bm(args, local, world)
    if args.descent_samples > 0:
        line["descent"] = bench_descent(args, local, world, rank)
    if args.rotor_samples > 0:
        line["rotor"] = bench_rotor(args, local, world, rank)
    if getattr(args, "pimc_samples", 0) > 0:
        line["pimc"] = bench_pimc(args, local, world, rank)

    if rank == 0 and not args.no_cpu:
        cb = cpu_sample(probs, args.cpu_budget, gpu_out=gpu_out)
        line["cpu_baseline"] = {k: cb[k] for k in ("value", "unit", "cores", "kind", "sample",
                                                   "checked_reads", "mismatches")}
    if rank == 0:
        print(json.dumps(line))
    if world > 1:
        dist.destroy_process_group()
    return 0


def main():
    args = parse_args()
    if args.impl == "reference":
        return run_reference(args)
    return run_ours(args)


if __name__ == "__main__":
    sys.exit(main())
