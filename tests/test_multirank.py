"""The multi-GPU paths on CPU.  The benchmark: two gloo ranks build their own
batches (same shapes, disjoint read seeds: weak scaling with no collective on
the data path) and agree on the slowest rank's time.  The sharded batch
(b200sa.shards): one batch partitioned across two ranks, annealed rank by rank
and gathered, equals the one-rank result byte for byte."""
import os
import socket
import sys
from types import SimpleNamespace

import numpy as np
import torch.multiprocessing as mp

from conftest import ROOT


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def _rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    for p in (ROOT, os.path.join(ROOT, "dwave-samplers_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from datetime import timedelta
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    import bench
    args = SimpleNamespace(problems=3, sweep_scale=1.0)
    probs = bench.workload(args, rank)
    slowest = bench.max_over_ranks(10.0 * (rank + 1), world, "cpu")
    out[rank] = (slowest, [p.n for p in probs], [int(p.seeds[0]) for p in probs],
                 [p.states.tobytes() for p in probs])
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_weak_scaling_and_max_timing():
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    (t0, n0, s0, st0), (t1, n1, s1, st1) = out[0], out[1]
    assert t0 == t1 == 20.0            # both ranks see the slowest rank's time
    assert n0 == n1 and st0 == st1     # same problem shapes and initial states
    assert set(s0).isdisjoint(s1)      # rank-specific read seeds


# ---- one batch split across ranks (b200sa.shards) -------------------------

def _small_batch():
    from b200sa import workloads
    probs = workloads.uneven_batch(num_problems=7, n_range=(20, 120), reads_range=(1, 9),
                                   sweeps_range=(5, 30), seed=71)
    probs.append(workloads.complete_graph(reads=13, sweeps=25, seed=71))  # Gibbs
    probs[2].randomize_order = True
    return probs


def _oracle_worker(sub):
    """The per-rank worker of the test: the CPU oracle in place of a GPU."""
    import oracle
    states, ens = [], []
    for p in sub:
        s, e = oracle.run(p.h, p.u, p.v, p.J, p.states, p.sweeps_per_beta, p.betas, p.seeds,
                          p.randomize_order, p.proposal.lower() == "gibbs")
        states.append(s)
        ens.append(e)
    return states, ens


def _shard_rank(rank, world, port, out, dst):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    for p in (ROOT, os.path.join(ROOT, "dwave-samplers_b200"), os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    from datetime import timedelta
    from b200sa import shards
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    probs = _small_batch()
    ens = shards.sample_batch_distributed(probs, group=None, dst=dst, worker=_oracle_worker)
    out[rank] = None if ens is None else ([p.states.tobytes() for p in probs],
                                          [e.tobytes() for e in ens])
    dist.barrier()
    dist.destroy_process_group()


def test_partition_covers_every_read_once_and_balances():
    for p in (os.path.join(ROOT, "dwave-samplers_b200"),):
        if p not in sys.path:
            sys.path.insert(0, p)
    from b200sa import shards, workloads
    probs = workloads.uneven_batch(num_problems=40, n_range=(64, 4096), reads_range=(32, 1024),
                                   sweeps_range=(2, 4), seed=5)
    for parts in (1, 2, 3, 8):
        plan = shards.partition(probs, parts)
        seen = [np.zeros(p.num_reads, int) for p in probs]
        loads = []
        for chunks in plan:
            load = 0
            for k, r0, r1 in chunks:
                seen[k][r0:r1] += 1
                load += (r1 - r0) * len(probs[k].betas) * probs[k].n
            loads.append(load)
        assert all((s == 1).all() for s in seen)
        assert max(loads) <= 1.05 * (sum(loads) / parts) + 1
        assert plan == shards.partition(probs, parts)  # deterministic


def test_two_rank_sharded_batch_equals_one_rank():
    """Two gloo ranks each anneal their shard (the oracle stands in for the
    GPU), exchange them and both hold the one-rank result byte for byte; with
    a destination rank only that rank does."""
    import oracle  # noqa: F401  (built before the ranks start)
    ref = _small_batch()
    want_e = []
    for p in ref:
        s, e = _oracle_worker([p])
        p.states[:] = s[0]
        want_e.append(e[0])
    want = ([p.states.tobytes() for p in ref], [e.tobytes() for e in want_e])
    world = 2
    for dst in (None, 1):
        mgr = mp.Manager()
        out = mgr.dict()
        mp.spawn(_shard_rank, args=(world, _free_port(), out, dst), nprocs=world, join=True)
        for r in range(world):
            if dst is None or r == dst:
                assert out[r] == want
            else:
                assert out[r] is None


# ---- Boltzmann-machine moments pooled across ranks (b200sa.autograd) -------

def _bm_problem():
    rng = np.random.default_rng(91)
    n = 24
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.3
    u, v = iu[keep].astype(np.int32), ju[keep].astype(np.int32)
    J = rng.normal(0, 0.5, u.shape[0])
    h = np.zeros(n)
    states = (2 * rng.integers(0, 2, (16, n)) - 1).astype(np.int8)
    seeds = np.arange(16, dtype=np.uint64) + 500
    return h, u, v, J, states, seeds


def _bm_sums(rows):
    """Moment sums (int64) of the oracle's Gibbs reads `rows` at beta = 1."""
    import oracle
    h, u, v, J, states, seeds = _bm_problem()
    s, _ = oracle.run(h, u, v, J, states[rows], 50, np.array([1.0]), seeds[rows], False, True)
    s = s.astype(np.int64)
    return s.sum(0), (s[:, u] * s[:, v]).sum(0)


def _bm_rank(rank, world, port, out):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    for p in (ROOT, os.path.join(ROOT, "dwave-samplers_b200"), os.path.join(ROOT, "oracle")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch
    import torch.distributed as dist
    from datetime import timedelta
    from b200sa.autograd import pool_sums
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=60))
    reads = 16 // world  # each rank samples its own reads [rank R, (rank + 1) R)
    s, ss = _bm_sums(np.arange(rank * reads, (rank + 1) * reads))
    ps, pss = pool_sums([torch.from_numpy(s)], [torch.from_numpy(ss)], None)
    out[rank] = (ps[0].numpy().tolist(), pss[0].numpy().tolist())
    dist.barrier()
    dist.destroy_process_group()


def test_two_rank_bm_moments_pool_to_the_one_rank_sums():
    """Each rank takes half of the reads (their seeds and initial states, as a
    SamplingSpec with a group does) and the moment sums are pooled by one
    all-reduce: both ranks hold exactly the sums of one run over all reads."""
    import oracle  # noqa: F401  (built before the ranks start)
    s, ss = _bm_sums(np.arange(16))
    world = 2
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_bm_rank, args=(world, _free_port(), out), nprocs=world, join=True)
    for r in range(world):
        assert out[r] == (s.tolist(), ss.tolist())
