"""The multi-GPU benchmark path on CPU: two gloo ranks build their own
batches (same shapes, disjoint read seeds: weak scaling with no collective on
the data path) and agree on the slowest rank's time."""
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
