"""Bit-exact parity at the benchmark sizes.

The per-read contract (dwave/samplers/sa/src/cpu_sa.cpp:283-284, 321-358):
read r of a call equals the reference run with num_samples=1, seed=seeds[r]
and the same initial state -- identical final spins and energies bit for bit.
Checked here on the full benchmark workloads, against the CPU oracle run on
all host threads:

* dense n=100 (1000 reads x 1000 geometric sweeps): every read;
* the uneven batch of 512 random-regular problems, annealed exactly as the
  benchmark anneals it (autotuned launches replayed as one CUDA graph): the
  first and the last read of every problem, and every read of the eight
  problems with the largest n;
* every read reports a near-tie count of zero.

The 3D lattice (L=32, 4096 sweeps) is checked in test_gpu_parity.py.
"""
import os
from concurrent.futures import ThreadPoolExecutor

import numpy as np
import pytest

import oracle
from b200sa import Plan, simulated_annealing, workloads
from conftest import bits

pytestmark = pytest.mark.gpu


def _threads():
    try:
        return len(os.sched_getaffinity(0))
    except AttributeError:
        return os.cpu_count() or 1


def _oracle_reads(jobs):
    """jobs: (key, instance, read indices); returns {key: (states, energies)}
    from the oracle, reads spread over all host threads (the oracle releases
    the GIL)."""
    def one(job):
        key, p, rows = job
        gibbs = p.proposal.lower() == "gibbs"
        return key, oracle.run(p.h, p.u, p.v, p.J, p.states[rows], p.sweeps_per_beta, p.betas,
                               p.seeds[rows], p.randomize_order, gibbs)
    with ThreadPoolExecutor(_threads()) as ex:
        return dict(ex.map(one, jobs))


def test_dense100_every_read():
    inst = workloads.dense_ising()
    st = inst.states.copy()
    stats = {}
    s, e = simulated_annealing(inst.num_reads, inst.h, inst.u, inst.v, inst.J, 1, inst.betas,
                               0, st, seeds=inst.seeds, stats=stats)
    assert stats["attempts"] == inst.attempts == 10**8
    assert stats["near_ties"] == 0 and not stats["near_ties_per_read"].any()
    chunk = 25
    jobs = [(r0, inst, np.arange(r0, min(r0 + chunk, inst.num_reads)))
            for r0 in range(0, inst.num_reads, chunk)]
    want = _oracle_reads(jobs)
    for r0, rows in ((j[0], j[2]) for j in jobs):
        ws, we = want[r0]
        np.testing.assert_array_equal(s[rows], ws)
        np.testing.assert_array_equal(bits(e[rows]), bits(we))


def test_uneven_batch_full_size_as_benchmarked(tmp_path):
    import torch
    probs = workloads.uneven_batch()
    with Plan(probs) as plan:
        plan.autotune(str(tmp_path / "tune.txt"), force=True)
        host = np.concatenate([p.states.ravel() for p in probs])
        sin = torch.from_numpy(host).cuda()
        sout = torch.empty_like(sin)
        en = torch.empty(plan.total_reads, dtype=torch.float64, device="cuda")
        st = plan.run(sin, sout, en, mode="graph", sync=True, per_read=True)
        assert st["attempts"] == sum(p.attempts for p in probs)
        assert st["near_ties"] == 0 and not st["near_ties_per_read"].any()
        out = sout.cpu().numpy()
        energies = en.cpu().numpy()
        so, ro = plan.state_offsets, plan.read_offsets
    largest = set(np.argsort([-p.n for p in probs], kind="stable")[:8].tolist())
    jobs = []
    for k, p in enumerate(probs):
        if k in largest:
            for r0 in range(0, p.num_reads, 16):
                jobs.append(((k, r0), p, np.arange(r0, min(r0 + 16, p.num_reads))))
        else:
            jobs.append(((k, 0), p, np.array(sorted({0, p.num_reads - 1}))))
    want = _oracle_reads(jobs)
    checked = 0
    for (k, r0), p, rows in jobs:
        ws, we = want[(k, r0)]
        got = out[so[k]:so[k + 1]].reshape(p.num_reads, p.n)[rows]
        np.testing.assert_array_equal(got, ws, err_msg=f"problem {k} reads {rows}")
        np.testing.assert_array_equal(bits(energies[ro[k]:ro[k + 1]][rows]), bits(we),
                                      err_msg=f"problem {k} reads {rows}")
        checked += len(rows)
    assert checked > 2 * len(probs)
