"""Plan features with no reference counterpart, checked against the plan's
own persistent runs and the oracle: CUDA-graph replay, in-place weight
updates, and the autotuner (its choices must not change any result)."""
import copy

import numpy as np
import pytest
import torch

import oracle
from b200sa import Plan, sample_batch, workloads
from b200sa.workloads import Instance, random_regular, random_states
from conftest import bits

pytestmark = pytest.mark.gpu


def mixed_batch(seed=31):
    """Small uneven problems plus one above the on-chip size (global state)."""
    probs = workloads.uneven_batch(num_problems=10, n_range=(64, 900), reads_range=(3, 24),
                                   sweeps_range=(10, 60), seed=seed)
    rng = np.random.default_rng(seed)
    n, u, v = random_regular(9000, 4, rng, graph_seed=seed)
    probs.append(Instance(rng.normal(0, 0.1, n), u, v, rng.normal(0, 1, u.shape[0]),
                          random_states(rng, 5, n), np.geomspace(0.1, 5.0, 8), 1,
                          np.arange(5, dtype=np.uint64) + 99))
    k16 = workloads.complete_graph(reads=16, sweeps=30, seed=seed)
    probs.append(k16)  # Gibbs
    return probs


def device_buffers(plan, probs):
    host = np.concatenate([p.states.ravel() for p in probs])
    sin = torch.from_numpy(host).cuda()
    out = torch.empty_like(sin)
    en = torch.empty(plan.total_reads, dtype=torch.float64, device="cuda")
    return sin, out, en


def test_graph_replay_equals_persistent():
    probs = mixed_batch()
    with Plan(probs) as plan:
        sin, ref, en_ref = device_buffers(plan, probs)
        plan.run(sin, ref, en_ref, mode="persistent")
        out = torch.empty_like(ref)
        en = torch.empty_like(en_ref)
        for _ in range(3):  # capture, then two replays
            out.zero_()
            st = plan.run(sin, out, en, mode="graph")
            assert torch.equal(out, ref) and torch.equal(en, en_ref)
            assert st["attempts"] == plan.attempts and st["launches"] >= 1
        out2 = torch.empty_like(ref)  # new buffers: captured again
        plan.run(sin, out2, en, mode="graph")
        assert torch.equal(out2, ref)


def test_set_weights_equals_fresh_plan():
    probs = mixed_batch(seed=37)[:6]
    probs.append(workloads.dense_ising(n=50, reads=12, sweeps=40, seed=6))  # dense updates
    rng = np.random.default_rng(5)
    new = copy.deepcopy(probs)
    for k in (1, 4, 6):
        new[k].h = rng.normal(0, 0.3, new[k].n)
        new[k].J = rng.normal(0, 1.0, new[k].J.shape[0])
    with Plan(probs) as plan, Plan(new) as fresh:
        sin, out, en = device_buffers(plan, probs)
        plan.run(sin, out, en, mode="graph")  # a captured graph survives the update
        for k in (1, 4, 6):
            plan.set_weights(k, new[k].h, new[k].J)
        plan.run(sin, out, en, mode="graph")
        _, out_f, en_f = device_buffers(fresh, new)
        fresh.run(sin, out_f, en_f)
        assert torch.equal(out, out_f) and torch.equal(en, en_f)
        p = new[1]
        ws, we = oracle.run(p.h, p.u, p.v, p.J, p.states, p.sweeps_per_beta, p.betas, p.seeds)
        o = int(plan.state_offsets[1])
        got = out[o:o + p.num_reads * p.n].cpu().numpy().reshape(p.num_reads, p.n)
        np.testing.assert_array_equal(got, ws)
        r = int(plan.read_offsets[1])
        np.testing.assert_array_equal(bits(en[r:r + p.num_reads].cpu().numpy()), bits(we))
    with Plan(probs) as plan:
        with pytest.raises(ValueError):
            plan.set_weights(len(probs), probs[0].h, probs[0].J)


def test_set_weights_device_equals_fresh_plan():
    """All problems' weights replaced from device tensors in one kernel,
    including problems with in-window resolution (dense; their back-neighbour
    couplings are copies of adjacency entries) and a captured graph."""
    probs = mixed_batch(seed=43)[:5]
    probs.append(workloads.dense_ising(n=60, reads=24, sweeps=30, seed=9))
    rng = np.random.default_rng(8)
    new = copy.deepcopy(probs)
    for p in new:
        p.h = rng.normal(0, 0.3, p.n)
        p.J = rng.normal(0, 1.0, p.J.shape[0])
    with Plan(probs) as plan, Plan(new) as fresh:
        sin, out, en = device_buffers(plan, probs)
        plan.run(sin, out, en, mode="graph")
        h_cat = torch.from_numpy(np.concatenate([p.h for p in new])).cuda()
        J_cat = torch.from_numpy(np.concatenate([p.J for p in new])).cuda()
        stream = torch.cuda.current_stream()
        for _ in range(2):  # the first call builds the scatter map, the second reuses it
            plan.set_weights_device(h_cat, J_cat, stream=stream)
            plan.run(sin, out, en, mode="graph", stream=stream)
        _, out_f, en_f = device_buffers(fresh, new)
        fresh.run(sin, out_f, en_f)
        assert torch.equal(out, out_f) and torch.equal(en, en_f)
        p = new[-1]
        ws, we = oracle.run(p.h, p.u, p.v, p.J, p.states, p.sweeps_per_beta, p.betas, p.seeds)
        o = int(plan.state_offsets[-2])
        got = out[o:o + p.num_reads * p.n].cpu().numpy().reshape(p.num_reads, p.n)
        np.testing.assert_array_equal(got, ws)


def test_autotune_keeps_results_and_caches(tmp_path):
    probs = mixed_batch(seed=41)
    cache = str(tmp_path / "tune.txt")
    with Plan(probs) as plan:
        sin, ref, en_ref = device_buffers(plan, probs)
        plan.run(sin, ref, en_ref)
        rep = plan.autotune(cache, force=True)
        assert rep and all(e["candidates"] >= 1 and e["from_cache"] == 0 for e in rep)
        assert all(e["warps_per_cta"] >= 1 and e["attempts_per_s"] > 0 for e in rep)
        assert all(e["registers"] in (64, 80, 128) for e in rep)
        assert sum(e["items"] for e in rep) == plan.total_reads
        out = torch.empty_like(ref)
        en = torch.empty_like(en_ref)
        for mode in ("persistent", "graph"):
            out.zero_()
            plan.run(sin, out, en, mode=mode)
            assert torch.equal(out, ref) and torch.equal(en, en_ref)
    lines = open(cache).read().splitlines()
    assert len(lines) >= 1 and all(len(x.split()) == 6 for x in lines)
    with Plan(probs) as plan:
        rep2 = plan.autotune(cache)
        assert all(e["from_cache"] == 1 and e["candidates"] == 0 for e in rep2)
        sin, out, en = device_buffers(plan, probs)
        plan.run(sin, out, en)
        assert torch.equal(out, ref)


def test_concurrent_global_buckets_do_not_share_slots():
    """Two problems above the on-chip size with different kernels run as two
    concurrent bucket launches; each must use its own global slots."""
    rng = np.random.default_rng(43)
    probs = []
    for k, crit in enumerate(("Metropolis", "Gibbs", "Metropolis")):
        n, u, v = random_regular(9000, 3 + k, rng, graph_seed=50 + k)
        probs.append(Instance(rng.normal(0, 0.1, n), u, v, rng.normal(0, 1, u.shape[0]),
                              random_states(rng, 6, n), np.geomspace(0.1, 5.0, 6), 1,
                              np.arange(6, dtype=np.uint64) + 7 * k, proposal=crit,
                              randomize_order=(k == 2)))
    with Plan(probs) as plan:
        sin, a, ea = device_buffers(plan, probs)
        plan.run(sin, a, ea, mode="persistent")
        b = torch.empty_like(a)
        eb = torch.empty_like(ea)
        plan.run(sin, b, eb, mode="plain")
        assert torch.equal(a, b) and torch.equal(ea, eb)
        for k in (0, 1):
            p = probs[k]
            ws, we = oracle.run(p.h, p.u, p.v, p.J, p.states, 1, p.betas, p.seeds,
                                False, p.proposal == "Gibbs")
            o = int(plan.state_offsets[k])
            got = a[o:o + p.num_reads * p.n].cpu().numpy().reshape(p.num_reads, p.n)
            np.testing.assert_array_equal(got, ws)


def test_batch_with_other_spin_values_matches_oracle():
    """Initial spins other than +-1 (the reference's int8 arithmetic is
    defined for them) mixed with ordinary reads in one batch, in every mode,
    against the oracle."""
    rng = np.random.default_rng(47)
    probs = []
    for k, crit in enumerate(("Metropolis", "Gibbs")):
        n, u, v = random_regular(300 + 50 * k, 5, rng, graph_seed=60 + k)
        st = random_states(rng, 10, n)
        st[1, 7] = 2
        st[4, :5] = [0, -3, 5, 127, -128]
        probs.append(Instance(rng.normal(0, 0.1, n), u, v, rng.normal(0, 1, u.shape[0]), st,
                              np.geomspace(0.1, 3.0, 20), 2, np.arange(10, dtype=np.uint64) + 3,
                              proposal=crit))
    with Plan(probs) as plan:
        sin, ref, en_ref = device_buffers(plan, probs)
        plan.run(sin, ref, en_ref, mode="persistent")
        for k, p in enumerate(probs):
            ws, we = oracle.run(p.h, p.u, p.v, p.J, p.states, p.sweeps_per_beta, p.betas,
                                p.seeds, False, p.proposal == "Gibbs")
            o = int(plan.state_offsets[k])
            got = ref[o:o + p.num_reads * p.n].cpu().numpy().reshape(p.num_reads, p.n)
            np.testing.assert_array_equal(got, ws)
            r = int(plan.read_offsets[k])
            np.testing.assert_array_equal(bits(en_ref[r:r + p.num_reads].cpu().numpy()),
                                          bits(we))
        for mode in ("plain", "graph"):
            out = torch.empty_like(ref)
            en = torch.empty_like(en_ref)
            st = plan.run(sin, out, en, mode=mode)
            assert torch.equal(out, ref) and torch.equal(en, en_ref), mode
            assert st["reads"] == plan.total_reads


def test_every_configuration_gives_identical_results(tmp_path):
    """Each state location (global slot, shared memory, spins shared with
    energies global) and register budget, forced through the tuning cache,
    reproduces the untuned run byte for byte."""
    probs = workloads.uneven_batch(num_problems=6, n_range=(100, 2500), reads_range=(20, 60),
                                   sweeps_range=(10, 40), seed=53)
    probs.append(workloads.complete_graph(reads=40, sweeps=20, seed=53))  # Gibbs
    cache = tmp_path / "tune.txt"
    with Plan(probs) as plan:
        sin, ref, en_ref = device_buffers(plan, probs)
        plan.run(sin, ref, en_ref)
        plan.autotune(str(cache), force=True)
    keys = [line.split()[0] for line in cache.read_text().splitlines()]
    assert keys
    for staging in (0, 1, 2):
        for regs in (0, 1, 2):
            cache.write_text("".join(f"{k} {staging} 1 0 {regs} 1.0\n" for k in keys))
            with Plan(probs) as plan:
                rep = plan.autotune(str(cache))
                assert all(e["from_cache"] == 1 for e in rep)
                for mode in ("persistent", "plain_tuned"):
                    out = torch.empty_like(ref)
                    en = torch.empty_like(en_ref)
                    plan.run(sin, out, en, mode=mode)
                    assert torch.equal(out, ref) and torch.equal(en, en_ref), (staging, regs, mode)


def test_bucket_report_matches_run_counters():
    """Per-bucket figures of a persistent run and of a graph replay add up to
    the run's counters, and each bucket launch has a device time."""
    probs = workloads.uneven_batch(num_problems=10, n_range=(64, 3000), reads_range=(8, 40),
                                   sweeps_range=(10, 30), seed=61)
    with Plan(probs) as plan:
        sin, out, en = device_buffers(plan, probs)
        for mode in ("persistent", "graph"):
            st = plan.run(sin, out, en, mode=mode)
            rep = plan.bucket_report()
            assert rep and sum(r["reads"] for r in rep) == plan.total_reads
            assert sum(r["attempts"] for r in rep) == st["attempts"]
            assert sum(r["flips"] for r in rep) == st["flips"]
            assert sum(r["passes"] for r in rep) == st["passes"]
            assert all(r["ms"] > 0 and r["model_bytes"] > 0 and r["grid"] > 0 for r in rep), rep


def test_sharded_batch_on_two_host_threads_equals_one_call():
    """b200sa.shards on one GPU driven as two devices (two host threads, two
    plans at once): the gathered result equals one batched call."""
    from b200sa import shards
    probs = mixed_batch(seed=47)
    a, b = copy.deepcopy(probs), copy.deepcopy(probs)
    ea = sample_batch(a, mode="persistent")
    eb = shards.sample_batch_devices(b, devices=[0, 0])
    for pa, pb, xa, xb in zip(a, b, ea, eb):
        np.testing.assert_array_equal(pa.states, pb.states)
        np.testing.assert_array_equal(bits(xa), bits(xb))


def test_band_location_in_every_register_budget(tmp_path):
    """A banded problem run with the band location forced through the tuning
    cache, in each register budget, reproduces the untuned run; problems that
    are not banded fall back to another location."""
    rng = np.random.default_rng(3)
    n = 10000
    u = rng.integers(0, n - 1, 3 * n)
    v = np.minimum(u + rng.integers(1, 50, u.shape[0]), n - 1)
    keep = u != v
    u, v = np.minimum(u[keep], v[keep]).astype(np.int32), np.maximum(u[keep], v[keep]).astype(np.int32)
    band = Instance(rng.normal(0, 0.1, n), u, v, rng.normal(0, 1, u.shape[0]),
                    random_states(rng, 12, n), np.geomspace(0.1, 3.0, 6), 1,
                    np.arange(12, dtype=np.uint64) + 5)
    probs = [band] + mixed_batch(seed=59)[:3]
    cache = tmp_path / "tune.txt"
    with Plan(probs) as plan:
        sin, ref, en_ref = device_buffers(plan, probs)
        plan.run(sin, ref, en_ref, mode="plain")
        plan.autotune(str(cache), force=True)
        out = torch.empty_like(ref)
        en = torch.empty_like(en_ref)
        plan.run(sin, out, en)
        assert torch.equal(out, ref) and torch.equal(en, en_ref)
    keys = [line.split()[0] for line in cache.read_text().splitlines()]
    for regs in (0, 1, 2):
        cache.write_text("".join(f"{k} 3 2 0 {regs} 1.0\n" for k in keys))
        with Plan(probs) as plan:
            plan.autotune(str(cache))
            for mode in ("persistent", "plain_tuned"):
                out = torch.empty_like(ref)
                en = torch.empty_like(en_ref)
                plan.run(sin, out, en, mode=mode)
                assert torch.equal(out, ref) and torch.equal(en, en_ref), (regs, mode)
            rep = plan.bucket_report()
            assert any(r["staging"] == 3 for r in rep)
