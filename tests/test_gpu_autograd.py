"""Differentiable sampling: the backward of LogPartition against exact log Z
by enumeration (n = 16), against the same gradient computed with NumPy from
the CPU oracle's samples (bit-identical samples => identical gradient), the
recompute-from-seed path, and batched Boltzmann-machine learning."""
import itertools

import numpy as np
import pytest
import torch

import oracle
from b200sa import workloads
from b200sa.autograd import (IsingModel, SamplingSpec, edge_moments, initial_states,
                             log_partition, read_seeds, sample_models)

pytestmark = pytest.mark.gpu


def exact_logz_and_grad(h, u, v, J, beta):
    """log Z, d logZ/dh, d logZ/dJ by enumerating all 2^n states (float64)."""
    n = len(h)
    s = np.array(list(itertools.product([-1, 1], repeat=n)), dtype=np.float64)
    E = s @ h + (s[:, u] * s[:, v]) @ J
    a = -beta * E
    amax = a.max()
    w = np.exp(a - amax)
    Z = w.sum()
    p = w / Z
    logz = amax + np.log(Z)
    gh = -beta * (p @ s)
    gJ = -beta * (p @ (s[:, u] * s[:, v]))
    return logz, gh, gJ


def k16(seed=4):
    inst = workloads.complete_graph(reads=8, sweeps=1, seed=seed)
    return inst.h, inst.u, inst.v, inst.J


def test_enumeration_gradient_matches_central_differences():
    h, u, v, J = k16()
    beta = 1.0
    _, gh, gJ = exact_logz_and_grad(h, u, v, J, beta)
    eps = 1e-4
    for i in (0, 5, 15):
        hp, hm = h.copy(), h.copy()
        hp[i] += eps
        hm[i] -= eps
        fd = (exact_logz_and_grad(hp, u, v, J, beta)[0] - exact_logz_and_grad(hm, u, v, J, beta)[0]) / (2 * eps)
        assert abs(fd - gh[i]) < 1e-7
    for c in (0, 40, 119):
        Jp, Jm = J.copy(), J.copy()
        Jp[c] += eps
        Jm[c] -= eps
        fd = (exact_logz_and_grad(h, u, v, Jp, beta)[0] - exact_logz_and_grad(h, u, v, Jm, beta)[0]) / (2 * eps)
        assert abs(fd - gJ[c]) < 1e-7


def test_sampled_gradient_within_4_standard_errors_of_exact():
    """K16, J~N(0,0.3), h~N(0,0.1), beta=1, Gibbs, 10000 sweeps, 4096 reads."""
    h, u, v, J = k16()
    beta, reads = 1.0, 4096
    model = IsingModel(16, u, v)
    spec = SamplingSpec([model], beta=beta, sweeps=10000, reads=reads, seed=3, init_seed=5)
    hh = torch.tensor(h, dtype=torch.float64, requires_grad=True)
    JJ = torch.tensor(J, dtype=torch.float64, requires_grad=True)
    log_partition(hh, JJ, spec).backward()
    _, gh, gJ = exact_logz_and_grad(h, u, v, J, beta)
    s = spec.last_samples[0].cpu().numpy().astype(np.float64)
    se_h = beta * s.std(axis=0, ddof=1) / np.sqrt(reads)
    ss = s[:, u] * s[:, v]
    se_J = beta * ss.std(axis=0, ddof=1) / np.sqrt(reads)
    zh = np.abs(hh.grad.numpy() - gh) / se_h
    zJ = np.abs(JJ.grad.numpy() - gJ) / se_J
    assert zh.max() < 4.0 and zJ.max() < 4.0, (zh.max(), zJ.max())
    # central differences of the exact log Z agree with the same expectations
    eps = 1e-4
    hp, hm = h.copy(), h.copy()
    hp[3] += eps
    hm[3] -= eps
    fd = (exact_logz_and_grad(hp, u, v, J, beta)[0] - exact_logz_and_grad(hm, u, v, J, beta)[0]) / (2 * eps)
    assert abs(hh.grad.numpy()[3] - fd) < 4.0 * se_h[3]


def test_gradient_equals_numpy_gradient_from_oracle_samples():
    """The oracle (reference algorithm on the CPU) run with the same seeds and
    initial states gives the same samples, hence exactly the same gradient."""
    h, u, v, J = k16(seed=9)
    beta, reads, sweeps = 1.0, 256, 2000
    model = IsingModel(16, u, v)
    spec = SamplingSpec([model], beta=beta, sweeps=sweeps, reads=reads, seed=21, init_seed=8)
    hh = torch.tensor(h, dtype=torch.float64, requires_grad=True)
    JJ = torch.tensor(J, dtype=torch.float64, requires_grad=True)
    log_partition(hh, JJ, spec).backward()
    init = initial_states(8, 0, reads, 16)
    seeds = read_seeds(21, 0, reads)
    st, _ = oracle.run(h, u, v, J, init, sweeps, [beta], seeds, False, True)
    s = st.astype(np.int64)
    np.testing.assert_array_equal(spec.last_samples[0].cpu().numpy(), st)
    np.testing.assert_array_equal(hh.grad.numpy(), -beta * (s.sum(axis=0) / reads))
    np.testing.assert_array_equal(JJ.grad.numpy(), -beta * ((s[:, u] * s[:, v]).sum(axis=0) / reads))


def test_recompute_from_seed_gives_identical_gradients():
    rng = np.random.default_rng(2)
    models, hs, Js = [], [], []
    for k, n in enumerate((40, 64, 90)):
        n, u, v = workloads.random_regular(n, 3 + k, rng, graph_seed=k + 1)
        models.append(IsingModel(n, u, v))
        hs.append(rng.normal(0, 0.1, n))
        Js.append(rng.normal(0, 0.5, u.shape[0]))
    h_cat = np.concatenate(hs)
    J_cat = np.concatenate(Js)
    grads = []
    for budget in (1 << 30, 0):  # keep samples / recompute them in chunks
        spec = SamplingSpec(models, beta=0.8, sweeps=300, reads=200, seed=4, init_seed=6,
                            memory_budget=budget, recompute_chunk=64)
        hh = torch.tensor(h_cat, requires_grad=True)
        JJ = torch.tensor(J_cat, requires_grad=True)
        log_partition(hh, JJ, spec).backward()
        assert (len(spec.last_samples) > 0) == (budget > 0)
        grads.append((hh.grad.numpy().copy(), JJ.grad.numpy().copy()))
    np.testing.assert_array_equal(grads[0][0], grads[1][0])
    np.testing.assert_array_equal(grads[0][1], grads[1][1])


def test_batched_moments_match_numpy():
    rng = np.random.default_rng(3)
    models, samples = [], []
    for n, m in ((30, 50), (200, 700), (1000, 9000)):
        u = rng.integers(0, n, m).astype(np.int32)
        v = rng.integers(0, n, m).astype(np.int32)
        models.append(IsingModel(n, u, v))
        samples.append(torch.from_numpy((2 * rng.integers(0, 2, (130, n)) - 1).astype(np.int8)).cuda())
    s_sum, ss_sum = edge_moments(models, samples)
    for mod, st, a, b in zip(models, samples, s_sum, ss_sum):
        x = st.cpu().numpy().astype(np.int64)
        np.testing.assert_array_equal(a.cpu().numpy(), x.sum(axis=0))
        np.testing.assert_array_equal(b.cpu().numpy(), (x[:, mod.u] * x[:, mod.v]).sum(axis=0))


def test_batched_boltzmann_machine_learning_reduces_correlation_error():
    from b200sa import bm
    truth = workloads.bm_models(num_models=3, n_range=(40, 64), d=3, J_sigma=0.5, seed=7)
    res = bm.fit(truth, beta=1.0, steps=40, reads=512, sweeps=200, lr=0.05, target_reads=2048,
                 target_sweeps=300, seed=3)
    assert res.corr_error[-1] < 0.5 * res.corr_error[0], res.corr_error[::8]
    assert res.steps_per_second > 0


@pytest.mark.parametrize("init_seed, model, read0, reads, n", [
    (8, 0, 0, 256, 16), (1, 3, 77, 5, 1), (2**40 + 5, 63, 1000, 33, 17), (0, 0, 0, 300, 2048)])
def test_device_initial_states_match_host(init_seed, model, read0, reads, n):
    from b200sa.autograd import device_initial_states
    out = torch.empty(reads * n, dtype=torch.int8, device="cuda")
    device_initial_states(out, init_seed, model, read0, reads, n)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(out.cpu().numpy().reshape(reads, n),
                                  initial_states(init_seed, model, reads, n, read0))


def _two_models():
    rng = np.random.default_rng(8)
    models, hs, Js = [], [], []
    for k, n in enumerate((40, 70)):
        n, u, v = workloads.random_regular(n, 3 + k, rng, graph_seed=k + 11)
        models.append(IsingModel(n, u, v))
        hs.append(rng.normal(0, 0.1, n))
        Js.append(rng.normal(0, 0.5, u.shape[0]))
    return models, np.concatenate(hs), np.concatenate(Js)


def _grads(reads, budget, group=None):
    models, h_cat, J_cat = _two_models()
    spec = SamplingSpec(models, beta=0.9, sweeps=80, reads=reads, seed=9, init_seed=10,
                        memory_budget=budget, recompute_chunk=16, group=group)
    hh = torch.tensor(h_cat, requires_grad=True)
    JJ = torch.tensor(J_cat, requires_grad=True)
    log_partition(hh, JJ, spec).backward()
    return hh.grad.numpy().tolist(), JJ.grad.numpy().tolist()


def _pooled_rank(rank, world, port, out):
    import os
    import sys
    from datetime import timedelta
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    from conftest import ROOT
    for p in (ROOT, os.path.join(ROOT, "dwave-samplers_b200")):
        if p not in sys.path:
            sys.path.insert(0, p)
    import torch.distributed as dist
    dist.init_process_group("gloo", rank=rank, world_size=world, timeout=timedelta(seconds=120))
    out[rank] = [_grads(24, budget, dist.group.WORLD) for budget in (1 << 30, 0)]
    dist.barrier()
    dist.destroy_process_group()


def test_moments_pooled_over_two_ranks_equal_one_rank_with_all_reads():
    """Two ranks (processes on one GPU, gloo between them) each sample 24
    reads of every model (reads [24 k, 24 k + 24) of the pooled set) and pool
    the moment sums in backward: both hold exactly the gradient of one
    process sampling all 48 reads, with the samples kept or recomputed."""
    import socket
    import torch.multiprocessing as mp
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        port = s.getsockname()[1]
    want = _grads(48, 1 << 30)
    mgr = mp.Manager()
    out = mgr.dict()
    mp.spawn(_pooled_rank, args=(2, port, out), nprocs=2, join=True)
    for r in range(2):
        for got in out[r]:
            assert [list(x) for x in got] == [list(x) for x in want]
