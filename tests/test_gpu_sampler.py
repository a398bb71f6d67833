"""SimulatedAnnealingSampler on the GPU: the reference's sampler-level tests
restated without dimod (tests/test_simulated_annealing_sampler.py)."""
import numpy as np
import pytest

from b200sa.sampler import Neal, SimulatedAnnealingSampler

pytestmark = pytest.mark.gpu


def test_ground_state_ferromagnet_and_timing():
    h = {i: -1.0 for i in range(12)}
    J = {(i, j): -1.0 for i in range(12) for j in range(i + 1, 12)}
    ss = SimulatedAnnealingSampler().sample_ising(h, J, num_reads=20, seed=3)
    assert len(ss) == 20
    assert ss.first.energy == pytest.approx(-12 - 66)
    assert ss.first.sample == {i: 1 for i in range(12)}
    for k in ("preprocessing_ns", "sampling_ns", "postprocessing_ns"):
        assert ss.info["timing"][k] > 0
    assert "beta_range" in ss.info and ss.info["beta_schedule_type"] == "geometric"
    # No read decided an exp() comparison inside the cross-libm tie band.
    assert ss.info["near_ties"] == 0 and ss.info["near_tie_reads"] == []
    assert Neal is SimulatedAnnealingSampler


def test_qubo_sampling_energies_and_values():
    Q = {(0, 0): -1.0, (1, 1): -1.0, (0, 1): 2.0, (1, 2): -0.5, (2, 2): 0.3}
    ss = SimulatedAnnealingSampler().sample_qubo(Q, num_reads=30, seed=9)
    for row, e in zip(ss.record.sample, ss.record.energy):
        x = dict(zip(ss.variables, row.tolist()))
        assert set(x.values()) <= {0, 1}
        assert e == pytest.approx(sum(w * x[a] * x[b] for (a, b), w in Q.items()))
    assert ss.first.energy == pytest.approx(-1.2)


def test_seed_determinism_and_num_sweeps_zero():
    h = {i: float(np.sin(i)) for i in range(30)}
    J = {(i, (i * 7 + 3) % 30): 0.5 for i in range(30) if i != (i * 7 + 3) % 30}
    s = SimulatedAnnealingSampler()
    a = s.sample_ising(h, J, num_reads=10, seed=42).record.sample
    b = s.sample_ising(h, J, num_reads=10, seed=42).record.sample
    assert np.array_equal(a, b)
    init = np.ones((4, 30), dtype=np.int8)
    ss = s.sample_ising(h, J, num_sweeps=0, initial_states=init, seed=1)
    assert np.array_equal(ss.record.sample, init)


def test_metropolis_ergodicity_breaking_null_model():
    # tests/test_simulated_annealing_sampler.py:678-700
    n = 100
    init = 1 - 2 * np.random.randint(2, size=n)
    for num_sweeps in range(3):
        ss = SimulatedAnnealingSampler().sample_ising(
            {i: 0.0 for i in range(n)}, {}, initial_states=[init], num_reads=1,
            num_sweeps=num_sweeps, beta_range=[0.1, 1])
        assert np.all(ss.record.sample == (-1) ** num_sweeps * init)


def interval(p, num, k=3):
    mu = num * p
    sig = np.sqrt(num * p * (1 - p))
    return mu - k * sig, mu + k * sig


def test_central_limits_random_updates():
    # tests/test_simulated_annealing_sampler.py:702-788, seed 2023
    n, seed = 10000, 2023
    up = np.ones((1, n), dtype=np.int8)
    s = SimulatedAnnealingSampler()
    zero = {i: 0.0 for i in range(n)}
    cases = [
        (0.5, dict(proposal_acceptance_criteria="Gibbs")),
        (np.cosh(1) * np.exp(-1), dict(randomize_order=True)),
        (1 / np.exp(1) + (1 - 1 / np.exp(1)) * 0.5,
         dict(randomize_order=True, proposal_acceptance_criteria="Gibbs")),
    ]
    for p, kw in cases:
        lo, hi = interval(p, n)
        ss = s.sample_ising(zero, {}, initial_states=up, num_reads=1, seed=seed, num_sweeps=1,
                            beta_range=[0.1, 1], **kw)
        stat = np.sum(ss.record.sample == 1)
        assert lo < stat < hi, (kw, stat, lo, hi)
    p = np.exp(-1.5) / (2 * np.cosh(1.5))
    lo, hi = interval(p, n)
    ss = s.sample_ising({i: 1.0 for i in range(n)}, {}, initial_states=up, num_reads=1,
                        seed=seed, proposal_acceptance_criteria="Gibbs",
                        beta_schedule_type="custom", beta_schedule=[1, 1.5], num_sweeps_per_beta=1)
    stat = np.sum(ss.record.sample == 1)
    assert lo < stat < hi


def test_greedy_limit_independent_spins():
    # tests/test_simulated_annealing_sampler.py:790-845
    n = 10000
    hv = np.random.default_rng(0).normal(size=n)
    h = {i: float(hv[i]) for i in range(n)}
    ground = np.array([-int(np.sign(hv[i])) for i in range(n)])
    lo, hi = interval(1 - np.exp(-1), n)
    s = SimulatedAnnealingSampler()
    for randomize_order in (False, True):
        for crit in ("Metropolis", "Gibbs"):
            kw = dict(num_reads=1, num_sweeps=1, randomize_order=randomize_order,
                      proposal_acceptance_criteria=crit, beta_schedule_type="custom",
                      beta_schedule=[float("inf")], seed=2023)
            ss = s.sample_ising(h, {}, initial_states=[ground], **kw)
            assert np.all(ss.record.sample == ground)
            ss = s.sample_ising(h, {}, initial_states=[-ground], **kw)
            if not randomize_order:
                assert np.all(ss.record.sample == ground)
            else:
                stat = np.sum(ss.record.sample == ground)
                assert lo < stat < hi


def test_interrupt_function_exception_stops_after_one_read():
    def boom():
        raise RuntimeError("stop")
    ss = SimulatedAnnealingSampler().sample_ising({0: 1.0, 1: -1.0}, {(0, 1): 0.5},
                                                  num_reads=10, interrupt_function=boom, seed=1)
    assert len(ss) == 1
