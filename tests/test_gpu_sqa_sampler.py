"""SQA sampler front ends on the GPU: each result equals a direct call of the
binding with the same schedule, states and seed; info keys and vartypes follow
the reference samplers."""
import numpy as np
import pytest

from b200sa.sampler import SimulatedAnnealingSampler, _IsingProblem
from b200sa.sqa import path_annealing, simulated_annealing as rotor_annealing
from b200sa.sqa_sampler import PathIntegralAnnealingSampler, RotorModelAnnealingSampler
from conftest import bits

pytestmark = pytest.mark.gpu


def frustrated(n=12, seed=3):
    rng = np.random.default_rng(seed)
    h = {i: float(rng.normal(0, 0.3)) for i in range(n)}
    J = {(i, j): float(rng.normal(0, 1)) for i in range(n) for j in range(i + 1, n)
         if rng.random() < 0.3}
    return h, J


def classical_energy(sample, h, J, variables):
    idx = {x: k for k, x in enumerate(variables)}
    e = sum(h[x] * sample[idx[x]] for x in h)
    return e + sum(w * sample[idx[a]] * sample[idx[b]] for (a, b), w in J.items())


def test_path_integral_equals_binding_and_reports_breaks():
    h, J = frustrated()
    s = PathIntegralAnnealingSampler()
    ss = s.sample_ising(h, J, num_reads=16, num_sweeps=20, beta_range=[0.2, 3.0], seed=11,
                        Hd_field=np.linspace(3.0, 0.5, 20), project_states=(True, False),
                        schedule_sample_interval=5)
    p = _IsingProblem(h, J, 0.0, "SPIN")
    init = SimulatedAnnealingSampler._initial_states(p, 16, None, "random", 11)
    nb = np.zeros(init.shape, np.intc)
    bo = np.zeros(10000, np.intc)
    w = path_annealing(16, p.h, p.u, p.v, p.J, 1, np.geomspace(0.2, 3.0, 20),
                       np.linspace(3.0, 0.5, 20), 1.0, 1.0, 1, 1, 11, init.copy(), True, False,
                       nb, np.zeros(1, np.intc), bo, 5)
    np.testing.assert_array_equal(ss.record.sample, w[0])
    np.testing.assert_array_equal(bits(ss.record.energy), bits(w[1]))
    for row, e in zip(ss.record.sample, ss.record.energy):
        assert e == pytest.approx(classical_energy(row, h, J, ss.variables))
    total = int(ss.info["num_breaks"].sum())
    assert ss.info["complete_break_specification"] and len(ss.info["break_positions"]) == total
    np.testing.assert_array_equal(ss.info["break_positions"], w[4][:total])
    assert ss.info["statistics"].shape == (16, 4, 12)


def test_path_integral_qubo_and_ground_state():
    # Ferromagnetic ring of 8: ground states all-equal, energy -8.
    J = {(i, (i + 1) % 8): -1.0 for i in range(8)}
    ss = PathIntegralAnnealingSampler().sample_ising(
        {i: 0.0 for i in range(8)}, J, num_reads=32, num_sweeps=200, beta_range=[0.1, 5.0],
        Hd_field=np.geomspace(2.0, 0.01, 200), seed=5)
    assert ss.record.energy.min() == -8.0
    Q = {(0, 0): -1.0, (1, 1): -1.0, (0, 1): 2.0}
    sq = PathIntegralAnnealingSampler().sample_qubo(Q, num_reads=8, num_sweeps=50, seed=2)
    assert set(np.unique(sq.record.sample)) <= {0, 1}
    for row, e in zip(sq.record.sample, sq.record.energy):
        x = dict(zip(sq.variables, row))
        assert e == pytest.approx(sum(w * x[a] * x[b] for (a, b), w in Q.items()))


def test_rotor_equals_binding_with_projection():
    h, J = frustrated(10, 4)
    s = RotorModelAnnealingSampler()
    ss = s.sample_ising(h, J, num_reads=12, num_sweeps=30, beta_range=[0.2, 4.0], seed=21,
                        Hd_field=np.linspace(2.0, 0.1, 30), project_states=(False, False),
                        schedule_sample_interval=10, trans_fields=0.7)
    p = _IsingProblem(h, J, 0.0, "SPIN")
    init = SimulatedAnnealingSampler._initial_states(p, 12, None, "random", 21)
    angles = np.ascontiguousarray(64 - 64 * init, dtype=np.uint8)
    a, e, st = rotor_annealing(12, p.h, p.u, p.v, p.J, 0.7 * np.ones(10), 1,
                               np.geomspace(0.2, 4.0, 30), np.linspace(2.0, 0.1, 30), 21, angles,
                               False, "MetropolisUniform", 10)
    np.testing.assert_array_equal(ss.info["rotor_states"], a)
    np.testing.assert_array_equal(bits(ss.record.energy), bits(e))
    np.testing.assert_array_equal(ss.info["statistics"], st)
    prng = np.random.default_rng(21)
    spins = np.array(1 - 2 * (np.cos(np.pi * a / 128) < 1 - 2 * prng.random(size=a.shape)),
                     dtype=np.int8)
    np.testing.assert_array_equal(ss.record.sample, spins)


def test_rotor_angle_initial_states_and_zero_sweeps():
    s = RotorModelAnnealingSampler()
    init = np.array([[0, 64, 128], [200, 10, 90]], dtype=np.uint8)
    ss = s.sample_ising({0: 0.1, 1: -0.2, 2: 0.0}, {(0, 1): 1.0, (1, 2): -0.5},
                        initial_states=init, num_sweeps=0, seed=9,
                        project_states=(False, False))
    np.testing.assert_array_equal(ss.info["rotor_states"], init)  # nothing to anneal
    assert ss.info["beta_range"] is None
