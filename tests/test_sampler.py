"""SimulatedAnnealingSampler front end: argument handling, beta schedules,
default beta range and QUBO conversion (no GPU needed)."""
import warnings

import numpy as np
import pytest

from b200sa.sampler import (SimulatedAnnealingSampler, _IsingProblem, build_schedule,
                            ising_beta_range)


def problem(h, J):
    return _IsingProblem(h, J, 0.0, "SPIN")


def test_parameters_and_properties():
    s = SimulatedAnnealingSampler()
    assert sorted(s.parameters) == sorted([
        'beta_range', 'beta_schedule', 'beta_schedule_type', 'initial_states',
        'initial_states_generator', 'interrupt_function', 'num_reads', 'num_sweeps',
        'num_sweeps_per_beta', 'proposal_acceptance_criteria', 'randomize_order', 'seed'])
    assert s.properties['beta_schedule_options'] == ('linear', 'geometric', 'custom')


def test_schedules():
    p = problem({0: 1.0, 1: -1.0}, {(0, 1): 0.5})
    br, sch = build_schedule(p, [0.1, 2.0], 10, 1, "geometric", None)
    np.testing.assert_array_equal(sch, np.geomspace(0.1, 2.0, 10))
    br, sch = build_schedule(p, [0.1, 2.0], 10, 2, "linear", None)
    np.testing.assert_array_equal(sch, np.linspace(0.1, 2.0, 5))
    br, sch = build_schedule(p, [0.1, 2.0], 1, 1, "geometric", None)
    np.testing.assert_array_equal(sch, [2.0])  # one beta: the target value
    br, sch = build_schedule(p, None, None, 1, "geometric", None)
    assert len(sch) == 1000 and sch[0] == pytest.approx(br[0]) and sch[-1] == pytest.approx(br[1])
    br, sch = build_schedule(p, None, 0, 1, "geometric", None)
    assert len(sch) == 0
    br, sch = build_schedule(p, None, None, 3, "custom", [0.5, 1.0])
    np.testing.assert_array_equal(sch, [0.5, 1.0])


@pytest.mark.parametrize("kwargs, err", [
    (dict(beta_schedule_type="custom"), "must be provided"),
    (dict(beta_schedule_type="custom", beta_schedule=[1, 2], num_sweeps=3), "consistent"),
    (dict(beta_schedule_type="custom", beta_schedule=[1, 2], beta_range=[0.5, 2]), "consistent"),
    (dict(beta_schedule_type="custom", beta_schedule=[-1, 2]), "negative"),
    (dict(beta_schedule=[1, 2]), "must be set to None"),
    (dict(num_sweeps=10, num_sweeps_per_beta=3), "divisible"),
    (dict(beta_range=[1, 2, 3]), "2-tuple"),
    (dict(beta_range=[-1, 2]), "2-tuple"),
    (dict(beta_range=[0, 2]), "non-zero"),
    (dict(beta_schedule_type="cubic"), "not implemented"),
])
def test_schedule_errors(kwargs, err):
    p = problem({0: 1.0}, {})
    args = dict(beta_range=None, num_sweeps=None, num_sweeps_per_beta=1,
                beta_schedule_type="geometric", beta_schedule=None)
    args.update(kwargs)
    with pytest.raises(ValueError, match=err):
        build_schedule(p, args["beta_range"], args["num_sweeps"], args["num_sweeps_per_beta"],
                       args["beta_schedule_type"], args["beta_schedule"])


def test_sample_argument_errors():
    s = SimulatedAnnealingSampler()
    with pytest.raises(TypeError):
        s.sample_ising({0: 1.0}, {}, seed=1.5)
    with pytest.raises(ValueError):
        s.sample_ising({0: 1.0}, {}, seed=2**31)
    with pytest.raises(TypeError):
        s.sample_ising({0: 1.0}, {}, num_sweeps_per_beta=1.0)
    with pytest.raises(ValueError):
        s.sample_ising({0: 1.0}, {}, num_sweeps_per_beta=0)
    with pytest.raises(TypeError):
        s.sample_ising({0: 1.0}, {}, interrupt_function=3)
    with pytest.raises(ValueError):
        s.sample_ising({0: 1.0, 1: 0.0}, {}, num_reads=3, initial_states=[[1, 1]],
                       initial_states_generator="none")


def test_default_beta_range():
    # one spin with |h| = 1: hot = ln2/2, cold = ln(1/0.01)/2
    hot, cold = ising_beta_range({0: 1.0}, {})
    assert hot == pytest.approx(np.log(2) / 2)
    assert cold == pytest.approx(np.log(100) / 2)
    # chain with |J| = 1 and h = 0: max field 2 on interior spins, min gap 1 on all 3
    hot, cold = ising_beta_range({0: 0, 1: 0, 2: 0}, {(0, 1): -1, (1, 2): 1})
    assert hot == pytest.approx(np.log(2) / 4)
    assert cold == pytest.approx(np.log(3 / 0.01) / 2)
    with warnings.catch_warnings(record=True) as w:
        warnings.simplefilter("always")
        assert ising_beta_range({0: 0}, {}) == [0.1, 1]
        assert any("All bqm biases are zero" in str(x.message) for x in w)
    with pytest.raises(ValueError):
        ising_beta_range({0: 1}, {}, max_single_qubit_excitation_rate=2)


def test_qubo_to_ising_preserves_energies():
    rng = np.random.default_rng(1)
    Q = {}
    for a in range(5):
        for b in range(a, 5):
            if rng.random() < 0.7:
                Q[(a, b)] = float(rng.normal())
    linear = {a: 0.0 for a in range(5)}
    quadratic = {}
    for (a, b), w in Q.items():
        if a == b:
            linear[a] += w
        else:
            quadratic[(a, b)] = w
    p = _IsingProblem(linear, quadratic, 0.0, "BINARY")
    for bits in range(32):
        x = np.array([(bits >> k) & 1 for k in range(5)], dtype=np.float64)
        s = 2 * x - 1
        eq = sum(w * x[a] * x[b] for (a, b), w in Q.items())
        es = p.offset + s @ p.h + sum(w * s[i] * s[j] for i, j, w in zip(p.u, p.v, p.J))
        assert es == pytest.approx(eq)


def test_initial_states_generators():
    p = problem({0: 1.0, 1: 0.0, 2: -1.0}, {})
    init = SimulatedAnnealingSampler._initial_states
    given = [[1, -1, 1]]
    assert init(p, 3, given, "tile", 5).tolist() == [[1, -1, 1]] * 3
    r = init(p, 4, given, "random", 5)
    assert r.shape == (4, 3) and r[0].tolist() == [1, -1, 1] and set(np.unique(r)) <= {-1, 1}
    assert init(p, None, given, "none", 5).shape == (1, 3)
    assert init(p, 1, [[1, -1, 1], [-1, -1, -1]], "none", 5).tolist() == [[1, -1, 1]]
    assert init(p, None, {0: -1, 1: 1, 2: 1}, "random", 5).tolist() == [[-1, 1, 1]]
