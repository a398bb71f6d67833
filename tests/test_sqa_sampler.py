"""SQA sampler front ends (path-integral and rotor model): schedules, argument
handling and break-buffer sizing, the parts that need no GPU."""
import numpy as np
import pytest

from b200sa.sampler import _IsingProblem
from b200sa.sqa_sampler import (PathIntegralAnnealingSampler, RotorModelAnnealingSampler,
                                build_fields)


def problem(h, J):
    return _IsingProblem(h, J, 0.0, "SPIN")


P = problem({0: 1.0, 1: -1.0, 2: 0.0}, {(0, 1): 0.5, (1, 2): -1.0})


@pytest.mark.parametrize("cls", [PathIntegralAnnealingSampler, RotorModelAnnealingSampler])
def test_parameters_and_properties(cls):
    s = cls()
    assert sorted(s.parameters) == sorted([
        "beta_range", "beta_schedule_type", "initial_states", "initial_states_generator",
        "interrupt_function", "num_reads", "num_sweeps", "num_sweeps_per_beta", "seed"])
    assert s.properties["beta_schedule_options"] == ("linear", "geometric", "custom")


def test_fields():
    br, hp, hd = build_fields(P, [0.1, 2.0], 10, 1, "geometric", None, None)
    np.testing.assert_array_equal(hp, np.geomspace(0.1, 2.0, 10))
    np.testing.assert_array_equal(hd, np.zeros(10))
    br, hp, hd = build_fields(P, [0.1, 2.0], 10, 2, "linear", None, np.arange(5.0))
    np.testing.assert_array_equal(hp, np.linspace(0.1, 2.0, 5))
    np.testing.assert_array_equal(hd, np.arange(5.0))
    br, hp, hd = build_fields(P, [0.1, 2.0], 1, 1, "geometric", None, None)
    np.testing.assert_array_equal(hp, [2.0])
    br, hp, hd = build_fields(P, None, None, 1, "geometric", None, None)
    assert len(hp) == 100 and hp[-1] == pytest.approx(br[1])  # default num_sweeps
    br, hp, hd = build_fields(P, None, None, 4, "custom", [0.5, 1.0], [2.0, 1.0, 0.0])
    np.testing.assert_array_equal(hp, [0.5, 1.0])
    br, hp, hd = build_fields(P, None, 0, 1, "geometric", None, None, zero_sweeps_empty=True)
    assert len(hp) == 0 and len(hd) == 0 and br is None


@pytest.mark.parametrize("args, match", [
    (dict(beta_schedule_type="custom"), "must be provided"),
    (dict(beta_schedule_type="custom", Hp_field=[1.0, -1.0], num_sweeps=None,
          beta_range=None), "negative"),
    (dict(beta_schedule_type="custom", Hp_field=[1.0, 2.0], num_sweeps=3), "num_sweeps"),
    (dict(beta_schedule_type="custom", Hp_field=[1.0, 2.0], beta_range=[1.0, 3.0],
          num_sweeps=None), "beta_range"),
    (dict(Hp_field=[1.0]), "must be set to None"),
    (dict(num_sweeps=7, num_sweeps_per_beta=2), "divisible"),
    (dict(beta_range=[1.0]), "2-tuple"),
    (dict(beta_range=[0.0, 1.0]), "non-zero"),
    (dict(beta_schedule_type="cubic"), "not implemented"),
    (dict(num_sweeps=4, Hd_field=[1.0]), "Hd_field incompatible"),
])
def test_field_errors(args, match):
    kw = dict(beta_range=[0.1, 1.0], num_sweeps=4, num_sweeps_per_beta=1,
              beta_schedule_type="geometric", Hp_field=None, Hd_field=None)
    kw.update(args)
    with pytest.raises(ValueError, match=match):
        build_fields(P, kw["beta_range"], kw["num_sweeps"], kw["num_sweeps_per_beta"],
                     kw["beta_schedule_type"], kw["Hp_field"], kw["Hd_field"])


@pytest.mark.parametrize("cls", [PathIntegralAnnealingSampler, RotorModelAnnealingSampler])
@pytest.mark.parametrize("kw, error", [
    (dict(seed=-1), ValueError),
    (dict(seed=2**31), ValueError),
    (dict(seed=1.5), TypeError),
    (dict(num_sweeps_per_beta=0), ValueError),
    (dict(num_sweeps_per_beta=1.0), TypeError),
    (dict(interrupt_function=3), TypeError),
    (dict(schedule_sample_interval=0), ValueError),
    (dict(schedule_sample_interval=99, num_sweeps=4), ValueError),
    (dict(initial_states_generator="bogus"), ValueError),
])
def test_sample_argument_errors(cls, kw, error):
    with pytest.raises(error):
        cls().sample_ising({0: 0.5, 1: -0.5}, {(0, 1): 1.0}, **kw)


def test_path_integral_break_buffer_checks():
    s = PathIntegralAnnealingSampler()
    with pytest.raises(ValueError, match="inconsistent"):
        s.sample_ising({0: 0.5, 1: -0.5}, {(0, 1): 1.0}, num_reads=3,
                       num_breaks=np.zeros((2, 2), np.intc))


def test_rotor_argument_checks():
    s = RotorModelAnnealingSampler()
    with pytest.raises(ValueError, match="trans_fields"):
        s.sample_ising({0: 0.5, 1: -0.5}, {(0, 1): 1.0}, trans_fields=[1.0])
    with pytest.raises(ValueError, match="Shape of initial_states"):
        s.sample_ising({0: 0.5, 1: -0.5}, {(0, 1): 1.0}, num_reads=3,
                       initial_states=np.zeros((2, 2), np.uint8))
    with pytest.raises(ValueError, match="neither np.uint8"):
        s.sample_ising({0: 0.5, 1: -0.5}, {(0, 1): 1.0},
                       initial_states=np.array([[0, 2]], np.int8))
