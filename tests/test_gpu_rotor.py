"""Rotor-model (SQA) annealing on the GPU against the reference: its golden
fixtures (every proposal, both orders, both seeding modes, statistics) and
the oracle on random problems."""
import numpy as np
import pytest

import oracle
from b200sa.sqa import simulated_annealing
from conftest import bits
from test_rotor_host import ROTOR, load, written

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", ROTOR)
def test_golden_fixtures(name):
    c = load(name)
    st0 = c["states0"].copy()
    s, e, st = simulated_annealing(
        st0.shape[0], c["h"], c["u"], c["v"], c["J"], c["tf"], int(c["spb"]), c["hp"], c["hd"],
        int(c["seed"]), st0, bool(c["order"]), str(c["proposal"]), int(c["interval"]),
        rng_stream="shared" if c["shared"] else "per_read")
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    np.testing.assert_array_equal(written(st, c), written(c["out_stats"], c))


@pytest.mark.parametrize("proposal", list(oracle.ROTOR_PROPOSALS))
@pytest.mark.parametrize("order", [False, True])
def test_random_problems_vs_oracle(proposal, order):
    rng = np.random.default_rng(len(proposal) + 3 * order)
    n = 300
    m = 900
    u = rng.integers(0, n, m).astype(np.int32)
    v = rng.integers(0, n, m).astype(np.int32)
    J = rng.normal(0, 1, m)
    h = rng.normal(0, 0.3, n)
    tf = rng.uniform(0, 2, n)
    hp = np.geomspace(0.1, 3.0, 20)
    hd = np.geomspace(3.0, 0.05, 20)
    R = 200
    st0 = rng.integers(0, 256, (R, n)).astype(np.uint8)
    seed = 77
    ws, we, wst = oracle.rotormc(h, u, v, J, tf, st0, 2, hp, hd, seed + np.arange(R), order,
                                 proposal, 4)
    s, e, st = simulated_annealing(R, h, u, v, J, tf, 2, hp, hd, seed, st0.copy(), order,
                                   proposal, 4)
    np.testing.assert_array_equal(s, ws)
    np.testing.assert_array_equal(bits(e), bits(we))
    np.testing.assert_array_equal(st, wst)


def test_interrupt_cuts_after_first_true():
    calls = []

    def stop():
        calls.append(1)
        return len(calls) == 3
    st0 = np.zeros((8, 5), np.uint8)
    s, e, st = simulated_annealing(8, [0.1] * 5, [0, 1], [1, 2], [1.0, -1.0], [1.0] * 5, 1,
                                   [1.0, 2.0], [1.0, 0.5], 5, st0, False, "MetropolisUniform",
                                   0, stop)
    assert len(s) == 3 and len(e) == 3 and len(calls) == 3


def test_empty_schedule_with_statistics():
    # No schedule steps: nothing is sampled and the statistics have no points.
    R, n = 4, 6
    st0 = np.full((R, n), 7, np.uint8)
    s, e, st = simulated_annealing(R, [0.1] * n, [0, 1], [1, 2], [1.0, -1.0], [1.0] * n, 1, [],
                                   [], 5, st0.copy(), False, "MetropolisUniform", 1)
    assert st.shape == (R, 0, n)
    np.testing.assert_array_equal(s, st0)
