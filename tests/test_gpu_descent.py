"""Steepest descent on the GPU against the reference: its golden fixtures
(both solver modes), the oracle on random problems of many sizes (shared-
memory and global-slot state), the step limit, and the solver front end
and composite."""
import numpy as np
import pytest

import oracle
from b200sa import workloads
from b200sa.greedy import (SteepestDescentComposite, SteepestDescentSolver,
                           steepest_gradient_descent)
from b200sa.sampler import SimulatedAnnealingSampler
from conftest import bits
from test_descent_host import DESCENT, load

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("name", DESCENT)
def test_golden_fixtures(name):
    c = load(name)
    st = c["states0"].copy()
    s, e, k = steepest_gradient_descent(st.shape[0], c["h"], c["u"], c["v"], c["J"], st,
                                        bool(c["large_sparse_opt"]))
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    np.testing.assert_array_equal(k, c["out_steps"])


@pytest.mark.parametrize("n", [1, 5, 33, 257, 1500, 4096, 9000])
@pytest.mark.parametrize("mode", [False, True])
def test_random_problems_vs_oracle(n, mode):
    rng = np.random.default_rng(n + 7 * mode)
    m = 3 * n
    u = rng.integers(0, n, m).astype(np.int32)
    v = rng.integers(0, n, m).astype(np.int32)
    keep = u != v
    u, v = u[keep], v[keep]
    J = rng.normal(0, 1, len(u))
    h = rng.normal(0, 0.3, n)
    R = 40 if n < 5000 else 6
    st = (2 * rng.integers(0, 2, (R, n)) - 1).astype(np.int8)
    ws, we, wk = oracle.descent(h, u, v, J, st, mode)
    s, e, k = steepest_gradient_descent(R, h, u, v, J, st.copy(), mode)
    np.testing.assert_array_equal(s, ws)
    np.testing.assert_array_equal(bits(e), bits(we))
    np.testing.assert_array_equal(k, wk)


def test_regular_graph_from_annealed_states():
    inst = workloads.uneven_batch(num_problems=1, n_range=(800, 800), reads_range=(64, 64),
                                  sweeps_range=(20, 20), seed=9)[0]
    for mode in (False, True):
        ws, we, wk = oracle.descent(inst.h, inst.u, inst.v, inst.J, inst.states, mode)
        s, e, k = steepest_gradient_descent(inst.num_reads, inst.h, inst.u, inst.v, inst.J,
                                            inst.states.copy(), mode)
        np.testing.assert_array_equal(s, ws)
        np.testing.assert_array_equal(bits(e), bits(we))
        np.testing.assert_array_equal(k, wk)


def test_positive_self_loop_stops_at_the_step_limit():
    # h = 0 and a self-loop J = +1: the flip energy alternates -2, -2, ...
    # and the reference would flip for ever; the call stops at max_steps.
    st = np.array([[1]], dtype=np.int8)
    with pytest.raises(TimeoutError):
        steepest_gradient_descent(1, [0.0], [0], [0], [1.0], st, False, max_steps=1000)


def test_solver_front_end_and_composite():
    h = {0: 2.0, 1: 2.0}
    J = {(0, 1): -1.0}
    ss = SteepestDescentSolver().sample_ising(h, J, num_reads=5, seed=1)
    assert len(ss) == 5 and np.all(ss.record.energy == -5.0)
    assert ss.first.sample == {0: -1, 1: -1}
    ss = SteepestDescentSolver().sample_qubo({(0, 0): -1.0, (1, 1): -1.0, (0, 1): 2.0},
                                             num_reads=8, seed=2)
    assert np.all(ss.record.energy == -1.0)
    # annealing then descent: every sample a local minimum, never worse
    inst = workloads.uneven_batch(num_problems=1, n_range=(300, 300), reads_range=(8, 8),
                                  sweeps_range=(5, 5), seed=3)[0]
    hh = {i: float(x) for i, x in enumerate(inst.h)}
    JJ = {(int(a), int(b)): float(w) for a, b, w in zip(inst.u, inst.v, inst.J)}
    sa = SimulatedAnnealingSampler().sample_ising(hh, JJ, num_reads=8, num_sweeps=5, seed=4)
    comp = SteepestDescentComposite(SimulatedAnnealingSampler()).sample_ising(
        hh, JJ, num_reads=8, num_sweeps=5, seed=4)
    assert np.all(comp.record.energy <= sa.record.energy + 1e-9)
    s = comp.record.sample.astype(np.float64)
    n = s.shape[1]
    for row in s:
        f = inst.h.copy()
        np.add.at(f, inst.u, inst.J * row[inst.v])
        np.add.at(f, inst.v, inst.J * row[inst.u])
        assert np.all(-2 * row * f >= -1e-9)  # no single flip lowers the energy
    assert n == 300
