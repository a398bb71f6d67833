"""Path-integral Monte Carlo (SQA) annealing without a GPU: the C restatement
(oracle) against the golden fixtures made by the reference's own localPIMC
extension, against that extension directly when it is built here, the
restated mt19937, and the binding's argument handling."""
import glob
import os

import numpy as np
import pytest

import oracle
from b200sa.sqa import path_annealing
from conftest import bits

PIMC_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "pimc")
PIMC = sorted(os.path.splitext(os.path.basename(p))[0]
              for p in glob.glob(os.path.join(PIMC_DIR, "*.npz")))


def load(name):
    with np.load(os.path.join(PIMC_DIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def compose_breaks(num_breaks, lists, size):
    """The reference's break buffer (localPIMC.cpp:185-200 called sample after
    sample, :700-703): a variable's positions are written only while the rest
    of the buffer holds them all; every sample starts its total count after
    the previous sample's start."""
    buf = np.zeros(size, dtype=np.intc)
    start = 0
    for r in range(num_breaks.shape[0]):
        capacity, p = size - start, start
        for v in range(num_breaks.shape[1]):
            c = int(num_breaks[r, v])
            if capacity >= c:
                buf[p:p + c] = lists[r, v, :c]
                p += c
                capacity -= c
        start += int(num_breaks[r].sum())
    return buf


def oracle_run(c, max_out=512):
    """The oracle on a fixture's inputs: one call over all samples (shared) or
    one call per sample with seed + r."""
    kw = dict(chain_coupler_strength=float(c["jchain"]), qubits_per_chain=int(c["qpc"]),
              qubits_per_update=int(c["qpu"]), project_inputs=bool(c["proj_in"]),
              project_outputs=bool(c["proj_out"]), interval=int(c["interval"]),
              max_out=max_out)
    args = (c["h"], c["u"], c["v"], c["J"])
    s0 = c["states0"]
    R, n = s0.shape
    if bool(c["shared"]):
        return oracle.pimc(*args, s0, int(c["spb"]), c["hp"], c["hd"], int(c["seed"]),
                           num_breaks=c["num_breaks0"], breaks_in=c["breaks_in"], **kw)
    per = n * n if not bool(c["proj_in"]) else 0
    outs = []
    for r in range(R):
        bin_r = c["breaks_in"][r * per:(r + 1) * per] if per else c["breaks_in"]
        outs.append(oracle.pimc(*args, s0[r:r + 1], int(c["spb"]), c["hp"], c["hd"],
                                int(c["seed"]) + r, num_breaks=c["num_breaks0"][r:r + 1],
                                breaks_in=bin_r, **kw))
    return tuple(np.concatenate([o[k] for o in outs]) for k in range(5))


def test_fixture_set():
    assert len(PIMC) == 12


def test_mt19937_check_value():
    # The C++ standard's check: the 10000th output of a default-constructed
    # std::mt19937 (seed 5489) is 4123659995.
    assert oracle.mt19937(5489, 10000)[-1] == 4123659995


@pytest.mark.parametrize("name", PIMC)
def test_oracle_matches_golden(name):
    c = load(name)
    s, e, st, nb, lists = oracle_run(c)
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    if int(c["interval"]):
        np.testing.assert_array_equal(st, c["out_stats"])
    if not bool(c["proj_out"]):
        np.testing.assert_array_equal(nb, c["out_num_breaks"])
        np.testing.assert_array_equal(compose_breaks(nb, lists, int(c["out_size"])),
                                      c["out_breaks"])


def _random_case(seed, n, m, R, qpc=1, qpu=1, hd_value=4.0):
    rng = np.random.default_rng(seed)
    u = rng.integers(0, n, m).astype(np.int32)
    v = rng.integers(0, n, m).astype(np.int32)
    return dict(h=rng.normal(0, 0.3, n), u=u, v=v, J=rng.normal(0, 1, m),
                states0=(2 * rng.integers(0, 2, (R, n)) - 1).astype(np.int8),
                spb=2, hp=np.geomspace(0.2, 2.0, 6), hd=np.full(6, hd_value),
                seed=int(rng.integers(1, 2**31)), qpc=qpc, qpu=qpu)


@pytest.mark.parametrize("mode", ["qubit", "chain"])
def test_oracle_matches_reference_extension(mode):
    ref = oracle.reference_pimc_module()
    if ref is None:
        pytest.skip("reference extension not built (bash oracle/build_ref.sh)")
    q = 1 if mode == "qubit" else 4
    c = _random_case(11 + q, 32, 60, 3, qpc=q, qpu=q)
    R, n = c["states0"].shape
    size = 1 << 15
    nb0 = np.zeros((R, n), np.intc)
    rs, re, _, rnb, rbo = ref.simulated_annealing(
        R, list(map(float, c["h"])), list(map(int, c["u"])), list(map(int, c["v"])),
        list(map(float, c["J"])), c["spb"], c["hp"], c["hd"], 1.0, -1.5, q, q, c["seed"],
        c["states0"].copy(), True, False, nb0.copy(), np.zeros(1, np.intc),
        np.zeros(size, np.intc), 0)
    s, e, _, nb, lists = oracle.pimc(c["h"], c["u"], c["v"], c["J"], c["states0"], c["spb"],
                                     c["hp"], c["hd"], c["seed"], -1.5, q, q, True, False,
                                     max_out=512)
    np.testing.assert_array_equal(s, rs)
    np.testing.assert_array_equal(bits(e), bits(re))
    np.testing.assert_array_equal(nb, rnb)
    np.testing.assert_array_equal(compose_breaks(nb, lists, size), rbo)


def _args(R=2, n=4):
    return dict(num_samples=R, h=[0.1] * n, coupler_starts=[0], coupler_ends=[1],
                coupler_weights=[1.0], sweeps_per_beta=1, Hp_field=[1.0], Hd_field=[1.0],
                Gamma=1.0, chain_coupler_strength=1.0, qubits_per_chain=1,
                qubits_per_update=1, seed=3, states_numpy=np.ones((R, n), np.int8),
                project_inputs=True, project_outputs=True,
                num_breaks_numpy=np.zeros((R, n), np.intc),
                breaks_in_numpy=np.zeros(1, np.intc),
                breaks_buffer_out_numpy=np.zeros(1, np.intc), schedule_sample_interval=0)


def test_empty_problem_shapes():
    a = _args()
    a.update(h=[], coupler_starts=[], coupler_ends=[], coupler_weights=[],
             states_numpy=np.ones((2, 0), np.int8), num_breaks_numpy=np.zeros((2, 0), np.intc))
    s, e, st, nb, bo = path_annealing(**a)
    assert s.shape == (2, 0) and list(e) == [0.0, 0.0] and st.size == 0 and bo.size == 0


@pytest.mark.parametrize("change, error", [
    (dict(states_numpy=np.ones((2, 4), np.int16)), ValueError),
    (dict(num_breaks_numpy=np.zeros((2, 4), np.int64)), ValueError),
    (dict(coupler_ends=[1, 2]), ValueError),
    (dict(seed=-1), OverflowError),
    (dict(seed=2**32), OverflowError),
    (dict(Hp_field=[]), ValueError),
    (dict(coupler_ends=[9]), ValueError),
    (dict(qubits_per_chain=0), ValueError),
    (dict(qubits_per_chain=8, qubits_per_update=8), ValueError),
    (dict(rng_stream="other"), ValueError),
])
def test_argument_errors(change, error):
    a = _args()
    a.update(change)
    with pytest.raises(error):
        path_annealing(**a)
