"""Rotor-model (SQA) annealing without a GPU: the C restatement (oracle)
against the golden fixtures made by the reference's own rotor Monte Carlo
extension, against that extension directly when it is built here, and the
binding's argument handling."""
import glob
import os

import numpy as np
import pytest

import oracle
from b200sa.sqa import simulated_annealing
from conftest import bits

ROTOR_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "rotor")
ROTOR = sorted(os.path.splitext(os.path.basename(p))[0]
               for p in glob.glob(os.path.join(ROTOR_DIR, "*.npz")))


def load(name):
    with np.load(os.path.join(ROTOR_DIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def compose_shared_stats(blocks, num_betas, interval):
    """One continued-stream call places sample r's block at
    r * n * (num_betas // interval) (cpu_rotormc.cpp:445); later samples
    overwrite the overlap."""
    R, points, n = blocks.shape
    flat = np.zeros(R * points * n, dtype=np.uint8)
    stride = n * (num_betas // interval)
    for r in range(R):
        flat[r * stride: r * stride + points * n] = blocks[r].ravel()
    return flat.reshape(R, points, n)


def written(stats, c):
    """The part of a statistics buffer the reference writes: with one
    continued stream its last (num_betas // interval) < points blocks leave
    the buffer's tail unwritten (np.empty in the binding)."""
    flat = np.asarray(stats).reshape(-1)
    if not c["shared"]:
        return flat
    R, points, n = np.asarray(stats).shape
    stride = n * (len(c["hp"]) // int(c["interval"]))
    return flat[: (R - 1) * stride + points * n]


def test_fixture_set():
    assert len(ROTOR) == 16


@pytest.mark.parametrize("name", ROTOR)
def test_oracle_matches_reference_fixture(name):
    c = load(name)
    seeds = [int(c["seed"])] if c["shared"] else [int(c["seed"]) + r for r in range(len(c["states0"]))]
    s, e, st = oracle.rotormc(c["h"], c["u"], c["v"], c["J"], c["tf"], c["states0"], int(c["spb"]),
                              c["hp"], c["hd"], seeds, bool(c["order"]), str(c["proposal"]),
                              int(c["interval"]))
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    if c["shared"]:
        st = compose_shared_stats(st, len(c["hp"]), int(c["interval"]))
    np.testing.assert_array_equal(written(st, c), written(c["out_stats"], c))


def test_oracle_matches_reference_extension_on_random_problems():
    ref = oracle.reference_rotormc_module()
    if ref is None:
        pytest.skip("reference rotor extension not built (oracle/build_ref.sh)")
    rng = np.random.default_rng(23)
    for trial in range(32):
        n = int(rng.integers(1, 30))
        m = int(rng.integers(0, 3 * n))
        u = rng.integers(0, n, m).astype(np.int32)
        v = rng.integers(0, n, m).astype(np.int32)
        J = rng.normal(0, 1, m)
        h = rng.normal(0, 0.3, n)
        tf = rng.uniform(0, 2, n)
        nb = int(rng.integers(1, 9))
        hp = np.geomspace(0.1, 3.0, nb)
        hd = np.geomspace(3.0, 0.05, nb)
        st0 = rng.integers(0, 256, (1, n)).astype(np.uint8)
        prop = list(oracle.ROTOR_PROPOSALS)[trial % 4]
        order = bool((trial // 4) % 2)
        seed = int(rng.integers(0, 2**31))
        a = oracle.rotormc(h, u, v, J, tf, st0, 2, hp, hd, [seed], order, prop, 2)
        b = ref.simulated_annealing(1, list(h), list(u), list(v), list(J), list(tf), 2, hp, hd,
                                    seed, st0.copy(), order, prop, 2)
        np.testing.assert_array_equal(a[0], np.asarray(b[0]))
        np.testing.assert_array_equal(bits(a[1]), bits(np.asarray(b[1])))
        np.testing.assert_array_equal(a[2], np.asarray(b[2]))


def test_binding_edge_cases_and_errors():
    s, e, st = simulated_annealing(0, [1.0], [], [], [], [1.0], 1, [1.0], [1.0], 1,
                                   np.empty((0, 1), np.uint8), False, "GibbsNonErgodic", 0)
    assert s.shape == (0, 1) and e.shape == (0,) and st.shape == (0,)
    with pytest.raises(ValueError):
        simulated_annealing(1, [1.0], [], [], [], [1.0], 1, [1.0], [1.0], 1,
                            np.zeros((1, 1), np.uint8), False, "Gibbs", 0)
    with pytest.raises(ValueError):
        simulated_annealing(1, [1.0, 2.0], [], [], [], [1.0, 1.0], 1, [1.0], [1.0], 1,
                            np.zeros((1, 1), np.uint8), False, "GibbsNonErgodic", 0)
    with pytest.raises(OverflowError):
        simulated_annealing(1, [1.0], [], [], [], [1.0], 1, [1.0], [1.0], -1,
                            np.zeros((1, 1), np.uint8), False, "GibbsNonErgodic", 0)
