"""Steepest descent without a GPU: the C restatement (oracle) against the
golden fixtures made by the reference's own descent extension, against that
extension directly when it is built here, and the Python binding's argument
handling."""
import glob
import os

import numpy as np
import pytest

import oracle
from b200sa.greedy import steepest_gradient_descent
from conftest import bits

DESCENT_DIR = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "descent")
DESCENT = sorted(os.path.splitext(os.path.basename(p))[0]
                 for p in glob.glob(os.path.join(DESCENT_DIR, "*.npz")))


def load(name):
    with np.load(os.path.join(DESCENT_DIR, name + ".npz")) as z:
        return {k: z[k] for k in z.files}


def test_fixture_set():
    assert len(DESCENT) == 12
    assert "convex_linear" in DESCENT and "convex_sparse" in DESCENT


@pytest.mark.parametrize("name", DESCENT)
def test_oracle_matches_reference_fixture(name):
    c = load(name)
    s, e, k = oracle.descent(c["h"], c["u"], c["v"], c["J"], c["states0"],
                             bool(c["large_sparse_opt"]))
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    np.testing.assert_array_equal(k, c["out_steps"])


def test_convex_example_of_the_reference_test():
    # tests/test_greedy.py:26-45: converges to (-1, -1) with energy -5
    for mode in (False, True):
        s, e, _ = oracle.descent([2, 2], [0], [1], [-1], np.array([[1, 1]], np.int8), mode)
        assert s.tolist() == [[-1, -1]] and e.tolist() == [-5.0]


def test_oracle_matches_reference_extension_on_random_problems():
    ref = oracle.reference_descent_module()
    if ref is None:
        pytest.skip("reference descent extension not built (oracle/build_ref.sh)")
    rng = np.random.default_rng(11)
    for trial in range(60):
        n = int(rng.integers(1, 80))
        m = int(rng.integers(0, 3 * n))
        u = rng.integers(0, n, m).astype(np.int32)
        v = rng.integers(0, n, m).astype(np.int32)
        keep = u != v  # a positive self-loop makes the reference descend for ever
        u, v = u[keep], v[keep]
        if trial % 2:
            J = rng.integers(-2, 3, len(u)).astype(float)
            h = rng.integers(-2, 3, n).astype(float)
        else:
            J = rng.normal(0, 1, len(u))
            h = rng.normal(0, 0.3, n)
        st = (2 * rng.integers(0, 2, (4, n)) - 1).astype(np.int8)
        mode = bool(trial % 3 == 0)
        a = oracle.descent(h, u, v, J, st, mode)
        b = ref.steepest_gradient_descent(4, list(h), list(u), list(v), list(J), st.copy(), mode)
        np.testing.assert_array_equal(a[0], b[0])
        np.testing.assert_array_equal(bits(a[1]), bits(np.asarray(b[1])))
        np.testing.assert_array_equal(a[2], np.asarray(b[2]))


def test_binding_edge_cases_and_errors():
    # descent.pyx:83-88: no samples or no variables short-circuit
    s, e, k = steepest_gradient_descent(0, [1.0], [], [], [], np.empty((0, 1), np.int8))
    assert s.shape == (0, 1) and e.shape == (0,) and k.dtype == np.uint32
    s, e, k = steepest_gradient_descent(3, [], [], [], [], np.empty((3, 0), np.int8))
    assert s.shape == (3, 0) and np.all(e == 0) and np.all(k == 0)
    with pytest.raises(ValueError):
        steepest_gradient_descent(2, [1.0, 2.0], [0], [1], [1.0], np.ones((2, 3), np.int8))
    with pytest.raises(ValueError):
        steepest_gradient_descent(1, [1.0, 2.0], [0], [1], [1.0],
                                  np.ones((1, 2), np.int16))
    with pytest.raises(ValueError):
        steepest_gradient_descent(1, [1.0, 2.0], [0, 1], [1], [1.0], np.ones((1, 2), np.int8))
