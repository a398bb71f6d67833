"""Pins the CPU oracle (oracle/sa_oracle.c) to the reference.

* against the committed golden vectors, produced by the reference's own code
  (tests/golden/make_golden.py);
* against the reference extension built from source (oracle/build_ref.sh),
  when that build is present.
"""
import numpy as np
import pytest

import oracle
from conftest import GOLDEN, bits, load_golden


@pytest.mark.parametrize("name", GOLDEN)
def test_oracle_matches_golden(name):
    c = load_golden(name)
    seeds = c["seeds"] if not bool(c["shared"]) else c["seeds"][:1]
    s, e = oracle.run(c["h"], c["u"], c["v"], c["J"], c["states0"], int(c["spb"]),
                      c["betas"], seeds, bool(c["order"]), int(c["proposal"]) == 0)
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))


def test_golden_set_is_complete():
    # The cases the parity tests rely on (edge cases of the reference tests).
    for need in ("fm_shared", "fm_per_read", "dense100", "lattice8", "sparse300",
                 "k16_gibbs", "random_metropolis", "random_gibbs", "beta_edges_metropolis",
                 "beta_edges_gibbs", "dups_metropolis", "dups_gibbs", "zero_sweeps",
                 "null_model", "huge_gibbs", "odd_spins"):
        assert need in GOLDEN


def test_rng_stream_matches_xorshift128plus():
    # cpu_sa.cpp:27-34, seed 0 replaced by 2^64-1 (cpu_sa.cpp:283).
    M = (1 << 64) - 1

    def stream(seed, k):
        s0, s1 = (seed or M), 0
        out = []
        for _ in range(k):
            a, b = s0, s1
            s0 = b
            a = (a ^ (a << 23)) & M
            s1 = a ^ b ^ (a >> 17) ^ (b >> 26)
            out.append((s1 + b) & M)
        return out

    for seed in (0, 1, 12345, 2**63 + 7):
        assert list(map(int, oracle.rng_stream(seed, 50))) == stream(seed, 50)


def _random_case(rng, n, p, selfloops=False, dups=False, integer=False):
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < p
    u, v = iu[keep], ju[keep]
    if selfloops:
        u = np.concatenate([u, np.arange(0, n, 3)])
        v = np.concatenate([v, np.arange(0, n, 3)])
    if dups and len(u):
        u = np.concatenate([u, u[:5]])
        v = np.concatenate([v, v[:5]])
    J = rng.uniform(-1, 1, u.shape[0])
    h = rng.uniform(-1, 1, n)
    if integer:
        J, h = np.round(3 * J), np.round(2 * h)
    return h, u.astype(np.int32), v.astype(np.int32), J


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("gibbs", [False, True])
def test_oracle_matches_reference_build(order, gibbs):
    ref = oracle.reference_module()
    if ref is None:
        pytest.skip("reference extension not built (oracle/build_ref.sh)")
    rng = np.random.default_rng(100 + 2 * order + gibbs)
    crit = "Gibbs" if gibbs else "Metropolis"
    for kw in ({}, {"selfloops": True, "dups": True}, {"integer": True}):
        n = int(rng.integers(10, 60))
        h, u, v, J = _random_case(rng, n, 0.3, **kw)
        st = (2 * rng.integers(0, 2, (6, n)) - 1).astype(np.int8)
        betas = np.geomspace(0.1, 4.0, 40)
        seeds = rng.integers(0, 2**40, 6).astype(np.uint64)
        # per read
        a, ea = oracle.run(h, u, v, J, st, 2, betas, seeds, bool(order), gibbs)
        b, eb = oracle.reference_per_read(h, u, v, J, st, 2, betas, seeds, bool(order), crit)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(bits(ea), bits(eb))
        # one stream continued across reads
        a, ea = oracle.run(h, u, v, J, st, 2, betas, seeds[:1], bool(order), gibbs)
        b, eb = ref.simulated_annealing(6, list(h), list(u), list(v), list(J), 2, betas,
                                        int(seeds[0]), st.copy(), bool(order), crit)
        np.testing.assert_array_equal(a, b)
        np.testing.assert_array_equal(bits(ea), bits(eb))
