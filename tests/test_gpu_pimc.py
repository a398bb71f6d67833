"""Path-integral Monte Carlo (SQA) annealing on the GPU against the reference:
its golden fixtures (single-qubit and chain updates, both seeding modes,
statistics, break positions, quantum initial states) and the oracle on
random problems."""
import ctypes

import numpy as np
import pytest

import oracle
from b200sa import _lib
from b200sa.sqa import path_annealing
from conftest import bits
from test_pimc_host import PIMC, _random_case, compose_breaks, load

pytestmark = pytest.mark.gpu


def run_fixture(c, **kw):
    s0 = c["states0"].copy()
    R, n = s0.shape
    nb = c["num_breaks0"].copy()
    bo = np.zeros(int(c["out_size"]), np.intc)
    return path_annealing(
        R, c["h"], c["u"], c["v"], c["J"], int(c["spb"]), c["hp"], c["hd"], 1.0,
        float(c["jchain"]), int(c["qpc"]), int(c["qpu"]), int(c["seed"]), s0,
        bool(c["proj_in"]), bool(c["proj_out"]), nb, c["breaks_in"].copy(), bo,
        int(c["interval"]), rng_stream="shared" if bool(c["shared"]) else "per_read", **kw)


@pytest.mark.parametrize("name", PIMC)
def test_golden_fixtures(name):
    c = load(name)
    s, e, st, nb, bo = run_fixture(c)
    np.testing.assert_array_equal(s, c["out_states"])
    np.testing.assert_array_equal(bits(e), bits(c["out_energies"]))
    if int(c["interval"]):
        np.testing.assert_array_equal(st, c["out_stats"])
    if not bool(c["proj_out"]):
        np.testing.assert_array_equal(nb, c["out_num_breaks"])
        np.testing.assert_array_equal(bo, c["out_breaks"])


def _call_abi(c, R, n, q, proj_out, capacity=0):
    """Calls the C ABI directly (per-sample seeds); returns (rc, states,
    energies, break counts, break buffer, near ties, error buffer)."""
    st = c["states0"].copy()
    en = np.zeros(R)
    nb = np.zeros((R, n), np.intc)
    bo = np.zeros(1 << 20, np.intc)
    seeds = (c["seed"] + np.arange(R)).astype(np.uint32)
    hp, hd = c["hp"], c["hd"]
    near = ctypes.c_int64(-1)
    err = _lib.errbuf()
    rc = _lib.load().b200sa_path_anneal(
        n, c["h"].ctypes.data, len(c["J"]), c["u"].ctypes.data, c["v"].ctypes.data,
        c["J"].ctypes.data, R, st.ctypes.data, en.ctypes.data, c["spb"], len(hd),
        hp.ctypes.data, hd.ctypes.data, -1.5, q, q, seeds.ctypes.data, R, 1,
        0 if not proj_out else 1, nb.ctypes.data, None, 0, bo.ctypes.data, len(bo), None, 0,
        capacity, 0, ctypes.byref(near), err, len(err))
    return rc, st, en, nb, bo, near.value, err


@pytest.mark.parametrize("mode", ["qubit", "chain"])
def test_random_problems_vs_oracle(mode):
    q = 1 if mode == "qubit" else 4
    R, n = 96, 64
    c = _random_case(100 + q, n, 160, R, qpc=q, qpu=q)
    rc, s, e, nb, bo, near, err = _call_abi(c, R, n, q, proj_out=False)
    _lib.check(rc, err)
    assert near == 0
    ws, we, wnb, wlists = [], [], [], []
    for r in range(R):
        o = oracle.pimc(c["h"], c["u"], c["v"], c["J"], c["states0"][r:r + 1], c["spb"],
                        c["hp"], c["hd"], c["seed"] + r, -1.5, q, q, True, False, max_out=512)
        ws.append(o[0])
        we.append(o[1])
        wnb.append(o[3])
        wlists.append(o[4])
    wnb = np.concatenate(wnb)
    np.testing.assert_array_equal(s, np.concatenate(ws))
    np.testing.assert_array_equal(bits(e), bits(np.concatenate(we)))
    np.testing.assert_array_equal(nb, wnb)
    np.testing.assert_array_equal(bo, compose_breaks(wnb, np.concatenate(wlists), len(bo)))


def test_capacity_exceeded_is_reported_and_retried(monkeypatch):
    import b200sa.sqa
    c = _random_case(7, 24, 40, 8, hd_value=30.0)
    rc, *_, err = _call_abi(c, 8, 24, 1, proj_out=True, capacity=4)
    assert rc == _lib.ERANGE and b"break_capacity" in err.value
    # The binding doubles an automatic capacity (here made too small) until
    # the run fits.
    monkeypatch.setattr(b200sa.sqa, "_breaks_capacity", lambda hd: 4)
    s0 = c["states0"].copy()
    nb = np.zeros(s0.shape, np.intc)
    s, e, *_ = path_annealing(8, c["h"], c["u"], c["v"], c["J"], 2, c["hp"], c["hd"], 1.0,
                              1.0, 1, 1, c["seed"], s0, True, True, nb, np.zeros(1, np.intc),
                              np.zeros(1, np.intc), 0)
    w = [oracle.pimc(c["h"], c["u"], c["v"], c["J"], c["states0"][r:r + 1], 2, c["hp"],
                     c["hd"], c["seed"] + r)[0] for r in range(8)]
    np.testing.assert_array_equal(s, np.concatenate(w))
    with pytest.raises(_lib.CapacityError):
        path_annealing(8, c["h"], c["u"], c["v"], c["J"], 2, c["hp"], c["hd"], 1.0, 1.0, 1, 1,
                       c["seed"], c["states0"].copy(), True, True, nb, np.zeros(1, np.intc),
                       np.zeros(1, np.intc), 0, break_capacity=4)


def test_interrupt_cuts_after_first_true():
    calls = []

    def stop():
        calls.append(1)
        return len(calls) == 2
    R, n = 6, 5
    out = path_annealing(R, [0.1] * n, [0, 1], [1, 2], [1.0, -1.0], 1, [1.0, 2.0], [1.0, 0.5],
                         1.0, 1.0, 1, 1, 5, np.ones((R, n), np.int8), True, True,
                         np.zeros((R, n), np.intc), np.zeros(1, np.intc), np.zeros(1, np.intc),
                         0, stop)
    assert len(out[0]) == 2 and len(out[1]) == 2 and len(calls) == 2


def test_empty_schedule_with_statistics():
    # No schedule steps: nothing is sampled, the statistics have no points and
    # the states come back unchanged.
    R, n = 4, 6
    st0 = np.ones((R, n), np.int8)
    s, e, st, nb, bo = path_annealing(R, [0.1] * n, [0, 1], [1, 2], [1.0, -1.0], 1, [], [], 1.0,
                                      1.0, 1, 1, 5, st0.copy(), True, True,
                                      np.zeros((R, n), np.intc), np.zeros(1, np.intc),
                                      np.zeros(1, np.intc), 1)
    assert st.shape == (R, 0, n)
    np.testing.assert_array_equal(s, st0)


def test_chain_updates_from_quantum_states_vs_oracle():
    # Chains of 4 starting from world lines with breaks (2 per variable), final
    # breaks returned, per-sample seeds; the oracle runs one call per sample.
    rng = np.random.default_rng(41)
    R, n, q = 24, 48, 4
    u = rng.integers(0, n, 120).astype(np.int32)
    v = rng.integers(0, n, 120).astype(np.int32)
    J, h = rng.normal(0, 1, 120), rng.normal(0, 0.3, n)
    st0 = (2 * rng.integers(0, 2, (R, n)) - 1).astype(np.int8)
    nb0 = np.full((R, n), 2, np.intc)
    bin_ = np.sort(rng.choice(65536, size=(R * n, 2), replace=False), axis=1).astype(np.intc)
    hp, hd = np.geomspace(0.2, 2.0, 6), np.full(6, 3.0)
    s, e, _, nb, bo = path_annealing(R, h, u, v, J, 2, hp, hd, 1.0, -1.2, q, q, 77, st0.copy(),
                                     False, False, nb0.copy(), bin_.ravel().copy(),
                                     np.zeros(1 << 16, np.intc), 0)
    ws, we, wnb, wl = [], [], [], []
    for r in range(R):
        o = oracle.pimc(h, u, v, J, st0[r:r + 1], 2, hp, hd, 77 + r, -1.2, q, q, False, False,
                        num_breaks=nb0[r:r + 1], breaks_in=bin_[r * n:(r + 1) * n].ravel(),
                        max_out=512)
        ws.append(o[0])
        we.append(o[1])
        wnb.append(o[3])
        wl.append(o[4])
    wnb = np.concatenate(wnb)
    np.testing.assert_array_equal(s, np.concatenate(ws))
    np.testing.assert_array_equal(bits(e), bits(np.concatenate(we)))
    np.testing.assert_array_equal(nb, wnb)
    np.testing.assert_array_equal(bo, compose_breaks(wnb, np.concatenate(wl), len(bo)))
