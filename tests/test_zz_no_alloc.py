"""b200sa_sample_noalloc: the entry point for callers that cannot allocate
device memory while they run (memory owned by a fixed pool, allocation only at
start-up, no cudaMalloc/cudaFree synchronization allowed).  Its working memory
is a fixed array inside the library, so it is checked here against the
regular entry point on two calls in a row (the second call must not be
affected by what the first left in the array), in both update orders, at the
size limits, and after a call that the array's error flag rejected.

Named to be collected last: it runs after every other test in a full run, and
must also pass alone in a fresh process."""
import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


def _problem(rng, n, degree, reads, sweeps, gibbs):
    perm = np.concatenate([rng.permutation(n) for _ in range(degree)])
    a, b = perm[: len(perm) // 2 * 2].reshape(-1, 2).T
    ok = a != b
    u = np.minimum(a[ok], b[ok]).astype(np.int32)
    v = np.maximum(a[ok], b[ok]).astype(np.int32)
    J = rng.normal(0, 1, u.shape[0])
    h = rng.normal(0, 0.1, n)
    states = (2 * rng.integers(0, 2, (reads, n)) - 1).astype(np.int8)
    betas = np.geomspace(0.1, 5.0, sweeps)
    seeds = rng.integers(0, 2**63, reads).astype(np.uint64)
    return h, u, v, J, states, betas, seeds, "Gibbs" if gibbs else "Metropolis"


def _noalloc(h, u, v, J, states, betas, seeds, crit, order=0, expect_rc=None):
    import torch
    from b200sa import _lib
    L = _lib.load()
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dh, du, dv, dJ, db, ds = d(h), d(u), d(v), d(J), d(betas), d(seeds.view(np.int64))
    sin = d(states)
    sout = torch.empty_like(sin)
    en = torch.empty(states.shape[0], dtype=torch.float64, device="cuda")
    ties = torch.full((states.shape[0],), 7, dtype=torch.int32, device="cuda")
    total = ctypes.c_int64(-1)
    torch.cuda.synchronize()
    err = _lib.errbuf()
    rc = L.b200sa_sample_noalloc(
        len(h), dh.data_ptr(), len(J), du.data_ptr(), dv.data_ptr(), dJ.data_ptr(),
        states.shape[0], sin.data_ptr(), sout.data_ptr(), en.data_ptr(), 1, len(betas),
        db.data_ptr(), ds.data_ptr(), order, 0 if crit == "Gibbs" else 1, 0, None,
        ties.data_ptr(), ctypes.byref(total), err, len(err))
    if expect_rc is not None:
        assert rc == expect_rc, err.value
        return err.value
    _lib.check(rc, err)
    assert torch.equal(sin.cpu(), torch.from_numpy(states))  # inputs untouched
    # Every read's near-tie count was written (expected 0) and so was the total.
    assert total.value == 0 and int(ties.abs().sum()) == 0
    return sout.cpu().numpy(), en.cpu().numpy()


def _check_twice(h, u, v, J, states, betas, seeds, crit, order):
    from b200sa import simulated_annealing
    reads = states.shape[0]
    want_s, want_e = simulated_annealing(reads, h, u, v, J, 1, betas, 0, states.copy(),
                                         bool(order), crit, seeds=seeds)
    for _ in range(2):  # two calls in a row share the fixed working memory
        got_s, got_e = _noalloc(h, u, v, J, states, betas, seeds, crit, order)
        np.testing.assert_array_equal(got_s, want_s)
        np.testing.assert_array_equal(got_e.view(np.uint64), want_e.view(np.uint64))


@pytest.mark.parametrize("order", [0, 1])
@pytest.mark.parametrize("gibbs", [False, True])
def test_noalloc_matches_regular_entry_point_twice(gibbs, order):
    rng = np.random.default_rng(31 + gibbs + 2 * order)
    for n, degree, reads, sweeps in ((700, 6, 96, 120), (300, 11, 40, 150)):
        _check_twice(*_problem(rng, n, degree, reads, sweeps, gibbs), order)


def test_noalloc_at_its_size_limits():
    """n = 4096 with 65536 couplers: the largest shared-memory region and the
    longest adjacency the fixed array holds."""
    rng = np.random.default_rng(77)
    h, u, v, J, states, betas, seeds, crit = _problem(rng, 4096, 33, 48, 24, False)
    u, v, J = u[:65536], v[:65536], J[:65536]
    assert len(J) == 65536
    _check_twice(h, u, v, J, states, betas, seeds, crit, 0)


def test_noalloc_bad_coupler_then_valid_call():
    """A coupler index outside the problem sets the array's error flag and the
    call returns EINVAL; the next valid call on the same array is unaffected."""
    from b200sa import _lib
    rng = np.random.default_rng(5)
    h, u, v, J, states, betas, seeds, crit = _problem(rng, 200, 5, 16, 30, False)
    bad_v = v.copy()
    bad_v[len(bad_v) // 2] = 200
    msg = _noalloc(h, u, bad_v, J, states, betas, seeds, crit, expect_rc=_lib.EINVAL)
    assert b"invalid variable" in msg
    _check_twice(h, u, v, J, states, betas, seeds, crit, 0)


def test_noalloc_refuses_stream_capture():
    """The call waits for its own work, so it refuses a capturing stream
    before enqueuing anything."""
    import torch
    from b200sa import _lib
    rng = np.random.default_rng(6)
    h, u, v, J, states, betas, seeds, crit = _problem(rng, 64, 3, 4, 4, False)
    L = _lib.load()
    s = torch.cuda.Stream()
    g = torch.cuda.CUDAGraph()
    err = _lib.errbuf()
    with torch.cuda.graph(g, stream=s):
        rc = L.b200sa_sample_noalloc(64, 1, 0, None, None, None, 4, 1, 1, 1, 1, 4, 1, 1,
                                     0, 1, 0, s.cuda_stream, None, None, err, len(err))
    assert rc == _lib.EINVAL and b"CUDA graph" in err.value


def test_noalloc_rejects_problems_beyond_its_fixed_memory():
    from b200sa import _lib
    L = _lib.load()
    err = _lib.errbuf()
    rc = L.b200sa_sample_noalloc(5000, 1, 0, None, None, None, 1, 1, 1, 1, 1, 1, 1, 1,
                                 0, 1, 0, None, None, None, err, len(err))
    assert rc == _lib.EINVAL and b"num_vars <= 4096" in err.value
    rc = L.b200sa_sample_noalloc(10, 1, 70000, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                 0, 1, 0, None, None, None, err, len(err))
    assert rc == _lib.EINVAL and b"num_couplers <= 65536" in err.value
