"""b200sa_sample_noalloc: the entry point for callers that cannot allocate
device memory while they run (memory owned by a fixed pool, allocation only at
start-up, no cudaMalloc/cudaFree synchronization allowed).  Its working memory
is a fixed array inside the library, so it is checked here against the
regular entry point on two calls in a row (the second call must not be
affected by what the first left in the array).

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


def _noalloc(h, u, v, J, states, betas, seeds, crit):
    import torch
    from b200sa import _lib
    L = _lib.load()
    d = lambda x: torch.from_numpy(np.ascontiguousarray(x)).cuda()
    dh, du, dv, dJ, db, ds = d(h), d(u), d(v), d(J), d(betas), d(seeds.view(np.int64))
    sin = d(states)
    sout = torch.empty_like(sin)
    en = torch.empty(states.shape[0], dtype=torch.float64, device="cuda")
    torch.cuda.synchronize()
    err = _lib.errbuf()
    rc = L.b200sa_sample_noalloc(
        len(h), dh.data_ptr(), len(J), du.data_ptr(), dv.data_ptr(), dJ.data_ptr(),
        states.shape[0], sin.data_ptr(), sout.data_ptr(), en.data_ptr(), 1, len(betas),
        db.data_ptr(), ds.data_ptr(), 0, 0 if crit == "Gibbs" else 1, 0, None, err, len(err))
    _lib.check(rc, err)
    assert torch.equal(sin.cpu(), torch.from_numpy(states))  # inputs untouched
    return sout.cpu().numpy(), en.cpu().numpy()


@pytest.mark.parametrize("gibbs", [False, True])
def test_noalloc_matches_regular_entry_point_twice(gibbs):
    from b200sa import simulated_annealing
    rng = np.random.default_rng(31 + gibbs)
    for n, degree, reads, sweeps in ((700, 6, 96, 120), (300, 11, 40, 150)):
        h, u, v, J, states, betas, seeds, crit = _problem(rng, n, degree, reads, sweeps, gibbs)
        want_s, want_e = simulated_annealing(reads, h, u, v, J, 1, betas, 0, states.copy(),
                                             False, crit, seeds=seeds)
        for _ in range(2):  # two calls in a row share the fixed working memory
            got_s, got_e = _noalloc(h, u, v, J, states, betas, seeds, crit)
            np.testing.assert_array_equal(got_s, want_s)
            np.testing.assert_array_equal(got_e.view(np.uint64), want_e.view(np.uint64))


def test_noalloc_rejects_problems_beyond_its_fixed_memory():
    from b200sa import _lib
    L = _lib.load()
    err = _lib.errbuf()
    rc = L.b200sa_sample_noalloc(5000, 1, 0, None, None, None, 1, 1, 1, 1, 1, 1, 1, 1,
                                 0, 1, 0, None, err, len(err))
    assert rc == _lib.EINVAL and b"num_vars <= 4096" in err.value
    rc = L.b200sa_sample_noalloc(10, 1, 70000, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1, 1,
                                 0, 1, 0, None, err, len(err))
    assert rc == _lib.EINVAL and b"num_couplers <= 65536" in err.value
