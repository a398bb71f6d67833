"""Host-side logic that needs no GPU: argument handling of the drop-in
binding, seed mapping, workload generators, and a CPU model of the kernel's
speculative-window and RNG-ring algorithm checked against the oracle."""
import math

import numpy as np
import pytest

import oracle
from b200sa import per_read_seeds, simulated_annealing
from b200sa import workloads


def test_empty_short_circuit():
    # simulated_annealing.pyx:134-136
    s, e = simulated_annealing(0, [1.0, 2.0], [], [], [], 1, [1.0], 1,
                               np.ones((0, 2), np.int8))
    assert s.shape == (0, 2) and e.shape == (0,)
    s, e = simulated_annealing(3, [], [], [], [], 1, [1.0], 1, np.ones((3, 0), np.int8))
    assert s.shape == (3, 0) and s.dtype == np.int8
    assert np.array_equal(e, np.zeros(3))


def test_argument_errors_match_reference():
    st = np.ones((2, 3), np.int8)
    h = [0.0, 0.0, 0.0]
    with pytest.raises(ValueError, match="Unknown proposal_acceptance_criteria"):
        simulated_annealing(2, h, [0], [1], [1.0], 1, [1.0], 1, st,
                            proposal_acceptance_criteria="heatbath")
    with pytest.raises(OverflowError):
        simulated_annealing(2, h, [0], [1], [1.0], 1, [1.0], -1, st)
    with pytest.raises(ValueError, match="mismatched"):
        simulated_annealing(2, h, [0, 1], [1], [1.0], 1, [1.0], 1, st)
    with pytest.raises(ValueError, match="dtype"):
        simulated_annealing(2, h, [0], [1], [1.0], 1, [1.0], 1, st.astype(np.int16))
    with pytest.raises(ValueError, match="C-contiguous"):
        simulated_annealing(2, h, [0], [1], [1.0], 1, [1.0], 1,
                            np.ones((3, 2), np.int8).T)
    with pytest.raises(ValueError, match="shape"):
        simulated_annealing(3, h, [0], [1], [1.0], 1, [1.0], 1, st)


def test_per_read_seeds_wrap():
    s = per_read_seeds(2**64 - 2, 4)
    assert list(map(int, s)) == [2**64 - 2, 2**64 - 1, 0, 1]
    assert list(map(int, per_read_seeds(5, 3))) == [5, 6, 7]


def test_workload_shapes():
    d = workloads.dense_ising(n=40, reads=3, sweeps=7)
    assert d.states.shape == (3, 40) and len(d.betas) == 7
    assert np.all(d.u < d.v) and d.attempts == 3 * 7 * 40
    lat = workloads.cubic_lattice(L=4, reads=2, sweeps=5)
    deg = np.bincount(np.concatenate([lat.u, lat.v]), minlength=64)
    assert lat.n == 64 and np.all(deg == 6) and set(np.unique(lat.J)) <= {-1.0, 1.0}
    b = workloads.uneven_batch(num_problems=3, n_range=(64, 128), reads_range=(4, 8),
                               sweeps_range=(16, 32))
    assert len(b) == 3
    for p in b:
        deg = np.bincount(np.concatenate([p.u, p.v]), minlength=p.n)
        assert len(set(deg.tolist())) == 1 and 3 <= deg[0] <= 16
        assert p.seeds.shape == (p.num_reads,)
    k = workloads.complete_graph(reads=5, sweeps=3)
    assert k.n == 16 and k.J.shape == (120,) and k.proposal == "Gibbs"


# ---- CPU model of the kernel algorithm -------------------------------------
M64 = (1 << 64) - 1
RING, HALF, PER = 512, 256, 8


def _adv(s0, s1):
    a, b = s0, s1
    s0 = b
    a = (a ^ (a << 23)) & M64
    return s0, a ^ b ^ (a >> 17) ^ (b >> 26)


def _jump_columns(steps):
    cols = []
    for bit in range(128):
        s0 = (1 << bit) if bit < 64 else 0
        s1 = 0 if bit < 64 else 1 << (bit - 64)
        for _ in range(steps):
            s0, s1 = _adv(s0, s1)
        cols.append((s0, s1))
    return cols


class _Ring:
    """The kernel's ring: 32 lanes each fill PER consecutive outputs per half,
    then jump their segment state HALF steps with the GF(2) matrix."""
    cols = None

    def __init__(self, seed):
        if _Ring.cols is None:
            _Ring.cols = _jump_columns(HALF)
        self.ring = [0] * RING
        s0, s1 = (seed or M64), 0
        self.T = []
        for lane in range(32):
            a, b = s0, s1
            for _ in range(lane * PER):
                a, b = _adv(a, b)
            self._fill(0, a, b, lane)
            a, b = self._jump(a, b)
            self._fill(HALF, a, b, lane)
            self.T.append(self._jump(a, b))
        self.q = self.base = 0

    def _jump(self, s0, s1):
        a0 = a1 = 0
        for bit in range(128):
            if ((s0 if bit < 64 else s1) >> (bit % 64)) & 1:
                a0 ^= self.cols[bit][0]
                a1 ^= self.cols[bit][1]
        return a0, a1

    def _fill(self, pos, a, b, lane):
        for t in range(PER):
            prev = b
            a, b = _adv(a, b)
            self.ring[(pos + lane * PER + t) & (RING - 1)] = (b + prev) & M64

    def refill(self):
        if self.q - self.base >= HALF:
            for lane in range(32):
                a, b = self.T[lane]
                self._fill(self.base + RING, a, b, lane)
                self.T[lane] = self._jump(a, b)
            self.base += HALF

    def get(self, pos):
        assert self.base <= pos < self.base + RING
        return self.ring[pos & (RING - 1)]


def test_ring_reproduces_stream():
    want = oracle.rng_stream(987654321, 3000)
    r = _Ring(987654321)
    got = []
    while r.q < 3000:
        r.refill()
        take = min(29, 3000 - r.q)
        got += [r.get(r.q + i) for i in range(take)]
        r.q += take
    assert got == list(map(int, want))


def _model_anneal(h, u, v, J, s, betas, spb, seed, gibbs, resolve=False):
    """Speculative 32-wide windows exactly as the sequential-order kernel.

    With ``resolve`` (used when no list names a target twice and every spin
    is +-1), a pass does not end at the first lane a committed flip could
    have changed: the flips just committed correct the delta energies of the
    later lanes they neighbour (in variable order, as the reference adds
    them), those lanes decide again with draws placed after the committed
    ones, and the pass goes on until the window is committed."""
    n = len(h)
    rows = [[] for _ in range(n)]
    for a, b, w in zip(u, v, J):
        rows[a].append((int(b), float(w)))
        rows[b].append((int(a), float(w)))
    dist = []
    for i in range(n):
        ds = [t - i for t, _ in rows[i] if t > i]
        dist.append(min([32] + ds))
    if resolve:
        assert all(len({t for t, _ in r}) == len(r) for r in rows)
        assert all(int(x) in (-1, 1) for x in s)
        # back[v]: {offset o in 1..31: J} for neighbours v - o
        back = [{i - t: w for t, w in rows[i] if 0 < i - t < 32} for i in range(n)]
    s = [int(x) for x in s]
    de = []
    for i in range(n):
        f = float(h[i])
        for t, w in rows[i]:
            f += s[t] * w
        de.append((-2 * s[i]) * f)
    R = _Ring(seed)
    for beta in betas:
        thr = 44.36142 / beta
        for _ in range(spb):
            p = 0
            while p < n:
                R.refill()
                L = min(32, n - p)
                d = [de[p + k] for k in range(L)]
                c, used, flips = 0, 0, []
                while c < L:
                    need, acc = [False] * L, [False] * L
                    for k in range(c, L):
                        consider = not (d[k] >= thr)
                        need[k] = consider if gibbs else (consider and not d[k] <= 0.0)
                        acc[k] = (not gibbs) and consider
                    cnt = 0
                    for k in range(c, L):
                        if need[k]:
                            r = float(R.get(R.q + used + cnt))
                            cnt += 1
                            if gibbs:
                                e = math.exp(d[k] * beta) if d[k] * beta < 709 else math.inf
                                acc[k] = 2.0 ** 64 > r * (1 + e)
                            else:
                                acc[k] = math.exp(-d[k] * beta) * 2.0 ** 64 > r
                    commit = min([L] + [k + dist[p + k] for k in range(c, L) if acc[k]])
                    used += sum(need[c:commit])
                    new = [k for k in range(c, commit) if acc[k]]
                    flips += [p + k for k in new]
                    c = commit
                    if not resolve:
                        break
                    for k in range(c, L):  # corrections, in variable order
                        for j in new:
                            w = back[p + k].get(k - j)
                            if w is not None:
                                d[k] = d[k] + ((4.0 * s[p + j]) * w) * s[p + k]
                R.q += used
                if flips:
                    _model_apply_flips(rows, de, s, flips)
                p += c
    return np.array(s, np.int8)


def _model_apply_flips(rows, de, s, flips):
    """The kernel's update rounds: the flips' adjacency entries concatenated
    in variable order, 32 per round; entries of a round naming the same slot
    are summed in entry order by the first of them."""
    entries = []
    for var in flips:
        m = float(np.int8(4 * s[var]))
        entries += [(t, (m * w) * s[t]) for t, w in rows[var]]
    for base in range(0, len(entries), 32):
        rnd = entries[base:base + 32]
        done = set()
        for i, (t, x) in enumerate(rnd):
            if t in done:
                continue
            acc = de[t]
            for t2, x2 in rnd[i:]:
                if t2 == t:
                    acc = acc + x2
            de[t] = acc
            done.add(t)
    for var in flips:
        s[var] = -s[var]
        de[var] = -de[var]


def _model_anneal_random(h, u, v, J, s, betas, spb, seed, gibbs):
    """Random order (cpu_sa.cpp:134-139) in speculative windows of the RNG
    stream: lane l takes position q + l as the variable draw of a possible
    attempt (var = rand % n) and position q + l + 1 as its acceptance draw.
    The attempts actually made form a chain (the next attempt's variable draw
    follows the previous attempt's draws); it is committed up to the first
    attempt whose variable an earlier accepted flip of the window touched
    (the flipped variable or a neighbour of it)."""
    n = len(h)
    rows = [[] for _ in range(n)]
    for a, b, w in zip(u, v, J):
        rows[a].append((int(b), float(w)))
        rows[b].append((int(a), float(w)))
    s = [int(x) for x in s]
    de = []
    for i in range(n):
        f = float(h[i])
        for t, w in rows[i]:
            f += s[t] * w
        de.append((-2 * s[i]) * f)
    R = _Ring(seed)
    for beta in betas:
        thr = 44.36142 / beta
        for _ in range(spb):
            rem = n
            while rem > 0:
                R.refill()
                var = [R.get(R.q + l) % n for l in range(32)]
                d = [de[x] for x in var]
                cons = [not (x >= thr) for x in d]
                need = [c if gibbs else (c and not x <= 0.0) for c, x in zip(cons, d)]
                chain, pos = [], 0
                while pos < 32 and len(chain) < rem:
                    chain.append(pos)
                    pos += 1 + int(need[pos])
                acc = {}
                for l in chain:
                    acc[l] = (not gibbs) and cons[l]
                    if need[l]:
                        r = float(R.get(R.q + l + 1))
                        if gibbs:
                            e = math.exp(d[l] * beta) if d[l] * beta < 709 else math.inf
                            acc[l] = 2.0 ** 64 > r * (1 + e)
                        else:
                            acc[l] = math.exp(-d[l] * beta) * 2.0 ** 64 > r
                touched, c = set(), len(chain)
                for i, l in enumerate(chain):
                    if var[l] in touched:
                        c = i
                        break
                    if acc[l]:
                        touched.add(var[l])
                        touched.update(t for t, _ in rows[var[l]])
                done = chain[:c]
                last = done[-1]
                R.q += last + 1 + int(need[last])
                rem -= len(done)
                flips = [var[l] for l in done if acc[l]]
                if flips:
                    _model_apply_flips(rows, de, s, flips)
    return np.array(s, np.int8)


@pytest.mark.parametrize("gibbs", [False, True])
def test_random_order_window_model_matches_oracle(gibbs):
    rng = np.random.default_rng(13 + gibbs)
    for n, p in ((90, 0.05), (40, 0.5), (7, 0.6)):
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(iu.shape[0]) < p
        u = np.concatenate([iu[keep], [2]]).astype(np.int32)   # and a self-loop
        v = np.concatenate([ju[keep], [2]]).astype(np.int32)
        J = rng.uniform(-1, 1, u.shape[0])
        h = rng.uniform(-1, 1, n)
        betas = np.geomspace(0.05, 4.0, 20)
        st = (2 * rng.integers(0, 2, (2, n)) - 1).astype(np.int8)
        seeds = np.array([9, 0], np.uint64)
        want, _ = oracle.run(h, u, v, J, st, 1, betas, seeds, True, gibbs)
        for r in range(2):
            got = _model_anneal_random(h, u, v, J, st[r], betas, 1, int(seeds[r]), gibbs)
            np.testing.assert_array_equal(got, want[r])


@pytest.mark.parametrize("gibbs", [False, True])
def test_in_window_resolution_model_matches_oracle(gibbs):
    """Passes that resolve in-window dependents (dense graphs, where almost
    every variable neighbours its successor, and a periodic lattice whose
    rows wrap inside the window) give the reference's results."""
    rng = np.random.default_rng(11 + gibbs)
    cases = []
    for n, p in ((70, 0.5), (45, 0.1)):
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(iu.shape[0]) < p
        cases.append((n, iu[keep].astype(np.int32), ju[keep].astype(np.int32),
                      rng.uniform(-1, 1, int(keep.sum())), rng.uniform(-1, 1, n)))
    L = 5
    lat = workloads.cubic_lattice(L=L, reads=1, sweeps=1, seed=3)
    cases.append((L ** 3, lat.u, lat.v, lat.J, lat.h))
    for n, u, v, J, h in cases:
        betas = np.geomspace(0.05, 4.0, 20)
        st = (2 * rng.integers(0, 2, (2, n)) - 1).astype(np.int8)
        seeds = np.array([5, 0], np.uint64)
        want, _ = oracle.run(h, u, v, J, st, 1, betas, seeds, False, gibbs)
        for r in range(2):
            got = _model_anneal(h, u, v, J, st[r], betas, 1, int(seeds[r]), gibbs, resolve=True)
            np.testing.assert_array_equal(got, want[r])


@pytest.mark.parametrize("gibbs", [False, True])
def test_speculative_window_model_matches_oracle(gibbs):
    rng = np.random.default_rng(7 + gibbs)
    for n, p in ((45, 0.08), (70, 0.5)):
        iu, ju = np.triu_indices(n, 1)
        keep = rng.random(iu.shape[0]) < p
        u = np.concatenate([iu[keep], [3, 9]]).astype(np.int32)   # a self-loop and a duplicate
        v = np.concatenate([ju[keep], [3, ju[keep][0]]]).astype(np.int32)
        u[-1] = iu[keep][0]
        J = rng.uniform(-1, 1, u.shape[0])
        h = rng.uniform(-1, 1, n)
        betas = np.geomspace(0.1, 4.0, 25)
        st = (2 * rng.integers(0, 2, (2, n)) - 1).astype(np.int8)
        seeds = np.array([3, 0], np.uint64)
        want, _ = oracle.run(h, u, v, J, st, 1, betas, seeds, False, gibbs)
        for r in range(2):
            got = _model_anneal(h, u, v, J, st[r], betas, 1, int(seeds[r]), gibbs)
            np.testing.assert_array_equal(got, want[r])


def test_bench_cpu_sample_checks_gpu_reads():
    """The benchmark's CPU-baseline leg compares every read it times with the
    GPU run's output: an oracle-made output passes, a corrupted read is
    counted as a mismatch."""
    import bench
    probs = workloads.uneven_batch(num_problems=3, n_range=(30, 60), reads_range=(2, 4),
                                   sweeps_range=(5, 10), seed=19)
    so = np.cumsum([0] + [p.num_reads * p.n for p in probs])
    ro = np.cumsum([0] + [p.num_reads for p in probs])
    states = np.zeros(so[-1], np.int8)
    energies = np.zeros(ro[-1])
    for k, p in enumerate(probs):
        s, e = oracle.run(p.h, p.u, p.v, p.J, p.states, p.sweeps_per_beta, p.betas, p.seeds)
        states[so[k]:so[k + 1]] = s.ravel()
        energies[ro[k]:ro[k + 1]] = e
    out = bench.cpu_sample(probs, 0, threads=2, max_reads=3, gpu_out=(states, energies, so, ro))
    assert out["checked_reads"] == 3 and out["mismatches"] == 0
    energies[ro[0]:ro[-1]] += 1.0
    out = bench.cpu_sample(probs, 0, threads=2, max_reads=3, gpu_out=(states, energies, so, ro))
    assert out["mismatches"] == 3
