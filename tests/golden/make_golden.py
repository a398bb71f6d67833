"""Generate golden vectors from the reference's own simulated-annealing code.

    bash oracle/build_ref.sh            # reference extension from its sources
    python tests/golden/make_golden.py  # writes tests/golden/*.npz

Each fixture stores the inputs and the reference's outputs.  Per-read
fixtures hold, for each read r, the result of one reference call with
num_samples=1 and seed=seeds[r].  "shared" fixtures hold one reference call
over all reads with a single seed (one RNG stream continued across reads).
The first case restates the problem of the reference test
tests/test_simulated_annealing.py:96-122 (ferromagnet with self-loops).
"""
from __future__ import annotations

import os
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, os.path.join(ROOT, "oracle"))
import oracle  # noqa: E402


def states(rng, R, n):
    return (2 * rng.integers(0, 2, size=(R, n)) - 1).astype(np.int8)


def run_reference(case):
    mod = oracle.reference_module()
    crit = "Gibbs" if case["proposal"] == 0 else "Metropolis"
    order = bool(case["order"])
    args = (list(map(float, case["h"])), list(map(int, case["u"])),
            list(map(int, case["v"])), list(map(float, case["J"])),
            int(case["spb"]), np.asarray(case["betas"], dtype=float))
    s0 = case["states0"]
    if case["shared"]:
        s, e = mod.simulated_annealing(s0.shape[0], *args[:5], args[5],
                                       int(case["seeds"][0]), s0.copy(), order, crit)
        return np.array(s), np.array(e)
    outs, ens = [], []
    for r in range(s0.shape[0]):
        s, e = mod.simulated_annealing(1, *args[:5], args[5], int(case["seeds"][r]),
                                       s0[r:r + 1].copy(), order, crit)
        outs.append(np.array(s[0]))
        ens.append(e[0])
    return np.stack(outs), np.array(ens)


def cases():
    rng = np.random.default_rng(20240601)
    out = {}

    # tests/test_simulated_annealing.py:96-122 problem (self-loops u == v).
    n = 10
    pairs = [(u, v) for u in range(n) for v in range(u, n)]
    fm = dict(h=-np.ones(n), u=np.array([p[0] for p in pairs]), v=np.array([p[1] for p in pairs]),
              J=-np.ones(len(pairs)), betas=np.linspace(0.01, 3, num=1000), spb=1,
              states0=(2 * np.random.RandomState(1234).randint(2, size=(100, n)).astype(np.int8) - 1),
              order=0, proposal=1)
    out["fm_shared"] = dict(fm, seeds=np.array([1], np.uint64), shared=True)
    out["fm_per_read"] = dict(fm, seeds=np.arange(1, 101, dtype=np.uint64), shared=False)

    # Dense n=100, edge prob 0.5, U[-1,1] (the dense benchmark shape, fewer reads).
    n = 100
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.5
    out["dense100"] = dict(h=rng.uniform(-1, 1, n), u=iu[keep], v=ju[keep],
                           J=rng.uniform(-1, 1, int(keep.sum())),
                           betas=np.geomspace(0.1, 4.2, 1000), spb=1, states0=states(rng, 8, n),
                           order=0, proposal=1, seeds=np.arange(1000, 1008, dtype=np.uint64),
                           shared=False)

    # Periodic cubic lattice L=8, J=+-1, h=0.
    L = 8
    x, y, z = [a.ravel() for a in np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")]
    idx = (x * L + y) * L + z
    nb = np.stack([(((x + 1) % L) * L + y) * L + z, (x * L + (y + 1) % L) * L + z,
                   (x * L + y) * L + (z + 1) % L], 1).ravel()
    m = nb.shape[0]
    out["lattice8"] = dict(h=np.zeros(L ** 3), u=np.repeat(idx, 3), v=nb,
                           J=np.where(rng.random(m) < 0.5, -1.0, 1.0),
                           betas=np.linspace(0.1, 3.0, 256), spb=1, states0=states(rng, 4, L ** 3),
                           order=0, proposal=1, seeds=np.arange(2000, 2004, dtype=np.uint64),
                           shared=False)

    # Random 7-regular-like sparse graph, J~N(0,1), h~N(0,0.1).
    n = 300
    perm = np.concatenate([rng.permutation(n) for _ in range(7)])
    a, b = perm[: len(perm) // 2 * 2].reshape(-1, 2).T
    ok = a != b
    a, b = np.minimum(a[ok], b[ok]), np.maximum(a[ok], b[ok])
    out["sparse300"] = dict(h=rng.normal(0, 0.1, n), u=a, v=b, J=rng.normal(0, 1, a.shape[0]),
                            betas=np.geomspace(0.1, 5.0, 300), spb=1, states0=states(rng, 4, n),
                            order=0, proposal=1, seeds=np.arange(3000, 3004, dtype=np.uint64),
                            shared=False)

    # K16 fixed beta=1 Gibbs (the autograd shape, fewer sweeps/reads).
    n = 16
    iu, ju = np.triu_indices(n, 1)
    out["k16_gibbs"] = dict(h=rng.normal(0, 0.1, n), u=iu, v=ju, J=rng.normal(0, 0.3, iu.shape[0]),
                            betas=np.array([1.0]), spb=500, states0=states(rng, 32, n),
                            order=0, proposal=0, seeds=np.arange(4000, 4032, dtype=np.uint64),
                            shared=False)

    # Random order, both acceptance rules.
    n = 50
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.1
    base = dict(h=rng.uniform(-1, 1, n), u=iu[keep], v=ju[keep], J=rng.uniform(-1, 1, int(keep.sum())),
                betas=np.geomspace(0.2, 3.0, 100), spb=1, states0=states(rng, 4, n), order=1,
                seeds=np.arange(5000, 5004, dtype=np.uint64), shared=False)
    out["random_metropolis"] = dict(base, proposal=1)
    out["random_gibbs"] = dict(base, proposal=0)
    out["random_metropolis_shared"] = dict(base, proposal=1, seeds=np.array([77], np.uint64), shared=True)

    # Beta edge values: 0 (threshold inf), inf (threshold 0), tiny, huge; 2 sweeps each.
    n = 40
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.2
    base = dict(h=rng.uniform(-1, 1, n), u=iu[keep], v=ju[keep], J=rng.uniform(-1, 1, int(keep.sum())),
                betas=np.array([0.0, 0.5, np.inf, 1e-300, 1e300, 2.0]), spb=2,
                states0=states(rng, 4, n), order=0, seeds=np.array([0, 1, 2**63, 2**64 - 1], np.uint64),
                shared=False)
    out["beta_edges_metropolis"] = dict(base, proposal=1)
    out["beta_edges_gibbs"] = dict(base, proposal=0)

    # Self-loops and repeated couplers with real weights, both rules.
    n = 30
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.25
    u = np.concatenate([iu[keep], np.arange(0, n, 3), iu[keep][:12]])
    v = np.concatenate([ju[keep], np.arange(0, n, 3), ju[keep][:12]])
    base = dict(h=rng.uniform(-1, 1, n), u=u, v=v, J=rng.uniform(-1, 1, u.shape[0]),
                betas=np.geomspace(0.1, 4.0, 200), spb=1, states0=states(rng, 4, n), order=0,
                seeds=np.arange(6000, 6004, dtype=np.uint64), shared=False)
    out["dups_metropolis"] = dict(base, proposal=1)
    out["dups_gibbs"] = dict(base, proposal=0)

    # Empty schedule (num_sweeps = 0): states unchanged, energies computed.
    out["zero_sweeps"] = dict(base, betas=np.zeros(0), proposal=1)

    # Null model (no fields, no couplers): Metropolis sequential flips every spin.
    n = 64
    out["null_model"] = dict(h=np.zeros(n), u=np.zeros(0, int), v=np.zeros(0, int), J=np.zeros(0),
                             betas=np.array([0.1, 0.55, 1.0]), spb=1, states0=states(rng, 3, n),
                             order=0, proposal=1, seeds=np.arange(7000, 7003, dtype=np.uint64),
                             shared=False)

    # Huge fields: exp over/underflow and infinite products in Gibbs.
    n = 24
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.3
    out["huge_gibbs"] = dict(h=rng.uniform(-1, 1, n) * 1e3, u=iu[keep], v=ju[keep],
                             J=rng.uniform(-1, 1, int(keep.sum())) * 300.0,
                             betas=np.geomspace(0.01, 10.0, 50), spb=1, states0=states(rng, 4, n),
                             order=0, proposal=0, seeds=np.arange(8000, 8004, dtype=np.uint64),
                             shared=False)

    # Spin values other than +-1 (the reference applies int8 arithmetic as is).
    n = 20
    iu, ju = np.triu_indices(n, 1)
    keep = rng.random(iu.shape[0]) < 0.3
    odd = rng.integers(-2, 3, size=(3, n)).astype(np.int8)
    out["odd_spins"] = dict(h=rng.uniform(-1, 1, n), u=iu[keep], v=ju[keep],
                            J=rng.uniform(-1, 1, int(keep.sum())), betas=np.geomspace(0.1, 3.0, 30),
                            spb=1, states0=odd, order=0, proposal=1,
                            seeds=np.arange(9000, 9003, dtype=np.uint64), shared=False)
    return out


def main():
    if oracle.reference_module() is None:
        raise SystemExit("build the reference first: bash oracle/build_ref.sh")
    for name, c in cases().items():
        c = dict(c)
        c["h"] = np.asarray(c["h"], np.float64)
        c["u"] = np.asarray(c["u"], np.int32)
        c["v"] = np.asarray(c["v"], np.int32)
        c["J"] = np.asarray(c["J"], np.float64)
        c["betas"] = np.asarray(c["betas"], np.float64)
        c["seeds"] = np.asarray(c["seeds"], np.uint64)
        s, e = run_reference(c)
        np.savez_compressed(os.path.join(HERE, f"{name}.npz"), out_states=s.astype(np.int8),
                            out_energies=e.astype(np.float64), **c)
        print(f"{name}: reads={s.shape[0]} n={s.shape[1]} couplers={c['J'].shape[0]}")


if __name__ == "__main__":
    main()
