"""Generate golden vectors from the reference's own simulated-annealing,
steepest-descent and SQA (rotor and path-integral) code.

    bash oracle/build_ref.sh            # reference extensions from their sources
    python tests/golden/make_golden.py  # writes tests/golden/*.npz and the
                                        # descent/, rotor/ and pimc/ subfolders

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


def descent_cases():
    """Steepest-descent fixtures: each runs in both solver modes.  The first
    restates the reference test tests/test_greedy.py:26-45 (convex section of
    a hyperbolic paraboloid).  No self-loops: a positive one makes the
    reference descend for ever."""
    rng = np.random.default_rng(20240602)
    out = {"convex": dict(h=np.array([2.0, 2.0]), u=np.array([0]), v=np.array([1]),
                          J=np.array([-1.0]), states0=np.array([[1, 1]], np.int8))}

    def sparse(n, m, integer):
        u = rng.integers(0, n, m)
        v = rng.integers(0, n, m)
        keep = u != v
        u, v = u[keep], v[keep]
        if integer:
            return rng.integers(-2, 3, n).astype(float), u, v, rng.integers(-2, 3, len(u)).astype(float)
        return rng.normal(0, 0.2, n), u, v, rng.normal(0, 1, len(u))

    h, u, v, J = sparse(300, 900, False)
    out["sparse300"] = dict(h=h, u=u, v=v, J=J, states0=states(rng, 32, 300))
    h, u, v, J = sparse(120, 400, True)  # many equal flip energies: lowest index wins
    out["integer_ties"] = dict(h=h, u=u, v=v, J=J, states0=states(rng, 32, 120))
    n = 50
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < 0.1]
    pairs = pairs + pairs[: len(pairs) // 3]  # repeated couplers
    out["duplicates"] = dict(h=rng.normal(0, 0.3, n), u=np.array([p[0] for p in pairs]),
                             v=np.array([p[1] for p in pairs]),
                             J=rng.normal(0, 1, len(pairs)), states0=states(rng, 16, n))
    n = 64
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n)]
    out["dense64"] = dict(h=rng.uniform(-1, 1, n), u=np.array([p[0] for p in pairs]),
                          v=np.array([p[1] for p in pairs]), J=rng.uniform(-1, 1, len(pairs)),
                          states0=states(rng, 16, n))
    h, u, v, J = sparse(2000, 6000, False)
    out["sparse2000"] = dict(h=h, u=u, v=v, J=J, states0=states(rng, 8, 2000))
    return out


def main_descent():
    mod = oracle.reference_descent_module()
    if mod is None:
        raise SystemExit("build the reference first: bash oracle/build_ref.sh")
    outdir = os.path.join(HERE, "descent")
    os.makedirs(outdir, exist_ok=True)
    for name, c in descent_cases().items():
        for mode in (False, True):
            h = np.asarray(c["h"], np.float64)
            u = np.asarray(c["u"], np.int32)
            v = np.asarray(c["v"], np.int32)
            J = np.asarray(c["J"], np.float64)
            s0 = np.asarray(c["states0"], np.int8)
            s, e, k = mod.steepest_gradient_descent(s0.shape[0], list(h), list(u), list(v),
                                                    list(J), s0.copy(), mode)
            tag = f"{name}_{'sparse' if mode else 'linear'}"
            np.savez_compressed(os.path.join(outdir, f"{tag}.npz"), h=h, u=u, v=v, J=J,
                                states0=s0, large_sparse_opt=np.array(mode),
                                out_states=np.asarray(s, np.int8),
                                out_energies=np.asarray(e, np.float64),
                                out_steps=np.asarray(k, np.uint32))
            print(f"descent/{tag}: samples={s0.shape[0]} n={len(h)} steps={int(np.sum(k))}")


def rotor_cases():
    """Rotor-model (SQA) fixtures: every proposal in both orders, statistics
    on, per-sample calls and one continued-stream call."""
    rng = np.random.default_rng(20240603)
    out = {}
    n = 40
    pairs = [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < 0.15]
    base = dict(h=rng.normal(0, 0.5, n), u=np.array([p[0] for p in pairs]),
                v=np.array([p[1] for p in pairs]), J=rng.normal(0, 1, len(pairs)),
                tf=rng.uniform(0.1, 2.0, n), spb=2, hp=np.geomspace(0.05, 4.0, 11),
                hd=np.geomspace(4.0, 0.02, 11), interval=3)
    for prop in ("GibbsNonErgodic", "MetropolisNonErgodic", "MetropolisUniform", "MetropolisTF"):
        for order in (False, True):
            for shared in (False, True):
                c = dict(base)
                c.update(states0=rng.integers(0, 256, (6, n)).astype(np.uint8),
                         seed=int(rng.integers(0, 2**31)), order=order, proposal=prop,
                         shared=shared)
                out[f"{prop}_{'random' if order else 'seq'}_{'shared' if shared else 'per_read'}"] = c
    return out


def main_rotor():
    mod = oracle.reference_rotormc_module()
    if mod is None:
        raise SystemExit("build the reference first: bash oracle/build_ref.sh")
    outdir = os.path.join(HERE, "rotor")
    os.makedirs(outdir, exist_ok=True)
    for name, c in rotor_cases().items():
        args = (list(map(float, c["h"])), list(map(int, c["u"])), list(map(int, c["v"])),
                list(map(float, c["J"])), list(map(float, c["tf"])), c["spb"], c["hp"], c["hd"])
        s0 = c["states0"]
        if c["shared"]:
            s, e, st = mod.simulated_annealing(s0.shape[0], *args, c["seed"], s0.copy(),
                                               c["order"], c["proposal"], c["interval"])
            s, e, st = np.asarray(s), np.asarray(e), np.asarray(st)
        else:
            outs = [mod.simulated_annealing(1, *args, c["seed"] + r, s0[r:r + 1].copy(),
                                            c["order"], c["proposal"], c["interval"])
                    for r in range(s0.shape[0])]
            s = np.concatenate([np.asarray(o[0]) for o in outs])
            e = np.concatenate([np.asarray(o[1]) for o in outs])
            st = np.concatenate([np.asarray(o[2]) for o in outs])
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), h=c["h"], u=c["u"].astype(np.int32),
                            v=c["v"].astype(np.int32), J=c["J"], tf=c["tf"], spb=c["spb"],
                            hp=c["hp"], hd=c["hd"], interval=c["interval"], states0=s0,
                            seed=np.uint64(c["seed"]), order=c["order"], proposal=c["proposal"],
                            shared=c["shared"], out_states=s.astype(np.uint8),
                            out_energies=e.astype(np.float64), out_stats=st.astype(np.uint8))
        print(f"rotor/{name}: samples={s0.shape[0]} n={len(c['h'])}")


def pimc_cases():
    """Path-integral (SQA) fixtures: single-qubit and chain updates, per-sample
    calls and continued-stream calls, statistics, final break positions (with
    a buffer too small for all of them in one case), quantum initial states,
    no transverse field, self-loops and repeated couplers."""
    rng = np.random.default_rng(20240715)
    out = {}

    def problem(n, p, extra=()):
        pairs = [(a, b) for a in range(n) for b in range(a + 1, n) if rng.random() < p]
        pairs += list(extra)
        return dict(h=rng.normal(0, 0.4, n), u=np.array([q[0] for q in pairs], np.int32),
                    v=np.array([q[1] for q in pairs], np.int32), J=rng.normal(0, 1, len(pairs)))

    def case(name, prob, R, hp, hd, spb=2, qpc=1, qpu=1, jchain=1.0, shared=False, interval=0,
             proj_in=True, proj_out=False, out_size=1 << 16):
        n = len(prob["h"])
        c = dict(prob, states0=states(rng, R, n), spb=spb, hp=np.asarray(hp, np.float64),
                 hd=np.asarray(hd, np.float64), qpc=qpc, qpu=qpu, jchain=jchain,
                 seed=int(rng.integers(1, 2**31)), shared=shared, interval=interval,
                 proj_in=proj_in, proj_out=proj_out, out_size=out_size)
        nb = np.zeros((R, n), np.intc)
        bin_ = np.zeros(1, np.intc)
        if not proj_in:  # n increasing positions per variable
            nb[:] = n
            bin_ = np.concatenate([np.sort(rng.choice(65536, n, replace=False))
                                   for _ in range(R * n)]).astype(np.intc)
        c.update(num_breaks0=nb, breaks_in=bin_)
        out[name] = c

    p24 = problem(24, 0.2)
    ramp = (np.geomspace(0.1, 3.0, 12), np.geomspace(4.0, 0.05, 12))
    case("qubit_per_read", p24, 6, *ramp, interval=3)
    case("qubit_shared", p24, 5, *ramp, shared=True, interval=4)
    case("qubit_high_field", p24, 5, np.full(6, 0.7), np.full(6, 8.0))
    case("qubit_no_field", p24, 5, np.geomspace(0.2, 4.0, 8), np.zeros(8), proj_out=True)
    case("qubit_small_buffer", p24, 4, np.full(5, 0.8), np.full(5, 6.0), shared=True,
         out_size=300)
    p16 = problem(16, 0.2)
    case("chain4_per_read", p16, 5, np.geomspace(0.2, 2.0, 8), np.full(8, 5.0), qpc=4, qpu=4,
         jchain=-1.8)
    case("chain2_shared", p16, 4, *ramp, qpc=2, qpu=2, jchain=-3.0, shared=True, interval=2)
    p18 = problem(18, 0.2)
    case("chain3_per_read", p18, 4, np.full(6, 0.5), np.full(6, 12.0), qpc=3, qpu=3,
         jchain=-0.4)
    p8 = problem(8, 0.3)
    case("quantum_inputs", p8, 3, np.geomspace(0.2, 2.0, 5), np.full(5, 2.0), proj_in=False)
    loops = problem(10, 0.25, extra=[(2, 2), (3, 7), (3, 7), (7, 3)])
    case("self_loops_repeats", loops, 4, np.full(6, 1.0), np.full(6, 3.0))
    # Any qubits_per_update other than 1 updates whole chains of qubits_per_chain;
    # with 1, chains are ignored.
    case("chain3_update2", p18, 3, np.full(5, 0.6), np.full(5, 4.0), qpc=3, qpu=2,
         jchain=-1.0)
    case("qubit_ignores_chains", p16, 3, np.full(5, 0.6), np.full(5, 4.0), qpc=4, qpu=1,
         jchain=-1.0)
    return out


def main_pimc():
    mod = oracle.reference_pimc_module()
    if mod is None:
        raise SystemExit("build the reference first: bash oracle/build_ref.sh")
    outdir = os.path.join(HERE, "pimc")
    os.makedirs(outdir, exist_ok=True)
    for name, c in pimc_cases().items():
        s0 = c["states0"]
        R, n = s0.shape
        args = (list(map(float, c["h"])), list(map(int, c["u"])), list(map(int, c["v"])),
                list(map(float, c["J"])), c["spb"], c["hp"], c["hd"], 1.0, c["jchain"],
                c["qpc"], c["qpu"])
        if c["shared"]:
            bo = np.zeros(c["out_size"], np.intc)
            s, e, st, nb, bo = mod.simulated_annealing(
                R, *args, c["seed"], s0.copy(), c["proj_in"], c["proj_out"],
                c["num_breaks0"].copy(), c["breaks_in"].copy(), bo, c["interval"])
            s, e, st, nb = map(np.asarray, (s, e, st, nb))
        else:
            outs, bufs = [], []
            per = n * n if not c["proj_in"] else 0
            for r in range(R):
                bo = np.zeros(c["out_size"], np.intc)
                bin_r = c["breaks_in"][r * per:(r + 1) * per] if per else c["breaks_in"]
                o = mod.simulated_annealing(
                    1, *args, c["seed"] + r, s0[r:r + 1].copy(), c["proj_in"], c["proj_out"],
                    c["num_breaks0"][r:r + 1].copy(), np.ascontiguousarray(bin_r), bo,
                    c["interval"])
                outs.append(o)
                bufs.append(np.asarray(o[4])[:int(np.asarray(o[3]).sum())])
            s = np.concatenate([np.asarray(o[0]) for o in outs])
            e = np.concatenate([np.asarray(o[1]) for o in outs])
            st = np.concatenate([np.asarray(o[2]) for o in outs])
            nb = np.concatenate([np.asarray(o[3]) for o in outs])
            bo = np.zeros(c["out_size"], np.intc)
            flat = np.concatenate(bufs) if bufs else np.zeros(0, np.intc)
            bo[:len(flat)] = flat
        if not c["interval"]:  # the binding returns an uninitialised array then
            st = np.zeros_like(np.asarray(st))
        np.savez_compressed(os.path.join(outdir, f"{name}.npz"), **c, out_states=s.astype(np.int8),
                            out_energies=e.astype(np.float64), out_stats=st.astype(np.int8),
                            out_num_breaks=nb.astype(np.intc), out_breaks=np.asarray(bo, np.intc))
        print(f"pimc/{name}: samples={R} n={n} breaks={int(nb.sum()) if not c['proj_out'] else '-'}")


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
    main_descent()
    main_rotor()
    main_pimc()
