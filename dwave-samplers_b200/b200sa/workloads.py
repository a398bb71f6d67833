"""Seeded synthetic Ising instances with the shapes of the benchmark workloads.

Every generator is deterministic in its seed and returns COO couplers in
generation order (that order fixes adjacency and energy summation order) plus
uniform +-1 int8 initial states.  The reference publishes no benchmark
instances; these stand in for them.

    dense_ising        n=100 dense, edge prob 0.5, J,h ~ U[-1,1]; 1000 reads x 1000
                       geometric sweeps 0.1->4.2, Metropolis, sequential
    cubic_lattice      3D periodic L=32 (32768 spins), J=+-1, h=0; 256 reads x 4096
                       linear sweeps 0.1->3.0
    uneven_batch       512 random-regular problems, n~U[64,4096], degree~U{3..16},
                       J~N(0,1), h~N(0,0.1), reads~U[32,1024], sweeps~U[256,2048],
                       geometric 0.1->5.0
    complete_graph     K16, J~N(0,0.3), h~N(0,0.1) (fixed beta Gibbs)
    bm_models          64 six-regular models, n~U[256,2048], J*~N(0,0.5), h*=0
"""
from __future__ import annotations

from dataclasses import dataclass, field

import numpy as np

from .simulated_annealing import per_read_seeds


@dataclass
class Instance:
    h: np.ndarray                 # float64 [n]
    u: np.ndarray                 # int32 [m]
    v: np.ndarray                 # int32 [m]
    J: np.ndarray                 # float64 [m]
    states: np.ndarray            # int8 [R, n] initial states
    betas: np.ndarray             # float64 beta schedule
    sweeps_per_beta: int = 1
    seeds: np.ndarray = field(default_factory=lambda: np.zeros(0, np.uint64))
    randomize_order: bool = False
    proposal: str = "Metropolis"

    @property
    def n(self) -> int:
        return int(self.h.shape[0])

    @property
    def num_reads(self) -> int:
        return int(self.states.shape[0])

    @property
    def attempts(self) -> int:
        """Spin-flip attempts: reads x sweeps x n."""
        return self.num_reads * self.sweeps_per_beta * len(self.betas) * self.n


def random_states(rng: np.random.Generator, reads: int, n: int) -> np.ndarray:
    return (2 * rng.integers(0, 2, size=(reads, n), dtype=np.int8) - 1).astype(np.int8)


def dense_ising(n=100, p=0.5, reads=1000, sweeps=1000, beta_range=(0.1, 4.2),
                seed=1, base_seed=1000) -> Instance:
    rng = np.random.default_rng(seed)
    iu, ju = np.triu_indices(n, k=1)  # lexicographic i<j
    keep = rng.random(iu.shape[0]) < p
    u = iu[keep].astype(np.int32)
    v = ju[keep].astype(np.int32)
    J = rng.uniform(-1.0, 1.0, u.shape[0])
    h = rng.uniform(-1.0, 1.0, n)
    states = random_states(rng, reads, n)
    betas = np.geomspace(beta_range[0], beta_range[1], sweeps)
    return Instance(h, u, v, J, states, betas, 1, per_read_seeds(base_seed, reads))


def cubic_lattice(L=32, reads=256, sweeps=4096, beta_range=(0.1, 3.0), seed=2,
                  base_seed=2000) -> Instance:
    rng = np.random.default_rng(seed)
    x, y, z = np.meshgrid(np.arange(L), np.arange(L), np.arange(L), indexing="ij")
    x, y, z = x.ravel(), y.ravel(), z.ravel()
    idx = (x * L + y) * L + z
    nx_ = (((x + 1) % L) * L + y) * L + z
    ny_ = (x * L + (y + 1) % L) * L + z
    nz_ = (x * L + y) * L + (z + 1) % L
    # per site, in index order: +x, +y, +z
    u = np.repeat(idx, 3).astype(np.int32)
    v = np.stack([nx_, ny_, nz_], axis=1).ravel().astype(np.int32)
    J = np.where(rng.random(u.shape[0]) < 0.5, -1.0, 1.0)
    n = L ** 3
    h = np.zeros(n)
    states = random_states(rng, reads, n)
    betas = np.linspace(beta_range[0], beta_range[1], sweeps)
    return Instance(h, u, v, J, states, betas, 1, per_read_seeds(base_seed, reads))


def random_regular(n, d, rng: np.random.Generator, graph_seed: int):
    """Random d-regular graph (networkx), edges sorted u<v lexicographically.
    If n*d is odd, n is increased by one."""
    import networkx as nx
    if (n * d) % 2:
        n += 1
    g = nx.random_regular_graph(d, n, seed=graph_seed)
    e = np.array(sorted((min(a, b), max(a, b)) for a, b in g.edges()), dtype=np.int32)
    return n, e[:, 0].copy(), e[:, 1].copy()


def uneven_batch(num_problems=512, n_range=(64, 4096), d_range=(3, 16),
                 reads_range=(32, 1024), sweeps_range=(256, 2048),
                 beta_range=(0.1, 5.0), seed=3, base_seed=3000) -> list[Instance]:
    rng = np.random.default_rng(seed)
    out = []
    next_seed = base_seed
    for p in range(num_problems):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        d = int(rng.integers(d_range[0], d_range[1] + 1))
        R = int(rng.integers(reads_range[0], reads_range[1] + 1))
        S = int(rng.integers(sweeps_range[0], sweeps_range[1] + 1))
        n, u, v = random_regular(n, d, rng, graph_seed=int(rng.integers(2**31)))
        J = rng.normal(0.0, 1.0, u.shape[0])
        h = rng.normal(0.0, 0.1, n)
        states = random_states(rng, R, n)
        betas = np.geomspace(beta_range[0], beta_range[1], S)
        out.append(Instance(h, u, v, J, states, betas, 1, per_read_seeds(next_seed, R)))
        next_seed += R
    return out


def complete_graph(n=16, J_sigma=0.3, h_sigma=0.1, reads=4096, sweeps=10000, beta=1.0,
                   seed=4, base_seed=4000) -> Instance:
    rng = np.random.default_rng(seed)
    iu, ju = np.triu_indices(n, k=1)
    J = rng.normal(0.0, J_sigma, iu.shape[0])
    h = rng.normal(0.0, h_sigma, n)
    states = random_states(rng, reads, n)
    return Instance(h, iu.astype(np.int32), ju.astype(np.int32), J, states,
                    np.array([beta]), sweeps, per_read_seeds(base_seed, reads),
                    proposal="Gibbs")


def bm_models(num_models=64, n_range=(256, 2048), d=6, J_sigma=0.5, seed=5):
    """Ground-truth sparse models for Boltzmann-machine learning:
    list of (h*, u, v, J*) with h* = 0."""
    rng = np.random.default_rng(seed)
    models = []
    for _ in range(num_models):
        n = int(rng.integers(n_range[0], n_range[1] + 1))
        n, u, v = random_regular(n, d, rng, graph_seed=int(rng.integers(2**31)))
        J = rng.normal(0.0, J_sigma, u.shape[0])
        models.append((np.zeros(n), u, v, J))
    return models
