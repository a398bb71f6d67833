"""Python access to the CPU oracle.  TEST INFRASTRUCTURE ONLY.

Only ``tests/``, ``__graft_entry__.smoke()`` and the CPU-baseline legs of
``bench.py`` import this module; the product package never does.

Two oracles are exposed:

* :func:`run` -- the C restatement in ``oracle/sa_oracle.c`` of the
  reference's ``general_simulated_annealing`` (dwave-samplers 1.8.0,
  ``dwave/samplers/sa/src/cpu_sa.cpp:253-362``).
* :func:`reference_module` -- the reference's own Cython extension
  (``dwave/samplers/sa/simulated_annealing.pyx``) built from its sources by
  ``oracle/build_ref.sh`` into ``oracle/_ref/``, when that build exists.
* :func:`rotormc` -- the C restatement of the reference's rotor-model
  (SQA) annealing (``dwave/samplers/sqa/src/cpu_rotormc.cpp:368-563``), and
  :func:`reference_rotormc_module`, its own extension built the same way.
* :func:`pimc` -- the C restatement of the reference's path-integral Monte
  Carlo annealing (``dwave/samplers/sqa/src/localPIMC.cpp``), with
  :func:`mt19937`, and :func:`reference_pimc_module`, its own extension.
* :func:`descent` -- the C restatement of the reference's steepest descent
  (``dwave/samplers/greedy/src/descent.cpp:315-405``), and
  :func:`reference_descent_module`, the reference's own ``descent`` extension
  built the same way.
"""
from __future__ import annotations

import ctypes
import importlib.util
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(HERE, "libsa_oracle.so")
_REF_DIR = os.path.join(HERE, "_ref")

_lib = None
_ref = None


def build() -> str:
    """Compile the C restatement (plain gcc) if it is missing or stale."""
    srcs = [os.path.join(HERE, f) for f in ("sa_oracle.c", "pimc_oracle.c")]
    if (not os.path.exists(_LIB_PATH)
            or os.path.getmtime(_LIB_PATH) < max(map(os.path.getmtime, srcs))):
        subprocess.check_call(["make", "-s", "-C", HERE, "libsa_oracle.so"])
    return _LIB_PATH


def lib() -> ctypes.CDLL:
    global _lib
    if _lib is None:
        build()
        L = ctypes.CDLL(_LIB_PATH)
        L.sa_oracle_run.restype = ctypes.c_int
        L.sa_oracle_run.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.sa_oracle_energy.restype = ctypes.c_double
        L.sa_oracle_energy.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.sd_oracle_run.restype = ctypes.c_int
        L.sd_oracle_run.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int]
        L.rmc_oracle_run.restype = ctypes.c_int
        L.rmc_oracle_run.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.pimc_oracle_run.restype = ctypes.c_int
        L.pimc_oracle_run.argtypes = [
            ctypes.c_int, ctypes.c_void_p, ctypes.c_long, ctypes.c_void_p, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
            ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_double, ctypes.c_int,
            ctypes.c_int, ctypes.c_uint32, ctypes.c_int, ctypes.c_int, ctypes.c_void_p,
            ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, ctypes.c_int]
        L.pimc_oracle_mt.restype = None
        L.pimc_oracle_mt.argtypes = [ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p]
        L.sa_oracle_rng_stream.restype = None
        L.sa_oracle_rng_stream.argtypes = [ctypes.c_uint64, ctypes.c_int,
                                           ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a: np.ndarray) -> int:
    return a.ctypes.data


def run(h, u, v, J, states, sweeps_per_beta, betas, seeds,
        randomize_order=False, gibbs=False):
    """Anneal ``states`` (R x n int8, copied) with the C restatement.

    ``seeds`` is either one seed (one stream continued across reads, the
    reference's multi-read behaviour) or one seed per read (each read equal to
    a reference call with ``num_samples=1, seed=seeds[r]``).
    Returns ``(states, energies)``.
    """
    h = np.ascontiguousarray(h, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    J = np.ascontiguousarray(J, dtype=np.float64)
    st = np.array(states, dtype=np.int8, order="C", copy=True)
    if st.ndim != 2 or st.shape[1] != h.shape[0]:
        raise ValueError("states must be (num_reads, num_vars)")
    betas = np.ascontiguousarray(betas, dtype=np.float64)
    seeds = np.atleast_1d(np.asarray(seeds, dtype=np.uint64))
    R, n = st.shape
    en = np.zeros(R, dtype=np.float64)
    rc = lib().sa_oracle_run(
        n, _ptr(h), len(J), _ptr(u), _ptr(v), _ptr(J), R, _ptr(st), _ptr(en),
        int(sweeps_per_beta), len(betas), _ptr(betas), _ptr(seeds), len(seeds),
        int(bool(randomize_order)), int(bool(gibbs)))
    if rc < 0:
        raise ValueError(f"oracle error {rc}")
    return st, en


def energy(h, u, v, J, state) -> float:
    h = np.ascontiguousarray(h, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    J = np.ascontiguousarray(J, dtype=np.float64)
    s = np.ascontiguousarray(state, dtype=np.int8)
    return lib().sa_oracle_energy(len(h), _ptr(h), len(J), _ptr(u), _ptr(v),
                                  _ptr(J), _ptr(s))


def rng_stream(seed: int, count: int) -> np.ndarray:
    out = np.zeros(count, dtype=np.uint64)
    lib().sa_oracle_rng_stream(int(seed), int(count), _ptr(out))
    return out


def descent(h, u, v, J, states, large_sparse_opt=False):
    """Steepest descent from every row of ``states`` (copied) with the C
    restatement.  Returns (states, energies, steps)."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    J = np.ascontiguousarray(J, dtype=np.float64)
    st = np.array(states, dtype=np.int8, order="C", copy=True)
    R = st.shape[0]
    en = np.zeros(R, dtype=np.float64)
    steps = np.zeros(R, dtype=np.uint32)
    rc = lib().sd_oracle_run(len(h), _ptr(h), len(J), _ptr(u), _ptr(v), _ptr(J), R, _ptr(st),
                             _ptr(en), _ptr(steps), 1 if large_sparse_opt else 0)
    if rc < 0:
        raise ValueError(f"oracle error {rc}")
    return st, en, steps


ROTOR_PROPOSALS = {"GibbsNonErgodic": 0, "MetropolisNonErgodic": 1, "MetropolisUniform": 2,
                   "MetropolisTF": 3}


def rotormc(h, u, v, J, trans_fields, states, sweeps_per_beta, hp, hd, seeds,
            randomize_order=False, proposal="MetropolisNonErgodic", interval=0):
    """Rotor-model annealing of every row of ``states`` (uint8 angles, copied).
    ``seeds``: one seed (one stream across samples) or one per sample.  Returns
    (states, energies, statistics) with statistics (samples, points, n), one
    block per sample."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    J = np.ascontiguousarray(J, dtype=np.float64)
    tf = np.ascontiguousarray(trans_fields, dtype=np.float64)
    hp = np.ascontiguousarray(hp, dtype=np.float64)
    hd = np.ascontiguousarray(hd, dtype=np.float64)
    seeds = np.atleast_1d(np.asarray(seeds, dtype=np.uint64))
    st = np.array(states, dtype=np.uint8, order="C", copy=True)
    R, n = st.shape
    en = np.zeros(R, dtype=np.float64)
    points = 1 + (len(hp) - 1) // interval if interval else 0
    stats = np.zeros((R, max(points, 1), n), dtype=np.uint8)
    rc = lib().rmc_oracle_run(n, _ptr(h), len(J), _ptr(u), _ptr(v), _ptr(J), _ptr(tf), R,
                              _ptr(st), _ptr(en), int(sweeps_per_beta), len(hp), _ptr(hp),
                              _ptr(hd), _ptr(seeds), len(seeds), 1 if randomize_order else 0,
                              ROTOR_PROPOSALS[proposal], _ptr(stats) if interval else None,
                              int(interval))
    if rc < 0:
        raise ValueError(f"oracle error {rc}")
    return st, en, stats[:, :points]


def pimc(h, u, v, J, states, sweeps_per_beta, hp, hd, seed, chain_coupler_strength=1.0,
         qubits_per_chain=1, qubits_per_update=1, project_inputs=True, project_outputs=True,
         num_breaks=None, breaks_in=None, interval=0, max_out=64):
    """Path-integral Monte Carlo annealing of every row of ``states`` (int8,
    copied) as ONE reference call (one mt19937 stream across the samples).
    Returns (states, energies, statistics (samples, points, n), num_breaks
    (samples, n), breaks (samples, n, max_out): the final break positions of
    every variable, valid up to num_breaks)."""
    h = np.ascontiguousarray(h, dtype=np.float64)
    u = np.ascontiguousarray(u, dtype=np.int32)
    v = np.ascontiguousarray(v, dtype=np.int32)
    J = np.ascontiguousarray(J, dtype=np.float64)
    hp = np.ascontiguousarray(hp, dtype=np.float64)
    hd = np.ascontiguousarray(hd, dtype=np.float64)
    st = np.array(states, dtype=np.int8, order="C", copy=True)
    R, n = st.shape
    en = np.zeros(R, dtype=np.float64)
    points = 1 + (len(hp) - 1) // interval if interval else 0
    stats = np.zeros((R, max(points, 1), n), dtype=np.int8)
    nbk = (np.zeros((R, n), dtype=np.int32) if num_breaks is None
           else np.array(num_breaks, dtype=np.int32, order="C", copy=True))
    bin_ = np.ascontiguousarray(np.zeros(1) if breaks_in is None else breaks_in, dtype=np.int32)
    bout = np.zeros((R, n, max_out), dtype=np.int32)
    rc = lib().pimc_oracle_run(n, _ptr(h), len(J), _ptr(u), _ptr(v), _ptr(J), R, _ptr(st),
                               _ptr(en), int(sweeps_per_beta), len(hp), _ptr(hp), _ptr(hd),
                               float(chain_coupler_strength), int(qubits_per_chain),
                               int(qubits_per_update), int(seed), 1 if project_inputs else 0,
                               1 if project_outputs else 0, _ptr(nbk), _ptr(bin_), _ptr(bout),
                               int(max_out), _ptr(stats) if interval else None, int(interval))
    if rc == -2:
        raise ValueError("a variable ended with more than max_out breaks")
    if rc < 0:
        raise ValueError(f"oracle error {rc}")
    return st, en, stats[:, :points], nbk, bout


def mt19937(seed, count):
    """First ``count`` outputs of std::mt19937(seed) as restated by the oracle."""
    out = np.zeros(count, dtype=np.uint32)
    lib().pimc_oracle_mt(int(seed), int(count), _ptr(out))
    return out


_ref_pimc = None


def reference_pimc_module():
    """The reference's path-integral annealing extension built from source, or None."""
    global _ref_pimc
    if _ref_pimc is not None:
        return _ref_pimc
    if not os.path.isdir(_REF_DIR):
        return None
    for name in os.listdir(_REF_DIR):
        if name.startswith("pimc_annealing") and name.endswith(".so"):
            spec = importlib.util.spec_from_file_location(
                "pimc_annealing", os.path.join(_REF_DIR, name))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            _ref_pimc = mod
            return _ref_pimc
    return None


_ref_rotormc = None


def reference_rotormc_module():
    """The reference's rotor-model annealing extension built from source, or None."""
    global _ref_rotormc
    if _ref_rotormc is not None:
        return _ref_rotormc
    if not os.path.isdir(_REF_DIR):
        return None
    for name in os.listdir(_REF_DIR):
        if name.startswith("rotormc_annealing") and name.endswith(".so"):
            spec = importlib.util.spec_from_file_location(
                "rotormc_annealing", os.path.join(_REF_DIR, name))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            _ref_rotormc = mod
            return _ref_rotormc
    return None


_ref_descent = None


def reference_descent_module():
    """The reference's steepest-descent extension built from source, or None."""
    global _ref_descent
    if _ref_descent is not None:
        return _ref_descent
    if not os.path.isdir(_REF_DIR):
        return None
    for name in os.listdir(_REF_DIR):
        if name.startswith("descent") and name.endswith(".so"):
            spec = importlib.util.spec_from_file_location("descent", os.path.join(_REF_DIR, name))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            _ref_descent = mod
            return _ref_descent
    return None


def reference_module():
    """The reference extension built from source, or None if not built."""
    global _ref
    if _ref is not None:
        return _ref
    if not os.path.isdir(_REF_DIR):
        return None
    for name in os.listdir(_REF_DIR):
        if name.startswith("simulated_annealing") and name.endswith(".so"):
            spec = importlib.util.spec_from_file_location(
                "simulated_annealing", os.path.join(_REF_DIR, name))
            mod = importlib.util.module_from_spec(spec)
            spec.loader.exec_module(mod)
            _ref = mod
            return _ref
    return None


def reference_per_read(h, u, v, J, states, sweeps_per_beta, betas, seeds,
                       randomize_order=False, proposal="Metropolis"):
    """Run the reference extension once per read (num_samples=1, seed=seeds[r])."""
    mod = reference_module()
    if mod is None:
        raise RuntimeError("reference extension not built (oracle/build_ref.sh)")
    st = np.array(states, dtype=np.int8, order="C", copy=True)
    en = np.zeros(st.shape[0])
    hl, ul, vl, Jl = list(map(float, h)), list(map(int, u)), list(map(int, v)), list(map(float, J))
    for r in range(st.shape[0]):
        row = st[r:r + 1].copy()
        s, e = mod.simulated_annealing(1, hl, ul, vl, Jl, int(sweeps_per_beta),
                                       np.asarray(betas, dtype=float), int(seeds[r]), row,
                                       randomize_order, proposal)
        st[r] = s[0]
        en[r] = e[0]
    return st, en
