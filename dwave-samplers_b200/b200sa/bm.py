"""Batched Boltzmann-machine learning on the B200 sampler (no reference
counterpart).

Fully visible Ising models in the reference's convention
(``p(s) ~ exp(-beta E(s))``, ``E = sum h s + sum J s s``).  The negative
log-likelihood of data with coupler correlations ``<s_u s_v>_data`` is

    NLL(J) = beta * sum_c J_c <s_u s_v>_data + log Z(J)

whose gradient ``beta <ss>_data - beta <ss>_model`` is obtained by autograd:
the data term is a torch expression and ``log Z`` is
:class:`b200sa.autograd.LogPartition` (fixed-beta Gibbs sampling forward,
moments kernel backward).  All models are sampled in one persistent batch and
reduced in one moments launch per step; Adam updates the couplings.
"""
from __future__ import annotations

import time
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np
import torch

from .autograd import (IsingModel, ModelSampler, SamplingSpec, edge_moments, log_partition,
                       pool_sums, sample_models)


@dataclass
class BMResult:
    J: list                      # fitted couplings per model (numpy)
    corr_error: list = field(default_factory=list)  # mean |<ss>_model - <ss>_data| per step
    step_seconds: list = field(default_factory=list)
    target_seconds: float = 0.0

    @property
    def steps_per_second(self) -> float:
        t = sum(self.step_seconds)
        return len(self.step_seconds) / t if t > 0 else float("nan")


def target_correlations(models: Sequence[IsingModel], hs, Js, beta: float, reads: int,
                        sweeps: int, seed: int, device: int = 0, autotune: bool = False,
                        group=None):
    """<s_u s_v> per coupler of the ground-truth models, from `reads` fixed-beta
    Gibbs reads of `sweeps` sweeps each (with `group`, `reads` per rank, the
    sums pooled over the ranks)."""
    sampler = ModelSampler(models, beta, sweeps, reads, "Gibbs", device, autotune)
    try:
        ranks, read0 = 1, 0
        if group is not None:
            ranks = torch.distributed.get_world_size(group)
            read0 = torch.distributed.get_rank(group) * reads
        samples = sample_models(models, hs, Js, beta, sweeps, reads, seed, seed + 1, read0,
                                "Gibbs", device, sampler)
        ss, sss = edge_moments(models, samples, device)
        if group is not None:
            _, sss = pool_sums(ss, sss, group)
        return [x.to(torch.float64) / (reads * ranks) for x in sss]
    finally:
        sampler.close()


def fit(truth: Sequence[tuple], beta: float = 1.0, steps: int = 500, reads: int = 1024,
        sweeps: int = 2000, lr: float = 1e-2, target_reads: int = 8192,
        target_sweeps: int = 2000, seed: int = 11, device: int = 0,
        callback: Callable[[int, float], None] | None = None,
        autotune: bool = True, group=None) -> BMResult:
    """Fit J (from zero, h fixed at the truth's h) to the truth's coupler
    correlations.  `truth` is a list of (h, u, v, J) ground-truth models.
    With `autotune` the sampling plan's launch shapes are measured once, at
    the first step (results are the same either way).  With `group` (a
    torch.distributed group, one rank per GPU) every rank samples `reads`
    and `target_reads` reads of every model and the moment sums are pooled
    by one all-reduce per step, so every rank takes the same Adam step."""
    dev = torch.device("cuda", device)
    models = [IsingModel(len(h), np.ascontiguousarray(u, np.int32), np.ascontiguousarray(v, np.int32))
              for h, u, v, _ in truth]
    hs = [np.asarray(h, np.float64) for h, _, _, _ in truth]
    t0 = time.perf_counter()
    corr_data = target_correlations(models, hs, [np.asarray(J, np.float64) for *_, J in truth],
                                    beta, target_reads, target_sweeps, seed, device, autotune,
                                    group)
    torch.cuda.synchronize(dev)
    res = BMResult(J=[], target_seconds=time.perf_counter() - t0)
    data = torch.cat(corr_data).to(dev)
    h_cat = torch.from_numpy(np.concatenate(hs)).to(dev)
    J = torch.zeros(data.shape[0], dtype=torch.float64, device=dev, requires_grad=True)
    opt = torch.optim.Adam([J], lr=lr)
    samplers = None  # one plan and graph for every step
    for step in range(steps):
        t = time.perf_counter()
        spec = SamplingSpec(models, beta=beta, sweeps=sweeps, reads=reads,
                            seed=seed + 1000 + step, init_seed=seed + 7 + step, device=device,
                            samplers=samplers, autotune=autotune, group=group)
        loss = beta * torch.dot(J, data) + log_partition(h_cat, J, spec)
        samplers = spec.samplers
        opt.zero_grad()
        loss.backward()
        opt.step()
        model_corr = torch.cat([x.to(torch.float64) for x in spec.last_moments[1]]) / spec.total_reads
        err = float(torch.mean(torch.abs(model_corr - data)))
        torch.cuda.synchronize(dev)
        res.step_seconds.append(time.perf_counter() - t)
        res.corr_error.append(err)
        if callback is not None:
            callback(step, err)
    Jn = J.detach().cpu().numpy()
    off = 0
    for m in models:
        res.J.append(Jn[off:off + m.num_couplers].copy())
        off += m.num_couplers
    return res


def main(argv=None):
    """Run the batched fit on seeded synthetic ground truths and write the
    correlation-error curve:

        python -m b200sa.bm [--steps 500] [--models 64] [--out curve.json]

    Defaults: 64 six-regular models, n ~ U[256, 2048], J* ~ N(0, 0.5), h* = 0,
    targets from 8192 reads at beta = 1, Adam lr 1e-2, 1024 reads x 2000 Gibbs
    sweeps per step."""
    import argparse
    import json
    from . import workloads
    ap = argparse.ArgumentParser(prog="python -m b200sa.bm")
    ap.add_argument("--steps", type=int, default=500)
    ap.add_argument("--models", type=int, default=64)
    ap.add_argument("--reads", type=int, default=1024)
    ap.add_argument("--sweeps", type=int, default=2000)
    ap.add_argument("--target-reads", type=int, default=8192)
    ap.add_argument("--lr", type=float, default=1e-2)
    ap.add_argument("--device", type=int, default=0)
    ap.add_argument("--out", default=None)
    a = ap.parse_args(argv)
    truth = workloads.bm_models(num_models=a.models, n_range=(256, 2048), d=6, J_sigma=0.5,
                                seed=5)
    t0 = time.perf_counter()

    def report(step, err):
        if step % 10 == 0 or step == a.steps - 1:
            print(f"step {step:4d}  corr_error {err:.5f}  {time.perf_counter() - t0:8.1f} s",
                  flush=True)

    res = fit(truth, beta=1.0, steps=a.steps, reads=a.reads, sweeps=a.sweeps, lr=a.lr,
              target_reads=a.target_reads, target_sweeps=a.sweeps, seed=3, device=a.device,
              callback=report)
    Jerr = float(np.mean([np.mean(np.abs(J - t[3])) for J, t in zip(res.J, truth)]))
    out = {"steps": a.steps, "models": a.models, "reads": a.reads, "sweeps": a.sweeps,
           "target_reads": a.target_reads, "lr": a.lr, "corr_error": res.corr_error,
           "step_seconds": res.step_seconds, "target_seconds": res.target_seconds,
           "steps_per_second_after_first": (len(res.step_seconds) - 1) /
                                           max(sum(res.step_seconds[1:]), 1e-9),
           "mean_abs_J_error": Jerr}
    if a.out:
        with open(a.out, "w") as f:
            json.dump(out, f)
    print(json.dumps({k: v for k, v in out.items() if k not in ("corr_error", "step_seconds")}))


if __name__ == "__main__":
    main()
