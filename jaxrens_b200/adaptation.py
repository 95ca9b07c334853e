"""Step-size adaptation by trial moves (``sampling/adaptation/``).

The host side of the reference's in-XLA bisection: the acceptance-rate
decision (``stepsize_handler.py:35-104`` ``_process_rate_jax``) in float32 as
the reference computes it, the per-run bisection loop
(``stepsize_handler.py:110-433`` ``adjust_step_size``) whose trial moves run
on the GPU through ``jr_move_trial``, and the per-move driver
(``manager.py:71-227`` ``build_adapt_step``).  Runs advance together like the
reference's vmapped ``while_loop``: every round launches the trials of all
runs at once, and a converged run keeps its carry.
"""

from __future__ import annotations

import dataclasses
from typing import Callable

import numpy as np

from . import prng

FLOOR_THRESHOLD = 1.0e-7
_f32 = np.float32


def process_rate(rate, step_size, step_size_prev, rate_prev, min_rate: float,
                 max_rate: float, adjust_factor: float, max_step_size: float):
    """One acceptance-rate decision (``stepsize_handler.py:35-104``), float32.

    Returns ``(new_step_size, converged, cap_hit, floor_hit, too_high,
    too_low)``; ``rate_prev < 0`` means no previous rate.  Arrays broadcast
    (one entry per run)."""
    rate = _f32(rate) if np.isscalar(rate) else np.asarray(rate, _f32)
    ss = np.asarray(step_size, _f32)
    ss_prev = np.asarray(step_size_prev, _f32)
    rate_prev = np.asarray(rate_prev, _f32)
    lo, hi = _f32(min_rate), _f32(max_rate)
    target = _f32(0.5 * (min_rate + max_rate))
    in_window = (rate > lo) & (rate < hi)
    has_prev = rate_prev >= _f32(0.0)
    brackets = has_prev & (np.minimum(rate, rate_prev) < lo) & (np.maximum(rate, rate_prev) > hi)
    prev_closer = np.abs(rate_prev - target) < np.abs(rate - target)
    bracket_ss = np.where(prev_closer, ss_prev, ss)
    too_high = rate >= hi
    too_low = rate < lo
    scale = np.where(too_low, _f32(1.0 / adjust_factor),
                     np.where(too_high, _f32(adjust_factor), _f32(1.0))).astype(_f32)
    proposed = (ss * scale).astype(_f32)
    cap_hit = proposed >= _f32(max_step_size)
    floor_hit = proposed <= _f32(FLOOR_THRESHOLD)
    adjusted = np.clip(proposed, _f32(FLOOR_THRESHOLD), _f32(max_step_size)).astype(_f32)
    new_ss = np.where(in_window, ss, np.where(brackets, bracket_ss, adjusted)).astype(_f32)
    return new_ss, in_window | brackets, cap_hit, floor_hit, too_high, too_low


@dataclasses.dataclass
class AdjustResult:
    """Per-run outcome of :func:`adjust_step_size` (its tuple, named)."""

    step_size: np.ndarray
    rate: np.ndarray
    counts: np.ndarray          # (P, 4): accepted / energy / cell / prior, last round
    n_rounds: np.ndarray
    converged: np.ndarray
    cap_hits: np.ndarray
    floor_hits: np.ndarray
    bracket_detected: np.ndarray
    trial_n_evaluations: np.ndarray
    trial_n_grad_evaluations: np.ndarray


def adjust_step_size(trial: Callable, n_walkers: int, step_size, emax, keys, n_samples: int,
                     min_rate: float, max_rate: float, adjust_factor: float,
                     max_step_size: float, max_rounds: int, evals_per_trial: int = 1,
                     grad_evals_per_trial: int = 0) -> AdjustResult:
    """Bisection of one move's step size for P runs (``stepsize_handler.py:110-433``).

    ``trial(walker_idx (P,n), keys (P,n,2), step (P,), emax (P,))`` runs the
    move once on each sampled walker under the contour and returns
    ``(accepted, reject_reason)`` arrays ``(P, n)``; it must not change the
    population.  Per round and run: ``key, k_sample, k_trials =
    split(key, 3)``, walkers ``randint(k_sample, (n,), 0, K)`` (``choice``
    with replacement), trial keys ``split(k_trials, n)``."""
    keys = np.asarray(keys, np.uint32).reshape(-1, 2)
    P = keys.shape[0]
    ss = np.broadcast_to(np.asarray(step_size, _f32), (P,)).copy()
    ss_prev = ss.copy()
    rate_prev = np.full(P, -1.0, _f32)
    rate = np.zeros(P, _f32)
    key = keys.copy()
    rounds = np.zeros(P, np.int32)
    converged = np.zeros(P, bool)
    counts = np.zeros((P, 4), np.int32)
    cap = np.zeros(P, np.int32)
    floor = np.zeros(P, np.int32)
    hi_seen = np.zeros(P, bool)
    lo_seen = np.zeros(P, bool)
    n_ev = np.zeros(P, np.int64)
    n_gr = np.zeros(P, np.int64)
    em = np.broadcast_to(np.asarray(emax, np.float64), (P,)).copy()
    while True:
        active = ~converged & (rounds < max_rounds)
        if not active.any():
            break
        widx = np.zeros((P, n_samples), np.int32)
        tkeys = np.zeros((P, n_samples, 2), np.uint32)
        new_key = key.copy()
        for p in range(P):
            k3 = prng.split(key[p], 3)
            new_key[p] = k3[0]
            widx[p] = prng.randint_array(k3[1], n_samples, 0, n_walkers)
            tkeys[p] = prng.split(k3[2], n_samples)
        acc, reason = trial(widx, tkeys, ss, em)
        acc = np.asarray(acc).reshape(P, n_samples)
        reason = np.asarray(reason).reshape(P, n_samples)
        r = (np.sum(acc != 0, axis=1).astype(_f32) / _f32(n_samples)).astype(_f32)
        cnt = np.stack([np.sum(reason == c, axis=1) for c in range(4)], axis=1).astype(np.int32)
        nss, conv, ch, fh, th, tl = process_rate(r, ss, ss_prev, rate_prev, min_rate, max_rate,
                                                 adjust_factor, max_step_size)
        # runs that already left the loop keep their carry (batched while_loop)
        a = active
        ss_prev = np.where(a, ss, ss_prev)
        ss = np.where(a, nss, ss).astype(_f32)
        rate_prev = np.where(a, r, rate_prev)
        rate = np.where(a, r, rate)
        key = np.where(a[:, None], new_key, key)
        rounds = rounds + a
        converged = converged | (a & conv)
        counts = np.where(a[:, None], cnt, counts)
        cap = cap + (a & ch)
        floor = floor + (a & fh)
        hi_seen = hi_seen | (a & th)
        lo_seen = lo_seen | (a & tl)
        n_ev = n_ev + a * n_samples * evals_per_trial
        n_gr = n_gr + a * n_samples * grad_evals_per_trial
    return AdjustResult(ss, rate, counts, rounds, converged, cap, floor, hi_seen & lo_seen,
                        n_ev, n_gr)


def build_adapt_step(step, adjust_n_samples: int = 50, adjust_factor: float = 1.5,
                     adjust_max_rounds: int = 15, adjust_interval: int = 1,
                     trial_factory: Callable | None = None):
    """``manager.py:71-227``: returns ``adapt_step(ns_state, emax, keys)`` or
    ``None`` when inactive.  Per move ``m`` (in order) and run:
    ``adapt_key, key_adjust = split(adapt_key, 2)``, bisect from the run's
    current step size (walker 0's, ``batch_descriptor.extract_step_sizes``),
    then write every walker's step sizes back.  ``trial_factory(m)`` builds
    the trial function of move ``m`` (default: the GPU ``TrialMove``)."""
    if adjust_interval <= 0 or step.n_moves == 0:
        return None
    descs = list(step.move_descriptors)

    def adapt_step(ns_state, emax, keys):
        import torch

        from .nested_sampling import TrialMove

        pop = ns_state.population
        P, K = pop.energy64.shape
        ss = pop.step_sizes[:, 0, :].detach().cpu().numpy().astype(_f32)
        adapt_key = np.asarray(keys, np.uint32).reshape(P, 2).copy()
        diag = []
        for m, desc in enumerate(descs):
            pairs = np.stack([prng.split(adapt_key[p], 2) for p in range(P)])
            adapt_key = pairs[:, 0].copy()
            key_adjust = pairs[:, 1].copy()
            if trial_factory is not None:
                trial = trial_factory(m)
            else:
                tm = TrialMove(step, m)

                def trial(widx, tkeys, s, e, tm=tm):
                    a, r = tm(ns_state, widx, tkeys, s, e)
                    return a.cpu().numpy(), r.cpu().numpy()
            spec = step.specs[m]
            n_grad = spec.n_evals if spec.type == 0 else 0
            res = adjust_step_size(trial, K, ss[:, m], emax, key_adjust, adjust_n_samples,
                                   desc.min_rate, desc.max_rate, adjust_factor,
                                   desc.step_size_max, adjust_max_rounds,
                                   evals_per_trial=spec.n_evals, grad_evals_per_trial=n_grad)
            ss[:, m] = res.step_size
            diag.append(res)
        new = torch.as_tensor(ss, device=pop.step_sizes.device)
        pop.step_sizes.copy_(new[:, None, :].expand_as(pop.step_sizes))
        return ns_state, diag, adapt_key

    return adapt_step
