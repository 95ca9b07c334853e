"""Thermodynamics of nested-sampling output (``postprocess/thermodynamics.py``).

float64 NumPy on the host, like the reference: the evidence from dead and
live points (:89-122), the partition function ``log Z(beta)`` (:125-176) and
the heat capacity ``beta^2 Var(E)`` in the deviation form (:179-230), with the
prior-mass weights of :mod:`jaxrens_b200.prior_mass`.  Dead energies are in
``.energies`` row order (``n_cull`` per iteration, descending).
"""

from __future__ import annotations

import numpy as np

from .prior_mass import log_dead_weights, log_live_weight


def _lse(x, axis=-1, keepdims=False):
    x = np.asarray(x, np.float64)
    m = np.max(x, axis=axis, keepdims=True)
    m = np.where(np.isfinite(m), m, 0.0)
    out = np.log(np.sum(np.exp(x - m), axis=axis, keepdims=True)) + m
    return out if keepdims else np.squeeze(out, axis=axis)


def _weights(n_dead: int, n_live: int, n_cull: int):
    return log_dead_weights(n_dead, n_live, n_cull), log_live_weight(n_dead, n_live, n_cull)


def log_evidence(dead_energies, live_energies, n_live: int, n_cull: int = 1):
    """``log Z`` from the dead points and the remaining live walkers."""
    dead = np.asarray(dead_energies, np.float64)
    live = np.asarray(live_energies, np.float64)
    wd, wl = _weights(dead.shape[-1], n_live, n_cull)
    return np.logaddexp(_lse(wd - dead), _lse(wl - live))


def _merged(beta, dead_energies, live_energies, n_live, n_cull):
    dead = np.asarray(dead_energies, np.float64)
    live = np.asarray(live_energies, np.float64)
    wd, wl = _weights(dead.shape[-1], n_live, n_cull)
    live_b = np.broadcast_to(live, dead.shape[:-1] + (live.shape[-1],))
    E = np.concatenate([dead, live_b], axis=-1)
    w = np.concatenate([wd, np.full(live.shape[-1], wl)])
    return E, w - np.asarray(beta, np.float64) * E


def partition_function(beta, dead_energies, live_energies, n_live: int, n_cull: int = 1):
    """``log Z(beta) = log sum_i w_i exp(-beta E_i)`` over dead + live points."""
    return _lse(_merged(beta, dead_energies, live_energies, n_live, n_cull)[1])


def heat_capacity(beta, dead_energies, live_energies, n_live: int, n_cull: int = 1):
    """``C_v(beta) = beta^2 sum_i p_i (E_i - <E>)^2`` (deviation form)."""
    E, lu = _merged(beta, dead_energies, live_energies, n_live, n_cull)
    p = np.exp(lu - _lse(lu, keepdims=True))
    mean = np.sum(p * E, axis=-1, keepdims=True)
    return np.asarray(beta, np.float64) ** 2 * np.sum(p * (E - mean) ** 2, axis=-1)


def cv_peak_temperature(temperatures, dead_energies, live_energies, n_live: int,
                        n_cull: int = 1, n_atoms: int = 1) -> float:
    """Temperature of the per-atom heat-capacity maximum on a grid (k_B = 1)."""
    T = np.asarray(temperatures, np.float64)
    cv = np.array([heat_capacity(1.0 / t, dead_energies, live_energies, n_live, n_cull)
                   for t in T]) / n_atoms
    return float(T[int(np.argmax(cv))])
