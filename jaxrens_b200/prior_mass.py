"""Prior-mass ladder of nested sampling with ``n_cull`` culls per iteration.

Restates the pymatnest convention used by jaxrens (``prior_mass.py``;
Martiniani et al., PRX 4, 031034 (2014), Eq. 3): one iteration contracts the
prior mass by ``(K + 1 - n_cull) / (K + 1)``; dead point ``n`` carries
``log a_n = log X_n - log(K + 1 - (n + 1) mod n_cull)``.
"""

from __future__ import annotations

import numpy as np


def _check(n_live: int, n_cull: int) -> None:
    if int(n_cull) < 1:
        raise ValueError(f"at least one walker is culled per iteration (n_cull={n_cull})")
    if int(n_cull) >= int(n_live):
        raise ValueError(f"cannot cull {n_cull} of {n_live} live walkers per iteration: "
                         "n_cull has to stay below n_live")


def _terms(n_terms: int, n_live: int, n_cull: int) -> np.ndarray:
    j = (np.arange(n_terms, dtype=np.int64) % n_cull).astype(np.float64)
    return np.log(float(n_live) - j) - np.log(float(n_live) + 1.0 - j)


def log_alpha(n_live: int, n_cull: int = 1) -> float:
    _check(n_live, n_cull)
    return float(np.log(n_live + 1.0 - n_cull) - np.log(n_live + 1.0))


def log_prior_mass(n_dead: int, n_live: int, n_cull: int = 1) -> np.ndarray:
    _check(n_live, n_cull)
    return np.cumsum(_terms(int(n_dead), n_live, n_cull))


def log_dead_weights(n_dead: int, n_live: int, n_cull: int = 1) -> np.ndarray:
    lx = log_prior_mass(n_dead, n_live, n_cull)
    nxt = (np.arange(1, int(n_dead) + 1, dtype=np.int64) % n_cull).astype(np.float64)
    return lx - np.log(float(n_live) + 1.0 - nxt)


def log_live_weight(n_dead: int, n_live: int, n_cull: int = 1) -> float:
    _check(n_live, n_cull)
    return float(np.sum(_terms(int(n_dead) + 1, n_live, n_cull)) - np.log(float(n_live)))


def iteration_offsets(n_live: int, n_cull: int = 1):
    """``(x_offset, w_offset)`` of the dead points inside one iteration."""
    return log_prior_mass(n_cull, n_live, n_cull), log_dead_weights(n_cull, n_live, n_cull)
