"""Synthetic uniform-gas walkers for the benchmark workloads.

Walker ``k`` draws from ``split(key, K)[k]``: its cubic cell volume is
``v_hi * (1 - u)`` (uniform in ``(0, v_hi]``) and its fractional
coordinates are uniform in ``[0, 1)^3`` -- the initialisation the LJ
benchmark configurations specify (``init/cells.py:82-137`` and
``init/positions.py:15-31`` give the reference's general forms).
"""

from __future__ import annotations

import numpy as np

from . import prng


def uniform_gas(key, n_walkers: int, n_atoms: int, v_hi: float):
    keys = prng.split(np.asarray(key, np.uint32), n_walkers)
    pos = np.zeros((n_walkers, n_atoms, 3), np.float32)
    cell = np.zeros((n_walkers, 3, 3), np.float32)
    third = float(np.float32(1.0) / np.float32(3.0))
    for k in range(n_walkers):
        kv, kp = prng.split(keys[k], 2)
        u = prng.uniform(kv, 1)[0]
        V = np.float32(v_hi) * (np.float32(1.0) - u)
        L = np.float32(float(V) ** third)
        cell[k] = np.eye(3, dtype=np.float32) * L
        frac = prng.uniform(kp, 3 * n_atoms).reshape(n_atoms, 3)
        pos[k] = (frac * L).astype(np.float32)
    return pos, cell
