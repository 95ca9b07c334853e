"""Fixed-contour burn-in before nested sampling (``init/burn_in.py``).

``walk_population`` is ``_one_walk`` (:48-127) on the GPU through
``jr_walk_population``: every walker of every run walks ``walklength`` MWG
steps at once, one CUDA group per walker.  ``initial_walk`` is the driver
(:151-460): contour = each run's maximum energy + ``emax_offset_per_atom *
n_atoms``, held for all walks; step sizes adapted every ``adjust_interval``
walks; the key schedule of the reference (``key, key_adapt = split(key)``
before an adaptation, ``key, sub, move_key = split(key, 3)`` per walk, run
keys ``split(sub, R)`` for batched runs, the move key shared by all runs).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib, prng
from .adaptation import build_adapt_step


def walk_population(ns_state, step, walklength: int, run_keys, move_key, emax) -> None:
    """Advance every walker in place (``burn_in.py:48-127``).  ``run_keys``
    ``(P, 2)``, ``move_key`` ``(2,)``, ``emax`` ``(P,)``."""
    import torch

    from .nested_sampling import _ptr, _stream, make_dims, state_buffers

    dev = ns_state.population.positions.device
    P = ns_state.population.energy64.shape[0]
    rk = torch.as_tensor(np.asarray(run_keys, np.uint32).reshape(P, 2).view(np.int32).copy(),
                         device=dev)
    mk = torch.as_tensor(np.asarray(move_key, np.uint32).reshape(2).view(np.int32).copy(),
                         device=dev)
    em = torch.as_tensor(np.broadcast_to(np.asarray(emax, np.float64), (P,)).copy(), device=dev)
    dims = make_dims(ns_state, step, 1, 0)
    sb = state_buffers(ns_state)
    rc = _lib.load().jr_walk_population(C.byref(dims), C.byref(step.params), C.byref(sb),
                                        int(walklength), _ptr(rk), _ptr(mk), _ptr(em), _stream())
    _lib.check(rc, "jr_walk_population")


def initial_walk(key, ns_state, step, *, n_walks: int, walklength: int, adjust_interval: int,
                 emax_offset_per_atom: float, n_atoms: int, adapt: bool = True,
                 adjust_n_samples: int = 50, adjust_factor: float = 1.5,
                 adjust_max_rounds: int = 15, trial_factory=None):
    """Decorrelate the live walkers at a fixed contour (``burn_in.py:151-460``).

    Returns the state (updated in place) and the per-adaptation diagnostics.
    ``adapt=False`` runs the walks without step-size adaptation (the
    reference's ``per_move_fns=None``)."""
    if n_walks == 0:
        return ns_state, []
    pop = ns_state.population
    emax = pop.energy64.max(dim=1).values.cpu().numpy() + float(emax_offset_per_atom) * n_atoms
    P = emax.shape[0]
    batched = bool(ns_state.batched)
    adapt_step = (build_adapt_step(step, adjust_n_samples, adjust_factor, adjust_max_rounds,
                                   adjust_interval, trial_factory) if adapt else None)
    key = np.asarray(key, np.uint32)
    diags = []
    for walk_i in range(n_walks):
        if adapt_step is not None and walk_i % adjust_interval == 0:
            key, key_adapt = prng.split(key, 2)
            ka = prng.split(key_adapt, P) if batched else key_adapt[None, :]
            ns_state, diag, _ = adapt_step(ns_state, emax, ka)
            diags.append(diag)
        key, sub, move_key = prng.split(key, 3)
        run_keys = prng.split(sub, P) if batched else sub[None, :]
        walk_population(ns_state, step, walklength, run_keys, move_key, emax)
    return ns_state, diags
