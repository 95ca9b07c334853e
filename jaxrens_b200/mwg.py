"""Metropolis-within-Gibbs assembly (``sampling/mwg.py:40-259``).

``build_mwg(backend, move_descriptors)`` returns ``(init_fn, step_fn,
per_move_fns)`` like the reference.  Here ``step_fn`` is an ``MWGStep``
descriptor holding the kernel parameters (``JrParams``); ``ns_step`` hands it
to the CUDA walk.  ``per_move_fns[k]`` runs move ``k`` on chosen walkers
through ``jr_move_trial`` (step-size trials, burn-in).
"""

from __future__ import annotations

import ctypes as C
import dataclasses

import numpy as np

from . import _lib
from .backends import Hamiltonian
from .moves import MoveKernel, MoveSpec


@dataclasses.dataclass
class MWGStep:
    backend: object
    move_descriptors: list
    specs: list
    params: _lib.JrParams
    move_probs: np.ndarray
    default_step_sizes: np.ndarray

    @property
    def n_moves(self) -> int:
        return len(self.specs)

    @property
    def move_names(self) -> list[str]:
        return [d.name for d in self.move_descriptors]

    def with_evidence(self, log_alpha: float, w_offset) -> _lib.JrParams:
        """Parameters with the prior-mass constants of one iteration:
        ``log_alpha`` and the dead-weight offsets ``w_offset`` (a scalar for
        n_cull = 1 or the ``(n_cull,)`` array of
        ``prior_mass.iteration_offsets``)."""
        p = _lib.JrParams()
        C.pointer(p)[0] = self.params
        p.log_alpha = log_alpha
        wo = np.atleast_1d(np.asarray(w_offset, np.float64))
        if wo.size > _lib.MAX_CULL:
            raise ValueError(f"at most {_lib.MAX_CULL} culls per iteration")
        for k, v in enumerate(wo):
            p.w_offset[k] = float(v)
        return p


def _move_params(specs: list[MoveSpec], probs_cum: np.ndarray) -> _lib.JrMoveParams:
    mv = _lib.JrMoveParams()
    M = len(specs)
    if M > _lib.MAX_MOVES:
        raise ValueError("at most 8 move types")
    mv.n_moves = M
    # one cell-geometry guard for every cell move (the CLI's `cell:` section);
    # the volume-prior flag comes from the volume move
    guards = {s.cell_guard[:3] for s in specs if s.cell_guard is not None}
    if len(guards) > 1:
        raise NotImplementedError("all cell moves must share one cell-geometry guard")
    max_vpa, min_vpa, min_aspect = guards.pop() if guards else (1e4, 1.0, 0.8)
    flat = any(bool(s.cell_guard[3]) for s in specs
               if s.cell_guard is not None and s.cell_guard[3] is not None)
    for m, s in enumerate(specs):
        mv.type[m] = s.type
        mv.n_reflect[m] = s.n_reflect
        mv.perturb_angle[m] = s.perturb_angle
        mv.cum_probs[m] = float(probs_cum[m])
    mv.max_vpa, mv.min_vpa, mv.min_aspect = max_vpa, min_vpa, min_aspect
    mv.flat_v_prior = int(flat)
    return mv


def build_mwg(backend, move_descriptors: list[MoveKernel], constraint_descriptors=()):
    """Build ``(init_fn, step_fn, per_move_fns)`` (``mwg.py:40-259``).
    ``constraint_descriptors`` (``constraints.min_distance_descriptor``) gate
    the moves that can violate them (``mwg.py:97-150``)."""
    from .constraints import move_gates

    gates, dmin = move_gates(tuple(constraint_descriptors), move_descriptors)
    if not isinstance(backend, Hamiltonian):
        backend = Hamiltonian(backend, [])
    specs = [d.build_kernel(backend, **d.kernel_kwargs) for d in move_descriptors]
    # move_probs = weights / weights.sum() in float32; choice() uses its cumsum
    weights = np.array([d.weight for d in move_descriptors], np.float32)
    probs = (weights / weights.sum(dtype=np.float32)).astype(np.float32)
    cum = np.cumsum(probs, dtype=np.float32)
    params = _lib.JrParams()
    params.model = backend.model_params()
    params.moves = _move_params(specs, cum)
    if dmin is not None:
        S = backend.model_params().n_species
        if dmin.shape != (S, S):
            raise ValueError(f"d_min matrix must be ({S}, {S}) for this model")
        for m, g in enumerate(gates):
            params.moves.gate[m] = g
        params.moves.dmin[: S * S] = [float(v) for v in dmin.reshape(-1)]
    defaults = np.array([d.step_size for d in move_descriptors], np.float32)
    step = MWGStep(backend, list(move_descriptors), specs, params, probs, defaults)

    def init_fn(positions, types, energy, cell=None, step_sizes=None, step_size=None,
                ensemble_params=None, max_neighbors: int = 0, max_neighbor_count_init=0):
        """Single-walker initial state (host numpy), as ``mwg.py:163-222``."""
        if cell is None:
            cell = np.zeros((3, 3), np.float32)
        if step_sizes is None:
            step_sizes = (np.full(len(specs), step_size, np.float32)
                          if step_size is not None else defaults)
        return {
            "positions": np.asarray(positions, np.float32),
            "types": np.asarray(types, np.int32),
            "energy": float(energy) if energy is not None else None,
            "cell": np.asarray(cell, np.float32),
            "step_sizes": np.asarray(step_sizes, np.float32),
            "direction": np.zeros_like(np.asarray(positions, np.float32)),
            "ensemble_params": ensemble_params or {},
        }

    from .nested_sampling import TrialMove

    per_move_fns = [TrialMove(step, k) for k in range(len(specs))]
    init_fn.step = step  # lets init_ns recover the descriptor
    return init_fn, step, per_move_fns
