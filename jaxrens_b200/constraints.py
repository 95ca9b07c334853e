"""Configuration constraints gated after moves (``constraints/``).

A ``ConstraintDescriptor`` (``constraints/base.py:60-98``) names the state
aspects its predicate reads; ``build_mwg`` gates exactly the moves whose
``mutates`` set meets them (``make_move_gate``, ``base.py:101-140``).  The
minimum-distance constraint (``constraints/min_distance.py``) is the one the
walk kernels evaluate: every pair closer than ``d_min[t_i][t_j]`` under the
minimum image rejects the move with reason 4.
"""

from __future__ import annotations

import dataclasses

import numpy as np

ASPECTS = frozenset({"positions", "cell", "types"})


@dataclasses.dataclass(frozen=True)
class ConstraintDescriptor:
    name: str
    depends_on: frozenset
    build_kwargs: dict = dataclasses.field(default_factory=dict)
    reject_reason: int = 4

    def __post_init__(self):
        unknown = self.depends_on - ASPECTS
        if unknown:
            raise ValueError(f"Constraint {self.name!r} declares unknown depends_on aspects "
                             f"{sorted(unknown)}; valid aspects are {sorted(ASPECTS)}.")


def min_distance_descriptor(d_min_matrix, *, type_dependent: bool) -> ConstraintDescriptor:
    """``min_distance.py:50-75``: thresholds ``(S, S)``; a type-dependent
    matrix also gates the moves that relabel species."""
    depends = {"positions", "cell"} | ({"types"} if type_dependent else set())
    return ConstraintDescriptor("minimum_distance", frozenset(depends),
                                {"d_min_matrix": np.asarray(d_min_matrix, np.float32)})


def move_gates(constraints, move_descriptors) -> tuple[list[int], np.ndarray | None]:
    """Per move, whether the minimum-distance gate applies; and its matrix."""
    dmin = None
    relevant = []
    for c in constraints:
        if c.name != "minimum_distance":
            raise NotImplementedError(f"constraint {c.name!r} has no CUDA kernel in this library")
        if dmin is not None:
            raise NotImplementedError("one minimum-distance constraint per sampler")
        dmin = np.asarray(c.build_kwargs["d_min_matrix"], np.float32)
        relevant.append(c)
    gates = [int(any(c.depends_on & d.mutates for c in relevant)) for d in move_descriptors]
    return gates, dmin
