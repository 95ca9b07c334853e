"""Move descriptors: the MWG move set of the B200 walk.

Mirrors ``sampling/move_kernel.py`` (``MoveKernel``) and the ``build_kernel``
entry points of ``sampling/moves/galilean.py``, ``volume.py``,
``alchemical.py`` and ``swap.py``.  A built kernel here is a small
descriptor; the arithmetic runs inside the CUDA walk.
"""

from __future__ import annotations

import dataclasses
from collections.abc import Callable
from dataclasses import field
from types import SimpleNamespace
from typing import Any

from . import _lib


@dataclasses.dataclass(frozen=True)
class MoveKernel:
    """One MWG move type (``sampling/move_kernel.py:16-71``)."""

    name: str
    build_kernel: Callable
    kernel_kwargs: dict[str, Any] = field(default_factory=dict)
    weight: float = 1.0
    step_size: float = 0.1
    step_size_max: float = 10.0
    min_rate: float = 0.25
    max_rate: float = 0.65
    extra_state_fields: dict[str, tuple[type, Callable]] = field(default_factory=dict)
    reject_reasons: frozenset[str] = field(default_factory=lambda: frozenset({"energy"}))
    mutates: frozenset[str] = field(
        default_factory=lambda: frozenset({"positions", "cell", "types"}))


@dataclasses.dataclass(frozen=True)
class MoveSpec:
    """What the CUDA walk needs to know about one built move."""

    type: int
    n_reflect: int = 0
    perturb_angle: float = 0.0
    cell_guard: tuple | None = None  # (max_vpa, min_vpa, min_aspect, flat_v_prior)
    n_evals: int = 1


def _galilean_build_kernel(backend, n_reflect: int = 5, perturb_angle: float = 0.1,
                           use_forces: bool = True, species=None,
                           direction_field: str = "direction",
                           refresh_direction: bool = False) -> MoveSpec:
    """Galilean move with n_reflect reflections (``galilean.py:98-302``)."""
    if not use_forces or species is not None or refresh_direction or direction_field != "direction":
        raise NotImplementedError(
            "the B200 galilean kernel implements use_forces=True, species=None, "
            "refresh_direction=False on the 'direction' field")
    if int(n_reflect) < 1:
        raise ValueError("n_reflect must be >= 1")
    return MoveSpec(_lib.MOVE_GALILEAN, int(n_reflect), float(perturb_angle),
                    n_evals=int(n_reflect))


def _volume_build_kernel(backend, n_atoms: int, max_vol_per_atom: float = 100.0,
                         min_vol_per_atom: float = 1.0, min_aspect: float = 0.5,
                         flat_v_prior: bool = False) -> MoveSpec:
    """Isotropic volume move (``volume.py:19-111``).  ``n_atoms`` is taken
    per replica from the state, so uneven replicas share one descriptor."""
    return MoveSpec(_lib.MOVE_VOLUME,
                    cell_guard=(float(max_vol_per_atom), float(min_vol_per_atom),
                                float(min_aspect), bool(flat_v_prior)))


def _morph_build_kernel(backend, n_species: int) -> MoveSpec:
    """alchemical_morph (``alchemical.py:26-81``): composition-changing."""
    if int(n_species) < 2:
        raise ValueError("alchemical_morph needs n_species >= 2")
    return MoveSpec(_lib.MOVE_MORPH)


def _swap_build_kernel(backend, n_species: int, species=None) -> MoveSpec:
    """species_swap (``swap.py:119-262``): composition-conserving."""
    if int(n_species) < 2:
        raise ValueError(
            f"swap.build_kernel requires n_species >= 2, got {n_species}")
    if species is not None and sorted(set(int(c) for c in species)) != list(range(int(n_species))):
        raise NotImplementedError("the B200 swap kernel exchanges over every species")
    return MoveSpec(_lib.MOVE_SWAP)


def _shear_build_kernel(backend, n_atoms: int, max_vol_per_atom: float = 100.0,
                        min_vol_per_atom: float = 1.0, min_aspect: float = 0.5) -> MoveSpec:
    """Volume-preserving shear of one cell vector (``shear.py:54-127``)."""
    return MoveSpec(_lib.MOVE_SHEAR, cell_guard=(float(max_vol_per_atom),
                                                 float(min_vol_per_atom), float(min_aspect),
                                                 None))


def _stretch_build_kernel(backend, n_atoms: int, max_vol_per_atom: float = 100.0,
                          min_vol_per_atom: float = 1.0, min_aspect: float = 0.5) -> MoveSpec:
    """Volume-preserving stretch along two axes (``stretch.py:18-104``)."""
    return MoveSpec(_lib.MOVE_STRETCH, cell_guard=(float(max_vol_per_atom),
                                                   float(min_vol_per_atom), float(min_aspect),
                                                   None))


galilean = SimpleNamespace(build_kernel=_galilean_build_kernel)
shear = SimpleNamespace(build_kernel=_shear_build_kernel)
stretch = SimpleNamespace(build_kernel=_stretch_build_kernel)
volume = SimpleNamespace(build_kernel=_volume_build_kernel)
alchemical = SimpleNamespace(build_morph_kernel=_morph_build_kernel)
swap = SimpleNamespace(build_kernel=_swap_build_kernel)

DIRECTION_FIELD = {"direction": (object, lambda pos, types: None)}


def gmc(name: str = "galilean", n_reflect: int = 10, step_size: float = 0.1,
        weight: float = 4.0, perturb_angle: float = 0.1) -> MoveKernel:
    """Convenience: the ``moves[].type: galilean`` descriptor."""
    return MoveKernel(name, galilean.build_kernel,
                      kernel_kwargs={"n_reflect": n_reflect, "perturb_angle": perturb_angle},
                      weight=weight, step_size=step_size,
                      extra_state_fields=DIRECTION_FIELD,
                      mutates=frozenset({"positions"}))


def volume_move(n_atoms: int, step_size: float = 0.3, weight: float = 1.0,
                max_volume_per_atom: float = 1e4, min_volume_per_atom: float = 1.0,
                min_aspect_ratio: float = 0.8, flat_v_prior: bool = False) -> MoveKernel:
    """Convenience: ``moves[].type: volume`` with the ``cell:`` section
    defaults of ``cli/schema/cell.py``."""
    return MoveKernel("volume", volume.build_kernel,
                      kernel_kwargs={"n_atoms": n_atoms,
                                     "max_vol_per_atom": max_volume_per_atom,
                                     "min_vol_per_atom": min_volume_per_atom,
                                     "min_aspect": min_aspect_ratio,
                                     "flat_v_prior": flat_v_prior},
                      weight=weight, step_size=step_size,
                      reject_reasons=frozenset({"energy", "cell", "prior"}),
                      mutates=frozenset({"positions", "cell"}))


def morph_move(n_species: int, weight: float = 1.0) -> MoveKernel:
    return MoveKernel("alchemical_morph", alchemical.build_morph_kernel,
                      kernel_kwargs={"n_species": n_species}, weight=weight,
                      step_size=0.0, mutates=frozenset({"types"}))


def swap_move(n_species: int, weight: float = 1.0) -> MoveKernel:
    return MoveKernel("species_swap", swap.build_kernel,
                      kernel_kwargs={"n_species": n_species}, weight=weight,
                      step_size=0.0, mutates=frozenset({"types"}))


def shear_move(n_atoms: int, step_size: float = 0.1, weight: float = 1.0,
               max_volume_per_atom: float = 1e4, min_volume_per_atom: float = 1.0,
               min_aspect_ratio: float = 0.8) -> MoveKernel:
    """Convenience: ``moves[].type: shear`` with the ``cell:`` section defaults."""
    return MoveKernel("shear", shear.build_kernel,
                      kernel_kwargs={"n_atoms": n_atoms, "max_vol_per_atom": max_volume_per_atom,
                                     "min_vol_per_atom": min_volume_per_atom,
                                     "min_aspect": min_aspect_ratio},
                      weight=weight, step_size=step_size,
                      reject_reasons=frozenset({"energy", "cell"}),
                      mutates=frozenset({"positions", "cell"}))


def stretch_move(n_atoms: int, step_size: float = 0.1, weight: float = 1.0,
                 max_volume_per_atom: float = 1e4, min_volume_per_atom: float = 1.0,
                 min_aspect_ratio: float = 0.8) -> MoveKernel:
    """Convenience: ``moves[].type: stretch`` with the ``cell:`` section defaults."""
    return MoveKernel("stretch", stretch.build_kernel,
                      kernel_kwargs={"n_atoms": n_atoms, "max_vol_per_atom": max_volume_per_atom,
                                     "min_vol_per_atom": min_volume_per_atom,
                                     "min_aspect": min_aspect_ratio},
                      weight=weight, step_size=step_size,
                      reject_reasons=frozenset({"energy", "cell"}),
                      mutates=frozenset({"positions", "cell"}))
