"""ctypes mirror of ``include/jaxrens_b200.h`` and the library loader.

The CUDA library is the only compute path: importing an operation whose
library is missing raises immediately (no CPU fallback exists).
"""

from __future__ import annotations

import ctypes as C
import os

MAX_SPECIES = 8
MAX_MOVES = 8
MAX_CULL = 32
MAX_IMAGES = 125
MAX_CENTERS = 8
MAX_ATOMS = 256

JR_OK = 0
ERRORS = {
    -1: "JR_ERR_SHAPE",
    -2: "JR_ERR_PARAM",
    -3: "JR_ERR_CUDA",
    -4: "JR_ERR_TIMEOUT",
    -5: "JR_ERR_WORKSPACE",
    -6: "JR_ERR_UNSUPPORTED",
}

MODEL_LJ, MODEL_GAUSS_MIX, MODEL_SW = 0, 1, 2
SW_MAX_ATOMS = 64
MOVE_GALILEAN, MOVE_VOLUME, MOVE_MORPH, MOVE_SWAP, MOVE_SHEAR, MOVE_STRETCH = 0, 1, 2, 3, 4, 5

_vp = C.c_void_p


class JrDims(C.Structure):
    _fields_ = [
        ("n_replicas", C.c_int32),
        ("n_walkers", C.c_int32),
        ("n_atoms_max", C.c_int32),
        ("n_moves", C.c_int32),
        ("n_mcmc_steps", C.c_int32),
        ("n_extra", C.c_int32),
        ("n_cull", C.c_int32),
        ("shared_move_key", C.c_int32),
    ]


class JrModelParams(C.Structure):
    _fields_ = [
        ("model", C.c_int32),
        ("n_species", C.c_int32),
        ("has_cutoff", C.c_int32),
        ("rc2", C.c_float),
        ("eps4", C.c_float * (MAX_SPECIES * MAX_SPECIES)),
        ("eps24", C.c_float * (MAX_SPECIES * MAX_SPECIES)),
        ("sig2", C.c_float * (MAX_SPECIES * MAX_SPECIES)),
        ("n_images", C.c_int32),
        ("img_off", C.c_float * (MAX_IMAGES * 3)),
        ("n_centers", C.c_int32),
        ("centers", C.c_float * (MAX_CENTERS * 3)),
        ("gm_sigma", C.c_float),
        ("sw_sigma", C.c_float),
        ("sw_rc", C.c_float),
        ("sw_gsig", C.c_float),
        ("sw_Aeps", C.c_float),
        ("sw_B", C.c_float),
        ("sw_leps", C.c_float),
    ]


class JrMoveParams(C.Structure):
    _fields_ = [
        ("n_moves", C.c_int32),
        ("type", C.c_int32 * MAX_MOVES),
        ("n_reflect", C.c_int32 * MAX_MOVES),
        ("perturb_angle", C.c_float * MAX_MOVES),
        ("cum_probs", C.c_float * MAX_MOVES),
        ("max_vpa", C.c_float),
        ("min_vpa", C.c_float),
        ("min_aspect", C.c_float),
        ("flat_v_prior", C.c_int32),
        ("gate", C.c_int32 * MAX_MOVES),
        ("dmin", C.c_float * (MAX_SPECIES * MAX_SPECIES)),
    ]


class JrParams(C.Structure):
    _fields_ = [
        ("model", JrModelParams),
        ("moves", JrMoveParams),
        ("log_alpha", C.c_double),
        ("w_offset", C.c_double * MAX_CULL),
    ]


class JrStateBuffers(C.Structure):
    _fields_ = [
        ("positions", _vp),
        ("direction", _vp),
        ("types", _vp),
        ("energy", _vp),
        ("energy64", _vp),
        ("cell", _vp),
        ("step_sizes", _vp),
        ("n_accepted", _vp),
        ("n_proposed", _vp),
        ("rng_key", _vp),
        ("log_evidence", _vp),
        ("iteration", _vp),
        ("emax", _vp),
        ("n_atoms", _vp),
        ("pressure", _vp),
        ("mu", _vp),
        ("move_key", _vp),
    ]


class JrInfoBuffers(C.Structure):
    _fields_ = [
        ("worst_idx", _vp),
        ("clone_idx", _vp),
        ("emax", _vp),
        ("log_evidence", _vp),
        ("dead_positions", _vp),
        ("dead_types", _vp),
        ("dead_cell", _vp),
        ("n_accepted", _vp),
        ("n_proposed", _vp),
        ("reject_reason_counts", _vp),
        ("n_evaluations", _vp),
        ("n_grad_evaluations", _vp),
        ("rounds", _vp),
        ("dead_energy", _vp),
        ("term_counts", _vp),
    ]


SUR_BASIS, SUR_HIDDEN, SUR_PARAMS = 16, 64, 5313


class JrSurrogate(C.Structure):
    _fields_ = [
        ("params", _vp),
        ("in_scale", C.c_float * SUR_BASIS),
        ("in_shift", C.c_float * SUR_BASIS),
        ("out_scale", C.c_float),
        ("out_shift", C.c_float),
        ("contour_shift", C.c_float),
        ("tau", C.c_float),
    ]


class JrSampleRing(C.Structure):
    _fields_ = [
        ("positions", _vp),
        ("cell", _vp),
        ("energy_u", _vp),
        ("capacity", C.c_int64),
        ("base", C.c_int64),
        ("n_surrogate_evaluations", _vp),
    ]


class JrLaunchConfig(C.Structure):
    _fields_ = [("threads", C.c_int32), ("tpa", C.c_int32), ("cluster", C.c_int32),
                ("warp_walkers", C.c_int32)]


#: Every symbol ``include/jaxrens_b200.h`` declares.
EXPORTED = (
    "jr_ns_iterate_workspace_size",
    "jr_ns_iterate",
    "jr_ns_iterate_static",
    "jr_move_trial",
    "jr_walk_population",
    "jr_energy_forces",
    "jr_re_swap",
    "jr_autotune",
    "jr_sur_descriptors",
    "jr_sur_train_workspace_size",
    "jr_sur_train_step",
    "jr_sur_energy_forces",
    "jr_ns_iterate_da",
    "jr_bench_fma_peak",
    "jr_last_error",
    "jr_version",
)

LIB_PATH = os.path.join(os.path.dirname(os.path.abspath(__file__)), "_lib",
                        "libjaxrens_b200.so")

_lib = None


class JrError(RuntimeError):
    """A C-ABI call returned a JR_ERR_* code."""

    def __init__(self, code: int, where: str, msg: str):
        super().__init__(f"{where}: {ERRORS.get(code, code)}: {msg}")
        self.code = code


def load():
    """Load the CUDA library (raises if it was not built)."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(LIB_PATH):
        raise RuntimeError(
            f"CUDA library missing at {LIB_PATH}; build it with "
            "`python -m jaxrens_b200._build` (there is no CPU fallback)"
        )
    L = C.CDLL(LIB_PATH)
    P = C.POINTER
    L.jr_last_error.restype = C.c_char_p
    L.jr_version.restype = C.c_int
    L.jr_ns_iterate_workspace_size.restype = C.c_size_t
    L.jr_ns_iterate_workspace_size.argtypes = [P(JrDims)]
    L.jr_ns_iterate.restype = C.c_int
    L.jr_ns_iterate.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), P(JrInfoBuffers), C.c_int32,
        P(JrLaunchConfig), _vp, C.c_size_t, _vp,
    ]
    L.jr_ns_iterate_static.restype = C.c_int
    L.jr_ns_iterate_static.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), P(JrInfoBuffers), C.c_int32,
        P(JrLaunchConfig), _vp,
    ]
    L.jr_move_trial.restype = C.c_int
    L.jr_move_trial.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), C.c_int32, C.c_int32, _vp, _vp,
        _vp, _vp, _vp, C.c_int32, _vp, _vp, _vp,
    ]
    L.jr_walk_population.restype = C.c_int
    L.jr_walk_population.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), C.c_int32, _vp, _vp, _vp, _vp,
    ]
    L.jr_energy_forces.restype = C.c_int
    L.jr_energy_forces.argtypes = [
        P(JrParams), C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp, _vp, _vp,
        _vp, _vp,
    ]
    L.jr_re_swap.restype = C.c_int
    L.jr_re_swap.argtypes = [
        P(JrDims), P(JrStateBuffers), C.c_uint32, C.c_uint32, C.c_int32, C.c_int32,
        _vp, _vp, _vp,
    ]
    L.jr_autotune.restype = C.c_int
    L.jr_autotune.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), C.c_int32, P(JrLaunchConfig), _vp,
    ]
    L.jr_sur_descriptors.restype = C.c_int
    L.jr_sur_descriptors.argtypes = [C.c_int32, C.c_int32, _vp, _vp, _vp, _vp]
    L.jr_sur_train_workspace_size.restype = C.c_size_t
    L.jr_sur_train_workspace_size.argtypes = [C.c_int32, C.c_int32]
    L.jr_sur_train_step.restype = C.c_int
    L.jr_sur_train_step.argtypes = [
        P(JrSurrogate), _vp, _vp, _vp, C.c_int32, C.c_int32, _vp, _vp, _vp, C.c_int32,
        C.c_float, _vp, _vp, C.c_size_t, _vp,
    ]
    L.jr_sur_energy_forces.restype = C.c_int
    L.jr_sur_energy_forces.argtypes = [
        P(JrSurrogate), C.c_int32, C.c_int32, _vp, _vp, _vp, _vp, _vp, _vp,
    ]
    L.jr_ns_iterate_da.restype = C.c_int
    L.jr_ns_iterate_da.argtypes = [
        P(JrDims), P(JrParams), P(JrStateBuffers), P(JrInfoBuffers), P(JrSurrogate),
        P(JrSampleRing), C.c_int32, P(JrLaunchConfig), _vp, C.c_size_t, _vp,
    ]
    L.jr_bench_fma_peak.restype = C.c_int
    L.jr_bench_fma_peak.argtypes = [C.c_int, C.c_int, _vp, C.POINTER(C.c_double), _vp]
    _lib = L
    return L


def check(rc: int, where: str) -> None:
    if rc != JR_OK:
        msg = load().jr_last_error().decode(errors="replace")
        raise JrError(rc, where, msg)
