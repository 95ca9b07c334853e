"""ctypes binding of the CPU oracle (TEST INFRASTRUCTURE ONLY).

The oracle restates jaxrens's nested-sampling walk in C (``jr_oracle.c``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg may import this module; the product package never does.  Parity status
is documented in the C header and in the repository's design notes:
threefry is pinned by the Random123 known-answer vectors, the LJ +
EnsembleTerm energy by the reference's committed ``lj8_npt`` trajectory
frames, and the JAX-specific transforms (normal via erf_inv) are restated
from the published algorithms without a JAX-produced pin.
"""

from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "libjr_oracle.so")

DEV, REF32, F64 = 0, 1, 2
GALILEAN, VOLUME, MORPH, SWAP = 0, 1, 2, 3
MODEL_LJ, MODEL_GAUSS_MIX, MODEL_SW = 0, 1, 2
MAX_SPECIES, MAX_MOVES, MAX_IMAGES, MAX_CENTERS = 8, 8, 125, 8

_f = C.POINTER(C.c_float)
_d = C.POINTER(C.c_double)
_i = C.POINTER(C.c_int32)
_u = C.POINTER(C.c_uint32)


class JroModel(C.Structure):
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


class JroMoves(C.Structure):
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


class JroReplica(C.Structure):
    _fields_ = [
        ("n_walkers", C.c_int32),
        ("n_atoms", C.c_int32),
        ("positions", _f),
        ("direction", _f),
        ("types", _i),
        ("energy", _d),
        ("cell", _f),
        ("step_sizes", _f),
        ("n_acc", _i),
        ("n_prop", _i),
        ("rng_key", _u),
        ("log_evidence", _d),
        ("iteration", _i),
        ("emax", _d),
        ("pressure", C.c_float),
        ("mu", C.c_float * MAX_SPECIES),
        ("has_mu", C.c_int32),
    ]


class JroIterInfo(C.Structure):
    _fields_ = [
        ("worst_idx", C.c_int32),
        ("clone_idx", C.c_int32),
        ("emax", C.c_double),
        ("dead_energy", C.c_double),
        ("n_acc", C.c_int32 * MAX_MOVES),
        ("n_prop", C.c_int32 * MAX_MOVES),
        ("rr", C.c_int32 * (MAX_MOVES * 4)),
        ("n_evals", C.c_int32 * MAX_MOVES),
        ("n_grad", C.c_int32 * MAX_MOVES),
        ("total_accepted", C.c_int32),
    ]


def build() -> str:
    """Compile the oracle with its Makefile (idempotent)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        L = C.CDLL(_LIB_PATH)
        L.jro_bits32.restype = C.c_uint32
        L.jro_uniform.restype = C.c_float
        L.jro_uniform.argtypes = [C.c_uint32, C.c_float, C.c_float]
        L.jro_normal.restype = C.c_float
        L.jro_normal.argtypes = [C.c_uint32]
        L.jro_erfinv.restype = C.c_float
        L.jro_erfinv.argtypes = [C.c_float]
        L.jro_sw_exp.restype = C.c_float
        L.jro_sw_exp.argtypes = [C.c_float]
        L.jro_randint.restype = C.c_int32
        L.jro_choice.restype = C.c_int32
        L.jro_det3.restype = C.c_float
        L.jro_energy.restype = C.c_double
        L.jro_energy.argtypes = [
            C.POINTER(JroModel), C.c_int32, C.c_int32, _f, _i, _f, C.c_float,
            _f, C.c_int32, _d, _d,
        ]
        L.jro_move_trial.restype = C.c_int32
        L.jro_move_trial.argtypes = [
            C.POINTER(JroModel), C.POINTER(JroMoves), C.c_int32, C.c_int32,
            _u, C.c_float, C.c_double, C.c_int32, _f, _f, _i, _f, _d,
            C.c_float, _f, C.c_int32, _i,
        ]
        L.jro_ns_step.argtypes = [
            C.POINTER(JroModel), C.POINTER(JroMoves), C.c_int32,
            C.POINTER(JroReplica), C.c_int32, C.c_int32, _u, C.c_double,
            C.c_double, C.POINTER(JroIterInfo), _f, _i, _f,
        ]
        L.jro_ns_step_n.argtypes = [
            C.POINTER(JroModel), C.POINTER(JroMoves), C.c_int32,
            C.POINTER(JroReplica), C.c_int32, C.c_int32, C.c_int32, _u, C.c_double,
            _d, C.POINTER(JroIterInfo), _i, _i, _d, _f, _i, _f,
        ]
        L.jro_min_distance_ok.argtypes = [C.POINTER(JroMoves), C.c_int32, C.c_int32, _f, _i,
                                          _f, C.c_int32]
        L.jro_walk_population.argtypes = [
            C.POINTER(JroModel), C.POINTER(JroMoves), C.c_int32, C.POINTER(JroReplica),
            C.c_int32, _u, _u, C.c_double,
        ]
        L.jro_ns_step_batched.argtypes = [
            C.POINTER(JroModel), C.POINTER(JroMoves), C.c_int32,
            C.POINTER(JroReplica), C.c_int32, C.c_int32, C.c_int32, C.c_int32,
            C.c_double, C.c_double, C.POINTER(JroIterInfo), C.c_int32,
        ]
        L.jro_re_step.argtypes = [
            C.POINTER(JroReplica), C.c_int32, _u, C.c_int32, C.c_int32, _i, _i,
        ]
        L.jro_init_walkers.argtypes = [_u, C.c_int32, C.c_int32, C.c_float, _f, _f]
        _lib = L
    return _lib


def _p(a, t):
    return a.ctypes.data_as(t)


# ---------------------------------------------------------------- RNG ----
def threefry2x32(key, ctr):
    out = np.zeros(2, np.uint32)
    lib().jro_threefry2x32(
        C.c_uint32(int(key[0])), C.c_uint32(int(key[1])),
        C.c_uint32(int(ctr[0])), C.c_uint32(int(ctr[1])), _p(out, _u),
    )
    return out


def key(seed: int) -> np.ndarray:
    """jax.random.key(seed) data for a 32-bit seed: (0, seed)."""
    return np.array([0, seed & 0xFFFFFFFF], np.uint32)


def split(k, n: int = 2) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    out = np.zeros((n, 2), np.uint32)
    for i in range(n):
        lib().jro_split(_p(k, _u), C.c_uint32(i), _p(out[i], _u))
    return out


def fold_in(k, data: int) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    out = np.zeros(2, np.uint32)
    lib().jro_fold_in(_p(k, _u), C.c_uint32(data), _p(out, _u))
    return out


def split_original(k, n: int = 2) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    out = np.zeros((n, 2), np.uint32)
    lib().jro_split_original(_p(k, _u), C.c_int32(n), _p(out, _u))
    return out


def random_bits(k, n: int) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    return np.array([lib().jro_bits32(_p(k, _u), C.c_uint32(i)) for i in range(n)], np.uint32)


def uniform(k, n: int) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    out = np.zeros(n, np.float32)
    lib().jro_uniform_array(_p(k, _u), C.c_int32(n), _p(out, _f))
    return out


def normal(k, n: int) -> np.ndarray:
    k = np.ascontiguousarray(k, np.uint32)
    out = np.zeros(n, np.float32)
    lib().jro_normal_array(_p(k, _u), C.c_int32(n), _p(out, _f))
    return out


def randint(k, lo: int, hi: int) -> int:
    k = np.ascontiguousarray(k, np.uint32)
    return int(lib().jro_randint(_p(k, _u), C.c_int32(lo), C.c_int32(hi)))


def choice(k, cum) -> int:
    k = np.ascontiguousarray(k, np.uint32)
    cum = np.ascontiguousarray(cum, np.float32)
    return int(lib().jro_choice(_p(k, _u), _p(cum, _f), C.c_int32(len(cum))))


# -------------------------------------------------------------- model ----
def make_model(eps4, eps24, sig2, rc2=None, img_off=None, model=MODEL_LJ,
               centers=None, gm_sigma=0.5) -> JroModel:
    m = JroModel()
    m.model = model
    eps4 = np.atleast_2d(np.asarray(eps4, np.float32))
    S = eps4.shape[0]
    m.n_species = S
    m.has_cutoff = 0 if rc2 is None else 1
    m.rc2 = np.float32(rc2 if rc2 is not None else np.inf)
    for name, arr in (("eps4", eps4), ("eps24", eps24), ("sig2", sig2)):
        a = np.atleast_2d(np.asarray(arr, np.float32)).reshape(-1)
        getattr(m, name)[: S * S] = a.tolist()
    if img_off is None:
        img_off = np.zeros((1, 3), np.float32)
    img_off = np.asarray(img_off, np.float32).reshape(-1, 3)
    m.n_images = img_off.shape[0]
    m.img_off[: img_off.size] = img_off.reshape(-1).tolist()
    if centers is not None:
        c = np.asarray(centers, np.float32).reshape(-1, 3)
        m.n_centers = c.shape[0]
        m.centers[: c.size] = c.reshape(-1).tolist()
        m.gm_sigma = np.float32(gm_sigma)
    return m


def make_sw_model(sw_sigma, sw_rc, sw_gsig, sw_Aeps, sw_B, sw_leps) -> JroModel:
    """Stillinger-Weber model from the float32 constants of the kernel
    contract (one species, the single minimum image)."""
    m = JroModel()
    m.model = MODEL_SW
    m.n_species = 1
    m.has_cutoff = 1
    m.sw_sigma, m.sw_rc, m.sw_gsig = (float(np.float32(v)) for v in (sw_sigma, sw_rc, sw_gsig))
    m.sw_Aeps, m.sw_B, m.sw_leps = (float(np.float32(v)) for v in (sw_Aeps, sw_B, sw_leps))
    m.rc2 = sw_cutoff_sq(sw_rc)
    m.n_images = 1
    return m


def sw_cutoff_sq(rc) -> np.float32:
    """The smallest float32 x whose float32 square root reaches rc: then
    r2 < x is exactly sqrt(r2) < rc."""
    rc = np.float32(rc)
    x = np.float32(rc * rc)
    while np.sqrt(x) >= rc:
        x = np.nextafter(x, np.float32(0))
    while np.sqrt(x) < rc:
        x = np.nextafter(x, np.float32(np.inf))
    return x


def sw_exp(x: float) -> float:
    """The SW kernel's float32 exp, evaluated by the oracle."""
    return float(lib().jro_sw_exp(float(x)))


def make_moves(types, n_reflect, perturb_angle, cum_probs, max_vpa=1e4,
               min_vpa=1.0, min_aspect=0.8, flat_v_prior=False, gate=None,
               dmin=None) -> JroMoves:
    mv = JroMoves()
    M = len(types)
    mv.n_moves = M
    mv.type[:M] = list(types)
    mv.n_reflect[:M] = list(n_reflect)
    mv.perturb_angle[:M] = [float(x) for x in perturb_angle]
    mv.cum_probs[:M] = [float(x) for x in np.asarray(cum_probs, np.float32)]
    mv.max_vpa = max_vpa
    mv.min_vpa = min_vpa
    mv.min_aspect = min_aspect
    mv.flat_v_prior = int(flat_v_prior)
    if gate is not None:
        mv.gate[:M] = [int(g) for g in gate]
    if dmin is not None:
        dm = np.asarray(dmin, np.float32).reshape(-1)
        mv.dmin[: dm.size] = dm.tolist()
    return mv


def energy(model, x, types, cell, pressure=0.0, mu=None, mode=DEV, forces=True):
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
    n = x.shape[0]
    t = np.ascontiguousarray(types, np.int32).reshape(n)
    c = np.ascontiguousarray(cell, np.float32).reshape(9)
    F = np.zeros((n, 3), np.float64) if forces else None
    u = C.c_double(0.0)
    has_mu = mu is not None
    muv = np.zeros(MAX_SPECIES, np.float32)
    if has_mu:
        muv[: len(mu)] = np.asarray(mu, np.float32)
    E = lib().jro_energy(
        C.byref(model), mode, n, _p(x, _f), _p(t, _i), _p(c, _f),
        C.c_float(pressure), _p(muv, _f), int(has_mu),
        _p(F, _d) if F is not None else None, C.byref(u),
    )
    return E, F, u.value


class Replica:
    """numpy-owned replica population for the oracle's ns_step."""

    def __init__(self, positions, types, energy, cell, step_sizes, rng_key,
                 pressure=0.0, mu=None, direction=None, log_evidence=-np.inf,
                 iteration=0, emax=np.inf):
        self.positions = np.ascontiguousarray(positions, np.float32).copy()
        K, N, _ = self.positions.shape
        self.direction = (np.zeros_like(self.positions) if direction is None
                          else np.ascontiguousarray(direction, np.float32).copy())
        self.types = np.ascontiguousarray(np.broadcast_to(types, (K, N)), np.int32).copy()
        self.energy = np.ascontiguousarray(energy, np.float64).copy()
        self.cell = np.ascontiguousarray(cell, np.float32).reshape(K, 3, 3).copy()
        self.step_sizes = np.ascontiguousarray(step_sizes, np.float32).copy()
        M = self.step_sizes.shape[1]
        self.n_acc = np.zeros((K, M), np.int32)
        self.n_prop = np.zeros((K, M), np.int32)
        self.rng_key = np.ascontiguousarray(rng_key, np.uint32).copy()
        self.log_evidence = np.array([log_evidence], np.float64)
        self.iteration = np.array([iteration], np.int32)
        self.emax = np.array([emax], np.float64)
        self.pressure = float(pressure)
        self.mu = mu

    def cstruct(self) -> JroReplica:
        r = JroReplica()
        K, N, _ = self.positions.shape
        r.n_walkers, r.n_atoms = K, N
        r.positions = _p(self.positions, _f)
        r.direction = _p(self.direction, _f)
        r.types = _p(self.types, _i)
        r.energy = _p(self.energy, _d)
        r.cell = _p(self.cell, _f)
        r.step_sizes = _p(self.step_sizes, _f)
        r.n_acc = _p(self.n_acc, _i)
        r.n_prop = _p(self.n_prop, _i)
        r.rng_key = _p(self.rng_key, _u)
        r.log_evidence = _p(self.log_evidence, _d)
        r.iteration = _p(self.iteration, _i)
        r.emax = _p(self.emax, _d)
        r.pressure = self.pressure
        if self.mu is not None:
            r.mu[: len(self.mu)] = [float(v) for v in np.asarray(self.mu, np.float32)]
            r.has_mu = 1
        return r


def ns_step(model, moves, rep: Replica, n_mcmc_steps, log_alpha, w_offset,
            n_extra=0, move_key=None, mode=DEV):
    info = JroIterInfo()
    K, N, _ = rep.positions.shape
    dx = np.zeros((N, 3), np.float32)
    dt = np.zeros(N, np.int32)
    dc = np.zeros((3, 3), np.float32)
    cs = rep.cstruct()
    mk = None if move_key is None else np.ascontiguousarray(move_key, np.uint32)
    lib().jro_ns_step(
        C.byref(model), C.byref(moves), mode, C.byref(cs), n_mcmc_steps, n_extra,
        _p(mk, _u) if mk is not None else None, log_alpha, w_offset,
        C.byref(info), _p(dx, _f), _p(dt, _i), _p(dc, _f),
    )
    return info, dx, dt, dc


def ns_step_n(model, moves, rep: Replica, n_mcmc_steps, log_alpha, w_offsets, n_cull,
              n_extra=0, move_key=None, mode=DEV):
    """ns_step with n_cull culls: returns (info, worst, clone, dead_energy,
    dead_positions, dead_types, dead_cell) with a leading (n_cull,) axis."""
    info = JroIterInfo()
    K, N, _ = rep.positions.shape
    wo = np.ascontiguousarray(np.broadcast_to(np.asarray(w_offsets, np.float64), (n_cull,)))
    worst = np.zeros(n_cull, np.int32)
    clone = np.zeros(n_cull, np.int32)
    de = np.zeros(n_cull, np.float64)
    dx = np.zeros((n_cull, N, 3), np.float32)
    dt = np.zeros((n_cull, N), np.int32)
    dc = np.zeros((n_cull, 3, 3), np.float32)
    cs = rep.cstruct()
    mk = None if move_key is None else np.ascontiguousarray(move_key, np.uint32)
    lib().jro_ns_step_n(
        C.byref(model), C.byref(moves), mode, C.byref(cs), n_mcmc_steps, n_cull, n_extra,
        _p(mk, _u) if mk is not None else None, log_alpha, _p(wo, _d), C.byref(info),
        _p(worst, _i), _p(clone, _i), _p(de, _d), _p(dx, _f), _p(dt, _i), _p(dc, _f),
    )
    return info, worst, clone, de, dx, dt, dc


def min_distance_ok(moves, n_species, x, types, cell, mode=DEV) -> bool:
    x = np.ascontiguousarray(x, np.float32).reshape(-1, 3)
    t = np.ascontiguousarray(types, np.int32)
    c = np.ascontiguousarray(cell, np.float32).reshape(9)
    return bool(lib().jro_min_distance_ok(C.byref(moves), n_species, x.shape[0], _p(x, _f),
                                          _p(t, _i), _p(c, _f), mode))


def walk_population(model, moves, rep: Replica, walklength, run_key, move_key, emax,
                    mode=DEV):
    """Burn-in walk of every walker of one run, in place."""
    cs = rep.cstruct()
    rk = np.ascontiguousarray(run_key, np.uint32)
    mk = np.ascontiguousarray(move_key, np.uint32)
    lib().jro_walk_population(C.byref(model), C.byref(moves), mode, C.byref(cs), int(walklength),
                              _p(rk, _u), _p(mk, _u), float(emax))


def ns_step_batched(model, moves, reps, n_mcmc_steps, log_alpha, w_offset,
                    n_extra=0, shared_move_key=True, mode=DEV, n_threads=1):
    arr = (JroReplica * len(reps))(*[r.cstruct() for r in reps])
    infos = (JroIterInfo * len(reps))()
    lib().jro_ns_step_batched(
        C.byref(model), C.byref(moves), mode, arr, len(reps), n_mcmc_steps,
        n_extra, int(shared_move_key), log_alpha, w_offset, infos, n_threads,
    )
    return list(infos)


def re_step(reps, key_, n_swap_cycles=1, mode=DEV):
    arr = (JroReplica * len(reps))(*[r.cstruct() for r in reps])
    k = np.ascontiguousarray(key_, np.uint32)
    acc = np.zeros(max(len(reps) - 1, 1), np.int32)
    att = np.zeros(max(len(reps) - 1, 1), np.int32)
    lib().jro_re_step(arr, len(reps), _p(k, _u), n_swap_cycles, mode,
                      _p(acc, _i), _p(att, _i))
    return acc, att


def init_walkers(key_, n_walkers, n_atoms, v_hi):
    k = np.ascontiguousarray(key_, np.uint32)
    pos = np.zeros((n_walkers, n_atoms, 3), np.float32)
    cell = np.zeros((n_walkers, 3, 3), np.float32)
    lib().jro_init_walkers(_p(k, _u), n_walkers, n_atoms, np.float32(v_hi),
                           _p(pos, _f), _p(cell, _f))
    return pos, cell


def move_trial(model, moves, move_idx, key_, step, emax, x, d, types, cell,
               energy_, pressure=0.0, mu=None, mode=DEV):
    x = np.ascontiguousarray(x, np.float32).copy()
    d = np.ascontiguousarray(d, np.float32).copy()
    t = np.ascontiguousarray(types, np.int32).copy()
    c = np.ascontiguousarray(cell, np.float32).reshape(9).copy()
    e = C.c_double(energy_)
    k = np.ascontiguousarray(key_, np.uint32)
    muv = np.zeros(MAX_SPECIES, np.float32)
    if mu is not None:
        muv[: len(mu)] = np.asarray(mu, np.float32)
    reason = C.c_int32(0)
    acc = lib().jro_move_trial(
        C.byref(model), C.byref(moves), mode, move_idx, _p(k, _u),
        C.c_float(step), C.c_double(emax), x.shape[0], _p(x, _f), _p(d, _f),
        _p(t, _i), _p(c, _f), C.byref(e), C.c_float(pressure), _p(muv, _f),
        int(mu is not None), C.byref(reason),
    )
    return bool(acc), x, d, t, c.reshape(3, 3), e.value, int(reason.value)
