"""Energy backends: LJ + EnsembleTerm composed in a Hamiltonian.

Mirrors the reference's backend API (``backends/lj.py``, ``backends/ensemble.py``,
``backends/hamiltonian.py``, ``backends/base.py``): ``create_lj`` builds an
``LJBackend`` from scalar, per-species (Lorentz-Berthelot) or full pair tables;
``Hamiltonian(model, [EnsembleTerm(...)])`` adds ``P*V - mu*N``.  Calling a
backend evaluates on the GPU through ``jr_energy_forces``; the descriptors are
also what the NS kernels read (``model_params``).
"""

from __future__ import annotations

import ctypes as C
from collections.abc import Sequence
from typing import Any, NamedTuple

import numpy as np

from . import _lib

_ScalarOrSeq = float | Sequence[float] | np.ndarray


def make_image_offsets(sc_a: int, sc_b: int, sc_c: int) -> np.ndarray:
    """Centred integer image offsets of a supercell (``_graph_neighbors.py:20-33``)."""
    a = np.arange(-(sc_a // 2), sc_a // 2 + 1)
    b = np.arange(-(sc_b // 2), sc_b // 2 + 1)
    c = np.arange(-(sc_c // 2), sc_c // 2 + 1)
    grid = np.stack(np.meshgrid(a, b, c, indexing="ij"), axis=-1)
    return grid.reshape(-1, 3)


class BackendResult(NamedTuple):
    """Return value of backend calls (``backends/base.py:33-71``)."""

    energy: Any
    forces: Any = None
    max_neighbor_count: Any = 0
    overflow: Any = False


class LJBackend:
    """All-pairs Lennard-Jones with triclinic minimum image, supercell images
    and a hard cutoff (``backends/lj.py:125-204``).

    ``epsilon``/``sigma``: scalars (one species), 1-D per-species tables
    (Lorentz-Berthelot mixing, the reference's mode), or -- beyond the
    reference -- full symmetric ``S x S`` pair tables (``pair_tables=True``),
    which express mixtures such as Kob-Andersen.
    """

    def __init__(self, epsilon: _ScalarOrSeq = 1.0, sigma: _ScalarOrSeq = 1.0,
                 cutoff: float | None = None,
                 supercell_trafo: tuple[int, int, int] = (1, 1, 1)):
        eps = np.asarray(epsilon, np.float32)
        sig = np.asarray(sigma, np.float32)
        if eps.ndim != sig.ndim:
            raise ValueError(
                f"epsilon (rank {eps.ndim}) and sigma (rank {sig.ndim}) differ in rank; "
                "pass two scalars, two per-species vectors or two pair tables")
        if eps.ndim > 2:
            raise ValueError(f"rank-{eps.ndim} epsilon/sigma: only scalars, per-species "
                             "vectors and S x S pair tables are accepted")
        if eps.ndim >= 1 and eps.shape != sig.shape:
            raise ValueError(
                f"epsilon has shape {eps.shape} but sigma has shape {sig.shape}; "
                "give both one entry per species")
        if eps.ndim >= 1 and eps.shape[0] == 0:
            raise ValueError("empty epsilon/sigma tables: a species table needs at least one entry")
        if eps.ndim == 2 and (eps.shape[0] != eps.shape[1] or not np.array_equal(eps, eps.T)
                              or not np.array_equal(sig, sig.T)):
            raise ValueError("pair tables must be square and symmetric")
        self.cutoff = cutoff
        self.r_cutoff = cutoff if cutoff is not None else 0.0
        sc = tuple(int(x) for x in supercell_trafo)
        if min(sc) < 1:
            raise ValueError(f"supercell_trafo entries must be >= 1, got {supercell_trafo}")
        self.supercell_trafo = sc
        self.image_offsets = make_image_offsets(*sc).astype(np.float32)
        if len(self.image_offsets) > _lib.MAX_IMAGES:
            raise ValueError("supercell_trafo gives more than 125 images")
        if eps.ndim == 0:
            # scalar mode: sigma**2 and 4*eps are Python-double constants the
            # reference folds into float32 (lj.py:193-196)
            e, s = float(epsilon), float(sigma)
            self.n_species = 1
            self.eps4 = np.array([[4.0 * e]], np.float32)
            self.eps24 = np.array([[24.0 * e]], np.float32)
            self.sig2 = np.array([[s * s]], np.float32)
            self.epsilon, self.sigma = e, s
        else:
            if eps.ndim == 1:
                # Lorentz-Berthelot in float32 (lj.py:175-189)
                eps_ij = np.sqrt(eps[:, None] * eps[None, :]).astype(np.float32)
                sig_ij = (np.float32(0.5) * (sig[:, None] + sig[None, :])).astype(np.float32)
            else:
                eps_ij, sig_ij = eps, sig
            self.n_species = int(eps_ij.shape[0])
            self.eps4 = (np.float32(4.0) * eps_ij).astype(np.float32)
            self.eps24 = (24.0 * eps_ij.astype(np.float64)).astype(np.float32)
            self.sig2 = (sig_ij * sig_ij).astype(np.float32)
            self.epsilon = self.sigma = None
        if self.n_species > _lib.MAX_SPECIES:
            raise ValueError("at most 8 species are supported")

    def model_params(self) -> _lib.JrModelParams:
        m = _lib.JrModelParams()
        m.model = _lib.MODEL_LJ
        S = self.n_species
        m.n_species = S
        m.has_cutoff = 0 if self.cutoff is None else 1
        m.rc2 = float(np.float32(self.cutoff ** 2)) if self.cutoff is not None else float("inf")
        m.eps4[: S * S] = self.eps4.reshape(-1).tolist()
        m.eps24[: S * S] = self.eps24.reshape(-1).tolist()
        m.sig2[: S * S] = self.sig2.reshape(-1).tolist()
        m.n_images = len(self.image_offsets)
        m.img_off[: self.image_offsets.size] = self.image_offsets.reshape(-1).tolist()
        return m

    def __call__(self, positions, species, cell, max_neighbors: int = 0,
                 ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self, None, positions, species, cell, forces=False)

    def energy_and_forces(self, positions, species, cell, max_neighbors: int = 0,
                          ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self, None, positions, species, cell, forces=True)


def create_lj(epsilon: _ScalarOrSeq = 1.0, sigma: _ScalarOrSeq = 1.0,
              cutoff: float | None = None,
              supercell_trafo: tuple[int, int, int] = (1, 1, 1)) -> LJBackend:
    return LJBackend(epsilon=epsilon, sigma=sigma, cutoff=cutoff,
                     supercell_trafo=supercell_trafo)


class GaussianMixtureBackend:
    """Gaussian-mixture toy (``backends/toy.py:163-204``) with analytic log Z;
    a validation target for the evidence accumulator."""

    def __init__(self, centers=None, sigma: float = 0.5):
        if centers is None:
            centers = [[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]]
        self.centers = np.asarray(centers, np.float32).reshape(-1, 3)
        if len(self.centers) > _lib.MAX_CENTERS:
            raise ValueError("at most 8 centers")
        self.sigma = float(sigma)
        self.r_cutoff = 0.0
        self.n_species = 1

    def model_params(self) -> _lib.JrModelParams:
        m = _lib.JrModelParams()
        m.model = _lib.MODEL_GAUSS_MIX
        m.n_species = 1
        m.n_images = 1
        m.n_centers = len(self.centers)
        m.centers[: self.centers.size] = self.centers.reshape(-1).tolist()
        m.gm_sigma = self.sigma
        m.eps4[0] = m.eps24[0] = m.sig2[0] = 0.0
        return m

    def log_evidence(self, half_width: float) -> float:
        """Analytic log Z for one atom, uniform prior on a cube of side
        ``2*half_width`` containing all the mixture mass."""
        return float(np.log(len(self.centers)) - 3.0 * np.log(2.0 * half_width))

    def __call__(self, positions, species, cell, max_neighbors=0, ensemble_params=None):
        return _evaluate(self, None, positions, species, cell, forces=False)

    def energy_and_forces(self, positions, species, cell, max_neighbors=0,
                          ensemble_params=None):
        return _evaluate(self, None, positions, species, cell, forces=True)


class StillingerWeberBackend:
    """Stillinger-Weber potential (F. H. Stillinger and T. A. Weber, Phys.
    Rev. B 31, 5262 (1985)) for one species with the exponents p = 4, q = 0:
    two-body ``A eps (B (sigma/r)^4 - 1) exp(sigma / (r - a sigma))`` and
    three-body ``lambda eps (cos theta + 1/3)^2 g(r_ij) g(r_ik)``,
    ``g(r) = exp(gamma sigma / (r - a sigma))``, zero beyond ``a sigma``,
    under the single minimum image.

    The reference has no such backend; it takes one through its
    ``EnergyBackend`` protocol (``backends/base.py:165-212``), which this
    class follows (``__call__``, ``energy_and_forces``, ``r_cutoff``).
    Defaults are the silicon parameters (eV, Angstrom).
    """

    def __init__(self, epsilon: float = 2.1683, sigma: float = 2.0951, a: float = 1.8,
                 lambda_: float = 21.0, gamma: float = 1.2, A: float = 7.049556277,
                 B: float = 0.6022245584, p: int = 4, q: int = 0):
        if int(p) != 4 or int(q) != 0:
            raise NotImplementedError(
                f"the Stillinger-Weber kernels take the exponents p = 4, q = 0 (got p={p}, q={q})")
        if min(epsilon, sigma, a) <= 0.0:
            raise ValueError("epsilon, sigma and a must be positive")
        self.epsilon, self.sigma, self.a = float(epsilon), float(sigma), float(a)
        self.lambda_, self.gamma, self.A, self.B = float(lambda_), float(gamma), float(A), float(B)
        self.n_species = 1
        self.cutoff = self.a * self.sigma
        self.r_cutoff = self.cutoff
        f = np.float32
        # the float32 constants of the kernel contract, rounded once here
        self.consts = dict(sw_sigma=f(sigma), sw_rc=f(self.a * self.sigma),
                           sw_gsig=f(self.gamma * self.sigma), sw_Aeps=f(self.A * self.epsilon),
                           sw_B=f(self.B), sw_leps=f(self.lambda_ * self.epsilon))
        # the pair test of the kernels is r^2 < rc2 with rc2 the smallest
        # float32 whose square root reaches the cutoff: exactly r < a sigma
        rc = self.consts["sw_rc"]
        x = np.float32(rc * rc)
        while np.sqrt(x) >= rc:
            x = np.nextafter(x, np.float32(0))
        while np.sqrt(x) < rc:
            x = np.nextafter(x, np.float32(np.inf))
        self.rc2 = x

    def model_params(self) -> _lib.JrModelParams:
        m = _lib.JrModelParams()
        m.model = _lib.MODEL_SW
        m.n_species = 1
        m.has_cutoff = 1
        m.rc2 = float(self.rc2)
        m.n_images = 1
        for k, v in self.consts.items():
            setattr(m, k, float(v))
        return m

    def __call__(self, positions, species, cell, max_neighbors: int = 0,
                 ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self, None, positions, species, cell, forces=False)

    def energy_and_forces(self, positions, species, cell, max_neighbors: int = 0,
                          ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self, None, positions, species, cell, forces=True)


def create_sw(epsilon: float = 2.1683, sigma: float = 2.0951, a: float = 1.8,
              lambda_: float = 21.0, gamma: float = 1.2, A: float = 7.049556277,
              B: float = 0.6022245584, p: int = 4, q: int = 0) -> StillingerWeberBackend:
    return StillingerWeberBackend(epsilon=epsilon, sigma=sigma, a=a, lambda_=lambda_,
                                  gamma=gamma, A=A, B=B, p=p, q=q)


#: eV / Angstrom^3 per GPa (pressures of the Stillinger-Weber workloads)
EV_PER_A3_PER_GPA = 0.006241509


class EnergyTerm:
    """Additive model-independent term (``backends/hamiltonian.py:54-86``)."""


class EnsembleTerm(EnergyTerm):
    """``P*V - mu*N`` (``backends/ensemble.py:90-133``); zero forces.  Per-run
    ``ensemble_params`` (``pressure``, ``chemical_potentials``) override the
    defaults given here."""

    def __init__(self, pressure: float = 0.0, chemical_potentials=None):
        self.pressure = pressure
        self.chemical_potentials = chemical_potentials

    def resolve(self, ensemble_params: dict | None):
        p, mu = self.pressure, self.chemical_potentials
        if ensemble_params is not None:
            p = ensemble_params.get("pressure", p)
            mu = ensemble_params.get("chemical_potentials", mu)
        return p, mu


class Hamiltonian:
    """``H = U_model + sum(terms)`` (``backends/hamiltonian.py:89-153``).  This
    build supports one model plus at most one ``EnsembleTerm``."""

    def __init__(self, model, terms: Sequence[EnergyTerm] = ()):
        if isinstance(model, Hamiltonian):
            terms = (*model.terms, *terms)
            model = model.model
        self.model = model
        self.terms = tuple(terms)
        ens = [t for t in self.terms if isinstance(t, EnsembleTerm)]
        if len(ens) > 1 or len(ens) != len(self.terms):
            raise NotImplementedError("only a single EnsembleTerm is supported as a term")
        self.ensemble = ens[0] if ens else None
        self.r_cutoff = model.r_cutoff

    @property
    def n_species(self) -> int:
        return self.model.n_species

    def with_terms(self, *terms: EnergyTerm) -> Hamiltonian:
        return Hamiltonian(self.model, (*self.terms, *terms))

    def model_params(self) -> _lib.JrModelParams:
        return self.model.model_params()

    def ensemble_values(self, ensemble_params: dict | None):
        if self.ensemble is None:
            return 0.0, None
        return self.ensemble.resolve(ensemble_params)

    def __call__(self, positions, species, cell, max_neighbors: int = 0,
                 ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self.model, self.ensemble_values(ensemble_params), positions,
                         species, cell, forces=False)

    def energy_and_forces(self, positions, species, cell, max_neighbors: int = 0,
                          ensemble_params: dict | None = None) -> BackendResult:
        return _evaluate(self.model, self.ensemble_values(ensemble_params), positions,
                         species, cell, forces=True)


def unwrap_model(backend):
    return backend.model if isinstance(backend, Hamiltonian) else backend


def eval_energy_and_forces(backend, positions, species, cell, max_neighbors=0,
                           ensemble_params=None) -> BackendResult:
    """``backends/base.py:74-113``: the native force path of the backend."""
    return backend.energy_and_forces(positions, species, cell, max_neighbors,
                                     ensemble_params=ensemble_params)


def _evaluate(model, ens, positions, species, cell, forces: bool) -> BackendResult:
    """Batch evaluation on the GPU.  ``positions`` (..., N, 3) torch or numpy;
    returns float64 energies (and float32 forces) as torch tensors on CUDA."""
    import torch

    from ._device import device

    dev = device()
    x = torch.as_tensor(positions, dtype=torch.float32, device=dev)
    single = x.dim() == 2
    if single:
        x = x[None]
    B, N, _ = x.shape
    t = torch.as_tensor(species, dtype=torch.int32, device=dev)
    t = t.expand(B, N).contiguous() if t.dim() == 1 else t.reshape(B, N).contiguous()
    c = torch.as_tensor(cell, dtype=torch.float32, device=dev).reshape(-1, 9)
    c = c.expand(B, 9).contiguous() if c.shape[0] == 1 else c.contiguous()
    pressure, mu = (0.0, None) if ens is None else ens
    pr = torch.as_tensor(pressure, dtype=torch.float32, device=dev).reshape(-1)
    pr = pr.expand(B).contiguous() if pr.numel() == 1 else pr.contiguous()
    mu_t = None
    if mu is not None:
        mu_t = torch.as_tensor(mu, dtype=torch.float32, device=dev).reshape(-1, model.n_species)
        mu_t = mu_t.expand(B, model.n_species).contiguous()
    x = x.contiguous()
    nat = torch.full((B,), N, dtype=torch.int32, device=dev)
    e64 = torch.empty(B, dtype=torch.float64, device=dev)
    f = torch.empty((B, N, 3), dtype=torch.float32, device=dev) if forces else None
    P = _lib.JrParams()
    P.model = model.model_params()
    L = _lib.load()
    stream = torch.cuda.current_stream(dev).cuda_stream
    rc = L.jr_energy_forces(
        C.byref(P), B, N, x.data_ptr(), t.data_ptr(), c.data_ptr(), nat.data_ptr(),
        pr.data_ptr(), mu_t.data_ptr() if mu_t is not None else None, e64.data_ptr(), None,
        f.data_ptr() if f is not None else None, stream)
    _lib.check(rc, "jr_energy_forces")
    if single:
        return BackendResult(energy=e64[0], forces=f[0] if f is not None else None)
    return BackendResult(energy=e64, forces=f)
