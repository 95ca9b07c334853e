"""Nested-sampling driver: the host side of the B200 walk.

Mirrors the reference's operator interface for the hot path
(``sampling/nested_sampling.py``): ``init_ns`` / ``init_ns_parallel`` build the
state, ``ns_step`` runs one iteration (cull, clone, walk, evidence) and
returns ``(ns_state, info)`` with the reference's info keys, and ``run_ns`` /
``run_ns_parallel`` drive the Python outer loop (termination, replica
exchange, callbacks).  The iteration itself is one ``jr_ns_iterate`` launch;
``ns_iterate`` runs many iterations per launch.

State is device resident (torch tensors on the current CUDA device) and is
advanced in place: ``ns_step`` returns the same ``NSState`` object with its
buffers updated, like a JAX call with donated arguments.
"""

from __future__ import annotations

import ctypes as C
import dataclasses
import math
from typing import Any

import numpy as np

from . import _lib, prior_mass, prng
from ._device import device
from .mwg import MWGStep


@dataclasses.dataclass
class MCState:
    """Walker population, leading axes ``(P, K)`` (``state/mc_state.py:48-102``)."""

    positions: Any      # (P,K,Nmax,3) float32
    direction: Any      # (P,K,Nmax,3) float32
    types: Any          # (P,K,Nmax) int32
    energy: Any         # (P,K) float32 view of energy64
    energy64: Any       # (P,K) float64 full ensemble potential
    cell: Any           # (P,K,3,3) float32
    step_sizes: Any     # (P,K,M) float32
    n_accepted: Any     # (P,K,M) int32
    n_proposed: Any     # (P,K,M) int32
    ensemble_params: dict
    n_atoms: Any        # (P,) int32

    def set(self, **kw) -> MCState:
        return dataclasses.replace(self, **kw)


@dataclasses.dataclass
class NSState:
    """NS state of P runs (``state/ns.py:29-83``) plus the launch workspace."""

    population: MCState
    log_evidence: Any   # (P,) float64
    iteration: Any      # (P,) int32
    emax: Any           # (P,) float64
    rng_key: Any        # (P,2) uint32 words stored as int32
    n_walkers: int = 0
    n_atoms: int = 0
    batched: bool = False
    workspace: Any = None

    def set(self, **kw) -> NSState:
        return dataclasses.replace(self, **kw)

    def clone(self) -> NSState:
        """An independent copy: every device buffer copied."""
        import torch

        def c(v):
            return v.clone() if isinstance(v, torch.Tensor) else v

        pop = dataclasses.replace(self.population, **{
            f.name: c(getattr(self.population, f.name))
            for f in dataclasses.fields(self.population)})
        return dataclasses.replace(self, population=pop, log_evidence=c(self.log_evidence),
                                   iteration=c(self.iteration), emax=c(self.emax),
                                   rng_key=c(self.rng_key), workspace=c(self.workspace))

    @property
    def n_runs(self) -> int:
        return int(self.log_evidence.shape[0])


def _ptr(t):
    return None if t is None else t.data_ptr()


def state_buffers(ns: NSState) -> _lib.JrStateBuffers:
    pop = ns.population
    b = _lib.JrStateBuffers()
    b.positions = _ptr(pop.positions)
    b.direction = _ptr(pop.direction)
    b.types = _ptr(pop.types)
    b.energy = _ptr(pop.energy)
    b.energy64 = _ptr(pop.energy64)
    b.cell = _ptr(pop.cell)
    b.step_sizes = _ptr(pop.step_sizes)
    b.n_accepted = _ptr(pop.n_accepted)
    b.n_proposed = _ptr(pop.n_proposed)
    b.rng_key = _ptr(ns.rng_key)
    b.log_evidence = _ptr(ns.log_evidence)
    b.iteration = _ptr(ns.iteration)
    b.emax = _ptr(ns.emax)
    b.n_atoms = _ptr(pop.n_atoms)
    b.pressure = _ptr(pop.ensemble_params["pressure"])
    mu = pop.ensemble_params.get("chemical_potentials")
    b.mu = _ptr(mu)
    return b


def make_dims(ns: NSState, step: MWGStep, n_mcmc_steps: int, n_extra: int,
              n_cull: int = 1) -> _lib.JrDims:
    d = _lib.JrDims()
    P, K, Nmax = ns.population.types.shape
    d.n_replicas, d.n_walkers, d.n_atoms_max = P, K, Nmax
    d.n_moves = step.n_moves
    d.n_mcmc_steps = int(n_mcmc_steps)
    d.n_extra = int(n_extra)
    d.n_cull = int(n_cull)
    d.shared_move_key = 1 if ns.batched else 0
    return d


def _stream():
    import torch

    return torch.cuda.current_stream(device()).cuda_stream


# ---------------------------------------------------------------- init ----

def _build_state(step: MWGStep, positions, types, energies, cells, rng_keys,
                 step_sizes, pressure, chemical_potentials, batched: bool) -> NSState:
    import torch

    dev = device()
    pos_list = [np.asarray(p, np.float32) for p in positions]
    P = len(pos_list)
    K = pos_list[0].shape[0]
    n_atoms = np.array([p.shape[1] for p in pos_list], np.int32)
    Nmax = int(n_atoms.max())
    if Nmax > _lib.MAX_ATOMS:
        raise ValueError(f"at most {_lib.MAX_ATOMS} atoms per walker")
    if any(p.shape[0] != K for p in pos_list):
        raise ValueError("every run needs the same number of walkers")
    M = step.n_moves
    X = np.zeros((P, K, Nmax, 3), np.float32)
    Tt = np.zeros((P, K, Nmax), np.int32)
    Cc = np.zeros((P, K, 3, 3), np.float32)
    for r in range(P):
        n = n_atoms[r]
        X[r, :, :n] = pos_list[r]
        t = np.asarray(types[r], np.int32)
        Tt[r, :, :n] = np.broadcast_to(t, (K, n))
        if cells is not None:
            Cc[r] = np.asarray(cells[r], np.float32).reshape(K, 3, 3)
    ss0 = step.default_step_sizes if step_sizes is None else step_sizes
    ss = np.broadcast_to(np.asarray(ss0, np.float32).reshape(-1, M), (P, M)).copy()
    S = step.backend.n_species
    pr = np.broadcast_to(np.asarray(pressure, np.float32).reshape(-1), (P,)).copy()
    mu = None
    if chemical_potentials is not None:
        mu = np.broadcast_to(np.asarray(chemical_potentials, np.float32).reshape(-1, S), (P, S)).copy()
    t32 = lambda a, dt: torch.as_tensor(np.ascontiguousarray(a), device=dev).to(dt)
    pop = MCState(
        positions=t32(X, torch.float32),
        direction=torch.zeros((P, K, Nmax, 3), dtype=torch.float32, device=dev),
        types=t32(Tt, torch.int32),
        energy=torch.zeros((P, K), dtype=torch.float32, device=dev),
        energy64=torch.zeros((P, K), dtype=torch.float64, device=dev),
        cell=t32(Cc, torch.float32),
        step_sizes=t32(np.repeat(ss[:, None, :], K, axis=1), torch.float32),
        n_accepted=torch.zeros((P, K, M), dtype=torch.int32, device=dev),
        n_proposed=torch.zeros((P, K, M), dtype=torch.int32, device=dev),
        ensemble_params={"pressure": t32(pr, torch.float32),
                         "chemical_potentials": None if mu is None else t32(mu, torch.float32)},
        n_atoms=t32(n_atoms, torch.int32),
    )
    keys = np.asarray(rng_keys, np.uint32).reshape(P, 2)
    ns = NSState(
        population=pop,
        log_evidence=torch.full((P,), -math.inf, dtype=torch.float64, device=dev),
        iteration=torch.zeros((P,), dtype=torch.int32, device=dev),
        emax=torch.full((P,), math.inf, dtype=torch.float64, device=dev),
        rng_key=torch.as_tensor(keys.view(np.int32).copy(), device=dev),
        n_walkers=K, n_atoms=Nmax, batched=batched,
    )
    d = make_dims(ns, step, 1, 0)
    ns.workspace = torch.zeros(int(_lib.load().jr_ns_iterate_workspace_size(C.byref(d))),
                               dtype=torch.uint8, device=dev)
    if energies is None:
        set_energies_from_backend(ns, step)
    else:
        e = np.zeros((P, K), np.float64)
        for r in range(P):
            e[r] = np.asarray(energies[r], np.float64)
        pop.energy64.copy_(torch.as_tensor(e, device=dev))
        pop.energy.copy_(pop.energy64.to(torch.float32))
    return ns


def set_energies_from_backend(ns: NSState, step: MWGStep) -> None:
    """Evaluate every walker's full potential on the GPU (float64)."""
    import torch

    pop = ns.population
    P, K, Nmax = pop.types.shape
    B = P * K
    params = _lib.JrParams()
    params.model = step.backend.model_params()
    nat = pop.n_atoms.repeat_interleave(K).contiguous()
    pr = pop.ensemble_params["pressure"].repeat_interleave(K).contiguous()
    mu = pop.ensemble_params.get("chemical_potentials")
    mu_b = None if mu is None else mu.repeat_interleave(K, dim=0).contiguous()
    e64 = torch.empty(B, dtype=torch.float64, device=pop.positions.device)
    rc = _lib.load().jr_energy_forces(
        C.byref(params), B, Nmax, pop.positions.data_ptr(), pop.types.data_ptr(),
        pop.cell.data_ptr(), nat.data_ptr(), pr.data_ptr(), _ptr(mu_b), e64.data_ptr(),
        None, None, _stream())
    _lib.check(rc, "jr_energy_forces")
    pop.energy64.copy_(e64.view(P, K))
    pop.energy.copy_(pop.energy64.to(torch.float32))


def _ens(ensemble_params, P):
    ep = ensemble_params or {}
    return ep.get("pressure", 0.0), ep.get("chemical_potentials")


def init_ns(init_fn, positions, types, energies, cells, rng_key, step_sizes=None,
            ensemble_params=None, restart_state=None, max_neighbors: int = 0,
            max_neighbor_counts=None) -> NSState:
    """One run (``nested_sampling.py:260-383``).  ``energies=None`` evaluates
    the Hamiltonian (model + EnsembleTerm) on the GPU."""
    step = init_fn.step
    pressure, mu = _ens(ensemble_params, 1)
    if ensemble_params is None and step.backend.ensemble is not None:
        pressure, mu = step.backend.ensemble.resolve(None)
    ns = _build_state(step, [positions], [types], None if energies is None else [energies],
                      None if cells is None else [cells], [np.asarray(rng_key, np.uint32)],
                      step_sizes, pressure, mu, batched=False)
    if restart_state is not None:
        _apply_restart(ns, restart_state)
    return ns


def init_ns_parallel(init_fn, positions, types, energies, cells, rng_keys,
                     step_sizes=None, ensemble_params=None) -> NSState:
    """R runs batched like ``VmapRuns`` (one shared move schedule).
    ``positions`` may be a list of ``(K, N_r, 3)`` arrays with uneven N_r."""
    step = init_fn.step
    R = len(positions)
    pressure, mu = _ens(ensemble_params, R)
    if ensemble_params is None and step.backend.ensemble is not None:
        pressure, mu = step.backend.ensemble.resolve(None)
    return _build_state(step, list(positions), list(types),
                        None if energies is None else list(energies),
                        None if cells is None else list(cells), rng_keys, step_sizes,
                        pressure, mu, batched=True)


def _apply_restart(ns: NSState, rs) -> None:
    import torch

    ns.log_evidence.fill_(float(rs.log_evidence))
    ns.iteration.fill_(int(rs.iteration))
    ns.emax.fill_(float(rs.emax))
    if getattr(rs, "rng_key_data", None) is not None:
        k = np.asarray(rs.rng_key_data, np.uint32).reshape(-1, 2)
        ns.rng_key.copy_(torch.as_tensor(k.view(np.int32), device=ns.rng_key.device))


# ----------------------------------------------------------- iterations ----

class InfoBuffers:
    """Device buffers for ``n_iter`` iterations of per-iteration outputs."""

    def __init__(self, ns: NSState, M: int, n_iter: int, dead: bool = True, n_cull: int = 1):
        import torch

        dev = ns.population.positions.device
        P, K, Nmax = ns.population.types.shape
        z = lambda shape, dt: torch.zeros(shape, dtype=dt, device=dev)
        c = () if n_cull == 1 else (n_cull,)   # per-cull axis after P when n_cull > 1
        self.n_iter = n_iter
        self.n_cull = n_cull
        self.worst_idx = z((n_iter, P) + c, torch.int32)
        self.clone_idx = z((n_iter, P) + c, torch.int32)
        self.dead_energy = z((n_iter, P) + c, torch.float64)
        self.emax = z((n_iter, P), torch.float64)
        self.log_evidence = z((n_iter, P), torch.float64)
        self.dead_positions = z((n_iter, P) + c + (Nmax, 3), torch.float32) if dead else None
        self.dead_types = z((n_iter, P) + c + (Nmax,), torch.int32) if dead else None
        self.dead_cell = z((n_iter, P) + c + (3, 3), torch.float32) if dead else None
        self.n_accepted = z((n_iter, P, M), torch.int32)
        self.n_proposed = z((n_iter, P, M), torch.int32)
        self.reject_reason_counts = z((n_iter, P, M, 4), torch.int32)
        self.n_evaluations = z((n_iter, P, M), torch.int32)
        self.n_grad_evaluations = z((n_iter, P, M), torch.int32)
        self.rounds = z((P,), torch.int32)
        # Stillinger-Weber work per iteration: pairs and triplets inside the
        # cutoff over the energy+force evaluations, then the energy-only ones
        self.term_counts = z((n_iter, P, 4), torch.int64)

    def cstruct(self) -> _lib.JrInfoBuffers:
        b = _lib.JrInfoBuffers()
        for f, _ in _lib.JrInfoBuffers._fields_:
            setattr(b, f, _ptr(getattr(self, f)))
        return b


def ns_iterate(ns_state: NSState, step_fn: MWGStep, n_iter: int, n_mcmc_steps: int = 20,
               n_extra: int = 0, n_cull: int = 1, info: InfoBuffers | None = None,
               cfg: _lib.JrLaunchConfig | None = None, move_key=None) -> InfoBuffers:
    """Run ``n_iter`` NS iterations on every run in one launch.  ``move_key``
    (one iteration only): the key of the move schedule, ``split(move_key,
    n_mcmc_steps)``, shared by every run, as the reference's ``ns_step``
    takes it; by default the schedule comes from the run keys."""
    K = ns_state.n_walkers
    la = prior_mass.log_alpha(K, n_cull)
    _, w_off = prior_mass.iteration_offsets(K, n_cull)
    params = step_fn.with_evidence(la, w_off)
    dims = make_dims(ns_state, step_fn, n_mcmc_steps, n_extra, n_cull)
    if info is None:
        info = InfoBuffers(ns_state, step_fn.n_moves, n_iter, n_cull=n_cull)
    if info.n_cull != n_cull:
        raise ValueError("info buffers were sized for a different n_cull")
    sb = state_buffers(ns_state)
    mk_dev = None
    if move_key is not None:
        import torch

        if n_iter != 1:
            raise ValueError("an explicit move_key drives exactly one iteration")
        words = np.asarray(move_key, np.uint32).reshape(2)
        mk_dev = torch.as_tensor(words.view(np.int32).copy(), device=ns_state.rng_key.device)
        dims.shared_move_key = 2
        sb.move_key = mk_dev.data_ptr()
    ib = info.cstruct()
    rc = _lib.load().jr_ns_iterate(
        C.byref(dims), C.byref(params), C.byref(sb), C.byref(ib), int(n_iter),
        C.byref(cfg) if cfg is not None else None, ns_state.workspace.data_ptr(),
        ns_state.workspace.numel(), _stream())
    _lib.check(rc, "jr_ns_iterate")
    return info


def info_dict(info: InfoBuffers, ns_state: NSState, n_mcmc_steps: int, n_extra: int,
              row: int = 0) -> dict:
    """The reference's ``info`` dict (``nested_sampling.py:653-685``) for one
    iteration, leading run axis ``(P, ...)``; device tensors.  The
    single-walker views (``worst_idx``, ``dead_walker``) are the contour cull,
    the last of the ``(n_cull,)``-wide ones."""
    import torch

    emax64 = info.emax[row]
    multi = info.n_cull > 1

    def wide(t):   # (P, n_cull, ...) view
        return None if t is None else (t[row] if multi else t[row][:, None])

    dws = {
        "positions": wide(info.dead_positions),
        "types": wide(info.dead_types),
        "energy": wide(info.dead_energy).to(torch.float32),
        "cell": wide(info.dead_cell),
    }
    dw = {k: (None if v is None else v[:, -1]) for k, v in dws.items()}
    n_acc = info.n_accepted[row]
    total = n_mcmc_steps * (info.n_cull + n_extra)
    worst = wide(info.worst_idx)
    clone = wide(info.clone_idx)
    d = {
        "emax": emax64.to(torch.float32),
        "emax64": emax64,
        "hmax": emax64.to(torch.float32),
        "worst_idx": worst[:, -1],
        "clone_idx": clone[:, -1],
        "worst_indices": worst,
        "clone_indices": clone,
        "acceptance_rate": n_acc.sum(-1).to(torch.float32) / float(total),
        "dead_walker": dw,
        "dead_walkers": dws,
        "n_accepted_per_move": n_acc,
        "n_proposed_per_move": info.n_proposed[row],
        "reject_reason_counts_per_move": info.reject_reason_counts[row],
        "n_evaluations_per_move": info.n_evaluations[row],
        "n_grad_evaluations_per_move": info.n_grad_evaluations[row],
        "log_evidence": info.log_evidence[row],
    }
    return d


def ns_step(ns_state: NSState, step_fn: MWGStep, n_mcmc_steps: int = 20, n_extra: int = 0,
            n_cull: int = 1, move_key=None):
    """One NS iteration (``nested_sampling.py:391-686``); returns
    ``(ns_state, info)``.  The run key and (for batched runs) the shared move
    schedule are derived on the device exactly as the reference does; a
    caller's ``move_key`` (the reference batcher's ``_shared_move_key``,
    ``batch_descriptor.py:177-195``) replaces the schedule key for every run."""
    info = ns_iterate(ns_state, step_fn, 1, n_mcmc_steps, n_extra, n_cull, move_key=move_key)
    return ns_state, info_dict(info, ns_state, n_mcmc_steps, n_extra, 0)


def final_log_evidence(ns_state: NSState, n_cull: int = 1):
    """Live-walker share of the remaining prior mass added to log Z
    (``nested_sampling.py:229-252``), float64, per run."""
    import torch

    K = ns_state.n_walkers
    la = prior_mass.log_alpha(K, n_cull)
    log_x = ns_state.iteration.to(torch.float64) * la + (math.log(K) - math.log(K + 1.0))
    log_live = log_x - math.log(K) + torch.logsumexp(-ns_state.population.energy64, dim=-1)
    return torch.logaddexp(ns_state.log_evidence, log_live)


# -------------------------------------------------------------- trials ----

class TrialMove:
    """``per_move_fns[k]``: move ``k`` applied to chosen walkers
    (``mwg.py:152-154``), e.g. the step-size trials of
    ``adaptation/stepsize_handler.py:246-255``."""

    def __init__(self, step: MWGStep, move_idx: int):
        self.step = step
        self.move_idx = move_idx

    def __call__(self, ns_state: NSState, walker_idx, keys, step_size, emax,
                 write_back: bool = False, move_keys=None):
        import torch

        dev = ns_state.population.positions.device
        widx = torch.as_tensor(walker_idx, dtype=torch.int32, device=dev).contiguous()
        P, n = widx.shape
        k = np.asarray(keys, np.uint32).reshape(P, n, 2).view(np.int32)
        kt = torch.as_tensor(k.copy(), device=dev)
        mkt = None
        if move_keys is not None:
            mk = np.asarray(move_keys, np.uint32).reshape(P, n, 2).view(np.int32)
            mkt = torch.as_tensor(mk.copy(), device=dev)
        st = torch.as_tensor(step_size, dtype=torch.float32, device=dev).reshape(-1).expand(P).contiguous()
        em = torch.as_tensor(emax, dtype=torch.float64, device=dev).reshape(-1).expand(P).contiguous()
        acc = torch.zeros((P, n), dtype=torch.int32, device=dev)
        reason = torch.zeros((P, n), dtype=torch.int32, device=dev)
        dims = make_dims(ns_state, self.step, 1, 0)
        sb = state_buffers(ns_state)
        rc = _lib.load().jr_move_trial(
            C.byref(dims), C.byref(self.step.params), C.byref(sb), n, self.move_idx,
            widx.data_ptr(), kt.data_ptr(), _ptr(mkt), st.data_ptr(), em.data_ptr(),
            int(write_back), acc.data_ptr(), reason.data_ptr(), _stream())
        _lib.check(rc, "jr_move_trial")
        return acc, reason


# ------------------------------------------------------------ outer loop ----

class IterationTermination:
    """Stop after a fixed number of iterations (``termination.py:55-65``)."""

    def __init__(self, max_iterations: int):
        self.max_iterations = max_iterations

    def check(self, iteration: int, emax: float) -> bool:
        return iteration >= self.max_iterations - 1

    def message(self) -> str:
        return f"Reached max iterations ({self.max_iterations})"


class PriorMassTermination:
    """Skilling-style remaining-mass test (``termination.py:68-112``)."""

    def __init__(self, n_live: int, threshold: float = 1e-3, n_cull: int = 1):
        self.n_live, self.n_cull, self.threshold = n_live, n_cull, threshold
        self._log_threshold = math.log(threshold)
        self._log_alpha = prior_mass.log_alpha(n_live, n_cull)
        self._log_evidence = -math.inf

    def update_evidence(self, log_evidence: float) -> None:
        self._log_evidence = log_evidence

    def check(self, iteration: int, emax: float) -> bool:
        if iteration * self.n_cull <= self.n_live:
            return False
        log_x = (iteration + 1) * self._log_alpha
        return log_x - float(emax) < float(self._log_evidence) + self._log_threshold

    def message(self) -> str:
        return "Prior mass negligible compared to evidence"


def check_any(criteria, iteration: int, emax: float):
    for c in criteria:
        if c.check(iteration, emax):
            return True, c.message()
    return False, ""


class InterREManager:
    """Pressure / semi-grand replica exchange every ``re_interval`` iterations
    (``sampling/inter_re_manager.py:191-273``), swaps on the GPU."""

    def __init__(self, re_interval: int, n_swap_cycles: int, rng_key):
        self.re_interval = int(re_interval)
        self.n_swap_cycles = int(n_swap_cycles)
        # run_loop.py:437-438: one scalar key derived before the loop
        self.key = prng.split(np.asarray(rng_key, np.uint32), 1)[0]

    def fires(self, iteration: int) -> bool:
        return self.re_interval > 0 and iteration > 0 and iteration % self.re_interval == 0

    def next_swap_key(self) -> np.ndarray:
        # run_loop.py:545: inter_re_key, key_re = split(inter_re_key);
        # inter_re_manager.py:251: rng_key, swap_key = split(key_re)
        ks = prng.split(self.key, 2)
        self.key, key_re = ks[0], ks[1]
        return prng.split(key_re, 2)[1]

    def apply(self, ns_state: NSState, step_fn: MWGStep):
        import torch

        R = ns_state.n_runs
        swap_key = self.next_swap_key()
        dims = make_dims(ns_state, step_fn, 1, 0)
        acc = torch.zeros(max(R - 1, 1), dtype=torch.int32, device=ns_state.emax.device)
        att = torch.zeros_like(acc)
        sb = state_buffers(ns_state)
        rc = _lib.load().jr_re_swap(C.byref(dims), C.byref(sb), int(swap_key[0]),
                                    int(swap_key[1]), self.n_swap_cycles,
                                    step_fn.backend.n_species, acc.data_ptr(),
                                    att.data_ptr(), _stream())
        _lib.check(rc, "jr_re_swap")
        return {"n_accepted_per_pair": acc, "n_attempted_per_pair": att}


def run_loop(ns_state: NSState, step_fn: MWGStep, n_mcmc_steps: int, n_extra: int,
             termination_criteria: list, callbacks: list | None = None,
             inter_re: InterREManager | None = None, n_cull: int = 1,
             check_interval: int = 1) -> NSState:
    """The Python outer loop (``sampling/run_loop.py:323-627``) without
    adaptation.  ``check_interval`` iterations run per launch; termination is
    evaluated for every one of them from the per-iteration info, so with the
    default 1 the loop stops exactly where the reference's would."""
    callbacks = callbacks or []
    i = 0
    while True:
        chunk = max(1, int(check_interval))
        if inter_re is not None and inter_re.re_interval > 0:
            # end the launch on the next iteration after which a swap fires
            re = inter_re.re_interval
            nxt = max(re, ((i + re - 1) // re) * re)
            chunk = min(chunk, nxt - i + 1)
        info = ns_iterate(ns_state, step_fn, chunk, n_mcmc_steps, n_extra, n_cull)
        lz = info.log_evidence.cpu().numpy()
        em = info.emax.cpu().numpy()
        stop = False
        n_keep = chunk
        for r in range(chunk):
            it = i + r
            if inter_re is not None and r == chunk - 1 and inter_re.fires(it):
                stats = inter_re.apply(ns_state, step_fn)
            else:
                stats = None
            d = info_dict(info, ns_state, n_mcmc_steps, n_extra, r)
            if stats is not None:
                d["inter_re_stats"] = stats
            for cb in callbacks:
                if hasattr(cb, "on_iteration"):
                    cb.on_iteration(it, ns_state, d)
            log_z = float(np.min(lz[r]))
            hmax = float(np.max(em[r]))
            for c in termination_criteria:
                if isinstance(c, PriorMassTermination):
                    c.update_evidence(log_z)
            stop, _ = check_any(termination_criteria, it, hmax)
            if stop:
                n_keep = r + 1
                break
        for cb in callbacks:
            if hasattr(cb, "on_launch"):
                cb.on_launch(i, info, n_keep)
        i += chunk
        if stop:
            return ns_state


def run_ns(positions, types, energies, cells, init_fn, step_fn, rng_key,
           max_iterations: int = 1000, n_mcmc_steps: int = 20, n_extra: int = 0,
           convergence_threshold: float | None = None, callbacks=None,
           ensemble_params=None, step_sizes=None, check_interval: int = 1,
           n_cull: int = 1):
    """Single run to termination (``nested_sampling.py:1065-1226``)."""
    ns = init_ns(init_fn, positions, types, energies, cells, rng_key,
                 step_sizes=step_sizes, ensemble_params=ensemble_params)
    crit = [IterationTermination(max_iterations)]
    if convergence_threshold is not None:
        crit.append(PriorMassTermination(ns.n_walkers, convergence_threshold, n_cull))
    run_loop(ns, step_fn, n_mcmc_steps, n_extra, crit, callbacks, n_cull=n_cull,
             check_interval=check_interval)
    return {"ns_state": ns, "log_evidence": final_log_evidence(ns, n_cull),
            "n_iterations": ns.iteration}


def run_ns_parallel(positions, types, energies, cells, init_fn, step_fn, rng_keys,
                    max_iterations: int = 1000, n_mcmc_steps: int = 20, n_extra: int = 0,
                    convergence_threshold: float | None = None, callbacks=None,
                    ensemble_params=None, re_interval: int = 0, n_swap_cycles: int = 1,
                    re_key=None, step_sizes=None, check_interval: int = 1,
                    n_cull: int = 1):
    """R runs batched (``nested_sampling.py:1341-1560``), with optional
    replica exchange every ``re_interval`` iterations."""
    ns = init_ns_parallel(init_fn, positions, types, energies, cells, rng_keys,
                          step_sizes=step_sizes, ensemble_params=ensemble_params)
    crit = [IterationTermination(max_iterations)]
    if convergence_threshold is not None:
        crit.append(PriorMassTermination(ns.n_walkers, convergence_threshold, n_cull))
    re = None
    if re_interval > 0 and ns.n_runs > 1:
        re = InterREManager(re_interval, n_swap_cycles,
                            re_key if re_key is not None else prng.key(0))
    run_loop(ns, step_fn, n_mcmc_steps, n_extra, crit, callbacks, inter_re=re,
             n_cull=n_cull, check_interval=check_interval)
    return {"ns_state": ns, "log_evidence": final_log_evidence(ns, n_cull),
            "n_iterations": ns.iteration}
