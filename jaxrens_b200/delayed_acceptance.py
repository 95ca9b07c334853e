"""Nested sampling with the delayed-acceptance walk on the learned surrogate.

``ns_iterate_da`` is ``ns_iterate`` for the Stillinger-Weber model with the
galilean and volume moves screened by the surrogate
(``jr_ns_iterate_da``): stage 1 accepts on the smoothed surrogate
constraint, stage 2 evaluates the exact potential, which decides every step.
The walk stores every exactly evaluated configuration in a ``SampleRing``;
``DelayedAcceptanceNS`` trains the surrogate on the ring's recent entries
every ``train_every`` iterations.

Before the surrogate has data the driver bootstraps it from the live
population (and the dead walkers of a few plain iterations, ``warmup_iters``),
evaluated exactly with ``jr_energy_forces``.

The reference has no learned potential on its walk; this module has no
counterpart there.  The per-iteration outputs are the reference's
(``ns_step``'s info, ``sampling/nested_sampling.py:653-685``), with
``n_evaluations`` counting exact evaluations and
``n_surrogate_evaluations`` the surrogate's.
"""

from __future__ import annotations

import ctypes as C
import math

import numpy as np

from . import _lib, prior_mass
from ._device import device
from .mwg import MWGStep
from .nested_sampling import (InfoBuffers, NSState, _stream, make_dims, ns_iterate,
                              state_buffers)
from .surrogate import Surrogate


def torch_det_abs(cell):
    """|det| of (..., 3, 3) cells in float64 (the triple product, elementwise)."""
    import torch

    c = cell.to(torch.float64)
    return (c[..., 0, :] * torch.linalg.cross(c[..., 1, :], c[..., 2, :])).sum(-1).abs()


class SampleRing:
    """Device ring of exactly evaluated configurations: positions
    ``(capacity, Nmax, 3)``, cells ``(capacity, 3, 3)`` and model energies
    ``energy_u`` (float64; NaN marks a slot without an evaluation).  Every
    MWG step of the walk owns one slot; ``base`` is the slot of the next
    launch's first step."""

    def __init__(self, capacity: int, n_atoms_max: int):
        import torch

        dev = device()
        self.capacity = int(capacity)
        self.n_atoms_max = int(n_atoms_max)
        self.positions = torch.zeros((self.capacity, n_atoms_max, 3), dtype=torch.float32,
                                     device=dev)
        self.cell = torch.zeros((self.capacity, 3, 3), dtype=torch.float32, device=dev)
        self.energy_u = torch.full((self.capacity,), math.nan, dtype=torch.float64, device=dev)
        self.base = 0
        self.reserved = 0  # slots handed out so far (all time)

    def cstruct(self, n_surrogate_evaluations=None) -> _lib.JrSampleRing:
        r = _lib.JrSampleRing()
        r.positions = self.positions.data_ptr()
        r.cell = self.cell.data_ptr()
        r.energy_u = self.energy_u.data_ptr()
        r.capacity = self.capacity
        r.base = self.base
        r.n_surrogate_evaluations = (None if n_surrogate_evaluations is None
                                     else n_surrogate_evaluations.data_ptr())
        return r

    def reserve(self, n: int) -> None:
        self.base = (self.base + int(n)) % self.capacity
        self.reserved += int(n)

    def push(self, positions, cells, energy_u) -> None:
        """Append configurations evaluated elsewhere (B, Nmax, 3), (B, 3, 3),
        (B,) at the ring's head."""
        import torch

        B = int(positions.shape[0])
        if B == 0:
            return
        if B > self.capacity:
            positions, cells, energy_u = positions[-self.capacity:], cells[-self.capacity:], \
                energy_u[-self.capacity:]
            B = self.capacity
        idx = (torch.arange(B, device=self.positions.device) + self.base) % self.capacity
        self.positions[idx] = positions.to(self.positions)
        self.cell[idx] = cells.reshape(B, 3, 3).to(self.cell)
        self.energy_u[idx] = energy_u.to(self.energy_u)
        self.reserve(B)

    def recent_valid(self, window: int):
        """Slots of the last ``window`` reserved steps holding an evaluation
        (device int64)."""
        import torch

        w = min(int(window), self.reserved, self.capacity)
        if w == 0:
            return torch.zeros(0, dtype=torch.int64, device=self.positions.device)
        idx = (torch.arange(self.base - w, self.base, device=self.positions.device)) % \
            self.capacity
        return idx[torch.isfinite(self.energy_u[idx])]


def ns_iterate_da(ns_state: NSState, step_fn: MWGStep, surrogate: Surrogate, n_iter: int,
                  n_mcmc_steps: int = 20, n_extra: int = 0, info: InfoBuffers | None = None,
                  ring: SampleRing | None = None, cfg: _lib.JrLaunchConfig | None = None,
                  move_key=None) -> InfoBuffers:
    """``n_iter`` NS iterations with the delayed-acceptance walk, in one
    launch.  ``info.n_surrogate_evaluations`` ``(n_iter, P, M)`` receives the
    surrogate evaluations per move; the walk's exact evaluations go to
    ``ring`` when given (its ``base`` advances by ``n_iter P (1 + n_extra)
    n_mcmc_steps``)."""
    import torch

    K = ns_state.n_walkers
    la = prior_mass.log_alpha(K, 1)
    _, w_off = prior_mass.iteration_offsets(K, 1)
    params = step_fn.with_evidence(la, w_off)
    dims = make_dims(ns_state, step_fn, n_mcmc_steps, n_extra, 1)
    if info is None:
        info = InfoBuffers(ns_state, step_fn.n_moves, n_iter)
    P = int(ns_state.population.types.shape[0])
    if getattr(info, "n_surrogate_evaluations", None) is None:
        info.n_surrogate_evaluations = torch.zeros((info.n_iter, P, step_fn.n_moves),
                                                   dtype=torch.int32, device=device())
    sb = state_buffers(ns_state)
    mk_dev = None
    if move_key is not None:
        if n_iter != 1:
            raise ValueError("an explicit move_key drives exactly one iteration")
        words = np.asarray(move_key, np.uint32).reshape(2)
        mk_dev = torch.as_tensor(words.view(np.int32).copy(), device=device())
        dims.shared_move_key = 2
        sb.move_key = mk_dev.data_ptr()
    ib = info.cstruct()
    if ring is not None:
        rs = ring.cstruct(info.n_surrogate_evaluations)
    else:
        rs = _lib.JrSampleRing()
        rs.n_surrogate_evaluations = info.n_surrogate_evaluations.data_ptr()
    sc = surrogate.cstruct()
    rc = _lib.load().jr_ns_iterate_da(
        C.byref(dims), C.byref(params), C.byref(sb), C.byref(ib), C.byref(sc), C.byref(rs),
        int(n_iter), C.byref(cfg) if cfg is not None else None, ns_state.workspace.data_ptr(),
        ns_state.workspace.numel(), _stream())
    _lib.check(rc, "jr_ns_iterate_da")
    if ring is not None:
        ring.reserve(n_iter * P * (1 + n_extra) * n_mcmc_steps)
    return info


def surrogate_energy_forces(surrogate: Surrogate, positions, cells, forces: bool = True):
    """The surrogate's U (float64, (B,)) and forces ((B, N, 3) or None) of
    configurations (B, N, 3) with cells (B, 3, 3), as the walk evaluates
    them (``jr_sur_energy_forces``)."""
    import torch

    dev = device()
    x = torch.as_tensor(positions, dtype=torch.float32, device=dev).contiguous()
    B, N, _ = x.shape
    c = torch.as_tensor(cells, dtype=torch.float32, device=dev).reshape(B, 9).contiguous()
    nat = torch.full((B,), N, dtype=torch.int32, device=dev)
    U = torch.empty(B, dtype=torch.float64, device=dev)
    F = torch.empty((B, N, 3), dtype=torch.float32, device=dev) if forces else None
    sc = surrogate.cstruct()
    rc = _lib.load().jr_sur_energy_forces(C.byref(sc), B, N, x.data_ptr(), c.data_ptr(),
                                          nat.data_ptr(), U.data_ptr(),
                                          F.data_ptr() if F is not None else None, _stream())
    _lib.check(rc, "jr_sur_energy_forces")
    return U, F


class DelayedAcceptanceNS:
    """Driver of the delayed-acceptance NS walk with online training.

    ``bootstrap()`` evaluates the live population (and the dead walkers of
    ``warmup_iters`` plain iterations) exactly, fills the ring, sets the
    surrogate's normalisation and trains ``bootstrap_steps`` Adam steps.
    ``run(n_iter)`` then walks blocks of ``block`` iterations with
    ``ns_iterate_da`` and, every ``train_every`` iterations, takes
    ``train_steps`` Adam steps on minibatches drawn from the ring's last
    ``train_window`` slots."""

    def __init__(self, ns_state: NSState, step_fn: MWGStep, surrogate: Surrogate | None = None,
                 n_mcmc_steps: int = 20, ring_capacity: int = 100_000, train_every: int = 50,
                 train_window: int = 100_000, train_steps: int = 16, batch: int = 256,
                 lr: float = 1e-3, warmup_iters: int = 0, bootstrap_steps: int = 200,
                 margin: float = 0.5, shift_sigmas: float = 0.0, seed: int = 0):
        import torch

        self.ns = ns_state
        self.step_fn = step_fn
        self.sur = surrogate if surrogate is not None else Surrogate(seed=seed)
        self.T = int(n_mcmc_steps)
        P, K, Nmax = ns_state.population.types.shape
        self.ring = SampleRing(ring_capacity, Nmax)
        self.train_every = int(train_every)
        self.train_window = int(train_window)
        self.train_steps = int(train_steps)
        self.batch = int(batch)
        self.lr = float(lr)
        self.warmup_iters = int(warmup_iters)
        self.margin = float(margin)
        self.shift_sigmas = float(shift_sigmas)
        self.bootstrap_steps = int(bootstrap_steps)
        self.gen = torch.Generator(device=device()).manual_seed(seed)
        self.since_train = 0
        self.iterations = 0

    def _exact_u(self, positions, cells):
        from .backends import _evaluate

        model = getattr(self.step_fn.backend, "model", self.step_fn.backend)
        B, N, _ = positions.shape
        return _evaluate(model, None, positions, np.zeros(N, np.int32), cells, False).energy

    def bootstrap(self, positions=None, cells=None) -> None:
        """Fill the ring with the live population, the configurations
        ``positions`` (B, N, 3) / ``cells`` (B, 3, 3) when given (e.g. the dead
        walkers of earlier iterations) and the dead walkers of
        ``warmup_iters`` plain iterations, all evaluated exactly; then set the
        normalisation, train and calibrate."""
        import torch

        pop = self.ns.population
        P, K, N = pop.types.shape
        xs = [pop.positions.reshape(P * K, N, 3).clone()]
        cs = [pop.cell.reshape(P * K, 3, 3).clone()]
        if positions is not None:
            xs.append(torch.as_tensor(positions, device=device()).reshape(-1, N, 3))
            cs.append(torch.as_tensor(cells, device=device()).reshape(-1, 3, 3))
        if self.warmup_iters > 0:
            info = ns_iterate(self.ns, self.step_fn, self.warmup_iters, self.T)
            xs.append(info.dead_positions.reshape(-1, N, 3))
            cs.append(info.dead_cell.reshape(-1, 3, 3))
            self.iterations += self.warmup_iters
        x = torch.cat(xs)
        c = torch.cat(cs)
        U = self._exact_u(x, c)
        self.ring.push(x, c, U)
        D = Surrogate.descriptors(x, c)
        self.sur.fit_normalisation(D, U, N)
        self.train(self.bootstrap_steps, renormalise=True)

    def _live_u_max(self):
        """The largest per-atom model energy of the live walkers (float)."""
        import torch

        pop = self.ns.population
        P, K, N = pop.types.shape
        vol = torch_det_abs(pop.cell)
        pr = pop.ensemble_params.get("pressure", 0.0)
        pr = torch.as_tensor(pr, dtype=torch.float64, device=vol.device).reshape(-1, 1)
        u = (pop.energy64 - pr * vol) / N
        return float(u.max())

    def training_set(self):
        """Ring slots to train and calibrate on: the last ``train_window``
        evaluated slots whose per-atom energy lies below the highest live
        walker's plus ``margin`` eV (the configurations near and inside the
        contour, where stage 1 decides)."""
        idx = self.ring.recent_valid(self.train_window)
        if idx.numel() == 0:
            return idx
        N = self.ring.n_atoms_max
        keep = self.ring.energy_u[idx] / N <= self._live_u_max() + self.margin
        return idx[keep]

    def calibrate(self, idx=None, n: int = 512) -> tuple[float, float]:
        """Set the surrogate constraint from its error d = U_sur - U on
        recent training configurations: with sigma = 1.4826 MAD(d),
        ``contour_shift`` = median(d) - shift_sigmas sigma (a surrogate
        contour moved inside the true one keeps trajectories inside it more
        often), ``tau`` = 0.6 sigma (a logistic of that scale follows the
        normal CDF of the error), at least 1e-3.  Either choice leaves the walk
        exact; they set how well stage 1 screens.  Returns (shift, tau)."""
        import torch

        idx = self.training_set() if idx is None else idx
        if idx.numel() == 0:
            return self.sur.contour_shift, self.sur.tau
        idx = idx[-n:]
        Us, _ = surrogate_energy_forces(self.sur, self.ring.positions[idx],
                                        self.ring.cell[idx], forces=False)
        d = Us - self.ring.energy_u[idx]
        med = d.median()
        sigma = 1.4826 * float((d - med).abs().median())
        self.sur.contour_shift = float(med) - self.shift_sigmas * sigma
        self.sur.tau = max(0.6 * sigma, 1e-3)
        return self.sur.contour_shift, self.sur.tau

    def train(self, steps: int, renormalise: bool = False) -> None:
        """``steps`` Adam steps on minibatches of the training set (after
        refitting the standardisation to it when ``renormalise``); then
        recalibrate."""
        import torch

        idx = self.training_set()
        if idx.numel() == 0 or steps <= 0:
            return
        N = self.ring.n_atoms_max
        if renormalise:
            sub = idx[-4096:]
            D = Surrogate.descriptors(self.ring.positions[sub], self.ring.cell[sub])
            self.sur.renormalise(D, self.ring.energy_u[sub], N)
        B = min(self.batch, int(idx.numel()))
        # every minibatch of the round drawn at once: one descriptor launch,
        # then one training launch per minibatch on its rows
        pick = idx[torch.randint(0, idx.numel(), (steps * B,), generator=self.gen,
                                 device=idx.device)]
        D = Surrogate.descriptors(self.ring.positions[pick], self.ring.cell[pick])
        Ub = self.ring.energy_u[pick].contiguous()
        rows = torch.arange(steps * B, dtype=torch.int32, device=idx.device).view(steps, B)
        for k in range(steps):
            self.sur.train_step(D, Ub, rows[k], self.lr)
        self.since_train = 0
        self.calibrate(idx)

    def run(self, n_iter: int, block: int = 10):
        """Walk ``n_iter`` iterations; returns the info buffers of the last
        block."""
        info = None
        done = 0
        while done < n_iter:
            b = min(block, n_iter - done)
            info = ns_iterate_da(self.ns, self.step_fn, self.sur, b, self.T, ring=self.ring)
            done += b
            self.iterations += b
            self.since_train += b
            if self.train_every > 0 and self.since_train >= self.train_every:
                self.train(self.train_steps)
        return info
