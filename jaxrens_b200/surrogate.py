"""The learned surrogate energy of the delayed-acceptance walk (host side).

A small network predicts the Stillinger-Weber model energy from radial
descriptors: per atom 16 Gaussians of the neighbour distances (centres
1.5..3.8 A, cosine cutoff 3.8 A), a 16-64-64-1 SiLU MLP, per-atom energies
summed.  It is trained online on configurations the walk itself evaluated
exactly, by the library's tensor-core training kernel (``jr_sur_train_step``:
bfloat16 products, float32 accumulation, Adam on float32 master weights),
and screens galilean and volume proposals in a two-stage delayed-acceptance
walk in which the exact potential decides every step.

The reference has no learned potential on its walk; this module has no
counterpart there.  The descriptor and network definitions are the ones the
CUDA kernels implement (``csrc/jr_sur.cuh``).
"""

from __future__ import annotations

import ctypes as C

import numpy as np

from . import _lib
from ._device import device

N_BASIS = _lib.SUR_BASIS
HIDDEN = _lib.SUR_HIDDEN
N_PARAMS = _lib.SUR_PARAMS
OFF_W1, OFF_B1 = 0, N_BASIS * HIDDEN
OFF_W2 = OFF_B1 + HIDDEN
OFF_B2 = OFF_W2 + HIDDEN * HIDDEN
OFF_W3 = OFF_B2 + HIDDEN
OFF_B3 = OFF_W3 + HIDDEN


def _stream():
    import torch

    return torch.cuda.current_stream(device()).cuda_stream


def flatten(p: dict) -> np.ndarray:
    """Parameters dict (W1 [16][64], b1, W2 [64][64], b2, w3, b3) -> the flat
    float32 layout of the kernels."""
    return np.concatenate([np.asarray(p["W1"], np.float32).reshape(-1),
                           np.asarray(p["b1"], np.float32),
                           np.asarray(p["W2"], np.float32).reshape(-1),
                           np.asarray(p["b2"], np.float32), np.asarray(p["w3"], np.float32),
                           np.atleast_1d(np.float32(p["b3"]))]).astype(np.float32)


def unflatten(v) -> dict:
    v = np.asarray(v, np.float32)
    return {"W1": v[OFF_W1:OFF_B1].reshape(N_BASIS, HIDDEN), "b1": v[OFF_B1:OFF_W2],
            "W2": v[OFF_W2:OFF_B2].reshape(HIDDEN, HIDDEN), "b2": v[OFF_B2:OFF_W3],
            "w3": v[OFF_W3:OFF_B3], "b3": np.float32(v[OFF_B3])}


def init_params(seed: int = 0) -> np.ndarray:
    """He-scaled random weights, zero biases (flat layout)."""
    rng = np.random.default_rng(seed)
    return flatten({
        "W1": rng.standard_normal((N_BASIS, HIDDEN)) / np.sqrt(N_BASIS),
        "b1": np.zeros(HIDDEN), "W2": rng.standard_normal((HIDDEN, HIDDEN)) / np.sqrt(HIDDEN),
        "b2": np.zeros(HIDDEN), "w3": rng.standard_normal(HIDDEN) / np.sqrt(HIDDEN), "b3": 0.0})


class Surrogate:
    """Parameters, Adam state and normalisation of the surrogate, on the GPU.

    ``contour_shift`` and ``tau`` set the smoothed surrogate constraint of
    the delayed-acceptance walk: ``s(x) = sigmoid((emax + contour_shift -
    H_sur(x)) / tau)`` with ``H_sur`` the surrogate energy plus the exact
    ensemble term."""

    def __init__(self, seed: int = 0, tau: float = 0.05, contour_shift: float = 0.0):
        import torch

        dev = device()
        self.params = torch.as_tensor(init_params(seed), device=dev)
        self.adam_m = torch.zeros(N_PARAMS, dtype=torch.float32, device=dev)
        self.adam_v = torch.zeros(N_PARAMS, dtype=torch.float32, device=dev)
        self.step = 0
        self.in_scale = np.ones(N_BASIS, np.float32)
        self.in_shift = np.zeros(N_BASIS, np.float32)
        self.out_scale = 1.0
        self.out_shift = 0.0
        self.tau = float(tau)
        self.contour_shift = float(contour_shift)
        self._ws = None
        self._loss = torch.zeros(1, dtype=torch.float32, device=dev)

    def cstruct(self) -> _lib.JrSurrogate:
        s = _lib.JrSurrogate()
        s.params = self.params.data_ptr()
        s.in_scale[:] = [float(v) for v in self.in_scale]
        s.in_shift[:] = [float(v) for v in self.in_shift]
        s.out_scale = float(self.out_scale)
        s.out_shift = float(self.out_shift)
        s.contour_shift = float(self.contour_shift)
        s.tau = float(self.tau)
        return s

    # ----------------------------------------------------------- data ----
    @staticmethod
    def descriptors(positions, cells):
        """D [B][N][16] float32 on the GPU of configurations (B, N, 3) with
        cells (B, 3, 3) (torch or numpy)."""
        import torch

        dev = device()
        x = torch.as_tensor(positions, dtype=torch.float32, device=dev).contiguous()
        B, N, _ = x.shape
        c = torch.as_tensor(cells, dtype=torch.float32, device=dev).reshape(B, 9).contiguous()
        D = torch.empty((B, N, N_BASIS), dtype=torch.float32, device=dev)
        rc = _lib.load().jr_sur_descriptors(B, N, x.data_ptr(), c.data_ptr(), D.data_ptr(),
                                            _stream())
        _lib.check(rc, "jr_sur_descriptors")
        return D

    def fit_normalisation(self, D, U, n_atoms: int) -> None:
        """Input standardisation from descriptors D (B, N, 16) and output
        scale and shift from the per-atom energies U / n (B,)."""
        import torch

        Df = D.reshape(-1, N_BASIS).double()
        mean, std = Df.mean(0), Df.std(0).clamp_min(1e-6)
        self.in_scale = (1.0 / std).float().cpu().numpy()
        self.in_shift = (-mean / std).float().cpu().numpy()
        u = torch.as_tensor(U, dtype=torch.float64).cpu() / n_atoms
        self.out_shift = float(u.mean())
        self.out_scale = float(max(float(u.std()), 1e-3))

    def renormalise(self, D, U, n_atoms: int) -> None:
        """Refit the input and output standardisation to (D, U) while keeping
        the function the network computes: W1 and b1 absorb the change of
        the input affine map, w3 and b3 the change of the output one.  The
        Adam moments restart."""
        import torch

        a, b = np.asarray(self.in_scale, np.float64), np.asarray(self.in_shift, np.float64)
        s, t = float(self.out_scale), float(self.out_shift)
        self.fit_normalisation(D, U, n_atoms)
        a2, b2 = np.asarray(self.in_scale, np.float64), np.asarray(self.in_shift, np.float64)
        s2, t2 = float(self.out_scale), float(self.out_shift)
        p = self.params.double()
        W1 = p[OFF_W1:OFF_B1].view(N_BASIS, HIDDEN)
        r = torch.as_tensor(a / a2, dtype=torch.float64, device=p.device)
        c = torch.as_tensor(b - b2 * (a / a2), dtype=torch.float64, device=p.device)
        b1 = p[OFF_B1:OFF_W2] + c @ W1
        W1 = W1 * r[:, None]
        w3 = p[OFF_W3:OFF_B3] * (s / s2)
        b3 = (p[OFF_B3] * s + t - t2) / s2
        self.params[OFF_W1:OFF_B1] = W1.reshape(-1).float()
        self.params[OFF_B1:OFF_W2] = b1.float()
        self.params[OFF_W3:OFF_B3] = w3.float()
        self.params[OFF_B3] = b3.float()
        self.adam_m.zero_()
        self.adam_v.zero_()
        self.step = 0

    # ------------------------------------------------------- training ----
    def train_step(self, D, U, batch_idx, lr: float = 1e-3) -> None:
        """One Adam step on the configurations batch_idx (int32, device) of
        (D, U); the batch loss lands in ``last_loss`` (device)."""
        import torch

        n_batch = int(batch_idx.numel())
        n_atoms = int(D.shape[1])
        L = _lib.load()
        need = int(L.jr_sur_train_workspace_size(n_batch, n_atoms))
        if self._ws is None or self._ws.numel() < need:
            self._ws = torch.zeros(need, dtype=torch.uint8, device=self.params.device)
        self.step += 1
        s = self.cstruct()
        rc = L.jr_sur_train_step(C.byref(s), D.data_ptr(), U.data_ptr(), batch_idx.data_ptr(),
                                 n_batch, n_atoms, self.params.data_ptr(), self.adam_m.data_ptr(),
                                 self.adam_v.data_ptr(), self.step, float(lr),
                                 self._loss.data_ptr(), self._ws.data_ptr(), self._ws.numel(),
                                 _stream())
        _lib.check(rc, "jr_sur_train_step")

    @property
    def last_loss(self):
        return self._loss

    def train_error(self) -> bool:
        """True if a bounded tensor-core wait of the last training step gave
        up (its update is then not valid)."""
        import torch

        return self._ws is not None and int(self._ws[:4].view(torch.int32).item()) != 0

    def fit(self, D, U, epochs: int = 2, batch: int = 1024, lr: float = 1e-3, seed: int = 0):
        """Epochs of shuffled minibatches over (D, U); returns the mean loss
        of the last epoch (a host float: one synchronisation)."""
        import torch

        n = int(D.shape[0])
        g = torch.Generator(device="cpu").manual_seed(seed)
        total = torch.zeros((), dtype=torch.float64, device=self.params.device)
        steps = 0
        for _ in range(epochs):
            perm = torch.randperm(n, generator=g).to(torch.int32).to(self.params.device)
            total.zero_()
            steps = 0
            for b0 in range(0, n, batch):
                idx = perm[b0:b0 + batch].contiguous()
                self.train_step(D, U, idx, lr)
                total += self._loss.double()[0]
                steps += 1
        return float(total.item()) / max(steps, 1)
