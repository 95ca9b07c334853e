"""CPU reference of the learned surrogate energy (TEST INFRASTRUCTURE ONLY).

The checker of the surrogate kernels: only tests/ and bench.py's CPU legs
use it.  The surrogate has no counterpart in the reference (jaxrens has no
learned potentials on its walk), so nothing external pins it; it is pinned
by this restatement, float64 finite differences and the gradients of its own
loss.

Model, for a configuration of n atoms in a periodic cell (single minimum
image, as the Stillinger-Weber walk):

* descriptor of atom i: ``D[i, k] = sum_j exp(-eta (r_ij - mu_k)^2) fc(r_ij)``
  over the other atoms within ``rc``, ``fc(r) = (cos(pi r / rc) + 1) / 2``,
  16 centres ``mu_k`` evenly spaced on [1.5, 3.8] A, ``eta = 1 / (2 dmu^2)``;
* input ``x = D * in_scale + in_shift`` (per feature);
* MLP ``h1 = silu(x W1 + b1)``, ``h2 = silu(h1 W2 + b2)``, ``e = h2 w3 + b3``
  with 16 -> 64 -> 64 -> 1 and ``silu(z) = z sigmoid(z)``;
* energy ``U = sum_i (e_i out_scale + out_shift)``.

The kernels run the matrix products in bfloat16 with float32 accumulation;
``bf=True`` rounds every matrix operand (inputs, weights, activations,
back-propagated gradients) to bfloat16 the same way, so kernel results agree
with it to float32 summation-order rounding.  ``bf=False`` evaluates
everything in float64 (the finite-difference yardstick).
"""

from __future__ import annotations

import numpy as np

N_BASIS = 16
HIDDEN = 64
RC = 3.8
MU = np.linspace(1.5, 3.8, N_BASIS)
ETA = 1.0 / (2.0 * (MU[1] - MU[0]) ** 2)


def bf16(a):
    """Round float32 values to bfloat16 (round to nearest even), as float32."""
    a = np.ascontiguousarray(a, np.float32)
    u = a.view(np.uint32).astype(np.uint64)
    rounded = ((u + 0x7FFF + ((u >> 16) & 1)) >> 16) << 16
    out = rounded.astype(np.uint32).view(np.float32)
    return np.where(np.isnan(a), a, out).astype(np.float32)


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def mic_pairs(x, cell):
    """Minimum-image displacements dr[i, j] = x_j - x_i and distances."""
    x = np.asarray(x, np.float64)
    c = np.asarray(cell, np.float64).reshape(3, 3)
    inv = np.linalg.inv(c)
    dr = x[None, :, :] - x[:, None, :]
    f = dr @ inv
    dr = dr - np.rint(f) @ c
    r = np.linalg.norm(dr, axis=-1)
    return dr, r


def descriptors(x, cell):
    """D [n][16] (float64), the displacements, distances and neighbour mask."""
    dr, r = mic_pairs(x, cell)
    n = len(x)
    inside = (r < RC) & ~np.eye(n, dtype=bool)
    fc = np.where(inside, 0.5 * (np.cos(np.pi * r / RC) + 1.0), 0.0)
    g = np.exp(-ETA * (r[..., None] - MU) ** 2)          # [n][n][16]
    phi = g * fc[..., None]
    D = phi.sum(axis=1)
    return D, dr, r, inside


def init_params(seed=0):
    """Random-init float32 parameters (He scale): W1 [16][64], b1 [64],
    W2 [64][64], b2 [64], w3 [64], b3, in/out normalisation."""
    rng = np.random.default_rng(seed)
    return {
        "W1": (rng.standard_normal((N_BASIS, HIDDEN)) / np.sqrt(N_BASIS)).astype(np.float32),
        "b1": np.zeros(HIDDEN, np.float32),
        "W2": (rng.standard_normal((HIDDEN, HIDDEN)) / np.sqrt(HIDDEN)).astype(np.float32),
        "b2": np.zeros(HIDDEN, np.float32),
        "w3": (rng.standard_normal(HIDDEN) / np.sqrt(HIDDEN)).astype(np.float32),
        "b3": np.float32(0.0),
        "in_scale": np.ones(N_BASIS, np.float32),
        "in_shift": np.zeros(N_BASIS, np.float32),
        "out_scale": np.float32(1.0),
        "out_shift": np.float32(0.0),
    }


def mlp_forward(D, p, bf=True):
    """Per-atom energies e and the intermediates of the backward pass."""
    dt = np.float32 if bf else np.float64
    r = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    x = r(np.asarray(D, dt) * p["in_scale"] + p["in_shift"])
    z1 = (x @ r(p["W1"])).astype(dt) + p["b1"]
    h1 = r(silu(z1))
    z2 = (h1 @ r(p["W2"])).astype(dt) + p["b2"]
    h2 = silu(z2).astype(dt)
    e = h2 @ p["w3"] + p["b3"]
    return e.astype(dt), dict(x=x, z1=z1, h1=h1, z2=z2, h2=h2)


def energy(x, cell, p, bf=True):
    D, *_ = descriptors(x, cell)
    e, _ = mlp_forward(D, p, bf)
    return float(np.sum(e.astype(np.float64) * p["out_scale"] + p["out_shift"]))


def energy_forces(x, cell, p, bf=True):
    """Surrogate energy U and forces -dU/dx (float64 descriptor geometry)."""
    r_ = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    D, dr, r, inside = descriptors(x, cell)
    e, it = mlp_forward(D, p, bf)
    U = float(np.sum(e.astype(np.float64) * p["out_scale"] + p["out_shift"]))
    # dU/de_i = out_scale
    g2 = r_(p["out_scale"] * p["w3"][None, :] * dsilu(it["z2"]))
    g1 = r_((g2 @ r_(p["W2"]).T) * dsilu(it["z1"]))
    gx = (g1 @ r_(p["W1"]).T).astype(np.float64)         # dU/dx [n][16]
    gD = gx * p["in_scale"]                               # dU/dD
    # dD_ik/dr_ij = g_k(r) [-2 eta (r - mu_k) fc + fc'(r)]
    fc = np.where(inside, 0.5 * (np.cos(np.pi * r / RC) + 1.0), 0.0)
    dfc = np.where(inside, -0.5 * np.pi / RC * np.sin(np.pi * r / RC), 0.0)
    g = np.exp(-ETA * (r[..., None] - MU) ** 2)
    dphi = g * (-2.0 * ETA * (r[..., None] - MU) * fc[..., None] + dfc[..., None])
    s = ((gD[:, None, :] + gD[None, :, :]) * dphi).sum(-1)   # [n][n]
    with np.errstate(invalid="ignore", divide="ignore"):
        coef = np.where(inside, s / r, 0.0)
    # F_i = sum_j coef_ij dr_ij
    F = (coef[..., None] * dr).sum(axis=1)
    return U, F


def loss_and_grads(Dbatch, U, p, n_atoms, bf=True):
    """Mean over configurations of ((sum_i e_i) out_scale + n out_shift - U)^2
    / n^2 and its gradients with respect to W1, b1, W2, b2, w3, b3 (the
    training kernel's loss).  Dbatch [B][n][16], U [B]."""
    r_ = bf16 if bf else (lambda a: np.asarray(a, np.float64))
    dt = np.float32 if bf else np.float64
    B, n, _ = Dbatch.shape
    e, it = mlp_forward(Dbatch.reshape(B * n, N_BASIS), p, bf)
    Epred = e.reshape(B, n).astype(np.float64).sum(1) * p["out_scale"] + n * p["out_shift"]
    err = (Epred - U) / n
    loss = float(np.mean(err ** 2))
    dE = (2.0 * err / n / B) * p["out_scale"]               # dL/d(sum_i e_i) per config
    de = np.repeat(dE, n).astype(dt)                         # dL/de_r
    h2, z2, h1, z1, x = it["h2"], it["z2"], it["h1"], it["z1"], it["x"]
    grads = {}
    grads["w3"] = (r_(h2).astype(np.float64).T @ r_(de)).astype(dt)
    grads["b3"] = dt(de.astype(np.float64).sum())
    g2 = r_(de[:, None] * p["w3"][None, :] * dsilu(z2))
    grads["W2"] = (h1.astype(np.float64).T @ g2).astype(dt)
    grads["b2"] = g2.astype(np.float64).sum(0).astype(dt)
    g1 = r_((g2 @ r_(p["W2"]).T) * dsilu(z1))
    grads["W1"] = (x.astype(np.float64).T @ g1).astype(dt)
    grads["b1"] = g1.astype(np.float64).sum(0).astype(dt)
    return loss, grads
