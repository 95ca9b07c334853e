"""The surrogate's CPU reference against finite differences (CPU only).

``oracle/surrogate_ref.py`` restates the surrogate energy (radial descriptors
+ 16-64-64-1 SiLU MLP) and its training loss; the GPU kernels are checked
against it.  Here it is pinned to calculus: forces are minus the gradient of
its energy, and its loss gradients are the derivatives of its loss, both by
central finite differences in float64 (the unrounded mode), plus the
descriptor's translation invariance and cutoff.
"""

import numpy as np
import pytest

from oracle import surrogate_ref as S


def _config(seed, n=20, side=8.0):
    rng = np.random.default_rng(seed)
    return rng.uniform(0, side, (n, 3)), np.eye(3) * side


def _params(seed=1):
    p = S.init_params(seed)
    rng = np.random.default_rng(seed + 100)
    p["b1"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b2"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["in_scale"] = np.full(16, 0.7, np.float32)
    p["in_shift"] = np.full(16, -0.2, np.float32)
    p["out_scale"] = np.float32(0.5)
    p["out_shift"] = np.float32(-1.0)
    return p


def _f64(p):
    return {k: np.asarray(v, np.float64) for k, v in p.items()}


def test_descriptors_translation_invariant_and_cut_off():
    x, c = _config(0)
    D1, *_ = S.descriptors(x, c)
    D2, *_ = S.descriptors(x + np.array([1.3, -0.4, 2.2]), c)
    np.testing.assert_allclose(D1, D2, atol=1e-12)
    # a lone atom pair beyond the cutoff contributes nothing
    D, *_ = S.descriptors(np.array([[0.0, 0.0, 0.0], [3.81, 0.0, 0.0]]), np.eye(3) * 20)
    assert np.abs(D).max() == 0.0


@pytest.mark.parametrize("seed", [0, 1])
def test_forces_are_minus_the_gradient(seed):
    x, c = _config(seed)
    p = _f64(_params())
    _, F = S.energy_forces(x, c, p, bf=False)
    h = 1e-5
    for i in range(0, len(x), 3):
        for q in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, q] += h
            xm[i, q] -= h
            fd = -(S.energy(xp, c, p, bf=False) - S.energy(xm, c, p, bf=False)) / (2 * h)
            assert abs(fd - F[i, q]) < 1e-5 * max(1.0, abs(F[i, q])), (i, q, fd, F[i, q])


def test_loss_gradients_match_finite_differences():
    rng = np.random.default_rng(5)
    B, n = 3, 12
    D = np.stack([S.descriptors(*_config(10 + b, n=n, side=6.0))[0] for b in range(B)])
    U = rng.uniform(-40, -20, B)
    p = _f64(_params(2))
    _, g = S.loss_and_grads(D, U, p, n, bf=False)
    h = 1e-6
    for name, idx in (("W1", (3, 5)), ("b1", (7,)), ("W2", (10, 20)), ("b2", (33,)),
                      ("w3", (40,)), ("b3", ())):
        pp, pm = {k: v.copy() for k, v in p.items()}, {k: v.copy() for k, v in p.items()}
        pp[name] = np.array(pp[name], np.float64)
        pm[name] = np.array(pm[name], np.float64)
        pp[name][idx] += h
        pm[name][idx] -= h
        fd = (S.loss_and_grads(D, U, pp, n, bf=False)[0] -
              S.loss_and_grads(D, U, pm, n, bf=False)[0]) / (2 * h)
        got = float(np.asarray(g[name])[idx])
        assert abs(fd - got) < 1e-4 * max(1e-3, abs(fd)), (name, fd, got)


def test_bf16_rounding_is_round_to_nearest_even():
    v = np.array([1.0, 1.00390625, 1.005859375, -3.0000002, 65504.0], np.float32)
    r = S.bf16(v)
    assert r[0] == 1.0 and r[1] == 1.0  # exact tie 1 + 2^-8 rounds to even
    assert r[2] == np.float32(1.0078125)
    assert r[3] == -3.0
