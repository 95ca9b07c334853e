"""The surrogate's training kernels on the GPU against the CPU reference (B200).

``oracle/surrogate_ref.py`` restates the descriptors, the network and the
loss; its bfloat16 mode rounds the matrix operands as the tensor-core
kernels do.  Checked here:

- descriptors of random configurations: 1e-4 relative (float32 geometry and
  exponentials against float64);
- one training step's loss and every gradient (W1, b1, W2, b2, w3, b3),
  recovered from Adam's first moment after one step from zero moments with a
  zero learning rate (m = 0.1 g): the loss to 1e-3 relative, the gradients to
  3e-2 of the largest entry of each tensor (bfloat16 operands, float32 sums
  in another order); odd and even batch sizes;
- training lowers the loss of a fit to the Stillinger-Weber energies of
  perturbed, rescaled 64-atom diamond silicon cells.
"""

import numpy as np
import pytest

from jaxrens_b200 import surrogate as sg
from oracle import surrogate_ref as S

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _configs(seed, B, n=64, side=None):
    rng = np.random.default_rng(seed)
    side = side if side is not None else (20.0 * n) ** (1.0 / 3.0)
    x = rng.uniform(0, side, (B, n, 3)).astype(np.float32)
    c = np.tile((np.eye(3) * side).astype(np.float32), (B, 1, 1))
    return x, c


@pytest.mark.parametrize("n", [20, 64])
def test_descriptors_match_reference(n):
    x, c = _configs(n, 5, n=n)
    D = sg.Surrogate.descriptors(x, c).cpu().numpy()
    for b in range(5):
        ref, *_ = S.descriptors(x[b], c[b])
        np.testing.assert_allclose(D[b], ref, rtol=1e-4, atol=1e-6)


def _surrogate_with(seed):
    sur = sg.Surrogate(seed=seed)
    rng = np.random.default_rng(seed + 7)
    p = sg.unflatten(sur.params.cpu().numpy())
    p["b1"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b2"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b3"] = np.float32(0.3)
    sur.params.copy_(torch.as_tensor(sg.flatten(p)))
    sur.in_scale = rng.uniform(0.5, 1.5, 16).astype(np.float32)
    sur.in_shift = rng.uniform(-1.0, 0.0, 16).astype(np.float32)
    sur.out_scale, sur.out_shift = 0.8, -2.0
    return sur


def _ref_params(sur):
    p = sg.unflatten(sur.params.cpu().numpy())
    p.update(in_scale=sur.in_scale, in_shift=sur.in_shift, out_scale=np.float32(sur.out_scale),
             out_shift=np.float32(sur.out_shift))
    return p


@pytest.mark.parametrize("B", [6, 5])
def test_train_step_gradients_match_reference(B):
    x, c = _configs(100 + B, 8)
    D = sg.Surrogate.descriptors(x, c)
    rng = np.random.default_rng(B)
    U = torch.as_tensor(rng.uniform(-150.0, -100.0, 8), dtype=torch.float64, device=D.device)
    idx_np = rng.permutation(8)[:B].astype(np.int32)
    idx = torch.as_tensor(idx_np, device=D.device)
    sur = _surrogate_with(3)
    p = _ref_params(sur)
    before = sur.params.cpu().numpy().copy()
    sur.train_step(D, U, idx, lr=0.0)
    torch.cuda.synchronize()
    assert not sur.train_error()
    g_gpu = sg.unflatten(sur.adam_m.cpu().numpy() / np.float32(0.1))
    loss, g = S.loss_and_grads(D.cpu().numpy()[idx_np], U.cpu().numpy()[idx_np], p, 64, bf=True)
    assert abs(float(sur.last_loss.item()) - loss) <= 1e-3 * max(loss, 1e-6)
    for name in ("W1", "b1", "W2", "b2", "w3", "b3"):
        a, b = np.atleast_1d(g_gpu[name]), np.atleast_1d(g[name])
        scale = max(np.abs(b).max(), 1e-12)
        assert np.abs(a - b).max() <= 3e-2 * scale, (name, np.abs(a - b).max(), scale)
    # a zero learning rate leaves the parameters as they were
    np.testing.assert_array_equal(sur.params.cpu().numpy(), before)


def perturbed_diamond(seed, B, amp=0.35):
    """B 64-atom silicon cells: the diamond lattice rescaled by up to +-6%
    in volume and every atom displaced by up to amp A (the solid-like
    configurations of a late nested-sampling run)."""
    from tests.test_oracle_sw import diamond

    rng = np.random.default_rng(seed)
    x0, c0 = diamond(2)
    xs, cs = [], []
    for _ in range(B):
        f = (1.0 + rng.uniform(-0.06, 0.06)) ** (1.0 / 3.0)
        xs.append((x0 * f + rng.uniform(-amp, amp, x0.shape)).astype(np.float32))
        cs.append((c0 * f).astype(np.float32))
    return np.stack(xs), np.stack(cs)


def test_training_lowers_the_loss_on_stillinger_weber_energies():
    from jaxrens_b200 import create_sw
    from oracle import oracle as O

    sw = create_sw()
    m = O.make_sw_model(**sw.consts)
    x, c = perturbed_diamond(7, 512)
    U = np.array([O.energy(m, x[b], np.zeros(64, np.int32), c[b], mode=O.F64, forces=False)[2]
                  for b in range(len(x))])
    D = sg.Surrogate.descriptors(x, c)
    Ut = torch.as_tensor(U, dtype=torch.float64, device=D.device)
    sur = sg.Surrogate(seed=1)
    sur.fit_normalisation(D, U, 64)
    first = sur.fit(D, Ut, epochs=1, batch=64, lr=3e-3)
    last = sur.fit(D, Ut, epochs=60, batch=64, lr=3e-3)
    assert not sur.train_error()
    assert last < 0.2 * first, (first, last)


def test_renormalise_keeps_the_function():
    """Refitting the standardisation rewrites W1, b1, w3 and b3 so that the
    float64 network computes the same energies as before."""
    x, c = _configs(41, 6)
    sur = _surrogate_with(8)
    before = _ref_params(sur)
    xs, cs = perturbed_diamond(3, 16)
    D = sg.Surrogate.descriptors(xs, cs)
    U = torch.as_tensor(np.linspace(-200.0, -150.0, 16), dtype=torch.float64)
    sur.renormalise(D, U, 64)
    after = _ref_params(sur)
    assert not np.allclose(before["in_scale"], after["in_scale"])
    for b in range(len(x)):
        e0 = S.energy(x[b], c[b], before, bf=False)
        e1 = S.energy(x[b], c[b], after, bf=False)
        assert abs(e0 - e1) <= 1e-5 * max(abs(e0), 1.0), (e0, e1)
