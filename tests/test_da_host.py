"""Host logic of the delayed-acceptance driver (CPU; the device set to the CPU).

- the sample ring: appends wrap around its capacity, `recent_valid` returns
  the evaluated slots of the last `window` reserved steps, newest last, and
  skips slots marked NaN;
- the triple-product volume matches numpy's determinant;
- refitting the surrogate's standardisation keeps the float64 network's
  energies (W1, b1, w3 and b3 absorb the change).
"""

import numpy as np
import pytest

torch = pytest.importorskip("torch")

from jaxrens_b200 import delayed_acceptance as da  # noqa: E402
from jaxrens_b200 import surrogate as sg  # noqa: E402
from oracle import surrogate_ref as S  # noqa: E402


@pytest.fixture
def on_cpu(monkeypatch):
    cpu = lambda: torch.device("cpu")  # noqa: E731
    monkeypatch.setattr(da, "device", cpu)
    monkeypatch.setattr(sg, "device", cpu)


def test_ring_wraps_and_selects_recent_valid_slots(on_cpu):
    ring = da.SampleRing(capacity=10, n_atoms_max=2)
    x = torch.arange(14 * 6, dtype=torch.float32).reshape(14, 2, 3)
    c = torch.eye(3).expand(14, 3, 3)
    u = torch.arange(14, dtype=torch.float64)
    u[12] = float("nan")  # a step without an exact evaluation
    ring.push(x[:8], c[:8], u[:8])
    assert ring.base == 8 and ring.reserved == 8
    ring.push(x[8:], c[8:], u[8:])
    assert ring.base == 4 and ring.reserved == 14
    # slot (i mod 10) holds entry i for the last 10 entries 4..13
    for i in range(4, 14):
        assert torch.equal(ring.positions[i % 10], x[i])
    idx = ring.recent_valid(5)  # entries 9..13 without 12
    assert ring.energy_u[idx].tolist() == [9.0, 10.0, 11.0, 13.0]
    assert ring.recent_valid(100).numel() == 9  # capacity bound, NaN skipped
    ring.reserve(3)  # a launch's steps: base moves on, slots keep old data
    assert ring.base == 7 and ring.reserved == 17


def test_triple_product_volume_matches_numpy():
    rng = np.random.default_rng(3)
    cells = rng.normal(size=(20, 3, 3))
    got = da.torch_det_abs(torch.as_tensor(cells)).numpy()
    np.testing.assert_allclose(got, np.abs(np.linalg.det(cells)), rtol=1e-12)


def test_renormalise_keeps_the_network_energies(on_cpu):
    sur = sg.Surrogate(seed=4)
    rng = np.random.default_rng(5)
    p = sg.unflatten(sur.params.numpy())
    p["b1"] = (0.1 * rng.standard_normal(64)).astype(np.float32)
    p["b3"] = np.float32(0.2)
    sur.params.copy_(torch.as_tensor(sg.flatten(p)))
    sur.in_scale = rng.uniform(0.5, 1.5, 16).astype(np.float32)
    sur.in_shift = rng.uniform(-1.0, 0.0, 16).astype(np.float32)
    sur.out_scale, sur.out_shift = 0.7, -3.0

    def ref_params():
        q = sg.unflatten(sur.params.numpy())
        q.update(in_scale=sur.in_scale, in_shift=sur.in_shift,
                 out_scale=np.float32(sur.out_scale), out_shift=np.float32(sur.out_shift))
        return q

    side = (20.0 * 16) ** (1.0 / 3.0)
    xs = rng.uniform(0, side, (4, 16, 3))
    cell = np.eye(3) * side
    before = [S.energy(x, cell, ref_params(), bf=False) for x in xs]
    D = torch.as_tensor(np.stack([S.descriptors(x, cell)[0] for x in xs]), dtype=torch.float32)
    sur.renormalise(D, torch.tensor([-40.0, -35.0, -30.0, -45.0], dtype=torch.float64), 16)
    after = [S.energy(x, cell, ref_params(), bf=False) for x in xs]
    np.testing.assert_allclose(after, before, rtol=1e-5, atol=1e-5)
    assert sur.step == 0 and float(sur.adam_m.abs().sum()) == 0.0
