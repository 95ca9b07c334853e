"""The Stillinger-Weber oracle against the model's closed forms (CPU only).

The reference has no Stillinger-Weber backend, so no reference output pins
this model ("parity unpinned" against any external implementation).  The
oracle is pinned instead by what the published functional form fixes
(F. H. Stillinger and T. A. Weber, Phys. Rev. B 31, 5262 (1985)):

- the dimer energy phi2(r) and its minimum -eps at r = 2^(1/6) sigma;
- an isolated triangle: three pair terms plus the three angle terms;
- the diamond lattice at a = 2^(1/6) sigma * 4 / sqrt(3) (5.431 A for the
  silicon parameters): -2 eps per atom, zero forces (cos theta = -1/3 kills
  the three-body term, second neighbours lie beyond a sigma);
- forces equal the negative gradient (central finite differences of the
  float64 energy);
- the kernel contract (DEV, float32 terms) against float64 within 1e-5;
- the project's float32 exp within 2 ulp of the double-precision exp.
"""

import numpy as np
import pytest

from jaxrens_b200 import create_sw
from oracle import oracle as O

SW = create_sw()
C = SW.consts


def _model():
    return O.make_sw_model(**C)


def _f64(v):
    return float(np.float64(v))


def phi2(r):
    s, rc, Ae, B = _f64(C["sw_sigma"]), _f64(C["sw_rc"]), _f64(C["sw_Aeps"]), _f64(C["sw_B"])
    if r >= rc:
        return 0.0
    return Ae * (B * (s / r) ** 4 - 1.0) * np.exp(s / (r - rc))


def g(r):
    rc, gs = _f64(C["sw_rc"]), _f64(C["sw_gsig"])
    return np.exp(gs / (r - rc)) if r < rc else 0.0


def h(rj, rk, cos):
    return _f64(C["sw_leps"]) * (cos + 1.0 / 3.0) ** 2 * g(rj) * g(rk)


def _energy(x, cell, mode, forces=True):
    x = np.asarray(x, np.float32)
    E, F, _ = O.energy(_model(), x, np.zeros(len(x), np.int32), cell, pressure=0.0, mode=mode,
                       forces=forces)
    return E, F


BIG = np.eye(3, dtype=np.float32) * 40.0


def test_sw_exp_within_two_ulp():
    xs = np.concatenate([np.linspace(-103.9, 0.0, 40001),
                         -np.exp(np.linspace(-20.0, 4.6, 4001))]).astype(np.float32)
    worst = 0.0
    for x in xs:
        y = O.sw_exp(float(x))
        ref = np.exp(np.float64(x))
        ulp = np.spacing(np.float32(ref)) if ref >= 1.2e-38 else 1.4e-45
        worst = max(worst, abs(y - ref) / ulp)
    assert worst <= 2.0, worst
    assert O.sw_exp(-200.0) == 0.0 and O.sw_exp(0.0) == 1.0


@pytest.mark.parametrize("r", [1.9, 2.2, 2.3517, 2.8, 3.5, 3.77])
def test_dimer_closed_form(r):
    x = [[0.0, 0.0, 0.0], [r, 0.0, 0.0]]
    rr = _f64(np.float32(r))
    ref = phi2(rr)
    e64, F64 = _energy(x, BIG, O.F64)
    assert abs(e64 - ref) <= 1e-12 * max(1.0, abs(ref))
    edev, Fdev = _energy(x, BIG, O.DEV)
    assert abs(edev - ref) <= 2e-6 * max(1.0, abs(ref))
    # Newton's third law, forces along the bond
    assert np.allclose(F64[0], -F64[1], rtol=0, atol=1e-12)
    assert abs(F64[0, 1]) < 1e-12 and abs(F64[0, 2]) < 1e-12


def test_dimer_minimum_is_minus_epsilon():
    rmin = 2.0 ** (1.0 / 6.0) * 2.0951
    e, F = _energy([[0.0, 0.0, 0.0], [rmin, 0.0, 0.0]], BIG, O.F64)
    assert abs(e + 2.1683) < 2e-6
    assert np.abs(F).max() < 1e-4


def test_triangle_closed_form():
    x = np.array([[0.0, 0.0, 0.0], [2.3, 0.0, 0.0], [0.6, 2.1, 0.3]], np.float32)
    xd = x.astype(np.float64)
    E = 0.0
    for i in range(3):
        for j in range(i + 1, 3):
            E += phi2(np.linalg.norm(xd[j] - xd[i]))
    for i in range(3):
        j, k = [q for q in range(3) if q != i]
        dj, dk = xd[j] - xd[i], xd[k] - xd[i]
        rj, rk = np.linalg.norm(dj), np.linalg.norm(dk)
        E += h(rj, rk, dj @ dk / (rj * rk))
    e64, _ = _energy(x, BIG, O.F64)
    edev, _ = _energy(x, BIG, O.DEV)
    assert abs(e64 - E) <= 1e-12 * abs(E)
    assert abs(edev - E) <= 1e-5 * abs(E)


def diamond(n_cells=2, a=5.431):
    base = np.array([[0, 0, 0], [0, 0.5, 0.5], [0.5, 0, 0.5], [0.5, 0.5, 0]], np.float64)
    basis = np.concatenate([base, base + 0.25])
    pts = []
    for i in range(n_cells):
        for j in range(n_cells):
            for k in range(n_cells):
                pts.append(basis + np.array([i, j, k]))
    x = np.concatenate(pts) * a
    return x.astype(np.float32), (np.eye(3) * a * n_cells).astype(np.float32)


def test_diamond_silicon_fixed_point():
    a = 2.0 ** (1.0 / 6.0) * 2.0951 * 4.0 / np.sqrt(3.0)
    assert abs(a - 5.431) < 2e-3
    x, cell = diamond(2, a)
    assert len(x) == 64
    for mode, tol in ((O.F64, 1e-6), (O.DEV, 1e-5)):
        e, F = _energy(x, cell, mode)
        assert abs(e / 64 + 2.0 * 2.1683) < tol * 4.3366, (mode, e / 64)
        assert np.abs(F).max() < 2e-3, (mode, np.abs(F).max())


def _random_config(seed, n=16, side=7.0, dmin=1.8):
    rng = np.random.default_rng(seed)
    x = []
    while len(x) < n:
        p = rng.uniform(0, side, 3)
        ok = True
        for q in x:
            d = p - q
            d -= side * np.round(d / side)
            if np.linalg.norm(d) < dmin:
                ok = False
                break
        if ok:
            x.append(p)
    return np.array(x, np.float32), (np.eye(3) * side).astype(np.float32)


@pytest.mark.parametrize("seed", [0, 1, 2])
def test_forces_are_minus_the_gradient(seed):
    x, cell = _random_config(seed)
    _, F = _energy(x, cell, O.F64)
    hstep = 1e-3
    worst = 0.0
    for i in range(len(x)):
        for q in range(3):
            xp, xm = x.copy(), x.copy()
            xp[i, q] += np.float32(hstep)
            xm[i, q] -= np.float32(hstep)
            dx = float(xp[i, q]) - float(xm[i, q])
            ep, _ = _energy(xp, cell, O.F64, forces=False)
            em, _ = _energy(xm, cell, O.F64, forces=False)
            worst = max(worst, abs(-(ep - em) / dx - F[i, q]))
    assert worst < 2e-4 * max(1.0, np.abs(F).max()), worst


@pytest.mark.parametrize("seed", [3, 4, 5, 6])
def test_kernel_contract_against_float64(seed):
    x, cell = _random_config(seed, n=24, side=8.0, dmin=1.7)
    e64, F64 = _energy(x, cell, O.F64)
    edev, Fdev = _energy(x, cell, O.DEV)
    assert abs(edev - e64) <= 1e-5 * max(1.0, abs(e64))
    assert np.abs(Fdev - F64).max() <= 1e-5 * max(1.0, np.abs(F64).max())


def test_triclinic_cell_minimum_image():
    # the same crystal in a sheared but equivalent cell: identical energy
    x, cell = diamond(2)
    c2 = cell.copy()
    c2[1] += cell[0]  # b' = b + a spans the same lattice
    e1, _ = _energy(x, cell, O.F64)
    e2, _ = _energy(x, c2, O.F64)
    assert abs(e1 - e2) < 1e-9 * abs(e1)
