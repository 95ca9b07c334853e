"""The oracle against every pin the reference offers (CPU only).

Pins: Random123 known-answer vectors for threefry2x32-20, JAX's documented
pre-partitionable ``split(key(0))``, the reference's committed lj8_npt
trajectory frames (LJ + EnsembleTerm energies), the closed forms and the
brute-force minimum-image reference of ``tests/backends/test_lj.py``, and the
reference's own numpy ``prior_mass.py`` outputs.
"""

import json
import os

import numpy as np
import pytest

from jaxrens_b200 import create_lj, prior_mass, prng
from oracle import oracle as O

GOLD = os.path.join(os.path.dirname(__file__), "golden")


def _lj_model(eps=1.0, sig=1.0, cutoff=2.5, supercell=(1, 1, 1)):
    lj = create_lj(epsilon=eps, sigma=sig, cutoff=cutoff, supercell_trafo=supercell)
    rc2 = None if cutoff is None else np.float32(cutoff ** 2)
    return O.make_model(lj.eps4, lj.eps24, lj.sig2, rc2, lj.image_offsets)


@pytest.mark.parametrize("key,ctr,expect", [
    ((0, 0), (0, 0), (0x6B200159, 0x99BA4EFE)),
    ((0xFFFFFFFF, 0xFFFFFFFF), (0xFFFFFFFF, 0xFFFFFFFF), (0x1CB996FC, 0xBB002BE7)),
    ((0x13198A2E, 0x03707344), (0x243F6A88, 0x85A308D3), (0xC4923A9C, 0x483DF7A0)),
])
def test_threefry_known_answers(key, ctr, expect):
    assert tuple(int(v) for v in O.threefry2x32(key, ctr)) == expect
    a, b = prng.threefry2x32(key[0], key[1], ctr[0], ctr[1])
    assert (int(a), int(b)) == expect


def test_split_layout_pinned_by_jax_documented_value():
    # jax.random.split(PRNGKey(0)) before the partitionable default flip
    assert O.split_original(O.key(0), 2).tolist() == [[4146024105, 967050713],
                                                      [2718843009, 1272950319]]


def test_partitionable_split_equals_fold_in_and_host_prng():
    k = O.key(1234)
    for i in range(6):
        assert np.array_equal(O.split(k, 6)[i], O.fold_in(k, i))
    assert np.array_equal(O.split(k, 6), prng.split(k, 6))
    assert np.array_equal(O.uniform(k, 64), prng.uniform(k, 64))


def test_uniform_and_normal_ranges():
    u = O.uniform(O.key(7), 4096)
    assert u.min() >= 0.0 and u.max() < 1.0
    z = O.normal(O.key(7), 20000)
    assert abs(float(z.mean())) < 0.03 and abs(float(z.std()) - 1.0) < 0.03


def test_erfinv_inverts_erf():
    from math import erf
    for x in np.linspace(-0.999, 0.999, 41):
        y = O.lib().jro_erfinv(np.float32(x))
        assert abs(erf(y) - float(np.float32(x))) < 2e-6


def test_randint_range_and_choice():
    for s in range(50):
        k = O.key(s)
        v = O.randint(k, 3, 17)
        assert 3 <= v < 17
    cum = np.cumsum(np.array([0.8, 0.2], np.float32), dtype=np.float32)
    picks = [O.choice(O.key(s), cum) for s in range(2000)]
    assert 0.76 < picks.count(0) / 2000 < 0.84


def _frames():
    return json.load(open(os.path.join(GOLD, "lj8_frames.json")))


@pytest.mark.parametrize("mode", [O.DEV, O.REF32, O.F64])
def test_lj8_golden_frames(mode):
    g = _frames()
    m = _lj_model()
    for fr in g["frames"]:
        x = np.array(fr["positions"], np.float32)
        c = np.array(fr["cell"], np.float32).reshape(3, 3)
        E, _, _ = O.energy(m, x, np.zeros(8, np.int32), c, pressure=0.1, mode=mode)
        assert abs(E - fr["ns_energy"]) / abs(fr["ns_energy"]) < 2.5e-7


def test_two_atom_closed_form_nonperiodic():
    m = _lj_model(cutoff=None)
    for r in (0.95, 1.2, 1.5, 2.3):
        x = np.array([[0, 0, 0], [r, 0, 0]], np.float32)
        E, F, _ = O.energy(m, x, [0, 0], np.zeros((3, 3)), mode=O.DEV)
        exp = 4.0 * ((1 / r) ** 12 - (1 / r) ** 6)
        assert abs(E - exp) <= 1e-5 * max(1.0, abs(exp))
        fexp = 24.0 * (2 * (1 / r) ** 13 - (1 / r) ** 7)  # on atom 1, +x
        assert abs(F[1, 0] - fexp) <= 1e-5 * max(1.0, abs(fexp))
        assert abs(F[0, 0] + F[1, 0]) <= 1e-5 * max(1.0, abs(fexp))


def test_lorentz_berthelot_mixing_value():
    lj = create_lj(epsilon=[1.0, 0.5], sigma=[1.0, 1.2])
    m = O.make_model(lj.eps4, lj.eps24, lj.sig2, None, lj.image_offsets)
    r = 1.4
    x = np.array([[0, 0, 0], [r, 0, 0]], np.float32)
    E, _, _ = O.energy(m, x, [0, 1], np.zeros((3, 3)))
    eps_ij, sig_ij = np.sqrt(0.5), 1.1
    assert abs(E - 4 * eps_ij * ((sig_ij / r) ** 12 - (sig_ij / r) ** 6)) < 1e-5


def _brute(pos, cell, cutoff, sc):
    pos = np.asarray(pos, np.float64)
    cell = np.asarray(cell, np.float64)
    inv = np.linalg.inv(cell)
    offs = [(a, b, c) for a in range(-(sc[0] // 2), sc[0] // 2 + 1)
            for b in range(-(sc[1] // 2), sc[1] // 2 + 1)
            for c in range(-(sc[2] // 2), sc[2] // 2 + 1)]
    e = 0.0
    for i in range(len(pos)):
        for j in range(len(pos)):
            dr = pos[j] - pos[i]
            dm = dr - np.round(dr @ inv) @ cell
            for off in offs:
                if i == j and off == (0, 0, 0):
                    continue
                d = dm + np.array(off, float) @ cell
                r2 = float(d @ d)
                if cutoff is not None and r2 >= cutoff ** 2:
                    continue
                s6 = (1.0 / r2) ** 3
                e += 0.5 * 4.0 * (s6 * s6 - s6)
    return e


def test_sheared_cell_matches_brute_force():
    rng = np.random.default_rng(0)
    cell = np.array([[5.0, 0.5, 0.0], [0.6, 5.0, 0.3], [0.2, 0.4, 5.0]], np.float32)
    pos = rng.uniform(-1.0, 6.0, (8, 3)).astype(np.float32)
    m = _lj_model()
    for mode in (O.DEV, O.REF32, O.F64):
        E, _, _ = O.energy(m, pos, np.zeros(8, np.int32), cell, mode=mode)
        ref = _brute(pos, cell, 2.5, (1, 1, 1))
        assert abs(E - ref) <= 1e-4 * max(1, abs(ref))


def test_tight_cell_picks_up_images():
    pos = np.array([[0, 0, 0], [1.2, 0, 0]], np.float32)
    cell = np.diag([3.55, 3.55, 3.55]).astype(np.float32)
    e1, _, _ = O.energy(_lj_model(supercell=(1, 1, 1)), pos, [0, 0], cell)
    e2, _, _ = O.energy(_lj_model(supercell=(2, 2, 2)), pos, [0, 0], cell)
    assert abs(e1 - _brute(pos, cell, 2.5, (1, 1, 1))) < 1e-4
    assert abs(e2 - _brute(pos, cell, 2.5, (2, 2, 2))) < 1e-4
    assert abs(e1 - e2) > 1e-3


def test_lattice_translation_invariance():
    rng = np.random.default_rng(1)
    cell = (np.eye(3) * 6.0034575).astype(np.float32)
    pos = rng.uniform(0, 6, (8, 3)).astype(np.float32)
    shifts = rng.integers(-8, 9, (8, 3)).astype(np.float32)
    shifted = (pos + shifts @ cell).astype(np.float32)
    m = _lj_model()
    a = O.energy(m, pos, np.zeros(8, np.int32), cell)[0]
    b = O.energy(m, shifted, np.zeros(8, np.int32), cell)[0]
    assert abs(a - b) < 1e-3


def test_dev_and_ref32_forces_match_f64_and_finite_differences():
    rng = np.random.default_rng(2)
    cell = (np.eye(3) * 4.6).astype(np.float32)
    pos = (rng.uniform(0, 1, (16, 3)) * 4.6).astype(np.float32)
    m = _lj_model()
    t = np.zeros(16, np.int32)
    E64, F64, _ = O.energy(m, pos, t, cell, mode=O.F64)
    for mode in (O.DEV, O.REF32):
        E, F, _ = O.energy(m, pos, t, cell, mode=mode)
        assert abs(E - E64) <= 1e-5 * max(1.0, abs(E64))
        assert np.abs(F - F64).max() <= 1e-5 * max(1.0, np.abs(F64).max())
    h = 1e-4
    for i, q in [(0, 0), (3, 1), (7, 2)]:
        p1, p2 = pos.astype(np.float64).copy(), pos.astype(np.float64).copy()
        p1[i, q] += h
        p2[i, q] -= h
        e1 = O.energy(m, p1.astype(np.float32), t, cell, mode=O.F64)[0]
        e2 = O.energy(m, p2.astype(np.float32), t, cell, mode=O.F64)[0]
        dx = float(np.float32(pos[i, q] + h)) - float(np.float32(pos[i, q] - h))
        assert abs(-(e1 - e2) / dx - F64[i, q]) < 2e-2 * max(1.0, abs(F64[i, q]))


def test_prior_mass_matches_reference_outputs():
    g = json.load(open(os.path.join(GOLD, "prior_mass.json")))
    for c in g["cases"]:
        K, nc = c["n_live"], c["n_cull"]
        assert prior_mass.log_alpha(K, nc) == c["log_alpha"]
        xo, wo = prior_mass.iteration_offsets(K, nc)
        np.testing.assert_array_equal(xo, c["x_offset"])
        np.testing.assert_array_equal(wo, c["w_offset"])
        np.testing.assert_allclose(prior_mass.log_dead_weights(30, K, nc),
                                   c["log_dead_weights_30"], rtol=0, atol=1e-14)
        assert abs(prior_mass.log_live_weight(30, K, nc) - c["log_live_weight_30"]) < 1e-12


def test_energies_file_format_pin():
    g = json.load(open(os.path.join(GOLD, "lj8_energies.json")))
    n_walkers, n_cull, n_dof, zero, n_atoms = g["header"].split()
    assert (int(n_walkers), int(n_cull), int(n_atoms)) == (32, 1, 8)
    it, H, V = g["rows"][0].split()
    assert int(it) == 0 and float(H) > 0 and float(V) > 0


def test_thermodynamics_match_reference_outputs():
    """postprocess/thermodynamics.py restated: log Z, log Z(beta) and C_v on
    the seeded fixture equal the reference module's own outputs."""
    from jaxrens_b200 import thermo

    g = json.load(open(os.path.join(GOLD, "thermo.json")))
    for c in g["cases"]:
        d, l, K, nc = np.array(c["dead"]), np.array(c["live"]), c["n_live"], c["n_cull"]
        assert abs(thermo.log_evidence(d, l, K, nc) - c["log_evidence"]) <= 1e-12 * abs(c["log_evidence"])
        for b, z, cv in zip(c["betas"], c["partition_function"], c["heat_capacity"]):
            assert abs(thermo.partition_function(b, d, l, K, nc) - z) <= 1e-12 * max(1, abs(z))
            assert abs(thermo.heat_capacity(b, d, l, K, nc) - cv) <= 1e-10 * max(1, abs(cv))
