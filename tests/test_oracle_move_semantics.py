"""The reference's own property tests of the walk, run against the oracle (CPU).

* Galilean trajectory semantics (``tests/sampling/moves/test_moves.py:358-510``):
  a move with no path below the contour is rejected and leaves the walker
  intact; on rejection the stored direction is minus the *perturbed* direction
  (not minus the incoming one); every accepted move ends below the contour;
  persistent-direction GMC keeps a uniform ensemble inside a harmonic contour
  uniform (``<r^2> = d/(d+2)``).  The harmonic well is the Gaussian-mixture
  toy with one centre at the origin (``backends/toy.py:163-204``): for one
  atom its energy is ``|x|^2/(2 sigma^2) + 1.5 log(2 pi sigma^2)``, a 3-D
  harmonic well, so the invariant is ``<r^2> = 3/5`` inside ``|x| < 1``.
* Semi-grand replica-exchange rebase
  (``tests/sampling/replica_exchange/test_semigrand.py:102-140``): the stored
  energy ``U - mu_self . N`` is re-based to the receiving run's ``mu`` on a
  swap, with the reference's hand-calculated values (5.0 and 1.0).
"""

import numpy as np

from jaxrens_b200 import build_mwg, create_lj, prng
from jaxrens_b200 import moves as mvs
from jaxrens_b200.backends import GaussianMixtureBackend
from oracle import oracle as O
from tests._cases import oracle_model, oracle_moves

E_CONST = 1.5 * np.log(2.0 * np.pi)  # the normalisation of a sigma = 1 component


def harmonic_case(step_size, n_reflect):
    g = GaussianMixtureBackend(centers=[[0.0, 0.0, 0.0]], sigma=1.0)
    _, step, _ = build_mwg(g, [mvs.gmc(n_reflect=n_reflect, step_size=step_size, weight=1.0)])
    return g, step, oracle_model(g), oracle_moves(step)


def harmonic_energy(x):
    x = np.asarray(x, np.float64)
    return 0.5 * np.sum(x.reshape(-1, 3) ** 2) + E_CONST


def uniform_ball(n, seed):
    """n points uniform in the unit 3-ball and n unit directions (float32)."""
    rng = np.random.default_rng(seed)
    x = rng.standard_normal((n, 3))
    x /= np.linalg.norm(x, axis=1, keepdims=True)
    x *= rng.uniform(size=(n, 1)) ** (1.0 / 3.0)
    v = rng.standard_normal((n, 3))
    v /= np.linalg.norm(v, axis=1, keepdims=True)
    return x.astype(np.float32).reshape(n, 1, 3), v.astype(np.float32).reshape(n, 1, 3)


X0 = np.array([[0.6, -0.4, 0.3]], np.float32)


def _trial(model, moves, key, step, emax, x, d, mode=O.REF32):
    return O.move_trial(model, moves, 0, key, step, emax, x, d, np.zeros(1, np.int32),
                        np.zeros((3, 3), np.float32), harmonic_energy(x), mode=mode)


def test_reject_when_no_path_below_constraint():
    _, _, model, moves = harmonic_case(0.5, 4)
    d0 = np.ones((1, 3), np.float32) / np.float32(np.sqrt(3.0))
    # a contour below the well's minimum: no trajectory can end under it
    acc, x, _, _, _, e, _ = _trial(model, moves, prng.key(0), 0.5, E_CONST - 0.1, X0, d0)
    assert not acc
    np.testing.assert_array_equal(x, X0)
    assert e == float(np.float32(harmonic_energy(X0)))  # the float32 MCState energy


def test_reject_flips_the_perturbed_direction():
    _, step, model, moves = harmonic_case(0.5, 4)
    d0 = np.ones((1, 3), np.float32) / np.float32(np.sqrt(3.0))
    key = prng.key(0)
    acc, _, d, _, _, _, _ = _trial(model, moves, key, 0.5, E_CONST - 0.1, X0, d0)
    assert not acc
    # the kernel's key split (init, perturb, reflect); perturbation 0.1 * normal
    _, k_perturb, _ = O.split(key, 3)
    used = d0 + np.float32(step.params.moves.perturb_angle[0]) * O.normal(k_perturb, 3).reshape(1, 3)
    used = used / np.linalg.norm(used)
    np.testing.assert_allclose(d, -used, atol=1e-6)
    assert not np.allclose(d, -d0, atol=1e-3)


def test_accepted_moves_advance_and_end_below_the_contour():
    _, _, model, moves = harmonic_case(0.05, 5)
    emax = E_CONST + 0.5
    x = X0 * np.float32(0.5)
    d = np.zeros((1, 3), np.float32)
    key = prng.key(7)
    n_acc = 0
    for _ in range(60):
        key, sub = O.split(key, 2)
        acc, xn, d, _, _, e, _ = _trial(model, moves, sub, 0.05, emax, x, d)
        if acc:
            n_acc += 1
            assert e < emax
            assert not np.array_equal(xn, x)
        else:
            np.testing.assert_array_equal(xn, x)
        x = xn
    assert n_acc > 5


def walk_uniform_ball(n, seed, n_calls, mode=O.REF32):
    """``n_calls`` persistent-direction GMC steps of every walker at the fixed
    contour |x| = 1 (step 0.15, 4 reflections), from a uniform start."""
    _, step, model, moves = harmonic_case(0.15, 4)
    x, v = uniform_ball(n, seed)
    e = np.array([harmonic_energy(p) for p in x])
    rep = O.Replica(x, np.zeros((n, 1), np.int32), e, np.zeros((n, 3, 3), np.float32),
                    np.full((n, 1), 0.15, np.float32), prng.key(seed), direction=v)
    keys = prng.split(prng.key(seed + 1), 2)
    O.walk_population(model, moves, rep, n_calls, keys[0], keys[1], E_CONST + 0.5, mode=mode)
    return rep, keys


def test_persistent_direction_keeps_the_uniform_ball_invariant():
    rep, _ = walk_uniform_ball(8000, 0, 100)
    r2 = np.sum(rep.positions.astype(np.float64) ** 2, axis=(1, 2))
    assert np.all(r2 < 1.0 + 1e-6)
    # standard error of <r^2> for 8000 uniform points in a 3-ball: 0.0029
    assert abs(r2.mean() - 0.6) < 0.009, r2.mean()
    assert rep.n_prop.sum() == 8000 * 100 and 0 < rep.n_acc.sum() < rep.n_prop.sum()


def _semigrand_replicas(K):
    lj = create_lj(epsilon=[1.0, 1.0], sigma=[1.0, 1.0], cutoff=2.5)
    mu_a, mu_b = [0.0, 0.0], [0.5, 1.0]
    xa = np.tile(np.array([[0.0, 0.0, 0.0], [1.5, 0.0, 0.0], [0.0, 1.5, 0.0]], np.float32), (K, 1, 1))
    xb = xa + np.float32(0.25)
    ta = np.tile(np.array([0, 0, 1], np.int32), (K, 1))  # N_A = [2, 1]
    tb = np.tile(np.array([1, 1, 0], np.int32), (K, 1))  # N_B = [1, 2]
    cells = np.zeros((K, 3, 3), np.float32)  # |det| = 0: no P V share
    stored_a = np.full(K, 3.0 - (mu_a[0] * 2 + mu_a[1] * 1))  # 3.0
    stored_b = np.full(K, 5.0 - (mu_b[0] * 1 + mu_b[1] * 2))  # 2.5
    ss = np.full((K, 2), 0.1, np.float32)
    a = O.Replica(xa, ta, stored_a, cells, ss, prng.key(1), mu=mu_a, emax=10.0)
    b = O.Replica(xb, tb, stored_b, cells, ss, prng.key(2), mu=mu_b, emax=10.0)
    return lj, (a, b), (xa, xb, ta, tb, stored_a, stored_b, mu_a, mu_b)


def test_semigrand_swap_rebases_to_the_receiving_chemical_potential():
    for mode in (O.DEV, O.REF32):
        _, (a, b), (xa, xb, ta, tb, *_) = _semigrand_replicas(1)
        acc, att = O.re_step([a, b], prng.key(0), n_swap_cycles=1, mode=mode)
        assert (int(acc[0]), int(att[0])) == (1, 1)
        # walker B now in run A: U_B - mu_A . N_B = 5.0; walker A in run B: 1.0
        assert abs(a.energy[0] - 5.0) < 1e-6 and abs(b.energy[0] - 1.0) < 1e-6
        np.testing.assert_array_equal(a.types[0], tb[0])
        np.testing.assert_array_equal(b.positions[0], xa[0])


def test_semigrand_swap_is_refused_above_either_contour():
    _, (a, b), _ = _semigrand_replicas(1)
    a.emax[0] = 4.0  # walker B would arrive in run A at 5.0
    acc, att = O.re_step([a, b], prng.key(0), n_swap_cycles=1)
    assert (int(acc[0]), int(att[0])) == (0, 1)
    assert a.energy[0] == 3.0 and b.energy[0] == 2.5


def test_ensemble_term_of_the_semigrand_case_is_minus_mu_n():
    lj, _, (xa, _, ta, *_) = _semigrand_replicas(1)
    model = oracle_model(lj)
    cell = np.eye(3, dtype=np.float32) * 20
    u = O.energy(model, xa[0], ta[0], cell, mode=O.DEV, forces=False)[0]
    g = O.energy(model, xa[0], ta[0], cell, mu=[0.5, 1.0], mode=O.DEV, forces=False)[0]
    # stored = U - mu . N with N_A = [2, 1]
    assert abs((u - g) - (0.5 * 2 + 1.0 * 1)) < 1e-12
