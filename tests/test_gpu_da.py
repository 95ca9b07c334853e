"""The delayed-acceptance walk on the learned surrogate (B200).

- the walk's surrogate energy and forces (``jr_sur_energy_forces``: the
  evaluation inside the walk, warp-level tensor-core products) against the
  CPU reference ``oracle/surrogate_ref.py`` in its bfloat16 mode: U to 2e-3
  of sum |e_i| out_scale, forces to 3e-2 of the largest component;
- a flat surrogate constraint (contour far above every energy) reduces the
  two-stage moves to the exact ones: with one-step galilean trajectories the
  walk is the plain walk, walker for walker and bit for bit;
- invariants of a walk with an untrained surrogate: every stored energy is
  the exact potential of its walker, the contour falls, every walker sits
  below it, the sample ring holds exactly the configurations the walk
  evaluated with their exact energies, and the counters add up (one exact
  evaluation per galilean or volume step at most, n_reflect or more
  surrogate evaluations per galilean step).
"""

import numpy as np
import pytest

from jaxrens_b200 import create_sw
from jaxrens_b200 import delayed_acceptance as da
from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200 import surrogate as sg
from oracle import surrogate_ref as S
from tests._cases import lj_case
from tests.test_gpu_parity import _np
from tests.test_gpu_surrogate import _ref_params, _surrogate_with, perturbed_diamond

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _gas(seed, B, n, vpa):
    rng = np.random.default_rng(seed)
    side = (vpa * n) ** (1.0 / 3.0)
    x = rng.uniform(0, side, (B, n, 3)).astype(np.float32)
    c = np.tile((np.eye(3) * side).astype(np.float32), (B, 1, 1))
    return x, c


@pytest.mark.parametrize("kind", ["gas64", "gas20", "diamond"])
def test_walk_surrogate_energy_forces_match_reference(kind):
    if kind == "gas64":
        x, c = _gas(5, 6, 64, 20.0)
    elif kind == "gas20":
        x, c = _gas(6, 6, 20, 30.0)
    else:
        x, c = perturbed_diamond(9, 6)
    sur = _surrogate_with(4)
    p = _ref_params(sur)
    U, F = da.surrogate_energy_forces(sur, x, c)
    U, F = _np(U), _np(F)
    for b in range(len(x)):
        Ur, Fr = S.energy_forces(x[b], c[b], p, bf=True)
        D, *_ = S.descriptors(x[b], c[b])
        e, _ = S.mlp_forward(D, p, bf=True)
        scale = float(np.abs(e.astype(np.float64) * p["out_scale"]).sum())
        assert abs(U[b] - Ur) <= 2e-3 * scale, (b, U[b], Ur, scale)
        fs = np.abs(Fr).max()
        assert np.abs(F[b] - Fr).max() <= 3e-2 * fs, (b, np.abs(F[b] - Fr).max(), fs)


P_SI = 0.1 * 0.006241509


def _sw_case(P, K, R, T, seed, vpa=30.0, weights=(4.0, 1.0)):
    return lj_case(P=P, K=K, N=64, seed=seed, n_reflect=R, T=T, pressure=P_SI,
                   v_hi_per_atom=vpa, step_sizes=(0.3, 2.0), backend=create_sw(),
                   weights=weights)


def _init(case):
    return nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                case["energies"], case["cells"], case["run_keys"],
                                ensemble_params={"pressure": case["pressures"],
                                                 "chemical_potentials": None})


def _flat_surrogate():
    """A surrogate whose smoothed constraint is 1 everywhere: the contour
    sits 1e30 above every energy."""
    sur = sg.Surrogate(seed=2, tau=0.05, contour_shift=1e30)
    return sur


def test_flat_surrogate_reduces_to_the_exact_walk():
    """One-step galilean trajectories (no reflection moves a position) and
    volume moves: with s(x) = 1 stage 1 always passes (the volume prior test
    is the exact move's, on the same draw) and stage 2 is the exact move's
    energy test, so the walk is the plain walk bit for bit."""
    case = _sw_case(P=2, K=12, R=1, T=6, seed=31)
    ns_a, ns_b = _init(case), _init(case)
    sur = _flat_surrogate()
    ia = nsm.ns_iterate(ns_a, case["step"], 5, case["T"])
    ib = da.ns_iterate_da(ns_b, case["step"], sur, 5, case["T"])
    torch.cuda.synchronize()
    pa, pb = ns_a.population, ns_b.population
    np.testing.assert_array_equal(_np(pa.positions), _np(pb.positions))
    np.testing.assert_array_equal(_np(pa.cell), _np(pb.cell))
    np.testing.assert_array_equal(_np(pa.energy64), _np(pb.energy64))
    np.testing.assert_array_equal(_np(ia.dead_energy), _np(ib.dead_energy))
    np.testing.assert_array_equal(_np(ia.log_evidence), _np(ib.log_evidence))
    np.testing.assert_array_equal(_np(ia.n_accepted), _np(ib.n_accepted))
    np.testing.assert_array_equal(_np(ia.n_proposed), _np(ib.n_proposed))
    # exact evaluations: the volume steps whose prior and cell passed, and
    # every galilean step; one surrogate evaluation per step at least
    ne_b = _np(ib.n_evaluations)
    assert (ne_b <= _np(ib.n_proposed)).all()
    assert (ne_b[..., 0] == _np(ib.n_proposed)[..., 0]).all()
    assert (_np(ib.n_surrogate_evaluations) >= _np(ib.n_proposed)).all()


def _exact_u(case, x, c):
    from jaxrens_b200.backends import _evaluate

    B, N, _ = x.shape
    return _np(_evaluate(case["H"].model, None, x, np.zeros(N, np.int32), c, False).energy)


def test_walk_with_untrained_surrogate_keeps_the_exact_invariants():
    R, T, n_iter = 3, 6, 4
    case = _sw_case(P=2, K=16, R=R, T=T, seed=32)
    ns = _init(case)
    pop = ns.population
    P, K, N = pop.types.shape
    sur = sg.Surrogate(seed=5, tau=0.2)
    x0 = pop.positions.reshape(P * K, N, 3)
    c0 = pop.cell.reshape(P * K, 3, 3)
    D = sg.Surrogate.descriptors(x0, c0)
    sur.fit_normalisation(D, torch.as_tensor(_exact_u(case, _np(x0), _np(c0))), N)
    ring = da.SampleRing(4096, N)
    info = da.ns_iterate_da(ns, case["step"], sur, n_iter, T, ring=ring)
    torch.cuda.synchronize()
    assert ring.reserved == n_iter * P * T
    # stored energies: the exact potential U + P V of each walker
    x, c = _np(pop.positions), _np(pop.cell)
    U = _exact_u(case, x.reshape(-1, N, 3), c.reshape(-1, 3, 3)).reshape(P, K)
    vol = np.abs(np.linalg.det(c.astype(np.float64)))
    e64 = _np(pop.energy64)
    np.testing.assert_allclose(e64, U + np.float32(P_SI) * vol.astype(np.float32), rtol=1e-6)
    # the contour falls and every walker sits below the last one
    dead = _np(info.dead_energy)
    assert (np.diff(dead, axis=0) <= 0).all()
    assert (e64 < dead[-1][:, None]).all()
    # counters per move (0 galilean, 1 volume)
    prop, ne = _np(info.n_proposed), _np(info.n_evaluations)
    nsur, acc = _np(info.n_surrogate_evaluations), _np(info.n_accepted)
    assert (acc <= ne).all() and (ne <= prop).all()
    assert (nsur[..., 0] >= R * prop[..., 0]).all()
    assert (nsur[..., 0] <= 2 * R * prop[..., 0]).all()
    assert (nsur[..., 1] == prop[..., 1]).all()
    # the ring: one slot per step, the evaluated ones with their exact U
    eu = _np(ring.energy_u)[:ring.reserved]
    ok = np.isfinite(eu)
    assert ok.sum() == ne.sum()
    xr = _np(ring.positions)[:ring.reserved][ok]
    cr = _np(ring.cell)[:ring.reserved][ok]
    np.testing.assert_allclose(eu[ok], _exact_u(case, xr, cr), rtol=1e-9, atol=1e-9)


def test_ablation_trained_surrogate_screens_better_than_untrained():
    """Same condensed-silicon walkers, keys and contours: after bootstrap
    training the surrogate's stage 1 passes proposals that the exact stage 2
    then accepts far more often than an untrained network with the same
    normalisation and constraint width does (accepted per exact evaluation of
    the galilean move)."""
    from jaxrens_b200 import EnsembleTerm, Hamiltonian, build_mwg, prng
    from jaxrens_b200 import moves as mvs

    P, K, T, R = 4, 128, 10, 10
    H = Hamiltonian(create_sw(), [EnsembleTerm(pressure=P_SI)])
    init_fn, step, _ = build_mwg(H, [mvs.gmc(n_reflect=R, step_size=0.05, weight=4.0),
                                     mvs.volume_move(64, step_size=0.5, weight=1.0)])
    pos, cells = zip(*[perturbed_diamond(40 + r, K) for r in range(P)])
    ns = nsm.init_ns_parallel(init_fn, list(pos), [np.zeros((K, 64), np.int32)] * P, None,
                              list(cells), prng.split(prng.key(41), P),
                              ensemble_params={"pressure": np.full(P, P_SI, np.float32)})
    drv = da.DelayedAcceptanceNS(ns, step, n_mcmc_steps=T, train_every=0,
                                 bootstrap_steps=400, seed=3)
    drv.bootstrap()
    untrained = sg.Surrogate(seed=9)
    untrained.in_scale, untrained.in_shift = drv.sur.in_scale, drv.sur.in_shift
    untrained.out_scale, untrained.out_shift = drv.sur.out_scale, drv.sur.out_shift
    untrained.tau, untrained.contour_shift = drv.sur.tau, drv.sur.contour_shift
    rate = {}
    for name, sur in (("trained", drv.sur), ("untrained", untrained)):
        s = ns.clone()
        info = da.ns_iterate_da(s, step, sur, 30, T)
        acc = _np(info.n_accepted)[..., 0].sum()
        ne = _np(info.n_evaluations)[..., 0].sum()
        rate[name] = acc / max(ne, 1)
    assert rate["trained"] > rate["untrained"] + 0.03, rate


def test_delayed_acceptance_samples_the_exact_constrained_prior():
    """Long chains (120 MWG steps per iteration) on 8 runs of 32 condensed
    silicon walkers: nested sampling with the delayed-acceptance walk (the
    surrogate trained on the population, its contour moved 1.5 robust
    standard deviations inside) and with the exact walk reach the same
    contour energies after the same iterations, within 4 standard errors of
    the 8-run ensembles.  A first stage that breaks detailed balance (a trajectory
    that reflects at its final point, a prior ratio clamped before the
    surrogate ratio) moves the contours down by several standard errors."""
    from jaxrens_b200 import EnsembleTerm, Hamiltonian, build_mwg, prng
    from jaxrens_b200 import moves as mvs

    P, K, T, R, n_iter = 8, 32, 120, 5, 48
    H = Hamiltonian(create_sw(), [EnsembleTerm(pressure=P_SI)])
    init_fn, step, _ = build_mwg(H, [mvs.gmc(n_reflect=R, step_size=0.05, weight=4.0),
                                     mvs.volume_move(64, step_size=0.5, weight=1.0)])
    pos, cells = zip(*[perturbed_diamond(60 + r, K) for r in range(P)])

    def fresh(seed):
        return nsm.init_ns_parallel(init_fn, list(pos), [np.zeros((K, 64), np.int32)] * P,
                                    None, list(cells), prng.split(prng.key(seed), P),
                                    ensemble_params={"pressure": np.full(P, P_SI, np.float32)})

    ns_exact, ns_da = fresh(61), fresh(62)
    drv = da.DelayedAcceptanceNS(ns_da, step, n_mcmc_steps=T, train_every=0,
                                 bootstrap_steps=300, shift_sigmas=1.5, seed=3)
    drv.bootstrap()
    ie = nsm.ns_iterate(ns_exact, step, n_iter, T)
    idd = da.ns_iterate_da(ns_da, step, drv.sur, n_iter, T)
    torch.cuda.synchronize()
    for row in (n_iter // 2 - 1, n_iter - 1):
        a, b = _np(ie.dead_energy)[row], _np(idd.dead_energy)[row]
        se = np.sqrt(a.var(ddof=1) / P + b.var(ddof=1) / P)
        assert abs(a.mean() - b.mean()) < 4 * se + 1e-9, (row, a, b)


def test_energy_only_path_gives_the_same_energy():
    """The walk's energy-only surrogate evaluation (trajectory steps) and the
    one with forces (reflections) give the same U bit for bit: both reduce
    the same per-thread partials by the same tree."""
    x, c = perturbed_diamond(11, 8)
    sur = _surrogate_with(6)
    U0, _ = da.surrogate_energy_forces(sur, x, c, forces=False)
    U1, F = da.surrogate_energy_forces(sur, x, c, forces=True)
    np.testing.assert_array_equal(_np(U0), _np(U1))
    assert np.isfinite(_np(F)).all()
