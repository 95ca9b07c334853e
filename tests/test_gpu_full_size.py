"""Size-independent properties of the walk at the full batched sizes (B200).

The oracle cannot follow thousands of walkers through hundreds of iterations
in a test's time, so at these sizes the checks are properties that hold at
any size, plus an oracle recomputation of a sample of walkers:

* the contour of every run never increases (nested sampling's ordering; a
  replica-exchange swap only brings in walkers below both contours);
* every live walker lies at or below its run's last contour;
* a stored float64 energy equals the oracle's energy of the stored state
  (positions, cell, species) in the kernel's arithmetic, to 1e-12;
* the per-iteration counters follow the move mix: n_mcmc_steps proposals per
  chain, n_reflect evaluations per galilean proposal, one per other move;
* log Z is the running logaddexp of the dead-point weights (recomputed on
  the host from the reported contours), finite and non-decreasing;
* worst and clone indices are valid and distinct.

Workloads: the batched LJ-32 NPT configuration (8 runs x 512 walkers,
n_mcmc_steps 40, 10 reflections, replica exchange every 10 iterations) and
the uneven semi-grand configuration (16 runs x 1024 walkers of binary LJ with
16 to 96 atoms, morph and swap identity moves).  A third case plants a NaN
energy (two coincident atoms) in a small population and follows the
reference's by-value NaN handling against the oracle.
"""

import numpy as np
import pytest

from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200 import _lib, prior_mass, prng
from oracle import oracle as O
from tests._cases import lj_case, oracle_replicas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _np(t):
    return t.detach().cpu().numpy()


def _init(case):
    return nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                case["energies"], case["cells"], case["run_keys"],
                                ensemble_params={"pressure": case["pressures"],
                                                 "chemical_potentials": case["mus"]})


def _walk(case, n_launch, n_iter, re_every=None):
    ns = _init(case)
    re = nsm.InterREManager(re_every, 1, prng.key(77)) if re_every else None
    infos, swaps = [], []
    for _ in range(n_launch):
        infos.append(nsm.ns_iterate(ns, case["step"], n_iter, case["T"], 0))
        if re is not None:
            swaps.append(re.apply(ns, case["step"]))
    torch.cuda.synchronize()
    cat = lambda name: np.concatenate([_np(getattr(i, name)) for i in infos], axis=0)
    return ns, {k: cat(k) for k in ("emax", "log_evidence", "worst_idx", "clone_idx",
                                    "n_accepted", "n_proposed", "n_evaluations",
                                    "n_grad_evaluations")}, swaps


def _check(case, ns, info, swaps, sample=12):
    K, T, P = case["K"], case["T"], case["P"]
    step = case["step"]
    em, lz = info["emax"], info["log_evidence"]  # (iterations, runs)
    n_it = em.shape[0]
    assert np.all(np.isfinite(em)) and np.all(np.isfinite(lz))
    # the contour never rises; log Z never falls
    assert np.all(np.diff(em, axis=0) <= 0.0)
    assert np.all(np.diff(lz, axis=0) >= 0.0)
    # log Z is the running logaddexp of i log(alpha) + w_offset - E_dead
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    z = np.full(P, -np.inf)
    for t in range(n_it):
        z = np.logaddexp(z, t * la + wo - em[t])
    np.testing.assert_allclose(lz[-1], z, rtol=1e-12)
    # live walkers at or below the last contour
    E = _np(ns.population.energy64)
    assert np.all(E <= _np(ns.emax)[:, None])
    assert np.all(_np(ns.iteration) == n_it)
    # indices
    w, c = info["worst_idx"], info["clone_idx"]
    assert np.all((w >= 0) & (w < K) & (c >= 0) & (c < K) & (w != c))
    # counters follow the move mix
    prop, ev, gr = info["n_proposed"], info["n_evaluations"], info["n_grad_evaluations"]
    assert np.all(prop.sum(axis=2) == T)
    assert np.all(info["n_accepted"] <= prop)
    types = [step.params.moves.type[m] for m in range(step.n_moves)]
    for m, ty in enumerate(types):
        gal = ty == _lib.MOVE_GALILEAN
        per = step.params.moves.n_reflect[m] if gal else 1
        np.testing.assert_array_equal(ev[:, :, m], per * prop[:, :, m])
        np.testing.assert_array_equal(gr[:, :, m], (per if gal else 0) * prop[:, :, m])
    for s in swaps:
        assert np.all(_np(s["n_accepted_per_pair"]) <= _np(s["n_attempted_per_pair"]))
    # stored energies of a sample of walkers against the oracle
    X, C_, Ty = _np(ns.population.positions), _np(ns.population.cell), _np(ns.population.types)
    rng = np.random.default_rng(5)
    for r in range(P):
        n = case["Ns"][r]
        mu = None if case["mus"] is None else case["mus"][r]
        for k in rng.choice(K, sample, replace=False):
            e = O.energy(case["model"], X[r, k, :n], Ty[r, k, :n], C_[r, k],
                         pressure=float(case["pressures"][r]), mu=mu, mode=O.DEV,
                         forces=False)[0]
            assert abs(E[r, k] - e) <= 1e-12 * max(1.0, abs(e)), (r, k, E[r, k], e)
            assert np.all((Ty[r, k, :n] >= 0) & (Ty[r, k, :n] < case["H"].model.n_species))


def test_batched_lj32_configuration_full_size():
    case = lj_case(P=8, K=512, N=32, seed=2024, n_reflect=10, T=40,
                   pressure=np.logspace(-2, 0, 8).astype(np.float32))
    ns, info, swaps = _walk(case, n_launch=12, n_iter=10, re_every=10)
    _check(case, ns, info, swaps)


def test_uneven_semigrand_configuration_full_size():
    Ns = [int(v) for v in np.random.default_rng(96).choice(np.arange(16, 97, 8), 16)]
    dmu = np.concatenate([-np.logspace(np.log10(2.0), -2, 8), np.logspace(-2, np.log10(2.0), 8)])
    mu = np.stack([np.zeros(16), dmu], axis=1)
    case = lj_case(P=16, K=1024, N=max(Ns), seed=2025, n_reflect=10, T=40, n_atoms_list=Ns,
                   identity="both", mu=mu, epsilon=[[1.0, 1.5], [1.5, 0.5]],
                   sigma=[[1.0, 0.8], [0.8, 0.88]])
    ns, info, _ = _walk(case, n_launch=4, n_iter=10)
    _check(case, ns, info, [], sample=6)


def test_nan_energy_population_matches_oracle():
    """One walker with two coincident atoms has a NaN energy: the contour is
    NaN (jnp.max propagates it), no walker equals it, walker 0 is culled,
    every E < NaN test fails, so every proposal of the iteration is rejected
    and log Z turns NaN -- on the GPU exactly as in the oracle."""
    case = lj_case(P=2, K=16, N=8, seed=31, n_reflect=3, T=4, pressure=np.array([0.1, 0.2]))
    x = case["positions"][0]
    x[5, 3] = x[5, 1]  # coincident atoms: r = 0
    e = O.energy(case["model"], x[5], case["types"][0][5], case["cells"][0][5],
                 pressure=0.1, forces=False)[0]
    assert np.isnan(e)
    case["energies"][0][5] = e
    ns = _init(case)
    infos = [nsm.ns_iterate(ns, case["step"], 3, case["T"], 0)]
    torch.cuda.synchronize()
    reps = oracle_replicas(case)
    la = prior_mass.log_alpha(16, 1)
    wo = float(prior_mass.iteration_offsets(16, 1)[1][0])
    hist = [O.ns_step_batched(case["model"], case["moves"], reps, case["T"], la, wo,
                              shared_move_key=True) for _ in range(3)]
    em = _np(infos[0].emax)
    w = _np(infos[0].worst_idx)
    acc = _np(infos[0].n_accepted)
    for t in range(3):
        assert np.isnan(em[t, 0]) and np.isfinite(em[t, 1])
        assert w[t, 0] == hist[t][0].worst_idx == 0
        assert acc[t, 0].sum() == 0
        assert w[t, 1] == hist[t][1].worst_idx
    assert np.isnan(_np(ns.log_evidence)[0])
    X = _np(ns.population.positions)
    E = _np(ns.population.energy64)
    for r, rep in enumerate(reps):
        np.testing.assert_array_equal(X[r], rep.positions)
        np.testing.assert_allclose(E[r], rep.energy, rtol=1e-12, equal_nan=True)
    np.testing.assert_array_equal(_np(ns.rng_key).view(np.uint32),
                                  np.stack([rp.rng_key for rp in reps]))
