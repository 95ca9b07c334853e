"""Burn-in and step-size adaptation on the B200 vs the CPU oracle.

``jr_walk_population`` (``init/burn_in.py`` ``_one_walk``) must leave every
walker exactly as the oracle's walk does; ``initial_walk`` with adaptation
(trial moves through ``jr_move_trial``) must choose the same step sizes and
end in the same state as the same driver fed by oracle trials and walks.
"""

import numpy as np
import pytest

from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200 import prng
from jaxrens_b200.adaptation import adjust_step_size
from jaxrens_b200.burn_in import initial_walk, walk_population
from oracle import oracle as O
from tests._cases import lj_case, oracle_replicas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _np(t):
    return t.detach().cpu().numpy()


def _init(case):
    if case["P"] > 1:
        return nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                    case["energies"], case["cells"], case["run_keys"],
                                    ensemble_params={"pressure": case["pressures"],
                                                     "chemical_potentials": case["mus"]})
    return nsm.init_ns(case["init_fn"], case["positions"][0], case["types"][0],
                       case["energies"][0], case["cells"][0], case["run_keys"][0],
                       ensemble_params={"pressure": float(case["pressures"][0])})


def _same(case, ns, reps):
    pop = ns.population
    for r, rep in enumerate(reps):
        n = case["Ns"][r]
        np.testing.assert_array_equal(_np(pop.positions)[r, :, :n], rep.positions)
        np.testing.assert_array_equal(_np(pop.direction)[r, :, :n], rep.direction)
        np.testing.assert_array_equal(_np(pop.cell)[r], rep.cell)
        np.testing.assert_array_equal(_np(pop.types)[r, :, :n], rep.types)
        np.testing.assert_allclose(_np(pop.energy64)[r], rep.energy, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(_np(pop.n_accepted)[r], rep.n_acc)
        np.testing.assert_array_equal(_np(pop.n_proposed)[r], rep.n_prop)
        np.testing.assert_array_equal(_np(pop.step_sizes)[r], rep.step_sizes)


@pytest.mark.parametrize("P", [1, 3])
def test_walk_population_matches_oracle(P):
    case = lj_case(P=P, K=20, N=8, seed=50 + P, n_reflect=3, T=1,
                   pressure=np.linspace(0.05, 0.4, P))
    ns = _init(case)
    reps = oracle_replicas(case)
    emax = _np(ns.population.energy64).max(axis=1) + 0.5 * 8
    run_keys = prng.split(prng.key(7), P)
    move_key = prng.key(8)
    walk_population(ns, case["step"], 6, run_keys, move_key, emax)
    torch.cuda.synchronize()
    for r, rep in enumerate(reps):
        O.walk_population(case["model"], case["moves"], rep, 6, run_keys[r], move_key, emax[r])
    _same(case, ns, reps)


def _oracle_initial_walk(case, reps, key, n_walks, walklength, adjust_interval, offset,
                         n_atoms, n_samples, max_rounds):
    """The burn-in driver of init/burn_in.py:151-460 on oracle replicas."""
    P = len(reps)
    step = case["step"]
    emax = np.array([r.energy.max() for r in reps]) + offset * n_atoms
    key = np.asarray(key, np.uint32)
    for walk_i in range(n_walks):
        if walk_i % adjust_interval == 0:
            key, key_adapt = prng.split(key, 2)
            adapt_key = prng.split(key_adapt, P) if P > 1 else key_adapt[None, :]
            ss = np.stack([r.step_sizes[0] for r in reps]).astype(np.float32)
            for m, desc in enumerate(step.move_descriptors):
                pairs = np.stack([prng.split(adapt_key[p], 2) for p in range(P)])
                adapt_key, key_adjust = pairs[:, 0].copy(), pairs[:, 1].copy()

                def trial(widx, tkeys, s, e, m=m):
                    acc = np.zeros(widx.shape, np.int32)
                    why = np.zeros(widx.shape, np.int32)
                    for p, rep in enumerate(reps):
                        for j, w in enumerate(widx[p]):
                            a, *_, reason = O.move_trial(
                                case["model"], case["moves"], m, tkeys[p, j], float(s[p]),
                                float(e[p]), rep.positions[w], rep.direction[w],
                                rep.types[w], rep.cell[w], float(rep.energy[w]),
                                pressure=float(rep.pressure))
                            acc[p, j] = a
                            why[p, j] = 0 if a else (reason if reason > 1 else 1)
                    return acc, why

                res = adjust_step_size(trial, len(reps[0].energy), ss[:, m], emax, key_adjust,
                                       n_samples, desc.min_rate, desc.max_rate, 1.5,
                                       desc.step_size_max, max_rounds)
                ss[:, m] = res.step_size
            for p, rep in enumerate(reps):
                rep.step_sizes[:] = ss[p][None, :]
        key, sub, move_key = prng.split(key, 3)
        run_keys = prng.split(sub, P) if P > 1 else sub[None, :]
        for p, rep in enumerate(reps):
            O.walk_population(case["model"], case["moves"], rep, walklength, run_keys[p],
                              move_key, emax[p])


@pytest.mark.parametrize("P", [1, 2])
def test_initial_walk_with_adaptation_matches_oracle(P):
    case = lj_case(P=P, K=16, N=6, seed=60 + P, n_reflect=2, T=1,
                   pressure=np.linspace(0.1, 0.3, P))
    ns = _init(case)
    reps = oracle_replicas(case)
    key = prng.key(11)
    kw = dict(n_walks=3, walklength=4, adjust_interval=2, emax_offset_per_atom=0.3, n_atoms=6)
    ns, diags = initial_walk(key, ns, case["step"], adjust_n_samples=12, adjust_max_rounds=4,
                             **kw)
    torch.cuda.synchronize()
    _oracle_initial_walk(case, reps, key, 3, 4, 2, 0.3, 6, 12, 4)
    assert len(diags) == 2 and all(len(d) == case["step"].n_moves for d in diags)
    _same(case, ns, reps)
