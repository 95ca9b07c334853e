"""ns_step with the caller's move-schedule key (B200).

The reference's batcher derives one move key outside its run ``vmap`` and
passes it to every replica's ``ns_step`` (``sampling/batch_descriptor.py``
``_wrap_batched_step``); ``ns_step(move_key=...)`` takes it the same way.
Checked against the oracle's ``ns_step`` given the same key, over several
iterations with a different caller key each, and against the default batched
schedule when the caller passes the key that schedule derives itself.
"""

import numpy as np
import pytest

from jaxrens_b200 import prior_mass, prng
from jaxrens_b200 import nested_sampling as nsm
from oracle import oracle as O
from tests._cases import lj_case, oracle_replicas
from tests.test_gpu_parity import _np

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _init(case):
    return nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                case["energies"], case["cells"], case["run_keys"],
                                ensemble_params={"pressure": case["pressures"]})


def test_explicit_move_key_matches_oracle():
    case = lj_case(P=3, K=20, N=8, seed=31, n_reflect=3, T=5)
    ns = _init(case)
    reps = oracle_replicas(case)
    K = case["K"]
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    for i in range(5):
        mk = prng.fold_in(prng.key(777), i)
        ns, info = nsm.ns_step(ns, case["step"], 5, 0, move_key=mk)
        for r, rep in enumerate(reps):
            oi = O.ns_step(case["model"], case["moves"], rep, 5, la, wo, move_key=mk)[0]
            assert int(_np(info["worst_idx"])[r]) == oi.worst_idx
            np.testing.assert_array_equal(_np(info["n_accepted_per_move"])[r],
                                          list(oi.n_acc)[: case["step"].n_moves])
    torch.cuda.synchronize()
    X = _np(ns.population.positions)
    E = _np(ns.population.energy64)
    for r, rep in enumerate(reps):
        np.testing.assert_array_equal(X[r], rep.positions)
        np.testing.assert_allclose(E[r], rep.energy, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(_np(ns.rng_key).view(np.uint32)[r], rep.rng_key)


def test_explicit_key_equal_to_the_derived_one_reproduces_the_batched_schedule():
    case = lj_case(P=2, K=16, N=8, seed=32, n_reflect=2, T=4)
    a, b = _init(case), _init(case)
    for _ in range(3):
        k0 = _np(a.rng_key).view(np.uint32)[0].copy()
        nsm.ns_step(a, case["step"], 4, 0, move_key=prng.fold_in(k0, 1))
        nsm.ns_step(b, case["step"], 4, 0)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(a.population.positions), _np(b.population.positions))
    np.testing.assert_array_equal(_np(a.rng_key), _np(b.rng_key))
