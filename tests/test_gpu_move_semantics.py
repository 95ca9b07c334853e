"""The reference's own property tests of the walk, on the B200 (C ABI).

* Persistent-direction GMC keeps a uniform ensemble inside a harmonic contour
  uniform (``tests/sampling/moves/test_moves.py:414-453``): 8000 one-atom
  walkers of the one-centre Gaussian-mixture well (a 3-D harmonic well) walk
  100 galilean steps each through ``jr_walk_population`` at the fixed contour
  ``|x| = 1``; ``<r^2>`` stays 3/5, and every walker ends exactly where the
  oracle's walk in the kernel's arithmetic leaves it.
* The semi-grand swap re-bases the stored ``U - mu . N`` to the receiving
  run (``tests/sampling/replica_exchange/test_semigrand.py:102-140``), through
  ``jr_re_swap``, with the reference's hand-calculated 5.0 and 1.0.
"""

import numpy as np
import pytest

from jaxrens_b200 import Hamiltonian, EnsembleTerm, build_mwg, prng
from jaxrens_b200 import moves as mvs
from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200.burn_in import walk_population
from oracle import oracle as O
from tests.test_oracle_move_semantics import (E_CONST, _semigrand_replicas, harmonic_case,
                                              harmonic_energy, uniform_ball, walk_uniform_ball)

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _np(t):
    return t.detach().cpu().numpy()


def test_uniform_ball_invariant_and_oracle_parity():
    n, seed, calls = 8000, 0, 100
    g = harmonic_case(0.15, 4)[0]
    init_fn, step, _ = build_mwg(g, [mvs.gmc(n_reflect=4, step_size=0.15, weight=1.0)])
    x, v = uniform_ball(n, seed)
    e = np.array([harmonic_energy(p) for p in x])
    ns = nsm.init_ns(init_fn, x, np.zeros((n, 1), np.int32), e, np.zeros((n, 3, 3), np.float32),
                     prng.key(seed))
    ns.population.direction.copy_(torch.as_tensor(v).reshape(ns.population.direction.shape))
    keys = prng.split(prng.key(seed + 1), 2)
    walk_population(ns, step, calls, keys[0][None], keys[1], E_CONST + 0.5)
    torch.cuda.synchronize()
    X = _np(ns.population.positions)[0]
    r2 = np.sum(X.astype(np.float64) ** 2, axis=(1, 2))
    assert np.all(r2 < 1.0 + 1e-6)
    assert abs(r2.mean() - 0.6) < 0.009, r2.mean()
    rep, _ = walk_uniform_ball(n, seed, calls, mode=O.DEV)
    np.testing.assert_array_equal(X, rep.positions)
    np.testing.assert_array_equal(_np(ns.population.direction)[0], rep.direction)
    np.testing.assert_array_equal(_np(ns.population.n_accepted)[0], rep.n_acc)
    np.testing.assert_allclose(_np(ns.population.energy64)[0], rep.energy, rtol=1e-12, atol=0)


def test_semigrand_swap_rebases_on_the_gpu():
    K = 4
    lj, (a, b), (xa, xb, ta, tb, sa, sb, mu_a, mu_b) = _semigrand_replicas(K)
    H = Hamiltonian(lj, [EnsembleTerm(pressure=0.0, chemical_potentials=[0.0, 0.0])])
    init_fn, step, _ = build_mwg(H, [mvs.gmc(n_reflect=2, step_size=0.1, weight=1.0),
                                     mvs.volume_move(3, step_size=0.1, weight=1.0)])
    cells = np.zeros((K, 3, 3), np.float32)
    ns = nsm.init_ns_parallel(init_fn, [xa, xb], [ta, tb], [sa, sb], [cells, cells],
                              prng.split(prng.key(3), 2),
                              ensemble_params={"pressure": np.zeros(2, np.float32),
                                               "chemical_potentials": np.array([mu_a, mu_b],
                                                                               np.float32)})
    ns.emax.fill_(10.0)
    re = nsm.InterREManager(10, 1, prng.key(0))
    swap_key = prng.split(prng.split(re.key, 2)[1], 2)[1]
    stats = re.apply(ns, step)
    torch.cuda.synchronize()
    assert int(_np(stats["n_accepted_per_pair"])[0]) == 1
    E = _np(ns.population.energy64)
    T = _np(ns.population.types)
    ia = np.flatnonzero(E[0] != 3.0)
    ib = np.flatnonzero(E[1] != 2.5)
    assert len(ia) == 1 and len(ib) == 1
    assert abs(E[0, ia[0]] - 5.0) < 1e-6 and abs(E[1, ib[0]] - 1.0) < 1e-6
    np.testing.assert_array_equal(T[0, ia[0]], tb[0])
    np.testing.assert_array_equal(T[1, ib[0]], ta[0])
    # the same pass on the oracle picks the same walkers
    O.re_step([a, b], swap_key, n_swap_cycles=1)
    np.testing.assert_allclose(E[0], a.energy, rtol=1e-12)
    np.testing.assert_allclose(E[1], b.energy, rtol=1e-12)
    np.testing.assert_array_equal(_np(ns.population.positions)[0], a.positions)
