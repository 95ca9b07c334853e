"""Accept decisions of the kernels' arithmetic against the reference's (CPU).

The CUDA walk follows the oracle's DEV contract (float32 terms, float64
sums); the reference evaluates in float32 in its own operation order, the
oracle's REF32 mode.  On identical walkers, keys and contours this test runs
galilean (one-step and four-step trajectories), volume, morph and swap trials
in both modes and checks:

- the proposal energies of the two modes differ by at most the stated
  margin, 4e-6 |E| (measured up to 1.9e-6 |E| on these states);
- every decision is the mode's own energy test, E_mode < Emax (the other
  tests -- cell, prior, identity draws -- never differ between the modes);
- therefore every flip of a one-step decision has |E - Emax| within the
  margin.  Contours are drawn both generically (a walker energy of the
  population) and near the threshold (Emax = E_REF32 (1 + delta), |delta| <=
  4e-6); the flip rates are reported on failure and recorded in the design
  notes;
- four-step galilean trajectories, whose intermediate reflections can also
  flip, flip on at most 2% of the generic contours.

The reference's own move tests: ``tests/sampling/moves/test_moves.py:358-510``.
"""

import numpy as np
import pytest

from oracle import oracle as O
from tests._cases import lj_case

MARGIN = 4e-6

CASES = {
    "npt": dict(P=1, K=40, N=16, seed=51, T=1, pressure=0.1, v_hi_per_atom=3.0),
    "semigrand": dict(P=1, K=40, N=16, seed=52, T=1, identity="both",
                      mu=np.array([[0.0, -0.5]]), epsilon=[[1.0, 1.5], [1.5, 0.5]],
                      sigma=[[1.0, 0.8], [0.8, 0.88]], v_hi_per_atom=3.0),
}


def _trial(c, k, m, key, emax, mode):
    return O.move_trial(c["model"], c["moves"], m, key, float(c["step"].default_step_sizes[m]),
                        emax, c["positions"][0][k], np.zeros_like(c["positions"][0][k]),
                        c["types"][0][k], c["cells"][0][k], c["energies"][0][k],
                        pressure=float(c["pressures"][0]),
                        mu=None if c["mus"] is None else c["mus"][0], mode=mode)


@pytest.mark.parametrize("name", sorted(CASES))
def test_decision_flips_lie_within_the_margin(name):
    c = lj_case(n_reflect=1, **CASES[name])
    rng = np.random.default_rng(3)
    M = c["step"].n_moves
    pop_e = np.asarray(c["energies"][0])
    stats = {"near": [0, 0], "generic": [0, 0]}  # [flips, decisions]
    for k in range(c["K"]):
        for m in range(M):
            key = O.fold_in(O.fold_in(O.key(7), k), m)
            probe = {mode: _trial(c, k, m, key, 1e300, mode) for mode in (O.DEV, O.REF32)}
            # without a contour the two modes take the same non-energy decisions
            assert probe[O.DEV][0] == probe[O.REF32][0], (k, m)
            assert probe[O.DEV][6] == probe[O.REF32][6], (k, m)
            if not probe[O.DEV][0]:
                continue
            e_dev, e_ref = probe[O.DEV][5], probe[O.REF32][5]
            assert abs(e_dev - e_ref) <= MARGIN * abs(e_ref), (k, m, e_dev, e_ref)
            contours = [("generic", float(rng.choice(pop_e)))]
            for _ in range(3):
                contours.append(("near", e_ref + rng.uniform(-MARGIN, MARGIN) * abs(e_ref)))
            for kind, emax in contours:
                a_dev = _trial(c, k, m, key, emax, O.DEV)[0]
                a_ref = _trial(c, k, m, key, emax, O.REF32)[0]
                assert a_dev == (e_dev < emax) and a_ref == (e_ref < emax), (k, m, kind)
                stats[kind][1] += 1
                if a_dev != a_ref:
                    stats[kind][0] += 1
                    assert abs(e_ref - emax) <= MARGIN * abs(e_ref), (k, m, kind, emax)
    assert stats["near"][1] > 100 and stats["generic"][1] > 40, stats
    assert stats["generic"][0] == 0, stats


def test_four_step_galilean_flips_are_rare():
    c = lj_case(n_reflect=4, **CASES["npt"])
    rng = np.random.default_rng(4)
    pop_e = np.asarray(c["energies"][0])
    flips = n = 0
    for k in range(c["K"]):
        key = O.fold_in(O.key(9), k)
        for emax in rng.choice(pop_e, 3):
            a_dev = _trial(c, k, 0, key, float(emax), O.DEV)[0]
            a_ref = _trial(c, k, 0, key, float(emax), O.REF32)[0]
            n += 1
            flips += int(a_dev != a_ref)
    assert flips <= 0.02 * n, (flips, n)
