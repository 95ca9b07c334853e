"""Step-size adaptation host logic (CPU): the rate decision against the
cases of the reference's tests/sampling/adaptation/test_stepsize_handler.py
and the bisection loop with stand-in trial functions."""

import numpy as np
import pytest

from jaxrens_b200 import prng
from jaxrens_b200.adaptation import adjust_step_size, process_rate
from oracle import oracle as O

ARGS = (0.2, 0.7, 1.5, 10.0)   # min_rate, max_rate, adjust_factor, max_step_size


def test_within_window_converges():
    ss, conv, cap, floor, hi, lo = process_rate(0.4, 0.1, 0.1, -1.0, *ARGS)
    assert conv and ss == np.float32(0.1) and not (cap or floor or hi or lo)


def test_below_min_decreases_above_max_increases():
    ss, conv, _, _, hi, lo = process_rate(0.1, 1.0, 1.0, -1.0, *ARGS)
    assert not conv and ss < 1.0 and lo and not hi
    assert ss == np.float32(1.0) * np.float32(1.0 / 1.5)
    ss, conv, _, _, hi, lo = process_rate(0.9, 0.1, 0.1, -1.0, *ARGS)
    assert not conv and ss > 0.1 and hi and not lo


def test_cap_and_floor():
    ss, _, cap, floor, _, _ = process_rate(0.95, 9.0, 9.0, -1.0, *ARGS)
    assert ss == np.float32(10.0) and cap and not floor
    ss, _, cap, floor, _, lo = process_rate(0.01, 1e-20, 1e-20, -1.0, *ARGS)
    assert ss == np.float32(1e-7) and floor and not cap and lo


@pytest.mark.parametrize("rate,rate_prev,expected", [(0.8, 0.15, 0.3), (0.75, 0.05, 0.5)])
def test_bracket_keeps_the_closer_step_size(rate, rate_prev, expected):
    ss, conv, *_ = process_rate(rate, 0.5, 0.3, rate_prev, *ARGS)
    assert conv and ss == np.float32(expected)


def _stub_trial(rate_of_step):
    """Trial stand-in: accepts the first round(rate * n) samples."""
    def trial(widx, tkeys, step, emax):
        P, n = widx.shape
        acc = np.zeros((P, n), np.int32)
        for p in range(P):
            acc[p, : int(round(rate_of_step(float(step[p])) * n))] = 1
        return acc, np.where(acc == 1, 0, 1)
    return trial


def test_bisection_converges_bounded_and_caps():
    # rate falls with the step size: converges inside the window from a small step
    res = adjust_step_size(_stub_trial(lambda s: np.exp(-s)), 64, [0.01, 0.05],
                           [0.0, 0.0], prng.split(prng.key(1), 2), 50, 0.25, 0.65, 1.5,
                           10.0, 15)
    assert res.converged.all() and ((res.rate > 0.25) & (res.rate < 0.65)).all()
    assert (res.n_rounds <= 15).all() and (res.trial_n_evaluations == 50 * res.n_rounds).all()
    # everything accepted: the step grows to the cap and stops at max_rounds
    res = adjust_step_size(_stub_trial(lambda s: 1.0), 64, [1.0], [0.0],
                           prng.key(2)[None], 20, 0.25, 0.65, 1.5, 10.0, 8)
    assert res.n_rounds[0] == 8 and not res.converged[0]
    assert res.step_size[0] == np.float32(10.0) and res.cap_hits[0] > 0


def test_sampling_keys_follow_the_reference_split_order():
    seen = {}

    def trial(widx, tkeys, step, emax):
        seen.setdefault("w", widx.copy())
        seen.setdefault("k", tkeys.copy())
        return np.ones_like(widx), np.zeros_like(widx)

    k = prng.key(9)
    adjust_step_size(trial, 30, [0.1], [0.0], k[None], 7, 0.25, 0.65, 1.5, 10.0, 1)
    _, ks, kt = prng.split(k, 3)
    assert seen["w"][0, 0] == O.randint(ks, 0, 30)
    np.testing.assert_array_equal(seen["w"][0], prng.randint_array(ks, 7, 0, 30))
    np.testing.assert_array_equal(seen["k"][0], prng.split(kt, 7))
    assert (seen["w"] >= 0).all() and (seen["w"] < 30).all()
