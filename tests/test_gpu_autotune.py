"""The project-written autotuner (``jr_autotune``) on the GPU.

It times candidate launch shapes on copies of the caller's state (every
candidate restored to the same pristine copy before each timed launch, the
median of three launches scored) and caches the winner for the dims.  The
checks: the caller's state is untouched; the chosen shape is a valid
configuration that a launch accepts; the next launch without an explicit
shape (which takes the cached one) and launches with the heuristic shape give
identical walkers, since results do not depend on the launch shape.
"""

import ctypes as C

import numpy as np
import pytest

from jaxrens_b200 import _lib, prior_mass
from jaxrens_b200 import nested_sampling as nsm
from tests._cases import lj_case
from tests.test_gpu_parity import _np, _run_gpu

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _tune(ns, step, T, n_iter):
    K = ns.n_walkers
    dims = nsm.make_dims(ns, step, T, 0)
    params = step.with_evidence(prior_mass.log_alpha(K, 1),
                                prior_mass.iteration_offsets(K, 1)[1])
    sb = nsm.state_buffers(ns)
    best = _lib.JrLaunchConfig()
    rc = _lib.load().jr_autotune(C.byref(dims), C.byref(params), C.byref(sb), n_iter,
                                 C.byref(best), torch.cuda.current_stream().cuda_stream)
    _lib.check(rc, "jr_autotune")
    torch.cuda.synchronize()
    return best


def _snapshot(ns):
    pop = ns.population
    return [_np(t).copy() for t in (pop.positions, pop.direction, pop.energy64, pop.cell,
                                    pop.n_accepted, ns.rng_key, ns.iteration, ns.log_evidence)]


@pytest.mark.parametrize("N,P", [(8, 2), (32, 3)])
def test_autotune_picks_a_valid_cached_shape_without_touching_the_state(N, P):
    case = lj_case(P=P, K=48, N=N, seed=40 + N, n_reflect=3, T=4)
    ns, _ = _run_gpu(case, 2, 4)
    before = _snapshot(ns)
    best = _tune(ns, case["step"], 4, 6)
    for a, b in zip(before, _snapshot(ns)):
        np.testing.assert_array_equal(a, b)
    assert best.threads in (32, 64, 128, 256, 512) and best.cluster >= 1
    assert best.tpa >= 1 and (best.tpa & (best.tpa - 1)) == 0
    # three ways to walk the same 6 iterations: the cached tuned shape (no
    # explicit shape), the tuned shape given explicitly, the heuristic shape
    heur = _lib.JrLaunchConfig(256 if N > 16 else 128, 8, 1, 0)
    outs = []
    for cfg in (None, best, heur):
        case_ns, _ = _run_gpu(case, 2, 4)
        nsm.ns_iterate(case_ns, case["step"], 6, 4, 0, cfg=cfg)
        torch.cuda.synchronize()
        outs.append(_snapshot(case_ns))
    for other in outs[1:]:
        for a, b in zip(outs[0], other):
            np.testing.assert_array_equal(a, b)
