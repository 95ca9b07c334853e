"""jr_ns_iterate_static vs jr_ns_iterate (B200), through the C ABI.

The allocation-free entry runs on the library's static device scratch; the
workspace entry on a caller-allocated workspace.  Started from identical
states, two calls in a row of each must leave identical walkers and report
identical per-iteration info (float64 energies and log Z to 1e-12 relative,
everything else exactly).  Batched runs are used because they read replica
0's key snapshot, the one thing the scratch holds.
"""

import ctypes as C

import numpy as np
import pytest

from jaxrens_b200 import _lib, prior_mass
from jaxrens_b200 import nested_sampling as nsm
from tests._cases import lj_case

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

RTOL = 1e-12


def _init(case):
    return nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                case["energies"], case["cells"], case["run_keys"],
                                ensemble_params={"pressure": case["pressures"],
                                                 "chemical_potentials": case["mus"]})


def _call(ns, step, n_iter, T, n_extra, static):
    K = ns.n_walkers
    la = prior_mass.log_alpha(K, 1)
    _, w_off = prior_mass.iteration_offsets(K, 1)
    params = step.with_evidence(la, float(w_off[0]))
    dims = nsm.make_dims(ns, step, T, n_extra, 1)
    info = nsm.InfoBuffers(ns, step.n_moves, n_iter)
    sb = nsm.state_buffers(ns)
    ib = info.cstruct()
    stream = torch.cuda.current_stream().cuda_stream
    L = _lib.load()
    if static:
        rc = L.jr_ns_iterate_static(C.byref(dims), C.byref(params), C.byref(sb), C.byref(ib),
                                    int(n_iter), None, stream)
        _lib.check(rc, "jr_ns_iterate_static")
    else:
        ws = torch.zeros(L.jr_ns_iterate_workspace_size(C.byref(dims)), dtype=torch.uint8,
                         device="cuda")
        rc = L.jr_ns_iterate(C.byref(dims), C.byref(params), C.byref(sb), C.byref(ib),
                             int(n_iter), None, ws.data_ptr(), ws.numel(), stream)
        _lib.check(rc, "jr_ns_iterate")
    torch.cuda.synchronize()
    return info


def _np(t):
    return t.detach().cpu().numpy()


def _same_state(a, b):
    for name in ("positions", "direction", "types", "cell", "n_accepted", "n_proposed"):
        np.testing.assert_array_equal(_np(getattr(a.population, name)),
                                      _np(getattr(b.population, name)), err_msg=name)
    np.testing.assert_allclose(_np(a.population.energy64), _np(b.population.energy64),
                               rtol=RTOL, atol=0)
    np.testing.assert_array_equal(_np(a.rng_key), _np(b.rng_key))
    np.testing.assert_array_equal(_np(a.iteration), _np(b.iteration))
    np.testing.assert_allclose(_np(a.log_evidence), _np(b.log_evidence), rtol=RTOL, atol=0)
    np.testing.assert_allclose(_np(a.emax), _np(b.emax), rtol=RTOL, atol=0)


def _same_info(a, b):
    for name in ("worst_idx", "clone_idx", "n_accepted", "n_proposed", "reject_reason_counts",
                 "n_evaluations", "n_grad_evaluations"):
        np.testing.assert_array_equal(_np(getattr(a, name)), _np(getattr(b, name)),
                                      err_msg=name)
    np.testing.assert_allclose(_np(a.emax), _np(b.emax), rtol=RTOL, atol=0)
    np.testing.assert_allclose(_np(a.log_evidence), _np(b.log_evidence), rtol=RTOL, atol=0)


@pytest.mark.parametrize("n_extra", [0, 2])
def test_static_scratch_entry_matches_workspace_entry(n_extra):
    case = lj_case(P=3, K=24, N=12, seed=21, n_reflect=3, T=4,
                   pressure=np.array([0.05, 0.1, 0.3]))
    ref = _init(case)
    got = _init(case)
    for _ in range(2):  # two calls in a row on each path
        ia = _call(ref, case["step"], 7, 4, n_extra, static=False)
        ib = _call(got, case["step"], 7, 4, n_extra, static=True)
        _same_info(ia, ib)
        _same_state(ref, got)
    assert int(_np(got.iteration)[0]) == 14


def test_static_scratch_entry_rejects_invalid_dims():
    case = lj_case(P=2, K=16, N=8, seed=22, n_reflect=2, T=2,
                   pressure=np.array([0.1, 0.2]))
    ns = _init(case)
    dims = nsm.make_dims(ns, case["step"], 2, 0, 1)
    dims.n_cull = 0
    params = case["step"].with_evidence(prior_mass.log_alpha(16, 1), 0.0)
    rc = _lib.load().jr_ns_iterate_static(C.byref(dims), C.byref(params),
                                          C.byref(nsm.state_buffers(ns)), None, 1, None,
                                          torch.cuda.current_stream().cuda_stream)
    assert _lib.ERRORS[rc] == "JR_ERR_SHAPE"
    assert b"n_cull" in _lib.load().jr_last_error()
