"""Stillinger-Weber walk on the GPU against the CPU oracle (B200).

The kernels follow the oracle's DEV contract: forces bit for bit, energies to
1e-12 relative (the float64 sum of float32 terms near the cutoff depends on
its order), against float64 within 1e-5; NS iterations walker for walker and
counter for counter, as the LJ parity tests check.
"""

import numpy as np
import pytest

from jaxrens_b200 import EnsembleTerm, Hamiltonian, create_sw
from jaxrens_b200.backends import EV_PER_A3_PER_GPA
from oracle import oracle as O
from tests._cases import lj_case, oracle_model
from tests.test_gpu_parity import _compare, _np, _run_gpu, _run_oracle
from tests.test_oracle_sw import diamond

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")

P_SI = 0.1 * EV_PER_A3_PER_GPA


def _configs(rng, B, N, L, triclinic=False):
    pos = (rng.uniform(0, 1, (B, N, 3)) * L).astype(np.float32)
    cell = np.tile(np.eye(3, dtype=np.float32) * L, (B, 1, 1))
    if triclinic:
        cell = cell + (rng.uniform(-0.6, 0.6, (B, 3, 3)) * (1 - np.eye(3))).astype(np.float32)
    return pos, cell.astype(np.float32)


@pytest.mark.parametrize("N,vpa,tric", [(8, 12.0, False), (17, 20.0, True), (33, 16.0, False),
                                        (64, 20.0, False), (64, 9.0, True), (64, 40.0, True)])
def test_sw_energy_forces_vs_oracle(N, vpa, tric):
    rng = np.random.default_rng(N * 7 + int(vpa))
    H = Hamiltonian(create_sw(), [EnsembleTerm(pressure=P_SI)])
    B = 12
    pos, cell = _configs(rng, B, N, (vpa * N) ** (1.0 / 3.0), triclinic=tric)
    types = np.zeros((B, N), np.int32)
    res = H.energy_and_forces(pos, types, cell)
    E, F = _np(res.energy), _np(res.forces)
    m = oracle_model(H)
    for b in range(B):
        e_o, f_o, _ = O.energy(m, pos[b], types[b], cell[b], pressure=P_SI, mode=O.DEV)
        assert abs(E[b] - e_o) <= 1e-12 * max(1.0, abs(e_o)), (b, E[b], e_o)
        np.testing.assert_array_equal(F[b], f_o.astype(np.float32))
        e64, f64, _ = O.energy(m, pos[b], types[b], cell[b], pressure=P_SI, mode=O.F64)
        assert abs(E[b] - e64) <= 1e-5 * max(1.0, abs(e64))
        assert np.abs(F[b] - f64).max() <= 1e-5 * max(1.0, np.abs(f64).max())


def test_sw_diamond_silicon_on_gpu():
    x, cell = diamond(2)
    res = create_sw().energy_and_forces(x, np.zeros(64, np.int32), cell)
    assert abs(float(_np(res.energy)) / 64 + 2.0 * 2.1683) < 1e-4
    assert np.abs(_np(res.forces)).max() < 2e-3


def _sw_case(P, K, N, seed, T, R, vpa, pressure=P_SI):
    return lj_case(P=P, K=K, N=N, seed=seed, n_reflect=R, T=T, pressure=pressure,
                   v_hi_per_atom=vpa, step_sizes=(0.3, 2.0), backend=create_sw())


def test_sw_single_run_matches_oracle():
    case = _sw_case(P=1, K=16, N=8, seed=21, T=4, R=3, vpa=25.0)
    ns, infos = _run_gpu(case, 12, 4, chunk=5)
    reps, hist = _run_oracle(case, 12, 4)
    _compare(case, ns, infos, reps, hist)


def test_sw_batched_64_atoms_matches_oracle():
    """The batched Stillinger-Weber shape: 64-atom silicon walkers, runs at
    two pressures, speculative iterations (the default launch covers them)."""
    case = _sw_case(P=2, K=12, N=64, seed=22, T=3, R=2, vpa=30.0,
                    pressure=np.array([P_SI, 3 * P_SI]))
    ns, infos = _run_gpu(case, 6, 3)
    reps, hist = _run_oracle(case, 6, 3)
    _compare(case, ns, infos, reps, hist)
    # the work counters of the iterations: every step evaluates the energy
    # (at most n(n-1)/2 pairs each); forces are evaluated only on the
    # galilean steps that reflect, at most once per counted evaluation
    tc = np.concatenate([_np(i.term_counts) for i in infos])
    ne = np.concatenate([_np(i.n_evaluations).sum(-1) for i in infos])
    ng = np.concatenate([_np(i.n_grad_evaluations).sum(-1) for i in infos])
    assert (tc[..., 2] > 0).all() and (tc[..., 2] <= ne * 64 * 63 // 2).all()
    assert (tc[..., 0] <= ng * 64 * 63 // 2).all()
    assert (tc[..., 1] <= ng * 64 * 63 * 62).all() and (tc[..., 3] >= 0).all()


def test_sw_launch_shapes_agree():
    """Results do not depend on the launch shape (CTA size, cluster)."""
    from jaxrens_b200 import _lib

    case = _sw_case(P=2, K=16, N=24, seed=23, T=3, R=3, vpa=25.0)
    ref_ns, _ = _run_gpu(case, 8, 3)
    for cfg in [_lib.JrLaunchConfig(128, 4, 1, 0), _lib.JrLaunchConfig(512, 16, 4, 0),
                _lib.JrLaunchConfig(256, 8, 8, 0)]:
        ns, _ = _run_gpu(case, 8, 3, cfg=cfg)
        np.testing.assert_array_equal(_np(ns.population.positions), _np(ref_ns.population.positions))
        np.testing.assert_allclose(_np(ns.population.energy64), _np(ref_ns.population.energy64),
                                   rtol=1e-12, atol=0)
