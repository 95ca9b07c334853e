"""Bulk .energies writing from run_loop on the B200 vs the oracle's dead points."""

import numpy as np
import pytest

from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200 import prior_mass
from jaxrens_b200.energy_log import EnergyLogCallback, EnergyLogger
from oracle import oracle as O
from tests._cases import lj_case, oracle_replicas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


@pytest.mark.parametrize("n_cull", [1, 2])
def test_energies_files_match_oracle_dead_points(tmp_path, n_cull):
    P, K, T, n_iter = 2, 20, 3, 9
    case = lj_case(P=P, K=K, N=6, seed=70 + n_cull, n_reflect=2, T=T,
                   pressure=np.array([0.1, 0.4]))
    ns = nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                              case["energies"], case["cells"], case["run_keys"],
                              ensemble_params={"pressure": case["pressures"],
                                               "chemical_potentials": case["mus"]})
    paths = [tmp_path / f"r{r}.energies" for r in range(P)]
    cb = EnergyLogCallback(paths, K, n_cull, n_atoms=6)
    nsm.run_loop(ns, case["step"], T, 0, [nsm.IterationTermination(n_iter)], [cb],
                 n_cull=n_cull, check_interval=4)
    cb.close()
    reps = oracle_replicas(case)
    la = prior_mass.log_alpha(K, n_cull)
    wo = prior_mass.iteration_offsets(K, n_cull)[1]
    want = [[] for _ in range(P)]
    for it in range(n_iter):
        mk = O.fold_in(reps[0].rng_key, 1)
        for r, rep in enumerate(reps):
            _, _, _, de, _, _, dc = O.ns_step_n(case["model"], case["moves"], rep, T, la, wo,
                                                 n_cull, move_key=mk)
            for k in range(n_cull):
                vol = float(abs(np.linalg.det(dc[k])))
                want[r].append(f"{it} {float(np.float32(de[k])):.10e} {vol:.10e}")
    for r in range(P):
        lines = open(paths[r]).read().splitlines()
        assert lines[0] == f"{K} {n_cull} 0 0.0 6"
        assert lines[1:] == want[r]
        assert len(EnergyLogger.read(paths[r]).iterations) == n_iter * n_cull
