"""Statistical parity on the B200: log Z and C_v against independent runs.

* Gaussian-mixture toy (backends/toy.py:163-204): the evidence of GPU runs
  matches the analytic log Z on its uniform prior cube.
* LJ8 NPT: an ensemble of GPU runs and an ensemble of runs of the oracle in
  the reference's float32 arithmetic (independent seeds) give the same log Z
  and the same heat-capacity peak temperature within statistical error.
* LJ-32 NPT at the bench shape (8 runs x 512 walkers, n_mcmc_steps 40, 10
  reflections): GPU and oracle ensembles give the same log Z after 6000
  iterations (prior mass about 1e-5), so the throughput is measured at
  matched log Z.
* LJ-32 on the bench's pressure ladder with replica exchange every 10
  iterations, 16 seeds per arm: per pressure, log Z and the seed-mean contour
  energy at fixed log X along the run agree with the oracle in the
  reference's float32 arithmetic.
"""

import numpy as np
import pytest

from jaxrens_b200 import GaussianMixtureBackend, build_mwg, prior_mass, prng, thermo
from jaxrens_b200 import moves as mvs
from jaxrens_b200 import nested_sampling as nsm
from oracle import oracle as O
from tests._cases import lj_case, oracle_replicas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _run_gpu(ns, step, n_iter, T, chunk=500):
    dead = []
    done = 0
    while done < n_iter:
        c = min(chunk, n_iter - done)
        info = nsm.ns_iterate(ns, step, c, T)
        dead.append(info.dead_energy.cpu().numpy())
        done += c
    torch.cuda.synchronize()
    return np.concatenate(dead, axis=0).T, ns.population.energy64.cpu().numpy()


def test_gaussian_mixture_log_evidence_is_analytic():
    g = GaussianMixtureBackend(centers=[[-1.0, 0.0, 0.0], [1.0, 0.0, 0.0]], sigma=0.5)
    h, K, P, T, n_iter = 3.0, 256, 4, 20, 2600
    init_fn, step, _ = build_mwg(g, [mvs.gmc(n_reflect=4, step_size=0.1, weight=1.0)])
    keys = prng.split(prng.key(31), P + 1)
    pos = [prng.uniform(keys[r], K * 3).reshape(K, 1, 3) * np.float32(2 * h) - np.float32(h)
           for r in range(P)]
    ns = nsm.init_ns_parallel(init_fn, pos, [np.zeros((K, 1), np.int32)] * P, None,
                              [np.zeros((K, 3, 3), np.float32)] * P,
                              prng.split(keys[P], P))
    dead, live = _run_gpu(ns, step, n_iter, T)
    want = g.log_evidence(h)
    lz = np.array([thermo.log_evidence(dead[r], live[r], K) for r in range(P)])
    # the kernel's own accumulator plus the live share agrees with post-processing
    np.testing.assert_allclose(nsm.final_log_evidence(ns).cpu().numpy(), lz, rtol=0, atol=1e-8)
    assert np.all(np.abs(lz - want) < 0.5), (lz, want)
    assert abs(lz.mean() - want) < 0.3, (lz, want)


def _cv_peak(dead, live, K, n_atoms):
    temps = np.linspace(0.05, 2.0, 196)
    return thermo.cv_peak_temperature(temps, dead, live, K, 1, n_atoms)


def test_lj8_npt_log_z_and_cv_peak_match_reference_arithmetic():
    P, K, N, T, n_iter = 8, 64, 8, 8, 2000
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    gcase = lj_case(P=P, K=K, N=N, seed=100, n_reflect=4, T=T, pressure=0.1)
    ns = nsm.init_ns_parallel(gcase["init_fn"], gcase["positions"], gcase["types"],
                              gcase["energies"], gcase["cells"], gcase["run_keys"],
                              ensemble_params={"pressure": gcase["pressures"]})
    dead_g, live_g = _run_gpu(ns, gcase["step"], n_iter, T)
    rcase = lj_case(P=P, K=K, N=N, seed=200, n_reflect=4, T=T, pressure=0.1)
    reps = oracle_replicas(rcase)
    dead_r = np.zeros((P, n_iter))
    for it in range(n_iter):
        infos = O.ns_step_batched(rcase["model"], rcase["moves"], reps, T, la, wo,
                                  shared_move_key=True, mode=O.REF32, n_threads=8)
        dead_r[:, it] = [i.dead_energy for i in infos]
    live_r = np.stack([r.energy for r in reps])
    lz_g = np.array([thermo.log_evidence(dead_g[r], live_g[r], K) for r in range(P)])
    lz_r = np.array([thermo.log_evidence(dead_r[r], live_r[r], K) for r in range(P)])
    se = np.sqrt(lz_g.var(ddof=1) / P + lz_r.var(ddof=1) / P)
    assert abs(lz_g.mean() - lz_r.mean()) < 4 * se + 0.05, (lz_g, lz_r)
    tg = np.array([_cv_peak(dead_g[r], live_g[r], K, N) for r in range(P)])
    tr = np.array([_cv_peak(dead_r[r], live_r[r], K, N) for r in range(P)])
    se_t = np.sqrt(tg.var(ddof=1) / P + tr.var(ddof=1) / P)
    assert abs(tg.mean() - tr.mean()) < 4 * se_t + 0.03, (tg, tr)


def test_lj32_npt_bench_shape_log_z_matches_reference_arithmetic():
    """Matched log Z at the bench shape: 8 runs x 512 walkers of 32-atom LJ
    NPT at one pressure (so the runs form one seed ensemble), n_mcmc_steps 40,
    10 reflections, 6000 iterations (prior mass exp(-6000/512), about 1e-5).
    The GPU ensemble and an independent ensemble of oracle runs in the
    reference's float32 arithmetic give the same log Z (dead points plus live
    walkers) and the same final contour within statistical error."""
    P, K, N, T, n_iter = 8, 512, 32, 40, 6000
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    gcase = lj_case(P=P, K=K, N=N, seed=300, n_reflect=10, T=T, pressure=0.1)
    ns = nsm.init_ns_parallel(gcase["init_fn"], gcase["positions"], gcase["types"],
                              gcase["energies"], gcase["cells"], gcase["run_keys"],
                              ensemble_params={"pressure": gcase["pressures"]})
    dead_g, live_g = _run_gpu(ns, gcase["step"], n_iter, T)
    rcase = lj_case(P=P, K=K, N=N, seed=400, n_reflect=10, T=T, pressure=0.1)
    reps = oracle_replicas(rcase)
    dead_r = np.zeros((P, n_iter))
    for it in range(n_iter):
        infos = O.ns_step_batched(rcase["model"], rcase["moves"], reps, T, la, wo,
                                  shared_move_key=True, mode=O.REF32, n_threads=8)
        dead_r[:, it] = [i.dead_energy for i in infos]
    live_r = np.stack([r.energy for r in reps])
    lz_g = np.array([thermo.log_evidence(dead_g[r], live_g[r], K) for r in range(P)])
    lz_r = np.array([thermo.log_evidence(dead_r[r], live_r[r], K) for r in range(P)])
    se = np.sqrt(lz_g.var(ddof=1) / P + lz_r.var(ddof=1) / P)
    print("log Z GPU %.4f +- %.4f, oracle %.4f +- %.4f" %
          (lz_g.mean(), lz_g.std(ddof=1), lz_r.mean(), lz_r.std(ddof=1)))
    assert abs(lz_g.mean() - lz_r.mean()) < 4 * se + 0.05, (lz_g, lz_r)
    eg, er = dead_g[:, -1], dead_r[:, -1]
    se_e = np.sqrt(eg.var(ddof=1) / P + er.var(ddof=1) / P)
    print("final contour GPU %.4f +- %.4f, oracle %.4f +- %.4f" %
          (eg.mean(), eg.std(ddof=1), er.mean(), er.std(ddof=1)))
    assert abs(eg.mean() - er.mean()) < 4 * se_e + 1e-3 * abs(er.mean()), (eg, er)


def test_lj32_pressure_ladder_with_replica_exchange_matches_reference_arithmetic():
    """The bench's pressure ladder (8 runs at pressures log-spaced over
    0.01-1.0, replica exchange every 10 iterations) with 16 independent seeds
    per arm: the GPU walk and the oracle in the reference's float32
    arithmetic.  Compared per pressure: log Z, and the low-variance statistic
    of the seed-mean contour energy at fixed log X (every 100 iterations
    along the run), each within 4 standard errors.  128 walkers of 32 atoms,
    n_mcmc_steps 20, 10 reflections, 1500 iterations (log X = -11.7)."""
    S, P, K, N, T, R, n_iter, every = 16, 8, 128, 32, 20, 10, 1500, 10
    pressures = np.logspace(-2, 0, P).astype(np.float32)
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    dead = {"gpu": np.zeros((S, P, n_iter)), "ref": np.zeros((S, P, n_iter))}
    lz = {"gpu": np.zeros((S, P)), "ref": np.zeros((S, P))}
    for s in range(S):
        c = lj_case(P=P, K=K, N=N, seed=1000 + s, n_reflect=R, T=T, pressure=pressures)
        ns = nsm.init_ns_parallel(c["init_fn"], c["positions"], c["types"], c["energies"],
                                  c["cells"], c["run_keys"],
                                  ensemble_params={"pressure": c["pressures"]})
        re = nsm.InterREManager(every, 1, prng.fold_in(prng.key(1000 + s), 5))
        rows = []
        for _ in range(n_iter // every):
            info = nsm.ns_iterate(ns, c["step"], every, T)
            rows.append(info.dead_energy.cpu().numpy())
            re.apply(ns, c["step"])
        dead["gpu"][s] = np.concatenate(rows, axis=0).T
        live = ns.population.energy64.cpu().numpy()
        lz["gpu"][s] = [thermo.log_evidence(dead["gpu"][s, r], live[r], K) for r in range(P)]
        c = lj_case(P=P, K=K, N=N, seed=2000 + s, n_reflect=R, T=T, pressure=pressures)
        reps = oracle_replicas(c)
        re = nsm.InterREManager(every, 1, prng.fold_in(prng.key(2000 + s), 5))
        for it in range(n_iter):
            infos = O.ns_step_batched(c["model"], c["moves"], reps, T, la, wo,
                                      shared_move_key=True, mode=O.REF32, n_threads=8)
            dead["ref"][s, :, it] = [i.dead_energy for i in infos]
            if (it + 1) % every == 0:
                O.re_step(reps, re.next_swap_key(), 1, mode=O.REF32)
        lz["ref"][s] = [thermo.log_evidence(dead["ref"][s, r], reps[r].energy, K)
                        for r in range(P)]
    for r in range(P):
        a, b = lz["gpu"][:, r], lz["ref"][:, r]
        se = np.sqrt(a.var(ddof=1) / S + b.var(ddof=1) / S)
        assert abs(a.mean() - b.mean()) < 4 * se + 0.05, (r, a, b)
        for it in range(every * 10 - 1, n_iter, 100):
            a, b = dead["gpu"][:, r, it], dead["ref"][:, r, it]
            se = np.sqrt(a.var(ddof=1) / S + b.var(ddof=1) / S)
            assert abs(a.mean() - b.mean()) < 4 * se + 1e-6 * abs(b.mean()), (r, it, a, b)
