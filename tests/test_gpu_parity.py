"""CUDA walk vs the CPU oracle on identical inputs and keys (B200).

The kernels follow the oracle's DEV contract (float32 pair terms with a fixed
FMA placement, float64 accumulation), so states are compared bit-for-bit:
positions, directions, cells, types, keys, culled/cloned indices and counters
exactly; float64 energies and log Z to 1e-12 relative (the only freedom is
the order of exact-or-near-exact float64 sums).
"""

import ctypes as C

import numpy as np
import pytest

from jaxrens_b200 import _lib, prior_mass, prng
from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200.backends import GaussianMixtureBackend, Hamiltonian, create_lj, EnsembleTerm
from oracle import oracle as O
from tests._cases import lj_case, oracle_model, oracle_replicas

pytestmark = pytest.mark.gpu

torch = pytest.importorskip("torch")


def _np(t):
    return t.detach().cpu().numpy()


# ------------------------------------------------------------- energies ----

def _configs(rng, B, N, L, triclinic=False, S=1):
    pos = (rng.uniform(0, 1, (B, N, 3)) * L).astype(np.float32)
    cell = np.tile(np.eye(3, dtype=np.float32) * L, (B, 1, 1))
    if triclinic:
        cell = cell + rng.uniform(-0.3, 0.3, (B, 3, 3)).astype(np.float32) * (1 - np.eye(3, dtype=np.float32))
    types = rng.integers(0, S, (B, N)).astype(np.int32)
    return pos, cell.astype(np.float32), types


@pytest.mark.parametrize("kind", ["cubic", "triclinic", "images", "lb", "pairtable",
                                  "nonperiodic", "nocutoff"])
def test_energy_forces_bitwise_vs_oracle(kind):
    rng = np.random.default_rng(11)
    S = 1
    sc = (1, 1, 1)
    cutoff = 2.5
    if kind == "lb":
        lj = create_lj(epsilon=[1.0, 0.5], sigma=[1.0, 1.2], cutoff=2.5)
        S = 2
    elif kind == "pairtable":
        lj = create_lj(epsilon=[[1.0, 1.5], [1.5, 0.5]], sigma=[[1.0, 0.8], [0.8, 0.88]], cutoff=2.5)
        S = 2
    else:
        if kind == "images":
            sc = (2, 2, 2)
        if kind == "nocutoff":
            cutoff = None
        lj = create_lj(epsilon=1.0, sigma=1.0, cutoff=cutoff, supercell_trafo=sc)
    H = Hamiltonian(lj, [EnsembleTerm(pressure=0.37)])
    B, N = 24, 32
    L = 3.6 if kind == "images" else 4.4
    pos, cell, types = _configs(rng, B, N, L, triclinic=(kind == "triclinic"), S=S)
    if kind == "nonperiodic":
        cell[:] = 0.0
    res = H.energy_and_forces(pos, types, cell)
    E = _np(res.energy)
    F = _np(res.forces)
    m = oracle_model(H)
    for b in range(B):
        e_o, f_o, _ = O.energy(m, pos[b], types[b], cell[b], pressure=0.37, mode=O.DEV)
        assert abs(E[b] - e_o) <= 1e-12 * max(1.0, abs(e_o)), (b, E[b], e_o)
        np.testing.assert_array_equal(F[b], f_o.astype(np.float32))
        e64, f64, _ = O.energy(m, pos[b], types[b], cell[b], pressure=0.37, mode=O.F64)
        assert abs(E[b] - e64) <= 1e-5 * max(1.0, abs(e64))
        assert np.abs(F[b] - f64).max() <= 1e-5 * max(1.0, np.abs(f64).max())


@pytest.mark.parametrize("N", [80, 100])
def test_energy_forces_large_walkers_bitwise_vs_oracle(N):
    """Walkers above 64 atoms: the pair-matrix path up to 96, the ordered
    pairs beyond, both bit-exact against the oracle."""
    rng = np.random.default_rng(N)
    lj = create_lj(epsilon=1.0, sigma=1.0, cutoff=2.5)
    H = Hamiltonian(lj, [EnsembleTerm(pressure=0.2)])
    L = 1.25 * N ** (1.0 / 3.0)
    pos, cell, types = _configs(rng, 6, N, L, triclinic=True)
    res = H.energy_and_forces(pos, types, cell)
    E, F = _np(res.energy), _np(res.forces)
    m = oracle_model(H)
    for b in range(6):
        e_o, f_o, _ = O.energy(m, pos[b], types[b], cell[b], pressure=0.2, mode=O.DEV)
        assert abs(E[b] - e_o) <= 1e-12 * max(1.0, abs(e_o)), (b, E[b], e_o)
        np.testing.assert_array_equal(F[b], f_o.astype(np.float32))


def test_large_walker_ns_run_matches_oracle():
    case = lj_case(P=1, K=12, N=80, seed=8, n_reflect=2, T=2, v_hi_per_atom=3.0)
    ns, infos = _run_gpu(case, 4, 2)
    reps, hist = _run_oracle(case, 4, 2)
    _compare(case, ns, infos, reps, hist)


def test_gauss_mix_energy_vs_oracle():
    g = GaussianMixtureBackend(centers=[[-1, 0, 0], [1, 0.5, 0]], sigma=0.5)
    rng = np.random.default_rng(3)
    pos = rng.uniform(-3, 3, (16, 1, 3)).astype(np.float32)
    res = g.energy_and_forces(pos, np.zeros((16, 1), np.int32), np.zeros((16, 3, 3), np.float32))
    m = oracle_model(g)
    for b in range(16):
        e_o, f_o, _ = O.energy(m, pos[b], [0], np.zeros((3, 3)))
        assert abs(float(_np(res.energy)[b]) - e_o) < 1e-12 * max(1, abs(e_o))
        np.testing.assert_allclose(_np(res.forces)[b], f_o, rtol=1e-6, atol=1e-7)


# ------------------------------------------------------------ NS steps ----

def _run_gpu(case, n_iter, T, n_extra=0, batched=None, cfg=None, chunk=None):
    P = case["P"]
    batched = P > 1 if batched is None else batched
    if batched:
        ns = nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                  case["energies"], case["cells"], case["run_keys"],
                                  ensemble_params={"pressure": case["pressures"],
                                                   "chemical_potentials": case["mus"]})
    else:
        ns = nsm.init_ns(case["init_fn"], case["positions"][0], case["types"][0],
                         case["energies"][0], case["cells"][0], case["run_keys"][0],
                         ensemble_params={"pressure": float(case["pressures"][0])})
    infos = []
    done = 0
    chunk = chunk or n_iter
    while done < n_iter:
        c = min(chunk, n_iter - done)
        infos.append(nsm.ns_iterate(ns, case["step"], c, T, n_extra, cfg=cfg))
        done += c
    torch.cuda.synchronize()
    return ns, infos


def _run_oracle(case, n_iter, T, n_extra=0, batched=None):
    P = case["P"]
    batched = P > 1 if batched is None else batched
    reps = oracle_replicas(case)
    K = case["K"]
    la = prior_mass.log_alpha(K, 1)
    wo = float(prior_mass.iteration_offsets(K, 1)[1][0])
    hist = []
    for _ in range(n_iter):
        if batched:
            infos = O.ns_step_batched(case["model"], case["moves"], reps, T, la, wo,
                                      n_extra=n_extra, shared_move_key=True)
        else:
            infos = [O.ns_step(case["model"], case["moves"], reps[0], T, la, wo,
                               n_extra=n_extra)[0]]
        hist.append([(i.worst_idx, i.clone_idx, i.emax, list(i.n_acc), list(i.n_prop),
                      list(i.rr), list(i.n_evals), float(r.log_evidence[0]))
                     for i, r in zip(infos, reps)])
    return reps, hist


def _compare(case, ns, infos, reps, hist):
    pop = ns.population
    X, D, T_, C_ = _np(pop.positions), _np(pop.direction), _np(pop.types), _np(pop.cell)
    E = _np(pop.energy64)
    keys = _np(ns.rng_key).view(np.uint32)
    M = case["step"].n_moves
    for r, rep in enumerate(reps):
        n = case["Ns"][r]
        np.testing.assert_array_equal(X[r, :, :n], rep.positions)
        np.testing.assert_array_equal(D[r, :, :n], rep.direction)
        np.testing.assert_array_equal(T_[r, :, :n], rep.types)
        np.testing.assert_array_equal(C_[r], rep.cell)
        np.testing.assert_allclose(E[r], rep.energy, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(keys[r], rep.rng_key)
        assert int(_np(ns.iteration)[r]) == int(rep.iteration[0])
        np.testing.assert_array_equal(_np(pop.n_accepted)[r], rep.n_acc)
        np.testing.assert_array_equal(_np(pop.n_proposed)[r], rep.n_prop)
        assert abs(float(_np(ns.log_evidence)[r]) - rep.log_evidence[0]) <= 1e-12 * max(1, abs(rep.log_evidence[0]))
    row = 0
    for info in infos:
        for j in range(info.n_iter):
            for r in range(len(reps)):
                w, c, em, nacc, nprop, rr, nev, lz = hist[row][r]
                assert int(_np(info.worst_idx)[j, r]) == w
                assert int(_np(info.clone_idx)[j, r]) == c
                assert abs(float(_np(info.emax)[j, r]) - em) <= 1e-12 * max(1, abs(em))
                np.testing.assert_array_equal(_np(info.n_accepted)[j, r], nacc[:M])
                np.testing.assert_array_equal(_np(info.n_proposed)[j, r], nprop[:M])
                np.testing.assert_array_equal(_np(info.reject_reason_counts)[j, r].reshape(-1), rr[: 4 * M])
                np.testing.assert_array_equal(_np(info.n_evaluations)[j, r], nev[:M])
                assert abs(float(_np(info.log_evidence)[j, r]) - lz) <= 1e-12 * max(1, abs(lz))
            row += 1


def test_single_run_matches_oracle():
    case = lj_case(P=1, K=32, N=8, seed=1, n_reflect=4, T=5)
    ns, infos = _run_gpu(case, 25, 5, chunk=7)
    reps, hist = _run_oracle(case, 25, 5)
    _compare(case, ns, infos, reps, hist)


def test_batched_shared_move_key_matches_oracle():
    case = lj_case(P=3, K=24, N=12, seed=2, n_reflect=3, T=4, pressure=np.array([0.05, 0.1, 0.3]))
    ns, infos = _run_gpu(case, 15, 4)
    reps, hist = _run_oracle(case, 15, 4)
    _compare(case, ns, infos, reps, hist)


def test_n_extra_matches_oracle():
    case = lj_case(P=2, K=20, N=8, seed=3, n_reflect=3, T=3)
    ns, infos = _run_gpu(case, 10, 3, n_extra=3)
    reps, hist = _run_oracle(case, 10, 3, n_extra=3)
    _compare(case, ns, infos, reps, hist)


def test_uneven_semigrand_identity_moves_match_oracle():
    lj_pair = dict(epsilon=[[1.0, 1.5], [1.5, 0.5]], sigma=[[1.0, 0.8], [0.8, 0.88]])
    case = lj_case(P=3, K=16, N=8, seed=4, n_reflect=3, T=6, n_atoms_list=[8, 12, 16],
                   identity="both", mu=np.array([[0.0, -1.0], [0.0, 0.0], [0.0, 1.5]]),
                   **lj_pair)
    ns, infos = _run_gpu(case, 12, 6)
    reps, hist = _run_oracle(case, 12, 6)
    _compare(case, ns, infos, reps, hist)


def test_uneven_semigrand_up_to_96_atoms_matches_oracle():
    """The uneven semi-grand shape of the batched binary configuration: runs of
    16, 56 and 96 atoms in one launch (Nmax 96, pair-matrix path with a
    per-run row stride), Kob-Andersen pair tables, Delta-mu, morph and swap
    identity moves."""
    lj_pair = dict(epsilon=[[1.0, 1.5], [1.5, 0.5]], sigma=[[1.0, 0.8], [0.8, 0.88]])
    case = lj_case(P=3, K=12, N=16, seed=9, n_reflect=2, T=3, n_atoms_list=[16, 56, 96],
                   identity="both", mu=np.array([[0.0, -2.0], [0.0, 0.3], [0.0, 2.0]]),
                   v_hi_per_atom=4.0, **lj_pair)
    ns, infos = _run_gpu(case, 6, 3)
    reps, hist = _run_oracle(case, 6, 3)
    _compare(case, ns, infos, reps, hist)


def test_supercell_images_match_oracle():
    case = lj_case(P=1, K=16, N=6, seed=5, n_reflect=3, T=3, supercell=(2, 2, 2),
                   v_hi_per_atom=6.0)
    ns, infos = _run_gpu(case, 8, 3)
    reps, hist = _run_oracle(case, 8, 3)
    _compare(case, ns, infos, reps, hist)


def test_shear_and_stretch_moves_match_oracle():
    """Shear (shear.py) and stretch (stretch.py) cell moves beside galilean and
    volume: walkers, keys and counters identical to the oracle; the sheared
    cells take the triclinic minimum-image path."""
    case = lj_case(P=2, K=16, N=6, seed=90, n_reflect=2, T=6, cell_moves=True,
                   pressure=np.array([0.1, 0.5]))
    ns, infos = _run_gpu(case, 14, 6, chunk=5)
    reps, hist = _run_oracle(case, 14, 6)
    _compare(case, ns, infos, reps, hist)
    cells = _np(ns.population.cell)
    off = cells * (1 - np.eye(3, dtype=np.float32))
    assert (np.abs(off) > 0).any()
    acc = sum(_np(i.n_accepted).sum(axis=(0, 1)) for i in infos)
    assert acc[2] > 0 and acc[3] > 0


@pytest.mark.parametrize("types_dep", [False, True])
def test_min_distance_gate_matches_oracle(types_dep):
    """A minimum-distance constraint (constraints/min_distance.py) gates the
    moves that can violate it; undone moves, reason-4 drops from the bucket
    counts and all walker state identical to the oracle."""
    dmin = [[0.6, 0.5], [0.5, 0.4]] if types_dep else 0.6
    case = lj_case(P=2, K=16, N=6, seed=80 + int(types_dep), n_reflect=2, T=4,
                   identity="morph", epsilon=[1.0, 0.5], sigma=[1.0, 0.9], d_min=dmin,
                   d_min_types=types_dep, pressure=np.array([0.1, 0.3]))
    ns, infos = _run_gpu(case, 12, 4)
    reps, hist = _run_oracle(case, 12, 4)
    _compare(case, ns, infos, reps, hist)
    n_prop = sum(_np(i.n_proposed).sum() for i in infos)
    n_rr = sum(_np(i.reject_reason_counts).sum() for i in infos)
    assert n_rr < n_prop   # the gate undid some accepted moves


@pytest.mark.parametrize("P,n_cull,n_extra", [(1, 3, 0), (1, 4, 2), (2, 2, 1)])
def test_multi_cull_matches_oracle(P, n_cull, n_extra):
    """n_cull > 1 (nested_sampling.py:195-212): lexsort cull order, permuted
    survivors as clone sources and extras, per-cull dead points, logsumexp
    evidence -- walkers, keys and per-cull info identical to the oracle."""
    case = lj_case(P=P, K=24, N=8, seed=40 + n_cull, n_reflect=3, T=3,
                   pressure=np.linspace(0.05, 0.3, P))
    K, T, n_iter = 24, 3, 8
    batched = P > 1
    if batched:
        ns = nsm.init_ns_parallel(case["init_fn"], case["positions"], case["types"],
                                  case["energies"], case["cells"], case["run_keys"],
                                  ensemble_params={"pressure": case["pressures"],
                                                   "chemical_potentials": case["mus"]})
    else:
        ns = nsm.init_ns(case["init_fn"], case["positions"][0], case["types"][0],
                         case["energies"][0], case["cells"][0], case["run_keys"][0],
                         ensemble_params={"pressure": float(case["pressures"][0])})
    info = nsm.ns_iterate(ns, case["step"], n_iter, T, n_extra, n_cull=n_cull)
    torch.cuda.synchronize()
    reps = oracle_replicas(case)
    la = prior_mass.log_alpha(K, n_cull)
    wo = prior_mass.iteration_offsets(K, n_cull)[1]
    for it in range(n_iter):
        mk = O.fold_in(reps[0].rng_key, 1) if batched else None
        for r, rep in enumerate(reps):
            oi, worst, clone, de, dx, dt, dc = O.ns_step_n(
                case["model"], case["moves"], rep, T, la, wo, n_cull, n_extra=n_extra,
                move_key=mk)
            np.testing.assert_array_equal(_np(info.worst_idx)[it, r], worst)
            np.testing.assert_array_equal(_np(info.clone_idx)[it, r], clone)
            np.testing.assert_allclose(_np(info.dead_energy)[it, r], de, rtol=1e-12, atol=0)
            np.testing.assert_array_equal(_np(info.dead_positions)[it, r], dx)
            assert abs(float(_np(info.emax)[it, r]) - oi.emax) <= 1e-12 * max(1, abs(oi.emax))
            lz = float(rep.log_evidence[0])
            assert abs(float(_np(info.log_evidence)[it, r]) - lz) <= 1e-12 * max(1, abs(lz))
            np.testing.assert_array_equal(_np(info.n_proposed)[it, r],
                                          list(oi.n_prop)[:case["step"].n_moves])
    pop = ns.population
    for r, rep in enumerate(reps):
        n = case["Ns"][r]
        np.testing.assert_array_equal(_np(pop.positions)[r, :, :n], rep.positions)
        np.testing.assert_array_equal(_np(pop.types)[r, :, :n], rep.types)
        np.testing.assert_allclose(_np(pop.energy64)[r], rep.energy, rtol=1e-12, atol=0)
        np.testing.assert_array_equal(_np(ns.rng_key).view(np.uint32)[r], rep.rng_key)


@pytest.mark.parametrize("cfg", [(128, 4, 1, 0), (256, 8, 2, 0), (256, 16, 4, 0),
                                 (512, 32, 8, 0), (256, 8, 12, 0), (32, 2, 1, 1),
                                 (128, 2, 1, 1), (64, 2, 4, 1), (128, 2, 8, 1),
                                 (32, 2, 16, 1)])
def test_launch_shape_and_speculation_do_not_change_results(cfg):
    case = lj_case(P=2, K=32, N=16, seed=6, n_reflect=4, T=4)
    ref_ns, ref_infos = _run_gpu(case, 20, 4, cfg=_lib.JrLaunchConfig(256, 8, 1, 0))
    ns, infos = _run_gpu(case, 20, 4, cfg=_lib.JrLaunchConfig(*cfg))
    # Indices, configurations and keys are identical.  float64 energies may
    # differ in the last bit when pair terms span more than 2^29 in magnitude
    # (overlapping atoms of the random-gas start, |E| ~ 1e15), because then the
    # float64 sums are not exact and their order follows the launch shape.
    for a, b in [(ref_ns.population.positions, ns.population.positions),
                 (ref_ns.population.direction, ns.population.direction),
                 (ref_ns.rng_key, ns.rng_key), (ref_ns.iteration, ns.iteration)]:
        assert torch.equal(a, b)
    for f in ("worst_idx", "clone_idx", "n_accepted", "n_proposed"):
        assert torch.equal(getattr(ref_infos[0], f), getattr(infos[0], f))
    for a, b in [(ref_ns.population.energy64, ns.population.energy64),
                 (ref_ns.log_evidence, ns.log_evidence),
                 (ref_infos[0].emax, infos[0].emax),
                 (ref_infos[0].log_evidence, infos[0].log_evidence)]:
        torch.testing.assert_close(a, b, rtol=1e-12, atol=0)


@pytest.mark.parametrize("cfg", [(256, 8, 8, 0), (128, 4, 4, 1)])
def test_speculation_commits_more_than_one_iteration_per_round(cfg):
    case = lj_case(P=2, K=64, N=8, seed=7, n_reflect=3, T=3)
    ns, infos = _run_gpu(case, 16, 3, cfg=_lib.JrLaunchConfig(*cfg))
    rounds = _np(infos[0].rounds)
    assert (rounds < 16).all() and (rounds >= 2).all()
    reps, hist = _run_oracle(case, 16, 3)
    _compare(case, ns, infos, reps, hist)


def test_re_swap_matches_oracle():
    case = lj_case(P=4, K=16, N=8, seed=8, n_reflect=3, T=3,
                   pressure=np.array([0.01, 0.05, 0.2, 1.0]))
    ns, _ = _run_gpu(case, 6, 3)
    reps, _ = _run_oracle(case, 6, 3)
    key = prng.key(99)
    re = nsm.InterREManager(10, 2, key)
    swap_key = prng.split(re.key, 2)[1]
    swap_key = prng.split(swap_key, 2)[1]
    stats = re.apply(ns, case["step"])
    acc, att = O.re_step(reps, swap_key, n_swap_cycles=2)
    torch.cuda.synchronize()
    np.testing.assert_array_equal(_np(stats["n_accepted_per_pair"]), acc)
    np.testing.assert_array_equal(_np(stats["n_attempted_per_pair"]), att)
    X = _np(ns.population.positions)
    E = _np(ns.population.energy64)
    for r, rep in enumerate(reps):
        np.testing.assert_array_equal(X[r], rep.positions)
        np.testing.assert_allclose(E[r], rep.energy, rtol=1e-12)


def test_move_trials_match_oracle():
    case = lj_case(P=2, K=16, N=10, seed=9, n_reflect=5, T=3)
    ns, _ = _run_gpu(case, 4, 3)
    reps, _ = _run_oracle(case, 4, 3)
    n = 8
    for m in range(case["step"].n_moves):
        widx = np.stack([np.arange(n), np.arange(n) + 4])
        keys = prng.split(prng.key(100 + m), 2 * n).reshape(2, n, 2)
        emax = _np(ns.emax)
        acc, reason = nsm.TrialMove(case["step"], m)(ns, widx, keys, [0.15, 0.2], emax)
        acc = _np(acc)
        for r in range(2):
            for t in range(n):
                rep = reps[r]
                k = widx[r, t]
                a, *_rest = O.move_trial(case["model"], case["moves"], m, keys[r, t],
                                         [0.15, 0.2][r], float(rep.emax[0]),
                                         rep.positions[k], rep.direction[k], rep.types[k],
                                         rep.cell[k], rep.energy[k], pressure=rep.pressure)
                assert bool(acc[r, t]) == a


def test_lazy_forces_work_counters():
    """A galilean step evaluates the energy and, only when it reflects off the
    contour, the forces: per iteration the energy-only pair count is exactly
    every counted evaluation's n(n-1)/2 unique pairs, and the pairs with
    forces are n(n-1)/2 per reflection, at most one per counted gradient
    evaluation.  The walk itself is pinned to the oracle by the other tests."""
    case = lj_case(P=2, K=24, N=12, seed=77, n_reflect=5, T=6)
    ns, infos = _run_gpu(case, 8, 6)
    np_ = 12 * 11 // 2
    for info in infos:
        tc = _np(info.term_counts)
        ne = _np(info.n_evaluations).sum(-1)
        ng = _np(info.n_grad_evaluations).sum(-1)
        np.testing.assert_array_equal(tc[..., 2], ne * np_)
        assert (tc[..., 0] % np_ == 0).all() and (tc[..., 0] <= ng * np_).all()
        assert (tc[..., 1] == 0).all() and (tc[..., 3] == 0).all()
