"""Host-side logic and the C ABI boundary (CPU only, no compute calls)."""

import ctypes as C
import os
import re
import subprocess
import tempfile

import numpy as np
import pytest

from jaxrens_b200 import _lib, create_lj, prior_mass, prng
from jaxrens_b200 import moves as mvs
from jaxrens_b200 import nested_sampling as nsm
from jaxrens_b200.backends import EnsembleTerm, Hamiltonian, make_image_offsets
from jaxrens_b200.mwg import build_mwg
from oracle import oracle as O

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
HEADER = os.path.join(ROOT, "include", "jaxrens_b200.h")


def _declared_functions():
    src = open(HEADER).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(jr_[a-z0-9_]+)\s*\(", src)))


def test_library_loads_and_exports_every_declared_symbol():
    from jaxrens_b200 import _build

    _build.build()
    L = C.CDLL(_lib.LIB_PATH)
    declared = _declared_functions()
    assert sorted(_lib.EXPORTED) == declared
    for name in declared:
        assert hasattr(L, name), name
    assert _lib.load().jr_version() >= 2


def test_struct_layout_matches_header():
    prog = r'''
#include <stdio.h>
#include <stddef.h>
#include "jaxrens_b200.h"
int main(void) {
  printf("%zu %zu %zu %zu %zu %zu %zu %zu %zu %zu %zu\n", sizeof(JrDims), sizeof(JrModelParams),
         sizeof(JrMoveParams), sizeof(JrParams), sizeof(JrStateBuffers), sizeof(JrInfoBuffers),
         sizeof(JrLaunchConfig), offsetof(JrParams, log_alpha), offsetof(JrModelParams, gm_sigma),
         offsetof(JrModelParams, sw_leps), offsetof(JrInfoBuffers, term_counts));
  return 0;
}
'''
    with tempfile.TemporaryDirectory() as d:
        c = os.path.join(d, "t.c")
        open(c, "w").write(prog)
        exe = os.path.join(d, "t")
        subprocess.run(["gcc", "-I", os.path.dirname(HEADER), c, "-o", exe], check=True)
        got = [int(v) for v in subprocess.run([exe], capture_output=True, text=True,
                                              check=True).stdout.split()]
    want = [C.sizeof(_lib.JrDims), C.sizeof(_lib.JrModelParams), C.sizeof(_lib.JrMoveParams),
            C.sizeof(_lib.JrParams), C.sizeof(_lib.JrStateBuffers), C.sizeof(_lib.JrInfoBuffers),
            C.sizeof(_lib.JrLaunchConfig), _lib.JrParams.log_alpha.offset,
            _lib.JrModelParams.gm_sigma.offset, _lib.JrModelParams.sw_leps.offset,
            _lib.JrInfoBuffers.term_counts.offset]
    assert got == want


def test_invalid_arguments_fail_loudly_without_a_gpu():
    L = _lib.load()
    d = _lib.JrDims(1, 16, 8, 2, 4, 0, 0, 0)  # n_cull = 0 is out of range
    p = _lib.JrParams()
    p.model.n_species = 1
    p.model.n_images = 1
    p.moves.n_moves = 2
    rc = L.jr_ns_iterate(C.byref(d), C.byref(p), C.byref(_lib.JrStateBuffers()), None, 1,
                         None, None, 0, None)
    assert _lib.ERRORS[rc] == "JR_ERR_SHAPE"
    assert b"n_cull" in L.jr_last_error()
    d.n_cull = 9  # 2 * n_cull + n_extra > n_walkers (the reference's own bound)
    rc = L.jr_ns_iterate(C.byref(d), C.byref(p), C.byref(_lib.JrStateBuffers()), None, 1,
                         None, None, 0, None)
    assert _lib.ERRORS[rc] == "JR_ERR_SHAPE"
    assert b"2*n_cull" in L.jr_last_error()
    with pytest.raises(_lib.JrError):
        _lib.check(rc, "jr_ns_iterate")


def test_lj_tables_follow_reference_rounding():
    a = create_lj(epsilon=0.7, sigma=0.9, cutoff=2.5)
    assert a.eps4[0, 0] == np.float32(4.0 * 0.7)
    assert a.sig2[0, 0] == np.float32(0.9 * 0.9)
    b = create_lj(epsilon=[0.7, 0.7], sigma=[0.9, 0.9])
    # the table path squares the float32 sigma (lj.py:186) -- may differ by 1 ulp
    assert abs(float(b.sig2[0, 1]) - 0.81) < 1e-6
    lb = create_lj(epsilon=[1.0, 0.5], sigma=[1.0, 1.2])
    assert lb.eps4[0, 1] == np.float32(4.0) * np.sqrt(np.float32(1.0) * np.float32(0.5))
    assert lb.sig2[0, 1] == np.float32(1.1) * np.float32(1.1)
    with pytest.raises(ValueError):
        create_lj(epsilon=[1.0, 1.0], sigma=1.0)
    with pytest.raises(ValueError):
        create_lj(supercell_trafo=(0, 1, 1))


def test_image_offsets_like_reference():
    assert make_image_offsets(1, 1, 1).tolist() == [[0, 0, 0]]
    assert len(make_image_offsets(2, 2, 2)) == 27
    assert len(make_image_offsets(4, 4, 4)) == 125


def test_build_mwg_probabilities_and_params():
    H = Hamiltonian(create_lj(cutoff=2.5), [EnsembleTerm(pressure=0.1)])
    _, step, per = build_mwg(H, [mvs.gmc(n_reflect=10, weight=4.0), mvs.volume_move(32)])
    assert step.params.moves.n_moves == 2
    assert np.float32(step.params.moves.cum_probs[0]) == np.float32(0.8)
    assert np.float32(step.params.moves.cum_probs[1]) == np.float32(1.0)
    assert step.params.moves.n_reflect[0] == 10
    assert len(per) == 2
    with pytest.raises(NotImplementedError):
        build_mwg(H, [mvs.MoveKernel("g", mvs.galilean.build_kernel,
                                     kernel_kwargs={"use_forces": False})])


def test_re_firing_schedule_and_key_chain():
    re = nsm.InterREManager(10, 1, prng.key(5))
    assert [i for i in range(35) if re.fires(i)] == [10, 20, 30]
    k0 = re.key.copy()
    sk = re.next_swap_key()
    a, b = prng.split(k0, 2)
    assert np.array_equal(re.key, a)
    assert np.array_equal(sk, prng.split(b, 2)[1])


def test_prior_mass_termination_semantics():
    t = nsm.PriorMassTermination(n_live=32, threshold=1e-3)
    assert not t.check(10, 5.0)  # never before every walker was replaced once
    t.update_evidence(-2.0)
    la = prior_mass.log_alpha(32, 1)
    it = 5000
    assert t.check(it, -((it + 1) * la) + 2.0 + 10.0) is True
    assert nsm.IterationTermination(100).check(99, 0.0)


def test_oracle_ns_step_counter_invariants_and_evidence():
    from tests._cases import lj_case, oracle_replicas

    case = lj_case(P=1, K=24, N=8, seed=12, n_reflect=3, T=6)
    rep = oracle_replicas(case)[0]
    la = prior_mass.log_alpha(24, 1)
    wo = float(prior_mass.iteration_offsets(24, 1)[1][0])
    last = -np.inf
    emaxes = []
    for _ in range(40):
        info, *_ = O.ns_step(case["model"], case["moves"], rep, 6, la, wo)
        for m in range(2):
            assert info.rr[4 * m] == info.n_acc[m]
            assert sum(info.rr[4 * m: 4 * m + 4]) == info.n_prop[m]
        assert sum(info.n_prop[:2]) == 6
        assert rep.log_evidence[0] >= last
        last = rep.log_evidence[0]
        emaxes.append(info.emax)
        assert rep.energy.max() <= info.emax
    assert all(b <= a for a, b in zip(emaxes, emaxes[1:]))


def test_worst_walker_ties_break_on_noise():
    from tests._cases import lj_case, oracle_replicas

    case = lj_case(P=1, K=16, N=4, seed=13, n_reflect=2, T=1)
    rep = oracle_replicas(case)[0]
    rep.energy[:] = 7.0
    key = rep.rng_key.copy()
    info, *_ = O.ns_step(case["model"], case["moves"], rep, 1, prior_mass.log_alpha(16, 1),
                         float(prior_mass.iteration_offsets(16, 1)[1][0]))
    kw = prng.split(key, 2)[1]
    assert info.worst_idx == int(np.argmax(prng.uniform(kw, 16)))


def test_oracle_replica_exchange_keeps_energies_in_receiving_frame():
    from tests._cases import lj_case, oracle_replicas

    case = lj_case(P=4, K=12, N=6, seed=14, n_reflect=2, T=2,
                   pressure=np.array([0.01, 0.1, 0.5, 1.0]))
    reps = oracle_replicas(case)
    for r in reps:
        r.emax[0] = np.inf
    acc, att = O.re_step(reps, prng.key(3), n_swap_cycles=3)
    assert att.sum() == 3 * 3 and acc.sum() > 0
    for r in reps:
        for k in range(12):
            e = O.energy(case["model"], r.positions[k], r.types[k], r.cell[k],
                         pressure=r.pressure, forces=False)[0]
            assert abs(e - r.energy[k]) <= 1e-9 * max(1.0, abs(e))


def test_host_prng_matches_oracle():
    k = prng.key(77)
    assert np.array_equal(prng.split(k, 9), O.split(k, 9))
    assert np.array_equal(prng.fold_in(k, 1), O.fold_in(k, 1))
    assert np.array_equal(prng.advance_iteration(k), O.split(O.split(k, 2)[0], 5)[0])


def test_oracle_multi_cull_invariants():
    """n_cull > 1 (nested_sampling.py:195-212): the culls are the n_cull
    highest energies in descending order, the contour is the last of them,
    clone sources and extras are distinct survivors, log Z only grows."""
    from tests._cases import lj_case, oracle_replicas

    K, nc, nx = 20, 3, 2
    case = lj_case(P=1, K=K, N=6, seed=15, n_reflect=2, T=2)
    rep = oracle_replicas(case)[0]
    la = prior_mass.log_alpha(K, nc)
    wo = prior_mass.iteration_offsets(K, nc)[1]
    last = -np.inf
    for _ in range(12):
        E = rep.energy.copy()
        info, worst, clone, de, *_ = O.ns_step_n(case["model"], case["moves"], rep, 2, la, wo,
                                                 nc, n_extra=nx)
        top = np.sort(E)[::-1][:nc]
        np.testing.assert_array_equal(E[worst], top)
        np.testing.assert_array_equal(de, top)
        assert info.emax == top[-1]
        assert len(set(clone.tolist())) == nc and not set(clone.tolist()) & set(worst.tolist())
        assert sum(info.n_prop) == 2 * (nc + nx)
        assert rep.log_evidence[0] >= last
        last = rep.log_evidence[0]
        assert rep.energy.max() <= info.emax


def test_min_distance_gates_the_moves_that_can_violate_it():
    """make_move_gate (constraints/base.py:101-140): a uniform threshold gates
    the position/cell moves only; a per-species one also the relabelling
    moves.  A violating accepted move is undone with reason 4, which the
    4-bucket reject counts drop (nested_sampling.py:562-570)."""
    from tests._cases import lj_case, oracle_replicas

    c = lj_case(P=1, K=16, N=6, seed=16, n_reflect=2, T=4, identity="morph",
                epsilon=[1.0, 0.5], sigma=[1.0, 0.9], d_min=0.6)
    assert [c["step"].params.moves.gate[m] for m in range(3)] == [1, 1, 0]
    c2 = lj_case(P=1, K=16, N=6, seed=16, n_reflect=2, T=4, identity="morph",
                 epsilon=[1.0, 0.5], sigma=[1.0, 0.9], d_min=[[0.6, 0.5], [0.5, 0.4]],
                 d_min_types=True)
    assert [c2["step"].params.moves.gate[m] for m in range(3)] == [1, 1, 1]
    rep = oracle_replicas(c)[0]
    dropped = 0
    for _ in range(20):
        info, *_ = O.ns_step(c["model"], c["moves"], rep, 4, prior_mass.log_alpha(16, 1),
                             float(prior_mass.iteration_offsets(16, 1)[1][0]))
        dropped += sum(info.n_prop[:3]) - sum(info.rr[:12])
        for m in range(3):
            assert info.rr[4 * m] == info.n_acc[m]
    assert dropped > 0   # some moves met the gate


def test_min_distance_predicate_matches_brute_force():
    """The oracle gate's verdict equals a float64 brute-force minimum-image
    distance check on random cubic configurations (away from the threshold)."""
    rng = np.random.default_rng(5)
    mv = O.make_moves([0], [1], [0.1], [1.0], gate=[1], dmin=[0.7])
    hits = 0
    for _ in range(40):
        L = 2.5
        x = rng.uniform(0, L, (6, 3)).astype(np.float32)
        cell = (np.eye(3) * L).astype(np.float32)
        d = x[:, None, :].astype(np.float64) - x[None, :, :]
        d -= L * np.round(d / L)
        r = np.sqrt((d ** 2).sum(-1))[np.triu_indices(6, 1)]
        if np.any(np.abs(r - 0.7) < 1e-4):
            continue
        want = bool(np.all(r >= 0.7))
        got = O.min_distance_ok(mv, 1, x, np.zeros(6, np.int32), cell)
        assert got == want
        hits += not want
    assert hits > 0


def test_oracle_shear_and_stretch_preserve_volume_and_fractions():
    """shear.py / stretch.py: both proposals keep the cell volume (to float32
    rounding) and map positions with the cell (fractional coordinates kept)."""
    from jaxrens_b200 import moves as mv_
    from tests._cases import lj_case, oracle_replicas

    c = lj_case(P=1, K=8, N=5, seed=17, n_reflect=2, T=1, cell_moves=True)
    assert [c["step"].params.moves.type[m] for m in range(4)] == [0, 1, 4, 5]
    rep = oracle_replicas(c)[0]
    for m in (2, 3):
        n_acc = 0
        for k in range(8):
            for s in range(6):
                key = prng.fold_in(prng.key(100 + s), k)
                acc, x, d, t, cell, e, reason = O.move_trial(
                    c["model"], c["moves"], m, key, 0.2, np.inf, rep.positions[k],
                    rep.direction[k], rep.types[k], rep.cell[k], rep.energy[k],
                    pressure=0.1)
                if not acc:
                    assert reason == 2   # infinite contour: only the cell guard rejects
                    continue
                n_acc += 1
                v0 = abs(np.linalg.det(rep.cell[k].astype(np.float64)))
                v1 = abs(np.linalg.det(cell.astype(np.float64)))
                assert abs(v1 - v0) <= 1e-5 * v0
                f0 = rep.positions[k].astype(np.float64) @ np.linalg.inv(rep.cell[k].astype(np.float64))
                f1 = x.astype(np.float64) @ np.linalg.inv(cell.astype(np.float64))
                assert np.abs(f1 - f0).max() < 1e-4
        assert n_acc > 0
    with pytest.raises(NotImplementedError):
        build_mwg(create_lj(), [mv_.volume_move(4, min_aspect_ratio=0.8),
                                mv_.shear_move(4, min_aspect_ratio=0.5)])


def test_uniform_gas_matches_the_oracle_bit_for_bit():
    """The host's synthetic initial walkers (init.uniform_gas) against the
    oracle's restatement (jro_init_walkers): cubic cell of volume
    v_hi * (1 - u), fractional coordinates uniform, walker k from
    split(key, K)[k] -- the same float32 values."""
    from jaxrens_b200 import init as jinit
    from jaxrens_b200 import prng
    from oracle import oracle as O

    for seed, K, N, v in ((0, 17, 8, 64.0), (5, 9, 32, 256.0), (11, 4, 64, 64 * 160.0)):
        key = prng.key(seed)
        p_host, c_host = jinit.uniform_gas(key, K, N, v)
        p_or, c_or = O.init_walkers(key, K, N, v)
        np.testing.assert_array_equal(p_host, p_or)
        np.testing.assert_array_equal(c_host, c_or)


def test_bernoulli_species_draws():
    """Species Bernoulli(0.5) from a threefry key: uniform(key, n) < 0.5,
    the same bits as the oracle's uniform stream."""
    from jaxrens_b200 import prng
    from oracle import oracle as O

    k = prng.key(3)
    b = prng.bernoulli(k, 4096, 0.5)
    np.testing.assert_array_equal(b, O.uniform(k, 4096) < np.float32(0.5))
    assert abs(b.mean() - 0.5) < 0.03


def test_reciprocal_seed_is_near_minimax():
    """The pair loop's reciprocal seed as_float(C - as_int(x)), C =
    0x7EF311C3: over the mantissas of one binade its largest relative error
    is 5.05%, within 1e-7 of the best offset a scan of C finds, and three
    Newton steps bring it below 1e-10 before rounding."""
    m = np.arange(0, 1 << 23, 13, dtype=np.uint32)
    xb = (m | 0x3F800000).astype(np.int64)
    x = (m | 0x3F800000).view(np.float32).astype(np.float64)

    def err(c):
        y = (np.int64(c) - xb).astype(np.uint32).view(np.float32).astype(np.float64)
        return np.abs(y * x - 1.0).max()

    e = err(0x7EF311C3)
    best = min(err(c) for c in range(0x7EF311C3 - 256, 0x7EF311C3 + 256, 4))
    assert 0.0504 < e < 0.0506 and e - best < 1e-7
    assert e ** 8 < 1e-10
