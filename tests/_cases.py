"""Shared builders for the parity tests: one configuration expressed both for
the CUDA package and for the CPU oracle from the same numpy arrays."""

from __future__ import annotations

import numpy as np

from jaxrens_b200 import Hamiltonian, EnsembleTerm, build_mwg, create_lj, init as jinit, prng
from jaxrens_b200 import moves as mvs
from jaxrens_b200.backends import GaussianMixtureBackend, StillingerWeberBackend
from oracle import oracle as O


def oracle_model(backend) -> O.JroModel:
    m = backend.model if hasattr(backend, "model") else backend
    if isinstance(m, StillingerWeberBackend):
        return O.make_sw_model(**m.consts)
    if isinstance(m, GaussianMixtureBackend):
        return O.make_model([[0.0]], [[0.0]], [[0.0]], None, None, O.MODEL_GAUSS_MIX,
                            m.centers, m.sigma)
    rc2 = None if m.cutoff is None else np.float32(m.cutoff ** 2)
    return O.make_model(m.eps4, m.eps24, m.sig2, rc2, m.image_offsets)


def oracle_moves(step) -> O.JroMoves:
    p = step.params.moves
    M = p.n_moves
    return O.make_moves([p.type[m] for m in range(M)], [p.n_reflect[m] for m in range(M)],
                        [p.perturb_angle[m] for m in range(M)],
                        [p.cum_probs[m] for m in range(M)], p.max_vpa, p.min_vpa,
                        p.min_aspect, bool(p.flat_v_prior), [p.gate[m] for m in range(M)],
                        list(p.dmin))


def lj_case(P=1, K=32, N=8, seed=0, n_reflect=4, T=5, pressure=0.1, epsilon=1.0,
            sigma=1.0, cutoff=2.5, supercell=(1, 1, 1), v_hi_per_atom=8.0,
            n_atoms_list=None, mu=None, identity=None, step_sizes=(0.1, 0.3),
            min_vpa=1.0, max_vpa=1e4, weights=(4.0, 1.0), d_min=None, d_min_types=False,
            cell_moves=False, backend=None):
    """LJ NPT (or semi-grand with identity moves) case with P runs; another
    backend (Stillinger-Weber) in place of LJ when ``backend`` is given."""
    lj = backend if backend is not None else create_lj(epsilon=epsilon, sigma=sigma,
                                                       cutoff=cutoff, supercell_trafo=supercell)
    S = lj.n_species
    H = Hamiltonian(lj, [EnsembleTerm(pressure=pressure, chemical_potentials=None)])
    Ns = list(n_atoms_list) if n_atoms_list is not None else [N] * P
    moves = [mvs.gmc(n_reflect=n_reflect, step_size=step_sizes[0], weight=weights[0]),
             mvs.volume_move(max(Ns), step_size=step_sizes[1], weight=weights[1],
                             min_volume_per_atom=min_vpa, max_volume_per_atom=max_vpa)]
    if cell_moves:
        moves.append(mvs.shear_move(max(Ns), step_size=0.15, weight=1.0,
                                    min_volume_per_atom=min_vpa, max_volume_per_atom=max_vpa))
        moves.append(mvs.stretch_move(max(Ns), step_size=0.15, weight=1.0,
                                      min_volume_per_atom=min_vpa, max_volume_per_atom=max_vpa))
    if identity == "morph":
        moves.append(mvs.morph_move(S, weight=1.0))
    elif identity == "swap":
        moves.append(mvs.swap_move(S, weight=1.0))
    elif identity == "both":
        moves.append(mvs.morph_move(S, weight=1.0))
        moves.append(mvs.swap_move(S, weight=1.0))
    cons = ()
    if d_min is not None:
        from jaxrens_b200.constraints import min_distance_descriptor

        dm = np.broadcast_to(np.asarray(d_min, np.float32), (S, S))
        cons = (min_distance_descriptor(dm, type_dependent=d_min_types),)
    init_fn, step, _ = build_mwg(H, moves, cons)
    root = prng.key(seed)
    keys = prng.split(root, P + 1)
    pos, cells, types = [], [], []
    for r in range(P):
        p_, c_ = jinit.uniform_gas(keys[r], K, Ns[r], v_hi_per_atom * Ns[r])
        pos.append(p_)
        cells.append(c_)
        if S > 1:
            # species uniform over S from threefry bits of a per-run key
            u = prng.uniform(prng.fold_in(keys[r], 7), K * Ns[r])
            types.append(np.minimum((u * S).astype(np.int32), S - 1).reshape(K, Ns[r]))
        else:
            types.append(np.zeros((K, Ns[r]), np.int32))
    run_keys = prng.split(keys[P], P)
    pressures = np.full(P, pressure, np.float32) if np.ndim(pressure) == 0 else np.asarray(pressure, np.float32)
    mus = None if mu is None else np.asarray(mu, np.float32).reshape(P, S)
    model = oracle_model(H)
    energies = []
    for r in range(P):
        e = np.zeros(K)
        for k in range(K):
            e[k] = O.energy(model, pos[r][k], types[r][k], cells[r][k], pressure=float(pressures[r]),
                            mu=None if mus is None else mus[r], forces=False)[0]
        energies.append(e)
    return dict(H=H, init_fn=init_fn, step=step, positions=pos, cells=cells, types=types,
                energies=energies, run_keys=run_keys, pressures=pressures, mus=mus,
                model=model, moves=oracle_moves(step), K=K, Ns=Ns, P=P, T=T)


def oracle_replicas(case):
    reps = []
    for r in range(case["P"]):
        M = case["step"].n_moves
        reps.append(O.Replica(case["positions"][r], case["types"][r], case["energies"][r],
                              case["cells"][r], np.tile(case["step"].default_step_sizes, (case["K"], 1)),
                              case["run_keys"][r], pressure=float(case["pressures"][r]),
                              mu=None if case["mus"] is None else case["mus"][r]))
        del M
    return reps
