"""jaxrens_b200 -- B200-native nested-sampling walk for jaxrens.

The hot path of jaxrens (the jitted ``ns_step``: max-energy cull and clone,
``n_mcmc_steps`` of Metropolis-within-Gibbs galilean / volume / identity
moves on the LJ + EnsembleTerm Hamiltonian, JAX threefry streams, evidence
accumulation) as hand-written CUDA for sm_100a behind a C ABI
(``include/jaxrens_b200.h``), with a Python host layer mirroring the
reference's operator interface.
"""

from .backends import (
    BackendResult,
    EnsembleTerm,
    GaussianMixtureBackend,
    Hamiltonian,
    LJBackend,
    StillingerWeberBackend,
    create_lj,
    create_sw,
    eval_energy_and_forces,
)
from .moves import (MoveKernel, alchemical, galilean, gmc, morph_move, shear, shear_move, stretch,
                    stretch_move, swap, swap_move, volume, volume_move)
from .adaptation import adjust_step_size, build_adapt_step, process_rate
from .burn_in import initial_walk, walk_population
from .energy_log import EnergyLogCallback, EnergyLogger
from .mwg import build_mwg
from . import thermo
from .nested_sampling import (
    InterREManager,
    IterationTermination,
    NSState,
    PriorMassTermination,
    final_log_evidence,
    init_ns,
    init_ns_parallel,
    ns_iterate,
    ns_step,
    run_loop,
    run_ns,
    run_ns_parallel,
)

__all__ = [
    "BackendResult", "EnsembleTerm", "GaussianMixtureBackend", "Hamiltonian", "LJBackend",
    "StillingerWeberBackend", "create_lj", "create_sw", "eval_energy_and_forces", "MoveKernel", "alchemical", "galilean", "gmc",
    "morph_move", "swap", "swap_move", "volume", "volume_move", "shear", "shear_move",
    "stretch", "stretch_move", "build_mwg",
    "InterREManager", "IterationTermination", "NSState", "PriorMassTermination",
    "final_log_evidence", "init_ns", "init_ns_parallel", "ns_iterate", "ns_step",
    "run_loop", "run_ns", "run_ns_parallel", "adjust_step_size", "build_adapt_step",
    "process_rate", "initial_walk", "walk_population", "EnergyLogCallback", "EnergyLogger",
]
