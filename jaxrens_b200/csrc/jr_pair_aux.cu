// jr_pair_aux.cu -- the pair family's move-trial, burn-in and energy
// kernels, compiled apart from its NS walk.
#define JR_INSTANTIATE_PAIR_AUX
#include "jr_host.cuh"

template int jrh::launch_trial_family<jr::kFamPair>(JR_TRIAL_ARGS);
template int jrh::launch_population_family<jr::kFamPair>(JR_POP_ARGS);
template int jrh::launch_energy_family<jr::kFamPair>(JR_ENERGY_ARGS);
