// jr_sw.cu -- the Stillinger-Weber family of the walk kernels.  The C-ABI
// entry points in jr_ns.cu dispatch here when params.model.model is
// JR_MODEL_SW; this translation unit instantiates the SW-family launch
// templates of jr_host.cuh (and with them the SW-family kernels of
// jr_kernels.cuh), compiled apart from the pair family.
#define JR_INSTANTIATE_SW
#include "jr_host.cuh"

template int jrh::launch_ns_family<jr::kFamSW>(JR_NS_WALK_ARGS);
template int jrh::launch_trial_family<jr::kFamSW>(JR_TRIAL_ARGS);
template int jrh::launch_population_family<jr::kFamSW>(JR_POP_ARGS);
template int jrh::launch_energy_family<jr::kFamSW>(JR_ENERGY_ARGS);
