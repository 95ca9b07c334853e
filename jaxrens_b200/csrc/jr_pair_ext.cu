// jr_pair_ext.cu -- the pair family's full NS walk (the minimum-distance
// gate and the shear and stretch cell moves), compiled apart from the lean
// walk of jr_ns.cu.
#define JR_INSTANTIATE_PAIR_EXT
#include "jr_host.cuh"

template int jrh::launch_ns_walk<jr::kFamPair, true>(JR_NS_WALK_ARGS);
