// Batched small-matrix kernel instantiations for limb counts 18..21.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(18)
LF_BATCHED_INSTANTIATE(19)
LF_BATCHED_INSTANTIATE(20)
LF_BATCHED_INSTANTIATE(21)
