// Batched small-matrix kernel instantiations for limb counts 14..17.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(14)
LF_BATCHED_INSTANTIATE(15)
LF_BATCHED_INSTANTIATE(16)
LF_BATCHED_INSTANTIATE(17)
