// Batched small-matrix kernel instantiations for limb counts 22..24.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(22)
LF_BATCHED_INSTANTIATE(23)
LF_BATCHED_INSTANTIATE(24)
