// Batched small-matrix kernel instantiations for limb counts 29..32.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(29)
LF_BATCHED_INSTANTIATE(30)
LF_BATCHED_INSTANTIATE(31)
LF_BATCHED_INSTANTIATE(32)
