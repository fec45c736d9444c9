// Batched small-matrix kernel instantiations for limb counts 31..32.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(31)
LF_BATCHED_INSTANTIATE(32)
