// Batched small-matrix kernel instantiations for limb counts 25..26.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(25)
LF_BATCHED_INSTANTIATE(26)
