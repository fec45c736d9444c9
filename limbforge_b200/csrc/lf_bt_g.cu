// Batched small-matrix kernel instantiations for limb counts 29..30.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(29)
LF_BATCHED_INSTANTIATE(30)
