// Batched small-matrix kernel instantiations for limb counts 27..28.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(27)
LF_BATCHED_INSTANTIATE(28)
