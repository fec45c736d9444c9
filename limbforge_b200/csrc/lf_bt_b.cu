// Batched small-matrix kernel instantiations for limb counts 9..13.
#include "lf_batched.cuh"
LF_BATCHED_INSTANTIATE(9)
LF_BATCHED_INSTANTIATE(10)
LF_BATCHED_INSTANTIATE(11)
LF_BATCHED_INSTANTIATE(12)
LF_BATCHED_INSTANTIATE(13)
