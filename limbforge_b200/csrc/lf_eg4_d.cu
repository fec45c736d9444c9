// Exact batched 4 x 4 product kernel instantiations for limb counts 27..32.
#include "lf_eg4.cuh"
LF_EG4_INSTANTIATE(27)
LF_EG4_INSTANTIATE(28)
LF_EG4_INSTANTIATE(29)
LF_EG4_INSTANTIATE(30)
LF_EG4_INSTANTIATE(31)
LF_EG4_INSTANTIATE(32)
