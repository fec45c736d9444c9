// Element-wise kernel instantiations for limb counts: 9 10 11 12 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(9)
LF_EW_INSTANTIATE(10)
LF_EW_INSTANTIATE(11)
LF_EW_INSTANTIATE(12)
