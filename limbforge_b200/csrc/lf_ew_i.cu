// Element-wise kernel instantiations for limb counts: 31 32 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(31)
LF_EW_INSTANTIATE(32)
