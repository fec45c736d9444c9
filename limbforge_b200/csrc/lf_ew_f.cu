// Element-wise kernel instantiations for limb counts: 25 26 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(25)
LF_EW_INSTANTIATE(26)
