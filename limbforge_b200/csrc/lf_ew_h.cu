// Element-wise kernel instantiations for limb counts: 27 28 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(27)
LF_EW_INSTANTIATE(28)
