// Element-wise kernel instantiations for limb counts: 21 22 23 24 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(21)
LF_EW_INSTANTIATE(22)
LF_EW_INSTANTIATE(23)
LF_EW_INSTANTIATE(24)
