// Element-wise kernel instantiations for limb counts: 13 14 15 16 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(13)
LF_EW_INSTANTIATE(14)
LF_EW_INSTANTIATE(15)
LF_EW_INSTANTIATE(16)
