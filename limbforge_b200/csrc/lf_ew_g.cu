// Element-wise kernel instantiations for limb counts: 29 30 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(29)
LF_EW_INSTANTIATE(30)
