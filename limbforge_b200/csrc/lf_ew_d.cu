// Element-wise kernel instantiations for limb counts: 17 18 19 20 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(17)
LF_EW_INSTANTIATE(18)
LF_EW_INSTANTIATE(19)
LF_EW_INSTANTIATE(20)
