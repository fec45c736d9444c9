// Element-wise kernel instantiations for limb counts: 2 3 4 5 6 7 8 (split so the widths compile in parallel).
#include "lf_elementwise.cuh"
LF_EW_INSTANTIATE(2)
LF_EW_INSTANTIATE(3)
LF_EW_INSTANTIATE(4)
LF_EW_INSTANTIATE(5)
LF_EW_INSTANTIATE(6)
LF_EW_INSTANTIATE(7)
LF_EW_INSTANTIATE(8)
