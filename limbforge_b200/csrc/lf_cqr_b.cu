// Complex Householder QR panel kernel instantiations for limb counts 8..12.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(8)
LF_CQR_INSTANTIATE(9)
LF_CQR_INSTANTIATE(10)
LF_CQR_INSTANTIATE(11)
LF_CQR_INSTANTIATE(12)
