// Complex Householder QR panel kernel instantiations for limb counts 2..7.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(2)
LF_CQR_INSTANTIATE(3)
LF_CQR_INSTANTIATE(4)
LF_CQR_INSTANTIATE(5)
LF_CQR_INSTANTIATE(6)
LF_CQR_INSTANTIATE(7)
