// Complex Householder QR panel kernel instantiations for limb counts 18..21.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(18)
LF_CQR_INSTANTIATE(19)
LF_CQR_INSTANTIATE(20)
LF_CQR_INSTANTIATE(21)
