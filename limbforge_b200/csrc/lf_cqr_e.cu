// Complex Householder QR panel kernel instantiations for limb counts 22..25.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(22)
LF_CQR_INSTANTIATE(23)
LF_CQR_INSTANTIATE(24)
LF_CQR_INSTANTIATE(25)
