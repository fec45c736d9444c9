// Complex Householder QR panel kernel instantiations for limb counts 26..28.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(26)
LF_CQR_INSTANTIATE(27)
LF_CQR_INSTANTIATE(28)
