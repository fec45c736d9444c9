// Complex Householder QR panel kernel instantiations for limb counts 31..32.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(31)
LF_CQR_INSTANTIATE(32)
