// Complex Householder QR panel kernel instantiations for limb counts 29..30.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(29)
LF_CQR_INSTANTIATE(30)
