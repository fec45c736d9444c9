// Householder QR panel kernel instantiations for limb counts 14..17.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(14)
LF_QR_INSTANTIATE(15)
LF_QR_INSTANTIATE(16)
LF_QR_INSTANTIATE(17)
