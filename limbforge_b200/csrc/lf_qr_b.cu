// Householder QR panel kernel instantiations for limb counts 6..9.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(6)
LF_QR_INSTANTIATE(7)
LF_QR_INSTANTIATE(8)
LF_QR_INSTANTIATE(9)
