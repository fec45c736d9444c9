// Householder QR panel kernel instantiations for limb counts 29..32.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(29)
LF_QR_INSTANTIATE(30)
LF_QR_INSTANTIATE(31)
LF_QR_INSTANTIATE(32)
