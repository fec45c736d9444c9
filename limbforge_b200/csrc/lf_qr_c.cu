// Householder QR panel kernel instantiations for limb counts 10..13.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(10)
LF_QR_INSTANTIATE(11)
LF_QR_INSTANTIATE(12)
LF_QR_INSTANTIATE(13)
