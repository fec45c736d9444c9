// Householder QR panel kernel instantiations for limb counts 2..5.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(2)
LF_QR_INSTANTIATE(3)
LF_QR_INSTANTIATE(4)
LF_QR_INSTANTIATE(5)
