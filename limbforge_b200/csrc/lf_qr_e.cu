// Householder QR panel kernel instantiations for limb counts 18..21.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(18)
LF_QR_INSTANTIATE(19)
LF_QR_INSTANTIATE(20)
LF_QR_INSTANTIATE(21)
