// Householder QR panel kernel instantiations for limb counts 25..28.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(25)
LF_QR_INSTANTIATE(26)
LF_QR_INSTANTIATE(27)
LF_QR_INSTANTIATE(28)
