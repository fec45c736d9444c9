// Householder QR panel kernel instantiations for limb counts 22..24.
#include "lf_qr.cuh"
LF_QR_INSTANTIATE(22)
LF_QR_INSTANTIATE(23)
LF_QR_INSTANTIATE(24)
