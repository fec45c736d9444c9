// Complex Householder QR panel kernel instantiations for limb counts 13..17.
#include "lf_cqr.cuh"
LF_CQR_INSTANTIATE(13)
LF_CQR_INSTANTIATE(14)
LF_CQR_INSTANTIATE(15)
LF_CQR_INSTANTIATE(16)
LF_CQR_INSTANTIATE(17)
