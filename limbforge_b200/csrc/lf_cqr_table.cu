// Width -> complex Householder QR panel kernel table.
#include "lf_cqr.cuh"
namespace lfd {
extern const CqrKernels cqr_kernels_2;
extern const CqrKernels cqr_kernels_3;
extern const CqrKernels cqr_kernels_4;
extern const CqrKernels cqr_kernels_5;
extern const CqrKernels cqr_kernels_6;
extern const CqrKernels cqr_kernels_7;
extern const CqrKernels cqr_kernels_8;
extern const CqrKernels cqr_kernels_9;
extern const CqrKernels cqr_kernels_10;
extern const CqrKernels cqr_kernels_11;
extern const CqrKernels cqr_kernels_12;
extern const CqrKernels cqr_kernels_13;
extern const CqrKernels cqr_kernels_14;
extern const CqrKernels cqr_kernels_15;
extern const CqrKernels cqr_kernels_16;
extern const CqrKernels cqr_kernels_17;
extern const CqrKernels cqr_kernels_18;
extern const CqrKernels cqr_kernels_19;
extern const CqrKernels cqr_kernels_20;
extern const CqrKernels cqr_kernels_21;
extern const CqrKernels cqr_kernels_22;
extern const CqrKernels cqr_kernels_23;
extern const CqrKernels cqr_kernels_24;
extern const CqrKernels cqr_kernels_25;
extern const CqrKernels cqr_kernels_26;
extern const CqrKernels cqr_kernels_27;
extern const CqrKernels cqr_kernels_28;
extern const CqrKernels cqr_kernels_29;
extern const CqrKernels cqr_kernels_30;
extern const CqrKernels cqr_kernels_31;
extern const CqrKernels cqr_kernels_32;
static const CqrKernels* const kCqr[33] = {nullptr, nullptr, &cqr_kernels_2, &cqr_kernels_3, &cqr_kernels_4, &cqr_kernels_5, &cqr_kernels_6, &cqr_kernels_7, &cqr_kernels_8, &cqr_kernels_9, &cqr_kernels_10, &cqr_kernels_11, &cqr_kernels_12, &cqr_kernels_13, &cqr_kernels_14, &cqr_kernels_15, &cqr_kernels_16, &cqr_kernels_17, &cqr_kernels_18, &cqr_kernels_19, &cqr_kernels_20, &cqr_kernels_21, &cqr_kernels_22, &cqr_kernels_23, &cqr_kernels_24, &cqr_kernels_25, &cqr_kernels_26, &cqr_kernels_27, &cqr_kernels_28, &cqr_kernels_29, &cqr_kernels_30, &cqr_kernels_31, &cqr_kernels_32};
const CqrKernels* cqr_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kCqr[limbs] : nullptr; }
}  // namespace lfd
