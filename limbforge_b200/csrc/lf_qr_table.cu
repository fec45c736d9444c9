// Width -> Householder QR panel kernel table.
#include "lf_qr.cuh"
namespace lfd {
extern const QrKernels qr_kernels_2;
extern const QrKernels qr_kernels_3;
extern const QrKernels qr_kernels_4;
extern const QrKernels qr_kernels_5;
extern const QrKernels qr_kernels_6;
extern const QrKernels qr_kernels_7;
extern const QrKernels qr_kernels_8;
extern const QrKernels qr_kernels_9;
extern const QrKernels qr_kernels_10;
extern const QrKernels qr_kernels_11;
extern const QrKernels qr_kernels_12;
extern const QrKernels qr_kernels_13;
extern const QrKernels qr_kernels_14;
extern const QrKernels qr_kernels_15;
extern const QrKernels qr_kernels_16;
extern const QrKernels qr_kernels_17;
extern const QrKernels qr_kernels_18;
extern const QrKernels qr_kernels_19;
extern const QrKernels qr_kernels_20;
extern const QrKernels qr_kernels_21;
extern const QrKernels qr_kernels_22;
extern const QrKernels qr_kernels_23;
extern const QrKernels qr_kernels_24;
extern const QrKernels qr_kernels_25;
extern const QrKernels qr_kernels_26;
extern const QrKernels qr_kernels_27;
extern const QrKernels qr_kernels_28;
extern const QrKernels qr_kernels_29;
extern const QrKernels qr_kernels_30;
extern const QrKernels qr_kernels_31;
extern const QrKernels qr_kernels_32;
static const QrKernels* const kQr[33] = {nullptr, nullptr, &qr_kernels_2, &qr_kernels_3, &qr_kernels_4, &qr_kernels_5, &qr_kernels_6, &qr_kernels_7, &qr_kernels_8, &qr_kernels_9, &qr_kernels_10, &qr_kernels_11, &qr_kernels_12, &qr_kernels_13, &qr_kernels_14, &qr_kernels_15, &qr_kernels_16, &qr_kernels_17, &qr_kernels_18, &qr_kernels_19, &qr_kernels_20, &qr_kernels_21, &qr_kernels_22, &qr_kernels_23, &qr_kernels_24, &qr_kernels_25, &qr_kernels_26, &qr_kernels_27, &qr_kernels_28, &qr_kernels_29, &qr_kernels_30, &qr_kernels_31, &qr_kernels_32};
const QrKernels* qr_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kQr[limbs] : nullptr; }
}  // namespace lfd
