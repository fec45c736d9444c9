// Width -> exact batched 4 x 4 product kernel table.
#include "lf_eg4.cuh"
namespace lfd {
extern const Eg4Kernels eg4_kernels_2;
extern const Eg4Kernels eg4_kernels_3;
extern const Eg4Kernels eg4_kernels_4;
extern const Eg4Kernels eg4_kernels_5;
extern const Eg4Kernels eg4_kernels_6;
extern const Eg4Kernels eg4_kernels_7;
extern const Eg4Kernels eg4_kernels_8;
extern const Eg4Kernels eg4_kernels_9;
extern const Eg4Kernels eg4_kernels_10;
extern const Eg4Kernels eg4_kernels_11;
extern const Eg4Kernels eg4_kernels_12;
extern const Eg4Kernels eg4_kernels_13;
extern const Eg4Kernels eg4_kernels_14;
extern const Eg4Kernels eg4_kernels_15;
extern const Eg4Kernels eg4_kernels_16;
extern const Eg4Kernels eg4_kernels_17;
extern const Eg4Kernels eg4_kernels_18;
extern const Eg4Kernels eg4_kernels_19;
extern const Eg4Kernels eg4_kernels_20;
extern const Eg4Kernels eg4_kernels_21;
extern const Eg4Kernels eg4_kernels_22;
extern const Eg4Kernels eg4_kernels_23;
extern const Eg4Kernels eg4_kernels_24;
extern const Eg4Kernels eg4_kernels_25;
extern const Eg4Kernels eg4_kernels_26;
extern const Eg4Kernels eg4_kernels_27;
extern const Eg4Kernels eg4_kernels_28;
extern const Eg4Kernels eg4_kernels_29;
extern const Eg4Kernels eg4_kernels_30;
extern const Eg4Kernels eg4_kernels_31;
extern const Eg4Kernels eg4_kernels_32;
static const Eg4Kernels* const kEg4[33] = {nullptr, nullptr, &eg4_kernels_2, &eg4_kernels_3, &eg4_kernels_4, &eg4_kernels_5, &eg4_kernels_6, &eg4_kernels_7, &eg4_kernels_8, &eg4_kernels_9, &eg4_kernels_10, &eg4_kernels_11, &eg4_kernels_12, &eg4_kernels_13, &eg4_kernels_14, &eg4_kernels_15, &eg4_kernels_16, &eg4_kernels_17, &eg4_kernels_18, &eg4_kernels_19, &eg4_kernels_20, &eg4_kernels_21, &eg4_kernels_22, &eg4_kernels_23, &eg4_kernels_24, &eg4_kernels_25, &eg4_kernels_26, &eg4_kernels_27, &eg4_kernels_28, &eg4_kernels_29, &eg4_kernels_30, &eg4_kernels_31, &eg4_kernels_32};
const Eg4Kernels* eg4_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kEg4[limbs] : nullptr; }
}  // namespace lfd
