// Width -> kernel tables of the exact products, factorizations and the residue engine.
#include "lf_residue.cuh"
namespace lfd {
extern const LinalgKernels linalg_kernels_2; extern const FactorKernels factor_kernels_2; extern const ResidueKernels residue_kernels_2;
extern const LinalgKernels linalg_kernels_3; extern const FactorKernels factor_kernels_3; extern const ResidueKernels residue_kernels_3;
extern const LinalgKernels linalg_kernels_4; extern const FactorKernels factor_kernels_4; extern const ResidueKernels residue_kernels_4;
extern const LinalgKernels linalg_kernels_5; extern const FactorKernels factor_kernels_5; extern const ResidueKernels residue_kernels_5;
extern const LinalgKernels linalg_kernels_6; extern const FactorKernels factor_kernels_6; extern const ResidueKernels residue_kernels_6;
extern const LinalgKernels linalg_kernels_7; extern const FactorKernels factor_kernels_7; extern const ResidueKernels residue_kernels_7;
extern const LinalgKernels linalg_kernels_8; extern const FactorKernels factor_kernels_8; extern const ResidueKernels residue_kernels_8;
extern const LinalgKernels linalg_kernels_9; extern const FactorKernels factor_kernels_9; extern const ResidueKernels residue_kernels_9;
extern const LinalgKernels linalg_kernels_10; extern const FactorKernels factor_kernels_10; extern const ResidueKernels residue_kernels_10;
extern const LinalgKernels linalg_kernels_11; extern const FactorKernels factor_kernels_11; extern const ResidueKernels residue_kernels_11;
extern const LinalgKernels linalg_kernels_12; extern const FactorKernels factor_kernels_12; extern const ResidueKernels residue_kernels_12;
extern const LinalgKernels linalg_kernels_13; extern const FactorKernels factor_kernels_13; extern const ResidueKernels residue_kernels_13;
extern const LinalgKernels linalg_kernels_14; extern const FactorKernels factor_kernels_14; extern const ResidueKernels residue_kernels_14;
extern const LinalgKernels linalg_kernels_15; extern const FactorKernels factor_kernels_15; extern const ResidueKernels residue_kernels_15;
extern const LinalgKernels linalg_kernels_16; extern const FactorKernels factor_kernels_16; extern const ResidueKernels residue_kernels_16;
extern const LinalgKernels linalg_kernels_17; extern const FactorKernels factor_kernels_17; extern const ResidueKernels residue_kernels_17;
extern const LinalgKernels linalg_kernels_18; extern const FactorKernels factor_kernels_18; extern const ResidueKernels residue_kernels_18;
extern const LinalgKernels linalg_kernels_19; extern const FactorKernels factor_kernels_19; extern const ResidueKernels residue_kernels_19;
extern const LinalgKernels linalg_kernels_20; extern const FactorKernels factor_kernels_20; extern const ResidueKernels residue_kernels_20;
extern const LinalgKernels linalg_kernels_21; extern const FactorKernels factor_kernels_21; extern const ResidueKernels residue_kernels_21;
extern const LinalgKernels linalg_kernels_22; extern const FactorKernels factor_kernels_22; extern const ResidueKernels residue_kernels_22;
extern const LinalgKernels linalg_kernels_23; extern const FactorKernels factor_kernels_23; extern const ResidueKernels residue_kernels_23;
extern const LinalgKernels linalg_kernels_24; extern const FactorKernels factor_kernels_24; extern const ResidueKernels residue_kernels_24;
extern const LinalgKernels linalg_kernels_25; extern const FactorKernels factor_kernels_25; extern const ResidueKernels residue_kernels_25;
extern const LinalgKernels linalg_kernels_26; extern const FactorKernels factor_kernels_26; extern const ResidueKernels residue_kernels_26;
extern const LinalgKernels linalg_kernels_27; extern const FactorKernels factor_kernels_27; extern const ResidueKernels residue_kernels_27;
extern const LinalgKernels linalg_kernels_28; extern const FactorKernels factor_kernels_28; extern const ResidueKernels residue_kernels_28;
extern const LinalgKernels linalg_kernels_29; extern const FactorKernels factor_kernels_29; extern const ResidueKernels residue_kernels_29;
extern const LinalgKernels linalg_kernels_30; extern const FactorKernels factor_kernels_30; extern const ResidueKernels residue_kernels_30;
extern const LinalgKernels linalg_kernels_31; extern const FactorKernels factor_kernels_31; extern const ResidueKernels residue_kernels_31;
extern const LinalgKernels linalg_kernels_32; extern const FactorKernels factor_kernels_32; extern const ResidueKernels residue_kernels_32;
static const LinalgKernels* const kLinalg[33] = {nullptr, nullptr, &linalg_kernels_2, &linalg_kernels_3, &linalg_kernels_4, &linalg_kernels_5, &linalg_kernels_6, &linalg_kernels_7, &linalg_kernels_8, &linalg_kernels_9, &linalg_kernels_10, &linalg_kernels_11, &linalg_kernels_12, &linalg_kernels_13, &linalg_kernels_14, &linalg_kernels_15, &linalg_kernels_16, &linalg_kernels_17, &linalg_kernels_18, &linalg_kernels_19, &linalg_kernels_20, &linalg_kernels_21, &linalg_kernels_22, &linalg_kernels_23, &linalg_kernels_24, &linalg_kernels_25, &linalg_kernels_26, &linalg_kernels_27, &linalg_kernels_28, &linalg_kernels_29, &linalg_kernels_30, &linalg_kernels_31, &linalg_kernels_32};
static const FactorKernels* const kFactor[33] = {nullptr, nullptr, &factor_kernels_2, &factor_kernels_3, &factor_kernels_4, &factor_kernels_5, &factor_kernels_6, &factor_kernels_7, &factor_kernels_8, &factor_kernels_9, &factor_kernels_10, &factor_kernels_11, &factor_kernels_12, &factor_kernels_13, &factor_kernels_14, &factor_kernels_15, &factor_kernels_16, &factor_kernels_17, &factor_kernels_18, &factor_kernels_19, &factor_kernels_20, &factor_kernels_21, &factor_kernels_22, &factor_kernels_23, &factor_kernels_24, &factor_kernels_25, &factor_kernels_26, &factor_kernels_27, &factor_kernels_28, &factor_kernels_29, &factor_kernels_30, &factor_kernels_31, &factor_kernels_32};
static const ResidueKernels* const kResidue[33] = {nullptr, nullptr, &residue_kernels_2, &residue_kernels_3, &residue_kernels_4, &residue_kernels_5, &residue_kernels_6, &residue_kernels_7, &residue_kernels_8, &residue_kernels_9, &residue_kernels_10, &residue_kernels_11, &residue_kernels_12, &residue_kernels_13, &residue_kernels_14, &residue_kernels_15, &residue_kernels_16, &residue_kernels_17, &residue_kernels_18, &residue_kernels_19, &residue_kernels_20, &residue_kernels_21, &residue_kernels_22, &residue_kernels_23, &residue_kernels_24, &residue_kernels_25, &residue_kernels_26, &residue_kernels_27, &residue_kernels_28, &residue_kernels_29, &residue_kernels_30, &residue_kernels_31, &residue_kernels_32};
const LinalgKernels* linalg_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kLinalg[limbs] : nullptr; }
const FactorKernels* factor_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kFactor[limbs] : nullptr; }
const ResidueKernels* residue_kernels(int limbs) { return limbs >= 2 && limbs <= 32 ? kResidue[limbs] : nullptr; }
}  // namespace lfd
