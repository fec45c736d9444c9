// Width -> launcher tables for the cast, tree-sum, segmented-dot and recurrence kernels.
#include "lf_reduce.cuh"
namespace lfd {
int cast_launch_2(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_2(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_3(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_3(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_4(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_4(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_5(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_5(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_6(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_6(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_7(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_7(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_8(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_8(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_9(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_9(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_10(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_10(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_11(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_11(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_12(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_12(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_13(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_13(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_14(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_14(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_15(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_15(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_16(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_16(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_17(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_17(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_18(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_18(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_19(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_19(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_20(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_20(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_21(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_21(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_22(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_22(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_23(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_23(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_24(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_24(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_25(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_25(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_26(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_26(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_27(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_27(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_28(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_28(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_29(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_29(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_30(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_30(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_31(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_31(bool, const u32*, u32*, u64, cudaStream_t);
int cast_launch_32(const u32*, u32*, u64, int, cudaStream_t); int tree_level_launch_32(bool, const u32*, u32*, u64, cudaStream_t);
static const CastLauncher kCast[33] = {nullptr, nullptr, cast_launch_2, cast_launch_3, cast_launch_4, cast_launch_5, cast_launch_6, cast_launch_7, cast_launch_8, cast_launch_9, cast_launch_10, cast_launch_11, cast_launch_12, cast_launch_13, cast_launch_14, cast_launch_15, cast_launch_16, cast_launch_17, cast_launch_18, cast_launch_19, cast_launch_20, cast_launch_21, cast_launch_22, cast_launch_23, cast_launch_24, cast_launch_25, cast_launch_26, cast_launch_27, cast_launch_28, cast_launch_29, cast_launch_30, cast_launch_31, cast_launch_32};
static const TreeLevelLauncher kTree[33] = {nullptr, nullptr, tree_level_launch_2, tree_level_launch_3, tree_level_launch_4, tree_level_launch_5, tree_level_launch_6, tree_level_launch_7, tree_level_launch_8, tree_level_launch_9, tree_level_launch_10, tree_level_launch_11, tree_level_launch_12, tree_level_launch_13, tree_level_launch_14, tree_level_launch_15, tree_level_launch_16, tree_level_launch_17, tree_level_launch_18, tree_level_launch_19, tree_level_launch_20, tree_level_launch_21, tree_level_launch_22, tree_level_launch_23, tree_level_launch_24, tree_level_launch_25, tree_level_launch_26, tree_level_launch_27, tree_level_launch_28, tree_level_launch_29, tree_level_launch_30, tree_level_launch_31, tree_level_launch_32};
CastLauncher cast_launcher(int limbs) { return limbs >= 2 && limbs <= 32 ? kCast[limbs] : nullptr; }
TreeLevelLauncher tree_level_launcher(int limbs) { return limbs >= 2 && limbs <= 32 ? kTree[limbs] : nullptr; }
extern const SequenceLaunchers sequence_launchers_2;
extern const SequenceLaunchers sequence_launchers_3;
extern const SequenceLaunchers sequence_launchers_4;
extern const SequenceLaunchers sequence_launchers_5;
extern const SequenceLaunchers sequence_launchers_6;
extern const SequenceLaunchers sequence_launchers_7;
extern const SequenceLaunchers sequence_launchers_8;
extern const SequenceLaunchers sequence_launchers_9;
extern const SequenceLaunchers sequence_launchers_10;
extern const SequenceLaunchers sequence_launchers_11;
extern const SequenceLaunchers sequence_launchers_12;
extern const SequenceLaunchers sequence_launchers_13;
extern const SequenceLaunchers sequence_launchers_14;
extern const SequenceLaunchers sequence_launchers_15;
extern const SequenceLaunchers sequence_launchers_16;
extern const SequenceLaunchers sequence_launchers_17;
extern const SequenceLaunchers sequence_launchers_18;
extern const SequenceLaunchers sequence_launchers_19;
extern const SequenceLaunchers sequence_launchers_20;
extern const SequenceLaunchers sequence_launchers_21;
extern const SequenceLaunchers sequence_launchers_22;
extern const SequenceLaunchers sequence_launchers_23;
extern const SequenceLaunchers sequence_launchers_24;
extern const SequenceLaunchers sequence_launchers_25;
extern const SequenceLaunchers sequence_launchers_26;
extern const SequenceLaunchers sequence_launchers_27;
extern const SequenceLaunchers sequence_launchers_28;
extern const SequenceLaunchers sequence_launchers_29;
extern const SequenceLaunchers sequence_launchers_30;
extern const SequenceLaunchers sequence_launchers_31;
extern const SequenceLaunchers sequence_launchers_32;
static const SequenceLaunchers* const kSeq[33] = {nullptr, nullptr, &sequence_launchers_2, &sequence_launchers_3, &sequence_launchers_4, &sequence_launchers_5, &sequence_launchers_6, &sequence_launchers_7, &sequence_launchers_8, &sequence_launchers_9, &sequence_launchers_10, &sequence_launchers_11, &sequence_launchers_12, &sequence_launchers_13, &sequence_launchers_14, &sequence_launchers_15, &sequence_launchers_16, &sequence_launchers_17, &sequence_launchers_18, &sequence_launchers_19, &sequence_launchers_20, &sequence_launchers_21, &sequence_launchers_22, &sequence_launchers_23, &sequence_launchers_24, &sequence_launchers_25, &sequence_launchers_26, &sequence_launchers_27, &sequence_launchers_28, &sequence_launchers_29, &sequence_launchers_30, &sequence_launchers_31, &sequence_launchers_32};
const SequenceLaunchers* sequence_launchers(int limbs) { return limbs >= 2 && limbs <= 32 ? kSeq[limbs] : nullptr; }
}  // namespace lfd
