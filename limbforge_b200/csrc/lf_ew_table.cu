// Width -> launcher tables for the element-wise and chain kernels.
#include "lf_elementwise.cuh"

namespace lfd {
#define LF_DECL(N) int ew_launch_##N(int, const EwParams&, cudaStream_t); int chain_launch_##N(const ChainParams&, cudaStream_t); \
    int ew_attr_##N(int, cudaFuncAttributes*);
LF_DECL(2) LF_DECL(3) LF_DECL(4) LF_DECL(5) LF_DECL(6) LF_DECL(7) LF_DECL(8) LF_DECL(9) LF_DECL(10) LF_DECL(11)
LF_DECL(12) LF_DECL(13) LF_DECL(14) LF_DECL(15) LF_DECL(16) LF_DECL(17) LF_DECL(18) LF_DECL(19) LF_DECL(20)
LF_DECL(21) LF_DECL(22) LF_DECL(23) LF_DECL(24) LF_DECL(25) LF_DECL(26) LF_DECL(27) LF_DECL(28) LF_DECL(29)
LF_DECL(30) LF_DECL(31) LF_DECL(32)
#undef LF_DECL
#define LF_ROW(N) ew_launch_##N,
static const EwLauncher kEw[33] = {nullptr, nullptr, LF_ROW(2) LF_ROW(3) LF_ROW(4) LF_ROW(5) LF_ROW(6) LF_ROW(7) LF_ROW(8)
    LF_ROW(9) LF_ROW(10) LF_ROW(11) LF_ROW(12) LF_ROW(13) LF_ROW(14) LF_ROW(15) LF_ROW(16) LF_ROW(17) LF_ROW(18) LF_ROW(19)
    LF_ROW(20) LF_ROW(21) LF_ROW(22) LF_ROW(23) LF_ROW(24) LF_ROW(25) LF_ROW(26) LF_ROW(27) LF_ROW(28) LF_ROW(29) LF_ROW(30)
    LF_ROW(31) LF_ROW(32)};
#undef LF_ROW
#define LF_ROW(N) chain_launch_##N,
static const ChainLauncher kChain[33] = {nullptr, nullptr, LF_ROW(2) LF_ROW(3) LF_ROW(4) LF_ROW(5) LF_ROW(6) LF_ROW(7) LF_ROW(8)
    LF_ROW(9) LF_ROW(10) LF_ROW(11) LF_ROW(12) LF_ROW(13) LF_ROW(14) LF_ROW(15) LF_ROW(16) LF_ROW(17) LF_ROW(18) LF_ROW(19)
    LF_ROW(20) LF_ROW(21) LF_ROW(22) LF_ROW(23) LF_ROW(24) LF_ROW(25) LF_ROW(26) LF_ROW(27) LF_ROW(28) LF_ROW(29) LF_ROW(30)
    LF_ROW(31) LF_ROW(32)};
#undef LF_ROW
#define LF_ROW(N) ew_attr_##N,
static const EwAttributes kAttr[33] = {nullptr, nullptr, LF_ROW(2) LF_ROW(3) LF_ROW(4) LF_ROW(5) LF_ROW(6) LF_ROW(7) LF_ROW(8)
    LF_ROW(9) LF_ROW(10) LF_ROW(11) LF_ROW(12) LF_ROW(13) LF_ROW(14) LF_ROW(15) LF_ROW(16) LF_ROW(17) LF_ROW(18) LF_ROW(19)
    LF_ROW(20) LF_ROW(21) LF_ROW(22) LF_ROW(23) LF_ROW(24) LF_ROW(25) LF_ROW(26) LF_ROW(27) LF_ROW(28) LF_ROW(29) LF_ROW(30)
    LF_ROW(31) LF_ROW(32)};
#undef LF_ROW
EwAttributes ew_attributes_of(int limbs) { return limbs >= 2 && limbs <= 32 ? kAttr[limbs] : nullptr; }
EwLauncher ew_launcher(int limbs) { return limbs >= 2 && limbs <= 32 ? kEw[limbs] : nullptr; }
ChainLauncher chain_launcher(int limbs) { return limbs >= 2 && limbs <= 32 ? kChain[limbs] : nullptr; }
}  // namespace lfd
