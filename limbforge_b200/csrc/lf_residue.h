// Int8-residue / CRT engine for exact dense products (tcgen05 kind::i8 MMAs, TMEM int32
// accumulators, one rounding per output).  run() returns false when the product is outside the
// engine's domain (the caller then uses the generic limb kernel, which gives identical bits).
#pragma once
#include "lf_linalg.cuh"
#include "lf_runtime.h"

namespace lfr {

struct ResidueEngine {
    DevBuf lines, planes, residues, tables, misc;
    bool run(int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc, uint64_t K, uint32_t* C,
             uint64_t ldc, bool subtract, bool lower, uint32_t* error, cudaStream_t s, bool forced, lf_linalg_report& report);
};

}  // namespace lfr
