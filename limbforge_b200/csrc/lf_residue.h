// Int8-residue / CRT engine for exact dense products (tcgen05 kind::i8 MMAs, TMEM int32
// accumulators, one rounding per output).  run() returns false when the product is outside the
// engine's domain (the caller then uses the generic limb kernel, which gives identical bits).
#pragma once
#include <memory>
#include "lf_linalg.cuh"
#include "lf_runtime.h"

namespace lfr {

struct ResidueEngine {
    DevBuf lines, planes, residues, tables, misc;
    size_t bytes() const { return lines.bytes + planes.bytes + residues.bytes + tables.bytes + misc.bytes; }
    void release() { lines = DevBuf{}; planes = DevBuf{}; residues = DevBuf{}; tables = DevBuf{}; misc = DevBuf{}; }
    bool run(int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc, uint64_t K, uint32_t* C,
             uint64_t ldc, bool subtract, bool lower, uint32_t* error, cudaStream_t s, bool forced, lf_linalg_report& report);
};

}  // namespace lfr

// Pieces of the engine for callers that supply every device buffer (the allocation-free entry point).
#include <cuda.h>
namespace lfd { struct ResTables; struct MmaParams; }
namespace lfr {
int residue_moduli_for(int bits, int G, uint64_t K);      // modulus count L, 0 above the table limit
int residue_max_band();
uint64_t residue_max_k();
void residue_tables_host(int L, lfd::ResTables& tables, int& qwords);
CUtensorMap residue_plane_map(void* base, uint64_t Kp, uint64_t rows_pad, int L);
void residue_mma_launch(dim3 grid, const CUtensorMap& ta1, const CUtensorMap& ta0, const CUtensorMap& tb1, const CUtensorMap& tb0,
                        const lfd::MmaParams& p, cudaStream_t s);
}  // namespace lfr

// Resident products planned on the GPU (Linalg::syrk / gemm on a CommandBatch): set up at record time for
// every modulus count the product could need; launched at submit with no host round trip (line
// analysis, plan, digit planes, residue products, CRT or the limb kernel, all on the stream).
namespace lfr {
struct ResidentProduct;
std::shared_ptr<ResidentProduct> resident_product_create(int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc,
                                                         uint64_t K, uint32_t* C, uint64_t ldc, bool subtract, bool lower,
                                                         bool mirror, bool limb_only);
void resident_product_launch(ResidentProduct& r, cudaStream_t s);
bool resident_product_done(ResidentProduct& r);              // the launch has completed on the GPU
size_t resident_product_bytes(const ResidentProduct& r);     // device workspace the product holds now
void resident_product_hold(ResidentProduct& r, bool held);  // recorded in a live batch, or that batch is gone
// Busy: recorded in a live batch and not launched yet, or launched and not completed.
bool resident_product_busy(ResidentProduct& r);
// Frees the product's device workspace unless it is busy (a completed product keeps its report on the host);
// returns the bytes freed.
size_t resident_product_release(ResidentProduct& r);
// Fills the engine, modulus count and band; returns false when a cluster overflowed the exact window.
bool resident_product_report(ResidentProduct& r, lf_linalg_report& rep);
}  // namespace lfr
