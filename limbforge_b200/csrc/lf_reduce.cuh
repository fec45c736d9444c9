// Precision casts and tree sums (the reference's Engine::cast / CommandBatch::cast and
// CommandBatch::tree_sum: engine.hpp:150-175, kernels.metal:60-112 and 251-266).
//  - cast: exact widening and round-to-nearest-even narrowing between any two widths, complex
//    componentwise.  A status element or a zero becomes a zero carrying that status.
//  - tree sum: the fixed adjacent-pair tree.  Each level adds elements 2i and 2i+1 (cadd for complex),
//    an odd last element is carried without a rounding, and the levels repeat until one element is
//    left.  An empty input sums to zero.  Every level is one launch.
#pragma once
#include "lf_arith.cuh"
#include <cuda_runtime.h>

namespace lfd {

// One component per thread; from_words source limbs (2..32), the target width N.
template <int N> __global__ void __launch_bounds__(128) cast_kernel(const u32* in, u32* out, u64 count, int from_words) {
    const u64 i = (u64)blockIdx.x * 128 + threadIdx.x;
    if (i >= count) return;
    const u32* src = in + i * (u64)(from_words + 3);
    const u32 st = src[from_words + 2];
    const int sign = (int)src[from_words + 1];
    u32* dst = out + i * (u64)(N + 3);
    if (st || !sign) { store<N>(dst, zero<N>(st)); return; }
    u32 x[33];
#pragma unroll
    for (int w = 0; w < 33; ++w) x[w] = w < from_words ? src[w] : 0u;
    store<N>(dst, round_general<N, 33>(x, (i64)(int)src[from_words] - (32 * (i64)from_words - 1), sign, 0));
}

// One level of the tree: out[i] = in[2i] + in[2i+1] (or in[2i] for an odd last element).
template <int N, bool CX> __global__ void __launch_bounds__(128) tree_level_kernel(const u32* in, u32* out, u64 count) {
    const u64 i = (u64)blockIdx.x * 128 + threadIdx.x;
    constexpr u64 E = N + 3;
    if (!count) {
        if (!i) { store<N>(out, zero<N>()); if (CX) store<N>(out + E, zero<N>()); }
        return;
    }
    if (i >= (count + 1) / 2) return;
    const u64 j = 2 * i;
    if constexpr (CX) {
        Cpx<N> x = cload<N>(in + 2 * E * j);
        if (j + 1 < count) x = cadd<N>(x, cload<N>(in + 2 * E * (j + 1)));
        cstore<N>(out + 2 * E * i, x);
    } else {
        Num<N> x = load<N>(in + E * j);
        if (j + 1 < count) x = add<N>(x, load<N>(in + E * (j + 1)));
        store<N>(out + E * i, x);
    }
}

template <int N> int launch_cast_n(const u32* in, u32* out, u64 count, int from_words, cudaStream_t s) {
    if (!count) return 0;
    cast_kernel<N><<<(unsigned)((count + 127) / 128), 128, 0, s>>>(in, out, count, from_words);
    return 0;
}
template <int N> int launch_tree_level_n(bool cx, const u32* in, u32* out, u64 count, cudaStream_t s) {
    const u64 threads = count ? (count + 1) / 2 : 1;
    const unsigned blocks = (unsigned)((threads + 127) / 128);
    if (cx) tree_level_kernel<N, true><<<blocks, 128, 0, s>>>(in, out, count);
    else tree_level_kernel<N, false><<<blocks, 128, 0, s>>>(in, out, count);
    return 0;
}
typedef int (*CastLauncher)(const u32*, u32*, u64, int, cudaStream_t);
typedef int (*TreeLevelLauncher)(bool, const u32*, u32*, u64, cudaStream_t);
CastLauncher cast_launcher(int limbs);
TreeLevelLauncher tree_level_launcher(int limbs);

}  // namespace lfd

#define LF_REDUCE_INSTANTIATE(N)                                                                          \
    namespace lfd {                                                                                       \
    int cast_launch_##N(const u32* i, u32* o, u64 c, int w, cudaStream_t s) { return launch_cast_n<N>(i, o, c, w, s); } \
    int tree_level_launch_##N(bool cx, const u32* i, u32* o, u64 c, cudaStream_t s) { return launch_tree_level_n<N>(cx, i, o, c, s); } \
    }
