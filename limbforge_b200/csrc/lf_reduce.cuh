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

// ---- Segmented dot products (Engine::segmented_dot, engine.hpp:30-32,205; kernels.metal:195-207):
// out[i] = the sequential fused chain s <- fma(a_ik, b_k, s) from s = 0, k = 0..length-1 (cfma for complex),
// with b_k = b[i * length + k], or b[k] when the right operand is shared.  One thread per segment.
template <int N, bool CX, bool SHARED> __global__ void __launch_bounds__(128) segdot_kernel(const u32* a, const u32* b, u32* out,
                                                                                            u64 segments, u64 length) {
    const u64 i = (u64)blockIdx.x * 128 + threadIdx.x;
    if (i >= segments) return;
    constexpr u64 S = CX ? 2 * (N + 3) : N + 3;
    const u64 base = i * length;
    if constexpr (CX) {
        Cpx<N> s = {zero<N>(), zero<N>()};
        for (u64 k = 0; k < length; ++k) s = cfma<N>(cload<N>(a + (base + k) * S), cload<N>(b + (SHARED ? k : base + k) * S), s);
        cstore<N>(out + i * S, s);
    } else {
        Num<N> s = zero<N>();
        for (u64 k = 0; k < length; ++k) s = fma<N>(load<N>(a + (base + k) * S), load<N>(b + (SHARED ? k : base + k) * S), s);
        store<N>(out + i * S, s);
    }
}
// ---- Four-term complex recurrence (Engine::recurrence, engine.hpp:218-223; kernels.metal:39-58): instance i keeps
// the ring (q0, q1, q2, q3) = seeds[j * count + i]; each step forms q = cadd(... cadd(0, cmul(w_0, q0)) ..., cmul(w_3, q3))
// in that order with w_j = weights[(step * 4 + j) * (count / spw) + i / spw], then shifts the ring (q0 <- q1, ..., q3 <- q).
// The output is q3.  One thread per instance.
template <int N> __global__ void __launch_bounds__(128) recurrence_kernel(const u32* seeds, const u32* weights, u32* out, u64 count,
                                                                          unsigned steps, unsigned spw) {
    const u64 i = (u64)blockIdx.x * 128 + threadIdx.x;
    if (i >= count) return;
    constexpr u64 S = 2 * (N + 3);
    Cpx<N> q0 = cload<N>(seeds + i * S), q1 = cload<N>(seeds + (count + i) * S), q2 = cload<N>(seeds + (2 * count + i) * S),
           q3 = cload<N>(seeds + (3 * count + i) * S);
    const u64 G = count / spw, g = i / spw;
    for (unsigned t = 0; t < steps; ++t) {
        const u32* w = weights + ((u64)t * 4 * G + g) * S;
        Cpx<N> sum = {zero<N>(), zero<N>()};
        sum = cadd<N>(sum, cmul<N>(cload<N>(w), q0));
        sum = cadd<N>(sum, cmul<N>(cload<N>(w + G * S), q1));
        sum = cadd<N>(sum, cmul<N>(cload<N>(w + 2 * G * S), q2));
        sum = cadd<N>(sum, cmul<N>(cload<N>(w + 3 * G * S), q3));
        q0 = q1; q1 = q2; q2 = q3; q3 = sum;
    }
    cstore<N>(out + i * S, q3);
}
template <int N> int launch_segdot_n(bool cx, bool shared, const u32* a, const u32* b, u32* out, u64 segments, u64 length, cudaStream_t s) {
    if (!segments) return 0;
    const unsigned blocks = (unsigned)((segments + 127) / 128);
    if (cx) { if (shared) segdot_kernel<N, true, true><<<blocks, 128, 0, s>>>(a, b, out, segments, length);
              else segdot_kernel<N, true, false><<<blocks, 128, 0, s>>>(a, b, out, segments, length); }
    else { if (shared) segdot_kernel<N, false, true><<<blocks, 128, 0, s>>>(a, b, out, segments, length);
           else segdot_kernel<N, false, false><<<blocks, 128, 0, s>>>(a, b, out, segments, length); }
    return 0;
}
template <int N> int launch_recurrence_n(const u32* seeds, const u32* weights, u32* out, u64 count, unsigned steps, unsigned spw, cudaStream_t s) {
    if (!count) return 0;
    recurrence_kernel<N><<<(unsigned)((count + 127) / 128), 128, 0, s>>>(seeds, weights, out, count, steps, spw);
    return 0;
}
typedef int (*SegDotLauncher)(bool, bool, const u32*, const u32*, u32*, u64, u64, cudaStream_t);
typedef int (*RecurrenceLauncher)(const u32*, const u32*, u32*, u64, unsigned, unsigned, cudaStream_t);
struct SequenceLaunchers { SegDotLauncher segdot; RecurrenceLauncher recurrence; };
const SequenceLaunchers* sequence_launchers(int limbs);

}  // namespace lfd

#define LF_REDUCE_INSTANTIATE(N)                                                                          \
    namespace lfd {                                                                                       \
    int cast_launch_##N(const u32* i, u32* o, u64 c, int w, cudaStream_t s) { return launch_cast_n<N>(i, o, c, w, s); } \
    int tree_level_launch_##N(bool cx, const u32* i, u32* o, u64 c, cudaStream_t s) { return launch_tree_level_n<N>(cx, i, o, c, s); } \
    extern const SequenceLaunchers sequence_launchers_##N; const SequenceLaunchers sequence_launchers_##N = {launch_segdot_n<N>, launch_recurrence_n<N>}; \
    }
