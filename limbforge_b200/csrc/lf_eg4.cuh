// The exact batched 4 x 4 product (the reference's benchmarks/experiments/exact_gemm4: README.md "Contract and
// dispatch", prototype.hpp:5-24): fixed row-major 4 x 4 matrices, matrix t of A, B and C at t * stride elements
// (stride 0 broadcasts an input).  Each real output component is RN(C_old + sum_k a_ik b_kj) with one rounding of the
// exact sum (C_old left out without accumulation), negated when asked; a complex component sums its eight signed real
// products.  Statuses: zero with the OR of every operand the component reads and C_old; no nonzero product gives C_old
// (or zero).  One thread per output component; the exact sum is a register window when the terms' spread fits it, else
// cluster_round over the component's terms (a window per cluster, streamed when a cluster is wider), so every spread
// is summed on the GPU.
#pragma once
#include "lf_linalg.cuh"

namespace lfd {

struct Eg4Params { const u32* A; const u32* B; u32* C; u64 count, sa, sb, sc; int accumulate, negative; };

// Terms of one component: products x_k y_k with signs (k < cnt) and the old value as the last term.
template <int N> struct Eg4Terms {
    const u32* x[8]; const u32* y[8]; int sg[8]; int cnt; Num<N> c;
    __device__ u64 count() const { return (u64)cnt + 1; }
    __device__ bool term(u64 k, i64& scale, i64& top, int& sign) const {
        if ((int)k == cnt) {
            if (!c.s) return false;
            scale = (i64)c.e - (32 * N - 1); top = scale + 32 * N; sign = c.s;
            return true;
        }
        const int sa = (int)x[k][N + 1], sb = (int)y[k][N + 1];
        if (!sa || !sb) return false;
        scale = (i64)(int)x[k][N] + (int)y[k][N] - 2 * (32 * N - 1);
        top = scale + 64 * N;
        sign = sg[k] * sa * sb;
        return true;
    }
    __device__ void add(u64 k, u32* acc, int len, i64 off) const {
        if ((int)k == cnt) { acc_add(acc, len, c.m, N, off); return; }
        const Num<N> a = load_plain<N>(x[k]), b = load_plain<N>(y[k]);
        u32 prod[2 * N];
        mant_mul<N>(a.m, b.m, prod);
        acc_add(acc, len, prod, 2 * N, off);
    }
};

// Register window for components whose terms span at most 32 W - 5 bits (the usual case): every product is added
// exactly into a two's-complement window of W = 2N + 8 words held in registers and rounded once; the term pointers
// follow from the term index, so nothing is indexed at run time.  Wider spreads (and widths above 512 bits, where
// the window would not fit in registers) take cluster_round.  Returns false to ask for the cluster path.
template <int N> constexpr int eg4_window() { return N <= 16 ? 2 * N + 8 : 0; }
template <int N, bool CX> __device__ __forceinline__ void eg4_term(const u32* a, const u32* b, int k, int part, const u32*& x,
                                                                 const u32*& y, int& sg) {
    constexpr u64 E = N + 3, S = CX ? 2 * E : E;
    if (!CX) { x = a + (u64)k * S; y = b + (u64)k * 4 * S; sg = 1; return; }
    const int kk = k >> 1, h = k & 1;
    const u32* ak = a + (u64)kk * S;
    const u32* bk = b + (u64)kk * 4 * S;
    if (part == 0) { x = ak + h * E; y = bk + h * E; sg = h ? -1 : 1; }             // re: a.re b.re - a.im b.im
    else { x = ak + h * E; y = bk + (1 - h) * E; sg = 1; }                        // im: a.re b.im + a.im b.re
}
template <int N, bool CX> __device__ bool eg4_window_sum(const u32* a, const u32* b, int part, const Num<N>& c, Num<N>& out) {
    constexpr int W = eg4_window<N>();
    if constexpr (W == 0) {
        return false;
    } else {
        constexpr int CNT = CX ? 8 : 4;
        i64 lo = INT64_MAX, hi = INT64_MIN;
#pragma unroll 1
        for (int k = 0; k < CNT; ++k) {
            const u32 *x, *y; int sg;
            eg4_term<N, CX>(a, b, k, part, x, y, sg);
            if (!x[N + 1] || !y[N + 1]) continue;
            const i64 sc = (i64)(int)x[N] + (int)y[N] - 2 * (32 * N - 1);
            lo = sc < lo ? sc : lo; hi = sc + 64 * N > hi ? sc + 64 * N : hi;
        }
        const i64 cs = (i64)c.e - (32 * N - 1);
        if (c.s) { lo = cs < lo ? cs : lo; hi = cs + 32 * N > hi ? cs + 32 * N : hi; }
        if (hi - lo + 5 > 32 * (i64)W) return false;
        u32 acc[W], t[W];
#pragma unroll
        for (int w = 0; w < W; ++w) acc[w] = 0;
#pragma unroll 1
        for (int k = 0; k < CNT; ++k) {
            const u32 *x, *y; int sg;
            eg4_term<N, CX>(a, b, k, part, x, y, sg);
            const int sa = (int)x[N + 1], sb = (int)y[N + 1];
            if (!sa || !sb) continue;
            const Num<N> xa = load_plain<N>(x), yb = load_plain<N>(y);
            u32 pr[2 * N];
            mant_mul<N>(xa.m, yb.m, pr);
            place_words<W, 2 * N>(t, pr, (i64)xa.e + yb.e - 2 * (32 * N - 1) - lo);
            accumulate<W>(acc, t, sg * sa * sb < 0);
        }
        if (c.s) {
            place_words<W, N>(t, c.m, cs - lo);
            accumulate<W>(acc, t, c.s < 0);
        }
        int sign = 1;
        if (acc[W - 1] >> 31) {
            sign = -1;
            u64 cy = 1;
#pragma unroll
            for (int w = 0; w < W; ++w) { const u64 v = (u64)(u32)~acc[w] + cy; acc[w] = (u32)v; cy = v >> 32; }
        }
        u32 any = 0;
#pragma unroll
        for (int w = 0; w < W; ++w) any |= acc[w];
        out = any ? round_general<N, W>(acc, lo, sign, 0) : zero<N>();
        return true;
    }
}

template <int N, bool CX> __global__ void __launch_bounds__(128) exact_gemm4_kernel(Eg4Params p) {
    constexpr u64 E = N + 3, S = CX ? 2 * E : E, P = CX ? 2 : 1;
    constexpr int CNT = CX ? 8 : 4;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.count * 16 * P) return;
    const u64 t = q / (16 * P), rest = q % (16 * P), oi = rest / P, part = rest % P;
    const u64 i = oi / 4, j = oi % 4;
    const u32* a = p.A + (t * p.sa + i * 4) * S;
    const u32* b = p.B + (t * p.sb + j) * S;
    u32* out = p.C + (t * p.sc + oi) * S + part * E;
    const Num<N> c = p.accumulate ? load_plain<N>(out) : zero<N>();
    u32 st = c.st;
    bool products = false;
#pragma unroll 1
    for (int k = 0; k < CNT; ++k) {
        const u32 *x, *y; int sg;
        eg4_term<N, CX>(a, b, k, (int)part, x, y, sg);
        st |= x[N + 2] | y[N + 2];
        products = products || (x[N + 1] && y[N + 1]);
    }
    Num<N> r;
    if (st) r = zero<N>(st);
    else if (!products) r = c;
    else if (!eg4_window_sum<N, CX>(a, b, (int)part, c, r)) {
        Eg4Terms<N> src;
        src.cnt = CNT;
        for (int k = 0; k < CNT; ++k) eg4_term<N, CX>(a, b, k, (int)part, src.x[k], src.y[k], src.sg[k]);
        src.c = c;
        r = cluster_round<N, 8 * N + 8>(src, nullptr);
    }
    if (p.negative) r = negate<N>(r);
    store<N>(out, r);
}

struct Eg4Kernels { void (*run)(const Eg4Params&, bool complex_, cudaStream_t); };
const Eg4Kernels* eg4_kernels(int limbs);

template <int N> void eg4_launch(const Eg4Params& p, bool cx, cudaStream_t s) {
    const u64 items = p.count * 16 * (cx ? 2 : 1);
    if (!items) return;
    const unsigned blocks = (unsigned)((items + 127) / 128);
    if (cx) exact_gemm4_kernel<N, true><<<blocks, 128, 0, s>>>(p);
    else exact_gemm4_kernel<N, false><<<blocks, 128, 0, s>>>(p);
}

}  // namespace lfd

#define LF_EG4_INSTANTIATE(N)                                                         \
    namespace lfd {                                                                   \
    extern const Eg4Kernels eg4_kernels_##N;                                          \
    const Eg4Kernels eg4_kernels_##N = {eg4_launch<N>};                               \
    }
