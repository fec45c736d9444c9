// The exact batched 4 x 4 product (the reference's benchmarks/experiments/exact_gemm4: README.md "Contract and
// dispatch", prototype.hpp:5-24): fixed row-major 4 x 4 matrices, matrix t of A, B and C at t * stride elements
// (stride 0 broadcasts an input).  Each real output component is RN(C_old + sum_k a_ik b_kj) with one rounding of the
// exact sum (C_old left out without accumulation), negated when asked; a complex component sums its eight signed real
// products.  Statuses: zero with the OR of every operand the component reads and C_old; no nonzero product gives C_old
// (or zero).  One thread per output component; the exact sum is cluster_round over the component's terms (a window per
// cluster, streamed when a cluster is wider), so every spread is summed on the GPU.
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

template <int N, bool CX> __global__ void __launch_bounds__(128) exact_gemm4_kernel(Eg4Params p) {
    constexpr u64 E = N + 3, S = CX ? 2 * E : E, P = CX ? 2 : 1;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.count * 16 * P) return;
    const u64 t = q / (16 * P), rest = q % (16 * P), oi = rest / P, part = rest % P;
    const u64 i = oi / 4, j = oi % 4;
    const u32* a = p.A + (t * p.sa + i * 4) * S;
    const u32* b = p.B + (t * p.sb + j) * S;
    u32* out = p.C + (t * p.sc + oi) * S + part * E;
    Eg4Terms<N> src;
    src.cnt = CX ? 8 : 4;
    for (int k = 0; k < 4; ++k) {
        const u32* ak = a + k * S;
        const u32* bk = b + (u64)k * 4 * S;
        if (!CX) { src.x[k] = ak; src.y[k] = bk; src.sg[k] = 1; }
        else if (part == 0) {                                  // re: a.re b.re - a.im b.im
            src.x[2 * k] = ak; src.y[2 * k] = bk; src.sg[2 * k] = 1;
            src.x[2 * k + 1] = ak + E; src.y[2 * k + 1] = bk + E; src.sg[2 * k + 1] = -1;
        } else {                                               // im: a.re b.im + a.im b.re
            src.x[2 * k] = ak; src.y[2 * k] = bk + E; src.sg[2 * k] = 1;
            src.x[2 * k + 1] = ak + E; src.y[2 * k + 1] = bk; src.sg[2 * k + 1] = 1;
        }
    }
    src.c = p.accumulate ? load_plain<N>(out) : zero<N>();
    u32 st = src.c.st;
    bool products = false;
    for (int k = 0; k < src.cnt; ++k) {
        st |= src.x[k][N + 2] | src.y[k][N + 2];
        products = products || (src.x[k][N + 1] && src.y[k][N + 1]);
    }
    Num<N> r;
    if (st) r = zero<N>(st);
    else if (!products) r = src.c;
    else r = cluster_round<N, 8 * N + 8>(src, nullptr);
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
