// Batched small-matrix kernels: 4x4 complex LU solve/inverse/determinant (kernels.metal:210-249
// sequence) and strided batched GEMM with ascending-k composed or fused updates
// (batched_linalg.metal:16-17, 24-37, 145-157 sequence).  One thread per matrix / per output
// entry; every arithmetic step is the correctly rounded device routine of lf_arith.cuh, so the
// bits follow the same rounding sequence as the reference.
#pragma once
#include "lf_arith.cuh"
#include <cuda_runtime.h>

namespace lfd {

struct Lu4Params {
    const u32* A; const u32* B; u32* X; u32* det; u32* status;
    u64 count; unsigned rhs; int fused, want_det, inverse;
};

template <int N> __device__ __forceinline__ Cpx<N> c_minus(const Cpx<N>& c, const Cpx<N>& a, const Cpx<N>& b, bool fused) {
    if (fused) { Cpx<N> r = cfms<N>(a, b, c); return {negate<N>(r.re), negate<N>(r.im)}; }   // -(a*b - c), one rounding each
    const Cpx<N> q = cmul<N>(a, b);
    return {subx<N>(c.re, q.re), subx<N>(c.im, q.im)};
}
template <int N> __device__ __forceinline__ Num<N> mag_of(const Cpx<N>& z) {               // max(|re|, |im|) by exact comparison
    return mag_cmp<N>(z.re, z.im) >= 0 ? z.re : z.im;
}

template <int N> __global__ void __launch_bounds__(64) lu4_kernel(Lu4Params p) {
    const u64 m = (u64)blockIdx.x * 64 + threadIdx.x;
    if (m >= p.count) return;
    constexpr u64 CE = 2 * (N + 3);
    Cpx<N> a[16];
    for (int i = 0; i < 16; ++i) a[i] = cload<N>(p.A + (m * 16 + i) * CE);
    unsigned perm[4] = {0, 1, 2, 3}, st = 0, swaps = 0;
    for (unsigned k = 0; k < 4 && !st; ++k) {
        unsigned piv = k;
        for (unsigned r = k + 1; r < 4; ++r)
            if (mag_cmp<N>(mag_of<N>(a[r * 4 + k]), mag_of<N>(a[piv * 4 + k])) > 0) piv = r;   // ties keep the lowest row
        if (!a[piv * 4 + k].re.s && !a[piv * 4 + k].im.s) { st = k + 1; break; }
        if (piv != k) {
            for (unsigned c = 0; c < 4; ++c) { Cpx<N> t = a[k * 4 + c]; a[k * 4 + c] = a[piv * 4 + c]; a[piv * 4 + c] = t; }
            unsigned t = perm[k]; perm[k] = perm[piv]; perm[piv] = t; ++swaps;
        }
        for (unsigned r = k + 1; r < 4; ++r) {
            const Cpx<N> l = cdiv<N>(a[r * 4 + k], a[k * 4 + k]);
            a[r * 4 + k] = l;
            for (unsigned c = k + 1; c < 4; ++c) a[r * 4 + c] = c_minus<N>(a[r * 4 + c], l, a[k * 4 + c], p.fused);
        }
    }
    p.status[m] = st;
    const Cpx<N> z = {zero<N>(), zero<N>()};
    if (p.want_det) {
        Cpx<N> d = z;
        if (!st) {
            d = a[0];
            for (int k = 1; k < 4; ++k) d = cmul<N>(d, a[k * 5]);
            if (swaps & 1) d = {negate<N>(d.re), negate<N>(d.im)};
        }
        cstore<N>(p.det + m * CE, d);
    }
    const unsigned R = p.inverse ? 4 : p.rhs;
    for (unsigned j = 0; j < R; ++j) {
        Cpx<N> y[4];
        for (unsigned i = 0; i < 4; ++i) {
            if (p.inverse) { y[i] = z; if (perm[i] == j) { y[i].re.m[N - 1] = 0x80000000u; y[i].re.s = 1; } }
            else y[i] = cload<N>(p.B + ((m * 4 + perm[i]) * R + j) * CE);
        }
        if (st) {
            const Cpx<N> e = {zero<N>(kDivZero), zero<N>(kDivZero)};
            for (unsigned i = 0; i < 4; ++i) cstore<N>(p.X + ((m * 4 + i) * R + j) * CE, e);
            continue;
        }
        for (unsigned i = 1; i < 4; ++i) for (unsigned t = 0; t < i; ++t) y[i] = c_minus<N>(y[i], a[i * 4 + t], y[t], p.fused);
        for (int i = 3; i >= 0; --i) {
            for (unsigned t = (unsigned)i + 1; t < 4; ++t) y[i] = c_minus<N>(y[i], a[i * 4 + t], y[t], p.fused);
            y[i] = cdiv<N>(y[i], a[i * 5]);
        }
        for (unsigned i = 0; i < 4; ++i) cstore<N>(p.X + ((m * 4 + i) * R + j) * CE, y[i]);
    }
}

struct SgParams {
    const u32* A; const u32* B; u32* C;
    u64 count, m, n, k, sa, sb, sc;
    int accumulate, fused, negative;
};
// One thread per output entry (instance t, row i, column j): sum over ascending k of
// (composed) add(mul(a,b), sum) / cadd(cmul(a,b), sum), or (fused) fma / cfma; negated at the end.
template <int N, bool CX, bool FUSED> __global__ void __launch_bounds__(128) strided_gemm_kernel(SgParams p) {
    const u64 q = (u64)blockIdx.x * 128 + threadIdx.x;
    const u64 cells = p.m * p.n;
    if (q >= p.count * cells) return;
    const u64 t = q / cells, cell = q % cells, i = cell / p.n, j = cell % p.n;
    constexpr u64 E = N + 3, S = CX ? 2 * E : E;
    u32* out = p.C + (t * p.sc + cell) * S;
    if constexpr (CX) {
        Cpx<N> sum = p.accumulate ? cload_plain<N>(out) : Cpx<N>{zero<N>(), zero<N>()};
        for (u64 kk = 0; kk < p.k; ++kk) {
            const Cpx<N> x = cload<N>(p.A + (t * p.sa + i * p.k + kk) * S);
            const Cpx<N> y = cload<N>(p.B + (t * p.sb + kk * p.n + j) * S);
            if constexpr (FUSED) sum = cfma<N>(x, y, sum); else sum = cadd<N>(cmul<N>(x, y), sum);
        }
        if (p.negative) sum = {negate<N>(sum.re), negate<N>(sum.im)};
        cstore<N>(out, sum);
    } else {
        Num<N> sum = p.accumulate ? load_plain<N>(out) : zero<N>();
        for (u64 kk = 0; kk < p.k; ++kk) {
            const Num<N> x = load<N>(p.A + (t * p.sa + i * p.k + kk) * S);
            const Num<N> y = load<N>(p.B + (t * p.sb + kk * p.n + j) * S);
            if constexpr (FUSED) sum = fma<N>(x, y, sum); else sum = addx<N>(mulx<N>(x, y), sum);
        }
        if (p.negative) sum = negate<N>(sum);
        store<N>(out, sum);
    }
}

template <int N> int launch_lu4_n(const Lu4Params& p, cudaStream_t s) {
    if (!p.count) return 0;
    lu4_kernel<N><<<(unsigned)((p.count + 63) / 64), 64, 0, s>>>(p);
    return 0;
}
template <int N> int launch_sg_n(bool cx, const SgParams& p, cudaStream_t s) {
    const u64 total = p.count * p.m * p.n;
    if (!total) return 0;
    const unsigned blocks = (unsigned)((total + 127) / 128);
    if (cx) { if (p.fused) strided_gemm_kernel<N, true, true><<<blocks, 128, 0, s>>>(p); else strided_gemm_kernel<N, true, false><<<blocks, 128, 0, s>>>(p); }
    else { if (p.fused) strided_gemm_kernel<N, false, true><<<blocks, 128, 0, s>>>(p); else strided_gemm_kernel<N, false, false><<<blocks, 128, 0, s>>>(p); }
    return 0;
}
typedef int (*Lu4Launcher)(const Lu4Params&, cudaStream_t);
typedef int (*SgLauncher)(bool, const SgParams&, cudaStream_t);
Lu4Launcher lu4_launcher(int limbs);
SgLauncher sg_launcher(int limbs);

}  // namespace lfd

#define LF_BATCHED_INSTANTIATE(N)                                                                   \
    namespace lfd {                                                                                 \
    int lu4_launch_##N(const Lu4Params& p, cudaStream_t s) { return launch_lu4_n<N>(p, s); }        \
    int sg_launch_##N(bool cx, const SgParams& p, cudaStream_t s) { return launch_sg_n<N>(cx, p, s); } \
    }
