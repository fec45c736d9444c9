// Arithmetic on 32-bit limb numbers: correctly rounded (round to nearest, ties to even)
// add/sub/mul/div/sqrt/fma and the exact multi-term sums behind complex fused operations.
// One source for the GPU kernels (nvcc, sm_100a) and the host-side scalar arithmetic of
// include/limbforge/core.hpp (any C++17 compiler): device-only forms (PTX carry chains, CUDA
// intrinsics) have portable host forms that compute the same integers.
//
// Element contract (the reference's include/limbforge/core.hpp:22-34): Number<N> is
// {u32 limb[N] little endian, top bit set when nonzero; i32 exponent; i32 sign; u32 status},
// value = sign * int(limb) * 2^(exponent-(32N-1)); canonical zero; any input status gives zero
// carrying the OR of the statuses; a rounded exponent outside [-1e9, 1e9] gives zero with
// exponent_overflow (core.hpp:77-85).  Every routine here computes the exact result (in a
// bounded window when a far term can only act as a sticky bit) and rounds it once, so the bits
// equal the reference's and MPFR's; the algorithms are this file's own (fixed windows and
// branch-free barrel shifts that keep every index static, so arrays live in registers).
#pragma once
#include <stdint.h>

#if defined(__CUDACC__)
#define LFD_FN __host__ __device__
#define LFD_INLINE __forceinline__
#define LFD_NOINLINE __noinline__
#define LFD_UNROLL _Pragma("unroll")
#define LFD_NOUNROLL _Pragma("unroll 1")
#else
#include <cmath>
#define LFD_FN
#define LFD_INLINE inline
#define LFD_NOINLINE __attribute__((noinline))
#define LFD_UNROLL
#define LFD_NOUNROLL
#endif

namespace lfd {

typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
typedef uint16_t u16;

constexpr i64 kEmax = 1000000000;
enum : u32 { kDivZero = 1, kOverflow = 2, kInvalid = 4 };

template <int N> struct Num { u32 m[N]; int e; int s; u32 st; };

// ---------------------------------------------------------------- intrinsics with host forms
// lf_fshl: the high word of (hi:lo) << (s mod 32); lf_fshr: the low word of (hi:lo) >> (s mod 32).
LFD_FN LFD_INLINE u32 lf_fshl(u32 lo, u32 hi, u32 s) {
#ifdef __CUDA_ARCH__
    return __funnelshift_l(lo, hi, s);
#else
    s &= 31u; return s ? (hi << s) | (lo >> (32u - s)) : hi;
#endif
}
LFD_FN LFD_INLINE u32 lf_fshr(u32 lo, u32 hi, u32 s) {
#ifdef __CUDA_ARCH__
    return __funnelshift_r(lo, hi, s);
#else
    s &= 31u; return s ? (lo >> s) | (hi << (32u - s)) : lo;
#endif
}
LFD_FN LFD_INLINE int lf_clz(u32 x) {             // leading zeros, 32 for zero
#ifdef __CUDA_ARCH__
    return __clz(x);
#else
    return x ? __builtin_clz(x) : 32;
#endif
}
LFD_FN LFD_INLINE u32 lf_ldg(const u32* p) {     // read-only (non-coherent) load on the GPU
#ifdef __CUDA_ARCH__
    return __ldg(p);
#else
    return *p;
#endif
}
LFD_FN LFD_INLINE double lf_rsqrt_start(double z) {   // 1 / sqrt(z), both steps correctly rounded
#ifdef __CUDA_ARCH__
    return __drcp_rn(__dsqrt_rn(z));
#else
    return 1.0 / std::sqrt(z);
#endif
}
LFD_FN LFD_INLINE void lf_flag(u32* error, u32 v) {
#ifdef __CUDA_ARCH__
    atomicExch(error, v);
#else
    *error = v;
#endif
}

template <int N> LFD_FN LFD_INLINE Num<N> zero(u32 st = 0) {
    Num<N> r;
LFD_UNROLL
    for (int i = 0; i < N; ++i) r.m[i] = 0;
    r.e = 0; r.s = 0; r.st = st;
    return r;
}
template <int N> LFD_FN LFD_INLINE Num<N> negate(Num<N> a) { a.s = -a.s; return a; }

// ---------------------------------------------------------------- element load / store
template <int N> LFD_FN LFD_INLINE Num<N> load(const u32* __restrict__ p) {
    Num<N> r;
LFD_UNROLL
    for (int i = 0; i < N; ++i) r.m[i] = lf_ldg(p + i);
    r.e = (int)lf_ldg(p + N); r.s = (int)lf_ldg(p + N + 1); r.st = lf_ldg(p + N + 2);
    return r;
}
template <int N> LFD_FN LFD_INLINE Num<N> load_plain(const u32* p) {   // for buffers written in the same kernel
    Num<N> r;
LFD_UNROLL
    for (int i = 0; i < N; ++i) r.m[i] = p[i];
    r.e = (int)p[N]; r.s = (int)p[N + 1]; r.st = p[N + 2];
    return r;
}
template <int N> LFD_FN LFD_INLINE void store(u32* p, const Num<N>& r) {
LFD_UNROLL
    for (int i = 0; i < N; ++i) p[i] = r.m[i];
    p[N] = (u32)r.e; p[N + 1] = (u32)r.s; p[N + 2] = r.st;
}

// ---------------------------------------------------------------- small helpers
template <int N> LFD_FN LFD_INLINE Num<N> pick(bool c, const Num<N>& a, const Num<N>& b) {
    Num<N> r;
LFD_UNROLL
    for (int i = 0; i < N; ++i) r.m[i] = c ? a.m[i] : b.m[i];
    r.e = c ? a.e : b.e; r.s = c ? a.s : b.s; r.st = c ? a.st : b.st;
    return r;
}
template <int N> LFD_FN LFD_INLINE int mag_cmp(const Num<N>& a, const Num<N>& b) {
    if (!a.s) return b.s ? -1 : 0;
    if (!b.s) return 1;
    if (a.e != b.e) return a.e > b.e ? 1 : -1;
    int c = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) c = (a.m[i] != b.m[i]) ? (a.m[i] > b.m[i] ? 1 : -1) : c;   // highest differing word wins
    return c;
}
// Rounded result r = sign * m * 2^(e-(32N-1)) with the increment decided by the caller.
template <int N> LFD_FN LFD_INLINE Num<N> finish(u32 (&m)[N], i64 e, int sign, bool up, u32 status) {
    u32 c = up ? 1u : 0u;
LFD_UNROLL
    for (int i = 0; i < N; ++i) { u32 t = m[i] + c; c = (c && t == 0) ? 1u : 0u; m[i] = t; }
    if (c) { m[N - 1] = 0x80000000u; e += 1; }
    if (e > kEmax || e < -kEmax) return zero<N>(status | kOverflow);
    Num<N> r;
LFD_UNROLL
    for (int i = 0; i < N; ++i) r.m[i] = m[i];
    r.e = (int)e; r.s = sign; r.st = status;
    return r;
}

// Words of x moved up by q words (q in [0, 2^stages)), zeros shifted in: a branch-free barrel
// shifter, so the array stays register resident whatever q is.
template <int W, int STAGES> LFD_FN LFD_INLINE void shift_up_words(u32 (&x)[W], u32 q) {
LFD_UNROLL
    for (int b = 0; b < STAGES; ++b) {
        const int s = 1 << b;
        if (s >= W) { if ((q >> b) & 1u) {
LFD_UNROLL
                for (int k = 0; k < W; ++k) x[k] = 0; }
            continue; }
        const bool on = (q >> b) & 1u;
LFD_UNROLL
        for (int k = W - 1; k >= 0; --k) x[k] = on ? (k >= s ? x[k - s] : 0u) : x[k];
    }
}
// x <<= r bits (0 <= r < 32) over W words
template <int W> LFD_FN LFD_INLINE void shift_up_bits(u32 (&x)[W], u32 r) {
LFD_UNROLL
    for (int k = W - 1; k > 0; --k) x[k] = lf_fshl(x[k - 1], x[k], r);
    x[0] = x[0] << r;   // r < 32
}
template <int W> LFD_FN constexpr int stages_for() { return W <= 1 ? 1 : W <= 2 ? 1 : W <= 4 ? 2 : W <= 8 ? 3 : W <= 16 ? 4 : W <= 32 ? 5 : W <= 64 ? 6 : W <= 128 ? 7 : 8; }

// RN(sign * int(x) * 2^scale) for a W-word magnitude with the top bit anywhere (x is clobbered).
template <int N, int W> LFD_FN LFD_INLINE Num<N> round_general(u32 (&x)[W], i64 scale, int sign, u32 status) {
    static_assert(W >= N + 1, "window narrower than the result");
    int t = -1;
LFD_UNROLL
    for (int k = 0; k < W; ++k) t = x[k] ? k : t;
    if (t < 0) return zero<N>(status);
    u32 top = 0;
LFD_UNROLL
    for (int k = 0; k < W; ++k) top = (k == t) ? x[k] : top;
    const int lz = lf_clz(top);
    const i64 e = scale + 32 * (i64)t + 31 - lz;
    shift_up_words<W, stages_for<W>()>(x, (u32)(W - 1 - t));
    shift_up_bits<W>(x, (u32)lz);
    u32 m[N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) m[i] = x[W - N + i];
    u32 below = (W > N) ? x[W - N - 1] : 0u;
    bool rb = below >> 31;
    u32 sticky = below & 0x7fffffffu;
LFD_UNROLL
    for (int k = 0; k < W - N - 1; ++k) sticky |= x[k];
    return finish<N>(m, e, sign, rb && (sticky || (m[0] & 1u)), status);
}

// ---------------------------------------------------------------- mul
// Carry-chain primitives (PTX add/mad with .cc): one IMAD per half word product.  GPU only; the host forms
// of the products below use 64-bit arithmetic instead.
#ifdef __CUDA_ARCH__
__device__ __forceinline__ u32 mad_lo_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("mad.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ u32 madc_lo_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.lo.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ u32 mad_hi_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("mad.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ u32 madc_hi_cc(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.hi.cc.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ u32 madc_hi(u32 a, u32 b, u32 c) { u32 r; asm volatile("madc.hi.u32 %0, %1, %2, %3;" : "=r"(r) : "r"(a), "r"(b), "r"(c)); return r; }
__device__ __forceinline__ u32 carry_out() { u32 r; asm volatile("addc.u32 %0, 0, 0;" : "=r"(r)); return r; }

#endif

// a (A words) * b (B words) = p (A + B words): schoolbook rows with explicit 32-bit carries.
template <int A, int B> LFD_FN LFD_INLINE void mul_words(const u32 (&a)[A], const u32 (&b)[B], u32 (&p)[A + B]) {
LFD_UNROLL
    for (int k = 0; k < A + B; ++k) p[k] = 0;
LFD_UNROLL
    for (int j = 0; j < B; ++j) {
        u32 c = 0;
LFD_UNROLL
        for (int i = 0; i < A; ++i) {
            const u64 t = (u64)a[i] * b[j] + p[i + j] + c;
            p[i + j] = (u32)t;
            c = (u32)(t >> 32);
        }
        p[j + A] = c;
    }
}

// p (2N words) = a * b, schoolbook by rows: for row i a low-half carry chain adds
// lo(a_i b_j) into p[i+j] and a high-half chain adds hi(a_i b_j) into p[i+j+1]; the running
// sum never exceeds 2^(32(i+N+1)), so the last high-half step cannot carry out.
template <int N> LFD_FN LFD_INLINE void mant_mul(const u32 (&a)[N], const u32 (&b)[N], u32 (&p)[2 * N]) {
#ifndef __CUDA_ARCH__
    mul_words<N, N>(a, b, p);
#else
LFD_UNROLL
    for (int k = 0; k < 2 * N; ++k) p[k] = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) {
        p[i] = mad_lo_cc(a[i], b[0], p[i]);
LFD_UNROLL
        for (int j = 1; j < N; ++j) p[i + j] = madc_lo_cc(a[i], b[j], p[i + j]);
        p[i + N] = carry_out();
        p[i + 1] = mad_hi_cc(a[i], b[0], p[i + 1]);
LFD_UNROLL
        for (int j = 1; j < N - 1; ++j) p[i + j + 1] = madc_hi_cc(a[i], b[j], p[i + j + 1]);
        p[i + N] = madc_hi(a[i], b[N - 1], p[i + N]);
    }
#endif
}
// Round a product of two normalized mantissas: its top bit is bit 64N-1 or 64N-2.
template <int N> LFD_FN LFD_INLINE Num<N> round_product(const u32 (&p)[2 * N], i64 e_sum, int sign, u32 status) {
    const u32 s = (p[2 * N - 1] >> 31) ? 0u : 1u;      // normalizing left shift
    u32 m[N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) m[i] = lf_fshl(p[N + i - 1], p[N + i], s);
    const u32 low = p[N - 1] << s;                    // round bit is its top bit
    u32 sticky = low & 0x7fffffffu;
LFD_UNROLL
    for (int k = 0; k < N - 1; ++k) sticky |= p[k];
    // (when s = 1 the bit shifted out of p[N-1] went into m[0], not lost)
    return finish<N>(m, e_sum + 1 - (i64)s, sign, (low >> 31) && (sticky || (m[0] & 1u)), status);
}
// RN(a * b) from the full 2N-word product.
template <int N> LFD_FN LFD_INLINE Num<N> mul_exact(const Num<N>& a, const Num<N>& b) {
    const u32 st = a.st | b.st;
    if (st || !a.s || !b.s) return zero<N>(st);
    u32 p[2 * N];
    mant_mul<N>(a.m, b.m, p);
    return round_product<N>(p, (i64)a.e + b.e, a.s * b.s, 0);
}
template <int N> LFD_FN LFD_NOINLINE Num<N> mul_exact_call(const Num<N> a, const Num<N> b) { return mul_exact<N>(a, b); }
// The same with b read inside the call, so a caller's fast path need not keep b's words live for it.
template <int N> LFD_FN LFD_NOINLINE Num<N> mul_exact_mem_call(const Num<N> a, const u32* b) { return mul_exact<N>(a, load_plain<N>(b)); }

// The same upper part T as mant_mul_high with b's words read from memory: row j adds b_j times a into
// the window through an explicit 32-bit carry (64-bit products, no condition code), so successive rows
// are plain data dependencies that the compiler can overlap, and only a and the window live in
// registers.  a_i b_j + h + c <= (2^32 - 1)^2 + 2 (2^32 - 1) = 2^64 - 1, so no step overflows.
template <int N> LFD_FN LFD_INLINE void mant_mul_high_mem(const u32 (&a)[N], const u32* b, u32 (&h)[N + 2]) {
    constexpr int B = N - 2;
LFD_UNROLL
    for (int k = 0; k < N + 2; ++k) h[k] = 0;
LFD_UNROLL
    for (int j = 0; j < N; ++j) {
        const u32 bj = b[j];
        const int i0 = B - j > 0 ? B - j : 0;
        u32 c = 0;
LFD_UNROLL
        for (int i = i0; i < N; ++i) {
            const u64 t = (u64)a[i] * bj + h[i + j - B] + c;
            h[i + j - B] = (u32)t;
            c = (u32)(t >> 32);
        }
        h[j + N - B] = c;        // rows before j end at word j + N - B - 1
    }
}
// Upper part of the product: h = T / 2^(32(N-2)) with T = sum of a_i b_j 2^(32(i+j)) over i + j >= N-2
// (words N-2 .. 2N-1; about 58% of the word products at N = 32).  The omitted products sum to
// D = sum_{i+j <= N-3} a_i b_j 2^(32(i+j)) < (N-2) 2^(32(N-1)) (1 + 2^-31), so the full product is T + D
// with D less than N units of word N-1.  Row carries follow mant_mul: T through row i is at most the
// full partial product, below 2^(32(i+N+1)), so the last high-half step of a row cannot carry out.
template <int N> LFD_FN LFD_INLINE void mant_mul_high(const u32 (&a)[N], const u32 (&b)[N], u32 (&h)[N + 2]) {
#ifndef __CUDA_ARCH__
    mant_mul_high_mem<N>(a, b, h);                 // the same products, summed with explicit carries
#else
    constexpr int B = N - 2;
LFD_UNROLL
    for (int k = 0; k < N + 2; ++k) h[k] = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) {
        const int j0 = B - i > 0 ? B - i : 0;
        h[i + j0 - B] = mad_lo_cc(a[i], b[j0], h[i + j0 - B]);
LFD_UNROLL
        for (int j = j0 + 1; j < N; ++j) h[i + j - B] = madc_lo_cc(a[i], b[j], h[i + j - B]);
        h[i + N - B] = carry_out();
        h[i + j0 + 1 - B] = mad_hi_cc(a[i], b[j0], h[i + j0 + 1 - B]);
LFD_UNROLL
        for (int j = j0 + 1; j < N - 1; ++j) h[i + j + 1 - B] = madc_hi_cc(a[i], b[j], h[i + j + 1 - B]);
        h[i + N - B] = madc_hi(a[i], b[N - 1], h[i + N - B]);
    }
#endif
}

// RN(a * b).  From N = 12 limbs on, the rounding is decided from the upper part T of the product when
// that is safe, and from the full product otherwise.  With s the normalizing shift, word N-1 of T
// shifted left by s holds the round bit (bit 31) and, below it, `low`.  The omitted part D adds less
// than N units to word N-1 (at most 2N after the shift), so when low + 2N stays below 2^31 every bit
// from the round bit up is exact.  Then a clear round bit rounds down, and a set round bit with low != 0
// rounds up: the discarded bits are nonzero, so there is no tie.  Any other case (a carry could reach
// the round bit, or the sticky bits depend on D) takes the full product: for random operands about
// once in 2^25 products.
constexpr int kShortMulLimbs = 12;
template <int N> LFD_FN LFD_INLINE Num<N> mul(const Num<N>& a, const Num<N>& b) {
    if constexpr (N < kShortMulLimbs) {
        return mul_exact<N>(a, b);
    } else {
        const u32 st = a.st | b.st;
        if (st || !a.s || !b.s) return zero<N>(st);
        u32 h[N + 2];
        mant_mul_high<N>(a.m, b.m, h);
        const u32 s = (h[N + 1] >> 31) ? 0u : 1u;
        const u32 lw = h[1] << s;
        const u32 low = lw & 0x7fffffffu;
        const bool rb = lw >> 31;
        if (low >= 0x80000000u - ((u32)N << s) || (rb && low == 0)) return mul_exact_call<N>(a, b);
        u32 m[N];
LFD_UNROLL
        for (int i = 0; i < N; ++i) m[i] = lf_fshl(h[i + 1], h[i + 2], s);
        return finish<N>(m, (i64)a.e + b.e + 1 - (i64)s, a.s * b.s, rb, 0);
    }
}

// RN(a * y) for y an element in memory (plain loads: y may have been written earlier in the same
// kernel).  The rounding rule is mul's, on the same T, so the result is mul(a, y) bit for bit.
template <int N> LFD_FN LFD_INLINE Num<N> mul_mem(const Num<N>& a, const u32* y) {
    if constexpr (N < kShortMulLimbs) {
        return mul_exact<N>(a, load_plain<N>(y));
    } else {
        const int ys = (int)y[N + 1];
        const u32 st = a.st | y[N + 2];
        if (st || !a.s || !ys) return zero<N>(st);
        u32 h[N + 2];
        mant_mul_high_mem<N>(a.m, y, h);
        const u32 s = (h[N + 1] >> 31) ? 0u : 1u;
        const u32 lw = h[1] << s;
        const u32 low = lw & 0x7fffffffu;
        const bool rb = lw >> 31;
        if (low >= 0x80000000u - ((u32)N << s) || (rb && low == 0)) return mul_exact_mem_call<N>(a, y);
        u32 m[N];
LFD_UNROLL
        for (int i = 0; i < N; ++i) m[i] = lf_fshl(h[i + 1], h[i + 2], s);
        return finish<N>(m, (i64)a.e + (int)y[N] + 1 - (i64)s, a.s * ys, rb, 0);
    }
}

// ---------------------------------------------------------------- add / sub
// Words of x moved down by q words (q in [0, 2^stages)), zeros shifted in; every word shifted out is
// ORed into `sticky` (branch-free barrel shifter, like shift_up_words).
template <int W, int STAGES> LFD_FN LFD_INLINE void shift_down_words(u32 (&x)[W], u32 q, u32& sticky) {
LFD_UNROLL
    for (int b = 0; b < STAGES; ++b) {
        const int s = 1 << b;
        const bool on = (q >> b) & 1u;
LFD_UNROLL
        for (int k = 0; k < (s < W ? s : W); ++k) sticky |= on ? x[k] : 0u;
LFD_UNROLL
        for (int k = 0; k < W; ++k) x[k] = on ? (k + s < W ? x[k + s] : 0u) : x[k];
    }
}
template <int W> LFD_FN LFD_INLINE void shift_down_bits(u32 (&x)[W], u32 r, u32& sticky) {   // r < 32
    sticky |= r ? (x[0] << (32 - r)) : 0u;
LFD_UNROLL
    for (int k = 0; k < W - 1; ++k) x[k] = lf_fshr(x[k], x[k + 1], r);
    x[W - 1] = x[W - 1] >> r;
}

// RN(a + b).  x = the larger magnitude, y = the smaller, gap = e_x - e_y.  Window of N + 4 words:
// x's significand at words [3, N+2] (three words below it, one word of headroom above).  y is aligned
// by shifting it down gap bits from x's position.  When gap <= 96 all of y stays in the window and the
// sum is exact.  Otherwise the bits shifted out are nonzero only if `lost` is set, and
// x +- y = V + phi with V = x + y_t or x - y_t - lost (y_t the kept part) and 0 <= phi < 1 (phi > 0 iff
// lost).  Setting bit 0 of V to lost then gives every bit that the rounding reads.  The result is at least
// x/2 here, so its round bit lies at bit 94 or higher, far above bit 0.  gap > 32N+2 returns x: y is below a
// quarter ulp of x, and RN(x +- y) = x.
template <int N> LFD_FN LFD_INLINE Num<N> add(const Num<N>& a, const Num<N>& b) {
    const u32 st = a.st | b.st;
    if (st) return zero<N>(st);
    if (!a.s) return b;
    if (!b.s) return a;
    const bool swap = mag_cmp<N>(a, b) < 0;
    const Num<N> x = pick<N>(swap, b, a);
    const Num<N> y = pick<N>(swap, a, b);
    const i64 gap = (i64)x.e - y.e;
    if (gap > 32 * N + 2) return x;
    constexpr int W = N + 4;
    u32 w[W], v[W];
LFD_UNROLL
    for (int k = 0; k < W; ++k) { w[k] = (k >= 3 && k < N + 3) ? x.m[k - 3] : 0u; v[k] = (k >= 3 && k < N + 3) ? y.m[k - 3] : 0u; }
    u32 lost = 0;
    shift_down_bits<W>(v, (u32)gap & 31u, lost);
    shift_down_words<W, stages_for<W>()>(v, (u32)gap >> 5, lost);
    const u32 l = lost ? 1u : 0u;
    if (x.s == y.s) {
        u64 c = 0;
LFD_UNROLL
        for (int k = 0; k < W; ++k) { u64 t = (u64)w[k] + v[k] + c; w[k] = (u32)t; c = t >> 32; }
    } else {
        u32 bo = l;                                         // x - y_t - lost
LFD_UNROLL
        for (int k = 0; k < W; ++k) { u64 t = (u64)v[k] + bo; u32 old = w[k]; w[k] = (u32)((u64)old - t); bo = (u64)old < t; }
    }
    w[0] |= l;
    return round_general<N, W>(w, (i64)x.e - (32 * N - 1) - 96, x.s, 0);
}
template <int N> LFD_FN LFD_INLINE Num<N> sub(const Num<N>& a, const Num<N>& b) { return add<N>(a, negate<N>(b)); }

// ---------------------------------------------------------------- div
// Two-by-one word division with a reused reciprocal (Moller & Granlund, "Improved division by
// invariant integers", IEEE TC 2011, algorithm 4).  d normalized, u1 < d, v = floor((2^64-1)/d)-2^32.
LFD_FN LFD_INLINE u32 div2by1(u32 u1, u32 u0, u32 d, u32 v, u32& rem) {
    u64 p = (u64)v * u1;
    u64 s = (p & 0xffffffffull) + u0;
    u32 q0 = (u32)s;
    u32 q1 = (u32)((p >> 32) + u1 + 1 + (s >> 32));
    u32 r = u0 - q1 * d;
    if (r > q0) { --q1; r += d; }
    if (r >= d) { ++q1; r -= d; }
    rem = r;
    return q1;
}
// Quotient Q = floor(A * 2^(32N-1+c) / B), c = (A < B), has exactly 32N bits; schoolbook long
// division by 32-bit digits (Knuth, TAOCP vol. 2, 4.3.1 algorithm D) with the digit estimate
// above; RNE from the remainder: 2R > B rounds up, 2R == B is a tie.
template <int N> LFD_FN LFD_INLINE Num<N> div(const Num<N>& a, const Num<N>& b) {
    const u32 st = a.st | b.st;
    if (st) return zero<N>(st);
    if (!b.s) return zero<N>(kDivZero);
    if (!a.s) return zero<N>();
    int cmp = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) cmp = (a.m[i] != b.m[i]) ? (a.m[i] > b.m[i] ? 1 : -1) : cmp;
    const int c = cmp < 0 ? 1 : 0;
    const i64 e = (i64)a.e - b.e - c;
    if (e > kEmax || e < -kEmax - 1) return zero<N>(kOverflow);
    u32 u[2 * N + 1];
LFD_UNROLL
    for (int k = 0; k <= 2 * N; ++k) u[k] = 0;
    if (c) {
LFD_UNROLL
        for (int i = 0; i < N; ++i) u[N + i] = a.m[i];
    } else {
        u[N - 1] = a.m[0] << 31;
LFD_UNROLL
        for (int i = 0; i < N; ++i) u[N + i] = (a.m[i] >> 1) | (i + 1 < N ? a.m[i + 1] << 31 : 0u);
    }
    const u32 d = b.m[N - 1], d2 = b.m[N - 2];
    const u32 v = (u32)(0xffffffffffffffffull / d - 0x100000000ull);
    u32 q[N];
LFD_UNROLL
    for (int j = N - 1; j >= 0; --j) {
        const u32 u1 = u[j + N], u0 = u[j + N - 1];
        u32 qh, rh;
        bool rbig;                                   // r-hat >= 2^32: the refinement cannot trigger
        if (u1 >= d) { qh = 0xffffffffu; u64 r = ((u64)u1 << 32 | u0) - (u64)qh * d; rbig = (r >> 32) != 0; rh = (u32)r; }
        else { qh = div2by1(u1, u0, d, v, rh); rbig = false; }
        const u32 u2 = u[j + N - 2];
LFD_NOUNROLL
        for (int it = 0; it < 2 && !rbig; ++it) {
            if ((u64)qh * d2 > (((u64)rh << 32) | u2)) { --qh; u64 nr = (u64)rh + d; rbig = (nr >> 32) != 0; rh = (u32)nr; }
            else break;
        }
        // u[j .. j+N] -= qh * B
        u64 borrow = 0;
LFD_UNROLL
        for (int i = 0; i < N; ++i) {
            u64 p = (u64)qh * b.m[i] + borrow;
            u32 lo = (u32)p, old = u[j + i];
            u[j + i] = old - lo;
            borrow = (p >> 32) + (old < lo ? 1u : 0u);
        }
        const bool under = (u64)u[j + N] < borrow;
        u[j + N] = (u32)((u64)u[j + N] - borrow);
        if (under) {
            --qh;
            u64 cy = 0;
LFD_UNROLL
            for (int i = 0; i < N; ++i) { u64 t = (u64)u[j + i] + b.m[i] + cy; u[j + i] = (u32)t; cy = t >> 32; }
            u[j + N] += (u32)cy;
        }
        q[j] = qh;
    }
    // remainder u[0..N-1]; compare 2R with B
    int half = 0;
    const bool topbit = u[N - 1] >> 31;
LFD_UNROLL
    for (int i = 0; i < N; ++i) {
        u32 tw = (u[i] << 1) | (i ? u[i - 1] >> 31 : 0u);
        half = (tw != b.m[i]) ? (tw > b.m[i] ? 1 : -1) : half;
    }
    if (topbit) half = 1;
    return finish<N>(q, e, a.s * b.s, half > 0 || (half == 0 && (q[0] & 1u)), 0);
}

// ---------------------------------------------------------------- sqrt
// Restoring digit-by-digit root of the 64N-bit radicand M * 2^(32N-1+odd); the root has 32N bits
// and no tie is possible: round up exactly when the remainder exceeds the root.
template <int N> LFD_FN LFD_INLINE Num<N> sqrt_restoring(const Num<N>& a) {
    if (a.st || !a.s) return zero<N>(a.st);
    if (a.s < 0) return zero<N>(kInvalid);
    int e = a.e / 2; if (a.e < 0 && (a.e % 2)) --e;
    const int odd = a.e - 2 * e;                    // 0 or 1
    // radicand Z = M << (32N - 1 + odd): 2N words
    u32 z[2 * N];
LFD_UNROLL
    for (int k = 0; k < 2 * N; ++k) z[k] = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) z[N + i] = a.m[i];
    // shift right by 1 - odd bits (0 or 1)
    if (!odd) {
LFD_UNROLL
        for (int k = 0; k < 2 * N; ++k) z[k] = (z[k] >> 1) | (k + 1 < 2 * N ? z[k + 1] << 31 : 0u);
    }
    u32 root[N + 1], rem[N + 2];
LFD_UNROLL
    for (int k = 0; k <= N; ++k) root[k] = 0;
LFD_UNROLL
    for (int k = 0; k < N + 2; ++k) rem[k] = 0;
LFD_NOUNROLL
    for (int pi = 32 * N - 1; pi >= 0; --pi) {
        // bring down two bits of z at position 2*pi
        u32 wsel = 0;
LFD_UNROLL
        for (int k = 0; k < 2 * N; ++k) wsel = (k == (2 * pi) / 32) ? z[k] : wsel;
        const u32 pair = (wsel >> ((2 * pi) % 32)) & 3u;
LFD_UNROLL
        for (int k = N + 1; k > 0; --k) rem[k] = (rem[k] << 2) | (rem[k - 1] >> 30);
        rem[0] = (rem[0] << 2) | pair;
        // trial = 4*root + 1, compared with rem
        u32 tr[N + 2];
        tr[0] = (root[0] << 2) | 1u;
LFD_UNROLL
        for (int k = 1; k <= N; ++k) tr[k] = (root[k] << 2) | (root[k - 1] >> 30);
        tr[N + 1] = root[N] >> 30;
        int c = 0;
LFD_UNROLL
        for (int k = 0; k < N + 2; ++k) c = (rem[k] != tr[k]) ? (rem[k] > tr[k] ? 1 : -1) : c;
LFD_UNROLL
        for (int k = N; k > 0; --k) root[k] = (root[k] << 1) | (root[k - 1] >> 31);
        root[0] <<= 1;
        if (c >= 0) {
            u32 bo = 0;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { u64 t = (u64)tr[k] + bo; u32 old = rem[k]; rem[k] = (u32)((u64)old - t); bo = (u64)old < t; }
            root[0] |= 1u;
        }
    }
    // round up iff rem > root
    int c = 0;
LFD_UNROLL
    for (int k = 0; k < N + 2; ++k) { u32 rk = k <= N ? root[k] : 0u; c = (rem[k] != rk) ? (rem[k] > rk ? 1 : -1) : c; }
    u32 m[N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) m[i] = root[i];
    return finish<N>(m, e, 1, c > 0, 0);
}
template <int N> LFD_FN LFD_NOINLINE Num<N> sqrt_restoring_call(const Num<N> a) { return sqrt_restoring<N>(a); }
template <int N> LFD_FN LFD_NOINLINE Num<N> add_call(const Num<N> a, const Num<N> b);
template <int N> LFD_FN LFD_NOINLINE Num<N> div_call(const Num<N> a, const Num<N> b);

// Reciprocal square root in fixed point, for the candidate of sqrt.  z = Z / 2^(64N) lies in [1/4, 1) and
// y = 1 / sqrt(z) in (1, 2].  At level M (M words) y is held as Y = y * 2^(32M - 2).  A start of 50 correct
// bits (a double) is refined by Newton's step y' = y + y (1 - z y^2) / 2 at word counts that double
// (4, 8, 16, ... capped at N), each giving min(2p - 2, 32M - 8) correct bits, until p >= 16N + 16.
LFD_FN constexpr int rsqrt_next_level(int N, int L) { return L == 2 ? (N < 4 ? N : 4) : (2 * L < N ? 2 * L : N); }
LFD_FN constexpr int rsqrt_prec_after(int p, int M) { return 2 * p - 2 < 32 * M - 8 ? 2 * p - 2 : 32 * M - 8; }
LFD_FN constexpr int rsqrt_final_prec(int N) {
    int p = 50, L = 2;
    while (p < 16 * N + 16) { const int M = rsqrt_next_level(N, L); p = rsqrt_prec_after(p, M); L = M; }
    return p;
}
// One Newton step from level L (y[0..L)) to level M >= L.  With Zm the top M words of Z:
//   P = Y^2 = y^2 2^(64M-4); T = Zm * top_M(P) = z y^2 2^(64M-4); H = 2^(64M-4) - T = (1 - z y^2) 2^(64M-4);
//   the correction y h / 2 at level M is Y * floor(H / 2^(32M)) / 2^(32M-3).
template <int N, int L, int M> LFD_FN LFD_INLINE void rsqrt_step(const u32 (&z)[2 * N], u32 (&y)[N]) {
    u32 Y[M], Zm[M], Pt[M], Ht[M];
LFD_UNROLL
    for (int i = 0; i < M; ++i) { Y[i] = i >= M - L ? y[i - (M - L)] : 0u; Zm[i] = z[2 * N - M + i]; }
    u32 P[2 * M];
    mul_words<M, M>(Y, Y, P);
LFD_UNROLL
    for (int i = 0; i < M; ++i) Pt[i] = P[M + i];
    u32 T[2 * M];
    mul_words<M, M>(Zm, Pt, T);
    u32 bo = 0;
LFD_UNROLL
    for (int k = 0; k < 2 * M; ++k) {
        const u64 v = (u64)T[k] + bo;
        const u32 kw = k == 2 * M - 1 ? 0x10000000u : 0u;
        const u32 d = (u32)((u64)kw - v);
        bo = (u64)kw < v;
        if (k >= M) Ht[k - M] = d;
    }
    const bool neg = Ht[M - 1] >> 31;                  // z y^2 > 1: y is too large
    if (neg) {
        u32 cy = 1;
LFD_UNROLL
        for (int i = 0; i < M; ++i) { const u64 v = (u64)(~Ht[i]) + cy; Ht[i] = (u32)v; cy = (u32)(v >> 32); }
    }
    u32 Q[2 * M];
    mul_words<M, M>(Y, Ht, Q);
    u64 cy = 0, bw = 0;
LFD_UNROLL
    for (int i = 0; i < M; ++i) {
        const u32 corr = lf_fshr(Q[M - 1 + i], M + i < 2 * M ? Q[M + i] : 0u, 29);     // Q >> (32M - 3)
        if (neg) { const u64 v = (u64)corr + bw; const u32 old = Y[i]; Y[i] = (u32)((u64)old - v); bw = (u64)old < v; }
        else { const u64 v = (u64)Y[i] + corr + cy; Y[i] = (u32)v; cy = v >> 32; }
    }
LFD_UNROLL
    for (int i = 0; i < M; ++i) y[i] = Y[i];
}
template <int N, int L, int P> LFD_FN LFD_INLINE void rsqrt_ladder(const u32 (&z)[2 * N], u32 (&y)[N]) {
    if constexpr (P < 16 * N + 16) {
        constexpr int M = rsqrt_next_level(N, L);
        rsqrt_step<N, L, M>(z, y);
        rsqrt_ladder<N, M, rsqrt_prec_after(P, M)>(z, y);
    } else if constexpr (L < N) {
LFD_UNROLL
        for (int i = N - 1; i >= 0; --i) y[i] = i >= N - L ? y[i - (N - L)] : 0u;     // to level N
    }
}
// Candidate C (N + 1 words, c[N] = 0, C in [2^(32N-1), 2^(32N))) for S = sqrt(Z), within a few units of S.
// C0 = Zt * Y / 2^(32N-2) (Zt the top N words of Z) is within 2^(32N-p+2) of S; one correction
// C1 = C0 + (Z - C0^2) / (2 S) = C0 + (Z - C0^2) * Y / 2^(64N-1) leaves a second-order error below a unit
// (p >= 16N + 16) plus the truncations below, under two units together.  Returns false when Z - C0^2 is
// larger than these bounds allow (never expected), and the caller takes the restoring routine.
template <int N> LFD_FN LFD_INLINE bool sqrt_candidate(const u32 (&z)[2 * N], u32 (&c)[N + 1]) {
    const u64 zt = ((u64)z[2 * N - 1] << 32) | z[2 * N - 2];
    const double y0 = lf_rsqrt_start((double)zt * 0x1p-64);                // (1, 2]
    const u64 Y0 = (u64)(y0 * 0x1p62);
    u32 y[N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) y[i] = 0;
    y[0] = (u32)Y0; y[1] = (u32)(Y0 >> 32);
    constexpr int P = rsqrt_final_prec(N);
    rsqrt_ladder<N, 2, 50>(z, y);
    // C0
    u32 Zt[N], R[2 * N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) Zt[i] = z[N + i];
    mul_words<N, N>(Zt, y, R);
LFD_UNROLL
    for (int i = 0; i <= N; ++i) c[i] = lf_fshr(R[N - 1 + i], N + i < 2 * N ? R[N + i] : 0u, 30);
    const auto clamp = [&c]() {
        if (c[N]) {
LFD_UNROLL
            for (int i = 0; i < N; ++i) c[i] = 0xffffffffu;
        } else if (!(c[N - 1] >> 31)) {
LFD_UNROLL
            for (int i = 0; i < N; ++i) c[i] = i == N - 1 ? 0x80000000u : 0u;
        }
        c[N] = 0;
    };
    clamp();
    // D0 = Z - C0^2 (sign and magnitude)
    u32 cm[N], sq[2 * N], d[2 * N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) cm[i] = c[i];
    mul_words<N, N>(cm, cm, sq);
    u32 bo = 0;
LFD_UNROLL
    for (int k = 0; k < 2 * N; ++k) { const u64 v = (u64)sq[k] + bo; d[k] = (u32)((u64)z[k] - v); bo = (u64)z[k] < v; }
    const bool neg = bo != 0;                          // C0^2 > Z
    if (neg) {
        u32 cy = 1;
LFD_UNROLL
        for (int k = 0; k < 2 * N; ++k) { const u64 v = (u64)(~d[k]) + cy; d[k] = (u32)v; cy = (u32)(v >> 32); }
    }
    // |D0| < 2^(64N - P + 3): words [DL, DH) carry it to within 2^-31 of a unit of the correction;
    // words [YL, N) of Y carry the product to within a quarter unit.
    constexpr int DL = N - 1;
    constexpr int DH = (64 * N - P + 4 + 31) / 32 < 2 * N ? (64 * N - P + 4 + 31) / 32 : 2 * N;
    constexpr int YL = (P - 6) / 32 < N - 1 ? (P - 6) / 32 : N - 1;
    static_assert(DH > DL, "correction window");
    u32 hi = 0;
LFD_UNROLL
    for (int k = DH; k < 2 * N; ++k) hi |= d[k];
    if (hi) return false;
    u32 dw[DH - DL], yw[N - YL], pr[DH - DL + N - YL];
LFD_UNROLL
    for (int k = 0; k < DH - DL; ++k) dw[k] = d[DL + k];
LFD_UNROLL
    for (int k = 0; k < N - YL; ++k) yw[k] = y[YL + k];
    mul_words<DH - DL, N - YL>(dw, yw, pr);
    // delta = pr >> SH with SH = 64N - 1 - 32 (DL + YL) bits
    constexpr int SH = 64 * N - 1 - 32 * (DL + YL);
    constexpr int SW = SH / 32, SB = SH % 32;
    constexpr int PW = DH - DL + N - YL;
    u64 cy = 0, bw = 0;
LFD_UNROLL
    for (int i = 0; i <= N; ++i) {
        const u32 lo = SW + i < PW ? pr[SW + i] : 0u;
        const u32 up = SW + i + 1 < PW ? pr[SW + i + 1] : 0u;
        const u32 dl = SB ? lf_fshr(lo, up, SB) : lo;
        if (neg) { const u64 v = (u64)dl + bw; const u32 old = c[i]; c[i] = (u32)((u64)old - v); bw = (u64)old < v; }
        else { const u64 v = (u64)c[i] + dl + cy; c[i] = (u32)v; cy = v >> 32; }
    }
    if (neg && (c[N] >> 31)) {                           // below zero: not reachable from C0 >= 2^(32N-1)
LFD_UNROLL
        for (int i = 0; i <= N; ++i) c[i] = i == N - 1 ? 0x80000000u : 0u;
    }
    clamp();
    return true;
}

// RN(sqrt(a)).  With Z the 2N-word radicand of sqrt_restoring and S = sqrt(Z) in [2^(32N-1), 2^(32N)),
// the result mantissa is the integer C nearest S (there are no ties: S is an integer or irrational), and C
// is nearest exactly when -C < Z - C^2 <= C.  The candidate from sqrt_candidate (multiplications only) is
// moved a unit at a time, with Z - C^2 updated exactly, until it passes.  A candidate that is not within a
// few units, which its error bounds rule out, takes the restoring routine.
template <int N> LFD_FN LFD_INLINE Num<N> sqrt(const Num<N>& a) {
    if (a.st || !a.s) return zero<N>(a.st);
    if (a.s < 0) return zero<N>(kInvalid);
    int e = a.e / 2; if (a.e < 0 && (a.e % 2)) --e;
    const int odd = a.e - 2 * e;                    // 0 or 1
    // Z (2N words) and D = Z - C^2 (2N + 1 words, two's complement)
    u32 z[2 * N];
LFD_UNROLL
    for (int k = 0; k < N; ++k) z[k] = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) z[N + i] = a.m[i];
    if (!odd) {
LFD_UNROLL
        for (int k = 0; k < 2 * N; ++k) z[k] = (z[k] >> 1) | (k + 1 < 2 * N ? z[k + 1] << 31 : 0u);
    }
    u32 c[N + 1];
    if (!sqrt_candidate<N>(z, c)) return sqrt_restoring_call<N>(a);
    u32 cm[N], p[2 * N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) cm[i] = c[i];
    mant_mul<N>(cm, cm, p);
    // D within N + 2 words: the words above must be the sign extension
    u32 d[N + 2];
    u32 bo = 0, hi_or = 0, hi_and = 0xffffffffu;
LFD_UNROLL
    for (int k = 0; k < 2 * N; ++k) {
        const u64 t = (u64)p[k] + bo;
        const u32 r = (u32)((u64)z[k] - t);
        bo = (u64)z[k] < t;
        if (k < N + 1) d[k] = r; else { hi_or |= r; hi_and &= r; }
    }
    const u32 ext = bo ? 0xffffffffu : 0u;           // sign word of Z - C^2
    if (N + 1 < 2 * N && (hi_or != ext || hi_and != ext)) return sqrt_restoring_call<N>(a);
    d[N + 1] = ext;
    // adjust: while D > C: D -= 2C + 1, C += 1; while D <= -C: D += 2C - 1, C -= 1
    bool done = false;
LFD_NOUNROLL
    for (int it = 0; it < 6 && !done; ++it) {
        const bool neg = d[N + 1] >> 31;
        // cmp = sign(D - C) for D >= 0, or sign(D + C) for D < 0
        u32 t[N + 2];
        if (!neg) {
            u32 b2 = 0;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { const u64 v = (u64)(k <= N ? c[k] : 0u) + b2; t[k] = (u32)((u64)d[k] - v); b2 = (u64)d[k] < v; }
            u32 o = 0;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) o |= t[k];
            if ((t[N + 1] >> 31) || o == 0) { done = true; break; }   // 0 <= D <= C
            // D -= 2C + 1; C += 1
            u32 b3 = 1;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { const u32 ck = k <= N ? c[k] : 0u; const u64 v = (u64)ck + ck + b3;
                const u64 dv = (u64)d[k] - (u32)v; d[k] = (u32)dv; b3 = (u32)(v >> 32) + (u32)((dv >> 32) & 1u); }
            u32 cy = 1;
LFD_UNROLL
            for (int k = 0; k <= N; ++k) { const u64 v = (u64)c[k] + cy; c[k] = (u32)v; cy = (u32)(v >> 32); }
        } else {
            u64 cy2 = 0;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { const u64 v = (u64)d[k] + (k <= N ? c[k] : 0u) + cy2; t[k] = (u32)v; cy2 = v >> 32; }
            if (!(t[N + 1] >> 31)) {                     // D + C >= 0 ... D > -C unless D + C == 0
                u32 o = 0;
LFD_UNROLL
                for (int k = 0; k < N + 2; ++k) o |= t[k];
                if (o != 0) { done = true; break; }       // -C < D < 0
            }
            // D <= -C: D += 2C - 1; C -= 1
            u64 cy3 = 0;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { const u32 ck = k <= N ? c[k] : 0u; const u64 v = (u64)d[k] + ck + ck + cy3; d[k] = (u32)v; cy3 = v >> 32; }
            u32 b4 = 1;
LFD_UNROLL
            for (int k = 0; k < N + 2; ++k) { const u64 v = (u64)1u * b4; const u32 old = d[k]; d[k] = old - (u32)v; b4 = old < (u32)v; }
            u32 b5 = 1;
LFD_UNROLL
            for (int k = 0; k <= N; ++k) { const u32 old = c[k]; c[k] = old - b5; b5 = old < b5; }
        }
    }
    if (!done) return sqrt_restoring_call<N>(a);
    u32 m[N];
    if (c[N]) {                                      // C = 2^(32N): rounds up into the next binade
LFD_UNROLL
        for (int i = 0; i < N; ++i) m[i] = 0xffffffffu;
        return finish<N>(m, e, 1, true, 0);
    }
LFD_UNROLL
    for (int i = 0; i < N; ++i) m[i] = c[i];
    if (!(m[N - 1] >> 31)) return sqrt_restoring_call<N>(a);   // below the binade: not a valid candidate
    return finish<N>(m, e, 1, false, 0);
}

// ---------------------------------------------------------------- division by a known reciprocal
// r = RN(1 / b) at N + 1 limbs, computed once per divisor (a Cholesky pivot, a triangular solve's diagonal).
template <int N> LFD_FN LFD_INLINE Num<N + 1> reciprocal(const Num<N>& b) {
    Num<N + 1> one, w;
LFD_UNROLL
    for (int i = 0; i <= N; ++i) { one.m[i] = 0; w.m[i] = i ? b.m[i - 1] : 0u; }
    one.m[N] = 0x80000000u; one.e = 0; one.s = 1; one.st = 0;
    w.e = b.e; w.s = b.s; w.st = b.st;
    return div<N + 1>(one, w);
}
// RN(a / b) from r = reciprocal(b).  r has relative error at most 2^-(32N+32), so the exact product a * r,
// normalized to N words, puts the quotient's 32 bits below its last place (g) within two units of those of
// a / b.  Unless g lies within 3 units of 0, of a half or of the wrap (an exact quotient, a tie, a carry into
// the last place or a power of two), the truncated words are those of a / b and g decides the rounding;
// those cases, zeros and statuses take the exact division.  The bits always equal div(a, b).
template <int N> LFD_FN LFD_INLINE Num<N> div_by(const Num<N>& a, const Num<N>& b, const Num<N + 1>& r) {
    if (a.st || b.st || r.st || !a.s || !b.s) return div_call<N>(a, b);
    // p = a * r in [2^(64N+30), 2^(64N+32)): the N x N product with r's top N words, shifted one word,
    // plus a times r's low word
    u32 rh[N], q[2 * N], p[2 * N + 1];
LFD_UNROLL
    for (int i = 0; i < N; ++i) rh[i] = r.m[i + 1];
    mant_mul<N>(a.m, rh, q);
    p[0] = 0;
LFD_UNROLL
    for (int i = 0; i < 2 * N; ++i) p[i + 1] = q[i];
    u32 c = 0;
LFD_UNROLL
    for (int i = 0; i < N; ++i) { const u64 t = (u64)a.m[i] * r.m[0] + p[i] + c; p[i] = (u32)t; c = (u32)(t >> 32); }
LFD_UNROLL
    for (int i = N; i < 2 * N + 1; ++i) { const u64 t = (u64)p[i] + c; p[i] = (u32)t; c = (u32)(t >> 32); }
    const u32 sh = (p[2 * N] >> 31) ? 0u : 1u;
    const u32 g = lf_fshl(p[N - 1], p[N], sh);
    if (g <= 3u || g >= 0xfffffffcu || (g >= 0x7ffffffdu && g <= 0x80000003u)) return div_call<N>(a, b);
    u32 m[N];
LFD_UNROLL
    for (int i = 0; i < N; ++i) m[i] = lf_fshl(p[N + i], p[N + 1 + i], sh);
    return finish<N>(m, (i64)a.e + r.e + 1 - (i64)sh, a.s * b.s, g > 0x80000000u, 0);
}

// ---------------------------------------------------------------- fma
// RN(a*b + c) with one rounding.  One two's-complement window of F = 3N+4 exact words above one
// sticky word, anchored 2 bits above the larger term's top bit.  A term that does not fit lies
// more than 100 bits below the other term's lowest bit (shown by the window sizes), so only its
// sign matters: it becomes +-1 in the sticky word, below every rounding decision.
template <int W, int LEN> LFD_FN LFD_INLINE void place_words(u32 (&v)[W], const u32 (&t)[LEN], i64 offset) {
    // v = t << offset (offset >= 0, the term fits: callers guarantee)
LFD_UNROLL
    for (int k = 0; k < W; ++k) v[k] = k < LEN ? t[k] : 0u;
    shift_up_bits<W>(v, (u32)(offset & 31));
    shift_up_words<W, stages_for<W>()>(v, (u32)(offset >> 5));
}
template <int W> LFD_FN LFD_INLINE void accumulate(u32 (&acc)[W], const u32 (&t)[W], bool negative) {
    if (!negative) { u64 cy = 0;
LFD_UNROLL
        for (int k = 0; k < W; ++k) { u64 x = (u64)acc[k] + t[k] + cy; acc[k] = (u32)x; cy = x >> 32; } }
    else { u32 bo = 0;
LFD_UNROLL
        for (int k = 0; k < W; ++k) { u64 x = (u64)t[k] + bo; u32 old = acc[k]; acc[k] = (u32)((u64)old - x); bo = (u64)old < x; } }
}
template <int N> LFD_FN LFD_INLINE Num<N> fma(const Num<N>& a, const Num<N>& b, const Num<N>& c) {
    const u32 st = a.st | b.st | c.st;
    if (st) return zero<N>(st);
    const bool pz = !a.s || !b.s;
    if (pz) return c.s ? c : zero<N>();
    u32 p[2 * N];
    mant_mul<N>(a.m, b.m, p);
    const int ps = a.s * b.s;
    if (!c.s) return round_product<N>(p, (i64)a.e + b.e, ps, 0);
    constexpr int F = 3 * N + 4, W = F + 1;
    const i64 sp = (i64)a.e + b.e - 2 * (32 * N - 1);
    const i64 tp = sp + 64 * N - 1 - ((p[2 * N - 1] >> 31) ? 0 : 1);
    const i64 sc = (i64)c.e - (32 * N - 1), tc = c.e;
    const i64 hi = tp > tc ? tp : tc;
    const i64 lo = hi + 3 - 32 * (i64)F;            // exponent of window bit 32
    u32 acc[W], t[W];
LFD_UNROLL
    for (int k = 0; k < W; ++k) acc[k] = 0;
    if (sp >= lo) place_words<W, 2 * N>(t, p, 32 + (sp - lo));
    else {
LFD_UNROLL
        for (int k = 0; k < W; ++k) t[k] = k == 0 ? 1u : 0u;
    }
    accumulate<W>(acc, t, ps < 0);
    if (sc >= lo) place_words<W, N>(t, c.m, 32 + (sc - lo));
    else {
LFD_UNROLL
        for (int k = 0; k < W; ++k) t[k] = k == 0 ? 1u : 0u;
    }
    accumulate<W>(acc, t, c.s < 0);
    int sign = 1;
    if (acc[W - 1] >> 31) {
        sign = -1; u64 cy = 1;
LFD_UNROLL
        for (int k = 0; k < W; ++k) { u64 x = (u64)(u32)~acc[k] + cy; acc[k] = (u32)x; cy = x >> 32; }
    }
    return round_general<N, W>(acc, lo - 32, sign, 0);
}
template <int N> LFD_FN LFD_INLINE Num<N> fms(const Num<N>& a, const Num<N>& b, const Num<N>& c) { return fma<N>(a, b, negate<N>(c)); }

// ---------------------------------------------------------------- exact sums by clusters
// acc (len words) += t << off; t has tw words; acc wide enough (callers check)
LFD_FN LFD_INLINE void acc_add(u32* acc, int len, const u32* t, int tw, i64 off) {
    const int ws = (int)(off >> 5), bs = (int)(off & 31);
    u64 cy = 0;
    int k = ws;
    for (int q = 0; q <= tw && k < len; ++q, ++k) {
        u32 v = q < tw ? t[q] << bs : 0u;
        if (bs && q > 0) v |= t[q - 1] >> (32 - bs);
        u64 s = (u64)acc[k] + v + cy; acc[k] = (u32)s; cy = s >> 32;
    }
    for (; cy && k < len; ++k) { u64 s = (u64)acc[k] + cy; acc[k] = (u32)s; cy = s >> 32; }
}

// Rounding record of a nonzero exact magnitude: N result words, exponent, round and sticky bits.
template <int N> struct Rounded { u32 m[N]; i64 e; bool rb, sb; };
template <int N> LFD_FN bool round_info(const u32* x, int len, i64 scale, Rounded<N>& r) {
    int t = -1;
    for (int k = len - 1; k >= 0; --k) if (x[k]) { t = k; break; }
    if (t < 0) return false;
    const int h = 32 * t + 31 - lf_clz(x[t]);
    r.e = scale + h;
    const int shift = h - (32 * N - 1);
    for (int i = 0; i < N; ++i) {
        const int p = shift + 32 * i;
        u32 v = 0;
        if (p <= -32) v = 0;
        else if (p < 0) v = x[0] << (-p);
        else { const int wi = p >> 5, bi = p & 31; v = wi < len ? x[wi] >> bi : 0u; if (bi && wi + 1 < len) v |= x[wi + 1] << (32 - bi); }
        r.m[i] = v;
    }
    r.rb = false; r.sb = false;
    if (shift > 0) {
        const int rbp = shift - 1;
        r.rb = (x[rbp >> 5] >> (rbp & 31)) & 1u;
        bool st = (rbp & 31) && (x[rbp >> 5] & ((1u << (rbp & 31)) - 1u));
        for (int k = 0; k < (rbp >> 5) && !st; ++k) st = x[k] != 0;
        r.sb = st;
    }
    return true;
}

// RN(sum of the nonzero terms of `src`) with one rounding, for any spread of exponents.  A term source has
//   u64 count() const;                                          term slots 0 .. count()-1
//   bool term(u64 k, i64& scale, i64& top, int& sign) const;    false for a zero slot; the term is
//                                                               sign * T * 2^scale with 0 < T < 2^(top - scale)
//   void add(u64 k, u32* acc, int len, i64 off) const;          acc (len words) += T << off
// ---- over-wide clusters: streaming with a sliding window
// The terms with top <= cutoff taken one at a time in the order (top descending, index ascending) are added into
// a window of CW words (positive and negative magnitudes) that covers bits [A - 32 CW, A).  A term that reaches
// below the window moves the window down when the partial sum is small enough to stay inside (nothing is lost);
// otherwise the partial sum lies at least 32 CW - 64N - 2 bits above the term and everything after it is tiny
// against it.
struct StreamPos { i64 top; u64 k; bool started; };
// The next term after `at` in the order (top descending, index ascending) among those with top <= cutoff.
template <class Src> LFD_FN bool stream_next(const Src& src, i64 cutoff, StreamPos& at, i64& scale, i64& top, int& sign) {
    const u64 n = src.count();
    bool found = false; i64 bt = 0; u64 bk = 0;
    for (u64 k = 0; k < n; ++k) {
        i64 s, tp; int sg;
        if (!src.term(k, s, tp, sg) || tp > cutoff) continue;
        if (at.started && (tp > at.top || (tp == at.top && k <= at.k))) continue;
        if (!found || tp > bt || (tp == bt && k < bk)) { found = true; bt = tp; bk = k; }
    }
    if (!found) return false;
    at.top = bt; at.k = bk; at.started = true;
    src.term(bk, scale, top, sign);
    return true;
}
// pos <- |pos - neg|, neg <- 0; returns the sign of pos - neg before (0 when equal).
template <int CW> LFD_FN int stream_normalize(u32* pos, u32* neg) {
    int cmp = 0;
    LFD_NOUNROLL for (int w = CW - 1; w >= 0 && !cmp; --w) if (pos[w] != neg[w]) cmp = pos[w] > neg[w] ? 1 : -1;
    if (cmp < 0) { LFD_NOUNROLL for (int w = 0; w < CW; ++w) { const u32 t = pos[w]; pos[w] = neg[w]; neg[w] = t; } }
    u32 bo = 0;
    LFD_NOUNROLL for (int w = 0; w < CW; ++w) { const u64 d = (u64)neg[w] + bo; const u32 o = pos[w]; pos[w] = (u32)((u64)o - d); bo = (u64)o < d; neg[w] = 0; }
    return cmp;
}
// Index of the highest set bit of x (CW words), -1 when zero.
template <int CW> LFD_FN int stream_msb(const u32* x) {
    LFD_NOUNROLL for (int w = CW - 1; w >= 0; --w) if (x[w]) return 32 * w + 31 - lf_clz(x[w]);
    return -1;
}
// x <- x * 2^d (d >= 0), words shifted out at the top dropped (the caller guarantees they are zero).
template <int CW> LFD_FN void stream_shift_up(u32* x, i64 d) {
    const int q = (int)(d >> 5), r = (int)(d & 31);
    LFD_NOUNROLL for (int w = CW - 1; w >= 0; --w) {
        const int a = w - q;
        u32 v = a >= 0 ? x[a] << r : 0u;
        if (r && a - 1 >= 0) v |= x[a - 1] >> (32 - r);
        x[w] = v;
    }
}
// Window state of one stream: magnitudes (pos, neg), sign of the partial sum after normalisation, anchor A.
template <int CW> struct StreamWin { u32 pos[CW], neg[CW]; i64 A; };
// Adds the terms after `at` (in order) until they run out (returns true) or one no longer fits while the partial sum
// is too large to move the window (returns false with that term pending in `at`, its data in scale/top/sign).
// mult flips every term's sign (-1).  logc: ceil(log2(terms + 2)).
template <int CW, class Src> LFD_FN LFD_NOINLINE bool stream_run(const Src& src, i64 cutoff, int mult, int logc, StreamWin<CW>& W, StreamPos& at,
                                                    i64& scale, i64& top, int& sign) {
    for (;;) {
        StreamPos nx = at;
        if (!stream_next(src, cutoff, nx, scale, top, sign)) return true;
        i64 bottom = W.A - 32 * (i64)CW;
        if (scale < bottom) {
            const int sg = stream_normalize<CW>(W.pos, W.neg);
            const int h = stream_msb<CW>(W.pos);
            if (sg == 0 || h < 0) {
                W.A = top + logc + 2;                                     // empty window: re-anchor at the term
            } else {
                const i64 m = bottom + h;                                 // highest set bit of |partial|
                const i64 A2 = (m + 2 > top + logc + 2) ? m + 2 : top + logc + 2;
                if (A2 - 32 * (i64)CW > scale) {                          // the partial sum dominates the rest
                    if (sg < 0) { LFD_NOUNROLL for (int w = 0; w < CW; ++w) { W.neg[w] = W.pos[w]; W.pos[w] = 0; } }
                    at = nx;
                    return false;
                }
                stream_shift_up<CW>(W.pos, W.A - A2);
                if (sg < 0) { LFD_NOUNROLL for (int w = 0; w < CW; ++w) { W.neg[w] = W.pos[w]; W.pos[w] = 0; } }
                W.A = A2;
            }
            bottom = W.A - 32 * (i64)CW;
        }
        src.add(nx.k, sign * mult > 0 ? W.pos : W.neg, CW, scale - bottom);
        at = nx;
    }
}
// Sign of X * 2^xscale * xsign + mult * (the terms after `at`, and the term at `at` itself when pending), exactly.
// X: xw words (nullptr when absent).
template <int CW, class Src> LFD_FN LFD_NOINLINE int stream_sign(const Src& src, i64 cutoff, StreamPos at, bool pending, int mult, int logc,
                                                    const u32* X, int xw, i64 xscale, int xsign) {
    StreamWin<CW> W;
    LFD_NOUNROLL for (int w = 0; w < CW; ++w) { W.pos[w] = 0; W.neg[w] = 0; }
    i64 xt = INT64_MIN;                                                   // X's highest bit + 1
    LFD_NOUNROLL for (int w = xw - 1; w >= 0; --w) if (X[w]) { xt = xscale + 32 * w + 32 - lf_clz(X[w]); break; }
    i64 s0 = 0, t0 = INT64_MIN; int g0 = 0;
    if (pending) src.term(at.k, s0, t0, g0);
    const i64 top = xt > t0 ? xt : t0;
    W.A = (top == INT64_MIN ? cutoff : top) + logc + 2;
    const i64 bottom = W.A - 32 * (i64)CW;
    if (pending) src.add(at.k, g0 * mult > 0 ? W.pos : W.neg, CW, s0 - bottom);
    if (xt != INT64_MIN) acc_add(xsign > 0 ? W.pos : W.neg, CW, X, xw, xscale - bottom);
    i64 sc, tp; int sg;
    stream_run<CW>(src, cutoff, mult, logc, W, at, sc, tp, sg);           // stops early only when the partial sum dominates
    return stream_normalize<CW>(W.pos, W.neg);
}
// RN of the exact sum of the terms with top <= cutoff, by streaming.  When the window cannot follow, the partial sum
// S is split at bit k = (pending top) + logc + 3 into S_hi (a multiple of 2^k) and S_lo < 2^k; with the tail t (all
// later terms, |t| < 2^(k - 2)) the rounding of S + t is that of S_hi + carry 2^k plus the sign of the remainder in
// [0, 2^k), and carry and remainder follow from the exact signs of S_lo + t and S_lo + t - 2^k.
template <int N, int CW, class Src> LFD_FN LFD_NOINLINE Num<N> stream_value(const Src& src, i64 cutoff, int logc) {
    StreamWin<CW> W;
    LFD_NOUNROLL for (int w = 0; w < CW; ++w) { W.pos[w] = 0; W.neg[w] = 0; }
    StreamPos at{0, 0, false};
    W.A = cutoff + logc + 2;
    i64 sc, tp; int sg;
    const bool done = stream_run<CW>(src, cutoff, 1, logc, W, at, sc, tp, sg);
    const int ssign = stream_normalize<CW>(W.pos, W.neg);
    const i64 bottom = W.A - 32 * (i64)CW;
    if (done) {
        if (!ssign) return zero<N>();
        Rounded<N> R;
        round_info<N>(W.pos, CW, bottom, R);
        return finish<N>(R.m, R.e, ssign, R.rb && (R.sb || (R.m[0] & 1u)), 0);
    }
    const i64 k = tp + logc + 3;                                          // S_lo = |S| mod 2^k
    u32 lo[CW];
    LFD_NOUNROLL for (int w = 0; w < CW; ++w) lo[w] = 0;
    const i64 kb = k - bottom;                                            // bit index of k in the window (> 0)
    LFD_NOUNROLL for (int w = 0; w < CW; ++w) {
        const i64 b0 = 32 * (i64)w;
        if (b0 + 32 <= kb) { lo[w] = W.pos[w]; W.pos[w] = 0; }
        else if (b0 < kb) { const u32 mask = (1u << (kb - b0)) - 1u; lo[w] = W.pos[w] & mask; W.pos[w] &= ~mask; }
    }
    // sign of S_lo + ssign * t, and of S_lo - 2^k + ssign * t
    const int c0 = stream_sign<CW>(src, cutoff, at, true, ssign, logc, lo, CW, bottom, 1);
    int carry = 0, sigma = 0;
    if (kb <= 0) {
        // the pending term lies wholly below the window: S is a multiple of 2^bottom > |t|, so only t's sign matters
        sigma = c0;
    } else {
        u32 hk[CW];                                                       // 2^k - S_lo
        LFD_NOUNROLL for (int w = 0; w < CW; ++w) hk[w] = 0;
        if (kb < 32 * (i64)CW) hk[kb >> 5] = 1u << (kb & 31);
        u32 bo = 0;
        LFD_NOUNROLL for (int w = 0; w < CW; ++w) { const u64 d = (u64)lo[w] + bo; const u32 o = hk[w]; hk[w] = (u32)((u64)o - d); bo = (u64)o < d; }
        const int c1 = stream_sign<CW>(src, cutoff, at, true, ssign, logc, hk, CW, bottom, -1);
        if (c0 < 0) { carry = -1; sigma = 1; }
        else if (c0 == 0) { carry = 0; sigma = 0; }
        else if (c1 < 0) { carry = 0; sigma = 1; }
        else if (c1 == 0) { carry = 1; sigma = 0; }
        else { carry = 1; sigma = 1; }
    }
    if (carry) {                                                          // S_hi +- 2^k (S_hi >> 2^k: no sign change)
        u32 one[1] = {1u};
        if (carry > 0) acc_add(W.pos, CW, one, 1, kb);
        else { LFD_NOUNROLL for (int w = 0; w < CW; ++w) W.neg[w] = 0; acc_add(W.neg, CW, one, 1, kb); stream_normalize<CW>(W.pos, W.neg); }
    }
    Rounded<N> R;
    round_info<N>(W.pos, CW, bottom, R);
    const bool up = R.rb && (R.sb || sigma > 0 || (sigma == 0 && (R.m[0] & 1u)));
    return finish<N>(R.m, R.e, ssign, up, 0);
}

// The terms are summed cluster by cluster from the highest: a cluster holds the highest remaining top and
// grows downwards while some remaining term reaches within gap = 32N + ceil(log2(count + 1)) + 4 bits of its
// lowest bit; it is summed exactly as positive and negative magnitudes in CW words.  The first nonzero
// cluster sum S is kept; everything below it is less than 2^(lowest bit of S - 32N - 2) in magnitude, so of
// the rest only the sign of the next nonzero cluster can matter (to exact ties and exact S).  A cluster wider
// than CW words is streamed (stream_value / stream_sign above), so no input fails.
// STREAM = false leaves the streaming path out (callers whose clusters provably fit: dot2_add's three terms); an
// over-wide cluster then sets *error and gives zero with status invalid.
template <int N, int CW, class Src, bool STREAM = true> LFD_FN Num<N> cluster_round(const Src& src, u32* error) {
    const u64 n = src.count();
    int count = 0;
    i64 T = INT64_MIN;
    for (u64 k = 0; k < n; ++k) {
        i64 s, tp; int sg;
        if (!src.term(k, s, tp, sg)) continue;
        T = tp > T ? tp : T;
        ++count;
    }
    if (!count) return zero<N>();
    int logc = 0;
    while ((1 << logc) < count + 1) ++logc;
    const i64 gap = 32 * N + logc + 4;
    u32 pos[CW], neg[CW];
    i64 cutoff = T;                        // inclusive bound on the tops still to visit
    bool have = false;
    Rounded<N> R; int rsign = 0, sigma = 0;
    for (;;) {
        i64 Tc = INT64_MIN;                // top of the next cluster
        for (u64 k = 0; k < n; ++k) {
            i64 s, tp; int sg;
            if (src.term(k, s, tp, sg) && tp <= cutoff && tp > Tc) Tc = tp;
        }
        if (Tc == INT64_MIN) break;
        i64 low = INT64_MAX;               // lowest bit: grow while a remaining term reaches within `gap`
        for (u64 k = 0; k < n; ++k) {
            i64 s, tp; int sg;
            if (src.term(k, s, tp, sg) && tp == Tc && s < low) low = s;
        }
        for (;;) {
            i64 nl = low;
            for (u64 k = 0; k < n; ++k) {
                i64 s, tp; int sg;
                if (src.term(k, s, tp, sg) && tp <= cutoff && tp > low - gap && s < nl) nl = s;
            }
            if (nl == low) break;
            low = nl;
        }
        const int len = (int)((Tc - low + logc + 2 + 31) / 32) + 1;
        if (len > CW) {
            if constexpr (STREAM) {
                // an over-wide cluster: stream everything from here (tops <= cutoff)
                if (!have) return stream_value<N, CW>(src, cutoff, logc);
                const int rest = stream_sign<CW>(src, cutoff, StreamPos{0, 0, false}, false, 1, logc, nullptr, 0, 0, 1);
                sigma = rest == 0 ? 0 : (rest == rsign ? 1 : -1);
                break;
            } else {
                if (error) lf_flag(error, 1u);
                return zero<N>(kInvalid);
            }
        }
        for (int w = 0; w < len; ++w) { pos[w] = 0; neg[w] = 0; }
        for (u64 k = 0; k < n; ++k) {
            i64 s, tp; int sg;
            if (!src.term(k, s, tp, sg) || !(tp <= cutoff && tp > low - gap)) continue;
            src.add(k, sg > 0 ? pos : neg, len, s - low);
        }
        cutoff = low - gap;
        int cmp = 0;
        for (int w = len - 1; w >= 0 && !cmp; --w) if (pos[w] != neg[w]) cmp = pos[w] > neg[w] ? 1 : -1;
        if (!cmp) continue;                // the cluster cancels exactly
        u32* big = cmp > 0 ? pos : neg;
        const u32* small = cmp > 0 ? neg : pos;
        u32 bo = 0;
        for (int w = 0; w < len; ++w) { u64 d = (u64)small[w] + bo; u32 o = big[w]; big[w] = (u32)((u64)o - d); bo = (u64)o < d; }
        if (!have) { round_info<N>(big, len, low, R); rsign = cmp; have = true; continue; }
        sigma = cmp == rsign ? 1 : -1;     // sign of everything below, relative to S
        break;
    }
    if (!have) return zero<N>();
    // RN(S + sigma * tiny): the tail decides only exact ties and exact S
    const bool up = R.rb && (R.sb || sigma > 0 || (sigma == 0 && (R.m[0] & 1u)));
    return finish<N>(R.m, R.e, rsign, up, 0);
}

// ---------------------------------------------------------------- RN(a*b + c*d + e)
// The two products and the addend as a term source for cluster_round (words in registers or local memory).
template <int N> struct Dot2Terms {
    const u32* w[3]; int len[3]; i64 scale[3]; int sign[3];
    LFD_FN u64 count() const { return 3; }
    LFD_FN bool term(u64 k, i64& s, i64& tp, int& sg) const {
        if (!sign[k]) return false;
        s = scale[k]; tp = scale[k] + 32 * len[k]; sg = sign[k];
        return true;
    }
    LFD_FN void add(u64 k, u32* acc, int alen, i64 off) const { acc_add(acc, alen, w[k], len[k], off); }
};
// One rounding of the exact sum.  Fast path: fma's window, widened to three terms.  One two's-complement window
// of F = 3N+4 words sits above a sticky word, anchored three bits above the highest term's top bit (three terms
// below 2^hi sum below 2^(hi+2), plus the sign).  With lo the window's lowest bit, a term whose lowest bit is at
// or above lo is placed exactly, and a term below 2^(lo-1) in magnitude becomes one unit of the sticky word with
// its sign.  Let P be the exact sum of the placed terms (a multiple of 2^lo) and R that of the dropped ones
// (|R| < 2^lo).  When the dropped terms share a sign, the window holds P' = P + u 2^(lo-32) with sign(u) =
// sign(R).  When moreover |P'| >= 2^(lo+32N), every rounding boundary of the result's binade (representable
// values and midpoints) is a multiple of 2^lo; P + R and P' lie within 2^lo of P on the same side of it (or both
// equal P), in the same binade, so they round alike and the window's rounding is RN(ab + cd + e).  Any other
// case (a term straddling lo, dropped terms of opposite signs, deep cancellation) sums the terms by clusters,
// the limb kernel's exact method, in 8N+4 words: three chained terms of at most 64N bits and two gaps below.
template <int N> LFD_FN LFD_NOINLINE Num<N> dot2_add(const Num<N>& a, const Num<N>& b, const Num<N>& c, const Num<N>& d, const Num<N>& e) {
    const u32 st = a.st | b.st | c.st | d.st | e.st;
    if (st) return zero<N>(st);
    const int s1 = a.s * b.s, s2 = c.s * d.s;
    if (!s1 && !s2) return e.s ? e : zero<N>();
    u32 p1[2 * N], p2[2 * N];
    i64 sc1 = 0, sc2 = 0, top = INT64_MIN;            // scales; top: above the highest term's top bit
    if (s1) { mant_mul<N>(a.m, b.m, p1); sc1 = (i64)a.e + b.e - 2 * (32 * N - 1); const i64 t = sc1 + 64 * N - ((p1[2 * N - 1] >> 31) ? 0 : 1); top = t > top ? t : top; }
    if (s2) { mant_mul<N>(c.m, d.m, p2); sc2 = (i64)c.e + d.e - 2 * (32 * N - 1); const i64 t = sc2 + 64 * N - ((p2[2 * N - 1] >> 31) ? 0 : 1); top = t > top ? t : top; }
    const i64 sce = (i64)e.e - (32 * N - 1);
    if (e.s) top = (i64)e.e + 1 > top ? (i64)e.e + 1 : top;
    constexpr int F = 3 * N + 4, W = F + 1;
    const i64 lo = top + 3 - 32 * (i64)F;
    u32 acc[W], t[W];
LFD_UNROLL
    for (int k = 0; k < W; ++k) acc[k] = 0;
    bool fast = true;
    int dropped = 0;                                  // sign of the sticky units so far
    const auto sticky = [&](int sg) {
        if (dropped && dropped != sg) fast = false;
        dropped = sg;
LFD_UNROLL
        for (int k = 0; k < W; ++k) t[k] = k == 0 ? 1u : 0u;
        accumulate<W>(acc, t, sg < 0);
    };
    if (s1) {
        if (sc1 >= lo) { place_words<W, 2 * N>(t, p1, 32 + (sc1 - lo)); accumulate<W>(acc, t, s1 < 0); }
        else if (sc1 + 64 * N <= lo - 1) sticky(s1);
        else fast = false;
    }
    if (s2 && fast) {
        if (sc2 >= lo) { place_words<W, 2 * N>(t, p2, 32 + (sc2 - lo)); accumulate<W>(acc, t, s2 < 0); }
        else if (sc2 + 64 * N <= lo - 1) sticky(s2);
        else fast = false;
    }
    if (e.s && fast) {
        if (sce >= lo) { place_words<W, N>(t, e.m, 32 + (sce - lo)); accumulate<W>(acc, t, e.s < 0); }
        else if ((i64)e.e + 1 <= lo - 1) sticky(e.s);
        else fast = false;
    }
    if (fast) {
        int sign = 1;
        if (acc[W - 1] >> 31) {
            sign = -1; u64 cy = 1;
LFD_UNROLL
            for (int k = 0; k < W; ++k) { u64 x = (u64)(u32)~acc[k] + cy; acc[k] = (u32)x; cy = x >> 32; }
        }
        int hw = -1;
LFD_UNROLL
        for (int k = 0; k < W; ++k) hw = acc[k] ? k : hw;
        if (hw < 0 && !dropped) return zero<N>();    // exact cancellation
        if (hw >= 0) {
            u32 topw = 0;
LFD_UNROLL
            for (int k = 0; k < W; ++k) topw = k == hw ? acc[k] : topw;
            if (32 * hw + 31 - lf_clz(topw) >= 32 + 32 * N + 1) return round_general<N, W>(acc, lo - 32, sign, 0);
        }
    }
    Dot2Terms<N> src{{p1, p2, e.m}, {2 * N, 2 * N, N}, {sc1, sc2, sce}, {s1, s2, e.s}};
    return cluster_round<N, 8 * N + 4, Dot2Terms<N>, false>(src, nullptr);
}

// ---------------------------------------------------------------- out-of-line forms
// Composite sequences (complex ops, batched LU, strided GEMM) call the wide routines through
// these non-inlined wrappers above 8 limbs: one copy of each routine per kernel keeps code size
// and compile time bounded, while a call costs little next to an N^2-word product.
template <int N> LFD_FN LFD_NOINLINE Num<N> mul_call(const Num<N> a, const Num<N> b) { return mul<N>(a, b); }
template <int N> LFD_FN LFD_NOINLINE Num<N> add_call(const Num<N> a, const Num<N> b) { return add<N>(a, b); }
template <int N> LFD_FN LFD_NOINLINE Num<N> div_call(const Num<N> a, const Num<N> b) { return div<N>(a, b); }
template <int N> LFD_FN LFD_INLINE Num<N> mulx(const Num<N>& a, const Num<N>& b) { if constexpr (N > 8) return mul_call<N>(a, b); else return mul<N>(a, b); }
template <int N> LFD_FN LFD_INLINE Num<N> addx(const Num<N>& a, const Num<N>& b) { if constexpr (N > 8) return add_call<N>(a, b); else return add<N>(a, b); }
template <int N> LFD_FN LFD_INLINE Num<N> subx(const Num<N>& a, const Num<N>& b) { return addx<N>(a, negate<N>(b)); }
template <int N> LFD_FN LFD_INLINE Num<N> divx(const Num<N>& a, const Num<N>& b) { if constexpr (N > 8) return div_call<N>(a, b); else return div<N>(a, b); }

// ---------------------------------------------------------------- complex (composed, core.hpp:353-419)
template <int N> struct Cpx { Num<N> re, im; };
template <int N> LFD_FN LFD_INLINE Cpx<N> cadd(const Cpx<N>& a, const Cpx<N>& b) { return {addx<N>(a.re, b.re), addx<N>(a.im, b.im)}; }
template <int N> LFD_FN LFD_INLINE Cpx<N> cmul(const Cpx<N>& a, const Cpx<N>& b) {
    return {subx<N>(mulx<N>(a.re, b.re), mulx<N>(a.im, b.im)), addx<N>(mulx<N>(a.re, b.im), mulx<N>(a.im, b.re))};
}
template <int N> LFD_FN LFD_INLINE Cpx<N> cdiv(const Cpx<N>& a, const Cpx<N>& b) {
    const Num<N> d = addx<N>(mulx<N>(b.re, b.re), mulx<N>(b.im, b.im));
    return {divx<N>(addx<N>(mulx<N>(a.re, b.re), mulx<N>(a.im, b.im)), d), divx<N>(subx<N>(mulx<N>(a.im, b.re), mulx<N>(a.re, b.im)), d)};
}
template <int N> LFD_FN LFD_INLINE Cpx<N> cfma(const Cpx<N>& a, const Cpx<N>& b, const Cpx<N>& c) {
    return {dot2_add<N>(a.re, b.re, negate<N>(a.im), b.im, c.re), dot2_add<N>(a.re, b.im, a.im, b.re, c.im)};
}
template <int N> LFD_FN LFD_INLINE Cpx<N> cfms(const Cpx<N>& a, const Cpx<N>& b, const Cpx<N>& c) {
    return cfma<N>(a, b, Cpx<N>{negate<N>(c.re), negate<N>(c.im)});
}
template <int N> LFD_FN LFD_INLINE Cpx<N> cload(const u32* p) { return {load<N>(p), load<N>(p + N + 3)}; }
template <int N> LFD_FN LFD_INLINE Cpx<N> cload_plain(const u32* p) { return {load_plain<N>(p), load_plain<N>(p + N + 3)}; }
template <int N> LFD_FN LFD_INLINE void cstore(u32* p, const Cpx<N>& z) { store<N>(p, z.re); store<N>(p + N + 3, z.im); }

}  // namespace lfd
