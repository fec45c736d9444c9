#pragma once
// Element types and scalar arithmetic of the limbforge API (the reference's include/limbforge/core.hpp).
// Number<N> = {uint32 limb[N] little endian (top bit set when nonzero), int exponent, int sign, uint32
// status}, value = sign * int(limb) * 2^(exponent - (32N-1)); Complex<N> = {re, im}.
//
// The scalar functions below (add, mul, div, sqrt, fma, dot2_add, the complex forms, pack and the word
// division) run on the calling host thread and are the same source as the GPU kernels
// (detail/arith.hpp, compiled here by the host compiler): every result is the correctly rounded value
// (round to nearest, ties to even) of the exact operation, bit for bit what the GPU returns.  Batched
// work belongs on Engine / CommandBatch (engine.hpp).
#include <cstdint>
#include <cstring>
#include "detail/arith.hpp"
#include "version.hpp"

namespace limbforge {
using word = std::uint32_t;
using dword = std::uint64_t;
using exponent_type = std::int64_t;
enum Status : word { ok = 0, division_by_zero = 1, exponent_overflow = 2, invalid = 4 };
template <int N> struct Number {
    word limb[N];
    int exponent;
    int sign;
    word status;
};
template <int Bits> struct FloatType {
    static_assert(Bits >= 64 && Bits <= 1024 && Bits % 32 == 0, "precision must be a multiple of 32 in [64,1024]");
    using type = Number<Bits / 32>;
};
template <int Bits> using Float = typename FloatType<Bits>::type;
template <int N> struct Complex { Number<N> re, im; };

template <int N> inline Number<N> zero(word status = ok) {
    Number<N> r;
    for (int i = 0; i < N; ++i) r.limb[i] = 0;
    r.exponent = 0; r.sign = 0; r.status = status;
    return r;
}
template <int N> inline Number<N> negate(Number<N> a) { a.sign = -a.sign; return a; }
// |a| <=> |b| by exact comparison (zero smallest).
template <int N> inline int magnitude_compare(const Number<N>& a, const Number<N>& b) {
    if (!a.sign) return b.sign ? -1 : 0;
    if (!b.sign) return 1;
    if (a.exponent != b.exponent) return a.exponent > b.exponent ? 1 : -1;
    for (int i = N - 1; i >= 0; --i) if (a.limb[i] != b.limb[i]) return a.limb[i] > b.limb[i] ? 1 : -1;
    return 0;
}

namespace detail {
// Number<N> and the arithmetic's element are the same 4N+12 bytes.
template <int N> inline lfd::Num<N> num(const Number<N>& a) {
    static_assert(sizeof(Number<N>) == sizeof(lfd::Num<N>), "element layouts differ");
    lfd::Num<N> r; std::memcpy(&r, &a, sizeof r); return r;
}
template <int N> inline Number<N> number(const lfd::Num<N>& a) { Number<N> r; std::memcpy(&r, &a, sizeof r); return r; }
template <int N> inline lfd::Cpx<N> cpx(const Complex<N>& a) { return {num(a.re), num(a.im)}; }
template <int N> inline Complex<N> complex_of(const lfd::Cpx<N>& a) { return {number(a.re), number(a.im)}; }
}  // namespace detail

// ---- bit helpers on word arrays (little endian)
template <int W> inline int highest(const word (&a)[W]) {                 // index of the top set bit, -1 for zero
    for (int i = W - 1; i >= 0; --i) if (a[i]) return 32 * i + 31 - lfd::lf_clz(a[i]);
    return -1;
}
template <int W> inline word extract(const word (&a)[W], int bit) {        // 32 bits from `bit` (zeros outside)
    if (bit < 0) return 0;
    const int i = bit / 32, s = bit % 32;
    const word lo = i < W ? a[i] : 0u, hi = i + 1 < W ? a[i + 1] : 0u;
    return lfd::lf_fshr(lo, hi, (unsigned)s);
}
template <int W> inline bool any_below(const word (&a)[W], int bit) {      // some set bit strictly below `bit`
    for (int i = 0; i < W && 32 * i < bit; ++i) {
        const int n = bit - 32 * i;
        if (n >= 32 ? a[i] != 0 : (a[i] & ((word(1) << n) - 1u)) != 0) return true;
    }
    return false;
}
// One unit added at the last place (a carry out of the top renormalizes).
template <int N> inline void increment(Number<N>& r) {
    for (int i = 0; i < N; ++i) if (++r.limb[i]) return;
    r.limb[N - 1] = word(1) << 31; ++r.exponent;
}
// Zero with exponent_overflow when the exponent left [-1e9, 1e9].
template <int N> inline Number<N> checked(Number<N> r) {
    if (r.exponent > 1000000000 || r.exponent < -1000000000) return zero<N>(r.status | exponent_overflow);
    return r;
}
// RN(sign * int(a) * 2^scale) to N limbs; exponent range as every operation.
template <int N, int W> inline Number<N> pack(const word (&a)[W], exponent_type scale, int sign, word status) {
    constexpr int X = W > N + 1 ? W : N + 1;
    word x[X];
    for (int i = 0; i < X; ++i) x[i] = i < W ? a[i] : 0u;
    return detail::number(lfd::round_general<N, X>(x, scale, sign, status));
}

// ---- real operations, one rounding each (Padded is accepted for source compatibility and changes nothing)
template <int N> inline Number<N> add(const Number<N>& a, const Number<N>& b) { return detail::number(lfd::add<N>(detail::num(a), detail::num(b))); }
template <int N> inline Number<N> sub(const Number<N>& a, const Number<N>& b) { return detail::number(lfd::sub<N>(detail::num(a), detail::num(b))); }
template <int N, bool Padded = true> inline Number<N> mul(const Number<N>& a, const Number<N>& b) { return detail::number(lfd::mul<N>(detail::num(a), detail::num(b))); }
template <int N> inline Number<N> square(const Number<N>& a) { return mul<N>(a, a); }
template <int N, bool Padded = true> inline Number<N> div(const Number<N>& a, const Number<N>& b) { return detail::number(lfd::div<N>(detail::num(a), detail::num(b))); }
template <int N> inline Number<N> sqrt(const Number<N>& a) { return detail::number(lfd::sqrt<N>(detail::num(a))); }
// RN(a*b + c) and RN(a*b - c)
template <int N> inline Number<N> fma(const Number<N>& a, const Number<N>& b, const Number<N>& c) { return detail::number(lfd::fma<N>(detail::num(a), detail::num(b), detail::num(c))); }
template <int N> inline Number<N> fms(const Number<N>& a, const Number<N>& b, const Number<N>& c) { return detail::number(lfd::fms<N>(detail::num(a), detail::num(b), detail::num(c))); }
// RN(a*b + c*d + e) with one rounding
template <int N> inline Number<N> dot2_add(const Number<N>& a, const Number<N>& b, const Number<N>& c, const Number<N>& d, const Number<N>& e) {
    return detail::number(lfd::dot2_add<N>(detail::num(a), detail::num(b), detail::num(c), detail::num(d), detail::num(e)));
}
template <int N> inline Number<N> dot2_add_rolled(const Number<N>& a, const Number<N>& b, const Number<N>& c, const Number<N>& d, const Number<N>& e) {
    return dot2_add<N>(a, b, c, d, e);
}

// ---- complex operations: composed (cadd, cmul, cdiv: each real step rounded) and fused (each component one rounding)
template <int N> inline Complex<N> cadd(const Complex<N>& a, const Complex<N>& b) { return detail::complex_of(lfd::cadd<N>(detail::cpx(a), detail::cpx(b))); }
template <int N> inline Complex<N> cmul(const Complex<N>& a, const Complex<N>& b) { return detail::complex_of(lfd::cmul<N>(detail::cpx(a), detail::cpx(b))); }
template <int N> inline Complex<N> cdiv(const Complex<N>& a, const Complex<N>& b) { return detail::complex_of(lfd::cdiv<N>(detail::cpx(a), detail::cpx(b))); }
template <int N> inline Complex<N> cfma(const Complex<N>& a, const Complex<N>& b, const Complex<N>& c) { return detail::complex_of(lfd::cfma<N>(detail::cpx(a), detail::cpx(b), detail::cpx(c))); }
template <int N> inline Complex<N> cfms(const Complex<N>& a, const Complex<N>& b, const Complex<N>& c) { return detail::complex_of(lfd::cfms<N>(detail::cpx(a), detail::cpx(b), detail::cpx(c))); }
template <int N> inline Complex<N> cfma_rolled(const Complex<N>& a, const Complex<N>& b, const Complex<N>& c) { return cfma<N>(a, b, c); }

// ---- word division with a reused reciprocal (Moller & Granlund 2011, algorithm 4): (high:low) / d for
// normalized d (top bit set), high < d, inv = floor((2^64 - 1) / d) - 2^32.
struct WordDivision { word quotient, remainder; };
inline WordDivision divide_word(word high, word low, word d, word inv) {
    word r = 0;
    const word q = lfd::div2by1(high, low, d, inv, r);
    return {q, r};
}
}  // namespace limbforge
