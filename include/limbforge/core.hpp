#pragma once
// Element types of the limbforge API (the layouts of the reference's include/limbforge/core.hpp:22-34):
// Number<N> = {uint32 limb[N] little endian (top bit set when nonzero), int exponent, int sign, uint32
// status}, value = sign * int(limb) * 2^(exponent - (32N-1)); Complex<N> = {re, im}.  The arithmetic on
// these types runs on the GPU through Engine / CommandBatch (engine.hpp); this header only defines
// the types and the non-arithmetic helpers.
#include <cstdint>

namespace limbforge {
using word = std::uint32_t;
using dword = std::uint64_t;
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
}  // namespace limbforge
