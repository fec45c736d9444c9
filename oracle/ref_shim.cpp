// C entry points over the reference's own CPU arithmetic (TEST INFRASTRUCTURE ONLY).
// Compiled by oracle/Makefile against the reference headers where they lie
// (include/limbforge/core.hpp, include/limbforge/linalg.hpp::exact_dot_add) into
// oracle/_ref/libref.so, which the tests use to pin the C oracle (lf_oracle.c) bit for bit.
// Nothing here is product code and nothing of the reference is copied: this file only
// instantiates the reference templates for the 31 widths and exports them with C linkage.
#include "limbforge/core.hpp"
#include "limbforge/linalg.hpp"
#include <cstring>
#include <cstddef>

namespace {
using namespace limbforge;
template<int N> int ew(int op, const void* a, const void* b, const void* c, void* out, std::size_t count) {
    using F = Number<N>; using C = Complex<N>;
    const bool cx = (op >= 4 && op <= 6) || op == 11 || op == 12;
    for (std::size_t i = 0; i < count; ++i) {
        if (cx) {
            C x, y, z, r; std::memcpy(&x, static_cast<const C*>(a) + i, sizeof(C));
            if (b) std::memcpy(&y, static_cast<const C*>(b) + i, sizeof(C));
            if (c) std::memcpy(&z, static_cast<const C*>(c) + i, sizeof(C));
            switch (op) {
            case 4: r = cadd(x, y); break; case 5: r = cmul(x, y); break; case 6: r = cdiv(x, y); break;
            case 11: r = cfma(x, y, z); break; case 12: r = cfms(x, y, z); break; default: return 1;
            }
            std::memcpy(static_cast<C*>(out) + i, &r, sizeof(C));
        } else {
            F x, y, z, r; std::memcpy(&x, static_cast<const F*>(a) + i, sizeof(F));
            if (b) std::memcpy(&y, static_cast<const F*>(b) + i, sizeof(F));
            if (c) std::memcpy(&z, static_cast<const F*>(c) + i, sizeof(F));
            switch (op) {
            case 0: r = add(x, y); break; case 1: r = sub(x, y); break; case 2: r = mul(x, y); break;
            case 3: r = div(x, y); break; case 7: r = square(x); break; case 8: r = limbforge::sqrt(x); break;
            case 9: r = fma(x, y, z); break; case 10: r = fms(x, y, z); break; default: return 1;
            }
            std::memcpy(static_cast<F*>(out) + i, &r, sizeof(F));
        }
    }
    return 0;
}
template<int N> int dot(const void* c, int subtract, const void* a, long sa, const void* b, long sb, std::size_t K, void* out) {
    using F = Number<N>;
    F r = exact_dot_add<N>(static_cast<const F*>(c), subtract != 0, static_cast<const F*>(a), sa, static_cast<const F*>(b), sb, K);
    std::memcpy(out, &r, sizeof(F));
    return 0;
}
template<int N> int d2(const void* a, const void* b, const void* c, const void* d, const void* e, void* out, std::size_t count) {
    using F = Number<N>;
    for (std::size_t i = 0; i < count; ++i) {
        F r = dot2_add<N>(static_cast<const F*>(a)[i], static_cast<const F*>(b)[i], static_cast<const F*>(c)[i],
                          static_cast<const F*>(d)[i], static_cast<const F*>(e)[i]);
        std::memcpy(static_cast<F*>(out) + i, &r, sizeof(F));
    }
    return 0;
}
template<int N = 2, class Fn> int by_limbs(int n, Fn&& f) {
    if constexpr (N <= 32) { if (n == N) return f(std::integral_constant<int, N>{}); return by_limbs<N + 1>(n, f); }
    else return 1;
}
}  // namespace

extern "C" {
int ref_elementwise(int bits, int op, const void* a, const void* b, const void* c, void* out, std::size_t count) {
    if (bits < 64 || bits > 1024 || bits % 32) return 1;
    return by_limbs(bits / 32, [&](auto n) { return ew<decltype(n)::value>(op, a, b, c, out, count); });
}
int ref_exact_dot_add(int bits, const void* c, int subtract, const void* a, long sa, const void* b, long sb, std::size_t K, void* out) {
    return by_limbs(bits / 32, [&](auto n) { return dot<decltype(n)::value>(c, subtract, a, sa, b, sb, K, out); });
}
int ref_dot2_add(int bits, const void* a, const void* b, const void* c, const void* d, const void* e, void* out, std::size_t count) {
    return by_limbs(bits / 32, [&](auto n) { return d2<decltype(n)::value>(a, b, c, d, e, out, count); });
}
int ref_divide_word(unsigned high, unsigned low, unsigned d, unsigned* q, unsigned* r) {
    auto res = divide_word(high, low, d, word(~dword(0) / d - (dword(1) << 32)));
    *q = res.quotient; *r = res.remainder; return 0;
}
}
