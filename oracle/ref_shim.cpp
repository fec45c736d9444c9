// C entry points over the reference's own CPU arithmetic (TEST INFRASTRUCTURE ONLY).
// Compiled by oracle/Makefile against the reference headers where they lie
// (include/limbforge/core.hpp, include/limbforge/linalg.hpp::exact_dot_add) into
// oracle/_ref/libref.so, which the tests use to pin the C oracle (lf_oracle.c) bit for bit.
// Nothing here is product code and nothing of the reference is copied: this file instantiates
// the reference templates for the 31 widths and exports them with C linkage, and restates one
// sequence (the blocked Householder QR) on top of those templates.
#include "limbforge/core.hpp"
#include "limbforge/linalg.hpp"
#include <cstring>
#include <vector>
#include <algorithm>
#include <climits>
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
// Unpivoted Householder QR in the blocked right-looking form of the reference library (src/linalg.mm:488-790 with
// every product on the host: panels column by column with the panel's W rows Wp and Gram columns, then one
// W = P(V^T X), Y = P(T^T W), X = D(X; V, Y) update per block), driven entirely by the reference's own arithmetic
// (exact_dot, exact_dot_add, sqrt, sub, div, mul, negate).  The sequence is restated here; the oracle's
// column-by-column form must give the same bits.
template<int N> Number<N> pow2(int e) { Number<N> x = zero<N>(); x.limb[N - 1] = 0x80000000u; x.sign = 1; x.exponent = e; return x; }
template<int N> Number<N> times2(Number<N> x, long e) {
    if (!x.sign) return x;
    const long r = long(x.exponent) - e;
    if (r > 1000000000L || r < -1000000000L) return zero<N>(x.status | exponent_overflow);
    x.exponent = int(r); return x;
}
template<int N> int qr_blocked(const void* Ain, std::size_t m, std::size_t n, std::size_t block, int rank_bits, void* Rout, void* Vout,
                               void* Tout, void* tauout, long* info) {
    using F = Number<N>;
    const F* A = static_cast<const F*>(Ain); F* R = static_cast<F*>(Rout); F* V = static_cast<F*>(Vout);
    F* T = static_cast<F*>(Tout); F* tau = static_cast<F*>(tauout);
    const std::size_t nb = block && block < n ? block : n, blocks = nb ? (n + nb - 1) / nb : 0;
    std::vector<F> W(A, A + m * n);
    std::fill(V, V + m * n, zero<N>()); std::fill(T, T + blocks * nb * nb, zero<N>()); std::fill(tau, tau + n, zero<N>());
    std::size_t rank = n; int reason = 0; word status = 0; long top = LONG_MIN;
    std::vector<F> Wb(nb * n + 1), Yb(nb * n + 1), Wp(nb * nb + 1), G(nb + 1), y(nb + 1);
    const F two = pow2<N>(1), one = pow2<N>(0);
    auto update = [&](std::size_t b, std::size_t c0, std::size_t c1) {
        const std::size_t k0 = b * nb, kb = std::min(n, k0 + nb) - k0, mr = m - k0;
        const F* Vb = V + k0 * n + k0; const F* Tb = T + b * nb * nb; F* Xb = W.data() + k0 * n;
        for (std::size_t i = 0; i < kb; ++i) for (std::size_t j = c0; j < c1; ++j) Wb[i * n + j] = exact_dot<N>(Vb + i, std::ptrdiff_t(n), Xb + j, std::ptrdiff_t(n), mr);
        for (std::size_t i = 0; i < kb; ++i) for (std::size_t j = c0; j < c1; ++j) Yb[i * n + j] = exact_dot<N>(Tb + i, std::ptrdiff_t(nb), Wb.data() + j, std::ptrdiff_t(n), kb);
        for (std::size_t r = 0; r < mr; ++r) for (std::size_t j = c0; j < c1; ++j)
            Xb[r * n + j] = exact_dot_add<N>(&Xb[r * n + j], true, Vb + r * n, 1, Yb.data() + j, std::ptrdiff_t(n), kb);
    };
    auto panel = [&](std::size_t k0, std::size_t k1) {
        const std::size_t kb = k1 - k0, mr = m - k0; F* Tb = T + (k0 / nb) * nb * nb;
        std::vector<F> Pt(kb * mr), Vt(kb * mr, zero<N>());
        for (std::size_t c = 0; c < kb; ++c) for (std::size_t r = 0; r < mr; ++r) Pt[c * mr + r] = W[(k0 + r) * n + k0 + c];
        for (std::size_t c = 0; c < kb; ++c) {
            const std::size_t j = k0 + c; F* x = Pt.data() + c * mr;
            const std::size_t q = std::min(j, rank) - k0;
            for (std::size_t i = 0; i < q; ++i) y[i] = exact_dot<N>(Tb + i, std::ptrdiff_t(nb), Wp.data() + c, std::ptrdiff_t(nb), i + 1);
            if (q) for (std::size_t r = 0; r < mr; ++r) x[r] = exact_dot_add<N>(&x[r], true, Vt.data() + r, std::ptrdiff_t(mr), y.data(), 1, q);
            if (rank < n) continue;
            F* xc = x + c; const std::size_t len = mr - c;
            const F s = exact_dot<N>(xc, 1, xc, 1, len);
            bool below = false; for (std::size_t r = 1; r < len; ++r) below |= xc[r].sign != 0;
            int why = s.status ? 3 : (!xc[0].sign && !below) ? 1 : 0;
            F beta = xc[0], v0 = one;
            if (!why && below) { beta = limbforge::sqrt(s); if (xc[0].sign >= 0) beta = negate(beta); v0 = sub(xc[0], beta); }
            if (!why && rank_bits > 0 && top != LONG_MIN && long(beta.exponent) + rank_bits < top) why = 2;
            if (why) { rank = j; reason = why; status = s.status; continue; }
            F* v = Vt.data() + c * mr + c; F tj = zero<N>();
            if (below) { const long e = v0.exponent; v[0] = times2<N>(v0, e); for (std::size_t r = 1; r < len; ++r) v[r] = times2<N>(xc[r], e);
                         tj = div(two, exact_dot<N>(v, 1, v, 1, len)); }
            else v[0] = one;
            xc[0] = beta; tau[j] = tj; top = std::max(top, long(beta.exponent));
            for (std::size_t u = 0; u + 1 < kb; ++u) {
                if (u < c) G[u] = exact_dot<N>(Vt.data() + u * mr + c, 1, v, 1, len);
                else Wp[c * nb + u + 1] = exact_dot<N>(v, 1, Pt.data() + (u + 1) * mr + c, 1, len);
            }
            Tb[c * nb + c] = tj;
            for (std::size_t l = 0; l < c; ++l) Tb[l * nb + c] = negate(mul(tj, exact_dot<N>(Tb + l * nb + l, 1, G.data() + l, 1, c - l)));
        }
        for (std::size_t c = 0; c < kb; ++c) for (std::size_t r = 0; r < mr; ++r) { W[(k0 + r) * n + k0 + c] = Pt[c * mr + r]; V[(k0 + r) * n + k0 + c] = Vt[c * mr + r]; }
        return std::min(k1, rank);
    };
    std::size_t k0 = 0, k1 = std::min(n, nb), p = n ? panel(0, k1) : 0;
    while (k1 < n) {
        const std::size_t b = k0 / nb;
        if (p < k1) { if (p > k0) update(b, k1, n); break; }
        update(b, k1, n);
        const std::size_t k2 = std::min(n, k1 + nb);
        p = panel(k1, k2); k0 = k1; k1 = k2;
    }
    for (std::size_t i = 0; i < n; ++i) for (std::size_t j = 0; j < n; ++j) R[i * n + j] = j >= std::min(i, rank) ? W[i * n + j] : zero<N>();
    info[0] = long(rank); info[1] = reason; info[2] = long(status); info[3] = 0;
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
int ref_qr_blocked(int bits, const void* A, std::size_t m, std::size_t n, std::size_t block, int rank_bits, void* R, void* V, void* T,
                   void* tau, long* info) {
    return by_limbs(bits / 32, [&](auto w) { return qr_blocked<decltype(w)::value>(A, m, n, block, rank_bits, R, V, T, tau, info); });
}
int ref_divide_word(unsigned high, unsigned low, unsigned d, unsigned* q, unsigned* r) {
    auto res = divide_word(high, low, d, word(~dword(0) / d - (dword(1) << 32)));
    *q = res.quotient; *r = res.remainder; return 0;
}
}
