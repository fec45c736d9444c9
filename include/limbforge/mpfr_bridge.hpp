#pragma once
// Host conversions between the element format and MPFR / MPC values (the reference's
// include/limbforge/mpfr_bridge.hpp): typed and runtime-width, single values and arrays split over host threads,
// from_decimal, and (beyond the reference) conversions straight into and out of an Engine buffer's pinned host mirror.
// Optional: include it only with <mpfr.h> on the include path and link MPFR and GMP; the mpc_t forms need <mpc.h> on
// the include path and no libmpc symbols (define LIMBFORGE_NO_MPC to leave them out).
//
// from_mpfr rounds to the element width, ties to even, by reading the MPFR significand directly: NaN and infinities give
// invalid, zero the canonical zero, an exponent outside [-1e9, 1e9] exponent_overflow; the MPFR inexact flag is raised
// when rounding discards bits.  to_mpfr is exact when the output's precision is at least the element width and rounds
// to nearest-even otherwise; an element with a status throws runtime_error.  Values land in the output's own
// significand; a result outside MPFR's current exponent range goes through mpfr_set_z_2exp, which applies MPFR's
// overflow and underflow rules.  The element's exponent range lies far inside MPFR's default range, so the caller's
// range only matters for ranges narrowed below +-1e9.
#include "core.hpp"
#include "engine.hpp"
#include <mpfr.h>
#if !defined(LIMBFORGE_NO_MPC) && __has_include(<mpc.h>)
#include <mpc.h>
#define LIMBFORGE_HAS_MPC 1
#endif
#include <algorithm>
#include <cstring>
#include <exception>
#include <stdexcept>
#include <string>
#include <system_error>
#include <thread>
#include <type_traits>
#include <vector>

namespace limbforge {
namespace bridge_detail {

// MPFR keeps a regular value's significand in ceil(prec / 64) GMP limbs, most significant bit set and the low bits
// zero.  On a little-endian host with 64-bit nail-free limbs those are, read as 32-bit words, the element's limb order.
#if defined(__BYTE_ORDER__) && __BYTE_ORDER__ == __ORDER_LITTLE_ENDIAN__ && GMP_NUMB_BITS == 64 && GMP_NAIL_BITS == 0
constexpr bool kDirect = true;
#else
constexpr bool kDirect = false;
#endif
constexpr long kExponentLimit = 1000000000L;

inline std::size_t words_of(mpfr_prec_t p) { return 2 * ((std::size_t(p) + 63) / 64); }
inline word get(const void* s, std::size_t i) { word w; std::memcpy(&w, static_cast<const char*>(s) + 4 * i, 4); return w; }

struct Range {
    mpfr_exp_t lo, hi;
    static Range current() { return {mpfr_get_emin(), mpfr_get_emax()}; }
    void adopt() const { mpfr_set_emin(lo); mpfr_set_emax(hi); }
};

// RN(q) to `keep` significant bits of an N-word significand whose top bit is set, in place; returns the carry out of
// the top (q is then 2^(32N-1)) and reports whether bits were discarded.
template <int N> inline bool round_words(word* q, int keep, bool& inexact) {
    const int cut = 32 * N - keep;                  // bits to clear, >= 1
    const int gw = (cut - 1) / 32, gb = (cut - 1) % 32, kw = cut / 32, kb = cut % 32;
    const bool guard = (q[gw] >> gb) & 1;
    bool sticky = (q[gw] & ((word(1) << gb) - 1)) != 0;
    for (int i = 0; !sticky && i < gw; ++i) sticky = q[i] != 0;
    const bool odd = kw < N && ((q[kw] >> kb) & 1);
    inexact = guard || sticky;
    for (int i = 0; i < kw; ++i) q[i] = 0;
    if (kw < N) q[kw] &= ~((word(1) << kb) - 1);
    if (!(guard && (sticky || odd))) return false;
    dword c = dword(q[kw]) + (dword(1) << kb);
    q[kw] = word(c);
    for (int i = kw + 1; (c >> 32) && i < N; ++i) { c = dword(q[i]) + 1; q[i] = word(c); }
    if (!(c >> 32)) return false;
    q[N - 1] = word(1) << 31;
    return true;
}

template <int N> inline Number<N> finish(Number<N> r, long e) {
    if (e > kExponentLimit || e < -kExponentLimit) return zero<N>(exponent_overflow);
    r.exponent = int(e);
    return r;
}

// Portable path (no direct limb access): the value rounded by MPFR to 32N bits, then exported as an integer.
template <int N> inline Number<N> from_general(mpfr_srcptr in) {
    mpfr_t t;
    mpfr_init2(t, 32 * N);
    const Range r = Range::current();
    mpfr_set_emin(mpfr_get_emin_min()); mpfr_set_emax(mpfr_get_emax_max());
    mpfr_set(t, in, MPFR_RNDN);
    r.adopt();
    Number<N> out = zero<N>();
    out.sign = mpfr_sgn(t) < 0 ? -1 : 1;
    const long e = long(mpfr_get_exp(t)) - 1;
    mpz_t z; mpz_init(z);
    mpfr_get_z_2exp(z, t);
    const std::size_t bits = mpz_sizeinbase(z, 2);
    mpz_mul_2exp(z, z, 32 * N - bits);
    std::size_t count = 0;
    mpz_export(out.limb, &count, -1, sizeof(word), 0, 0, z);
    mpz_clear(z); mpfr_clear(t);
    return finish<N>(out, e);
}

template <int N> inline Number<N> from(mpfr_srcptr in) {
    if (!mpfr_number_p(in)) return zero<N>(invalid);
    if (mpfr_zero_p(in)) return zero<N>();
    if (!kDirect) return from_general<N>(in);
    const void* s = mpfr_custom_get_significand(in);
    const std::size_t M = words_of(mpfr_get_prec(in));
    Number<N> r;
    r.status = ok;
    r.sign = mpfr_signbit(in) ? -1 : 1;
    long e = long(mpfr_get_exp(in)) - 1;
    if (M <= std::size_t(N)) {
        std::memset(r.limb, 0, 4 * (N - M));
        std::memcpy(r.limb + (N - M), s, 4 * M);
        return finish<N>(r, e);
    }
    // keep the top N words; the word below gives the guard bit, everything lower the sticky bit
    const std::size_t low = M - N;
    std::memcpy(r.limb, static_cast<const char*>(s) + 4 * low, 4 * N);
    const word g = get(s, low - 1);
    bool sticky = (g & 0x7fffffffu) != 0;
    for (std::size_t i = 0; !sticky && i + 1 < low; ++i) sticky = get(s, i) != 0;
    const bool guard = g >> 31;
    if (guard || sticky) mpfr_set_inexflag();
    if (guard && (sticky || (r.limb[0] & 1))) {
        int i = 0;
        while (i < N && ++r.limb[i] == 0) ++i;
        if (i == N) { r.limb[N - 1] = word(1) << 31; ++e; }
    }
    return finish<N>(r, e);
}

[[noreturn]] inline void status_error(word st) { throw std::runtime_error("WolfNum arithmetic status " + std::to_string(st)); }

// x (status 0) into out at out's precision, through MPFR's own rounding and range rules.
template <int N> inline void to_general(mpfr_ptr out, const Number<N>& x) {
    mpz_t z; mpz_init(z);
    mpz_import(z, N, -1, sizeof(word), 0, 0, x.limb);
    if (x.sign < 0) mpz_neg(z, z);
    mpfr_set_z_2exp(out, z, mpfr_exp_t(x.exponent) - (32 * N - 1), MPFR_RNDN);
    mpz_clear(z);
}

template <int N> inline void to(mpfr_ptr out, const Number<N>& x) {
    if (x.status) status_error(x.status);
    if (!x.sign) { mpfr_set_zero(out, 1); return; }
    if (!kDirect) { to_general<N>(out, x); return; }
    const mpfr_prec_t p = mpfr_get_prec(out);
    const std::size_t D = words_of(p);
    mpfr_exp_t e = mpfr_exp_t(x.exponent) + 1;
    word q[N];
    std::memcpy(q, x.limb, sizeof q);
    bool inexact = false;
    if (p < 32 * N && round_words<N>(q, int(p), inexact)) ++e;
    if (e < mpfr_get_emin() || e > mpfr_get_emax()) { to_general<N>(out, x); return; }
    if (inexact) mpfr_set_inexflag();
    char* s = static_cast<char*>(mpfr_custom_get_significand(out));
    if (D >= std::size_t(N)) {
        std::memset(s, 0, 4 * (D - N));
        std::memcpy(s + 4 * (D - N), q, 4 * N);
    } else {
        std::memcpy(s, q + (N - D), 4 * D);        // the words below are zero after rounding to p <= 32 D bits
    }
    mpfr_custom_init_set(out, x.sign < 0 ? -MPFR_REGULAR_KIND : MPFR_REGULAR_KIND, e, p, s);
}

// f(begin, end) over contiguous chunks of [0, n) on up to `threads` host threads (0: one per `grain` values, at most
// the core count).  MPFR's exponent range is per thread, so workers take the caller's; after every chunk has run, the
// exception of the lowest failing chunk is rethrown.
template <class F> inline void chunks(std::size_t n, unsigned threads, std::size_t grain, F&& f) {
    if (!n) return;
    const Range range = Range::current();
    if (!threads) {
        const std::size_t want = std::max<std::size_t>(1, n / std::max<std::size_t>(1, grain));
        threads = unsigned(std::min<std::size_t>(want, std::max(1u, std::thread::hardware_concurrency())));
    }
    threads = unsigned(std::min<std::size_t>(threads, n));
    if (threads <= 1) { f(std::size_t(0), n); return; }
    const std::size_t step = (n + threads - 1) / threads;
    std::vector<std::exception_ptr> errors(threads);
    std::vector<std::thread> pool;
    for (unsigned t = 1; t < threads; ++t) {
        const std::size_t b = t * step, e = std::min(n, b + step);
        if (b >= e) break;
        auto body = [&f, &errors, range, t, b, e] {
            try { range.adopt(); f(b, e); } catch (...) { errors[t] = std::current_exception(); }
            mpfr_free_cache2(MPFR_FREE_LOCAL_CACHE);
        };
        try { pool.emplace_back(body); }
        catch (const std::system_error&) { try { f(b, e); } catch (...) { errors[t] = std::current_exception(); } }
    }
    try { f(std::size_t(0), std::min(n, step)); } catch (...) { errors[0] = std::current_exception(); }
    for (auto& w : pool) w.join();
    for (auto& err : errors) if (err) std::rethrow_exception(err);
}
template <int Bits> constexpr std::size_t real_grain() { return (std::size_t(1) << 22) / Bits; }
template <int Bits> constexpr std::size_t complex_grain() { return (std::size_t(1) << 21) / Bits; }

template <int Bits = 64, class F> inline void for_width(int bits, F&& f) {
    if (bits == Bits) { f(std::integral_constant<int, Bits>{}); return; }
    if constexpr (Bits < 1024) for_width<Bits + 32>(bits, f);
}
template <class T> inline void put(void* p, const T& v) { std::memcpy(p, &v, sizeof(T)); }
template <class T> inline T take(const void* p) { T v; std::memcpy(&v, p, sizeof(T)); return v; }
inline void need(bool ok, const char* what) { if (!ok) throw std::invalid_argument(what); }
}  // namespace bridge_detail

// ---- typed forms
template <int Bits> inline Float<Bits> from_mpfr(mpfr_srcptr input) { return bridge_detail::from<Bits / 32>(input); }
template <int Bits> inline void to_mpfr(mpfr_ptr out, const Float<Bits>& x) { bridge_detail::to<Bits / 32>(out, x); }
template <int Bits> inline void from_mpfr_array(const mpfr_t* in, Float<Bits>* out, std::size_t n, unsigned threads = 0) {
    bridge_detail::chunks(n, threads, bridge_detail::real_grain<Bits>(), [&](std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e; ++i) out[i] = bridge_detail::from<Bits / 32>(in[i]);
    });
}
// Element by element as to_mpfr; on a status, elements of other chunks may already be written.
template <int Bits> inline void to_mpfr_array(mpfr_t* out, const Float<Bits>* in, std::size_t n, unsigned threads = 0) {
    bridge_detail::chunks(n, threads, bridge_detail::real_grain<Bits>(), [&](std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e; ++i) bridge_detail::to<Bits / 32>(out[i], in[i]);
    });
}
template <int Bits> inline Float<Bits> from_decimal(const std::string& text) {
    mpfr_t x;
    mpfr_init2(x, Bits);
    if (mpfr_set_str(x, text.c_str(), 10, MPFR_RNDN)) { mpfr_clear(x); throw std::invalid_argument("invalid decimal number"); }
    const Float<Bits> r = from_mpfr<Bits>(x);
    mpfr_clear(x);
    return r;
}

#ifdef LIMBFORGE_HAS_MPC
template <int Bits> inline Complex<Bits / 32> from_mpc(mpc_srcptr z) {
    return {bridge_detail::from<Bits / 32>(mpc_realref(z)), bridge_detail::from<Bits / 32>(mpc_imagref(z))};
}
// Each part as to_mpfr; throws before writing either part when one has a status.
template <int Bits> inline void to_mpc(mpc_ptr out, const Complex<Bits / 32>& x) {
    if (x.re.status | x.im.status) bridge_detail::status_error(x.re.status | x.im.status);
    bridge_detail::to<Bits / 32>(mpc_realref(out), x.re);
    bridge_detail::to<Bits / 32>(mpc_imagref(out), x.im);
}
template <int Bits> inline void from_mpc_array(const mpc_t* in, Complex<Bits / 32>* out, std::size_t n, unsigned threads = 0) {
    bridge_detail::chunks(n, threads, bridge_detail::complex_grain<Bits>(), [&](std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e; ++i) out[i] = from_mpc<Bits>(in[i]);
    });
}
template <int Bits> inline void to_mpc_array(mpc_t* out, const Complex<Bits / 32>* in, std::size_t n, unsigned threads = 0) {
    bridge_detail::chunks(n, threads, bridge_detail::complex_grain<Bits>(), [&](std::size_t b, std::size_t e) {
        for (std::size_t i = b; i < e; ++i) to_mpc<Bits>(out[i], in[i]);
    });
}
#endif

// ---- runtime width: byte storage holding the same Float<bits> / Complex<bits/32> structs, no alignment required
inline std::size_t bridge_element_bytes(int bits, bool complex = false) {
    if (bits < 64 || bits > 1024 || bits % 32) throw std::invalid_argument("bridge bits must be a multiple of 32 in [64,1024]");
    return std::size_t(bits / 8 + 12) * (complex ? 2 : 1);
}
inline void from_mpfr(int bits, mpfr_srcptr input, void* out) {
    bridge_element_bytes(bits);
    bridge_detail::need(input && out, "null bridge operand");
    bridge_detail::for_width(bits, [&](auto b) { bridge_detail::put(out, from_mpfr<b.value>(input)); });
}
inline void to_mpfr(int bits, mpfr_ptr out, const void* input) {
    bridge_element_bytes(bits);
    bridge_detail::need(input && out, "null bridge operand");
    bridge_detail::for_width(bits, [&](auto b) { to_mpfr<b.value>(out, bridge_detail::take<Float<b.value>>(input)); });
}
inline void from_mpfr_array(int bits, const mpfr_t* input, void* out, std::size_t count, unsigned threads = 0) {
    const std::size_t bytes = bridge_element_bytes(bits);
    bridge_detail::need(!count || (input && out), "null bridge array");
    bridge_detail::need(count <= std::size_t(-1) / bytes, "bridge array size overflow");
    bridge_detail::for_width(bits, [&](auto b) {
        bridge_detail::chunks(count, threads, bridge_detail::real_grain<b.value>(), [&](std::size_t lo, std::size_t hi) {
            for (std::size_t i = lo; i < hi; ++i)
                bridge_detail::put(static_cast<char*>(out) + i * bytes, bridge_detail::from<b.value / 32>(input[i]));
        });
    });
}
inline void to_mpfr_array(int bits, mpfr_t* out, const void* input, std::size_t count, unsigned threads = 0) {
    const std::size_t bytes = bridge_element_bytes(bits);
    bridge_detail::need(!count || (input && out), "null bridge array");
    bridge_detail::need(count <= std::size_t(-1) / bytes, "bridge array size overflow");
    bridge_detail::for_width(bits, [&](auto b) {
        bridge_detail::chunks(count, threads, bridge_detail::real_grain<b.value>(), [&](std::size_t lo, std::size_t hi) {
            for (std::size_t i = lo; i < hi; ++i)
                bridge_detail::to<b.value / 32>(out[i], bridge_detail::take<Float<b.value>>(static_cast<const char*>(input) + i * bytes));
        });
    });
}
#ifdef LIMBFORGE_HAS_MPC
inline void from_mpc(int bits, mpc_srcptr input, void* out) {
    bridge_element_bytes(bits, true);
    bridge_detail::need(input && out, "null bridge operand");
    bridge_detail::for_width(bits, [&](auto b) { bridge_detail::put(out, from_mpc<b.value>(input)); });
}
inline void to_mpc(int bits, mpc_ptr out, const void* input) {
    bridge_element_bytes(bits, true);
    bridge_detail::need(input && out, "null bridge operand");
    bridge_detail::for_width(bits, [&](auto b) { to_mpc<b.value>(out, bridge_detail::take<Complex<b.value / 32>>(input)); });
}
inline void from_mpc_array(int bits, const mpc_t* input, void* out, std::size_t count, unsigned threads = 0) {
    const std::size_t bytes = bridge_element_bytes(bits, true);
    bridge_detail::need(!count || (input && out), "null bridge array");
    bridge_detail::need(count <= std::size_t(-1) / bytes, "bridge array size overflow");
    bridge_detail::for_width(bits, [&](auto b) {
        bridge_detail::chunks(count, threads, bridge_detail::complex_grain<b.value>(), [&](std::size_t lo, std::size_t hi) {
            for (std::size_t i = lo; i < hi; ++i) bridge_detail::put(static_cast<char*>(out) + i * bytes, from_mpc<b.value>(input[i]));
        });
    });
}
inline void to_mpc_array(int bits, mpc_t* out, const void* input, std::size_t count, unsigned threads = 0) {
    const std::size_t bytes = bridge_element_bytes(bits, true);
    bridge_detail::need(!count || (input && out), "null bridge array");
    bridge_detail::need(count <= std::size_t(-1) / bytes, "bridge array size overflow");
    bridge_detail::for_width(bits, [&](auto b) {
        bridge_detail::chunks(count, threads, bridge_detail::complex_grain<b.value>(), [&](std::size_t lo, std::size_t hi) {
            for (std::size_t i = lo; i < hi; ++i)
                to_mpc<b.value>(out[i], bridge_detail::take<Complex<b.value / 32>>(static_cast<const char*>(input) + i * bytes));
        });
    });
}
#endif

// ---- engine buffers: conversion into a buffer's pinned host mirror, which the next submission that uses the buffer
// uploads (one host pass, no staging copy); and out of a buffer through one download.
template <class T> inline void from_mpfr_buffer(const mpfr_t* in, Buffer<T>& out, std::size_t n, unsigned threads = 0) {
    static_assert(!detail::Format<T>::complex && detail::Format<T>::bits != 0, "real arithmetic buffer required");
    bridge_detail::need(n <= out.size(), "bridge array exceeds the buffer");
    from_mpfr_array<detail::Format<T>::bits>(in, out.mapped(), n, threads);
}
template <class T> inline void to_mpfr_buffer(mpfr_t* out, const Buffer<T>& in, std::size_t n, unsigned threads = 0) {
    static_assert(!detail::Format<T>::complex && detail::Format<T>::bits != 0, "real arithmetic buffer required");
    bridge_detail::need(n <= in.size(), "bridge array exceeds the buffer");
    std::vector<T> host(n);
    in.download(host.data(), n);
    to_mpfr_array<detail::Format<T>::bits>(out, host.data(), n, threads);
}
}  // namespace limbforge
