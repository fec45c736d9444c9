// The MPFR/MPC bridge (include/limbforge/mpfr_bridge.hpp) against MPFR's own rounding and the element format.
//   bridge check <in.bin> <count> <out.bin>   in: count 1024-bit elements; out, per element and per width W of
//        64, 96, 256, 736, 1024: from_mpfr<W> of the exact MPFR value, then to_mpfr at precision W read back at 1024 bits
//   bridge self                                 internal checks; prints "bridge ok"
//   bridge time <count> <samples>               ns per value, as the reference's benchmarks/bridge.cpp reports
#include "limbforge/mpfr_bridge.hpp"
#include "limbforge/mpc_staging.hpp"
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <memory>
#include <random>
#include <iostream>

using namespace limbforge;

#define CHECK(c, what) do { if (!(c)) { std::printf("FAILED: %s (line %d)\n", what, __LINE__); std::exit(1); } } while (0)

struct MP {   // an array of initialised mpfr_t
    std::unique_ptr<mpfr_t[]> a; std::size_t n;
    MP(std::size_t n, mpfr_prec_t p) : a(new mpfr_t[n]), n(n) { for (std::size_t i = 0; i < n; ++i) mpfr_init2(a[i], p); }
    ~MP() { for (std::size_t i = 0; i < n; ++i) mpfr_clear(a[i]); }
};
template <int N> static bool same(const Number<N>& x, const Number<N>& y) { return !std::memcmp(&x, &y, sizeof x); }

// Exact value of x by integer import (independent of the fast path): x at 32N bits of precision.
template <int N> static void exact(mpfr_ptr out, const Number<N>& x) { bridge_detail::to_general<N>(out, x); }

static int check(const char* in_path, std::size_t count, const char* out_path) {
    constexpr int N = 32;
    std::vector<Number<N>> x(count);
    std::ifstream(in_path, std::ios::binary).read(reinterpret_cast<char*>(x.data()), count * sizeof(Number<N>));
    std::ofstream out(out_path, std::ios::binary);
    mpfr_t v, w;
    mpfr_init2(v, 1024);
    for (std::size_t i = 0; i < count; ++i) {
        exact<N>(v, x[i]);
        auto emit = [&](auto b) {
            constexpr int W = decltype(b)::value;
            const Float<W> f = from_mpfr<W>(v);
            out.write(reinterpret_cast<const char*>(&f), sizeof f);
            mpfr_init2(w, W);
            to_mpfr<1024>(w, x[i]);
            const Float<1024> g = from_mpfr<1024>(w);
            out.write(reinterpret_cast<const char*>(&g), sizeof g);
            mpfr_clear(w);
        };
        emit(std::integral_constant<int, 64>{}); emit(std::integral_constant<int, 96>{}); emit(std::integral_constant<int, 256>{});
        emit(std::integral_constant<int, 736>{}); emit(std::integral_constant<int, 1024>{});
        // precisions that are not whole words: the fast path against MPFR rounding the exact value
        for (mpfr_prec_t p : {1, 2, 33, 100, 333, 1000, 1100}) {
            mpfr_t a, r;
            mpfr_init2(a, p); mpfr_init2(r, p);
            to_mpfr<1024>(a, x[i]);
            mpfr_set(r, v, MPFR_RNDN);
            CHECK(mpfr_equal_p(a, r) || (mpfr_zero_p(a) && mpfr_zero_p(r)), "to_mpfr rounding vs mpfr_set");
            mpfr_clear(a); mpfr_clear(r);
        }
    }
    mpfr_clear(v);
    return 0;
}

template <int Bits> static Float<Bits> pow2(long e, int sign = 1) {
    Float<Bits> r = zero<Bits / 32>(); r.limb[Bits / 32 - 1] = 0x80000000u; r.exponent = int(e); r.sign = sign; return r;
}

static int self_checks() {
    mpfr_t x; mpfr_init2(x, 2000);
    // specials
    mpfr_set_nan(x); CHECK(from_mpfr<256>(x).status == invalid && from_mpfr<256>(x).sign == 0, "NaN");
    mpfr_set_inf(x, -1); CHECK(from_mpfr<256>(x).status == invalid, "Inf");
    mpfr_set_zero(x, -1); CHECK(same(from_mpfr<256>(x), zero<8>()), "zero");
    mpfr_set_si(x, 1, MPFR_RNDN); mpfr_mul_2si(x, x, 1000000000L, MPFR_RNDN);
    CHECK(same(from_mpfr<64>(x), pow2<64>(1000000000L)), "exponent limit");
    mpfr_mul_2si(x, x, 1, MPFR_RNDN); CHECK(from_mpfr<64>(x).status == exponent_overflow, "exponent overflow");
    mpfr_set_si(x, -1, MPFR_RNDN); mpfr_mul_2si(x, x, -1000000001L, MPFR_RNDN);
    CHECK(from_mpfr<64>(x).status == exponent_overflow, "exponent underflow");
    // rounding carries into the next binade: (1 - 2^-1500) 2^7 -> 2^7 at every width, inexact
    mpfr_set_si(x, 1, MPFR_RNDN); mpfr_mul_2si(x, x, -1500, MPFR_RNDN);
    { mpfr_t one; mpfr_init2(one, 2000); mpfr_set_si(one, 1, MPFR_RNDN); mpfr_t d; mpfr_init2(d, 2000);
      mpfr_sub(d, one, x, MPFR_RNDN); mpfr_mul_2si(d, d, 7, MPFR_RNDN);
      mpfr_clear_inexflag(); CHECK(same(from_mpfr<64>(d), pow2<64>(6 + 1)), "carry"); CHECK(mpfr_inexflag_p(), "inexact flag");
      mpfr_clear(one); mpfr_clear(d); }
    // exact conversions leave the inexact flag clear
    mpfr_set_si(x, -3, MPFR_RNDN); mpfr_clear_inexflag();
    const Float<128> m3 = from_mpfr<128>(x);
    CHECK(!mpfr_inexflag_p() && m3.sign == -1 && m3.exponent == 1 && m3.limb[3] == 0xC0000000u, "exact small integer");
    // to_mpfr: status throws, zero, exact at wider precision, ties to even at narrower
    bool threw = false;
    try { to_mpfr<64>(x, zero<2>(division_by_zero)); } catch (const std::runtime_error& e) { threw = std::string(e.what()).find("status 1") != std::string::npos; }
    CHECK(threw, "status throws");
    to_mpfr<64>(x, zero<2>()); CHECK(mpfr_zero_p(x) && !mpfr_signbit(x), "to_mpfr zero");
    Float<64> t = pow2<64>(0); t.limb[0] = 0x80000000u;        // 1 + 2^-32 ... then 3 significant bits: ties
    { mpfr_t s; mpfr_init2(s, 33); mpfr_clear_inexflag(); to_mpfr<64>(s, t); CHECK(!mpfr_inexflag_p(), "33-bit exact flag");
      Float<64> back = from_mpfr<64>(s); CHECK(same(back, t), "33-bit exact"); mpfr_clear(s); }
    { mpfr_t s; mpfr_init2(s, 32); mpfr_clear_inexflag(); to_mpfr<64>(s, t);
      CHECK(mpfr_inexflag_p() && same(from_mpfr<64>(s), pow2<64>(0)), "tie to even (down)"); mpfr_clear(s); }
    t.limb[1] |= 1u;                                             // odd last kept bit: the tie goes up
    { mpfr_t s; mpfr_init2(s, 32); to_mpfr<64>(s, t); Float<64> up = pow2<64>(0); up.limb[1] |= 2u;
      CHECK(same(from_mpfr<64>(s), up), "tie to even (up)"); mpfr_clear(s); }
    // results outside MPFR's exponent range follow MPFR's overflow rule
    { const mpfr_exp_t emax = mpfr_get_emax(); mpfr_set_emax(100); mpfr_t s; mpfr_init2(s, 64);
      to_mpfr<64>(s, pow2<64>(200)); CHECK(mpfr_inf_p(s), "overflow to infinity"); mpfr_set_emax(emax); mpfr_clear(s); }
    // arrays, threads, runtime width, errors
    const std::size_t n = 5000;
    MP a(n, 300), b(n, 448);
    std::mt19937_64 rng(7);
    std::vector<Float<448>> v(n), w(n), u(n);
    for (std::size_t i = 0; i < n; ++i) {
        Float<448> r = zero<14>(); for (int k = 0; k < 14; ++k) r.limb[k] = word(rng());
        r.limb[13] |= 0x80000000u; r.exponent = int(rng() % 4001) - 2000; r.sign = (rng() & 1) ? 1 : -1;
        v[i] = (i % 97 == 5) ? zero<14>() : r;
    }
    to_mpfr_array<448>(b.a.get(), v.data(), n, 3);
    from_mpfr_array<448>(b.a.get(), w.data(), n, 0);
    for (std::size_t i = 0; i < n; ++i) CHECK(same(w[i], v[i]), "array round trip");
    to_mpfr_array<448>(a.a.get(), v.data(), n, 1);               // rounds to 300 bits
    from_mpfr_array(448, a.a.get(), u.data(), n, 4);
    for (std::size_t i = 0; i < n; ++i) { Float<448> s; from_mpfr(448, a.a[i], &s); CHECK(same(s, u[i]), "runtime width"); }
    std::vector<Float<448>> bad = v; bad[4321].status = invalid;
    threw = false;
    try { to_mpfr_array<448>(b.a.get(), bad.data(), n, 4); } catch (const std::runtime_error&) { threw = true; }
    CHECK(threw, "array status throws");
    threw = false;
    try { bridge_element_bytes(48); } catch (const std::invalid_argument&) { threw = true; }
    CHECK(threw && bridge_element_bytes(448, true) == 2 * (56 + 12), "element bytes");
    // decimal
    const Float<256> tenth = from_decimal<256>("0.1");
    CHECK(same(tenth, div(pow2<256>(0), from_decimal<256>("10"))), "from_decimal vs division");
    threw = false;
    try { from_decimal<256>("zz"); } catch (const std::invalid_argument&) { threw = true; }
    CHECK(threw, "bad decimal");
#ifdef LIMBFORGE_HAS_MPC
    {
        mpc_t z; mpfr_init2(mpc_realref(z), 256); mpfr_init2(mpc_imagref(z), 256);
        Complex<8> c{from_decimal<256>("0.1"), from_decimal<256>("-3")};
        to_mpc<256>(z, c);
        const Complex<8> back = from_mpc<256>(z);
        CHECK(same(back.re, c.re) && same(back.im, c.im), "mpc round trip");
        Complex<8> st{c.re, zero<8>(invalid)};
        threw = false;
        try { to_mpc<256>(z, st); } catch (const std::runtime_error&) { threw = true; }
        CHECK(threw && same(from_mpc<256>(z).re, c.re), "mpc status throws before writing");
        std::vector<Complex<8>> cs(100, c), cb(100);
        std::unique_ptr<mpc_t[]> zs(new mpc_t[100]);
        for (auto i = 0; i < 100; ++i) { mpfr_init2(mpc_realref(zs[i]), 256); mpfr_init2(mpc_imagref(zs[i]), 256); }
        to_mpc_array(256, zs.get(), cs.data(), 100, 2);
        from_mpc_array<256>(zs.get(), cb.data(), 100, 3);
        for (auto& q : cb) CHECK(same(q.re, c.re) && same(q.im, c.im), "mpc arrays");
        for (auto i = 0; i < 100; ++i) { mpfr_clear(mpc_realref(zs[i])); mpfr_clear(mpc_imagref(zs[i])); }
        mpfr_clear(mpc_realref(z)); mpfr_clear(mpc_imagref(z));
    }
    {   // describe_inline_mpc: records of values whose significands sit in one page-aligned allocation
        const std::size_t page = 4096, bytes = 2 * page;
        void* mem = std::aligned_alloc(page, bytes);
        std::memset(mem, 0, bytes);
        mpc_t v[3];
        const mpc_srcptr ptrs[3] = {v[0], v[1], v[2]};
        char* at = static_cast<char*>(mem) + 64;
        for (auto& q : v)
            for (mpfr_ptr part : {mpc_realref(q), mpc_imagref(q)}) {
                mpfr_custom_init(at, 96);
                mpfr_custom_init_set(part, MPFR_ZERO_KIND, 0, 96, at);
                at += 16;
            }
        to_mpc<96>(v[0], Complex<3>{from_decimal<96>("1.5"), from_decimal<96>("-0.1")});
        mpfr_set_nan(mpc_realref(v[1]));
        to_mpc<96>(v[2], Complex<3>{pow2<96>(1000000000L), pow2<96>(-5, -1)});
        mpfr_mul_2si(mpc_realref(v[2]), mpc_realref(v[2]), 1, MPFR_RNDN);
        const auto rec = describe_inline_mpc(96, mem, bytes, ptrs, 3);
        CHECK(rec[0].real_offset == 64 && rec[0].real_exponent == 0 && rec[0].real_sign == 1 && rec[0].imag_offset == 80 &&
              rec[0].imag_sign == -1 && rec[0].imag_exponent == -4, "inline records");
        CHECK(rec[1].real_status == invalid && rec[1].imag_sign == 0 && rec[1].imag_status == 0, "inline specials");
        CHECK(rec[2].real_status == exponent_overflow && rec[2].imag_exponent == -5 && rec[2].imag_sign == -1, "inline exponent range");
        threw = false;
        try { describe_inline_mpc(128, mem, bytes, ptrs, 3); } catch (const std::invalid_argument&) { threw = true; }
        CHECK(threw, "inline precision must match");
        threw = false;
        try { describe_inline_mpc(96, static_cast<char*>(mem) + page, page, ptrs, 3); } catch (const std::invalid_argument&) { threw = true; }
        CHECK(threw, "inline significand outside allocation");
        std::free(mem);
    }
#endif
    mpfr_clear(x);
    std::printf("bridge ok\n");
    return 0;
}

// ns per value, median of `samples`, scalar and array forms, one thread and all threads; the mpz route
// (to_general / from_general) timed beside as the reference's benchmark times its mpz route.
template <int Bits> static void timing(std::size_t count, int samples) {
    constexpr int N = Bits / 32;
    using Clock = std::chrono::steady_clock;
    auto ns = [&](auto&& run) {
        run();
        std::vector<double> t;
        for (int s = 0; s < samples; ++s) {
            const auto a = Clock::now(); run();
            t.push_back(std::chrono::duration<double, std::nano>(Clock::now() - a).count() / double(count));
        }
        std::sort(t.begin(), t.end());
        return t[t.size() / 2];
    };
    std::mt19937_64 rng(Bits);
    std::vector<Float<Bits>> v(count), w(count);
    for (auto& r : v) {
        r = zero<N>(); for (int k = 0; k < N; ++k) r.limb[k] = word(rng());
        r.limb[N - 1] |= 0x80000000u; r.exponent = int(rng() % 2001) - 1000; r.sign = (rng() & 1) ? 1 : -1;
    }
    for (mpfr_prec_t prec : {mpfr_prec_t(Bits), mpfr_prec_t(Bits + 64), mpfr_prec_t(Bits - 32)}) {
        MP m(count, prec);
        const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
        const double to_gen = ns([&] { for (std::size_t i = 0; i < count; ++i) bridge_detail::to_general<N>(m.a[i], v[i]); });
        const double from_gen = ns([&] { for (std::size_t i = 0; i < count; ++i) w[i] = bridge_detail::from_general<N>(m.a[i]); });
        const double to1 = ns([&] { to_mpfr_array<Bits>(m.a.get(), v.data(), count, 1); });
        const double toN = ns([&] { to_mpfr_array<Bits>(m.a.get(), v.data(), count, 0); });
        const double from1 = ns([&] { from_mpfr_array<Bits>(m.a.get(), w.data(), count, 1); });
        const double fromN = ns([&] { from_mpfr_array<Bits>(m.a.get(), w.data(), count, 0); });
        std::printf("{\"bits\": %d, \"mpfr_prec\": %ld, \"count\": %zu, \"threads\": %u, \"to_mpz_ns\": %.2f, \"to_ns\": %.2f, "
                    "\"to_threads_ns\": %.2f, \"from_mpz_ns\": %.2f, \"from_ns\": %.2f, \"from_threads_ns\": %.2f}\n",
                    Bits, long(prec), count, hw, to_gen, to1, toN, from_gen, from1, fromN);
    }
}

int main(int argc, char** argv) {
    try {
        const std::string mode = argc > 1 ? argv[1] : "self";
        if (mode == "check" && argc == 5) return check(argv[2], std::strtoull(argv[3], nullptr, 10), argv[4]);
        if (mode == "self") return self_checks();
        if (mode == "time") {
            const std::size_t count = argc > 2 ? std::strtoull(argv[2], nullptr, 10) : 65536;
            const int samples = argc > 3 ? std::atoi(argv[3]) : 9;
            timing<224>(count, samples); timing<256>(count, samples); timing<384>(count, samples); timing<1024>(count, samples);
            return 0;
        }
        std::printf("usage: bridge self | check <in> <count> <out> | time [count] [samples]\n");
        return 2;
    } catch (const std::exception& e) {
        std::printf("exception: %s\n", e.what());
        return 1;
    }
}
