// The bridge's engine-buffer forms and the inline MPC import on the GPU (include/limbforge/mpfr_bridge.hpp,
// mpc_staging.hpp, BatchedLinalg::import_inline_complex): MPFR values go into a buffer's pinned mirror, a batch adds
// each value to itself, and the results come back through to_mpfr_buffer equal to MPFR's own doubling (exact); mpc_t
// values whose significands sit in one page-aligned allocation are imported on the GPU and read back equal to
// from_mpc.  Prints "bridge gpu ok".
#include "limbforge/batched_linalg.hpp"
#include "limbforge/mpc_staging.hpp"
#include <cstdio>
#include <cstdlib>
#include <memory>
#include <random>
#include <vector>

using namespace limbforge;
#define CHECK(c, what) do { if (!(c)) { std::printf("FAILED: %s (line %d)\n", what, __LINE__); return 1; } } while (0)

int main() {
    try {
        constexpr int B = 448;
        const std::size_t n = 3000;
        Engine e;
        std::mt19937_64 rng(5);
        std::unique_ptr<mpfr_t[]> in(new mpfr_t[n]), out(new mpfr_t[n]);
        for (std::size_t i = 0; i < n; ++i) {
            mpfr_init2(in[i], B); mpfr_init2(out[i], B);
            Float<B> x = zero<B / 32>();
            for (int k = 0; k < B / 32; ++k) x.limb[k] = word(rng());
            x.limb[B / 32 - 1] |= 0x80000000u; x.exponent = int(rng() % 801) - 400; x.sign = (rng() & 1) ? 1 : -1;
            to_mpfr<B>(in[i], i % 41 == 3 ? zero<B / 32>() : x);
        }
        auto buf = e.make_buffer<Float<B>>(n), dbl = e.make_buffer<Float<B>>(n);
        from_mpfr_buffer(in.get(), buf, n, 4);
        auto batch = e.batch();
        batch.run(Operation::add, buf, buf, dbl);
        batch.submit().wait();
        to_mpfr_buffer(out.get(), dbl, n, 4);
        for (std::size_t i = 0; i < n; ++i) {
            mpfr_t want; mpfr_init2(want, B);
            mpfr_mul_2si(want, in[i], 1, MPFR_RNDN);
            CHECK(mpfr_equal_p(out[i], want) || (mpfr_zero_p(out[i]) && mpfr_zero_p(want)), "buffer round trip through a GPU add");
            mpfr_clear(want);
        }
        for (std::size_t i = 0; i < n; ++i) { mpfr_clear(in[i]); mpfr_clear(out[i]); }

        // inline MPC import: 64 values, significands scattered over two pages
        constexpr int C = 256;
        const std::size_t m = 64, page = 4096, bytes = 4 * page;
        void* mem = std::aligned_alloc(page, bytes);
        std::unique_ptr<mpc_t[]> z(new mpc_t[m]);
        std::vector<mpc_srcptr> ptrs(m);
        for (std::size_t i = 0; i < m; ++i) {
            for (int part = 0; part < 2; ++part) {
                mpfr_ptr f = part ? mpc_imagref(z[i]) : mpc_realref(z[i]);
                void* at = static_cast<char*>(mem) + page + part * m * 32 + ((i * 7) % m) * 32;   // scattered, disjoint
                mpfr_custom_init(at, C);
                mpfr_custom_init_set(f, MPFR_ZERO_KIND, 0, C, at);
            }
            Float<C> re = zero<C / 32>(), im = zero<C / 32>();
            for (int k = 0; k < C / 32; ++k) { re.limb[k] = word(rng()); im.limb[k] = word(rng()); }
            re.limb[C / 32 - 1] |= 0x80000000u; im.limb[C / 32 - 1] |= 0x80000000u;
            re.exponent = int(i) - 30; im.exponent = -int(i); re.sign = 1; im.sign = (i & 1) ? -1 : 1;
            to_mpc<C>(z[i], Complex<C / 32>{re, i % 9 == 4 ? zero<C / 32>() : im});
            ptrs[i] = z[i];
        }
        const auto records = describe_inline_mpc(C, mem, bytes, ptrs.data(), m);
        BatchedLinalg bl(e);
        auto cz = e.make_buffer<Complex<C / 32>>(m);
        auto b2 = e.batch();
        bl.import_inline_complex(b2, mem, bytes, records.data(), m, cz);
        b2.submit().wait();
        std::vector<Complex<C / 32>> got(m);
        cz.download(got.data(), m);
        for (std::size_t i = 0; i < m; ++i) {
            const Complex<C / 32> want = from_mpc<C>(z[i]);
            CHECK(!std::memcmp(&got[i], &want, sizeof want), "inline import");
        }
        std::free(mem);
        std::printf("bridge gpu ok\n");
        return 0;
    } catch (const std::exception& ex) {
        std::printf("exception: %s\n", ex.what());
        return 1;
    }
}
