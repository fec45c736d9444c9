// Host-side scalar arithmetic of include/limbforge/core.hpp and linalg.hpp (exact_dot_add), built with the host
// compiler alone: reads operand arrays from a file, applies every scalar operation at one width, and writes
// the results, which tests/test_host_arith.py compares with the oracle bit for bit.
//   host_arith <bits> <in> <out>   in: count, then a, b, c, d, e (count elements each, N + 3 words); out: results
#include "limbforge/linalg.hpp"
#include <cstdio>
#include <cstdlib>
#include <vector>

using namespace limbforge;

template <int N> int run(const char* in_path, const char* out_path) {
    std::FILE* in = std::fopen(in_path, "rb");
    if (!in) return 2;
    std::uint64_t count = 0;
    if (std::fread(&count, 8, 1, in) != 1) return 2;
    std::vector<Number<N>> v[5];
    for (auto& x : v) {
        x.resize(count);
        if (std::fread(x.data(), sizeof(Number<N>), count, in) != count) return 2;
    }
    std::fclose(in);
    const auto &a = v[0], &b = v[1], &c = v[2], &d = v[3], &e = v[4];
    std::vector<Number<N>> out;
    for (std::uint64_t i = 0; i < count; ++i) {
        out.push_back(add(a[i], b[i]));
        out.push_back(sub(a[i], b[i]));
        out.push_back(mul(a[i], b[i]));
        out.push_back(div(a[i], b[i]));
        out.push_back(square(a[i]));
        Number<N> r = a[i]; r.sign = r.sign < 0 ? -r.sign : r.sign;
        out.push_back(limbforge::sqrt(r));
        out.push_back(fma(a[i], b[i], c[i]));
        out.push_back(fms(a[i], b[i], c[i]));
        out.push_back(dot2_add(a[i], b[i], c[i], d[i], e[i]));
        const Complex<N> x{a[i], b[i]}, y{c[i], d[i]}, z{e[i], a[i]};
        for (const Complex<N>& w : {cadd(x, y), cmul(x, y), cdiv(x, y), cfma(x, y, z), cfms(x, y, z)}) { out.push_back(w.re); out.push_back(w.im); }
    }
    // exact dots: RN(c_0 - sum_k a_k b_k) over the whole arrays, and RN(sum_k a_k d_k)
    out.push_back(exact_dot_add(c[0], true, a.data(), 1, b.data(), 1, count));
    out.push_back(exact_dot(a.data(), 1, d.data(), 1, count));
    std::FILE* o = std::fopen(out_path, "wb");
    if (!o) return 2;
    std::fwrite(out.data(), sizeof(Number<N>), out.size(), o);
    std::fclose(o);
    return 0;
}

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    switch (std::atoi(argv[1])) {
    case 64: return run<2>(argv[2], argv[3]);
    case 256: return run<8>(argv[2], argv[3]);
    case 416: return run<13>(argv[2], argv[3]);
    case 1024: return run<32>(argv[2], argv[3]);
    default: return 2;
    }
}
