// Exact sums whose clusters are wider than the window (include/limbforge/detail/arith.hpp cluster_round's streaming
// path) against the same sums with a window wide enough for every cluster.  Terms are products a_k b_k of random
// numbers whose exponents form chains spaced below the cluster gap (so one cluster spans thousands of bits), with
// random signs, exact cancellations (a term and its negation), sparse significands (exact ties) and a few far terms.
// Prints "checked K, mismatches M"; exits 1 on a mismatch.
#include "limbforge/detail/arith.hpp"
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

using namespace lfd;

template <int N> struct Pairs {
    const std::vector<Num<N>>* a; const std::vector<Num<N>>* b;
    u64 count() const { return a->size(); }
    bool term(u64 k, i64& scale, i64& top, int& sign) const {
        const Num<N>& x = (*a)[k]; const Num<N>& y = (*b)[k];
        if (!x.s || !y.s) return false;
        scale = (i64)x.e + y.e - 2 * (32 * N - 1); top = scale + 64 * N; sign = x.s * y.s;
        return true;
    }
    void add(u64 k, u32* acc, int len, i64 off) const {
        u32 p[2 * N];
        mul_words<N, N>((*a)[k].m, (*b)[k].m, p);
        acc_add(acc, len, p, 2 * N, off);
    }
};

template <int N> Num<N> rnd(std::mt19937_64& g, int e, bool sparse) {
    Num<N> x{};
    for (int i = 0; i < N; ++i) x.m[i] = sparse ? 0u : (u32)g();
    x.m[N - 1] |= 0x80000000u;
    if (sparse) for (int t = 0; t < 3; ++t) { const int b = (int)(g() % (32 * N)); x.m[b / 32] |= 1u << (b % 32); }
    x.e = e; x.s = (g() & 1) ? 1 : -1; x.st = 0;
    return x;
}

template <int N> int run(std::mt19937_64& g, int cases) {
    constexpr int SMALL = 8 * N + 4, BIG = 2048;
    int bad = 0;
    for (int c = 0; c < cases; ++c) {
        const int K = 2 + (int)(g() % 60);
        std::vector<Num<N>> a(K), b(K);
        const int spacing = 1 + (int)(g() % (32 * N + 6));       // below the gap: the terms chain into one cluster
        int e = 0;
        const bool sparse = g() % 3 == 0;
        for (int k = 0; k < K; ++k) {
            a[k] = rnd<N>(g, e, sparse); b[k] = rnd<N>(g, 0, sparse);
            if (g() % 7 == 0) e -= 5000 + (int)(g() % 3000);       // a far term: a new cluster
            else e -= spacing / 2 + (int)(g() % (spacing / 2 + 1));
        }
        if (K > 3 && g() % 4 == 0) { a[K / 2] = a[0]; b[K / 2] = b[0]; a[K / 2].s = -a[0].s; }    // exact cancellation of the top
        if (K > 5 && g() % 5 == 0) { a[K - 1] = a[1]; b[K - 1] = b[1]; a[K - 1].s = -a[1].s; }
        for (int k = 0; k < K; ++k) if (g() % 29 == 0) a[k].s = 0, std::memset(a[k].m, 0, sizeof a[k].m), a[k].e = 0;
        const Pairs<N> src{&a, &b};
        u32 e1 = 0, e2 = 0;
        const Num<N> x = cluster_round<N, SMALL>(src, &e1), y = cluster_round<N, BIG>(src, &e2);
        const bool same = x.s == y.s && x.st == y.st && (!x.s || (x.e == y.e && !std::memcmp(x.m, y.m, sizeof x.m)));
        if (!same || e1 || e2) ++bad;
    }
    return bad;
}

int main() {
    std::mt19937_64 g(20261204);
    int bad = 0, total = 0;
    bad += run<2>(g, 3000); total += 3000;
    bad += run<4>(g, 3000); total += 3000;
    bad += run<7>(g, 2000); total += 2000;
    bad += run<8>(g, 2000); total += 2000;
    bad += run<16>(g, 500); total += 500;
    bad += run<32>(g, 200); total += 200;
    std::printf("checked %d, mismatches %d\n", total, bad);
    return bad ? 1 : 0;
}
