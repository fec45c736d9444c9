// Householder QR panel kernels (the unpivoted sequence of the reference's src/linalg.mm:488-790; the
// column-by-column statement its tests/test_qr.cpp:33-68 checks gives the same bits).  P(x, y) = RN(sum x_k y_k)
// and D(c; x, y) = RN(c - sum x_k y_k) with one rounding each.
//
// A panel of kb columns starting at column k0 is copied column-contiguous (Pt: entry (c, r) at c * mr + r,
// mr = m - k0 rows), its reflectors are built in Vt with the same layout, and every column step runs as four
// launches with no host round trip: the rows of the column reduced by the panel's earlier reflectors (one warp
// per row), the reflector (one block: the squared norm, sqrt, the scaled reflector and tau), the panel W row and
// Gram column (one block per dot), then one block that writes the T column and the next column's y.  Failures (zero, small or status columns) are recorded in a device-side state that the following launches
// and the host read; the trailing matrix is updated by the compact-WY products on the exact GEMM engine.
#pragma once
#include "lf_linalg.cuh"

namespace lfd {

// Progress of one factorization, written by the panel kernels and read by the next launches and the host.
struct QrState {
    long long rank;      // n while every column so far gave a reflector; the first failing column otherwise
    int reason;          // 0 full rank, 1 zero column, 2 small column (rank test), 3 status column
    u32 status;          // the failing column's status
    long long top;       // the largest exponent of an r_jj so far (valid when have_top)
    int have_top;
    u32 arrivals;        // blocks of the current dots launch that have finished
    u32 recomputed;      // column pivoting: downdated squared norms recomputed from the reduced column
};

struct QrPanel {
    u32* Wk; u64 m, n;           // the work matrix (m x n), reduced in place
    u32* V; u32* T; u32* tau;    // the factor: V (m x n), T (blocks of nb x nb), tau (n)
    u32* Pt; u32* Vt;            // the panel's columns and reflectors, entry (c, r) at c * mr + r
    u32* Wp; u32* G; u32* y;     // the panel W rows (nb x nb: Wp[c][c'] = P(v_c, a_c')), Gram column, next y
    u64 k0, kb, nb, mr;
    int rank_bits;
    QrState* st;
    u32* error;                  // set when an exact sum exceeds the cluster window
    // column pivoting (pivot != 0): W and Y rows of the trailing columns (nb x n), squared column norms nu and their
    // last exact values nuref (n), the permutation (n) and the recomputation flags (n)
    int pivot;
    u32* Wr; u32* Yr; u32* nu; u32* nuref; u64* perm; u32* flag;
};

constexpr int kQrThreads = 256;
// Window words of the block-wide exact dot: the product width plus headroom for the spread of the products'
// exponents (about 800 bits up to 512-bit numbers, 320 bits beyond); wider spreads take the cluster method.
template <int N> __host__ __device__ constexpr int qr_window() { return 2 * N + 10 + (N <= 16 ? 16 : 4); }
// The block-wide sums reduce the threads' windows with two shuffle levels to kQrRows partial windows, which go to
// shared memory as rows of qr_row_words words (odd: conflict-free rows and columns) and are summed by columns.
constexpr int kQrRows = kQrThreads / 4;
template <int N> __host__ __device__ constexpr int qr_row_words() { return qr_window<N>() | 1; }
template <int N> __host__ __device__ constexpr int qr_dot_words() {
    return kQrRows * qr_row_words<N>() + 1 + 8 * qr_window<N>() + 6 * (kQrThreads / 32) + N + 8;
}

template <int N> __device__ __forceinline__ Num<N> qr_pow2(int e) {
    Num<N> x = zero<N>();
    x.m[N - 1] = 0x80000000u; x.s = 1; x.e = e;
    return x;
}
// x * 2^-e exactly; a result exponent outside [-1e9, 1e9] gives zero with exponent_overflow (linalg.mm:492).
template <int N> __device__ __forceinline__ Num<N> qr_scaled(Num<N> x, long long e) {
    if (!x.s) return x;
    const long long r = (long long)x.e - e;
    if (r > kEmax || r < -kEmax) return zero<N>(x.st | kOverflow);
    x.e = (int)r;
    return x;
}

// Operands of term k of a strided dot: x[k sx] and y[k sy].  fallback: the cluster method on one thread.
template <int N, bool RO> struct StridedPair {
    const u32* x; i64 sx; const u32* y; i64 sy; u64 K;
    __device__ void operands(u64 k, Num<N>& a, Num<N>& b) const {
        constexpr i64 E = N + 3;
        a = ldn<N, RO>(x + (i64)k * sx * E); b = ldn<N, RO>(y + (i64)k * sy * E);
    }
    __device__ Num<N> fallback(u32* error) const { return exact_dot_add_dev<N, RO>(nullptr, false, x, sx, y, sy, K, error); }
};

// RN(sum_{k<K} a_k b_k) with one rounding for the operands a_k, b_k that src gives, computed by the whole block
// (kQrThreads threads) and returned to every thread; the contract of exact_dot (statuses first; no nonzero product
// gives zero).  Pass 1 reduces the statuses, the number of nonzero products and the range of their scales; each
// thread then adds its products into a two's-complement window anchored at the lowest scale, the warps sum their
// windows with shuffles and thread 0 adds the warps' sums and rounds once.  A range wider than the window goes to
// src.fallback (the cluster method) on thread 0.  sm: qr_dot_words<N>() words of shared memory, 8-byte aligned.
// keep (optional, qr_keep_words<N>() words): thread 0 leaves there the exact window of the sum (valid flag, lo, hi,
// logc, the two's-complement words) so that it can add terms to the exact sum and round again (qr_resum).
// The window reductions run as rolled loops: these kernels are latency-bound on one or a few blocks, where the
// instruction fetch of fully unrolled code, not the arithmetic, sets the time.
template <int N> __host__ __device__ constexpr int qr_keep_words() { return qr_window<N>() + 6; }
template <int N, class Src> __device__ __noinline__ Num<N> block_exact_sum(const Src& src, u64 K, u32* sm, u32* error, u32* keep = nullptr) {
    constexpr int W = qr_window<N>();
    constexpr int WARPS = kQrThreads / 32;
    constexpr int WP = qr_row_words<N>(), P0 = (kQrRows * WP + 1) & ~1;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    u32* s_rows = sm;                                                // kQrRows partial windows
    u64* s_part = reinterpret_cast<u64*>(sm + P0);                   // 4 column sums of 16 rows each, per column
    long long* s_lo = reinterpret_cast<long long*>(s_part + 4 * W);
    long long* s_hi = s_lo + WARPS;
    u32* s_st = reinterpret_cast<u32*>(s_hi + WARPS);
    u32* s_cnt = s_st + WARPS;
    u32* s_res = s_cnt + WARPS;                                      // N + 3 words
    u32 st = 0, cnt = 0;
    long long lo = INT64_MAX, hi = INT64_MIN;
    for (u64 k = tid; k < K; k += kQrThreads) {
        Num<N> a, b;
        src.operands(k, a, b);
        st |= a.st | b.st;
        if (a.s && b.s) {
            const long long s = (long long)a.e + b.e - 2 * (32 * N - 1);
            lo = s < lo ? s : lo; hi = s + 64 * N > hi ? s + 64 * N : hi; ++cnt;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        st |= __shfl_xor_sync(0xffffffffu, st, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        const long long l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo; hi = h2 > hi ? h2 : hi;
    }
    if (lane == 0) { s_lo[warp] = lo; s_hi[warp] = hi; s_st[warp] = st; s_cnt[warp] = cnt; }
    __syncthreads();
    st = 0; cnt = 0; lo = INT64_MAX; hi = INT64_MIN;
#pragma unroll
    for (int w = 0; w < WARPS; ++w) {
        st |= s_st[w]; cnt += s_cnt[w];
        lo = s_lo[w] < lo ? s_lo[w] : lo; hi = s_hi[w] > hi ? s_hi[w] : hi;
    }
    __syncthreads();                                                 // the slots are reused by the next call
    if (keep && tid == 0) keep[0] = 0;
    if (st) return zero<N>(st);
    if (!cnt) return zero<N>();
    int logc = 0;
    while ((1u << logc) < cnt + 2) ++logc;
    Num<N> r = zero<N>();
    if (hi - lo + logc + 1 >= 32 * (long long)W) {
        if (tid == 0) store<N>(s_res, src.fallback(error));
        __syncthreads();
        r = load_plain<N>(s_res);
        __syncthreads();
        return r;
    }
    u32 acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    for (u64 k = tid; k < K; k += kQrThreads) {
        Num<N> a, b;
        src.operands(k, a, b);
        if (!a.s || !b.s) continue;
        u32 p[2 * N], t[W];
        mant_mul<N>(a.m, b.m, p);
        place_words<W, 2 * N>(t, p, (i64)a.e + b.e - 2 * (32 * N - 1) - lo);
        accumulate<W>(acc, t, a.s * b.s < 0);
    }
#pragma unroll 1
    for (int o = 16; o >= 32 / (kQrThreads / kQrRows); o >>= 1) {
        u32 other[W];
#pragma unroll
        for (int w = 0; w < W; ++w) other[w] = __shfl_down_sync(0xffffffffu, acc[w], o);
        accumulate<W>(acc, other, false);
    }
    constexpr int PER_WARP = kQrRows / WARPS;
    if (lane < PER_WARP) {
        u32* row = s_rows + (warp * PER_WARP + lane) * WP;
#pragma unroll
        for (int w = 0; w < W; ++w) row[w] = acc[w];
    }
    __syncthreads();
    for (int job = tid; job < 4 * W; job += kQrThreads) {            // job q * W + col: rows [16q, 16q + 16) of col
        const int q = job / W, col = job - q * W;
        const u32* at = s_rows + q * (kQrRows / 4) * WP + col;
        u64 s0 = 0, s1 = 0;
#pragma unroll
        for (int l = 0; l < kQrRows / 4; l += 2) { s0 += at[l * WP]; s1 += at[(l + 1) * WP]; }
        s_part[job] = s0 + s1;
    }
    __syncthreads();
    if (warp == 0) {
        constexpr int R = (W + 31) / 32;
        u32 v[R], h[R];
#pragma unroll
        for (int q = 0; q < R; ++q) {
            const int w = lane + 32 * q;
            const u64 sum = w < W ? s_part[w] + s_part[W + w] + s_part[2 * W + w] + s_part[3 * W + w] : 0;
            v[q] = (u32)sum; h[q] = (u32)(sum >> 32);
        }
        if (keep && lane == 0) {
            keep[0] = 1;
            keep[1] = (u32)(u64)lo; keep[2] = (u32)((u64)lo >> 32);
            keep[3] = (u32)(u64)hi; keep[4] = (u32)((u64)hi >> 32);
            keep[5] = (u32)logc;
        }
        const Num<N> res = warp_round_columns<N, W>(v, h, lo, keep ? keep + 6 : nullptr);
        if (lane == 0) store<N>(s_res, res);
    }
    __syncthreads();
    r = load_plain<N>(s_res);
    __syncthreads();
    return r;
}
template <int N, bool RO> __device__ Num<N> block_exact_dot(const u32* x, i64 sx, const u32* y, i64 sy, u64 K, u32* sm, u32* error,
                                                    u32* keep = nullptr) {
    return block_exact_sum<N>(StridedPair<N, RO>{x, sx, y, sy, K}, K, sm, error, keep);
}
// P(v, v) of a reflector from the kept window of s = P(x, x) (thread 0): v = 2^-e (v0, x_1, ...), so P(v, v) =
// 2^-2e RN(s_exact - x0^2 + v0^2) exactly, as long as every 2^-e x_r stays inside the exponent range and the window has
// room for v0^2; false when it does not (the caller then sums v afresh).  For a complex column x0 and v0 are the real
// parts of alpha and v0 (the imaginary part of v0 is alpha's).
template <int N> __device__ bool qr_resum(const u32* keep, const Num<N>& x0, const Num<N>& v0, long long e, Num<N>& out) {
    constexpr int W = qr_window<N>();
    if (!keep[0] || !v0.s || v0.st || x0.st) return false;
    const long long lo = (long long)((u64)keep[1] | ((u64)keep[2] << 32));
    const long long hi = (long long)((u64)keep[3] | ((u64)keep[4] << 32));
    const int logc = (int)keep[5];
    const long long xe_lo = (lo + 2 * (32 * N - 1)) / 2 - 1, xe_hi = (hi - 2) / 2 + 1;    // exponents of the entries
    if (xe_lo - e < -kEmax || xe_hi - e > kEmax) return false;
    const long long sv = 2 * (long long)v0.e - 2 * (32 * N - 1);
    const long long top = sv + 64 * N > hi ? sv + 64 * N : hi;
    if (sv < lo || top - lo + logc + 4 >= 32 * (long long)W) return false;
    u32 acc[W], p[2 * N], t[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = keep[6 + w];
    if (x0.s) {
        mant_mul<N>(x0.m, x0.m, p);
        place_words<W, 2 * N>(t, p, 2 * (long long)x0.e - 2 * (32 * N - 1) - lo);
        accumulate<W>(acc, t, true);
    }
    mant_mul<N>(v0.m, v0.m, p);
    place_words<W, 2 * N>(t, p, sv - lo);
    accumulate<W>(acc, t, false);
    if (acc[W - 1] >> 31) return false;
    out = qr_scaled<N>(round_general<N, W>(acc, lo, 1, 0), 2 * e);
    return true;
}

// Pt <- the panel's columns of Wk, Vt <- 0.
template <int N> __global__ void qr_load_kernel(QrPanel p) {
    constexpr u64 E = N + 3;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.kb * p.mr) return;
    const u64 c = q / p.mr, r = q % p.mr;
    const u32* src = p.Wk + ((p.k0 + r) * p.n + p.k0 + c) * E;
    u32* dst = p.Pt + q * E;
    u32* vt = p.Vt + q * E;
#pragma unroll
    for (u64 w = 0; w < E; ++w) { dst[w] = src[w]; vt[w] = 0; }
}
// The panel's columns and reflectors back into Wk and V; with pivoting only the columns before a failing one
// (linalg.mm:718: the failing column stays as it was at the block start, swapped into place).
template <int N> __global__ void qr_store_kernel(QrPanel p) {
    constexpr u64 E = N + 3;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.kb * p.mr) return;
    const u64 c = q / p.mr, r = q % p.mr;
    const long long rank = p.st->rank;
    if (p.pivot && rank < (long long)p.n && rank >= (long long)p.k0 && c >= (u64)(rank - (long long)p.k0)) return;
    const u64 at = ((p.k0 + r) * p.n + p.k0 + c) * E;
#pragma unroll
    for (u64 w = 0; w < E; ++w) { p.Wk[at + w] = p.Pt[q * E + w]; p.V[at + w] = p.Vt[q * E + w]; }
}

// Column c (j = k0 + c) by the panel's reflectors so far: x_r = D(x_r; Vt[0..q)[r], y[0..q)) for every row of the
// panel, q = min(j, rank) - k0.  One warp per row.
template <int N> __global__ void __launch_bounds__(256) qr_update_kernel(QrPanel p, u64 c) {
    constexpr u64 E = N + 3;
    const long long rank = p.st->rank, j = (long long)(p.k0 + c);
    const long long q = (rank < j ? rank : j) - (long long)p.k0;
    if (q <= 0) return;
    const u64 r = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= p.mr) return;
    u32* x = p.Pt + (c * p.mr + r) * E;
    const Num<N> v = warp_exact_dot<N, true>(x, true, p.Vt + r * E, (i64)p.mr, p.y, 1, (u64)q, p.error);
    if ((threadIdx.x & 31) == 0) store<N>(x, v);
}

// Reflector of column c from its reduced entries x = Pt[c][c..mr) (linalg.mm:675-690): s = P(x, x); a zero or
// status column, or one failing the rank test, ends the factorization there; otherwise beta = -sgn(x0) sqrt(s),
// v0 = RN(x0 - beta), v = 2^-e (v0, x1, ...) with e = exponent(v0) and tau = RN(2 / P(v, v)) (nothing below the
// diagonal: tau = 0, v = e_c, beta = x0); r_jj = beta, T_cc = tau.  One block.
template <int N> __global__ void __launch_bounds__(kQrThreads) qr_reflect_kernel(QrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    __shared__ u32 s_keep[qr_keep_words<N>()];
    __shared__ long long s_e;
    __shared__ int s_go, s_fast;
    constexpr u64 E = N + 3;
    QrState* st = p.st;
    if (st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, len = p.mr - c;
    u32* xc = p.Pt + (c * p.mr + c) * E;
    u32* v = p.Vt + (c * p.mr + c) * E;
    const Num<N> s = block_exact_dot<N, true>(xc, 1, xc, 1, len, sm, p.error, s_keep);
    int below = 0;
    for (u64 r = 1 + threadIdx.x; r < len; r += kQrThreads) below |= ldw<true>(xc + r * E + N + 1) != 0;
    below = __syncthreads_or(below);
    Num<N> beta = zero<N>(), v0 = qr_pow2<N>(0), x0 = zero<N>();
    if (threadIdx.x == 0) {
        x0 = load_plain<N>(xc);
        int reason = s.st ? 3 : (!x0.s && !below) ? 1 : 0;
        beta = x0;
        if (!reason && below) {
            beta = sqrt<N>(s);
            if (x0.s >= 0) beta = negate<N>(beta);
            v0 = subx<N>(x0, beta);
        }
        if (!reason && p.rank_bits > 0 && st->have_top && (long long)beta.e + p.rank_bits < st->top) reason = 2;
        if (reason) { st->rank = (long long)j; st->reason = reason; st->status = s.st; s_go = 0; }
        else { s_go = 1; s_e = below ? (long long)v0.e : 0; }
    }
    __syncthreads();
    if (!s_go) return;
    const long long e = s_e;
    // Thread 0 forms P(v, v) from the kept window and tau while warps 1.. scale the rest of the reflector.
    Num<N> tj = zero<N>();
    if (threadIdx.x == 0) {
        store<N>(v, below ? qr_scaled<N>(v0, e) : qr_pow2<N>(0));
        Num<N> pv;
        const int fast = below && qr_resum<N>(s_keep, x0, v0, e, pv);
        if (fast) tj = divx<N>(qr_pow2<N>(1), pv);
        s_fast = fast;
    }
    if (below && threadIdx.x >= 32)
        for (u64 r = 1 + threadIdx.x - 32; r < len; r += kQrThreads - 32) store<N>(v + r * E, qr_scaled<N>(load_plain<N>(xc + r * E), e));
    __syncthreads();
    if (below && !s_fast) {
        const Num<N> pv = block_exact_dot<N, false>(v, 1, v, 1, len, sm, p.error);
        if (threadIdx.x == 0) tj = divx<N>(qr_pow2<N>(1), pv);
    }
    if (threadIdx.x == 0) {
        store<N>(xc, beta);
        store<N>(p.tau + j * E, tj);
        store<N>(p.T + ((p.k0 / p.nb) * p.nb * p.nb + c * p.nb + c) * E, tj);
        if (!st->have_top || (long long)beta.e > st->top) st->top = beta.e;
        st->have_top = 1;
    }
}

// After reflector c: block u < c gives G[u] = P(v_u, v_c), block u >= c the W row entry Wp[c][u+1] = P(v_c,
// a_{u+1}) (the block-start column), both over rows [c, mr) (linalg.mm:636-645).  kb - 1 blocks.
template <int N> __global__ void __launch_bounds__(kQrThreads) qr_dots_kernel(QrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    constexpr u64 E = N + 3;
    QrState* st = p.st;
    const long long rank = st->rank;
    const bool reflected = rank == (long long)p.n;
    const u64 len = p.mr - c, u = blockIdx.x;
    if (reflected && u + 1 < p.kb) {
        const u32* v = p.Vt + (c * p.mr + c) * E;
        const Num<N> d = u < c ? block_exact_dot<N, true>(p.Vt + (u * p.mr + c) * E, 1, v, 1, len, sm, p.error)
                               : block_exact_dot<N, true>(v, 1, p.Pt + ((u + 1) * p.mr + c) * E, 1, len, sm, p.error);
        if (threadIdx.x == 0) store<N>(u < c ? p.G + u * E : p.Wp + (c * p.nb + u + 1) * E, d);
    }
}
// T column c, T_lc = -RN(tau * P(T[l][l..c), G[l..c))) (linalg.mm:713), then the next column's y_i = P(T[0..i][i],
// Wp[0..i][c+1]) for i < min(j + 1, rank) - k0 (linalg.mm:668): one warp per entry, 16 warps (a 32-column block's
// entries in two rounds).  One block, after the dots kernel.
constexpr int kQrTcolThreads = 512;
template <int N> __global__ void __launch_bounds__(kQrTcolThreads) qr_tcol_kernel(QrPanel p, u64 c) {
    constexpr u64 E = N + 3;
    const long long rank = p.st->rank;
    const bool reflected = rank == (long long)p.n;
    const u64 j = p.k0 + c;
    u32* Tb = p.T + (p.k0 / p.nb) * p.nb * p.nb * E;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int WARPS = kQrTcolThreads / 32;
    if (reflected) {
        const Num<N> tj = ldn<N, false>(p.tau + j * E);
        for (u64 l = warp; l < c; l += WARPS) {
            const Num<N> d = warp_exact_dot<N, false>(nullptr, false, Tb + (l * p.nb + l) * E, 1, p.G + l * E, 1, c - l, p.error);
            if (lane == 0) store<N>(Tb + (l * p.nb + c) * E, negate<N>(mulx<N>(tj, d)));
        }
    }
    __syncthreads();
    if (c + 1 < p.kb) {
        const long long qn = (rank < (long long)j + 1 ? rank : (long long)j + 1) - (long long)p.k0;
        for (long long i = warp; i < qn; i += WARPS) {
            const Num<N> d = warp_exact_dot<N, false>(nullptr, false, Tb + i * E, (i64)p.nb, p.Wp + (c + 1) * E, (i64)p.nb,
                                                      (u64)i + 1, p.error);
            if (lane == 0) store<N>(p.y + i * E, d);
        }
    }
}

// ---- column pivoting (the pivoted branch of linalg.mm:600-719; xGEQP3 order) ----
// Exact order of two squared norms for the pivot choice: +1 if x > y, -1 if x < y, 0 if equal; a status ranks above
// every value and two statuses are equal (linalg.mm:541-547).
template <int N> __device__ __forceinline__ int qr_order(const u32* x, const u32* y) {
    const u32 sx = x[N + 2], sy = y[N + 2];
    if (sx || sy) return (sx != 0) - (sy != 0);
    const int a = (int)x[N + 1], b = (int)y[N + 1];
    if (a != b) return a > b ? 1 : -1;
    if (!a) return 0;
    int c = 0;
    if (x[N] != y[N]) c = (int)x[N] > (int)y[N] ? 1 : -1;
    for (int i = N - 1; i >= 0 && !c; --i) if (x[i] != y[i]) c = x[i] > y[i] ? 1 : -1;
    return a > 0 ? c : -c;
}
// nu_k = nuref_k = P(a_k, a_k) over all rows; perm = identity.  One block per column.
template <int N> __global__ void __launch_bounds__(kQrThreads) qrp_norms_kernel(QrPanel p) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    constexpr u64 E = N + 3;
    const u64 k = blockIdx.x;
    const Num<N> d = block_exact_dot<N, true>(p.Wk + k * E, (i64)p.n, p.Wk + k * E, (i64)p.n, p.m, sm, p.error);
    if (threadIdx.x == 0) { store<N>(p.nu + k * E, d); store<N>(p.nuref + k * E, d); p.perm[k] = k; }
}
// Step j = k0 + c: the remaining column with the largest nu (a status first; ties to the lowest original index) is
// swapped with column j everywhere: Wk, the W and Y rows of this block's earlier steps, nu, nuref, perm.  One block.
template <int N> __global__ void __launch_bounds__(kQrThreads) qrp_pivot_kernel(QrPanel p, u64 c) {
    __shared__ u32 s_best[kQrThreads];
    constexpr u64 E = N + 3;
    if (p.st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c;
    constexpr u32 kNone = 0xffffffffu;
    auto better = [&](u32 a, u32 b) {
        if (b == kNone) return a != kNone;
        if (a == kNone) return false;
        const int o = qr_order<N>(p.nu + (u64)a * E, p.nu + (u64)b * E);
        return o > 0 || (o == 0 && p.perm[a] < p.perm[b]);
    };
    u32 best = kNone;
    for (u64 k = j + threadIdx.x; k < p.n; k += kQrThreads)
        if (better((u32)k, best)) best = (u32)k;
    s_best[threadIdx.x] = best;
    __syncthreads();
    for (int h = kQrThreads / 2; h; h >>= 1) {
        if ((int)threadIdx.x < h && better(s_best[threadIdx.x + h], s_best[threadIdx.x])) s_best[threadIdx.x] = s_best[threadIdx.x + h];
        __syncthreads();
    }
    const u64 q = s_best[0];
    if (q == j || q == kNone) return;
    for (u64 r = threadIdx.x; r < p.m; r += kQrThreads)
        for (u64 w = 0; w < E; ++w) {
            u32* a = p.Wk + (r * p.n + j) * E + w; u32* b = p.Wk + (r * p.n + q) * E + w;
            const u32 t = *a; *a = *b; *b = t;
        }
    for (u64 i = threadIdx.x; i < c; i += kQrThreads)
        for (u64 w = 0; w < E; ++w) {
            u32* a = p.Wr + (i * p.n + j) * E + w; u32* b = p.Wr + (i * p.n + q) * E + w;
            u32 t = *a; *a = *b; *b = t;
            a = p.Yr + (i * p.n + j) * E + w; b = p.Yr + (i * p.n + q) * E + w;
            t = *a; *a = *b; *b = t;
        }
    if (threadIdx.x == 0) {
        for (u64 w = 0; w < E; ++w) {
            u32 t = p.nu[j * E + w]; p.nu[j * E + w] = p.nu[q * E + w]; p.nu[q * E + w] = t;
            t = p.nuref[j * E + w]; p.nuref[j * E + w] = p.nuref[q * E + w]; p.nuref[q * E + w] = t;
        }
        const u64 t = p.perm[j]; p.perm[j] = p.perm[q]; p.perm[q] = t;
    }
}
// Column j reduced by this block's reflectors so far with its Y entries from the earlier steps:
// Pt[c][r] = D(a_{k0+r,j}; V_{k0+r}[k0, k0+c), Y[0..c)[j]) for every row of the panel (linalg.mm:662, 668-670).
// One warp per row.
template <int N> __global__ void __launch_bounds__(256) qrp_column_kernel(QrPanel p, u64 c) {
    constexpr u64 E = N + 3;
    if (p.st->rank < (long long)p.n) return;
    const u64 r = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= p.mr) return;
    const u64 j = p.k0 + c;
    const u32* a = p.Wk + ((p.k0 + r) * p.n + j) * E;
    u32* x = p.Pt + (c * p.mr + r) * E;
    const Num<N> v = c ? warp_exact_dot<N, true>(a, true, p.Vt + r * E, (i64)p.mr, p.Yr + j * E, (i64)p.n, c, p.error)
                       : ldn<N, true>(a);
    if ((threadIdx.x & 31) == 0) store<N>(x, v);
}
// After reflector j: block u < c gives the Gram entry G[u] = P(v_u, v_j) over the panel rows [c, mr); block u >= c
// the W row entry W[c][k] = P(v_j, a_k) over rows [j, m) of trailing column k = j + 1 + (u - c) (block-start values,
// linalg.mm:636-645).  The last block to arrive writes the T column (linalg.mm:713).
template <int N> __global__ void __launch_bounds__(kQrThreads) qrp_gramw_kernel(QrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    __shared__ int s_last;
    constexpr u64 E = N + 3;
    QrState* st = p.st;
    if (st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, len = p.mr - c, u = blockIdx.x;
    const u32* v = p.Vt + (c * p.mr + c) * E;
    if (u < c) {
        const Num<N> d = block_exact_dot<N, true>(p.Vt + (u * p.mr + c) * E, 1, v, 1, len, sm, p.error);
        if (threadIdx.x == 0) store<N>(p.G + u * E, d);
    } else if (j + 1 + (u - c) < p.n) {
        const u64 k = j + 1 + (u - c);
        const Num<N> d = block_exact_dot<N, true>(v, 1, p.Wk + (j * p.n + k) * E, (i64)p.n, len, sm, p.error);
        if (threadIdx.x == 0) store<N>(p.Wr + (c * p.n + k) * E, d);
    }
    if (threadIdx.x == 0) {
        __threadfence();
        const u32 before = atomicAdd(&st->arrivals, 1u);
        s_last = before == gridDim.x - 1;
        if (s_last) st->arrivals = 0;
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    u32* Tb = p.T + (p.k0 / p.nb) * p.nb * p.nb * E;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const Num<N> tj = ldn<N, false>(p.tau + j * E);
    for (u64 l = warp; l < c; l += kQrThreads / 32) {
        const Num<N> d = warp_exact_dot<N, false>(nullptr, false, Tb + (l * p.nb + l) * E, 1, p.G + l * E, 1, c - l, p.error);
        if (lane == 0) store<N>(Tb + (l * p.nb + c) * E, negate<N>(mulx<N>(tj, d)));
    }
}
// Every trailing column k > j: Y[c][k] = P(T[0..c][c], W[0..c][k]), r_jk = D(a_jk; V_j[k0..j], Y[0..c][k]) and
// nu_k = D(nu_k; r_jk, r_jk); flag_k when nu_k drops to <= 0 or more than bits/2 binades below nuref_k (nuref_k a
// status-free nonzero, nu_k status-free) (linalg.mm:714-723).  One warp per column.
template <int N> __global__ void __launch_bounds__(256) qrp_trailing_kernel(QrPanel p, u64 c) {
    constexpr u64 E = N + 3;
    if (p.st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c;
    const u64 k = j + 1 + (((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (k >= p.n) return;
    const int lane = threadIdx.x & 31;
    const u32* Tb = p.T + (p.k0 / p.nb) * p.nb * p.nb * E;
    const Num<N> y = warp_exact_dot<N, true>(nullptr, false, Tb + c * E, (i64)p.nb, p.Wr + k * E, (i64)p.n, c + 1, p.error);
    if (lane == 0) store<N>(p.Yr + (c * p.n + k) * E, y);
    __syncwarp();
    const Num<N> r = warp_exact_dot<N, false>(p.Wk + (j * p.n + k) * E, true, p.Vt + c * E, (i64)p.mr, p.Yr + k * E, (i64)p.n, c + 1,
                                              p.error);
    if (lane == 0) {
        const Num<N> nu = negate<N>(fms<N>(r, r, ldn<N, false>(p.nu + k * E)));
        const Num<N> ref = ldn<N, false>(p.nuref + k * E);
        store<N>(p.nu + k * E, nu);
        p.flag[k] = ref.s && !ref.st && !nu.st && (nu.s <= 0 || (long long)nu.e + 16 * N < (long long)ref.e);
    }
}
// Operands of the recomputed squared norm: z_i = D(a_{k0+i,k}; V_{k0+i}[k0..j], Y[0..c][k]) for the panel rows i in
// (c, mr), squared.  The fallback runs the cluster method over the same terms.
template <int N> struct ReducedSquares {
    const QrPanel* p; u64 c, k;
    __device__ Num<N> z(u64 q) const {
        constexpr u64 E = N + 3;
        const u64 i = c + 1 + q;
        return exact_dot_add_dev<N, true>(p->Wk + ((p->k0 + i) * p->n + k) * E, true, p->Vt + i * E, (i64)p->mr, p->Yr + k * E,
                                          (i64)p->n, c + 1, p->error);
    }
    __device__ void operands(u64 q, Num<N>& a, Num<N>& b) const { a = z(q); b = a; }
    // the cluster-method source: term q is z_q^2
    __device__ u64 count() const { return p->mr - c - 1; }
    __device__ bool term(u64 q, i64& scale, i64& top, int& sign) const {
        const Num<N> a = z(q);
        if (!a.s) return false;
        scale = 2 * (i64)a.e - 2 * (32 * N - 1); top = scale + 64 * N; sign = 1;
        return true;
    }
    __device__ void add(u64 q, u32* acc, int len, i64 off) const {
        const Num<N> a = z(q);
        u32 prod[2 * N];
        mant_mul<N>(a.m, a.m, prod);
        acc_add(acc, len, prod, 2 * N, off);
    }
    __device__ Num<N> fallback(u32* error) const {
        u32 st = 0;
        for (u64 q = 0; q < count(); ++q) st |= z(q).st;
        if (st) return zero<N>(st);
        return cluster_round<N, kClusterWords>(*this, error);
    }
};
// Flagged columns: nu_k = nuref_k = P(z, z) over the reduced column below row j (linalg.mm:724-727).  One block per
// trailing column; unflagged blocks return at once.
template <int N> __global__ void __launch_bounds__(kQrThreads) qrp_recompute_kernel(QrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    constexpr u64 E = N + 3;
    if (p.st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, k = j + 1 + blockIdx.x;
    if (k >= p.n || !p.flag[k]) return;
    const ReducedSquares<N> src{&p, c, k};
    const Num<N> d = block_exact_sum<N>(src, src.count(), sm, p.error);
    if (threadIdx.x == 0) {
        store<N>(p.nu + k * E, d); store<N>(p.nuref + k * E, d);
        atomicAdd(&p.st->recomputed, 1u);
    }
}

// R (n x n) <- the upper triangle of Wk's first n rows; with rank p < n, rows i >= p keep columns j >= p.
template <int N> __global__ void qr_extract_kernel(const u32* Wk, u32* R, u64 n, const QrState* st) {
    constexpr u64 E = N + 3;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * n) return;
    const u64 i = q / n, j = q % n, rank = (u64)st->rank;
    const bool keep = j >= (i < rank ? i : rank);
#pragma unroll
    for (u64 w = 0; w < E; ++w) R[q * E + w] = keep ? Wk[q * E + w] : 0u;
}
// dst (rows x cols, row stride ld_dst) <- src (row stride ld_src), element copies.
template <int N> __global__ void qr_copy_kernel(const u32* src, u64 ld_src, u32* dst, u64 ld_dst, u64 rows, u64 cols) {
    constexpr u64 E = N + 3;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= rows * cols) return;
    const u64 i = q / cols, j = q % cols;
#pragma unroll
    for (u64 w = 0; w < E; ++w) dst[(i * ld_dst + j) * E + w] = src[(i * ld_src + j) * E + w];
}

struct QrKernels {
    void (*load)(const QrPanel&, cudaStream_t);
    void (*update)(const QrPanel&, u64 c, cudaStream_t);
    void (*reflect)(const QrPanel&, u64 c, cudaStream_t);
    void (*dots)(const QrPanel&, u64 c, cudaStream_t);
    void (*tcol)(const QrPanel&, u64 c, cudaStream_t);
    void (*store)(const QrPanel&, cudaStream_t);
    void (*extract)(const u32* Wk, u32* R, u64 n, const QrState* st, cudaStream_t);
    void (*copy)(const u32* src, u64 ld_src, u32* dst, u64 ld_dst, u64 rows, u64 cols, cudaStream_t);
    // column pivoting
    void (*norms)(const QrPanel&, cudaStream_t);
    void (*pivot)(const QrPanel&, u64 c, cudaStream_t);
    void (*column)(const QrPanel&, u64 c, cudaStream_t);
    void (*gramw)(const QrPanel&, u64 c, cudaStream_t);
    void (*trailing)(const QrPanel&, u64 c, cudaStream_t);
    void (*recompute)(const QrPanel&, u64 c, cudaStream_t);
};
const QrKernels* qr_kernels(int limbs);

inline unsigned qr_grid(u64 items, unsigned threads) { return (unsigned)((items + threads - 1) / threads); }
template <int N> void qr_load_launch(const QrPanel& p, cudaStream_t s) {
    if (p.kb * p.mr) qr_load_kernel<N><<<qr_grid(p.kb * p.mr, 128), 128, 0, s>>>(p);
}
template <int N> void qr_store_launch(const QrPanel& p, cudaStream_t s) {
    if (p.kb * p.mr) qr_store_kernel<N><<<qr_grid(p.kb * p.mr, 128), 128, 0, s>>>(p);
}
template <int N> void qr_update_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    if (p.mr) qr_update_kernel<N><<<qr_grid(p.mr * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void qr_reflect_launch(const QrPanel& p, u64 c, cudaStream_t s) { qr_reflect_kernel<N><<<1, kQrThreads, 0, s>>>(p, c); }
template <int N> void qr_dots_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    if (p.kb > 1) qr_dots_kernel<N><<<(unsigned)(p.kb - 1), kQrThreads, 0, s>>>(p, c);
}
template <int N> void qr_tcol_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    if (p.kb > 1) qr_tcol_kernel<N><<<1, kQrTcolThreads, 0, s>>>(p, c);
}
template <int N> void qr_extract_launch(const u32* Wk, u32* R, u64 n, const QrState* st, cudaStream_t s) {
    if (n) qr_extract_kernel<N><<<qr_grid(n * n, 128), 128, 0, s>>>(Wk, R, n, st);
}
template <int N> void qr_copy_launch(const u32* src, u64 ld_src, u32* dst, u64 ld_dst, u64 rows, u64 cols, cudaStream_t s) {
    if (rows * cols) qr_copy_kernel<N><<<qr_grid(rows * cols, 128), 128, 0, s>>>(src, ld_src, dst, ld_dst, rows, cols);
}

template <int N> void qrp_norms_launch(const QrPanel& p, cudaStream_t s) {
    if (p.n) qrp_norms_kernel<N><<<(unsigned)p.n, kQrThreads, 0, s>>>(p);
}
template <int N> void qrp_pivot_launch(const QrPanel& p, u64 c, cudaStream_t s) { qrp_pivot_kernel<N><<<1, kQrThreads, 0, s>>>(p, c); }
template <int N> void qrp_column_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    if (p.mr) qrp_column_kernel<N><<<qr_grid(p.mr * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void qrp_gramw_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    const u64 trailing = p.n - (p.k0 + c) - 1, blocks = c + trailing;
    qrp_gramw_kernel<N><<<(unsigned)(blocks ? blocks : 1), kQrThreads, 0, s>>>(p, c);
}
template <int N> void qrp_trailing_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    const u64 trailing = p.n - (p.k0 + c) - 1;
    if (trailing) qrp_trailing_kernel<N><<<qr_grid(trailing * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void qrp_recompute_launch(const QrPanel& p, u64 c, cudaStream_t s) {
    const u64 trailing = p.n - (p.k0 + c) - 1;
    if (trailing) qrp_recompute_kernel<N><<<(unsigned)trailing, kQrThreads, 0, s>>>(p, c);
}

}  // namespace lfd

#define LF_QR_INSTANTIATE(N)                                                                                        \
    namespace lfd {                                                                                                 \
    extern const QrKernels qr_kernels_##N;                                                                          \
    const QrKernels qr_kernels_##N = {qr_load_launch<N>, qr_update_launch<N>, qr_reflect_launch<N>, qr_dots_launch<N>, \
                                      qr_tcol_launch<N>, qr_store_launch<N>, qr_extract_launch<N>, qr_copy_launch<N>, qrp_norms_launch<N>,  \
                                      qrp_pivot_launch<N>, qrp_column_launch<N>, qrp_gramw_launch<N>,                   \
                                      qrp_trailing_launch<N>, qrp_recompute_launch<N>};                                 \
    }
