// Complex Householder QR panel kernels (the reference's src/linalg_complex.mm:125-306: zgeqrf convention,
// H = I - tau v v^H with complex tau and real beta).  Every complex dot product or update is two real exact dot
// products over the interleaved (re, im) operand sequences, one rounding per component; a complex array of
// elements (re, im) is read as such a real sequence with unit stride.  The panel mirrors the real one (lf_qr.cuh):
// column-contiguous Pt (the panel's columns), Vt (reflectors) and Vi (i v), plus Vr (the reflectors by rows,
// entry (r, c) at r * nb + c), four launches per column and a device-side state; the trailing updates are the
// real compact-WY products on the 2 x 2-block real embeddings of V and T ([[re, -im], [im, re]]) applied to the
// work matrix split by rows (row 2r = Re of row r, 2r + 1 = Im).
#pragma once
#include "lf_qr.cuh"

namespace lfd {

struct CqrPanel {
    u32* Wk; u64 m, n;               // the row-split work matrix (2m x n real), reduced in place
    u32* V; u32* T; u32* tau;        // the complex factor: V (m x n), T (blocks of nb x nb), tau (n)
    u32* EV; u32* ET;                // real embeddings: EV (2m x 2n), ET (blocks of 2nb x 2nb)
    u32* Pt; u32* Vt; u32* Vi; u32* Vr;
    u32* Wp; u32* G; u32* Gc; u32* Gic; u32* yc; u32* yic;
    u32* scr;                        // per y entry: the T column, i times it and the W column (3 nb complex)
    u64 k0, kb, nb, mr;
    int rank_bits;
    QrState* st;
    u32* error;
    // column pivoting (pivot != 0): the W and Y rows of the trailing columns as real rows (2 nb x n: row 2c = Re,
    // 2c + 1 = Im of step c), real squared norms nu and nuref (n), the permutation and recomputation flags (n), the
    // reflectors by rows as conj(v) (Vrc) and i conj(v) (Vri), and the T column with i times it (tc, 2 nb complex)
    int pivot;
    u32* Wr; u32* Yr; u32* nu; u32* nuref; u64* perm; u32* flag;
    u32* Vrc; u32* Vri; u32* tc;
};

template <int N> __device__ __forceinline__ void cq_store(u32* p, const Num<N>& re, const Num<N>& im) { store<N>(p, re); store<N>(p + N + 3, im); }
// i z, conj(z), i conj(z) of the complex element at p, written to q
template <int N> __device__ __forceinline__ void cq_times_i(u32* q, const u32* p) {
    const Num<N> re = load_plain<N>(p), im = load_plain<N>(p + N + 3);
    cq_store<N>(q, negate<N>(im), re);
}
template <int N> __device__ __forceinline__ void cq_conj(u32* q, const u32* p) {
    const Num<N> re = load_plain<N>(p), im = load_plain<N>(p + N + 3);
    cq_store<N>(q, re, negate<N>(im));
}
template <int N> __device__ __forceinline__ void cq_i_conj(u32* q, const u32* p) {
    const Num<N> re = load_plain<N>(p), im = load_plain<N>(p + N + 3);
    cq_store<N>(q, im, re);
}
// The 2 x 2 real block [[re, -im], [im, re]] of the complex element at z, written at (2r, 2c) of M (row stride ld).
template <int N> __device__ __forceinline__ void cq_embed(u32* M, u64 ld, u64 r, u64 c, const u32* z) {
    constexpr u64 E = N + 3;
    const Num<N> re = load_plain<N>(z), im = load_plain<N>(z + E);
    store<N>(M + (2 * r * ld + 2 * c) * E, re); store<N>(M + (2 * r * ld + 2 * c + 1) * E, negate<N>(im));
    store<N>(M + ((2 * r + 1) * ld + 2 * c) * E, im); store<N>(M + ((2 * r + 1) * ld + 2 * c + 1) * E, re);
}

// Pt <- the panel's columns of the row-split Wk; Vt, Vi, Vr <- 0.
template <int N> __global__ void cqr_load_kernel(CqrPanel p) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= p.mr * p.nb) return;
    for (u64 w = 0; w < C2; ++w) p.Vr[q * C2 + w] = 0;
    if (p.pivot)
        for (u64 w = 0; w < C2; ++w) { p.Vrc[q * C2 + w] = 0; p.Vri[q * C2 + w] = 0; }
    if (q >= p.kb * p.mr) return;
    const u64 c = q / p.mr, r = q % p.mr;
    const u32* re = p.Wk + (2 * (p.k0 + r) * p.n + p.k0 + c) * E;
    const u32* im = re + p.n * E;
    for (u64 w = 0; w < E; ++w) { p.Pt[q * C2 + w] = re[w]; p.Pt[q * C2 + E + w] = im[w]; }
    for (u64 w = 0; w < C2; ++w) { p.Vt[q * C2 + w] = 0; p.Vi[q * C2 + w] = 0; }
}
// Column c by the panel's reflectors so far: x_r = (D(Re x_r; Vr[r][0..q), conj y), D(Im x_r; Vr[r][0..q), i conj y))
// over 2q real terms each (linalg_complex.mm:188-193).  One warp per row.
template <int N> __global__ void __launch_bounds__(256) cqr_update_kernel(CqrPanel p, u64 c) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    const long long rank = p.st->rank, j = (long long)(p.k0 + c);
    const long long q = (rank < j ? rank : j) - (long long)p.k0;
    if (q <= 0) return;
    const u64 r = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= p.mr) return;
    u32* x = p.Pt + (c * p.mr + r) * C2;
    const u32* vr = p.Vr + r * p.nb * C2;
    const Num<N> re = warp_exact_dot<N, true>(x, true, vr, 1, p.yc, 1, 2 * (u64)q, p.error);
    const Num<N> im = warp_exact_dot<N, true>(x + E, true, vr, 1, p.yic, 1, 2 * (u64)q, p.error);
    if ((threadIdx.x & 31) == 0) cq_store<N>(x, re, im);
}
// Reflector of column c (linalg_complex.mm:205-226): s = P(x^H x); a zero or status column, or one failing the rank
// test, ends the factorization; otherwise, when anything lies below the diagonal or Im alpha != 0, beta =
// -sgn(Re alpha) sqrt(s), v0 = (RN(Re alpha - beta), Im alpha), v = 2^-e (v0, x_1, ...) with e = exponent(Re v0) and
// tau = (RN(2 / P(v^H v)), 0) when Im v0 = 0, else with a = P(v^H v) / 2, b = RN(2^-e beta Im v0), d = RN(a^2 + b^2):
// tau = (RN(a / d), -RN(b / d)); nothing to reflect: tau = 0, v = e_c, r_jj = alpha.  r_jj = (beta, 0), T_cc = tau,
// and the rows of v and i v from row c (Vt, Vi, Vr).  One block.
template <int N> __global__ void __launch_bounds__(kQrThreads) cqr_reflect_kernel(CqrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    __shared__ u32 s_keep[qr_keep_words<N>()];
    __shared__ long long s_e;
    __shared__ int s_go, s_needs, s_fast;
    constexpr u64 E = N + 3, C2 = 2 * E;
    QrState* st = p.st;
    if (st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, len = p.mr - c;
    u32* xc = p.Pt + (c * p.mr + c) * C2;
    u32* v = p.Vt + (c * p.mr + c) * C2;
    u32* iv = p.Vi + (c * p.mr + c) * C2;
    const Num<N> s = block_exact_dot<N, true>(xc, 1, xc, 1, 2 * len, sm, p.error, s_keep);
    int below = 0;
    for (u64 k = 2 + threadIdx.x; k < 2 * len; k += kQrThreads) below |= ldw<true>(xc + k * E + N + 1) != 0;
    below = __syncthreads_or(below);
    Num<N> beta = zero<N>(), v0 = qr_pow2<N>(0), are = zero<N>(), aim = zero<N>();
    if (threadIdx.x == 0) {
        are = load_plain<N>(xc); aim = load_plain<N>(xc + E);
        const int needs = below || aim.s;
        int reason = s.st ? 3 : (!are.s && !aim.s && !below) ? 1 : 0;
        beta = are;
        if (!reason && needs) {
            beta = sqrt<N>(s);
            if (are.s >= 0) beta = negate<N>(beta);
            v0 = subx<N>(are, beta);
        }
        if (!reason && p.rank_bits > 0 && st->have_top && (long long)beta.e + p.rank_bits < st->top) reason = 2;
        if (reason) { st->rank = (long long)j; st->reason = reason; st->status = s.st; s_go = 0; }
        else {
            s_go = 1; s_needs = needs; s_e = needs ? (long long)v0.e : 0;
            if (needs) cq_store<N>(v, qr_scaled<N>(v0, s_e), qr_scaled<N>(aim, s_e));
            else cq_store<N>(v, qr_pow2<N>(0), zero<N>());
        }
    }
    __syncthreads();
    if (!s_go) return;
    const long long e = s_e;
    const bool needs = s_needs;
    Num<N> tre = zero<N>(), tim = zero<N>();
    auto tau_of = [&](const Num<N>& sv) {                             // thread 0
        const Num<N> vim = load_plain<N>(v + E);
        if (!vim.s && !vim.st) tre = divx<N>(qr_pow2<N>(1), sv);
        else {
            const Num<N> a = qr_scaled<N>(sv, 1), b = mulx<N>(qr_scaled<N>(beta, e), vim);
            const Num<N> d = dot2_add<N>(a, a, b, b, zero<N>());
            tre = divx<N>(a, d); tim = negate<N>(divx<N>(b, d));
        }
    };
    // Thread 0 forms P(v^H v) from the kept window and tau while warps 1.. scale the rest of the reflector.
    if (threadIdx.x == 0) {
        Num<N> sv;
        const int fast = needs && qr_resum<N>(s_keep, are, v0, e, sv);
        if (fast) tau_of(sv);
        s_fast = fast;
    }
    if (needs && threadIdx.x >= 32)
        for (u64 r = 1 + threadIdx.x - 32; r < len; r += kQrThreads - 32)
            cq_store<N>(v + r * C2, qr_scaled<N>(load_plain<N>(xc + r * C2), e), qr_scaled<N>(load_plain<N>(xc + r * C2 + E), e));
    __syncthreads();
    if (needs && !s_fast) {
        const Num<N> sv = block_exact_dot<N, false>(v, 1, v, 1, 2 * len, sm, p.error);
        if (threadIdx.x == 0) tau_of(sv);
    }
    if (threadIdx.x == 0) {
        cq_store<N>(xc, beta, zero<N>());
        cq_store<N>(p.tau + j * C2, tre, tim);
        cq_store<N>(p.T + ((p.k0 / p.nb) * p.nb * p.nb + c * p.nb + c) * C2, tre, tim);
        if (!st->have_top || (long long)beta.e > st->top) st->top = beta.e;
        st->have_top = 1;
    }
    for (u64 r = threadIdx.x; r < len; r += kQrThreads) {
        cq_times_i<N>(iv + r * C2, v + r * C2);
        for (u64 w = 0; w < C2; ++w) p.Vr[((c + r) * p.nb + c) * C2 + w] = v[r * C2 + w];
        if (p.pivot) {
            cq_conj<N>(p.Vrc + ((c + r) * p.nb + c) * C2, v + r * C2);
            cq_i_conj<N>(p.Vri + ((c + r) * p.nb + c) * C2, v + r * C2);
        }
    }
}
// After reflector c: block u < c gives G[u] = P(v_u^H v_c), block u >= c the W row entry Wp[c][u+1] = P(v_c^H a_{u+1})
// (the block-start column), over rows [c, mr), two real dots each.  kb - 1 blocks.
template <int N> __global__ void __launch_bounds__(kQrThreads) cqr_dots_kernel(CqrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    constexpr u64 E = N + 3, C2 = 2 * E;
    const long long rank = p.st->rank;
    const bool reflected = rank == (long long)p.n;
    const u64 len = p.mr - c, u = blockIdx.x;
    if (reflected && u + 1 < p.kb) {
        const u32* v = p.Vt + (c * p.mr + c) * C2;
        const u32* iv = p.Vi + (c * p.mr + c) * C2;
        const u32 *a0, *a1, *b0;
        u32* out;
        if (u < c) { a0 = p.Vt + (u * p.mr + c) * C2; a1 = p.Vi + (u * p.mr + c) * C2; b0 = v; out = p.G + u * C2; }
        else { a0 = v; a1 = iv; b0 = p.Pt + ((u + 1) * p.mr + c) * C2; out = p.Wp + (c * p.nb + u + 1) * C2; }
        const Num<N> re = block_exact_dot<N, true>(a0, 1, b0, 1, 2 * len, sm, p.error);
        const Num<N> im = block_exact_dot<N, true>(a1, 1, b0, 1, 2 * len, sm, p.error);
        if (threadIdx.x == 0) cq_store<N>(out, re, im);
    }
}

// T column c, T_lc = -(tau * P(T[l][l..c) G[l..c))) with one rounding per component (cfma, linalg_complex.mm:237),
// then the next column's conj y and i conj y for y_i = P(T[0..i][i]^H Wp[0..i][c+1]) (linalg_complex.mm:186-187): one
// warp per entry, 16 warps.  One block, after the dots kernel.
constexpr int kCqrTcolThreads = 512;
template <int N> __global__ void __launch_bounds__(kCqrTcolThreads) cqr_tcol_kernel(CqrPanel p, u64 c) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    const long long rank = p.st->rank;
    const bool reflected = rank == (long long)p.n;
    const u64 j = p.k0 + c;
    u32* Tb = p.T + (p.k0 / p.nb) * p.nb * p.nb * C2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int WARPS = kCqrTcolThreads / 32;
    if (reflected) {
        for (u64 l = threadIdx.x; l < c; l += kCqrTcolThreads) { cq_conj<N>(p.Gc + l * C2, p.G + l * C2); cq_i_conj<N>(p.Gic + l * C2, p.G + l * C2); }
        __syncthreads();
        const Num<N> tre = ldn<N, false>(p.tau + j * C2), tim = ldn<N, false>(p.tau + j * C2 + E);
        for (u64 l = warp; l < c; l += WARPS) {
            const u32* trow = Tb + (l * p.nb + l) * C2;
            const Num<N> pre = warp_exact_dot<N, false>(nullptr, false, trow, 1, p.Gc + l * C2, 1, 2 * (c - l), p.error);
            const Num<N> pim = warp_exact_dot<N, false>(nullptr, false, trow, 1, p.Gic + l * C2, 1, 2 * (c - l), p.error);
            if (lane == 0) {
                const Cpx<N> z = cfma<N>(Cpx<N>{tre, tim}, Cpx<N>{pre, pim}, Cpx<N>{zero<N>(), zero<N>()});
                cq_store<N>(Tb + (l * p.nb + c) * C2, negate<N>(z.re), negate<N>(z.im));
            }
        }
    }
    __syncthreads();
    if (c + 1 < p.kb) {
        const long long qn = (rank < (long long)j + 1 ? rank : (long long)j + 1) - (long long)p.k0;
        for (long long i = warp; i < qn; i += WARPS) {
            u32* tcol = p.scr + (u64)i * 3 * p.nb * C2;
            u32* itcol = tcol + p.nb * C2;
            u32* wl = itcol + p.nb * C2;
            for (long long l = lane; l <= i; l += 32) {
                const u32* t = Tb + ((u64)l * p.nb + (u64)i) * C2;
                for (u64 w = 0; w < C2; ++w) { tcol[l * C2 + w] = t[w]; wl[l * C2 + w] = p.Wp[((u64)l * p.nb + c + 1) * C2 + w]; }
                cq_times_i<N>(itcol + l * C2, t);
            }
            __syncwarp();
            const Num<N> yre = warp_exact_dot<N, false>(nullptr, false, tcol, 1, wl, 1, 2 * ((u64)i + 1), p.error);
            const Num<N> yim = warp_exact_dot<N, false>(nullptr, false, itcol, 1, wl, 1, 2 * ((u64)i + 1), p.error);
            if (lane == 0) { cq_store<N>(p.yc + i * C2, yre, negate<N>(yim)); cq_store<N>(p.yic + i * C2, yim, yre); }
        }
    }
}
// ---- column pivoting (linalg_complex.mm:136-139, 160-255): the real pivoted sequence on complex columns.  The
// squared norms are real sums over the 2m split rows (qrp_norms_kernel on the split matrix); conj(v) and i conj(v)
// by rows turn every complex reduction into two real dots against the real Y rows read with stride n.
// Step j = k0 + c: the remaining column with the largest nu (a status first; ties to the lowest original index) is
// swapped with column j in the 2m split rows of Wk, rows [0, 2c) of the W and Y rows, nu, nuref and perm.  One block.
template <int N> __global__ void __launch_bounds__(kQrThreads) cqrp_pivot_kernel(CqrPanel p, u64 c) {
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
    auto swap = [&](u32* base, u64 row) {
        for (u64 w = 0; w < E; ++w) {
            u32* a = base + (row * p.n + j) * E + w; u32* b = base + (row * p.n + q) * E + w;
            const u32 t = *a; *a = *b; *b = t;
        }
    };
    for (u64 r = threadIdx.x; r < 2 * p.m; r += kQrThreads) swap(p.Wk, r);
    for (u64 i = threadIdx.x; i < 2 * c; i += kQrThreads) { swap(p.Wr, i); swap(p.Yr, i); }
    if (threadIdx.x == 0) {
        for (u64 w = 0; w < E; ++w) {
            u32 t = p.nu[j * E + w]; p.nu[j * E + w] = p.nu[q * E + w]; p.nu[q * E + w] = t;
            t = p.nuref[j * E + w]; p.nuref[j * E + w] = p.nuref[q * E + w]; p.nuref[q * E + w] = t;
        }
        const u64 t = p.perm[j]; p.perm[j] = p.perm[q]; p.perm[q] = t;
    }
}
// Column j of the panel reduced by this block's reflectors with its Y rows from the earlier steps:
// x_r = (D(Re a_rj; conj v_r[0..c), Y[0..2c)[j]), D(Im a_rj; i conj v_r[0..c), Y[0..2c)[j])) over 2c real terms each
// (linalg_complex.mm:188-193 with y read from the Y rows).  One warp per row.
template <int N> __global__ void __launch_bounds__(256) cqrp_column_kernel(CqrPanel p, u64 c) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    if (p.st->rank < (long long)p.n) return;
    const u64 r = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    if (r >= p.mr) return;
    const u64 j = p.k0 + c;
    const u32* are = p.Wk + (2 * (p.k0 + r) * p.n + j) * E;
    const u32* aim = are + p.n * E;
    u32* x = p.Pt + (c * p.mr + r) * C2;
    Num<N> re, im;
    if (c) {
        re = warp_exact_dot<N, true>(are, true, p.Vrc + r * p.nb * C2, 1, p.Yr + j * E, (i64)p.n, 2 * c, p.error);
        im = warp_exact_dot<N, true>(aim, true, p.Vri + r * p.nb * C2, 1, p.Yr + j * E, (i64)p.n, 2 * c, p.error);
    } else {
        re = ldn<N, true>(are);
        im = ldn<N, true>(aim);
    }
    if ((threadIdx.x & 31) == 0) cq_store<N>(x, re, im);
}
// After reflector j: block u < c gives G[u] = P(v_u^H v_j) over the panel rows [c, mr); block u >= c the W rows of
// trailing column k = j + 1 + (u - c): W[2c][k] = P(v_j . a_k), W[2c + 1][k] = P(i v_j . a_k) over the split rows
// from 2j (block-start values).  The last block to arrive writes the T column (cfma, linalg_complex.mm:237) and then
// the column with i times it for the Y rows.
template <int N> __global__ void __launch_bounds__(kQrThreads) cqrp_gramw_kernel(CqrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    __shared__ int s_last;
    constexpr u64 E = N + 3, C2 = 2 * E;
    QrState* st = p.st;
    if (st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, len = p.mr - c, u = blockIdx.x;
    const u32* v = p.Vt + (c * p.mr + c) * C2;
    const u32* iv = p.Vi + (c * p.mr + c) * C2;
    if (u < c) {
        const Num<N> re = block_exact_dot<N, true>(p.Vt + (u * p.mr + c) * C2, 1, v, 1, 2 * len, sm, p.error);
        const Num<N> im = block_exact_dot<N, true>(p.Vi + (u * p.mr + c) * C2, 1, v, 1, 2 * len, sm, p.error);
        if (threadIdx.x == 0) cq_store<N>(p.G + u * C2, re, im);
    } else if (j + 1 + (u - c) < p.n) {
        const u64 k = j + 1 + (u - c);
        const u32* a = p.Wk + (2 * j * p.n + k) * E;
        const Num<N> re = block_exact_dot<N, true>(v, 1, a, (i64)p.n, 2 * len, sm, p.error);
        const Num<N> im = block_exact_dot<N, true>(iv, 1, a, (i64)p.n, 2 * len, sm, p.error);
        if (threadIdx.x == 0) { store<N>(p.Wr + (2 * c * p.n + k) * E, re); store<N>(p.Wr + ((2 * c + 1) * p.n + k) * E, im); }
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
    u32* Tb = p.T + (p.k0 / p.nb) * p.nb * p.nb * C2;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    constexpr int WARPS = kQrThreads / 32;
    for (u64 l = threadIdx.x; l < c; l += kQrThreads) { cq_conj<N>(p.Gc + l * C2, p.G + l * C2); cq_i_conj<N>(p.Gic + l * C2, p.G + l * C2); }
    __syncthreads();
    const Num<N> tre = ldn<N, false>(p.tau + j * C2), tim = ldn<N, false>(p.tau + j * C2 + E);
    for (u64 l = warp; l < c; l += WARPS) {
        const u32* trow = Tb + (l * p.nb + l) * C2;
        const Num<N> pre = warp_exact_dot<N, false>(nullptr, false, trow, 1, p.Gc + l * C2, 1, 2 * (c - l), p.error);
        const Num<N> pim = warp_exact_dot<N, false>(nullptr, false, trow, 1, p.Gic + l * C2, 1, 2 * (c - l), p.error);
        if (lane == 0) {
            const Cpx<N> z = cfma<N>(Cpx<N>{tre, tim}, Cpx<N>{pre, pim}, Cpx<N>{zero<N>(), zero<N>()});
            cq_store<N>(Tb + (l * p.nb + c) * C2, negate<N>(z.re), negate<N>(z.im));
        }
    }
    __syncthreads();
    for (u64 l = threadIdx.x; l <= c; l += kQrThreads) {
        const u32* t = Tb + (l * p.nb + c) * C2;
        for (u64 w = 0; w < C2; ++w) p.tc[l * C2 + w] = t[w];
        cq_times_i<N>(p.tc + (p.nb + l) * C2, t);
    }
}
// Every trailing column k > j: the Y rows Y[2c][k] = P(T[0..c][c] . W[0..2c+2)[k]), Y[2c + 1][k] = P(i T[0..c][c] .
// W[0..2c+2)[k]); r_jk = (D(Re a_jk; conj v_j[0..c], Y[..][k]), D(Im a_jk; i conj v_j[0..c], Y[..][k])) and nu_k =
// RN(nu_k - |r_jk|^2); flag_k as the real rule (linalg_complex.mm:238-250).  One warp per column.
template <int N> __global__ void __launch_bounds__(256) cqrp_trailing_kernel(CqrPanel p, u64 c) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    if (p.st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c;
    const u64 k = j + 1 + (((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 5);
    if (k >= p.n) return;
    const int lane = threadIdx.x & 31;
    const Num<N> yre = warp_exact_dot<N, true>(nullptr, false, p.tc, 1, p.Wr + k * E, (i64)p.n, 2 * (c + 1), p.error);
    const Num<N> yim = warp_exact_dot<N, true>(nullptr, false, p.tc + p.nb * C2, 1, p.Wr + k * E, (i64)p.n, 2 * (c + 1), p.error);
    if (lane == 0) { store<N>(p.Yr + (2 * c * p.n + k) * E, yre); store<N>(p.Yr + ((2 * c + 1) * p.n + k) * E, yim); }
    __syncwarp();
    const u32* are = p.Wk + (2 * j * p.n + k) * E;
    const Num<N> rre = warp_exact_dot<N, false>(are, true, p.Vrc + c * p.nb * C2, 1, p.Yr + k * E, (i64)p.n, 2 * (c + 1), p.error);
    const Num<N> rim = warp_exact_dot<N, false>(are + p.n * E, true, p.Vri + c * p.nb * C2, 1, p.Yr + k * E, (i64)p.n, 2 * (c + 1),
                                                p.error);
    if (lane == 0) {
        const Num<N> nu = dot2_add<N>(negate<N>(rre), rre, negate<N>(rim), rim, ldn<N, false>(p.nu + k * E));
        const Num<N> ref = ldn<N, false>(p.nuref + k * E);
        store<N>(p.nu + k * E, nu);
        p.flag[k] = ref.s && !ref.st && !nu.st && (nu.s <= 0 || (long long)nu.e + 16 * N < (long long)ref.e);
    }
}
// Operands of a recomputed squared norm: the reduced column below row j, term 2q + part the square of component
// `part` of z_i = a_ik reduced by v_i[0..c] and the Y rows (i = c + 1 + q, a panel row).
template <int N> struct CReducedSquares {
    const CqrPanel* p; u64 c, k;
    __device__ Num<N> z(u64 t) const {
        constexpr u64 E = N + 3, C2 = 2 * E;
        const u64 i = c + 1 + t / 2, part = t & 1;
        return exact_dot_add_dev<N, true>(p->Wk + ((2 * (p->k0 + i) + part) * p->n + k) * E, true,
                                          (part ? p->Vri : p->Vrc) + i * p->nb * C2, 1, p->Yr + k * E, (i64)p->n, 2 * (c + 1),
                                          p->error);
    }
    __device__ void operands(u64 t, Num<N>& a, Num<N>& b) const { a = z(t); b = a; }
    __device__ u64 count() const { return 2 * (p->mr - c - 1); }
    __device__ bool term(u64 t, i64& scale, i64& top, int& sign) const {
        const Num<N> a = z(t);
        if (!a.s) return false;
        scale = 2 * (i64)a.e - 2 * (32 * N - 1); top = scale + 64 * N; sign = 1;
        return true;
    }
    __device__ void add(u64 t, u32* acc, int len, i64 off) const {
        const Num<N> a = z(t);
        u32 prod[2 * N];
        mant_mul<N>(a.m, a.m, prod);
        acc_add(acc, len, prod, 2 * N, off);
    }
    __device__ Num<N> fallback(u32* error) const {
        u32 st = 0;
        for (u64 t = 0; t < count(); ++t) st |= z(t).st;
        if (st) return zero<N>(st);
        return cluster_round<N, kClusterWords>(*this, error);
    }
};
// Flagged columns: nu_k = nuref_k = P(z^H z) over the reduced column below row j (linalg_complex.mm:251-254).  One
// block per trailing column; unflagged blocks return at once.
template <int N> __global__ void __launch_bounds__(kQrThreads) cqrp_recompute_kernel(CqrPanel p, u64 c) {
    __shared__ __align__(16) u32 sm[qr_dot_words<N>()];
    constexpr u64 E = N + 3;
    if (p.st->rank < (long long)p.n) return;
    const u64 j = p.k0 + c, k = j + 1 + blockIdx.x;
    if (k >= p.n || !p.flag[k]) return;
    const CReducedSquares<N> src{&p, c, k};
    const Num<N> d = block_exact_sum<N>(src, src.count(), sm, p.error);
    if (threadIdx.x == 0) {
        store<N>(p.nu + k * E, d); store<N>(p.nuref + k * E, d);
        atomicAdd(&p.st->recomputed, 1u);
    }
}

// The panel back into the row-split Wk, V (complex) and its embedding EV; the block's T into ET (entries l <= c).
template <int N> __global__ void cqr_store_kernel(CqrPanel p) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q < p.kb * p.kb) {
        const u64 l = q / p.kb, c = q % p.kb;
        if (l <= c) {
            const u64 b = p.k0 / p.nb;
            cq_embed<N>(p.ET + b * 4 * p.nb * p.nb * E, 2 * p.nb, l, c, p.T + (b * p.nb * p.nb + l * p.nb + c) * C2);
        }
    }
    if (q >= p.kb * p.mr) return;
    const u64 c = q / p.mr, r = q % p.mr;
    // with pivoting, a failing column and those after it stay as they were at the block start, swapped into place
    const long long rank = p.st->rank;
    if (p.pivot && rank < (long long)p.n && rank >= (long long)p.k0 && c >= (u64)(rank - (long long)p.k0)) return;
    const u32* x = p.Pt + q * C2;
    const u32* v = p.Vt + q * C2;
    u32* re = p.Wk + (2 * (p.k0 + r) * p.n + p.k0 + c) * E;
    for (u64 w = 0; w < E; ++w) { re[w] = x[w]; re[p.n * E + w] = x[E + w]; }
    for (u64 w = 0; w < C2; ++w) p.V[((p.k0 + r) * p.n + p.k0 + c) * C2 + w] = v[w];
    cq_embed<N>(p.EV, 2 * p.n, p.k0 + r, p.k0 + c, v);
}
// R (complex, n x n) <- the upper triangle of the row-split Wk (rows i >= rank keep columns j >= rank), and its
// real embedding ER (2n x 2n) for the solves.
template <int N> __global__ void cqr_extract_kernel(const u32* Wk, u32* R, u32* ER, u64 n, const QrState* st) {
    constexpr u64 E = N + 3, C2 = 2 * E;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n * n) return;
    const u64 i = q / n, j = q % n, rank = (u64)st->rank;
    const bool keep = j >= (i < rank ? i : rank);
    for (u64 w = 0; w < E; ++w) {
        R[q * C2 + w] = keep ? Wk[(2 * i * n + j) * E + w] : 0u;
        R[q * C2 + E + w] = keep ? Wk[((2 * i + 1) * n + j) * E + w] : 0u;
    }
    cq_embed<N>(ER, 2 * n, i, j, R + q * C2);
}

struct CqrKernels {
    void (*load)(const CqrPanel&, cudaStream_t);
    void (*update)(const CqrPanel&, u64 c, cudaStream_t);
    void (*reflect)(const CqrPanel&, u64 c, cudaStream_t);
    void (*dots)(const CqrPanel&, u64 c, cudaStream_t);
    void (*tcol)(const CqrPanel&, u64 c, cudaStream_t);
    void (*store)(const CqrPanel&, cudaStream_t);
    void (*extract)(const u32* Wk, u32* R, u32* ER, u64 n, const QrState* st, cudaStream_t);
    void (*pivot)(const CqrPanel&, u64 c, cudaStream_t);
    void (*column)(const CqrPanel&, u64 c, cudaStream_t);
    void (*gramw)(const CqrPanel&, u64 c, cudaStream_t);
    void (*trailing)(const CqrPanel&, u64 c, cudaStream_t);
    void (*recompute)(const CqrPanel&, u64 c, cudaStream_t);
};
const CqrKernels* cqr_kernels(int limbs);

template <int N> void cqr_load_launch(const CqrPanel& p, cudaStream_t s) {
    if (p.mr * p.nb) cqr_load_kernel<N><<<qr_grid(p.mr * p.nb, 128), 128, 0, s>>>(p);
}
template <int N> void cqr_update_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    if (p.mr) cqr_update_kernel<N><<<qr_grid(p.mr * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void cqr_reflect_launch(const CqrPanel& p, u64 c, cudaStream_t s) { cqr_reflect_kernel<N><<<1, kQrThreads, 0, s>>>(p, c); }
template <int N> void cqr_dots_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    if (p.kb > 1) cqr_dots_kernel<N><<<(unsigned)(p.kb - 1), kQrThreads, 0, s>>>(p, c);
}
template <int N> void cqr_tcol_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    if (p.kb > 1) cqr_tcol_kernel<N><<<1, kCqrTcolThreads, 0, s>>>(p, c);
}
template <int N> void cqr_store_launch(const CqrPanel& p, cudaStream_t s) {
    const u64 items = p.kb * p.mr > p.kb * p.kb ? p.kb * p.mr : p.kb * p.kb;
    if (items) cqr_store_kernel<N><<<qr_grid(items, 128), 128, 0, s>>>(p);
}
template <int N> void cqr_extract_launch(const u32* Wk, u32* R, u32* ER, u64 n, const QrState* st, cudaStream_t s) {
    if (n) cqr_extract_kernel<N><<<qr_grid(n * n, 128), 128, 0, s>>>(Wk, R, ER, n, st);
}

template <int N> void cqrp_pivot_launch(const CqrPanel& p, u64 c, cudaStream_t s) { cqrp_pivot_kernel<N><<<1, kQrThreads, 0, s>>>(p, c); }
template <int N> void cqrp_column_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    if (p.mr) cqrp_column_kernel<N><<<qr_grid(p.mr * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void cqrp_gramw_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    const u64 blocks = c + (p.n - (p.k0 + c) - 1);
    cqrp_gramw_kernel<N><<<(unsigned)(blocks ? blocks : 1), kQrThreads, 0, s>>>(p, c);
}
template <int N> void cqrp_trailing_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    const u64 trailing = p.n - (p.k0 + c) - 1;
    if (trailing) cqrp_trailing_kernel<N><<<qr_grid(trailing * 32, 256), 256, 0, s>>>(p, c);
}
template <int N> void cqrp_recompute_launch(const CqrPanel& p, u64 c, cudaStream_t s) {
    const u64 trailing = p.n - (p.k0 + c) - 1;
    if (trailing) cqrp_recompute_kernel<N><<<(unsigned)trailing, kQrThreads, 0, s>>>(p, c);
}

}  // namespace lfd

#define LF_CQR_INSTANTIATE(N)                                                                                   \
    namespace lfd {                                                                                             \
    extern const CqrKernels cqr_kernels_##N;                                                                    \
    const CqrKernels cqr_kernels_##N = {cqr_load_launch<N>, cqr_update_launch<N>, cqr_reflect_launch<N>,        \
                                        cqr_dots_launch<N>, cqr_tcol_launch<N>, cqr_store_launch<N>,            \
                                        cqr_extract_launch<N>,                                                  \
                                        cqrp_pivot_launch<N>, cqrp_column_launch<N>, cqrp_gramw_launch<N>,      \
                                        cqrp_trailing_launch<N>, cqrp_recompute_launch<N>};                     \
    }
