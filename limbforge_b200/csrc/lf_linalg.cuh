// Exact dense products on the GPU: C[i][j] = RN(c_ij -/+ sum_k L(i,k) R(j,k)) with one rounding per
// output (the contract of the reference's Linalg::gemm/syrk and exact_dot_add, linalg.hpp:1-7,
// 268-318).  Operands are strided "line" views of AoS element matrices: element (line, k) of a view
// sits at base + (line * ls + k * ks) elements.
//
// This file holds the per-line analysis and the generic limb kernel: one thread per output sums
// the exact 2N-word limb products cluster by cluster (terms sorted implicitly by scanning for the
// next-highest term; a new cluster starts where every remaining term lies more than
// 32N + ceil(log2(count+1)) + 4 bits below the current cluster's lowest bit, linalg.hpp:269-273),
// keeps the first nonzero cluster sum S exactly and only the sign of the next nonzero cluster, and
// rounds S once.  It serves every input (any exponent spread, statuses, zeros) and is the plain
// limb-kernel baseline of the residue/CRT engine (lf_residue.cu), which must match it bit for bit.
#pragma once
#include "lf_arith.cuh"
#include <cuda_runtime.h>

namespace lfd {

struct LineView { const u32* base; u64 ls, ks; };
struct LineInfo { u32 status; int top; int bottom; u32 nonzero; };

// One warp per line: OR of statuses, largest and smallest exponent of the nonzero, status-free
// entries (linalg.mm:82-112 pass 1).
template <int N> __global__ void analyze_kernel(LineView v, u64 lines, u64 K, LineInfo* out) {
    const u64 line = (u64)blockIdx.x * (blockDim.x / 32) + threadIdx.x / 32;
    const int lane = threadIdx.x & 31;
    if (line >= lines) return;
    constexpr u64 E = N + 3;
    u32 st = 0, nz = 0;
    int top = INT_MIN, bottom = INT_MAX;
    for (u64 k = lane; k < K; k += 32) {
        const u32* p = v.base + (line * v.ls + k * v.ks) * E;
        const u32 s = __ldg(p + N + 2);
        const int sg = (int)__ldg(p + N + 1), e = (int)__ldg(p + N);
        st |= s;
        if (!s && sg) { nz += 1; top = max(top, e); bottom = min(bottom, e); }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        st |= __shfl_xor_sync(0xffffffffu, st, o);
        nz += __shfl_xor_sync(0xffffffffu, nz, o);
        top = max(top, __shfl_xor_sync(0xffffffffu, top, o));
        bottom = min(bottom, __shfl_xor_sync(0xffffffffu, bottom, o));
    }
    if (!lane) out[line] = LineInfo{st, top, bottom, nz};
}

// Plan of a product whose engine is chosen on the GPU (resident products): mode 1 runs the residue
// engine with the modulus count L and the tables of that count, mode 0 the generic limb kernel.
struct ResPlan {
    int mode, G;
    int L, qwords, NB, Kp, NS; u32 tmem_cols;        // CRT operand of L
    int dNB; u32 dtmem;                               // digit operand of L
    const void* tab; const unsigned char* crt_bimg; const unsigned char* dig_bimg;
};

struct DotParams {
    LineView left, right;
    const LineInfo* linfo; const LineInfo* rinfo;
    u32* C; u64 ldc;                 // output element (i, j) at C + (i * ldc + j) * E
    u64 M, Nc, K;
    u64 row0, col0;                  // output offsets of this launch (tiles of a larger product)
    int subtract, lower;             // lower: only j <= i (global indices i = row0 + r, j = col0 + c)
    u32* error;                      // set to 1 when a cluster exceeds the accumulator
    const ResPlan* plan;             // planned on the GPU: nothing to do when the plan chose the residue engine
};

constexpr int kClusterWords = 192;   // 6144-bit exact window per cluster (pos/neg magnitudes)

// RN(c -/+ sum_{k<K} x[k*sx] y[k*sy]) with one rounding, c == nullptr a zero addend: the contract
// of exact_dot_add (linalg.hpp:268-318).  Statuses: zero carrying the OR of c's and every x[k],
// y[k] status; no nonzero product returns c itself (or zero).  `error` is set when one cluster
// is wider than kClusterWords words (the result is then zero with status invalid).
// RO: the operands are read-only for the whole kernel (read-only cache loads); kernels that write
// entries they read later (the factorization panels and solves) use RO = false, coherent loads.
template <bool RO> __device__ __forceinline__ u32 ldw(const u32* p) { if constexpr (RO) return __ldg(p); else return *(volatile const u32*)p; }
template <int N, bool RO> __device__ __forceinline__ Num<N> ldn(const u32* p) {
    Num<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.m[i] = ldw<RO>(p + i);
    r.e = (int)ldw<RO>(p + N); r.s = (int)ldw<RO>(p + N + 1); r.st = ldw<RO>(p + N + 2);
    return r;
}
// Terms of one output as a source for cluster_round: slot k < K is the product x_k y_k (top bound
// scale + 64N), slot K the addend c (top scale + 32N).
template <int N, bool RO> struct LineTerms {
    const u32* x; i64 sx; const u32* y; i64 sy; u64 K; bool subtract; Num<N> c;
    __device__ u64 count() const { return K + 1; }
    __device__ bool term(u64 k, i64& scale, i64& top, int& sign) const {
        constexpr i64 E = N + 3;
        if (k == K) {
            if (!c.s) return false;
            scale = (i64)c.e - (32 * N - 1); top = scale + 32 * N; sign = c.s;
            return true;
        }
        const u32* a = x + (i64)k * sx * E; const u32* b = y + (i64)k * sy * E;
        const int sa = (int)ldw<RO>(a + N + 1), sb = (int)ldw<RO>(b + N + 1);
        if (!sa || !sb) return false;
        scale = (i64)(int)ldw<RO>(a + N) + (int)ldw<RO>(b + N) - 2 * (32 * N - 1);
        top = scale + 64 * N;
        sign = subtract ? -sa * sb : sa * sb;
        return true;
    }
    __device__ void add(u64 k, u32* acc, int len, i64 off) const {
        constexpr i64 E = N + 3;
        if (k == K) { acc_add(acc, len, c.m, N, off); return; }
        const Num<N> a = ldn<N, RO>(x + (i64)k * sx * E), b = ldn<N, RO>(y + (i64)k * sy * E);
        u32 prod[2 * N];
        mant_mul<N>(a.m, b.m, prod);
        acc_add(acc, len, prod, 2 * N, off);
    }
};
template <int N, bool RO = true> __device__ __noinline__ Num<N> exact_dot_add_dev(const u32* cp, bool subtract, const u32* x, i64 sx, const u32* y, i64 sy,
                                                     u64 K, u32* error) {
    constexpr i64 E = N + 3;
    const Num<N> c = cp ? load_plain<N>(cp) : zero<N>();
    u32 st = c.st;
    for (u64 k = 0; k < K; ++k) st |= ldw<RO>(x + (i64)k * sx * E + N + 2) | ldw<RO>(y + (i64)k * sy * E + N + 2);
    if (st) return zero<N>(st);
    bool products = false;
    for (u64 k = 0; k < K && !products; ++k)
        products = ldw<RO>(x + (i64)k * sx * E + N + 1) && ldw<RO>(y + (i64)k * sy * E + N + 1);
    if (!products) return cp ? c : zero<N>();
    const LineTerms<N, RO> src{x, sx, y, sy, K, subtract, c};
    return cluster_round<N, kClusterWords>(src, error);
}

template <int N> __global__ void __launch_bounds__(128) exact_dot_kernel(DotParams p) {
    if (p.plan && p.plan->mode == 1) return;
    const u64 r = (u64)blockIdx.y * blockDim.y + threadIdx.y;
    const u64 q = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (r >= p.M || q >= p.Nc) return;
    const u64 i = p.row0 + r, j = p.col0 + q;
    if (p.lower && j > i) return;
    constexpr u64 E = N + 3;
    u32* out = p.C + (r * p.ldc + q) * E;
    const Num<N> v = exact_dot_add_dev<N>(p.subtract ? out : nullptr, p.subtract, p.left.base + i * p.left.ls * E, (i64)p.left.ks,
                                          p.right.base + j * p.right.ls * E, (i64)p.right.ks, p.K, p.error);
    store<N>(out, v);
}

// Lower triangle mirrored into the upper one (full SYRK output).
template <int N> __global__ void mirror_kernel(u32* C, u64 n, u64 ldc) {
    const u64 i = (u64)blockIdx.y * blockDim.y + threadIdx.y, j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || j >= n || j <= i) return;
    constexpr u64 E = N + 3;
    const u32* src = C + (j * ldc + i) * E;
    u32* dst = C + (i * ldc + j) * E;
    for (int w = 0; w < (int)E; ++w) dst[w] = src[w];
}

typedef void (*AnalyzeFn)(LineView, u64, u64, LineInfo*, cudaStream_t);
typedef void (*DotFn)(const DotParams&, cudaStream_t);
typedef void (*MirrorFn)(u32*, u64, u64, cudaStream_t);
struct LinalgKernels { AnalyzeFn analyze; DotFn dot; MirrorFn mirror; };
const LinalgKernels* linalg_kernels(int limbs);

template <int N> void analyze_launch(LineView v, u64 lines, u64 K, LineInfo* out, cudaStream_t s) {
    if (!lines) return;
    analyze_kernel<N><<<(unsigned)((lines + 3) / 4), 128, 0, s>>>(v, lines, K, out);
}
template <int N> void dot_launch(const DotParams& p, cudaStream_t s) {
    if (!p.M || !p.Nc) return;
    dim3 block(32, 4), grid((unsigned)((p.Nc + 31) / 32), (unsigned)((p.M + 3) / 4));
    exact_dot_kernel<N><<<grid, block, 0, s>>>(p);
}
template <int N> void mirror_launch(u32* C, u64 n, u64 ldc, cudaStream_t s) {
    if (n < 2) return;
    dim3 block(32, 4), grid((unsigned)((n + 31) / 32), (unsigned)((n + 3) / 4));
    mirror_kernel<N><<<grid, block, 0, s>>>(C, n, ldc);
}

}  // namespace lfd

#define LF_LINALG_INSTANTIATE(N)                                                                      \
    namespace lfd {                                                                                   \
    extern const LinalgKernels linalg_kernels_##N; const LinalgKernels linalg_kernels_##N = {analyze_launch<N>, dot_launch<N>, mirror_launch<N>};    \
    }

namespace lfd {

// ---------------------------------------------------------------- warp-cooperative exact dot
// exact_dot_add with the terms spread over the 32 lanes of a warp (k = lane, lane + 32, ...).  When
// every nonzero term and the addend fit one two's-complement window of W = 2N + 10 words
// (64N + 320 bits: products of the same magnitude class, as in factorization panels), each lane sums
// its terms exactly in the window (the addend goes to lane K mod 32, which has one term fewer when K is
// not a multiple of 32), the warp adds the windows exactly and rounds once: with shared rows (srow, from
// the caller's dynamic shared memory) by warp_round_window, otherwise by a shuffle tree and lane 0.  A
// spread too wide for the window takes the generic cluster routine on lane 0.  Every lane receives the
// result.
template <int N> __device__ __forceinline__ Num<N> warp_broadcast(const Num<N>& v) {
    Num<N> r;
#pragma unroll
    for (int i = 0; i < N; ++i) r.m[i] = __shfl_sync(0xffffffffu, v.m[i], 0);
    r.e = __shfl_sync(0xffffffffu, v.e, 0); r.s = __shfl_sync(0xffffffffu, v.s, 0); r.st = __shfl_sync(0xffffffffu, v.st, 0);
    return r;
}
// Shared memory of the window reduction: one row of dot_row_words words per lane (odd stride: the row
// writes and the column reads are free of bank conflicts).
template <int N> __host__ __device__ constexpr int dot_row_words() { return (2 * N + 10) | 1; }
template <int N> __host__ __device__ constexpr size_t dot_smem_bytes(int warps) { return (size_t)warps * 32 * dot_row_words<N>() * 4; }

// RN(T * 2^lo) for T = sum_w S_w 2^(32w) mod 2^(32W), lane l holding the column sums S_{l+32r} as v[r] (low word)
// and hi[r] (high word); every lane of the warp returns the result.  keep (optional): the resolved two's-complement
// words T_w go to keep[w] before the rounding.
template <int N, int W> __device__ __forceinline__ Num<N> warp_round_columns(u32 (&v)[(W + 31) / 32], const u32 (&hi)[(W + 31) / 32],
                                                                            i64 lo, u32* keep);
// RN(T * 2^lo) for T the sum, mod 2^(32W), of the 32 lanes' two's-complement windows, computed by the whole
// warp; every lane returns the result.  The windows go to shared memory (srow: 32 rows) and lane l sums
// column l (+32, +64) over the rows; the column sums' high parts and the carries between columns are
// resolved with ballots (carries c = ((G|P) + G) ^ (G|P) ^ G for generate G and propagate P); the sign,
// the magnitude, the top word and the round and sticky bits follow with ballots and shuffles.  The
// bits equal those of round_general on the summed window.
template <int N, int W> __device__ __forceinline__ Num<N> warp_round_window(const u32 (&acc)[W], i64 lo, u32* srow) {
    constexpr int WP = dot_row_words<N>();
    static_assert(WP >= W, "row shorter than the window");
    constexpr int R = (W + 31) / 32;
    constexpr u32 FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    u32* row = srow + lane * WP;
#pragma unroll
    for (int w = 0; w < W; ++w) row[w] = acc[w];
    __syncwarp();
    u32 v[R], hi[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int w = lane + 32 * r;
        u64 s0 = 0, s1 = 0;
        if (w < W) {
#pragma unroll
            for (int l = 0; l < 32; l += 2) { s0 += srow[l * WP + w]; s1 += srow[(l + 1) * WP + w]; }
        }
        const u64 sum = s0 + s1;
        v[r] = (u32)sum; hi[r] = (u32)(sum >> 32);
    }
    __syncwarp();                                            // the rows may be rewritten by the next call
    return warp_round_columns<N, W>(v, hi, lo, nullptr);
}
template <int N, int W> __device__ __forceinline__ Num<N> warp_round_columns(u32 (&v)[(W + 31) / 32], const u32 (&hi)[(W + 31) / 32],
                                                                            i64 lo, u32* keep) {
    constexpr int R = (W + 31) / 32;
    constexpr u32 FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    u32 G[R], P[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {                            // u_w = low(S_w) + high(S_{w-1})
        u32 hp = __shfl_up_sync(FULL, hi[r], 1);
        const u32 hl = r ? __shfl_sync(FULL, hi[r ? r - 1 : 0], 31) : 0u;
        if (lane == 0) hp = hl;
        const u64 u = (u64)v[r] + hp;
        const bool valid = lane + 32 * r < W;
        v[r] = valid ? (u32)u : 0u;
        G[r] = __ballot_sync(FULL, valid && (u >> 32));
        P[r] = __ballot_sync(FULL, valid && (u32)u == FULL);
    }
    u32 cy = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const u32 X = G[r] | P[r];
        const u64 sum = (u64)X + G[r] + cy;
        const u32 Cm = (u32)sum ^ X ^ G[r];                  // carry into each column of this round
        cy = (u32)(sum >> 32);
        if (lane + 32 * r < W) v[r] += (Cm >> lane) & 1u;     // the carry out of the window is dropped (mod 2^(32W))
    }
    if (keep)
#pragma unroll
        for (int r = 0; r < R; ++r)
            if (lane + 32 * r < W) keep[lane + 32 * r] = v[r];
    constexpr int RT = (W - 1) / 32, LT = (W - 1) % 32;
    const bool neg = __shfl_sync(FULL, v[RT], LT) >> 31;
    if (neg) {                                               // magnitude: ~T + 1
        bool zero_below = true;
        const u32 lowmask = (1u << lane) - 1u;
#pragma unroll
        for (int r = 0; r < R; ++r) {
            const bool valid = lane + 32 * r < W;
            const u32 Z = __ballot_sync(FULL, !valid || v[r] == 0);
            const bool cin = zero_below && (Z & lowmask) == lowmask;
            v[r] = valid ? ~v[r] + (cin ? 1u : 0u) : 0u;
            zero_below = zero_below && Z == FULL;
        }
    }
    int top = -1;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const u32 T = __ballot_sync(FULL, v[r] != 0);
        if (T) top = 32 * r + 31 - __clz(T);
    }
    if (top < 0) return zero<N>();
    u32 vt = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) vt = (r == (top >> 5)) ? v[r] : vt;
    vt = __shfl_sync(FULL, vt, top & 31);
    const int lz = __clz(vt);
    u32 sh[R];
#pragma unroll
    for (int r = 0; r < R; ++r) {                            // sh_w = high word of (a_w : a_{w-1}) << lz
        u32 pv = __shfl_up_sync(FULL, v[r], 1);
        const u32 pl = r ? __shfl_sync(FULL, v[r ? r - 1 : 0], 31) : 0u;
        if (lane == 0) pv = pl;
        sh[r] = __funnelshift_l(pv, v[r], lz);
    }
    const int c = top - N;                                   // column whose top bit is the round bit
    bool any = false;
#pragma unroll
    for (int r = 0; r < R; ++r) {
        const int w = lane + 32 * r;
        const u32 part = w < c - 1 ? v[r] : w == c - 1 ? (v[r] << lz) : w == c ? (sh[r] & 0x7fffffffu) : 0u;
        any = any || part != 0;
    }
    const bool sticky = __any_sync(FULL, any);
    u32 rbw = 0;
#pragma unroll
    for (int r = 0; r < R; ++r) rbw = (r == (c >> 5)) ? sh[r] : rbw;
    rbw = __shfl_sync(FULL, rbw, c & 31);
    const bool rb = c >= 0 && (rbw >> 31);
    u32 m[N];
#pragma unroll
    for (int i = 0; i < N; ++i) {
        const int col = c + 1 + i;
        u32 x = 0;
#pragma unroll
        for (int r = 0; r < R; ++r) x = (r == (col >> 5)) ? sh[r] : x;
        x = __shfl_sync(FULL, x, col & 31);
        m[i] = col >= 0 ? x : 0u;
    }
    return finish<N>(m, lo + 32 * (i64)top + 31 - lz, neg ? -1 : 1, rb && (sticky || (m[0] & 1u)), 0);
}

template <int N, bool RO> __device__ __noinline__ Num<N> warp_exact_dot(const u32* cp, bool subtract, const u32* x, i64 sx, const u32* y, i64 sy,
                                                          u64 K, u32* error, u32* srow = nullptr) {
    constexpr int W = 2 * N + 10;
    constexpr i64 E = N + 3;
    const int lane = threadIdx.x & 31;
    const Num<N> c = cp ? ldn<N, RO>(cp) : zero<N>();
    u32 st = 0; int cnt = 0;
    i64 lo = INT64_MAX, hi = INT64_MIN;
    for (u64 k = lane; k < K; k += 32) {
        const u32* a = x + (i64)k * sx * E; const u32* b = y + (i64)k * sy * E;
        st |= ldw<RO>(a + N + 2) | ldw<RO>(b + N + 2);
        const int sa = (int)ldw<RO>(a + N + 1), sb = (int)ldw<RO>(b + N + 1);
        if (sa && sb) {
            const i64 s = (i64)(int)ldw<RO>(a + N) + (int)ldw<RO>(b + N) - 2 * (32 * N - 1);
            lo = s < lo ? s : lo; hi = s + 64 * N > hi ? s + 64 * N : hi; ++cnt;
        }
    }
#pragma unroll
    for (int o = 16; o; o >>= 1) {
        st |= __shfl_xor_sync(0xffffffffu, st, o);
        cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
        const i64 l2 = __shfl_xor_sync(0xffffffffu, lo, o), h2 = __shfl_xor_sync(0xffffffffu, hi, o);
        lo = l2 < lo ? l2 : lo; hi = h2 > hi ? h2 : hi;
    }
    st |= c.st;
    if (st) return zero<N>(st);
    if (!cnt) return cp ? c : zero<N>();
    if (c.s) {
        const i64 sc = (i64)c.e - (32 * N - 1);
        lo = sc < lo ? sc : lo; hi = (i64)c.e + 1 > hi ? (i64)c.e + 1 : hi;
    }
    int logc = 0;
    while ((1 << logc) < cnt + 2) ++logc;
    if (hi - lo + logc + 1 >= 32 * (i64)W) {
        Num<N> r = zero<N>();
        if (lane == 0) r = exact_dot_add_dev<N, RO>(cp, subtract, x, sx, y, sy, K, error);
        return warp_broadcast<N>(r);
    }
    u32 acc[W];
#pragma unroll
    for (int w = 0; w < W; ++w) acc[w] = 0;
    for (u64 k = lane; k < K; k += 32) {
        const Num<N> a = ldn<N, RO>(x + (i64)k * sx * E), b = ldn<N, RO>(y + (i64)k * sy * E);
        if (!a.s || !b.s) continue;
        u32 p[2 * N], t[W];
        mant_mul<N>(a.m, b.m, p);
        place_words<W, 2 * N>(t, p, (i64)a.e + b.e - 2 * (32 * N - 1) - lo);
        accumulate<W>(acc, t, (subtract ? -a.s * b.s : a.s * b.s) < 0);
    }
    if (lane == (int)(K % 32) && c.s) {                     // the addend goes to a lane with one term fewer
        u32 t[W];
        place_words<W, N>(t, c.m, (i64)c.e - (32 * N - 1) - lo);
        accumulate<W>(acc, t, c.s < 0);
    }
    if (srow) return warp_round_window<N, W>(acc, lo, srow);
#pragma unroll 1
    for (int o = 16; o; o >>= 1) {
        u32 other[W];
#pragma unroll
        for (int w = 0; w < W; ++w) other[w] = __shfl_down_sync(0xffffffffu, acc[w], o);
        accumulate<W>(acc, other, false);
    }
    Num<N> r = zero<N>();
    if (lane == 0) {
        int sign = 1;
        if (acc[W - 1] >> 31) {
            sign = -1; u64 cy = 1;
#pragma unroll
            for (int w = 0; w < W; ++w) { u64 v = (u64)(u32)~acc[w] + cy; acc[w] = (u32)v; cy = v >> 32; }
        }
        r = round_general<N, W>(acc, lo, sign, 0);
    }
    return warp_broadcast<N>(r);
}

// ---------------------------------------------------------------- blocked Cholesky pieces
// W: n x n row-major work matrix (element stride E).  D(c; x, y; K) = RN(c - sum x_k y_k), one rounding.
struct CholParams { u32* W; u64 n, k0, k1; long long* info; u32* error; };
constexpr u64 kRecips = 32;       // pivot reciprocals a panel-row or solve block keeps in shared memory

// Diagonal block [k0, k1) column by column: s_jj = D(w_jj; row j [k0,j)), l_jj = sqrt(s_jj) (or the
// failing pivot recorded in info = {pivot, sign, status}); l_ij = RN(D(w_ij; row i, row j; [k0,j)) / l_jj)
// for the block rows i > j.  The same formulas in the same dependency order as the row-by-row host
// panel of linalg.mm:418-430, so every entry gets identical bits.  For each column every dot product
// (the diagonal's and the rows') runs at once, one warp each, and D is parked in w_ij; the square
// root follows on the diagonal's warp, then one thread per row divides.  After a failure the column's
// parked values are overwritten with invalid zeros by chol_prepare_kernel.
template <int N> constexpr int diag_threads() { return N <= 8 ? 512 : N <= 16 ? 256 : 128; }   // registers per thread
template <int N> __global__ void __launch_bounds__(diag_threads<N>()) chol_diag_kernel(CholParams p) {
    constexpr u64 E = N + 3;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    extern __shared__ u32 dot_rows[];
    u32* srow = dot_rows + warp * 32 * dot_row_words<N>();
    __shared__ int failed;
    if (!threadIdx.x) failed = 0;
    __syncthreads();
    for (u64 j = p.k0; j < p.k1; ++j) {
        u32* wjj = p.W + (j * p.n + j) * E;
        for (u64 u = warp; u < p.k1 - j; u += nw) {                 // u = 0: the diagonal, u > 0: row j + u
            const u64 i = j + u;
            u32* wij = p.W + (i * p.n + j) * E;
            const Num<N> v = warp_exact_dot<N, false>(wij, true, p.W + (i * p.n + p.k0) * E, 1, p.W + (j * p.n + p.k0) * E, 1, j - p.k0, p.error,
                                                      srow);
            if (lane == 0) {
                if (u) store<N>(wij, v);
                else if (v.st || v.s <= 0) { p.info[0] = (long long)j; p.info[1] = v.st ? 0 : v.s; p.info[2] = v.st; failed = 1; }
                else store<N>(wjj, lfd::sqrt<N>(v));
            }
        }
        __syncthreads();
        if (failed) return;
        for (u64 i = j + 1 + threadIdx.x; i < p.k1; i += blockDim.x) {
            u32* wij = p.W + (i * p.n + j) * E;
            store<N>(wij, div<N>(ldn<N, false>(wij), ldn<N, false>(wjj)));
        }
        __syncthreads();
    }
}
// Rows i in [r0, n) below the diagonal block: l_ij = RN(D(w_ij; row i, row j; [k0,j)) / l_jj) for
// j in [k0, jend), left to right (jend = the failing pivot, or k1).  One warp per row.
// The block first forms the reciprocals of its first kRecips pivots l_jj in shared memory, one per thread,
// and divides through them (div_by: the bits of div); later columns of a wider block use div.
template <int N> __global__ void __launch_bounds__(128) chol_rows_kernel(CholParams p, u64 r0, u64 jend) {
    constexpr u64 E = N + 3, ER = N + 4;
    const u64 i = r0 + ((u64)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    extern __shared__ u32 dot_rows[];
    u32* srow = dot_rows + (threadIdx.x >> 5) * 32 * dot_row_words<N>();
    u32* srec = dot_rows + (blockDim.x >> 5) * 32 * dot_row_words<N>();
    if (threadIdx.x < jend - p.k0 && threadIdx.x < kRecips) {
        const u64 j = p.k0 + threadIdx.x;
        store<N + 1>(srec + threadIdx.x * ER, reciprocal<N>(ldn<N, false>(p.W + (j * p.n + j) * E)));
    }
    __syncthreads();
    if (i >= p.n) return;
    for (u64 j = p.k0; j < jend; ++j) {
        u32* wij = p.W + (i * p.n + j) * E;
        const Num<N> v = warp_exact_dot<N, false>(wij, true, p.W + (i * p.n + p.k0) * E, 1, p.W + (j * p.n + p.k0) * E, 1, j - p.k0, p.error,
                                                  srow);
        if (lane == 0) {
            const Num<N> ljj = ldn<N, false>(p.W + (j * p.n + j) * E);
            store<N>(wij, j - p.k0 < kRecips ? div_by<N>(v, ljj, load_plain<N + 1>(srec + (j - p.k0) * ER)) : div<N>(v, ljj));
        }
        __syncwarp();
    }
}
// W = lower triangle of A (upper zero); after a failure at pivot p: entries (i, j), p <= j <= i, are
// zero with status invalid.
template <int N> __global__ void chol_prepare_kernel(const u32* A, u32* W, u64 n, u64 fail) {
    constexpr u64 E = N + 3;
    const u64 i = (u64)blockIdx.y * blockDim.y + threadIdx.y, j = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n || j >= n) return;
    u32* w = W + (i * n + j) * E;
    if (fail < n) {
        if (j >= fail && j <= i) store<N>(w, zero<N>(kInvalid));
        return;
    }
    if (j > i) store<N>(w, zero<N>());
    else if (A != W) { const u32* a = A + (i * n + j) * E; for (int q = 0; q < (int)E; ++q) w[q] = a[q]; }
}

// ---------------------------------------------------------------- triangular solves (linalg.mm:459-488)
// X: n x nrhs, L: n x n lower.  Forward block [r0, r1): x_i = RN(D(x_i; l_i[r0,i), x[r0,i)) / l_ii),
// i ascending; backward block: x_i = RN(D(x_i; column i of L below i within (i, r1), x(i, r1)) / l_ii),
// i descending (upper: R = L^T stored by rows).  One thread per right-hand side.
struct SolveParams { const u32* L; u32* X; u64 n, nrhs, r0, r1; int upper; u32* error; };
// Reciprocals of the block's first kRecips diagonal entries l_ii, i in [r0, r1), in shared memory: one per
// thread, before any thread leaves.  Rows beyond them divide with div.
template <int N> __device__ __forceinline__ void solve_reciprocals(const SolveParams& p, u32* srec) {
    constexpr u64 E = N + 3;
    if (threadIdx.x < p.r1 - p.r0 && threadIdx.x < kRecips) {
        const u64 i = p.r0 + threadIdx.x;
        store<N + 1>(srec + threadIdx.x * (N + 4), reciprocal<N>(ldn<N, false>(p.L + (i * p.n + i) * E)));
    }
    __syncthreads();
}
template <int N> __device__ __forceinline__ Num<N> solve_divide(const SolveParams& p, const Num<N>& v, u64 i, const u32* srec) {
    const Num<N> lii = ldn<N, false>(p.L + (i * p.n + i) * (N + 3));
    return i - p.r0 < kRecips ? div_by<N>(v, lii, load_plain<N + 1>(srec + (i - p.r0) * (N + 4))) : div<N>(v, lii);
}
// One warp per right-hand side.
template <int N> __global__ void __launch_bounds__(128) solve_forward_kernel(SolveParams p) {
    constexpr u64 E = N + 3;
    const u64 c = ((u64)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    extern __shared__ u32 dot_rows[];
    u32* srow = dot_rows + (threadIdx.x >> 5) * 32 * dot_row_words<N>();
    u32* srec = dot_rows + (blockDim.x >> 5) * 32 * dot_row_words<N>();
    solve_reciprocals<N>(p, srec);
    if (c >= p.nrhs) return;
    for (u64 i = p.r0; i < p.r1; ++i) {
        u32* x = p.X + (i * p.nrhs + c) * E;
        const Num<N> v = warp_exact_dot<N, false>(x, true, p.L + (i * p.n + p.r0) * E, 1, p.X + (p.r0 * p.nrhs + c) * E, (i64)p.nrhs, i - p.r0, p.error,
                                                  srow);
        if (lane == 0) store<N>(x, solve_divide<N>(p, v, i, srec));
        __syncwarp();
    }
}
template <int N> __global__ void __launch_bounds__(128) solve_backward_kernel(SolveParams p) {
    constexpr u64 E = N + 3;
    const u64 c = ((u64)blockIdx.x * blockDim.x + threadIdx.x) / 32;
    const int lane = threadIdx.x & 31;
    extern __shared__ u32 dot_rows[];
    u32* srow = dot_rows + (threadIdx.x >> 5) * 32 * dot_row_words<N>();
    u32* srec = dot_rows + (blockDim.x >> 5) * 32 * dot_row_words<N>();
    solve_reciprocals<N>(p, srec);
    if (c >= p.nrhs) return;
    for (u64 i = p.r1; i-- > p.r0;) {
        u32* x = p.X + (i * p.nrhs + c) * E;
        Num<N> v;
        if (i + 1 < p.r1) {
            const u32* col = p.upper ? p.L + (i * p.n + i + 1) * E : p.L + ((i + 1) * p.n + i) * E;
            v = warp_exact_dot<N, false>(x, true, col, p.upper ? 1 : (i64)p.n, p.X + ((i + 1) * p.nrhs + c) * E, (i64)p.nrhs, p.r1 - i - 1, p.error,
                                         srow);
        } else {
            v = ldn<N, false>(x);
        }
        if (lane == 0) store<N>(x, solve_divide<N>(p, v, i, srec));
        __syncwarp();
    }
}

typedef void (*CholDiagFn)(const CholParams&, cudaStream_t);
typedef void (*CholRowsFn)(const CholParams&, u64, u64, cudaStream_t);
typedef void (*CholPrepFn)(const u32*, u32*, u64, u64, cudaStream_t);
typedef void (*SolveFn)(const SolveParams&, bool, cudaStream_t);
struct FactorKernels { CholDiagFn diag; CholRowsFn rows; CholPrepFn prep; SolveFn solve; };
const FactorKernels* factor_kernels(int limbs);

template <int N> void chol_diag_launch(const CholParams& p, cudaStream_t s) {
    const size_t smem = dot_smem_bytes<N>(diag_threads<N>() / 32);
    cudaFuncSetAttribute(chol_diag_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    chol_diag_kernel<N><<<1, diag_threads<N>(), smem, s>>>(p);
}
template <int N> void chol_rows_launch(const CholParams& p, u64 r0, u64 jend, cudaStream_t s) {
    if (r0 >= p.n || jend <= p.k0) return;
    const u64 rows = p.n - r0;
    chol_rows_kernel<N><<<(unsigned)((rows + 3) / 4), 128, dot_smem_bytes<N>(4) + kRecips * (N + 4) * 4, s>>>(p, r0, jend);
}
template <int N> void chol_prep_launch(const u32* A, u32* W, u64 n, u64 fail, cudaStream_t s) {
    if (!n) return;
    dim3 block(32, 4), grid((unsigned)((n + 31) / 32), (unsigned)((n + 3) / 4));
    chol_prepare_kernel<N><<<grid, block, 0, s>>>(A, W, n, fail);
}
template <int N> void solve_launch(const SolveParams& p, bool forward, cudaStream_t s) {
    if (!p.nrhs || p.r1 <= p.r0) return;
    const unsigned blocks = (unsigned)((p.nrhs + 3) / 4);
    const size_t smem = dot_smem_bytes<N>(4) + kRecips * (N + 4) * 4;
    if (forward) solve_forward_kernel<N><<<blocks, 128, smem, s>>>(p);
    else solve_backward_kernel<N><<<blocks, 128, smem, s>>>(p);
}

}  // namespace lfd

#define LF_FACTOR_INSTANTIATE(N)                                                                               \
    namespace lfd {                                                                                            \
    extern const FactorKernels factor_kernels_##N; const FactorKernels factor_kernels_##N = {chol_diag_launch<N>, chol_rows_launch<N>, chol_prep_launch<N>, solve_launch<N>}; \
    }
