// Int8-residue / CRT exact products (the reference's plan D6, linalg.mm:305-404 and
// linalg.metal:23-152, redesigned for sm_100a):
//
//  1. digits: every entry of a line becomes the exact integer X = mantissa * 2^(e - bottom(line))
//     (< 2^(32N+G), G = widest line spread), reduced modulo L primes m_l < 2^16 to a balanced
//     residue r = 256 d1 + d0 with int8 digits; planes D1/D0 [L][rows][Kp] (K-major, zero padded).
//  2. mma: per modulus and 128x128 output tile, tcgen05.mma kind::i8 with int32 accumulators in
//     TMEM: S11 = D1a D1b^T, S00 = D0a D0b^T, Smid = D1a D0b^T + D0a D1b^T; operands fed by TMA
//     (128-byte swizzle, no multicast); epilogue r = (65536 S11 + 256 Smid + S00) mod m -> uint16.
//  3. reconstruct: per output, CRT of the L residues (X = sum_l t_l (M/m_l) - q M, q = round of the
//     fixed-point sum of t_l/m_l; the modulus product exceeds 4 max|X| so the rounding of q is never
//     close), then RN(c - X 2^scale) (or RN(X 2^scale)) with one rounding.
// Every step is exact integer arithmetic, so the outputs equal the generic limb kernel's bit for bit.
#pragma once
#include "lf_linalg.cuh"
#include <cuda.h>

namespace lfd {

constexpr int kResMaxModuli = 160;
constexpr int kResMaxQWords = 80;          // words of M / m_l
struct ResTables {
    u32 m[kResMaxModuli];                  // moduli, descending primes < 2^16
    u64 barrett[kResMaxModuli];            // floor(2^64 / m)
    u32 w[kResMaxModuli];                  // (M / m_l)^{-1} mod m_l
    u64 frac[kResMaxModuli];               // floor(2^48 / m_l)
    u32 q[kResMaxModuli][kResMaxQWords];   // M / m_l, little-endian words
    u32 M[kResMaxQWords + 1];              // product of the moduli
    u32 pw[kResMaxModuli][40];             // 2^(32 w) mod m_l for the integer words (<= 40)
};

__device__ __forceinline__ u32 mod_barrett(u64 x, u32 m, u64 r) {
    u64 q = __umul64hi(x, r);
    u64 t = x - q * m;
    while (t >= m) t -= m;                 // at most twice
    return (u32)t;
}

// ---------------------------------------------------------------- 1. digit planes
struct DigitParams {
    LineView v; u64 lines, K, Kp, rows_pad; int L; int xwords;
    const LineInfo* info; const ResTables* tab;
    signed char* d1; signed char* d0;      // [L][rows_pad][Kp]
};
template <int N> __global__ void __launch_bounds__(128) digits_kernel(DigitParams p) {
    const u64 k = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    const u64 line = blockIdx.y;                          // rows_pad lines: padding rows are zero
    if (k >= p.Kp || line >= p.rows_pad) return;
    u32 x[40];
    for (int w = 0; w < 40; ++w) x[w] = 0;
    bool nz = false, negative = false;
    if (k < p.K && line < p.lines) {
        const Num<N> a = load<N>(p.v.base + (line * p.v.ls + k * p.v.ks) * (u64)(N + 3));
        if (!a.st && a.s) {
            nz = true; negative = a.s < 0;
            const int sh = a.e - p.info[line].bottom;       // 0 <= sh <= G
            const int ws = sh >> 5, bs = sh & 31;
            for (int i = 0; i <= N; ++i) {
                u32 v = i < N ? a.m[i] << bs : 0u;
                if (bs && i > 0) v |= a.m[i - 1] >> (32 - bs);
                x[i + ws] = v;
            }
        }
    }
    const u64 plane = p.rows_pad * p.Kp;
    for (int l = 0; l < p.L; ++l) {
        int r = 0;
        if (nz) {
            const u32 m = p.tab->m[l];
            u64 acc = 0;
            for (int w = 0; w < p.xwords; ++w) acc += (u64)x[w] * p.tab->pw[l][w];     // < 2^54
            u32 u = mod_barrett(acc, m, p.tab->barrett[l]);
            if (negative && u) u = m - u;                     // residue of -X
            r = (int)u;
            if (r > (int)(m >> 1)) r -= (int)m;               // balanced: |r| <= (m-1)/2 <= 32639
        }
        const int lo = (int)(signed char)(r & 0xff);
        const int hi = (r - lo) >> 8;                         // in [-128, 127] because m <= 65279
        p.d1[l * plane + line * p.Kp + k] = (signed char)hi;
        p.d0[l * plane + line * p.Kp + k] = (signed char)lo;
    }
}

// ---------------------------------------------------------------- 2. tcgen05 residue products
constexpr int kTileM = 128, kTileN = 128, kTileK = 128;      // K tile in int8 elements = one 128-byte row
constexpr int kStages = 3;                                    // 3 x 64 KB of operand tiles (of 227 KB shared)
constexpr int kTileBytes = kTileM * kTileK;                   // 16 KB per operand tile
constexpr int kStageBytes = 4 * kTileBytes;                   // D1a, D0a, D1b, D0b
constexpr u32 kSpinLimit = 1u << 28;                          // bounded mbarrier waits
constexpr int kMmaThreads = 256;                              // warps w and w + 4 share TMEM lanes 32 (w % 4) ..
constexpr int kDigitThreads = 256;                            // digit planes: the same lane sharing
constexpr int kCrtThreads = 256;                              // CRT column sums: the same lane sharing

struct MmaParams {
    u16* res;                               // [L][M][Nc] residues (0 <= r < m)
    const ResTables* tab;
    u64 M, Nc, Kp;
    int lower;                              // skip tiles strictly above the diagonal (SYRK)
    u32* error;
    const ResPlan* plan;                    // planned on the GPU: moduli at or above plan->L have no work
    u32 poll_limit;                         // polls of a barrier wait before it gives up (0: kSpinLimit)
    int no_loads;                           // failure test only: the producer issues no loads, so the first wait runs out
};

__device__ __forceinline__ u32 smem_u32(const void* p) { return (u32)__cvta_generic_to_shared(p); }
__device__ __forceinline__ void mbar_init(u64* bar, u32 count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" :: "r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ void mbar_expect_tx(u64* bar, u32 bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" :: "r"(smem_u32(bar)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(u64* bar, u32 phase) {
    u32 ok;
    asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(ok) : "r"(smem_u32(bar)), "r"(phase) : "memory");
    return ok != 0;
}
// Bounded wait: false (and the error flag set) when the barrier has not completed after `limit` polls.
__device__ __forceinline__ bool mbar_wait(u64* bar, u32 phase, u32* error, u32 limit = kSpinLimit) {
    for (u32 it = 0; it < limit; ++it)
        if (mbar_try_wait(bar, phase)) return true;
    atomicExch(error, 2u);
    return false;
}
__device__ __forceinline__ void tma_load_3d(void* dst, const CUtensorMap* map, u64* bar, int c0, int c1, int c2) {
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%3, %4, %5}], [%2];"
                 :: "r"(smem_u32(dst)), "l"((u64)map), "r"(smem_u32(bar)), "r"(c0), "r"(c1), "r"(c2) : "memory");
}
// K-major operand in 128-byte-swizzled 8-row atoms (1024 B): LBO 16 B, SBO 1024 B, layout SWIZZLE_128B.
__device__ __forceinline__ u64 smem_desc(const void* p) {
    const u64 start = (smem_u32(p) >> 4) & 0x3FFFu;
    return start | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// kind::i8: D s32, A s8, B s8, both K-major, M = 128, N = 128.
constexpr u32 kIdesc = (2u << 4) | (1u << 7) | (1u << 10) | ((u32)(kTileN >> 3) << 17) | ((u32)(kTileM >> 4) << 24);

__device__ __forceinline__ void mma_i8(u32 d_tmem, u64 a, u64 b, bool accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                 :: "r"(d_tmem), "l"(a), "l"(b), "r"(kIdesc), "r"((u32)accumulate), "r"(0u));
}
__device__ __forceinline__ void mma_commit(u64* bar) {
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" :: "r"(smem_u32(bar)) : "memory");
}
__device__ __forceinline__ void tmem_ld32(u32 taddr, u32 (&r)[32]) {
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x32.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, %15, "
                 "%16, %17, %18, %19, %20, %21, %22, %23, %24, %25, %26, %27, %28, %29, %30, %31}, [%32];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
                   "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15]),
                   "=r"(r[16]), "=r"(r[17]), "=r"(r[18]), "=r"(r[19]), "=r"(r[20]), "=r"(r[21]), "=r"(r[22]), "=r"(r[23]),
                   "=r"(r[24]), "=r"(r[25]), "=r"(r[26]), "=r"(r[27]), "=r"(r[28]), "=r"(r[29]), "=r"(r[30]), "=r"(r[31])
                 : "r"(taddr));
}

#ifdef LF_RESIDUE_MMA_KERNEL
// One CTA = one 128 x 128 output tile of one modulus (grid z).  Warp 0 lane 0 issues TMA loads,
// warp 1 lane 0 issues the MMAs; then all eight warps reduce the accumulators: warp w reads TMEM lanes
// 32 (w % 4) .. + 31 (rows) for the columns of half w / 4 and stores 32 residues of a row with four
// 16-byte stores when the row stride allows.
__global__ void __launch_bounds__(kMmaThreads, 1) residue_mma_kernel(const __grid_constant__ CUtensorMap ta1, const __grid_constant__ CUtensorMap ta0,
                                                              const __grid_constant__ CUtensorMap tb1, const __grid_constant__ CUtensorMap tb0,
                                                              MmaParams p) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)smem_raw + 1023) & ~(uintptr_t)1023);
    __shared__ __align__(8) u64 full[kStages], empty[kStages], done;
    __shared__ u32 tmem_slot;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const ResTables* tab = p.tab;
    if (p.plan) {
        if (p.plan->mode != 1 || blockIdx.z >= (unsigned)p.plan->L) return;
        tab = static_cast<const ResTables*>(p.plan->tab);
    }
    const int tm = blockIdx.y, tn = blockIdx.x, l = blockIdx.z;
    if (p.lower && (u64)tn * kTileN > (u64)tm * kTileM + kTileM - 1) return;      // whole tile above the diagonal
    if (threadIdx.x == 0) {
        for (int s = 0; s < kStages; ++s) { mbar_init(&full[s], 1); mbar_init(&empty[s], 1); }
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], 512;" :: "r"(smem_u32(&tmem_slot)));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const u32 tmem = tmem_slot;
    const u32 acc11 = tmem, acc00 = tmem + kTileN, accm = tmem + 2 * kTileN;
    const int kblocks = (int)(p.Kp / kTileK);
    const u32 polls = p.poll_limit ? p.poll_limit : kSpinLimit;
    __shared__ int abort_flag, issued, consumed;          // stages loaded by the producer / read by the MMA issuer
    if (threadIdx.x == 0) { abort_flag = 0; issued = 0; consumed = kblocks; }
    __syncthreads();
    if (warp == 0 && lane == 0) {
        // producer; stops issuing once the MMA issuer has given up
        for (int kb = 0; kb < kblocks && !p.no_loads; ++kb) {
            const int s = kb % kStages;
            const u32 ph = (u32)((kb / kStages) & 1);
            if (kb >= kStages && !mbar_wait(&empty[s], ph ^ 1u, p.error, polls)) { abort_flag = 1; break; }
            if (*(volatile int*)&abort_flag) break;
            unsigned char* st = smem + s * kStageBytes;
            mbar_expect_tx(&full[s], kStageBytes);
            tma_load_3d(st, &ta1, &full[s], kb * kTileK, tm * kTileM, l);
            tma_load_3d(st + kTileBytes, &ta0, &full[s], kb * kTileK, tm * kTileM, l);
            tma_load_3d(st + 2 * kTileBytes, &tb1, &full[s], kb * kTileK, tn * kTileN, l);
            tma_load_3d(st + 3 * kTileBytes, &tb0, &full[s], kb * kTileK, tn * kTileN, l);
            issued = kb + 1;
        }
    } else if (warp == 1 && lane == 0) {
        // MMA issuer
        bool ok = true;
        for (int kb = 0; kb < kblocks && ok; ++kb) {
            const int s = kb % kStages;
            const u32 ph = (u32)((kb / kStages) & 1);
            if (!mbar_wait(&full[s], ph, p.error, polls)) { ok = false; consumed = kb; *(volatile int*)&abort_flag = 1; break; }
            asm volatile("tcgen05.fence::after_thread_sync;");
            unsigned char* st = smem + s * kStageBytes;
            const u64 a1 = smem_desc(st), a0 = smem_desc(st + kTileBytes), b1 = smem_desc(st + 2 * kTileBytes),
                      b0 = smem_desc(st + 3 * kTileBytes);
#pragma unroll
            for (int kk = 0; kk < kTileK / 32; ++kk) {
                const u64 off = (u64)(kk * 32) >> 4;           // 32 bytes along K inside the swizzled row
                const bool acc = kb > 0 || kk > 0;
                mma_i8(acc11, a1 + off, b1 + off, acc);
                mma_i8(acc00, a0 + off, b0 + off, acc);
                mma_i8(accm, a1 + off, b0 + off, acc);
                mma_i8(accm, a0 + off, b1 + off, true);
            }
            mma_commit(&empty[s]);                            // stage free once these MMAs have read it
        }
        mma_commit(&done);                                    // arrives after every MMA issued above
    }
    __syncthreads();
    if (abort_flag && threadIdx.x == 0) {
        // An abandoned wait leaves loads in flight into shared memory: let every stage that was loaded and
        // not read complete (bounded) before the CTA releases its resources.
        for (int kb = consumed; kb < issued; ++kb) mbar_wait(&full[kb % kStages], (u32)((kb / kStages) & 1), p.error, polls);
    }
    const bool fine = mbar_wait(&done, 0, p.error, polls) && !abort_flag;
    asm volatile("tcgen05.fence::after_thread_sync;");
    if (fine) {
        const u32 m = tab->m[l];
        const u64 br = tab->barrett[l];
        const u32 moff = m - mod_barrett(1ull << 49, m, br);  // m - (2^49 mod m), in (0, m]
        const int q = warp & 3, half = warp >> 2;
        const u64 row = (u64)tm * kTileM + q * 32 + lane;
        const u32 lane_base = (u32)(q * 32) << 16;
        const bool vec = (p.Nc & 7) == 0;                      // rows start on 16-byte boundaries
        for (int c0 = half * (kTileN / 2); c0 < (half + 1) * (kTileN / 2); c0 += 32) {
            u32 s11[32], s00[32], sm[32];
            tmem_ld32(acc11 + lane_base + c0, s11);
            tmem_ld32(acc00 + lane_base + c0, s00);
            tmem_ld32(accm + lane_base + c0, sm);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
            if (row < p.M) {
                const u64 col0 = (u64)tn * kTileN + c0;
                u16* out = p.res + ((u64)l * p.M + row) * p.Nc + col0;
                u32 r[32];
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    // 65536 S11 + 256 Smid + S00 (|.| < 2^48), made nonnegative by 2^49 and reduced
                    const long long v = (long long)(int)s11[c] * 65536 + (long long)(int)sm[c] * 256 + (long long)(int)s00[c];
                    const u32 t = mod_barrett((u64)(v + (1ll << 49)), m, br) + moff;     // in (0, 2m)
                    r[c] = t >= m ? t - m : t;
                }
                if (vec && col0 + 32 <= p.Nc) {
                    uint4* o = reinterpret_cast<uint4*>(out);
#pragma unroll
                    for (int v = 0; v < 4; ++v)
                        o[v] = make_uint4(r[8 * v] | (r[8 * v + 1] << 16), r[8 * v + 2] | (r[8 * v + 3] << 16),
                                          r[8 * v + 4] | (r[8 * v + 5] << 16), r[8 * v + 6] | (r[8 * v + 7] << 16));
                } else {
#pragma unroll
                    for (int c = 0; c < 32; ++c)
                        if (col0 + c < p.Nc) out[c] = (u16)r[c];
                }
            }
        }
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, 512;" :: "r"(tmem));
}

// Plans a product on the GPU from its line analysis (the rule of the host driver): the residue engine
// when some line is nonzero and status free, every such line spans at most max_band bits (G = the
// widest) and 0 < K <= max_k; L is then the smallest count whose log2 product cum[L] exceeds
// 2(32 limbs + G) + ceil(log2 K) + 3.  Otherwise the limb kernel.  One block.
struct PlanParams {
    const LineInfo* linfo; const LineInfo* rinfo; u64 M, Nc, K; int limbs;
    const ResPlan* cands; const double* cum; int Lmin, count;     // candidate i is L = Lmin + i
    int max_band; u64 max_k;
    ResPlan* out;
};
__global__ void __launch_bounds__(256) plan_kernel(PlanParams p) {
    __shared__ int sg[256], sa[256];
    int G = 0, any = 0;
    for (u64 i = threadIdx.x; i < p.M + p.Nc; i += blockDim.x) {
        const LineInfo li = i < p.M ? p.linfo[i] : p.rinfo[i - p.M];
        if (!li.status && li.nonzero) { G = max(G, li.top - li.bottom); any = 1; }
    }
    sg[threadIdx.x] = G; sa[threadIdx.x] = any;
    __syncthreads();
    for (int o = 128; o; o >>= 1) {
        if ((int)threadIdx.x < o) { sg[threadIdx.x] = max(sg[threadIdx.x], sg[threadIdx.x + o]); sa[threadIdx.x] |= sa[threadIdx.x + o]; }
        __syncthreads();
    }
    if (threadIdx.x) return;
    ResPlan r{};
    r.mode = 0; r.G = sg[0];
    if (sa[0] && sg[0] <= p.max_band && p.K && p.K <= p.max_k) {
        int logk = 0;
        while ((1ull << logk) < p.K) ++logk;
        const double need = 2.0 * (32 * p.limbs + sg[0]) + logk + 3;
        for (int i = 0; i < p.count; ++i)
            if (p.cum[i] > need) { r = p.cands[i]; r.mode = 1; r.G = sg[0]; break; }
    }
    *p.out = r;
}

#endif  // LF_RESIDUE_MMA_KERNEL

// ---------------------------------------------------------------- 3. reconstruction and rounding
struct RecParams {
    const u16* res; const ResTables* tab; int L; int qwords;
    const LineInfo* linfo; const LineInfo* rinfo;
    u32* C; u64 ldc, M, Nc;
    int subtract, lower;
};
// RN(sign_x * X * 2^sx + c) with one rounding for an exact multiword X: both terms in one exact
// window when they are close, otherwise the far smaller term as a sticky unit (as in fma).
// acc (len words, two's complement) -= t << off (t has tw words), borrow carried to the top.
__device__ __forceinline__ void acc_sub(u32* acc, int len, const u32* t, int tw, i64 off) {
    const int ws = (int)(off >> 5), bs = (int)(off & 31);
    u32 bo = 0;
    int k = ws;
    for (int q = 0; q <= tw && k < len; ++q, ++k) {
        u32 v = q < tw ? t[q] << bs : 0u;
        if (bs && q > 0) v |= t[q - 1] >> (32 - bs);
        const u64 d = (u64)v + bo;
        const u32 old = acc[k];
        acc[k] = (u32)((u64)old - d);
        bo = (u64)old < d;
    }
    for (; bo && k < len; ++k) { const u32 old = acc[k]; acc[k] = old - 1u; bo = old == 0u; }
}
__device__ __forceinline__ void acc_unit(u32* acc, int len, bool negative) {   // acc +-= 1
    if (negative) { for (int k = 0; k < len; ++k) { const u32 old = acc[k]; acc[k] = old - 1u; if (old) break; } }
    else { for (int k = 0; k < len; ++k) { if (++acc[k]) break; } }
}
// Scratch words round_sum2 needs for an X of xw words (the window below); callers pass that much.
template <int N> __host__ __device__ constexpr int round_sum2_words(int xw) { return xw + 2 * N + 8; }
template <int N> __device__ Num<N> round_sum2(const u32* X, int xw, i64 sx, int signx, const Num<N>& c, u32* acc) {
    // One two's-complement window of xw + 2N + 8 words under the larger top, two bits of headroom
    // above it: a term below the window lies at least 2N + 6 words under that top, beyond every
    // rounding decision, and counts as +-1 in the lowest word.  The window lives in the caller's
    // scratch (shared memory in crt_round_kernel).
    const int CW = round_sum2_words<N>(xw);
    int tx = -1;
    for (int w = xw - 1; w >= 0; --w) if (X[w]) { tx = w; break; }
    if (tx < 0) return c;                                       // no product term left
    const i64 topx = sx + 32 * (i64)tx + 31 - __clz(X[tx]);
    if (!c.s) {
        Rounded<N> R; round_info<N>(X, xw, sx, R);
        return finish<N>(R.m, R.e, signx, R.rb && (R.sb || (R.m[0] & 1u)), 0);
    }
    const i64 sc = (i64)c.e - (32 * N - 1), topc = c.e;
    const i64 hi = topx > topc ? topx : topc;
    const i64 lo = hi + 3 - 32 * (i64)(CW - 1);               // exponent of window bit 32
    for (int w = 0; w < CW; ++w) acc[w] = 0;
    if (sx >= lo) { if (signx > 0) acc_add(acc, CW, X, xw, 32 + (sx - lo)); else acc_sub(acc, CW, X, xw, 32 + (sx - lo)); }
    else acc_unit(acc, CW, signx < 0);
    if (sc >= lo) { if (c.s > 0) acc_add(acc, CW, c.m, N, 32 + (sc - lo)); else acc_sub(acc, CW, c.m, N, 32 + (sc - lo)); }
    else acc_unit(acc, CW, c.s < 0);
    const bool negative = acc[CW - 1] >> 31;
    if (negative) { u32 cy = 1; for (int w = 0; w < CW; ++w) { const u32 v = ~acc[w] + cy; cy = cy && v == 0; acc[w] = v; } }
    Rounded<N> R;
    if (!round_info<N>(acc, CW, lo - 32, R)) return zero<N>();   // exact cancellation
    return finish<N>(R.m, R.e, negative ? -1 : 1, R.rb && (R.sb || (R.m[0] & 1u)), 0);
}

// From S = sum_l t_l (M / m_l) (qwords + 2 words, clobbered) and F = sum_l t_l floor(2^48 / m_l):
// X = S - round(F / 2^48) M, the signed exact product sum; returns RN(c -/+ X 2^scale) (subtract) or
// RN(X 2^scale), one rounding.  The modulus product exceeds 4 max|X|, so the quotient's rounding is
// never close.
template <int N> __device__ __forceinline__ Num<N> crt_tail(u32* S, int qwords, u64 F, const ResTables* tab, i64 scale,
                                                          bool subtract, const Num<N>& c, u32* scratch) {
    const u64 q = (F + (1ull << 47)) >> 48;                  // round(F): X = S - q M
    // D = S - q*M (two's complement over qwords+2 words)
    u64 borrow = 0;
    for (int w = 0; w <= qwords + 1; ++w) {
        const u64 qm = (w <= qwords ? (u64)tab->M[w] : 0ull) * q + borrow;
        const u32 lo = (u32)qm;
        const u32 old = S[w];
        S[w] = old - lo;
        borrow = (qm >> 32) + (old < lo ? 1u : 0u);
    }
    int sign = 1;
    const int xw = qwords + 2;
    if (S[xw - 1] >> 31) {
        sign = -1; u64 c1 = 1;
        for (int w = 0; w < xw; ++w) { u64 v = (u64)(u32)~S[w] + c1; S[w] = (u32)v; c1 = v >> 32; }
    }
    // a zero exact sum X with the addend falls back to c itself, as exact_dot_add
    return round_sum2<N>(S, xw, scale, subtract ? -sign : sign, c, scratch);
}

// ---------------------------------------------------------------- 4. tiled limb-kernel product
// The generic limb kernel's fast form: C[i][j] = RN(c -/+ sum_k L(i,k) R(j,k)) with every product summed exactly in
// one window per output and rounded once (round_sum2 with the old entry), the same bits as exact_dot_add.  The line
// analysis bounds every product of output (i, j): a nonzero, status-free entry of line i has its exponent in
// [bottom_i, top_i], so the products' scales lie in [base, base + spread_i + spread_j] with base = bottom_i +
// bottom_j - 2(32N - 1), each below 2^(scale + 64N), and K of them sum below 2^(base + spread_i + spread_j + 64N +
// ceil(log2 K)).  When that fits kWinWords(N) words, the output adds each signed product, shifted to its bit offset
// (scale - base), word by word into signed 64-bit column sums: no carry runs between the words of a product, so the
// adds of one product are independent, and K < 2^28 products of 32-bit words cannot overflow a column.  One carry pass
// at the end turns the columns into a two's-complement window that is rounded once with the old entry; wider
// outputs take exact_dot_add_dev's cluster method in the same kernel.  A block computes an 8 x 8 tile of outputs and
// stages the 8 + 8 lines' next kWinTK entries in shared memory, so each entry is read from memory once per tile
// instead of once per output; the column sums live in shared memory (one row per thread, an odd number of 64-bit
// words apart).
constexpr int kWinTM = 8, kWinTN = 8, kWinThreads = kWinTM * kWinTN, kWinTK = 8;
template <int N> __host__ __device__ constexpr int win_words() { return 2 * N + 8; }
// Row of one thread: W + 1 64-bit column sums (the sum's sign in the last), later the window (round_sum2's scratch is
// thread-local, used once per output); the row is an odd number of 64-bit words long.
template <int N> __host__ __device__ constexpr int win_row_words() { return 2 * ((win_words<N>() + 1) | 1); }
constexpr unsigned long long kWinMaxK = 1ull << 28;          // column sums of 32-bit words stay below 2^62
template <int N> __host__ __device__ constexpr size_t win_smem_bytes() {
    return (size_t)4 * ((kWinTM + kWinTN) * kWinTK * (N + 3) + kWinThreads * win_row_words<N>());
}
// col (len signed 64-bit column sums) +/-= t (TW words) << (32 ws + bs), one independent add per word
template <int TW> __device__ __forceinline__ void win_add_cols(long long* col, int len, const u32 (&t)[TW], int ws, int bs, bool negative) {
#pragma unroll
    for (int q = 0; q <= TW; ++q) {
        const int k = ws + q;
        if (k >= len) break;
        const u32 v = lf_fshl(q ? t[q - 1] : 0u, q < TW ? t[q] : 0u, (u32)bs);
        col[k] += negative ? -(long long)v : (long long)v;
    }
}
struct WinParams {
    DotParams d;                    // operands, output, modes, error word
    const LineInfo* linfo; const LineInfo* rinfo;   // analysis of the M left and Nc right lines
};
template <int N> __global__ void __launch_bounds__(kWinThreads) window_dot_kernel(const WinParams wp) {
    const DotParams& p = wp.d;
    constexpr int E = N + 3, W = win_words<N>();
    extern __shared__ __align__(16) u32 win_park[];
    u32* sA = win_park;                                  // [kWinTK][kWinTM] entries
    u32* sB = sA + kWinTK * kWinTM * E;                  // [kWinTK][kWinTN] entries
    const int t = threadIdx.x, r = t / kWinTN, q = t % kWinTN;
    u32* row = sB + kWinTK * kWinTN * E + t * win_row_words<N>();
    long long* col = reinterpret_cast<long long*>(row);  // W column sums; then the window
    const u64 r0 = (u64)blockIdx.y * kWinTM, q0 = (u64)blockIdx.x * kWinTN;
    const u64 ro = r0 + r, qo = q0 + q;                  // this thread's output (local row, column)
    const u64 i = p.row0 + ro, j = p.col0 + qo;          // its lines
    bool live = ro < p.M && qo < p.Nc && !(p.lower && j > i);
    u32* out = p.C + (ro * p.ldc + qo) * E;
    const Num<N> c = (live && p.subtract) ? load_plain<N>(out) : zero<N>();
    LineInfo li{}, ri{};
    if (live) { li = wp.linfo[ro]; ri = wp.rinfo[qo]; }
    const u32 st = (p.subtract ? c.st : 0u) | li.status | ri.status;
    const bool products = li.nonzero && ri.nonzero;
    int logk = 0;
    while ((1ull << logk) < p.K) ++logk;
    const i64 span = products ? (i64)(li.top - li.bottom) + (ri.top - ri.bottom) + 64 * N + logk : 0;
    const bool window = live && !st && products && span <= 32 * W && p.K < kWinMaxK;
    constexpr int W1 = W + 1;                            // one more column for the sign of the signed sum
    if (window) for (int w = 0; w < W1; ++w) col[w] = 0;
    const int ebase = li.bottom + ri.bottom;
    // all threads stage the tiles (the barriers include threads without a window)
    for (u64 k0 = 0; k0 < p.K; k0 += kWinTK) {
        __syncthreads();
        // word by word over the staged entries, consecutive words to consecutive threads: entries of one k that
        // are consecutive in memory (unit line stride) make coalesced runs
        for (int x = t; x < (kWinTM + kWinTN) * kWinTK * E; x += kWinThreads) {
            const int e = x / E, w = x - e * E;
            const bool left = e < kWinTM * kWinTK;
            const int y = left ? e : e - kWinTM * kWinTK;
            const int kk = y / (left ? kWinTM : kWinTN), line = y - kk * (left ? kWinTM : kWinTN);
            const u64 lo_line = (left ? r0 : q0) + line, k = k0 + kk;
            const bool in = k < p.K && lo_line < (left ? p.M : p.Nc);
            const LineView& v = left ? p.left : p.right;
            win_park[x] = in ? __ldg(v.base + (((left ? p.row0 : p.col0) + lo_line) * v.ls + k * v.ks) * (u64)E + w) : 0u;
        }
        __syncthreads();
        if (!window) continue;
        const int kmax = p.K - k0 < (u64)kWinTK ? (int)(p.K - k0) : kWinTK;
        for (int kk = 0; kk < kmax; ++kk) {
            const u32* a = sA + (kk * kWinTM + r) * E;
            const u32* b = sB + (kk * kWinTN + q) * E;
            const int sa = (int)a[N + 1], sb = (int)b[N + 1];
            if (!sa || !sb) continue;
            u32 am[N], bm[N], pr[2 * N];
#pragma unroll
            for (int w = 0; w < N; ++w) { am[w] = a[w]; bm[w] = b[w]; }
            mant_mul<N>(am, bm, pr);
            const int off = (int)a[N] + (int)b[N] - ebase;           // 0 <= off <= spread_i + spread_j
            win_add_cols<2 * N>(col, W1, pr, off >> 5, off & 31, (sa * sb > 0) == (p.subtract != 0));
        }
    }
    if (!live) return;
    if (st) { store<N>(out, zero<N>(st)); return; }
    if (!products) { store<N>(out, p.subtract ? c : zero<N>()); return; }
    if (!window) {                                       // wide output: the cluster method, from memory
        const Num<N> v = exact_dot_add_dev<N>(p.subtract ? out : nullptr, p.subtract, p.left.base + i * p.left.ls * E, (i64)p.left.ks,
                                              p.right.base + j * p.right.ls * E, (i64)p.right.ks, p.K, p.error);
        store<N>(out, v);
        return;
    }
    // one carry pass: the columns become the two's-complement window X (in place: word w is written after column w,
    // which starts at word 2w, has been read), its sign the final carry's
    u32* X = row;
    long long carry = 0;
    for (int w = 0; w < W1; ++w) {
        const long long v = col[w] + carry;
        X[w] = (u32)v;
        carry = v >> 32;
    }
    int cmp = carry < 0 ? -1 : 0;
    if (cmp < 0) {
        u32 cy = 1;
        for (int w = 0; w < W1; ++w) { const u32 v = ~X[w] + cy; cy = cy && v == 0; X[w] = v; }
    } else {
        for (int w = 0; w < W1 && !cmp; ++w) if (X[w]) cmp = 1;
    }
    // round_sum2 adds the old entry c with its own sign (it computes RN(sign * X * 2^scale + c))
    u32 scratch[round_sum2_words<N>(W1)];
    store<N>(out, round_sum2<N>(X, W1, (i64)ebase - 2 * (32 * N - 1), cmp, c, scratch));
}

template <int N> __global__ void __launch_bounds__(128) reconstruct_kernel(RecParams p) {
    const u64 j = (u64)blockIdx.x * blockDim.x + threadIdx.x, i = blockIdx.y;
    if (j >= p.Nc || i >= p.M) return;
    if (p.lower && j > i) return;
    constexpr u64 E = N + 3;
    u32* out = p.C + (i * p.ldc + j) * E;
    const Num<N> c = p.subtract ? load_plain<N>(out) : zero<N>();
    const LineInfo li = p.linfo[i], ri = p.rinfo[j];
    const u32 st = (p.subtract ? c.st : 0u) | li.status | ri.status;
    if (st) { store<N>(out, zero<N>(st)); return; }
    if (!li.nonzero || !ri.nonzero) { store<N>(out, p.subtract ? c : zero<N>()); return; }
    // S = sum_l t_l (M/m_l) in 64-bit column sums, F = sum_l t_l floor(2^48/m_l)
    u64 col[kResMaxQWords + 1];
    for (int w = 0; w <= p.qwords; ++w) col[w] = 0;
    u64 F = 0;
    bool any = false;
    for (int l = 0; l < p.L; ++l) {
        const u32 r = p.res[((u64)l * p.M + i) * p.Nc + j];
        any |= r != 0;
        const u32 m = p.tab->m[l];
        const u32 t = mod_barrett((u64)r * p.tab->w[l], m, p.tab->barrett[l]);
        F += (u64)t * p.tab->frac[l];
        for (int w = 0; w < p.qwords; ++w) col[w] += (u64)t * p.tab->q[l][w];
    }
    if (!any) { store<N>(out, p.subtract ? c : zero<N>()); return; }       // X == 0
    u32 S[kResMaxQWords + 2];
    u64 cy = 0;
    for (int w = 0; w <= p.qwords; ++w) { u64 v = col[w] + cy; S[w] = (u32)v; cy = v >> 32; }
    S[p.qwords + 1] = (u32)cy;
    u32 scratch[round_sum2_words<N>(kResMaxQWords + 2)];
    store<N>(out, crt_tail<N>(S, p.qwords, F, p.tab, (i64)li.bottom + ri.bottom - 2 * (32 * N - 1), p.subtract != 0, c, scratch));
}

// ---------------------------------------------------------------- 3b. CRT on the tensor cores
// S and F as one unsigned int8 GEMM.  With t_l = 256 th_l + tl_l (bytes) and q_{l,b} the bytes of
// M/m_l, byte column b of S gets P[b] = sum_l (tl_l q_{l,b} + th_l q_{l,b-1}), so that
// S = sum_b P[b] 2^(8b); F likewise from the bytes of floor(2^48/m_l).  Row o of the A operand holds
// (tl_0, th_0, tl_1, th_1, ...) for output o.  B is the constant [NB][Kp] byte matrix of those
// (shifted) bytes, uploaded once per modulus count already in the 128-byte-swizzled K-major layout
// of shared memory.  Each P[b] is below 2L * 255^2 < 2^25, so the int32 accumulators are exact.  One
// CTA computes 128 outputs per tile and is persistent over the tiles:
//   - eight warps build the rows of A from the residues (r -> t = r w_l mod m_l), warps q and q + 4
//     taking alternate groups of 16 moduli of the same rows;
//   - one thread issues tcgen05.mma kind::i8 (u8 x u8 -> s32, M = 128, N <= 256 per instruction)
//     into TMEM;
//   - each thread of warps 0-3 reads its TMEM lane and carries the byte columns into S and F, which
//     go to memory for crt_round_kernel (or are rounded here with crt_tail).
struct CrtParams {
    const u16* res; const ResTables* tab; const unsigned char* bimg;
    int L, qwords, NB, Kp, NS;             // B rows (multiple of 16), K bytes (multiple of 32), S byte columns
    u32 tmem_cols;
    const LineInfo* linfo; const LineInfo* rinfo;
    u32* C; u64 ldc, M, Nc;
    int subtract, lower;
    u32* error;
    const ResPlan* plan;                   // planned on the GPU: L and its operand come from the plan
    u32* sf;                               // not null: S (qwords + 2 words) and F (2 words) go here, word-major
                                           // (word w of output o at sf[w * M * Nc + o]), and crt_round_kernel rounds
};
__device__ __forceinline__ void mma_i8_u(u32 d_tmem, u64 a, u64 b, u32 idesc, bool accumulate) {
    asm volatile("{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                 "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, {%5, %5, %5, %5}, p;\n\t}"
                 :: "r"(d_tmem), "l"(a), "l"(b), "r"(idesc), "r"((u32)accumulate), "r"(0u));
}
__device__ __forceinline__ u64 crt_desc(u32 saddr) {       // K-major, SW128, SBO 1024 B, as smem_desc
    return (u64)((saddr >> 4) & 0x3FFFu) | (1ull << 16) | (64ull << 32) | (1ull << 46) | (2ull << 61);
}
// byte offset of (row, k) in a [rows][128-byte K block] tile, 128-byte swizzle (the TMA SW128 image)
__host__ __device__ __forceinline__ u32 sw128_offset(u32 row, u32 k) {
    return (row >> 3) * 1024u + (row & 7u) * 128u + ((((k >> 4) ^ row) & 7u) << 4) + (k & 15u);
}
template <int N> __global__ void __launch_bounds__(kCrtThreads, 2) crt_mma_kernel(const CrtParams pin) {
    CrtParams p = pin;
    if (pin.plan) {
        const ResPlan& r = *pin.plan;
        if (r.mode != 1) return;
        p.tab = static_cast<const ResTables*>(r.tab); p.bimg = r.crt_bimg; p.L = r.L; p.qwords = r.qwords;
        p.NB = r.NB; p.Kp = r.Kp; p.NS = r.NS; p.tmem_cols = r.tmem_cols;
    }
    extern __shared__ __align__(1024) unsigned char crt_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)crt_raw + 1023) & ~(uintptr_t)1023);
    const int kblocks = p.Kp / 128 + (p.Kp % 128 ? 1 : 0);
    unsigned char* sA = smem;                                  // kblocks x [128 rows][128 B]
    unsigned char* sB = smem + kblocks * 16384;                // kblocks x [NB rows][128 B]
    __shared__ __align__(8) u64 done;
    __shared__ u32 tmem_slot;
    __shared__ u32 s_m[kResMaxModuli], s_w[kResMaxModuli], s_r[kResMaxModuli];   // m_l, (M/m_l)^-1, floor(2^32/m_l)
    __shared__ unsigned char s_any[2][128];                    // some residue of the row is nonzero, per half
    const int warp = threadIdx.x >> 5;
    const u64 bbytes = (u64)kblocks * p.NB * 128;
    for (u64 o = (u64)threadIdx.x * 16; o < bbytes; o += (u64)blockDim.x * 16)
        *reinterpret_cast<uint4*>(sB + o) = *reinterpret_cast<const uint4*>(p.bimg + o);
    for (int l = threadIdx.x; l < p.L; l += blockDim.x) {
        s_m[l] = p.tab->m[l];
        s_w[l] = p.tab->w[l];
        s_r[l] = (u32)(p.tab->barrett[l] >> 32);               // floor(2^64 / m) >> 32 = floor(2^32 / m)
    }
    if (threadIdx.x == 0) {
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(&tmem_slot)), "r"(p.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const u32 tmem = tmem_slot;
    const int N1 = p.NB < 256 ? p.NB : 256, N2 = p.NB - N1;
    const u32 id1 = (2u << 4) | ((u32)(N1 >> 3) << 17) | ((u32)(128 >> 4) << 24);
    const u32 id2 = (2u << 4) | ((u32)(N2 >> 3) << 17) | ((u32)(128 >> 4) << 24);
    const u64 outputs = p.M * p.Nc, tiles = (outputs + 127) / 128;
    // Warps q and q + 4 stage alternate groups of 16 moduli of the same 128 rows; warps 0-3 then carry the
    // byte columns of their TMEM lanes 32 q .. into S and F.
    const int half = warp >> 2;
    const u32 row = (u32)((warp & 3) * 32 + (threadIdx.x & 31)), lane_base = (u32)((warp & 3) * 32) << 16;
    u32 phase = 0;
    for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        if (p.lower) {                                         // a tile inside one row, wholly above the diagonal
            const u64 o0 = tile * 128, o1 = (o0 + 127 < outputs ? o0 + 127 : outputs - 1);
            if (o0 / p.Nc == o1 / p.Nc && o0 % p.Nc > o0 / p.Nc) continue;
        }
        const u64 o = tile * 128 + row;
        const bool valid = o < outputs;
        bool any = false;
        for (int l0 = half * 16; l0 < p.L; l0 += 32) {          // row of A: t_l as two bytes; 16 loads in flight
            u32 r[16];
#pragma unroll
            for (int q = 0; q < 16; ++q) r[q] = (valid && l0 + q < p.L) ? p.res[(u64)(l0 + q) * outputs + o] : 0u;
#pragma unroll
            for (int q = 0; q < 16; ++q) {
                const int l = l0 + q;
                if (l >= p.L) break;
                any |= r[q] != 0;
                // t = r w mod m: r < m and w < m, so r w < 2^32 and one 32-bit Barrett step leaves [0, 2m)
                const u32 m = s_m[l], x = r[q] * s_w[l];
                u32 t = x - __umulhi(x, s_r[l]) * m;
                if (t >= m) t -= m;
                const u32 k = 2u * l;
                *reinterpret_cast<u16*>(sA + (k >> 7) * 16384u + sw128_offset(row, k & 127u)) = (u16)t;
            }
        }
        for (u32 k = 2u * p.L + 2u * half; k < (u32)kblocks * 128u; k += 4)
            *reinterpret_cast<u16*>(sA + (k >> 7) * 16384u + sw128_offset(row, k & 127u)) = 0;
        s_any[half][row] = any ? 1 : 0;
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // generic writes -> tensor core reads
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            for (int ks = 0; ks < p.Kp / 32; ++ks) {
                const int kb = ks >> 2;
                const u64 koff = (u64)((ks & 3) * 32) >> 4;
                const u64 ad = crt_desc(smem_u32(sA + kb * 16384)) + koff;
                const u32 bbase = smem_u32(sB + (u64)kb * p.NB * 128);
                mma_i8_u(tmem, ad, crt_desc(bbase) + koff, id1, ks > 0);
                if (N2) mma_i8_u(tmem + 256, ad, crt_desc(bbase + 256 * 128) + koff, id2, ks > 0);
            }
            mma_commit(&done);
        }
        const bool fine = __syncthreads_and(mbar_wait(&done, phase, p.error));
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (!fine) break;
        any = (s_any[0][row] | s_any[1][row]) != 0;
        // S and F from the byte columns of this row (every thread of warps 0-3 reads its lane: .sync.aligned)
        if (half == 0 && p.sf) {                                // S and F to global memory, word-major
            int sw = 0;
            u64 acc = 0, F = 0;
            u32* dst = p.sf + o;
            for (int c0 = 0; c0 < p.NB; c0 += 32) {
                u32 P[32];
                tmem_ld32(tmem + lane_base + (u32)c0, P);
                asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
                for (int c = 0; c < 32; ++c) {
                    const int col = c0 + c;
                    if (col < p.NS) {
                        acc += (u64)P[c] << (8 * (col & 3));
                        if ((col & 3) == 3) { if (valid) dst[(u64)sw * outputs] = (u32)acc; ++sw; acc >>= 32; }
                    } else if (col < p.NS + 6) {
                        F += (u64)P[c] << (8 * (col - p.NS));
                    }
                }
            }
            if (valid) {
                while (sw < p.qwords + 2) { dst[(u64)sw * outputs] = (u32)acc; ++sw; acc >>= 32; }
                dst[(u64)(p.qwords + 2) * outputs] = (u32)F;
                dst[(u64)(p.qwords + 3) * outputs] = (u32)(F >> 32);
            }
        } else if (half == 0) {                                 // S and F in registers, rounded here
        u32 S[kResMaxQWords + 2];
        int sw = 0;
        u64 acc = 0, F = 0;
        for (int c0 = 0; c0 < p.NB; c0 += 32) {
            u32 P[32];
            tmem_ld32(tmem + lane_base + (u32)c0, P);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int c = 0; c < 32; ++c) {
                const int col = c0 + c;
                if (col < p.NS) {
                    acc += (u64)P[c] << (8 * (col & 3));
                    if ((col & 3) == 3) { S[sw++] = (u32)acc; acc >>= 32; }
                } else if (col < p.NS + 6) {
                    F += (u64)P[c] << (8 * (col - p.NS));
                }
            }
        }
        while (sw < p.qwords + 2) { S[sw++] = (u32)acc; acc >>= 32; }
        if (valid) {
            const u64 i = o / p.Nc, j = o % p.Nc;
            if (!(p.lower && j > i)) {
                constexpr u64 E = N + 3;
                u32* out = p.C + (i * p.ldc + j) * E;
                const Num<N> c = p.subtract ? load_plain<N>(out) : zero<N>();
                const LineInfo li = p.linfo[i], ri = p.rinfo[j];
                const u32 st = (p.subtract ? c.st : 0u) | li.status | ri.status;
                if (st) store<N>(out, zero<N>(st));
                else if (!li.nonzero || !ri.nonzero || !any) store<N>(out, p.subtract ? c : zero<N>());
                else {
                    u32 scratch[round_sum2_words<N>(kResMaxQWords + 2)];
                    store<N>(out, crt_tail<N>(S, p.qwords, F, p.tab, (i64)li.bottom + ri.bottom - 2 * (32 * N - 1), p.subtract != 0, c, scratch));
                }
            }
        }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();                                        // TMEM and A are free for the next tile
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(p.tmem_cols));
}

// ---------------------------------------------------------------- 1b. digit planes on the tensor cores
// X mod m_l for all L moduli as one unsigned int8 GEMM: with x_b the bytes of X (4 xwords of them) and
// T_l[b] = 2^(8b) mod m_l = 256 th + tl, the columns 2l, 2l+1 of P = [x bytes] x [tl; th] give
// X == P_2l + 256 P_2l+1 (mod m_l), each P below 160 * 255^2 < 2^24.  Rows are the padded entries
// (line, k) in plane order, 128 per tile; B is the constant [2L][4 xwords] byte table, uploaded per
// (L, xwords) as its swizzled shared-memory image.  The epilogue reduces, negates for negative
// entries, balances and splits each residue into the two int8 digits, and writes them to the planes
// (consecutive rows are consecutive plane bytes).
struct DigitMmaParams {
    LineView v; u64 lines, K, Kp, rows_pad; int L; int xwords;
    const LineInfo* info; const ResTables* tab;
    const unsigned char* bimg; int NB, KB; u32 tmem_cols;
    signed char* d1; signed char* d0;
    u32* error;
    const ResPlan* plan;                   // planned on the GPU: L and its operand come from the plan
};
template <int N> __global__ void __launch_bounds__(kDigitThreads, 1) digits_mma_kernel(const DigitMmaParams pin) {
    DigitMmaParams p = pin;
    if (pin.plan) {
        const ResPlan& r = *pin.plan;
        if (r.mode != 1) return;
        p.tab = static_cast<const ResTables*>(r.tab); p.bimg = r.dig_bimg; p.L = r.L; p.NB = r.dNB; p.tmem_cols = r.dtmem;
    }
    extern __shared__ __align__(1024) unsigned char dig_raw[];
    unsigned char* smem = (unsigned char*)(((uintptr_t)dig_raw + 1023) & ~(uintptr_t)1023);
    const int kblocks = p.KB / 128 + (p.KB % 128 ? 1 : 0);
    unsigned char* sA = smem;
    unsigned char* sB = smem + kblocks * 16384;
    __shared__ __align__(8) u64 done;
    __shared__ u32 tmem_slot;
    __shared__ u32 s_m[kResMaxModuli], s_r[kResMaxModuli];     // m_l and floor(2^32 / m_l)
    __shared__ unsigned char s_neg[128];                       // row holds a negative entry
    const int warp = threadIdx.x >> 5;
    const u64 bbytes = (u64)kblocks * p.NB * 128;
    for (u64 o = (u64)threadIdx.x * 16; o < bbytes; o += (u64)blockDim.x * 16)
        *reinterpret_cast<uint4*>(sB + o) = *reinterpret_cast<const uint4*>(p.bimg + o);
    for (int l = threadIdx.x; l < p.L; l += blockDim.x) {
        s_m[l] = p.tab->m[l];
        s_r[l] = (u32)(p.tab->barrett[l] >> 32);               // floor(2^64 / m) >> 32 = floor(2^32 / m)
    }
    if (threadIdx.x == 0) {
        mbar_init(&done, 1);
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    if (warp == 0) {
        asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" :: "r"(smem_u32(&tmem_slot)), "r"(p.tmem_cols));
        asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
    }
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;");
    const u32 tmem = tmem_slot;
    const int N1 = p.NB < 256 ? p.NB : 256, N2 = p.NB - N1;
    const u32 id1 = (2u << 4) | ((u32)(N1 >> 3) << 17) | ((u32)(128 >> 4) << 24);
    const u32 id2 = (2u << 4) | ((u32)(N2 >> 3) << 17) | ((u32)(128 >> 4) << 24);
    const u64 plane = p.rows_pad * p.Kp, tiles = plane / 128;     // Kp is a multiple of 128
    const int q = warp & 3, half = warp >> 2;                  // warps q and q + 4 share TMEM lanes 32 q ..
    const u32 row = (u32)(q * 32 + (threadIdx.x & 31)), lane_base = (u32)(q * 32) << 16;
    // The first four warps stage the entries of a tile (one row each); the entry of the next tile is
    // loaded before the current tile's epilogue so that its latency hides behind the digit work.
    Num<N> a = zero<N>();
    u64 aline = 0;
    auto fetch = [&](u64 t) {
        a = zero<N>();
        const u64 e = t * 128 + row;
        aline = e / p.Kp;
        const u64 k = e % p.Kp;
        if (t < tiles && k < p.K && aline < p.lines) a = load<N>(p.v.base + (aline * p.v.ls + k * p.v.ks) * (u64)(N + 3));
    };
    if (half == 0) fetch(blockIdx.x);
    u32 phase = 0;
    for (u64 tile = blockIdx.x; tile < tiles; tile += gridDim.x) {
        const u64 e = tile * 128 + row;
        if (half == 0) {
            // row of A: the bytes of X = |entry| 2^(e - bottom) (0 <= shift <= G), zero beyond its words
#pragma unroll
            for (int c = 0; c < 16; ++c) {                      // up to 2 K blocks of 8 chunks
                if (c >= kblocks * 8) break;
                *reinterpret_cast<uint4*>(sA + (c >> 3) * 16384u + sw128_offset(row, (u32)(c & 7) * 16u)) = make_uint4(0, 0, 0, 0);
            }
            bool negative = false;
            if (!a.st && a.s) {
                negative = a.s < 0;
                const int sh = a.e - p.info[aline].bottom;
                const int ws = sh >> 5, bs = sh & 31;
#pragma unroll
                for (int i = 0; i <= N; ++i) {
                    u32 v = i < N ? a.m[i] << bs : 0u;
                    if (bs && i > 0) v |= a.m[i - 1] >> (32 - bs);
                    const u32 byte = (u32)(i + ws) * 4u;      // word i + ws < xwords <= KB / 4
                    *reinterpret_cast<u32*>(sA + (byte >> 7) * 16384u + sw128_offset(row, byte & 127u)) = v;
                }
            }
            s_neg[row] = negative ? 1 : 0;
        }
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncthreads();
        if (threadIdx.x == 0) {
            asm volatile("tcgen05.fence::after_thread_sync;");
            for (int ks = 0; ks < p.KB / 32; ++ks) {
                const int kb = ks >> 2;
                const u64 koff = (u64)((ks & 3) * 32) >> 4;
                const u64 ad = crt_desc(smem_u32(sA + kb * 16384)) + koff;
                const u32 bbase = smem_u32(sB + (u64)kb * p.NB * 128);
                mma_i8_u(tmem, ad, crt_desc(bbase) + koff, id1, ks > 0);
                if (N2) mma_i8_u(tmem + 256, ad, crt_desc(bbase + 256 * 128) + koff, id2, ks > 0);
            }
            mma_commit(&done);
        }
        const bool fine = __syncthreads_and(mbar_wait(&done, phase, p.error));
        phase ^= 1u;
        asm volatile("tcgen05.fence::after_thread_sync;");
        if (!fine) break;
        if (half == 0) fetch(tile + gridDim.x);                // sA is rewritten only after the barrier below
        const bool negative = s_neg[row] != 0;
        signed char* d1 = p.d1 + e;
        signed char* d0 = p.d0 + e;
        // X == P_2l + 256 P_2l+1 (mod m_l) with both P below 160 * 255^2, so the sum stays below 2^32 and one
        // 32-bit Barrett step with floor(2^32 / m) leaves it in [0, 2m).
        for (int c0 = half * 32; c0 < 2 * p.L; c0 += 64) {
            u32 P[32];
            tmem_ld32(tmem + lane_base + (u32)c0, P);
            asm volatile("tcgen05.wait::ld.sync.aligned;");
#pragma unroll
            for (int c = 0; c < 32; c += 2) {
                const int l = (c0 + c) >> 1;
                if (l >= p.L) break;
                const u32 m = s_m[l];
                const u32 x = P[c] + (P[c + 1] << 8);
                u32 u = x - __umulhi(x, s_r[l]) * m;
                if (u >= m) u -= m;
                if (negative && u) u = m - u;                   // residue of -X
                const int r = (int)u - (u > (m >> 1) ? (int)m : 0);   // balanced: |r| <= 32639
                const int lo = (int)(signed char)(r & 0xff);
                d1[(u64)l * plane] = (signed char)((r - lo) >> 8);
                d0[(u64)l * plane] = (signed char)lo;
            }
        }
        asm volatile("tcgen05.fence::before_thread_sync;");
        __syncthreads();
    }
    asm volatile("tcgen05.fence::before_thread_sync;");
    __syncthreads();
    if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" :: "r"(tmem), "r"(p.tmem_cols));
}

// The rounding half of the CRT when crt_mma_kernel wrote S and F: one thread per output.  Each thread's S and
// rounding window live in shared memory (crt_round_words words per thread, an odd stride so that the 32 lanes of a
// warp touching the same word index hit 32 banks), so the data-dependent word indexing of crt_tail costs no local-
// memory traffic to L2 and DRAM.  An output whose residues were all zero has S = F = 0, which crt_tail turns into
// c itself (or zero), as the fused path does.
constexpr int kCrtRoundThreads = 64;
template <int N> __host__ __device__ constexpr int crt_round_words(int qwords) {
    return ((qwords + 2) + round_sum2_words<N>(qwords + 2)) | 1;
}
template <int N> __global__ void __launch_bounds__(kCrtRoundThreads) crt_round_kernel(const CrtParams pin) {
    CrtParams p = pin;
    if (pin.plan) {
        if (pin.plan->mode != 1) return;
        p.tab = static_cast<const ResTables*>(pin.plan->tab); p.qwords = pin.plan->qwords;
    }
    extern __shared__ u32 crt_round_park[];
    const u64 outputs = p.M * p.Nc, o = (u64)blockIdx.x * kCrtRoundThreads + threadIdx.x;
    if (o >= outputs) return;
    const u64 i = o / p.Nc, j = o % p.Nc;
    if (p.lower && j > i) return;
    constexpr u64 E = N + 3;
    u32* out = p.C + (i * p.ldc + j) * E;
    const Num<N> c = p.subtract ? load_plain<N>(out) : zero<N>();
    const LineInfo li = p.linfo[i], ri = p.rinfo[j];
    const u32 st = (p.subtract ? c.st : 0u) | li.status | ri.status;
    if (st) { store<N>(out, zero<N>(st)); return; }
    if (!li.nonzero || !ri.nonzero) { store<N>(out, p.subtract ? c : zero<N>()); return; }
    u32* S = crt_round_park + threadIdx.x * crt_round_words<N>(p.qwords);
    for (int w = 0; w < p.qwords + 2; ++w) S[w] = p.sf[(u64)w * outputs + o];
    const u64 F = (u64)p.sf[(u64)(p.qwords + 2) * outputs + o] | ((u64)p.sf[(u64)(p.qwords + 3) * outputs + o] << 32);
    store<N>(out, crt_tail<N>(S, p.qwords, F, p.tab, (i64)li.bottom + ri.bottom - 2 * (32 * N - 1), p.subtract != 0, c, S + p.qwords + 2));
}

typedef void (*DigitFn)(const DigitParams&, cudaStream_t);
typedef void (*RecFn)(const RecParams&, cudaStream_t);
typedef void (*CrtFn)(const CrtParams&, unsigned grid, size_t smem, cudaStream_t);
typedef void (*DigitMmaFn)(const DigitMmaParams&, unsigned grid, size_t smem, cudaStream_t);
typedef void (*WindowDotFn)(const WinParams&, cudaStream_t);
struct ResidueKernels { DigitFn digits; RecFn rec; CrtFn crt; DigitMmaFn digits_mma; WindowDotFn window_dot; };
const ResidueKernels* residue_kernels(int limbs);

template <int N> void digits_launch(const DigitParams& p, cudaStream_t s) {
    if (!p.rows_pad || !p.Kp) return;
    dim3 grid((unsigned)((p.Kp + 127) / 128), (unsigned)p.rows_pad);
    digits_kernel<N><<<grid, 128, 0, s>>>(p);
}
template <int N> void crt_launch(const CrtParams& p, unsigned grid, size_t smem, cudaStream_t s) {
    if (!p.M || !p.Nc) return;
    cudaFuncSetAttribute(crt_mma_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    crt_mma_kernel<N><<<grid, kCrtThreads, smem, s>>>(p);
    if (p.sf) {
        // the planned form learns qwords on the GPU: size the rounding scratch for the largest table
        const int qw = p.plan ? kResMaxQWords : p.qwords;
        const size_t rsmem = (size_t)kCrtRoundThreads * crt_round_words<N>(qw) * 4;
        if (rsmem > 48 * 1024) cudaFuncSetAttribute(crt_round_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rsmem);
        crt_round_kernel<N><<<(unsigned)((p.M * p.Nc + kCrtRoundThreads - 1) / kCrtRoundThreads), kCrtRoundThreads, rsmem, s>>>(p);
    }
}
template <int N> void digits_mma_launch(const DigitMmaParams& p, unsigned grid, size_t smem, cudaStream_t s) {
    if (!p.rows_pad || !p.Kp) return;
    cudaFuncSetAttribute(digits_mma_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    digits_mma_kernel<N><<<grid, kDigitThreads, smem, s>>>(p);
}
template <int N> void window_dot_launch(const WinParams& p, cudaStream_t s) {
    if (!p.d.M || !p.d.Nc) return;
    const size_t smem = win_smem_bytes<N>();
    if (smem > 48 * 1024) cudaFuncSetAttribute(window_dot_kernel<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    dim3 grid((unsigned)((p.d.Nc + kWinTN - 1) / kWinTN), (unsigned)((p.d.M + kWinTM - 1) / kWinTM));
    window_dot_kernel<N><<<grid, kWinThreads, smem, s>>>(p);
}
template <int N> void rec_launch(const RecParams& p, cudaStream_t s) {
    if (!p.M || !p.Nc) return;
    dim3 grid((unsigned)((p.Nc + 127) / 128), (unsigned)p.M);
    reconstruct_kernel<N><<<grid, 128, 0, s>>>(p);
}

}  // namespace lfd

#define LF_RESIDUE_INSTANTIATE(N)                                                                  \
    namespace lfd {                                                                                \
    extern const ResidueKernels residue_kernels_##N; const ResidueKernels residue_kernels_##N = {digits_launch<N>, rec_launch<N>, crt_launch<N>, digits_mma_launch<N>, window_dot_launch<N>}; \
    }
