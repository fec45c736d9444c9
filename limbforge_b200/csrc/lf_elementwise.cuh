// Element-wise kernels: one value per thread, the reference's element layout (AoS) in HBM.
// Broadcast operands are read at (i / stride) % period (kernels.metal:7).  Op codes follow
// limbforge::Operation (engine.hpp:13).  The mul-chain kernel keeps the running value in
// registers across every step (the fused form of a resident CommandBatch chain).
#pragma once
#include "lf_arith.cuh"
#include <cuda_runtime.h>
#include <cstdint>

namespace lfd {

struct EwParams {
    const u32* a; const u32* b; const u32* c; u32* out;
    u64 count, bs, bp, cs, cp;
};
struct ChainStep { const u32* b; u32* out; u64 bs, bp; int op; int pad; };
constexpr int kMaxChain = 32;
struct ChainParams {
    const u32* a; u64 count; int steps; int lanes;      // lanes: 2 runs stageable multiplication chains on lane pairs
    ChainStep step[kMaxChain];
};

__device__ __forceinline__ u64 bidx(u64 i, u64 s, u64 p) { u64 j = s > 1 ? i / s : i; return p ? j % p : j; }

constexpr int kEwThreads = 128;

template <int N, int OP> __global__ void __launch_bounds__(kEwThreads) ew_kernel(EwParams p) {
    const u64 i = (u64)blockIdx.x * kEwThreads + threadIdx.x;
    if (i >= p.count) return;
    constexpr u64 E = N + 3;
    if constexpr (OP == 4 || OP == 5 || OP == 6 || OP == 11 || OP == 12) {
        const Cpx<N> x = cload<N>(p.a + 2 * E * i);
        const Cpx<N> y = cload<N>(p.b + 2 * E * bidx(i, p.bs, p.bp));
        Cpx<N> z;
        if constexpr (OP == 4) z = cadd<N>(x, y);
        else if constexpr (OP == 5) z = cmul<N>(x, y);
        else if constexpr (OP == 6) z = cdiv<N>(x, y);
        else {
            const Cpx<N> w = cload<N>(p.c + 2 * E * bidx(i, p.cs, p.cp));
            z = OP == 11 ? cfma<N>(x, y, w) : cfms<N>(x, y, w);
        }
        cstore<N>(p.out + 2 * E * i, z);
    } else {
        const Num<N> x = load<N>(p.a + E * i);
        Num<N> z;
        if constexpr (OP == 7) z = mul<N>(x, x);
        else if constexpr (OP == 8) z = lfd::sqrt<N>(x);
        else {
            const Num<N> y = load<N>(p.b + E * bidx(i, p.bs, p.bp));
            if constexpr (OP == 0) z = add<N>(x, y);
            else if constexpr (OP == 1) z = sub<N>(x, y);
            else if constexpr (OP == 2) z = mul<N>(x, y);
            else if constexpr (OP == 3) z = div<N>(x, y);
            else {
                const Num<N> w = load<N>(p.c + E * bidx(i, p.cs, p.cp));
                z = OP == 9 ? fma<N>(x, y, w) : fms<N>(x, y, w);
            }
        }
        store<N>(p.out + E * i, z);
    }
}

// v <- op_s(v, b_s[...]) for every step; out_s written where non-null.  Steps are uniform across
// the grid, so the switch never diverges.  Products read the factor's words from memory inside the
// product (mul_mem), which keeps the kernel at about 120 registers; 64-thread blocks spread a
// one-wave grid evenly over the SMs.
constexpr int kChainThreads = 64;
template <int N, bool MUL_ONLY> __global__ void __launch_bounds__(kChainThreads) chain_kernel(const __grid_constant__ ChainParams p) {
    const u64 i = (u64)blockIdx.x * kChainThreads + threadIdx.x;
    if (i >= p.count) return;
    constexpr u64 E = N + 3;
    Num<N> v = load_plain<N>(p.a + E * i);
#pragma unroll 1
    for (int s = 0; s < p.steps; ++s) {
        const ChainStep& st = p.step[s];
        const u32* y = st.b + E * bidx(i, st.bs, st.bp);
        if constexpr (MUL_ONLY) v = mul_mem<N>(v, y);
        else switch (st.op) {
        case 0: v = add<N>(v, load_plain<N>(y)); break;
        case 1: v = sub<N>(v, load_plain<N>(y)); break;
        case 2: v = mul_mem<N>(v, y); break;
        default: v = div<N>(v, load_plain<N>(y)); break;
        }
        if (st.out) store<N>(st.out + E * i, v);
    }
}

// Multiplication chains whose factors are contiguous (no broadcast) and read nowhere that a step writes:
// a block of 32 values copies the next step's 32 factors (one contiguous tile of 32 (N+3) words, a
// multiple of 16 bytes) into shared memory with cp.async while the current products run, so the product
// reads its factor words from shared memory.  A partial last block reads its factors directly.
constexpr int kStagedThreads = 32;
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
    const unsigned a = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" :: "r"(a), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int G> __device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" :: "n"(G) : "memory"); }

template <int N> __global__ void __launch_bounds__(kStagedThreads) chain_staged_kernel(const __grid_constant__ ChainParams p) {
    constexpr u64 E = N + 3;
    constexpr int T = kStagedThreads, TILE = T * (int)E, CH = TILE / 4;
    static_assert(TILE % 4 == 0, "tiles of whole 16-byte chunks");
    const u64 base = (u64)blockIdx.x * T, i = base + threadIdx.x;
    if (base + T > p.count) {
        if (i >= p.count) return;
        Num<N> v = load_plain<N>(p.a + E * i);
#pragma unroll 1
        for (int s = 0; s < p.steps; ++s) {
            v = mul_mem<N>(v, p.step[s].b + E * i);
            if (p.step[s].out) store<N>(p.step[s].out + E * i, v);
        }
        return;
    }
    extern __shared__ __align__(16) u32 chain_stage[];
    const auto fetch = [&](int s) {
        const u32* src = p.step[s].b + E * base;
        u32* dst = chain_stage + (s & 1) * TILE;
        for (int c = threadIdx.x; c < CH; c += T) cp_async16(dst + 4 * c, src + 4 * c);
        cp_async_commit();
    };
    fetch(0);
    Num<N> v = load_plain<N>(p.a + E * i);
#pragma unroll 1
    for (int s = 0; s < p.steps; ++s) {
        if (s + 1 < p.steps) { fetch(s + 1); cp_async_wait<1>(); } else cp_async_wait<0>();
        __syncthreads();                                     // every thread's chunks of this step's tile
        v = mul_mem<N>(v, chain_stage + (s & 1) * TILE + threadIdx.x * E);
        if (p.step[s].out) store<N>(p.step[s].out + E * i, v);
        __syncthreads();                                     // the tile is refilled for step s + 2
    }
}
// ---- Lane pairs: one value over two lanes (N even, N >= 12).  Both lanes hold the running value a.  Lane p forms
// the rows j = 2m + p of the upper part T of a * y (the products a_i y_j with i + j >= N - 2, as mant_mul_high_mem),
// each row a carry chain, into its own window; lane p's window index w'' stands for word w'' - 1 + p of T, which
// keeps every index static.  Lane 1's row 2m + 1 starts one product earlier than lane 0's row 2m; lane 0 takes that
// product with a zero operand.  One exchange of the windows (a shuffle per word) gives both lanes T, and both round
// it exactly as mul does, so the pair ends the step holding RN(a * y) bit for bit as one thread would.
template <int N> __device__ __forceinline__ Num<N> mul_pair(const Num<N>& a, const u32* y, int pl) {
    static_assert(N % 2 == 0 && N >= kShortMulLimbs, "lane pairs need an even width of at least kShortMulLimbs");
    constexpr int B = N - 2, W = N + 2;
    const int ys = (int)y[N + 1];
    const u32 st = a.st | y[N + 2];
    if (st || !a.s || !ys) return zero<N>(st);
    u32 h[W + 1];
#pragma unroll
    for (int k = 0; k <= W; ++k) h[k] = 0;
#pragma unroll
    for (int m = 0; m < N / 2; ++m) {
        const u32 bj = y[2 * m + pl];
        const int i1 = B - 2 * m - 1 > 0 ? B - 2 * m - 1 : 0;           // lane 1's first product (static)
        const bool mask0 = B - 2 * m - 1 >= 0;                           // lane 0 starts one later: zero operand
        u32 c = 0;
#pragma unroll
        for (int i = i1; i < N; ++i) {
            const u32 ai = (i == i1 && mask0 && !pl) ? 0u : a.m[i];
            const u64 t = (u64)ai * bj + h[i + 2 * m - B + 1] + c;
            h[i + 2 * m - B + 1] = (u32)t;
            c = (u32)(t >> 32);
        }
        h[2 * m + 3] = c;                                                // N - 1 + 2m - B + 2
    }
    // T word w = h0[w + 1] + h1[w]: each lane sends its share of word w and adds the partner's.  The exchange names
    // only the two lanes of the pair: other pairs of the warp may have left (a zero or status operand above, or a
    // value past the end), and both lanes of a pair always take the same path (they hold the same a and y).
    const u32 pair = 3u << ((threadIdx.x & 31) & ~1u);
    u32 cy = 0;
#pragma unroll
    for (int w = 0; w < W; ++w) {
        const u32 mine = pl ? h[w] : h[w + 1];
        const u32 other = __shfl_xor_sync(pair, mine, 1);
        const u64 t = (u64)mine + other + cy;
        h[w] = (u32)t;
        cy = (u32)(t >> 32);
    }
    const u32 sh = (h[N + 1] >> 31) ? 0u : 1u;
    const u32 lw = h[1] << sh;
    const u32 low = lw & 0x7fffffffu;
    const bool rb = lw >> 31;
    if (low >= 0x80000000u - ((u32)N << sh) || (rb && low == 0)) return mul_exact_mem_call<N>(a, y);
    u32 m[N];
#pragma unroll
    for (int i = 0; i < N; ++i) m[i] = __funnelshift_l(h[i + 1], h[i + 2], sh);
    return finish<N>(m, (i64)a.e + (int)y[N] + 1 - (i64)sh, a.s * ys, rb, 0);
}
constexpr int kPairThreads = 64;                          // 32 values per block
template <int N> __global__ void __launch_bounds__(kPairThreads, 10) chain_pair_kernel(const __grid_constant__ ChainParams p) {
    constexpr u64 E = N + 3;
    constexpr int V = kPairThreads / 2, TILE = V * (int)E, CH = TILE / 4;
    static_assert(TILE % 4 == 0, "tiles of whole 16-byte chunks");
    const int pl = threadIdx.x & 1, vi = threadIdx.x >> 1;
    const u64 base = (u64)blockIdx.x * V, i = base + vi;
    if (base + V > p.count) {                                       // partial block: factors straight from memory
        if (i >= p.count) return;                                    // both lanes of a pair leave together
        Num<N> v = load_plain<N>(p.a + E * i);
#pragma unroll 1
        for (int s = 0; s < p.steps; ++s) {
            v = mul_pair<N>(v, p.step[s].b + E * i, pl);
            if (p.step[s].out && !pl) store<N>(p.step[s].out + E * i, v);
        }
        return;
    }
    extern __shared__ __align__(16) u32 pair_stage[];
    const auto fetch = [&](int s) {
        const u32* src = p.step[s].b + E * base;
        u32* dst = pair_stage + (s & 1) * TILE;
        for (int c = threadIdx.x; c < CH; c += kPairThreads) cp_async16(dst + 4 * c, src + 4 * c);
        cp_async_commit();
    };
    fetch(0);
    Num<N> v = load_plain<N>(p.a + E * i);
#pragma unroll 1
    for (int s = 0; s < p.steps; ++s) {
        if (s + 1 < p.steps) { fetch(s + 1); cp_async_wait<1>(); } else cp_async_wait<0>();
        __syncthreads();
        v = mul_pair<N>(v, pair_stage + (s & 1) * TILE + vi * E, pl);
        if (p.step[s].out && !pl) store<N>(p.step[s].out + E * i, v);
        __syncthreads();
    }
}

// The staged kernel applies when every factor is contiguous, 16-byte aligned and disjoint from every output.
inline bool chain_can_stage(const ChainParams& p, u64 E) {
    const u64 bytes = p.count * E * 4;
    for (int k = 0; k < p.steps; ++k) {
        const ChainStep& st = p.step[k];
        if (st.op != 2 || st.bs != 1 || st.bp != 0 || ((uintptr_t)st.b & 15)) return false;
        const uintptr_t b0 = (uintptr_t)st.b, b1 = b0 + bytes;
        for (int q = 0; q < p.steps; ++q) {
            if (!p.step[q].out) continue;
            const uintptr_t o0 = (uintptr_t)p.step[q].out, o1 = o0 + bytes;
            if (b0 < o1 && o0 < b1) return false;
        }
    }
    return true;
}

template <int N> int launch_ew(int op, const EwParams& p, cudaStream_t s) {
    if (!p.count) return 0;
    const unsigned blocks = (unsigned)((p.count + kEwThreads - 1) / kEwThreads);
    switch (op) {
    case 0: ew_kernel<N, 0><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 1: ew_kernel<N, 1><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 2: ew_kernel<N, 2><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 3: ew_kernel<N, 3><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 4: ew_kernel<N, 4><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 5: ew_kernel<N, 5><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 6: ew_kernel<N, 6><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 7: ew_kernel<N, 7><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 8: ew_kernel<N, 8><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 9: ew_kernel<N, 9><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 10: ew_kernel<N, 10><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 11: ew_kernel<N, 11><<<blocks, kEwThreads, 0, s>>>(p); break;
    case 12: ew_kernel<N, 12><<<blocks, kEwThreads, 0, s>>>(p); break;
    default: return 1;
    }
    return 0;
}
template <int N> int launch_chain(const ChainParams& p, cudaStream_t s) {
    if (!p.count) return 0;
    const unsigned blocks = (unsigned)((p.count + kChainThreads - 1) / kChainThreads);
    bool mul_only = true;
    for (int k = 0; k < p.steps; ++k) mul_only = mul_only && p.step[k].op == 2;
    if (mul_only && chain_can_stage(p, N + 3)) {
        if constexpr (N % 2 == 0 && N >= kShortMulLimbs) {
            if (p.lanes == 2) {
                const unsigned pb = (unsigned)((p.count + kPairThreads / 2 - 1) / (kPairThreads / 2));
                chain_pair_kernel<N><<<pb, kPairThreads, 2 * (kPairThreads / 2) * (N + 3) * 4, s>>>(p);
                return 0;
            }
        }
        const unsigned sb = (unsigned)((p.count + kStagedThreads - 1) / kStagedThreads);
        chain_staged_kernel<N><<<sb, kStagedThreads, 2 * kStagedThreads * (N + 3) * 4, s>>>(p);
    } else if (mul_only) chain_kernel<N, true><<<blocks, kChainThreads, 0, s>>>(p);     // registers of mul alone
    else chain_kernel<N, false><<<blocks, kChainThreads, 0, s>>>(p);
    return 0;
}

// Attributes of the element-wise kernel of one operation (the query also loads the kernel's module, which a
// first launch would otherwise do): Engine::prewarm and Engine::pipeline_info.
template <int N> int ew_attributes(int op, cudaFuncAttributes* a) {
    switch (op) {
    case 0: return cudaFuncGetAttributes(a, ew_kernel<N, 0>);
    case 1: return cudaFuncGetAttributes(a, ew_kernel<N, 1>);
    case 2: return cudaFuncGetAttributes(a, ew_kernel<N, 2>);
    case 3: return cudaFuncGetAttributes(a, ew_kernel<N, 3>);
    case 4: return cudaFuncGetAttributes(a, ew_kernel<N, 4>);
    case 5: return cudaFuncGetAttributes(a, ew_kernel<N, 5>);
    case 6: return cudaFuncGetAttributes(a, ew_kernel<N, 6>);
    case 7: return cudaFuncGetAttributes(a, ew_kernel<N, 7>);
    case 8: return cudaFuncGetAttributes(a, ew_kernel<N, 8>);
    case 9: return cudaFuncGetAttributes(a, ew_kernel<N, 9>);
    case 10: return cudaFuncGetAttributes(a, ew_kernel<N, 10>);
    case 11: return cudaFuncGetAttributes(a, ew_kernel<N, 11>);
    case 12: return cudaFuncGetAttributes(a, ew_kernel<N, 12>);
    default: return (int)cudaErrorInvalidValue;
    }
}

// Dispatch tables filled by the per-width translation units (lf_ew_*.cu).
typedef int (*EwLauncher)(int, const EwParams&, cudaStream_t);
typedef int (*ChainLauncher)(const ChainParams&, cudaStream_t);
typedef int (*EwAttributes)(int, cudaFuncAttributes*);
EwLauncher ew_launcher(int limbs);
ChainLauncher chain_launcher(int limbs);
EwAttributes ew_attributes_of(int limbs);

}  // namespace lfd

#define LF_EW_INSTANTIATE(N)                                                             \
    namespace lfd {                                                                      \
    int ew_launch_##N(int op, const EwParams& p, cudaStream_t s) { return launch_ew<N>(op, p, s); } \
    int chain_launch_##N(const ChainParams& p, cudaStream_t s) { return launch_chain<N>(p, s); } \
    int ew_attr_##N(int op, cudaFuncAttributes* a) { return ew_attributes<N>(op, a); } \
    }
