// Batched small-matrix kernels: 4x4 complex LU solve/inverse/determinant (the rounding sequence of
// kernels.metal:210-249) and strided batched GEMM with ascending-k composed or fused updates
// (batched_linalg.metal:16-17, 24-37, 145-157 sequence).  Every arithmetic step is the correctly
// rounded device routine of lf_arith.cuh, applied to the same operands in the same order as the
// reference's sequence, so the bits are the same however the steps are spread over threads.
#pragma once
#include "lf_arith.cuh"
#include <cuda_runtime.h>

namespace lfd {

struct Lu4Params {
    const u32* A; const u32* B; u32* X; u32* det; u32* status;
    u64 count; unsigned rhs; int fused, want_det, inverse;
};

template <int N, bool FUSED> __device__ __forceinline__ Cpx<N> c_minus(const Cpx<N>& c, const Cpx<N>& a, const Cpx<N>& b) {
    if constexpr (FUSED) { Cpx<N> r = cfms<N>(a, b, c); return {negate<N>(r.re), negate<N>(r.im)}; }   // -(a*b - c), one rounding each
    const Cpx<N> q = cmul<N>(a, b);
    return {subx<N>(c.re, q.re), subx<N>(c.im, q.im)};
}
template <int N> __device__ __forceinline__ Num<N> mag_of(const Cpx<N>& z) {               // max(|re|, |im|) by exact comparison
    return mag_cmp<N>(z.re, z.im) >= 0 ? z.re : z.im;
}

// ---- 4x4 complex LU: one quad of lanes per system.
// The quad parks its system in shared memory: the 16 matrix entries, then 4 solve values.  Lane r owns row r
// of the elimination.  At step k every lane finds the same pivot (the row r >= k of largest max(|re|, |im|),
// ties to the lowest row) by reading column k, lane c swaps column c of the two rows, and lane r > k forms its
// multiplier l = a_rk / a_kk and updates a_rc -= l a_kc (c > k) from the pivot row.  The solves give lane i
// row i of the right-hand side: forward, y_i -= a_it y_t in ascending t as each y_t becomes final; backward,
// y_i -= a_it y_t (t = i+1..3, ascending) then y_i /= a_ii, row after row.  Lane 0 forms the determinant while
// the other lanes start the forward pass.  A grid-stride loop over systems accepts any grid; the block size
// must be a multiple of four.
constexpr unsigned kLuLanes = 4;
template <int N> constexpr u32 lu_quad_words() { return 20u * 2u * (N + 3); }
template <int N> __device__ __forceinline__ Cpx<N> lu_get(const u32* q, unsigned idx) { return cload_plain<N>(q + idx * 2 * (N + 3)); }
template <int N> __device__ __forceinline__ void lu_put(u32* q, unsigned idx, const Cpx<N>& z) { cstore<N>(q + idx * 2 * (N + 3), z); }

template <int N, bool FUSED> __global__ void __launch_bounds__(256) lu4_kernel(Lu4Params p) {
    constexpr u64 CE = 2 * (N + 3);
    extern __shared__ __align__(16) u32 lu_park[];
    const unsigned lane = threadIdx.x & 3u;
    u32* const q = lu_park + (threadIdx.x >> 2) * lu_quad_words<N>();
    u32* const Y = q + 16 * CE;
    const unsigned qmask = 0xFu << (threadIdx.x & 28u);
    const u64 quads = ((u64)gridDim.x * blockDim.x) >> 2;
    const Cpx<N> z = {zero<N>(), zero<N>()};
    for (u64 m = ((u64)blockIdx.x * blockDim.x + threadIdx.x) >> 2; m < p.count; m += quads) {
        const u32* src = p.A + m * 16 * CE;                  // 16 contiguous entries, copied word by word
        for (u32 w = lane; w < 16 * CE; w += kLuLanes) q[w] = __ldg(src + w);
        __syncwarp(qmask);
        unsigned perm = 0x03020100u, st = 0, swaps = 0;     // row of step i in byte i
        for (unsigned k = 0; k < 4; ++k) {
            unsigned piv = k;
            for (unsigned r = k + 1; r < 4; ++r)
                if (mag_cmp<N>(mag_of<N>(lu_get<N>(q, r * 4 + k)), mag_of<N>(lu_get<N>(q, piv * 4 + k))) > 0) piv = r;
            const Cpx<N> pv = lu_get<N>(q, piv * 4 + k);
            __syncwarp(qmask);                              // column k read by every lane before it moves
            if (!pv.re.s && !pv.im.s) { st = k + 1; break; }
            if (piv != k) {
                const Cpx<N> x = lu_get<N>(q, k * 4 + lane), y = lu_get<N>(q, piv * 4 + lane);
                lu_put<N>(q, k * 4 + lane, y);
                lu_put<N>(q, piv * 4 + lane, x);
                const unsigned a = (perm >> (8 * k)) & 0xffu, b = (perm >> (8 * piv)) & 0xffu;
                perm ^= ((a ^ b) << (8 * k)) | ((a ^ b) << (8 * piv));
                ++swaps;
                __syncwarp(qmask);
            }
            if (lane > k) {
                const Cpx<N> l = cdiv<N>(lu_get<N>(q, lane * 4 + k), lu_get<N>(q, k * 5));
                lu_put<N>(q, lane * 4 + k, l);
                for (unsigned c = k + 1; c < 4; ++c) lu_put<N>(q, lane * 4 + c, c_minus<N, FUSED>(lu_get<N>(q, lane * 4 + c), l, lu_get<N>(q, k * 4 + c)));
            }
            __syncwarp(qmask);
        }
        if (lane == 0) {
            p.status[m] = st;
            if (p.want_det) {
                Cpx<N> d = z;
                if (!st) {
                    d = lu_get<N>(q, 0);
                    for (unsigned k = 1; k < 4; ++k) d = cmul<N>(d, lu_get<N>(q, k * 5));
                    if (swaps & 1) d = {negate<N>(d.re), negate<N>(d.im)};
                }
                cstore<N>(p.det + m * CE, d);
            }
        }
        const unsigned R = p.inverse ? 4 : p.rhs;
        for (unsigned j = 0; j < R; ++j) {
            u32* xo = p.X + ((m * 4 + lane) * R + j) * CE;
            if (st) { cstore<N>(xo, Cpx<N>{zero<N>(kDivZero), zero<N>(kDivZero)}); continue; }
            Cpx<N> y;
            const unsigned row = (perm >> (8 * lane)) & 0xffu;
            if (p.inverse) { y = z; if (row == j) { y.re.m[N - 1] = 0x80000000u; y.re.s = 1; } }
            else y = cload<N>(p.B + ((m * 4 + row) * R + j) * CE);
            if (lane == 0) lu_put<N>(Y, 0, y);
            __syncwarp(qmask);
            for (unsigned t = 0; t < 3; ++t) {                // y_t is final after step t - 1
                if (lane > t) {
                    y = c_minus<N, FUSED>(y, lu_get<N>(q, lane * 4 + t), lu_get<N>(Y, t));
                    if (lane == t + 1) lu_put<N>(Y, lane, y);
                }
                __syncwarp(qmask);
            }
            for (int i = 3; i >= 0; --i) {
                if ((int)lane == i) {
                    for (unsigned t = (unsigned)i + 1; t < 4; ++t) y = c_minus<N, FUSED>(y, lu_get<N>(q, i * 4 + t), lu_get<N>(Y, t));
                    y = cdiv<N>(y, lu_get<N>(q, (unsigned)i * 5));
                    lu_put<N>(Y, (unsigned)i, y);
                }
                __syncwarp(qmask);
            }
            cstore<N>(xo, y);
        }
        __syncwarp(qmask);                                  // the parked system is read to the end before the next one
    }
}

// GEMM work of one launch.  Work units are output entries (real) or entry components (complex: unit g
// is component g & 1 of entry g >> 1); `cells` counts units.  Ragged form (items != nullptr): entries of
// every item of one precision class numbered consecutively (item t owns entries [cell0, cell0 + m n)),
// units cut into chunks of `chunk`, and chunk_item[c] the item owning the first unit of chunk c; operands are word
// offsets from `base`.  Uniform form (items == nullptr): the StridedGemm shape below.  With `counter`
// the kernel is persistent (blocks take chunks from the counter until none are left); without it
// block b computes chunk b.  With out_override every output cell g goes to out_override + g * S
// instead of its C (the autotuner's trial runs leave the caller's outputs untouched).
struct GemmItem { u64 a, b, c, cell0; u32 m, n, k, flags; };          // flags: 1 accumulate, 2 negative
struct GemmWork {
    const GemmItem* items; const u32* chunk_item; const u32* base;
    u64 cells; u32 nchunks, chunk;
    u32* counter; u32* out_override; u32* out_base;
    const u32* A; const u32* B; u32* C; u64 m, n, k, sa, sb, sc; int accumulate, negative;
};
// One output entry (real) or one component of one (complex: comp 0 = re, 1 = im), summed over
// ascending k from C (accumulate) or zero and negated at the end.  The components of a complex entry
// are independent rounding sequences, so each has its own thread:
//   composed re: add(sub(mul(ar, br), mul(ai, bi)), sum)   im: add(add(mul(ar, bi), mul(ai, br)), sum)
//   fused    re: dot2_add(ar, br, -ai, bi, sum)             im: dot2_add(ar, bi, ai, br, sum)
// exactly the re / im parts of cadd(cmul(a, b), sum) and cfma(a, b, sum).
// One k step of one complex component: sum <- the composed or fused update with x = a_ik, y = b_kj.
// Operands are loaded next to their use (the second factor of a product word by word inside it, mul_mem),
// so only the running sum lives across products; above 8 limbs
// the step is an out-of-line call, which keeps the kernel's register allocation to that sum.
template <int N, bool FUSED> __device__ __forceinline__ void cx_step_body(Num<N>& sum, const u32* x, const u32* y, int comp) {
    constexpr u64 E = N + 3;
    const u32* yr = y + (comp ? E : 0);                 // im swaps the roles of br and bi
    const u32* yi = y + (comp ? 0 : E);
    if constexpr (FUSED) {
        const Num<N> xi = load<N>(x + E);
        sum = dot2_add<N>(load<N>(x), load<N>(yr), comp ? xi : negate<N>(xi), load<N>(yi), sum);
    } else {
        const Num<N> p1 = mul_mem<N>(load<N>(x), yr);
        const Num<N> p2 = mul_mem<N>(load<N>(x + E), yi);
        sum = add<N>(comp ? add<N>(p1, p2) : sub<N>(p1, p2), sum);
    }
}
template <int N, bool FUSED> __device__ __noinline__ void cx_step_call(Num<N>& sum, const u32* x, const u32* y, int comp) {
    cx_step_body<N, FUSED>(sum, x, y, comp);
}
template <int N, bool FUSED> __device__ __forceinline__ void cx_step(Num<N>& sum, const u32* x, const u32* y, int comp) {
    if constexpr (N > 8) cx_step_call<N, FUSED>(sum, x, y, comp); else cx_step_body<N, FUSED>(sum, x, y, comp);
}

// Composed complex entries of 17+ limbs park their running sum and first product in shared memory (a slot of
// 2(N+3) words per thread, word w at slot[w * stride]) while the next product runs.  The kernel then needs
// the registers of one product or one sum at a time (128), which raises the warps an SM holds from 10 to 16 at 1024 bits.
template <int N, bool CX, bool FUSED> constexpr bool parked_state() { return CX && !FUSED && N >= 17; }
template <int N> __device__ __forceinline__ void park(u32* slot, u32 stride, const Num<N>& v) {
#pragma unroll
    for (int w = 0; w < N; ++w) slot[w * stride] = v.m[w];
    slot[N * stride] = (u32)v.e; slot[(N + 1) * stride] = (u32)v.s; slot[(N + 2) * stride] = v.st;
}
template <int N> __device__ __forceinline__ Num<N> unpark(const u32* slot, u32 stride) {
    Num<N> v;
#pragma unroll
    for (int w = 0; w < N; ++w) v.m[w] = slot[w * stride];
    v.e = (int)slot[N * stride]; v.s = (int)slot[(N + 1) * stride]; v.st = slot[(N + 2) * stride];
    return v;
}
template <int N> __device__ void gemm_cell_parked(const u32* A, const u32* B, const u32* in, u32* out, u64 n, u64 k, u64 i, u64 j,
                                                  int comp, bool accumulate, bool negative, u32* slot, u32 stride) {
    constexpr u64 E = N + 3, S = 2 * E;
    u32* ssum = slot;
    u32* sp1 = slot + E * stride;
    park<N>(ssum, stride, accumulate ? load_plain<N>(in) : zero<N>());
    for (u64 kk = 0; kk < k; ++kk) {
        const u32* x = A + (i * k + kk) * S;
        const u32* y = B + (kk * n + j) * S;
        park<N>(sp1, stride, mul_mem<N>(load<N>(x), y + (comp ? E : 0)));
        const Num<N> p2 = mul_mem<N>(load<N>(x + E), y + (comp ? 0 : E));
        const Num<N> p1 = unpark<N>(sp1, stride);
        park<N>(sp1, stride, comp ? add<N>(p1, p2) : sub<N>(p1, p2));
        park<N>(ssum, stride, add<N>(unpark<N>(sp1, stride), unpark<N>(ssum, stride)));
    }
    Num<N> sum = unpark<N>(ssum, stride);
    if (negative) sum = negate<N>(sum);
    store<N>(out, sum);
}
template <int N, bool CX, bool FUSED> __device__ __forceinline__ void gemm_cell(const u32* A, const u32* B, const u32* in, u32* out,
                                                                              u64 n, u64 k, u64 i, u64 j, int comp, bool accumulate,
                                                                              bool negative) {
    constexpr u64 E = N + 3, S = CX ? 2 * E : E;
    Num<N> sum = accumulate ? load_plain<N>(in) : zero<N>();
    for (u64 kk = 0; kk < k; ++kk) {
        const u32* x = A + (i * k + kk) * S;
        const u32* y = B + (kk * n + j) * S;
        if constexpr (CX) {
            cx_step<N, FUSED>(sum, x, y, comp);
        } else {
            const Num<N> xr = load<N>(x), yr = load<N>(y);
            if constexpr (FUSED) sum = fma<N>(xr, yr, sum); else sum = addx<N>(mulx<N>(xr, yr), sum);
        }
    }
    if (negative) sum = negate<N>(sum);
    store<N>(out, sum);
}
template <int N, bool CX, bool FUSED> __global__ void __launch_bounds__(256, (parked_state<N, CX, FUSED>() ? 2 : 1)) gemm_kernel(GemmWork p) {
    constexpr u64 E = N + 3, S = CX ? 2 * E : E;
    __shared__ u32 s_chunk;
    extern __shared__ u32 gemm_park[];                              // parked_state: 2E words per thread
    for (u32 round = 0;; ++round) {
        u32 c;
        if (p.counter) {
            __syncthreads();                                        // everyone has read the previous chunk index
            if (threadIdx.x == 0) s_chunk = atomicAdd(p.counter, 1u);
            __syncthreads();
            c = s_chunk;
        } else {
            if (round) return;
            c = blockIdx.x;
        }
        if (c >= p.nchunks) return;
        const u64 g = (u64)c * p.chunk + threadIdx.x;              // work unit: an entry, or one component of one
        if (threadIdx.x >= p.chunk || g >= p.cells) continue;
        const u64 gc = CX ? g >> 1 : g;
        const int comp = CX ? (int)(g & 1) : 0;
        if (p.items) {
            u32 t = p.chunk_item[c];
            GemmItem it = p.items[t];
            while (gc >= it.cell0 + (u64)it.m * it.n) it = p.items[++t];   // owner of entry gc (empty items skipped)
            const u64 cell = gc - it.cell0, i = cell / it.n, j = cell % it.n;
            const u32* in = p.base + it.c + cell * S + comp * E;
            u32* out = p.out_override ? p.out_override + gc * S + comp * E : p.out_base + it.c + cell * S + comp * E;
            if constexpr (parked_state<N, CX, FUSED>())
                gemm_cell_parked<N>(p.base + it.a, p.base + it.b, in, out, it.n, it.k, i, j, comp, it.flags & 1, it.flags & 2,
                                    gemm_park + threadIdx.x, blockDim.x);
            else
                gemm_cell<N, CX, FUSED>(p.base + it.a, p.base + it.b, in, out, it.n, it.k, i, j, comp, it.flags & 1, it.flags & 2);
        } else {
            const u64 cells = p.m * p.n, t = gc / cells, cell = gc % cells;
            u32* out = p.C + (t * p.sc + cell) * S + comp * E;
            if constexpr (parked_state<N, CX, FUSED>())
                gemm_cell_parked<N>(p.A + t * p.sa * S, p.B + t * p.sb * S, out, out, p.n, p.k, cell / p.n, cell % p.n, comp,
                                    p.accumulate, p.negative, gemm_park + threadIdx.x, blockDim.x);
            else
                gemm_cell<N, CX, FUSED>(p.A + t * p.sa * S, p.B + t * p.sb * S, out, out, p.n, p.k, cell / p.n, cell % p.n, comp,
                                        p.accumulate, p.negative);
        }
    }
}

// Launchers.  grid == 0 asks for the number of resident blocks per SM at this block size instead (0 when
// the block's parked systems do not fit in shared memory; the LU launcher then refuses the launch too).
template <int N, bool FUSED> int launch_lu4_v(const Lu4Params& p, unsigned grid, unsigned block, cudaStream_t s) {
    const size_t smem = (size_t)(block / kLuLanes) * lu_quad_words<N>() * 4;
    if (block % kLuLanes || smem > 227 * 1024) return grid ? 1 : 0;
    if (smem > 48 * 1024) cudaFuncSetAttribute(lu4_kernel<N, FUSED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (!grid) { int b = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lu4_kernel<N, FUSED>, (int)block, smem); return b; }
    if (!p.count) return 0;
    lu4_kernel<N, FUSED><<<grid, block, smem, s>>>(p);
    return 0;
}
template <int N> int launch_lu4_n(const Lu4Params& p, unsigned grid, unsigned block, cudaStream_t s) {
    return p.fused ? launch_lu4_v<N, true>(p, grid, block, s) : launch_lu4_v<N, false>(p, grid, block, s);
}
template <int N, bool CX, bool FUSED> int launch_gemm_v(const GemmWork& p, unsigned grid, unsigned block, cudaStream_t s) {
    const size_t smem = parked_state<N, CX, FUSED>() ? (size_t)block * 2 * (N + 3) * 4 : 0;
    if (smem > 48 * 1024) cudaFuncSetAttribute(gemm_kernel<N, CX, FUSED>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (!grid) { int b = 0; cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, gemm_kernel<N, CX, FUSED>, (int)block, smem); return b; }
    if (!p.nchunks) return 0;
    gemm_kernel<N, CX, FUSED><<<grid, block, smem, s>>>(p);
    return 0;
}
template <int N> int launch_gemm_n(bool cx, bool fused, const GemmWork& p, unsigned grid, unsigned block, cudaStream_t s) {
    if (cx) return fused ? launch_gemm_v<N, true, true>(p, grid, block, s) : launch_gemm_v<N, true, false>(p, grid, block, s);
    return fused ? launch_gemm_v<N, false, true>(p, grid, block, s) : launch_gemm_v<N, false, false>(p, grid, block, s);
}
typedef int (*Lu4Launcher)(const Lu4Params&, unsigned grid, unsigned block, cudaStream_t);
typedef int (*GemmLauncher)(bool cx, bool fused, const GemmWork&, unsigned grid, unsigned block, cudaStream_t);
Lu4Launcher lu4_launcher(int limbs);
GemmLauncher gemm_launcher(int limbs);

}  // namespace lfd

#define LF_BATCHED_INSTANTIATE(N)                                                                   \
    namespace lfd {                                                                                 \
    int lu4_launch_##N(const Lu4Params& p, unsigned g, unsigned b, cudaStream_t s) { return launch_lu4_n<N>(p, g, b, s); } \
    int gemm_launch_##N(bool cx, bool f, const GemmWork& p, unsigned g, unsigned b, cudaStream_t s) { return launch_gemm_n<N>(cx, f, p, g, b, s); } \
    }
