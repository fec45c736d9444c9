// C ABI of the batched small-matrix paths: Engine::lu4 / CommandBatch::lu4 (engine.hpp:164,208;
// engine.mm:199-222,363-374,515-521) and BatchedLinalg::gemm host and resident forms
// (batched_linalg.hpp:86,97; batched_linalg.mm:150-173), with the reference's validation rules.
#include <algorithm>
#include "lf_runtime.h"
#include "lf_batched.cuh"

namespace lfr {

void launch_lu4(int bits, const lf_batched4& s, const void* A, const void* B, void* X, void* det, uint32_t* status,
                cudaStream_t st) {
    if (!s.count) return;
    lfd::Lu4Params p{static_cast<const uint32_t*>(A), static_cast<const uint32_t*>(B), static_cast<uint32_t*>(X),
                     static_cast<uint32_t*>(det), status, s.count, s.rhs, s.fused, s.determinant, s.inverse};
    const uint64_t lanes = (uint64_t)s.count * lfd::kLuLanes;           // one quad of lanes per system
    if (lfd::lu4_launcher(bits / 32)(p, (unsigned)std::min<uint64_t>((lanes + 63) / 64, 1u << 30), 64, st))
        throw runtime_error("lu4 launch: block does not fit");
    cuda_check(cudaGetLastError(), "lu4 launch");
}
void launch_strided_gemm(int bits, bool complex, const lf_strided_gemm& s, const void* A, const void* B, void* C,
                         cudaStream_t st) {
    lfd::GemmWork p{};
    p.A = static_cast<const uint32_t*>(A); p.B = static_cast<const uint32_t*>(B); p.C = static_cast<uint32_t*>(C);
    p.m = s.m; p.n = s.n; p.k = s.k; p.sa = s.stride_a; p.sb = s.stride_b; p.sc = s.stride_c;
    p.accumulate = s.accumulate; p.negative = s.negative;
    p.cells = (uint64_t)s.count * s.m * s.n * (complex ? 2 : 1);        // work units
    p.chunk = 128;
    p.nchunks = (uint32_t)((p.cells + 127) / 128);
    if (!p.nchunks) return;
    lfd::gemm_launcher(bits / 32)(complex, s.fused != 0, p, p.nchunks, 128, st);
    cuda_check(cudaGetLastError(), "strided gemm launch");
}

Lu4Sizes lu4_elements(int bits, const lf_batched4& s) {                         // engine.mm lu4_elements
    validate(bits, s.count);
    if (s.count > 0xffffffffull / 16) throw invalid_argument("batched 4x4 exceeds 32-bit indexing");
    if (s.inverse && s.rhs) throw invalid_argument("inverse uses no right-hand sides");
    unsigned R = s.inverse ? 4 : s.rhs;
    return {s.count * 16, checked_size(s.count * 4, s.rhs), checked_size(s.count * 4, R), s.determinant ? s.count : 0, s.count};
}
static size_t mul_size(size_t a, size_t b) {
    if (a && b > SIZE_MAX / a) throw invalid_argument("batched algebra: size overflow");
    return a * b;
}
static size_t extent(size_t count, size_t stride, size_t matrix) {                      // batched_linalg.mm:20
    if (!count || !matrix) return 0;
    size_t n = mul_size(count - 1, stride);
    if (matrix > SIZE_MAX - n) throw invalid_argument("batched algebra: stride overflow");
    return n + matrix;
}
struct SgSizes { size_t A, B, C; };
static SgSizes sg_elements(int bits, const lf_strided_gemm& s) {                       // batched_linalg.mm:163-167
    if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
    size_t as = mul_size(s.m, s.k), bs = mul_size(s.k, s.n), cs = mul_size(s.m, s.n);
    if (mul_size(s.count, cs) > 0xffffffffull) throw invalid_argument("batched algebra: grid exceeds 32-bit indexing");
    if (s.count > 1 && s.stride_c < cs) throw invalid_argument("batched GEMM: output matrices overlap");
    return {extent(s.count, s.stride_a, as), extent(s.count, s.stride_b, bs), extent(s.count, s.stride_c, cs)};
}

}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};

extern "C" {

int lf_engine_lu4(lf_engine* e, int bits, const lf_batched4* shape, const void* A, const void* B, void* X, void* det,
                  uint32_t* status, lf_timing* timing) {
    LF_API_BEGIN
    if (!e || !shape) throw invalid_argument("null argument");
    const lf_batched4 s = *shape;
    Lu4Sizes n = lu4_elements(bits, s);
    const unsigned R = s.inverse ? 4 : s.rhs;
    if (timing) *timing = {0, 0};
    if (!s.count) return LF_OK;
    if (!A || (s.rhs && !B) || (R && !X) || (s.determinant && !det) || !status) throw invalid_argument("null batched 4x4 buffer");
    auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const size_t es = element_bytes(bits, true);
    void* dA = e->scratch[0].get(n.A * es);
    void* dB = n.B ? e->scratch[1].get(n.B * es) : nullptr;
    void* dX = n.X ? e->scratch[2].get(n.X * es) : nullptr;
    void* dD = n.det ? e->scratch[3].get(n.det * es) : nullptr;
    uint32_t* dS = static_cast<uint32_t*>(e->scratch[4].get(n.status * 4));
    cudaStream_t st = e->stream;
    cuda_check(cudaMemcpyAsync(dA, A, n.A * es, cudaMemcpyHostToDevice, st), "upload");
    if (n.B) cuda_check(cudaMemcpyAsync(dB, B, n.B * es, cudaMemcpyHostToDevice, st), "upload");
    cuda_check(cudaEventRecord(e->e0, st), "event");
    launch_lu4(bits, s, dA, dB, dX, dD, dS, st);
    cuda_check(cudaEventRecord(e->e1, st), "event");
    if (n.X) cuda_check(cudaMemcpyAsync(X, dX, n.X * es, cudaMemcpyDeviceToHost, st), "download");
    if (n.det) cuda_check(cudaMemcpyAsync(det, dD, n.det * es, cudaMemcpyDeviceToHost, st), "download");
    cuda_check(cudaMemcpyAsync(status, dS, n.status * 4, cudaMemcpyDeviceToHost, st), "download");
    cuda_check(cudaStreamSynchronize(st), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

int lf_batch_lu4(lf_batch* bt, int bits, const lf_batched4* shape, lf_buffer* A, lf_buffer* B, lf_buffer* X,
                 lf_buffer* det, lf_buffer* status) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    if (!shape) throw invalid_argument("null shape");
    const lf_batched4 s = *shape;
    Lu4Sizes n = lu4_elements(bits, s);
    const size_t es = element_bytes(bits, true);
    auto need = [](Buffer* b, size_t bytes, bool required) {
        if (!required) return;
        if (!b || b->bytes < bytes) throw invalid_argument("batched 4x4: undersized buffer");
    };
    need(A, n.A * es, n.A > 0); need(B, n.B * es, n.B > 0); need(X, n.X * es, n.X > 0);
    need(det, n.det * es, n.det > 0); need(status, n.status * 4, n.status > 0);
    if (n.A) bt->retain(A);
    if (n.B) bt->retain(B);
    if (n.X) bt->retain(X, true);
    if (n.det) bt->retain(det, true);
    if (n.status) bt->retain(status, true);
    if (!s.count) return LF_OK;
    Op o;
    o.kind = kLu4; o.bits = bits; o.lu = s;
    o.a = A; o.b = n.B ? B : nullptr; o.c = n.X ? X : nullptr; o.out = n.det ? det : nullptr; o.e = status;
    bt->ops.push_back(o);
    LF_API_END
}

int lf_batched_gemm(lf_engine* e, int bits, int complex_, const lf_strided_gemm* shape, const void* A, const void* B,
                    void* C, lf_timing* timing) {
    LF_API_BEGIN
    if (!e || !shape) throw invalid_argument("null argument");
    const lf_strided_gemm s = *shape;
    SgSizes n = sg_elements(bits, s);
    if (timing) *timing = {0, 0};
    if (!n.C) return LF_OK;
    if ((n.A && !A) || (n.B && !B) || !C) throw invalid_argument("null batched algebra operand");
    auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const size_t es = element_bytes(bits, complex_ != 0);
    void* dA = e->scratch[0].get(n.A * es + 16);
    void* dB = e->scratch[1].get(n.B * es + 16);
    void* dC = e->scratch[2].get(n.C * es);
    cudaStream_t st = e->stream;
    if (n.A) cuda_check(cudaMemcpyAsync(dA, A, n.A * es, cudaMemcpyHostToDevice, st), "upload");
    if (n.B) cuda_check(cudaMemcpyAsync(dB, B, n.B * es, cudaMemcpyHostToDevice, st), "upload");
    cuda_check(cudaMemcpyAsync(dC, C, n.C * es, cudaMemcpyHostToDevice, st), "upload");   // padding between outputs is kept
    cuda_check(cudaEventRecord(e->e0, st), "event");
    launch_strided_gemm(bits, complex_ != 0, s, dA, dB, dC, st);
    cuda_check(cudaEventRecord(e->e1, st), "event");
    cuda_check(cudaMemcpyAsync(C, dC, n.C * es, cudaMemcpyDeviceToHost, st), "download");
    cuda_check(cudaStreamSynchronize(st), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

int lf_batch_strided_gemm(lf_batch* bt, int bits, int complex_, const lf_strided_gemm* shape, lf_buffer* A, lf_buffer* B,
                          lf_buffer* C) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    if (!shape) throw invalid_argument("null shape");
    const lf_strided_gemm s = *shape;
    SgSizes n = sg_elements(bits, s);
    const size_t es = element_bytes(bits, complex_ != 0);
    auto size_ok = [](Buffer* b, size_t bytes) { if (bytes && (!b || b->bytes < bytes)) throw invalid_argument("batched algebra: undersized buffer"); };
    size_ok(A, n.A * es); size_ok(B, n.B * es); size_ok(C, n.C * es);
    if (C && (C == A || C == B)) throw invalid_argument("batched algebra: output aliases an input");
    if (!s.count || !n.C) return LF_OK;
    if (n.A) bt->retain(A);
    if (n.B) bt->retain(B);
    bt->retain(C, true);
    Op o;
    o.kind = kStridedGemm; o.bits = bits; o.complex = complex_ != 0; o.sg = s;
    o.a = A; o.b = B; o.out = C;
    bt->ops.push_back(o);
    LF_API_END
}

}  // extern "C"
