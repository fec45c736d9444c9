// C ABI of the exact batched 4 x 4 product (the reference's experimental ExactGemm4, benchmarks/experiments/exact_gemm4/
// prototype.hpp:5-33): the host-array call and the resident form recorded into a CommandBatch.  Every component is summed
// exactly on the GPU (no host repair), so the report counts every component as a GPU component.
#include "lf_runtime.h"
#include "lf_eg4.cuh"

#include <chrono>

namespace lfr {

// Element counts of A, B and C for the shape, validated as the reference validates them (prototype.mm:14-16, 47-50):
// matrix t at t * stride, stride 0 broadcasting; inputs may overlap, output matrices may not.
static size_t eg4_extent(size_t count, size_t stride) {
    if (!count) return 0;
    const size_t v = checked_size(count - 1, stride);
    if (v > SIZE_MAX - 16) throw invalid_argument("exact_gemm4: stride overflow");
    return v + 16;
}
static void eg4_elements(int bits, const lf_exact_gemm4_shape& s, size_t n[3]) {
    validate(bits, s.count);
    if (s.count > 1 && s.stride_c < 16) throw invalid_argument("exact_gemm4: output matrices overlap");
    if (checked_size(s.count, 16) > 0xffffffffull) throw invalid_argument("exact_gemm4: grid exceeds 32 bits");
    n[0] = eg4_extent(s.count, s.stride_a);
    n[1] = eg4_extent(s.count, s.stride_b);
    n[2] = eg4_extent(s.count, s.stride_c);
}
static void eg4_run(int bits, bool cx, const lf_exact_gemm4_shape& s, const void* A, const void* B, void* C, cudaStream_t st) {
    const lfd::Eg4Params p{static_cast<const uint32_t*>(A), static_cast<const uint32_t*>(B), static_cast<uint32_t*>(C),
                           s.count, s.stride_a, s.stride_b, s.stride_c, s.accumulate ? 1 : 0, s.negative ? 1 : 0};
    lfd::eg4_kernels(bits / 32)->run(p, cx, st);
    cuda_check(cudaGetLastError(), "exact_gemm4 launch");
}

}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};

extern "C" {

int lf_engine_exact_gemm4(lf_engine* e, int bits, int complex_, const lf_exact_gemm4_shape* shape, const void* A, const void* B, void* C,
                          lf_exact_gemm4_report* report, lf_timing* timing) {
    LF_API_BEGIN
    if (!e || !shape) throw invalid_argument("null argument");
    size_t n[3];
    eg4_elements(bits, *shape, n);
    if (timing) *timing = {0, 0};
    if (report) *report = lf_exact_gemm4_report{0, 0, 0};
    if (!shape->count) return LF_OK;
    if (!A || !B || !C) throw invalid_argument("exact_gemm4: null host matrix");
    const auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const size_t es = element_bytes(bits, complex_ != 0);
    const size_t ab = checked_size(n[0], es), bb = checked_size(n[1], es), cb = checked_size(n[2], es);
    void* da = e->scratch[0].get(ab + 16);
    void* db = e->scratch[1].get(bb + 16);
    void* dc = e->scratch[2].get(cb + 16);
    cudaStream_t s = e->stream;
    cuda_check(cudaMemcpyAsync(da, A, ab, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaMemcpyAsync(db, B, bb, cudaMemcpyHostToDevice, s), "upload");
    // C is uploaded whole: the padding between output matrices comes back untouched
    cuda_check(cudaMemcpyAsync(dc, C, cb, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaEventRecord(e->e0, s), "event");
    eg4_run(bits, complex_ != 0, *shape, da, db, dc, s);
    cuda_check(cudaEventRecord(e->e1, s), "event");
    cuda_check(cudaMemcpyAsync(C, dc, cb, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (report) *report = lf_exact_gemm4_report{shape->count * 16 * (complex_ ? 2 : 1), 0, 0};
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

int lf_batch_exact_gemm4(lf_batch* bt, int bits, int complex_, const lf_exact_gemm4_shape* shape, lf_buffer* A, lf_buffer* B,
                         lf_buffer* C) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    if (!shape) throw invalid_argument("null argument");
    size_t n[3];
    eg4_elements(bits, *shape, n);
    if (!A || !B || !C) throw invalid_argument("missing exact_gemm4 buffer");
    if (C == A || C == B) throw invalid_argument("exact_gemm4: output aliases input");
    const size_t es = element_bytes(bits, complex_ != 0);
    if (A->bytes < checked_size(n[0], es) || B->bytes < checked_size(n[1], es) || C->bytes < checked_size(n[2], es))
        throw invalid_argument("exact_gemm4: undersized buffer");
    bt->retain(A);
    bt->retain(B);
    bt->retain(C, true);
    if (!shape->count) return LF_OK;
    Op o;
    o.kind = kCustom;
    const lf_exact_gemm4_shape d = *shape;
    const bool cx = complex_ != 0;
    Buffer* x = A; Buffer* y = B; Buffer* z = C;
    o.custom = [=](cudaStream_t s) { eg4_run(bits, cx, d, x->dev, y->dev, z->dev, s); };
    bt->ops.push_back(o);
    LF_API_END
}

}  // extern "C"
