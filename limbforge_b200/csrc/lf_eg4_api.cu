// C ABI of the exact batched 4 x 4 product (the reference's experimental ExactGemm4, benchmarks/experiments/exact_gemm4/
// prototype.hpp:5-33): the host-array call and the resident form recorded into a CommandBatch.  Every component is summed
// exactly on the GPU (no host repair), so the report counts every component as a GPU component.
#include "lf_runtime.h"
#include "lf_eg4.cuh"

#include <algorithm>
#include <chrono>
#include <cstring>

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

// Host copy split over the host threads (large staging copies run at memory bandwidth rather than one core's rate).
static void par_copy(void* dst, const void* src, size_t bytes) {
    constexpr size_t kPiece = size_t(1) << 20;
    const long long pieces = (long long)((bytes + kPiece - 1) / kPiece);
#pragma omp parallel for schedule(static) if (pieces > 1)
    for (long long q = 0; q < pieces; ++q) {
        const size_t off = (size_t)q * kPiece, len = std::min(kPiece, bytes - off);
        std::memcpy(static_cast<char*>(dst) + off, static_cast<const char*>(src) + off, len);
    }
}

// Host arrays with dense strides (16 elements, or 0 for a broadcast input): the matrices run in chunks through two
// pinned staging slots and two streams, so that the host copies of one chunk overlap the transfers and the product
// of the other.  Returns the summed device time of the products.
static double eg4_host_pipelined(Engine* e, int bits, bool cx, const lf_exact_gemm4_shape& s, const void* A, const void* B, void* C) {
    constexpr size_t kChunkBytes = size_t(8) << 20;               // per staged operand and slot
    const size_t per = 16 * element_bytes(bits, cx);              // one matrix
    const size_t cm = std::max<size_t>(1, kChunkBytes / per);     // matrices per chunk
    const size_t chunks = (s.count + cm - 1) / cm;
    const bool ba = s.stride_a == 0, bb = s.stride_b == 0;
    const size_t slot = ((ba ? 0 : cm) + (bb ? 0 : cm) + cm) * per;
    char* pin[2] = {static_cast<char*>(e->staging[0].get(slot)), static_cast<char*>(e->staging[1].get(slot))};
    char* dev[2] = {static_cast<char*>(e->scratch[0].get(slot)), static_cast<char*>(e->scratch[1].get(slot))};
    char* da0 = static_cast<char*>(e->scratch[2].get(per)), *db0 = static_cast<char*>(e->scratch[3].get(per));
    if (ba) cuda_check(cudaMemcpy(da0, A, per, cudaMemcpyHostToDevice), "upload");
    if (bb) cuda_check(cudaMemcpy(db0, B, per, cudaMemcpyHostToDevice), "upload");
    cudaStream_t st[2] = {nullptr, nullptr};
    cudaEvent_t done[2] = {nullptr, nullptr}, k0[2] = {nullptr, nullptr}, k1[2] = {nullptr, nullptr};
    double gpu = 0;
    size_t pending[2] = {SIZE_MAX, SIZE_MAX};                       // chunk whose result sits in slot q
    auto drain = [&](int q) {                                       // wait for slot q's chunk and copy its C out
        if (pending[q] == SIZE_MAX) return;
        cuda_check(cudaEventSynchronize(done[q]), "execution");
        float ms = 0;
        cudaEventElapsedTime(&ms, k0[q], k1[q]);
        gpu += ms * 1e-3;
        const size_t t0 = pending[q] * cm, nt = std::min(cm, s.count - t0);
        const size_t coff = ((ba ? 0 : cm) + (bb ? 0 : cm)) * per;
        par_copy(static_cast<char*>(C) + t0 * per, pin[q] + coff, nt * per);
        pending[q] = SIZE_MAX;
    };
    try {
        for (int q = 0; q < 2; ++q) {
            cuda_check(cudaStreamCreateWithFlags(&st[q], cudaStreamNonBlocking), "stream");
            cuda_check(cudaEventCreate(&done[q]), "event");
            cuda_check(cudaEventCreate(&k0[q]), "event");
            cuda_check(cudaEventCreate(&k1[q]), "event");
        }
        for (size_t i = 0; i < chunks; ++i) {
            const int q = int(i & 1);
            drain(q);
            const size_t t0 = i * cm, nt = std::min(cm, s.count - t0);
            char* h = pin[q];
            size_t off = 0, aoff = 0, boff = 0;
            if (!ba) { par_copy(h, static_cast<const char*>(A) + t0 * per, nt * per); aoff = off; off += cm * per; }
            if (!bb) { par_copy(h + off, static_cast<const char*>(B) + t0 * per, nt * per); boff = off; off += cm * per; }
            const size_t coff = off;
            if (s.accumulate) par_copy(h + coff, static_cast<const char*>(C) + t0 * per, nt * per);
            char* d = dev[q];
            if (!ba) cuda_check(cudaMemcpyAsync(d + aoff, h + aoff, nt * per, cudaMemcpyHostToDevice, st[q]), "upload");
            if (!bb) cuda_check(cudaMemcpyAsync(d + boff, h + boff, nt * per, cudaMemcpyHostToDevice, st[q]), "upload");
            if (s.accumulate) cuda_check(cudaMemcpyAsync(d + coff, h + coff, nt * per, cudaMemcpyHostToDevice, st[q]), "upload");
            lf_exact_gemm4_shape cs = s;
            cs.count = nt;
            cuda_check(cudaEventRecord(k0[q], st[q]), "event");
            eg4_run(bits, cx, cs, ba ? da0 : d + aoff, bb ? db0 : d + boff, d + coff, st[q]);
            cuda_check(cudaEventRecord(k1[q], st[q]), "event");
            cuda_check(cudaMemcpyAsync(h + coff, d + coff, nt * per, cudaMemcpyDeviceToHost, st[q]), "download");
            cuda_check(cudaEventRecord(done[q], st[q]), "event");
            pending[q] = i;
        }
        drain(int(chunks & 1));
        drain(int((chunks + 1) & 1));
    } catch (...) {
        for (int q = 0; q < 2; ++q) if (st[q]) cudaStreamSynchronize(st[q]);
        for (int q = 0; q < 2; ++q) {
            if (st[q]) cudaStreamDestroy(st[q]);
            if (done[q]) cudaEventDestroy(done[q]);
            if (k0[q]) cudaEventDestroy(k0[q]);
            if (k1[q]) cudaEventDestroy(k1[q]);
        }
        throw;
    }
    for (int q = 0; q < 2; ++q) {
        cudaStreamDestroy(st[q]); cudaEventDestroy(done[q]); cudaEventDestroy(k0[q]); cudaEventDestroy(k1[q]);
    }
    return gpu;
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
    const bool dense = (shape->stride_a == 16 || shape->stride_a == 0) && (shape->stride_b == 16 || shape->stride_b == 0) &&
                       (shape->stride_c == 16 || shape->count == 1);
    if (dense) {
        lf_exact_gemm4_shape d = *shape;
        d.stride_c = 16;
        const double g = eg4_host_pipelined(e, bits, complex_ != 0, d, A, B, C);
        if (report) *report = lf_exact_gemm4_report{shape->count * 16 * (complex_ ? 2 : 1), 0, 0};
        if (timing) *timing = {g, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
        return LF_OK;
    }
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
