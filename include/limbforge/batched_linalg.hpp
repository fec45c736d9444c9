#pragma once
// limbforge::BatchedLinalg strided batched products (the reference's include/limbforge/batched_linalg.hpp:
// 7-14, 77-98): C_b (+)= A_b B_b over ascending k, composed (mul then add) or fused (fma / cfma) steps,
// optionally negated; host and resident forms over the C ABI.
#include "engine.hpp"
#include <algorithm>
#include <memory>
#include <vector>

namespace limbforge {
struct StridedGemm {
    std::size_t count = 1, m = 0, n = 0, k = 0, stride_a = 0, stride_b = 0, stride_c = 0;
    bool accumulate = false, fused = false, negative = false;
};
// Intermediate buffers BatchedLinalg keeps for product3 (batched_linalg.hpp:77-79), in bytes.
struct BatchedWorkspaces { std::size_t idle_bytes = 0, busy_bytes = 0, busy_workspaces = 0; };
// Metadata for an external allocation of whole aligned pages holding inline MPFR significands
// (batched_linalg.hpp:53-60): offsets address little-endian 64-bit MPFR limbs of exactly the target width.  The
// allocation stays alive and unchanged until the batch has been submitted.
struct InlineComplexRecord {
    std::uint64_t real_offset = 0, imag_offset = 0;
    std::int32_t real_exponent = 0, imag_exponent = 0, real_sign = 0, imag_sign = 0;
    std::uint32_t real_status = 0, imag_status = 0;
};
static_assert(sizeof(InlineComplexRecord) == sizeof(lf_inline_complex_record), "record layout is the C ABI's");
class BatchedLinalg {
    Engine* engine_;
    // product3 intermediates: idle when no batch or unwaited submission holds them, and then reused
    std::vector<std::shared_ptr<detail::BufferRef>> spaces_;
    template <class T> Buffer<T> space(std::size_t count) {
        const std::size_t bytes = count * sizeof(T);
        for (auto& r : spaces_)
            if (lf_buffer_holders(r->h) == 0 && lf_buffer_bytes(r->h) >= bytes) return detail::Access::view<T>(r, count);
        Buffer<T> b = engine_->make_buffer<T>(count);
        spaces_.push_back(detail::Access::ref(b));
        return b;
    }
    BatchedWorkspaces tally() const {
        BatchedWorkspaces w;
        for (auto& r : spaces_) {
            const std::size_t b = lf_buffer_bytes(r->h);
            if (lf_buffer_holders(r->h) == 0) w.idle_bytes += b; else { w.busy_bytes += b; ++w.busy_workspaces; }
        }
        return w;
    }
    static lf_strided_gemm shape(const StridedGemm& s) {
        return {s.count, s.m, s.n, s.k, s.stride_a, s.stride_b, s.stride_c, s.accumulate, s.fused, s.negative};
    }
public:
    explicit BatchedLinalg(Engine& e) : engine_(&e) {}
    Timing gemm(int bits, bool complex, const StridedGemm& s, const void* A, const void* B, void* C) {
        lf_strided_gemm sh = shape(s);
        lf_timing t{};
        detail::check(lf_batched_gemm(engine_->handle(), bits, complex, &sh, A, B, C, &t));
        return detail::timing(t);
    }
    template <class T> void gemm(CommandBatch& b, const StridedGemm& s, const Buffer<T>& A, const Buffer<T>& B, Buffer<T>& C) {
        lf_strided_gemm sh = shape(s);
        detail::check(lf_batch_strided_gemm(b.handle(), detail::Format<T>::bits, detail::Format<T>::complex, &sh, A.handle(), B.handle(), C.handle()));
    }
    Timing gemm_sequential(int bits, bool complex, const StridedGemm& s, const void* A, const void* B, void* C) { return gemm(bits, complex, s, A, B, C); }
    template <class T> void gemm_sequential(CommandBatch& b, const StridedGemm& s, const Buffer<T>& A, const Buffer<T>& B, Buffer<T>& C) { gemm(b, s, A, B, C); }
    // Two-stage product C_b = (A_b B_b) D_b (batched_linalg.hpp:99-110): the intermediate
    // [first.count][first.m][first.n] lives in a workspace of this BatchedLinalg; neither stage accumulates.
    // Complex values gathered on the GPU from MPFR significands inside `allocation` (batched_linalg.hpp:146-148).
    template <class T> void import_inline_complex(CommandBatch& b, const void* allocation, std::size_t bytes,
                                                  const InlineComplexRecord* records, std::size_t count, Buffer<T>& out) {
        static_assert(detail::Format<T>::complex, "inline complex staging needs complex output");
        if (out.size() < count) throw std::invalid_argument("inline staging: undersized buffer");
        detail::check(lf_batch_import_inline_complex(b.handle(), detail::Format<T>::bits, allocation, bytes,
                                                     reinterpret_cast<const lf_inline_complex_record*>(records), count, out.handle()));
    }
    template <class T> void product3(CommandBatch& b, StridedGemm first, StridedGemm second, const Buffer<T>& A, const Buffer<T>& B,
                                     const Buffer<T>& D, Buffer<T>& C, bool negative = false) {
        if (first.count != second.count || first.m != second.m || first.n != second.k || first.accumulate || second.accumulate)
            throw std::invalid_argument("product3: incompatible shapes or accumulation");
        if (first.m && first.n > std::size_t(-1) / first.m) throw std::invalid_argument("product3: size overflow");
        first.stride_c = first.m * first.n;
        second.stride_a = first.stride_c;
        if (first.count && first.stride_c > std::size_t(-1) / first.count) throw std::invalid_argument("product3: size overflow");
        second.negative = negative;
        Buffer<T> tmp = space<T>(std::max<std::size_t>(first.count * first.stride_c, 1));
        gemm(b, first, A, B, tmp);
        gemm(b, second, tmp, D, C);
    }
    // Retained intermediates (batched_linalg.hpp:78-79): release drops the idle ones now and detaches the busy
    // ones, which are freed when their batches let go; the result is what was retained before the release.
    BatchedWorkspaces workspaces() const { return tally(); }
    BatchedWorkspaces release_workspaces() { const BatchedWorkspaces w = tally(); spaces_.clear(); return w; }
};
}  // namespace limbforge
