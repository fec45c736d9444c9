#pragma once
// limbforge::BatchedLinalg strided batched products (the reference's include/limbforge/batched_linalg.hpp:
// 7-14, 77-98): C_b (+)= A_b B_b over ascending k, composed (mul then add) or fused (fma / cfma) steps,
// optionally negated; host and resident forms over the C ABI.
#include "engine.hpp"

namespace limbforge {
struct StridedGemm {
    std::size_t count = 1, m = 0, n = 0, k = 0, stride_a = 0, stride_b = 0, stride_c = 0;
    bool accumulate = false, fused = false, negative = false;
};
class BatchedLinalg {
    Engine* engine_;
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
};
}  // namespace limbforge
