#pragma once
// wolfnum::experimental::ExactGemm4, the exact batched 4 x 4 product (the reference's
// benchmarks/experiments/exact_gemm4/prototype.hpp:4-33), over the C ABI.  Fixed row-major 4 x 4 matrices; matrix t of
// A, B and C at t * stride elements, stride 0 broadcasting an input.  Each real component is RN(C_old + sum of exact
// signed products), then optionally negated exactly; C_old is left out without accumulation; complex components sum
// eight real products with one rounding; statuses are ORed per component across its operands.  Every component is
// summed exactly on the GPU, so the report counts no host components, no read inside the batch is provisional, and a
// ticket resolves once the batch's submission has been waited for.
#include "engine.hpp"
#include <atomic>
#include <chrono>
#include <memory>

namespace wolfnum::experimental {
struct ExactGemm4Shape { std::size_t count = 1, stride_a = 16, stride_b = 16, stride_c = 16; bool accumulate = false, negative = false; };
struct ExactGemm4Report { std::size_t gpu_components = 0, host_components = 0; bool provisional_reads = false; };
struct ExactGemm4State { std::atomic<bool> done{false}; ExactGemm4Report report; };

class ExactGemm4Ticket {
    std::shared_ptr<ExactGemm4State> state_;
    friend class ExactGemm4;
    explicit ExactGemm4Ticket(std::shared_ptr<ExactGemm4State> s) : state_(std::move(s)) {}
public:
    bool resolved() const { return state_ && state_->done.load(std::memory_order_acquire); }
    ExactGemm4Report report() const {
        if (!resolved()) throw std::logic_error("exact GEMM4: wait for submission before reading report");
        return state_->report;
    }
};

class ExactGemm4 {
    limbforge::Engine* engine_;
    static lf_exact_gemm4_shape raw(const ExactGemm4Shape& s) {
        return lf_exact_gemm4_shape{s.count, s.stride_a, s.stride_b, s.stride_c, s.accumulate, s.negative};
    }
public:
    explicit ExactGemm4(limbforge::Engine& e) : engine_(&e) {}
    ExactGemm4(const ExactGemm4&) = delete;
    ExactGemm4& operator=(const ExactGemm4&) = delete;

    // Resident buffers, recorded into the batch (prototype.hpp:28-30).
    template <class T> ExactGemm4Ticket gemm(limbforge::CommandBatch& b, const ExactGemm4Shape& s, const limbforge::Buffer<T>& a,
                                             const limbforge::Buffer<T>& bb, limbforge::Buffer<T>& c) {
        static_assert(limbforge::detail::Format<T>::bits != 0, "arithmetic elements required");
        const lf_exact_gemm4_shape d = raw(s);
        limbforge::detail::check(lf_batch_exact_gemm4(b.handle(), limbforge::detail::Format<T>::bits, limbforge::detail::Format<T>::complex,
                                                      &d, a.handle(), bb.handle(), c.handle()));
        auto state = std::make_shared<ExactGemm4State>();
        state->report.gpu_components = s.count * 16 * (limbforge::detail::Format<T>::complex ? 2 : 1);
        b.on_wait([state] { state->done.store(true, std::memory_order_release); });
        return ExactGemm4Ticket(state);
    }
    // Host arrays (prototype.hpp:32): c is read (with accumulation) and written in place.
    limbforge::Timing gemm(int bits, bool complex, const ExactGemm4Shape& s, const void* a, const void* b, void* c,
                           ExactGemm4Report* report = nullptr) {
        const lf_exact_gemm4_shape d = raw(s);
        lf_exact_gemm4_report r{};
        lf_timing t{};
        limbforge::detail::check(lf_engine_exact_gemm4(engine_->handle(), bits, complex, &d, a, b, c, &r, &t));
        if (report) *report = ExactGemm4Report{r.gpu_components, r.host_components, r.provisional_reads != 0};
        return limbforge::detail::timing(t);
    }
};
}  // namespace wolfnum::experimental
