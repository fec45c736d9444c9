#pragma once
// limbforge::Engine / Buffer / CommandBatch / Submission (the reference's include/limbforge/engine.hpp
// interface) as inline wrappers over the C ABI of liblimbforge_b200.so (include/limbforge_b200.h).
// Errors are rethrown as the reference's exception classes: std::invalid_argument, std::logic_error,
// std::runtime_error.
#include "core.hpp"
#include "../limbforge_b200.h"
#include <cstddef>
#include <cstdint>
#include <functional>
#include <future>
#include <memory>
#include <stdexcept>
#include <string>
#include <utility>
#include <vector>

namespace limbforge {
enum class Operation { add, sub, mul, div, complex_add, complex_mul, complex_div, square, sqrt, fma, fms, complex_fma, complex_fms };
inline bool operation_is_complex(Operation op) { return (int(op) >= 4 && int(op) <= 6) || op == Operation::complex_fma || op == Operation::complex_fms; }
inline bool operation_is_unary(Operation op) { return op == Operation::square || op == Operation::sqrt; }
inline bool operation_is_ternary(Operation op) { return int(op) >= 9 && int(op) <= 12; }
inline bool operation_is_valid(Operation op) { return int(op) >= 0 && int(op) <= 12; }
struct Timing { double gpu_seconds, wall_seconds; };
struct Broadcast { std::size_t stride = 1, period = 0; };
inline std::size_t broadcast_elements(std::size_t count, Broadcast b) {
    if (!b.stride) throw std::invalid_argument("broadcast stride must be positive");
    std::size_t n = count / b.stride + (count % b.stride != 0);
    return b.period && b.period < n ? b.period : n;
}
struct EngineOptions { unsigned threads_per_threadgroup = 0; bool cooperative_reductions = true; bool cooperative_recurrence = true; };
struct Batched4 { std::size_t count = 0; unsigned rhs = 0; bool inverse = false, determinant = false, fused = false; };
struct PipelineInfo { unsigned simd_width, max_threads, threads_per_threadgroup; };
// Segmented dot products: out[i] = sum_{k<length} a[i*length+k] * b[i*length+k] (or b[k] when shared_right),
// as the sequential fma / cfma chain from k = 0.
struct SegmentedDot { std::size_t segments = 0, length = 0; bool shared_right = false; };
// Shape of Engine::vector_recurrence (the reference's engine.hpp:37-49); that entry point is declared for source
// compatibility and is not provided by this library (it throws std::runtime_error).
struct VectorRecurrence {
    std::size_t lanes = 0; unsigned steps = 0;
    unsigned lanes_per_weight = 1;
    bool affine = false, matrix = false, all_steps = false, reverse = false, tangent = false;
    unsigned lanes_per_base = 1, lanes_per_tangent = 1;
    bool fused = false;
};
// Kernels to prepare ahead of use (Engine::prewarm).  The kernels are compiled ahead for sm_100a; a prewarm
// validates the widths and operations and loads the element-wise kernels of `operations` for every width.
struct Prewarm {
    std::vector<int> bits;
    std::vector<Operation> operations;
    bool recurrence = false, reductions = false;
    std::vector<VectorRecurrence> vector_shapes;
    std::vector<SegmentedDot> real_dots, complex_dots;
    std::vector<Batched4> lu4;
};

namespace detail {
inline void check(int rc) {
    if (rc == LF_OK) return;
    const std::string m = lf_last_error();
    if (rc == LF_INVALID_ARGUMENT) throw std::invalid_argument(m);
    if (rc == LF_LOGIC_ERROR) throw std::logic_error(m);
    throw std::runtime_error(m);
}
inline Timing timing(const lf_timing& t) { return {t.gpu_seconds, t.wall_seconds}; }
template <class T> struct Format;
template <int N> struct Format<Number<N>> { static constexpr int bits = 32 * N; static constexpr bool complex = false; };
template <int N> struct Format<Complex<N>> { static constexpr int bits = 32 * N; static constexpr bool complex = true; };
template <> struct Format<std::uint32_t> { static constexpr int bits = 0; static constexpr bool complex = false; };
template <> struct Format<std::int32_t> { static constexpr int bits = 0; static constexpr bool complex = false; };
struct BufferRef {
    lf_buffer* h = nullptr;
    explicit BufferRef(lf_buffer* b) : h(b) {}
    ~BufferRef() { if (h) lf_buffer_release(h); }
};
struct Access;
}  // namespace detail

template <class T> class Buffer {
    std::shared_ptr<detail::BufferRef> ref_;
    std::size_t count_ = 0;
    Buffer(std::shared_ptr<detail::BufferRef> r, std::size_t n) : ref_(std::move(r)), count_(n) {}
    friend class Engine; friend class CommandBatch; friend struct detail::Access;
public:
    Buffer() = default;
    std::size_t size() const { return count_; }
    lf_buffer* handle() const { return ref_ ? ref_->h : nullptr; }
    T* mapped() { void* p = nullptr; detail::check(lf_buffer_mapped(handle(), &p)); return static_cast<T*>(p); }
    const T* mapped() const { void* p = nullptr; detail::check(lf_buffer_mapped(handle(), &p)); return static_cast<const T*>(p); }
    void upload(const T* source, std::size_t count) {
        if (count > count_) throw std::invalid_argument("upload exceeds buffer");
        detail::check(lf_buffer_upload(handle(), source, count * sizeof(T)));
    }
    void download(T* target, std::size_t count) const {
        if (count > count_) throw std::invalid_argument("download exceeds buffer");
        detail::check(lf_buffer_download(handle(), target, count * sizeof(T)));
    }
};
namespace detail {
struct Access {
    template <class T> static lf_buffer* h(const Buffer<T>& b) { return b.handle(); }
    template <class T> static std::shared_ptr<BufferRef> ref(const Buffer<T>& b) { return b.ref_; }
    template <class T> static Buffer<T> view(std::shared_ptr<BufferRef> r, std::size_t n) { return Buffer<T>(std::move(r), n); }
};
}

class Submission {
    struct Del { void operator()(lf_submission* s) const { lf_submission_destroy(s); } };
    std::unique_ptr<lf_submission, Del> s_;
    std::vector<std::function<void()>> done_;     // run once waited for (tickets of operations in the batch)
    Submission(lf_submission* s, std::vector<std::function<void()>> done) : s_(s), done_(std::move(done)) {}
    friend class CommandBatch;
public:
    Submission() = default;
    bool ready() const {
        if (!s_) throw std::logic_error("empty submission");
        int r = 0; detail::check(lf_submission_ready(s_.get(), &r)); return r != 0;
    }
    Timing wait() {
        if (!s_) throw std::logic_error("empty submission");
        lf_timing t{}; detail::check(lf_submission_wait(s_.get(), &t));
        for (auto& f : done_) f();
        done_.clear();
        return detail::timing(t);
    }
};

class CommandBatch {
    struct Del { void operator()(lf_batch* b) const { lf_batch_destroy(b); } };
    std::unique_ptr<lf_batch, Del> b_;
    std::vector<std::function<void()>> done_;
    explicit CommandBatch(lf_batch* b) : b_(b) {}
    friend class Engine;
    lf_batch* open() const { if (!b_) throw std::logic_error("batch already submitted or moved"); return b_.get(); }
    template <class T> void encode(Operation op, const Buffer<T>& a, const Buffer<T>* b, const Buffer<T>* c, Buffer<T>& out,
                                   std::size_t count, Broadcast bi, Broadcast ci) {
        detail::check(lf_batch_run(open(), detail::Format<T>::bits, detail::Format<T>::complex, int(op), a.handle(),
                                   b ? b->handle() : nullptr, c ? c->handle() : nullptr, out.handle(), count,
                                   lf_broadcast{bi.stride, bi.period}, lf_broadcast{ci.stride, ci.period}));
    }
public:
    lf_batch* handle() const { return b_.get(); }
    // f runs when the submission of this batch has been waited for.
    void on_wait(std::function<void()> f) { open(); done_.push_back(std::move(f)); }
    template <class T> void run(Operation op, const Buffer<T>& a, const Buffer<T>& b, Buffer<T>& out) {
        if (operation_is_unary(op) || operation_is_ternary(op)) throw std::invalid_argument("operation requires a different number of inputs");
        if (a.size() != b.size() || a.size() != out.size()) throw std::invalid_argument("buffer counts must match");
        encode<T>(op, a, &b, nullptr, out, a.size(), {}, {});
    }
    template <class T> void run(Operation op, const Buffer<T>& a, const Buffer<T>& b, Buffer<T>& out, Broadcast b_index) {
        if (operation_is_unary(op) || operation_is_ternary(op)) throw std::invalid_argument("operation requires a different number of inputs");
        if (a.size() != out.size() || b.size() < broadcast_elements(a.size(), b_index)) throw std::invalid_argument("buffer counts do not match the broadcast");
        encode<T>(op, a, &b, nullptr, out, a.size(), b_index, {});
    }
    template <class T> void run(Operation op, const Buffer<T>& a, const Buffer<T>& b, const Buffer<T>& c, Buffer<T>& out, Broadcast b_index, Broadcast c_index) {
        if (!operation_is_ternary(op)) throw std::invalid_argument("operation does not take three inputs");
        if (a.size() != out.size() || b.size() < broadcast_elements(a.size(), b_index) || c.size() < broadcast_elements(a.size(), c_index))
            throw std::invalid_argument("buffer counts do not match the broadcast");
        encode(op, a, &b, &c, out, a.size(), b_index, c_index);
    }
    template <class T> void run(Operation op, const Buffer<T>& a, const Buffer<T>& b, const Buffer<T>& c, Buffer<T>& out) {
        if (!operation_is_ternary(op)) throw std::invalid_argument("operation does not take three inputs");
        if (a.size() != b.size() || a.size() != c.size() || a.size() != out.size()) throw std::invalid_argument("buffer counts must match");
        encode(op, a, &b, &c, out, a.size(), {}, {});
    }
    template <class T> void run(Operation op, const Buffer<T>& a, Buffer<T>& out) {
        if (!operation_is_unary(op)) throw std::invalid_argument("operation requires two inputs");
        if (a.size() != out.size()) throw std::invalid_argument("buffer counts must match");
        encode(op, a, static_cast<const Buffer<T>*>(nullptr), static_cast<const Buffer<T>*>(nullptr), out, a.size(), {}, {});
    }
    template <class T> void lu4(const Batched4& s, const Buffer<T>& A, const Buffer<T>& B, Buffer<T>& X, Buffer<T>& det,
                                Buffer<std::uint32_t>& status) {
        static_assert(detail::Format<T>::complex, "batched 4x4 systems use complex buffers");
        lf_batched4 sh{s.count, s.rhs, s.inverse, s.determinant, s.fused};
        detail::check(lf_batch_lu4(open(), detail::Format<T>::bits, &sh, A.handle(), B.handle(), X.handle(), det.handle(), status.handle()));
    }
    // Precision cast (exact widening, RNE narrowing, complex componentwise) and the adjacent-pair tree sum.
    template <class From, class To> void cast(const Buffer<From>& in, Buffer<To>& out) {
        static_assert(detail::Format<From>::complex == detail::Format<To>::complex, "cast keeps real or complex");
        if (in.size() != out.size()) throw std::invalid_argument("cast buffer counts must match");
        detail::check(lf_batch_cast(open(), detail::Format<From>::bits, detail::Format<To>::bits, detail::Format<To>::complex,
                                    in.handle(), out.handle(), in.size()));
    }
    template <class T> void segmented_dot(const SegmentedDot& shape, const Buffer<T>& a, const Buffer<T>& b, Buffer<T>& out) {
        static_assert(detail::Format<T>::bits, "segmented dots use arithmetic buffers");
        lf_segmented_dot d{shape.segments, shape.length, shape.shared_right};
        detail::check(lf_batch_segmented_dot(open(), detail::Format<T>::bits, detail::Format<T>::complex, &d, a.handle(), b.handle(),
                                             out.handle()));
    }
    // Declared for source compatibility with the reference; not provided by this library.
    template <class T> void vector_recurrence(const VectorRecurrence&, const Buffer<T>&, const Buffer<T>&, const Buffer<T>&, const Buffer<T>&,
                                              Buffer<T>&, const Buffer<T>& = Buffer<T>(), const Buffer<T>& = Buffer<T>(),
                                              const Buffer<T>& = Buffer<T>()) {
        static_assert(detail::Format<T>::complex, "vector recurrences use complex buffers");
        throw std::runtime_error("vector_recurrence is not provided by this library");
    }
    template <class T> void tree_sum(const Buffer<T>& input, Buffer<T>& out) {
        if (out.size() != 1) throw std::invalid_argument("tree_sum output must contain one element");
        detail::check(lf_batch_tree_sum(open(), detail::Format<T>::bits, detail::Format<T>::complex, input.handle(), out.handle(),
                                        input.size()));
    }
    Submission submit() {
        lf_submission* s = nullptr;
        detail::check(lf_batch_submit(open(), &s));
        b_.reset();
        return Submission(s, std::move(done_));
    }
};

// One Engine per host thread.
class Engine {
    struct Del { void operator()(lf_engine* e) const { lf_engine_destroy(e); } };
    std::unique_ptr<lf_engine, Del> e_;
public:
    explicit Engine(EngineOptions options = {}) {
        lf_engine_options o{options.threads_per_threadgroup, options.cooperative_reductions, options.cooperative_recurrence, 0};
        lf_engine* e = nullptr;
        detail::check(lf_engine_create(&o, &e));
        e_.reset(e);
    }
    Engine(const Engine&) = delete;
    Engine& operator=(const Engine&) = delete;
    lf_engine* handle() const { return e_.get(); }
    std::string device_name() const { char b[256]; detail::check(lf_engine_device_name(e_.get(), b, sizeof b)); return b; }
    // Validates the request and loads the element-wise kernels it names; the other fields need no preparation.
    void prewarm(const Prewarm& request) {
        std::vector<int> ops;
        for (Operation op : request.operations) ops.push_back(int(op));
        detail::check(lf_engine_prewarm(e_.get(), request.bits.data(), request.bits.size(), ops.data(), ops.size()));
    }
    // The same on a background thread; errors surface from the future.
    std::future<void> prewarm_async(Prewarm request) {
        return std::async(std::launch::async, [this, r = std::move(request)]() { prewarm(r); });
    }
    PipelineInfo pipeline_info(int bits, Operation op) {
        PipelineInfo p{};
        detail::check(lf_engine_pipeline_info(e_.get(), bits, int(op), &p.simd_width, &p.max_threads, &p.threads_per_threadgroup));
        return p;
    }
    Timing segmented_dot(int bits, bool complex, const SegmentedDot& shape, const void* a, const void* b, void* out) {
        lf_segmented_dot d{shape.segments, shape.length, shape.shared_right};
        lf_timing t{}; detail::check(lf_engine_segmented_dot(e_.get(), bits, complex, &d, a, b, out, &t)); return detail::timing(t);
    }
    Timing recurrence(int bits, const void* seeds, const void* weights, void* out, std::size_t count, unsigned steps,
                      unsigned states_per_weight = 1) {
        lf_timing t{};
        detail::check(lf_engine_recurrence(e_.get(), bits, seeds, weights, out, count, steps, states_per_weight, &t));
        return detail::timing(t);
    }
    // Declared for source compatibility with the reference; not provided by this library.
    Timing vector_recurrence(int, const VectorRecurrence&, const void*, const void*, const void*, const void*, void*,
                             const void* = nullptr, const void* = nullptr, const void* = nullptr) {
        throw std::runtime_error("vector_recurrence is not provided by this library");
    }
    template <class T> Buffer<T> make_buffer(std::size_t count) {
        static_assert(!detail::Format<T>::bits || sizeof(T) == std::size_t(detail::Format<T>::bits / 8 + 12) * (detail::Format<T>::complex ? 2 : 1),
                      "buffer layout mismatch");
        if (count > std::size_t(-1) / sizeof(T)) throw std::invalid_argument("buffer size overflow");
        lf_buffer* b = nullptr;
        detail::check(lf_buffer_create(e_.get(), count * sizeof(T), &b));
        return Buffer<T>(std::make_shared<detail::BufferRef>(b), count);
    }
    CommandBatch batch() { lf_batch* b = nullptr; detail::check(lf_batch_create(e_.get(), &b)); return CommandBatch(b); }
    Timing run(int bits, Operation op, const void* a, const void* b, void* out, std::size_t count, Broadcast b_index = {}) {
        lf_timing t{}; detail::check(lf_engine_run(e_.get(), bits, int(op), a, b, out, count, {b_index.stride, b_index.period}, &t));
        return detail::timing(t);
    }
    Timing run_unary(int bits, Operation op, const void* a, void* out, std::size_t count) {
        lf_timing t{}; detail::check(lf_engine_run_unary(e_.get(), bits, int(op), a, out, count, &t)); return detail::timing(t);
    }
    Timing run_ternary(int bits, Operation op, const void* a, const void* b, const void* c, void* out, std::size_t count,
                       Broadcast b_index = {}, Broadcast c_index = {}) {
        lf_timing t{};
        detail::check(lf_engine_run_ternary(e_.get(), bits, int(op), a, b, c, out, count, {b_index.stride, b_index.period},
                                            {c_index.stride, c_index.period}, &t));
        return detail::timing(t);
    }
    // Host-array precision cast between any two supported widths (complex: componentwise).
    Timing cast(int from_bits, int to_bits, bool complex, const void* in, void* out, std::size_t count) {
        lf_timing t{}; detail::check(lf_engine_cast(e_.get(), from_bits, to_bits, complex, in, out, count, &t)); return detail::timing(t);
    }
    Timing lu4(int bits, const Batched4& s, const void* A, const void* B, void* X, void* det, std::uint32_t* status) {
        lf_batched4 sh{s.count, s.rhs, s.inverse, s.determinant, s.fused};
        lf_timing t{}; detail::check(lf_engine_lu4(e_.get(), bits, &sh, A, B, X, det, status, &t)); return detail::timing(t);
    }
};
}  // namespace limbforge
