#pragma once
// limbforge::Linalg (the reference's include/limbforge/linalg.hpp:141-218 interface): exact dense
// products with one rounding per output, blocked Cholesky and multi-RHS triangular solves, as
// inline wrappers over the C ABI.  Every product runs on the GPU.
#include "engine.hpp"
#include <vector>

namespace limbforge {
struct LinalgOptions {
    int band_bits = 64; int max_bands = 4; int max_spread = 512; unsigned host_threads = 0;
    bool force_fallback = false; int resident_bands = 2;
    int method = 0;   // 0 auto (int8 residue engine where it applies), 1 generic limb kernel, 2 residue engine only
};
struct FactorOptions { std::size_t block = 32; double host_macs = 5e4; double solve_host_macs = 4e5; bool gpu = true; };
struct CholeskyInfo {
    std::size_t pivot = 0; int pivot_sign = 0; word pivot_status = 0;
    Timing timing{0, 0};
    std::size_t blocks = 0, gpu_updates = 0, host_updates = 0;
    double panel_seconds = 0, update_seconds = 0;
};
// Device memory a Linalg retains between calls (linalg.hpp:46-52), in bytes.
struct LinalgWorkspaces { std::size_t scratch_bytes = 0, idle_bytes = 0, busy_bytes = 0, busy_workspaces = 0; };
struct LinalgReport {
    std::size_t m = 0, n = 0, k = 0, gpu_outputs = 0, trivial_outputs = 0, gemm_rows = 0, gemm_cols = 0, int8_gemms = 0, moduli = 0, band_bits = 0;
    double analysis_seconds = 0, gpu_seconds = 0;
    int method = 0;
};

// Handle of a resident product (linalg.hpp:60-66): C is final after the batch's Submission::wait().
class LinalgTicket {
    struct Del { void operator()(lf_linalg_ticket* t) const { lf_linalg_ticket_destroy(t); } };
    std::shared_ptr<lf_linalg_ticket> t_;
    mutable LinalgReport r_;
    explicit LinalgTicket(lf_linalg_ticket* t) : t_(t, Del{}) {}
    friend class Linalg;
public:
    LinalgTicket() = default;
    bool resolved() const { int r = 0; detail::check(lf_linalg_ticket_resolved(t_.get(), &r)); return r != 0; }
    const LinalgReport& report() const {
        lf_linalg_report c{};
        detail::check(lf_linalg_ticket_report(t_.get(), &c));
        r_ = {c.m, c.n, c.k, c.gpu_outputs, c.trivial_outputs, c.gemm_rows, c.gemm_cols, c.int8_gemms, c.moduli, c.band_bits,
              c.analysis_seconds, c.gpu_seconds, c.method};
        return r_;
    }
    // Later operations of the batch read C in stream order after the product, so no read is provisional.
    bool provisional_reads() const { (void)report(); return false; }
};

// One Linalg per host thread.
class Linalg {
    struct Del { void operator()(lf_linalg* l) const { lf_linalg_destroy(l); } };
    std::unique_ptr<lf_linalg, Del> l_;
    LinalgOptions o_;
    mutable LinalgReport r_;
    static lf_factor_options fo(const FactorOptions& o) { return {o.block, o.host_macs, o.solve_host_macs, o.gpu}; }
    void make(lf_engine* e, LinalgOptions o) {
        o_ = o;
        lf_linalg_options c{o.band_bits, o.max_bands, o.max_spread, o.host_threads, o.force_fallback, o.resident_bands, o.method};
        lf_linalg* l = nullptr;
        detail::check(lf_linalg_create(e, &c, &l));
        l_.reset(l);
    }
public:
    explicit Linalg(LinalgOptions options = {}) { make(nullptr, options); }
    explicit Linalg(Engine& engine, LinalgOptions options = {}) { make(engine.handle(), options); }
    Linalg(const Linalg&) = delete;
    Linalg& operator=(const Linalg&) = delete;
    const LinalgOptions& options() const { return o_; }
    const LinalgReport& report() const {
        lf_linalg_report c{};
        detail::check(lf_linalg_get_report(l_.get(), &c));
        r_ = {c.m, c.n, c.k, c.gpu_outputs, c.trivial_outputs, c.gemm_rows, c.gemm_cols, c.int8_gemms, c.moduli, c.band_bits,
              c.analysis_seconds, c.gpu_seconds, c.method};
        return r_;
    }
    // Retained memory and its release (linalg.hpp:173-180): scratch and idle resident workspaces are freed now,
    // busy ones with their batches; the result is what was retained before the release.  Call between this
    // Linalg's calls, on its host thread.
    LinalgWorkspaces workspaces() const {
        lf_linalg_workspaces w{}; detail::check(lf_linalg_get_workspaces(l_.get(), &w));
        return {w.scratch_bytes, w.idle_bytes, w.busy_bytes, w.busy_workspaces};
    }
    LinalgWorkspaces release_workspaces() {
        lf_linalg_workspaces w{}; detail::check(lf_linalg_release_workspaces(l_.get(), &w));
        return {w.scratch_bytes, w.idle_bytes, w.busy_bytes, w.busy_workspaces};
    }
    Timing syrk(int bits, const void* A, std::size_t rows, std::size_t cols, void* C, bool lower_only = true, bool subtract = false) {
        lf_timing t{}; detail::check(lf_linalg_syrk(l_.get(), bits, A, rows, cols, C, lower_only, subtract, &t)); return detail::timing(t);
    }
    Timing gemm(int bits, bool transpose_a, const void* A, const void* B, std::size_t m, std::size_t n, std::size_t k, void* C,
                bool subtract = false) {
        lf_timing t{}; detail::check(lf_linalg_gemm(l_.get(), bits, transpose_a, A, B, m, n, k, C, subtract, &t)); return detail::timing(t);
    }
    CholeskyInfo cholesky(int bits, const void* A, std::size_t n, void* L, const FactorOptions& options = {}) {
        lf_factor_options o = fo(options);
        lf_cholesky_info i{};
        detail::check(lf_linalg_cholesky(l_.get(), bits, A, n, L, &o, &i));
        return {i.pivot, i.pivot_sign, i.pivot_status, detail::timing(i.timing), i.blocks, i.gpu_updates, i.host_updates,
                i.panel_seconds, i.update_seconds};
    }
    Timing trsm(int bits, bool transpose, const void* L, std::size_t n, const void* B, std::size_t nrhs, void* X, const FactorOptions& options = {}) {
        lf_factor_options o = fo(options);
        lf_timing t{}; detail::check(lf_linalg_trsm(l_.get(), bits, transpose, L, n, B, nrhs, X, &o, &t)); return detail::timing(t);
    }
    Timing cholesky_solve(int bits, const void* L, std::size_t n, const void* B, std::size_t nrhs, void* X, const FactorOptions& options = {}) {
        lf_factor_options o = fo(options);
        lf_timing t{}; detail::check(lf_linalg_cholesky_solve(l_.get(), bits, L, n, B, nrhs, X, &o, &t)); return detail::timing(t);
    }
    // Resident products (linalg.hpp:190-195): recorded into the batch; analysis, engine choice and modulus
    // count are GPU passes of the batch.
    template <class T> LinalgTicket syrk(CommandBatch& batch, const Buffer<T>& A, std::size_t rows, std::size_t cols, Buffer<T>& C,
                                         bool lower_only = true, bool subtract = false) {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "dense linear algebra uses real Float<bits> buffers");
        lf_linalg_ticket* t = nullptr;
        detail::check(lf_linalg_batch_syrk(l_.get(), batch.handle(), detail::Format<T>::bits, A.handle(), rows, cols, C.handle(),
                                           lower_only, subtract, &t));
        return LinalgTicket(t);
    }
    template <class T> LinalgTicket gemm(CommandBatch& batch, bool transpose_a, const Buffer<T>& A, const Buffer<T>& B, std::size_t m,
                                         std::size_t n, std::size_t k, Buffer<T>& C, bool subtract = false) {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "dense linear algebra uses real Float<bits> buffers");
        lf_linalg_ticket* t = nullptr;
        detail::check(lf_linalg_batch_gemm(l_.get(), batch.handle(), detail::Format<T>::bits, transpose_a, A.handle(), B.handle(), m, n, k,
                                           C.handle(), subtract, &t));
        return LinalgTicket(t);
    }
    template <class T> LinalgTicket gemm_exact(CommandBatch& b, bool ta, const Buffer<T>& A, const Buffer<T>& B, std::size_t m, std::size_t n,
                                               std::size_t k, Buffer<T>& C, bool sub = false) { return gemm(b, ta, A, B, m, n, k, C, sub); }
    template <class T> LinalgTicket syrk_exact(CommandBatch& b, const Buffer<T>& A, std::size_t rows, std::size_t cols, Buffer<T>& C,
                                               bool lower_only = true, bool sub = false) { return syrk(b, A, rows, cols, C, lower_only, sub); }
    // explicit contract names (linalg.hpp:203-208)
    Timing gemm_exact(int bits, bool ta, const void* A, const void* B, std::size_t m, std::size_t n, std::size_t k, void* C, bool sub = false) {
        return gemm(bits, ta, A, B, m, n, k, C, sub);
    }
    Timing syrk_exact(int bits, const void* A, std::size_t rows, std::size_t cols, void* C, bool lower_only = true, bool sub = false) {
        return syrk(bits, A, rows, cols, C, lower_only, sub);
    }
    CholeskyInfo cholesky_blocked(int bits, const void* A, std::size_t n, void* L, const FactorOptions& o = {}) { return cholesky(bits, A, n, L, o); }
    Timing cholesky_solve_blocked(int bits, const void* L, std::size_t n, const void* B, std::size_t nrhs, void* X, const FactorOptions& o = {}) {
        return cholesky_solve(bits, L, n, B, nrhs, X, o);
    }
};
}  // namespace limbforge
