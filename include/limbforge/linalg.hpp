#pragma once
// limbforge::Linalg (the reference's include/limbforge/linalg.hpp:141-218 interface): exact dense
// products with one rounding per output, blocked Cholesky, multi-RHS triangular solves and Householder
// QR, as inline wrappers over the C ABI.  Every product runs on the GPU.
#include "engine.hpp"
#include <cstring>
#include <future>
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
// Kernels to prepare ahead of use (Linalg::prewarm); the widths and inner sizes are validated.
struct LinalgPrewarm {
    std::vector<int> bits;
    std::vector<std::size_t> inner_sizes;
    bool resident = false;
};
struct LinalgPair { unsigned left_band, right_band, rows, cols, moduli; };
// Diagnostics of the last call (the reference's fields, filled from the GPU analysis: every nonzero, status-free
// line is one band of the residue engine here, so left_bands[1] / right_bands[1] count them and left_bands[0] /
// right_bands[0] the zero or status lines; outputs the reference sends to its host fallback run on the GPU, so
// the *_fallback counts are 0), and the engine used here.
struct LinalgReport {
    std::size_t m = 0, n = 0, k = 0;
    std::vector<std::size_t> left_bands, right_bands;
    std::size_t left_fallback = 0, right_fallback = 0;
    std::size_t gpu_outputs = 0, multi_band_outputs = 0, fallback_outputs = 0, trivial_outputs = 0;
    std::vector<LinalgPair> pairs;
    std::size_t gemm_rows = 0, gemm_cols = 0, int8_gemms = 0;
    bool zero_copy_output = false;
    bool resident_overflow = false;
    double analysis_seconds = 0, upload_seconds = 0, gpu_seconds = 0, assembly_seconds = 0, fallback_seconds = 0;
    std::size_t moduli = 0, band_bits = 0;
    int method = 0;   // 1 generic limb kernel, 2 int8 residue engine
};
namespace detail {
inline LinalgReport report_of(const lf_linalg_report& c) {
    LinalgReport r;
    r.m = c.m; r.n = c.n; r.k = c.k;
    r.gpu_outputs = c.gpu_outputs; r.trivial_outputs = c.trivial_outputs;
    r.gemm_rows = c.gemm_rows; r.gemm_cols = c.gemm_cols; r.int8_gemms = c.int8_gemms;
    r.moduli = c.moduli; r.band_bits = c.band_bits; r.method = c.method;
    r.analysis_seconds = c.analysis_seconds; r.gpu_seconds = c.gpu_seconds;
    r.left_bands = {c.left_zero_lines, c.left_lines};
    r.right_bands = {c.right_zero_lines, c.right_lines};
    if (c.method == 2) r.pairs.push_back({1, 1, (unsigned)c.gemm_rows, (unsigned)c.gemm_cols, (unsigned)c.moduli});
    return r;
}
}  // namespace detail

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
        r_ = detail::report_of(c);
        return r_;
    }
    // Later operations of the batch read C in stream order after the product, so no read is provisional.
    bool provisional_reads() const { (void)report(); return false; }
};

// Householder QR (linalg.hpp:88-137): FactorOptions (block; the GPU/host split fields only place work and never change
// a bit) and an optional rank test (rank_bits > 0 also stops at the first column whose |r_jj| lies more than rank_bits
// binades below the largest earlier |r_kk|); pivot: column pivoting (xGEQP3 order).
struct QROptions : FactorOptions { int rank_bits = 0; bool pivot = false; };
struct QRInfo {
    enum Reason { full_rank = 0, zero_column = 1, small_column = 2, status_column = 3 };
    std::size_t rank = 0; int reason = full_rank; word status = 0;
    Timing timing{0, 0};
    std::size_t blocks = 0, gpu_updates = 0, host_updates = 0;
    double panel_seconds = 0, update_seconds = 0;
    std::size_t norm_recomputations = 0;
};
class Linalg;
// Owning QR factor of an m x n matrix (m >= n): Q = H_0 ... H_{n-1}, H_j = I - tau_j v_j v_j^T, and R.  Row-major
// Float<bits> arrays owned by the factor: R (n x n, upper; with rank p < n rows i >= p hold the remainder in columns
// j >= p), V (m x n, column j is v_j), tau (n), T (blocks of nb x nb, block b at b*nb*nb).  The Linalg that made it
// must outlive it; calls follow the Linalg threading rule.
class QRFactor {
    struct Del { void operator()(lf_qr* q) const { lf_qr_destroy(q); } };
    std::unique_ptr<lf_qr, Del> q_;
    int bits_ = 0; std::size_t m_ = 0, n_ = 0, nb_ = 0; bool pivoted_ = false; QRInfo info_{};
    explicit QRFactor(lf_qr* q) : q_(q) {
        lf_qr_info i{}; int piv = 0;
        detail::check(lf_qr_describe(q, &bits_, &m_, &n_, &nb_, &piv, &i));
        pivoted_ = piv != 0;
        info_.rank = i.rank; info_.reason = i.reason; info_.status = i.status; info_.timing = detail::timing(i.timing);
        info_.blocks = i.blocks; info_.gpu_updates = i.gpu_updates; info_.host_updates = i.host_updates;
        info_.panel_seconds = i.panel_seconds; info_.update_seconds = i.update_seconds; info_.norm_recomputations = i.norm_recomputations;
    }
    const lf_qr* get() const { if (!q_) throw std::logic_error("empty QR factor"); return q_.get(); }
    const void* host(const void* p) const {
        if (!p && n_) throw std::runtime_error(std::string("QR factor arrays: ") + lf_last_error());
        return p;
    }
    friend class Linalg;
public:
    QRFactor() = default;
    QRFactor(QRFactor&&) noexcept = default;
    QRFactor& operator=(QRFactor&&) noexcept = default;
    bool empty() const { return !q_; }
    int bits() const { (void)get(); return bits_; }
    std::size_t rows() const { (void)get(); return m_; }
    std::size_t cols() const { (void)get(); return n_; }
    std::size_t block() const { (void)get(); return nb_; }
    const QRInfo& info() const { (void)get(); return info_; }
    bool full_rank() const { (void)get(); return info_.rank == n_; }
    // R, V and T are copied from the device on the first call; a failed copy throws.
    const void* r() const { return host(lf_qr_r(get())); }
    const void* v() const { return host(lf_qr_v(get())); }
    const void* tau() const { return lf_qr_tau(get()); }
    const void* t() const { return host(lf_qr_t(get())); }
    bool pivoted() const { (void)get(); return pivoted_; }
    const std::size_t* permutation() const { return lf_qr_permutation(get()); }
    // Least squares X (n x nrhs) for B (m x nrhs); X must not overlap B (linalg.hpp:127).
    Timing solve(const void* B, std::size_t nrhs, void* X) const {
        lf_timing t{}; detail::check(lf_qr_solve(get(), B, nrhs, X, &t)); return detail::timing(t);
    }
    // B (m x nrhs) <- Q^T B (transpose) or Q B, in place (linalg.hpp:129).
    Timing apply_q(void* B, std::size_t nrhs, bool transpose) const {
        lf_timing t{}; detail::check(lf_qr_apply_q(get(), B, nrhs, transpose, &t)); return detail::timing(t);
    }
    template <class T> Timing solve(const Buffer<T>& B, std::size_t nrhs, Buffer<T>& X) const {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "QR uses real Float<bits> buffers");
        lf_timing t{}; detail::check(lf_qr_solve_buffers(get(), B.handle(), nrhs, X.handle(), &t)); return detail::timing(t);
    }
    template <class T> Timing apply_q(Buffer<T>& B, std::size_t nrhs, bool transpose) const {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "QR uses real Float<bits> buffers");
        lf_timing t{}; detail::check(lf_qr_apply_q_buffer(get(), B.handle(), nrhs, transpose, &t)); return detail::timing(t);
    }
};

// Owning complex QR factor (linalg.hpp:331-350): H_j = I - tau_j v_j v_j^H with complex tau_j (zgeqrf), R upper with a
// real diagonal; row-major Complex<bits/32> arrays.  Same options, rank and status rules as QRFactor; column pivoting of
// complex factors is not built (factor_qr_complex throws std::runtime_error).
class ComplexQRFactor {
    QRFactor f_;
    explicit ComplexQRFactor(QRFactor f) : f_(std::move(f)) {}
    friend class Linalg;
public:
    ComplexQRFactor() = default;
    bool empty() const { return f_.empty(); }
    int bits() const { return f_.bits(); }
    std::size_t rows() const { return f_.rows(); }
    std::size_t cols() const { return f_.cols(); }
    std::size_t block() const { return f_.block(); }
    const QRInfo& info() const { return f_.info(); }
    bool full_rank() const { return f_.full_rank(); }
    const void* r() const { return f_.r(); }
    const void* v() const { return f_.v(); }
    const void* tau() const { return f_.tau(); }
    const void* t() const { return f_.t(); }
    bool pivoted() const { return f_.pivoted(); }
    const std::size_t* permutation() const { return f_.permutation(); }
    // X (n x nrhs, complex) = least-squares solution for B (m x nrhs, complex); X must not overlap B.
    Timing solve(const void* B, std::size_t nrhs, void* X) const { return f_.solve(B, nrhs, X); }
    // B (m x nrhs, complex) <- Q^H B (adjoint) or Q B, in place.
    Timing apply_q(void* B, std::size_t nrhs, bool adjoint) const { return f_.apply_q(B, nrhs, adjoint); }
};

// One Linalg per host thread.
class Linalg {
    struct Del { void operator()(lf_linalg* l) const { lf_linalg_destroy(l); } };
    std::unique_ptr<lf_linalg, Del> l_;
    LinalgOptions o_;
    mutable LinalgReport r_;
    static lf_factor_options fo(const FactorOptions& o) { return {o.block, o.host_macs, o.solve_host_macs, o.gpu}; }
    static lf_qr_options qo(const QROptions& o) { return {o.block, o.host_macs, o.solve_host_macs, o.gpu, o.rank_bits, o.pivot}; }
    template <class T> Timing solve_buffers(int passes, const Buffer<T>& L, std::size_t n, const Buffer<T>& B, std::size_t nrhs, Buffer<T>& X,
                                            const FactorOptions& options) {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "dense linear algebra uses real Float<bits> buffers");
        lf_factor_options o = fo(options);
        lf_timing t{};
        detail::check(lf_linalg_solve_buffers(l_.get(), detail::Format<T>::bits, passes, L.handle(), n, B.handle(), nrhs, X.handle(), &o, &t));
        return detail::timing(t);
    }
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
    // The kernels are compiled ahead for sm_100a; a prewarm validates the widths and inner sizes.
    void prewarm(const LinalgPrewarm& request) {
        for (int b : request.bits)
            if (b < 64 || b > 1024 || b % 32) throw std::invalid_argument("bits must be a multiple of 32 in [64,1024]");
        for (std::size_t k : request.inner_sizes)
            if (k > 65472) throw std::invalid_argument("resident inner size above 65472");
    }
    std::future<void> prewarm_async(LinalgPrewarm request) {
        return std::async(std::launch::async, [this, r = std::move(request)]() { prewarm(r); });
    }
    std::string device_name() const {
        char b[256]; detail::check(lf_linalg_device_name(l_.get(), b, sizeof b)); return b;
    }
    const LinalgReport& report() const {
        lf_linalg_report c{};
        detail::check(lf_linalg_get_report(l_.get(), &c));
        r_ = detail::report_of(c);
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
    // Householder QR of A (m x n, row-major, m >= n); A is only read (linalg.hpp:164).
    QRFactor factor_qr(int bits, const void* A, std::size_t m, std::size_t n, const QROptions& options = {}) {
        lf_qr_options o = qo(options); lf_qr* q = nullptr;
        detail::check(lf_linalg_factor_qr(l_.get(), bits, A, m, n, &o, &q));
        return QRFactor(q);
    }
    // Complex Householder QR of A (m x n Complex<bits/32>, row-major, m >= n) (linalg.hpp:170).
    ComplexQRFactor factor_qr_complex(int bits, const void* A, std::size_t m, std::size_t n, const QROptions& options = {}) {
        lf_qr_options o = qo(options); lf_qr* q = nullptr;
        detail::check(lf_linalg_factor_qr_complex(l_.get(), bits, A, m, n, &o, &q));
        return ComplexQRFactor(QRFactor(q));
    }
    // QR of the augmented Levenberg-Marquardt matrix [J; diag(d)] ((m + n) x n) (linalg.hpp:168).
    QRFactor factor_qr_augmented(int bits, const void* J, std::size_t m, std::size_t n, const void* d, const QROptions& options = {}) {
        lf_qr_options o = qo(options); lf_qr* q = nullptr;
        detail::check(lf_linalg_factor_qr_augmented(l_.get(), bits, J, m, n, d, &o, &q));
        return QRFactor(q);
    }
    template <class T> QRFactor factor_qr(const Buffer<T>& A, std::size_t m, std::size_t n, const QROptions& options = {}) {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "QR uses real Float<bits> buffers");
        lf_qr_options o = qo(options); lf_qr* q = nullptr;
        detail::check(lf_linalg_factor_qr_buffer(l_.get(), detail::Format<T>::bits, A.handle(), m, n, &o, &q));
        return QRFactor(q);
    }
    // Factorization and solves on Buffer operands of the Linalg's engine (linalg.hpp:194-199): synchronous, outside any
    // batch, the buffers used in place; they must be idle (logic_error otherwise).  Same bits as the host-array calls.
    template <class T> CholeskyInfo cholesky(const Buffer<T>& A, std::size_t n, Buffer<T>& L, const FactorOptions& options = {}) {
        static_assert(detail::Format<T>::bits && !detail::Format<T>::complex, "dense linear algebra uses real Float<bits> buffers");
        lf_factor_options o = fo(options);
        lf_cholesky_info i{};
        detail::check(lf_linalg_cholesky_buffers(l_.get(), detail::Format<T>::bits, A.handle(), n, L.handle(), &o, &i));
        return {i.pivot, i.pivot_sign, i.pivot_status, detail::timing(i.timing), i.blocks, i.gpu_updates, i.host_updates,
                i.panel_seconds, i.update_seconds};
    }
    template <class T> Timing trsm(bool transpose, const Buffer<T>& L, std::size_t n, const Buffer<T>& B, std::size_t nrhs, Buffer<T>& X,
                                   const FactorOptions& options = {}) {
        return solve_buffers<T>(transpose ? 2 : 1, L, n, B, nrhs, X, options);
    }
    template <class T> Timing cholesky_solve(const Buffer<T>& L, std::size_t n, const Buffer<T>& B, std::size_t nrhs, Buffer<T>& X,
                                             const FactorOptions& options = {}) {
        return solve_buffers<T>(3, L, n, B, nrhs, X, options);
    }
    template <class T> CholeskyInfo cholesky_blocked(const Buffer<T>& A, std::size_t n, Buffer<T>& L, const FactorOptions& o = {}) {
        return cholesky(A, n, L, o);
    }
    template <class T> Timing cholesky_solve_blocked(const Buffer<T>& L, std::size_t n, const Buffer<T>& B, std::size_t nrhs, Buffer<T>& X,
                                                     const FactorOptions& o = {}) {
        return cholesky_solve(L, n, B, nrhs, X, o);
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

// ---- Exact dot products on the host (linalg.hpp:268-321): RN(c -/+ sum_k a[k*sa] b[k*sb]) with one rounding, the
// contract every GPU product here meets; the same cluster method as the GPU limb kernel.  Statuses: zero carrying the
// OR of c's and every operand's status; no nonzero product returns c (or zero).
namespace detail {
template <int N> struct HostDotTerms {
    const Number<N>* a; long sa; const Number<N>* b; long sb; std::size_t K; bool subtract; lfd::Num<N> c;
    lfd::u64 count() const { return K + 1; }
    bool term(lfd::u64 k, lfd::i64& scale, lfd::i64& top, int& sign) const {
        if (k == K) {
            if (!c.s) return false;
            scale = (lfd::i64)c.e - (32 * N - 1); top = scale + 32 * N; sign = c.s;
            return true;
        }
        const Number<N>& x = a[(long)k * sa];
        const Number<N>& y = b[(long)k * sb];
        if (!x.sign || !y.sign) return false;
        scale = (lfd::i64)x.exponent + y.exponent - 2 * (32 * N - 1); top = scale + 64 * N;
        sign = subtract ? -x.sign * y.sign : x.sign * y.sign;
        return true;
    }
    void add(lfd::u64 k, lfd::u32* acc, int len, lfd::i64 off) const {
        if (k == K) { lfd::acc_add(acc, len, c.m, N, off); return; }
        lfd::u32 p[2 * N];
        lfd::mant_mul<N>(a[(long)k * sa].limb, b[(long)k * sb].limb, p);
        lfd::acc_add(acc, len, p, 2 * N, off);
    }
};
}  // namespace detail
template <int N> inline Number<N> exact_dot_add(const Number<N>& c, bool subtract, const Number<N>* a, long sa, const Number<N>* b, long sb,
                                                std::size_t K) {
    word st = c.status;
    bool products = false;
    for (std::size_t k = 0; k < K; ++k) {
        st |= a[(long)k * sa].status | b[(long)k * sb].status;
        products = products || (a[(long)k * sa].sign && b[(long)k * sb].sign);
    }
    if (st) return zero<N>(st);
    if (!products) return c;
    const detail::HostDotTerms<N> src{a, sa, b, sb, K, subtract, detail::num(c)};
    lfd::u32 error = 0;
    const Number<N> r = detail::number(lfd::cluster_round<N, 8 * N + 64>(src, &error));
    if (error) throw std::runtime_error("exact_dot_add: a cluster of terms exceeds the exact window");
    return r;
}
template <int N> inline Number<N> exact_dot(const Number<N>* a, long sa, const Number<N>* b, long sb, std::size_t K) {
    return exact_dot_add<N>(zero<N>(), false, a, sa, b, sb, K);
}
}  // namespace limbforge
