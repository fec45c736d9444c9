// C ABI of the exact dense products and factorizations (the reference's Linalg, linalg.hpp:141-218,
// linalg.mm:176-488): host-array and device-resident forms of gemm/syrk, blocked Cholesky with the
// reference's fixed rounding sequence, and multi-RHS triangular solves.  Every product runs on the
// GPU (no host fallback): the residue/CRT tensor-core engine where it applies, the generic exact limb
// kernel otherwise; both give identical bits.
#include "lf_runtime.h"
#include "lf_linalg.cuh"
#include "lf_residue.h"
#include "lf_residue.cuh"
#include "lf_qr.cuh"
#include "lf_cqr.cuh"

#include <algorithm>
#include <cstdio>
#include <chrono>

namespace lfr {

struct Linalg {
    Engine* engine = nullptr;
    bool own_engine = false;
    lf_linalg_options options{};
    lf_linalg_report report{};
    DevBuf work[6];
    DevBuf qr[13];                  // Householder QR scratch: W/Y blocks, panel, state, right-hand sides, pivoting
    DevBuf info_buf, error_buf, lines;
    ResidueEngine residue;
    // the factorizations' second product lane: trailing updates beyond the next block run on `side` while the
    // next panel runs on the engine's stream (look-ahead), with their own residue-engine workspaces
    ResidueEngine residue2;
    DevBuf lines2;
    cudaStream_t side = nullptr;
    cudaEvent_t ev_panel = nullptr, ev_side = nullptr;
    std::vector<std::weak_ptr<ResidentProduct>> resident;   // recorded resident products, for workspaces()
    ~Linalg() {
        if (ev_panel) cudaEventDestroy(ev_panel);
        if (ev_side) cudaEventDestroy(ev_side);
        if (side) cudaStreamDestroy(side);
    }
};

using Clock = std::chrono::steady_clock;
static double since(Clock::time_point t) { return std::chrono::duration<double>(Clock::now() - t).count(); }
static void check_bits(int bits) { if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]"); }

// Workspaces of one stream of exact products: residue engine, line analysis and the error word.
struct ProductLane { ResidueEngine* residue; DevBuf* lines; uint32_t* err; };
// The main lane (the engine's stream; error word 1 of the Linalg's error buffer; word 0 belongs to the panel and
// solve kernels of a factorization) and the factorizations' side lane (error word 2).
static ProductLane main_lane(Linalg& la) { return {&la.residue, &la.lines, static_cast<uint32_t*>(la.error_buf.get(16)) + 1}; }
static ProductLane side_lane(Linalg& la) {
    if (!la.side) {
        cuda_check(cudaStreamCreateWithFlags(&la.side, cudaStreamNonBlocking), "stream");
        cuda_check(cudaEventCreateWithFlags(&la.ev_panel, cudaEventDisableTiming), "event");
        cuda_check(cudaEventCreateWithFlags(&la.ev_side, cudaEventDisableTiming), "event");
    }
    return {&la.residue2, &la.lines2, static_cast<uint32_t*>(la.error_buf.get(16)) + 2};
}

// C (M x Nc at ldc) <- RN(C - L R^T) (subtract) or RN(L R^T), L/R given as line views; lower: only j <= i.  On `lane`
// and stream s; with `check`, the call waits for the product and raises a cluster overflow, otherwise the caller reads
// the lane's error word later (its word is not cleared here then).
void exact_product_on(Linalg& la, const ProductLane& lane, int bits, lfd::LineView left, lfd::LineView right, uint64_t M,
                      uint64_t Nc, uint64_t K, uint32_t* C, uint64_t ldc, bool subtract, bool lower, cudaStream_t s,
                      int* method_used, bool check) {
    if (!M || !Nc) return;
    const int n = bits / 32;
    uint32_t* err = lane.err;
    if (check) cuda_check(cudaMemsetAsync(err, 0, 4, s), "memset");
    int method = la.options.method;                    // 0 auto, 1 limb kernel, 2 residue engine
    bool used_residue = false;
    if (method != 1 && !la.options.force_fallback)
        used_residue = lane.residue->run(bits, left, right, M, Nc, K, C, ldc, subtract, lower, err, s, method == 2, la.report);
    if (!used_residue) {
        // the tiled limb kernel: line analysis, then one exact window per output (cluster method for wide outputs)
        lfd::WinParams wp{};
        lfd::DotParams& p = wp.d;
        p.left = left; p.right = right; p.C = C; p.ldc = ldc; p.M = M; p.Nc = Nc; p.K = K;
        p.row0 = 0; p.col0 = 0; p.subtract = subtract; p.lower = lower; p.error = err;
        auto* linfo = static_cast<lfd::LineInfo*>(lane.lines->get(sizeof(lfd::LineInfo) * (M + Nc) + 64));
        lfd::linalg_kernels(n)->analyze(left, M, K, linfo, s);
        lfd::linalg_kernels(n)->analyze(right, Nc, K, linfo + M, s);
        wp.linfo = linfo; wp.rinfo = linfo + M;
        lfd::residue_kernels(n)->window_dot(wp, s);
        cuda_check(cudaGetLastError(), "exact product launch");
    }
    if (method_used) *method_used = used_residue ? 2 : 1;
    if (!check) return;
    uint32_t e = 0;
    cuda_check(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "exact product");
    if (e) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
}
void exact_product(Linalg& la, int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc, uint64_t K,
                   uint32_t* C, uint64_t ldc, bool subtract, bool lower, cudaStream_t s, int* method_used) {
    exact_product_on(la, main_lane(la), bits, left, right, M, Nc, K, C, ldc, subtract, lower, s, method_used, true);
}

static void validate_dims(size_t M, size_t Nc, size_t K, size_t stride) {
    const size_t limit = size_t(1) << 31;
    if (M >= limit || Nc >= limit || K >= limit || M * stride >= limit) throw invalid_argument("matrix dimensions exceed 32-bit indexing");
}

}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};
struct lf_linalg : Linalg {};

extern "C" {

int lf_linalg_create(lf_engine* engine, const lf_linalg_options* options, lf_linalg** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null handle");
    lf_linalg_options o{64, 4, 512, 0, 0, 2, 0};
    if (options) o = *options;
    if (o.band_bits < 0 || o.band_bits > 1024 || o.max_bands < 0 || o.max_spread < 0 || o.max_spread > 8192)
        throw invalid_argument("linalg options: band_bits in [0,1024], max_bands >= 0, max_spread in [0,8192]");
    auto* la = new lf_linalg();
    la->options = o;
    if (engine) la->engine = engine;
    else {
        lf_engine* e = nullptr;
        int rc = lf_engine_create(nullptr, &e);
        if (rc) { delete la; throw runtime_error(lf_last_error()); }
        la->engine = e; la->own_engine = true;
    }
    *out = la;
    LF_API_END
}
void lf_linalg_destroy(lf_linalg* la) {
    if (!la) return;
    if (la->own_engine) lf_engine_destroy(static_cast<lf_engine*>(la->engine));
    delete la;
}
int lf_linalg_device_name(lf_linalg* la, char* name, size_t capacity) {
    LF_API_BEGIN
    if (!la || !name || !capacity) throw invalid_argument("null argument");
    cudaDeviceProp p{};
    cuda_check(cudaGetDeviceProperties(&p, la->engine->device), "device properties");
    std::snprintf(name, capacity, "%s", p.name);
    LF_API_END
}

int lf_linalg_get_report(lf_linalg* la, lf_linalg_report* r) {
    LF_API_BEGIN
    if (!la || !r) throw invalid_argument("null argument");
    *r = la->report;
    LF_API_END
}

// Linalg::gemm (linalg.hpp:155; linalg.mm:181-185): C (m x n) = op(A) B, or RN(C - op(A) B).
int lf_linalg_gemm(lf_linalg* la, int bits, int transpose_a, const void* A, const void* B, size_t m, size_t n, size_t k,
                   void* C, int subtract, lf_timing* timing) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    validate_dims(m, n, k, n);
    if (m && n && !C) throw invalid_argument("null output");
    if (m * n && k && (!A || !B)) throw invalid_argument("null input");
    auto w0 = Clock::now();
    la->report = lf_linalg_report{};
    la->report.m = m; la->report.n = n; la->report.k = k;
    if (timing) *timing = {0, 0};
    if (!m || !n) return LF_OK;
    Engine& e = *la->engine;
    e.activate();
    const size_t E = bits / 32 + 3, eb = 4 * E;
    cudaStream_t s = e.stream;
    uint32_t* dA = static_cast<uint32_t*>(la->work[0].get(m * k * eb + 16));
    uint32_t* dB = static_cast<uint32_t*>(la->work[1].get(k * n * eb + 16));
    uint32_t* dC = static_cast<uint32_t*>(la->work[2].get(m * n * eb));
    if (k) {
        cuda_check(cudaMemcpyAsync(dA, A, m * k * eb, cudaMemcpyHostToDevice, s), "upload");
        cuda_check(cudaMemcpyAsync(dB, B, k * n * eb, cudaMemcpyHostToDevice, s), "upload");
    }
    if (subtract) cuda_check(cudaMemcpyAsync(dC, C, m * n * eb, cudaMemcpyHostToDevice, s), "upload");
    lfd::LineView lv = transpose_a ? lfd::LineView{dA, 1, m} : lfd::LineView{dA, k, 1};
    lfd::LineView rv{dB, 1, n};
    cuda_check(cudaEventRecord(e.e0, s), "event");
    int method = 1;
    exact_product(*la, bits, lv, rv, m, n, k, dC, n, subtract != 0, false, s, &method);
    cuda_check(cudaEventRecord(e.e1, s), "event");
    cuda_check(cudaMemcpyAsync(C, dC, m * n * eb, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0; cudaEventElapsedTime(&ms, e.e0, e.e1);
    la->report.gpu_seconds = ms * 1e-3; la->report.gpu_outputs = m * n; la->report.method = method;
    if (timing) *timing = {ms * 1e-3, since(w0)};
    LF_API_END
}

// Linalg::syrk (linalg.hpp:152; linalg.mm:176-180): C (cols x cols) = A^T A, lower or full.
int lf_linalg_syrk(lf_linalg* la, int bits, const void* A, size_t rows, size_t cols, void* C, int lower_only, int subtract,
                   lf_timing* timing) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    if (subtract && !lower_only) throw invalid_argument("syrk: subtract updates the lower triangle only (lower_only)");
    validate_dims(cols, cols, rows, cols);
    if (cols && !C) throw invalid_argument("null output");
    if (cols && rows && !A) throw invalid_argument("null input");
    auto w0 = Clock::now();
    la->report = lf_linalg_report{};
    la->report.m = cols; la->report.n = cols; la->report.k = rows;
    if (timing) *timing = {0, 0};
    if (!cols) return LF_OK;
    Engine& e = *la->engine;
    e.activate();
    const size_t E = bits / 32 + 3, eb = 4 * E;
    cudaStream_t s = e.stream;
    uint32_t* dA = static_cast<uint32_t*>(la->work[0].get(rows * cols * eb + 16));
    uint32_t* dC = static_cast<uint32_t*>(la->work[2].get(cols * cols * eb));
    if (rows) cuda_check(cudaMemcpyAsync(dA, A, rows * cols * eb, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaMemcpyAsync(dC, C, cols * cols * eb, cudaMemcpyHostToDevice, s), "upload");   // keeps the untouched triangle
    lfd::LineView v{dA, 1, cols};
    cuda_check(cudaEventRecord(e.e0, s), "event");
    int method = 1;
    exact_product(*la, bits, v, v, cols, cols, rows, dC, cols, subtract != 0, true, s, &method);
    if (!lower_only) lfd::linalg_kernels(bits / 32)->mirror(dC, cols, cols, s);
    cuda_check(cudaEventRecord(e.e1, s), "event");
    cuda_check(cudaMemcpyAsync(C, dC, cols * cols * eb, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0; cudaEventElapsedTime(&ms, e.e0, e.e1);
    la->report.gpu_seconds = ms * 1e-3; la->report.gpu_outputs = cols * (cols + 1) / 2; la->report.method = method;
    if (timing) *timing = {ms * 1e-3, since(w0)};
    LF_API_END
}

}  // extern "C"

namespace lfr {

// Blocked right-looking Cholesky of the device matrix W (n x n, already holding A's lower triangle):
// panels on the GPU (diagonal block, then the rows below), trailing updates as exact SYRK products
// of one rounding per entry (linalg.mm:411-457 sequence).  Look-ahead: block k's trailing update is split into
// the next block column (rows k1.., columns [k1, k2), on the engine's stream, so the next panel follows it there)
// and the rest (rows and columns k2.., on the side stream), which runs while the next panel is factored.  Every
// entry still receives block 0's update, then block 1's, ... in order: the next block column's update waits for the
// previous remainder update, which covered those columns too.
static lf_cholesky_info cholesky_device(Linalg& la, int bits, uint32_t* W, size_t n, size_t block) {
    lf_cholesky_info info{};
    info.pivot = n;
    auto w0 = Clock::now();
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3;
    const auto* fk = lfd::factor_kernels(limbs);
    const size_t nb = block ? std::min(block, n) : n;
    long long* dinfo = static_cast<long long*>(la.info_buf.get(64));
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane_a = main_lane(la), lane_b = side_lane(la);
    cudaStream_t s2 = la.side;
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    bool side_pending = false;                           // a remainder update is queued on s2 (ev_side after it)
    size_t fail = n;
    for (size_t k0 = 0; k0 < n && fail == n; k0 += nb) {
        const size_t k1 = std::min(n, k0 + nb);
        auto t = Clock::now();
        long long init[3] = {(long long)n, 0, 0};
        cuda_check(cudaMemcpyAsync(dinfo, init, sizeof init, cudaMemcpyHostToDevice, s), "info");
        lfd::CholParams p{W, n, k0, k1, dinfo, err};
        fk->diag(p, s);
        cuda_check(cudaGetLastError(), "cholesky diagonal block");
        long long got[3];
        cuda_check(cudaMemcpyAsync(got, dinfo, sizeof got, cudaMemcpyDeviceToHost, s), "info");
        cuda_check(cudaStreamSynchronize(s), "panel");
        ++info.blocks;
        if ((size_t)got[0] < n) {
            fail = (size_t)got[0];
            info.pivot = fail; info.pivot_sign = (int)got[1]; info.pivot_status = (uint32_t)got[2];
            fk->rows(p, k1, fail, s);                   // rows below the block: columns [k0, fail)
            cuda_check(cudaGetLastError(), "cholesky panel rows");
            cuda_check(cudaStreamSynchronize(s), "panel");
            info.panel_seconds += since(t);
            break;
        }
        fk->rows(p, k1, k1, s);
        cuda_check(cudaGetLastError(), "cholesky panel rows");
        info.panel_seconds += since(t);
        if (k1 < n) {
            t = Clock::now();
            const size_t k2 = std::min(n, k1 + nb);
            cuda_check(cudaEventRecord(la.ev_panel, s), "event");               // panel k0 complete
            // the next block column: rows [k1, n) x columns [k1, k2), after the previous remainder update
            if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
            lfd::LineView rows_k1{W + (k1 * n + k0) * E, n, 1}, rows_k1b{W + (k1 * n + k0) * E, n, 1};
            exact_product_on(la, lane_a, bits, rows_k1, rows_k1b, n - k1, k2 - k1, k1 - k0, W + (k1 * n + k1) * E, n, true, true, s,
                             nullptr, false);
            // the rest: rows and columns [k2, n), on the side stream after the panel
            if (k2 < n) {
                cuda_check(cudaStreamWaitEvent(s2, la.ev_panel, 0), "event wait");
                lfd::LineView rows_k2{W + (k2 * n + k0) * E, n, 1};
                exact_product_on(la, lane_b, bits, rows_k2, rows_k2, n - k2, n - k2, k1 - k0, W + (k2 * n + k2) * E, n, true, true, s2,
                                 nullptr, false);
                cuda_check(cudaEventRecord(la.ev_side, s2), "event");
                side_pending = true;
            }
            ++info.gpu_updates;
            info.update_seconds += since(t);
        }
    }
    if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
    if (fail < n) fk->prep(nullptr, W, n, fail, s);
    cuda_check(cudaGetLastError(), "cholesky clear");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "cholesky");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1] | ev[2]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    info.timing = {ms * 1e-3, since(w0)};
    return info;
}

// X (device, n x nrhs) holds B; passes 1 forward, 2 backward (L^T), 3 both (linalg.mm:459-488).  Look-ahead as
// in the factorization: after the diagonal block of rows [r0, r1), the update of the next block's rows runs on the
// engine's stream (the next diagonal block follows it there) and the update of the rows beyond on the side stream,
// while the next diagonal block is solved; each row still receives the blocks' updates in order.
// upper (backward pass only): L holds an upper triangular R = L^T itself, row i of R in place of column i of L (the
// least-squares solve of the QR factor; the same sequence, linalg.mm:471-480).
static double solve_device(Linalg& la, int bits, const uint32_t* L, size_t n, uint32_t* X, size_t nrhs, size_t block, int passes,
                           bool upper = false) {
    if (!n || !nrhs) return 0;
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3;
    const auto* fk = lfd::factor_kernels(limbs);
    const size_t nb = block ? std::min(block, n) : n;
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));      // word 0: the solve kernels' flag
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane_a = main_lane(la), lane_b = side_lane(la);
    cudaStream_t s2 = la.side;
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    bool side_pending = false;
    // rows [a, b) of X updated by the block [r0, r1): X[a..b) -= L(a..b, r0..r1) X[r0..r1) (forward), or with the
    // columns of L (backward, line i = column i of L from row r0)
    auto update = [&](bool forward, size_t r0, size_t r1, size_t a, size_t b, const ProductLane& lane, cudaStream_t st) {
        if (a >= b) return;
        const lfd::LineView lv = forward || upper ? lfd::LineView{L + (a * n + r0) * E, n, 1} : lfd::LineView{L + (r0 * n + a) * E, 1, n};
        const lfd::LineView xv{X + r0 * nrhs * E, 1, nrhs};
        exact_product_on(la, lane, bits, lv, xv, b - a, nrhs, r1 - r0, X + a * nrhs * E, nrhs, true, false, st, nullptr, false);
    };
    // after the diagonal block [r0, r1): the next block's rows [na, nb_) on s, the rest [ra, rb) on s2
    auto split = [&](bool forward, size_t r0, size_t r1, size_t na, size_t nbb, size_t ra, size_t rb) {
        cuda_check(cudaEventRecord(la.ev_panel, s), "event");
        if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
        update(forward, r0, r1, na, nbb, lane_a, s);
        if (ra < rb) {
            cuda_check(cudaStreamWaitEvent(s2, la.ev_panel, 0), "event wait");
            update(forward, r0, r1, ra, rb, lane_b, s2);
            cuda_check(cudaEventRecord(la.ev_side, s2), "event");
            side_pending = true;
        }
    };
    if (passes & 1)
        for (size_t r0 = 0; r0 < n; r0 += nb) {
            const size_t r1 = std::min(n, r0 + nb);
            fk->solve(lfd::SolveParams{L, X, n, nrhs, r0, r1, 0, err}, true, s);
            cuda_check(cudaGetLastError(), "forward substitution");
            if (r1 < n) {
                const size_t r2 = std::min(n, r1 + nb);
                split(true, r0, r1, r1, r2, r2, n);
            }
        }
    if (side_pending) { cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait"); side_pending = false; }
    if (passes & 2)
        for (size_t r0 = (n - 1) / nb * nb;; r0 -= nb) {
            const size_t r1 = std::min(n, r0 + nb);
            fk->solve(lfd::SolveParams{L, X, n, nrhs, r0, r1, upper ? 1 : 0, err}, false, s);
            cuda_check(cudaGetLastError(), "back substitution");
            if (r0) {
                const size_t q0 = r0 - nb;                     // the next block (below in the order) is [q0, r0)
                split(false, r0, r1, q0, r0, 0, q0);
            }
            if (!r0) break;
        }
    if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "solve");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1] | ev[2]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    return ms * 1e-3;
}

static bool overlap(const void* a, size_t na, const void* b, size_t nb) {
    auto x = reinterpret_cast<uintptr_t>(a), y = reinterpret_cast<uintptr_t>(b);
    return na && nb && x < y + nb && y < x + na;
}

}  // namespace lfr

extern "C" {

// Linalg::cholesky (linalg.hpp:158): L may equal A; otherwise they must not overlap.
int lf_linalg_cholesky(lf_linalg* la, int bits, const void* A, size_t n, void* L, const lf_factor_options* fo,
                       lf_cholesky_info* out) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    validate_dims(n, n, n, n);
    const size_t eb = size_t(bits / 8 + 12);
    if (n && (!A || !L)) throw invalid_argument("null matrix");
    if (A != L && overlap(A, n * n * eb, L, n * n * eb)) throw invalid_argument("cholesky: L overlaps A");
    const size_t block = fo ? fo->block : 32;
    lf_cholesky_info info{};
    info.pivot = n;
    if (n) {
        Engine& e = *la->engine;
        e.activate();
        uint32_t* dA = static_cast<uint32_t*>(la->work[3].get(n * n * eb));
        uint32_t* W = static_cast<uint32_t*>(la->work[4].get(n * n * eb));
        auto w0 = Clock::now();
        cuda_check(cudaMemcpyAsync(dA, A, n * n * eb, cudaMemcpyHostToDevice, e.stream), "upload");
        lfd::factor_kernels(bits / 32)->prep(dA, W, n, n, e.stream);
        cuda_check(cudaGetLastError(), "cholesky prepare");
        info = cholesky_device(*la, bits, W, n, block);
        cuda_check(cudaMemcpyAsync(L, W, n * n * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        cuda_check(cudaStreamSynchronize(e.stream), "download");
        info.timing.wall_seconds = since(w0);
    }
    if (out) *out = info;
    LF_API_END
}

static int solve_common(lf_linalg* la, int bits, int passes, const void* L, size_t n, const void* B, size_t nrhs, void* X,
                        const lf_factor_options* fo, lf_timing* timing) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    validate_dims(n, nrhs, n, nrhs);
    const size_t eb = size_t(bits / 8 + 12);
    if (timing) *timing = {0, 0};
    if (!n || !nrhs) return LF_OK;
    if (!L || !B || !X) throw invalid_argument("null matrix");
    if (X != B && (overlap(X, n * nrhs * eb, B, n * nrhs * eb) || overlap(X, n * nrhs * eb, L, n * n * eb)))
        throw invalid_argument("trsm: X overlaps B or L");
    Engine& e = *la->engine;
    e.activate();
    auto w0 = Clock::now();
    uint32_t* dL = static_cast<uint32_t*>(la->work[3].get(n * n * eb));
    uint32_t* dX = static_cast<uint32_t*>(la->work[5].get(n * nrhs * eb));
    cuda_check(cudaMemcpyAsync(dL, L, n * n * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    cuda_check(cudaMemcpyAsync(dX, B, n * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    const double g = solve_device(*la, bits, dL, n, dX, nrhs, fo ? fo->block : 32, passes);
    cuda_check(cudaMemcpyAsync(X, dX, n * nrhs * eb, cudaMemcpyDeviceToHost, e.stream), "download");
    cuda_check(cudaStreamSynchronize(e.stream), "download");
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}
// Linalg::trsm (linalg.hpp:161): L X = B, or L^T X = B with transpose.
int lf_linalg_trsm(lf_linalg* la, int bits, int transpose, const void* L, size_t n, const void* B, size_t nrhs, void* X,
                   const lf_factor_options* fo, lf_timing* timing) {
    return solve_common(la, bits, transpose ? 2 : 1, L, n, B, nrhs, X, fo, timing);
}
// Linalg::cholesky_solve (linalg.hpp:163): L L^T X = B.
int lf_linalg_cholesky_solve(lf_linalg* la, int bits, const void* L, size_t n, const void* B, size_t nrhs, void* X,
                             const lf_factor_options* fo, lf_timing* timing) {
    return solve_common(la, bits, 3, L, n, B, nrhs, X, fo, timing);
}

// Buffer forms of the factorization and the solves (linalg.hpp:194-199): synchronous, outside any batch, on
// buffers of the Linalg's engine used in place; the buffers must be idle (a buffer in an unwaited submission
// throws logic_error) and are held like a submission's until the call returns.  Results equal the host-array
// calls bit for bit.
namespace {
struct BufferClaim {
    std::vector<lf_buffer*> held;
    void take(lf_buffer* b, uint64_t owner) {
        if (!b) throw invalid_argument("missing buffer");
        if (b->owner != owner) throw invalid_argument("buffer belongs to another engine");
        for (lf_buffer* h : held) if (h == b) return;
        bool idle = false;
        if (!b->busy.compare_exchange_strong(idle, true)) throw logic_error("buffer is in use by an unwaited submission");
        held.push_back(b);
    }
    ~BufferClaim() { for (lf_buffer* b : held) b->busy.store(false); }
};
}  // namespace

int lf_linalg_cholesky_buffers(lf_linalg* la, int bits, lf_buffer* A, size_t n, lf_buffer* L, const lf_factor_options* fo,
                               lf_cholesky_info* out) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    validate_dims(n, n, n, n);
    const size_t eb = size_t(bits / 8 + 12);
    Engine& e = *la->engine;
    BufferClaim claim;
    claim.take(A, e.identity);
    claim.take(L, e.identity);
    if (A->bytes < n * n * eb || L->bytes < n * n * eb) throw invalid_argument("cholesky: buffer smaller than n x n");
    lf_cholesky_info info{};
    info.pivot = n;
    if (n) {
        e.activate();
        auto w0 = Clock::now();
        A->sync_to_device(e.stream);
        if (L != A) L->host_authoritative = false;          // every entry of L is written below
        uint32_t* W = static_cast<uint32_t*>(L->dev);
        lfd::factor_kernels(bits / 32)->prep(static_cast<const uint32_t*>(A->dev), W, n, n, e.stream);
        cuda_check(cudaGetLastError(), "cholesky prepare");
        info = cholesky_device(*la, bits, W, n, fo ? fo->block : 32);
        cuda_check(cudaStreamSynchronize(e.stream), "cholesky");
        info.timing.wall_seconds = since(w0);
    }
    if (out) *out = info;
    LF_API_END
}

int lf_linalg_solve_buffers(lf_linalg* la, int bits, int passes, lf_buffer* L, size_t n, lf_buffer* B, size_t nrhs, lf_buffer* X,
                            const lf_factor_options* fo, lf_timing* timing) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    if (passes < 1 || passes > 3) throw invalid_argument("passes must be 1 (L X = B), 2 (L^T X = B) or 3 (L L^T X = B)");
    check_bits(bits);
    validate_dims(n, nrhs, n, nrhs);
    const size_t eb = size_t(bits / 8 + 12);
    Engine& e = *la->engine;
    BufferClaim claim;
    claim.take(L, e.identity);
    claim.take(B, e.identity);
    claim.take(X, e.identity);
    if (L->bytes < n * n * eb || B->bytes < n * nrhs * eb || X->bytes < n * nrhs * eb) throw invalid_argument("trsm: buffer too small");
    if (X == L) throw invalid_argument("trsm: X overlaps L");
    if (timing) *timing = {0, 0};
    if (!n || !nrhs) return LF_OK;
    e.activate();
    auto w0 = Clock::now();
    L->sync_to_device(e.stream);
    B->sync_to_device(e.stream);
    uint32_t* dX = static_cast<uint32_t*>(X->dev);
    if (X != B) {
        X->host_authoritative = false;
        cuda_check(cudaMemcpyAsync(dX, B->dev, n * nrhs * eb, cudaMemcpyDeviceToDevice, e.stream), "right-hand sides");
    }
    const double g = solve_device(*la, bits, static_cast<const uint32_t*>(L->dev), n, dX, nrhs, fo ? fo->block : 32, passes);
    cuda_check(cudaStreamSynchronize(e.stream), "solve");
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}

// Device-pointer exact product for CUDA callers (no reference counterpart): C <- RN(C -/+ L R^T)
// over line views (element (line, k) at base + (line * ls + k * ks) elements).
int lf_dev_exact_product(lf_linalg* la, int bits, const void* left, size_t left_ls, size_t left_ks, const void* right,
                         size_t right_ls, size_t right_ks, size_t M, size_t Nc, size_t K, void* C, size_t ldc, int subtract,
                         int lower, void* stream) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    lfd::LineView lv{static_cast<const uint32_t*>(left), left_ls, left_ks}, rv{static_cast<const uint32_t*>(right), right_ls, right_ks};
    int method = 1;
    exact_product(*la, bits, lv, rv, M, Nc, K, static_cast<uint32_t*>(C), ldc, subtract != 0, lower != 0,
                  stream ? static_cast<cudaStream_t>(stream) : la->engine->stream, &method);
    la->report.method = method;
    LF_API_END
}

}  // extern "C"

// ---------------------------------------------------------------- resident products (linalg.hpp:190-195)
// Linalg::syrk / gemm on a CommandBatch: recorded now, planned and run on the GPU at submit (line analysis,
// engine choice and modulus count are kernels of the batch), final after Submission::wait.  C equals the
// host-array call bit for bit.  The ticket reports the engine and modulus count once the batch has run.
struct lf_linalg_ticket { std::shared_ptr<lfr::ResidentProduct> prod; };

namespace {
void resident_common(lf_linalg* la, lf_batch* bt, lf_buffer* C) {
    if (!la) throw invalid_argument("null linalg");
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    if (la->engine != bt->engine) throw invalid_argument("resident product: the batch belongs to another engine than the Linalg");
    if (!C) throw invalid_argument("missing output buffer");
}
void resident_record(lf_linalg* la, lf_batch* bt, std::shared_ptr<ResidentProduct> prod, lf_linalg_ticket** out) {
    auto& list = la->resident;
    list.erase(std::remove_if(list.begin(), list.end(), [](const std::weak_ptr<ResidentProduct>& w) { return w.expired(); }), list.end());
    list.push_back(prod);
    // the product counts as held by the batch until the batch's last copy of the op is gone
    struct BatchHold {
        std::shared_ptr<ResidentProduct> p;
        ~BatchHold() { if (p) resident_product_hold(*p, false); }
    };
    auto hold = std::make_shared<BatchHold>();
    hold->p = prod;
    resident_product_hold(*prod, true);
    Op o;
    o.kind = kCustom;
    o.custom = [hold](cudaStream_t s) { resident_product_launch(*hold->p, s); };
    bt->ops.push_back(o);
    *out = new lf_linalg_ticket{std::move(prod)};
}
}  // namespace

extern "C" {

int lf_linalg_batch_gemm(lf_linalg* la, lf_batch* bt, int bits, int transpose_a, lf_buffer* A, lf_buffer* B, size_t m, size_t n,
                         size_t k, lf_buffer* C, int subtract, lf_linalg_ticket** out) {
    LF_API_BEGIN
    resident_common(la, bt, C);
    if (!out) throw invalid_argument("null ticket");
    check_bits(bits);
    validate_dims(m, n, k, n);
    const size_t eb = size_t(bits / 8 + 12);
    if (!A || !B) throw invalid_argument("missing input buffer");
    if (A == C || B == C) throw invalid_argument("resident product: C must not be A or B");
    if (A->bytes < m * k * eb || B->bytes < k * n * eb || C->bytes < m * n * eb) throw invalid_argument("resident product: undersized buffer");
    bt->retain(A); bt->retain(B); bt->retain(C, true);
    bt->engine->activate();
    const bool limb = la->options.method == 1 || la->options.force_fallback;
    const auto* a = static_cast<const uint32_t*>(A->dev);
    lfd::LineView lv = transpose_a ? lfd::LineView{a, 1, m} : lfd::LineView{a, k, 1};
    lfd::LineView rv{static_cast<const uint32_t*>(B->dev), 1, n};
    resident_record(la, bt, resident_product_create(bits, lv, rv, m, n, k, static_cast<uint32_t*>(C->dev), n, subtract != 0, false, false, limb),
                    out);
    LF_API_END
}

int lf_linalg_batch_syrk(lf_linalg* la, lf_batch* bt, int bits, lf_buffer* A, size_t rows, size_t cols, lf_buffer* C, int lower_only,
                         int subtract, lf_linalg_ticket** out) {
    LF_API_BEGIN
    resident_common(la, bt, C);
    if (!out) throw invalid_argument("null ticket");
    check_bits(bits);
    if (subtract && !lower_only) throw invalid_argument("syrk: subtract updates the lower triangle only (lower_only)");
    validate_dims(cols, cols, rows, cols);
    const size_t eb = size_t(bits / 8 + 12);
    if (!A) throw invalid_argument("missing input buffer");
    if (A == C) throw invalid_argument("resident product: C must not be A");
    if (A->bytes < rows * cols * eb || C->bytes < cols * cols * eb) throw invalid_argument("resident product: undersized buffer");
    bt->retain(A); bt->retain(C, true);
    bt->engine->activate();
    const bool limb = la->options.method == 1 || la->options.force_fallback;
    lfd::LineView v{static_cast<const uint32_t*>(A->dev), 1, cols};
    resident_record(la, bt, resident_product_create(bits, v, v, cols, cols, rows, static_cast<uint32_t*>(C->dev), cols, subtract != 0, true,
                                                !lower_only, limb), out);
    LF_API_END
}

// LinalgTicket::resolved (linalg.hpp:61): the product has run (its submission completed).
int lf_linalg_ticket_resolved(lf_linalg_ticket* t, int* resolved) {
    LF_API_BEGIN
    if (!t || !resolved) throw invalid_argument("null argument");
    *resolved = resident_product_done(*t->prod) ? 1 : 0;
    LF_API_END
}
// LinalgTicket::report (linalg.hpp:62): the engine, modulus count and band the GPU chose; logic_error before
// the product has run, runtime_error when a cluster of terms overflowed the exact window.
int lf_linalg_ticket_report(lf_linalg_ticket* t, lf_linalg_report* rep) {
    LF_API_BEGIN
    if (!t || !rep) throw invalid_argument("null argument");
    if (!resident_product_done(*t->prod)) throw logic_error("ticket not resolved: wait for the submission first");
    if (!resident_product_report(*t->prod, *rep)) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    LF_API_END
}
void lf_linalg_ticket_destroy(lf_linalg_ticket* t) { delete t; }

// Linalg::workspaces / release_workspaces (linalg.hpp:173-180): device memory the Linalg retains between
// calls.  Scratch is the staging and work memory of the host-array calls and factorizations; a resident
// product's workspace is idle once its batch has run and busy while the batch is unsubmitted or in flight.
static lf_linalg_workspaces linalg_workspaces(Linalg& la) {
    lf_linalg_workspaces w{};
    for (auto& b : la.work) w.scratch_bytes += b.bytes;
    for (auto& b : la.qr) w.scratch_bytes += b.bytes;
    w.scratch_bytes += la.info_buf.bytes + la.error_buf.bytes + la.lines.bytes + la.residue.bytes() + la.lines2.bytes + la.residue2.bytes();
    for (auto& weak : la.resident) {
        auto r = weak.lock();
        if (!r) continue;
        const size_t b = resident_product_bytes(*r);
        if (!b) continue;                               // released
        if (resident_product_busy(*r)) { w.busy_bytes += b; ++w.busy_workspaces; }
        else w.idle_bytes += b;
    }
    return w;
}
int lf_linalg_get_workspaces(lf_linalg* la, lf_linalg_workspaces* out) {
    LF_API_BEGIN
    if (!la || !out) throw invalid_argument("null argument");
    la->engine->activate();
    *out = linalg_workspaces(*la);
    LF_API_END
}
// Frees the scratch and the idle resident workspaces now (their tickets keep their reports); busy ones stay
// with their batches and are freed with them.  Returns what was retained before the release.  Later calls
// allocate afresh.  Call between this Linalg's calls, on its host thread.
int lf_linalg_release_workspaces(lf_linalg* la, lf_linalg_workspaces* out) {
    LF_API_BEGIN
    if (!la) throw invalid_argument("null linalg");
    la->engine->activate();
    cuda_check(cudaStreamSynchronize(la->engine->stream), "release workspaces");
    const lf_linalg_workspaces w = linalg_workspaces(*la);
    for (auto& b : la->work) b = DevBuf{};
    for (auto& b : la->qr) b = DevBuf{};
    la->info_buf = DevBuf{}; la->error_buf = DevBuf{}; la->lines = DevBuf{}; la->lines2 = DevBuf{};
    la->residue.release();
    la->residue2.release();
    auto& list = la->resident;
    for (auto& weak : list) if (auto r = weak.lock()) resident_product_release(*r);
    list.erase(std::remove_if(list.begin(), list.end(), [](const std::weak_ptr<ResidentProduct>& x) {
        auto r = x.lock();
        return !r || resident_product_bytes(*r) == 0;
    }), list.end());
    if (out) *out = w;
    LF_API_END
}

}  // extern "C"

// ---- Householder QR (linalg.hpp:88-137, linalg.mm:488-849) ----
namespace lfr {

struct QrFactor {
    Linalg* owner = nullptr;
    int bits = 0;
    size_t m = 0, n = 0, nb = 0, block = 32;    // nb: the factor's block; block: the option the solves use
    bool pivot = false;
    bool cplx = false;                           // a complex factor (linalg_complex.mm): complex arrays, real embeddings
    lf_qr_info info{};
    // The accessors' arrays.  The factor keeps R, V and T on the device and copies them to these arrays the first
    // time an accessor asks (host_pending): a factorization followed by solves or Q applications moves no factor data
    // to the host.
    mutable std::vector<uint32_t> R, V, T, tau;
    std::vector<size_t> perm;
    DevBuf dV, dT, dR;                           // device copies for the solves and Q applications (complex: the embeddings)
    DevBuf cV, cT, cR;                           // complex: the factor's own complex arrays, for the accessors
    mutable bool host_pending = false;
    mutable std::mutex host_mutex;
    void materialize() const {
        std::lock_guard<std::mutex> lock(host_mutex);
        if (!host_pending) return;
        const size_t E = size_t(bits / 32 + 3) * (cplx ? 2 : 1), eb = 4 * E, blocks = nb ? (n + nb - 1) / nb : 0;
        const void* sR = cplx ? cR.p : dR.p;
        const void* sV = cplx ? cV.p : dV.p;
        const void* sT = cplx ? cT.p : dT.p;
        Engine& e = *owner->engine;
        e.activate();
        R.resize(n * n * E); V.resize(m * n * E); T.resize(blocks * nb * nb * E);
        cuda_check(cudaMemcpyAsync(R.data(), sR, n * n * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        cuda_check(cudaMemcpyAsync(V.data(), sV, m * n * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        if (blocks) cuda_check(cudaMemcpyAsync(T.data(), sT, blocks * nb * nb * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        cuda_check(cudaStreamSynchronize(e.stream), "download");
        host_pending = false;
    }
};

// Block b of the compact-WY factor (V: mE x nE, T: blocks of nbE x nbE, all real) applied to columns [c0, c1) of X
// (row stride ld): W = P(V_b^T X) over rows [k0, mE), Y = P(T_b^T W) (qt) or P(T_b W), X = D(X; V_b, Y), each with the
// whole block; with have_y, Y is given (qr_block, linalg.mm:550-567).  The complex factor passes its real embeddings
// with doubled dimensions and its row-split work matrix.
static void qr_block_update(Linalg& la, const ProductLane& lane, int bits, const uint32_t* V, const uint32_t* T, size_t mE, size_t nE,
                            size_t nbE, size_t b, uint32_t* X, size_t ld, size_t c0, size_t c1, bool qt, uint32_t* Wb, uint32_t* Yb,
                            bool have_y, cudaStream_t q) {
    const size_t E = bits / 32 + 3;
    const size_t k0 = b * nbE, kb = std::min(nE, k0 + nbE) - k0, mr = mE - k0, c = c1 - c0;
    if (!c || !kb) return;
    const uint32_t* Vb = V + (k0 * nE + k0) * E;
    const uint32_t* Tb = T + b * nbE * nbE * E;
    uint32_t* Xb = X + (k0 * ld + c0) * E;
    if (!have_y) {
        exact_product_on(la, lane, bits, {Vb, 1, nE}, {Xb, 1, ld}, kb, c, mr, Wb + c0 * E, ld, false, false, q, nullptr, false);
        const lfd::LineView tv = qt ? lfd::LineView{Tb, 1, nbE} : lfd::LineView{Tb, nbE, 1};
        exact_product_on(la, lane, bits, tv, {Wb + c0 * E, 1, ld}, kb, c, kb, Yb + c0 * E, ld, false, false, q, nullptr, false);
    }
    exact_product_on(la, lane, bits, {Vb, nE, 1}, {Yb + c0 * E, 1, ld}, mr, c, kb, Xb, ld, true, false, q, nullptr, false);
}

// Factor the device matrix Wk (m x n, reduced in place) into V, T, tau and R (all device).  Right-looking with
// one block of look-ahead (linalg.mm:721-745): after panel b, block b updates the next panel's columns on the
// engine's stream, and the rest of the trailing matrix on the side stream while the next panel is factored.
// After a failing column p in block b, block b (its reflectors before p; the rest of its V and T are zero) is
// applied to the columns after the block, unless p is the block's first column, and the factorization stops.
static lf_qr_info qr_device(Linalg& la, int bits, uint32_t* Wk, size_t m, size_t n, size_t nb, int rank_bits, uint32_t* V,
                            uint32_t* T, uint32_t* tau, uint32_t* R) {
    lf_qr_info info{};
    info.rank = n;
    auto w0 = Clock::now();
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3, eb = E * 4;
    const auto* qk = lfd::qr_kernels(limbs);
    const size_t blocks = nb ? (n + nb - 1) / nb : 0;
    cuda_check(cudaMemsetAsync(V, 0, m * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(T, 0, blocks * nb * nb * eb, s), "memset");
    cuda_check(cudaMemsetAsync(tau, 0, n * eb, s), "memset");
    uint32_t* Wb = static_cast<uint32_t*>(la.qr[0].get(nb * n * eb + 16));
    uint32_t* Yb = static_cast<uint32_t*>(la.qr[1].get(nb * n * eb + 16));
    uint32_t* Pt = static_cast<uint32_t*>(la.qr[2].get(nb * m * eb + 16));
    uint32_t* Vt = static_cast<uint32_t*>(la.qr[3].get(nb * m * eb + 16));
    uint32_t* Wp = static_cast<uint32_t*>(la.qr[4].get(nb * nb * eb + 16));
    uint32_t* G = static_cast<uint32_t*>(la.qr[5].get(nb * eb + 16));
    uint32_t* y = static_cast<uint32_t*>(la.qr[6].get(nb * eb + 16));
    auto* st = static_cast<lfd::QrState*>(la.qr[7].get(sizeof(lfd::QrState)));
    lfd::QrState host{};
    host.rank = (long long)n;
    cuda_check(cudaMemcpyAsync(st, &host, sizeof host, cudaMemcpyHostToDevice, s), "state");
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane_a = main_lane(la), lane_b = side_lane(la);
    cudaStream_t s2 = la.side;
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    lfd::QrPanel P{Wk, m, n, V, T, tau, Pt, Vt, Wp, G, y, 0, 0, nb, 0, rank_bits, st, err};
    // panel [k0, k1) on the engine's stream; returns min(k1, rank) (the host reads the state once per panel)
    auto panel = [&](size_t k0, size_t k1) -> size_t {
        auto t = Clock::now();
        P.k0 = k0; P.kb = k1 - k0; P.mr = m - k0;
        qk->load(P, s);
        for (size_t c = 0; c < P.kb; ++c) {
            if (c) qk->update(P, c, s);
            qk->reflect(P, c, s);
            qk->dots(P, c, s);
            qk->tcol(P, c, s);
        }
        qk->store(P, s);
        cuda_check(cudaGetLastError(), "qr panel");
        cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
        cuda_check(cudaStreamSynchronize(s), "qr panel");
        ++info.blocks;
        info.panel_seconds += since(t);
        return std::min(k1, (size_t)host.rank);
    };
    // block b on columns [c0, c1): W = P(V_b^T X), Y = P(T_b^T W), X = D(X; V_b, Y) (qr_block, linalg.mm:550-567)
    auto update = [&](size_t b, size_t c0, size_t c1, const ProductLane& lane, cudaStream_t q) {
        auto t = Clock::now();
        qr_block_update(la, lane, bits, V, T, m, n, nb, b, Wk, n, c0, c1, true, Wb, Yb, false, q);
        ++info.gpu_updates;
        info.update_seconds += since(t);
    };
    bool side_pending = false;
    size_t k0 = 0, k1 = std::min(n, nb), p = n ? panel(0, k1) : 0;
    while (k1 < n) {
        const size_t b = k0 / nb;
        // block b-1's remainder update (side stream) covered the columns from k1 on
        if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
        if (p < k1) {
            if (p > k0) update(b, k1, n, lane_a, s);
            break;
        }
        const size_t k2 = std::min(n, k1 + nb);
        update(b, k1, k2, lane_a, s);
        if (k2 < n) {
            // panel b is complete (the host read its state), so the side stream may read V_b and T_b
            update(b, k2, n, lane_b, s2);
            cuda_check(cudaEventRecord(la.ev_side, s2), "event");
            side_pending = true;
        }
        p = panel(k1, k2);
        k0 = k1; k1 = k2;
    }
    if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
    qk->extract(Wk, R, n, st, s);
    cuda_check(cudaGetLastError(), "qr extract");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "qr");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1] | ev[2]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    info.rank = (size_t)host.rank; info.reason = host.reason; info.status = host.status;
    info.timing = {ms * 1e-3, since(w0)};
    return info;
}

// Column-pivoted factorization (the pivoted branch of linalg.mm:600-731; no look-ahead: the next panel's columns
// are chosen during it).  Each step picks the pivot, reduces the column with its Y entries, forms the reflector,
// the Gram column and the W rows of every trailing column, then their Y rows, row j of R and the downdated norms
// (recomputed where they collapse).  After the panel the block updates the trailing columns with those Y rows,
// X = D(X; V_b, Y); after a failing column p it forms W and Y afresh for columns [p, n) and stops.  perm (n) receives
// the permutation.
static lf_qr_info qr_device_pivoted(Linalg& la, int bits, uint32_t* Wk, size_t m, size_t n, size_t nb, int rank_bits, uint32_t* V,
                                    uint32_t* T, uint32_t* tau, uint32_t* R, size_t* perm_out) {
    lf_qr_info info{};
    info.rank = n;
    auto w0 = Clock::now();
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3, eb = E * 4;
    const auto* qk = lfd::qr_kernels(limbs);
    const size_t blocks = nb ? (n + nb - 1) / nb : 0;
    cuda_check(cudaMemsetAsync(V, 0, m * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(T, 0, blocks * nb * nb * eb, s), "memset");
    cuda_check(cudaMemsetAsync(tau, 0, n * eb, s), "memset");
    uint32_t* Wb = static_cast<uint32_t*>(la.qr[0].get(nb * n * eb + 16));
    uint32_t* Yb = static_cast<uint32_t*>(la.qr[1].get(nb * n * eb + 16));
    cuda_check(cudaMemsetAsync(Wb, 0, nb * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(Yb, 0, nb * n * eb, s), "memset");
    uint32_t* Pt = static_cast<uint32_t*>(la.qr[2].get(nb * m * eb + 16));
    uint32_t* Vt = static_cast<uint32_t*>(la.qr[3].get(nb * m * eb + 16));
    uint32_t* G = static_cast<uint32_t*>(la.qr[5].get(nb * eb + 16));
    auto* st = static_cast<lfd::QrState*>(la.qr[7].get(sizeof(lfd::QrState)));
    uint32_t* nu = static_cast<uint32_t*>(la.qr[11].get(2 * n * eb + 16));
    auto* perm = static_cast<uint64_t*>(la.qr[12].get(n * 12 + 16));
    uint32_t* flag = reinterpret_cast<uint32_t*>(perm + n);
    cuda_check(cudaMemsetAsync(flag, 0, n * 4, s), "memset");
    lfd::QrState host{};
    host.rank = (long long)n;
    cuda_check(cudaMemcpyAsync(st, &host, sizeof host, cudaMemcpyHostToDevice, s), "state");
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane = main_lane(la);
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    lfd::QrPanel P{Wk, m, n, V, T, tau, Pt, Vt, nullptr, G, nullptr, 0, 0, nb, 0, rank_bits, st, err,
                   1, Wb, Yb, nu, nu + n * E, perm, flag};
    qk->norms(P, s);
    for (size_t k0 = 0; k0 < n; k0 += nb) {
        const size_t k1 = std::min(n, k0 + nb), b = k0 / nb;
        auto t = Clock::now();
        P.k0 = k0; P.kb = k1 - k0; P.mr = m - k0;
        qk->load(P, s);
        for (size_t c = 0; c < P.kb; ++c) {
            qk->pivot(P, c, s);
            qk->column(P, c, s);
            qk->reflect(P, c, s);
            qk->gramw(P, c, s);
            qk->trailing(P, c, s);
            qk->recompute(P, c, s);
        }
        qk->store(P, s);
        cuda_check(cudaGetLastError(), "pivoted qr panel");
        cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
        cuda_check(cudaStreamSynchronize(s), "pivoted qr panel");
        ++info.blocks;
        info.panel_seconds += since(t);
        t = Clock::now();
        const size_t p = std::min(k1, (size_t)host.rank), kb = k1 - k0, mr = m - k0;
        const uint32_t* Vb = V + (k0 * n + k0) * E;
        const uint32_t* Tb = T + b * nb * nb * E;
        if (p < k1) {
            // reflectors [k0, p) on columns [p, n) with W and Y formed afresh (qr_block without have_y)
            if (p > k0) {
                const size_t c = n - p;
                exact_product_on(la, lane, bits, {Vb, 1, n}, {Wk + (k0 * n + p) * E, 1, n}, kb, c, mr, Wb + p * E, n, false, false, s,
                                 nullptr, false);
                exact_product_on(la, lane, bits, {Tb, 1, nb}, {Wb + p * E, 1, n}, kb, c, kb, Yb + p * E, n, false, false, s, nullptr, false);
                exact_product_on(la, lane, bits, {Vb, n, 1}, {Yb + p * E, 1, n}, mr, c, kb, Wk + (k0 * n + p) * E, n, true, false, s,
                                 nullptr, false);
                ++info.gpu_updates;
            }
            info.update_seconds += since(t);
            break;
        }
        if (k1 < n) {
            // X = D(X; V_b, Y) with the Y rows of the panel
            exact_product_on(la, lane, bits, {Vb, n, 1}, {Yb + k1 * E, 1, n}, mr, n - k1, kb, Wk + (k0 * n + k1) * E, n, true, false, s,
                             nullptr, false);
            ++info.gpu_updates;
        }
        info.update_seconds += since(t);
    }
    qk->extract(Wk, R, n, st, s);
    cuda_check(cudaGetLastError(), "qr extract");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    std::vector<uint64_t> hp(n);
    cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
    cuda_check(cudaMemcpyAsync(hp.data(), perm, n * 8, cudaMemcpyDeviceToHost, s), "permutation");
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "pivoted qr");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    for (size_t k = 0; k < n; ++k) perm_out[k] = (size_t)hp[k];
    info.rank = (size_t)host.rank; info.reason = host.reason; info.status = host.status;
    info.norm_recomputations = host.recomputed;
    info.timing = {ms * 1e-3, since(w0)};
    return info;
}

// Complex factorization (linalg_complex.mm:125-306) of the row-split device matrix Wk (2m x n real, reduced in place) into
// V, T, tau, R (complex) and the real embeddings EV (2m x 2n), ET (blocks of 2nb x 2nb), ER (2n x 2n).  The loop and the
// look-ahead are the real factorization's; the trailing updates are qr_block_update on the embeddings.
static lf_qr_info cqr_device(Linalg& la, int bits, uint32_t* Wk, size_t m, size_t n, size_t nb, int rank_bits, uint32_t* V, uint32_t* T,
                             uint32_t* tau, uint32_t* R, uint32_t* EV, uint32_t* ET, uint32_t* ER) {
    lf_qr_info info{};
    info.rank = n;
    auto w0 = Clock::now();
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3, eb = E * 4, cb = 2 * eb;
    const auto* ck = lfd::cqr_kernels(limbs);
    const size_t blocks = nb ? (n + nb - 1) / nb : 0;
    cuda_check(cudaMemsetAsync(V, 0, m * n * cb, s), "memset");
    cuda_check(cudaMemsetAsync(T, 0, blocks * nb * nb * cb, s), "memset");
    cuda_check(cudaMemsetAsync(tau, 0, n * cb, s), "memset");
    cuda_check(cudaMemsetAsync(EV, 0, 4 * m * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(ET, 0, 4 * blocks * nb * nb * eb, s), "memset");
    uint32_t* Wb = static_cast<uint32_t*>(la.qr[0].get(2 * nb * n * eb + 16));
    uint32_t* Yb = static_cast<uint32_t*>(la.qr[1].get(2 * nb * n * eb + 16));
    uint32_t* Pt = static_cast<uint32_t*>(la.qr[2].get(4 * nb * m * cb + 16));       // Pt, Vt, Vi, Vr
    uint32_t* Vt = Pt + nb * m * 2 * E;
    uint32_t* Vi = Vt + nb * m * 2 * E;
    uint32_t* Vr = Vi + nb * m * 2 * E;
    uint32_t* Wp = static_cast<uint32_t*>(la.qr[4].get((nb * nb + 6 * nb) * cb + 3 * nb * nb * cb + 16));
    uint32_t* G = Wp + nb * nb * 2 * E;
    uint32_t* Gc = G + nb * 2 * E;
    uint32_t* Gic = Gc + nb * 2 * E;
    uint32_t* yc = Gic + nb * 2 * E;
    uint32_t* yic = yc + nb * 2 * E;
    uint32_t* scr = yic + 2 * nb * 2 * E;
    auto* st = static_cast<lfd::QrState*>(la.qr[7].get(sizeof(lfd::QrState)));
    lfd::QrState host{};
    host.rank = (long long)n;
    cuda_check(cudaMemcpyAsync(st, &host, sizeof host, cudaMemcpyHostToDevice, s), "state");
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane_a = main_lane(la), lane_b = side_lane(la);
    cudaStream_t s2 = la.side;
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    lfd::CqrPanel P{Wk, m, n, V, T, tau, EV, ET, Pt, Vt, Vi, Vr, Wp, G, Gc, Gic, yc, yic, scr, 0, 0, nb, 0, rank_bits, st, err};
    auto panel = [&](size_t k0, size_t k1) -> size_t {
        auto t = Clock::now();
        P.k0 = k0; P.kb = k1 - k0; P.mr = m - k0;
        ck->load(P, s);
        for (size_t c = 0; c < P.kb; ++c) {
            if (c) ck->update(P, c, s);
            ck->reflect(P, c, s);
            ck->dots(P, c, s);
            ck->tcol(P, c, s);
        }
        ck->store(P, s);
        cuda_check(cudaGetLastError(), "complex qr panel");
        cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
        cuda_check(cudaStreamSynchronize(s), "complex qr panel");
        ++info.blocks;
        info.panel_seconds += since(t);
        return std::min(k1, (size_t)host.rank);
    };
    auto update = [&](size_t b, size_t c0, size_t c1, const ProductLane& lane, cudaStream_t q) {
        auto t = Clock::now();
        qr_block_update(la, lane, bits, EV, ET, 2 * m, 2 * n, 2 * nb, b, Wk, n, c0, c1, true, Wb, Yb, false, q);
        ++info.gpu_updates;
        info.update_seconds += since(t);
    };
    bool side_pending = false;
    size_t k0 = 0, k1 = std::min(n, nb), p = n ? panel(0, k1) : 0;
    while (k1 < n) {
        const size_t b = k0 / nb;
        if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
        if (p < k1) {
            if (p > k0) update(b, k1, n, lane_a, s);
            break;
        }
        const size_t k2 = std::min(n, k1 + nb);
        update(b, k1, k2, lane_a, s);
        if (k2 < n) {
            update(b, k2, n, lane_b, s2);
            cuda_check(cudaEventRecord(la.ev_side, s2), "event");
            side_pending = true;
        }
        p = panel(k1, k2);
        k0 = k1; k1 = k2;
    }
    if (side_pending) cuda_check(cudaStreamWaitEvent(s, la.ev_side, 0), "event wait");
    ck->extract(Wk, R, ER, n, st, s);
    cuda_check(cudaGetLastError(), "complex qr extract");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "complex qr");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1] | ev[2]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    info.rank = (size_t)host.rank; info.reason = host.reason; info.status = host.status;
    info.timing = {ms * 1e-3, since(w0)};
    return info;
}

// Column-pivoted complex QR (linalg_complex.mm:136-139, 160-290): per column step the pivot choice and swap, the
// column's reduction with its Y rows, the reflector, the Gram entries with the W rows of every trailing column and
// the T column, the Y rows with the downdated norms, and recomputation of collapsed norms; after each panel the
// trailing matrix is updated with the panel's Y rows (X = D(X; EV_b, Y)).  No look-ahead, as in the reference.  After
// a failing column p in block b, block b (formed afresh) is applied to the columns [p, n) and the factorization stops.
static lf_qr_info cqr_device_pivoted(Linalg& la, int bits, uint32_t* Wk, size_t m, size_t n, size_t nb, int rank_bits, uint32_t* V,
                                     uint32_t* T, uint32_t* tau, uint32_t* R, uint32_t* EV, uint32_t* ET, uint32_t* ER, size_t* perm_out) {
    lf_qr_info info{};
    info.rank = n;
    auto w0 = Clock::now();
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const int limbs = bits / 32;
    const size_t E = limbs + 3, eb = E * 4, cb = 2 * eb;
    const auto* ck = lfd::cqr_kernels(limbs);
    const auto* qk = lfd::qr_kernels(limbs);
    const size_t blocks = nb ? (n + nb - 1) / nb : 0;
    cuda_check(cudaMemsetAsync(V, 0, m * n * cb, s), "memset");
    cuda_check(cudaMemsetAsync(T, 0, blocks * nb * nb * cb, s), "memset");
    cuda_check(cudaMemsetAsync(tau, 0, n * cb, s), "memset");
    cuda_check(cudaMemsetAsync(EV, 0, 4 * m * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(ET, 0, 4 * blocks * nb * nb * eb, s), "memset");
    uint32_t* Wb = static_cast<uint32_t*>(la.qr[0].get(2 * nb * n * eb + 16));
    uint32_t* Yb = static_cast<uint32_t*>(la.qr[1].get(2 * nb * n * eb + 16));
    cuda_check(cudaMemsetAsync(Wb, 0, 2 * nb * n * eb, s), "memset");
    cuda_check(cudaMemsetAsync(Yb, 0, 2 * nb * n * eb, s), "memset");
    uint32_t* Pt = static_cast<uint32_t*>(la.qr[2].get(4 * nb * m * cb + 16));       // Pt, Vt, Vi, Vr
    uint32_t* Vt = Pt + nb * m * 2 * E;
    uint32_t* Vi = Vt + nb * m * 2 * E;
    uint32_t* Vr = Vi + nb * m * 2 * E;
    uint32_t* Wp = static_cast<uint32_t*>(la.qr[4].get((nb * nb + 6 * nb) * cb + 3 * nb * nb * cb + 16));
    uint32_t* G = Wp + nb * nb * 2 * E;
    uint32_t* Gc = G + nb * 2 * E;
    uint32_t* Gic = Gc + nb * 2 * E;
    uint32_t* Vrc = static_cast<uint32_t*>(la.qr[6].get((2 * nb * m + 2 * nb) * cb + 16));   // Vrc, Vri, tc
    uint32_t* Vri = Vrc + nb * m * 2 * E;
    uint32_t* tc = Vri + nb * m * 2 * E;
    auto* st = static_cast<lfd::QrState*>(la.qr[7].get(sizeof(lfd::QrState)));
    uint32_t* nu = static_cast<uint32_t*>(la.qr[11].get(2 * n * eb + 16));
    auto* perm = static_cast<uint64_t*>(la.qr[12].get(n * 12 + 16));
    uint32_t* flag = reinterpret_cast<uint32_t*>(perm + n);
    cuda_check(cudaMemsetAsync(flag, 0, n * 4, s), "memset");
    lfd::QrState host{};
    host.rank = (long long)n;
    cuda_check(cudaMemcpyAsync(st, &host, sizeof host, cudaMemcpyHostToDevice, s), "state");
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane = main_lane(la);
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    // squared norms over the 2m split rows: the real kernel on the split matrix
    lfd::QrPanel Q{};
    Q.Wk = Wk; Q.m = 2 * m; Q.n = n; Q.st = st; Q.error = err; Q.pivot = 1; Q.nu = nu; Q.nuref = nu + n * E; Q.perm = perm;
    qk->norms(Q, s);
    lfd::CqrPanel P{Wk, m, n, V, T, tau, EV, ET, Pt, Vt, Vi, Vr, Wp, G, Gc, Gic, nullptr, nullptr, nullptr, 0, 0, nb, 0, rank_bits, st, err,
                    1, Wb, Yb, nu, nu + n * E, perm, flag, Vrc, Vri, tc};
    for (size_t k0 = 0; k0 < n; k0 += nb) {
        const size_t k1 = std::min(n, k0 + nb), b = k0 / nb;
        auto t = Clock::now();
        P.k0 = k0; P.kb = k1 - k0; P.mr = m - k0;
        ck->load(P, s);
        for (size_t c = 0; c < P.kb; ++c) {
            ck->pivot(P, c, s);
            ck->column(P, c, s);
            ck->reflect(P, c, s);
            ck->gramw(P, c, s);
            ck->trailing(P, c, s);
            ck->recompute(P, c, s);
        }
        ck->store(P, s);
        cuda_check(cudaGetLastError(), "pivoted complex qr panel");
        cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
        cuda_check(cudaStreamSynchronize(s), "pivoted complex qr panel");
        ++info.blocks;
        info.panel_seconds += since(t);
        t = Clock::now();
        const size_t p = std::min(k1, (size_t)host.rank);
        if (p < k1) {
            if (p > k0) {
                qr_block_update(la, lane, bits, EV, ET, 2 * m, 2 * n, 2 * nb, b, Wk, n, p, n, true, Wb, Yb, false, s);
                ++info.gpu_updates;
            }
            info.update_seconds += since(t);
            break;
        }
        if (k1 < n) {
            qr_block_update(la, lane, bits, EV, ET, 2 * m, 2 * n, 2 * nb, b, Wk, n, k1, n, true, Wb, Yb, true, s);
            ++info.gpu_updates;
        }
        info.update_seconds += since(t);
    }
    ck->extract(Wk, R, ER, n, st, s);
    cuda_check(cudaGetLastError(), "complex qr extract");
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev[3] = {0, 0, 0};
    std::vector<uint64_t> pm(n);
    cuda_check(cudaMemcpyAsync(&host, st, sizeof host, cudaMemcpyDeviceToHost, s), "state");
    cuda_check(cudaMemcpyAsync(ev, err, 12, cudaMemcpyDeviceToHost, s), "error flag");
    if (n) cuda_check(cudaMemcpyAsync(pm.data(), perm, n * 8, cudaMemcpyDeviceToHost, s), "permutation");
    cuda_check(cudaStreamSynchronize(s), "pivoted complex qr");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev[0] | ev[1] | ev[2]) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    for (size_t k = 0; k < n; ++k) perm_out[k] = (size_t)pm[k];
    info.rank = (size_t)host.rank; info.reason = host.reason; info.status = host.status;
    info.norm_recomputations = host.recomputed;
    info.timing = {ms * 1e-3, since(w0)};
    return info;
}

// C (device, m x nrhs) <- Q^T C (qt: blocks in order) or Q C (blocks in reverse) over the blocks holding reflectors
// [0, rank) (qr_apply_n, linalg.mm:750-766).  Returns the device seconds.
static double qr_apply_device(Linalg& la, const QrFactor& f, uint32_t* C, size_t nrhs, bool qt) {
    const size_t nb = f.nb, blocks = nb ? (f.info.rank + nb - 1) / nb : 0;
    if (!blocks || !nrhs || !f.m) return 0;
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    const size_t k = f.cplx ? 2 : 1;                    // a complex factor applies its real embeddings to row-split C
    const size_t eb = (f.bits / 32 + 3) * 4;
    uint32_t* Wb = static_cast<uint32_t*>(la.qr[0].get(k * nb * nrhs * eb + 16));
    uint32_t* Yb = static_cast<uint32_t*>(la.qr[1].get(k * nb * nrhs * eb + 16));
    uint32_t* err = static_cast<uint32_t*>(la.error_buf.get(16));
    cuda_check(cudaMemsetAsync(err, 0, 16, s), "memset");
    const ProductLane lane = main_lane(la);
    cudaEvent_t g0, g1;
    cuda_check(cudaEventCreate(&g0), "event"); cuda_check(cudaEventCreate(&g1), "event");
    cuda_check(cudaEventRecord(g0, s), "event");
    for (size_t q = 0; q < blocks; ++q)
        qr_block_update(la, lane, f.bits, static_cast<const uint32_t*>(f.dV.p), static_cast<const uint32_t*>(f.dT.p), k * f.m, k * f.n,
                        k * nb, qt ? q : blocks - 1 - q, C, nrhs, 0, nrhs, qt, Wb, Yb, false, s);
    cuda_check(cudaEventRecord(g1, s), "event");
    uint32_t ev = 0;
    cuda_check(cudaMemcpyAsync(&ev, lane.err, 4, cudaMemcpyDeviceToHost, s), "error flag");
    cuda_check(cudaStreamSynchronize(s), "qr apply");
    float ms = 0; cudaEventElapsedTime(&ms, g0, g1);
    cudaEventDestroy(g0); cudaEventDestroy(g1);
    if (ev) throw runtime_error("exact product: a device error word was set (a bounded wait gave up)");
    return ms * 1e-3;
}

// Least squares on the device: C (m x nrhs, holding B) <- Q^T C, then the backward substitution with R (upper;
// pivoted: its leading rank x rank block) on C's first rows (qr_solve_n, linalg.mm:768-786).  Returns the device
// seconds; the caller reads the first min(rank, n) rows.  Callers handle the rank-deficient cases that write
// invalid zeros.
static double qr_solve_device(Linalg& la, const QrFactor& f, uint32_t* C, size_t nrhs) {
    double g = qr_apply_device(la, f, C, nrhs, true);
    // complex: the real backward substitution of the 2n x 2n embedding of R, blocks 2 min(nb, p) (linalg_complex.mm:339-342)
    const size_t k = f.cplx ? 2 : 1, p = k * f.info.rank, n = k * f.n;
    const size_t block = f.cplx ? 2 * std::min(f.nb, f.info.rank) : f.block;
    if (!p) return g;
    if (p < n) {
        const size_t eb = (f.bits / 32 + 3) * 4;
        uint32_t* R11 = static_cast<uint32_t*>(la.qr[9].get(p * p * eb + 16));
        lfd::qr_kernels(f.bits / 32)->copy(static_cast<const uint32_t*>(f.dR.p), n, R11, p, p, p, la.engine->stream);
        cuda_check(cudaGetLastError(), "qr leading block");
        g += solve_device(la, f.bits, R11, p, C, nrhs, block, 2, true);
    } else {
        g += solve_device(la, f.bits, static_cast<const uint32_t*>(f.dR.p), n, C, nrhs, block, 2, true);
    }
    return g;
}
// A complex matrix (rows x cols elements of (re, im), E words each) to the row-split real layout, on the device: one
// thread per word of A.
__global__ void split_rows_kernel(const uint32_t* A, uint32_t* W, uint64_t rows, uint64_t cols, uint64_t E) {
    const uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= rows * cols * 2 * E) return;
    const uint64_t el = q / (2 * E), k = q % (2 * E), part = k / E, w = k % E;
    const uint64_t r = el / cols, c = el % cols;
    W[((2 * r + part) * cols + c) * E + w] = A[q];
}
// Complex host arrays <-> the row-split real layout the device works on (row 2r = Re of row r, 2r + 1 = Im).
static void split_rows(const uint32_t* A, size_t rows, size_t cols, size_t E, std::vector<uint32_t>& out) {
    out.resize(2 * rows * cols * E);
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < cols; ++c) {
            const uint32_t* z = A + (r * cols + c) * 2 * E;
            std::memcpy(&out[(2 * r * cols + c) * E], z, E * 4);
            std::memcpy(&out[((2 * r + 1) * cols + c) * E], z + E, E * 4);
        }
}
static void join_rows(const uint32_t* W, size_t rows, size_t cols, size_t E, uint32_t* out) {
    for (size_t r = 0; r < rows; ++r)
        for (size_t c = 0; c < cols; ++c) {
            uint32_t* z = out + (r * cols + c) * 2 * E;
            std::memcpy(z, W + (2 * r * cols + c) * E, E * 4);
            std::memcpy(z + E, W + ((2 * r + 1) * cols + c) * E, E * 4);
        }
}

static void check_qr_size(size_t n, size_t rows) {
    if (n >= 46341 || n * rows >= (size_t(1) << 31)) throw invalid_argument("matrix dimensions exceed 32-bit indexing");
}

// Factor the matrix already on the device at dA (m x n, left unchanged) into f's device arrays, then copy the
// factor to f's host arrays.
static void qr_factor_common(Linalg& la, QrFactor& f, const uint32_t* dA, int rank_bits) {
    const size_t eb = size_t(f.bits / 8 + 12), m = f.m, n = f.n;
    const size_t blocks = f.nb ? (n + f.nb - 1) / f.nb : 0;
    auto w0 = Clock::now();
    f.R.clear(); f.V.clear(); f.T.clear();
    f.host_pending = false;
    f.tau.assign(n * (eb / 4), 0);
    f.perm.resize(n);
    for (size_t k = 0; k < n; ++k) f.perm[k] = k;
    f.info = lf_qr_info{};
    f.info.rank = n;
    if (!n) return;
    Engine& e = *la.engine;
    cudaStream_t s = e.stream;
    uint32_t* Wk = static_cast<uint32_t*>(la.work[4].get(m * n * eb));
    cuda_check(cudaMemcpyAsync(Wk, dA, m * n * eb, cudaMemcpyDeviceToDevice, s), "work matrix");
    uint32_t* V = static_cast<uint32_t*>(f.dV.get(m * n * eb));
    uint32_t* T = static_cast<uint32_t*>(f.dT.get(blocks * f.nb * f.nb * eb + 16));
    uint32_t* R = static_cast<uint32_t*>(f.dR.get(n * n * eb));
    uint32_t* tau = static_cast<uint32_t*>(la.qr[10].get(n * eb));
    f.info = f.pivot ? qr_device_pivoted(la, f.bits, Wk, m, n, f.nb, rank_bits, V, T, tau, R, f.perm.data())
                     : qr_device(la, f.bits, Wk, m, n, f.nb, rank_bits, V, T, tau, R);
    (void)R; (void)V; (void)T;                   // kept on the device; copied on the first accessor call
    cuda_check(cudaMemcpyAsync(f.tau.data(), tau, n * eb, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "download");
    f.host_pending = true;
    f.info.timing.wall_seconds = since(w0);
}

}  // namespace lfr

struct lf_qr : QrFactor {};

extern "C" {

static QrFactor* qr_prepare(lf_linalg* la, int bits, size_t m, size_t n, const lf_qr_options* o) {
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    if (m < n) throw invalid_argument("factor_qr: rows >= columns required");
    check_qr_size(n, m);
    const lf_qr_options opts = o ? *o : lf_qr_options{32, 0, 0, 1, 0, 0};
    if (opts.rank_bits < 0) throw invalid_argument("factor_qr: rank_bits >= 0");
    auto* f = new lf_qr();
    f->owner = la; f->bits = bits; f->m = m; f->n = n;
    f->block = opts.block; f->nb = opts.block ? std::min(opts.block, n) : n; f->pivot = opts.pivot != 0;
    return f;
}

// Linalg::factor_qr (linalg.hpp:164): Householder QR of A (m x n, row-major, m >= n); A is only read.
int lf_linalg_factor_qr(lf_linalg* la, int bits, const void* A, size_t m, size_t n, const lf_qr_options* o, lf_qr** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null output");
    *out = nullptr;
    std::unique_ptr<lf_qr> f(static_cast<lf_qr*>(qr_prepare(la, bits, m, n, o)));
    if (m * n && !A) throw invalid_argument("null matrix");
    const size_t eb = size_t(bits / 8 + 12);
    auto w0 = Clock::now();
    if (n) {
        Engine& e = *la->engine;
        e.activate();
        uint32_t* dA = static_cast<uint32_t*>(la->work[3].get(m * n * eb));
        cuda_check(cudaMemcpyAsync(dA, A, m * n * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    }
    qr_factor_common(*la, *f, static_cast<const uint32_t*>(la->work[3].p), o ? o->rank_bits : 0);
    f->info.timing.wall_seconds = since(w0);
    *out = f.release();
    LF_API_END
}

// Linalg::factor_qr_augmented (linalg.hpp:168): the factor of [J; diag(d)] ((m + n) x n).
int lf_linalg_factor_qr_augmented(lf_linalg* la, int bits, const void* J, size_t m, size_t n, const void* d, const lf_qr_options* o,
                                  lf_qr** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null output");
    *out = nullptr;
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    check_qr_size(n, m + n);
    if (n && (!d || (m && !J))) throw invalid_argument("null matrix");
    const size_t eb = size_t(bits / 8 + 12);
    std::vector<unsigned char> S((m + n) * n * eb, 0);
    if (m * n) std::memcpy(S.data(), J, m * n * eb);
    for (size_t i = 0; i < n; ++i) std::memcpy(S.data() + ((m + i) * n + i) * eb, static_cast<const unsigned char*>(d) + i * eb, eb);
    const int rc = lf_linalg_factor_qr(la, bits, S.data(), m + n, n, o, out);
    if (rc != LF_OK) return rc;
    LF_API_END
}

// Linalg::factor_qr on a Buffer (linalg.hpp:200): synchronous, outside any batch; the buffer must be idle.
int lf_linalg_factor_qr_buffer(lf_linalg* la, int bits, lf_buffer* A, size_t m, size_t n, const lf_qr_options* o, lf_qr** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null output");
    *out = nullptr;
    std::unique_ptr<lf_qr> f(static_cast<lf_qr*>(qr_prepare(la, bits, m, n, o)));
    const size_t eb = size_t(bits / 8 + 12);
    Engine& e = *la->engine;
    BufferClaim claim;
    claim.take(A, e.identity);
    if (A->bytes < m * n * eb) throw invalid_argument("factor_qr: buffer smaller than m x n");
    auto w0 = Clock::now();
    e.activate();
    A->sync_to_device(e.stream);
    qr_factor_common(*la, *f, static_cast<const uint32_t*>(A->dev), o ? o->rank_bits : 0);
    f->info.timing.wall_seconds = since(w0);
    *out = f.release();
    LF_API_END
}

void lf_qr_destroy(lf_qr* f) { delete f; }

int lf_qr_describe(const lf_qr* f, int* bits, size_t* rows, size_t* cols, size_t* block, int* pivoted, lf_qr_info* info) {
    LF_API_BEGIN
    if (!f) throw logic_error("empty QR factor");
    if (bits) *bits = f->bits;
    if (rows) *rows = f->m;
    if (cols) *cols = f->n;
    if (block) *block = f->nb;
    if (pivoted) *pivoted = f->pivot ? 1 : 0;
    if (info) *info = f->info;
    LF_API_END
}
// The first call on a real factor copies R, V and T from the device; a failing copy gives nullptr and the error
// message (lf_last_error).
static const QrFactor* qr_host(const lf_qr* f) {
    if (!f) return nullptr;
    try { f->materialize(); } catch (const std::exception& e) { set_error(e.what()); return nullptr; }
    return f;
}
const void* lf_qr_r(const lf_qr* f) { const QrFactor* q = qr_host(f); return q && !q->R.empty() ? q->R.data() : nullptr; }
const void* lf_qr_v(const lf_qr* f) { const QrFactor* q = qr_host(f); return q && !q->V.empty() ? q->V.data() : nullptr; }
const void* lf_qr_tau(const lf_qr* f) { return f && !f->tau.empty() ? f->tau.data() : nullptr; }
const void* lf_qr_t(const lf_qr* f) { const QrFactor* q = qr_host(f); return q && !q->T.empty() ? q->T.data() : nullptr; }
const size_t* lf_qr_permutation(const lf_qr* f) { return f && !f->perm.empty() ? f->perm.data() : nullptr; }

// QRFactor::solve (linalg.hpp:127): X (n x nrhs) = the least-squares solution for each column of B (m x nrhs).
// A rank-deficient unpivoted factor writes zero with invalid to every entry; a status column zero with invalid and
// its status.  X must not overlap B.
int lf_qr_solve(const lf_qr* f, const void* B, size_t nrhs, void* X, lf_timing* timing) {
    LF_API_BEGIN
    if (!f) throw logic_error("empty QR factor");
    check_qr_size(f->cplx ? 2 * f->n : f->n, nrhs);
    check_qr_size(1, (f->cplx ? 4 : 1) * f->m * nrhs);
    if (timing) *timing = {0, 0};
    if (!f->n || !nrhs) return LF_OK;
    if (!B || !X) throw invalid_argument("null matrix");
    const size_t k = f->cplx ? 2 : 1;                    // components per element
    const size_t eb = size_t(f->bits / 8 + 12), E = eb / 4, m = f->m, n = f->n, p = f->info.rank;
    if (overlap(X, n * nrhs * k * eb, B, m * nrhs * k * eb)) throw invalid_argument("solve: X overlaps B");
    auto w0 = Clock::now();
    if (p < n && (!f->pivot || f->info.reason == 3)) {
        const uint32_t st = 4u | (f->pivot ? f->info.status : 0u);
        auto* x = static_cast<uint32_t*>(X);
        std::memset(x, 0, n * nrhs * k * eb);
        for (size_t q = 0; q < k * n * nrhs; ++q) x[q * E + E - 1] = st;
        if (timing) *timing = {0, since(w0)};
        return LF_OK;
    }
    Linalg& la = *f->owner;
    Engine& e = *la.engine;
    e.activate();
    // the device works on k m real rows (complex: split by rows); the solution is its first k min(p, n) rows
    uint32_t* C = static_cast<uint32_t*>(la.qr[8].get(k * m * nrhs * eb));
    std::vector<uint32_t> split;
    if (f->cplx) {
        split_rows(static_cast<const uint32_t*>(B), m, nrhs, E, split);
        cuda_check(cudaMemcpyAsync(C, split.data(), 2 * m * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    } else {
        cuda_check(cudaMemcpyAsync(C, B, m * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    }
    const double g = qr_solve_device(la, *f, C, nrhs);
    const size_t rows = std::min(p, n);
    std::vector<uint32_t> Z(k * rows * nrhs * E + 1), Zc;
    if (rows) cuda_check(cudaMemcpyAsync(Z.data(), C, k * rows * nrhs * eb, cudaMemcpyDeviceToHost, e.stream), "download");
    cuda_check(cudaStreamSynchronize(e.stream), "download");
    const uint32_t* z = Z.data();
    if (f->cplx) {
        Zc.resize(2 * rows * nrhs * E + 1);
        join_rows(Z.data(), rows, nrhs, E, Zc.data());
        z = Zc.data();
    }
    auto* x = static_cast<uint32_t*>(X);
    if (rows < n) std::memset(x, 0, n * nrhs * k * eb);
    for (size_t i = 0; i < rows; ++i) std::memcpy(x + f->perm[i] * nrhs * k * E, z + i * nrhs * k * E, nrhs * k * eb);
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}

// QRFactor::apply_q (linalg.hpp:129): B (m x nrhs) <- Q^T B (transpose) or Q B, in place; a complex factor's adjoint is Q^H.
int lf_qr_apply_q(const lf_qr* f, void* B, size_t nrhs, int transpose, lf_timing* timing) {
    LF_API_BEGIN
    if (!f) throw logic_error("empty QR factor");
    check_qr_size(f->cplx ? 2 * f->n : f->n, nrhs);
    check_qr_size(1, (f->cplx ? 4 : 1) * f->m * nrhs);
    if (timing) *timing = {0, 0};
    if (!f->m || !nrhs) return LF_OK;
    if (!B) throw invalid_argument("null matrix");
    const size_t k = f->cplx ? 2 : 1;
    const size_t eb = size_t(f->bits / 8 + 12), E = eb / 4, m = f->m;
    auto w0 = Clock::now();
    Linalg& la = *f->owner;
    Engine& e = *la.engine;
    e.activate();
    uint32_t* C = static_cast<uint32_t*>(la.qr[8].get(k * m * nrhs * eb));
    std::vector<uint32_t> split;
    if (f->cplx) {
        split_rows(static_cast<const uint32_t*>(B), m, nrhs, E, split);
        cuda_check(cudaMemcpyAsync(C, split.data(), 2 * m * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    } else {
        cuda_check(cudaMemcpyAsync(C, B, m * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "upload");
    }
    const double g = qr_apply_device(la, *f, C, nrhs, transpose != 0);
    if (f->cplx) {
        cuda_check(cudaMemcpyAsync(split.data(), C, 2 * m * nrhs * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        cuda_check(cudaStreamSynchronize(e.stream), "download");
        join_rows(split.data(), m, nrhs, E, static_cast<uint32_t*>(B));
    } else {
        cuda_check(cudaMemcpyAsync(B, C, m * nrhs * eb, cudaMemcpyDeviceToHost, e.stream), "download");
        cuda_check(cudaStreamSynchronize(e.stream), "download");
    }
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}

// Linalg::factor_qr_complex (linalg.hpp:170): complex Householder QR of A (m x n Complex<bits/32>, row-major, m >= n);
// the factor's arrays are complex and its solve and apply_q take complex matrices; with pivoting, column j of the
// factor is column perm[j] of A.
int lf_linalg_factor_qr_complex(lf_linalg* la, int bits, const void* A, size_t m, size_t n, const lf_qr_options* o, lf_qr** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null output");
    *out = nullptr;
    if (!la) throw invalid_argument("null linalg");
    check_bits(bits);
    if (m < n) throw invalid_argument("factor_qr_complex: rows >= columns required");
    if (2 * n >= 46341 || 4 * n * m >= (size_t(1) << 31)) throw invalid_argument("matrix dimensions exceed 32-bit indexing");
    if (m * n && !A) throw invalid_argument("null matrix");
    const lf_qr_options opts = o ? *o : lf_qr_options{32, 0, 0, 1, 0, 0};
    if (opts.rank_bits < 0) throw invalid_argument("factor_qr_complex: rank_bits >= 0");
    std::unique_ptr<lf_qr> f(new lf_qr());
    f->owner = la; f->bits = bits; f->m = m; f->n = n; f->cplx = true; f->pivot = opts.pivot != 0;
    f->block = opts.block; f->nb = opts.block ? std::min(opts.block, n) : n;
    const size_t eb = size_t(bits / 8 + 12), E = eb / 4, cb = 2 * eb;
    const size_t blocks = f->nb ? (n + f->nb - 1) / f->nb : 0;
    auto w0 = Clock::now();
    f->tau.assign(n * 2 * E, 0);
    f->perm.resize(n);
    for (size_t k = 0; k < n; ++k) f->perm[k] = k;
    f->info.rank = n;
    if (n) {
        Engine& e = *la->engine;
        e.activate();
        cudaStream_t s = e.stream;
        // A as it is, then split by rows on the device
        uint32_t* Ac = static_cast<uint32_t*>(la->qr[8].get(2 * m * n * eb));
        uint32_t* Wk = static_cast<uint32_t*>(la->work[4].get(2 * m * n * eb));
        cuda_check(cudaMemcpyAsync(Ac, A, 2 * m * n * eb, cudaMemcpyHostToDevice, s), "upload");
        const uint64_t words = 2 * (uint64_t)m * n * E;
        split_rows_kernel<<<(unsigned)((words + 255) / 256), 256, 0, s>>>(Ac, Wk, m, n, E);
        cuda_check(cudaGetLastError(), "split rows");
        DevBuf dtau;
        uint32_t* V = static_cast<uint32_t*>(f->cV.get(m * n * cb));
        uint32_t* T = static_cast<uint32_t*>(f->cT.get(blocks * f->nb * f->nb * cb + 16));
        uint32_t* R = static_cast<uint32_t*>(f->cR.get(n * n * cb));
        uint32_t* tau = static_cast<uint32_t*>(dtau.get(n * cb));
        uint32_t* EV = static_cast<uint32_t*>(f->dV.get(4 * m * n * eb));
        uint32_t* ET = static_cast<uint32_t*>(f->dT.get(4 * blocks * f->nb * f->nb * eb + 16));
        uint32_t* ER = static_cast<uint32_t*>(f->dR.get(4 * n * n * eb));
        f->info = f->pivot ? cqr_device_pivoted(*la, bits, Wk, m, n, f->nb, opts.rank_bits, V, T, tau, R, EV, ET, ER, f->perm.data())
                           : cqr_device(*la, bits, Wk, m, n, f->nb, opts.rank_bits, V, T, tau, R, EV, ET, ER);
        cuda_check(cudaMemcpyAsync(f->tau.data(), tau, n * cb, cudaMemcpyDeviceToHost, s), "download");
        cuda_check(cudaStreamSynchronize(s), "download");
        f->host_pending = true;                  // R, V and T are copied on the first accessor call
    } else {
        f->info.rank = 0;
    }
    f->info.timing.wall_seconds = since(w0);
    *out = f.release();
    LF_API_END
}
int lf_qr_is_complex(const lf_qr* f) { return f && f->cplx ? 1 : 0; }

// QRFactor::solve / apply_q on Buffers (linalg.hpp:131-134): synchronous, outside any batch, buffers idle.
int lf_qr_solve_buffers(const lf_qr* f, lf_buffer* B, size_t nrhs, lf_buffer* X, lf_timing* timing) {
    LF_API_BEGIN
    if (!f) throw logic_error("empty QR factor");
    if (f->cplx) throw invalid_argument("complex QR factors have no Buffer forms");
    check_qr_size(f->n, nrhs);
    check_qr_size(1, f->m * nrhs);
    const size_t eb = size_t(f->bits / 8 + 12), E = eb / 4, m = f->m, n = f->n, p = f->info.rank;
    Linalg& la = *f->owner;
    Engine& e = *la.engine;
    BufferClaim claim;
    claim.take(B, e.identity);
    claim.take(X, e.identity);
    if (B->bytes < m * nrhs * eb || X->bytes < n * nrhs * eb) throw invalid_argument("solve: buffer too small");
    if (X == B) throw invalid_argument("solve: X overlaps B");
    if (timing) *timing = {0, 0};
    if (!n || !nrhs) return LF_OK;
    auto w0 = Clock::now();
    e.activate();
    B->sync_to_device(e.stream);
    X->host_authoritative = false;
    uint32_t* dX = static_cast<uint32_t*>(X->dev);
    if (p < n && (!f->pivot || f->info.reason == 3)) {
        std::vector<uint32_t> z(n * nrhs * E, 0);
        const uint32_t st = 4u | (f->pivot ? f->info.status : 0u);
        for (size_t q = 0; q < n * nrhs; ++q) z[q * E + E - 1] = st;
        cuda_check(cudaMemcpyAsync(dX, z.data(), n * nrhs * eb, cudaMemcpyHostToDevice, e.stream), "invalid solution");
        cuda_check(cudaStreamSynchronize(e.stream), "solve");
        if (timing) *timing = {0, since(w0)};
        return LF_OK;
    }
    uint32_t* C = static_cast<uint32_t*>(la.qr[8].get(m * nrhs * eb));
    cuda_check(cudaMemcpyAsync(C, B->dev, m * nrhs * eb, cudaMemcpyDeviceToDevice, e.stream), "right-hand sides");
    const double g = qr_solve_device(la, *f, C, nrhs);
    const size_t rows = std::min(p, n);
    if (f->pivot) {
        cuda_check(cudaMemsetAsync(dX, 0, n * nrhs * eb, e.stream), "memset");
        for (size_t i = 0; i < rows; ++i)
            cuda_check(cudaMemcpyAsync(dX + f->perm[i] * nrhs * E, C + i * nrhs * E, nrhs * eb, cudaMemcpyDeviceToDevice, e.stream), "permute");
    } else {
        cuda_check(cudaMemcpyAsync(dX, C, n * nrhs * eb, cudaMemcpyDeviceToDevice, e.stream), "solution");
    }
    cuda_check(cudaStreamSynchronize(e.stream), "solve");
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}
int lf_qr_apply_q_buffer(const lf_qr* f, lf_buffer* B, size_t nrhs, int transpose, lf_timing* timing) {
    LF_API_BEGIN
    if (!f) throw logic_error("empty QR factor");
    if (f->cplx) throw invalid_argument("complex QR factors have no Buffer forms");
    check_qr_size(f->n, nrhs);
    check_qr_size(1, f->m * nrhs);
    const size_t eb = size_t(f->bits / 8 + 12), m = f->m;
    Linalg& la = *f->owner;
    Engine& e = *la.engine;
    BufferClaim claim;
    claim.take(B, e.identity);
    if (B->bytes < m * nrhs * eb) throw invalid_argument("apply_q: buffer too small");
    if (timing) *timing = {0, 0};
    if (!m || !nrhs) return LF_OK;
    auto w0 = Clock::now();
    e.activate();
    B->sync_to_device(e.stream);
    const double g = qr_apply_device(la, *f, static_cast<uint32_t*>(B->dev), nrhs, transpose != 0);
    cuda_check(cudaStreamSynchronize(e.stream), "apply_q");
    if (timing) *timing = {g, since(w0)};
    LF_API_END
}

}  // extern "C"
