/* C ABI of the B200 implementation of the LimbForge/WolfNum batched multiprecision path.
 *
 * The reference exposes a C++17 header API (namespace limbforge, include/limbforge/engine.hpp,
 * linalg.hpp, batched_linalg.hpp) and no C ABI.  This header is the language-neutral boundary
 * those classes map onto one to one; the headers include/limbforge/NAME.hpp in this repository are the
 * thin inline C++ wrappers that keep user code source compatible.  Each entry point cites the
 * reference interface it replaces (file:line, paths inside the reference project).
 *
 * Conventions
 *   - Every function returns LF_OK (0) or an error class mirroring the reference's exceptions:
 *     LF_INVALID_ARGUMENT (std::invalid_argument), LF_LOGIC_ERROR (std::logic_error),
 *     LF_RUNTIME_ERROR (std::runtime_error).  lf_last_error() returns the message of the last
 *     failure on the calling thread.  Arithmetic errors are never reported here: they are the
 *     per-element status bits (division_by_zero=1, exponent_overflow=2, invalid=4).
 *   - Elements are the reference's structs, byte for byte: a real element of `bits` (64..1024,
 *     multiple of 32) is bits/32 little-endian uint32 limbs, int32 exponent, int32 sign,
 *     uint32 status (bits/8+12 bytes); a complex element is {re, im}.
 *   - Host-array calls take host pointers, copy in and out and return after completion.
 *   - Operation codes are limbforge::Operation (engine.hpp:13).
 */
#ifndef LIMBFORGE_B200_H
#define LIMBFORGE_B200_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { LF_OK = 0, LF_INVALID_ARGUMENT = 1, LF_LOGIC_ERROR = 2, LF_RUNTIME_ERROR = 3 };
enum lf_operation {
    LF_ADD = 0, LF_SUB = 1, LF_MUL = 2, LF_DIV = 3, LF_COMPLEX_ADD = 4, LF_COMPLEX_MUL = 5, LF_COMPLEX_DIV = 6,
    LF_SQUARE = 7, LF_SQRT = 8, LF_FMA = 9, LF_FMS = 10, LF_COMPLEX_FMA = 11, LF_COMPLEX_FMS = 12
};

typedef struct lf_timing { double gpu_seconds, wall_seconds; } lf_timing;              /* engine.hpp:18 */
typedef struct lf_broadcast { size_t stride, period; } lf_broadcast;                   /* engine.hpp:21 */
typedef struct lf_engine_options {                                                      /* engine.hpp:28 */
    unsigned threads_per_threadgroup; int cooperative_reductions, cooperative_recurrence; int device;
} lf_engine_options;
typedef struct lf_batched4 { size_t count; unsigned rhs; int inverse, determinant, fused; } lf_batched4; /* engine.hpp:36 */
typedef struct lf_strided_gemm {                                                        /* batched_linalg.hpp:11-14 */
    size_t count, m, n, k, stride_a, stride_b, stride_c; int accumulate, fused, negative;
} lf_strided_gemm;

typedef struct lf_linalg_options {                                                      /* linalg.hpp:18-25 */
    int band_bits, max_bands, max_spread; unsigned host_threads; int force_fallback, resident_bands;
    int method;   /* 0 auto (residue engine where it applies), 1 generic limb kernel, 2 residue engine only */
} lf_linalg_options;
typedef struct lf_factor_options { size_t block; double host_macs, solve_host_macs; int gpu; } lf_factor_options; /* linalg.hpp:73-78 */
typedef struct lf_cholesky_info {                                                       /* linalg.hpp:82-87 */
    size_t pivot; int pivot_sign; uint32_t pivot_status; lf_timing timing;
    size_t blocks, gpu_updates, host_updates; double panel_seconds, update_seconds;
} lf_cholesky_info;
typedef struct lf_linalg_report {                                                       /* linalg.hpp:35-45 */
    size_t m, n, k, gpu_outputs, trivial_outputs, gemm_rows, gemm_cols, int8_gemms, moduli, band_bits;
    double analysis_seconds, gpu_seconds;
    int method;   /* 1 generic limb kernel, 2 residue engine */
    /* lines (rows of the left operand, columns of the right) with a nonzero status-free entry, and the others
     * (all zero, or a status entry), as the residue engine's analysis found them; 0 when the limb kernel ran */
    size_t left_lines, left_zero_lines, right_lines, right_zero_lines;
} lf_linalg_report;

typedef struct lf_engine lf_engine;
typedef struct lf_linalg lf_linalg;
typedef struct lf_buffer lf_buffer;
typedef struct lf_batch lf_batch;
typedef struct lf_submission lf_submission;

const char* lf_last_error(void);
/* library version string and the GPU architecture the kernels were built for */
const char* lf_version(void);
/* the limbforge API version the library implements (version.hpp: library_version) */
void lf_api_version(unsigned* major, unsigned* minor, unsigned* patch);

/* ---- Engine (engine.hpp:184-227) ---- */
int lf_engine_create(const lf_engine_options* options, lf_engine** out);               /* Engine::Engine */
void lf_engine_destroy(lf_engine* engine);                                              /* Engine::~Engine */
int lf_engine_device_name(lf_engine* engine, char* name, size_t capacity);              /* Engine::device_name */
/* Engine::prewarm (engine.hpp:190): validates the widths and operations and loads their element-wise kernels now */
int lf_engine_prewarm(lf_engine* engine, const int* bits, size_t nbits, const int* ops, size_t nops);
/* Engine::pipeline_info (engine.hpp:193): warp width, largest block of the kernel, block size it is launched with */
int lf_engine_pipeline_info(lf_engine* engine, int bits, int op, unsigned* simd_width, unsigned* max_threads, unsigned* threads);
/* Engine::run (engine.hpp:202): out[i] = op(a[i], b[(i/stride)%period]) for binary real/complex ops */
int lf_engine_run(lf_engine* engine, int bits, int op, const void* a, const void* b, void* out, size_t count,
                  lf_broadcast b_index, lf_timing* timing);
/* Engine::run_unary (engine.hpp:203): square, sqrt */
int lf_engine_run_unary(lf_engine* engine, int bits, int op, const void* a, void* out, size_t count, lf_timing* timing);
/* Engine::run_ternary (engine.hpp:204): fma, fms, complex_fma, complex_fms */
int lf_engine_run_ternary(lf_engine* engine, int bits, int op, const void* a, const void* b, const void* c, void* out,
                          size_t count, lf_broadcast b_index, lf_broadcast c_index, lf_timing* timing);
/* Engine::lu4 (engine.hpp:208): batched 4x4 complex LU solve / inverse / determinant */
int lf_engine_lu4(lf_engine* engine, int bits, const lf_batched4* shape, const void* A, const void* B, void* X,
                  void* det, uint32_t* status, lf_timing* timing);

/* ---- BatchedLinalg (batched_linalg.hpp:77-118) ---- */
/* BatchedLinalg::gemm host form (batched_linalg.hpp:86): sequential ascending-k products, one
 * rounding per step (composed) or per fused step; C is read (accumulate) and written */
int lf_batched_gemm(lf_engine* engine, int bits, int complex_, const lf_strided_gemm* shape, const void* A,
                    const void* B, void* C, lf_timing* timing);

/* ---- Linalg (linalg.hpp:141-218): exact products, blocked Cholesky, triangular solves ---- */
int lf_linalg_create(lf_engine* engine, const lf_linalg_options* options, lf_linalg** out); /* Linalg::Linalg (engine may be NULL) */
void lf_linalg_destroy(lf_linalg* linalg);
int lf_linalg_get_report(lf_linalg* linalg, lf_linalg_report* report);                 /* Linalg::report */
int lf_linalg_device_name(lf_linalg* linalg, char* name, size_t capacity);              /* Linalg::device_name */
/* Linalg::gemm (linalg.hpp:155): C (m x n) = op(A) B, or RN(C - op(A) B) with subtract */
int lf_linalg_gemm(lf_linalg* linalg, int bits, int transpose_a, const void* A, const void* B, size_t m, size_t n, size_t k,
                   void* C, int subtract, lf_timing* timing);
/* Linalg::syrk (linalg.hpp:152): C (cols x cols) = A^T A, lower triangle or full */
int lf_linalg_syrk(lf_linalg* linalg, int bits, const void* A, size_t rows, size_t cols, void* C, int lower_only,
                   int subtract, lf_timing* timing);
/* Linalg::cholesky (linalg.hpp:158) */
int lf_linalg_cholesky(lf_linalg* linalg, int bits, const void* A, size_t n, void* L, const lf_factor_options* options,
                       lf_cholesky_info* info);
/* Linalg::trsm (linalg.hpp:161) */
int lf_linalg_trsm(lf_linalg* linalg, int bits, int transpose, const void* L, size_t n, const void* B, size_t nrhs, void* X,
                   const lf_factor_options* options, lf_timing* timing);
/* Linalg::cholesky_solve (linalg.hpp:163) */
int lf_linalg_cholesky_solve(lf_linalg* linalg, int bits, const void* L, size_t n, const void* B, size_t nrhs, void* X,
                             const lf_factor_options* options, lf_timing* timing);
/* Buffer forms (linalg.hpp:194-199): Linalg::cholesky / trsm / cholesky_solve on idle buffers of the Linalg's engine,
 * used in place, synchronous; passes 1 = L X = B, 2 = L^T X = B, 3 = L L^T X = B.  Same results as the host-array calls. */
int lf_linalg_cholesky_buffers(lf_linalg* linalg, int bits, lf_buffer* A, size_t n, lf_buffer* L, const lf_factor_options* options,
                               lf_cholesky_info* info);
int lf_linalg_solve_buffers(lf_linalg* linalg, int bits, int passes, lf_buffer* L, size_t n, lf_buffer* B, size_t nrhs, lf_buffer* X,
                            const lf_factor_options* options, lf_timing* timing);

/* ---- Householder QR (linalg.hpp:88-137; linalg.mm:488-849).  Options: the FactorOptions fields (block is the
 * compact-WY block; host_macs, solve_host_macs and gpu only place work and never change a bit), rank_bits (> 0:
 * the factorization also stops at the first column whose |r_jj| lies more than rank_bits binades below the
 * largest earlier |r_kk|) and pivot (column pivoting, as xGEQP3).  A factor owns row-major arrays R (n x n, upper;
 * with rank p < n rows i >= p hold the remainder in columns j >= p), V (m x n, column j is v_j, zero above row j),
 * tau (n) and T (blocks of nb x nb compact-WY upper triangles, block b at b*nb*nb); it uses the Linalg that made
 * it, which must outlive it.  info.reason: 0 full rank, 1 zero column, 2 small column, 3 status column. */
typedef struct lf_qr_options { size_t block; double host_macs, solve_host_macs; int gpu; int rank_bits; int pivot; } lf_qr_options; /* linalg.hpp:94 */
typedef struct lf_qr_info {                                                               /* linalg.hpp:98-105 */
    size_t rank; int reason; uint32_t status; lf_timing timing;
    size_t blocks, gpu_updates, host_updates; double panel_seconds, update_seconds; size_t norm_recomputations;
} lf_qr_info;
typedef struct lf_qr lf_qr;                                                               /* QRFactor, linalg.hpp:112 */
/* Linalg::factor_qr (linalg.hpp:164): A (m x n, m >= n) is only read; *out owns the factor (lf_qr_destroy) */
int lf_linalg_factor_qr(lf_linalg* linalg, int bits, const void* A, size_t m, size_t n, const lf_qr_options* options, lf_qr** out);
/* Linalg::factor_qr_augmented (linalg.hpp:168): the factor of [J; diag(d)] ((m + n) x n) */
int lf_linalg_factor_qr_augmented(lf_linalg* linalg, int bits, const void* J, size_t m, size_t n, const void* d,
                                  const lf_qr_options* options, lf_qr** out);
/* Linalg::factor_qr on a Buffer (linalg.hpp:200): synchronous, the buffer idle */
int lf_linalg_factor_qr_buffer(lf_linalg* linalg, int bits, lf_buffer* A, size_t m, size_t n, const lf_qr_options* options, lf_qr** out);
void lf_qr_destroy(lf_qr* qr);
/* QRFactor::bits/rows/cols/block/pivoted/info (linalg.hpp:115-116) */
int lf_qr_describe(const lf_qr* qr, int* bits, size_t* rows, size_t* cols, size_t* block, int* pivoted, lf_qr_info* info);
/* QRFactor::r/v/tau/t/permutation (linalg.hpp:121-123): arrays owned by the factor; NULL when empty */
const void* lf_qr_r(const lf_qr* qr);
const void* lf_qr_v(const lf_qr* qr);
const void* lf_qr_tau(const lf_qr* qr);
const void* lf_qr_t(const lf_qr* qr);
const size_t* lf_qr_permutation(const lf_qr* qr);
/* QRFactor::solve (linalg.hpp:127): least-squares X (n x nrhs) from B (m x nrhs); X must not overlap B */
int lf_qr_solve(const lf_qr* qr, const void* B, size_t nrhs, void* X, lf_timing* timing);
/* QRFactor::apply_q (linalg.hpp:129): B (m x nrhs) <- Q^T B (transpose) or Q B, in place */
int lf_qr_apply_q(const lf_qr* qr, void* B, size_t nrhs, int transpose, lf_timing* timing);
/* Buffer forms of solve / apply_q (linalg.hpp:131-134): synchronous, buffers idle (real factors) */
int lf_qr_solve_buffers(const lf_qr* qr, lf_buffer* B, size_t nrhs, lf_buffer* X, lf_timing* timing);
int lf_qr_apply_q_buffer(const lf_qr* qr, lf_buffer* B, size_t nrhs, int transpose, lf_timing* timing);
/* Linalg::factor_qr_complex (linalg.hpp:170, ComplexQRFactor linalg.hpp:331-350): complex A (m x n Complex<bits/32>,
 * m >= n); the factor's r/v/tau/t are complex arrays (R with a real diagonal), lf_qr_solve and lf_qr_apply_q take
 * complex matrices (transpose selects Q^H).  Column pivoting of complex factors is not built (runtime error). */
int lf_linalg_factor_qr_complex(lf_linalg* linalg, int bits, const void* A, size_t m, size_t n, const lf_qr_options* options,
                                lf_qr** out);
int lf_qr_is_complex(const lf_qr* qr);
/* Exact product on device line views (CUDA callers; no reference counterpart): element (line, k)
 * at base + (line * ls + k * ks) elements; C element (i, j) at C + i * ldc + j elements. */
int lf_dev_exact_product(lf_linalg* linalg, int bits, const void* left, size_t left_ls, size_t left_ks, const void* right,
                         size_t right_ls, size_t right_ks, size_t M, size_t N, size_t K, void* C, size_t ldc, int subtract,
                         int lower, void* stream);

/* Allocation-free form of lf_dev_exact_product (no reference counterpart).  For callers that cannot
 * allocate device memory when they need a product (a fixed device-memory plan, threads that must not
 * take the allocator's locks, embedding runtimes that forbid allocation): all temporary device data
 * lives in a 32 MiB static device array of the library, so no cudaMalloc/cudaFree is called.  Same
 * operands and result as lf_dev_exact_product; at most 8192 lines (M + N), larger products are
 * rejected with LF_INVALID_ARGUMENT.  A product whose residue planes would not fit the array runs on
 * the generic limb kernel (same bits, slower).  Calls share the array, so calls that overlapped on the
 * GPU would race: the library serializes them process-wide with one lock held until the product is
 * done, and each call blocks until then (synchronous on `stream`).  The first call on a device, and
 * the first after that device's context was recreated (a device reset), resolves the array's address:
 * make that call before any stream capture. */
int lf_dev_exact_product_static(int bits, const void* left, size_t left_ls, size_t left_ks, const void* right,
                                size_t right_ls, size_t right_ks, size_t M, size_t N, size_t K, void* C, size_t ldc,
                                int subtract, int lower, void* stream);

/* ---- Buffers (engine.hpp:74-86, 194-198): device-resident typed storage of one engine ---- */
int lf_buffer_create(lf_engine* engine, size_t bytes, lf_buffer** out);                /* Engine::make_buffer */
void lf_buffer_release(lf_buffer* buffer);                                              /* last reference frees */
size_t lf_buffer_bytes(const lf_buffer* buffer);                                        /* Buffer::size (bytes) */
int lf_buffer_holders(const lf_buffer* buffer);   /* batches and unwaited submissions holding the buffer (workspace accounting) */
int lf_buffer_upload(lf_buffer* buffer, const void* source, size_t bytes);              /* Buffer::upload */
int lf_buffer_download(lf_buffer* buffer, void* target, size_t bytes);                  /* Buffer::download */
/* Buffer::mapped (engine.hpp:82): a host view, current as of this call; host writes through it
 * reach the device at the next submission that uses the buffer. */
int lf_buffer_mapped(lf_buffer* buffer, void** host);
/* Page-locked host memory for fast transfers to and from buffers (no reference counterpart:
 * the reference's unified memory needs none). */
int lf_host_alloc(size_t bytes, void** host);
void lf_host_free(void* host);
/* Device address of the storage (CUDA interop; no reference counterpart). */
int lf_buffer_device_pointer(lf_buffer* buffer, void** device);

/* ---- Command batches and submissions (engine.hpp:93-182) ---- */
int lf_batch_create(lf_engine* engine, lf_batch** out);                                 /* Engine::batch */
void lf_batch_destroy(lf_batch* batch);                                                 /* CommandBatch::~CommandBatch */
/* CommandBatch::run (engine.hpp:120-147): counts in elements; b/c may be NULL where unused */
int lf_batch_run(lf_batch* batch, int bits, int complex_, int op, lf_buffer* a, lf_buffer* b, lf_buffer* c,
                 lf_buffer* out, size_t count, lf_broadcast b_index, lf_broadcast c_index);
/* CommandBatch::lu4 (engine.hpp:164) */
int lf_batch_lu4(lf_batch* batch, int bits, const lf_batched4* shape, lf_buffer* A, lf_buffer* B, lf_buffer* X,
                 lf_buffer* det, lf_buffer* status);
/* BatchedLinalg::gemm resident form (batched_linalg.hpp:97): C_b (+)= A_b B_b, strides in elements */
int lf_batch_strided_gemm(lf_batch* batch, int bits, int complex_, const lf_strided_gemm* shape, lf_buffer* A,
                          lf_buffer* B, lf_buffer* C);
int lf_batch_submit(lf_batch* batch, lf_submission** out);                             /* CommandBatch::submit */
int lf_submission_ready(lf_submission* submission, int* ready);                        /* Submission::ready */
int lf_submission_wait(lf_submission* submission, lf_timing* timing);                  /* Submission::wait */
void lf_submission_destroy(lf_submission* submission);                                  /* waits, then frees */

/* ---- Device-pointer entry points (resident CUDA memory, caller's stream; no reference
 *      counterpart: they are the kernels behind the calls above, for CUDA callers) ---- */
int lf_dev_elementwise(int bits, int op, const void* a, const void* b, const void* c, void* out, size_t count,
                       lf_broadcast b_index, lf_broadcast c_index, void* stream);
/* x <- x * f_s for s = 0..steps-1, every step rounded, the running value held in registers:
 * the fused form of CommandBatch::run(mul, x, f_s, x) repeated (engine.mm:332-346).
 * factors: steps arrays of count elements at factors + s * factor_stride elements. */
int lf_dev_mul_chain(int bits, const void* x, const void* factors, size_t factor_stride, unsigned steps, void* out,
                     size_t count, void* stream);
/* The same with a choice of lanes per value (no reference counterpart): 1, one value per thread; 2, one value per
 * lane pair, each lane forming half of every product's rows and one shuffle exchange per product (even widths of
 * 384 bits and more, contiguous factors; other chains run one value per thread).  Identical bits either way. */
int lf_dev_mul_chain_lanes(int bits, int lanes, const void* x, const void* factors, size_t factor_stride, unsigned steps,
                           void* out, size_t count, void* stream);

/* ---- Resident products (linalg.hpp:60-66,190-195): Linalg::syrk / gemm recorded into a CommandBatch on
 * buffers of the Linalg's engine (row-major, sizes as the host calls).  Line analysis, the choice of engine
 * and the modulus count are GPU passes of the batch (no host round trip); after the submission is waited C
 * equals the host-array call bit for bit.  C must not be A or B. */
typedef struct lf_linalg_ticket lf_linalg_ticket;                                        /* LinalgTicket */
int lf_linalg_batch_gemm(lf_linalg* la, lf_batch* batch, int bits, int transpose_a, lf_buffer* A, lf_buffer* B, size_t m,
                         size_t n, size_t k, lf_buffer* C, int subtract, lf_linalg_ticket** out);
int lf_linalg_batch_syrk(lf_linalg* la, lf_batch* batch, int bits, lf_buffer* A, size_t rows, size_t cols, lf_buffer* C,
                         int lower_only, int subtract, lf_linalg_ticket** out);
int lf_linalg_ticket_resolved(lf_linalg_ticket* ticket, int* resolved);                 /* LinalgTicket::resolved */
int lf_linalg_ticket_report(lf_linalg_ticket* ticket, lf_linalg_report* report);         /* LinalgTicket::report */
void lf_linalg_ticket_destroy(lf_linalg_ticket* ticket);
/* Linalg::workspaces / release_workspaces (linalg.hpp:46-52, 173-180): bytes of device memory the Linalg retains:
 * scratch of the host-array calls and factorizations; resident-product workspaces idle (their batch has run)
 * or busy (unsubmitted or in flight).  release frees the scratch and the idle workspaces (tickets keep their
 * reports) and returns what was retained before it; busy workspaces are freed with their batches. */
typedef struct lf_linalg_workspaces { size_t scratch_bytes, idle_bytes, busy_bytes, busy_workspaces; } lf_linalg_workspaces;
int lf_linalg_get_workspaces(lf_linalg* linalg, lf_linalg_workspaces* out);
int lf_linalg_release_workspaces(lf_linalg* linalg, lf_linalg_workspaces* out);

/* ---- Precision casts and tree sums (engine.hpp:150-175,205; kernels.metal:60-112,251-266).
 * cast: exact widening, round-to-nearest-even narrowing, complex componentwise; a status element or a
 * zero becomes a zero with that status.  tree_sum: the fixed adjacent-pair tree (elements 2i and 2i+1
 * added, an odd last element carried unrounded, repeated to one element; empty input -> zero). */
int lf_engine_cast(lf_engine* engine, int from_bits, int to_bits, int complex_, const void* in, void* out, size_t count,
                   lf_timing* timing);                                                   /* Engine::cast */
int lf_batch_cast(lf_batch* batch, int from_bits, int to_bits, int complex_, lf_buffer* in, lf_buffer* out,
                  size_t count);                                                         /* CommandBatch::cast */
int lf_batch_tree_sum(lf_batch* batch, int bits, int complex_, lf_buffer* in, lf_buffer* out,
                      size_t count);                                                     /* CommandBatch::tree_sum */
/* Segmented dot products (engine.hpp:30-32,205; kernels.metal:195-207): out[i] is the fused chain s <- fma(a[i*length+k],
 * b[i*length+k] (or b[k] when shared_right), s) from s = 0 over k = 0..length-1, cfma for complex. */
typedef struct lf_segmented_dot { size_t segments, length; int shared_right; } lf_segmented_dot;   /* engine.hpp:32 */
int lf_engine_segmented_dot(lf_engine* engine, int bits, int complex_, const lf_segmented_dot* shape, const void* a, const void* b,
                            void* out, lf_timing* timing);                               /* Engine::segmented_dot */
int lf_batch_segmented_dot(lf_batch* batch, int bits, int complex_, const lf_segmented_dot* shape, lf_buffer* a, lf_buffer* b,
                           lf_buffer* out);                                              /* CommandBatch::segmented_dot */
/* Engine::recurrence (engine.hpp:218-223; kernels.metal:39-58): complex four-value rings, seeds[j*count+i],
 * weights[(step*4+j)*(count/states_per_weight)+i/states_per_weight]; each step q <- sum_j w_j q_j as
 * cadd(cadd(cadd(cadd(0, cmul(w_0, q_0)), ...))) and the ring shifts; out[i] is the last value (the fourth
 * seed after zero steps). */
int lf_engine_recurrence(lf_engine* engine, int bits, const void* seeds, const void* weights, void* out, size_t count,
                         unsigned steps, unsigned states_per_weight, lf_timing* timing);
/* The exact batched 4 x 4 product, wolfnum::experimental::ExactGemm4 (benchmarks/experiments/exact_gemm4/prototype.hpp:
 * 4-33): row-major 4 x 4 matrices, matrix t of A, B, C at t * stride elements (stride 0 broadcasts an input); each real
 * component RN(C_old + sum_k a_ik b_kj) with one rounding of the exact sum (C_old left out without accumulate), then
 * negated when `negative`; complex components sum eight signed real products.  Output matrices may not overlap
 * (stride_c >= 16 when count > 1), inputs may; the output may not alias an input.  Every component is summed on the
 * GPU: the report's host_components and provisional_reads are always 0. */
typedef struct lf_exact_gemm4_shape {
    size_t count, stride_a, stride_b, stride_c;
    int accumulate, negative;
} lf_exact_gemm4_shape;                                                                  /* ExactGemm4Shape */
typedef struct lf_exact_gemm4_report {
    size_t gpu_components, host_components;
    int provisional_reads;
} lf_exact_gemm4_report;                                                                 /* ExactGemm4Report */
int lf_engine_exact_gemm4(lf_engine* engine, int bits, int complex_, const lf_exact_gemm4_shape* shape, const void* A,
                          const void* B, void* C, lf_exact_gemm4_report* report,
                          lf_timing* timing);                                            /* ExactGemm4::gemm (host arrays) */
int lf_batch_exact_gemm4(lf_batch* batch, int bits, int complex_, const lf_exact_gemm4_shape* shape, lf_buffer* A,
                         lf_buffer* B, lf_buffer* C);                                    /* ExactGemm4::gemm (CommandBatch&) */
/* Import of complex values whose MPFR significands live inside one caller allocation (BatchedLinalg::
 * import_inline_complex, batched_linalg.hpp:53-60,146-148): offsets address little-endian 64-bit MPFR limbs of a
 * significand of exactly `bits` bits; the allocation owns whole aligned pages and stays unchanged until the batch has
 * been submitted.  out[i] gets both parts of record i (a status or a zero sign gives zero with that status). */
typedef struct lf_inline_complex_record {
    uint64_t real_offset, imag_offset;
    int32_t real_exponent, imag_exponent, real_sign, imag_sign;
    uint32_t real_status, imag_status;
} lf_inline_complex_record;                                                              /* InlineComplexRecord */
int lf_batch_import_inline_complex(lf_batch* batch, int bits, const void* allocation, size_t bytes,
                                   const lf_inline_complex_record* records, size_t count,
                                   lf_buffer* out);                                      /* import_inline_complex */

/* Device-pointer forms (no reference counterpart), asynchronous on `stream`; tree_sum's scratch holds
 * 2 * ceil(count / 2) elements (unused for count <= 2). */
int lf_dev_cast(int from_bits, int to_bits, int complex_, const void* in, void* out, size_t count, void* stream);
int lf_dev_tree_sum(int bits, int complex_, const void* in, size_t count, void* out, void* scratch, void* stream);

/* ---- Ragged mixed-precision batches.  No reference counterpart: the reference's
 * BatchedLinalg::gemm (batched_linalg.hpp:86; batched_linalg.mm:163-173) runs one StridedGemm per
 * call, one shape and one precision, so a ragged batch there is a loop of calls grouped by shape.
 * A plan holds a list of GEMM instances, each with its own precision and shape, and optionally one
 * batched 4x4 LU job (Engine::lu4 semantics, engine.hpp:164), all over one device arena.  Running it
 * is one CUDA graph launch: one persistent kernel per precision class (blocks take chunks of output
 * cells from a counter, heaviest instances first) and the LU kernel, on parallel graph branches.
 * Block sizes and grids come from an autotuner that times the candidates on the plan itself.
 * Instance i computes C_i (+)= A_i B_i exactly as a one-instance StridedGemm at bits_i would. */
typedef struct lf_ragged_gemm {
    int bits;                  /* 64..1024, multiple of 32 */
    uint32_t m, n, k;          /* A_i m x k, B_i k x n, C_i m x n, row-major */
    uint64_t a, b, c;          /* byte offsets in the arena, multiples of 16 */
    int accumulate, negative;  /* as lf_strided_gemm */
} lf_ragged_gemm;
typedef struct lf_ragged_lu4 {
    int bits; lf_batched4 shape;
    uint64_t A, B, X, det, status;   /* byte offsets in the arena (multiples of 16); unused ones ignored */
} lf_ragged_lu4;
typedef struct lf_ragged_class_info {
    int bits; size_t items, cells;    /* instances and output entries of this precision */
    unsigned block, grid;             /* launch shape in use */
    double trial_ms;                  /* measured time of that shape when tuned, else 0 */
} lf_ragged_class_info;
typedef struct lf_ragged_info {
    size_t classes; lf_ragged_class_info cls[31];
    unsigned lu4_block, lu4_grid; double lu4_trial_ms;
    int tuned;
} lf_ragged_info;
typedef struct lf_ragged_plan lf_ragged_plan;

/* Host only: assigns packed offsets (A, B, C of each instance in turn, then the LU job's A, B, X,
 * det, status when lu4 is given), 256-byte aligned, and returns the arena size in bytes. */
int lf_ragged_pack(int complex_, lf_ragged_gemm* items, size_t count, lf_ragged_lu4* lu4, uint64_t* arena_bytes);
/* Validates the instances against an arena of arena_bytes (extents, alignment, no output overlapping
 * another output or any input) and builds the work lists.  lu4 may be null. */
int lf_ragged_plan_create(lf_engine* engine, int complex_, int fused, const lf_ragged_gemm* items, size_t count,
                          const lf_ragged_lu4* lu4, uint64_t arena_bytes, lf_ragged_plan** out);
/* Autotuner: times every candidate block size (and, for the LU job, grid form) of every precision
 * class on this arena's data, with trial outputs written to plan-owned scratch so the arena is not
 * modified, and keeps the fastest.  Synchronous.  Until it runs, defaults are used. */
int lf_ragged_plan_tune(lf_ragged_plan* plan, const void* arena);
/* One graph launch on `stream` (null = the legacy default stream); asynchronous.  Runs of one plan
 * are ordered after each other whatever their streams.  The graph is rebuilt when the arena moves. */
int lf_ragged_plan_run(lf_ragged_plan* plan, void* arena, void* stream);
int lf_ragged_plan_get_info(const lf_ragged_plan* plan, lf_ragged_info* info);
void lf_ragged_plan_destroy(lf_ragged_plan* plan);

/* ---- Failure-detection test hook (no reference counterpart): one tile of the residue products whose loads are
 * left out, so the first barrier wait of the tensor-core kernel runs out after `polls` polls; the kernel records
 * error 2, frees its tensor memory and returns, and *error_word receives the kernel's error word. */
int lf_test_residue_wait_limit(unsigned polls, uint32_t* error_word);

/* ---- Measurement helper (no reference counterpart): the device's rate of 32 x 32 -> 64-bit integer
 * multiply-adds, the word product of every limb kernel, measured by a kernel of independent
 * multiply-add chains on every SM (CUDA events).  The denominator of the integer-pipe roofline. */
int lf_probe_word_mac_rate(int device, double* word_macs_per_s);

#ifdef __cplusplus
}
#endif
#endif
