// Host driver of the int8-residue / CRT exact product engine (kernels in lf_residue.cuh).
//
// Domain: every nonzero, status-free line of each side fits one exponent band of width
// G <= kMaxBand bits (G = the widest such line's exponent spread) and K <= kMaxK.  Outside it the
// caller runs the generic limb kernel, which gives the same bits.
//
// Moduli: primes <= 65279, descending (as the reference, linalg.mm:39-40: a balanced residue
// |r| <= 32639 then splits into two int8 digits); L is the smallest count whose product exceeds
// 2^(2(32N+G) + ceil(log2 K) + 3) > 4 K max|entry|^2, so the signed CRT value and the rounding of
// the fixed-point quotient are both unambiguous.
#include "lf_residue.h"
#define LF_RESIDUE_MMA_KERNEL
#include "lf_residue.cuh"

#include <cuda.h>
#include <algorithm>
#include <cmath>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace lfr {

namespace {
constexpr int kMaxBand = 192;
constexpr uint64_t kMaxK = 65472;

const std::vector<uint32_t>& primes() {
    static const std::vector<uint32_t> p = [] {
        std::vector<uint32_t> r;
        for (uint32_t q = 65279; r.size() < (size_t)lfd::kResMaxModuli; --q) {
            bool prime = q > 1;
            for (uint32_t d = 2; d * d <= q && prime; ++d) prime = q % d != 0;
            if (prime) r.push_back(q);
        }
        return r;
    }();
    return p;
}
uint32_t inverse_mod(uint64_t a, uint64_t m) {                // extended Euclid
    int64_t t = 0, nt = 1, r = (int64_t)m, nr = (int64_t)(a % m);
    while (nr) { int64_t q = r / nr, x = t - q * nt; t = nt; nt = x; x = r - q * nr; r = nr; nr = x; }
    return (uint32_t)(t < 0 ? t + (int64_t)m : t);
}
// Multiword helpers for the host-side tables.
void mul_small(std::vector<uint32_t>& x, uint32_t m) {
    uint64_t c = 0;
    for (auto& w : x) { uint64_t t = (uint64_t)w * m + c; w = (uint32_t)t; c = t >> 32; }
    if (c) x.push_back((uint32_t)c);
}
uint32_t mod_small(const std::vector<uint32_t>& x, uint32_t m) {
    uint64_t r = 0;
    for (size_t i = x.size(); i-- > 0;) r = ((r << 32) | x[i]) % m;
    return (uint32_t)r;
}

// Device tables of one modulus count: the ResTables and the byte matrix B of the tensor-core CRT
// (NB rows of byte columns: S bytes 0..NS-1, then 6 bytes of F; Kp = 2L bytes rounded up to 32),
// stored as the 128-byte-swizzled shared-memory image of each 128-byte K block.
struct TableSet {
    lfd::ResTables* dev = nullptr; int L = 0, qwords = 0;
    unsigned char* bimg = nullptr; int NB = 0, Kp = 0, NS = 0; unsigned tmem_cols = 0;
};
std::mutex g_table_mutex;
std::map<std::pair<int, int>, TableSet> g_tables;            // (device, L)

TableSet tables_for(int device, int L) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    auto key = std::make_pair(device, L);
    auto it = g_tables.find(key);
    if (it != g_tables.end()) return it->second;
    auto* h = new lfd::ResTables();
    const auto& m = primes();
    std::vector<uint32_t> M{1};
    for (int l = 0; l < L; ++l) mul_small(M, m[l]);
    int qwords = 0;
    for (int l = 0; l < L; ++l) {
        h->m[l] = m[l];
        h->barrett[l] = ~0ull / m[l] + ((~0ull % m[l]) + 1 == m[l] ? 1 : 0);   // floor(2^64 / m)
        h->frac[l] = (1ull << 48) / m[l];
        std::vector<uint32_t> q{1};
        for (int t = 0; t < L; ++t) if (t != l) mul_small(q, m[t]);
        if ((int)q.size() > lfd::kResMaxQWords) throw runtime_error("residue engine: modulus table too large");
        qwords = std::max(qwords, (int)q.size());
        for (size_t w = 0; w < q.size(); ++w) h->q[l][w] = q[w];
        h->w[l] = inverse_mod(mod_small(q, m[l]), m[l]);
        uint64_t pw = 1;
        for (int w = 0; w < 40; ++w) { h->pw[l][w] = (uint32_t)pw; pw = (pw << 32) % m[l]; }
    }
    if ((int)M.size() > lfd::kResMaxQWords + 1) throw runtime_error("residue engine: modulus product too large");
    for (size_t w = 0; w < M.size(); ++w) h->M[w] = M[w];
    TableSet t;
    t.L = L; t.qwords = std::max(qwords, (int)M.size() - 1);
    cuda_check(cudaMalloc(&t.dev, sizeof(lfd::ResTables)), "residue tables");
    // cudaMemcpy from pageable memory may return before its DMA lands, and the kernels that read the
    // tables run on non-blocking streams: wait for the copy before the table is handed out.
    cuda_check(cudaMemcpy(t.dev, h, sizeof(lfd::ResTables), cudaMemcpyHostToDevice), "residue tables");
    cuda_check(cudaStreamSynchronize(0), "residue tables");
    // tensor-core CRT operand: row b < NS: byte b - h of M/m_l in column 2l + h; row NS + b: byte b - h of
    // floor(2^48/m_l)
    t.NS = 4 * t.qwords + 1;
    t.NB = (t.NS + 6 + 15) / 16 * 16;
    t.Kp = (2 * L + 31) / 32 * 32;
    t.tmem_cols = 32;
    while ((int)t.tmem_cols < t.NB) t.tmem_cols *= 2;
    const int kblocks = (t.Kp + 127) / 128;
    std::vector<unsigned char> img((size_t)kblocks * t.NB * 128, 0);
    auto qbyte = [&](int l, int b) -> unsigned { return b < 0 || b >= 4 * lfd::kResMaxQWords ? 0u : (h->q[l][b / 4] >> (8 * (b % 4))) & 255u; };
    auto fbyte = [&](int l, int b) -> unsigned { return b < 0 || b >= 8 ? 0u : (unsigned)((h->frac[l] >> (8 * b)) & 255u); };
    for (int n = 0; n < t.NB; ++n)
        for (int k = 0; k < 2 * L; ++k) {
            const int l = k / 2, hb = k % 2;
            const unsigned v = n < t.NS ? qbyte(l, n - hb) : n < t.NS + 6 ? fbyte(l, n - t.NS - hb) : 0u;
            img[(size_t)(k / 128) * t.NB * 128 + lfd::sw128_offset((uint32_t)n, (uint32_t)(k % 128))] = (unsigned char)v;
        }
    cuda_check(cudaMalloc(&t.bimg, img.size()), "residue CRT operand");
    cuda_check(cudaMemcpy(t.bimg, img.data(), img.size(), cudaMemcpyHostToDevice), "residue CRT operand");
    cuda_check(cudaStreamSynchronize(0), "residue CRT operand");
    delete h;
    g_tables[key] = t;
    return t;
}

// Digit-plane operand of one (L, xwords): B[2l + h][b] = byte h of 2^(8b) mod m_l, as the swizzled image.
struct DigitTable { unsigned char* bimg = nullptr; int NB = 0, KB = 0; unsigned tmem_cols = 0; };
std::map<std::tuple<int, int, int>, DigitTable> g_digit_tables;     // (device, L, xwords)
DigitTable digit_table_for(int device, int L, int xwords) {
    std::lock_guard<std::mutex> lock(g_table_mutex);
    const auto key = std::make_tuple(device, L, xwords);
    auto it = g_digit_tables.find(key);
    if (it != g_digit_tables.end()) return it->second;
    DigitTable t;
    t.NB = (2 * L + 15) / 16 * 16;
    t.KB = (4 * xwords + 31) / 32 * 32;
    t.tmem_cols = 32;
    while ((int)t.tmem_cols < t.NB) t.tmem_cols *= 2;
    const int kblocks = (t.KB + 127) / 128;
    std::vector<unsigned char> img((size_t)kblocks * t.NB * 128, 0);
    const auto& m = primes();
    for (int l = 0; l < L; ++l) {
        uint64_t pw = 1 % m[l];
        for (int b = 0; b < 4 * xwords; ++b) {
            for (int h = 0; h < 2; ++h)
                img[(size_t)(b / 128) * t.NB * 128 + lfd::sw128_offset((uint32_t)(2 * l + h), (uint32_t)(b % 128))] = (unsigned char)(pw >> (8 * h));
            pw = (pw << 8) % m[l];
        }
    }
    cuda_check(cudaMalloc(&t.bimg, img.size()), "digit operand");
    cuda_check(cudaMemcpy(t.bimg, img.data(), img.size(), cudaMemcpyHostToDevice), "digit operand");
    cuda_check(cudaStreamSynchronize(0), "digit operand");
    g_digit_tables[key] = t;
    return t;
}
// Persistent launch shape of the tcgen05 kernels that hold `tmem_cols` TMEM columns per CTA: as many
// CTAs per SM as TMEM allows (512 columns), shared memory sized so that no more are resident.
void tmem_launch_shape(unsigned tmem_cols, size_t smem_need, int sms, uint64_t tiles, unsigned& grid, size_t& smem) {
    const int per_sm = (int)(512 / tmem_cols);
    smem = std::max(smem_need, (size_t)(228 * 1024) / (per_sm + 1) + 1024);
    if (smem > 227 * 1024) throw runtime_error("residue engine: operand tiles exceed shared memory");
    grid = (unsigned)std::min<uint64_t>(tiles, (uint64_t)sms * per_sm);
}

typedef CUresult (*EncodeTiled)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*, const cuuint64_t*,
                                const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                                CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiled encoder() {
    static EncodeTiled fn = [] {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return reinterpret_cast<EncodeTiled>(f);
    }();
    if (!fn) throw runtime_error("cuTensorMapEncodeTiled unavailable");
    return fn;
}
// [L][rows_pad][Kp] int8 planes, 128 x 128 boxes with the 128-byte swizzle.
CUtensorMap plane_map(void* base, uint64_t Kp, uint64_t rows_pad, int L) {
    CUtensorMap map;
    const cuuint64_t dims[3] = {Kp, rows_pad, (cuuint64_t)L};
    const cuuint64_t strides[2] = {Kp, rows_pad * Kp};
    const cuuint32_t box[3] = {lfd::kTileK, lfd::kTileM, 1};
    const cuuint32_t estr[3] = {1, 1, 1};
    CUresult r = encoder()(&map, CU_TENSOR_MAP_DATA_TYPE_UINT8, 3, base, dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
                           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) throw runtime_error("cuTensorMapEncodeTiled failed");
    return map;
}
}  // namespace

bool ResidueEngine::run(int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc, uint64_t K, uint32_t* C,
                        uint64_t ldc, bool subtract, bool lower, uint32_t* error, cudaStream_t s, bool forced,
                        lf_linalg_report& report) {
    const int n = bits / 32;
    auto refuse = [&](const char* why) -> bool {
        if (forced) throw runtime_error(std::string("residue engine: ") + why);
        return false;
    };
    if (!K) return refuse("empty inner dimension");
    if (K > kMaxK) return refuse("inner dimension above 65472");
    const bool same = left.base == right.base && left.ls == right.ls && left.ks == right.ks && M == Nc;
    const auto* lk = lfd::linalg_kernels(n);
    const auto* rk = lfd::residue_kernels(n);
    auto* linfo = static_cast<lfd::LineInfo*>(lines.get(sizeof(lfd::LineInfo) * (M + Nc) + 64));
    auto* rinfo = same ? linfo : linfo + M;
    lk->analyze(left, M, K, linfo, s);
    if (!same) lk->analyze(right, Nc, K, rinfo, s);
    std::vector<lfd::LineInfo> h(M + (same ? 0 : Nc));
    cuda_check(cudaMemcpyAsync(h.data(), linfo, sizeof(lfd::LineInfo) * h.size(), cudaMemcpyDeviceToHost, s), "line info");
    cuda_check(cudaStreamSynchronize(s), "line analysis");
    int G = 0;
    bool any = false;
    report.left_lines = report.left_zero_lines = report.right_lines = report.right_zero_lines = 0;
    for (size_t i = 0; i < h.size(); ++i) {
        const auto& li = h[i];
        const bool live = !li.status && li.nonzero;
        if (live) { G = std::max(G, li.top - li.bottom); any = true; }
        if (i < M) (live ? report.left_lines : report.left_zero_lines) += 1;
        if (i >= M || same) (live ? report.right_lines : report.right_zero_lines) += 1;
    }
    if (!any) return refuse("no nonzero lines");
    if (G > kMaxBand) return refuse("a line spans more than 192 exponent bits");
    const int P = 32 * n + G;
    int logk = 0;
    while ((1ull << logk) < K) ++logk;
    const double need = 2.0 * P + logk + 3;
    double have = 0;
    int L = 0;
    while (have <= need) {
        if (L >= lfd::kResMaxModuli) return refuse("modulus count above the table limit");
        have += std::log2((double)primes()[L++]);
    }
    int dev = 0;
    cudaGetDevice(&dev);
    TableSet tab = tables_for(dev, L);
    const uint64_t Kp = (K + lfd::kTileK - 1) / lfd::kTileK * lfd::kTileK;
    const uint64_t Mp = (M + lfd::kTileM - 1) / lfd::kTileM * lfd::kTileM, Np = (Nc + lfd::kTileN - 1) / lfd::kTileN * lfd::kTileN;
    const uint64_t aplane = (uint64_t)L * Mp * Kp, bplane = same ? 0 : (uint64_t)L * Np * Kp;
    auto* pl = static_cast<signed char*>(planes.get(2 * (aplane + bplane) + 256));
    signed char *a1 = pl, *a0 = pl + aplane, *b1 = same ? a1 : pl + 2 * aplane, *b0 = same ? a0 : pl + 2 * aplane + bplane;
    auto* res = static_cast<uint16_t*>(residues.get(sizeof(uint16_t) * (uint64_t)L * M * Nc + 64));
    const int xwords = n + (G + 31) / 32 + 1;
    int sms = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev), "SM count");
    {
        const DigitTable dt = digit_table_for(dev, L, xwords);
        const int kblocks = (dt.KB + 127) / 128;
        auto planes_of = [&](lfd::LineView v, uint64_t lines, uint64_t rows_pad, const lfd::LineInfo* info, signed char* d1, signed char* d0) {
            unsigned grid = 0; size_t smem = 0;
            tmem_launch_shape(dt.tmem_cols, 1024 + (size_t)kblocks * 16384 + (size_t)kblocks * dt.NB * 128, sms, rows_pad * Kp / 128, grid, smem);
            rk->digits_mma(lfd::DigitMmaParams{v, lines, K, Kp, rows_pad, L, xwords, info, tab.dev, dt.bimg, dt.NB, dt.KB, dt.tmem_cols,
                                               d1, d0, error}, grid, smem, s);
        };
        planes_of(left, M, Mp, linfo, a1, a0);
        if (!same) planes_of(right, Nc, Np, rinfo, b1, b0);
        cuda_check(cudaGetLastError(), "digit planes");
    }
    const CUtensorMap ta1 = plane_map(a1, Kp, Mp, L), ta0 = plane_map(a0, Kp, Mp, L);
    const CUtensorMap tb1 = plane_map(b1, Kp, same ? Mp : Np, L), tb0 = plane_map(b0, Kp, same ? Mp : Np, L);
    const size_t smem = lfd::kStages * lfd::kStageBytes + 1024;
    cuda_check(cudaFuncSetAttribute(lfd::residue_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem");
    lfd::MmaParams mp{res, tab.dev, M, Nc, Kp, lower ? 1 : 0, error};
    dim3 grid((unsigned)(Np / lfd::kTileN), (unsigned)(Mp / lfd::kTileM), (unsigned)L);
    lfd::residue_mma_kernel<<<grid, lfd::kMmaThreads, smem, s>>>(ta1, ta0, tb1, tb0, mp);
    cuda_check(cudaGetLastError(), "residue products");
    {
        // persistent CRT: as many CTAs per SM as TMEM holds (512 columns per SM), shared memory sized
        // so that no more than that are resident
        const int kblocks = (tab.Kp + 127) / 128;
        unsigned grid = 0; size_t smem = 0;
        tmem_launch_shape(tab.tmem_cols, 1024 + (size_t)kblocks * 16384 + (size_t)kblocks * tab.NB * 128, sms, (M * Nc + 127) / 128,
                          grid, smem);
        auto* sf = static_cast<uint32_t*>(misc.get(sizeof(uint32_t) * (uint64_t)(tab.qwords + 4) * M * Nc + 64));
        lfd::CrtParams cp{res, tab.dev, tab.bimg, L, tab.qwords, tab.NB, tab.Kp, tab.NS, tab.tmem_cols, linfo, rinfo, C, ldc, M, Nc,
                          subtract ? 1 : 0, lower ? 1 : 0, error, nullptr, sf};
        rk->crt(cp, grid, smem, s);
        cuda_check(cudaGetLastError(), "reconstruction");
    }
    report.moduli = (size_t)L;
    report.band_bits = (size_t)G;
    report.int8_gemms = 4 * (size_t)L;
    report.gemm_rows = M;
    report.gemm_cols = Nc;
    return true;
}

}  // namespace lfr

// ---------------------------------------------------------------- pieces for the allocation-free entry point
// (lf_noalloc.cu): the same kernels and tables, with every device buffer supplied by the caller.
namespace lfr {

int residue_moduli_for(int bits, int G, uint64_t K) {
    const int P = 32 * (bits / 32) + G;
    int logk = 0;
    while ((1ull << logk) < K) ++logk;
    const double need = 2.0 * P + logk + 3;
    double have = 0;
    int L = 0;
    while (have <= need) {
        if (L >= lfd::kResMaxModuli) return 0;
        have += std::log2((double)primes()[L++]);
    }
    return L;
}
int residue_max_band() { return kMaxBand; }
uint64_t residue_max_k() { return kMaxK; }

void residue_tables_host(int L, lfd::ResTables& h, int& qwords_out) {
    const auto& m = primes();
    std::vector<uint32_t> M{1};
    for (int l = 0; l < L; ++l) mul_small(M, m[l]);
    int qwords = 0;
    for (int l = 0; l < L; ++l) {
        h.m[l] = m[l];
        h.barrett[l] = ~0ull / m[l] + ((~0ull % m[l]) + 1 == m[l] ? 1 : 0);
        h.frac[l] = (1ull << 48) / m[l];
        std::vector<uint32_t> q{1};
        for (int t = 0; t < L; ++t) if (t != l) mul_small(q, m[t]);
        qwords = std::max(qwords, (int)q.size());
        for (size_t w = 0; w < q.size(); ++w) h.q[l][w] = q[w];
        h.w[l] = inverse_mod(mod_small(q, m[l]), m[l]);
        uint64_t pw = 1;
        for (int w = 0; w < 40; ++w) { h.pw[l][w] = (uint32_t)pw; pw = (pw << 32) % m[l]; }
    }
    for (size_t w = 0; w < M.size(); ++w) h.M[w] = M[w];
    qwords_out = std::max(qwords, (int)M.size() - 1);
}

CUtensorMap residue_plane_map(void* base, uint64_t Kp, uint64_t rows_pad, int L) { return plane_map(base, Kp, rows_pad, L); }

void residue_mma_launch(dim3 grid, const CUtensorMap& ta1, const CUtensorMap& ta0, const CUtensorMap& tb1, const CUtensorMap& tb0,
                        const lfd::MmaParams& p, cudaStream_t s) {
    const size_t smem = lfd::kStages * lfd::kStageBytes + 1024;
    cuda_check(cudaFuncSetAttribute(lfd::residue_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem");
    lfd::residue_mma_kernel<<<grid, lfd::kMmaThreads, smem, s>>>(ta1, ta0, tb1, tb0, p);
    cuda_check(cudaGetLastError(), "residue products");
}

}  // namespace lfr

// ---------------------------------------------------------------- resident products planned on the GPU
namespace lfr {

struct ResidentProduct {
    int bits = 0, n = 0;
    lfd::LineView left{}, right{};
    uint64_t M = 0, Nc = 0, K = 0, ldc = 0;
    uint32_t* C = nullptr;
    bool subtract = false, lower = false, mirror = false, same = false, residue = false;
    int device = 0, sms = 0, Lmin = 0, Lmax = 0, xwords = 0;
    DevBuf lines, planes, res, plan, cands, cum, error, sf;
    uint64_t Kp = 0, Mp = 0, Np = 0;
    int maxNB = 0, maxKp = 0, maxDNB = 0, KB = 0; unsigned maxTmem = 0, maxDTmem = 0;
    CUtensorMap ta1{}, ta0{}, tb1{}, tb0{};
    cudaEvent_t done = nullptr;
    bool launched = false;
    bool in_batch = false;              // recorded in a batch that still exists
    bool kept = false;                  // plan and error word copied to the host
    lfd::ResPlan kept_plan{};
    uint32_t kept_error = 0;
    ~ResidentProduct() { if (done) cudaEventDestroy(done); }
};

static int moduli_for_band(int n, int G, uint64_t K) {
    int logk = 0;
    while ((1ull << logk) < K) ++logk;
    const double need = 2.0 * (32 * n + G) + logk + 3;
    double have = 0;
    int L = 0;
    while (have <= need) {
        if (L >= lfd::kResMaxModuli) return 0;
        have += std::log2((double)primes()[L++]);
    }
    return L;
}

std::shared_ptr<ResidentProduct> resident_product_create(int bits, lfd::LineView left, lfd::LineView right, uint64_t M, uint64_t Nc,
                                                         uint64_t K, uint32_t* C, uint64_t ldc, bool subtract, bool lower,
                                                         bool mirror, bool limb_only) {
    auto r = std::make_shared<ResidentProduct>();
    r->bits = bits; r->n = bits / 32; r->left = left; r->right = right; r->M = M; r->Nc = Nc; r->K = K; r->C = C; r->ldc = ldc;
    r->subtract = subtract; r->lower = lower; r->mirror = mirror;
    r->same = left.base == right.base && left.ls == right.ls && left.ks == right.ks && M == Nc;
    cuda_check(cudaGetDevice(&r->device), "cudaGetDevice");
    cuda_check(cudaDeviceGetAttribute(&r->sms, cudaDevAttrMultiProcessorCount, r->device), "SM count");
    cuda_check(cudaEventCreateWithFlags(&r->done, cudaEventDisableTiming), "event");
    r->error.get(16);
    r->plan.get(sizeof(lfd::ResPlan));
    r->lines.get(sizeof(lfd::LineInfo) * (M + Nc) + 64);
    r->Lmin = moduli_for_band(r->n, 0, K);
    r->Lmax = moduli_for_band(r->n, kMaxBand, K);
    r->residue = !limb_only && K && K <= kMaxK && r->Lmin && r->Lmax;
    if (!r->residue) return r;
    // candidates: every modulus count a band of 0..kMaxBand bits can need, with their tables
    r->xwords = r->n + (kMaxBand + 31) / 32 + 1;
    const int count = r->Lmax - r->Lmin + 1;
    std::vector<lfd::ResPlan> cand(count);
    std::vector<double> cum(count);
    for (int i = 0; i < count; ++i) {
        const int L = r->Lmin + i;
        const TableSet t = tables_for(r->device, L);
        const DigitTable d = digit_table_for(r->device, L, r->xwords);
        lfd::ResPlan& c = cand[i];
        c.mode = 1; c.L = L; c.qwords = t.qwords; c.NB = t.NB; c.Kp = t.Kp; c.NS = t.NS; c.tmem_cols = t.tmem_cols;
        c.dNB = d.NB; c.dtmem = d.tmem_cols; c.tab = t.dev; c.crt_bimg = t.bimg; c.dig_bimg = d.bimg;
        double have = 0;
        for (int l = 0; l < L; ++l) have += std::log2((double)primes()[l]);
        cum[i] = have;
        r->maxNB = std::max(r->maxNB, t.NB); r->maxKp = std::max(r->maxKp, t.Kp); r->maxTmem = std::max(r->maxTmem, t.tmem_cols);
        r->maxDNB = std::max(r->maxDNB, d.NB); r->maxDTmem = std::max(r->maxDTmem, d.tmem_cols); r->KB = d.KB;
    }
    cuda_check(cudaMemcpy(r->cands.get(sizeof(lfd::ResPlan) * count), cand.data(), sizeof(lfd::ResPlan) * count, cudaMemcpyHostToDevice), "plan candidates");
    cuda_check(cudaMemcpy(r->cum.get(sizeof(double) * count), cum.data(), sizeof(double) * count, cudaMemcpyHostToDevice), "plan candidates");
    cuda_check(cudaStreamSynchronize(0), "plan candidates");
    r->Kp = (K + lfd::kTileK - 1) / lfd::kTileK * lfd::kTileK;
    r->Mp = (M + lfd::kTileM - 1) / lfd::kTileM * lfd::kTileM;
    r->Np = (Nc + lfd::kTileN - 1) / lfd::kTileN * lfd::kTileN;
    const uint64_t aplane = (uint64_t)r->Lmax * r->Mp * r->Kp, bplane = r->same ? 0 : (uint64_t)r->Lmax * r->Np * r->Kp;
    auto* pl = static_cast<signed char*>(r->planes.get(2 * (aplane + bplane) + 256));
    signed char *a1 = pl, *a0 = pl + aplane, *b1 = r->same ? a1 : pl + 2 * aplane, *b0 = r->same ? a0 : pl + 2 * aplane + bplane;
    r->res.get(sizeof(uint16_t) * (uint64_t)r->Lmax * M * Nc + 64);
    int maxq = 0;
    for (const auto& c : cand) maxq = std::max(maxq, c.qwords);
    r->sf.get(sizeof(uint32_t) * (uint64_t)(maxq + 4) * M * Nc + 64);
    r->ta1 = plane_map(a1, r->Kp, r->Mp, r->Lmax); r->ta0 = plane_map(a0, r->Kp, r->Mp, r->Lmax);
    r->tb1 = plane_map(b1, r->Kp, r->same ? r->Mp : r->Np, r->Lmax); r->tb0 = plane_map(b0, r->Kp, r->same ? r->Mp : r->Np, r->Lmax);
    return r;
}

void resident_product_launch(ResidentProduct& r, cudaStream_t s) {
    if (!r.error.p) throw std::logic_error("resident product: its workspace was released");
    uint32_t* err = static_cast<uint32_t*>(r.error.p);
    cuda_check(cudaMemsetAsync(err, 0, 4, s), "memset");
    const auto* lk = lfd::linalg_kernels(r.n);
    const lfd::ResPlan* plan = nullptr;
    auto* linfo = static_cast<lfd::LineInfo*>(r.lines.p);
    auto* rinfo = r.same ? linfo : linfo + r.M;
    if (r.residue) {
        const auto* rk = lfd::residue_kernels(r.n);
        lk->analyze(r.left, r.M, r.K, linfo, s);
        if (!r.same) lk->analyze(r.right, r.Nc, r.K, rinfo, s);
        auto* pdev = static_cast<lfd::ResPlan*>(r.plan.p);
        lfd::PlanParams pp{linfo, rinfo, r.M, r.Nc, r.K, r.n, static_cast<const lfd::ResPlan*>(r.cands.p),
                           static_cast<const double*>(r.cum.p), r.Lmin, r.Lmax - r.Lmin + 1, kMaxBand, kMaxK, pdev};
        lfd::plan_kernel<<<1, 256, 0, s>>>(pp);
        cuda_check(cudaGetLastError(), "product plan");
        plan = pdev;
        const uint64_t aplane = (uint64_t)r.Lmax * r.Mp * r.Kp, bplane = r.same ? 0 : (uint64_t)r.Lmax * r.Np * r.Kp;
        auto* pl = static_cast<signed char*>(r.planes.p);
        signed char *a1 = pl, *a0 = pl + aplane, *b1 = r.same ? a1 : pl + 2 * aplane, *b0 = r.same ? a0 : pl + 2 * aplane + bplane;
        auto* res = static_cast<uint16_t*>(r.res.p);
        const int kblocks = (r.KB + 127) / 128;
        auto planes_of = [&](lfd::LineView v, uint64_t lines, uint64_t rows_pad, const lfd::LineInfo* info, signed char* d1, signed char* d0) {
            unsigned grid = 0; size_t smem = 0;
            tmem_launch_shape(r.maxDTmem, 1024 + (size_t)kblocks * 16384 + (size_t)kblocks * r.maxDNB * 128, r.sms, rows_pad * r.Kp / 128,
                              grid, smem);
            lfd::DigitMmaParams dp{v, lines, r.K, r.Kp, rows_pad, 0, r.xwords, info, nullptr, nullptr, 0, r.KB, 0, d1, d0, err, plan};
            rk->digits_mma(dp, grid, smem, s);
        };
        planes_of(r.left, r.M, r.Mp, linfo, a1, a0);
        if (!r.same) planes_of(r.right, r.Nc, r.Np, rinfo, b1, b0);
        cuda_check(cudaGetLastError(), "digit planes");
        const size_t smem = lfd::kStages * lfd::kStageBytes + 1024;
        cuda_check(cudaFuncSetAttribute(lfd::residue_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem");
        lfd::MmaParams mp{res, nullptr, r.M, r.Nc, r.Kp, r.lower ? 1 : 0, err, plan};
        dim3 grid((unsigned)(r.Np / lfd::kTileN), (unsigned)(r.Mp / lfd::kTileM), (unsigned)r.Lmax);
        lfd::residue_mma_kernel<<<grid, lfd::kMmaThreads, smem, s>>>(r.ta1, r.ta0, r.tb1, r.tb0, mp);
        cuda_check(cudaGetLastError(), "residue products");
        const int ckb = (r.maxKp + 127) / 128;
        unsigned cgrid = 0; size_t csmem = 0;
        tmem_launch_shape(r.maxTmem, 1024 + (size_t)ckb * 16384 + (size_t)ckb * r.maxNB * 128, r.sms, (r.M * r.Nc + 127) / 128, cgrid, csmem);
        lfd::CrtParams cp{res, nullptr, nullptr, 0, 0, 0, 0, 0, 0, linfo, rinfo, r.C, r.ldc, r.M, r.Nc, r.subtract ? 1 : 0, r.lower ? 1 : 0, err, plan,
                          static_cast<uint32_t*>(r.sf.p)};
        rk->crt(cp, cgrid, csmem, s);
        cuda_check(cudaGetLastError(), "reconstruction");
    }
    // the limb kernel: the whole product when the plan chose it (or there is no residue set-up), else nothing
    lfd::DotParams dp{};
    dp.left = r.left; dp.right = r.right; dp.C = r.C; dp.ldc = r.ldc; dp.M = r.M; dp.Nc = r.Nc; dp.K = r.K;
    dp.subtract = r.subtract; dp.lower = r.lower; dp.error = err; dp.plan = plan;
    lk->dot(dp, s);
    cuda_check(cudaGetLastError(), "exact product launch");
    if (r.mirror) lk->mirror(r.C, r.M, r.ldc, s);
    cuda_check(cudaEventRecord(r.done, s), "event");
    r.launched = true;
}

bool resident_product_done(ResidentProduct& r) {
    if (!r.launched) return false;
    const cudaError_t e = cudaEventQuery(r.done);
    if (e == cudaErrorNotReady) return false;
    cuda_check(e, "resident product");
    return true;
}

static void keep_outcome(ResidentProduct& r) {
    if (r.kept) return;
    cuda_check(cudaEventSynchronize(r.done), "resident product");
    if (r.residue) cuda_check(cudaMemcpy(&r.kept_plan, r.plan.p, sizeof r.kept_plan, cudaMemcpyDeviceToHost), "plan");
    cuda_check(cudaMemcpy(&r.kept_error, r.error.p, 4, cudaMemcpyDeviceToHost), "error word");
    r.kept = true;
}

size_t resident_product_bytes(const ResidentProduct& r) {
    return r.lines.bytes + r.planes.bytes + r.res.bytes + r.plan.bytes + r.cands.bytes + r.cum.bytes + r.error.bytes + r.sf.bytes;
}

void resident_product_hold(ResidentProduct& r, bool held) { r.in_batch = held; }

bool resident_product_busy(ResidentProduct& r) { return r.launched ? !resident_product_done(r) : r.in_batch; }

size_t resident_product_release(ResidentProduct& r) {
    if (resident_product_busy(r)) return 0;
    if (r.launched) keep_outcome(r);
    const size_t b = resident_product_bytes(r);
    r.lines = DevBuf{}; r.planes = DevBuf{}; r.res = DevBuf{}; r.plan = DevBuf{}; r.cands = DevBuf{}; r.cum = DevBuf{};
    r.error = DevBuf{}; r.sf = DevBuf{};
    return b;
}

bool resident_product_report(ResidentProduct& r, lf_linalg_report& rep) {
    keep_outcome(r);
    const lfd::ResPlan p = r.kept_plan;
    const uint32_t e = r.kept_error;
    rep = lf_linalg_report{};
    rep.m = r.M; rep.n = r.Nc; rep.k = r.K;
    rep.method = p.mode == 1 ? 2 : 1;
    if (p.mode == 1) {
        rep.moduli = (size_t)p.L; rep.band_bits = (size_t)p.G; rep.int8_gemms = 4 * (size_t)p.L;
        rep.gemm_rows = r.M; rep.gemm_cols = r.Nc;
    }
    rep.gpu_outputs = r.lower ? r.M * (r.M + 1) / 2 : r.M * r.Nc;
    return e == 0;
}

}  // namespace lfr

// ---------------------------------------------------------------- failure detection test hook
// One 128 x 128 tile of the residue products with the producer's loads left out, so the MMA issuer's first
// barrier wait never completes and gives up after `polls` polls: the kernel records error 2, frees its TMEM and
// returns, and the context stays usable.  The value of the error word comes back in *error_word.
extern "C" int lf_test_residue_wait_limit(unsigned polls, uint32_t* error_word) {
    using namespace lfr;
    LF_API_BEGIN
    if (!error_word || !polls) throw invalid_argument("polls must be positive and error_word not null");
    int dev = 0;
    cuda_check(cudaGetDevice(&dev), "cudaGetDevice");
    const TableSet tab = tables_for(dev, 1);
    DevBuf planes, res, err;
    const uint64_t Kp = lfd::kTileK, Mp = lfd::kTileM;
    auto* pl = static_cast<signed char*>(planes.get(4 * Mp * Kp + 256));
    cuda_check(cudaMemset(pl, 0, 4 * Mp * Kp + 256), "planes");
    auto* r16 = static_cast<uint16_t*>(res.get(64));
    auto* e = static_cast<uint32_t*>(err.get(16));
    cuda_check(cudaMemset(e, 0, 16), "error word");
    const CUtensorMap t1 = plane_map(pl, Kp, Mp, 1), t0 = plane_map(pl + Mp * Kp, Kp, Mp, 1);
    const CUtensorMap u1 = plane_map(pl + 2 * Mp * Kp, Kp, Mp, 1), u0 = plane_map(pl + 3 * Mp * Kp, Kp, Mp, 1);
    lfd::MmaParams mp{r16, tab.dev, 1, 1, Kp, 0, e, nullptr, polls, 1};
    const size_t smem = lfd::kStages * lfd::kStageBytes + 1024;
    cuda_check(cudaFuncSetAttribute(lfd::residue_mma_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem), "smem");
    lfd::residue_mma_kernel<<<dim3(1, 1, 1), lfd::kMmaThreads, smem, nullptr>>>(t1, t0, u1, u0, mp);
    cuda_check(cudaGetLastError(), "launch");
    cuda_check(cudaDeviceSynchronize(), "bounded wait");
    cuda_check(cudaMemcpy(error_word, e, 4, cudaMemcpyDeviceToHost), "error word");
    LF_API_END
}
