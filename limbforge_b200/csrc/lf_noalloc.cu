// Allocation-free exact product: the same result as lf_dev_exact_product, for callers that must not
// allocate device memory.  Some callers cannot call cudaMalloc at the point where they need a product:
// code running under a memory budget fixed up front (a planner that owns every device byte), host
// threads that must not take the allocator's locks or synchronize the device, and library code
// embedded in another runtime that forbids device allocations.  This entry point therefore keeps all
// of its temporary device data (line table, int8 digit planes, residues, modulus tables and the error
// word) in one file-scope static device array of kScratchBytes, which every GPU that loads this
// library holds until the process exits.  It calls no cudaMalloc, cudaFree or other allocating
// routine; the caller still owns the inputs and the output.
//
// The array is shared by every call and keeps the last call's contents: whatever must start at zero
// (the error word) is cleared by each call, and two calls that overlap on the GPU (different streams or
// threads without ordering between them) would race on the array.  Inside this library the calls are
// serialized process-wide by one lock that is held until the product has completed, so a second host
// thread waits for the first.  The first call on a device (and the first after that device's context was
// destroyed and recreated, which the call detects from the context id) looks up the array's device
// address with cudaGetSymbolAddress (with that device current); make that first call before any stream
// capture.
//
// The residue engine's digit planes and residues must fit the array.  When they do not, the product runs
// on the generic limb kernel, which needs only the error word and gives the same bits; only products of
// more than kMaxLines lines (the line table) are refused.
#include "lf_residue.h"
#include "lf_residue.cuh"

#include <cstring>
#include <mutex>
#include <string>

namespace {

constexpr size_t kScratchBytes = size_t(32) << 20;      // 32 MiB per device
constexpr int kMaxDevices = 64;
constexpr size_t kMaxLines = 8192;                      // left + right lines of one product

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mutex;
unsigned char* g_base[kMaxDevices];                     // device address of g_scratch, per device
unsigned long long g_context[kMaxDevices];              // id of the context that address belongs to
int g_tables_L[kMaxDevices];                            // modulus count whose tables the array holds
int g_tables_qwords[kMaxDevices];                       // their quotient word count
lfd::ResTables g_host_tables;                           // staging for the table upload (host, static)
lfd::LineInfo g_host_lines[kMaxLines];

size_t up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// Unique id of the current context (cuCtxGetId through the runtime's driver entry points): a device
// reset or a destroyed primary context gives the next call a new id.
unsigned long long current_context_id() {
    typedef CUresult (*GetCurrent)(CUcontext*);
    typedef CUresult (*GetId)(CUcontext, unsigned long long*);
    static GetCurrent get_current = nullptr;
    static GetId get_id = nullptr;
    if (!get_current || !get_id) {
        void* f = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
            throw lfr::runtime_error("cuCtxGetCurrent unavailable");
        get_current = reinterpret_cast<GetCurrent>(f);
        if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) != cudaSuccess || q != cudaDriverEntryPointSuccess)
            throw lfr::runtime_error("cuCtxGetId unavailable");
        get_id = reinterpret_cast<GetId>(f);
    }
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (get_current(&ctx) != CUDA_SUCCESS || !ctx || get_id(ctx, &id) != CUDA_SUCCESS) throw lfr::runtime_error("no current CUDA context");
    return id;
}

// Device address of the static array on the current device: set up on the first call per device and
// again whenever the device's context has changed since (the tables uploaded into the old context are
// gone with it).
unsigned char* scratch_base(int device) {
    const unsigned long long ctx = current_context_id();
    if (!g_base[device] || g_context[device] != ctx) {
        void* p = nullptr;
        lfr::cuda_check(cudaGetSymbolAddress(&p, g_scratch), "scratch symbol address");
        g_base[device] = static_cast<unsigned char*>(p);
        g_context[device] = ctx;
        g_tables_L[device] = 0;
    }
    return g_base[device];
}

}  // namespace

using namespace lfr;

extern "C" int lf_dev_exact_product_static(int bits, const void* left, size_t left_ls, size_t left_ks, const void* right,
                                           size_t right_ls, size_t right_ks, size_t M, size_t N, size_t K, void* C, size_t ldc,
                                           int subtract, int lower, void* stream) {
    LF_API_BEGIN
    if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
    if (M >= (size_t(1) << 31) || N >= (size_t(1) << 31) || K >= (size_t(1) << 31)) throw invalid_argument("matrix dimensions exceed 32-bit indexing");
    if (M + N > kMaxLines) throw invalid_argument("static-scratch product: more than 8192 lines (left + right)");
    if (M && N && (!C || (K && (!left || !right)))) throw invalid_argument("null operand");
    std::lock_guard<std::mutex> lock(g_mutex);
    int device = 0;
    cuda_check(cudaGetDevice(&device), "cudaGetDevice");
    if (device < 0 || device >= kMaxDevices) throw runtime_error("device index out of range");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");  // initializes the device's primary context and makes it current
    unsigned char* base = scratch_base(device);
    if (!M || !N) return LF_OK;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    const int n = bits / 32;
    // layout: [error word][tables][line info][digit planes][residues]
    uint32_t* err = reinterpret_cast<uint32_t*>(base);
    auto* tables = reinterpret_cast<lfd::ResTables*>(base + 256);
    const size_t lines_off = up(256 + sizeof(lfd::ResTables), 256);
    auto* linfo = reinterpret_cast<lfd::LineInfo*>(base + lines_off);
    const size_t planes_off = up(lines_off + sizeof(lfd::LineInfo) * (M + N), 256);
    cuda_check(cudaMemsetAsync(err, 0, 4, s), "clear error word");
    const lfd::LineView lv{static_cast<const uint32_t*>(left), left_ls, left_ks};
    const lfd::LineView rv{static_cast<const uint32_t*>(right), right_ls, right_ks};
    uint32_t* out = static_cast<uint32_t*>(C);
    auto limb_kernel = [&] {                            // the generic limb kernel needs only the error word
        lfd::DotParams p{};
        p.left = lv; p.right = rv; p.C = out; p.ldc = ldc; p.M = M; p.Nc = N; p.K = K;
        p.subtract = subtract != 0; p.lower = lower != 0; p.error = err;
        lfd::linalg_kernels(n)->dot(p, s);
        cuda_check(cudaGetLastError(), "exact product launch");
    };
    bool residue = K > 0 && K <= residue_max_k();
    int G = 0, L = 0;
    if (residue) {
        lfd::linalg_kernels(n)->analyze(lv, M, K, linfo, s);
        lfd::linalg_kernels(n)->analyze(rv, N, K, linfo + M, s);
        cuda_check(cudaMemcpyAsync(g_host_lines, linfo, sizeof(lfd::LineInfo) * (M + N), cudaMemcpyDeviceToHost, s), "line info");
        cuda_check(cudaStreamSynchronize(s), "line analysis");
        bool any = false;
        for (size_t i = 0; i < M + N; ++i)
            if (!g_host_lines[i].status && g_host_lines[i].nonzero) { G = std::max(G, g_host_lines[i].top - g_host_lines[i].bottom); any = true; }
        residue = any && G <= residue_max_band() && (L = residue_moduli_for(bits, G, K)) > 0;
    }
    uint64_t Kp = 0, Mp = 0, Np = 0, aplane = 0, bplane = 0;
    size_t res_off = 0;
    if (residue) {                                      // planes and residues must fit the array
        Kp = up(K, lfd::kTileK); Mp = up(M, lfd::kTileM); Np = up(N, lfd::kTileN);
        aplane = (uint64_t)L * Mp * Kp; bplane = (uint64_t)L * Np * Kp;
        res_off = up(planes_off + 2 * (aplane + bplane), 256);
        residue = res_off + sizeof(uint16_t) * (uint64_t)L * M * N <= kScratchBytes;
    }
    if (!residue) {
        limb_kernel();
    } else {
        if (g_tables_L[device] != L) {
            std::memset(&g_host_tables, 0, sizeof(g_host_tables));
            int qw = 0;
            residue_tables_host(L, g_host_tables, qw);
            cuda_check(cudaMemcpyAsync(tables, &g_host_tables, sizeof(lfd::ResTables), cudaMemcpyHostToDevice, s), "modulus tables");
            cuda_check(cudaStreamSynchronize(s), "modulus tables");
            g_tables_L[device] = L;
            g_tables_qwords[device] = qw;
        }
        const int qwords = g_tables_qwords[device];
        auto* pl = reinterpret_cast<signed char*>(base + planes_off);
        signed char *a1 = pl, *a0 = pl + aplane, *b1 = pl + 2 * aplane, *b0 = pl + 2 * aplane + bplane;
        auto* res = reinterpret_cast<uint16_t*>(base + res_off);
        const int xwords = n + (G + 31) / 32 + 1;
        const auto* rk = lfd::residue_kernels(n);
        rk->digits(lfd::DigitParams{lv, M, K, Kp, Mp, L, xwords, linfo, tables, a1, a0}, s);
        rk->digits(lfd::DigitParams{rv, N, K, Kp, Np, L, xwords, linfo + M, tables, b1, b0}, s);
        cuda_check(cudaGetLastError(), "digit planes");
        const CUtensorMap ta1 = residue_plane_map(a1, Kp, Mp, L), ta0 = residue_plane_map(a0, Kp, Mp, L);
        const CUtensorMap tb1 = residue_plane_map(b1, Kp, Np, L), tb0 = residue_plane_map(b0, Kp, Np, L);
        lfd::MmaParams mp{res, tables, M, N, Kp, lower ? 1 : 0, err};
        residue_mma_launch(dim3((unsigned)(Np / lfd::kTileN), (unsigned)(Mp / lfd::kTileM), (unsigned)L), ta1, ta0, tb1, tb0, mp, s);
        rk->rec(lfd::RecParams{res, tables, L, qwords, linfo, linfo + M, out, ldc, M, N, subtract ? 1 : 0, lower ? 1 : 0}, s);
        cuda_check(cudaGetLastError(), "reconstruction");
    }
    uint32_t e = 0;
    cuda_check(cudaMemcpyAsync(&e, err, 4, cudaMemcpyDeviceToHost, s), "error word");
    cuda_check(cudaStreamSynchronize(s), "static-scratch product");
    if (e) throw runtime_error("static-scratch product: device error " + std::to_string(e));
    LF_API_END
}
