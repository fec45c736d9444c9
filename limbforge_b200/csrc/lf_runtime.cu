// C ABI of the engine, buffers, command batches and submissions (the reference's
// include/limbforge/engine.hpp:74-227 and src/engine.mm), on one CUDA device per engine:
// device-resident buffers, one in-order CUDA stream per engine, CUDA events for timing.
#include "lf_runtime.h"
#include "lf_elementwise.cuh"

#include <algorithm>
#include <cstdio>

namespace lfr {

static thread_local std::string g_error;
void set_error(const std::string& m) { g_error = m; }
void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) throw runtime_error(std::string("CUDA ") + what + ": " + cudaGetErrorString(e));
}
static std::atomic<uint64_t> g_identity{1};

void Batch::retain(Buffer* r, bool write) {
    if (!r || r->owner != engine->identity) throw invalid_argument("buffer belongs to another engine");
    if (r->busy.load(std::memory_order_acquire)) throw logic_error("buffer belongs to an unwaited submission");
    if (std::find(resources.begin(), resources.end(), r) == resources.end()) {
        r->refs.fetch_add(1);
        resources.push_back(r);
    }
    if (write && std::find(written.begin(), written.end(), r) == written.end()) written.push_back(r);
}
static void release(Buffer* b) { if (b && b->refs.fetch_sub(1) == 1) delete b; }
Batch::~Batch() { for (auto* r : resources) release(r); }

void Submission::finish() {
    if (done) return;
    cudaError_t e = cudaEventSynchronize(end);
    if (e == cudaSuccess) {
        float ms = 0;
        cudaEventElapsedTime(&ms, start, end);
        timing.gpu_seconds = ms * 1e-3;
    } else {
        error = cudaGetErrorString(e);
    }
    timing.wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - wall0).count();
    for (auto* r : resources) { r->busy.store(false, std::memory_order_release); release(r); }
    resources.clear();
    keep.clear();
    done = true;
}
Submission::~Submission() {
    finish();
    if (start) cudaEventDestroy(start);
    if (end) cudaEventDestroy(end);
}

void launch_elementwise(int bits, int op, const void* a, const void* b, const void* c, void* out, size_t count,
                        lf_broadcast bi, lf_broadcast ci, cudaStream_t s) {
    if (!count) return;
    auto f = lfd::ew_launcher(bits / 32);
    if (!f) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
    lfd::EwParams p{static_cast<const uint32_t*>(a), static_cast<const uint32_t*>(b), static_cast<const uint32_t*>(c),
                    static_cast<uint32_t*>(out), count, bi.stride, bi.period, ci.stride, ci.period};
    if (f(op, p, s)) throw invalid_argument("unknown arithmetic operation");
    cuda_check(cudaGetLastError(), "element-wise launch");
}

// One fused chain of binary real ops whose running value stays in registers.
static void launch_chain(int bits, const Op* const* steps, int n, const bool* write, cudaStream_t s) {
    lfd::ChainParams p{};
    p.a = static_cast<const uint32_t*>(steps[0]->a->dev);
    p.count = steps[0]->count;
    p.steps = n;
    for (int k = 0; k < n; ++k) {
        p.step[k].b = static_cast<const uint32_t*>(steps[k]->b->dev);
        p.step[k].out = write[k] ? static_cast<uint32_t*>(steps[k]->out->dev) : nullptr;
        p.step[k].bs = steps[k]->bi.stride; p.step[k].bp = steps[k]->bi.period;
        p.step[k].op = steps[k]->op;
    }
    auto f = lfd::chain_launcher(bits / 32);
    f(p, s);
    cuda_check(cudaGetLastError(), "chain launch");
}

static bool chainable(const Op& o) {
    return o.kind == kElementwise && !o.complex && o.op >= 0 && o.op <= 3 && o.count > 0;
}

// Launches the batch in order.  Runs of dependent binary real ops (a_k = out_{k-1}, same width
// and count, b_k not written earlier in the run) become one chain kernel; an intermediate
// output is stored only when no later step of the run overwrites the same buffer.
static void launch_ops(Engine& eng, std::vector<Op>& ops) {
    cudaStream_t s = eng.stream;
    size_t i = 0;
    while (i < ops.size()) {
        Op& o = ops[i];
        if (chainable(o)) {
            std::vector<const Op*> run{&o};
            std::vector<Buffer*> outs{o.out};
            size_t j = i + 1;
            while (j < ops.size() && run.size() < (size_t)lfd::kMaxChain) {
                const Op& q = ops[j];
                if (!chainable(q) || q.bits != o.bits || q.count != o.count || q.a != run.back()->out) break;
                if (std::find(outs.begin(), outs.end(), q.b) != outs.end()) break;
                run.push_back(&q); outs.push_back(q.out); ++j;
            }
            if (run.size() >= 2) {
                std::vector<char> write(run.size(), 1);
                for (size_t k = 0; k < run.size(); ++k)
                    for (size_t m = k + 1; m < run.size(); ++m)
                        if (run[m]->out == run[k]->out) { write[k] = 0; break; }
                launch_chain(o.bits, run.data(), (int)run.size(), reinterpret_cast<const bool*>(write.data()), s);
                i = j;
                continue;
            }
        }
        switch (o.kind) {
        case kElementwise:
            launch_elementwise(o.bits, o.op, o.a->dev, o.b ? o.b->dev : nullptr, o.c ? o.c->dev : nullptr, o.out->dev, o.count,
                               o.bi, o.ci, s);
            break;
        case kLu4:
            launch_lu4(o.bits, o.lu, o.a ? o.a->dev : nullptr, o.b ? o.b->dev : nullptr, o.c ? o.c->dev : nullptr, o.out ? o.out->dev : nullptr,
                       o.e ? static_cast<uint32_t*>(o.e->dev) : nullptr, s);
            break;
        case kStridedGemm:
            launch_strided_gemm(o.bits, o.complex, o.sg, o.a ? o.a->dev : nullptr, o.b ? o.b->dev : nullptr, o.out->dev, s);
            break;
        default:
            o.custom(s);
        }
        ++i;
    }
}

}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};
struct lf_submission : Submission {};

extern "C" {

const char* lf_last_error(void) { return g_error.c_str(); }
const char* lf_version(void) { return "limbforge_b200 1.3.1 (sm_100a)"; }

// Engine::prewarm (engine.hpp:190): the kernels are compiled ahead for sm_100a, so preparing a width means
// validating it and loading the requested element-wise kernels' modules now instead of at their first launch.
int lf_engine_prewarm(lf_engine* e, const int* bits, size_t nbits, const int* ops, size_t nops) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    for (size_t i = 0; i < nbits; ++i) validate(bits[i], 0);
    for (size_t j = 0; j < nops; ++j) if (!op_valid(ops[j])) throw invalid_argument("invalid operation");
    e->activate();
    for (size_t i = 0; i < nbits; ++i)
        for (size_t j = 0; j < nops; ++j) {
            cudaFuncAttributes a{};
            cuda_check(static_cast<cudaError_t>(lfd::ew_attributes_of(bits[i] / 32)(ops[j], &a)), "kernel load");
        }
    LF_API_END
}
// Engine::pipeline_info (engine.hpp:193): warp width, the kernel's largest block and the block it is launched with.
int lf_engine_pipeline_info(lf_engine* e, int bits, int op, unsigned* simd_width, unsigned* max_threads, unsigned* threads) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    validate(bits, 0);
    if (!op_valid(op)) throw invalid_argument("invalid operation");
    e->activate();
    cudaFuncAttributes a{};
    cuda_check(static_cast<cudaError_t>(lfd::ew_attributes_of(bits / 32)(op, &a)), "kernel attributes");
    if (simd_width) *simd_width = 32;
    if (max_threads) *max_threads = (unsigned)a.maxThreadsPerBlock;
    if (threads) *threads = (unsigned)lfd::kEwThreads;
    LF_API_END
}
void lf_api_version(unsigned* major, unsigned* minor, unsigned* patch) {
    if (major) *major = 1;
    if (minor) *minor = 3;
    if (patch) *patch = 1;
}

int lf_engine_create(const lf_engine_options* options, lf_engine** out) {
    LF_API_BEGIN
    if (!out) throw invalid_argument("null engine handle");
    int count = 0;
    cuda_check(cudaGetDeviceCount(&count), "device query");
    int device = options ? options->device : 0;
    if (device < 0 || device >= count) throw runtime_error("no CUDA GPU available");
    auto* e = new lf_engine();
    e->device = device;
    if (options) e->options = *options;
    e->identity = g_identity.fetch_add(1);
    try {
        e->activate();
        cudaDeviceProp prop{};
        cuda_check(cudaGetDeviceProperties(&prop, device), "device properties");
        e->name = prop.name;
        cuda_check(cudaStreamCreateWithFlags(&e->stream, cudaStreamNonBlocking), "stream");
        cuda_check(cudaEventCreate(&e->e0), "event");
        cuda_check(cudaEventCreate(&e->e1), "event");
    } catch (...) { delete e; throw; }
    *out = e;
    LF_API_END
}
void lf_engine_destroy(lf_engine* e) {
    if (!e) return;
    cudaSetDevice(e->device);
    cudaStreamSynchronize(e->stream);
    cudaEventDestroy(e->e0); cudaEventDestroy(e->e1);
    cudaStreamDestroy(e->stream);
    delete e;
}
int lf_engine_device_name(lf_engine* e, char* name, size_t capacity) {
    LF_API_BEGIN
    if (!e || !name || !capacity) throw invalid_argument("null argument");
    std::snprintf(name, capacity, "%s", e->name.c_str());
    LF_API_END
}

// Host-array element-wise call: copy in, one kernel, copy out (engine.mm:254-280 contract).
static void host_dispatch(Engine& e, int bits, int op, const void* a, const void* b, const void* c, void* out, size_t count,
                          lf_broadcast bi, lf_broadcast ci, lf_timing* timing) {
    auto w0 = std::chrono::steady_clock::now();
    e.activate();
    const size_t stride = element_bytes(bits, op_complex(op));
    const size_t bytes = checked_size(count, stride);
    const size_t bb = op_unary(op) ? 0 : checked_size(broadcast_elements(count, bi), stride);
    const size_t cb = op_ternary(op) ? checked_size(broadcast_elements(count, ci), stride) : 0;
    void* da = e.scratch[0].get(bytes);
    void* db = bb ? e.scratch[1].get(bb) : nullptr;
    void* dc = cb ? e.scratch[2].get(cb) : nullptr;
    void* dout = e.scratch[3].get(bytes);
    cudaStream_t s = e.stream;
    cuda_check(cudaMemcpyAsync(da, a, bytes, cudaMemcpyHostToDevice, s), "upload");
    if (bb) cuda_check(cudaMemcpyAsync(db, b, bb, cudaMemcpyHostToDevice, s), "upload");
    if (cb) cuda_check(cudaMemcpyAsync(dc, c, cb, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaEventRecord(e.e0, s), "event");
    launch_elementwise(bits, op, da, db, dc, dout, count, bi, ci, s);
    cuda_check(cudaEventRecord(e.e1, s), "event");
    cuda_check(cudaMemcpyAsync(out, dout, bytes, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e.e0, e.e1);
    if (timing) {
        timing->gpu_seconds = ms * 1e-3;
        timing->wall_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count();
    }
}

int lf_engine_run(lf_engine* e, int bits, int op, const void* a, const void* b, void* out, size_t count,
                  lf_broadcast bi, lf_timing* timing) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    validate(bits, count);
    if (!op_valid(op)) throw invalid_argument("unknown arithmetic operation");
    if (op_ternary(op)) throw invalid_argument("use run_ternary for fused operations");
    if (timing) *timing = {0, 0};
    if (!count) return LF_OK;
    if (!a || (!b && !op_unary(op)) || !out) throw invalid_argument("null arithmetic buffer");
    host_dispatch(*e, bits, op, a, b, nullptr, out, count, bi, lf_broadcast{1, 0}, timing);
    LF_API_END
}
int lf_engine_run_unary(lf_engine* e, int bits, int op, const void* a, void* out, size_t count, lf_timing* timing) {
    LF_API_BEGIN
    if (!op_unary(op)) throw invalid_argument("operation requires two inputs");
    int rc = lf_engine_run(e, bits, op, a, nullptr, out, count, lf_broadcast{1, 0}, timing);
    if (rc) return rc;
    LF_API_END
}
int lf_engine_run_ternary(lf_engine* e, int bits, int op, const void* a, const void* b, const void* c, void* out,
                          size_t count, lf_broadcast bi, lf_broadcast ci, lf_timing* timing) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    validate(bits, count);
    if (!op_ternary(op)) throw invalid_argument("operation does not take three inputs");
    if (timing) *timing = {0, 0};
    if (!count) return LF_OK;
    if (!a || !b || !c || !out) throw invalid_argument("null arithmetic buffer");
    host_dispatch(*e, bits, op, a, b, c, out, count, bi, ci, timing);
    LF_API_END
}

// ---- buffers
// A cudaMemcpy from pageable host memory may return before its DMA has landed, and work on the
// engines' non-blocking streams is not ordered after the legacy default stream that carried it:
// every host-to-device transfer outside a stream is followed by this wait.
static void landed() { cuda_check(cudaStreamSynchronize(0), "host-to-device transfer"); }
int lf_buffer_create(lf_engine* e, size_t bytes, lf_buffer** out) {
    LF_API_BEGIN
    if (!e || !out) throw invalid_argument("null argument");
    e->activate();
    auto* b = new lf_buffer();
    b->owner = e->identity; b->device = e->device; b->bytes = bytes;
    cudaError_t r = cudaMalloc(&b->dev, bytes ? bytes : 16);
    if (r != cudaSuccess) { b->dev = nullptr; delete b; throw runtime_error(std::string("CUDA buffer allocation: ") + cudaGetErrorString(r)); }
    r = cudaMemset(b->dev, 0, bytes ? bytes : 16);
    if (r == cudaSuccess) r = cudaStreamSynchronize(0);        // the memset is asynchronous to the host
    if (r != cudaSuccess) { cudaFree(b->dev); b->dev = nullptr; delete b; throw runtime_error(std::string("CUDA buffer clear: ") + cudaGetErrorString(r)); }
    *out = b;
    LF_API_END
}
void lf_buffer_release(lf_buffer* b) { release(b); }
size_t lf_buffer_bytes(const lf_buffer* b) { return b ? b->bytes : 0; }
// References to the buffer besides its owner's: batches that recorded it and submissions not yet waited.
int lf_buffer_holders(const lf_buffer* b) { return b ? b->refs.load(std::memory_order_acquire) - 1 : 0; }
static void idle(const Buffer* b) {
    if (!b) throw invalid_argument("empty buffer handle");
    if (b->busy.load(std::memory_order_acquire)) throw logic_error("buffer belongs to an unwaited submission");
}
int lf_buffer_upload(lf_buffer* b, const void* src, size_t bytes) {
    LF_API_BEGIN
    idle(b);
    if (bytes > b->bytes || (!src && bytes)) throw invalid_argument("invalid transfer");
    cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
    if (b->host_authoritative && bytes < b->bytes) {           // keep the mapped tail
        cuda_check(cudaMemcpy(b->dev, b->host, b->bytes, cudaMemcpyHostToDevice), "mirror upload");
    }
    b->host_authoritative = false;
    if (bytes) cuda_check(cudaMemcpy(b->dev, src, bytes, cudaMemcpyHostToDevice), "upload");
    landed();
    LF_API_END
}
int lf_buffer_download(lf_buffer* b, void* dst, size_t bytes) {
    LF_API_BEGIN
    idle(b);
    if (bytes > b->bytes || (!dst && bytes)) throw invalid_argument("invalid transfer");
    if (!bytes) return LF_OK;
    if (b->host_authoritative) std::memcpy(dst, b->host, bytes);
    else { cuda_check(cudaSetDevice(b->device), "cudaSetDevice"); cuda_check(cudaMemcpy(dst, b->dev, bytes, cudaMemcpyDeviceToHost), "download"); }
    LF_API_END
}
int lf_buffer_mapped(lf_buffer* b, void** host) {
    LF_API_BEGIN
    idle(b);
    if (!host) throw invalid_argument("null argument");
    cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
    if (!b->host) cuda_check(cudaMallocHost(&b->host, b->bytes ? b->bytes : 16), "host mirror");
    if (!b->host_authoritative && b->bytes) cuda_check(cudaMemcpy(b->host, b->dev, b->bytes, cudaMemcpyDeviceToHost), "mirror download");
    b->host_authoritative = true;
    *host = b->host;
    LF_API_END
}
int lf_host_alloc(size_t bytes, void** host) {
    LF_API_BEGIN
    if (!host) throw invalid_argument("null argument");
    cuda_check(cudaMallocHost(host, bytes ? bytes : 16), "pinned host allocation");
    LF_API_END
}
void lf_host_free(void* host) { if (host) cudaFreeHost(host); }
int lf_buffer_device_pointer(lf_buffer* b, void** device) {
    LF_API_BEGIN
    idle(b);
    if (!device) throw invalid_argument("null argument");
    if (b->host_authoritative) {
        cuda_check(cudaSetDevice(b->device), "cudaSetDevice");
        cuda_check(cudaMemcpy(b->dev, b->host, b->bytes, cudaMemcpyHostToDevice), "mirror upload");
        landed();
        b->host_authoritative = false;
    }
    *device = b->dev;
    LF_API_END
}

// ---- batches
int lf_batch_create(lf_engine* e, lf_batch** out) {
    LF_API_BEGIN
    if (!e || !out) throw invalid_argument("null argument");
    auto* b = new lf_batch();
    b->engine = e;
    *out = b;
    LF_API_END
}
void lf_batch_destroy(lf_batch* b) { delete b; }
static void open(lf_batch* b) { if (!b || b->submitted) throw logic_error("batch already submitted or moved"); }
static void need(const Buffer* b, size_t bytes, const char* what) {
    if (!b) throw invalid_argument(std::string("missing ") + what + " buffer");
    if (b->bytes < bytes) throw invalid_argument("buffer counts do not match the broadcast");
}
int lf_batch_run(lf_batch* bt, int bits, int complex_, int op, lf_buffer* a, lf_buffer* b, lf_buffer* c, lf_buffer* out,
                 size_t count, lf_broadcast bi, lf_broadcast ci) {
    LF_API_BEGIN
    open(bt);
    validate(bits, count);
    if (!op_valid(op) || op_complex(op) != (complex_ != 0)) throw invalid_argument("operation and buffer format mismatch");
    const size_t stride = element_bytes(bits, complex_ != 0);
    need(a, checked_size(count, stride), "a");
    need(out, checked_size(count, stride), "out");
    if (!op_unary(op)) need(b, checked_size(broadcast_elements(count, bi), stride), "b");
    if (op_ternary(op)) need(c, checked_size(broadcast_elements(count, ci), stride), "c");
    bt->retain(a);
    if (!op_unary(op)) bt->retain(b);
    if (op_ternary(op)) bt->retain(c);
    bt->retain(out, true);
    if (!count) return LF_OK;
    Op o;
    o.kind = kElementwise; o.bits = bits; o.op = op; o.complex = complex_ != 0;
    o.a = a; o.b = op_unary(op) ? nullptr : b; o.c = op_ternary(op) ? c : nullptr; o.out = out;
    o.count = count; o.bi = bi; o.ci = ci;
    bt->ops.push_back(o);
    LF_API_END
}
int lf_batch_submit(lf_batch* bt, lf_submission** out) {
    LF_API_BEGIN
    open(bt);
    if (!out) throw invalid_argument("null submission handle");
    Engine& e = *bt->engine;
    size_t claimed = 0;
    for (auto* r : bt->resources) {
        bool expected = false;
        if (!r->busy.compare_exchange_strong(expected, true)) {
            for (size_t i = 0; i < claimed; ++i) bt->resources[i]->busy.store(false);
            throw logic_error("buffer belongs to an unwaited submission");
        }
        ++claimed;
    }
    auto* sub = new lf_submission();
    sub->engine = &e;
    sub->wall0 = std::chrono::steady_clock::now();
    try {
        e.activate();
        cuda_check(cudaEventCreate(&sub->start), "event");
        cuda_check(cudaEventCreate(&sub->end), "event");
        for (auto* r : bt->resources) r->sync_to_device(e.stream);
        cuda_check(cudaEventRecord(sub->start, e.stream), "event");
        launch_ops(e, bt->ops);
        cuda_check(cudaEventRecord(sub->end, e.stream), "event");
    } catch (...) {
        cudaStreamSynchronize(e.stream);
        for (auto* r : bt->resources) r->busy.store(false);
        delete sub;
        throw;
    }
    sub->resources.swap(bt->resources);     // references move to the submission
    sub->keep.swap(bt->keep);
    bt->submitted = true;
    *out = sub;
    LF_API_END
}
int lf_submission_ready(lf_submission* s, int* ready) {
    LF_API_BEGIN
    if (!s || !ready) throw logic_error("empty submission");
    if (s->done) { *ready = 1; return LF_OK; }
    cudaError_t r = cudaEventQuery(s->end);
    *ready = (r == cudaSuccess || r != cudaErrorNotReady) ? 1 : 0;
    LF_API_END
}
int lf_submission_wait(lf_submission* s, lf_timing* timing) {
    LF_API_BEGIN
    if (!s) throw logic_error("empty submission");
    s->finish();
    if (!s->error.empty()) throw runtime_error("CUDA execution: " + s->error);
    if (timing) *timing = s->timing;
    LF_API_END
}
void lf_submission_destroy(lf_submission* s) { delete s; }

// ---- device-pointer entry points
int lf_dev_elementwise(int bits, int op, const void* a, const void* b, const void* c, void* out, size_t count,
                       lf_broadcast bi, lf_broadcast ci, void* stream) {
    LF_API_BEGIN
    validate(bits, count);
    if (!op_valid(op)) throw invalid_argument("unknown arithmetic operation");
    if (!count) return LF_OK;
    if (!a || !out || (!op_unary(op) && !b) || (op_ternary(op) && !c)) throw invalid_argument("null arithmetic buffer");
    if (!op_unary(op)) broadcast_elements(count, bi);
    if (op_ternary(op)) broadcast_elements(count, ci);
    launch_elementwise(bits, op, a, b, c, out, count, bi, ci, static_cast<cudaStream_t>(stream));
    LF_API_END
}
int lf_dev_mul_chain(int bits, const void* x, const void* factors, size_t factor_stride, unsigned steps, void* out,
                     size_t count, void* stream) {
    return lf_dev_mul_chain_lanes(bits, 1, x, factors, factor_stride, steps, out, count, stream);
}
int lf_dev_mul_chain_lanes(int bits, int lanes, const void* x, const void* factors, size_t factor_stride, unsigned steps, void* out,
                           size_t count, void* stream) {
    LF_API_BEGIN
    if (lanes != 1 && lanes != 2) throw invalid_argument("lanes must be 1 or 2");
    validate(bits, count);
    if (!count) return LF_OK;
    if (!x || !out || (steps && !factors)) throw invalid_argument("null arithmetic buffer");
    const size_t E = (size_t)bits / 32 + 3;
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (!steps) {
        if (x != out) cuda_check(cudaMemcpyAsync(out, x, count * E * 4, cudaMemcpyDeviceToDevice, s), "copy");
        return LF_OK;
    }
    const uint32_t* f = static_cast<const uint32_t*>(factors);
    const void* src = x;
    for (unsigned s0 = 0; s0 < steps; s0 += lfd::kMaxChain) {
        lfd::ChainParams p{};
        p.a = static_cast<const uint32_t*>(src);
        p.count = count;
        p.lanes = lanes;
        p.steps = (int)std::min<unsigned>(lfd::kMaxChain, steps - s0);
        for (int k = 0; k < p.steps; ++k) {
            p.step[k].b = f + (size_t)(s0 + k) * factor_stride * E;
            p.step[k].out = k + 1 == p.steps ? static_cast<uint32_t*>(out) : nullptr;
            p.step[k].bs = 1; p.step[k].bp = 0; p.step[k].op = 2;
        }
        lfd::chain_launcher(bits / 32)(p, s);
        cuda_check(cudaGetLastError(), "chain launch");
        src = out;
    }
    LF_API_END
}

}  // extern "C"
