// C ABI of precision casts and tree sums: Engine::cast (engine.hpp:205), CommandBatch::cast and
// CommandBatch::tree_sum (engine.hpp:150-175), and device-pointer forms.
#include "lf_runtime.h"
#include "lf_reduce.cuh"

#include <chrono>

namespace lfr {

static void check_width(int bits) {
    if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
}
static void launch_cast(int from_bits, int to_bits, bool complex, const void* in, void* out, size_t count, cudaStream_t s) {
    if (!count) return;
    lfd::cast_launcher(to_bits / 32)(static_cast<const uint32_t*>(in), static_cast<uint32_t*>(out), count * (complex ? 2 : 1),
                                     from_bits / 32, s);
    cuda_check(cudaGetLastError(), "cast launch");
}
// Levels of the adjacent-pair tree; scratch holds two arrays of ceil(count/2) elements.
static void launch_tree_sum(int bits, bool complex, const void* in, size_t count, void* out, void* scratch, cudaStream_t s) {
    const auto level = lfd::tree_level_launcher(bits / 32);
    const size_t es = element_bytes(bits, complex), half = (count + 1) / 2;
    unsigned char* buf[2] = {static_cast<unsigned char*>(scratch), static_cast<unsigned char*>(scratch) + half * es};
    const uint32_t* src = static_cast<const uint32_t*>(in);
    size_t c = count;
    int k = 0;
    do {
        const size_t next = c ? (c + 1) / 2 : 1;
        uint32_t* dst = next == 1 ? static_cast<uint32_t*>(out) : reinterpret_cast<uint32_t*>(buf[k]);
        level(complex, src, dst, c, s);
        cuda_check(cudaGetLastError(), "tree sum launch");
        src = dst; c = next; k ^= 1;
    } while (c > 1);
}

// Element counts of a, b and out of a segmented dot (engine.mm dot_elements rule).
static void dot_elements(int bits, const lf_segmented_dot& d, size_t n[3]) {
    validate(bits, d.segments);
    if (d.segments > 0xffffffffull || d.length > 0xffffffffull) throw invalid_argument("segmented dot exceeds 32-bit indexing");
    n[0] = checked_size(d.segments, d.length);
    n[1] = d.shared_right ? d.length : n[0];
    n[2] = d.segments;
}
static void launch_segdot(int bits, bool complex, const lf_segmented_dot& d, const void* a, const void* b, void* out, cudaStream_t s) {
    if (!d.segments) return;
    lfd::sequence_launchers(bits / 32)->segdot(complex, d.shared_right != 0, static_cast<const uint32_t*>(a), static_cast<const uint32_t*>(b),
                                               static_cast<uint32_t*>(out), d.segments, d.length, s);
    cuda_check(cudaGetLastError(), "segmented dot launch");
}

}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};

extern "C" {

int lf_engine_cast(lf_engine* e, int from_bits, int to_bits, int complex_, const void* in, void* out, size_t count, lf_timing* timing) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    check_width(from_bits); check_width(to_bits);
    validate(to_bits, count);
    if (timing) *timing = {0, 0};
    if (!count) return LF_OK;
    if (!in || !out) throw invalid_argument("null cast operand");
    const auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const bool cx = complex_ != 0;
    const size_t ib = checked_size(count, element_bytes(from_bits, cx)), ob = checked_size(count, element_bytes(to_bits, cx));
    void* din = e->scratch[0].get(ib);
    void* dout = e->scratch[1].get(ob);
    cudaStream_t s = e->stream;
    cuda_check(cudaMemcpyAsync(din, in, ib, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaEventRecord(e->e0, s), "event");
    launch_cast(from_bits, to_bits, cx, din, dout, count, s);
    cuda_check(cudaEventRecord(e->e1, s), "event");
    cuda_check(cudaMemcpyAsync(out, dout, ob, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

int lf_batch_cast(lf_batch* bt, int from_bits, int to_bits, int complex_, lf_buffer* in, lf_buffer* out, size_t count) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    check_width(from_bits); check_width(to_bits);
    validate(to_bits, count);
    const bool cx = complex_ != 0;
    if (!in || !out) throw invalid_argument("missing cast buffer");
    if (in->bytes < checked_size(count, element_bytes(from_bits, cx)) || out->bytes < checked_size(count, element_bytes(to_bits, cx)))
        throw invalid_argument("cast: buffer counts do not match");
    if (in == out && from_bits != to_bits) throw invalid_argument("cast: input and output alias with different widths");
    bt->retain(in);
    bt->retain(out, true);
    if (!count) return LF_OK;
    Op o;
    o.kind = kCustom;
    Buffer* a = in; Buffer* z = out;
    o.custom = [=](cudaStream_t s) { launch_cast(from_bits, to_bits, cx, a->dev, z->dev, count, s); };
    bt->ops.push_back(o);
    LF_API_END
}

int lf_batch_tree_sum(lf_batch* bt, int bits, int complex_, lf_buffer* in, lf_buffer* out, size_t count) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    check_width(bits);
    validate(bits, count);
    const bool cx = complex_ != 0;
    const size_t es = element_bytes(bits, cx);
    if (!in || !out) throw invalid_argument("missing tree sum buffer");
    if (in->bytes < checked_size(count, es)) throw invalid_argument("tree sum: input smaller than its count");
    if (out->bytes < es) throw invalid_argument("tree sum output must contain one element");
    bt->retain(in);
    bt->retain(out, true);
    Op o;
    o.kind = kCustom;
    Buffer* a = in; Buffer* z = out;
    Engine* eng = bt->engine;
    o.custom = [=](cudaStream_t s) {
        void* scratch = eng->scratch[5].get(2 * ((count + 1) / 2) * es + 16);
        launch_tree_sum(bits, cx, a->dev, count, z->dev, scratch, s);
    };
    bt->ops.push_back(o);
    LF_API_END
}

int lf_engine_segmented_dot(lf_engine* e, int bits, int complex_, const lf_segmented_dot* shape, const void* a, const void* b,
                            void* out, lf_timing* timing) {
    LF_API_BEGIN
    if (!e || !shape) throw invalid_argument("null argument");
    size_t n[3];
    dot_elements(bits, *shape, n);
    if (timing) *timing = {0, 0};
    if (!shape->segments) return LF_OK;
    if ((n[0] && !a) || (n[1] && !b) || !out) throw invalid_argument("null segmented dot buffer");
    const auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const size_t es = element_bytes(bits, complex_ != 0);
    const size_t ab = checked_size(n[0], es), bb = checked_size(n[1], es), ob = checked_size(n[2], es);
    void* da = e->scratch[0].get(ab + 16);
    void* db = e->scratch[1].get(bb + 16);
    void* dout = e->scratch[2].get(ob);
    cudaStream_t s = e->stream;
    if (ab) cuda_check(cudaMemcpyAsync(da, a, ab, cudaMemcpyHostToDevice, s), "upload");
    if (bb) cuda_check(cudaMemcpyAsync(db, b, bb, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaEventRecord(e->e0, s), "event");
    launch_segdot(bits, complex_ != 0, *shape, da, db, dout, s);
    cuda_check(cudaEventRecord(e->e1, s), "event");
    cuda_check(cudaMemcpyAsync(out, dout, ob, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

int lf_batch_segmented_dot(lf_batch* bt, int bits, int complex_, const lf_segmented_dot* shape, lf_buffer* a, lf_buffer* b,
                           lf_buffer* out) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    if (!shape) throw invalid_argument("null argument");
    size_t n[3];
    dot_elements(bits, *shape, n);
    const size_t es = element_bytes(bits, complex_ != 0);
    if (!a || !b || !out) throw invalid_argument("missing segmented dot buffer");
    if (a->bytes < checked_size(n[0], es) || b->bytes < checked_size(n[1], es) || out->bytes < checked_size(n[2], es))
        throw invalid_argument("segmented dot buffer too small");
    bt->retain(a);
    bt->retain(b);
    bt->retain(out, true);
    if (!shape->segments) return LF_OK;
    Op o;
    o.kind = kCustom;
    const lf_segmented_dot d = *shape;
    const bool cx = complex_ != 0;
    Buffer* x = a; Buffer* y = b; Buffer* z = out;
    o.custom = [=](cudaStream_t s) { launch_segdot(bits, cx, d, x->dev, y->dev, z->dev, s); };
    bt->ops.push_back(o);
    LF_API_END
}

int lf_engine_recurrence(lf_engine* e, int bits, const void* seeds, const void* weights, void* out, size_t count, unsigned steps,
                         unsigned states_per_weight, lf_timing* timing) {
    LF_API_BEGIN
    if (!e) throw invalid_argument("null engine");
    validate(bits, count);
    if (!states_per_weight || count % states_per_weight) throw invalid_argument("count must be divisible by states_per_weight");
    if (timing) *timing = {0, 0};
    if (!count) return LF_OK;
    if (!seeds || !out || (steps && !weights)) throw invalid_argument("null recurrence buffer");
    if (count > 0xffffffffull / 4 || (steps && (uint64_t)steps * 4 * (count / states_per_weight) > 0xffffffffull))
        throw invalid_argument("recurrence exceeds 32-bit indexing");
    const auto w0 = std::chrono::steady_clock::now();
    e->activate();
    const size_t es = element_bytes(bits, true);
    const size_t sb = checked_size(checked_size(count, es), 4), wb = checked_size(checked_size(count / states_per_weight, es), (size_t)steps * 4);
    void* ds = e->scratch[0].get(sb);
    void* dw = e->scratch[1].get(wb + 16);
    void* dout = e->scratch[2].get(count * es);
    cudaStream_t s = e->stream;
    cuda_check(cudaMemcpyAsync(ds, seeds, sb, cudaMemcpyHostToDevice, s), "upload");
    if (wb) cuda_check(cudaMemcpyAsync(dw, weights, wb, cudaMemcpyHostToDevice, s), "upload");
    cuda_check(cudaEventRecord(e->e0, s), "event");
    lfd::sequence_launchers(bits / 32)->recurrence(static_cast<const uint32_t*>(ds), static_cast<const uint32_t*>(dw),
                                                   static_cast<uint32_t*>(dout), count, steps, states_per_weight, s);
    cuda_check(cudaGetLastError(), "recurrence launch");
    cuda_check(cudaEventRecord(e->e1, s), "event");
    cuda_check(cudaMemcpyAsync(out, dout, count * es, cudaMemcpyDeviceToHost, s), "download");
    cuda_check(cudaStreamSynchronize(s), "execution");
    float ms = 0;
    cudaEventElapsedTime(&ms, e->e0, e->e1);
    if (timing) *timing = {ms * 1e-3, std::chrono::duration<double>(std::chrono::steady_clock::now() - w0).count()};
    LF_API_END
}

// Device-pointer forms (no reference counterpart): asynchronous on `stream`.
int lf_dev_cast(int from_bits, int to_bits, int complex_, const void* in, void* out, size_t count, void* stream) {
    LF_API_BEGIN
    check_width(from_bits); check_width(to_bits);
    validate(to_bits, count);
    if (count && (!in || !out)) throw invalid_argument("null cast operand");
    launch_cast(from_bits, to_bits, complex_ != 0, in, out, count, static_cast<cudaStream_t>(stream));
    LF_API_END
}
int lf_dev_tree_sum(int bits, int complex_, const void* in, size_t count, void* out, void* scratch, void* stream) {
    LF_API_BEGIN
    check_width(bits);
    validate(bits, count);
    if (!out || (count && !in) || (count > 2 && !scratch)) throw invalid_argument("null tree sum operand");
    launch_tree_sum(bits, complex_ != 0, in, count, out, scratch, static_cast<cudaStream_t>(stream));
    LF_API_END
}

}  // extern "C"
