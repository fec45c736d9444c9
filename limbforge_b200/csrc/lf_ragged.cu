// Ragged mixed-precision batches: many small GEMM instances of different shapes and precisions plus
// an optional batched 4x4 LU job, run as one CUDA graph launch.  The reference has no such entry
// point: its BatchedLinalg::gemm (batched_linalg.mm:163-173) takes one StridedGemm shape at one
// precision per call, so a ragged batch is a host loop over groups there.  Every instance computes
// exactly what a one-instance StridedGemm at its precision computes (same kernel body, gemm_cell).
//
// Plan: instances are grouped by limb count; inside a class they are ordered by inner dimension and
// then size, heaviest first, and their output cells numbered consecutively.  Each class runs as one
// persistent kernel whose blocks take chunks of `block` consecutive cells from a counter, so a block
// spans several small instances and the heavy ones start first.  The graph holds one memset of the
// counters, then one branch per class and one for the LU job, joined at the end.
//
// Autotuner: for each class it times every block size in {32, 64, 128, 256} (grid = SMs x resident
// blocks per SM at that size) on the arena's own data, writing outputs to plan-owned scratch, and
// keeps the fastest; for the LU job it times block sizes in {32, 64, 128, 256} with one thread per
// system or a persistent grid-stride grid.
#include "lf_runtime.h"
#include "lf_batched.cuh"

#include <algorithm>
#include <map>
#include <numeric>
#include <vector>

namespace lfr {
namespace {

constexpr unsigned kBlocks[] = {32, 64, 128, 256};
constexpr uint64_t kAlign = 256;

uint64_t up(uint64_t x, uint64_t a) { return (x + a - 1) / a * a; }
uint64_t mul64(uint64_t a, uint64_t b) {
    if (a && b > UINT64_MAX / a) throw invalid_argument("ragged batch: size overflow");
    return a * b;
}

struct Interval { uint64_t lo, hi; };       // [lo, hi) bytes

}  // namespace

struct ClassPlan {
    int limbs = 0;
    std::vector<lfd::GemmItem> items;        // sorted, cell0 filled
    uint64_t cells = 0;
    DevBuf d_items, d_chunks;
    unsigned block = 128, grid = 0;          // grid 0: not yet sized
    unsigned chunk_block = 0;                // block size the uploaded chunk table was built for
    uint32_t nchunks = 0;
    double trial_ms = 0;
};

struct RaggedPlan {
    Engine* engine = nullptr;
    bool cx = false, fused = false;
    uint64_t arena_bytes = 0;
    std::vector<ClassPlan> classes;
    bool has_lu = false;
    lf_ragged_lu4 lu{};
    Lu4Sizes lu_n{};
    unsigned lu_block = 64, lu_grid = 0; double lu_trial_ms = 0;
    bool tuned = false;
    int sms = 0;
    DevBuf counters, scratch;
    cudaStream_t streams[33] = {};
    cudaEvent_t fork = nullptr, joins[33] = {}, done = nullptr;
    bool done_recorded = false;
    cudaGraphExec_t exec = nullptr;
    const void* graph_arena = nullptr;

    ~RaggedPlan() {
        if (exec) cudaGraphExecDestroy(exec);
        for (auto& s : streams) if (s) cudaStreamDestroy(s);
        for (auto& e : joins) if (e) cudaEventDestroy(e);
        if (fork) cudaEventDestroy(fork);
        if (done) cudaEventDestroy(done);
    }

    uint64_t cell_words(int limbs) const { return uint64_t(limbs + 3) * (cx ? 2 : 1); }

    uint64_t units(const ClassPlan& c) const { return c.cells * (cx ? 2 : 1); }   // a thread per entry or component
    // Chunk table of a class for block size b: chunk c covers units [c b, (c+1) b); its first unit belongs
    // to entry (c b) / (units per entry), owned by item t.
    void build_chunks(ClassPlan& c, unsigned b, cudaStream_t s) {
        if (c.chunk_block == b) return;
        const uint64_t nch = (units(c) + b - 1) / b;
        if (nch > 0x7fffffffull) throw invalid_argument("ragged batch: too many output cells in one precision");
        std::vector<uint32_t> first(nch);
        size_t t = 0;
        for (uint64_t ch = 0; ch < nch; ++ch) {
            const uint64_t g = ch * b / (cx ? 2 : 1);
            while (g >= c.items[t].cell0 + (uint64_t)c.items[t].m * c.items[t].n) ++t;
            first[ch] = (uint32_t)t;
        }
        void* d = c.d_chunks.get(nch * 4 + 16);
        cuda_check(cudaMemcpyAsync(d, first.data(), nch * 4, cudaMemcpyHostToDevice, s), "ragged chunk table");
        cuda_check(cudaStreamSynchronize(s), "ragged chunk table");   // `first` is pageable and local
        c.chunk_block = b;
        c.nchunks = (uint32_t)nch;
    }
    unsigned class_grid(const ClassPlan& c, unsigned b) const {
        const int occ = lfd::gemm_launcher(c.limbs)(cx, fused, lfd::GemmWork{}, 0, b, nullptr);
        return (unsigned)std::max(1, occ) * (unsigned)sms;
    }
    lfd::GemmWork work(const ClassPlan& c, const void* arena, uint32_t* counter, uint32_t* override_out) const {
        lfd::GemmWork w{};
        w.items = static_cast<const lfd::GemmItem*>(c.d_items.p);
        w.chunk_item = static_cast<const uint32_t*>(c.d_chunks.p);
        w.base = static_cast<const uint32_t*>(arena);
        w.out_base = static_cast<uint32_t*>(const_cast<void*>(arena));
        w.cells = units(c); w.nchunks = c.nchunks; w.chunk = c.chunk_block;
        w.counter = counter; w.out_override = override_out;
        return w;
    }
    lfd::Lu4Params lu_params(const void* arena, bool to_scratch) const {
        auto at = [&](uint64_t off) { return static_cast<uint32_t*>(const_cast<void*>(arena)) + off / 4; };
        const lf_batched4& s = lu.shape;
        lfd::Lu4Params p{at(lu.A), lu_n.B ? at(lu.B) : nullptr, lu_n.X ? at(lu.X) : nullptr, lu_n.det ? at(lu.det) : nullptr,
                         at(lu.status), s.count, s.rhs, s.fused, s.determinant, s.inverse};
        if (to_scratch) {                      // trial outputs: X, det, status in the scratch area
            const uint64_t ces = element_bytes(lu.bits, true);
            auto* base = static_cast<unsigned char*>(scratch.p);
            p.X = lu_n.X ? reinterpret_cast<uint32_t*>(base) : nullptr;
            p.det = lu_n.det ? reinterpret_cast<uint32_t*>(base + up(lu_n.X * ces, kAlign)) : nullptr;
            p.status = reinterpret_cast<uint32_t*>(base + up(lu_n.X * ces, kAlign) + up(lu_n.det * ces, kAlign));
        }
        return p;
    }
    void launch_lu(const void* arena, bool to_scratch, unsigned block, unsigned grid, cudaStream_t s) const {
        const lfd::Lu4Params p = lu_params(arena, to_scratch);
        if (lfd::lu4_launcher(lu.bits / 32)(p, grid, block, s)) throw runtime_error("ragged lu4 launch: block does not fit");
        cuda_check(cudaGetLastError(), "ragged lu4 launch");
    }
    // Grid of the LU job at `block` threads (a quad of lanes per system): one quad per system, or a
    // persistent grid of resident blocks; 0 when the block's parked systems exceed shared memory.
    unsigned lu_grid_for(unsigned block, bool persistent) const {
        const int occ = lfd::lu4_launcher(lu.bits / 32)(lfd::Lu4Params{}, 0, block, nullptr);
        if (occ <= 0) return 0;
        if (!persistent) return (unsigned)std::min<uint64_t>((lu.shape.count * lfd::kLuLanes + block - 1) / block, 1u << 30);
        return (unsigned)occ * (unsigned)sms;
    }
};

namespace {

// Instance extents in bytes (empty when the operand is not read / written).
struct Extents { Interval a, b, c; };
Extents extents(const lf_ragged_gemm& it, bool cx) {
    const uint64_t es = element_bytes(it.bits, cx);
    const uint64_t cells = mul64(it.m, it.n);
    Extents e{{it.a, it.a}, {it.b, it.b}, {it.c, it.c}};
    if (!cells) return e;
    e.c.hi = it.c + mul64(cells, es);
    if (it.k) { e.a.hi = it.a + mul64(mul64(it.m, it.k), es); e.b.hi = it.b + mul64(mul64(it.k, it.n), es); }
    return e;
}

void check_bits(int bits) {
    if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
}

}  // namespace
}  // namespace lfr

using namespace lfr;
struct lf_engine : Engine {};
struct lf_ragged_plan : RaggedPlan {};

extern "C" {

int lf_ragged_pack(int complex_, lf_ragged_gemm* items, size_t count, lf_ragged_lu4* lu4, uint64_t* arena_bytes) {
    LF_API_BEGIN
    if (!arena_bytes || (count && !items)) throw invalid_argument("null argument");
    uint64_t off = 0;
    for (size_t i = 0; i < count; ++i) {
        lf_ragged_gemm& it = items[i];
        check_bits(it.bits);
        const uint64_t es = element_bytes(it.bits, complex_ != 0);
        it.a = off; off = up(off + mul64(mul64(it.m, it.k), es), kAlign);
        it.b = off; off = up(off + mul64(mul64(it.k, it.n), es), kAlign);
        it.c = off; off = up(off + mul64(mul64(it.m, it.n), es), kAlign);
    }
    if (lu4) {
        const Lu4Sizes n = lu4_elements(lu4->bits, lu4->shape);
        const uint64_t ces = element_bytes(lu4->bits, true);
        lu4->A = off; off = up(off + mul64(n.A, ces), kAlign);
        lu4->B = off; off = up(off + mul64(n.B, ces), kAlign);
        lu4->X = off; off = up(off + mul64(n.X, ces), kAlign);
        lu4->det = off; off = up(off + mul64(n.det, ces), kAlign);
        lu4->status = off; off = up(off + mul64(n.status, 4), kAlign);
    }
    *arena_bytes = off;
    LF_API_END
}

int lf_ragged_plan_create(lf_engine* e, int complex_, int fused, const lf_ragged_gemm* items, size_t count,
                          const lf_ragged_lu4* lu4, uint64_t arena_bytes, lf_ragged_plan** out) {
    LF_API_BEGIN
    if (!e || !out) throw invalid_argument("null argument");
    if (count && !items) throw invalid_argument("null instance list");
    if (count > 0x7fffffffull) throw invalid_argument("ragged batch: more than 2^31 instances");
    const bool cx = complex_ != 0;
    std::vector<Interval> outs, ins;
    std::vector<std::vector<size_t>> byclass(33);
    for (size_t i = 0; i < count; ++i) {
        const lf_ragged_gemm& it = items[i];
        check_bits(it.bits);
        if ((it.a | it.b | it.c) % 16) throw invalid_argument("ragged batch: operand offsets must be multiples of 16 bytes");
        const Extents x = extents(it, cx);
        for (const Interval& v : {x.a, x.b, x.c})
            if (v.hi < v.lo || v.hi > arena_bytes) throw invalid_argument("ragged batch: operand outside the arena");
        if (x.c.hi > x.c.lo) {                               // an accumulating C is read only by the cell that writes it
            outs.push_back(x.c);
            byclass[it.bits / 32].push_back(i);
        }
        if (x.a.hi > x.a.lo) ins.push_back(x.a);
        if (x.b.hi > x.b.lo) ins.push_back(x.b);
    }
    Lu4Sizes lun{};
    if (lu4) {
        lun = lu4_elements(lu4->bits, lu4->shape);
        const uint64_t ces = element_bytes(lu4->bits, true);
        if ((lu4->A | lu4->B | lu4->X | lu4->det | lu4->status) % 16) throw invalid_argument("ragged batch: operand offsets must be multiples of 16 bytes");
        auto span = [&](uint64_t off, uint64_t elems, uint64_t size) -> Interval {
            const Interval v{off, off + mul64(elems, size)};
            if (v.hi < v.lo || v.hi > arena_bytes) throw invalid_argument("ragged batch: operand outside the arena");
            return v;
        };
        const Interval A = span(lu4->A, lun.A, ces), B = span(lu4->B, lun.B, ces), X = span(lu4->X, lun.X, ces),
                       D = span(lu4->det, lun.det, ces), S = span(lu4->status, lun.status, 4);
        for (const Interval& v : {A, B}) if (v.hi > v.lo) ins.push_back(v);
        for (const Interval& v : {X, D, S}) if (v.hi > v.lo) outs.push_back(v);
    }
    // no output overlaps another output, nor an input
    std::sort(outs.begin(), outs.end(), [](const Interval& x, const Interval& y) { return x.lo < y.lo; });
    for (size_t i = 1; i < outs.size(); ++i)
        if (outs[i].lo < outs[i - 1].hi) throw invalid_argument("ragged batch: output matrices overlap");
    std::sort(ins.begin(), ins.end(), [](const Interval& x, const Interval& y) { return x.lo < y.lo; });
    std::vector<Interval> merged;
    for (const Interval& v : ins) {
        if (!merged.empty() && v.lo < merged.back().hi) merged.back().hi = std::max(merged.back().hi, v.hi);
        else merged.push_back(v);
    }
    for (const Interval& o : outs) {
        auto it = std::upper_bound(merged.begin(), merged.end(), o.lo, [](uint64_t x, const Interval& v) { return x < v.lo; });
        for (auto j = it == merged.begin() ? it : it - 1; j != merged.end() && j->lo < o.hi; ++j)
            if (j->lo < o.hi && o.lo < j->hi) throw invalid_argument("ragged batch: an output overlaps an input");
    }
    auto* p = new lf_ragged_plan();
    try {
        p->engine = e; p->cx = cx; p->fused = fused != 0; p->arena_bytes = arena_bytes;
        e->activate();
        cuda_check(cudaDeviceGetAttribute(&p->sms, cudaDevAttrMultiProcessorCount, e->device), "SM count");
        for (int limbs = 32; limbs >= 2; --limbs) {                    // widest (heaviest) class first
            const auto& idx = byclass[limbs];
            if (idx.empty()) continue;
            ClassPlan c;
            c.limbs = limbs;
            std::vector<size_t> order(idx);
            std::stable_sort(order.begin(), order.end(), [&](size_t x, size_t y) {
                const lf_ragged_gemm &a = items[x], &b = items[y];
                if (a.k != b.k) return a.k > b.k;
                return (uint64_t)a.m * a.n > (uint64_t)b.m * b.n;
            });
            uint64_t cell = 0;
            for (size_t i : order) {
                const lf_ragged_gemm& it = items[i];
                lfd::GemmItem g{it.a / 4, it.b / 4, it.c / 4, cell, it.m, it.n, it.k,
                                (it.accumulate ? 1u : 0u) | (it.negative ? 2u : 0u)};
                c.items.push_back(g);
                cell += (uint64_t)it.m * it.n;
            }
            c.items.push_back(lfd::GemmItem{0, 0, 0, cell, 0, 0, 0, 0});   // sentinel: the walk never passes it
            c.cells = cell;
            void* d = c.d_items.get(c.items.size() * sizeof(lfd::GemmItem));
            cuda_check(cudaMemcpy(d, c.items.data(), c.items.size() * sizeof(lfd::GemmItem), cudaMemcpyHostToDevice), "ragged items");
            cuda_check(cudaStreamSynchronize(0), "ragged items");
            p->classes.push_back(std::move(c));
        }
        if (lu4 && lu4->shape.count) { p->has_lu = true; p->lu = *lu4; p->lu_n = lun; }
        const size_t nstreams = p->classes.size() + (p->has_lu ? 1 : 0);
        for (size_t i = 0; i < std::max<size_t>(nstreams, 1); ++i) {
            cuda_check(cudaStreamCreateWithFlags(&p->streams[i], cudaStreamNonBlocking), "stream");
            cuda_check(cudaEventCreateWithFlags(&p->joins[i], cudaEventDisableTiming), "event");
        }
        cuda_check(cudaEventCreateWithFlags(&p->fork, cudaEventDisableTiming), "event");
        cuda_check(cudaEventCreateWithFlags(&p->done, cudaEventDisableTiming), "event");
        p->counters.get(4 * 33);
        for (auto& c : p->classes) {
            p->build_chunks(c, c.block, p->streams[0]);
            c.grid = p->class_grid(c, c.block);
        }
        if (p->has_lu) p->lu_grid = p->lu_grid_for(p->lu_block, false);
    } catch (...) {
        delete p;
        throw;
    }
    *out = p;
    LF_API_END
}

int lf_ragged_plan_tune(lf_ragged_plan* p, const void* arena) {
    LF_API_BEGIN
    if (!p) throw invalid_argument("null plan");
    if (p->classes.empty() && !p->has_lu) { p->tuned = true; return LF_OK; }
    if (!arena) throw invalid_argument("null arena");
    p->engine->activate();
    cudaStream_t s = p->streams[0];
    if (p->done_recorded) cuda_check(cudaStreamWaitEvent(s, p->done, 0), "ragged order");
    // scratch: the largest class's outputs, or the LU job's X, det and status
    uint64_t need = 16;
    for (auto& c : p->classes) need = std::max(need, c.cells * p->cell_words(c.limbs) * 4);
    if (p->has_lu) {
        const uint64_t ces = element_bytes(p->lu.bits, true);
        need = std::max(need, up(p->lu_n.X * ces, kAlign) + up(p->lu_n.det * ces, kAlign) + p->lu_n.status * 4 + 16);
    }
    p->scratch.get(need);
    cudaEvent_t t0, t1;
    cuda_check(cudaEventCreate(&t0), "event"); cuda_check(cudaEventCreate(&t1), "event");
    auto timed = [&](auto launch) {
        launch();                                                // warm-up
        cuda_check(cudaEventRecord(t0, s), "event");
        launch();
        cuda_check(cudaEventRecord(t1, s), "event");
        cuda_check(cudaEventSynchronize(t1), "ragged tune");
        float ms = 0; cudaEventElapsedTime(&ms, t0, t1);
        return (double)ms;
    };
    uint32_t* ctr = static_cast<uint32_t*>(p->counters.p);
    try {
        for (size_t ci = 0; ci < p->classes.size(); ++ci) {
            ClassPlan& c = p->classes[ci];
            double best = 1e300; unsigned best_b = c.block;
            for (unsigned b : kBlocks) {
                p->build_chunks(c, b, s);
                const unsigned grid = p->class_grid(c, b);
                const double ms = timed([&] {
                    cuda_check(cudaMemsetAsync(ctr + ci, 0, 4, s), "ragged counter");
                    lfd::gemm_launcher(c.limbs)(p->cx, p->fused, p->work(c, arena, ctr + ci, static_cast<uint32_t*>(p->scratch.p)), grid, b, s);
                    cuda_check(cudaGetLastError(), "ragged gemm launch");
                });
                if (ms < best) { best = ms; best_b = b; }
            }
            p->build_chunks(c, best_b, s);
            c.block = best_b; c.grid = p->class_grid(c, best_b); c.trial_ms = best;
        }
        if (p->has_lu) {
            double best = 1e300;
            for (unsigned b : kBlocks)
                for (int persistent = 0; persistent < 2; ++persistent) {
                    const unsigned grid = p->lu_grid_for(b, persistent != 0);
                    if (!grid) continue;
                    const double ms = timed([&] { p->launch_lu(arena, true, b, grid, s); });
                    if (ms < best) { best = ms; p->lu_block = b; p->lu_grid = grid; }
                }
            p->lu_trial_ms = best;
        }
    } catch (...) {
        cudaEventDestroy(t0); cudaEventDestroy(t1);
        throw;
    }
    cudaEventDestroy(t0); cudaEventDestroy(t1);
    p->tuned = true;
    if (p->exec) { cudaGraphExecDestroy(p->exec); p->exec = nullptr; p->graph_arena = nullptr; }
    LF_API_END
}

int lf_ragged_plan_run(lf_ragged_plan* p, void* arena, void* stream) {
    LF_API_BEGIN
    if (!p) throw invalid_argument("null plan");
    if (p->classes.empty() && !p->has_lu) return LF_OK;              // nothing to run
    if (!arena) throw invalid_argument("null arena");
    p->engine->activate();
    cudaStream_t user = static_cast<cudaStream_t>(stream);
    if (!p->exec || p->graph_arena != arena) {
        if (p->exec) { cudaGraphExecDestroy(p->exec); p->exec = nullptr; }
        cudaStream_t s0 = p->streams[0];
        cudaGraph_t g = nullptr;
        cuda_check(cudaStreamBeginCapture(s0, cudaStreamCaptureModeThreadLocal), "graph capture");
        try {
            uint32_t* ctr = static_cast<uint32_t*>(p->counters.p);
            if (!p->classes.empty()) cuda_check(cudaMemsetAsync(ctr, 0, 4 * p->classes.size(), s0), "ragged counters");
            cuda_check(cudaEventRecord(p->fork, s0), "fork");
            size_t branch = 0;
            auto on_branch = [&](auto launch) {
                cudaStream_t sb = p->streams[branch];
                if (branch) cuda_check(cudaStreamWaitEvent(sb, p->fork, 0), "fork");
                launch(sb);
                if (branch) cuda_check(cudaEventRecord(p->joins[branch], sb), "join");
                ++branch;
            };
            for (size_t ci = 0; ci < p->classes.size(); ++ci) {
                const ClassPlan& c = p->classes[ci];
                on_branch([&](cudaStream_t sb) {
                    lfd::gemm_launcher(c.limbs)(p->cx, p->fused, p->work(c, arena, ctr + ci, nullptr), c.grid, c.block, sb);
                    cuda_check(cudaGetLastError(), "ragged gemm launch");
                });
            }
            if (p->has_lu) on_branch([&](cudaStream_t sb) { p->launch_lu(arena, false, p->lu_block, p->lu_grid, sb); });
            for (size_t b = 1; b < branch; ++b) cuda_check(cudaStreamWaitEvent(s0, p->joins[b], 0), "join");
        } catch (...) {
            cudaStreamEndCapture(s0, &g);
            if (g) cudaGraphDestroy(g);
            throw;
        }
        cuda_check(cudaStreamEndCapture(s0, &g), "graph capture");
        cudaError_t r = cudaGraphInstantiate(&p->exec, g, 0);
        cudaGraphDestroy(g);
        cuda_check(r, "graph instantiate");
        p->graph_arena = arena;
    }
    if (p->done_recorded) cuda_check(cudaStreamWaitEvent(user, p->done, 0), "ragged order");
    cuda_check(cudaGraphLaunch(p->exec, user), "graph launch");
    cuda_check(cudaEventRecord(p->done, user), "ragged order");
    p->done_recorded = true;
    LF_API_END
}

int lf_ragged_plan_get_info(const lf_ragged_plan* p, lf_ragged_info* info) {
    LF_API_BEGIN
    if (!p || !info) throw invalid_argument("null argument");
    *info = lf_ragged_info{};
    info->classes = p->classes.size();
    for (size_t i = 0; i < p->classes.size(); ++i) {
        const ClassPlan& c = p->classes[i];
        info->cls[i] = lf_ragged_class_info{32 * c.limbs, c.items.size() - 1, c.cells, c.block, c.grid, c.trial_ms};
    }
    info->lu4_block = p->has_lu ? p->lu_block : 0; info->lu4_grid = p->has_lu ? p->lu_grid : 0;
    info->lu4_trial_ms = p->lu_trial_ms;
    info->tuned = p->tuned;
    LF_API_END
}

void lf_ragged_plan_destroy(lf_ragged_plan* p) {
    if (!p) return;
    if (p->done_recorded) cudaEventSynchronize(p->done);
    delete p;
}

}  // extern "C"
