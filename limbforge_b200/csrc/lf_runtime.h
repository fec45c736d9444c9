// Internal runtime objects behind the C ABI (engine, buffers, batches, submissions).
#pragma once
#include "limbforge_b200.h"
#include <cuda_runtime.h>
#include <atomic>
#include <chrono>
#include <cstdint>
#include <cstring>
#include <functional>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

namespace lfr {

struct invalid_argument : std::invalid_argument { using std::invalid_argument::invalid_argument; };
struct logic_error : std::logic_error { using std::logic_error::logic_error; };
struct runtime_error : std::runtime_error { using std::runtime_error::runtime_error; };

void set_error(const std::string& message);
void cuda_check(cudaError_t e, const char* what);

inline void validate(int bits, size_t count) {
    if (bits < 64 || bits > 1024 || bits % 32) throw invalid_argument("bits must be a multiple of 32 in [64,1024]");
    if (count > 0xffffffffull) throw invalid_argument("batch exceeds 32-bit indexing");
}
inline size_t checked_size(size_t count, size_t stride) {
    if (stride && count > SIZE_MAX / stride) throw invalid_argument("buffer size overflow");
    return count * stride;
}
inline size_t broadcast_elements(size_t count, lf_broadcast b) {                        // engine.hpp:22-25
    if (!b.stride) throw invalid_argument("broadcast stride must be positive");
    size_t n = count / b.stride + (count % b.stride != 0);
    return b.period && b.period < n ? b.period : n;
}
inline bool op_complex(int op) { return (op >= 4 && op <= 6) || op == 11 || op == 12; }
inline bool op_unary(int op) { return op == 7 || op == 8; }
inline bool op_ternary(int op) { return op >= 9 && op <= 12; }
inline bool op_valid(int op) { return op >= 0 && op <= 12; }
inline size_t element_bytes(int bits, bool complex) { return size_t(bits / 8 + 12) * (complex ? 2 : 1); }

// Grow-only device allocation owned by one engine (scratch for host-array calls).
struct DevBuf {
    void* p = nullptr; size_t bytes = 0;
    DevBuf() = default;
    DevBuf(const DevBuf&) = delete;
    DevBuf& operator=(const DevBuf&) = delete;
    DevBuf(DevBuf&& o) noexcept : p(o.p), bytes(o.bytes) { o.p = nullptr; o.bytes = 0; }
    DevBuf& operator=(DevBuf&& o) noexcept {
        if (this != &o) { if (p) cudaFree(p); p = o.p; bytes = o.bytes; o.p = nullptr; o.bytes = 0; }
        return *this;
    }
    void* get(size_t n) {
        if (n > bytes) {
            if (p) cudaFree(p);
            p = nullptr; bytes = 0;
            cuda_check(cudaMalloc(&p, n ? n : 16), "device allocation");
            bytes = n;
        }
        return p;
    }
    ~DevBuf() { if (p) cudaFree(p); }
};
// Pinned host staging that grows on demand (host-array calls that pipeline their transfers).
struct PinnedBuf {
    void* p = nullptr; size_t bytes = 0;
    PinnedBuf() = default;
    PinnedBuf(const PinnedBuf&) = delete;
    PinnedBuf& operator=(const PinnedBuf&) = delete;
    void* get(size_t n) {
        if (n > bytes) {
            if (p) cudaFreeHost(p);
            p = nullptr; bytes = 0;
            cuda_check(cudaMallocHost(&p, n ? n : 16), "pinned staging allocation");
            bytes = n;
        }
        return p;
    }
    ~PinnedBuf() { if (p) cudaFreeHost(p); }
};

struct Engine {
    int device = 0;
    uint64_t identity = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    DevBuf scratch[6];
    PinnedBuf staging[2];
    std::string name;
    lf_engine_options options{};
    void activate() const { cuda_check(cudaSetDevice(device), "cudaSetDevice"); }
};

// Device storage of a Buffer<T>.  The device copy is authoritative except after mapped(),
// which hands out a host mirror; the next submission (or upload/download) that uses the
// buffer brings the device copy up to date.
struct Buffer {
    std::atomic<int> refs{1};
    uint64_t owner = 0; int device = 0;
    void* dev = nullptr; size_t bytes = 0;
    void* host = nullptr;
    bool host_authoritative = false;
    std::atomic<bool> busy{false};
    ~Buffer() { if (dev) cudaFree(dev); if (host) cudaFreeHost(host); }
    void sync_to_device(cudaStream_t s) {
        if (host_authoritative && bytes) cuda_check(cudaMemcpyAsync(dev, host, bytes, cudaMemcpyHostToDevice, s), "host mirror upload");
        host_authoritative = false;
    }
};

enum OpKind { kElementwise = 0, kLu4 = 1, kStridedGemm = 2, kCustom = 3 };
struct Op {
    int kind = kElementwise; int bits = 0; int op = 0; bool complex = false;
    Buffer* a = nullptr; Buffer* b = nullptr; Buffer* c = nullptr; Buffer* out = nullptr; Buffer* e = nullptr;
    size_t count = 0; lf_broadcast bi{1, 0}, ci{1, 0};
    lf_batched4 lu{}; lf_strided_gemm sg{};
    std::function<void(cudaStream_t)> custom;
};

struct Batch {
    Engine* engine = nullptr;
    std::vector<Op> ops;
    std::vector<Buffer*> resources;   // each retained once
    std::vector<Buffer*> written;
    std::vector<std::shared_ptr<void>> keep;   // objects the recorded operations use, freed when the submission completes
    bool submitted = false;
    void retain(Buffer* r, bool write = false);
    ~Batch();
};

struct Submission {
    Engine* engine = nullptr;
    cudaEvent_t start = nullptr, end = nullptr;
    std::vector<Buffer*> resources;
    std::vector<std::shared_ptr<void>> keep;
    bool done = false; std::string error;
    lf_timing timing{0, 0};
    std::chrono::steady_clock::time_point wall0;
    void finish();
    ~Submission();
};

// Kernel launch entry points shared by host-array calls, batches and the device-pointer ABI.
void launch_elementwise(int bits, int op, const void* a, const void* b, const void* c, void* out, size_t count,
                        lf_broadcast bi, lf_broadcast ci, cudaStream_t s);
void launch_lu4(int bits, const lf_batched4& shape, const void* A, const void* B, void* X, void* det, uint32_t* status,
                cudaStream_t s);
void launch_strided_gemm(int bits, bool complex, const lf_strided_gemm& s, const void* A, const void* B, void* C,
                         cudaStream_t st);
// Element counts of the operands of a batched 4x4 job (A, B, X, det, status), validated as
// Engine::lu4 validates them (engine.mm lu4_elements).
struct Lu4Sizes { size_t A, B, X, det, status; };
Lu4Sizes lu4_elements(int bits, const lf_batched4& s);

}  // namespace lfr

#define LF_API_BEGIN try {
#define LF_API_END                                                             \
    return LF_OK;                                                              \
    } catch (const lfr::invalid_argument& e) { lfr::set_error(e.what()); return LF_INVALID_ARGUMENT; } \
    catch (const std::invalid_argument& e) { lfr::set_error(e.what()); return LF_INVALID_ARGUMENT; }   \
    catch (const std::logic_error& e) { lfr::set_error(e.what()); return LF_LOGIC_ERROR; }             \
    catch (const std::exception& e) { lfr::set_error(e.what()); return LF_RUNTIME_ERROR; }             \
    catch (...) { lfr::set_error("unknown error"); return LF_RUNTIME_ERROR; }
