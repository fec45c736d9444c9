// Import of complex values whose MPFR significands live inside one caller allocation (the reference's
// BatchedLinalg::import_inline_complex, batched_linalg.hpp:53-60,146-148; batched_linalg.mm:234-248;
// batched_linalg.metal:108-117).  The allocation is copied to the device once, in the submission's stream order, and
// one thread per complex element gathers both parts: a part with a status or a zero sign is zero (with that status);
// otherwise its N words are the top N 32-bit words of ceil(N/2) little-endian 64-bit MPFR limbs at the record's
// offset, with the record's exponent and sign, and an exponent outside [-1e9, 1e9] gives exponent_overflow.
#include "lf_runtime.h"

#include <unistd.h>
#include <array>
#include <memory>
#include <utility>
#include <vector>

namespace {
typedef uint32_t u32;
typedef uint64_t u64;

template <int N> __device__ void import_part(const unsigned char* bytes, u64 offset, int exponent, int sign, u32 status, u32* out) {
    if (status || !sign) {
        for (int j = 0; j < N + 3; ++j) out[j] = 0;
        out[N + 2] = status;
        return;
    }
    if (exponent > 1000000000 || exponent < -1000000000) {
        for (int j = 0; j < N + 3; ++j) out[j] = 0;
        out[N + 2] = 2u;
        return;
    }
    const u32* s = reinterpret_cast<const u32*>(bytes + offset) + (N % 2);   // odd widths: one low padding word
    for (int j = 0; j < N; ++j) out[j] = s[j];
    out[N] = static_cast<u32>(exponent);
    out[N + 1] = static_cast<u32>(sign);
    out[N + 2] = 0;
}

template <int N> __global__ void __launch_bounds__(128) inline_complex_kernel(const unsigned char* bytes, const lf_inline_complex_record* r,
                                                                              u32* out, u64 count) {
    const u64 i = static_cast<u64>(blockIdx.x) * blockDim.x + threadIdx.x;
    if (i >= count) return;
    const lf_inline_complex_record d = r[i];
    u32* o = out + i * 2 * (N + 3);
    import_part<N>(bytes, d.real_offset, d.real_exponent, d.real_sign, d.real_status, o);
    import_part<N>(bytes, d.imag_offset, d.imag_exponent, d.imag_sign, d.imag_status, o + N + 3);
}

typedef void (*InlineLaunch)(const unsigned char*, const lf_inline_complex_record*, u32*, u64, cudaStream_t);
template <int N> void inline_launch(const unsigned char* b, const lf_inline_complex_record* r, u32* o, u64 n, cudaStream_t s) {
    inline_complex_kernel<N><<<static_cast<unsigned>((n + 127) / 128), 128, 0, s>>>(b, r, o, n);
}
template <int... I> constexpr auto inline_table(std::integer_sequence<int, I...>) {
    return std::array<InlineLaunch, sizeof...(I)>{inline_launch<I + 2>...};
}
const auto kInlineLaunch = inline_table(std::make_integer_sequence<int, 31>{});

// Device copies of one import: the allocation and the records, freed when the submission completes.
struct InlineStage {
    void* bytes = nullptr; void* records = nullptr;
    ~InlineStage() { if (bytes) cudaFree(bytes); if (records) cudaFree(records); }
};
}  // namespace

using namespace lfr;
struct lf_buffer : Buffer {};
struct lf_batch : Batch {};

extern "C" {

int lf_batch_import_inline_complex(lf_batch* bt, int bits, const void* allocation, size_t bytes, const lf_inline_complex_record* records,
                                   size_t count, lf_buffer* out) {
    LF_API_BEGIN
    if (!bt || bt->submitted) throw logic_error("batch already submitted or moved");
    validate(bits, count);
    if (count > 0xffffffffull) throw invalid_argument("inline staging: grid exceeds 32 bits");
    if (!out) throw invalid_argument("missing inline staging output");
    if (out->bytes < checked_size(count, element_bytes(bits, true))) throw invalid_argument("inline staging: undersized buffer");
    if (!count) { bt->retain(out, true); return LF_OK; }
    const size_t page = static_cast<size_t>(sysconf(_SC_PAGESIZE));
    if (!allocation || reinterpret_cast<uintptr_t>(allocation) % page || !bytes || bytes % page || !records)
        throw invalid_argument("inline staging: allocation must own complete aligned pages");
    const size_t source = 8 * ((static_cast<size_t>(bits) + 63) / 64);
    for (size_t i = 0; i < count; ++i)
        for (uint64_t off : {records[i].real_offset, records[i].imag_offset})
            if (off % 8 || off > bytes || source > bytes - off)
                throw invalid_argument("inline staging: significand out of bounds or unaligned");
    bt->retain(out, true);
    auto stage = std::make_shared<InlineStage>();
    bt->engine->activate();
    cuda_check(cudaMalloc(&stage->bytes, bytes), "inline staging allocation");
    cuda_check(cudaMalloc(&stage->records, count * sizeof(lf_inline_complex_record)), "inline staging allocation");
    // the records are taken now; the allocation is read when the batch runs, so it must stay unchanged until then
    auto meta = std::make_shared<std::vector<lf_inline_complex_record>>(records, records + count);
    bt->keep.push_back(stage);
    bt->keep.push_back(meta);
    Op o;
    o.kind = kCustom;
    const int limbs = bits / 32;
    Buffer* z = out;
    o.custom = [=](cudaStream_t s) {
        cuda_check(cudaMemcpyAsync(stage->bytes, allocation, bytes, cudaMemcpyHostToDevice, s), "inline staging upload");
        cuda_check(cudaMemcpyAsync(stage->records, meta->data(), count * sizeof(lf_inline_complex_record), cudaMemcpyHostToDevice, s),
                   "inline staging upload");
        kInlineLaunch[limbs - 2](static_cast<const unsigned char*>(stage->bytes), static_cast<const lf_inline_complex_record*>(stage->records),
                                 static_cast<u32*>(z->dev), count, s);
        cuda_check(cudaGetLastError(), "inline staging launch");
    };
    bt->ops.push_back(o);
    LF_API_END
}

}  // extern "C"
