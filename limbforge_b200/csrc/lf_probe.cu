// Measurement helper with no reference counterpart: the rate at which one GPU forms 32 x 32 -> 64-bit word
// products with a 64-bit addend (the step of every limb kernel's schoolbook product), the denominator of the
// integer-pipe roofline that bench.py reports beside the HBM one.  Every thread runs eight independent
// multiply-add chains, acc <- hi(acc) * y + acc (one wide integer multiply-add each, loop-carried, so nothing
// can be hoisted), on a grid that fills every SM; the rate is timed with CUDA events over several launches.
#include <algorithm>
#include "lf_runtime.h"

namespace {

constexpr int kProbeChains = 8;
constexpr int kProbeThreads = 256;

__global__ void __launch_bounds__(kProbeThreads) word_mac_probe(const uint32_t* seed, uint64_t* out, int iters) {
    uint64_t acc[kProbeChains];
    uint32_t y[kProbeChains];
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) {
        acc[k] = ((uint64_t)seed[(threadIdx.x + k) & 31] << 32) | (blockIdx.x + k);
        y[k] = seed[(threadIdx.x + 3 * k + 1) & 31] | 1u;
    }
#pragma unroll 1
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int r = 0; r < 4; ++r) {
#pragma unroll
            for (int k = 0; k < kProbeChains; ++k) acc[k] = (uint64_t)(uint32_t)(acc[k] >> 32) * y[k] + acc[k];
        }
    }
    uint64_t s = 0;
#pragma unroll
    for (int k = 0; k < kProbeChains; ++k) s ^= acc[k];
    out[(size_t)blockIdx.x * kProbeThreads + threadIdx.x] = s;
}

}  // namespace

using namespace lfr;

extern "C" int lf_probe_word_mac_rate(int device, double* word_macs_per_s) {
    LF_API_BEGIN
    if (!word_macs_per_s) throw invalid_argument("null argument");
    cuda_check(cudaSetDevice(device), "cudaSetDevice");
    int sms = 0, per_sm = 0;
    cuda_check(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device), "SM count");
    cuda_check(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, word_mac_probe, kProbeThreads, 0), "occupancy");
    const unsigned grid = (unsigned)(sms * std::max(per_sm, 1));
    const int iters = 2048;
    DevBuf seed, out;
    seed.get(32 * 4);
    out.get((size_t)grid * kProbeThreads * 8);
    uint32_t h[32];
    for (int i = 0; i < 32; ++i) h[i] = 0x9e3779b9u * (uint32_t)(i + 1);
    cuda_check(cudaMemcpy(seed.p, h, sizeof h, cudaMemcpyHostToDevice), "probe seed");
    cudaStream_t s = nullptr;
    cudaEvent_t e0, e1;
    cuda_check(cudaEventCreate(&e0), "event");
    cuda_check(cudaEventCreate(&e1), "event");
    const auto launch = [&] { word_mac_probe<<<grid, kProbeThreads, 0, s>>>(static_cast<const uint32_t*>(seed.p), static_cast<uint64_t*>(out.p), iters); };
    for (int w = 0; w < 3; ++w) launch();
    const int reps = 10;
    cuda_check(cudaEventRecord(e0, s), "event");
    for (int r = 0; r < reps; ++r) launch();
    cuda_check(cudaEventRecord(e1, s), "event");
    cuda_check(cudaEventSynchronize(e1), "probe");
    cuda_check(cudaGetLastError(), "probe launch");
    float ms = 0;
    cuda_check(cudaEventElapsedTime(&ms, e0, e1), "event time");
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    const double macs = (double)reps * grid * kProbeThreads * (double)iters * 4.0 * kProbeChains;
    *word_macs_per_s = macs / (ms * 1e-3);
    LF_API_END
}
