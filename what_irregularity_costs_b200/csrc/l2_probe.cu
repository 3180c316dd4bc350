// Measured L2 ceilings of the GPU the library runs on: the denominators of
// the roofline fractions of the kernels whose working set stays in L2 (the
// band walk's per-voxel reductions, finish's tiles of touched blocks).
//
// No counterpart in the reference, which measures its kernels against
// nothing but their own durations (cpp/bench/bench_arms.cu). Each probe is
// one kernel over a device buffer of the requested size (L2-resident when
// well below the 126 MB L2), a persistent grid of 8 x 256-thread CTAs per
// SM, timed with CUDA events after one warm-up launch:
//
//   kind 0  red.global.add.u64 to pseudo-random 8-byte words (no return):
//           the band walk's fixed-point sums;          result: G ops/s
//   kind 1  red.global.add.u32 to pseudo-random 4-byte words:
//           the band walk's counts;                    result: G ops/s
//   kind 2  atom.global.add.u32 with return to pseudo-random words:
//           the group pass's place tickets;            result: G ops/s
//   kind 3  16-byte loads through L2 (ld.global.cg), streamed over the
//           buffer again and again: tile reads;       result: GB/s
//   kind 4  4-byte loads through L2 at pseudo-random words: the walk's
//           weight gathers and table probes;          result: G loads/s
#include <cstdio>

#include "../../include/osn_tsdf_b200.h"

namespace {

constexpr int kProbeThreads = 256;
constexpr int kProbeCtasPerSm = 8;

// A counter-based word index: splitmix64 of (thread, iteration), so every
// thread visits a different pseudo-random sequence spread over the buffer.
__device__ __forceinline__ unsigned long long mix(unsigned long long x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

template <int KIND>
__global__ void __launch_bounds__(kProbeThreads)
l2_probe_kernel(void* buf, unsigned long long n_words, int iters, unsigned* sink) {
    const unsigned long long tid = blockIdx.x * (unsigned long long)blockDim.x + threadIdx.x;
    const unsigned long long nthreads = (unsigned long long)gridDim.x * blockDim.x;
    unsigned acc = 0u;
    if (KIND == 3) {
        // Streamed 16-byte loads: consecutive threads read consecutive vectors.
        const uint4* v = static_cast<const uint4*>(buf);
        const unsigned long long n_vec = n_words / 2;  // words are 8 bytes here
        const unsigned long long step = nthreads % n_vec;
        unsigned long long i = tid % n_vec;
        for (int it = 0; it < iters; ++it) {
            const uint4 x = __ldcg(v + i);
            acc ^= x.x ^ x.y ^ x.z ^ x.w;
            i += step;  // i, step < n_vec
            if (i >= n_vec) i -= n_vec;
        }
    } else {
        unsigned long long h = mix(tid);
        for (int it = 0; it < iters; ++it) {
            h = mix(h);
            const unsigned long long w = h % n_words;
            if (KIND == 0) {
                asm volatile("red.global.add.u64 [%0], %1;" ::"l"(static_cast<unsigned long long*>(buf) + w),
                             "l"(1ull));
            } else if (KIND == 1) {
                asm volatile("red.global.add.u32 [%0], %1;" ::"l"(static_cast<unsigned*>(buf) + w), "r"(1u));
            } else if (KIND == 2) {
                acc += atomicAdd(static_cast<unsigned*>(buf) + w, 1u);
            } else {
                acc += __ldcg(static_cast<const unsigned*>(buf) + w);
            }
        }
    }
    if (acc == 0x12345678u) atomicAdd(sink, 1u);  // keeps the loads and returns live
}

template <int KIND>
cudaError_t run_probe(void* buf, unsigned long long n_words, int iters, int grid, unsigned* sink,
                      cudaStream_t s) {
    l2_probe_kernel<KIND><<<grid, kProbeThreads, 0, s>>>(buf, n_words, iters, sink);
    return cudaGetLastError();
}

cudaError_t launch_probe(int kind, void* buf, unsigned long long n_words, int iters, int grid, unsigned* sink,
                         cudaStream_t s) {
    switch (kind) {
        case 0: return run_probe<0>(buf, n_words, iters, grid, sink, s);
        case 1: return run_probe<1>(buf, n_words, iters, grid, sink, s);
        case 2: return run_probe<2>(buf, n_words, iters, grid, sink, s);
        case 3: return run_probe<3>(buf, n_words, iters, grid, sink, s);
        case 4: return run_probe<4>(buf, n_words, iters, grid, sink, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

extern "C" int32_t osn_tsdf_cuda_l2_probe(int32_t kind, int64_t bytes, int32_t iters, double* result) {
    if (kind < 0 || kind > 4 || bytes < (1 << 20) || bytes > (int64_t(1) << 31) || iters < 1 ||
        iters > (1 << 16) || !result)
        return 1;
    int dev = 0, sms = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
        return 3;
    // Words of 8 bytes for the 64-bit probe and the streamed loads, 4 bytes otherwise.
    const unsigned long long word = (kind == 0 || kind == 3) ? 8ull : 4ull;
    const unsigned long long n_words = (unsigned long long)bytes / word;
    void* buf = nullptr;
    unsigned* sink = nullptr;
    cudaStream_t s = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    int32_t rc = 3;
    const int grid = sms * kProbeCtasPerSm;
    if (cudaMalloc(&buf, (size_t)bytes) == cudaSuccess && cudaMalloc(&sink, sizeof(unsigned)) == cudaSuccess &&
        cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) == cudaSuccess &&
        cudaEventCreate(&e0) == cudaSuccess && cudaEventCreate(&e1) == cudaSuccess &&
        cudaMemsetAsync(buf, 0, (size_t)bytes, s) == cudaSuccess &&
        launch_probe(kind, buf, n_words, iters, grid, sink, s) == cudaSuccess &&  // warm-up
        cudaEventRecord(e0, s) == cudaSuccess &&
        launch_probe(kind, buf, n_words, iters, grid, sink, s) == cudaSuccess &&
        cudaEventRecord(e1, s) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess) {
        float ms = 0.0f;
        if (cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess && ms > 0.0f) {
            const double ops = (double)grid * kProbeThreads * iters;
            // G ops/s, or GB/s for the streamed 16-byte loads.
            *result = (kind == 3 ? ops * 16.0 : ops) / (ms * 1e-3) / 1e9;
            rc = 0;
        }
    }
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    if (s) cudaStreamDestroy(s);
    cudaFree(sink);
    cudaFree(buf);
    return rc;
}
