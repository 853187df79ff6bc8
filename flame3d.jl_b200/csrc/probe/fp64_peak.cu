// fp64_peak.cu — measured FP64 FMA throughput of the GPU, the compute roof of the plain FP64
// stage (whose kernels are bound by FP64 issue, not by HBM).  Built into libflame3d_probe.so,
// apart from the reference-facing library; bench.py times it with CUDA events.
//
// Every thread runs kChains independent fused multiply-add chains (enough independent work to
// cover the FP64 pipe latency) for `iters` rounds; the chains contract towards a fixed point,
// so the values stay finite and the compiler cannot drop the loop (the sum is stored).
#include <cuda_runtime.h>

namespace {

constexpr int kChains = 8;

__global__ void __launch_bounds__(256) k_fp64_fma(int iters, double a, double b, double *out) {
    double x[kChains];
#pragma unroll
    for (int c = 0; c < kChains; ++c) x[c] = threadIdx.x * 1e-3 + c;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int c = 0; c < kChains; ++c) x[c] = fma(x[c], a, b);
    }
    double s = 0;
#pragma unroll
    for (int c = 0; c < kChains; ++c) s += x[c];
    out[blockIdx.x * blockDim.x + threadIdx.x] = s;
}

}  // namespace

// Launches blocks x 256 threads, each doing kChains * iters FMAs, on `stream`; out must hold
// blocks * 256 doubles.  Returns the FLOPs issued (2 per FMA), or -1 on a launch error.
extern "C" double flame_probe_fp64_fma(int blocks, int iters, double *out, cudaStream_t stream) {
    k_fp64_fma<<<blocks, 256, 0, stream>>>(iters, 0.999999, 1e-6, out);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    return 2.0 * kChains * (double)iters * blocks * 256;
}
