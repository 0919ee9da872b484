// FP32 FMA-pipe throughput probe: the measured FP32 peak used as the roofline denominator of
// the fit kernels (they run on the FP32/MUFU pipes, not on tensor cores or at the HBM bound).
// Each thread runs 8 independent FMA chains; nothing touches memory until the final store.
#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/photonpy_b200.h"

namespace {
__global__ void __launch_bounds__(256) fma_probe_kernel(int iters, float a, float b, float* out) {
    float x0 = threadIdx.x * 1e-7f, x1 = x0 + 1e-7f, x2 = x0 + 2e-7f, x3 = x0 + 3e-7f;
    float x4 = x0 + 4e-7f, x5 = x0 + 5e-7f, x6 = x0 + 6e-7f, x7 = x0 + 7e-7f;
    for (int i = 0; i < iters; i++) {
#pragma unroll
        for (int u = 0; u < 16; u++) {
            x0 = fmaf(x0, a, b); x1 = fmaf(x1, a, b); x2 = fmaf(x2, a, b); x3 = fmaf(x3, a, b);
            x4 = fmaf(x4, a, b); x5 = fmaf(x5, a, b); x6 = fmaf(x6, a, b); x7 = fmaf(x7, a, b);
        }
    }
    const float s = ((x0 + x1) + (x2 + x3)) + ((x4 + x5) + (x6 + x7));
    if (s == 1.2345f) out[blockIdx.x] = s;  // practically never true; keeps the chains alive
}
}  // namespace

extern "C" double PB200_Fp32ProbeLaunch(int blocks, int threads, int iters, float* d_out, void* stream) {
    fma_probe_kernel<<<blocks, threads, 0, (cudaStream_t)stream>>>(iters, 0.9999999f, 1e-7f, d_out);
    if (cudaGetLastError() != cudaSuccess) return -1.0;
    return 2.0 * 8.0 * 16.0 * (double)iters * (double)blocks * (double)threads;  // FLOPs issued
}
