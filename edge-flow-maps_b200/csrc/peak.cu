// FP32 FMA throughput probe: the denominator of the FP32 roofline fraction
// reported for the interpolation kernels (the march, the face maps), which
// are bound by SIMT FMA issue rather than by HBM.
#include <cuda_runtime.h>

#include "edge_b200.h"

namespace {

// eight independent FMA chains per thread keep every FMA pipe busy
__global__ void __launch_bounds__(256) k_fma_peak(float* out, int iters, float a, float b) {
    float x[8];
#pragma unroll
    for (int q = 0; q < 8; q++) x[q] = (float)(threadIdx.x + q) * 1e-7f;
    for (int it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 16; r++)
#pragma unroll
            for (int q = 0; q < 8; q++) x[q] = fmaf(x[q], a, b);
    }
    float s = 0.0f;
#pragma unroll
    for (int q = 0; q < 8; q++) s += x[q];
    if (s == 12345.678f) out[0] = s;  // keeps the chains alive; never taken for these inputs
}

}  // namespace

extern "C" int edge_fma_peak(int blocks, int iters, float* out, double* flops, void* stream) {
    if (blocks <= 0 || iters <= 0 || !out || !flops) return EDGE_EINVAL;
    k_fma_peak<<<blocks, 256, 0, (cudaStream_t)stream>>>(out, iters, 0.999999f, 1e-7f);
    *flops = 2.0 * 8 * 16 * (double)iters * 256.0 * blocks;
    cudaError_t e = cudaPeekAtLastError();
    return e == cudaSuccess ? EDGE_OK : (int)e;
}
