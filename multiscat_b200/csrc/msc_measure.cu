// msc_measure.cu -- CUDA-core FMA peak of this GPU, measured in-tree.
//
// The channel coupling (and the SIMT block inverse) run on the CUDA cores'
// FMA pipes, so their roofline denominator is the FMA throughput the GPU
// reaches at its current clocks, not the HBM bandwidth.  This kernel issues
// nothing but independent fused multiply-adds (eight chains per thread, a
// full grid of resident warps per SM) and is timed with CUDA events on the
// caller's stream.  Measurement only; no counterpart in the reference.
#include <cuda_runtime.h>

#include "../../include/multiscat_b200.h"

namespace {

constexpr int kChains = 8;

__device__ double g_fma_sink[256];

template <typename R>
__global__ void __launch_bounds__(256) k_fma_peak(int iters, R a, R b)
{
    R x[kChains];
#pragma unroll
    for (int k = 0; k < kChains; ++k) x[k] = (R)(threadIdx.x + k) * (R)1e-3;
    for (int i = 0; i < iters; ++i) {
#pragma unroll
        for (int k = 0; k < kChains; ++k) x[k] = fma(x[k], a, b);
    }
    R acc = 0;
#pragma unroll
    for (int k = 0; k < kChains; ++k) acc += x[k];
    if (acc == (R)-12345.0) g_fma_sink[threadIdx.x] = (double)acc;   // never true; keeps the chains live
}

template <typename R>
msc_status run(int32_t iters, double *flops, float *ms, cudaStream_t st)
{
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return MSC_ERR_CUDA;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) return MSC_ERR_CUDA;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_fma_peak<R>, 256, 0) != cudaSuccess)
        return MSC_ERR_CUDA;
    const int grid = sms * (per_sm > 0 ? per_sm : 1);
    cudaEvent_t a, b;
    if (cudaEventCreate(&a) != cudaSuccess) return MSC_ERR_CUDA;
    if (cudaEventCreate(&b) != cudaSuccess) {
        cudaEventDestroy(a);
        return MSC_ERR_CUDA;
    }
    k_fma_peak<R><<<grid, 256, 0, st>>>(iters / 8 + 1, (R)0.999, (R)1e-4);   // warm-up
    cudaEventRecord(a, st);
    k_fma_peak<R><<<grid, 256, 0, st>>>(iters, (R)0.999, (R)1e-4);
    cudaEventRecord(b, st);
    cudaError_t e = cudaEventSynchronize(b);
    float t = 0.f;
    if (e == cudaSuccess) e = cudaEventElapsedTime(&t, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    if (e != cudaSuccess || cudaGetLastError() != cudaSuccess) return MSC_ERR_CUDA;
    *flops = 2.0 * kChains * (double)iters * grid * 256;
    *ms = t;
    return MSC_OK;
}

}  // namespace

extern "C" msc_status msc_measure_fma_peak(int32_t precision, int32_t iterations, double *flops,
                                           float *ms, void *stream)
{
    if (!flops || !ms || iterations <= 0) return MSC_ERR_ARG;
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (precision == MSC_PRECISION_FP64) return run<double>(iterations, flops, ms, st);
    if (precision == MSC_PRECISION_MIXED) return run<float>(iterations, flops, ms, st);
    return MSC_ERR_ARG;
}
