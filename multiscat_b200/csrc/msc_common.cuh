// msc_common.cuh -- shared helpers of the B200 close-coupling solver.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <cmath>

namespace msc {

// Complex arithmetic on interleaved pairs.
__host__ __device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__host__ __device__ __forceinline__ double2 cadd(double2 a, double2 b) {
    return make_double2(a.x + b.x, a.y + b.y);
}
__host__ __device__ __forceinline__ double2 csub(double2 a, double2 b) {
    return make_double2(a.x - b.x, a.y - b.y);
}
__host__ __device__ __forceinline__ double2 cconj(double2 a) { return make_double2(a.x, -a.y); }
__host__ __device__ __forceinline__ double cabs2(double2 a) { return a.x * a.x + a.y * a.y; }
__host__ __device__ __forceinline__ double2 cscale(double2 a, double s) {
    return make_double2(a.x * s, a.y * s);
}
// a / b with scaling (Smith's algorithm).
__host__ __device__ __forceinline__ double2 cdiv(double2 a, double2 b) {
    if (fabs(b.x) >= fabs(b.y)) {
        double r = b.y / b.x, d = b.x + b.y * r;
        return make_double2((a.x + a.y * r) / d, (a.y - a.x * r) / d);
    } else {
        double r = b.x / b.y, d = b.y + b.x * r;
        return make_double2((a.x * r + a.y) / d, (a.y * r - a.x) / d);
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// mbarriers and bulk copies (cp.async.bulk global -> shared, completion
// counted in bytes on an mbarrier), shared by the tcgen05 block inverse and
// the streamed Arnoldi reduction.
constexpr long long kSpinLimit = 1ll << 26;   // polls before a wait is declared hung

__device__ __forceinline__ uint32_t smem_u32(const void *p)
{
    return (uint32_t)__cvta_generic_to_shared(p);
}

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

__device__ __forceinline__ void mbar_fence_init()
{
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}

__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity)
{
    uint32_t ok;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(ok)
        : "r"(smem_u32(bar)), "r"(parity)
        : "memory");
    return ok != 0;
}

// Bounded wait: true when the phase completed, false after kSpinLimit polls.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity)
{
    for (long long i = 0; i < kSpinLimit; ++i)
        if (mbar_try_wait(bar, parity)) return true;
    return false;
}

__device__ __forceinline__ void bulk_g2s(void *smem_dst, const void *gsrc, uint32_t bytes, uint64_t *bar)
{
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
            smem_u32(smem_dst)),
        "l"(gsrc), "r"(bytes), "r"(smem_u32(bar))
        : "memory");
}

__device__ __forceinline__ void fence_proxy_async()
{
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Row tiles: every tile holds up to kTileRows consecutive channel rows of
// ONE system, so per-tile partial reductions add up per system.
constexpr int kTileRows = 8;
constexpr int kMaxNz = 1024;
constexpr int kWideNz = 512;   // above this the block inverse stages 4 rows per pass
constexpr int kMaxRestart = 64;
constexpr int kMaxTaps = 2048;

struct Tiles {
    const int *row0;   // first row of the tile
    const int *nrow;   // rows in the tile (1..kTileRows)
    const int *sys;    // system of the tile
    int count;
};

}  // namespace msc
