// msc_tc.cuh -- tcgen05 (5th-generation tensor core) block-diagonal inverse
// for the FP32 inner solve of the mixed form.
//
//   u = D^-1 x  per channel:  xt = E^T x ;  yt = (xt + beta e_n)/(pkd + lam) ;  u = E yt
//
// Both products are real GEMMs with M = n (nodes), K = n, N = 2 * channels
// (re/im columns).  They run as BF16x3 split products on tcgen05:
//   A B ~= A_hi B_hi + A_hi B_lo + A_lo B_hi      (FP32 accumulate in TMEM)
// where v_hi = bf16(v), v_lo = bf16(v - v_hi), which keeps ~16 bits of the
// FP32 operands.
//
// Layout.  The eigenvector matrix E (zero padded to Kp x Kp, Kp = n rounded
// up to 16) is stored once in shared memory as 8x8 core matrices (128 bytes:
// 8 rows of z, each with 8 consecutive k).  The same bytes are
//   - the K-major A operand of u = E yt        (M = z, K = k), and
//   - the MN-major A operand of xt = E^T x     (M = k, K = z),
// so one copy of E_hi and E_lo serves both GEMMs.  The image is prepared on
// the host in exactly this order and brought in with cp.async.bulk once per
// CTA.  The B operands (x, then yt) are staged per tile of channels by the
// threads themselves (FP32 -> BF16 hi/lo, re/im de-interleaved).
//
// Execution.  Persistent CTAs (one per SM, 256 threads = 8 warps).  Per tile:
// stage B, one thread issues the MMAs and commits to an mbarrier, all warps
// read the accumulator with tcgen05.ld (warp w owns TMEM lanes
// 32 (w % 4)..32 (w % 4) + 31 and the column half w / 4),
// form the Sherman-Morrison scalars and yt (pkd + lam in FP64), stage yt as
// the next B operand, second GEMM, store u.  Every mbarrier wait is bounded;
// on time-out the kernel records an error code, stops issuing work and still
// releases its TMEM.
#pragma once

#include <cuda_bf16.h>

#include "msc_common.cuh"

namespace msc {
namespace tc {

constexpr int kThreads = 256;   // 8 warps: warp w reads TMEM lanes 32 (w % 4).., columns half w / 4
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

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory"); }

__device__ __forceinline__ void tmem_alloc(uint32_t *smem_dst, uint32_t ncols)
{
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(smem_dst)),
                 "r"(ncols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}

__device__ __forceinline__ void tmem_dealloc(uint32_t taddr, uint32_t ncols)
{
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(taddr), "r"(ncols) : "memory");
}

// D[tmem] (+)= A[smem] * B[smem], kind::f16 (BF16 in, FP32 accumulate).
__device__ __forceinline__ void mma_bf16(uint32_t d_tmem, uint64_t a_desc, uint64_t b_desc, uint32_t idesc,
                                         uint32_t accumulate)
{
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "setp.ne.b32 p, %4, 0;\n\t"
        "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}" ::"r"(d_tmem),
        "l"(a_desc), "l"(b_desc), "r"(idesc), "r"(accumulate), "r"(0u), "r"(0u), "r"(0u), "r"(0u)
        : "memory");
}

__device__ __forceinline__ void mma_commit(uint64_t *bar)
{
    asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                     smem_u32(bar))
                 : "memory");
}

// 32 lanes x 16 consecutive 32-bit columns.
__device__ __forceinline__ void tmem_ld16(uint32_t taddr, float *v)
{
    uint32_t r[16];
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// Shared-memory matrix descriptor (no swizzle, canonical 8x16-byte core matrices).
__device__ __forceinline__ uint64_t make_desc(uint32_t saddr, uint32_t lbo_bytes, uint32_t sbo_bytes)
{
    uint64_t d = 0;
    d |= (uint64_t)((saddr & 0x3FFFFu) >> 4);
    d |= (uint64_t)((lbo_bytes >> 4) & 0x3FFFu) << 16;
    d |= (uint64_t)((sbo_bytes >> 4) & 0x3FFFu) << 32;
    d |= (uint64_t)1 << 46;            // descriptor version for sm_100
    // base offset 0, absolute LBO mode 0, layout type 0 (no swizzle)
    return d;
}

// Instruction descriptor: BF16 x BF16 -> FP32, M = 128, given N and A major-ness.
__host__ __device__ constexpr uint32_t make_idesc(int n, int a_mn_major)
{
    return (1u << 4)                         // D format F32
           | (1u << 7)                       // A format BF16
           | (1u << 10)                      // B format BF16
           | ((uint32_t)a_mn_major << 15)    // A major: 0 K-major, 1 MN-major
           | (0u << 16)                      // B K-major
           | ((uint32_t)(n >> 3) << 17)      // N / 8
           | ((uint32_t)(128 >> 4) << 24);   // M / 16
}

struct TcParams {
    int n;             // nodes
    int kp;            // n rounded up to 16 (E padded to kp x kp)
    int mt;            // M tiles of 128 (ceil(n / 128))
    int rows;          // total channel rows R
    int tile_rows;     // channels per tile (N / 2)
    int ntiles;        // ceil(R / tile_rows)
    const __nv_bfloat16 *e_img;   // [2][kp/8][kp/8][8][8]  hi part then lo part
    const double *lam, *en, *row_pkd, *row_fn;
    const double2 *row_c;
    const int *row_sys;           // [R]
    const int *gate;              // [B] or null
    const float2 *x;
    float2 *out;
    int *error;                   // set to a nonzero code on a time-out
};

// Offsets (bytes) of element (row c, k) of a K-major operand with `rows` rows.
__device__ __forceinline__ uint32_t kmaj_off(int c, int k, int rows)
{
    return (uint32_t)(((k >> 3) * (rows >> 3) + (c >> 3)) * 128 + (c & 7) * 16 + (k & 7) * 2);
}

template <int N>
__global__ void __launch_bounds__(kThreads, 1) k_block_inverse_tc(TcParams prm)
{
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N must be a multiple of 16 in [16, 256]");
    // Supports n <= 256 (at most two M tiles of 128).
    constexpr int TR = N / 2;                 // channels per tile
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_e, bar_mma;
    __shared__ uint32_t tmem_base_s;
    __shared__ float sm_part[8][2][N];        // Sherman-Morrison partial sums [warp][M tile][col]
    __shared__ float2 beta_s[TR];
    __shared__ double pkd_s[TR];

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int lq = warp & 3;                              // TMEM lane quarter of this warp
    constexpr int HALF = (N >= 32) ? N / 2 : N;           // columns per warp group
    const int c_begin = (N >= 32) ? (warp >> 2) * HALF : 0;
    const bool epi = (N >= 32) || warp < 4;               // N = 16: warps 4-7 sit out the epilogues
    const int n = prm.n, kp = prm.kp, mt_count = prm.mt;
    const int kb = kp >> 3;                               // 8-blocks along z and k
    const uint32_t part_bytes = (uint32_t)kp * kp * 2u;   // one of E_hi / E_lo
    unsigned char *e_hi = smem;
    unsigned char *e_lo = smem + part_bytes;
    unsigned char *b_hi = smem + 2 * part_bytes;
    unsigned char *b_lo = b_hi + (size_t)N * kp * 2;
    const uint32_t sz = (uint32_t)kb * 128u;              // stride of a z 8-block in E
    const uint32_t sk = 128u;                             // stride of a k 8-block in E
    const uint32_t b_lbo = (uint32_t)N * 16u;             // B: stride between k 8-blocks
    uint32_t ncols = 32;
    while (ncols < (uint32_t)(2 * mt_count * N)) ncols <<= 1;

    if (warp == 0) tmem_alloc(&tmem_base_s, ncols);
    if (tid == 0) {
        mbar_init(&bar_e, 1);
        mbar_init(&bar_mma, 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    bool ok = true;

    if (tid == 0) {
        mbar_expect_tx(&bar_e, 2u * part_bytes);
        bulk_g2s(e_hi, prm.e_img, part_bytes, &bar_e);
        bulk_g2s(e_lo, reinterpret_cast<const unsigned char *>(prm.e_img) + part_bytes, part_bytes, &bar_e);
    }
    bool e_ok = false;          // E image arrival is awaited just before the first MMA
    bool e_waited = false;
    uint32_t mma_phase = 0;
    bool mma_pending = false;
    const uint32_t idesc_mn = make_idesc(N, 1);   // GEMM 1: A = E^T via the MN-major view
    const uint32_t idesc_k = make_idesc(N, 0);    // GEMM 2: A = E, K-major
    const uint32_t e_hi_a = smem_u32(e_hi), e_lo_a = smem_u32(e_lo);
    const uint32_t b_hi_a = smem_u32(b_hi), b_lo_a = smem_u32(b_lo);
    const int ksteps = kp >> 4;

    for (int tile = blockIdx.x; tile < prm.ntiles && ok; tile += gridDim.x) {
        const int row0 = tile * TR;
        const int nrow = min(TR, prm.rows - row0);
        int any = 1;
        if (tid == 0 && prm.gate) {
            any = 0;
            const int s0 = prm.row_sys[row0], s1 = prm.row_sys[row0 + nrow - 1];
            for (int s = s0; s <= s1 && !any; ++s) any = prm.gate[s] != 0;
        }
        for (int j = tid; j < TR; j += kThreads) pkd_s[j] = (j < nrow) ? prm.row_pkd[row0 + j] : 0.0;
        if (!__syncthreads_or(tid == 0 ? any : 0)) continue;

        // ---- stage x as the B operand of GEMM 1 (rows = 2 TR re/im columns, K = z).
        // Loads are batched (kBatch per thread in flight) because one CTA per
        // SM has only four warps to hide memory latency with.
        constexpr int kBatch = 16;
        for (int base = tid; base < TR * kp; base += kThreads * kBatch) {
            float2 v[kBatch];
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int idx = base + u * kThreads;
                const int j = idx / kp, z = idx - j * kp;
                v[u] = make_float2(0.f, 0.f);
                if (idx < TR * kp && j < nrow && z < n) v[u] = prm.x[(size_t)(row0 + j) * n + z];
            }
#pragma unroll
            for (int u = 0; u < kBatch; ++u) {
                const int idx = base + u * kThreads;
                if (idx >= TR * kp) break;
                const int j = idx / kp, z = idx - j * kp;
                const __nv_bfloat16 hr = __float2bfloat16_rn(v[u].x), hi = __float2bfloat16_rn(v[u].y);
                const __nv_bfloat16 lr = __float2bfloat16_rn(v[u].x - __bfloat162float(hr));
                const __nv_bfloat16 li = __float2bfloat16_rn(v[u].y - __bfloat162float(hi));
                const uint32_t o_re = kmaj_off(2 * j, z, N), o_im = kmaj_off(2 * j + 1, z, N);
                *reinterpret_cast<__nv_bfloat16 *>(b_hi + o_re) = hr;
                *reinterpret_cast<__nv_bfloat16 *>(b_hi + o_im) = hi;
                *reinterpret_cast<__nv_bfloat16 *>(b_lo + o_re) = lr;
                *reinterpret_cast<__nv_bfloat16 *>(b_lo + o_im) = li;
            }
        }
        fence_proxy_async();
        if (!e_waited) {
            e_ok = mbar_wait(&bar_e, 0);
            e_waited = true;
            if (!__syncthreads_and(e_ok)) { ok = false; break; }
        }
        __syncthreads();

        // ---- GEMM 1: D1[m] = E^T x   (M = k, K = z); accumulator columns [m N, m N + N)
        if (tid == 0) {
            tc_fence_after();
            for (int m = 0; m < mt_count; ++m) {
                const uint32_t d = tmem + (uint32_t)(m * N);
                for (int s = 0; s < ksteps; ++s) {
                    // A (MN-major view): M-block stride = sk, K-block stride = sz
                    const uint32_t a_off = (uint32_t)(m * 16) * sk + (uint32_t)(2 * s) * sz;
                    const uint64_t ah = make_desc(e_hi_a + a_off, sz, sk);
                    const uint64_t al = make_desc(e_lo_a + a_off, sz, sk);
                    const uint32_t b_off = (uint32_t)(2 * s) * b_lbo;
                    const uint64_t bh = make_desc(b_hi_a + b_off, b_lbo, 128);
                    const uint64_t bl = make_desc(b_lo_a + b_off, b_lbo, 128);
                    mma_bf16(d, ah, bh, idesc_mn, s > 0 ? 1u : 0u);
                    mma_bf16(d, ah, bl, idesc_mn, 1u);
                    mma_bf16(d, al, bh, idesc_mn, 1u);
                }
            }
            mma_commit(&bar_mma);
        }
        mma_pending = true;
        if (mbar_wait(&bar_mma, mma_phase)) {
            mma_phase ^= 1u;
            mma_pending = false;
        } else {
            ok = false;
        }
        tc_fence_after();
        if (!__syncthreads_and(ok)) { ok = false; break; }

        // ---- epilogue 1a: Sherman-Morrison sums s_j = sum_k en_k xt_kj / (pkd_j + lam_k)
        for (int m = 0; m < mt_count && epi; ++m) {
            const int k = m * 128 + lq * 32 + lane;
            const bool valid = k < n;
            const double lam_k = valid ? prm.lam[k] : 0.0;
            const float en_k = valid ? (float)prm.en[k] : 0.f;
            for (int c0 = c_begin; c0 < c_begin + HALF; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(m * N + c0), v);
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    const int j = (c0 + c) >> 1;
                    float wr = 0.f, wi = 0.f;
                    if (valid && j < nrow) {
                        const float w = en_k / (float)(pkd_s[j] + lam_k);
                        wr = w * v[c];
                        wi = w * v[c + 1];
                    }
                    wr = warp_sum(wr);
                    wi = warp_sum(wi);
                    if (lane == 0) {
                        sm_part[warp][m][c0 + c] = wr;
                        sm_part[warp][m][c0 + c + 1] = wi;
                    }
                }
            }
        }
        __syncthreads();
        for (int j = tid; j < TR; j += kThreads) {
            double2 b = make_double2(0.0, 0.0);
            if (j < nrow) {
                double sr = 0.0, si = 0.0;   // fixed summation order: deterministic
                const int wg = (N >= 32) ? ((2 * j) / HALF) * 4 : 0;   // warps that own column 2j
                for (int m = 0; m < mt_count; ++m)
                    for (int w = wg; w < wg + 4; ++w) {
                        sr += sm_part[w][m][2 * j];
                        si += sm_part[w][m][2 * j + 1];
                    }
                const double2 c = prm.row_c[row0 + j];
                const double fn = prm.row_fn[row0 + j];
                b = cdiv(cmul(c, make_double2(sr, si)), make_double2(1.0 - c.x * fn, -c.y * fn));
            }
            beta_s[j] = make_float2((float)b.x, (float)b.y);
        }
        __syncthreads();

        // ---- epilogue 1b: yt = (xt + beta en) / (pkd + lam) as the B operand of GEMM 2
        // (rows = 2 TR columns, K = k; rows k >= kp are never read, k in [n, kp) are zero)
        for (int m = 0; m < mt_count && epi; ++m) {
            const int k = m * 128 + lq * 32 + lane;
            const bool valid = k < n;
            const bool stage = k < kp;
            const double lam_k = valid ? prm.lam[k] : 0.0;
            const float en_k = valid ? (float)prm.en[k] : 0.f;
            for (int c0 = c_begin; c0 < c_begin + HALF; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(m * N + c0), v);
                if (!stage) continue;
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    const int j = (c0 + c) >> 1;
                    float yr = 0.f, yi = 0.f;
                    if (valid && j < nrow) {
                        const float inv = 1.0f / (float)(pkd_s[j] + lam_k);
                        const float2 b = beta_s[j];
                        yr = (v[c] + b.x * en_k) * inv;
                        yi = (v[c + 1] + b.y * en_k) * inv;
                    }
                    const __nv_bfloat16 hr = __float2bfloat16_rn(yr), hi = __float2bfloat16_rn(yi);
                    const __nv_bfloat16 lr = __float2bfloat16_rn(yr - __bfloat162float(hr));
                    const __nv_bfloat16 li = __float2bfloat16_rn(yi - __bfloat162float(hi));
                    const uint32_t o_re = kmaj_off(c0 + c, k, N), o_im = kmaj_off(c0 + c + 1, k, N);
                    *reinterpret_cast<__nv_bfloat16 *>(b_hi + o_re) = hr;
                    *reinterpret_cast<__nv_bfloat16 *>(b_hi + o_im) = hi;
                    *reinterpret_cast<__nv_bfloat16 *>(b_lo + o_re) = lr;
                    *reinterpret_cast<__nv_bfloat16 *>(b_lo + o_im) = li;
                }
            }
        }
        tc_fence_before();
        fence_proxy_async();
        __syncthreads();

        // ---- GEMM 2: D2[m] = E yt   (M = z, K = k); accumulator columns after D1
        if (tid == 0) {
            tc_fence_after();
            for (int m = 0; m < mt_count; ++m) {
                const uint32_t d = tmem + (uint32_t)((mt_count + m) * N);
                for (int s = 0; s < ksteps; ++s) {
                    // A (K-major): row-block (z) stride = sz (SBO), K-block (k) stride = sk (LBO)
                    const uint32_t a_off = (uint32_t)(m * 16) * sz + (uint32_t)(2 * s) * sk;
                    const uint64_t ah = make_desc(e_hi_a + a_off, sk, sz);
                    const uint64_t al = make_desc(e_lo_a + a_off, sk, sz);
                    const uint32_t b_off = (uint32_t)(2 * s) * b_lbo;
                    const uint64_t bh = make_desc(b_hi_a + b_off, b_lbo, 128);
                    const uint64_t bl = make_desc(b_lo_a + b_off, b_lbo, 128);
                    mma_bf16(d, ah, bh, idesc_k, s > 0 ? 1u : 0u);
                    mma_bf16(d, ah, bl, idesc_k, 1u);
                    mma_bf16(d, al, bh, idesc_k, 1u);
                }
            }
            mma_commit(&bar_mma);
        }
        mma_pending = true;
        if (mbar_wait(&bar_mma, mma_phase)) {
            mma_phase ^= 1u;
            mma_pending = false;
        } else {
            ok = false;
        }
        tc_fence_after();
        if (!__syncthreads_and(ok)) { ok = false; break; }

        // ---- epilogue 2: u rows to global (z contiguous across lanes)
        for (int m = 0; m < mt_count && epi; ++m) {
            const int z = m * 128 + lq * 32 + lane;
            for (int c0 = c_begin; c0 < c_begin + HALF; c0 += 16) {
                float v[16];
                tmem_ld16(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)((mt_count + m) * N + c0), v);
                if (z < n) {
#pragma unroll
                    for (int c = 0; c < 16; c += 2) {
                        const int j = (c0 + c) >> 1;
                        if (j < nrow) prm.out[(size_t)(row0 + j) * n + z] = make_float2(v[c], v[c + 1]);
                    }
                }
            }
        }
        tc_fence_before();
        __syncthreads();
    }

    if (!ok && tid == 0 && prm.error) atomicExch(prm.error, 1);
    // Drain on a time-out: give the copy or MMAs still in flight a bounded
    // chance to finish before the accumulator columns are released.
    if (tid == 0 && !e_ok) (void)mbar_wait(&bar_e, 0);   // copy issued but not yet seen complete
    if (tid == 0 && mma_pending) (void)mbar_wait(&bar_mma, mma_phase);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem, ncols);
}

}  // namespace tc
}  // namespace msc
