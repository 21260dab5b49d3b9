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
// Execution.  Persistent CTAs (one per SM, 512 threads = 16 warps).  Per
// tile: stage x as B with 16-byte stores; one thread issues the MMAs and
// commits to an mbarrier; all warps read the accumulator with tcgen05.ld
// (warp w owns TMEM lanes 32 (w % 4)..32 (w % 4) + 31 and the columns of
// its column group w / 4: a quarter of N with one group), reduce
// the Sherman-Morrison sums over k with a reduce-scatter butterfly, form
// yt (pkd + lam in FP64) and stage it as the MN-major B operand of the second
// GEMM with 16-byte stores, store u.  beta is formed from the accumulator
// before the division by pkd + lam (adding the correction after the second
// GEMM instead, u = u0 + beta (H0 + pkd)^-1 e_n, cancels two large terms in
// FP32 near resonances of H0 + pkd and stalls the refinement).  Every mbarrier wait is bounded;
// on time-out the kernel records an error code, stops issuing work and still
// releases its TMEM.
//
// The epilogues are chains of short dependent steps (TMEM load, FP64 sum
// and SFU reciprocal, shuffles); 16 warps keep four per scheduler to hide
// them, with at most 128 registers per thread (the accumulator is read 32
// columns at a time).
//
// Warp groups.  With G = 2 the 16 warps form two groups of 8 (each group's
// warps cover the four TMEM lane quarters and two column halves); each group has
// its own B buffer, TMEM columns, mbarrier and named barrier and runs its own
// tile loop (tiles 2 b + g, stride 2 gridDim), so one group's staging and
// epilogues can overlap the other's MMAs.  G is autotuned with N.
#pragma once

#include <cuda_bf16.h>

#include "msc_common.cuh"

namespace msc {
namespace tc {

constexpr int kThreads = 512;   // 16 warps: warp w reads TMEM lanes 32 (w % 4).. of its column group

// Named barrier `id` over `count` threads (a warp group's tile loop; barrier
// 0 stays the CTA-wide __syncthreads).
__device__ __forceinline__ void group_sync(int id, int count)
{
    asm volatile("bar.sync %0, %1;" ::"r"(id), "r"(count) : "memory");
}

// Named barrier that also returns the AND of `v` over the participating threads.
__device__ __forceinline__ bool group_and(int id, int count, bool v)
{
    uint32_t r;
    asm volatile(
        "{\n\t.reg .pred p, q;\n\t"
        "setp.ne.u32 p, %1, 0;\n\t"
        "bar.red.and.pred q, %2, %3, p;\n\t"
        "selp.u32 %0, 1, 0, q;\n\t}"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(id), "r"(count)
        : "memory");
    return r != 0;
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

// 32 lanes x 16 consecutive 32-bit columns, issued without waiting: several
// loads go out back to back and one tmem_wait_ld completes them (the
// epilogues read up to 64 columns per warp and M tile at once instead of
// paying the load latency per 16).
__device__ __forceinline__ void tmem_ld16_nowait(uint32_t taddr, uint32_t (&r)[16])
{
    asm volatile(
        "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
          "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
        : "r"(taddr));
}
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory"); }

// Up to kLdChunks 16-column chunks starting at column c (warp-uniform count
// nch), one wait for all of them.
constexpr int kLdChunks = 2;
__device__ __forceinline__ void tmem_ld_chunks(uint32_t taddr, int nch, float (&v)[kLdChunks][16])
{
    uint32_t r[kLdChunks][16];
#pragma unroll
    for (int q = 0; q < kLdChunks; ++q)
        if (q < nch) tmem_ld16_nowait(taddr + (uint32_t)(16 * q), r[q]);
    tmem_wait_ld();
#pragma unroll
    for (int q = 0; q < kLdChunks; ++q)
#pragma unroll
        for (int i = 0; i < 16; ++i) v[q][i] = __uint_as_float(r[q][i]);
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

// Instruction descriptor: BF16 x BF16 -> FP32, M = 128, given N and the
// major-ness of A and B (0 K-major, 1 MN-major).
__host__ __device__ constexpr uint32_t make_idesc(int n, int a_mn_major, int b_mn_major)
{
    return (1u << 4)                         // D format F32
           | (1u << 7)                       // A format BF16
           | (1u << 10)                      // B format BF16
           | ((uint32_t)a_mn_major << 15)    // A major
           | ((uint32_t)b_mn_major << 16)    // B major
           | ((uint32_t)(n >> 3) << 17)      // N / 8
           | ((uint32_t)(128 >> 4) << 24);   // M / 16
}

// Reduce-scatter of 16 per-lane values over a warp: returns, in every lane,
// the sum over all 32 lanes of value (lane >> 1) & 15 (lanes 2i and 2i + 1
// hold the same column).  15 + 1 shuffles instead of 16 x 5; the order of
// the additions is fixed, so the result is deterministic.
__device__ __forceinline__ float warp_reduce_scatter16(float (&v)[16], int lane)
{
#pragma unroll
    for (int i = 0; i < 8; ++i) {          // lanes with bit 4 set keep columns 8..15
        const bool up = lane & 16;
        const float send = up ? v[i] : v[i + 8];
        const float keep = up ? v[i + 8] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 16);
    }
#pragma unroll
    for (int i = 0; i < 4; ++i) {          // bit 3: upper 4 of the 8
        const bool up = lane & 8;
        const float send = up ? v[i] : v[i + 4];
        const float keep = up ? v[i + 4] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 8);
    }
#pragma unroll
    for (int i = 0; i < 2; ++i) {          // bit 2
        const bool up = lane & 4;
        const float send = up ? v[i] : v[i + 2];
        const float keep = up ? v[i + 2] : v[i];
        v[i] = keep + __shfl_xor_sync(0xffffffffu, send, 4);
    }
    {                                      // bit 1
        const bool up = lane & 2;
        const float send = up ? v[0] : v[1];
        const float keep = up ? v[1] : v[0];
        v[0] = keep + __shfl_xor_sync(0xffffffffu, send, 2);
    }
    return v[0] + __shfl_xor_sync(0xffffffffu, v[0], 1);
}

// 1 / (pkd + lam_k): the sum in FP64 (pkd and lam_k cancel near a channel
// resonance), the reciprocal by the SFU's approximate FP32 divide (two
// instructions instead of the correctly rounded sequence; its 2-ulp error
// is far below the BF16x3 products').  Both epilogues call it, so the
// Sherman-Morrison sums and yt use the same values.
__device__ __forceinline__ float shifted_inverse(double pkd, double lam)
{
    return __fdividef(1.0f, (float)(pkd + lam));
}

struct TcParams {
    int n;             // nodes
    int kp;            // n rounded up to 16 (E padded to kp x kp)
    int mt;            // M tiles of 128 (ceil(n / 128))
    int rows;          // total channel rows R
    int tile_rows;     // channels per tile (N / 2)
    int ntiles;        // ceil(R / tile_rows)
    const __nv_bfloat16 *e_img;   // [2][kp/8][kp/8][8][8]  hi part then lo part
    const double *lam, *en, *row_pkd;
    const double2 *row_cf;        // [R] c / (1 - c f_n) of each row (Sherman-Morrison factor)
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

// G = 1: the CTA's 16 warps work on one tile at a time.  G = 2: two groups
// of 8 warps (warps 0-7, 8-15), each with its own B buffer, TMEM columns,
// mbarrier and named barrier, run independent tile loops over the shared E
// image, so that one group's staging and epilogues overlap the other's MMAs.
template <int N, int G>
__global__ void __launch_bounds__(kThreads, 1) k_block_inverse_tc(TcParams prm)
{
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "N must be a multiple of 16 in [16, 256]");
    static_assert(G == 1 || (G == 2 && N <= 128), "two groups take N <= 128");
    // Supports n <= 256 (at most two M tiles of 128).
    constexpr int GT = kThreads / G;          // threads per group
    constexpr int NW = GT / 32;               // warps per group
    constexpr int TR = N / 2;                 // channels per tile
    constexpr int P = GT / TR;                // staging threads per channel
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_e, bar_mma[G], bar_pf[G];
    __shared__ uint32_t tmem_base_s;
    __shared__ float sm_part[G][4][2][N];     // Sherman-Morrison partial sums [group][lane quarter][M tile][col]
    __shared__ float2 beta_s[G][TR];
    __shared__ double pkd_s[G][TR];
    __shared__ double2 cf_s[G][TR];            // the tile's c_j / (1 - c_j fn_j), loaded with pkd
    __shared__ double lam_s[256];             // eigenvalues of H0 (k < n <= 256), 0 past n
    __shared__ float en_s[256];               // last components E[n-1, k] (FP32), 0 past n

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int g = (G == 1) ? 0 : warp / NW;               // group of this thread
    const int gtid = tid - g * GT, wl = warp - g * NW;    // thread / warp index within the group
    const int bar_id = 1 + g;                             // the group's named barrier
    const int lq = warp & 3;                              // TMEM lane quarter of this warp
    constexpr int NCG = NW / 4;                           // column groups (warps per lane quarter)
    constexpr int CW = (N / NCG >= 16) ? N / NCG : 16;    // columns per warp
    const int c_begin = (wl >> 2) * CW;
    constexpr bool kInvCache = CW == 16 * kLdChunks;      // one TMEM pass per M tile
    float invc[2][kInvCache ? CW / 2 : 1];                // 1 / (pkd_j + lam_k) of epilogue 1a
    const bool epi = c_begin < N;                         // narrow tiles: surplus column groups sit out
    const int n = prm.n, kp = prm.kp, mt_count = prm.mt;
    const int kb = kp >> 3;                               // 8-blocks along z and k
    const uint32_t part_bytes = (uint32_t)kp * kp * 2u;   // one of E_hi / E_lo
    unsigned char *e_hi = smem;
    unsigned char *e_lo = smem + part_bytes;
    unsigned char *b_hi = smem + 2 * part_bytes + (size_t)g * 4 * N * kp;
    unsigned char *b_lo = b_hi + (size_t)N * kp * 2;
    const uint32_t sz = (uint32_t)kb * 128u;              // stride of a z 8-block in E
    const uint32_t sk = 128u;                             // stride of a k 8-block in E
    const uint32_t b_lbo = (uint32_t)N * 16u;             // B: stride between k 8-blocks
    uint32_t ncols = 32;                                  // TMEM columns of one group
    while (ncols < (uint32_t)(2 * mt_count * N)) ncols <<= 1;

    if (warp == 0) tmem_alloc(&tmem_base_s, G * ncols);
    for (int k = tid; k < 256; k += kThreads) {
        lam_s[k] = k < n ? prm.lam[k] : 0.0;
        en_s[k] = k < n ? (float)prm.en[k] : 0.f;
    }
    if (tid == 0) {
        mbar_init(&bar_e, 1);
        for (int q = 0; q < G; ++q) mbar_init(&bar_mma[q], 1);
        for (int q = 0; q < G; ++q) mbar_init(&bar_pf[q], 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s + (uint32_t)g * ncols;
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
    const uint32_t idesc_mn = make_idesc(N, 1, 0);   // GEMM 1: A = E^T via the MN-major view, B K-major
    const uint32_t idesc_k = make_idesc(N, 0, 1);    // GEMM 2: A = E K-major, B MN-major
    const uint32_t e_hi_a = smem_u32(e_hi), e_lo_a = smem_u32(e_lo);
    const uint32_t b_hi_a = smem_u32(b_hi), b_lo_a = smem_u32(b_lo);
    const int ksteps = kp >> 4;
    const int sj = gtid % TR, sp = gtid / TR;             // staging: channel, z-block phase

    // Staging units: thread (channel sj, z-blocks sp, sp + P, ...) handles 8
    // consecutive z (64 contiguous bytes of x) and writes four 16-byte units
    // (re/im x hi/lo) of the K-major B operand of GEMM 1.
    auto write_unit = [&](int zb, const float2 (&v)[8]) {
        uint32_t rh[4], ih[4], rl[4], il[4];
#pragma unroll
        for (int u = 0; u < 8; u += 2) {
            const __nv_bfloat162 hr = __floats2bfloat162_rn(v[u].x, v[u + 1].x);
            const __nv_bfloat162 hi = __floats2bfloat162_rn(v[u].y, v[u + 1].y);
            const float2 fr = __bfloat1622float2(hr), fi = __bfloat1622float2(hi);
            const __nv_bfloat162 lr = __floats2bfloat162_rn(v[u].x - fr.x, v[u + 1].x - fr.y);
            const __nv_bfloat162 li = __floats2bfloat162_rn(v[u].y - fi.x, v[u + 1].y - fi.y);
            rh[u >> 1] = *reinterpret_cast<const uint32_t *>(&hr);
            ih[u >> 1] = *reinterpret_cast<const uint32_t *>(&hi);
            rl[u >> 1] = *reinterpret_cast<const uint32_t *>(&lr);
            il[u >> 1] = *reinterpret_cast<const uint32_t *>(&li);
        }
        const uint32_t o_re = kmaj_off(2 * sj, zb * 8, N), o_im = o_re + 16;
        *reinterpret_cast<uint4 *>(b_hi + o_re) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4 *>(b_hi + o_im) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4 *>(b_lo + o_re) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4 *>(b_lo + o_im) = make_uint4(il[0], il[1], il[2], il[3]);
    };
    // Prefetch: once the second GEMM has consumed the B buffer, the next
    // tile's raw x rows ([TR][n] complex FP32 = 8 TR n bytes, within the B
    // buffer's 4 N kp = 8 TR kp bytes; one contiguous range of x) arrive in
    // it by one bulk copy on the group's mbarrier while the current tile is
    // stored; the next staging converts them from shared memory.  Needs a
    // 16-byte aligned range (n even, x 16-byte aligned) and at most kMaxPf
    // units per thread held in registers (raw and converted data share the
    // buffer).
    constexpr int kMaxPf = 4;
    const int upt = (kb + P - 1) / P;
    const bool use_pf = (n % 2 == 0) && upt <= kMaxPf &&
                        (reinterpret_cast<uintptr_t>(prm.x) & 15u) == 0;
    float2 *raw = reinterpret_cast<float2 *>(b_hi);
    uint32_t pf_phase = 0;
    bool pf_pending = false;
    auto prefetch = [&](int t) {
        if (gtid == 0) {
            const int r0 = t * TR, nr = min(TR, prm.rows - r0);
            const uint32_t bytes = (uint32_t)nr * (uint32_t)n * 8u;
            mbar_expect_tx(&bar_pf[g], bytes);
            bulk_g2s(raw, prm.x + (size_t)r0 * n, bytes, &bar_pf[g]);
        }
        pf_pending = true;
    };
    // first active tile of this group at or after t (stride G gridDim.x); the
    // group's thread 0
    auto find_active = [&](int t) {
        for (; t < prm.ntiles; t += G * gridDim.x) {
            if (!prm.gate) return t;
            const int r0 = t * TR, nr = min(TR, prm.rows - r0);
            const int s0 = prm.row_sys[r0], s1 = prm.row_sys[r0 + nr - 1];
            for (int q = s0; q <= s1; ++q)
                if (prm.gate[q]) return t;
        }
        return prm.ntiles;
    };
    __shared__ int next_s[G];
    if (gtid == 0) next_s[g] = find_active(G * blockIdx.x + g);
    __syncthreads();
    int tile = next_s[g];
    __syncthreads();            // every thread has read next_s before the loop rewrites it
    if (use_pf && tile < prm.ntiles) prefetch(tile);

    while (tile < prm.ntiles && ok) {
        const int row0 = tile * TR;
        const int nrow = min(TR, prm.rows - row0);
        for (int j = gtid; j < TR; j += GT) {
            const bool in = j < nrow;
            pkd_s[g][j] = in ? prm.row_pkd[row0 + j] : 0.0;
            cf_s[g][j] = in ? prm.row_cf[row0 + j] : make_double2(0.0, 0.0);
        }

        // ---- stage x as the B operand of GEMM 1 (K-major: rows = 2 TR re/im
        // columns, K = z)
        {
            const bool jok = sj < nrow;
            if (use_pf) {
                const bool got = mbar_wait(&bar_pf[g], pf_phase);
                if (!group_and(bar_id, GT, got)) { ok = false; break; }   // the raw tile is complete
                pf_phase ^= 1u;
                pf_pending = false;
                // two z per 16-byte load: the rows' 8 n-byte stride then
                // spreads a warp's 32 channels over all banks
                float2 v[kMaxPf][8];
                const float4 *raw4 = reinterpret_cast<const float4 *>(raw);
#pragma unroll
                for (int u = 0; u < kMaxPf; ++u) {
                    const int zb = sp + u * P;
#pragma unroll
                    for (int e = 0; e < 8; e += 2) {
                        const int z = zb * 8 + e;
                        float4 t = make_float4(0.f, 0.f, 0.f, 0.f);
                        if (u < upt && zb < kb && jok && z < n) t = raw4[((size_t)sj * n + z) >> 1];
                        v[u][e] = make_float2(t.x, t.y);
                        v[u][e + 1] = make_float2(t.z, t.w);
                    }
                }
                group_sync(bar_id, GT);                // raw reads done before B is overwritten
#pragma unroll
                for (int u = 0; u < kMaxPf; ++u) {
                    const int zb = sp + u * P;
                    if (u < upt && zb < kb) write_unit(zb, v[u]);
                }
            } else {
                const float2 *xr = prm.x + (size_t)(row0 + sj) * n;
                for (int zb = sp; zb < kb; zb += P) {
                    float2 v[8];
#pragma unroll
                    for (int u = 0; u < 8; ++u) {
                        const int z = zb * 8 + u;
                        v[u] = (jok && z < n) ? xr[z] : make_float2(0.f, 0.f);
                    }
                    write_unit(zb, v);
                }
            }
        }
        fence_proxy_async();
        if (!e_waited) {
            e_ok = mbar_wait(&bar_e, 0);
            e_waited = true;
            if (!group_and(bar_id, GT, e_ok)) { ok = false; break; }
        }
        group_sync(bar_id, GT);

        // ---- GEMM 1: D1[m] = E^T x   (M = k, K = z); accumulator columns [m N, m N + N)
        if (gtid == 0) {
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
            mma_commit(&bar_mma[g]);
        }
        // the next active tile (its search reads gate and row_sys from
        // global memory) is found by warp 1 while the MMAs run (on the
        // issuing thread it held up the wait that follows); every thread of
        // the group read next_s before the previous tile's last barrier
        if (gtid == 32) next_s[g] = find_active(tile + G * gridDim.x);
        mma_pending = true;
        if (mbar_wait(&bar_mma[g], mma_phase)) {
            mma_phase ^= 1u;
            mma_pending = false;
        } else {
            ok = false;
        }
        tc_fence_after();
        if (!group_and(bar_id, GT, ok)) { ok = false; break; }

        // ---- epilogue 1a: Sherman-Morrison sums s_j = sum_k en_k xt_kj / (pkd_j + lam_k)
        // from the accumulator itself (so beta is consistent with the xt that
        // GEMM 2 consumes; pkd + lam in FP64).  Each 16-column chunk is
        // reduced over the warp's 32 k-lanes by a reduce-scatter butterfly
        // (16 shuffles), then over lane quarters and M tiles in a fixed order.
        // With one TMEM pass per M tile (CW = 32) the thread keeps its
        // 1 / (pkd_j + lam_k) values for epilogue 1b.
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            if (m >= mt_count || !epi) break;
            const int k = m * 128 + lq * 32 + lane;
            const bool valid = k < n;
            const double lam_k = lam_s[k];
            const float en_k = en_s[k];
#pragma unroll
            for (int cb = c_begin; cb < c_begin + CW; cb += 16 * kLdChunks) {
            const int nch = min(kLdChunks, (c_begin + CW - cb) >> 4);
            float vv[kLdChunks][16];
            tmem_ld_chunks(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(m * N + cb), nch, vv);
#pragma unroll
            for (int q = 0; q < kLdChunks; ++q) {
                if (q >= nch) continue;
                const int c0 = cb + 16 * q;
                float (&v)[16] = vv[q];
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    // select, not multiply: accumulator rows k >= kp of the last
                    // M tile come from bytes past E in shared memory and may hold
                    // NaN, which a zero weight would not remove
                    const int j = (c0 + c) >> 1;
                    if (valid && j < nrow) {
                        const float iv = shifted_inverse(pkd_s[g][j], lam_k);
                        if constexpr (kInvCache) invc[m][(16 * q + c) >> 1] = iv;
                        const float w = en_k * iv;
                        v[c] *= w;
                        v[c + 1] *= w;
                    } else {
                        v[c] = 0.f;
                        v[c + 1] = 0.f;
                    }
                }
                const float sum = warp_reduce_scatter16(v, lane);
                if ((lane & 1) == 0) sm_part[g][lq][m][c0 + ((lane >> 1) & 15)] = sum;
            }
            }
        }
        group_sync(bar_id, GT);
        for (int j = gtid; j < TR; j += GT) {
            double2 b = make_double2(0.0, 0.0);
            if (j < nrow) {
                double sr = 0.0, si = 0.0;   // fixed summation order: deterministic
                // the 4 warps (one per lane quarter) that own column 2j
                for (int m = 0; m < mt_count; ++m)
                    for (int w = 0; w < 4; ++w) {
                        sr += sm_part[g][w][m][2 * j];
                        si += sm_part[g][w][m][2 * j + 1];
                    }
                b = cmul(cf_s[g][j], make_double2(sr, si));
            }
            beta_s[g][j] = make_float2((float)b.x, (float)b.y);
        }
        group_sync(bar_id, GT);

        // ---- epilogue 1b: yt = (xt + beta en) / (pkd + lam) as the B operand of
        // GEMM 2 in the MN-major layout: one thread holds one k and 16
        // consecutive columns, i.e. two 16-byte units per hi / lo part
        // (rows k >= kp are never read; k in [n, kp) are zero).
#pragma unroll
        for (int m = 0; m < 2; ++m) {
            if (m >= mt_count || !epi) break;
            const int k = m * 128 + lq * 32 + lane;
            const bool valid = k < n;
            const bool stage = k < kp;
            const double lam_k = lam_s[k];
            const float en_k = en_s[k];
#pragma unroll
            for (int cb = c_begin; cb < c_begin + CW; cb += 16 * kLdChunks) {
            const int nch = min(kLdChunks, (c_begin + CW - cb) >> 4);
            float vv[kLdChunks][16];
            tmem_ld_chunks(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)(m * N + cb), nch, vv);
            if (!stage) continue;
#pragma unroll
            for (int q = 0; q < kLdChunks; ++q) {
                if (q >= nch) continue;
                const int c0 = cb + 16 * q;
                const float (&v)[16] = vv[q];
                uint32_t hw[8], lw[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    const int j = (c0 + c) >> 1;
                    float yr = 0.f, yi = 0.f;
                    if (valid && j < nrow) {
                        float inv;
                        if constexpr (kInvCache) inv = invc[m][(16 * q + c) >> 1];
                        else inv = shifted_inverse(pkd_s[g][j], lam_k);
                        const float2 b = beta_s[g][j];
                        yr = (v[c] + b.x * en_k) * inv;
                        yi = (v[c + 1] + b.y * en_k) * inv;
                    }
                    const __nv_bfloat162 h = __floats2bfloat162_rn(yr, yi);
                    const float2 fh = __bfloat1622float2(h);
                    const __nv_bfloat162 l = __floats2bfloat162_rn(yr - fh.x, yi - fh.y);
                    hw[c >> 1] = *reinterpret_cast<const uint32_t *>(&h);
                    lw[c >> 1] = *reinterpret_cast<const uint32_t *>(&l);
                }
                // MN-major core matrix: (k, c) at ((k/8)(N/8) + c/8) 128 + (k%8) 16 + (c%8) 2
                const uint32_t o = (uint32_t)(((k >> 3) * (N >> 3) + (c0 >> 3)) * 128 + (k & 7) * 16);
                *reinterpret_cast<uint4 *>(b_hi + o) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *reinterpret_cast<uint4 *>(b_hi + o + 128) = make_uint4(hw[4], hw[5], hw[6], hw[7]);
                *reinterpret_cast<uint4 *>(b_lo + o) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                *reinterpret_cast<uint4 *>(b_lo + o + 128) = make_uint4(lw[4], lw[5], lw[6], lw[7]);
            }
            }
        }
        tc_fence_before();
        fence_proxy_async();
        group_sync(bar_id, GT);

        // ---- GEMM 2: D2[m] = E yt   (M = z, K = k); accumulator columns after D1
        if (gtid == 0) {
            tc_fence_after();
            for (int m = 0; m < mt_count; ++m) {
                const uint32_t d = tmem + (uint32_t)((mt_count + m) * N);
                for (int s = 0; s < ksteps; ++s) {
                    // A (K-major): row-block (z) stride = sz (SBO), K-block (k) stride = sk (LBO)
                    const uint32_t a_off = (uint32_t)(m * 16) * sz + (uint32_t)(2 * s) * sk;
                    const uint64_t ah = make_desc(e_hi_a + a_off, sk, sz);
                    const uint64_t al = make_desc(e_lo_a + a_off, sk, sz);
                    // B (MN-major): K-block (k) stride = 16 N (LBO), N-block stride = 128 (SBO)
                    const uint32_t b_off = (uint32_t)(2 * s) * b_lbo;
                    const uint64_t bh = make_desc(b_hi_a + b_off, b_lbo, 128);
                    const uint64_t bl = make_desc(b_lo_a + b_off, b_lbo, 128);
                    mma_bf16(d, ah, bh, idesc_k, s > 0 ? 1u : 0u);
                    mma_bf16(d, ah, bl, idesc_k, 1u);
                    mma_bf16(d, al, bh, idesc_k, 1u);
                }
            }
            mma_commit(&bar_mma[g]);
        }
        mma_pending = true;
        if (mbar_wait(&bar_mma[g], mma_phase)) {
            mma_phase ^= 1u;
            mma_pending = false;
        } else {
            ok = false;
        }
        tc_fence_after();
        if (!group_and(bar_id, GT, ok)) { ok = false; break; }
        // the B buffer is free: start the next tile's copy
        const int next = next_s[g];
        if (use_pf && next < prm.ntiles) prefetch(next);

        // ---- epilogue 2: u rows to global (z contiguous across lanes)
        for (int m = 0; m < mt_count && epi; ++m) {
            const int z = m * 128 + lq * 32 + lane;
            for (int cb = c_begin; cb < c_begin + CW; cb += 16 * kLdChunks) {
                const int nch = min(kLdChunks, (c_begin + CW - cb) >> 4);
                float vv[kLdChunks][16];
                tmem_ld_chunks(tmem + ((uint32_t)(lq * 32) << 16) + (uint32_t)((mt_count + m) * N + cb),
                               nch, vv);
                if (z < n) {
#pragma unroll
                    for (int q = 0; q < kLdChunks; ++q) {
                        if (q >= nch) continue;
#pragma unroll
                        for (int c = 0; c < 16; c += 2) {
                            const int j = (cb + 16 * q + c) >> 1;
                            if (j < nrow)
                                prm.out[(size_t)(row0 + j) * n + z] = make_float2(vv[q][c], vv[q][c + 1]);
                        }
                    }
                }
            }
        }
        tc_fence_before();
        group_sync(bar_id, GT);
        tile = next;
    }

    if (!ok && gtid == 0 && prm.error) atomicExch(prm.error, 1);
    // no copy may land after the kernel leaves
    if (gtid == 0 && pf_pending) (void)mbar_wait(&bar_pf[g], pf_phase);
    // Drain on a time-out: give the copy or MMAs still in flight a bounded
    // chance to finish before the accumulator columns are released.
    if (gtid == 0 && !e_ok) (void)mbar_wait(&bar_e, 0);   // copy issued but not yet seen complete
    if (gtid == 0 && mma_pending) (void)mbar_wait(&bar_mma[g], mma_phase);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem_base_s, G * ncols);
}

}  // namespace tc
}  // namespace msc
