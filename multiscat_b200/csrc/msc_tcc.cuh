// msc_tcc.cuh -- tcgen05 block-diagonal inverse with the channel rows as the
// M dimension ("channel-major" form of k_block_inverse_tc).
//
//   u = D^-1 x  per channel:  xt = E^T x ;  yt = (xt + beta e_n)/(pkd + lam) ;  u = E yt
//
// Here both GEMMs put the tile's 64 channels (128 rows: re and im of each,
// interleaved) on M = 128 and the nodes on N = kp (n rounded up to 16):
//   GEMM 1  D1[c, k] = sum_z x[c, z] E[z, k]    A = x tile (K-major, K = z),
//                                               B = E (MN-major view, N = k)
//   GEMM 2  D2[c, z] = sum_k yt[c, k] E[z, k]   A = yt tile (K-major, K = k),
//                                               B = E (K-major view, N = z)
// so the MMAs cover kp columns instead of two 128-row M tiles (n = 150:
// 160 against 256 rows), and each accumulator row belongs to one channel:
// the Sherman-Morrison sum over k is a sum along the thread's own columns
// (no warp butterfly), and pkd is one value per thread.  The same E image
// (8x8 core matrices: 8 rows of z, 8 consecutive k per 16-byte row) serves
// both B operands, as in k_block_inverse_tc; the A buffer takes the x tile,
// then yt, then (as raw FP32 rows) the next tile's x by one bulk copy.
// TMEM: D1 at columns [0, kp), D2 at [256, 256 + kp).
//
// BF16x3 products (A_hi B_hi + A_hi B_lo + A_lo B_hi), FP32 accumulation,
// pkd + lam in FP64 and the SFU reciprocal, every mbarrier wait bounded: on
// a time-out the kernel sets the error word, drains what it issued, frees
// its TMEM and returns.
#pragma once

#include "msc_tc.cuh"

namespace msc {
namespace tc {

// 16 accumulator columns of this warp's 32 lanes, waited for.
__device__ __forceinline__ void tmem_ld16f(uint32_t taddr, float (&v)[16])
{
    uint32_t r[16];
    tmem_ld16_nowait(taddr, r);
    tmem_wait_ld();
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}

// One CTA per SM, 512 threads: warp w reads TMEM lanes 32 (w % 4) .. + 31
// (rows c, i.e. 16 channels) and the column group w / 4 (a quarter of kp,
// in 16-column chunks).
__global__ void __launch_bounds__(kThreads, 1) k_block_inverse_tcc(TcParams prm)
{
    constexpr int TR = 64;                    // channels per tile
    constexpr int ROWS = 2 * TR;              // M
    constexpr int P = kThreads / TR;          // staging threads per channel
    extern __shared__ __align__(1024) unsigned char smem[];
    __shared__ __align__(8) uint64_t bar_e, bar_mma, bar_pf;
    __shared__ uint32_t tmem_base_s;
    __shared__ double sm_part[4][ROWS];       // Sherman-Morrison partial sums [column group][row]
    __shared__ float2 beta_s[TR];
    __shared__ double pkd_s[TR];
    __shared__ double2 cf_s[TR];              // c_j / (1 - c_j fn_j)
    __shared__ double lam_s[256];
    __shared__ float en_s[256];
    __shared__ int next_s;

    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int lq = warp & 3, cg = warp >> 2;
    const int n = prm.n, kp = prm.kp;
    const int kb = kp >> 3;                               // 8-blocks along z and k
    const int nch = kp >> 4;                              // 16-column chunks of an accumulator
    const int ch0 = (cg * nch) >> 2, ch1 = ((cg + 1) * nch) >> 2;   // this warp's chunks
    const uint32_t part_bytes = (uint32_t)kp * kp * 2u;   // one of E_hi / E_lo
    unsigned char *e_hi = smem;
    unsigned char *e_lo = smem + part_bytes;
    unsigned char *a_hi = smem + 2 * part_bytes;
    unsigned char *a_lo = a_hi + (size_t)ROWS * kp * 2;
    const uint32_t sz = (uint32_t)kb * 128u;              // E: stride of a z 8-block
    const uint32_t sk = 128u;                             // E: stride of a k 8-block
    const uint32_t a_lbo = (uint32_t)ROWS * 16u;          // A: stride of a K 8-block
    const int c = lq * 32 + lane;                         // accumulator row of this thread
    const int jc = c >> 1;                                // its channel in the tile

    if (warp == 0) tmem_alloc(&tmem_base_s, 512);
    for (int k = tid; k < 256; k += kThreads) {
        lam_s[k] = k < n ? prm.lam[k] : 0.0;
        en_s[k] = k < n ? (float)prm.en[k] : 0.f;
    }
    if (tid == 0) {
        mbar_init(&bar_e, 1);
        mbar_init(&bar_mma, 1);
        mbar_init(&bar_pf, 1);
        mbar_fence_init();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tmem_base_s;
    const uint32_t d1 = tmem, d2 = tmem + 256u;
    bool ok = true;

    if (tid == 0) {
        mbar_expect_tx(&bar_e, 2u * part_bytes);
        bulk_g2s(e_hi, prm.e_img, part_bytes, &bar_e);
        bulk_g2s(e_lo, reinterpret_cast<const unsigned char *>(prm.e_img) + part_bytes, part_bytes, &bar_e);
    }
    bool e_ok = false, e_waited = false;
    uint32_t mma_phase = 0, pf_phase = 0;
    bool mma_pending = false, pf_pending = false;
    const uint32_t idesc1 = make_idesc(kp, 0, 1);   // A K-major, B (E) MN-major
    const uint32_t idesc2 = make_idesc(kp, 0, 0);   // A K-major, B (E) K-major
    const uint32_t e_hi_a = smem_u32(e_hi), e_lo_a = smem_u32(e_lo);
    const uint32_t a_hi_a = smem_u32(a_hi), a_lo_a = smem_u32(a_lo);
    const int ksteps = kp >> 4;
    const int sj = tid % TR, sp = tid / TR;               // staging: channel, z-block phase

    // x (8 consecutive z of channel sj) as four 16-byte units of the K-major
    // A operand: re and im rows 2 sj and 2 sj + 1, hi and lo parts
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
        const uint32_t o_re = kmaj_off(2 * sj, zb * 8, ROWS), o_im = o_re + 16;
        *reinterpret_cast<uint4 *>(a_hi + o_re) = make_uint4(rh[0], rh[1], rh[2], rh[3]);
        *reinterpret_cast<uint4 *>(a_hi + o_im) = make_uint4(ih[0], ih[1], ih[2], ih[3]);
        *reinterpret_cast<uint4 *>(a_lo + o_re) = make_uint4(rl[0], rl[1], rl[2], rl[3]);
        *reinterpret_cast<uint4 *>(a_lo + o_im) = make_uint4(il[0], il[1], il[2], il[3]);
    };
    // The next tile's raw x rows (TR n complex FP32 = 8 TR n bytes, one
    // contiguous range of x, within the A buffer's 4 ROWS kp bytes) arrive by
    // one bulk copy once GEMM 2 has consumed the buffer.  Needs n even, x
    // 16-byte aligned and at most kMaxPf staging units per thread.
    constexpr int kMaxPf = 4;
    const int upt = (kb + P - 1) / P;
    const bool use_pf = (n % 2 == 0) && upt <= kMaxPf &&
                        (reinterpret_cast<uintptr_t>(prm.x) & 15u) == 0;
    float2 *raw = reinterpret_cast<float2 *>(a_hi);
    auto prefetch = [&](int t) {
        if (tid == 0) {
            const int r0 = t * TR, nr = min(TR, prm.rows - r0);
            const uint32_t bytes = (uint32_t)nr * (uint32_t)n * 8u;
            mbar_expect_tx(&bar_pf, bytes);
            bulk_g2s(raw, prm.x + (size_t)r0 * n, bytes, &bar_pf);
        }
        pf_pending = true;
    };
    auto find_active = [&](int t) {
        for (; t < prm.ntiles; t += gridDim.x) {
            if (!prm.gate) return t;
            const int r0 = t * TR, nr = min(TR, prm.rows - r0);
            const int s0 = prm.row_sys[r0], s1 = prm.row_sys[r0 + nr - 1];
            for (int q = s0; q <= s1; ++q)
                if (prm.gate[q]) return t;
        }
        return prm.ntiles;
    };
    if (tid == 0) next_s = find_active(blockIdx.x);
    __syncthreads();
    int tile = next_s;
    __syncthreads();            // every thread has read next_s before the loop rewrites it
    if (use_pf && tile < prm.ntiles) prefetch(tile);

    while (tile < prm.ntiles && ok) {
        const int row0 = tile * TR;
        const int nrow = min(TR, prm.rows - row0);
        for (int j = tid; j < TR; j += kThreads) {
            const bool in = j < nrow;
            pkd_s[j] = in ? prm.row_pkd[row0 + j] : 0.0;
            cf_s[j] = in ? prm.row_cf[row0 + j] : make_double2(0.0, 0.0);
        }

        // ---- stage x as the A operand of GEMM 1 (K-major: rows = 2 TR re/im, K = z)
        {
            const bool jok = sj < nrow;
            if (use_pf) {
                const bool got = mbar_wait(&bar_pf, pf_phase);
                if (!__syncthreads_and(got)) { ok = false; break; }   // the raw tile is complete
                pf_phase ^= 1u;
                pf_pending = false;
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
                __syncthreads();                       // raw reads done before A is overwritten
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
            if (!__syncthreads_and(e_ok)) { ok = false; break; }
        }
        __syncthreads();

        // ---- GEMM 1: D1[c, k] = sum_z x[c, z] E[z, k]   (M = 128 rows, N = kp, K = z)
        if (tid == 0) {
            tc_fence_after();
            for (int s = 0; s < ksteps; ++s) {
                // A (x, K-major): K 8-block stride a_lbo (LBO), row-block stride 128 (SBO)
                const uint64_t ah = make_desc(a_hi_a + (uint32_t)(2 * s) * a_lbo, a_lbo, 128);
                const uint64_t al = make_desc(a_lo_a + (uint32_t)(2 * s) * a_lbo, a_lbo, 128);
                // B (E, MN-major view, N = k): z-block stride sz (LBO), k-block stride sk (SBO)
                const uint64_t bh = make_desc(e_hi_a + (uint32_t)(2 * s) * sz, sz, sk);
                const uint64_t bl = make_desc(e_lo_a + (uint32_t)(2 * s) * sz, sz, sk);
                mma_bf16(d1, ah, bh, idesc1, s > 0 ? 1u : 0u);
                mma_bf16(d1, ah, bl, idesc1, 1u);
                mma_bf16(d1, al, bh, idesc1, 1u);
            }
            mma_commit(&bar_mma);
        }
        // the next active tile is found by warp 1 while the MMAs run; every
        // thread read next_s before the previous tile's last barrier
        if (tid == 32) next_s = find_active(tile + gridDim.x);
        mma_pending = true;
        if (mbar_wait(&bar_mma, mma_phase)) {
            mma_phase ^= 1u;
            mma_pending = false;
        } else {
            ok = false;
        }
        tc_fence_after();
        if (!__syncthreads_and(ok)) { ok = false; break; }

        const bool row_ok = jc < nrow;
        const int part = c & 1;
        const double pkd_j = pkd_s[jc];
        const uint32_t lane_base = (uint32_t)(lq * 32) << 16;

        // ---- epilogue 1a: Sherman-Morrison partial sums over this warp's
        // columns, s_c = sum_k en_k D1[c, k] / (pkd_j + lam_k)
        {
            // (the thread's sum runs in FP64: its ~kp/4 terms come in sequence,
            // not as a tree, and near a resonance of H0 + pkd they cancel)
            double sacc = 0.0;
            for (int q = ch0; q < ch1; ++q) {
                float v[16];
                tmem_ld16f(d1 + lane_base + (uint32_t)(16 * q), v);
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const int k = 16 * q + e;
                    // select, not multiply: columns past n carry nothing
                    if (k < n) sacc = fma((double)(en_s[k] * shifted_inverse(pkd_j, lam_s[k])), (double)v[e], sacc);
                }
            }
            sm_part[cg][c] = row_ok ? sacc : 0.0;
        }
        __syncthreads();
        for (int j = tid; j < TR; j += kThreads) {
            double2 b = make_double2(0.0, 0.0);
            if (j < nrow) {
                double sr = 0.0, si = 0.0;   // fixed summation order: deterministic
                for (int w = 0; w < 4; ++w) {
                    sr += sm_part[w][2 * j];
                    si += sm_part[w][2 * j + 1];
                }
                b = cmul(cf_s[j], make_double2(sr, si));
            }
            beta_s[j] = make_float2((float)b.x, (float)b.y);
        }
        __syncthreads();

        // ---- epilogue 1b: yt[c, k] = (D1[c, k] + beta_j en_k) / (pkd_j + lam_k)
        // as the K-major A operand of GEMM 2 (one row per thread, 8 k per
        // 16-byte unit; columns past n are zero)
        {
            const float bpart = part ? beta_s[jc].y : beta_s[jc].x;
            for (int q = ch0; q < ch1; ++q) {
                float v[16];
                tmem_ld16f(d1 + lane_base + (uint32_t)(16 * q), v);
                uint32_t hw[8], lw[8];
#pragma unroll
                for (int e = 0; e < 16; e += 2) {
                    const int k = 16 * q + e;
                    float y0 = 0.f, y1 = 0.f;
                    if (row_ok && k < n)
                        y0 = (v[e] + bpart * en_s[k]) * shifted_inverse(pkd_j, lam_s[k]);
                    if (row_ok && k + 1 < n)
                        y1 = (v[e + 1] + bpart * en_s[k + 1]) * shifted_inverse(pkd_j, lam_s[k + 1]);
                    const __nv_bfloat162 h = __floats2bfloat162_rn(y0, y1);
                    const float2 fh = __bfloat1622float2(h);
                    const __nv_bfloat162 l = __floats2bfloat162_rn(y0 - fh.x, y1 - fh.y);
                    hw[e >> 1] = *reinterpret_cast<const uint32_t *>(&h);
                    lw[e >> 1] = *reinterpret_cast<const uint32_t *>(&l);
                }
                const int k0 = 16 * q;
                const uint32_t o0 = kmaj_off(c, k0, ROWS), o1 = kmaj_off(c, k0 + 8, ROWS);
                *reinterpret_cast<uint4 *>(a_hi + o0) = make_uint4(hw[0], hw[1], hw[2], hw[3]);
                *reinterpret_cast<uint4 *>(a_hi + o1) = make_uint4(hw[4], hw[5], hw[6], hw[7]);
                *reinterpret_cast<uint4 *>(a_lo + o0) = make_uint4(lw[0], lw[1], lw[2], lw[3]);
                *reinterpret_cast<uint4 *>(a_lo + o1) = make_uint4(lw[4], lw[5], lw[6], lw[7]);
            }
        }
        tc_fence_before();
        fence_proxy_async();
        __syncthreads();

        // ---- GEMM 2: D2[c, z] = sum_k yt[c, k] E[z, k]   (M = 128 rows, N = kp, K = k)
        if (tid == 0) {
            tc_fence_after();
            for (int s = 0; s < ksteps; ++s) {
                const uint64_t ah = make_desc(a_hi_a + (uint32_t)(2 * s) * a_lbo, a_lbo, 128);
                const uint64_t al = make_desc(a_lo_a + (uint32_t)(2 * s) * a_lbo, a_lbo, 128);
                // B (E, K-major view, N = z): k-block stride sk (LBO), z-block stride sz (SBO)
                const uint64_t bh = make_desc(e_hi_a + (uint32_t)(2 * s) * sk, sk, sz);
                const uint64_t bl = make_desc(e_lo_a + (uint32_t)(2 * s) * sk, sk, sz);
                mma_bf16(d2, ah, bh, idesc2, s > 0 ? 1u : 0u);
                mma_bf16(d2, ah, bl, idesc2, 1u);
                mma_bf16(d2, al, bh, idesc2, 1u);
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
        // the A buffer is free: start the next tile's copy
        const int next = next_s;
        if (use_pf && next < prm.ntiles) prefetch(next);

        // ---- epilogue 2: u rows to global.  Lanes 2i and 2i + 1 hold the re
        // and im rows of one channel; one shuffle per pair of values gives
        // each lane 8 complex values of consecutive z (the even lane the
        // chunk's first half), stored as 16-byte pairs where aligned.
        {
            const bool odd = lane & 1;
            float2 *orow = prm.out + (size_t)(row0 + jc) * n;
            const bool pairs = (n % 2 == 0) && (reinterpret_cast<uintptr_t>(prm.out) & 15u) == 0;
            for (int q = ch0; q < ch1; ++q) {
                float v[16];
                tmem_ld16f(d2 + lane_base + (uint32_t)(16 * q), v);
                float2 o[8];
#pragma unroll
                for (int i = 0; i < 8; ++i) {
                    const float send = odd ? v[i] : v[8 + i];
                    const float recv = __shfl_xor_sync(0xffffffffu, send, 1);
                    o[i] = odd ? make_float2(recv, v[8 + i]) : make_float2(v[i], recv);
                }
                const int zb = 16 * q + (odd ? 8 : 0);
                if (!row_ok) continue;
                if (pairs) {
#pragma unroll
                    for (int i = 0; i < 8; i += 2)
                        if (zb + i < n)
                            *reinterpret_cast<float4 *>(orow + zb + i) =
                                make_float4(o[i].x, o[i].y, o[i + 1].x, o[i + 1].y);
                } else {
#pragma unroll
                    for (int i = 0; i < 8; ++i)
                        if (zb + i < n) orow[zb + i] = o[i];
                }
            }
        }
        tc_fence_before();
        __syncthreads();
        tile = next;
    }

    if (!ok && tid == 0 && prm.error) atomicExch(prm.error, 1);
    // Drain on a time-out: no copy may land and no MMA may write after the
    // kernel frees its TMEM and leaves (each wait bounded).
    if (tid == 0 && pf_pending) (void)mbar_wait(&bar_pf, pf_phase);
    if (tid == 0 && !e_ok) (void)mbar_wait(&bar_e, 0);
    if (tid == 0 && mma_pending) (void)mbar_wait(&bar_mma, mma_phase);
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    if (warp == 0) tmem_dealloc(tmem_base_s, 512);
}

}  // namespace tc
}  // namespace msc
