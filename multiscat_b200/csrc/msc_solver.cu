// msc_solver.cu -- plan, restarted GMRES orchestration and the C-ABI.
//
// One plan = one potential (z grid, coupling torus) + a batch of beams
// (systems).  The solve is right-preconditioned restarted GMRES(m):
//     A M y = b,  psi = M y,  M = D^-1 (block-diagonal, per channel)
// in FP64.  Each restart cycle recomputes the true residual b - A psi, so
// the stop rule ||b - A psi|| <= rtol ||b|| is checked on the real operator.
// The reference solves the same A psi = b with block Gauss-Seidel left
// preconditioning and unrestarted MGS GMRES
// (multiscat_gmres.f90:452-618); the converged psi is the same.
//
// Execution: one CUDA graph per restart cycle start (true residual + norm)
// and one for the m Arnoldi steps + solution update.  Per-system activity
// flags live on the device, so systems that converge early stop doing work
// while the rest of the batch carries on.  The host reads one counter per
// cycle.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <tuple>
#include <map>
#include <mutex>
#include <new>
#include <numeric>
#include <string>
#include <type_traits>
#include <vector>

#include "../../include/multiscat_b200.h"
#include "msc_common.cuh"
#include "msc_eigh.hpp"
#include "msc_eigh_gpu.cuh"
#include "msc_kernels.cuh"
#include "msc_tc.cuh"
#include "msc_tcc.cuh"

namespace {

thread_local std::string g_last_error;

msc_status fail(msc_status st, const std::string &msg)
{
    g_last_error = msg;
    return st;
}

#define MSC_CUDA(call)                                                                  \
    do {                                                                                \
        cudaError_t _e = (call);                                                        \
        if (_e != cudaSuccess) {                                                        \
            return fail(MSC_ERR_CUDA, std::string(#call) + ": " + cudaGetErrorString(_e)); \
        }                                                                               \
    } while (0)

// Plan memory comes from a memory pool owned by the library, one per device.
// A destroyed plan's buffers go back to the pool and later plans reuse them
// without cudaMalloc / cudaFree (a multi-GB cudaFree synchronises the device
// and unmaps, tens of ms); up to kPoolKeepBytes of unused memory stays
// reserved until msc_release_cached_memory.
constexpr int kPoolMaxDevices = 64;
constexpr uint64_t kPoolKeepBytes = 32ull << 30;
std::mutex g_pool_mutex;
cudaMemPool_t g_pool[kPoolMaxDevices] = {};

cudaError_t plan_pool(cudaMemPool_t *out)
{
    int dev = -1;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= kPoolMaxDevices) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lock(g_pool_mutex);
    if (!g_pool[dev]) {
        cudaMemPoolProps props{};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = dev;
        cudaMemPool_t pool;
        e = cudaMemPoolCreate(&pool, &props);
        if (e != cudaSuccess) return e;
        uint64_t keep = kPoolKeepBytes;
        e = cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (e != cudaSuccess) return e;
        g_pool[dev] = pool;
    }
    *out = g_pool[dev];
    return cudaSuccess;
}

template <typename T>
struct DevBuf {
    T *p = nullptr;
    size_t count = 0;
    // Allocation and release are ordered on the legacy stream; alloc waits
    // for the allocation, and the plan synchronises the device before it
    // releases anything that work may still use.
    cudaError_t alloc(size_t c)
    {
        release();
        count = c;
        if (c == 0) return cudaSuccess;
        cudaMemPool_t pool;
        cudaError_t e = plan_pool(&pool);
        if (e != cudaSuccess) return e;
        e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&p), c * sizeof(T), pool, 0);
        if (e != cudaSuccess) {
            p = nullptr;
            count = 0;
            return e;
        }
        // Debugging aid: MSC_POISON_ALLOC=1 fills new buffers with 0xFF bytes
        // (NaN in FP32 and FP64) so that a read of an unwritten element shows.
        static const bool poison = [] {
            const char *v = std::getenv("MSC_POISON_ALLOC");
            return v && v[0] == '1';
        }();
        if (poison) {
            e = cudaMemsetAsync(p, 0xff, c * sizeof(T), 0);
            if (e != cudaSuccess) return e;
        }
        return cudaStreamSynchronize(0);
    }
    void release()
    {
        if (p) cudaFreeAsync(p, 0);
        p = nullptr;
        count = 0;
    }
};

struct SystemHost {
    int C = 0;
    int spec = 0;
    std::vector<int> ix, iy;
    std::vector<double> pkd;
    std::vector<double2> b, c;
    double2 a_spec{0.0, 0.0};
    bool set = false;
};

}  // namespace

struct msc_plan {
    msc_plan_desc desc{};
    int n = 0, nkx = 0, nky = 0, B = 0, m = 30;
    bool potential_set = false;
    bool finalized = false;
    // potential
    std::vector<double> T_host, v00_host, lam_host, E_host, en_host;
    std::vector<std::pair<int, int>> taps;     // (dx, dy) storage offsets
    std::vector<double2> Vt_host;              // [K][n]
    std::vector<double2> Vt_adj_host;          // [K][n] taps of A^H: conj(V_{-d}) at offset d
    int K = 0;
    bool adjoint = false;                      // operator in use: A (false) or A^H (true)
    std::vector<SystemHost> sys;
    // rows / tiles
    int R = 0, ntiles = 0;
    std::vector<int> tile_row0_h, tile_nrow_h, tile_sys_h, sys_tile0_h, sys_row0_h, row_sys_h;
    // device data
    DevBuf<double> E, ET, Tm, lam, en, v00, row_pkd, row_fn;
    DevBuf<double2> Vt, row_c, row_b, row_rhs, sys_aspec;
    DevBuf<double2> row_cf;        // c / (1 - c f_n) per row (tcgen05 block inverse)
    std::vector<double2> row_c_h, rhs_default_h;   // c per row; default right-hand side
    DevBuf<int> row_pos, pos_map;                  // [R] torus position; [B][nkx*nky] row or -1
    DevBuf<int> sys_row0;                          // [B + 1] first row of each system
    DevBuf<int> nbr, tile_row0, tile_nrow, tile_sys, sys_tile0, sys_spec_row, row_sys;
    // solver state
    DevBuf<double2> X, W, U, TMP, Q, partial;
    DevBuf<double2> H, cs, sn, g, h1, h2, y;
    DevBuf<double2> Hraw, dsum, dcoef, gsave;   // DCGS2 Arnoldi step (see k_dcgs_reduce)
    // block Gauss-Seidel (flags bit 5, and the lower-block entry points):
    // level sets of every system's rows (k_gs_sweep)
    bool gs = false;
    bool gs_ready = false;
    bool gs_e64_smem = false, gs_e32_smem = false;   // E held in the sweep's shared memory
    DevBuf<int> gs_sys_lvl, gs_lvl_start, gs_lvl_rows, gs_low_ptr, gs_low_tap, gs_low_row;
    bool dcgs = true;              // DCGS2 (two basis passes per step); false: CGS2
    // FP32 DCGS2 passes streaming the basis by bulk copies: 2 reduction and
    // update, 1 reduction only, 0 neither
    int bulk_arnoldi = 0;
    DevBuf<int> wait_error;        // set by a kernel whose bounded wait timed out
    DevBuf<double> scale, bnorm, resid, est, beta0;
    // mixed form: FP32 copies of the operator data and the FP32 Krylov space
    bool mixed = false;
    bool cgs1_inner = false;       // single Gram-Schmidt pass in the FP32 inner solve
    double inner_rtol = 0.0;
    int max_cycles = 0;
    DevBuf<float> E32, ET32, lam32, en32, row_pkd32, row_fn32;
    DevBuf<float2> Vt32, row_c32, Q32, W32, U32, T32;
    DevBuf<double2> T64;            // von Neumann preconditioner term (order > 0)
    DevBuf<double2> X0;             // initial guess of the next solve (warm start)
    bool has_x0 = false;
    DevBuf<double2> R64;
    // tcgen05 block inverse (mixed form)
    bool use_tc = false;
    int tc_n = 0, tc_tile_rows = 0, tc_ntiles = 0, tc_grid = 0;
    int tc_groups = 1;          // warp groups with their own tile loop (1 or 2), or
                                // kTcChannelMajor: k_block_inverse_tcc
    int tc2_max = 0;            // widest N the two-group kernel may take (0: none)
    size_t tc_smem = 0, tc2_smem = 0;
    bool tcc_ok = false;        // the channel-major kernel fits (E and one A buffer)
    size_t tcc_smem = 0;
    DevBuf<__nv_bfloat16> e_img;
    DevBuf<int> tc_error;
    DevBuf<int> active, kcyc, iters, projv, cycles, unfinished, status, counter;
    int *counter_host = nullptr;   // pinned
    // Arnoldi blocks: runs of rows of one system ("chunks", first projection)
    // and row tiles split `split` ways (update + second projection)
    int nchunks = 0;
    int split = 1;
    DevBuf<int> chunk_row0, chunk_nrow, chunk_sys, sys_chunk0;
    // halo-tiled coupling
    bool use_halo = false;             // halo tables built (taps reach <= 8)
    int halo32 = 0, halo64 = 0;    // autotuned coupling kind per precision (0 nbr, 1/2 halo)
    int halo_hx = 0, halo_hy = 0, nwork = 0;
    // separable coupling (coupling kind 3): p, q, kappa per z when every tap
    // window factorises (see k_coupling_sep); host copies for the adjoint
    bool sep_ok = false;
    std::vector<double2> sep_p_h, sep_q_h, sep_k_h;   // [2hx+1][n], [2HY+1][n], [n]
    DevBuf<double2> sep64;                           // p | q | kappa
    DevBuf<float2> sep32;
    // autotuning record: microseconds per candidate
    std::vector<std::pair<std::string, float>> tune_log;
    std::string tune_report;
    DevBuf<int> work, tap_window;
    DevBuf<int2> taps_d;                      // [K] tap offsets (dx, dy)
    DevBuf<int> sys_counter;       // per-system arrival counters of the fused Arnoldi kernels
    cudaStream_t stream = nullptr;
    cudaGraphExec_t g_start = nullptr, g_start0 = nullptr, g_iter = nullptr;
    int pstride = 0;
    // measurement
    bool timing = false;
    static constexpr int kKinds = 5;      // block inverse, coupling, projection 1, projection 2, normalize
    std::vector<cudaEvent_t> tev;        // [kKinds][m + 1 slots][start, stop]
    double t_ms[kKinds] = {};
    int64_t t_launches[kKinds] = {};
    int *kcyc_host = nullptr;            // pinned [B]
    int64_t launches_last = 0;
    int cycles_last = 0;
    int fallbacks_last = 0;              // systems re-solved in FP64 by the last msc_solve
    int64_t launches_start = 0, launches_start0 = 0, launches_iter = 0;   // kernel nodes per graph

    ~msc_plan()
    {
        if (g_start) cudaGraphExecDestroy(g_start);
        if (g_start0) cudaGraphExecDestroy(g_start0);
        if (g_iter) cudaGraphExecDestroy(g_iter);
        if (counter_host) cudaFreeHost(counter_host);
        if (kcyc_host) cudaFreeHost(kcyc_host);
        for (cudaEvent_t e : tev) cudaEventDestroy(e);
        if (stream) cudaStreamDestroy(stream);
        E.release(); ET.release(); Tm.release(); lam.release(); en.release(); v00.release();
        row_pkd.release(); row_fn.release(); Vt.release(); row_c.release(); row_b.release();
        row_cf.release();
        row_rhs.release(); sys_aspec.release(); row_pos.release(); pos_map.release();
        sys_row0.release(); nbr.release(); tile_row0.release();
        tile_nrow.release(); tile_sys.release(); sys_tile0.release(); sys_spec_row.release();
        chunk_row0.release(); chunk_nrow.release(); chunk_sys.release(); sys_chunk0.release();
        row_sys.release(); X.release(); W.release(); U.release(); TMP.release(); Q.release();
        partial.release(); H.release(); cs.release(); sn.release(); g.release(); h1.release();
        h2.release(); y.release(); scale.release(); bnorm.release(); resid.release();
        est.release(); active.release(); kcyc.release(); iters.release(); projv.release();
        cycles.release();
        unfinished.release(); status.release(); counter.release(); beta0.release();
        sys_counter.release(); work.release(); tap_window.release(); taps_d.release();
        E32.release(); ET32.release(); lam32.release(); en32.release(); row_pkd32.release();
        row_fn32.release(); Vt32.release(); row_c32.release(); Q32.release(); W32.release();
        T32.release(); T64.release(); X0.release();
        U32.release(); R64.release(); e_img.release(); tc_error.release(); wait_error.release();
        Hraw.release(); dsum.release(); dcoef.release(); gsave.release();
        gs_sys_lvl.release(); gs_lvl_start.release(); gs_lvl_rows.release();
        gs_low_ptr.release(); gs_low_tap.release(); gs_low_row.release();
        sep64.release(); sep32.release();
    }

    msc::Tiles tiles() const
    {
        return msc::Tiles{tile_row0.p, tile_nrow.p, tile_sys.p, ntiles};
    }
    msc::Tiles chunks() const
    {
        return msc::Tiles{chunk_row0.p, chunk_nrow.p, chunk_sys.p, nchunks};
    }
    msc::GmresState state() const
    {
        msc::GmresState s;
        s.H = H.p; s.cs = cs.p; s.sn = sn.p; s.g = g.p; s.h1 = h1.p; s.h2 = h2.p; s.y = y.p;
        s.scale = scale.p; s.bnorm = bnorm.p; s.resid = resid.p; s.est = est.p; s.beta0 = beta0.p;
        s.active = active.p; s.kcyc = kcyc.p; s.iters = iters.p; s.projv = projv.p;
        s.cycles = cycles.p;
        s.unfinished = unfinished.p; s.status = status.p; s.counter = counter.p;
        return s;
    }
    msc::DcgsState dstate() const
    {
        msc::DcgsState d;
        d.Hraw = Hraw.p; d.dsum = dsum.p; d.coef = dcoef.p; d.gsave = gsave.p;
        d.cstride = 2 * m + 4;
        return d;
    }
};

namespace {

template <typename T>
cudaError_t upload(DevBuf<T> &buf, const std::vector<T> &h)
{
    cudaError_t e = buf.alloc(h.size());
    if (e != cudaSuccess) return e;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpy(buf.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

// Overwrite an allocated buffer in place (device pointers captured in the
// solve graphs stay valid).
template <typename T>
cudaError_t refill(DevBuf<T> &buf, const std::vector<T> &h)
{
    if (h.size() != buf.count) return cudaErrorInvalidValue;
    if (h.empty()) return cudaSuccess;
    return cudaMemcpy(buf.p, h.data(), h.size() * sizeof(T), cudaMemcpyHostToDevice);
}

int block_inverse_rows(int n) { return n <= msc::kWideNz ? 8 : 4; }
size_t smem_block_inverse(int n) { return (size_t)2 * n * 2 * block_inverse_rows(n) * sizeof(double); }
void launch_block_inverse(msc_plan *p, const int *gate, const double2 *x, double2 *out, int acc,
                          cudaStream_t st);
size_t smem_residual(int n) { return (size_t)n * 2 * msc::kTileRows * sizeof(double); }
size_t smem_coupling(int K) { return (size_t)msc::kTileRows * K * sizeof(int); }

// --- kernel launch wrappers ---------------------------------------------------

template <typename R>
struct OpData;   // operator data of one precision

template <>
struct OpData<double> {
    static const double *E(msc_plan *p) { return p->E.p; }
    static const double *ET(msc_plan *p) { return p->ET.p; }
    static const double *lam(msc_plan *p) { return p->lam.p; }
    static const double *en(msc_plan *p) { return p->en.p; }
    static const double *pkd(msc_plan *p) { return p->row_pkd.p; }
    static const double *fn(msc_plan *p) { return p->row_fn.p; }
    static const double2 *c(msc_plan *p) { return p->row_c.p; }
    static const double2 *Vt(msc_plan *p) { return p->Vt.p; }
};

template <>
struct OpData<float> {
    static const float *E(msc_plan *p) { return p->E32.p; }
    static const float *ET(msc_plan *p) { return p->ET32.p; }
    static const float *lam(msc_plan *p) { return p->lam32.p; }
    static const float *en(msc_plan *p) { return p->en32.p; }
    static const float *pkd(msc_plan *p) { return p->row_pkd32.p; }
    static const float *fn(msc_plan *p) { return p->row_fn32.p; }
    static const float2 *c(msc_plan *p) { return p->row_c32.p; }
    static const float2 *Vt(msc_plan *p) { return p->Vt32.p; }
};

template <typename R>
using C2 = typename msc::CT<R>::t;

template <typename R>
size_t smem_block_inverse_t(int n) { return (size_t)2 * n * 2 * block_inverse_rows(n) * sizeof(R); }

// tc_groups code of the channel-major tcgen05 kernel (k_block_inverse_tcc)
constexpr int kTcChannelMajor = 3;

void launch_block_inverse_tc(msc_plan *p, const int *gate, const float2 *x, float2 *out,
                             cudaStream_t st)
{
    msc::tc::TcParams prm;
    prm.n = p->n;
    prm.kp = (p->n + 15) / 16 * 16;
    prm.mt = (p->n + 127) / 128;
    prm.rows = p->R;
    prm.tile_rows = p->tc_tile_rows;
    prm.ntiles = p->tc_ntiles;
    prm.e_img = p->e_img.p;
    prm.lam = p->lam.p;
    prm.en = p->en.p;
    prm.row_pkd = p->row_pkd.p;
    prm.row_cf = p->row_cf.p;
    prm.row_sys = p->row_sys.p;
    prm.gate = gate;
    prm.x = x;
    prm.out = out;
    prm.error = p->tc_error.p;
    using msc::tc::k_block_inverse_tc;
    constexpr int T = msc::tc::kThreads;
    if (p->tc_groups == kTcChannelMajor) {
        msc::tc::k_block_inverse_tcc<<<p->tc_grid, T, p->tcc_smem, st>>>(prm);
        return;
    }
    if (p->tc_groups == 2) {
        const size_t sm = p->tc2_smem;
        switch (p->tc_n) {
        case 16: k_block_inverse_tc<16, 2><<<p->tc_grid, T, sm, st>>>(prm); break;
        case 32: k_block_inverse_tc<32, 2><<<p->tc_grid, T, sm, st>>>(prm); break;
        case 64: k_block_inverse_tc<64, 2><<<p->tc_grid, T, sm, st>>>(prm); break;
        default: k_block_inverse_tc<128, 2><<<p->tc_grid, T, sm, st>>>(prm); break;
        }
        return;
    }
    const size_t sm = p->tc_smem;
    switch (p->tc_n) {
    case 16: k_block_inverse_tc<16, 1><<<p->tc_grid, T, sm, st>>>(prm); break;
    case 32: k_block_inverse_tc<32, 1><<<p->tc_grid, T, sm, st>>>(prm); break;
    case 64: k_block_inverse_tc<64, 1><<<p->tc_grid, T, sm, st>>>(prm); break;
    case 128: k_block_inverse_tc<128, 1><<<p->tc_grid, T, sm, st>>>(prm); break;
    default: k_block_inverse_tc<256, 1><<<p->tc_grid, T, sm, st>>>(prm); break;
    }
}

template <typename R>
void launch_block_inverse_t(msc_plan *p, const int *gate, const C2<R> *x, C2<R> *out, int acc,
                            cudaStream_t st)
{
    using D = OpData<R>;
    if constexpr (std::is_same<R, float>::value) {
        if (p->use_tc && !acc) {
            launch_block_inverse_tc(p, gate, x, out, st);
            return;
        }
    }
    if (block_inverse_rows(p->n) == 8)
        msc::k_block_inverse<8, R><<<p->ntiles, 256, smem_block_inverse_t<R>(p->n), st>>>(
            p->tiles(), gate, p->n, D::E(p), D::ET(p), p->lam.p, p->en.p, p->row_pkd.p,
            p->row_c.p, p->row_fn.p, x, out, acc);
    else
        msc::k_block_inverse<4, R><<<p->ntiles, 256, smem_block_inverse_t<R>(p->n), st>>>(
            p->tiles(), gate, p->n, D::E(p), D::ET(p), p->lam.p, p->en.p, p->row_pkd.p,
            p->row_c.p, p->row_fn.p, x, out, acc);
}

void launch_block_inverse(msc_plan *p, const int *gate, const double2 *x, double2 *out, int acc,
                          cudaStream_t st)
{
    launch_block_inverse_t<double>(p, gate, x, out, acc, st);
}

void launch_residual_diag(msc_plan *p, const int *gate, const double2 *x, double2 *out, int with_b,
                          cudaStream_t st)
{
    const int nt = 2 * p->n <= 512 ? (2 * p->n + 31) / 32 * 32 : 256;
    msc::k_residual_diag<<<p->ntiles, nt, smem_residual(p->n), st>>>(
        p->tiles(), gate, p->n, p->Tm.p, p->v00.p, p->row_pkd.p, p->row_c.p, p->row_rhs.p, x, out,
        with_b);
}

constexpr int kHaloBX = 8;
template <typename R> constexpr int halo_zc() { return std::is_same<R, float>::value ? 32 : 16; }

size_t halo_smem(int hx, int hy, int zc, size_t elem)
{
    return (size_t)(kHaloBX + 2 * hx) * (8 + 2 * hy) * zc * elem +
           (size_t)(2 * hx + 1) * (2 * hy + 1) * zc * elem +
           (size_t)(kHaloBX + 2 * hx) * (8 + 2 * hy) * sizeof(int);
}

template <int HY, int YS, typename R, int MASK = 0>
void launch_halo(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                 C2<R> *out, cudaStream_t st)
{
    constexpr int ZC = halo_zc<R>();
    msc::CouplingTiles ct{p->work.p, p->pos_map.p, p->tap_window.p, p->nwork, p->nkx, p->nky,
                          p->halo_hx, p->K};
    dim3 grid(p->nwork, (p->n + ZC - 1) / ZC);
    msc::k_coupling_halo<HY, kHaloBX, ZC, YS, R, MASK>
        <<<grid, kHaloBX * ZC * (8 / YS), halo_smem(p->halo_hx, HY, ZC, sizeof(C2<R>)), st>>>(
            ct, gate, p->n, OpData<R>::Vt(p), src, in0, sgn, out);
}

template <int YS, typename R, int MASK = 0>
void launch_halo_ys(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                    C2<R> *out, cudaStream_t st)
{
    switch (p->halo_hy) {
    case 1: launch_halo<1, YS, R, MASK>(p, gate, src, in0, sgn, out, st); return;
    case 2: launch_halo<2, YS, R, MASK>(p, gate, src, in0, sgn, out, st); return;
    case 4: launch_halo<4, YS, R, MASK>(p, gate, src, in0, sgn, out, st); return;
    default: launch_halo<8, YS, R, MASK>(p, gate, src, in0, sgn, out, st); return;
    }
}

size_t sep_smem(int hx, int hy, int zc, size_t elem)
{
    const size_t hxw = kHaloBX + 2 * hx, hyw = 8 + 2 * hy;
    return (hxw * hyw + (2 * hx + 1) + (2 * hy + 1) + 1) * zc * elem + hxw * hyw * sizeof(int);
}

template <int HY, int ZC, typename R>
void launch_sep(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                C2<R> *out, cudaStream_t st)
{
    msc::CouplingTiles ct{p->work.p, p->pos_map.p, p->tap_window.p, p->nwork, p->nkx, p->nky,
                          p->halo_hx, p->K};
    const size_t np = (size_t)(2 * p->halo_hx + 1) * p->n, nq = (size_t)(2 * p->halo_hy + 1) * p->n;
    const C2<R> *base = std::is_same<R, float>::value
                            ? reinterpret_cast<const C2<R> *>(p->sep32.p)
                            : reinterpret_cast<const C2<R> *>(p->sep64.p);
    const msc::SepTaps sep{base, base + np, base + np + nq};
    dim3 grid(p->nwork, (p->n + ZC - 1) / ZC);
    const size_t sm = sep_smem(p->halo_hx, HY, ZC, sizeof(C2<R>));
    if (p->halo_hx == HY)       // square window: the x reach at compile time
        msc::k_coupling_sep<HY, kHaloBX, ZC, R, HY><<<grid, kHaloBX * ZC, sm, st>>>(
            ct, gate, p->n, sep, src, in0, sgn, out);
    else
        msc::k_coupling_sep<HY, kHaloBX, ZC, R><<<grid, kHaloBX * ZC, sm, st>>>(
            ct, gate, p->n, sep, src, in0, sgn, out);
}

// The row-wise separable kernel: square windows (hx = hy), x reach as a
// template parameter.
bool sep_rows_ok(const msc_plan *p)
{
    return p->sep_ok && p->halo_hx == p->halo_hy &&
           (p->halo_hx == 1 || p->halo_hx == 2 || p->halo_hx == 4 || p->halo_hx == 8);
}

template <int H, typename R>
void launch_sep_rows_h(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                       C2<R> *out, cudaStream_t st)
{
    constexpr int ZC = halo_zc<R>();
    msc::CouplingTiles ct{p->work.p, p->pos_map.p, p->tap_window.p, p->nwork, p->nkx, p->nky,
                          p->halo_hx, p->K};
    const size_t np = (size_t)(2 * H + 1) * p->n, nq = (size_t)(2 * H + 1) * p->n;
    const C2<R> *base = std::is_same<R, float>::value
                            ? reinterpret_cast<const C2<R> *>(p->sep32.p)
                            : reinterpret_cast<const C2<R> *>(p->sep64.p);
    const msc::SepTaps sep{base, base + np, base + np + nq};
    dim3 grid(p->nwork, (p->n + ZC - 1) / ZC);
    msc::k_coupling_sep_rows<H, kHaloBX, ZC, R, H>
        <<<grid, kHaloBX * ZC, sep_smem(H, H, ZC, sizeof(C2<R>)), st>>>(ct, gate, p->n, sep, src,
                                                                        in0, sgn, out);
}

template <typename R>
void launch_sep_rows(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                     C2<R> *out, cudaStream_t st)
{
    switch (p->halo_hx) {
    case 1: launch_sep_rows_h<1, R>(p, gate, src, in0, sgn, out, st); return;
    case 2: launch_sep_rows_h<2, R>(p, gate, src, in0, sgn, out, st); return;
    case 4: launch_sep_rows_h<4, R>(p, gate, src, in0, sgn, out, st); return;
    default: launch_sep_rows_h<8, R>(p, gate, src, in0, sgn, out, st); return;
    }
}

// ZC: z values per block (the halo kernel's, or half of it: half the shared
// memory, twice the resident blocks to hide the halo loads)
template <int ZC, typename R>
void launch_sep_hy(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                   C2<R> *out, cudaStream_t st)
{
    switch (p->halo_hy) {
    case 1: launch_sep<1, ZC, R>(p, gate, src, in0, sgn, out, st); return;
    case 2: launch_sep<2, ZC, R>(p, gate, src, in0, sgn, out, st); return;
    case 4: launch_sep<4, ZC, R>(p, gate, src, in0, sgn, out, st); return;
    default: launch_sep<8, ZC, R>(p, gate, src, in0, sgn, out, st); return;
    }
}

template <typename R>
void launch_coupling_t(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0, R sgn,
                       C2<R> *out, cudaStream_t st)
{
    // coupling kind per precision: 0 neighbour table, 1 halo (8 y/thread), 2 halo (4 y/thread),
    // 3 separable (two 1-D passes; only when the tap windows factorise),
    // 4 separable with half the z per block, 5 separable with the x pass
    // along the halo rows (square windows; otherwise the column form)
    const int kind = p->use_halo ? (std::is_same<R, float>::value ? p->halo32 : p->halo64) : 0;
    if (kind == 5 && p->sep_ok) {
        if (sep_rows_ok(p)) launch_sep_rows<R>(p, gate, src, in0, sgn, out, st);
        else launch_sep_hy<halo_zc<R>(), R>(p, gate, src, in0, sgn, out, st);
        return;
    }
    if (kind == 1) { launch_halo_ys<8, R>(p, gate, src, in0, sgn, out, st); return; }
    if (kind == 2) { launch_halo_ys<4, R>(p, gate, src, in0, sgn, out, st); return; }
    if (kind == 3 && p->sep_ok) {
        launch_sep_hy<halo_zc<R>(), R>(p, gate, src, in0, sgn, out, st);
        return;
    }
    if (kind == 4 && p->sep_ok) {
        launch_sep_hy<halo_zc<R>() / 2, R>(p, gate, src, in0, sgn, out, st);
        return;
    }

    dim3 grid(p->ntiles, (p->n + 31) / 32);
    dim3 block(32, msc::kTileRows);
    msc::k_coupling<R><<<grid, block, smem_coupling(std::max(p->K, 1)), st>>>(
        p->tiles(), gate, p->n, p->K, OpData<R>::Vt(p), p->nbr.p, src, in0, sgn, out);
}

void launch_coupling(msc_plan *p, const int *gate, const double2 *src, const double2 *in0,
                     double sgn, double2 *out, cudaStream_t st)
{
    launch_coupling_t<double>(p, gate, src, in0, sgn, out, st);
}

// Lower (mask 1) or upper (mask 2) part of the coupling in plan row order:
// the halo kernel with the row test when the plan has halo tables, else
// the neighbour table.
template <typename R>
void launch_coupling_masked_t(msc_plan *p, const int *gate, const C2<R> *src, const C2<R> *in0,
                              R sgn, int mask, C2<R> *out, cudaStream_t st)
{
    if (p->use_halo) {
        if (mask == 1) launch_halo_ys<4, R, 1>(p, gate, src, in0, sgn, out, st);
        else launch_halo_ys<4, R, 2>(p, gate, src, in0, sgn, out, st);
        return;
    }
    dim3 grid(p->ntiles, (p->n + 31) / 32);
    dim3 block(32, msc::kTileRows);
    msc::k_coupling_masked<R><<<grid, block, smem_coupling(std::max(p->K, 1)), st>>>(
        p->tiles(), gate, p->n, p->K, OpData<R>::Vt(p), p->nbr.p, src, in0, sgn, mask, out);
}

// Shared memory of the Gauss-Seidel sweep: E with row stride n + 1 when
// e_in_smem, then the s and t buffers of kGsRows rows.
template <typename R>
size_t gs_smem(int n, bool e_in_smem)
{
    const size_t e = e_in_smem ? ((size_t)n * (n + 1) * sizeof(R) + 15) / 16 * 16 : 0;
    return e + 2 * (size_t)msc::kGsRows * n * sizeof(C2<R>);
}

// y = L^-1 x (block Gauss-Seidel forward sweep), one CTA per system.
template <typename R>
void launch_gs_sweep_t(msc_plan *p, const int *gate, const C2<R> *x, C2<R> *y, cudaStream_t st)
{
    const msc::GsLevels lv{p->gs_sys_lvl.p, p->gs_lvl_start.p, p->gs_lvl_rows.p,
                           p->gs_low_ptr.p, p->gs_low_tap.p, p->gs_low_row.p};
    const bool es = std::is_same<R, float>::value ? p->gs_e32_smem : p->gs_e64_smem;
    msc::k_gs_sweep<R><<<p->B, 256, gs_smem<R>(p->n, es), st>>>(
        p->B, gate, p->n, p->K, OpData<R>::Vt(p), p->nbr.p, lv, OpData<R>::E(p), es ? 1 : 0,
        p->lam.p, p->en.p, p->row_pkd.p, p->row_c.p, p->row_fn.p, x, y);
}

template <typename R>
void launch_dots_t(msc_plan *p, const int *gate, const C2<R> *Q, int nvec, const C2<R> *W,
                   int with_norm, cudaStream_t st)
{
    msc::k_dots<R><<<p->ntiles, 256, 0, st>>>(p->tiles(), gate, p->n, Q, (size_t)p->R * p->n, nvec,
                                               W, with_norm, p->partial.p, p->pstride);
}

void launch_reduce(msc_plan *p, const int *gate, int nslot, double2 *out, cudaStream_t st)
{
    msc::k_reduce_partials<<<p->B, 256, 0, st>>>(p->sys_tile0.p, p->B, gate, p->partial.p,
                                                  p->pstride, nslot, out, p->m + 2);
}

dim3 elementwise_grid(msc_plan *p)
{
    return dim3(p->ntiles, (msc::kTileRows * p->n + 255) / 256);
}

template <typename R>
void launch_update_t(msc_plan *p, const int *gate, const C2<R> *Q, int nvec, const int *nvec_sys,
                     const double2 *coef, int cstride, const C2<R> *W, const double *scale,
                     C2<R> *dst, int sum_only, cudaStream_t st)
{
    // one block per row chunk of one system (~4096 elements)
    msc::k_update<R><<<dim3(p->nchunks, 1), 256, 0, st>>>(p->chunks(), gate, p->n, Q,
                                                          (size_t)p->R * p->n, nvec, nvec_sys,
                                                          coef, cstride, W, scale, dst, sum_only);
}

void launch_update(msc_plan *p, const int *gate, int nvec, const int *nvec_sys,
                   const double2 *coef, int cstride, const double2 *W, const double *scale,
                   double2 *dst, int sum_only, cudaStream_t st)
{
    launch_update_t<double>(p, gate, p->Q.p, nvec, nvec_sys, coef, cstride, W, scale, dst,
                            sum_only, st);
}

int sys_blocks(int B) { return (B + 127) / 128; }

// Shared scratch of the register-streamed DCGS2 passes' last-block work.
size_t dcgs_scratch_bytes(int m) { return (size_t)msc::dcgs_block_scratch(m) * sizeof(double2); }
size_t dcgs_update_scratch_bytes(int m) { return (size_t)(5 * m + 3) * sizeof(double2); }

// Block layout of an Arnoldi kernel: large row chunks (P1) or row tiles
// split into about 600 blocks in all (P2).
msc::ArnoldiArgs arnoldi_args(msc_plan *p, const int *gate, bool chunks)
{
    msc::ArnoldiArgs a;
    a.tiles = chunks ? p->chunks() : p->tiles();
    a.sys_tile0 = chunks ? p->sys_chunk0.p : p->sys_tile0.p;
    a.gate = gate;
    a.n = p->n;
    a.split = chunks ? 1 : p->split;
    a.qstride = (size_t)p->R * p->n;
    a.partial = p->partial.p;
    a.pstride = p->pstride;
    a.counter = p->sys_counter.p;
    return a;
}

cudaEvent_t tev_at(msc_plan *p, int kind, int slot, int which)
{
    return p->tev[((size_t)kind * (p->m + 1) + slot) * 2 + which];
}

// Event record node inside a captured graph (External: a real record at launch).
void mark(msc_plan *p, int kind, int slot, int which, cudaStream_t st)
{
    cudaEventRecordWithFlags(tev_at(p, kind, slot, which), st, cudaEventRecordExternal);
}

// Cycle start (both forms): r = b - A x in FP64, its norm, activation.
// FP64 form: r lands in Q0 and is scaled in place.  Mixed form: r lands in
// R64 and its normalised FP32 copy becomes the first inner Krylov vector, so
// every cycle is one step of iterative refinement with an FP64 residual.
void record_cycle_start_t(msc_plan *p, bool x_zero, cudaStream_t st)
{
    double2 *r64 = p->mixed ? p->R64.p : p->Q.p;
    cudaMemsetAsync(p->counter.p, 0, sizeof(int), st);
    if (x_zero) {
        msc::k_rhs_residual<<<elementwise_grid(p), 256, 0, st>>>(p->tiles(), p->unfinished.p, p->n,
                                                                 p->row_rhs.p, r64);
    } else {
        launch_residual_diag(p, p->unfinished.p, p->X.p, p->TMP.p, 1, st);
        launch_coupling(p, p->unfinished.p, p->X.p, p->TMP.p, -1.0, r64, st);
    }
    launch_dots_t<double>(p, p->unfinished.p, p->Q.p, 0, r64, 1, st);
    launch_reduce(p, p->unfinished.p, 1, p->h2.p, st);
    msc::k_cycle_start<<<sys_blocks(p->B), 128, 0, st>>>(p->state(), p->B, p->m, p->h2.p,
                                                         p->m + 2, p->desc.rtol,
                                                         p->desc.max_iterations, p->max_cycles);
    if (p->mixed) {
        msc::k_convert_scaled<<<elementwise_grid(p), 256, 0, st>>>(p->tiles(), p->active.p, p->n,
                                                                   r64, p->scale.p, p->Q32.p);
    } else {
        launch_update(p, p->active.p, 0, nullptr, p->h1.p, p->m + 2, r64, p->scale.p, r64, 0, st);
    }
    cudaMemcpyAsync(p->counter_host, p->counter.p, sizeof(int), cudaMemcpyDeviceToHost, st);
}

void record_cycle_start(msc_plan *p, cudaStream_t st) { record_cycle_start_t(p, false, st); }

// First cycle of a solve from x = 0 (no warm start): r = b without the
// residual's T GEMM and FP64 coupling.
void record_cycle_start_zero(msc_plan *p, cudaStream_t st) { record_cycle_start_t(p, true, st); }

// m Arnoldi steps (CGS2) in precision R and the solution update x += M (Q y).
// out = M x with the von Neumann preconditioner of order k,
// M = sum_{i<=k} (-D^-1 V)^i D^-1: term_0 = D^-1 x, term_i = -D^-1 V term_{i-1}.
// Order 0 is one block inverse.  `scratch` and `term` are work vectors of the
// plan (the input x is not overwritten unless it is `scratch`, which is read
// only by the first block inverse).
template <typename R>
void apply_precond_t(msc_plan *p, const int *gate, const C2<R> *x, C2<R> *out, C2<R> *scratch,
                     C2<R> *term, cudaStream_t st)
{
    const int k = p->desc.precond_order;
    // block-diagonal form: base D^-1, coupling V; Gauss-Seidel form: base
    // L^-1 (forward sweep), coupling U (strictly upper part), so that order 1
    // is the reference's Neumann-preconditioned Gauss-Seidel operator
    // (multiscat_gmres.f90:452-475, _gmres.py:55-71)
    auto base = [&](const C2<R> *in, C2<R> *o) {
        if (p->gs)
            launch_gs_sweep_t<R>(p, gate, in, o, st);
        else
            launch_block_inverse_t<R>(p, gate, in, o, 0, st);
    };
    if (k <= 0) {
        base(x, out);
        return;
    }
    base(x, term);
    msc::k_copy_add<R><<<elementwise_grid(p), 256, 0, st>>>(p->tiles(), gate, p->n, term, out, 0);
    for (int i = 0; i < k; ++i) {
        if (p->gs)
            launch_coupling_masked_t<R>(p, gate, term, nullptr, R(-1), 2, scratch, st);
        else
            launch_coupling_t<R>(p, gate, term, nullptr, R(-1), scratch, st);
        base(scratch, term);
        msc::k_copy_add<R><<<elementwise_grid(p), 256, 0, st>>>(p->tiles(), gate, p->n, term, out, 1);
    }
}

template <typename R> C2<R> *precond_term(msc_plan *p);
template <> C2<float> *precond_term<float>(msc_plan *p) { return p->T32.p; }
template <> C2<double> *precond_term<double>(msc_plan *p) { return p->T64.p; }

template <typename R>
void record_iterations_t(msc_plan *p, C2<R> *Q, C2<R> *W, C2<R> *U, cudaStream_t st)
{
    const size_t vs = (size_t)p->R * p->n;
    const bool tm = p->timing;
    const double inner = p->mixed ? p->inner_rtol : 0.0;
    for (int j = 0; j < p->m; ++j) {
        C2<R> *Qj = Q + (size_t)j * vs;
        C2<R> *Qn = Q + (size_t)(j + 1) * vs;
        if (tm) mark(p, 0, j, 0, st);
        apply_precond_t<R>(p, p->active.p, Qj, U, W, precond_term<R>(p), st);
        if (tm) mark(p, 0, j, 1, st);
        if (tm) mark(p, 1, j, 0, st);
        // w = A M q_j.  (D + V) M_k = I + (-1)^k (V D^-1)^{k+1} telescopes, so
        // w = q_j + V term_k with term_k = (-D^-1 V)^k D^-1 q_j the last term
        // of the series (for k = 0, term_0 = U = D^-1 q_j).
        // Gauss-Seidel form: (L + U) M_k = I + (-1)^k (U L^-1)^{k+1} likewise,
        // so w = q_j + U term_k with the strictly upper coupling only
        const C2<R> *last = p->desc.precond_order > 0 ? precond_term<R>(p) : U;
        if (p->gs)
            launch_coupling_masked_t<R>(p, p->active.p, last, Qj, R(1), 2, W, st);
        else
            launch_coupling_t<R>(p, p->active.p, last, Qj, R(1), W, st);
        if (tm) mark(p, 1, j, 1, st);
        const msc::ArnoldiArgs a1 = arnoldi_args(p, p->active.p, true);
        const msc::ArnoldiArgs a2 = arnoldi_args(p, p->active.p, false);
        const unsigned nblk1 = (unsigned)p->nchunks;
        if (p->dcgs) {
            // DCGS2: the reduction finalises column j - 1 and forms the
            // update coefficients; the update writes q_j and the next
            // candidate into slots j and j + 1 and runs the stop test.
            if (tm) mark(p, 2, j, 0, st);
            if constexpr (std::is_same<R, float>::value) {
                if (p->bulk_arnoldi > 0)
                    msc::k_dcgs_reduce_bulk<<<nblk1, 256, msc::dcgs_bulk_smem(), st>>>(
                        a1, Q, j, W, p->state(), p->dstate(), p->m, p->desc.rtol, inner,
                        p->wait_error.p);
                else
                    msc::k_dcgs_reduce<R><<<nblk1, 256, dcgs_scratch_bytes(p->m), st>>>(a1, Q, j, W, p->state(),
                                                                 p->dstate(), p->m, p->desc.rtol,
                                                                 inner);
            } else {
                msc::k_dcgs_reduce<R><<<nblk1, 256, dcgs_scratch_bytes(p->m), st>>>(a1, Q, j, W, p->state(), p->dstate(),
                                                             p->m, p->desc.rtol, inner);
            }
            if (tm) mark(p, 2, j, 1, st);
            if (tm) mark(p, 3, j, 0, st);
            bool updated = false;
            if constexpr (std::is_same<R, float>::value) {
                if (p->bulk_arnoldi > 1) {
                    msc::k_dcgs_update_bulk<<<nblk1, 256, msc::dcgs_bulk_smem(), st>>>(
                        a1, Q, j, W, p->state(), p->dstate(), p->m, p->desc.rtol,
                        p->desc.max_iterations, inner, p->wait_error.p);
                    updated = true;
                }
            }
            if (!updated)
                msc::k_dcgs_update<R><<<nblk1, 256, dcgs_update_scratch_bytes(p->m), st>>>(a1, Q, j, W, p->state(), p->dstate(),
                                                             p->m, p->desc.rtol,
                                                             p->desc.max_iterations, inner);
            if (tm) mark(p, 3, j, 1, st);
            continue;
        }
        const unsigned nblk2 = (unsigned)(p->ntiles * p->split);
        // Two Gram-Schmidt passes; the mixed form may opt into one pass with
        // the Pythagorean norm (the FP64 true residual of the next refinement
        // step absorbs the loss of orthogonality, at the price of iterations).
        const int cgs2 = p->cgs1_inner ? 0 : 1;
        if (cgs2) {
            if (tm) mark(p, 2, j, 0, st);
            msc::k_arnoldi_p1<R><<<nblk1, 256, 0, st>>>(a1, Q, j + 1, W, p->h1.p, p->m + 2);
            if (tm) mark(p, 2, j, 1, st);
        }
        if (tm) mark(p, 3, j, 0, st);
        msc::k_arnoldi_p2<R><<<nblk2, 256, 0, st>>>(a2, Q, j + 1, W, p->state(), p->m, j,
                                                   p->desc.rtol, p->desc.max_iterations, inner,
                                                   cgs2);
        if (tm) mark(p, 3, j, 1, st);
        if (tm) mark(p, 4, j, 0, st);
        launch_update_t<R>(p, p->active.p, Q, j + 1, nullptr, p->h2.p, p->m + 2, W, p->scale.p, Qn,
                           0, st);
        if (tm) mark(p, 4, j, 1, st);
    }
    msc::k_trisolve<<<sys_blocks(p->B), 128, 0, st>>>(p->state(), p->B, p->m);
    launch_update_t<R>(p, p->kcyc.p, Q, 0, p->kcyc.p, p->y.p, p->m, nullptr, nullptr, U, 1, st);
    if (tm) mark(p, 0, p->m, 0, st);
    if (p->gs || p->desc.precond_order > 0) {
        // W = M U (U is free after the first block inverse and serves as scratch)
        apply_precond_t<R>(p, p->kcyc.p, U, W, U, precond_term<R>(p), st);
        if (!p->mixed)
            msc::k_copy_add<R><<<elementwise_grid(p), 256, 0, st>>>(
                p->tiles(), p->kcyc.p, p->n, W, reinterpret_cast<C2<R> *>(p->X.p), 1);
    } else if (p->mixed) {
        launch_block_inverse_t<R>(p, p->kcyc.p, U, W, 0, st);
    } else {
        launch_block_inverse_t<R>(p, p->kcyc.p, U, reinterpret_cast<C2<R> *>(p->X.p), 1, st);
    }
    if (tm) mark(p, 0, p->m, 1, st);
    if (p->mixed) {
        msc::k_accumulate_f32<<<elementwise_grid(p), 256, 0, st>>>(
            p->tiles(), p->kcyc.p, p->n, reinterpret_cast<const float2 *>(W), p->X.p);
    }
    cudaMemcpyAsync(p->kcyc_host, p->kcyc.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, st);
}

void record_cycle_iterations(msc_plan *p, cudaStream_t st)
{
    if (p->mixed)
        record_iterations_t<float>(p, p->Q32.p, p->W32.p, p->U32.p, st);
    else
        record_iterations_t<double>(p, p->Q.p, p->W.p, p->U.p, st);
}

// Kernel nodes in a captured graph (launch accounting).
int64_t count_kernel_nodes(cudaGraph_t g)
{
    size_t n = 0;
    if (cudaGraphGetNodes(g, nullptr, &n) != cudaSuccess) return 0;
    std::vector<cudaGraphNode_t> nodes(n);
    if (cudaGraphGetNodes(g, nodes.data(), &n) != cudaSuccess) return 0;
    int64_t k = 0;
    for (cudaGraphNode_t nd : nodes) {
        cudaGraphNodeType t;
        if (cudaGraphNodeGetType(nd, &t) == cudaSuccess && t == cudaGraphNodeTypeKernel) ++k;
    }
    return k;
}

// Add the device time of the timed launches of the last iteration graph.
void accumulate_timing(msc_plan *p)
{
    int maxk = 0;
    for (int s = 0; s < p->B; ++s) maxk = std::max(maxk, p->kcyc_host[s]);
    if (maxk == 0) return;
    for (int kind = 0; kind < msc_plan::kKinds; ++kind) {
        for (int j = 0; j < maxk; ++j) {
            float ms = 0.f;
            if (cudaEventElapsedTime(&ms, tev_at(p, kind, j, 0), tev_at(p, kind, j, 1)) == cudaSuccess) {
                p->t_ms[kind] += ms;
                p->t_launches[kind] += 1;
            } else {
                (void)cudaGetLastError();   // timing is best effort; keep the error state clean
            }
        }
    }
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, tev_at(p, 0, p->m, 0), tev_at(p, 0, p->m, 1)) == cudaSuccess) {
        p->t_ms[0] += ms;
        p->t_launches[0] += 1;
    } else {
        (void)cudaGetLastError();
    }
}

msc_status capture(msc_plan *p, void (*rec)(msc_plan *, cudaStream_t), cudaGraphExec_t *out,
                   int64_t *kernel_nodes)
{
    cudaGraph_t graph = nullptr;
    if (*out) {
        cudaGraphExecDestroy(*out);
        *out = nullptr;
    }
    MSC_CUDA(cudaStreamBeginCapture(p->stream, cudaStreamCaptureModeThreadLocal));
    rec(p, p->stream);
    cudaError_t e = cudaStreamEndCapture(p->stream, &graph);
    if (e != cudaSuccess) return fail(MSC_ERR_CUDA, std::string("graph capture: ") + cudaGetErrorString(e));
    if (kernel_nodes) *kernel_nodes = count_kernel_nodes(graph);
    e = cudaGraphInstantiate(out, graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return fail(MSC_ERR_CUDA, std::string("graph instantiate: ") + cudaGetErrorString(e));
    return MSC_OK;
}

msc_status set_kernel_attributes(int n, int K)
{
    MSC_CUDA(cudaFuncSetAttribute(msc::k_block_inverse<8, double>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_block_inverse(msc::kWideNz)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_block_inverse<4, double>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_block_inverse(msc::kMaxNz)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_block_inverse<8, float>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_block_inverse(msc::kWideNz)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_block_inverse<4, float>,
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_block_inverse(msc::kMaxNz)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_coupling(msc::kMaxTaps)));
#define MSC_HALO_ATTR(HY, R)                                                                     \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_halo<HY, kHaloBX, halo_zc<R>(), 8, R>,        \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(halo_smem(8, HY, halo_zc<R>(), sizeof(C2<R>)), 232448))); \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_halo<HY, kHaloBX, halo_zc<R>(), 4, R>,        \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(halo_smem(8, HY, halo_zc<R>(), sizeof(C2<R>)), 232448)));;
#define MSC_SEP_ATTR(HY, R)                                                                      \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_sep<HY, kHaloBX, halo_zc<R>(), R>,              \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(sep_smem(8, HY, halo_zc<R>(), sizeof(C2<R>)), 232448))); \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_sep<HY, kHaloBX, halo_zc<R>(), R, HY>,          \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(sep_smem(HY, HY, halo_zc<R>(), sizeof(C2<R>)), 232448))); \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_sep<HY, kHaloBX, halo_zc<R>() / 2, R, HY>,      \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(sep_smem(HY, HY, halo_zc<R>() / 2, sizeof(C2<R>)), 232448))); \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_sep<HY, kHaloBX, halo_zc<R>() / 2, R>,          \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(sep_smem(8, HY, halo_zc<R>() / 2, sizeof(C2<R>)), 232448)));
#define MSC_SEP_ROWS_ATTR(H, R)                                                                  \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_sep_rows<H, kHaloBX, halo_zc<R>(), R, H>,      \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(sep_smem(H, H, halo_zc<R>(), sizeof(C2<R>)), 232448)));
    MSC_SEP_ROWS_ATTR(1, float) MSC_SEP_ROWS_ATTR(2, float)
    MSC_SEP_ROWS_ATTR(4, float) MSC_SEP_ROWS_ATTR(8, float)
    MSC_SEP_ROWS_ATTR(1, double) MSC_SEP_ROWS_ATTR(2, double)
    MSC_SEP_ROWS_ATTR(4, double) MSC_SEP_ROWS_ATTR(8, double)
#undef MSC_SEP_ROWS_ATTR
    MSC_SEP_ATTR(1, float)
    MSC_SEP_ATTR(2, float)
    MSC_SEP_ATTR(4, float)
    MSC_SEP_ATTR(8, float)
    MSC_SEP_ATTR(1, double)
    MSC_SEP_ATTR(2, double)
    MSC_SEP_ATTR(4, double)
    MSC_SEP_ATTR(8, double)
#undef MSC_SEP_ATTR
#define MSC_HALO_MASK_ATTR(HY, R, M)                                                              \
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_halo<HY, kHaloBX, halo_zc<R>(), 4, R, M>,       \
                                  cudaFuncAttributeMaxDynamicSharedMemorySize,                   \
                                  (int)std::min<size_t>(halo_smem(8, HY, halo_zc<R>(), sizeof(C2<R>)), 232448)));
    MSC_HALO_MASK_ATTR(1, float, 1) MSC_HALO_MASK_ATTR(2, float, 1)
    MSC_HALO_MASK_ATTR(4, float, 1) MSC_HALO_MASK_ATTR(8, float, 1)
    MSC_HALO_MASK_ATTR(1, float, 2) MSC_HALO_MASK_ATTR(2, float, 2)
    MSC_HALO_MASK_ATTR(4, float, 2) MSC_HALO_MASK_ATTR(8, float, 2)
    MSC_HALO_MASK_ATTR(1, double, 1) MSC_HALO_MASK_ATTR(2, double, 1)
    MSC_HALO_MASK_ATTR(4, double, 1) MSC_HALO_MASK_ATTR(8, double, 1)
    MSC_HALO_MASK_ATTR(1, double, 2) MSC_HALO_MASK_ATTR(2, double, 2)
    MSC_HALO_MASK_ATTR(4, double, 2) MSC_HALO_MASK_ATTR(8, double, 2)
#undef MSC_HALO_MASK_ATTR
    MSC_HALO_ATTR(1, float)
    MSC_HALO_ATTR(2, float)
    MSC_HALO_ATTR(4, float)
    MSC_HALO_ATTR(8, float)
    MSC_HALO_ATTR(1, double)
    MSC_HALO_ATTR(2, double)
    MSC_HALO_ATTR(4, double)
    MSC_HALO_ATTR(8, double)
#undef MSC_HALO_ATTR
    MSC_CUDA(cudaFuncSetAttribute(msc::k_residual_diag, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_residual(msc::kMaxNz)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_coupling(msc::kMaxTaps)));
    (void)n;
    (void)K;
    return MSC_OK;
}

// Shared memory the tensor-core kernel needs for tile width N and G warp
// groups (bytes of the dynamic part: E_hi, E_lo and one B buffer per group),
// including the bytes its padded M tiles may read past E.
size_t tc_smem_bytes(int n, int N, int G = 1)
{
    const size_t kp = (size_t)(n + 15) / 16 * 16;
    const size_t kb = kp / 8, mt = (size_t)(n + 127) / 128;
    const size_t part = kp * kp * 2, sz = kb * 128;
    const size_t read1 = (16 * mt - 1) * 128 + (kb - 1) * sz + 128;
    const size_t read2 = (16 * mt - 1) * sz + (kb - 1) * 128 + 128;
    const size_t need = std::max(2 * part + (size_t)G * 4 * N * kp, part + std::max(read1, read2));
    return (need + 1023) / 1024 * 1024 + 1024;
}

// TMEM columns one CTA allocates: a power of two >= 32 per group.
int tc_tmem_cols(int n, int N, int G)
{
    const int mt = (n + 127) / 128;
    int ncols = 32;
    while (ncols < 2 * mt * N) ncols <<= 1;
    return G * ncols;
}

template <int N, int G>
cudaError_t tc_set_smem(size_t bytes)
{
    return cudaFuncSetAttribute(msc::tc::k_block_inverse_tc<N, G>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

template <int N, int G>
size_t tc_static_smem()
{
    cudaFuncAttributes a{};
    if (cudaFuncGetAttributes(&a, msc::tc::k_block_inverse_tc<N, G>) != cudaSuccess) return 1u << 30;
    return a.sharedSizeBytes;
}

size_t tc_static_for(int N, int G = 1)
{
    if (G == 2) {
        switch (N) {
        case 16: return tc_static_smem<16, 2>();
        case 32: return tc_static_smem<32, 2>();
        case 64: return tc_static_smem<64, 2>();
        default: return tc_static_smem<128, 2>();
        }
    }
    switch (N) {
    case 16: return tc_static_smem<16, 1>();
    case 32: return tc_static_smem<32, 1>();
    case 64: return tc_static_smem<64, 1>();
    case 128: return tc_static_smem<128, 1>();
    default: return tc_static_smem<256, 1>();
    }
}

cudaError_t tc_set_smem_for(int N, int G, size_t bytes)
{
    if (G == 2) {
        switch (N) {
        case 16: return tc_set_smem<16, 2>(bytes);
        case 32: return tc_set_smem<32, 2>(bytes);
        case 64: return tc_set_smem<64, 2>(bytes);
        default: return tc_set_smem<128, 2>(bytes);
        }
    }
    switch (N) {
    case 16: return tc_set_smem<16, 1>(bytes);
    case 32: return tc_set_smem<32, 1>(bytes);
    case 64: return tc_set_smem<64, 1>(bytes);
    case 128: return tc_set_smem<128, 1>(bytes);
    default: return tc_set_smem<256, 1>(bytes);
    }
}

// Shared-memory request of a kernel variant: what it needs, padded so that
// no more CTAs fit on one SM than its 512 TMEM columns can serve.
size_t tc_request_bytes(int n, int N, int G)
{
    const size_t max_ctas = 512 / (size_t)tc_tmem_cols(n, N, G);
    const size_t sm_bytes = 233472;   // 228 KB of shared memory per SM
    const size_t floor_bytes = sm_bytes / (max_ctas + 1) + 1024;
    return std::max(tc_smem_bytes(n, N, G), floor_bytes);
}

// Decide whether the mixed form uses the tcgen05 block inverse and with what
// tile width; build the BF16 hi/lo image of E in the kernel's smem order.
msc_status setup_tensor_core(msc_plan *p)
{
    p->use_tc = false;
    if (!p->mixed || (p->desc.flags & 1) || p->n > 256) return MSC_OK;
    int dev = 0, sms = 0, cc_major = 0, cc_minor = 0, optin = 0;
    MSC_CUDA(cudaGetDevice(&dev));
    MSC_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev));
    MSC_CUDA(cudaDeviceGetAttribute(&cc_major, cudaDevAttrComputeCapabilityMajor, dev));
    MSC_CUDA(cudaDeviceGetAttribute(&cc_minor, cudaDevAttrComputeCapabilityMinor, dev));
    MSC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    if (cc_major != 10 || cc_minor != 0) return MSC_OK;   // tcgen05 path is built for sm_100a
    const int n = p->n;
    int chosen = 0;
    for (int N = 16; N <= 256; N *= 2) {
        if (tc_tmem_cols(n, N, 1) > 512) break;
        if (tc_smem_bytes(n, N) + tc_static_for(N) > (size_t)optin) break;
        const int tiles = (p->R + N / 2 - 1) / (N / 2);
        chosen = N;
        if (tiles <= sms) break;   // enough tiles for every SM already at this width
    }
    if (chosen == 0) return MSC_OK;
    p->tc_n = chosen;
    p->tc_groups = 1;
    p->tc_tile_rows = chosen / 2;
    p->tc_ntiles = (p->R + p->tc_tile_rows - 1) / p->tc_tile_rows;
    p->tc_grid = std::min(p->tc_ntiles, sms);
    // every width up to `chosen` may be picked by the autotuner; all launch
    // with the same (largest) shared-memory request
    p->tc_smem = tc_request_bytes(n, chosen, 1);
    if (p->tc_smem + tc_static_for(chosen) > (size_t)optin) return MSC_OK;
    for (int N = 16; N <= chosen; N *= 2) {
        cudaError_t e = tc_set_smem_for(N, 1, p->tc_smem);
        if (e != cudaSuccess) return fail(MSC_ERR_CUDA, std::string("tc smem attribute: ") + cudaGetErrorString(e));
    }
    // two-group variants: widths whose two TMEM regions and two B buffers fit
    p->tc2_max = 0;
    for (int N = 16; N <= std::min(chosen, 128); N *= 2) {
        if (tc_tmem_cols(n, N, 2) > 512) break;
        if (tc_request_bytes(n, N, 2) + tc_static_for(N, 2) > (size_t)optin) break;
        p->tc2_max = N;
    }
    if (p->tc2_max > 0) {
        p->tc2_smem = tc_request_bytes(n, p->tc2_max, 2);
        for (int N = 16; N <= p->tc2_max; N *= 2) {
            cudaError_t e = tc_set_smem_for(N, 2, p->tc2_smem);
            if (e != cudaSuccess) return fail(MSC_ERR_CUDA, std::string("tc smem attribute: ") + cudaGetErrorString(e));
        }
    }
    // channel-major kernel: E_hi, E_lo and one A buffer of 128 rows x kp
    {
        const size_t kpc = (size_t)(n + 15) / 16 * 16;
        cudaFuncAttributes fa{};
        p->tcc_smem = 4 * kpc * kpc + 512 * kpc + 1024;
        p->tcc_ok = kpc <= 256 &&
                    cudaFuncGetAttributes(&fa, msc::tc::k_block_inverse_tcc) == cudaSuccess &&
                    p->tcc_smem + fa.sharedSizeBytes <= (size_t)optin;
        if (p->tcc_ok) {
            cudaError_t e = cudaFuncSetAttribute(msc::tc::k_block_inverse_tcc,
                                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)p->tcc_smem);
            if (e != cudaSuccess) return fail(MSC_ERR_CUDA, std::string("tcc smem attribute: ") + cudaGetErrorString(e));
        }
    }
    // E image: [hi|lo][z/8][k/8][z%8][k%8], zero padded to kp x kp
    const int kp = (n + 15) / 16 * 16, kb = kp / 8;
    std::vector<__nv_bfloat16> img((size_t)2 * kp * kp, __float2bfloat16(0.f));
    for (int z = 0; z < n; ++z)
        for (int k = 0; k < n; ++k) {
            const double v = p->E_host[(size_t)z * n + k];
            const __nv_bfloat16 hi = __float2bfloat16_rn((float)v);
            const __nv_bfloat16 lo = __float2bfloat16_rn((float)(v - (double)__bfloat162float(hi)));
            const size_t off = ((size_t)(z / 8) * kb + k / 8) * 64 + (z % 8) * 8 + (k % 8);
            img[off] = hi;
            img[(size_t)kp * kp + off] = lo;
        }
    MSC_CUDA(upload(p->e_img, img));
    MSC_CUDA(p->tc_error.alloc(1));
    MSC_CUDA(cudaMemset(p->tc_error.p, 0, sizeof(int)));
    p->use_tc = true;
    return MSC_OK;
}

// Device time of one call of `f` on the plan's stream (mean of 3 after a warm-up).
template <typename F>
float time_launch(msc_plan *p, F f)
{
    cudaEvent_t a, b;
    cudaEventCreate(&a);
    cudaEventCreate(&b);
    f(p->stream);
    cudaEventRecord(a, p->stream);
    for (int i = 0; i < 3; ++i) f(p->stream);
    cudaEventRecord(b, p->stream);
    cudaEventSynchronize(b);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, a, b);
    cudaEventDestroy(a);
    cudaEventDestroy(b);
    return ms * 1000.f / 3.f;
}

// Autotuner: time the kernel variants this plan can use on its own data
// and keep the fastest.  Coupling: halo tiles vs neighbour table, for each
// precision the solve uses.  Mixed form: tcgen05 tile width N (and the SIMT
// FP32 kernel).  Runs once per plan, before the solve graphs are captured.
struct TuneKey {
    int n, R, K, nkx, nky, B, mixed, hx, hy, tcmax, flags, sep;
    bool operator<(const TuneKey &o) const
    {
        return std::tie(n, R, K, nkx, nky, B, mixed, hx, hy, tcmax, flags, sep) <
               std::tie(o.n, o.R, o.K, o.nkx, o.nky, o.B, o.mixed, o.hx, o.hy, o.tcmax, o.flags,
                        o.sep);
    }
};
struct TuneChoice {
    int halo64, halo32, use_tc, tc_n, tc_groups;
};
std::mutex g_tune_mutex;
std::map<TuneKey, TuneChoice> g_tune_cache;

msc_status autotune_measure(msc_plan *p);

void apply_tc_width(msc_plan *p, int N, int G = 1)
{
    int sms = 148, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (G == kTcChannelMajor) {
        if (p->tcc_ok) {
            p->tc_n = 128;                 // M rows: 64 channels
            p->tc_groups = G;
            p->tc_tile_rows = 64;
            p->tc_ntiles = (p->R + 63) / 64;
            p->tc_grid = std::min(p->tc_ntiles, sms);
            return;
        }
        G = 1;
        N = std::min(N, 128);
    }
    if (G == 2 && N > p->tc2_max) G = 1;
    p->tc_n = N;
    p->tc_groups = G;
    p->tc_tile_rows = N / 2;
    p->tc_ntiles = (p->R + N / 2 - 1) / (N / 2);
    p->tc_grid = std::min((p->tc_ntiles + G - 1) / G, sms);
}

// Autotuner front end: reuse the choices of an earlier plan of the same
// shape (same sizes, batch, tap reach and options), else measure.
// MSC_TUNE="c64=K,c32=K,bi=N[,bg=G]" fixes the choices (K: 0 neighbour
// table, 1 halo 8 y/thread, 2 halo 4 y/thread; N: tcgen05 tile width,
// 0 = SIMT; G: 1 or 2 warp groups in the tcgen05 kernel, default 1).
// Profiling runs use it so that a profiler's overhead cannot change what the
// autotuner picks.
bool tune_from_env(msc_plan *p)
{
    const char *env = std::getenv("MSC_TUNE");
    if (!env || !*env) return false;
    int c64 = p->halo64, c32 = p->halo32, bi = p->use_tc ? p->tc_n : 0, bg = 1;
    std::sscanf(env, "c64=%d,c32=%d,bi=%d,bg=%d", &c64, &c32, &bi, &bg);
    const int kmax = p->sep_ok ? 5 : 2;
    p->halo64 = p->use_halo ? std::max(0, std::min(kmax, c64)) : 0;
    p->halo32 = p->use_halo ? std::max(0, std::min(kmax, c32)) : 0;
    if (p->use_tc) {
        if (bi == 0) {
            p->use_tc = false;
        } else {
            int N = 16;
            while (N < bi && N < p->tc_n) N *= 2;
            apply_tc_width(p, N, (bg == 2 || bg == kTcChannelMajor) ? bg : 1);
        }
    }
    p->tune_log.push_back({"from_MSC_TUNE", 1.f});
    return true;
}

msc_status autotune(msc_plan *p)
{
    if (tune_from_env(p)) return MSC_OK;
    const TuneKey key{p->n, p->R, p->K, p->nkx, p->nky, p->B, p->mixed ? 1 : 0, p->halo_hx,
                      p->halo_hy, p->use_tc ? p->tc_n : 0, p->desc.flags, p->sep_ok ? 1 : 0};
    {
        std::lock_guard<std::mutex> lock(g_tune_mutex);
        auto it = g_tune_cache.find(key);
        if (it != g_tune_cache.end()) {
            p->halo64 = it->second.halo64;
            p->halo32 = it->second.halo32;
            if (p->use_tc) {
                p->use_tc = it->second.use_tc != 0;
                if (p->use_tc) apply_tc_width(p, it->second.tc_n, it->second.tc_groups);
            }
            p->tune_log.push_back({"cached", 1.f});
            return MSC_OK;
        }
    }
    msc_status st = autotune_measure(p);
    if (st != MSC_OK) return st;
    std::lock_guard<std::mutex> lock(g_tune_mutex);
    g_tune_cache[key] = TuneChoice{p->halo64, p->halo32, p->use_tc ? 1 : 0, p->tc_n, p->tc_groups};
    return MSC_OK;
}

msc_status autotune_measure(msc_plan *p)
{
    const size_t vs = (size_t)p->R * p->n;
    MSC_CUDA(cudaMemsetAsync(p->X.p, 0, vs * sizeof(double2), p->stream));
    MSC_CUDA(cudaMemsetAsync(p->TMP.p, 0, vs * sizeof(double2), p->stream));
    const char *kind_name[6] = {"neighbour", "halo_y8", "halo_y4", "separable", "separable_z2",
                                "separable_rows"};
    const int nkinds = sep_rows_ok(p) ? 6 : p->sep_ok ? 5 : 3;
    if (p->use_halo) {
        float best = 0.f;
        int best_k = 0;
        for (int k = 0; k < nkinds; ++k) {
            p->halo64 = k;
            const float t = time_launch(p, [&](cudaStream_t st) {
                launch_coupling_t<double>(p, nullptr, p->X.p, p->TMP.p, -1.0, p->TMP.p, st);
            });
            p->tune_log.push_back({std::string("coupling64_") + kind_name[k] + "_us", t});
            if (k == 0 || t < best) {
                best = t;
                best_k = k;
            }
        }
        p->halo64 = best_k;
    }
    if (p->mixed) {
        float2 *a = p->Q32.p, *b = p->W32.p, *c = p->U32.p;
        MSC_CUDA(cudaMemsetAsync(a, 0, vs * sizeof(float2), p->stream));
        MSC_CUDA(cudaMemsetAsync(c, 0, vs * sizeof(float2), p->stream));
        if (p->use_halo) {
            float best = 0.f;
            int best_k = 0;
            for (int k = 0; k < nkinds; ++k) {
                p->halo32 = k;
                const float t = time_launch(p, [&](cudaStream_t st) {
                    launch_coupling_t<float>(p, nullptr, a, c, 1.0f, b, st);
                });
                p->tune_log.push_back({std::string("coupling32_") + kind_name[k] + "_us", t});
                if (k == 0 || t < best) {
                    best = t;
                    best_k = k;
                }
            }
            p->halo32 = best_k;
        }
        if (p->use_tc) {
            const int best_n0 = p->tc_n;
            int best_n = 0, best_g = 1;
            float best_t = 0.f;
            p->use_tc = false;
            const float t_simt = time_launch(p, [&](cudaStream_t st) {
                launch_block_inverse_t<float>(p, nullptr, a, b, 0, st);
            });
            p->tune_log.push_back({"block_inverse32_simt_us", t_simt});
            p->use_tc = true;
            // (the channel-major form, MSC_TUNE bg=3, is left out: 243 against
            // 250 us per full-batch launch on the 512-beam cfg2 batch, but the
            // batch was not faster end to end with it)
            for (int G = 1; G <= 2; ++G)
                for (int N = 16; N <= (G == 1 ? best_n0 : p->tc2_max); N *= 2) {
                    apply_tc_width(p, N, G);
                    const float t = time_launch(p, [&](cudaStream_t st) {
                        launch_block_inverse_t<float>(p, nullptr, a, b, 0, st);
                    });
                    p->tune_log.push_back({std::string("block_inverse32_tc") + (G == 2 ? "2" : "") +
                                               "_N" + std::to_string(N) + "_us",
                                           t});
                    if (best_n == 0 || t < best_t) {
                        best_n = N;
                        best_g = G;
                        best_t = t;
                    }
                }
            int tc_err = 0;
            MSC_CUDA(cudaMemcpy(&tc_err, p->tc_error.p, sizeof(int), cudaMemcpyDeviceToHost));
            if (tc_err) return fail(MSC_ERR_CUDA, "tensor-core block inverse timed out during tuning");
            if (t_simt < best_t && !(p->desc.flags & 2)) {
                p->use_tc = false;
            } else {
                apply_tc_width(p, best_n, best_g);
            }
        }
    }
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

// Build rows, tiles, neighbour tables; upload everything; allocate state.
// Set-up phase timer: MSC_PROFILE_SETUP=1 prints the wall time of each plan
// set-up phase (device synchronised at the marks) to stderr.
struct SetupTimer {
    bool on = false;
    std::chrono::steady_clock::time_point t0;
    SetupTimer()
    {
        const char *e = std::getenv("MSC_PROFILE_SETUP");
        on = e && e[0] == '1';
        t0 = std::chrono::steady_clock::now();
    }
    void mark(const char *what)
    {
        if (!on) return;
        cudaDeviceSynchronize();
        const auto t = std::chrono::steady_clock::now();
        std::fprintf(stderr, "msc setup %-22s %8.2f ms\n", what,
                     std::chrono::duration<double, std::milli>(t - t0).count());
        t0 = t;
    }
};

msc_status ensure_gs_levels(msc_plan *p);

// Separable coupling: for every z, the tap window W[sdx][sdy] (signed
// offsets, zero where there is no tap, the centre free) is tested for the
// form p_sdx q_sdy.  The pivot is the largest entry off the centre row and
// column; p is its column, q its row divided by it, and every tap must
// match p q to 1e-13 of the potential's scale at that z, max(|W|, |V_00|):
// the rounding the potential's own 2-D FFT leaves in its small components
// (~1e-15 of that scale for the square-lattice Morse potentials) passes,
// anything structural fails.  A window of zeros gives p = q = 0.  Any z that
// fails (a hexagonal lattice's coupling, taps only on the centre cross)
// leaves the plan on the direct kernels.
void separable_factors(msc_plan *p, const std::vector<int> &win)
{
    p->sep_ok = false;
    const int n = p->n, hx = p->halo_hx, hy = p->halo_hy;
    const int wx = 2 * hx + 1, wy = 2 * hy + 1;
    std::vector<double2> P((size_t)wx * n), Q((size_t)wy * n), Kc(n);
    std::vector<double2> W((size_t)wx * wy);
    for (int z = 0; z < n; ++z) {
        double wmax = 0.0;
        for (int c = 0; c < wx * wy; ++c) {
            const int t = win[c];
            W[c] = t >= 0 ? p->Vt_host[(size_t)t * n + z] : double2{0.0, 0.0};
            wmax = std::max(wmax, std::sqrt(msc::cabs2(W[c])));
        }
        int pa = -1, pb = -1;
        double best = 0.0;
        for (int a = 0; a < wx; ++a)
            for (int b = 0; b < wy; ++b) {
                if (a == hx || b == hy) continue;
                const double m = msc::cabs2(W[(size_t)a * wy + b]);
                if (m > best) {
                    best = m;
                    pa = a;
                    pb = b;
                }
            }
        if (pa < 0) {
            if (wmax > 0.0) return;          // taps on the centre cross only: not a product
            for (int a = 0; a < wx; ++a) P[(size_t)a * n + z] = double2{0.0, 0.0};
            for (int b = 0; b < wy; ++b) Q[(size_t)b * n + z] = double2{0.0, 0.0};
            Kc[z] = double2{0.0, 0.0};
            continue;
        }
        const double2 piv = W[(size_t)pa * wy + pb];
        for (int a = 0; a < wx; ++a) P[(size_t)a * n + z] = W[(size_t)a * wy + pb];
        for (int b = 0; b < wy; ++b) Q[(size_t)b * n + z] = msc::cdiv(W[(size_t)pa * wy + b], piv);
        for (int a = 0; a < wx; ++a)
            for (int b = 0; b < wy; ++b) {
                if (a == hx && b == hy) continue;
                const double2 pq = msc::cmul(P[(size_t)a * n + z], Q[(size_t)b * n + z]);
                const double2 d = msc::csub(W[(size_t)a * wy + b], pq);
                if (std::sqrt(msc::cabs2(d)) > 1e-13 * std::max(wmax, std::fabs(p->v00_host[z])))
                    return;
            }
        Kc[z] = msc::cmul(P[(size_t)hx * n + z], Q[(size_t)hy * n + z]);
    }
    p->sep_p_h.swap(P);
    p->sep_q_h.swap(Q);
    p->sep_k_h.swap(Kc);
    p->sep_ok = true;
}

// Upload p | q | kappa of the operator in use (A: as found; A^H, whose tap
// at d is conj(V_{-d}): p_sdx -> conj(p_{-sdx}), q likewise, kappa -> conj).
msc_status upload_separable(msc_plan *p)
{
    const int n = p->n, wx = 2 * p->halo_hx + 1, wy = 2 * p->halo_hy + 1;
    std::vector<double2> all;
    all.reserve((size_t)(wx + wy + 1) * n);
    for (int a = 0; a < wx; ++a)
        for (int z = 0; z < n; ++z) {
            const double2 v = p->sep_p_h[(size_t)(p->adjoint ? wx - 1 - a : a) * n + z];
            all.push_back(p->adjoint ? msc::cconj(v) : v);
        }
    for (int b = 0; b < wy; ++b)
        for (int z = 0; z < n; ++z) {
            const double2 v = p->sep_q_h[(size_t)(p->adjoint ? wy - 1 - b : b) * n + z];
            all.push_back(p->adjoint ? msc::cconj(v) : v);
        }
    for (int z = 0; z < n; ++z) all.push_back(p->adjoint ? msc::cconj(p->sep_k_h[z]) : p->sep_k_h[z]);
    std::vector<float2> all32(all.size());
    for (size_t i = 0; i < all.size(); ++i) all32[i] = make_float2((float)all[i].x, (float)all[i].y);
    if (p->sep64.count == all.size()) {
        MSC_CUDA(refill(p->sep64, all));
        MSC_CUDA(refill(p->sep32, all32));
    } else {
        MSC_CUDA(upload(p->sep64, all));
        MSC_CUDA(upload(p->sep32, all32));
    }
    return MSC_OK;
}

msc_status finalize(msc_plan *p)
{
    if (p->finalized) return MSC_OK;
    SetupTimer tm;
    if (!p->potential_set) return fail(MSC_ERR_ARG, "potential not set");
    for (int s = 0; s < p->B; ++s)
        if (!p->sys[s].set) return fail(MSC_ERR_ARG, "system " + std::to_string(s) + " not set");
    const int n = p->n;
    // rows and tiles
    p->R = 0;
    p->sys_row0_h.assign(p->B + 1, 0);
    p->sys_tile0_h.assign(p->B + 1, 0);
    p->tile_row0_h.clear(); p->tile_nrow_h.clear(); p->tile_sys_h.clear(); p->row_sys_h.clear();
    for (int s = 0; s < p->B; ++s) {
        p->sys_row0_h[s] = p->R;
        p->sys_tile0_h[s] = (int)p->tile_row0_h.size();
        const int C = p->sys[s].C;
        for (int r = 0; r < C; r += msc::kTileRows) {
            p->tile_row0_h.push_back(p->R + r);
            p->tile_nrow_h.push_back(std::min(msc::kTileRows, C - r));
            p->tile_sys_h.push_back(s);
        }
        for (int r = 0; r < C; ++r) p->row_sys_h.push_back(s);
        p->R += C;
    }
    p->sys_row0_h[p->B] = p->R;
    p->sys_tile0_h[p->B] = (int)p->tile_row0_h.size();
    p->ntiles = (int)p->tile_row0_h.size();
    // per-row data and neighbour table
    // per-row data; position tables (row of each torus position per system)
    const int ntor = p->nkx * p->nky;
    std::vector<double> pkd(p->R);
    std::vector<double2> rc(p->R), rb(p->R), bspec(p->B), aspec(p->B);
    std::vector<int> spec_row(p->B), row_pos(p->R), pos_map((size_t)p->B * ntor, -1);
    for (int s = 0; s < p->B; ++s) {
        const SystemHost &sh = p->sys[s];
        const int r0 = p->sys_row0_h[s];
        int *map = pos_map.data() + (size_t)s * ntor;
        for (int j = 0; j < sh.C; ++j) {
            const int row = r0 + j;
            const int q = sh.ix[j] * p->nky + sh.iy[j];
            row_pos[row] = q;
            map[q] = row;
            pkd[row] = sh.pkd[j];
            rc[row] = sh.c[j];
            rb[row] = sh.b[j];
        }
        spec_row[s] = r0 + sh.spec;
        bspec[s] = sh.b[sh.spec];
        aspec[s] = sh.a_spec;
    }
    std::vector<double> bn(p->B);
    for (int s = 0; s < p->B; ++s) bn[s] = std::sqrt(msc::cabs2(bspec[s]));
    // right-hand side: the scattering source b_spec at z_n of each specular row
    p->rhs_default_h.assign(p->R, double2{0.0, 0.0});
    for (int s = 0; s < p->B; ++s) p->rhs_default_h[spec_row[s]] = bspec[s];
    p->row_c_h = rc;

    tm.mark("host row tables");
    MSC_CUDA(upload(p->row_pkd, pkd));
    MSC_CUDA(upload(p->row_c, rc));
    MSC_CUDA(upload(p->row_b, rb));
    MSC_CUDA(upload(p->row_rhs, p->rhs_default_h));
    MSC_CUDA(upload(p->sys_row0, p->sys_row0_h));
    MSC_CUDA(upload(p->sys_aspec, aspec));
    MSC_CUDA(upload(p->sys_spec_row, spec_row));
    MSC_CUDA(upload(p->row_pos, row_pos));
    MSC_CUDA(upload(p->pos_map, pos_map));
    MSC_CUDA(upload(p->row_sys, p->row_sys_h));
    {
        std::vector<int2> taps(std::max(p->K, 1), make_int2(0, 0));
        for (int t = 0; t < p->K; ++t) taps[t] = make_int2(p->taps[t].first, p->taps[t].second);
        MSC_CUDA(upload(p->taps_d, taps));
    }
    MSC_CUDA(p->row_fn.alloc(p->R));
    MSC_CUDA(p->nbr.alloc((size_t)p->R * std::max(p->K, 1)));
    if (p->K == 0) MSC_CUDA(cudaMemset(p->nbr.p, 0xff, p->nbr.count * sizeof(int)));
    if (p->mixed) MSC_CUDA(p->row_fn32.alloc(p->R));
    msc::k_row_tables<<<std::min((p->R + 255) / 256, 4096), 256>>>(
        p->R, n, p->K, p->nkx, p->nky, p->row_pos.p, p->row_sys.p, p->pos_map.p, p->taps_d.p,
        p->row_pkd.p, p->en.p, p->lam.p, p->row_fn.p, p->mixed ? p->row_fn32.p : nullptr,
        p->K > 0 ? p->nbr.p : nullptr);
    MSC_CUDA(cudaGetLastError());
    MSC_CUDA(p->row_cf.alloc(p->R));
    msc::k_row_cfac<<<std::min((p->R + 255) / 256, 4096), 256>>>(p->R, p->row_c.p, p->row_fn.p,
                                                                 p->row_cf.p);
    MSC_CUDA(cudaGetLastError());
    MSC_CUDA(cudaDeviceSynchronize());
    tm.mark("row tables (device)");
    {
        // Halo-tiled coupling: signed tap reach, tap window, position->row
        // tables and the list of 8 x kHaloBX position patches that hold
        // channels of each system.
        int hx = 0, hy = 0;
        std::vector<std::pair<int, int>> sgn(p->K);
        for (int t = 0; t < p->K; ++t) {
            int dx = p->taps[t].first, dy = p->taps[t].second;
            if (dx > p->nkx / 2) dx -= p->nkx;
            if (dy > p->nky / 2) dy -= p->nky;
            sgn[t] = {dx, dy};
            hx = std::max(hx, std::abs(dx));
            hy = std::max(hy, std::abs(dy));
        }
        int hyt = 1;
        while (hyt < hy) hyt <<= 1;
        p->use_halo = (hx <= 8 && hyt <= 8 &&
                       halo_smem(hx, hyt, 16, sizeof(double2)) <= 225 * 1024 &&
                       halo_smem(hx, hyt, 32, sizeof(float2)) <= 225 * 1024);
        if (p->use_halo) {
            p->halo_hx = hx;
            p->halo_hy = hyt;
            const int wy = 2 * hyt + 1;
            std::vector<int> win((size_t)(2 * hx + 1) * wy, -1);
            for (int t = 0; t < p->K; ++t)
                win[(size_t)(sgn[t].first + hx) * wy + (sgn[t].second + hyt)] = t;
            std::vector<int> wl;
            const int nbx = (p->nkx + kHaloBX - 1) / kHaloBX, nby = (p->nky + 7) / 8;
            for (int s2 = 0; s2 < p->B; ++s2) {
                const SystemHost &sh = p->sys[s2];
                std::vector<char> occ((size_t)nbx * nby, 0);
                for (int j = 0; j < sh.C; ++j)
                    occ[(size_t)(sh.ix[j] / kHaloBX) * nby + sh.iy[j] / 8] = 1;
                for (int bx = 0; bx < nbx; ++bx)
                    for (int by = 0; by < nby; ++by)
                        if (occ[(size_t)bx * nby + by]) {
                            wl.push_back(s2);
                            wl.push_back(bx * kHaloBX);
                            wl.push_back(by * 8);
                        }
            }
            p->nwork = (int)(wl.size() / 3);
            MSC_CUDA(upload(p->tap_window, win));
            MSC_CUDA(upload(p->work, wl));
            separable_factors(p, win);
            if (p->sep_ok) {
                msc_status sst = upload_separable(p);
                if (sst != MSC_OK) return sst;
            }
        }
    }
    tm.mark("halo tables");
    MSC_CUDA(upload(p->tile_row0, p->tile_row0_h));
    MSC_CUDA(upload(p->tile_nrow, p->tile_nrow_h));
    MSC_CUDA(upload(p->tile_sys, p->tile_sys_h));
    MSC_CUDA(upload(p->sys_tile0, p->sys_tile0_h));
    MSC_CUDA(upload(p->bnorm, bn));
    if (p->mixed) {
        std::vector<float> pkd32(p->R);
        std::vector<float2> c32(p->R);
        for (int r = 0; r < p->R; ++r) {
            pkd32[r] = (float)pkd[r];
            c32[r] = make_float2((float)rc[r].x, (float)rc[r].y);
        }
        MSC_CUDA(upload(p->row_pkd32, pkd32));
        MSC_CUDA(upload(p->row_c32, c32));
    }

    tm.mark("tile uploads");
    const size_t vs = (size_t)p->R * n;
    const int m = p->m;
    p->pstride = 2 * m + 2;      // slots per block: 2 (m + 1) dots of a DCGS2 reduction
    MSC_CUDA(p->X.alloc(vs));
    MSC_CUDA(p->TMP.alloc(vs));
    if (p->mixed) {
        MSC_CUDA(p->R64.alloc(vs));
        MSC_CUDA(p->Q32.alloc(vs * (m + 1)));
        MSC_CUDA(p->W32.alloc(vs));
        MSC_CUDA(p->U32.alloc(vs));
        if (p->desc.precond_order > 0) MSC_CUDA(p->T32.alloc(vs));
    } else {
        MSC_CUDA(p->W.alloc(vs));
        MSC_CUDA(p->U.alloc(vs));
        if (p->desc.precond_order > 0) MSC_CUDA(p->T64.alloc(vs));
        MSC_CUDA(p->Q.alloc(vs * (m + 1)));
    }
    {
        // Arnoldi chunks: about 4096 elements (16 per thread) per block, each
        // block followed by one per-system reduction, but at least ~600
        // blocks to fill the GPU; a chunk never spans two systems.
        const int crow = std::max(1, std::min(std::max(1, 4096 / n), p->R / 600));
        std::vector<int> c0, cn, cs, sc0(p->B + 1);
        for (int s = 0; s < p->B; ++s) {
            sc0[s] = (int)c0.size();
            const int r0 = p->sys_row0_h[s], C = p->sys[s].C;
            const int nch = (C + crow - 1) / crow;
            for (int c = 0; c < nch; ++c) {
                const int a = r0 + (int)((long long)C * c / nch);
                const int b = r0 + (int)((long long)C * (c + 1) / nch);
                c0.push_back(a);
                cn.push_back(b - a);
                cs.push_back(s);
            }
        }
        sc0[p->B] = (int)c0.size();
        p->nchunks = (int)c0.size();
        // the streamed reduction takes chunks of at most kBulkChunk elements
        // on 16-byte boundaries (n even: every chunk starts on an even element)
        const int max_rows = cn.empty() ? 0 : *std::max_element(cn.begin(), cn.end());
        const char *rmode = std::getenv("MSC_ARNOLDI_STREAM");
        const bool bulk_ok = p->mixed && n % 2 == 0 && (long long)max_rows * n <= msc::kBulkChunk;
        // Small chunks (a few rows: small batches, single systems) leave most
        // of a streamed block's threads idle; the register-streamed passes
        // split them across warps instead (cfg1, one 1681-row system in
        // 400-element chunks: 52 + 24 against 73 + 40 us per step).
        const bool bulk_big = (long long)max_rows * n >= msc::kBulkChunk / 2;
        // (MSC_ARNOLDI_STREAM=registers selects the register-streamed passes,
        // =reduce the streamed reduction with the register-streamed update,
        // =bulk both streamed wherever the chunks allow it)
        p->bulk_arnoldi = (bulk_ok && bulk_big) ? 2 : 0;
        if (bulk_ok && rmode && std::strcmp(rmode, "bulk") == 0) p->bulk_arnoldi = 2;
        if (bulk_ok && rmode && std::strcmp(rmode, "registers") == 0) p->bulk_arnoldi = 0;
        if (bulk_ok && rmode && std::strcmp(rmode, "reduce") == 0) p->bulk_arnoldi = 1;
        MSC_CUDA(p->wait_error.alloc(1));
        MSC_CUDA(cudaMemset(p->wait_error.p, 0, sizeof(int)));
        // the register-streamed reduction's last block stages its scalar work
        // in dynamic shared memory (up to the largest restart)
        MSC_CUDA(cudaFuncSetAttribute(msc::k_dcgs_reduce<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)dcgs_scratch_bytes(msc::kMaxRestart)));
        MSC_CUDA(cudaFuncSetAttribute(msc::k_dcgs_reduce<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                      (int)dcgs_scratch_bytes(msc::kMaxRestart)));
        if (p->bulk_arnoldi > 0)
            MSC_CUDA(cudaFuncSetAttribute(msc::k_dcgs_reduce_bulk,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)msc::dcgs_bulk_smem()));
        if (p->bulk_arnoldi > 1)
            MSC_CUDA(cudaFuncSetAttribute(msc::k_dcgs_update_bulk,
                                          cudaFuncAttributeMaxDynamicSharedMemorySize,
                                          (int)msc::dcgs_bulk_smem()));
        MSC_CUDA(upload(p->chunk_row0, c0));
        MSC_CUDA(upload(p->chunk_nrow, cn));
        MSC_CUDA(upload(p->chunk_sys, cs));
        MSC_CUDA(upload(p->sys_chunk0, sc0));
    }
    {
        // P2: enough blocks to fill the GPU (about 600 blocks of 256 threads)
        // without splitting a tile below 256 elements per block.
        const int tile_elems = msc::kTileRows * n;
        const int max_split = std::max(1, tile_elems / 256);
        p->split = std::max(1, std::min(max_split, (600 + p->ntiles - 1) / p->ntiles));
    }
    MSC_CUDA(p->partial.alloc((size_t)std::max(p->ntiles * p->split, p->nchunks) * p->pstride));
    MSC_CUDA(p->sys_counter.alloc(p->B));
    MSC_CUDA(cudaMemset(p->sys_counter.p, 0, p->B * sizeof(int)));
    MSC_CUDA(p->H.alloc((size_t)p->B * (m + 1) * m));
    MSC_CUDA(p->cs.alloc((size_t)p->B * m));
    MSC_CUDA(p->sn.alloc((size_t)p->B * m));
    MSC_CUDA(p->g.alloc((size_t)p->B * (m + 1)));
    MSC_CUDA(p->h1.alloc((size_t)p->B * (m + 2)));
    MSC_CUDA(p->h2.alloc((size_t)p->B * (m + 2)));
    MSC_CUDA(p->y.alloc((size_t)p->B * m));
    MSC_CUDA(p->Hraw.alloc((size_t)p->B * (m + 1) * m));
    MSC_CUDA(p->dsum.alloc((size_t)p->B * 2 * (m + 1)));
    MSC_CUDA(p->dcoef.alloc((size_t)p->B * (2 * m + 4)));
    MSC_CUDA(p->gsave.alloc(p->B));
    MSC_CUDA(cudaMemset(p->Hraw.p, 0, p->Hraw.count * sizeof(double2)));
    MSC_CUDA(cudaMemset(p->dcoef.p, 0, p->dcoef.count * sizeof(double2)));
    MSC_CUDA(p->scale.alloc(p->B));
    MSC_CUDA(p->resid.alloc(p->B));
    MSC_CUDA(p->beta0.alloc(p->B));
    MSC_CUDA(p->est.alloc(p->B));
    MSC_CUDA(p->active.alloc(p->B));
    MSC_CUDA(p->kcyc.alloc(p->B));
    MSC_CUDA(p->iters.alloc(p->B));
    MSC_CUDA(p->projv.alloc(p->B));
    MSC_CUDA(p->cycles.alloc(p->B));
    MSC_CUDA(p->unfinished.alloc(p->B));
    MSC_CUDA(p->status.alloc(p->B));
    MSC_CUDA(p->counter.alloc(1));
    MSC_CUDA(cudaMemset(p->H.p, 0, p->H.count * sizeof(double2)));
    MSC_CUDA(cudaMemset(p->h1.p, 0, p->h1.count * sizeof(double2)));
    MSC_CUDA(cudaMemset(p->y.p, 0, p->y.count * sizeof(double2)));

    tm.mark("solver allocations");
    {
        msc_status tst = setup_tensor_core(p);
        if (tst != MSC_OK) return tst;
    }
    tm.mark("tensor-core setup");
    {
        msc_status tst = autotune(p);
        if (tst != MSC_OK) return tst;
    }
    tm.mark("autotune");
    if (p->gs) {
        msc_status gst = ensure_gs_levels(p);
        if (gst != MSC_OK) return gst;
        tm.mark("Gauss-Seidel levels");
    }
    MSC_CUDA(cudaMallocHost(&p->kcyc_host, p->B * sizeof(int)));
    for (int s = 0; s < p->B; ++s) p->kcyc_host[s] = 0;
    p->tev.resize((size_t)msc_plan::kKinds * (m + 1) * 2);
    for (cudaEvent_t &e : p->tev) MSC_CUDA(cudaEventCreate(&e));
    msc_status st = capture(p, record_cycle_start, &p->g_start, &p->launches_start);
    if (st != MSC_OK) return st;
    st = capture(p, record_cycle_start_zero, &p->g_start0, &p->launches_start0);
    if (st != MSC_OK) return st;
    st = capture(p, record_cycle_iterations, &p->g_iter, &p->launches_iter);
    if (st != MSC_OK) return st;
    tm.mark("graph capture");
    p->finalized = true;
    return MSC_OK;
}

// Level sets of the block Gauss-Seidel sweep: a row's level is one more
// than the highest level among its lower neighbours (neighbour rows of the
// same system with a smaller row index, through any coupling tap), so the
// rows of one level can be solved at the same time.  Built once per plan.
msc_status ensure_gs_levels(msc_plan *p)
{
    if (p->gs_ready) return MSC_OK;
    const int ntor = p->nkx * p->nky;
    std::vector<int> sys_lvl(p->B + 1, 0), lvl_start, rows;
    std::vector<int> low_ptr(1, 0), low_tap, low_row;   // lower neighbours per row (CSR)
    rows.reserve(p->R);
    low_ptr.reserve(p->R + 1);
    std::vector<int> pos_row(ntor, -1);
    for (int s = 0; s < p->B; ++s) {
        const SystemHost &sh = p->sys[s];
        const int r0 = p->sys_row0_h[s];
        for (int j = 0; j < sh.C; ++j) pos_row[sh.ix[j] * p->nky + sh.iy[j]] = j;
        std::vector<int> lvl(sh.C, 0);
        int nlvl = 0;
        for (int j = 0; j < sh.C; ++j) {
            int best = -1;
            for (int t = 0; t < p->K; ++t) {
                int sx = sh.ix[j] - p->taps[t].first;
                sx += sx < 0 ? p->nkx : 0;
                int sy = sh.iy[j] - p->taps[t].second;
                sy += sy < 0 ? p->nky : 0;
                const int q = pos_row[sx * p->nky + sy];
                if (q >= 0 && q < j) {
                    best = std::max(best, lvl[q]);
                    low_tap.push_back(t);
                    low_row.push_back(r0 + q);
                }
            }
            low_ptr.push_back((int)low_tap.size());
            lvl[j] = best + 1;
            nlvl = std::max(nlvl, lvl[j] + 1);
        }
        sys_lvl[s] = (int)lvl_start.size();
        std::vector<int> count(nlvl + 1, 0);
        for (int j = 0; j < sh.C; ++j) ++count[lvl[j] + 1];
        for (int l = 0; l < nlvl; ++l) count[l + 1] += count[l];
        const int base = (int)rows.size();
        rows.resize(base + sh.C);
        std::vector<int> fill(count.begin(), count.end() - 1);
        for (int j = 0; j < sh.C; ++j) rows[base + fill[lvl[j]]++] = p->sys_row0_h[s] + j;
        for (int l = 0; l < nlvl; ++l) lvl_start.push_back(base + count[l]);
        for (int j = 0; j < sh.C; ++j) pos_row[sh.ix[j] * p->nky + sh.iy[j]] = -1;
    }
    sys_lvl[p->B] = (int)lvl_start.size();
    lvl_start.push_back((int)rows.size());
    if (low_tap.empty()) {
        low_tap.push_back(0);
        low_row.push_back(0);
    }
    MSC_CUDA(upload(p->gs_low_ptr, low_ptr));
    MSC_CUDA(upload(p->gs_low_tap, low_tap));
    MSC_CUDA(upload(p->gs_low_row, low_row));
    MSC_CUDA(upload(p->gs_sys_lvl, sys_lvl));
    MSC_CUDA(upload(p->gs_lvl_start, lvl_start));
    MSC_CUDA(upload(p->gs_lvl_rows, rows));
    int dev = 0, optin = 0;
    MSC_CUDA(cudaGetDevice(&dev));
    MSC_CUDA(cudaDeviceGetAttribute(&optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev));
    const size_t room = (size_t)optin - 1024;    // static shared memory of the kernel
    p->gs_e64_smem = gs_smem<double>(p->n, true) <= room;
    p->gs_e32_smem = p->E32.p && gs_smem<float>(p->n, true) <= room;
    MSC_CUDA(cudaFuncSetAttribute(msc::k_gs_sweep<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)gs_smem<double>(p->n, p->gs_e64_smem)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_gs_sweep<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)gs_smem<float>(p->n, p->gs_e32_smem)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_masked<double>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_coupling(msc::kMaxTaps)));
    MSC_CUDA(cudaFuncSetAttribute(msc::k_coupling_masked<float>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)smem_coupling(msc::kMaxTaps)));
    p->gs_ready = true;
    return MSC_OK;
}

// FP64 eigen-decomposition H = E diag(w) E^T of a symmetric n x n host
// matrix on the current device (msc_eigh_gpu.cuh): Householder reduction and
// both O(n^3) accumulations on the GPU, the O(n^2) tridiagonal QR iteration
// on the host.  w ascending; E row-major, eigenvector k in column k.
msc_status device_symmetric_eigh(int n, const double *H, double *w, double *E)
{
    namespace eg = msc::eig;
    DevBuf<double> A, R, d, e, Zt, Ed, rc, rs;
    DevBuf<int> applied, rk, dest;
    std::vector<double> Hh(H, H + (size_t)n * n);
    MSC_CUDA(upload(A, Hh));
    MSC_CUDA(R.alloc((size_t)n * n));
    MSC_CUDA(d.alloc(n));
    MSC_CUDA(e.alloc(n));
    MSC_CUDA(applied.alloc(n));
    MSC_CUDA(cudaMemset(R.p, 0, (size_t)n * n * sizeof(double)));
    MSC_CUDA(cudaMemset(e.p, 0, (size_t)n * sizeof(double)));
    const size_t tri_smem = n <= eg::kTriSmemMaxN ? (size_t)n * n * sizeof(double) : 0;
    MSC_CUDA(cudaFuncSetAttribute(eg::k_tridiagonalize, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)((size_t)eg::kTriSmemMaxN * eg::kTriSmemMaxN * sizeof(double))));
    eg::k_tridiagonalize<<<1, eg::kTriThreads, tri_smem>>>(n, A.p, R.p, d.p, e.p, applied.p);
    MSC_CUDA(cudaGetLastError());
    std::vector<double> dh(n), eh(n);
    MSC_CUDA(cudaMemcpy(dh.data(), d.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    MSC_CUDA(cudaMemcpy(eh.data(), e.p, n * sizeof(double), cudaMemcpyDeviceToHost));
    eh[n - 1] = 0.0;
    std::vector<int> rkh;
    std::vector<double> rch, rsh;
    rkh.reserve((size_t)n * n);
    rch.reserve((size_t)n * n);
    rsh.reserve((size_t)n * n);
    if (msc::tridiagonal_qr_rotations(n, dh, eh, rkh, rch, rsh) != 0)
        return fail(MSC_ERR_EIGEN, "eigensolver did not converge");
    const int nrot = (int)rkh.size();
    if (nrot > 0) {
        MSC_CUDA(upload(rk, rkh));
        MSC_CUDA(upload(rc, rch));
        MSC_CUDA(upload(rs, rsh));
    }
    MSC_CUDA(Zt.alloc((size_t)n * n));
    // rows of Z per CTA: as many as fit 200 KB of shared memory (32 or 16)
    if ((size_t)n * 32 * sizeof(double) <= 200 * 1024) {
        const size_t sm = (size_t)n * 32 * sizeof(double);
        MSC_CUDA(cudaFuncSetAttribute(eg::k_apply_rotations<32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        eg::k_apply_rotations<32><<<(n + 31) / 32, 32, sm>>>(n, nrot, rk.p, rc.p, rs.p, Zt.p);
    } else {
        const size_t sm = (size_t)n * 16 * sizeof(double);
        MSC_CUDA(cudaFuncSetAttribute(eg::k_apply_rotations<16>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        eg::k_apply_rotations<16><<<(n + 15) / 16, 16, sm>>>(n, nrot, rk.p, rc.p, rs.p, Zt.p);
    }
    MSC_CUDA(cudaGetLastError());
    // ascending order: column j of Q_H Z goes to column dest[j]
    std::vector<int> order(n), desth(n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int i, int j) { return dh[i] < dh[j]; });
    for (int k = 0; k < n; ++k) {
        desth[order[k]] = k;
        w[k] = dh[order[k]];
    }
    MSC_CUDA(upload(dest, desth));
    MSC_CUDA(Ed.alloc((size_t)n * n));
    if ((size_t)n * 32 * sizeof(double) <= 200 * 1024) {
        const size_t sm = (size_t)n * 32 * sizeof(double);
        MSC_CUDA(cudaFuncSetAttribute(eg::k_back_transform<32>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        eg::k_back_transform<32><<<(n + 31) / 32, 256, sm>>>(n, R.p, applied.p, Zt.p, dest.p, Ed.p);
    } else {
        const size_t sm = (size_t)n * 16 * sizeof(double);
        MSC_CUDA(cudaFuncSetAttribute(eg::k_back_transform<16>,
                                      cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
        eg::k_back_transform<16><<<(n + 15) / 16, 256, sm>>>(n, R.p, applied.p, Zt.p, dest.p, Ed.p);
    }
    MSC_CUDA(cudaGetLastError());
    MSC_CUDA(cudaMemcpy(E, Ed.p, (size_t)n * n * sizeof(double), cudaMemcpyDeviceToHost));
    return MSC_OK;
}

// Process-wide caches.  Sweeps build many plans over one potential (new
// beams, same z grid): the H0 eigen-decomposition and the autotuner's
// choices are reused instead of recomputed.
struct EigenEntry {
    std::vector<double> H, lam, E;
};
std::mutex g_cache_mutex;
std::vector<EigenEntry> g_eigen_cache;   // few entries, most recent last

bool eigen_cache_lookup(const std::vector<double> &H, std::vector<double> &lam, std::vector<double> &E)
{
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    for (const EigenEntry &e : g_eigen_cache)
        if (e.H.size() == H.size() && std::memcmp(e.H.data(), H.data(), H.size() * sizeof(double)) == 0) {
            lam = e.lam;
            E = e.E;
            return true;
        }
    return false;
}

void eigen_cache_store(const std::vector<double> &H, const std::vector<double> &lam,
                       const std::vector<double> &E)
{
    std::lock_guard<std::mutex> lock(g_cache_mutex);
    if (g_eigen_cache.size() >= 8) g_eigen_cache.erase(g_eigen_cache.begin());
    g_eigen_cache.push_back({H, lam, E});
}

// FP64 recovery of the systems a mixed-precision solve left unconverged.
// The FP32 inner solve of a hard beam can stall near its own rounding level
// (residual ~1e-5) before max_refinements runs out.  Those systems are
// solved again by a plain FP64 plan over the same potential, holding only
// them: same operator (forward or adjoint), same right-hand sides, the mixed
// solution as the initial guess (zero for a system whose state went
// non-finite), FP64 restart and iteration limits of the parent's options.
// Their rows of the parent's x are then replaced by the FP64 solution and
// their iteration counts, status and residual by the FP64 solve's.
msc_status fp64_recover(msc_plan *p, const std::vector<int> &failed, const std::vector<int> &status,
                        std::vector<msc_result> &out)
{
    const int nf = (int)failed.size();
    const int n = p->n;
    msc_plan_desc d = p->desc;
    d.precision = MSC_PRECISION_FP64;
    d.n_systems = nf;
    d.flags = 0;
    msc_plan *c = nullptr;
    msc_status st = msc_plan_create(&c, &d);
    if (st != MSC_OK) return st;
    struct Guard {
        msc_plan *c;
        ~Guard() { msc_plan_destroy(c); }
    } guard{c};
    // the potential in its [nkx][nky][n] layout from the parent's taps and V_00
    std::vector<double2> V((size_t)p->nkx * p->nky * n, double2{0.0, 0.0});
    for (int k = 0; k < n; ++k) V[k] = double2{p->v00_host[k], 0.0};
    for (int t = 0; t < p->K; ++t) {
        double2 *dst = V.data() + ((size_t)p->taps[t].first * p->nky + p->taps[t].second) * n;
        std::copy(p->Vt_host.begin() + (size_t)t * n, p->Vt_host.begin() + (size_t)(t + 1) * n, dst);
    }
    st = msc_plan_set_potential(c, reinterpret_cast<const double *>(V.data()), p->T_host.data());
    if (st != MSC_OK) return st;
    for (int k = 0; k < nf; ++k) {
        const SystemHost &sh = p->sys[failed[k]];
        c->sys[k] = sh;
    }
    st = finalize(c);
    if (st != MSC_OK) return st;
    if (p->adjoint) {
        st = msc_plan_set_adjoint(c, 1);
        if (st != MSC_OK) return st;
    }
    // right-hand sides and initial guesses: the parent's rows of each system
    const size_t vs = (size_t)c->R * n;
    MSC_CUDA(c->X0.alloc(vs));
    cudaStream_t cs = c->stream;
    for (int k = 0; k < nf; ++k) {
        const int s = failed[k];
        const int r0 = p->sys_row0_h[s], C = p->sys[s].C, q0 = c->sys_row0_h[k];
        MSC_CUDA(cudaMemcpyAsync(c->row_rhs.p + q0, p->row_rhs.p + r0, C * sizeof(double2),
                                 cudaMemcpyDeviceToDevice, cs));
        if (status[s] == MSC_ERR_NONFINITE)
            MSC_CUDA(cudaMemsetAsync(c->X0.p + (size_t)q0 * n, 0, (size_t)C * n * sizeof(double2), cs));
        else
            MSC_CUDA(cudaMemcpyAsync(c->X0.p + (size_t)q0 * n, p->X.p + (size_t)r0 * n,
                                     (size_t)C * n * sizeof(double2), cudaMemcpyDeviceToDevice, cs));
    }
    msc::k_system_norms<<<c->B, 256, 0, cs>>>(c->sys_row0.p, c->row_rhs.p, c->bnorm.p);
    MSC_CUDA(cudaGetLastError());
    MSC_CUDA(cudaStreamSynchronize(cs));
    c->has_x0 = true;
    out.assign(nf, msc_result{});
    st = msc_solve(c, nullptr, nullptr, out.data(), cs);
    if (st != MSC_OK && st != MSC_ERR_NOT_CONVERGED && st != MSC_ERR_NONFINITE) return st;
    for (int k = 0; k < nf; ++k) {
        const int s = failed[k];
        const int r0 = p->sys_row0_h[s], C = p->sys[s].C, q0 = c->sys_row0_h[k];
        MSC_CUDA(cudaMemcpyAsync(p->X.p + (size_t)r0 * n, c->X.p + (size_t)q0 * n,
                                 (size_t)C * n * sizeof(double2), cudaMemcpyDeviceToDevice, cs));
    }
    MSC_CUDA(cudaStreamSynchronize(cs));
    return MSC_OK;
}

}  // namespace

extern "C" {

const char *msc_last_error(void) { return g_last_error.c_str(); }
const char *msc_version(void) { return "multiscat_b200 0.1 (sm_100a)"; }

msc_status msc_plan_create(msc_plan **plan, const msc_plan_desc *desc)
{
    if (!plan || !desc) return fail(MSC_ERR_ARG, "null argument");
    *plan = nullptr;
    if (desc->n_z <= 1 || desc->n_z > msc::kMaxNz || desc->nkx <= 0 || desc->nky <= 0 ||
        desc->n_systems <= 0)
        return fail(MSC_ERR_DIMS, "bad plan dimensions");
    if (desc->restart < 1 || desc->restart > msc::kMaxRestart || desc->max_iterations < 1 ||
        !(desc->rtol > 0.0))
        return fail(MSC_ERR_ARG, "bad solver options");
    if (desc->precision != MSC_PRECISION_FP64 && desc->precision != MSC_PRECISION_MIXED)
        return fail(MSC_ERR_ARG, "unknown precision");
    if (desc->precision == MSC_PRECISION_MIXED &&
        (desc->inner_restart < 0 || desc->inner_restart > msc::kMaxRestart || desc->inner_rtol < 0.0 ||
         desc->max_refinements < 0))
        return fail(MSC_ERR_ARG, "bad mixed-precision options");
    if (desc->precond_order < 0 || desc->precond_order > 8)
        return fail(MSC_ERR_ARG, "precond_order must be in 0..8");
    msc_plan *p = new (std::nothrow) msc_plan();
    if (!p) return fail(MSC_ERR_CUDA, "host allocation failed");
    p->desc = *desc;
    p->n = desc->n_z;
    p->nkx = desc->nkx;
    p->nky = desc->nky;
    p->B = desc->n_systems;
    p->m = desc->restart;
    p->mixed = desc->precision == MSC_PRECISION_MIXED;
    if (p->mixed) {
        // The inner FP32 solve only has to gain inner_rtol (3e-6) per
        // refinement step, which takes ~15-20 iterations here; longer inner
        // cycles only add launches of systems that already stopped.  (On the
        // 512-beam cfg2 batch 3e-6 saves refinement steps against 1e-5:
        // 6929 against 6720 solves/s; 3e-5 is slower again.)
        p->m = desc->inner_restart > 0 ? desc->inner_restart : std::min(desc->restart, 20);
        p->inner_rtol = desc->inner_rtol > 0.0 ? desc->inner_rtol : 3e-6;
        p->cgs1_inner = (desc->flags & 4) != 0;
        if (p->cgs1_inner) p->dcgs = false;
        p->max_cycles = desc->max_refinements > 0 ? desc->max_refinements : 30;
    }
    if (desc->flags & 16) p->dcgs = false;     // classical Gram-Schmidt, two passes (CGS2)
    if (desc->flags & 32) p->gs = true;        // block Gauss-Seidel preconditioner M = L^-1
    p->sys.resize(p->B);
    msc_status st = set_kernel_attributes(p->n, 0);
    if (st != MSC_OK) { delete p; return st; }
    cudaError_t e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaMallocHost(&p->counter_host, sizeof(int));
    if (e != cudaSuccess) {
        delete p;
        return fail(MSC_ERR_CUDA, std::string("plan create: ") + cudaGetErrorString(e));
    }
    *plan = p;
    return MSC_OK;
}

msc_status msc_plan_destroy(msc_plan *plan)
{
    if (!plan) return MSC_OK;
    SetupTimer tm;
    cudaStreamSynchronize(plan->stream);
    cudaDeviceSynchronize();     // nothing may still use the buffers going back to the pool
    delete plan;
    tm.mark("plan destroy");
    return MSC_OK;
}

msc_status msc_release_cached_memory(void)
{
    cudaMemPool_t pool;
    MSC_CUDA(plan_pool(&pool));
    MSC_CUDA(cudaDeviceSynchronize());
    MSC_CUDA(cudaMemPoolTrimTo(pool, 0));
    return MSC_OK;
}

msc_status msc_plan_set_potential(msc_plan *p, const double *potential_values, const double *kinetic)
{
    if (!p || !potential_values || !kinetic) return fail(MSC_ERR_ARG, "null argument");
    if (p->finalized) return fail(MSC_ERR_ARG, "plan already finalized");
    const int n = p->n, nkx = p->nkx, nky = p->nky;
    const double2 *V = reinterpret_cast<const double2 *>(potential_values);
    // H0 = T + diag Re V00
    std::vector<double> H(kinetic, kinetic + (size_t)n * n);
    p->T_host.assign(kinetic, kinetic + (size_t)n * n);
    p->v00_host.resize(n);
    for (int k = 0; k < n; ++k) {
        p->v00_host[k] = V[k].x;   // storage (0, 0)
        H[(size_t)k * n + k] += V[k].x;
    }
    for (double hv : H)
        if (!std::isfinite(hv)) return fail(MSC_ERR_NONFINITE, "non-finite kinetic or V00");
    if (!eigen_cache_lookup(H, p->lam_host, p->E_host)) {
        p->lam_host.resize(n);
        p->E_host.resize((size_t)n * n);
        msc_status est = device_symmetric_eigh(n, H.data(), p->lam_host.data(), p->E_host.data());
        if (est != MSC_OK) return est;
        eigen_cache_store(H, p->lam_host, p->E_host);
    }
    p->en_host.resize(n);
    for (int k = 0; k < n; ++k) p->en_host[k] = p->E_host[(size_t)(n - 1) * n + k];
    std::vector<double> ET((size_t)n * n);
    for (int z = 0; z < n; ++z)
        for (int k = 0; k < n; ++k) ET[(size_t)k * n + z] = p->E_host[(size_t)z * n + k];
    // coupling taps: every offset d != 0 with V_d or V_{-d} nonzero (the set is
    // closed under d -> -d so that A^H, whose tap at d is conj(V_{-d}), runs on
    // the same offsets and tables)
    p->taps.clear();
    p->Vt_host.clear();
    p->Vt_adj_host.clear();
    auto nonzero = [&](int dx, int dy) {
        const double2 *v = V + ((size_t)dx * nky + dy) * n;
        for (int k = 0; k < n; ++k)
            if (v[k].x != 0.0 || v[k].y != 0.0) return true;
        return false;
    };
    for (int dx = 0; dx < nkx; ++dx)
        for (int dy = 0; dy < nky; ++dy) {
            if (dx == 0 && dy == 0) continue;
            const int mx = (nkx - dx) % nkx, my = (nky - dy) % nky;
            if (!nonzero(dx, dy) && !nonzero(mx, my)) continue;
            const double2 *v = V + ((size_t)dx * nky + dy) * n;
            const double2 *vm = V + ((size_t)mx * nky + my) * n;
            p->taps.emplace_back(dx, dy);
            p->Vt_host.insert(p->Vt_host.end(), v, v + n);
            for (int k = 0; k < n; ++k) p->Vt_adj_host.push_back(msc::cconj(vm[k]));
        }
    p->adjoint = false;
    p->K = (int)p->taps.size();
    if (p->K > msc::kMaxTaps) return fail(MSC_ERR_DIMS, "too many nonzero coupling taps");
    for (const double2 &v : p->Vt_host)
        if (!std::isfinite(v.x) || !std::isfinite(v.y)) return fail(MSC_ERR_NONFINITE, "non-finite potential");
    MSC_CUDA(upload(p->E, p->E_host));
    MSC_CUDA(upload(p->ET, ET));
    MSC_CUDA(upload(p->Tm, p->T_host));
    MSC_CUDA(upload(p->lam, p->lam_host));
    MSC_CUDA(upload(p->en, p->en_host));
    MSC_CUDA(upload(p->v00, p->v00_host));
    if (p->K > 0) {
        MSC_CUDA(upload(p->Vt, p->Vt_host));
    } else {
        std::vector<double2> dummy(1, double2{0.0, 0.0});
        MSC_CUDA(upload(p->Vt, dummy));
    }
    if (p->mixed) {
        auto to32 = [](const std::vector<double> &v) {
            return std::vector<float>(v.begin(), v.end());
        };
        MSC_CUDA(upload(p->E32, to32(p->E_host)));
        MSC_CUDA(upload(p->ET32, to32(ET)));
        MSC_CUDA(upload(p->lam32, to32(p->lam_host)));
        MSC_CUDA(upload(p->en32, to32(p->en_host)));
        std::vector<float2> vt32(std::max<size_t>(p->Vt_host.size(), 1), make_float2(0.f, 0.f));
        for (size_t i = 0; i < p->Vt_host.size(); ++i)
            vt32[i] = make_float2((float)p->Vt_host[i].x, (float)p->Vt_host[i].y);
        MSC_CUDA(upload(p->Vt32, vt32));
    }
    p->potential_set = true;
    return MSC_OK;
}

msc_status msc_plan_set_system(msc_plan *p, int32_t s, int32_t n_channels, const int32_t *channel_ix,
                               const int32_t *channel_iy, const double *pkd, const double *wave_b,
                               const double *wave_c, int32_t specular, const double *wave_a_spec)
{
    if (!p || !channel_ix || !channel_iy || !pkd || !wave_b || !wave_c)
        return fail(MSC_ERR_ARG, "null argument");
    if (p->finalized) return fail(MSC_ERR_ARG, "plan already finalized");
    if (s < 0 || s >= p->B) return fail(MSC_ERR_ARG, "system index out of range");
    if (n_channels <= 0 || n_channels > p->nkx * p->nky) return fail(MSC_ERR_DIMS, "bad channel count");
    if (specular < 0 || specular >= n_channels) return fail(MSC_ERR_ARG, "bad specular index");
    SystemHost &sh = p->sys[s];
    sh.C = n_channels;
    sh.spec = specular;
    sh.ix.assign(channel_ix, channel_ix + n_channels);
    sh.iy.assign(channel_iy, channel_iy + n_channels);
    std::vector<char> seen((size_t)p->nkx * p->nky, 0);
    for (int j = 0; j < n_channels; ++j) {
        if (sh.ix[j] < 0 || sh.ix[j] >= p->nkx || sh.iy[j] < 0 || sh.iy[j] >= p->nky)
            return fail(MSC_ERR_DIMS, "channel position outside the torus");
        char &f = seen[(size_t)sh.ix[j] * p->nky + sh.iy[j]];
        if (f) return fail(MSC_ERR_DIMS, "duplicate channel position");
        f = 1;
    }
    sh.pkd.assign(pkd, pkd + n_channels);
    sh.b.resize(n_channels);
    sh.c.resize(n_channels);
    for (int j = 0; j < n_channels; ++j) {
        sh.b[j] = double2{wave_b[2 * j], wave_b[2 * j + 1]};
        sh.c[j] = double2{wave_c[2 * j], wave_c[2 * j + 1]};
        if (!std::isfinite(sh.pkd[j]) || !std::isfinite(sh.c[j].x) || !std::isfinite(sh.c[j].y))
            return fail(MSC_ERR_NONFINITE, "non-finite channel data");
    }
    sh.a_spec = wave_a_spec ? double2{wave_a_spec[0], wave_a_spec[1]} : double2{0.0, 0.0};
    if (sh.b[specular].x == 0.0 && sh.b[specular].y == 0.0)
        return fail(MSC_ERR_ARG, "specular channel is closed (b = 0)");
    sh.set = true;
    return MSC_OK;
}

msc_status msc_plan_set_systems(msc_plan *p, int32_t first, int32_t count, const int64_t *offsets,
                                const int32_t *channel_ix, const int32_t *channel_iy, const double *pkd,
                                const double *wave_b, const double *wave_c, const int32_t *specular,
                                const double *wave_a_spec)
{
    if (!p || !offsets || !specular) return fail(MSC_ERR_ARG, "null argument");
    if (count < 0 || first < 0 || (int64_t)first + count > p->B)
        return fail(MSC_ERR_ARG, "system range out of range");
    if (offsets[0] != 0) return fail(MSC_ERR_ARG, "offsets[0] must be 0");
    for (int32_t k = 0; k < count; ++k) {
        const int64_t lo = offsets[k], hi = offsets[k + 1];
        if (hi < lo || hi - lo > (int64_t)p->nkx * p->nky) return fail(MSC_ERR_DIMS, "bad channel count");
        msc_status st = msc_plan_set_system(p, first + k, (int32_t)(hi - lo), channel_ix + lo,
                                            channel_iy + lo, pkd + lo, wave_b + 2 * lo, wave_c + 2 * lo,
                                            specular[k], wave_a_spec ? wave_a_spec + 2 * k : nullptr);
        if (st != MSC_OK) return st;
    }
    return MSC_OK;
}

int64_t msc_plan_total_rows(const msc_plan *p)
{
    if (!p) return -1;
    int64_t r = 0;
    for (const SystemHost &sh : p->sys) r += sh.C;
    return r;
}

msc_status msc_solve(msc_plan *p, double *psi_out, double *intensities_out, msc_result *results,
                     void *stream)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t user = reinterpret_cast<cudaStream_t>(stream);
    cudaStream_t ps = p->stream;
    cudaEvent_t ev;
    MSC_CUDA(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    MSC_CUDA(cudaEventRecord(ev, user));
    MSC_CUDA(cudaStreamWaitEvent(ps, ev, 0));
    // reset state (x = the warm-start guess when one is set, else 0)
    const size_t vs = (size_t)p->R * p->n;
    if (p->has_x0)
        MSC_CUDA(cudaMemcpyAsync(p->X.p, p->X0.p, vs * sizeof(double2), cudaMemcpyDeviceToDevice, ps));
    else
        MSC_CUDA(cudaMemsetAsync(p->X.p, 0, vs * sizeof(double2), ps));
    MSC_CUDA(cudaMemsetAsync(p->iters.p, 0, p->B * sizeof(int), ps));
    MSC_CUDA(cudaMemsetAsync(p->projv.p, 0, p->B * sizeof(int), ps));
    MSC_CUDA(cudaMemsetAsync(p->cycles.p, 0, p->B * sizeof(int), ps));
    MSC_CUDA(cudaMemsetAsync(p->status.p, 0, p->B * sizeof(int), ps));
    MSC_CUDA(cudaMemsetAsync(p->kcyc.p, 0, p->B * sizeof(int), ps));
    {
        std::vector<int> ones(p->B, 1);
        MSC_CUDA(cudaMemcpyAsync(p->unfinished.p, ones.data(), p->B * sizeof(int),
                                 cudaMemcpyHostToDevice, ps));
        MSC_CUDA(cudaStreamSynchronize(ps));
    }
    const int max_cycles = p->desc.max_iterations + 2;
    int cycle = 0;
    int64_t launches = 0;
    bool pending = false;
    for (; cycle < max_cycles; ++cycle) {
        const bool x_zero = cycle == 0 && !p->has_x0;
        MSC_CUDA(cudaGraphLaunch(x_zero ? p->g_start0 : p->g_start, ps));
        launches += x_zero ? p->launches_start0 : p->launches_start;
        MSC_CUDA(cudaStreamSynchronize(ps));
        if (pending && p->timing) accumulate_timing(p);
        pending = false;
        if (*p->counter_host == 0) break;
        MSC_CUDA(cudaGraphLaunch(p->g_iter, ps));
        launches += p->launches_iter;
        pending = true;
    }
    p->launches_last = launches;
    p->cycles_last = cycle;
    MSC_CUDA(cudaGetLastError());
    if (p->use_tc) {
        int tc_err = 0;
        MSC_CUDA(cudaMemcpy(&tc_err, p->tc_error.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (tc_err) return fail(MSC_ERR_CUDA, "tensor-core block inverse timed out on an mbarrier wait");
    }
    {
        int w_err = 0;
        MSC_CUDA(cudaMemcpy(&w_err, p->wait_error.p, sizeof(int), cudaMemcpyDeviceToHost));
        if (w_err) return fail(MSC_ERR_CUDA, "a bulk-copy wait of the streamed Arnoldi passes timed out");
    }
    std::vector<int> iters(p->B), cycles(p->B), status(p->B), unfinished(p->B), fallback(p->B, 0);
    std::vector<int> projv(p->B);
    std::vector<double> resid(p->B);
    MSC_CUDA(cudaMemcpyAsync(iters.data(), p->iters.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaMemcpyAsync(projv.data(), p->projv.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaMemcpyAsync(cycles.data(), p->cycles.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaMemcpyAsync(status.data(), p->status.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaMemcpyAsync(unfinished.data(), p->unfinished.p, p->B * sizeof(int), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaMemcpyAsync(resid.data(), p->resid.p, p->B * sizeof(double), cudaMemcpyDeviceToHost, ps));
    MSC_CUDA(cudaStreamSynchronize(ps));
    for (int s = 0; s < p->B; ++s)
        if (unfinished[s]) status[s] = MSC_ERR_NOT_CONVERGED;
    p->fallbacks_last = 0;
    if (p->mixed && !(p->desc.flags & 8)) {
        std::vector<int> failed;
        for (int s = 0; s < p->B; ++s)
            if (status[s] == MSC_ERR_NOT_CONVERGED || status[s] == MSC_ERR_NONFINITE) failed.push_back(s);
        if (!failed.empty()) {
            std::vector<msc_result> rec;
            msc_status rst = fp64_recover(p, failed, status, rec);
            if (rst != MSC_OK) {
                cudaEventDestroy(ev);
                return rst;
            }
            for (size_t k = 0; k < failed.size(); ++k) {
                const int s = failed[k];
                iters[s] += rec[k].iterations;
                projv[s] += rec[k].basis_vectors;
                cycles[s] += rec[k].refinements;
                status[s] = rec[k].status;
                resid[s] = rec[k].residual;
                fallback[s] = 1;
            }
            p->fallbacks_last = (int)failed.size();
        }
    }
    if (psi_out)
        MSC_CUDA(cudaMemcpyAsync(psi_out, p->X.p, vs * sizeof(double2), cudaMemcpyDeviceToDevice, ps));
    if (intensities_out) {
        msc::k_intensities<<<(p->R + 255) / 256, 256, 0, ps>>>(
            p->R, 0, p->n, p->row_sys.p, p->sys_spec_row.p, p->sys_aspec.p, p->row_b.p, p->X.p,
            intensities_out);
        MSC_CUDA(cudaGetLastError());
    }
    MSC_CUDA(cudaEventRecord(ev, ps));
    MSC_CUDA(cudaStreamWaitEvent(user, ev, 0));
    MSC_CUDA(cudaStreamSynchronize(ps));
    cudaEventDestroy(ev);
    msc_status worst = MSC_OK;
    for (int s = 0; s < p->B; ++s) {
        const int sst = status[s];
        if (results) {
            results[s].iterations = iters[s];
            results[s].refinements = cycles[s];
            results[s].status = sst;
            results[s].fp64_fallback = fallback[s];
            results[s].residual = resid[s];
            results[s].basis_vectors = projv[s];
            results[s].reserved = 0;
        }
        if (sst != MSC_OK && worst == MSC_OK) worst = (msc_status)sst;
    }
    if (worst != MSC_OK) g_last_error = "at least one system did not converge";
    return worst;
}

msc_status msc_plan_get_info(const msc_plan *p, msc_plan_info *info)
{
    if (!p || !info) return fail(MSC_ERR_ARG, "null argument");
    info->total_rows = msc_plan_total_rows(p);
    info->n_taps = p->K;
    info->n_tiles = p->ntiles;
    info->launches_last = p->launches_last;
    info->cycles_last = p->cycles_last;
    info->fallbacks_last = p->fallbacks_last;
    return MSC_OK;
}

msc_status msc_plan_set_kernel_timing(msc_plan *p, int enable)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    const bool want = enable != 0;
    if (want == p->timing) return MSC_OK;
    p->timing = want;
    for (int k = 0; k < msc_plan::kKinds; ++k) {
        p->t_ms[k] = 0.0;
        p->t_launches[k] = 0;
    }
    return capture(p, record_cycle_iterations, &p->g_iter, &p->launches_iter);
}

msc_status msc_plan_kernel_timing(msc_plan *p, double *ms, int64_t *launches)
{
    if (!p || !ms || !launches) return fail(MSC_ERR_ARG, "null argument");
    for (int k = 0; k < msc_plan::kKinds; ++k) {
        ms[k] = p->t_ms[k];
        launches[k] = p->t_launches[k];
        p->t_ms[k] = 0.0;
        p->t_launches[k] = 0;
    }
    return MSC_OK;
}

msc_status msc_debug_apply_coupling(msc_plan *p, const double *x, double *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    launch_coupling(p, nullptr, reinterpret_cast<const double2 *>(x), nullptr, 1.0,
                    reinterpret_cast<double2 *>(y), s);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_debug_apply_block_inverse(msc_plan *p, const double *x, double *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    launch_block_inverse(p, nullptr, reinterpret_cast<const double2 *>(x),
                         reinterpret_cast<double2 *>(y), 0, s);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_debug_apply_operator(msc_plan *p, const double *x, double *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // y = -(b - D x) with b switched off, then y += V_off x
    launch_residual_diag(p, nullptr, reinterpret_cast<const double2 *>(x), p->TMP.p, 0, s);
    launch_coupling(p, nullptr, reinterpret_cast<const double2 *>(x), p->TMP.p, -1.0,
                    reinterpret_cast<double2 *>(y), s);
    // y currently holds -(D x + V_off x)
    const size_t cnt = (size_t)p->R * p->n;
    msc::k_scale<<<(unsigned)std::min<size_t>((cnt + 255) / 256, 4096), 256, 0, s>>>(
        reinterpret_cast<double2 *>(y), cnt, -1.0);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_apply_lower_block(msc_plan *p, const double *x, double *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    if (x == y) return fail(MSC_ERR_ARG, "x and y must be different buffers");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    st = ensure_gs_levels(p);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    // y = -(-D x - V^lower x)
    launch_residual_diag(p, nullptr, reinterpret_cast<const double2 *>(x), p->TMP.p, 0, s);
    launch_coupling_masked_t<double>(p, nullptr, reinterpret_cast<const double2 *>(x), p->TMP.p,
                                     -1.0, 1, reinterpret_cast<double2 *>(y), s);
    const size_t cnt = (size_t)p->R * p->n;
    msc::k_scale<<<(unsigned)std::min<size_t>((cnt + 255) / 256, 4096), 256, 0, s>>>(
        reinterpret_cast<double2 *>(y), cnt, -1.0);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_solve_lower_block(msc_plan *p, const double *x, double *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    if (x == y) return fail(MSC_ERR_ARG, "x and y must be different buffers");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    st = ensure_gs_levels(p);
    if (st != MSC_OK) return st;
    launch_gs_sweep_t<double>(p, nullptr, reinterpret_cast<const double2 *>(x),
                              reinterpret_cast<double2 *>(y), reinterpret_cast<cudaStream_t>(stream));
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

const char *msc_plan_tuning_report(msc_plan *p)
{
    if (!p) return "";
    std::string r = "{";
    for (size_t i = 0; i < p->tune_log.size(); ++i) {
        if (i) r += ", ";
        r += "\"" + p->tune_log[i].first + "\": " + std::to_string(p->tune_log[i].second);
    }
    if (!r.empty() && r.size() > 1) r += ", ";
    const char *kn[6] = {"neighbour", "halo_y8", "halo_y4", "separable", "separable_z2",
                         "separable_rows"};
    r += "\"halo_hx\": " + std::to_string(p->use_halo ? p->halo_hx : 0) + ", \"halo_hy\": " +
         std::to_string(p->use_halo ? p->halo_hy : 0) + ", ";
    r += "\"chosen\": \"coupling64=" + std::string(p->use_halo ? kn[p->halo64] : kn[0]) +
         ",coupling32=" + std::string(p->use_halo ? kn[p->halo32] : kn[0]) +
         ",block_inverse32=" + (!p->use_tc ? std::string("simt")
                                : p->tc_groups == kTcChannelMajor ? std::string("tcc")
                                : std::string(p->tc_groups == 2 ? "tc2_N" : "tc_N") + std::to_string(p->tc_n)) +
         "\", \"arnoldi_stream\": \"" + (p->mixed && p->dcgs && p->bulk_arnoldi > 0 ? (p->bulk_arnoldi > 1 ? "bulk" : "bulk_reduce") : "registers") +
         "\"}";
    p->tune_report = r;
    return p->tune_report.c_str();
}

msc_status msc_debug_apply_block_inverse_f32(msc_plan *p, const float *x, float *y, void *stream)
{
    if (!p || !x || !y) return fail(MSC_ERR_ARG, "null argument");
    if (!p->mixed) return fail(MSC_ERR_ARG, "plan is not a mixed-precision plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    launch_block_inverse_t<float>(p, nullptr, reinterpret_cast<const float2 *>(x),
                                  reinterpret_cast<float2 *>(y), 0, s);
    MSC_CUDA(cudaGetLastError());
    if (p->use_tc) {
        int tc_err = 0;
        MSC_CUDA(cudaMemcpyAsync(&tc_err, p->tc_error.p, sizeof(int), cudaMemcpyDeviceToHost, s));
        MSC_CUDA(cudaStreamSynchronize(s));
        if (tc_err) return fail(MSC_ERR_CUDA, "tensor-core block inverse timed out on an mbarrier wait");
    }
    return MSC_OK;
}

int msc_plan_uses_tensor_cores(const msc_plan *p) { return (p && p->use_tc) ? p->tc_n : 0; }

msc_status msc_debug_symmetric_eigh(int32_t n, const double *a, double *w, double *v)
{
    if (!a || !w || !v) return fail(MSC_ERR_ARG, "null argument");
    if (n < 2 || n > msc::kMaxNz) return fail(MSC_ERR_DIMS, "n must be in 2..1024");
    for (size_t i = 0; i < (size_t)n * n; ++i)
        if (!std::isfinite(a[i])) return fail(MSC_ERR_NONFINITE, "non-finite matrix entry");
    return device_symmetric_eigh(n, a, w, v);
}

// ---------------------------------------------------------------------------
// Adjoint solves and the potential gradient (no counterpart in the reference;
// the operator they transpose is the one of multiscat_gmres.f90:452-687).
// ---------------------------------------------------------------------------
msc_status msc_plan_set_initial_guess(msc_plan *p, const double *psi0, int32_t on_device, void *stream)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    if (!psi0) {
        p->has_x0 = false;
        return MSC_OK;
    }
    const size_t vs = (size_t)p->R * p->n;
    if (!p->X0.p) MSC_CUDA(p->X0.alloc(vs));
    cudaStream_t us = reinterpret_cast<cudaStream_t>(stream);
    MSC_CUDA(cudaMemcpyAsync(p->X0.p, psi0, vs * sizeof(double2),
                             on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, us));
    if (!on_device) MSC_CUDA(cudaStreamSynchronize(us));
    p->has_x0 = true;
    return MSC_OK;
}

msc_status msc_plan_set_adjoint(msc_plan *p, int32_t adjoint)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    const bool want = adjoint != 0;
    if (want == p->adjoint) return MSC_OK;
    // nothing of this plan may be in flight while its operator data changes
    MSC_CUDA(cudaDeviceSynchronize());
    const std::vector<double2> &vt = want ? p->Vt_adj_host : p->Vt_host;
    std::vector<double2> rc = p->row_c_h;
    if (want)
        for (double2 &c : rc) c = msc::cconj(c);
    if (p->K > 0) MSC_CUDA(refill(p->Vt, vt));
    MSC_CUDA(refill(p->row_c, rc));
    msc::k_row_cfac<<<std::min((p->R + 255) / 256, 4096), 256>>>(p->R, p->row_c.p, p->row_fn.p,
                                                                 p->row_cf.p);
    MSC_CUDA(cudaGetLastError());
    MSC_CUDA(cudaDeviceSynchronize());    // the factors are in place before the next solve
    p->adjoint = want;
    if (p->sep_ok) {
        msc_status sst = upload_separable(p);
        if (sst != MSC_OK) return sst;
    }
    if (p->mixed) {
        if (p->K > 0) {
            std::vector<float2> vt32(vt.size());
            for (size_t i = 0; i < vt.size(); ++i) vt32[i] = make_float2((float)vt[i].x, (float)vt[i].y);
            MSC_CUDA(refill(p->Vt32, vt32));
        }
        std::vector<float2> c32(rc.size());
        for (size_t i = 0; i < rc.size(); ++i) c32[i] = make_float2((float)rc[i].x, (float)rc[i].y);
        MSC_CUDA(refill(p->row_c32, c32));
    }
    p->adjoint = want;
    return MSC_OK;
}

int msc_plan_is_adjoint(const msc_plan *p) { return (p && p->adjoint) ? 1 : 0; }

msc_status msc_plan_set_boundary_rhs(msc_plan *p, const double *rhs, int32_t on_device, void *stream)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t us = reinterpret_cast<cudaStream_t>(stream);
    const size_t bytes = (size_t)p->R * sizeof(double2);
    if (!rhs)
        MSC_CUDA(cudaMemcpyAsync(p->row_rhs.p, p->rhs_default_h.data(), bytes, cudaMemcpyHostToDevice, us));
    else
        MSC_CUDA(cudaMemcpyAsync(p->row_rhs.p, rhs, bytes,
                                 on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, us));
    msc::k_system_norms<<<p->B, 256, 0, us>>>(p->sys_row0.p, p->row_rhs.p, p->bnorm.p);
    MSC_CUDA(cudaGetLastError());
    if (!on_device || !rhs) MSC_CUDA(cudaStreamSynchronize(us));
    return MSC_OK;
}

msc_status msc_plan_set_adjoint_rhs(msc_plan *p, const double *psi, const double *dl_dintensity,
                                    const double *dl_damplitude, void *stream)
{
    if (!p) return fail(MSC_ERR_ARG, "null plan");
    if (dl_dintensity && !psi) return fail(MSC_ERR_ARG, "dl_dintensity needs psi");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    cudaStream_t us = reinterpret_cast<cudaStream_t>(stream);
    msc::k_adjoint_rhs<<<(p->R + 255) / 256, 256, 0, us>>>(
        p->R, p->n, p->row_sys.p, p->sys_spec_row.p, p->sys_aspec.p, p->row_b.p,
        reinterpret_cast<const double2 *>(psi), dl_dintensity,
        reinterpret_cast<const double2 *>(dl_damplitude), p->row_rhs.p);
    MSC_CUDA(cudaGetLastError());
    msc::k_system_norms<<<p->B, 256, 0, us>>>(p->sys_row0.p, p->row_rhs.p, p->bnorm.p);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_potential_gradient(msc_plan *p, const double *psi, const double *lambda,
                                  int32_t half_x, int32_t half_y, double *grad, void *stream)
{
    if (!p || !psi || !lambda || !grad) return fail(MSC_ERR_ARG, "null argument");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    const int nkx = p->nkx, nky = p->nky, n = p->n, ntor = nkx * nky;
    int wx = nkx, hx = 0, wy = nky, hy = 0;
    if (half_x >= 0 && 2 * half_x + 1 < nkx) {
        wx = 2 * half_x + 1;
        hx = half_x;
    }
    if (half_y >= 0 && 2 * half_y + 1 < nky) {
        wy = 2 * half_y + 1;
        hy = half_y;
    }
    cudaStream_t us = reinterpret_cast<cudaStream_t>(stream);
    MSC_CUDA(cudaMemsetAsync(grad, 0, (size_t)ntor * n * sizeof(double2), us));
    const int per_block = 8 * msc::kGradPerWarp;
    dim3 grid((wx * wy + per_block - 1) / per_block, (n + 31) / 32);
    msc::k_potential_gradient<<<grid, 256, 0, us>>>(
        nkx, nky, n, p->B, p->sys_row0.p, p->row_pos.p, p->pos_map.p, wx, wy, hx, hy,
        reinterpret_cast<const double2 *>(psi), reinterpret_cast<const double2 *>(lambda),
        reinterpret_cast<double2 *>(grad));
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

msc_status msc_intensities(msc_plan *p, int32_t s, const double *psi, double *intensities, void *stream)
{
    if (!p || !psi || !intensities) return fail(MSC_ERR_ARG, "null argument");
    msc_status st = finalize(p);
    if (st != MSC_OK) return st;
    if (s < 0 || s >= p->B) return fail(MSC_ERR_ARG, "system index out of range");
    cudaStream_t cs = reinterpret_cast<cudaStream_t>(stream);
    const int r0 = p->sys_row0_h[s], C = p->sys[s].C;
    msc::k_intensities<<<(C + 255) / 256, 256, 0, cs>>>(
        C, r0, p->n, p->row_sys.p + r0, p->sys_spec_row.p, p->sys_aspec.p, p->row_b.p + r0,
        reinterpret_cast<const double2 *>(psi), intensities);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}

int msc_run_multiscat(int gmres_preconditioner_flag, int convergence_significant_figures, int nkx,
                      int nky, int nz, const double *potential_values,
                      const double *perpendicular_kinetic_difference, const double *wave_a,
                      const double *wave_b, const double *wave_c,
                      const double *parallel_kinetic_energy, double *scattered_state_out,
                      int *iterations_out)
{
    (void)gmres_preconditioner_flag;
    if (nkx <= 0 || nky <= 0 || nz <= 0) return MSC_ERR_DIMS;
    if (!potential_values || !perpendicular_kinetic_difference || !wave_b || !wave_c ||
        !parallel_kinetic_energy || !scattered_state_out)
        return MSC_ERR_ARG;
    msc_plan_desc d{};
    d.n_z = nz;
    d.nkx = nkx;
    d.nky = nky;
    d.n_systems = 1;
    d.restart = 30;
    d.max_iterations = 2000;
    d.rtol = 5e-4 * std::pow(10.0, -(double)convergence_significant_figures);
    d.precision = MSC_PRECISION_FP64;
    msc_plan *p = nullptr;
    msc_status st = msc_plan_create(&p, &d);
    if (st != MSC_OK) return st;
    const int C = nkx * nky;
    std::vector<int32_t> ix(C), iy(C);
    for (int i = 0; i < nkx; ++i)
        for (int j = 0; j < nky; ++j) {
            ix[i * nky + j] = i;
            iy[i * nky + j] = j;
        }
    st = msc_plan_set_potential(p, potential_values, parallel_kinetic_energy);
    if (st == MSC_OK)
        st = msc_plan_set_system(p, 0, C, ix.data(), iy.data(), perpendicular_kinetic_difference,
                                 wave_b, wave_c, 0, wave_a);
    double *psi_dev = nullptr;
    msc_result res{};
    if (st == MSC_OK) {
        if (cudaMalloc(&psi_dev, (size_t)C * nz * sizeof(double2)) != cudaSuccess) st = MSC_ERR_CUDA;
    }
    if (st == MSC_OK) st = msc_solve(p, psi_dev, nullptr, &res, nullptr);
    if (st == MSC_OK || st == MSC_ERR_NOT_CONVERGED) {
        if (cudaMemcpy(scattered_state_out, psi_dev, (size_t)C * nz * sizeof(double2),
                       cudaMemcpyDeviceToHost) != cudaSuccess)
            st = MSC_ERR_CUDA;
    }
    if (iterations_out) *iterations_out = res.iterations;
    if (psi_dev) cudaFree(psi_dev);
    msc_plan_destroy(p);
    return st;
}

}  // extern "C"

// ===========================================================================
// Allocation-free operator apply.
//
// Some callers cannot call cudaMalloc at all: code that runs inside another
// framework's memory pool or under a strict device-memory budget, plug-ins
// that must not grow the process's allocations, and callers that work only
// on buffers handed to them.  msc_apply_operator_noalloc gives them y = A x
// for one full-grid system using only the buffers they pass plus a fixed
// scratch area that is part of this library's image: a file-scope
// __device__ array of kNoAllocScratchBytes (32 MiB) that every GPU which
// loads the library holds until the process exits.  The scratch keeps the
// tap table, neighbour table, row tiles and the D x intermediate of the
// last call; each call rewrites every byte it reads, so nothing has to start
// at zero.  All calls share the one array: calls that overlap on the GPU
// (different streams, or threads using the same device) race on it.
// ===========================================================================
namespace {

constexpr size_t kNoAllocScratchBytes = 32u << 20;
constexpr int kNoAllocMaxDevices = 64;

__device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

std::mutex g_noalloc_mutex;
void *g_noalloc_base[kNoAllocMaxDevices] = {};

// Nonzero coupling taps of V (storage offsets != (0, 0)) in (dx, dy)
// row-major order, Re V_00 into v00, the tap count into *count.  One block;
// order-preserving compaction so the tap order equals the plan builder's.
__global__ void __launch_bounds__(1024)
k_noalloc_scan_taps(int nkx, int nky, int n, const double2 *__restrict__ V, int *count,
                    int2 *__restrict__ taps, double *__restrict__ v00)
{
    __shared__ int warp_off[32];
    __shared__ int base;
    for (int z = threadIdx.x; z < n; z += blockDim.x) v00[z] = V[z].x;
    if (threadIdx.x == 0) {
        base = 0;
        count[1] = 0;   // non-finite flag, raised by k_noalloc_check_finite
    }
    __syncthreads();
    const int total = nkx * nky;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nwarps = blockDim.x >> 5;
    for (int c0 = 0; c0 < total; c0 += blockDim.x) {
        const int c = c0 + threadIdx.x;
        int flag = 0;
        if (c > 0 && c < total) {
            const double2 *v = V + (size_t)c * n;
            for (int z = 0; z < n && !flag; ++z) flag = (v[z].x != 0.0 || v[z].y != 0.0);
        }
        const unsigned m = __ballot_sync(0xffffffffu, flag);
        const int in_warp = __popc(m & ((1u << lane) - 1u));
        if (lane == 0) warp_off[warp] = __popc(m);
        __syncthreads();
        if (warp == 0) {
            const int own = (lane < nwarps) ? warp_off[lane] : 0;
            int inc = own;
            for (int o = 1; o < 32; o <<= 1) {
                const int up = __shfl_up_sync(0xffffffffu, inc, o);
                if (lane >= o) inc += up;
            }
            if (lane < nwarps) warp_off[lane] = inc - own;
        }
        __syncthreads();
        const int pos = base + warp_off[warp] + in_warp;
        if (flag) taps[pos] = make_int2(c / nky, c % nky);
        __syncthreads();
        if (threadIdx.x == blockDim.x - 1) base = pos + flag;
        __syncthreads();
    }
    if (threadIdx.x == 0) *count = base;
}

// Tap values, neighbour table and row tiles for one full-grid system.
__global__ void k_noalloc_tables(int nkx, int nky, int n, int K, const double2 *__restrict__ V,
                                 const int2 *__restrict__ taps, double2 *__restrict__ Vt,
                                 int *__restrict__ nbr, int *__restrict__ tile_row0,
                                 int *__restrict__ tile_nrow, int *__restrict__ tile_sys, int ntiles)
{
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    const int C = nkx * nky;
    for (size_t i = tid; i < (size_t)K * n; i += stride) {
        const int t = (int)(i / n), z = (int)(i - (size_t)t * n);
        Vt[i] = V[((size_t)taps[t].x * nky + taps[t].y) * n + z];
    }
    for (size_t i = tid; i < (size_t)C * K; i += stride) {
        const int r = (int)(i / K), t = (int)(i - (size_t)r * K);
        const int ix = r / nky, iy = r - ix * nky;
        const int sx = ((ix - taps[t].x) % nkx + nkx) % nkx;
        const int sy = ((iy - taps[t].y) % nky + nky) % nky;
        nbr[i] = sx * nky + sy;
    }
    for (size_t i = tid; i < (size_t)ntiles; i += stride) {
        tile_row0[i] = (int)i * msc::kTileRows;
        tile_nrow[i] = min(msc::kTileRows, C - (int)i * msc::kTileRows);
        tile_sys[i] = 0;
    }
}

// Raise *flag if any input of the operator is NaN or infinite (the plan
// builder rejects such inputs with MSC_ERR_NONFINITE; so does this path).
__global__ void k_noalloc_check_finite(int C, int n, const double2 *__restrict__ V,
                                       const double *__restrict__ T, const double *__restrict__ pkd,
                                       const double2 *__restrict__ wc, int *flag)
{
    const size_t tid = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    const size_t stride = (size_t)gridDim.x * blockDim.x;
    bool bad = false;
    for (size_t i = tid; i < (size_t)C * n; i += stride) bad |= !isfinite(V[i].x) || !isfinite(V[i].y);
    for (size_t i = tid; i < (size_t)n * n; i += stride) bad |= !isfinite(T[i]);
    for (size_t i = tid; i < (size_t)C; i += stride)
        bad |= !isfinite(pkd[i]) || !isfinite(wc[i].x) || !isfinite(wc[i].y);
    if (__any_sync(0xffffffffu, bad) && (threadIdx.x & 31) == 0) atomicOr(flag, 1);
}

size_t round256(size_t b) { return (b + 255) & ~(size_t)255; }

// Device address of the scratch array on the current device (set-up on the
// first call per device: symbol lookup and kernel shared-memory limits).
msc_status noalloc_scratch(unsigned char **out)
{
    int dev = -1;
    MSC_CUDA(cudaGetDevice(&dev));
    if (dev < 0 || dev >= kNoAllocMaxDevices) return fail(MSC_ERR_ARG, "device index out of range");
    std::lock_guard<std::mutex> lock(g_noalloc_mutex);
    if (!g_noalloc_base[dev]) {
        void *ptr = nullptr;
        cudaError_t e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
        if (e != cudaSuccess || ptr == nullptr)
            return fail(MSC_ERR_CUDA, std::string("cudaGetSymbolAddress(scratch): ") + cudaGetErrorString(e));
        msc_status st = set_kernel_attributes(0, 0);
        if (st != MSC_OK) return st;
        g_noalloc_base[dev] = ptr;
    }
    *out = static_cast<unsigned char *>(g_noalloc_base[dev]);
    return MSC_OK;
}

}  // namespace

extern "C" msc_status msc_apply_operator_noalloc(int32_t nkx, int32_t nky, int32_t n_z,
                                                 const double *potential_values,
                                                 const double *kinetic, const double *pkd,
                                                 const double *wave_c, const double *x, double *y,
                                                 void *stream)
{
    if (!potential_values || !kinetic || !pkd || !wave_c || !x || !y)
        return fail(MSC_ERR_ARG, "null argument");
    if (nkx <= 0 || nky <= 0 || n_z < 2 || n_z > msc::kMaxNz)
        return fail(MSC_ERR_DIMS, "bad dimensions");
    // channel count in 64 bits before any other arithmetic uses it
    if ((int64_t)nkx * nky - 1 > msc::kMaxTaps) return fail(MSC_ERR_DIMS, "more than 2049 channels");
    const int C = nkx * nky;
    const int n = n_z;
    const int kmax = std::max(C - 1, 1);
    const int ntiles = (C + msc::kTileRows - 1) / msc::kTileRows;
    // scratch layout (256-byte aligned pieces)
    size_t off = 0;
    const size_t o_count = off;  off += round256(2 * sizeof(int));   // tap count, non-finite flag
    const size_t o_taps = off;   off += round256(sizeof(int2) * (size_t)kmax);
    const size_t o_v00 = off;    off += round256(sizeof(double) * (size_t)n);
    const size_t o_vt = off;     off += round256(sizeof(double2) * (size_t)kmax * n);
    const size_t o_nbr = off;    off += round256(sizeof(int) * (size_t)C * kmax);
    const size_t o_t0 = off;     off += round256(sizeof(int) * (size_t)ntiles);
    const size_t o_tn = off;     off += round256(sizeof(int) * (size_t)ntiles);
    const size_t o_ts = off;     off += round256(sizeof(int) * (size_t)ntiles);
    const size_t o_tmp = off;    off += round256(sizeof(double2) * (size_t)C * n);
    if (off > kNoAllocScratchBytes)
        return fail(MSC_ERR_DIMS, "problem needs " + std::to_string(off) +
                                      " bytes of scratch; the allocation-free entry point has " +
                                      std::to_string(kNoAllocScratchBytes));
    unsigned char *base = nullptr;
    msc_status st = noalloc_scratch(&base);
    if (st != MSC_OK) return st;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int *count = reinterpret_cast<int *>(base + o_count);
    int2 *taps = reinterpret_cast<int2 *>(base + o_taps);
    double *v00 = reinterpret_cast<double *>(base + o_v00);
    double2 *Vt = reinterpret_cast<double2 *>(base + o_vt);
    int *nbr = reinterpret_cast<int *>(base + o_nbr);
    int *t0 = reinterpret_cast<int *>(base + o_t0);
    int *tn = reinterpret_cast<int *>(base + o_tn);
    int *ts = reinterpret_cast<int *>(base + o_ts);
    double2 *tmp = reinterpret_cast<double2 *>(base + o_tmp);
    const double2 *V = reinterpret_cast<const double2 *>(potential_values);

    k_noalloc_scan_taps<<<1, 1024, 0, s>>>(nkx, nky, n, V, count, taps, v00);
    MSC_CUDA(cudaGetLastError());
    k_noalloc_check_finite<<<128, 256, 0, s>>>(C, n, V, kinetic, pkd,
                                               reinterpret_cast<const double2 *>(wave_c), count + 1);
    MSC_CUDA(cudaGetLastError());
    int kf[2] = {0, 0};
    MSC_CUDA(cudaMemcpyAsync(kf, count, 2 * sizeof(int), cudaMemcpyDeviceToHost, s));
    MSC_CUDA(cudaStreamSynchronize(s));
    const int K = kf[0];
    if (kf[1]) return fail(MSC_ERR_NONFINITE, "non-finite potential, kinetic or channel data");
    if (K < 0 || K > kmax) return fail(MSC_ERR_CUDA, "tap scan returned an invalid count");
    k_noalloc_tables<<<256, 256, 0, s>>>(nkx, nky, n, K, V, taps, Vt, nbr, t0, tn, ts, ntiles);
    MSC_CUDA(cudaGetLastError());
    const msc::Tiles tiles{t0, tn, ts, ntiles};
    msc::k_residual_diag<<<ntiles, 256, smem_residual(n), s>>>(
        tiles, nullptr, n, kinetic, v00, pkd, reinterpret_cast<const double2 *>(wave_c), nullptr,
        reinterpret_cast<const double2 *>(x), tmp, 0);
    MSC_CUDA(cudaGetLastError());
    dim3 grid(ntiles, (n + 31) / 32);
    dim3 block(32, msc::kTileRows);
    msc::k_coupling<<<grid, block, smem_coupling(std::max(K, 1)), s>>>(
        tiles, nullptr, n, K, Vt, nbr, reinterpret_cast<const double2 *>(x), tmp, -1.0,
        reinterpret_cast<double2 *>(y));
    MSC_CUDA(cudaGetLastError());
    const size_t cnt = (size_t)C * n;
    msc::k_scale<<<(unsigned)std::min<size_t>((cnt + 255) / 256, 4096), 256, 0, s>>>(
        reinterpret_cast<double2 *>(y), cnt, -1.0);
    MSC_CUDA(cudaGetLastError());
    return MSC_OK;
}
