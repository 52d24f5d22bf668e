// mixed2d.cu -- iterative-refinement form of the 2D implicit timestep.
//
// tl2d_refine_solve_step solves one timestep's system A u = u0 (the operator
// of 2d/c_kernels/omp3/cg.c:9-85 with the reflective boundary) to a stated
// relative residual ||u0 - A u||_2 / ||u0||_2 <= rel_tol, with one algorithm
// (refine2d.cuh: CG on T-stored vectors and coefficients, arithmetic in T,
// FP64 dot products and scalars, FP64 solution with reliable FP64 residual
// replacement) in
// two storage precisions on identical inputs: T = float (48 B per cell per
// iteration) and T = double (96 B).
//
// Around the solve the timestep is the reference's: energy/density halos,
// cg_init, u0 = u (cg_driver.c:30-62), and energy = u / density afterwards
// (solver_methods.c finalise). Device-resident loop as in driver2d.cu: the
// last block of each reduction computes alpha, beta and the update/stop
// decisions; the FP64 fold and residual kernels are launched every trip and
// return at once unless an update was requested.
#include "host_maths.hpp"
#include "pcblock2d.cuh"
#include "refine2d.cuh"
#include "rftma2d.cuh"
#include "suite2d_impl.hpp"

#include <cmath>

using namespace tl2d;
using namespace tl2d::rf;

namespace {

constexpr int kBatch = 16;

template <typename T, bool FUSE_P>
__global__ void __launch_bounds__(BX, Pack<T>::MINB) k_rf_w(Lay L, const MxState* __restrict__ st,
                                                            const T* __restrict__ p_in, T* __restrict__ p_out,
                                                            const T* __restrict__ r, T* __restrict__ w,
                                                            const T* __restrict__ kx, const T* __restrict__ ky,
                                                            ReduceSlots rs, FinMxW fin)
{
    if (mx_idle(st)) return;
    const double bt = FUSE_P ? st->beta : 0.0;
    double acc[1] = {rf_w_tile<T, FUSE_P, false, typename RfMath<T>::M>(L, blockIdx.x, blockIdx.y, bt, p_in, p_out,
                                                                         r, w, kx, ky)};
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

template <typename T>
__global__ void __launch_bounds__(BX, Pack<T>::MINB) k_rf_ur(Lay L, const MxState* __restrict__ st, T* __restrict__ xs,
                                                             const T* __restrict__ p, T* __restrict__ r,
                                                             const T* __restrict__ w, ReduceSlots rs, FinMxUr fin)
{
    if (mx_idle(st)) return;
    double acc[1] = {rf_ur_tile<T, false, typename RfMath<T>::M>(L, blockIdx.x, blockIdx.y, st->alpha, xs, p, r, w)};
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// Inner step pp < ni - 1 of the PPCG preconditioner z = q(A) r (FOLD 1 for
// pp == 0: sd = r / theta, z = sd; else FOLD 2 with the coefficients of
// pp - 1).
template <typename T, int FOLD>
__global__ void __launch_bounds__(BX, Pack<T>::MINB - 2) k_rf_pc(Lay L, const MxState* __restrict__ st, double theta,
                                                               const double* __restrict__ alphas,
                                                               const double* __restrict__ betas, int pp,
                                                               const T* __restrict__ sd_in, T* __restrict__ sd_out,
                                                               const T* __restrict__ s_in, T* __restrict__ s_out,
                                                               T* __restrict__ z, const T* __restrict__ kx,
                                                               const T* __restrict__ ky)
{
    if (mx_idle(st)) return;
    const double fa = FOLD == 2 ? alphas[pp - 1] : 0.0, fb = FOLD == 2 ? betas[pp - 1] : 0.0;
    rf_pc_tile<T, FOLD, FOLD == 2>(L, blockIdx.x, blockIdx.y, theta, fa, fb, sd_in, sd_out, s_in, s_out, z, kx, ky);
}

// Last inner step (pp = ni - 1) of the preconditioner and r.z -> beta.
template <typename T, int FOLD>
__global__ void __launch_bounds__(BX, Pack<T>::MINB - 2) k_rf_pc_last(Lay L, const MxState* __restrict__ st,
                                                                  double theta, const double* __restrict__ alphas,
                                                                  const double* __restrict__ betas, int pp,
                                                                  const T* __restrict__ sd,
                                                                  const T* __restrict__ s_in, T* __restrict__ z,
                                                                  const T* __restrict__ r, ReduceSlots rs,
                                                                  FinPcgZ fin)
{
    if (mx_idle(st)) return;
    const double fa = FOLD == 2 ? alphas[pp - 1] : 0.0, fb = FOLD == 2 ? betas[pp - 1] : 0.0;
    double acc[1] = {rf_pc_last_tile<T, FOLD>(L, blockIdx.x, blockIdx.y, theta, fa, fb, sd, s_in, z, r)};
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// Resumes the iteration after the CG phase stopped for the switch (reason 2).
__global__ void k_rf_resume(MxState* st)
{
    if (threadIdx.x == 0 && st->reason == 2) {
        st->done = 0;
        st->reason = 0;
    }
}

template <typename T>
__global__ void __launch_bounds__(BX) k_rf_fold(Lay L, const MxState* __restrict__ st, int gx, int hd,
                                                double* __restrict__ u, T* __restrict__ xs)
{
    if (mx_no_update(st)) return;
    rf_fold_tile<T>(L, blockIdx.x, blockIdx.y, gx, hd, u, xs);
}

template <typename T>
__global__ void __launch_bounds__(BX) k_rf_resid(Lay L, const MxState* __restrict__ st, int gx, int hd,
                                                 const double* __restrict__ u, const double* __restrict__ u0,
                                                 const double* __restrict__ kx, const double* __restrict__ ky,
                                                 T* __restrict__ rT, ReduceSlots rs, FinMxRes fin)
{
    if (mx_no_update(st)) return;
    double acc[2] = {0.0, 0.0};
    rf_resid_tile<T>(L, blockIdx.x, blockIdx.y, gx, hd, u, u0, kx, ky, rT, acc);
    tl::grid_sum<2, BX>(acc, rs, block_id(), block_count(), fin);
}

// ------------------------------------------------------------ host side --

enum RfField { RF_KX = 0, RF_KY, RF_P0, RF_P1, RF_W, RF_R, RF_XS, RF_SD0, RF_SD1, RF_S0, RF_S1, RF_Z, RF_COUNT };

template <typename T>
struct RfBuffers {
    T* f[RF_COUNT];
    MxState* st;
    Lay L;
};

// The state word and `fields` T arrays in the suite's slab (grown on demand).
template <typename T>
RfBuffers<T> rf_buffers(TlSuite2D* s, int fields)
{
    constexpr int N = Pack<T>::N;
    RfBuffers<T> b{};
    const int nx = s->g.x - 2 * s->g.hd, ny = s->g.y - 2 * s->g.hd;
    // tile rows for whole waves of the TMA sweeps (the default path; the
    // per-thread-load sweeps keep the same tiles so both give the same sums)
    b.L = make_lay<T>(nx, ny, choose_rows(tl::ceil_div(nx, N), ny, s->sm_count, kRfTmaBlocks, 64));
    {
        const dim3 t = lay_tiles<T>(b.L);   // the reduction partials must fit
        if ((long)t.x * t.y * tl::kMaxSums > s->partial_capacity) b.L.rows = s->g.rows;
    }
    const size_t field = ((size_t)b.L.cells() * sizeof(T) + 255) & ~(size_t)255;
    const size_t need = 256 + field * fields;
    if (!s->mx_slab || s->mx_bytes < need) {
        if (s->mx_slab) cudaFree(s->mx_slab);
        s->mx_slab = nullptr;
        s->mx_bytes = 0;
        if (!TL_CUDA(cudaMalloc(&s->mx_slab, need))) return RfBuffers<T>{};
        s->mx_bytes = need;
    }
    char* base = (char*)s->mx_slab;
    static_assert(sizeof(MxState) <= 256, "the state word sits in the slab's first 256 bytes");
    b.st = (MxState*)base;
    for (int k = 0; k < fields; ++k) b.f[k] = (T*)(base + 256 + field * k);
    return b;
}

// Tensor map of a refinement array (T layout: xp x (ny + 2)): tile rows
// (RfRowsW<T>::W x kRfRows) or the 16-byte ring boxes.
template <typename T>
const CUtensorMap* rf_map(TlSuite2D* s, const Lay& L, const T* ptr, bool ring)
{
    const int kind = 16 + (sizeof(T) == 4 ? 0 : 8) + (ring ? 1 : 0);
    return tma_lookup(s, ptr, kind, [&](CUtensorMap* m) {
        return tl::tma_encode_3d(m, ptr, L.xp, L.ny + 2, 1, ring ? RfRowsW<T>::H : RfRowsW<T>::W, kRfRows, 1,
                                 (int)sizeof(T));
    });
}

// The refinement w sweep (k_rf_w semantics), by TMA where the maps encode.
// Internal linkage with the kernels, as the drop-in helpers.
template <typename T, bool FUSE_P>
void rf_w(TlSuite2D* s, const RfBuffers<T>& b, dim3 gl, const char* name, const T* p_in, T* p_out, const T* r,
          FinMxW fin)
{
    if (s->tma) {
        const CUtensorMap *mp = rf_map(s, b.L, p_in, false), *mph = rf_map(s, b.L, p_in, true);
        const CUtensorMap *mr = rf_map(s, b.L, r, false), *mrh = rf_map(s, b.L, r, true);
        const CUtensorMap *mkx = rf_map<T>(s, b.L, b.f[RF_KX], false), *mkxh = rf_map<T>(s, b.L, b.f[RF_KX], true);
        const CUtensorMap* mky = rf_map<T>(s, b.L, b.f[RF_KY], false);
        if (mp && mph && mr && mrh && mkx && mkxh && mky) {
            const RfWMaps m{*mp, *mr, *mkx, *mky, *mph, *mrh, *mkxh};
            constexpr size_t smem = rf_w_tma_bytes<T>();
            static unsigned attr_set = 0;
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k_rf_w_tma<T, FUSE_P>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
                attr_set |= 1u << (s->device & 31);
            }
            TL_LAUNCH(s, name, (k_rf_w_tma<T, FUSE_P><<<gl, BX, smem, s->stream>>>(
                                   b.L, b.st, m, p_out, b.f[RF_W], s->rs, fin, s->d_mirror + kTmaErrWord2)));
            return;
        }
    }
    TL_LAUNCH(s, name, (k_rf_w<T, FUSE_P><<<gl, BX, 0, s->stream>>>(b.L, b.st, p_in, p_out, r, b.f[RF_W],
                                                                     b.f[RF_KX], b.f[RF_KY], s->rs, fin)));
}

// The refinement u/r update (k_rf_ur semantics), by TMA where the maps encode.
template <typename T>
void rf_ur(TlSuite2D* s, const RfBuffers<T>& b, dim3 gl, const char* name, const T* p, T* r, FinMxUr fin)
{
    if (s->tma) {
        const CUtensorMap* mx = rf_map<T>(s, b.L, b.f[RF_XS], false);
        const CUtensorMap* mp = rf_map(s, b.L, p, false);
        const CUtensorMap* mr = rf_map<T>(s, b.L, r, false);
        const CUtensorMap* mw = rf_map<T>(s, b.L, b.f[RF_W], false);
        if (mx && mp && mr && mw) {
            const RfUMaps m{*mx, *mp, *mr, *mw};
            constexpr size_t smem = rf_u_tma_bytes<T>();
            static unsigned attr_set = 0;
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k_rf_ur_tma<T>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem));
                attr_set |= 1u << (s->device & 31);
            }
            TL_LAUNCH(s, name, (k_rf_ur_tma<T><<<gl, BX, smem, s->stream>>>(b.L, b.st, m, b.f[RF_XS], r, s->rs, fin,
                                                                           s->d_mirror + kTmaErrWord2)));
            return;
        }
    }
    TL_LAUNCH(s, name, (k_rf_ur<T><<<gl, BX, 0, s->stream>>>(b.L, b.st, b.f[RF_XS], p, r, b.f[RF_W], s->rs, fin)));
}

// Launches trips t = 0.. in batches of kBatch, looking at the mapped done word
// of the previous batch while the current one runs (as driver2d.cu).
template <typename F>
void batched(TlSuite2D* s, int max_trips, F&& launch_trip)
{
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int t = 0, batch = 0;
    bool pending_prev = false;
    while (t < max_trips && !tl::failed()) {
        const int end = std::min(max_trips, t + kBatch);
        for (; t < end; ++t) launch_trip(t);
        cudaEventRecord(ev[batch & 1], s->stream);
        if (pending_prev) {
            cudaEventSynchronize(ev[(batch + 1) & 1]);
            if (*(volatile int*)&s->h_mirror[0]) break;
        }
        pending_prev = true;
        ++batch;
    }
    cudaStreamSynchronize(s->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

template <typename T>
struct Names;
template <>
struct Names<float> {
    static constexpr const char* n[6] = {"k_rf_init<f32>", "k_rf_w<f32>", "k_rf_ur<f32>", "k_rf_fold<f32>",
                                         "k_rf_resid<f32>", "k_rf_pc<f32>"};
};
template <>
struct Names<double> {
    static constexpr const char* n[6] = {"k_rf_init<f64>", "k_rf_w<f64>", "k_rf_ur<f64>", "k_rf_fold<f64>",
                                         "k_rf_resid<f64>", "k_rf_pc<f64>"};
};

// CG in T storage with FP64 refinement; returns the trips run.
template <typename T>
int solve_refined(TlSuite2D* s, Chunk* chunk, int max_iters, double rel_tol, int* updates, double* rtrue,
                  double* bb)
{
    RfBuffers<T> b = rf_buffers<T>(s, RF_SD0);
    if (!b.st) return 0;
    const char* const* nm = Names<T>::n;
    const Lay L = b.L;
    const dim3 gl = lay_tiles<T>(L);
    s->h_mirror[0] = 0;
    // grid-stride init: as many blocks as the reduction partials hold (3 sums each)
    const int init_blocks = (int)std::max<long>(1, std::min<long>(s->sm_count * 4L, s->partial_capacity / 3));
    TL_LAUNCH(s, nm[0], (k_rf_init<T><<<init_blocks, 256, 0, s->stream>>>(
                            s->g.x, s->g.hd, L, chunk->r, chunk->u0, chunk->kx, chunk->ky, b.f[RF_KX], b.f[RF_KY], b.f[RF_R],
                            b.f[RF_P0], b.f[RF_P1], b.f[RF_W], b.f[RF_XS], s->rs,
                            FinMxInit{b.st, rel_tol * rel_tol, 0.0, max_iters, s->d_mirror})));
    T* pb[2] = {b.f[RF_P0], b.f[RF_P1]};
    int cur = 0;
    batched(s, max_iters, [&](int t) {
        if (t == 0) {
            rf_w<T, false>(s, b, gl, nm[1], pb[cur], pb[cur], b.f[RF_R], FinMxW{b.st});
        } else {
            rf_w<T, true>(s, b, gl, nm[1], pb[cur], pb[cur ^ 1], b.f[RF_R], FinMxW{b.st});
            cur ^= 1;
        }
        rf_ur<T>(s, b, gl, nm[2], pb[cur], b.f[RF_R], FinMxUr{b.st, s->d_mirror});
        TL_LAUNCH(s, nm[3], (k_rf_fold<T><<<gl, BX, 0, s->stream>>>(L, b.st, s->g.x, s->g.hd, chunk->u,
                                                                     b.f[RF_XS])));
        TL_LAUNCH(s, nm[4], (k_rf_resid<T><<<gl, BX, 0, s->stream>>>(L, b.st, s->g.x, s->g.hd, chunk->u,
                                                                      chunk->u0, chunk->kx, chunk->ky, b.f[RF_R],
                                                                      s->rs, FinMxRes{b.st, s->d_mirror})));
    });
    MxState st{};
    TL_CUDA(cudaMemcpy(&st, b.st, sizeof(MxState), cudaMemcpyDeviceToHost));
    *updates = st.updates;
    *rtrue = st.rtrue;
    *bb = st.bb;
    return st.trip;
}

// One launch of the blocked preconditioner (pcblock2d.cuh).
template <typename T, bool FIRST, bool LAST>
void pc_launch(TlSuite2D* s, dim3 grid, const PcArgs& a, const RfBuffers<T>& b, const T* sd_in, const T* s_in,
               T* sd_out, T* s_out, T* z, const T* r)
{
    static const char* const name = sizeof(T) == 4 ? "k_rf_pc_blocked<f32>" : "k_rf_pc_blocked<f64>";
    constexpr size_t smem = pc_smem<T>();
    TL_CUDA(cudaFuncSetAttribute(k_rf_pc_blocked<T, FIRST, LAST>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem));
    TL_LAUNCH(s, name, (k_rf_pc_blocked<T, FIRST, LAST><<<grid, kPcThreads, smem, s->stream>>>(
                           b.L, b.st, a, sd_in, s_in, sd_out, s_out, z, b.f[RF_KX], b.f[RF_KY], r, s->rs,
                           FinPcgZ{b.st})));
}

// PPCG in T storage with FP64 refinement. As 2d/drivers/ppcg_driver.c: CG
// trips recording the FP64 alphas and betas until the reference's switch test
// holds (more than presteps trips and error < 1, or with error_switch more
// than 20 trips and error < eps_lim), an FP64 residual replacement on the
// switch trip (the reference recomputes r = u0 - A u there too), the Lanczos
// eigenvalue bounds and Chebyshev coefficients of the inner steps on the host
// in FP64 (eigenvalue_driver.c, cheby_driver.c:163-183). The outer steps then
// use the inner Chebyshev recurrence (ppcg.c:9-61) as a polynomial
// preconditioner in standard PCG: z = q(A) r from ppcg_inner_steps steps on
// A z = r from z = 0, beta = r.z / r.z_old, p = z + beta p, w = A p, alpha =
// r.z / p.w, u += alpha p, r -= alpha w, with r.r driving the stop test and
// the residual replacements. (The reference applies the polynomial to u and r
// themselves and takes beta from r.r; that recurrence drifts from the true
// residual on ill-conditioned meshes and cannot be refined to a fixed
// residual.) Returns the trips run (CG + PPCG outer).
template <typename T>
int solve_refined_ppcg(TlSuite2D* s, Chunk* chunk, Settings* settings, double rel_tol, int* updates, double* rtrue,
                       double* bb, int* cg_trips)
{
    RfBuffers<T> b = rf_buffers<T>(s, RF_COUNT);
    if (!b.st) return 0;
    const char* const* nm = Names<T>::n;
    const Lay L = b.L;
    const dim3 gl = lay_tiles<T>(L);
    const int max_iters = settings->max_iters, ni = settings->ppcg_inner_steps;   // checked by the caller
    s->h_mirror[0] = 0;
    const size_t fb = (size_t)L.cells() * sizeof(T);
    for (int f : {RF_SD0, RF_SD1, RF_S0, RF_S1, RF_Z}) TL_CUDA(cudaMemsetAsync(b.f[f], 0, fb, s->stream));
    const int init_blocks = (int)std::max<long>(1, std::min<long>(s->sm_count * 4L, s->partial_capacity / 3));
    TL_LAUNCH(s, nm[0], (k_rf_init<T><<<init_blocks, 256, 0, s->stream>>>(
                            s->g.x, s->g.hd, L, chunk->r, chunk->u0, chunk->kx, chunk->ky, b.f[RF_KX], b.f[RF_KY],
                            b.f[RF_R], b.f[RF_P0], b.f[RF_P1], b.f[RF_W], b.f[RF_XS], s->rs,
                            FinMxInit{b.st, rel_tol * rel_tol, 0.0, max_iters, s->d_mirror})));
    T* pb[2] = {b.f[RF_P0], b.f[RF_P1]};
    T* sb[2] = {b.f[RF_SD0], b.f[RF_SD1]};
    T* qb[2] = {b.f[RF_S0], b.f[RF_S1]};
    T* const r = b.f[RF_R];
    T* const z = b.f[RF_Z];
    int cur = 0;
    auto fold_resid = [&](double* betas) {
        TL_LAUNCH(s, nm[3], (k_rf_fold<T><<<gl, BX, 0, s->stream>>>(L, b.st, s->g.x, s->g.hd, chunk->u,
                                                                     b.f[RF_XS])));
        TL_LAUNCH(s, nm[4], (k_rf_resid<T><<<gl, BX, 0, s->stream>>>(L, b.st, s->g.x, s->g.hd, chunk->u,
                                                                      chunk->u0, chunk->kx, chunk->ky, r, s->rs,
                                                                      FinMxRes{b.st, s->d_mirror, betas})));
    };
    auto w_sweep = [&](int t, double* alphas) {
        if (t == 0) {
            rf_w<T, false>(s, b, gl, nm[1], pb[cur], pb[cur], r, FinMxW{b.st, alphas});
        } else {
            rf_w<T, true>(s, b, gl, nm[1], pb[cur], pb[cur ^ 1], r, FinMxW{b.st, alphas});
            cur ^= 1;
        }
    };
    // CG trips up to the switch (2d/shared.h:41-42 for the constants)
    const FinMxUr cg_fin = settings->error_switch
                               ? FinMxUr{b.st, s->d_mirror, s->d_cg_betas, 20, settings->eps_lim}
                               : FinMxUr{b.st, s->d_mirror, s->d_cg_betas, settings->presteps, 1.0};
    batched(s, max_iters, [&](int t) {
        w_sweep(t, s->d_cg_alphas);
        rf_ur<T>(s, b, gl, nm[2], pb[cur], r, cg_fin);
        fold_resid(s->d_cg_betas);
    });
    MxState st{};
    TL_CUDA(cudaMemcpy(&st, b.st, sizeof(MxState), cudaMemcpyDeviceToHost));
    *cg_trips = st.trip;
    if (st.done && st.reason == 2) {
        // the inner steps' polynomial from the presteps' FP64 Lanczos matrix
        const int ncg = st.trip;
        TL_CUDA(cudaMemcpy(chunk->cg_alphas, s->d_cg_alphas, sizeof(double) * ncg, cudaMemcpyDeviceToHost));
        TL_CUDA(cudaMemcpy(chunk->cg_betas, s->d_cg_betas, sizeof(double) * ncg, cudaMemcpyDeviceToHost));
        if (!tl::eigen_bounds(chunk, ncg)) return st.trip;
        tl::cheby_coefs(chunk, ni);
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, chunk->cheby_alphas, sizeof(double) * ni, cudaMemcpyHostToDevice,
                                s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, chunk->cheby_betas, sizeof(double) * ni, cudaMemcpyHostToDevice,
                                s->stream));
        const double theta = chunk->theta;
        TL_LAUNCH(s, "k_rf_resume", (k_rf_resume<<<1, 32, 0, s->stream>>>(b.st)));
        TL_CUDA(cudaStreamSynchronize(s->stream));
        s->h_mirror[0] = 0;
        const double* ca = s->d_cheby_alphas;
        const double* cb = s->d_cheby_betas;
        // the blocked preconditioner reduces r.z with one partial per tile
        const dim3 pg = pc_grid(L);
        const bool blocked = s->temporal_blocking && (long)pg.x * pg.y <= s->partial_capacity;
        batched(s, max_iters - ncg, [&](int) {
            // z = q(A) r and beta
            if (ni == 1) {
                TL_LAUNCH(s, nm[5], (k_rf_pc_last<T, 1><<<gl, BX, 0, s->stream>>>(
                                        L, b.st, theta, ca, cb, 0, sb[0], r, z, r, s->rs, FinPcgZ{b.st})));
            } else if (blocked) {
                // ni - 1 stencil steps in launches of up to kPcMax, the last one with the final fold and r.z
                int c = 0;
                for (int pp = 0; pp < ni - 1;) {
                    const int h = std::min(kPcMax, ni - 1 - pp);
                    const PcArgs pa{h, pp, theta, ca, cb};
                    const bool first = pp == 0, last = pp + h == ni - 1;
                    const T* s_in = first ? r : qb[c];
                    if (first && last)
                        pc_launch<T, true, true>(s, pg, pa, b, sb[c], s_in, sb[c ^ 1], qb[c ^ 1], z, r);
                    else if (first)
                        pc_launch<T, true, false>(s, pg, pa, b, sb[c], s_in, sb[c ^ 1], qb[c ^ 1], z, r);
                    else if (last)
                        pc_launch<T, false, true>(s, pg, pa, b, sb[c], s_in, sb[c ^ 1], qb[c ^ 1], z, r);
                    else
                        pc_launch<T, false, false>(s, pg, pa, b, sb[c], s_in, sb[c ^ 1], qb[c ^ 1], z, r);
                    c ^= 1;
                    pp += h;
                }
            } else {
                TL_LAUNCH(s, nm[5], (k_rf_pc<T, 1><<<gl, BX, 0, s->stream>>>(L, b.st, theta, ca, cb, 0, sb[1], sb[0],
                                                                             r, qb[0], z, b.f[RF_KX], b.f[RF_KY])));
                int c = 0;
                for (int pp = 1; pp < ni - 1; ++pp, c ^= 1)
                    TL_LAUNCH(s, nm[5], (k_rf_pc<T, 2><<<gl, BX, 0, s->stream>>>(
                                            L, b.st, theta, ca, cb, pp, sb[c], sb[c ^ 1], qb[c], qb[c ^ 1], z,
                                            b.f[RF_KX], b.f[RF_KY])));
                TL_LAUNCH(s, nm[5], (k_rf_pc_last<T, 2><<<gl, BX, 0, s->stream>>>(
                                        L, b.st, theta, ca, cb, ni - 1, sb[c], qb[c], z, r, s->rs, FinPcgZ{b.st})));
            }
            // p = z + beta p, w = A p, alpha = r.z / p.w
            rf_w<T, true>(s, b, gl, nm[1], pb[cur], pb[cur ^ 1], z, FinMxW{b.st, nullptr, true});
            cur ^= 1;
            rf_ur<T>(s, b, gl, nm[2], pb[cur], r, FinMxUr{b.st, s->d_mirror});
            fold_resid(nullptr);
        });
        TL_CUDA(cudaMemcpy(&st, b.st, sizeof(MxState), cudaMemcpyDeviceToHost));
    }
    *updates = st.updates;
    *rtrue = st.rtrue;
    *bb = st.bb;
    return st.trip;
}

}  // namespace

extern "C" int tl2d_refine_solve_step(Chunk* chunk, Settings* settings, int tt, double rel_tol, int precision,
                                      TlRefineStats* stats)
{
    (void)tt;
    if (tl::failed()) return tl::error_state().code;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return tl::error_state().code;
    if (precision != 32 && precision != 64) {
        tl::fail(40, "tl2d_refine_solve_step: precision must be 32 or 64 (got %d)", precision);
        return 40;
    }
    if (!(rel_tol > 0.0)) {
        tl::fail(41, "tl2d_refine_solve_step: rel_tol must be positive (got %g)", rel_tol);
        return 41;
    }
    const Faces fc = faces_of(chunk);
    if (settings->num_chunks_per_rank != 1 || !(fc.l && fc.r && fc.b && fc.t)) {
        tl::fail(42, "tl2d_refine_solve_step: one chunk with four external faces is required");
        return 42;
    }
    if (settings->coefficient != TL_CONDUCTIVITY && settings->coefficient != TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return 7;
    }
    if (settings->solver == TL_PPCG_SOLVER) {
        if (settings->max_iters > s->table_len) {
            tl::fail(32, "max_iters %d exceeds the %d the chunk was initialised with", settings->max_iters,
                     s->table_len);
            return 32;
        }
        if (settings->ppcg_inner_steps < 1 || settings->ppcg_inner_steps > s->table_len) {
            tl::fail(43, "tl2d_refine_solve_step: ppcg_inner_steps %d outside 1..%d", settings->ppcg_inner_steps,
                     s->table_len);
            return 43;
        }
    }
    TlRefineStats local{};
    TlRefineStats* out = stats ? stats : &local;
    *out = TlRefineStats{};
    flush(s, chunk);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);

    // solve(): dt, rx, ry; energy/density halos; cg_init; halos of u, p; u0 = u
    const double dt = chunk->dt_init < settings->dt_init ? chunk->dt_init : settings->dt_init;
    const double rx = dt / (settings->dx * settings->dx);
    const double ry = dt / (settings->dy * settings->dy);
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
    s->pend.halo[TL_FIELD_ENERGY1] = s->pend.halo[TL_FIELD_DENSITY] = 2;
    flush(s, chunk);
    TL_LAUNCH(s, "k_cg_init", k_cg_init<<<full_grid(s->g), FB, 0, s->stream>>>(
                                  s->g, settings->coefficient, rx, ry, chunk->density, chunk->energy, chunk->u,
                                  chunk->p, s->alt[ALT_P], chunk->r, chunk->w, chunk->kx, chunk->ky, s->rs,
                                  FinCgInit{s->d_state, s->d_mirror}));
    s->pend.halo[TL_FIELD_U] = s->pend.halo[TL_FIELD_P] = 1;
    flush(s, chunk);
    TL_LAUNCH(s, "k_copy_u", k_copy_u<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u0, chunk->u));

    double rtrue = 0.0, bb = 0.0;
    const int max_iters = settings->max_iters;
    if (settings->solver == TL_PPCG_SOLVER)
        out->iterations =
            precision == 32
                ? solve_refined_ppcg<float>(s, chunk, settings, rel_tol, &out->residual_updates, &rtrue, &bb,
                                            &out->cg_trips)
                : solve_refined_ppcg<double>(s, chunk, settings, rel_tol, &out->residual_updates, &rtrue, &bb,
                                             &out->cg_trips);
    else
        out->iterations = precision == 32
                              ? solve_refined<float>(s, chunk, max_iters, rel_tol, &out->residual_updates, &rtrue, &bb)
                              : solve_refined<double>(s, chunk, max_iters, rel_tol, &out->residual_updates, &rtrue, &bb);
    if (settings->solver != TL_PPCG_SOLVER) out->cg_trips = out->iterations;
    // finalise (solver_methods.c), energy halo as solve_finished_driver
    TL_LAUNCH(s, "k_finalise", k_finalise<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->energy,
                                                                                     chunk->density, chunk->u));
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
    s->pend.halo[TL_FIELD_ENERGY1] = 1;
    flush(s, chunk);
    cudaEventRecord(e1, s->stream);
    TL_CUDA(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    out->device_ms = ms;
    out->rel_residual = bb > 0.0 ? std::sqrt(rtrue / bb) : 0.0;
    out->converged = out->rel_residual <= rel_tol ? 1 : 0;
    if (tma_failed(s)) tl::fail(35, "a TMA row load of the refinement sweeps did not complete (bounded barrier wait gave up)");
    return tl::failed() ? tl::error_state().code : 0;
}
