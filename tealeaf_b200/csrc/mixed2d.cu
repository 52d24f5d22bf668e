// mixed2d.cu -- iterative-refinement form of the 2D implicit timestep.
//
// tl2d_refine_solve_step solves one timestep's system A u = u0 (the operator
// of 2d/c_kernels/omp3/cg.c:9-85 with the reflective boundary) to a stated
// relative residual ||u0 - A u||_2 / ||u0||_2 <= rel_tol, with one algorithm
// in two storage precisions on identical inputs:
//
//  * CG whose vectors (p, r, w, the solution correction xs) and operator
//    coefficients (kx, ky) are stored in T (float or double). Every kernel
//    computes in FP64 registers and every dot product (p.w, r.r) is
//    accumulated in FP64, so w is the FP64 image of the stored p and only the
//    stores round.
//  * The solution is accumulated in FP64 (the chunk's u): when r.r of the
//    stored residual has dropped by kUpdateDelta^2 since the last replacement
//    (or looks converged), xs is folded into u, the residual u0 - A u is
//    recomputed in FP64 with the FP64 coefficients and replaces the stored
//    one, and the search direction is kept (reliable updates / residual
//    replacement: Sleijpen & van der Vorst 1996; van der Vorst & Ye 2000).
//    Convergence is only ever declared on that FP64 residual.
//
// With T = float one iteration moves 48 B per cell instead of 96.
//
// Layout of the T arrays: interior cells only, row pitch xp (>= nx + 2 cells
// per thread, a multiple of 64), one zero row above and below, so element
// (k, j) of the interior is at (j + 1) * xp + k. The face coefficient
// arrays hold kx of the face left of cell k and ky of the face below cell j,
// with the boundary faces set to zero: with the depth-1 reflective halo the
// boundary terms of the 5-point operator cancel (neighbour = centre), so the
// operator is the same in exact arithmetic and the sweeps need no boundary
// branches. Each thread owns 8 bytes of a row (2 floats or 1 double).
//
// Around the solve the timestep is the reference's: energy/density halos,
// cg_init, u0 = u (cg_driver.c:30-62), and energy = u / density afterwards
// (solver_methods.c finalise). Device-resident loop as in driver2d.cu: the
// last block of each reduction computes alpha, beta and the update/stop
// decisions; the FP64 fold and residual kernels are launched every trip and
// return at once unless an update was requested.
#include "suite2d_impl.hpp"

#include <cmath>

using namespace tl2d;

namespace {

constexpr int kBatch = 16;
constexpr double kUpdateDelta = 0.1;   // replace the residual when ||r|| fell by this factor

struct MxState {
    double rr;       // r.r of the stored residual (FP64 sum)
    double pw, alpha, beta;
    double bb;       // u0.u0
    double tol2bb;   // rel_tol^2 * bb
    double rref;     // r.r right after the last replacement
    double rtrue;    // FP64 r.r of the last FP64 residual
    double rsloppy;  // r.r of the stored residual when the last update was requested
    int trip, done, upd, updates, reason, max_iters;
};

__device__ __forceinline__ int vol_read(const int* p) { return *(volatile const int*)p; }
__device__ __forceinline__ bool mx_idle(const MxState* st) { return vol_read(&st->done) != 0; }
__device__ __forceinline__ bool mx_no_update(const MxState* st)
{
    return vol_read(&st->done) != 0 || vol_read(&st->upd) == 0;
}
__device__ __forceinline__ void mirror(const MxState* st, int* hm)
{
    if (hm) {
        hm[0] = st->done;
        hm[1] = st->trip;
        hm[2] = st->reason;
    }
}

struct FinMxInit {   // t: rT.rT, u0.u0, r.r (FP64 residual of cg_init)
    MxState* st;
    double tol2;
    int max_iters;
    int* hm;
    __device__ void operator()(const double* t) const
    {
        st->rr = t[0];
        st->rref = t[0];
        st->bb = t[1];
        st->tol2bb = tol2 * t[1];
        st->rtrue = t[2];
        st->rsloppy = t[0];
        st->pw = st->alpha = st->beta = 0.0;
        st->trip = 0;
        st->upd = 0;
        st->updates = 0;
        st->max_iters = max_iters;
        st->done = 0;
        st->reason = 0;
        if (t[2] <= st->tol2bb) {
            st->done = 1;
            st->reason = 1;
        } else if (max_iters <= 0) {
            st->done = 1;
            st->reason = 3;
        }
        mirror(st, hm);
    }
};

struct FinMxW {   // alpha = rr / pw
    MxState* st;
    __device__ void operator()(const double* t) const
    {
        st->pw = t[0];
        st->alpha = st->rr / t[0];
    }
};

struct FinMxUr {   // beta = rrn / rr, or request an FP64 residual replacement
    MxState* st;
    int* hm;
    __device__ void operator()(const double* t) const
    {
        const double rrn = t[0];
        st->trip += 1;
        const bool upd = rrn < kUpdateDelta * kUpdateDelta * st->rref || rrn <= st->tol2bb ||
                         st->trip >= st->max_iters || !(rrn == rrn);
        if (upd) {
            st->upd = 1;
            st->rsloppy = rrn;
        } else {
            st->beta = rrn / st->rr;
            st->rr = rrn;
        }
        mirror(st, hm);
    }
};

struct FinMxRes {   // t: r.r (FP64 residual), rT.rT
    MxState* st;
    int* hm;
    __device__ void operator()(const double* t) const
    {
        st->rtrue = t[0];
        st->updates += 1;
        st->upd = 0;
        if (t[0] <= st->tol2bb) {
            st->done = 1;
            st->reason = 1;
        } else if (st->trip >= st->max_iters || !(t[0] == t[0])) {
            st->done = 1;
            st->reason = 3;
        } else {
            st->beta = t[1] / st->rr;
            st->rr = t[1];
            st->rref = t[1];
        }
        mirror(st, hm);
    }
};

// ----------------------------------------------------------- T layout ----

// Cells per thread (8 bytes of a row) and resident blocks per SM of the
// sweeps (FP64 arithmetic on N cells needs 48 / 40 registers a thread).
template <typename T> struct Pack;
template <> struct Pack<float> {
    static constexpr int N = 2;
    static constexpr int MINB = 10;
    using V = float2;
};
template <> struct Pack<double> {
    static constexpr int N = 1;
    static constexpr int MINB = 12;
    using V = double;
};

template <typename T>
union Cells {
    typename Pack<T>::V v;
    T e[Pack<T>::N];
};

template <typename T>
__device__ __forceinline__ Cells<T> ld(const T* p)
{
    Cells<T> c;
    c.v = *reinterpret_cast<const typename Pack<T>::V*>(p);
    return c;
}
template <typename T>
__device__ __forceinline__ void st8(T* p, const Cells<T>& c)
{
    *reinterpret_cast<typename Pack<T>::V*>(p) = c.v;
}

struct Lay {
    int nx, ny, xp, rows;
    __host__ __device__ long cells() const { return (long)(ny + 2) * xp; }
};

// Interior column range and rows of this thread.
template <int N>
struct Span {
    int c0, cc, j0, j1, lane;
    bool any;   // at least one of the N cells is interior
    __device__ Span(const Lay& L)
    {
        c0 = (blockIdx.x * BX + threadIdx.x) * N;
        cc = min(c0, L.xp - N);   // clamped: lanes past the row load valid padding cells
        j0 = blockIdx.y * L.rows;
        j1 = min(j0 + L.rows, L.ny);
        lane = threadIdx.x & 31;
        any = c0 < L.nx;
    }
};

template <typename T>
dim3 lay_grid(const Lay& L)
{
    constexpr int N = Pack<T>::N;
    return dim3(tl::ceil_div(tl::ceil_div(L.nx, N), BX), tl::ceil_div(L.ny, L.rows));
}

// Fills the T arrays from the FP64 state after cg_init, padding included:
// kxT/kyT (interior faces; boundary faces and padding 0), rT = p0 = r,
// p1 = w = xs = 0. Sums rT.rT, u0.u0 and r.r over the interior.
template <typename T, typename Finish>
__global__ void __launch_bounds__(256) k_rf_init(Geo g, Lay L, const double* __restrict__ r,
                                                 const double* __restrict__ u0, const double* __restrict__ kx,
                                                 const double* __restrict__ ky, T* __restrict__ kxT,
                                                 T* __restrict__ kyT, T* __restrict__ rT, T* __restrict__ p0,
                                                 T* __restrict__ p1, T* __restrict__ w, T* __restrict__ xs,
                                                 ReduceSlots rs, Finish fin)
{
    double acc[3] = {0.0, 0.0, 0.0};
    const long n = L.cells();
    for (long e = blockIdx.x * (long)blockDim.x + threadIdx.x; e < n; e += (long)gridDim.x * blockDim.x) {
        const int k = (int)(e % L.xp);
        const int j = (int)(e / L.xp) - 1;
        const bool in = k < L.nx && j >= 0 && j < L.ny;
        const long i = in ? (long)(g.hd + k) + (long)(g.hd + j) * g.x : 0;
        T kxv = 0, kyv = 0, rv = 0;
        if (in) {
            if (k >= 1) kxv = (T)kx[i];
            if (j >= 1) kyv = (T)ky[i];
            const double r64 = r[i];
            rv = (T)r64;
            acc[0] += (double)rv * (double)rv;
            acc[1] += u0[i] * u0[i];
            acc[2] += r64 * r64;
        }
        kxT[e] = kxv;
        kyT[e] = kyv;
        rT[e] = rv;
        p0[e] = rv;
        p1[e] = 0;
        w[e] = 0;
        xs[e] = 0;
    }
    tl::grid_sum<3, 256>(acc, rs, blockIdx.x, gridDim.x, fin);
}

// CG sweep 1 on the T layout, FP64 arithmetic: [p = beta p + r] (rounded to
// T as stored), w = A p, sum(w p) over the stored values.
template <typename T, bool FUSE_P>
__global__ void __launch_bounds__(BX, Pack<T>::MINB) k_rf_w(Lay L, const MxState* __restrict__ st,
                                                        const T* __restrict__ p_in, T* __restrict__ p_out,
                                                        const T* __restrict__ r, T* __restrict__ w,
                                                        const T* __restrict__ kx, const T* __restrict__ ky,
                                                        ReduceSlots rs, FinMxW fin)
{
    constexpr int N = Pack<T>::N;
    if (mx_idle(st)) return;
    double acc[1] = {0.0};
    const Span<N> s(L);
    const double bt = FUSE_P ? st->beta : 0.0;
    auto cur = [&](long idx) -> Cells<T> {
        Cells<T> c = ld(p_in + idx);
        if (FUSE_P) {
            const Cells<T> q = ld(r + idx);
#pragma unroll
            for (int m = 0; m < N; ++m) c.e[m] = (T)(bt * (double)c.e[m] + (double)q.e[m]);
        }
        return c;
    };
    auto cur1 = [&](long idx) -> T {
        return FUSE_P ? (T)(bt * (double)p_in[idx] + (double)r[idx]) : p_in[idx];
    };
    const long xp = L.xp;
    long i = (long)(s.j0 + 1) * xp + s.cc;
    Cells<T> pc = cur(i), pd = cur(i - xp), kyc = ld(ky + i);
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
    for (int j = s.j0; j < s.j1; ++j, i += xp) {
        const Cells<T> pu = cur(i + xp), kyu = ld(ky + i + xp), kxc = ld(kx + i);
        T pl = __shfl_up_sync(kFull, pc.e[N - 1], 1);
        T pr = __shfl_down_sync(kFull, pc.e[0], 1);
        T kxr = __shfl_down_sync(kFull, kxc.e[0], 1);
        if (s.lane == 0) pl = cur1(i - 1);
        if (s.lane == 31) {
            pr = cur1(i + N);
            kxr = kx[i + N];
        }
        Cells<T> wv;
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const double c = (double)pc.e[m];
            const double l = m == 0 ? (double)pl : (double)pc.e[m - 1];
            const double rr = m == N - 1 ? (double)pr : (double)pc.e[m + 1];
            const double kr = m == N - 1 ? (double)kxr : (double)kxc.e[m + 1];
            wv.e[m] = (T)smvp((double)kxc.e[m], kr, (double)kyc.e[m], (double)kyu.e[m], c, l, rr, (double)pd.e[m],
                              (double)pu.e[m]);
        }
        if (s.any) {
            st8(w + i, wv);
            if (FUSE_P) st8(p_out + i, pc);
#pragma unroll
            for (int m = 0; m < N; ++m)
                if (s.c0 + m < L.nx) acc[0] += (double)wv.e[m] * (double)pc.e[m];
        }
        pd = pc;
        pc = pu;
        kyc = kyu;
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// CG sweep 2 on the T layout: xs += alpha p ; r -= alpha w ; sum(r r).
template <typename T>
__global__ void __launch_bounds__(BX, Pack<T>::MINB) k_rf_ur(Lay L, const MxState* __restrict__ st, T* __restrict__ xs,
                                                         const T* __restrict__ p, T* __restrict__ r,
                                                         const T* __restrict__ w, ReduceSlots rs, FinMxUr fin)
{
    constexpr int N = Pack<T>::N;
    if (mx_idle(st)) return;
    const Span<N> s(L);
    double acc[1] = {0.0};
    if (s.any) {
        const double a = st->alpha;
        long i = (long)(s.j0 + 1) * L.xp + s.c0;
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += L.xp) {
            Cells<T> xv = ld(xs + i), rv = ld(r + i);
            const Cells<T> pv = ld(p + i), wv = ld(w + i);
#pragma unroll
            for (int m = 0; m < N; ++m) {
                xv.e[m] = (T)((double)xv.e[m] + a * (double)pv.e[m]);
                rv.e[m] = (T)((double)rv.e[m] - a * (double)wv.e[m]);
                if (s.c0 + m < L.nx) acc[0] += (double)rv.e[m] * (double)rv.e[m];
            }
            st8(xs + i, xv);
            st8(r + i, rv);
        }
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// Reliable update, part 1 (only when requested): u += xs (FP64), xs = 0.
template <typename T>
__global__ void __launch_bounds__(BX) k_rf_fold(Geo g, Lay L, const MxState* __restrict__ st, double* __restrict__ u,
                                                T* __restrict__ xs)
{
    if (mx_no_update(st)) return;
    Strip s(g);
    if (!s.active) return;
    const int k = s.k - g.hd;
    long i = s.k + (long)s.j0 * g.x;
    for (int j = s.j0; j < s.j1; ++j, i += g.x) {
        const long e = (long)(j - g.hd + 1) * L.xp + k;
        u[i] += (double)xs[e];
        xs[e] = 0;
    }
}

// Reliable update, part 2: r = u0 - A u in FP64 with the FP64 coefficients
// and the reflective boundary; rT = r; sums r.r and rT.rT.
template <typename T>
__global__ void __launch_bounds__(BX) k_rf_resid(Geo g, Lay L, const MxState* __restrict__ st,
                                                 const double* __restrict__ u, const double* __restrict__ u0,
                                                 const double* __restrict__ kx, const double* __restrict__ ky,
                                                 T* __restrict__ rT, ReduceSlots rs, FinMxRes fin)
{
    if (mx_no_update(st)) return;
    double acc[2] = {0.0, 0.0};
    const StripC s(g);
    const int x = g.x;
    const int jt = g.y - g.hd - 1;
    long i = s.kk + (long)s.j0 * x;
    double uc = u[i];
    double ud = (s.j0 == g.hd) ? uc : u[i - x];
    double kyc = ky[i];
    for (int j = s.j0; j < s.j1; ++j, i += x) {
        const double uu = (j == jt) ? uc : u[i + x];
        const double kyu = ky[i + x];
        const double kxc = kx[i];
        double ul = __shfl_up_sync(kFull, uc, 1);
        double ur = __shfl_down_sync(kFull, uc, 1);
        double kxr = __shfl_down_sync(kFull, kxc, 1);
        if (s.at_l) ul = uc;
        else if (s.lane == 0) ul = u[i - 1];
        if (s.at_r) ur = uc;
        else if (s.lane == 31) ur = u[i + 1];
        if (s.at_r || s.lane == 31) kxr = kx[i + 1];
        const double rv = u0[i] - smvp(kxc, kxr, kyc, kyu, uc, ul, ur, ud, uu);
        const T rt = (T)rv;
        if (s.active) {
            rT[(long)(j - g.hd + 1) * L.xp + (s.k - g.hd)] = rt;
            acc[0] += rv * rv;
            acc[1] += (double)rt * (double)rt;
        }
        ud = uc;
        uc = uu;
        kyc = kyu;
    }
    tl::grid_sum<2, BX>(acc, rs, block_id(), block_count(), fin);
}

// ------------------------------------------------------------ host side --

enum RfField { RF_KX = 0, RF_KY, RF_P0, RF_P1, RF_W, RF_R, RF_XS, RF_COUNT };

template <typename T>
struct RfBuffers {
    T* f[RF_COUNT];
    MxState* st;
    Lay L;
};

template <typename T>
RfBuffers<T> rf_buffers(TlSuite2D* s)
{
    constexpr int N = Pack<T>::N;
    RfBuffers<T> b{};
    const int nx = s->g.x - 2 * s->g.hd, ny = s->g.y - 2 * s->g.hd;
    b.L.nx = nx;
    b.L.ny = ny;
    b.L.xp = ((nx + 2 * N + 63) / 64) * 64;
    b.L.rows = choose_rows(tl::ceil_div(nx, N), ny, s->sm_count, Pack<T>::MINB);
    {
        const dim3 t = lay_grid<T>(b.L);   // the reduction partials must fit
        if ((long)t.x * t.y * tl::kMaxSums > s->partial_capacity) b.L.rows = s->g.rows;
    }
    const size_t field = ((size_t)b.L.cells() * sizeof(T) + 255) & ~(size_t)255;
    const size_t need = field * RF_COUNT + 256;
    if (!s->mx_slab || s->mx_bytes < need) {
        if (s->mx_slab) cudaFree(s->mx_slab);
        s->mx_slab = nullptr;
        s->mx_bytes = 0;
        if (!TL_CUDA(cudaMalloc(&s->mx_slab, need))) return RfBuffers<T>{};
        s->mx_bytes = need;
    }
    char* base = (char*)s->mx_slab;
    for (int k = 0; k < RF_COUNT; ++k) b.f[k] = (T*)(base + field * k);
    b.st = (MxState*)(base + field * RF_COUNT);
    return b;
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
    static constexpr const char* n[5] = {"k_rf_init<f32>", "k_rf_w<f32>", "k_rf_ur<f32>", "k_rf_fold<f32>",
                                         "k_rf_resid<f32>"};
};
template <>
struct Names<double> {
    static constexpr const char* n[5] = {"k_rf_init<f64>", "k_rf_w<f64>", "k_rf_ur<f64>", "k_rf_fold<f64>",
                                         "k_rf_resid<f64>"};
};

// CG in T storage with FP64 refinement; returns the trips run.
template <typename T>
int solve_refined(TlSuite2D* s, Chunk* chunk, int max_iters, double rel_tol, int* updates, double* rtrue,
                  double* bb)
{
    RfBuffers<T> b = rf_buffers<T>(s);
    if (!b.st) return 0;
    const char* const* nm = Names<T>::n;
    const Lay L = b.L;
    const dim3 gl = lay_grid<T>(L), gi = interior_grid(s->g);
    s->h_mirror[0] = 0;
    TL_LAUNCH(s, nm[0], (k_rf_init<T><<<s->sm_count * 4, 256, 0, s->stream>>>(
                            s->g, L, chunk->r, chunk->u0, chunk->kx, chunk->ky, b.f[RF_KX], b.f[RF_KY], b.f[RF_R],
                            b.f[RF_P0], b.f[RF_P1], b.f[RF_W], b.f[RF_XS], s->rs,
                            FinMxInit{b.st, rel_tol * rel_tol, max_iters, s->d_mirror})));
    T* pb[2] = {b.f[RF_P0], b.f[RF_P1]};
    int cur = 0;
    batched(s, max_iters, [&](int t) {
        if (t == 0) {
            TL_LAUNCH(s, nm[1], (k_rf_w<T, false><<<gl, BX, 0, s->stream>>>(
                                    L, b.st, pb[cur], pb[cur], b.f[RF_R], b.f[RF_W], b.f[RF_KX], b.f[RF_KY], s->rs,
                                    FinMxW{b.st})));
        } else {
            TL_LAUNCH(s, nm[1], (k_rf_w<T, true><<<gl, BX, 0, s->stream>>>(
                                    L, b.st, pb[cur], pb[cur ^ 1], b.f[RF_R], b.f[RF_W], b.f[RF_KX], b.f[RF_KY],
                                    s->rs, FinMxW{b.st})));
            cur ^= 1;
        }
        TL_LAUNCH(s, nm[2], (k_rf_ur<T><<<gl, BX, 0, s->stream>>>(L, b.st, b.f[RF_XS], pb[cur], b.f[RF_R],
                                                                   b.f[RF_W], s->rs, FinMxUr{b.st, s->d_mirror})));
        TL_LAUNCH(s, nm[3], (k_rf_fold<T><<<gi, BX, 0, s->stream>>>(s->g, L, b.st, chunk->u, b.f[RF_XS])));
        TL_LAUNCH(s, nm[4], (k_rf_resid<T><<<gi, BX, 0, s->stream>>>(s->g, L, b.st, chunk->u, chunk->u0, chunk->kx,
                                                                      chunk->ky, b.f[RF_R], s->rs,
                                                                      FinMxRes{b.st, s->d_mirror})));
    });
    MxState st{};
    TL_CUDA(cudaMemcpy(&st, b.st, sizeof(MxState), cudaMemcpyDeviceToHost));
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
    out->iterations = precision == 32
                          ? solve_refined<float>(s, chunk, max_iters, rel_tol, &out->residual_updates, &rtrue, &bb)
                          : solve_refined<double>(s, chunk, max_iters, rel_tol, &out->residual_updates, &rtrue, &bb);
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
    return tl::failed() ? tl::error_state().code : 0;
}
