// refine2d.cuh -- CG with FP64 refinement on the padded "T layout" (2D):
// the solver state, the finishers and the tile sweeps shared by the
// iterative-refinement timestep (mixed2d.cu) and the batched solver
// (batch2d.cu).
//
// CG whose vectors (p, r, w, the solution correction xs) and operator
// coefficients (kx, ky) are stored in T (float or double). The refinement
// timestep's and the batched solver's sweeps compute in T (the stencil and
// vector updates in FP32 for FP32 storage; RfMath, BatchM); every dot
// product (p.w, r.r) is accumulated in FP64.
// The solution is accumulated in FP64 (the chunk's u): when r.r of the stored
// residual has dropped by kUpdateDelta^2 since the last replacement (or looks
// converged), xs is folded into u, the residual u0 - A u is recomputed in
// FP64 with the FP64 coefficients and replaces the stored one, and the search
// direction is kept (reliable updates / residual replacement: Sleijpen & van
// der Vorst 1996; van der Vorst & Ye 2000). Convergence is only ever declared
// on that FP64 residual. With T = float one iteration moves 48 B per cell.
//
// T layout: interior cells only, row pitch xp (>= nx + 2 cells per thread, a
// multiple of 64), one zero row above and below, so element (k, j) of the
// interior is at (j + 1) * xp + k. The face coefficient arrays hold kx of the
// face left of cell k and ky of the face below cell j, with the boundary faces
// set to zero: with the depth-1 reflective halo the boundary terms of the
// 5-point operator cancel (neighbour = centre), so the operator is the same
// in exact arithmetic and the sweeps need no boundary branches. The padding
// stays zero through the iteration (zero coefficients, zero start). A tile is
// BX threads x N cells (8 bytes of a row per thread) x L.rows rows.
#pragma once

#include <type_traits>

#include "kernels2d.cuh"

namespace tl2d {
namespace rf {

constexpr double kUpdateDelta = 0.1;   // replace the residual when ||r|| fell by this factor

struct MxState {
    double rr;       // r.r of the stored residual (FP64 sum)
    double pw, alpha, beta;
    double bb;       // u0.u0
    double tol2bb;   // stop when the FP64 r.r <= tol2bb
    double rref;     // r.r right after the last replacement
    double rtrue;    // FP64 r.r of the last FP64 residual
    double rsloppy;  // r.r of the stored residual when the last update was requested
    double rz;       // PPCG: r.z of the last preconditioned residual (0 before the first)
    int trip, done, upd, updates, reason, max_iters;
    int sw;          // the switch to PPCG is due after the pending replacement
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

// t: rT.rT, u0.u0, r.r (FP64 residual of cg_init). Stop test: FP64 r.r <=
// tol2 * u0.u0 (relative), or <= abs_eps when abs_eps > 0 (the reference's
// r.r < eps of 2d/diffuse.c, on the FP64 residual).
struct FinMxInit {
    MxState* st;
    double tol2;
    double abs_eps;
    int max_iters;
    int* hm;
    __device__ void operator()(const double* t) const
    {
        st->rr = t[0];
        st->rref = t[0];
        st->bb = t[1];
        st->tol2bb = abs_eps > 0.0 ? abs_eps : tol2 * t[1];
        st->rtrue = t[2];
        st->rsloppy = t[0];
        st->pw = st->alpha = st->beta = st->rz = 0.0;
        st->trip = 0;
        st->upd = 0;
        st->sw = 0;
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

struct FinMxW {   // alpha = rr / pw (PCG: rz / pw) [recorded in alphas[trip]]
    MxState* st;
    double* alphas = nullptr;
    bool pcg = false;
    __device__ void operator()(const double* t) const
    {
        st->pw = t[0];
        st->alpha = (pcg ? st->rz : st->rr) / t[0];
        if (alphas) alphas[st->trip] = st->alpha;
    }
};

// With sw_after >= 0 the CG-to-PPCG switch test of 2d/drivers/ppcg_driver.c:
// 27-29 runs on the trips completed and error = rrn (switch once more than
// sw_after trips ran and rrn < sw_below); a due switch requests a residual
// replacement, after which FinMxRes stops the CG phase with reason 2.
struct FinMxUr {   // beta = rrn / rr [recorded in betas[trip]], or request an FP64 residual replacement
    MxState* st;
    int* hm;
    double* betas = nullptr;
    int sw_after = -1;
    double sw_below = 0.0;
    __device__ void operator()(const double* t) const
    {
        const double rrn = t[0];
        const int tt = st->trip;
        st->trip = tt + 1;
        const bool sw = sw_after >= 0 && st->trip > sw_after && rrn < sw_below;
        if (sw) st->sw = 1;
        const bool upd = sw || rrn < kUpdateDelta * kUpdateDelta * st->rref || rrn <= st->tol2bb ||
                         st->trip >= st->max_iters || !(rrn == rrn);
        if (upd) {
            st->upd = 1;
            st->rsloppy = rrn;
            if (betas) betas[tt] = rrn / st->rr;   // the recurrence's beta for the Lanczos matrix
        } else {
            st->beta = rrn / st->rr;
            st->rr = rrn;
            if (betas) betas[tt] = st->beta;
        }
        mirror(st, hm);
    }
};

// PCG: t = r.z of the new preconditioned residual; beta = rz / rz_old (0 on
// the first step after the switch, which restarts the directions at p = z).
struct FinPcgZ {
    MxState* st;
    __device__ void operator()(const double* t) const
    {
        st->beta = st->rz > 0.0 ? t[0] / st->rz : 0.0;
        st->rz = t[0];
    }
};

struct FinMxRes {   // t: r.r (FP64 residual), rT.rT [beta recorded in betas[trip - 1]]
    MxState* st;
    int* hm;
    double* betas = nullptr;
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
            if (betas && st->trip > 0) betas[st->trip - 1] = st->beta;
            if (st->sw) {
                st->sw = 0;
                st->done = 1;
                st->reason = 2;
            }
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

// Arithmetic type of the refinement timestep's CG sweeps for storage type T:
// the storage precision itself (TL2D_RF_MATH_T 1: FP32 arithmetic for FP32
// storage, measured 9.81 against 10.61 s for the 8192^2 CG timestep to
// 1e-10 with FP64 arithmetic, same iterations) or FP64 (0). Dot products, the
// scalars and the FP64 residual stay FP64 either way. The tile functions'
// M defaults to double; the batched solver picks its own (BatchM).
#ifndef TL2D_RF_MATH_T
#define TL2D_RF_MATH_T 1
#endif
template <typename T>
struct RfMath {
    using M = double;
};
template <>
struct RfMath<float> {
    using M = std::conditional_t<TL2D_RF_MATH_T != 0, float, double>;
};
// The 5-point operator in type M, in the operand order of smvp.
template <typename M>
__device__ __forceinline__ M smvp_m(M kxc, M kxr, M kyc, M kyu, M c, M l, M r, M d, M u)
{
    return (M(1) + (kxr + kxc) + (kyu + kyc)) * c - (kxr * r + kxc * l) - (kyu * u + kyc * d);
}

template <typename T>
__device__ __forceinline__ Cells<T> ld(const T* p)
{
    Cells<T> c;
    c.v = *reinterpret_cast<const typename Pack<T>::V*>(p);
    return c;
}
// Loads for arrays that other blocks of the same (persistent) launch write
// between phases: CG = true reads through L2 (ld.global.cg), never from a
// stale L1 line or the read-only path; false is a plain load.
template <bool CG, typename T>
__device__ __forceinline__ Cells<T> ldc(const T* p)
{
    if (!CG) return ld(p);
    Cells<T> c;
    c.v = __ldcg(reinterpret_cast<const typename Pack<T>::V*>(p));
    return c;
}
template <bool CG, typename T>
__device__ __forceinline__ T ldc1(const T* p)
{
    return CG ? __ldcg(p) : *p;
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

template <typename T>
inline Lay make_lay(int nx, int ny, int rows)
{
    constexpr int N = Pack<T>::N;
    Lay L;
    L.nx = nx;
    L.ny = ny;
    L.xp = ((nx + 2 * N + 63) / 64) * 64;
    L.rows = rows;
    return L;
}

template <typename T>
inline dim3 lay_tiles(const Lay& L)
{
    constexpr int N = Pack<T>::N;
    return dim3(tl::ceil_div(tl::ceil_div(L.nx, N), BX), tl::ceil_div(L.ny, L.rows));
}

// Columns and rows of this thread in tile (tx, ty).
template <int N>
struct Span {
    int c0, cc, j0, j1, lane;
    bool any;   // at least one of the N cells is interior
    __device__ Span(const Lay& L, int tx, int ty)
    {
        c0 = (tx * BX + threadIdx.x) * N;
        cc = min(c0, L.xp - N);   // clamped: lanes past the row load valid padding cells
        j0 = ty * L.rows;
        j1 = min(j0 + L.rows, L.ny);
        lane = threadIdx.x & 31;
        any = c0 < L.nx;
    }
};

// Fills the T arrays from the FP64 state after cg_init, padding included:
// kxT/kyT (interior faces; boundary faces and padding 0), rT = p0 = r,
// p1 = w = xs = 0. Sums rT.rT, u0.u0 and r.r over the interior. gx: row
// length of the FP64 chunk arrays, hd: their halo depth.
template <typename T, typename Finish>
__global__ void __launch_bounds__(256) k_rf_init(int gx, int hd, Lay L, const double* __restrict__ r,
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
        const long i = in ? (long)(hd + k) + (long)(hd + j) * gx : 0;
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

// CG sweep 1 over tile (tx, ty), arithmetic in M: [p = beta p + r] (rounded
// to T as stored), w = A p; returns this thread's share of sum(w p) over the
// stored values. All threads of the block take part (warp shuffles).
template <typename T, bool FUSE_P, bool CG = false, typename M = double>
__device__ __forceinline__ double rf_w_tile(const Lay& L, int tx, int ty, double bt_, const T* __restrict__ p_in,
                                            T* __restrict__ p_out, const T* __restrict__ r, T* __restrict__ w,
                                            const T* __restrict__ kx, const T* __restrict__ ky)
{
    constexpr int N = Pack<T>::N;
    double acc = 0.0;
    const Span<N> s(L, tx, ty);
    const M bt = (M)bt_;
    auto cur = [&](long idx) -> Cells<T> {
        Cells<T> c = ldc<CG>(p_in + idx);
        if (FUSE_P) {
            const Cells<T> q = ldc<CG>(r + idx);
#pragma unroll
            for (int m = 0; m < N; ++m) c.e[m] = (T)(bt * (M)c.e[m] + (M)q.e[m]);
        }
        return c;
    };
    auto cur1 = [&](long idx) -> T {
        return FUSE_P ? (T)(bt * (M)ldc1<CG>(p_in + idx) + (M)ldc1<CG>(r + idx)) : ldc1<CG>(p_in + idx);
    };
    const long xp = L.xp;
    long i = (long)(s.j0 + 1) * xp + s.cc;
    Cells<T> pc = cur(i), pd = cur(i - xp), kyc = ldc<CG>(ky + i);
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
    for (int j = s.j0; j < s.j1; ++j, i += xp) {
        const Cells<T> pu = cur(i + xp), kyu = ldc<CG>(ky + i + xp), kxc = ldc<CG>(kx + i);
        T pl = __shfl_up_sync(kFull, pc.e[N - 1], 1);
        T pr = __shfl_down_sync(kFull, pc.e[0], 1);
        T kxr = __shfl_down_sync(kFull, kxc.e[0], 1);
        if (s.lane == 0) pl = cur1(i - 1);
        if (s.lane == 31) {
            pr = cur1(i + N);
            kxr = ldc1<CG>(kx + i + N);
        }
        Cells<T> wv;
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const M c = (M)pc.e[m];
            const M l = m == 0 ? (M)pl : (M)pc.e[m - 1];
            const M rr = m == N - 1 ? (M)pr : (M)pc.e[m + 1];
            const M kr = m == N - 1 ? (M)kxr : (M)kxc.e[m + 1];
            wv.e[m] = (T)smvp_m<M>((M)kxc.e[m], kr, (M)kyc.e[m], (M)kyu.e[m], c, l, rr, (M)pd.e[m], (M)pu.e[m]);
        }
        if (s.any) {
            st8(w + i, wv);
            if (FUSE_P) st8(p_out + i, pc);
#pragma unroll
            for (int m = 0; m < N; ++m)
                if (s.c0 + m < L.nx) acc += (double)wv.e[m] * (double)pc.e[m];
        }
        pd = pc;
        pc = pu;
        kyc = kyu;
    }
    return acc;
}

// CG sweep 2 over tile (tx, ty): xs += alpha p ; r -= alpha w ; returns this
// thread's share of sum(r r).
template <typename T, bool CG = false, typename M = double>
__device__ __forceinline__ double rf_ur_tile(const Lay& L, int tx, int ty, double a_, T* __restrict__ xs,
                                             const T* __restrict__ p, T* __restrict__ r, const T* __restrict__ w)
{
    const M a = (M)a_;
    constexpr int N = Pack<T>::N;
    const Span<N> s(L, tx, ty);
    double acc = 0.0;
    if (s.any) {
        long i = (long)(s.j0 + 1) * L.xp + s.c0;
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += L.xp) {
            Cells<T> xv = ldc<CG>(xs + i), rv = ldc<CG>(r + i);
            const Cells<T> pv = ldc<CG>(p + i), wv = ldc<CG>(w + i);
#pragma unroll
            for (int m = 0; m < N; ++m) {
                xv.e[m] = (T)((M)xv.e[m] + a * (M)pv.e[m]);
                rv.e[m] = (T)((M)rv.e[m] - a * (M)wv.e[m]);
                if (s.c0 + m < L.nx) acc += (double)rv.e[m] * (double)rv.e[m];
            }
            st8(xs + i, xv);
            st8(r + i, rv);
        }
    }
    return acc;
}

// Preconditioner arithmetic in T with explicit fused multiply-adds (the
// file is compiled without contraction; the one-step and the blocked kernels
// share these, so their results are bit-identical).
__device__ __forceinline__ float fma_t(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_t(double a, double b, double c) { return __fma_rn(a, b, c); }

// A sd at a cell: (1 + kx_c + kx_r + ky_c + ky_u) c - kx_c l - kx_r r - ky_c d - ky_u u.
template <typename T>
__device__ __forceinline__ T pc_op(T kxc, T kxr, T kyc, T kyu, T c, T l, T r, T d, T u)
{
    const T dg = T(1) + (kxr + kxc) + (kyu + kyc);
    return fma_t(dg, c, -fma_t(kxc, l, kxr * r)) - fma_t(kyc, d, kyu * u);
}

// The Chebyshev fold sd = a sd + b s (pp > 0).
template <typename T>
__device__ __forceinline__ T pc_fold(T a, T b, T sd, T s)
{
    return fma_t(a, sd, b * s);
}

// Chebyshev inner step of the PPCG preconditioner over tile (tx, ty): the
// recurrence of ppcg.c:29-61 applied to A z = r from z = 0 (s: its residual),
// on the T layout in T arithmetic (the preconditioner only steers the
// iteration; the dot products, the solution and the residual replacements
// stay FP64). sd = fold(sd_in, s_in) (FOLD 1: s / theta; FOLD 2: fa sd +
// fb s), read at the stencil points; s_out = s_in - A sd; z = sd (ACC false)
// or z += sd; sd_out = sd.
template <typename T, int FOLD, bool ACC>
__device__ __forceinline__ void rf_pc_tile(const Lay& L, int tx, int ty, double theta, double fa, double fb,
                                           const T* __restrict__ sd_in, T* __restrict__ sd_out,
                                           const T* __restrict__ s_in, T* __restrict__ s_out, T* __restrict__ z,
                                           const T* __restrict__ kx, const T* __restrict__ ky)
{
    constexpr int N = Pack<T>::N;
    const Span<N> s(L, tx, ty);
    const T th = (T)theta, ta = (T)fa, tb = (T)fb;
    auto fold1 = [&](T sdv, T sv) -> T { return FOLD == 1 ? sv / th : pc_fold(ta, tb, sdv, sv); };
    auto cur = [&](long idx) -> Cells<T> {
        Cells<T> a = ld(s_in + idx);
        if (FOLD == 1) {
#pragma unroll
            for (int m = 0; m < N; ++m) a.e[m] = fold1(a.e[m], a.e[m]);
        } else {
            const Cells<T> d = ld(sd_in + idx);
#pragma unroll
            for (int m = 0; m < N; ++m) a.e[m] = fold1(d.e[m], a.e[m]);
        }
        return a;
    };
    auto cur1 = [&](long idx) -> T { return fold1(FOLD == 1 ? T(0) : sd_in[idx], s_in[idx]); };
    const long xp = L.xp;
    long i = (long)(s.j0 + 1) * xp + s.cc;
    Cells<T> sc = cur(i), sdn = cur(i - xp), kyc = ld(ky + i);
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
    for (int j = s.j0; j < s.j1; ++j, i += xp) {
        const Cells<T> su = cur(i + xp), kyu = ld(ky + i + xp), kxc = ld(kx + i);
        T sl = __shfl_up_sync(kFull, sc.e[N - 1], 1);
        T sr = __shfl_down_sync(kFull, sc.e[0], 1);
        T kxr = __shfl_down_sync(kFull, kxc.e[0], 1);
        if (s.lane == 0) sl = cur1(i - 1);
        if (s.lane == 31) {
            sr = cur1(i + N);
            kxr = kx[i + N];
        }
        if (s.any) {
            const Cells<T> rc = ld(s_in + i);
            Cells<T> rn, zv;
            if (ACC) zv = ld(z + i);
#pragma unroll
            for (int m = 0; m < N; ++m) {
                const T c = sc.e[m];
                const T l = m == 0 ? sl : sc.e[m - 1];
                const T rr = m == N - 1 ? sr : sc.e[m + 1];
                const T kr = m == N - 1 ? kxr : kxc.e[m + 1];
                const T v = pc_op<T>(kxc.e[m], kr, kyc.e[m], kyu.e[m], c, l, rr, sdn.e[m], su.e[m]);
                rn.e[m] = rc.e[m] - v;
                zv.e[m] = ACC ? zv.e[m] + c : c;
            }
            st8(s_out + i, rn);
            st8(sd_out + i, sc);
            st8(z + i, zv);
        }
        sdn = sc;
        sc = su;
        kyc = kyu;
    }
}

// Last inner step of the PPCG preconditioner over tile (tx, ty), cell-local:
// sd = fold(sd, s) as rf_pc_tile; z = sd (FOLD 1) or z += sd (FOLD 2), in T
// arithmetic. Returns this thread's share of sum(r z) over the stored values,
// accumulated in FP64.
template <typename T, int FOLD>
__device__ __forceinline__ double rf_pc_last_tile(const Lay& L, int tx, int ty, double theta, double fa, double fb,
                                                  const T* __restrict__ sd, const T* __restrict__ s_in,
                                                  T* __restrict__ z, const T* __restrict__ r)
{
    constexpr int N = Pack<T>::N;
    const Span<N> s(L, tx, ty);
    const T th = (T)theta, ta = (T)fa, tb = (T)fb;
    double acc = 0.0;
    if (s.any) {
        long i = (long)(s.j0 + 1) * L.xp + s.c0;
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += L.xp) {
            const Cells<T> sv = ld(s_in + i), rv = ld(r + i);
            Cells<T> zv;
            Cells<T> dv;
            if (FOLD == 2) {
                zv = ld(z + i);
                dv = ld(sd + i);
            }
#pragma unroll
            for (int m = 0; m < N; ++m) {
                const T d = FOLD == 1 ? sv.e[m] / th : pc_fold(ta, tb, dv.e[m], sv.e[m]);
                zv.e[m] = FOLD == 1 ? d : zv.e[m] + d;
                if (s.c0 + m < L.nx) acc += (double)rv.e[m] * (double)zv.e[m];
            }
            st8(z + i, zv);
        }
    }
    return acc;
}

// Reliable update, part 1, tile (tx, ty): u += xs in FP64 (u in the chunk
// layout: row length gx, halo depth hd), xs = 0.
template <typename T, bool CG = false>
__device__ __forceinline__ void rf_fold_tile(const Lay& L, int tx, int ty, int gx, int hd, double* __restrict__ u,
                                             T* __restrict__ xs)
{
    constexpr int N = Pack<T>::N;
    const Span<N> s(L, tx, ty);
    for (int j = s.j0; j < s.j1; ++j)
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const int k = s.c0 + m;
            if (k >= L.nx) break;
            const long e = (long)(j + 1) * L.xp + k;
            double* ue = u + (long)(hd + k) + (long)(hd + j) * gx;
            *ue = ldc1<CG>(ue) + (double)ldc1<CG>(xs + e);
            xs[e] = 0;
        }
}

// Reliable update, part 2, tile (tx, ty): r = u0 - A u in FP64 with the FP64
// coefficients and the reflective boundary (a neighbour outside the interior
// is the centre value); rT = r; adds r.r and rT.rT to acc.
template <typename T, bool CG = false>
__device__ __forceinline__ void rf_resid_tile(const Lay& L, int tx, int ty, int gx, int hd,
                                              const double* __restrict__ u, const double* __restrict__ u0,
                                              const double* __restrict__ kx, const double* __restrict__ ky,
                                              T* __restrict__ rT, double (&acc)[2])
{
    constexpr int N = Pack<T>::N;
    const Span<N> s(L, tx, ty);
    for (int j = s.j0; j < s.j1; ++j)
#pragma unroll
        for (int m = 0; m < N; ++m) {
            const int k = s.c0 + m;
            if (k >= L.nx) break;
            const long i = (long)(hd + k) + (long)(hd + j) * gx;
            const double c = ldc1<CG>(u + i);
            const double l = k > 0 ? ldc1<CG>(u + i - 1) : c;
            const double rr = k < L.nx - 1 ? ldc1<CG>(u + i + 1) : c;
            const double d = j > 0 ? ldc1<CG>(u + i - gx) : c;
            const double up = j < L.ny - 1 ? ldc1<CG>(u + i + gx) : c;
            const double rv = u0[i] - smvp(kx[i], kx[i + 1], ky[i], ky[i + gx], c, l, rr, d, up);
            const T rt = (T)rv;
            rT[(long)(j + 1) * L.xp + k] = rt;
            acc[0] += rv * rv;
            acc[1] += (double)rt * (double)rt;
        }
}

}  // namespace rf
}  // namespace tl2d
