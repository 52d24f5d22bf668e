// rftma2d.cuh -- the refinement form's CG sweeps (refine2d.cuh, T layout)
// with their operand rows brought into shared memory by TMA (tma.cuh).
//
// A tile's row is BX threads x N cells = 1024 bytes (256 floats or 128
// doubles), the largest box a map allows in x, so the one-cell column ring of
// the w sweep comes in by two extra 16-byte boxes per row (left of the tile,
// right of it). Stages of kRfRows rows in a kRfStages ring, completed on
// shared-memory barriers with bounded waits. The threads keep the tiles, the
// rows in order and the arithmetic of rf_w_tile / rf_ur_tile, so results and
// reduction partials are bit-identical to k_rf_w / k_rf_ur. Every box starts
// on a 16-byte boundary: tile columns are multiples of 1024 bytes, the left
// ring box starts 16 bytes before the tile (a negative start at the first
// tile reads zeros, as the padding would), and rows are xp elements (a
// multiple of 64).
#pragma once

#include "refine2d.cuh"
#include "tma.cuh"

namespace tl2d {
namespace rf {

#ifndef TL2D_RF_ROWS
#define TL2D_RF_ROWS 4
#endif
#ifndef TL2D_RF_STAGES
#define TL2D_RF_STAGES 3
#endif
#ifndef TL2D_RF_STAGES_U
#define TL2D_RF_STAGES_U 3
#endif
#ifndef TL2D_RF_BLOCKS
#define TL2D_RF_BLOCKS 4
#endif
constexpr int kRfRows = TL2D_RF_ROWS;
constexpr int kRfStages = TL2D_RF_STAGES;      // w sweep ring
constexpr int kRfStagesU = TL2D_RF_STAGES_U;   // u/r sweep ring
constexpr int kRfTmaBlocks = TL2D_RF_BLOCKS;   // resident blocks per SM of the TMA sweeps the tiles are cut for

template <typename T>
struct RfRowsW {
    static constexpr int W = BX * Pack<T>::N;     // tile row: 1024 bytes
    static constexpr int H = 16 / (int)sizeof(T);   // ring box: 16 bytes
    static_assert(W * sizeof(T) == 1024 && H * sizeof(T) == 16,
                  "TMA boxes of the refinement sweeps: 1024-byte tile rows (the widest box) and 16-byte rings");
    alignas(128) T P[kRfRows][W];
    alignas(128) T R[kRfRows][W];
    alignas(128) T KX[kRfRows][W];
    alignas(128) T KY[kRfRows][W];
    alignas(128) T PL[kRfRows][H];
    alignas(128) T PR[kRfRows][H];
    alignas(128) T RL[kRfRows][H];
    alignas(128) T RR[kRfRows][H];
    alignas(128) T KXR[kRfRows][H];
};

template <typename T>
struct RfRowsU {
    static constexpr int W = BX * Pack<T>::N;
    alignas(128) T X[kRfRows][W];
    alignas(128) T P[kRfRows][W];
    alignas(128) T R[kRfRows][W];
    alignas(128) T Wv[kRfRows][W];
};

// Maps of the w sweep: tile rows (W x kRfRows) of p, r, kx, ky and ring
// boxes (H x kRfRows) of p, r, kx.
struct RfWMaps {
    CUtensorMap p, r, kx, ky, ph, rh, kxh;
};
struct RfUMaps {
    CUtensorMap xs, p, r, w;
};

template <typename T>
constexpr size_t rf_w_tma_bytes()
{
    return kRfStages * sizeof(RfRowsW<T>) + kRfStages * 8 + 128;
}
template <typename T>
constexpr size_t rf_u_tma_bytes()
{
    return kRfStagesU * sizeof(RfRowsU<T>) + kRfStagesU * 8 + 128;
}

// k_rf_w by TMA. Stage b holds T-layout rows j0 + 4b .. j0 + 4b + 3 (interior
// rows j0-1+4b ..): the rows of interior rows j0+4b .. j0+4b+3 and their
// upper neighbours are in stages b and b+1.
template <typename T, bool FUSE_P>
__global__ void __launch_bounds__(BX, 4) k_rf_w_tma(Lay L, const MxState* __restrict__ st,
                                                    const __grid_constant__ RfWMaps m, T* __restrict__ p_out,
                                                    T* __restrict__ w, ReduceSlots rs, FinMxW fin, int* err)
{
    extern __shared__ __align__(128) unsigned char rw_raw[];
    using S = RfRowsW<T>;
    constexpr int N = Pack<T>::N, W = S::W, H = S::H;
    if (mx_idle(st)) return;
    unsigned char* base = rw_raw + ((128 - (tl::smem_addr(rw_raw) & 127)) & 127);
    S* ring = reinterpret_cast<S*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kRfStages * sizeof(S));
    const double bt = FUSE_P ? st->beta : 0.0;
    const Span<N> s(L, blockIdx.x, blockIdx.y);
    const int tid = threadIdx.x;
    const int cb = blockIdx.x * W;
    const int np = (s.j1 - s.j0 + 2 + kRfRows - 1) / kRfRows;
    constexpr unsigned kMain = sizeof(T) * kRfRows * W, kRing = sizeof(T) * kRfRows * H;
    auto issue = [&](int b) {
        S& Q = ring[b % kRfStages];
        unsigned long long* bar = &bars[b % kRfStages];
        const int y0 = s.j0 + b * kRfRows;
        tl::mbar_expect_tx(bar, kMain * (FUSE_P ? 4u : 3u) + kRing * (FUSE_P ? 5u : 3u));
        tl::tma_load_3d(&Q.P[0][0], &m.p, cb, y0, 0, bar);
        tl::tma_load_3d(&Q.PL[0][0], &m.ph, cb - H, y0, 0, bar);
        tl::tma_load_3d(&Q.PR[0][0], &m.ph, cb + W, y0, 0, bar);
        if (FUSE_P) {
            tl::tma_load_3d(&Q.R[0][0], &m.r, cb, y0, 0, bar);
            tl::tma_load_3d(&Q.RL[0][0], &m.rh, cb - H, y0, 0, bar);
            tl::tma_load_3d(&Q.RR[0][0], &m.rh, cb + W, y0, 0, bar);
        }
        tl::tma_load_3d(&Q.KX[0][0], &m.kx, cb, y0, 0, bar);
        tl::tma_load_3d(&Q.KXR[0][0], &m.kxh, cb + W, y0, 0, bar);
        tl::tma_load_3d(&Q.KY[0][0], &m.ky, cb, y0, 0, bar);
    };
    if (tid == 0) {
        for (int q = 0; q < kRfStages; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int b = 0; b < kRfStages - 1 && b < np; ++b) issue(b);
    // t: T-layout row - j0
    auto stage = [&](int t) -> const S& { return ring[(t / kRfRows) % kRfStages]; };
    using M = typename RfMath<T>::M;
    const M btm = (M)bt;
    auto fuse1 = [&](T pv, T rv) -> T { return FUSE_P ? (T)(btm * (M)pv + (M)rv) : pv; };
    auto cur = [&](int t) -> Cells<T> {
        const S& Q = stage(t);
        Cells<T> c;
#pragma unroll
        for (int k = 0; k < N; ++k) c.e[k] = fuse1(Q.P[t % kRfRows][tid * N + k], Q.R[t % kRfRows][tid * N + k]);
        return c;
    };
    auto left1 = [&](int t) -> T {
        const S& Q = stage(t);
        return tid == 0 ? fuse1(Q.PL[t % kRfRows][H - 1], Q.RL[t % kRfRows][H - 1])
                        : fuse1(Q.P[t % kRfRows][tid * N - 1], Q.R[t % kRfRows][tid * N - 1]);
    };
    auto right1 = [&](int t) -> T {
        const S& Q = stage(t);
        return tid == BX - 1 ? fuse1(Q.PR[t % kRfRows][0], Q.RR[t % kRfRows][0])
                             : fuse1(Q.P[t % kRfRows][tid * N + N], Q.R[t % kRfRows][tid * N + N]);
    };
    auto row = [&](const T (*A)[W], int t) -> Cells<T> {
        Cells<T> c;
#pragma unroll
        for (int k = 0; k < N; ++k) c.e[k] = A[t % kRfRows][tid * N + k];
        return c;
    };
    double acc = 0.0;
    Cells<T> pc, pd, kyc;
    long i = (long)(s.j0 + 1) * L.xp + s.cc;
    for (int b = 0; b * kRfRows < s.j1 - s.j0; ++b) {
        __syncthreads();   // every thread is past the rows of block b-1: stage b-1 is free
        if (tid == 0 && b + kRfStages - 1 < np) issue(b + kRfStages - 1);
        tl::mbar_wait(&bars[b % kRfStages], (unsigned)(b / kRfStages) & 1u, err);
        if (b + 1 < np) tl::mbar_wait(&bars[(b + 1) % kRfStages], (unsigned)((b + 1) / kRfStages) & 1u, err);
        if (b == 0) {
            pc = cur(1);
            pd = cur(0);
            kyc = row(stage(1).KY, 1);
        }
#pragma unroll
        for (int u = 0; u < kRfRows; ++u) {
            const int j = s.j0 + b * kRfRows + u;
            if (j >= s.j1) break;
            const int t = j + 1 - s.j0;
            const S& Q = stage(t);
            const Cells<T> pu = cur(t + 1), kyu = row(stage(t + 1).KY, t + 1), kxc = row(Q.KX, t);
            T pl = __shfl_up_sync(kFull, pc.e[N - 1], 1);
            T pr = __shfl_down_sync(kFull, pc.e[0], 1);
            T kxr = __shfl_down_sync(kFull, kxc.e[0], 1);
            if (s.lane == 0) pl = left1(t);
            if (s.lane == 31) {
                pr = right1(t);
                kxr = tid == BX - 1 ? Q.KXR[t % kRfRows][0] : Q.KX[t % kRfRows][tid * N + N];
            }
            Cells<T> wv;
#pragma unroll
            for (int k = 0; k < N; ++k) {
                const M c = (M)pc.e[k];
                const M l = k == 0 ? (M)pl : (M)pc.e[k - 1];
                const M rr = k == N - 1 ? (M)pr : (M)pc.e[k + 1];
                const M kr = k == N - 1 ? (M)kxr : (M)kxc.e[k + 1];
                wv.e[k] = (T)smvp_m<M>((M)kxc.e[k], kr, (M)kyc.e[k], (M)kyu.e[k], c, l, rr, (M)pd.e[k], (M)pu.e[k]);
            }
            if (s.any) {
                st8(w + i, wv);
                if (FUSE_P) st8(p_out + i, pc);
#pragma unroll
                for (int k = 0; k < N; ++k)
                    if (s.c0 + k < L.nx) acc += (double)wv.e[k] * (double)pc.e[k];
            }
            pd = pc;
            pc = pu;
            kyc = kyu;
            i += L.xp;
        }
    }
    double a1[1] = {acc};
    tl::grid_sum<1, BX>(a1, rs, block_id(), block_count(), fin);
}

// k_rf_ur by TMA: stage b holds T-layout rows j0+1+4b .. (interior rows
// j0+4b ..).
template <typename T>
__global__ void __launch_bounds__(BX, 4) k_rf_ur_tma(Lay L, const MxState* __restrict__ st,
                                                     const __grid_constant__ RfUMaps m, T* __restrict__ xs,
                                                     T* __restrict__ r, ReduceSlots rs, FinMxUr fin, int* err)
{
    extern __shared__ __align__(128) unsigned char ru_raw[];
    using S = RfRowsU<T>;
    constexpr int N = Pack<T>::N, W = S::W;
    if (mx_idle(st)) return;
    unsigned char* base = ru_raw + ((128 - (tl::smem_addr(ru_raw) & 127)) & 127);
    S* ring = reinterpret_cast<S*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kRfStagesU * sizeof(S));
    const Span<N> s(L, blockIdx.x, blockIdx.y);
    const int tid = threadIdx.x;
    const int cb = blockIdx.x * W;
    const int np = (s.j1 - s.j0 + kRfRows - 1) / kRfRows;
    auto issue = [&](int b) {
        S& Q = ring[b % kRfStagesU];
        unsigned long long* bar = &bars[b % kRfStagesU];
        const int y0 = s.j0 + 1 + b * kRfRows;
        tl::mbar_expect_tx(bar, 4u * sizeof(T) * kRfRows * W);
        tl::tma_load_3d(&Q.X[0][0], &m.xs, cb, y0, 0, bar);
        tl::tma_load_3d(&Q.P[0][0], &m.p, cb, y0, 0, bar);
        tl::tma_load_3d(&Q.R[0][0], &m.r, cb, y0, 0, bar);
        tl::tma_load_3d(&Q.Wv[0][0], &m.w, cb, y0, 0, bar);
    };
    if (tid == 0) {
        for (int q = 0; q < kRfStagesU; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0)
        for (int b = 0; b < kRfStagesU - 1 && b < np; ++b) issue(b);
    using M = typename RfMath<T>::M;
    const M a = (M)st->alpha;
    double acc = 0.0;
    long i = (long)(s.j0 + 1) * L.xp + s.c0;
    for (int b = 0; b < np; ++b) {
        __syncthreads();   // every thread is past stage b-1: its slot is free
        if (tid == 0 && b + kRfStagesU - 1 < np) issue(b + kRfStagesU - 1);
        tl::mbar_wait(&bars[b % kRfStagesU], (unsigned)(b / kRfStagesU) & 1u, err);
        const S& Q = ring[b % kRfStagesU];
#pragma unroll
        for (int u = 0; u < kRfRows; ++u) {
            if (s.j0 + b * kRfRows + u >= s.j1) break;
            if (s.any) {
                Cells<T> xv, rv;
#pragma unroll
                for (int k = 0; k < N; ++k) {
                    const int c = tid * N + k;
                    xv.e[k] = (T)((M)Q.X[u][c] + a * (M)Q.P[u][c]);
                    rv.e[k] = (T)((M)Q.R[u][c] - a * (M)Q.Wv[u][c]);
                    if (s.c0 + k < L.nx) acc += (double)rv.e[k] * (double)rv.e[k];
                }
                st8(xs + i, xv);
                st8(r + i, rv);
            }
            i += L.xp;
        }
    }
    double a1[1] = {acc};
    tl::grid_sum<1, BX>(a1, rs, block_id(), block_count(), fin);
}

}  // namespace rf
}  // namespace tl2d
