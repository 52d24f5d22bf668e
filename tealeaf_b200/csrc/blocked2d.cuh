// blocked2d.cuh -- temporally blocked Chebyshev trips and PPCG inner steps
// (2D, FP64, one chunk with four external faces).
//
// Between two norm evaluations a Chebyshev trip (cheby.c:57-85) and a PPCG
// inner step (ppcg.c:29-61) are local stencil updates with no global
// reduction, so L of them (L <= Blk::TB) run in one launch: a block takes its
// tile of Blk::TX x Blk::TY cells plus an L-cell halo on chip, each thread holding a
// 16-row column segment of the carried fields, u0 (resp. u) and the face
// coefficients in registers, advances them L times (each step's valid region
// shrinks by one cell per side; the domain boundary is the depth-1 reflective
// halo applied on the fly, in regions that reach it), and writes the tile
// back once. Every cell goes through exactly the operations of the one-step
// kernels (k_cheby_trip, k_ppcg_step) in the same order, so the results are
// bit-identical; global traffic per step drops from 56 B (64 B) per cell to
// about 13 B (15 B) at L = 5. The reflective depth-1 halo of the written
// stencil field (u, resp. sd) is stored by the boundary tiles. A norm the
// last step needs is not reduced here: k_norm2_fin sums the stored residual
// over the interior strip partition, the partition and order of the one-step
// kernels, so the norms (and the PPCG beta) are bit-identical too.
//
// Chebyshev (MODE 0), carried fields A = u, B = p, state (u_{n-1}, p_{n-1})
// with the add pending:   A += B ;  B = a_n B + b_n (u0 - A A)
// (or, with add_end, state (u_n, p_n):   B = a B + b (u0 - A A) ;  A += B,
// the order of run_cheby_iterate, cheby.c:57-85)
// PPCG (MODE 1), A = sd, B = r, fold index pp:
//   A = pp == 0 ? B / theta : a_{pp-1} A + b_{pp-1} B ;  B -= A A ;  u += A
#pragma once

#include "kernels2d.cuh"

#include <type_traits>

namespace tl2d {

constexpr int kTW = 64;                 // region columns: one per thread of a row group
#ifndef TL2D_TSEG
#define TL2D_TSEG 8
#endif
constexpr int kTSeg = TL2D_TSEG;        // region rows per thread (a column segment in registers; 8: 512
                                        // threads at 128 registers, 16 warps per SM)
constexpr int kTRows = 64 / kTSeg;      // row groups
constexpr int kTBThreads = kTW * kTRows;   // 512
constexpr int kTH = kTSeg * kTRows;     // region rows (64)

// Tile shape of each mode. The margin TB is the most steps one launch can
// take (the valid region shrinks by one cell per step); the tile is the
// region less the margin on each side. Chebyshev (MODE 0): margin 6, whose
// even value keeps the TMA-staged regions' boxes 16-byte aligned; PPCG
// (MODE 1): margin 5 with per-thread region loads, which measured faster
// for it than the staged kernel (bench.py --solver ppcg at 4096^2).
template <int MODE>
struct Blk {
    static constexpr int TB = MODE == 0 ? 6 : 5;
    static constexpr int TX = kTW - 2 * TB;   // tile columns (52 / 54)
    static constexpr int TY = kTH - 2 * TB;   // tile rows
    static_assert(TX > 0 && TY > 0, "the margin must leave a tile");
};

struct BlockedArgs {
    int steps;          // L <= the mode's margin (Blk<MODE>::TB)
    int first;          // Chebyshev: coefficient index of the first trip; PPCG: pp of the first step
    int wr_last;        // Chebyshev: write w and r of the last trip
    double theta;       // PPCG fold of pp == 0
    const double* alphas;
    const double* betas;
    int add_end;        // Chebyshev: each trip ends with its u += p (the kernel-interface calls'
                        // order) instead of starting with the previous trip's
};

// Thread (cx, cy) holds column cx of the region, rows cy * kTSeg .. + kTSeg,
// in registers: the two carried fields, u0 (Chebyshev) or u (PPCG, tile cells)
// and the face coefficients. Each step's stencil field A goes through shared
// memory (two buffers, alternating by step) for the neighbours held by other
// warps (one column per warp) and other segments (one row each side);
// neighbours within a warp come by shuffle, within the segment from
// registers. A neighbour outside the interior is the cell itself (the
// reflective depth-1 halo); cells outside the interior or beyond the loaded
// margin compute values nothing valid reads.
// The operand region of a tile (kTW x kTH cells from grid column xs =
// X0 - TB, row ys = Y0 - TB): src.a / b / c / kx / ky (gi, ry, cx) give the
// value of a field at grid index gi, region row ry, region column cx; kxr the
// face coefficient one column to the right.
struct GlobalRegion {
    const double* A;
    const double* B;
    const double* C;
    const double* KX;
    const double* KY;
    __device__ __forceinline__ double a(long gi, int, int) const { return A[gi]; }
    __device__ __forceinline__ double b(long gi, int, int) const { return B[gi]; }
    __device__ __forceinline__ double c(long gi, int, int) const { return C[gi]; }
    __device__ __forceinline__ double kx(long gi, int, int) const { return KX[gi]; }
    __device__ __forceinline__ double kxr(long gi, int, int) const { return KX[gi + 1]; }
    __device__ __forceinline__ double ky(long gi, int, int) const { return KY[gi]; }
};

// One tile: L <= TB steps of MODE on the region given by `src`, then the
// tile written back. S0, S1: the two kTH x kTW stencil buffers; loaded() runs
// in every thread once the region is in registers.
template <int MODE, typename Src, typename Loaded>
__device__ __forceinline__ void blocked_tile(const Geo& g, const BlockedArgs& a, int X0, int Y0, const Src& src,
                                             double* A_out, double* __restrict__ B_out, double* __restrict__ u,
                                             double* __restrict__ w, double* __restrict__ r, double* const S0,
                                             double* const S1, Loaded loaded)
{
    const int x = g.x, hd = g.hd;
    const int ilo = hd, ihi = g.x - hd, jlo = hd, jhi = g.y - hd;   // interior [lo, hi)
    const int H = a.steps;
    const int tid = threadIdx.x, cx = tid % kTW, cy = tid / kTW, lane = tid & 31;
    const int gx = X0 - Blk<MODE>::TB + cx;    // grid column of this thread
    const int oy = Y0 - Blk<MODE>::TB;         // grid row of region row 0
    const int r0 = cy * kTSeg;       // first region row of this thread
    const bool colin = gx >= ilo && gx < ihi;
    const int mxc = max(max(Blk<MODE>::TB - cx, cx - (Blk<MODE>::TB + Blk<MODE>::TX - 1)), 0);   // column distance outside the tile
    const bool at_l = gx == ilo, at_r = gx == ihi - 1;
    const bool hi_half = cx >= 32;
    const int edge_lane = hi_half ? 0 : 31, edge_dx = hi_half ? -1 : 1;
    // does the region reach the domain boundary (then neighbours are reflected)?
    const bool touches = X0 - Blk<MODE>::TB <= ilo || X0 - Blk<MODE>::TB + kTW > ihi - 1 || oy <= jlo || oy + kTH > jhi - 1;

    double av[kTSeg], bv[kTSeg], cv[kTSeg], kxc[kTSeg], kxr[kTSeg], kyc[kTSeg + 1];
#pragma unroll
    for (int k = 0; k <= kTSeg; ++k) {
        const int ry = r0 + k, gy = oy + ry;
        const int my = max(max(Blk<MODE>::TB - ry, ry - (Blk<MODE>::TB + Blk<MODE>::TY - 1)), 0);
        const bool in = colin && gy >= jlo && gy < jhi && max(mxc, my) <= H;
        const long gi = gx + (long)gy * x;
        // ky of rows jlo..jhi: the face above the top interior row is read as the one-step kernels do
        const bool in_ky = colin && gy >= jlo && gy <= jhi && max(mxc, my) <= H + 1;
        kyc[k] = in_ky ? src.ky(gi, ry, cx) : 0.0;   // k == kTSeg: ky_u of the segment's top row
        if (k == kTSeg) break;
        av[k] = in ? src.a(gi, ry, cx) : 0.0;
        bv[k] = in ? src.b(gi, ry, cx) : 0.0;
        if (MODE == 0) cv[k] = in ? src.c(gi, ry, cx) : 0.0;
        else cv[k] = (in && mxc == 0 && my == 0) ? src.c(gi, ry, cx) : 0.0;
        kxc[k] = in ? src.kx(gi, ry, cx) : 0.0;
        kxr[k] = in ? src.kxr(gi, ry, cx) : 0.0;
    }
    loaded();
    for (int i = 0; i < H; ++i) {
        double* const As = (i & 1) ? S1 : S0;
        // pass A, pointwise
        {
            const int pp = a.first + i;
            const double fa = (MODE == 1 && pp > 0) ? a.alphas[pp - 1] : 0.0;
            const double fb = (MODE == 1 && pp > 0) ? a.betas[pp - 1] : 0.0;
            if (MODE == 1 && pp == 0) {
#pragma unroll
                for (int k = 0; k < kTSeg; ++k) {
                    av[k] = bv[k] / a.theta;
                    As[(r0 + k) * kTW + cx] = av[k];
                }
            } else if (MODE == 0 && a.add_end && i == 0) {
#pragma unroll
                for (int k = 0; k < kTSeg; ++k) As[(r0 + k) * kTW + cx] = av[k];
            } else {
#pragma unroll
                for (int k = 0; k < kTSeg; ++k) {
                    av[k] = MODE == 0 ? av[k] + bv[k] : fa * av[k] + fb * bv[k];
                    As[(r0 + k) * kTW + cx] = av[k];
                }
            }
        }
        __syncthreads();
        // pass B, the stencil on A (reflection only in regions at the boundary)
        auto pass_b = [&](auto reflect) {
            constexpr bool REFLECT = decltype(reflect)::value;
            const bool last = i == H - 1;
            const double ca = MODE == 0 ? a.alphas[a.first + i] : 0.0;
            const double cb = MODE == 0 ? a.betas[a.first + i] : 0.0;
#pragma unroll
            for (int k = 0; k < kTSeg; ++k) {
                const int ry = r0 + k, gy = oy + ry, o = ry * kTW + cx;
                const double c = av[k];
                double dn = k > 0 ? av[k - 1] : (ry > 0 ? As[o - kTW] : 0.0);
                double up = k < kTSeg - 1 ? av[k + 1] : (ry < kTH - 1 ? As[o + kTW] : 0.0);
                double l = __shfl_up_sync(kFull, c, 1);
                double rr = __shfl_down_sync(kFull, c, 1);
                // lane 0 / 31 at the region's edges keep 0 (nb is 0 off the edge lane)
                const double nb = lane == edge_lane ? As[o + edge_dx] : 0.0;
                if (lane == 0) l = nb;
                if (lane == 31) rr = nb;
                if (REFLECT) {
                    if (at_l) l = c;
                    if (at_r) rr = c;
                    if (gy == jlo) dn = c;
                    if (gy == jhi - 1) up = c;
                }
                const double v = smvp(kxc[k], kxr[k], kyc[k], kyc[k + 1], c, l, rr, dn, up);
                if (MODE == 0) {
                    const double res = cv[k] - v;
                    bv[k] = ca * bv[k] + cb * res;
                    const bool in_tile = colin && mxc == 0 && ry >= Blk<MODE>::TB && ry < Blk<MODE>::TB + Blk<MODE>::TY && gy < jhi;
                    if (last && in_tile && a.wr_last) {
                        const long gi = gx + (long)gy * x;
                        w[gi] = v;
                        r[gi] = res;
                    }
                } else {
                    bv[k] = bv[k] - v;
                    cv[k] += c;   // u; only tile cells (loaded, written back) matter
                }
            }
        };
        if (touches) pass_b(std::true_type());
        else pass_b(std::false_type());
    }
    // write the tile: A (u, resp. sd) with its reflective depth-1 halo, B (p,
    // resp. r). With add_end the last trip's u += p is applied here, and the
    // halo mirrors u before that add: the value a call-by-call sequence
    // leaves there (its depth-1 halo update comes before each call).
    const bool add_now = MODE == 0 && a.add_end && H > 0;
    if (colin && mxc == 0) {
#pragma unroll
        for (int k = 0; k < kTSeg; ++k) {
            const int ry = r0 + k, gy = oy + ry;
            if (ry < Blk<MODE>::TB || ry >= Blk<MODE>::TB + Blk<MODE>::TY || gy >= jhi) continue;
            const long gi = gx + (long)gy * x;
            const double hv = av[k];
            const double av_ = add_now ? av[k] + bv[k] : av[k];
            A_out[gi] = av_;
            B_out[gi] = bv[k];
            if (MODE == 1) u[gi] = cv[k];
            if (at_l) A_out[gi - 1] = hv;
            if (at_r) A_out[gi + 1] = hv;
            if (gy == jlo) A_out[gi - x] = hv;
            if (gy == jhi - 1) A_out[gi + x] = hv;
        }
    }
}

template <int MODE>
static __global__ void __launch_bounds__(kTBThreads, 1) k_blocked(Geo g, BlockedArgs a, const double* __restrict__ A_in,
                                                                  const double* __restrict__ B_in, double* A_out,
                                                                  double* __restrict__ B_out,
                                                                  const double* __restrict__ u0,
                                                                  double* __restrict__ u, double* __restrict__ w,
                                                                  double* __restrict__ r,
                                                                  const double* __restrict__ kx,
                                                                  const double* __restrict__ ky,
                                                                  const int* __restrict__ done)
{
    extern __shared__ double tb_smem[];
    double* const S0 = tb_smem;           // [kTH * kTW]
    double* const S1 = S0 + kTH * kTW;    // [kTH * kTW]
    if (gate_closed(done)) return;
    const GlobalRegion src{A_in, B_in, MODE == 0 ? u0 : u, kx, ky};
    blocked_tile<MODE>(g, a, g.hd + blockIdx.x * Blk<MODE>::TX, g.hd + blockIdx.y * Blk<MODE>::TY, src, A_out, B_out, u, w, r, S0, S1,
                       [] {});
}

// ------------------------------------------------------ TMA-staged form --
// k_blocked as a persistent kernel whose tile regions arrive by TMA: one
// block per SM walks tiles blockIdx.x, + gridDim.x, ...; one thread issues
// the five region boxes (kTW x kTH cells of A, B, C = u0 or u, kx, ky, from
// grid column X0 - Blk<MODE>::TB, row Y0 - Blk<MODE>::TB) of the block's NEXT tile into a
// shared-memory staging area as soon as every thread has taken the current
// tile's region into registers, so the loads of tile t+1 overlap the steps
// of tile t. Boxes start on a 16-byte boundary when the halo depth and Blk<MODE>::TB
// are even (X0 - Blk<MODE>::TB = hd - Blk<MODE>::TB + Blk<MODE>::TX bx); cells outside the array read as
// zero and, as in k_blocked, only cells inside the interior and the margin
// are taken. The two cells the staging lacks (kx one column right of the
// region, ky one row above it) only feed cells beyond the valid margin.
// Every wait is bounded (err); every issued region is waited for.
struct BlockedMaps {
    CUtensorMap a, b, c, kx, ky;
};
constexpr size_t kBlockedFieldDoubles = (size_t)kTH * kTW;
constexpr size_t kBlockedTmaBytes = sizeof(double) * 7 * kBlockedFieldDoubles + 8 + 128;

struct StagedRegion {
    const double* s;   // a, b, c, kx, ky: kTH x kTW each
    __device__ __forceinline__ double at(int f, int ry, int cx) const { return s[(f * kTH + ry) * kTW + cx]; }
    __device__ __forceinline__ double a(long, int ry, int cx) const { return at(0, ry, cx); }
    __device__ __forceinline__ double b(long, int ry, int cx) const { return at(1, ry, cx); }
    __device__ __forceinline__ double c(long, int ry, int cx) const { return at(2, ry, cx); }
    __device__ __forceinline__ double kx(long, int ry, int cx) const { return at(3, ry, cx); }
    __device__ __forceinline__ double kxr(long, int ry, int cx) const { return cx + 1 < kTW ? at(3, ry, cx + 1) : 0.0; }
    __device__ __forceinline__ double ky(long, int ry, int cx) const { return ry < kTH ? at(4, ry, cx) : 0.0; }
};

template <int MODE>
static __global__ void __launch_bounds__(kTBThreads, 1) k_blocked_tma(Geo g, BlockedArgs a,
                                                                      const __grid_constant__ BlockedMaps maps,
                                                                      double* A_out, double* __restrict__ B_out,
                                                                      double* __restrict__ u, double* __restrict__ w,
                                                                      double* __restrict__ r,
                                                                      const int* __restrict__ done, int* err)
{
    extern __shared__ __align__(128) unsigned char tbt_raw[];
    double* const S0 = reinterpret_cast<double*>(tbt_raw + ((128 - (tl::smem_addr(tbt_raw) & 127)) & 127));
    double* const S1 = S0 + kBlockedFieldDoubles;
    double* const stg = S1 + kBlockedFieldDoubles;
    unsigned long long* const bar = reinterpret_cast<unsigned long long*>(stg + 5 * kBlockedFieldDoubles);
    if (gate_closed(done)) return;
    const int ntx = (g.x - 2 * g.hd + Blk<MODE>::TX - 1) / Blk<MODE>::TX;
    const int ntiles = ntx * ((g.y - 2 * g.hd + Blk<MODE>::TY - 1) / Blk<MODE>::TY);
    const int tid = threadIdx.x;
    auto issue = [&](int t) {
        const int xs = g.hd + (t % ntx) * Blk<MODE>::TX - Blk<MODE>::TB, ys = g.hd + (t / ntx) * Blk<MODE>::TY - Blk<MODE>::TB;
        tl::mbar_expect_tx(bar, (unsigned)(5 * kBlockedFieldDoubles * sizeof(double)));
        tl::tma_load_3d(stg, &maps.a, xs, ys, 0, bar);
        tl::tma_load_3d(stg + kBlockedFieldDoubles, &maps.b, xs, ys, 0, bar);
        tl::tma_load_3d(stg + 2 * kBlockedFieldDoubles, &maps.c, xs, ys, 0, bar);
        tl::tma_load_3d(stg + 3 * kBlockedFieldDoubles, &maps.kx, xs, ys, 0, bar);
        tl::tma_load_3d(stg + 4 * kBlockedFieldDoubles, &maps.ky, xs, ys, 0, bar);
    };
    if (tid == 0) {
        tl::mbar_init(bar, 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (tid == 0 && (int)blockIdx.x < ntiles) issue(blockIdx.x);
    unsigned phase = 0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x, phase ^= 1u) {
        tl::mbar_wait(bar, phase, err);
        const int X0 = g.hd + (t % ntx) * Blk<MODE>::TX, Y0 = g.hd + (t / ntx) * Blk<MODE>::TY;
        blocked_tile<MODE>(g, a, X0, Y0, StagedRegion{stg}, A_out, B_out, u, w, r, S0, S1, [&] {
            __syncthreads();   // every thread holds the region: the staging is free for the next tile
            if (tid == 0 && t + (int)gridDim.x < ntiles) issue(t + gridDim.x);
        });
    }
}

// sum(b^2) over the interior with the interior-sweep partition (as k_norm2),
// then `fin` with the total; skipped once the loop has ended.
template <typename Finish>
static __global__ void __launch_bounds__(BX) k_norm2_fin(Geo g, const double* __restrict__ b, ReduceSlots rs,
                                                       const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        long i = s.k + (long)s.j0 * g.x;
        for (int j = s.j0; j < s.j1; ++j, i += g.x) acc[0] += b[i] * b[i];
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// `fin` alone (a block of trips without a norm); skipped once the loop has ended.
template <typename Finish>
static __global__ void k_finish_only(const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done) || threadIdx.x != 0) return;
    const double t[1] = {0.0};
    fin(t);
}

template <int MODE>
constexpr size_t blocked_smem()
{
    return sizeof(double) * 2 * kTH * kTW;
}

template <int MODE>
inline dim3 blocked_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, Blk<MODE>::TX), tl::ceil_div(g.y - 2 * g.hd, Blk<MODE>::TY));
}

}  // namespace tl2d
