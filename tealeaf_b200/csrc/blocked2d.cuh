// blocked2d.cuh -- temporally blocked Chebyshev trips and PPCG inner steps
// (2D, FP64, one chunk with four external faces).
//
// Between two norm evaluations a Chebyshev trip (cheby.c:57-85) and a PPCG
// inner step (ppcg.c:29-61) are local stencil updates with no global
// reduction, so L of them (L <= kTB) run in one launch: a block takes its
// tile of kTX x kTY cells plus an L-cell halo on chip, each thread holding a
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

constexpr int kTB = 5;                  // most steps per launch
constexpr int kTW = 64;                 // region columns: one per thread of a row group
constexpr int kTSeg = 16;               // region rows per thread (a column segment in registers)
constexpr int kTRows = 4;               // row groups
constexpr int kTBThreads = kTW * kTRows;   // 256
constexpr int kTH = kTSeg * kTRows;     // region rows (64)
constexpr int kTX = kTW - 2 * kTB;      // tile columns (54)
constexpr int kTY = kTH - 2 * kTB;      // tile rows (54)

struct BlockedArgs {
    int steps;          // L <= kTB
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
    const int x = g.x, hd = g.hd;
    const int ilo = hd, ihi = g.x - hd, jlo = hd, jhi = g.y - hd;   // interior [lo, hi)
    const int X0 = hd + blockIdx.x * kTX, Y0 = hd + blockIdx.y * kTY;
    const int H = a.steps;
    const int tid = threadIdx.x, cx = tid % kTW, cy = tid / kTW, lane = tid & 31;
    const int gx = X0 - kTB + cx;    // grid column of this thread
    const int oy = Y0 - kTB;         // grid row of region row 0
    const int r0 = cy * kTSeg;       // first region row of this thread
    const bool colin = gx >= ilo && gx < ihi;
    const int mxc = max(max(kTB - cx, cx - (kTB + kTX - 1)), 0);   // column distance outside the tile
    const bool at_l = gx == ilo, at_r = gx == ihi - 1;
    const bool hi_half = cx >= 32;
    const int edge_lane = hi_half ? 0 : 31, edge_dx = hi_half ? -1 : 1;
    // does the region reach the domain boundary (then neighbours are reflected)?
    const bool touches = X0 - kTB <= ilo || X0 - kTB + kTW > ihi - 1 || oy <= jlo || oy + kTH > jhi - 1;

    double av[kTSeg], bv[kTSeg], cv[kTSeg], kxc[kTSeg], kxr[kTSeg], kyc[kTSeg + 1];
#pragma unroll
    for (int k = 0; k <= kTSeg; ++k) {
        const int ry = r0 + k, gy = oy + ry;
        const int my = max(max(kTB - ry, ry - (kTB + kTY - 1)), 0);
        const bool in = colin && gy >= jlo && gy < jhi && max(mxc, my) <= H;
        const long gi = gx + (long)gy * x;
        // ky of rows jlo..jhi: the face above the top interior row is read as the one-step kernels do
        const bool in_ky = colin && gy >= jlo && gy <= jhi && max(mxc, my) <= H + 1;
        kyc[k] = in_ky ? ky[gi] : 0.0;   // k == kTSeg: ky_u of the segment's top row
        if (k == kTSeg) break;
        av[k] = in ? A_in[gi] : 0.0;
        bv[k] = in ? B_in[gi] : 0.0;
        if (MODE == 0) cv[k] = in ? u0[gi] : 0.0;
        else cv[k] = (in && mxc == 0 && my == 0) ? u[gi] : 0.0;
        kxc[k] = in ? kx[gi] : 0.0;
        kxr[k] = in ? kx[gi + 1] : 0.0;
    }
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
                    const bool in_tile = colin && mxc == 0 && ry >= kTB && ry < kTB + kTY && gy < jhi;
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
    // the last trip's u += p when each trip ends with its add
    if (MODE == 0 && a.add_end && H > 0) {
#pragma unroll
        for (int k = 0; k < kTSeg; ++k) av[k] = av[k] + bv[k];
    }
    // write the tile: A (u, resp. sd) with its reflective depth-1 halo, B (p, resp. r)
    if (colin && mxc == 0) {
#pragma unroll
        for (int k = 0; k < kTSeg; ++k) {
            const int ry = r0 + k, gy = oy + ry;
            if (ry < kTB || ry >= kTB + kTY || gy >= jhi) continue;
            const long gi = gx + (long)gy * x;
            const double av_ = av[k];
            A_out[gi] = av_;
            B_out[gi] = bv[k];
            if (MODE == 1) u[gi] = cv[k];
            if (at_l) A_out[gi - 1] = av_;
            if (at_r) A_out[gi + 1] = av_;
            if (gy == jlo) A_out[gi - x] = av_;
            if (gy == jhi - 1) A_out[gi + x] = av_;
        }
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

inline dim3 blocked_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, kTX), tl::ceil_div(g.y - 2 * g.hd, kTY));
}

// End of a block of Chebyshev trips: advances the trip and coefficient
// counters trip by trip (end_of_trip, as FinChebyTrip does per trip); only
// the last trip can take the norm (blocks end at norm trips).
struct FinChebyBlock {
    DevState* st;
    DevParams prm;
    int* host_mirror;
    int steps;
    int norm_last;
    __device__ void operator()(const double* t) const
    {
        for (int i = 0; i < steps; ++i) {
            const bool norm = norm_last && i == steps - 1;
            st->nch += 1;
            end_of_trip(st, prm, norm ? t[0] : st->error, host_mirror);
        }
    }
};

}  // namespace tl2d
