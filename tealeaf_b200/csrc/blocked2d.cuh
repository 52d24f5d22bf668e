// blocked2d.cuh -- temporally blocked Chebyshev trips and PPCG inner steps
// (2D, FP64, one chunk with four external faces).
//
// Between two norm evaluations a Chebyshev trip (cheby.c:57-85) and a PPCG
// inner step (ppcg.c:29-61) are local stencil updates with no global
// reduction, so L of them (L <= kTB) run in one launch: a block loads its
// tile of kTX x kTY cells plus an L-cell halo of the two carried fields into
// shared memory, advances them L times on chip (each step's valid region
// shrinks by one cell per side; the domain boundary is the depth-1 reflective
// halo applied on the fly, so boundary tiles need no halo data), and writes
// the tile back once. Every cell goes through exactly the operations of the
// one-step kernels (k_cheby_trip, k_ppcg_step) in the same order, so the
// results are bit-identical; global traffic per step drops from 56 B (64 B)
// per cell to about 13 B (15 B) at L = 5. The reflective depth-1 halo of the
// written stencil field (u, resp. sd) is stored by the boundary tiles. A norm
// the last step needs is not reduced here: k_norm2_fin sums the stored
// residual over the interior strip partition, the partition and order of the
// one-step kernels, so the norms (and the PPCG beta) are bit-identical too.
//
// Chebyshev (MODE 0), carried fields A = u, B = p, state (u_{n-1}, p_{n-1})
// with the add pending:   A += B ;  B = a_n B + b_n (u0 - A A)
// PPCG (MODE 1), A = sd, B = r, fold index pp:
//   A = pp == 0 ? B / theta : a_{pp-1} A + b_{pp-1} B ;  B -= A A ;  u += A
#pragma once

#include "kernels2d.cuh"

namespace tl2d {

constexpr int kTB = 5;                  // most steps per launch
constexpr int kTW = 64;                 // shared row pitch: one column per thread of a row group
constexpr int kTH = 48;                 // shared rows
constexpr int kTX = kTW - 2 * kTB;      // tile columns (54)
constexpr int kTY = kTH - 2 * kTB;      // tile rows (38)
constexpr int kTBThreads = 256;
constexpr int kTRows = kTBThreads / kTW;   // row groups (4): thread = (column, row group)

struct BlockedArgs {
    int steps;          // L <= kTB
    int first;          // Chebyshev: coefficient index of the first trip; PPCG: pp of the first step
    int wr_last;        // Chebyshev: write w and r of the last trip
    double theta;       // PPCG fold of pp == 0
    const double* alphas;
    const double* betas;
};

template <int MODE>
static __global__ void __launch_bounds__(kTBThreads) k_blocked(Geo g, BlockedArgs a, const double* __restrict__ A_in,
                                                               const double* __restrict__ B_in, double* A_out,
                                                               double* __restrict__ B_out, const double* __restrict__ u0,
                                                               double* __restrict__ u, double* __restrict__ w,
                                                               double* __restrict__ r, const double* __restrict__ kx,
                                                               const double* __restrict__ ky,
                                                               const int* __restrict__ done)
{
    extern __shared__ double tb_smem[];
    double* As = tb_smem;             // [kTH * kTW]
    double* Bs = As + kTH * kTW;      // [kTH * kTW]
    double* Us = Bs + kTH * kTW;      // [kTX * kTY], PPCG only
    if (gate_closed(done)) return;
    const int x = g.x, hd = g.hd;
    const int ilo = hd, ihi = g.x - hd, jlo = hd, jhi = g.y - hd;   // interior [lo, hi)
    const int X0 = hd + blockIdx.x * kTX, Y0 = hd + blockIdx.y * kTY;
    const int X1 = min(X0 + kTX, ihi), Y1 = min(Y0 + kTY, jhi);
    const int H = a.steps;
    const int ox = X0 - kTB, oy = Y0 - kTB;   // shared origin
    const int tid = threadIdx.x;

    // Thread (cx, cy): shared column cx of every kTRows-th row from cy; the
    // region of margin m of this tile is [xl, xh) x [yl, yh).
    const int cx = tid % kTW, cy = tid / kTW;
    const int gxc = ox + cx;   // this thread's grid column
    auto bounds = [&](int m, int& xl, int& xh, int& yl, int& yh) {
        xl = max(ilo, X0 - m);
        xh = min(ihi, X1 + m);
        yl = max(jlo, Y0 - m);
        yh = min(jhi, Y1 + m);
    };
    // first row >= yl of this thread's row group
    auto first_row = [&](int yl) { return yl + ((cy - (yl - oy)) % kTRows + kTRows) % kTRows; };

    // load the region of margin H (interior cells only)
    {
        int xl, xh, yl, yh;
        bounds(H, xl, xh, yl, yh);
        if (gxc >= xl && gxc < xh) {
            for (int yy = first_row(yl); yy < yh; yy += kTRows) {
                const long gi = gxc + (long)yy * x;
                const int s = (yy - oy) * kTW + cx;
                As[s] = A_in[gi];
                Bs[s] = B_in[gi];
                if (MODE == 1 && gxc >= X0 && gxc < X1 && yy >= Y0 && yy < Y1)
                    Us[(yy - Y0) * kTX + (gxc - X0)] = u[gi];
            }
        }
    }
    __syncthreads();
    for (int i = 0; i < H; ++i) {
        // pass A: pointwise over margin H - i
        {
            int xl, xh, yl, yh;
            bounds(H - i, xl, xh, yl, yh);
            double fa = 0.0, fb = 0.0;
            const int pp = a.first + i;
            if (MODE == 1 && pp > 0) {
                fa = a.alphas[pp - 1];
                fb = a.betas[pp - 1];
            }
            if (gxc >= xl && gxc < xh) {
                for (int yy = first_row(yl); yy < yh; yy += kTRows) {
                    const int s = (yy - oy) * kTW + cx;
                    if (MODE == 0) As[s] = As[s] + Bs[s];
                    else As[s] = pp == 0 ? Bs[s] / a.theta : fa * As[s] + fb * Bs[s];
                }
            }
        }
        __syncthreads();
        // pass B: stencil over margin H - i - 1
        {
            int xl, xh, yl, yh;
            bounds(H - i - 1, xl, xh, yl, yh);
            const bool last = i == H - 1;
            double ca = 0.0, cb = 0.0;
            if (MODE == 0) {
                ca = a.alphas[a.first + i];
                cb = a.betas[a.first + i];
            }
            if (gxc >= xl && gxc < xh) {
                const bool in_tx = gxc >= X0 && gxc < X1;
                for (int yy = first_row(yl); yy < yh; yy += kTRows) {
                    const int s = (yy - oy) * kTW + cx;
                    const long gi = gxc + (long)yy * x;
                    const double cc = As[s];
                    const double l = gxc == ilo ? cc : As[s - 1];
                    const double rr = gxc == ihi - 1 ? cc : As[s + 1];
                    const double d = yy == jlo ? cc : As[s - kTW];
                    const double up = yy == jhi - 1 ? cc : As[s + kTW];
                    const double v = smvp(__ldg(kx + gi), __ldg(kx + gi + 1), __ldg(ky + gi), __ldg(ky + gi + x), cc,
                                          l, rr, d, up);
                    const bool in_tile = in_tx && yy >= Y0 && yy < Y1;
                    if (MODE == 0) {
                        const double res = __ldg(u0 + gi) - v;
                        Bs[s] = ca * Bs[s] + cb * res;
                        if (last && in_tile && a.wr_last) {
                            w[gi] = v;
                            r[gi] = res;
                        }
                    } else {
                        Bs[s] = Bs[s] - v;
                        if (in_tile) Us[(yy - Y0) * kTX + (gxc - X0)] += cc;
                    }
                }
            }
        }
        __syncthreads();
    }
    // write the tile: A (u, resp. sd) with its reflective depth-1 halo, B (p, resp. r)
    if (gxc >= X0 && gxc < X1) {
        for (int yy = first_row(Y0); yy < Y1; yy += kTRows) {
            const int s = (yy - oy) * kTW + cx;
            const long gi = gxc + (long)yy * x;
            const double av = As[s];
            A_out[gi] = av;
            B_out[gi] = Bs[s];
            if (MODE == 1) u[gi] = Us[(yy - Y0) * kTX + (gxc - X0)];
            if (gxc == ilo) A_out[gi - 1] = av;
            if (gxc == ihi - 1) A_out[gi + 1] = av;
            if (yy == jlo) A_out[gi - x] = av;
            if (yy == jhi - 1) A_out[gi + x] = av;
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
    return sizeof(double) * (2 * kTH * kTW + (MODE == 1 ? kTX * kTY : 0));
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
