// pcblock2d.cuh -- temporally blocked inner steps of the PPCG preconditioner
// of the refinement form (the T layout of refine2d.cuh).
//
// z = q(A) r takes ppcg_inner_steps Chebyshev steps on A z = r from z = 0
// (ppcg.c:29-61): ni - 1 stencil steps and a final cell-local fold. Between
// the dot products of the outer PCG step nothing global happens, so up to
// kPcMax stencil steps run in one launch: a block takes a 64 x 64 region (its
// 54 x 54 tile plus a halo of `steps` cells) on chip, each thread holding a
// column segment of 16 rows in registers (sd, s, z and the face
// coefficients); only the folded sd of the current step goes through shared
// memory (two buffers, alternating by step, one barrier per step), for the
// neighbours in other warps and segments. The valid region shrinks by one
// cell per side and step, and the tile is written back once. Cells outside
// the interior hold 0 and stay 0 (their face coefficients are 0, as in the T
// layout). Every tile cell goes through the operations of k_rf_pc /
// k_rf_pc_last (pc_fold, pc_op) in the same order and precision, so the
// fields are bit-identical to the one-step chain; with `last` the launch also
// applies the final fold and sums r.z over its tile (a different partition
// from k_rf_pc_last: the sum may differ in the last bits).
#pragma once

#include "refine2d.cuh"

namespace tl2d {
namespace rf {

constexpr int kPcMax = 5;                        // most stencil steps per launch
constexpr int kPcW = 64;                         // region columns: one per thread of a row group
constexpr int kPcSeg = 16;                       // region rows per thread
constexpr int kPcGroups = 4;                     // row groups
constexpr int kPcThreads = kPcW * kPcGroups;     // 256
constexpr int kPcH = kPcSeg * kPcGroups;         // region rows (64)
constexpr int kPcX = kPcW - 2 * kPcMax;          // tile columns (54)
constexpr int kPcY = kPcH - 2 * kPcMax;          // tile rows (54)

struct PcArgs {
    int steps;               // stencil steps of this launch, 1..kPcMax
    int first;               // inner step index pp of the first of them
    double theta;            // fold of pp == 0: sd = s / theta
    const double* alphas;    // Chebyshev coefficients (fold of pp > 0 uses pp - 1)
    const double* betas;
};

// A0, A1: the folded sd, alternating by step, kPcH x kPcW each.
template <typename T>
constexpr size_t pc_smem()
{
    return sizeof(T) * 2 * kPcH * kPcW;
}

inline dim3 pc_grid(const Lay& L) { return dim3(tl::ceil_div(L.nx, kPcX), tl::ceil_div(L.ny, kPcY)); }

// FIRST: the launch starts at pp = 0 (s_in is r, sd_in and z are not read,
// z starts at 0). LAST: after the stencil steps the final inner step
// pp = first + steps folds sd, adds it to z, writes z only and reduces r.z
// into `fin`; otherwise sd, s and z of the tile are written to sd_out, s_out
// and z. sd_out / s_out must not alias sd_in / s_in (neighbouring tiles read
// the halo of the inputs); z is read and written at tile cells only.
template <typename T, bool FIRST, bool LAST>
__global__ void __launch_bounds__(kPcThreads, sizeof(T) == 4 ? 2 : 1)
    k_rf_pc_blocked(Lay L, const MxState* __restrict__ st, PcArgs a, const T* __restrict__ sd_in,
                    const T* __restrict__ s_in, T* __restrict__ sd_out, T* __restrict__ s_out, T* __restrict__ z,
                    const T* __restrict__ kx, const T* __restrict__ ky, const T* __restrict__ r, ReduceSlots rs,
                    FinPcgZ fin)
{
    extern __shared__ __align__(16) unsigned char pc_raw[];
    T* const A0 = reinterpret_cast<T*>(pc_raw);
    T* const A1 = A0 + kPcH * kPcW;
    if (mx_idle(st)) return;
    const int tid = threadIdx.x, cx = tid % kPcW, cy = tid / kPcW, lane = tid & 31;
    const int X0 = blockIdx.x * kPcX, Y0 = blockIdx.y * kPcY;
    const int gx = X0 - kPcMax + cx;   // interior column of this thread
    const int oy = Y0 - kPcMax;        // interior row of region row 0
    const int r0 = cy * kPcSeg;        // first region row of this thread
    const int H = a.steps;
    const bool colin = gx >= 0 && gx < L.nx;
    const int mxc = max(max(kPcMax - cx, cx - (kPcMax + kPcX - 1)), 0);   // column distance outside the tile
    // the one neighbour column of this warp held by another warp (none at the region's edges)
    const bool hi_half = cx >= 32;
    const int edge_lane = hi_half ? 0 : 31, edge_dx = hi_half ? -1 : 1;

    T av[kPcSeg], bv[kPcSeg], zv[kPcSeg], kxc[kPcSeg], kxr[kPcSeg], kyc[kPcSeg + 1];
#pragma unroll
    for (int k = 0; k <= kPcSeg; ++k) {
        const int ry = r0 + k, gy = oy + ry;
        const int my = max(max(kPcMax - ry, ry - (kPcMax + kPcY - 1)), 0);
        const bool in = colin && gy >= 0 && gy < L.ny && max(mxc, my) <= H;
        const long gi = (long)(gy + 1) * L.xp + gx;
        kyc[k] = in ? ky[gi] : T(0);   // k == kPcSeg: ky_u of the segment's top row
        if (k == kPcSeg) break;
        const bool tile = in && mxc == 0 && my == 0;
        av[k] = (!FIRST && in) ? sd_in[gi] : T(0);
        bv[k] = in ? s_in[gi] : T(0);
        zv[k] = (!FIRST && tile) ? z[gi] : T(0);
        kxc[k] = in ? kx[gi] : T(0);
        kxr[k] = in ? kx[gi + 1] : T(0);
    }
    const T th = (T)a.theta;
    // one stencil step on the folded av[] (in As): s -= A sd ; z += sd (z = sd when INIT)
    auto stencil = [&](const T* As, bool init) {
#pragma unroll
        for (int k = 0; k < kPcSeg; ++k) {
            const int ry = r0 + k, o = ry * kPcW + cx;
            const T c = av[k];
            const T d = k > 0 ? av[k - 1] : (ry > 0 ? As[o - kPcW] : T(0));
            const T u = k < kPcSeg - 1 ? av[k + 1] : (ry < kPcH - 1 ? As[o + kPcW] : T(0));
            T l = __shfl_up_sync(kFull, c, 1);
            T rr = __shfl_down_sync(kFull, c, 1);
            const bool edge = lane == edge_lane;
            const T nb = edge ? As[o + edge_dx] : T(0);
            if (lane == 0) l = hi_half ? nb : T(0);
            if (lane == 31) rr = hi_half ? T(0) : nb;
            const T v = pc_op<T>(kxc[k], kxr[k], kyc[k], kyc[k + 1], c, l, rr, d, u);
            bv[k] = bv[k] - v;
            zv[k] = init ? c : zv[k] + c;
        }
    };
    for (int i = 0; i < H; ++i) {
        const int pp = a.first + i;
        T* const As = (i & 1) ? A1 : A0;
        if (FIRST && i == 0) {
#pragma unroll
            for (int k = 0; k < kPcSeg; ++k) {
                av[k] = bv[k] / th;
                As[(r0 + k) * kPcW + cx] = av[k];
            }
            __syncthreads();
            stencil(As, true);
        } else {
            const T fa = (T)a.alphas[pp - 1], fb = (T)a.betas[pp - 1];
#pragma unroll
            for (int k = 0; k < kPcSeg; ++k) {
                av[k] = pc_fold(fa, fb, av[k], bv[k]);
                As[(r0 + k) * kPcW + cx] = av[k];
            }
            __syncthreads();
            stencil(As, false);
        }
    }
    double acc[1] = {0.0};
    const T fa = LAST ? (T)a.alphas[a.first + H - 1] : T(0), fb = LAST ? (T)a.betas[a.first + H - 1] : T(0);
    if (colin && mxc == 0) {
#pragma unroll
        for (int k = 0; k < kPcSeg; ++k) {
            const int ry = r0 + k, gy = oy + ry;
            if (ry < kPcMax || ry >= kPcMax + kPcY || gy >= L.ny) continue;
            const long gi = (long)(gy + 1) * L.xp + gx;
            if (LAST) {
                const T zn = zv[k] + pc_fold(fa, fb, av[k], bv[k]);
                z[gi] = zn;
                acc[0] += (double)r[gi] * (double)zn;
            } else {
                sd_out[gi] = av[k];
                s_out[gi] = bv[k];
                z[gi] = zv[k];
            }
        }
    }
    if (LAST) tl::grid_sum<1, kPcThreads>(acc, rs, block_id(), block_count(), fin);
}

}  // namespace rf
}  // namespace tl2d
