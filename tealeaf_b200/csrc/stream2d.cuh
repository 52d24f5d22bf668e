// stream2d.cuh -- the 2D CG sweeps as persistent kernels that stream their
// operand rows through one TMA ring across every strip a block owns.
//
// The interior is cut into the same strips as every other interior sweep
// (BX columns x Geo::rows rows; strip sid = bx + by * gx, the block index of
// the one-strip-per-block sweeps). A launch has at most sm_count x 4 blocks;
// block b takes strips b, b + gridDim.x, ... in turn. One thread per block
// issues cp.async.bulk.tensor row boxes into a kStages-deep ring of
// shared-memory stages completed on mbarriers, and keeps issuing into the
// next strip while the block still computes the current one, so a block's
// rows arrive as one continuous stream with no per-strip ramp-up. Each stage
// is consumed exactly once, in order: a row's values are read from shared
// memory when its stage is current and carried in registers while the row
// below it is computed (the vertical stencil neighbours), so the stage in
// use plus kStages - 1 in flight is the whole schedule.
//
// Results are bit-identical to the one-strip-per-block sweeps: every thread
// computes the same rows, in the same order, with the same operands and
// arithmetic; each strip's block sum goes to partial slot sid and the last
// block to finish adds the partials in the order tl::grid_sum uses.
//
// The reflective halos the fused sweeps write (the new p's depth-1 halo, the
// pending u halo) are written by the threads that own the mirrored interior
// cells as they reach them, with the values the halo-duty block row of the
// one-strip sweeps wrote.
//
// Launch: programmatic dependent launch (the stream-serialisation attribute).
// A block initialises its barriers, then waits (griddepcontrol.wait) until
// the previous kernel of the stream has completed and its writes are
// visible, before it reads any operand; it lets the next kernel be launched
// (griddepcontrol.launch_dependents) once it has started, so the next
// sweep's blocks are scheduled as this sweep's blocks retire.
#pragma once

#include "kernels2d.cuh"

namespace tl2d {

// Waits for the previous kernel of the stream (no-op without the attribute).
__device__ __forceinline__ void pdl_wait() { asm volatile("griddepcontrol.wait;\n" ::: "memory"); }
// Allows the next kernel of the stream to be launched.
__device__ __forceinline__ void pdl_launch_next() { asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory"); }

#ifndef TL2D_PDL_LATE
#define TL2D_PDL_LATE 0
#endif
constexpr int kStreamBlocksPerSm = 4;

// Strip `sid` of the interior grid (gx strips per row of strips).
struct StripAt {
    int k0, j0, j1;
    __device__ __forceinline__ StripAt(const Geo& g, int gx, int sid)
    {
        const int bx = sid % gx, by = sid / gx;
        k0 = g.hd + bx * BX;
        j0 = g.hd + by * g.rows;
        j1 = min(j0 + g.rows, g.y - g.hd);
    }
};

__device__ __forceinline__ int strips_x(const Geo& g) { return (g.x - 2 * g.hd + BX - 1) / BX; }
__device__ __forceinline__ int strips_total(const Geo& g)
{
    return strips_x(g) * ((g.y - 2 * g.hd + g.rows - 1) / g.rows);
}

// Block sum of strip sid into partial slot sid (thread 0 stores it).
template <int N>
__device__ __forceinline__ void strip_partial(double (&v)[N], const ReduceSlots& rs, int sid,
                                              double (*smem)[BX / tl::kWarp])
{
    __syncthreads();   // the previous strip's block sum has read smem
    tl::block_sum<N, BX>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) rs.partials[(long)sid * N + r] = v[r];
    }
}

// After a block's last strip: the last block to arrive adds the nstrips
// partials (thread t: slots t, t + BX, ...; then a block sum, as
// tl::grid_sum does) and publishes the totals.
template <int N, typename Finish>
__device__ __forceinline__ void strips_finish(const ReduceSlots& rs, int nstrips, const Finish& fin,
                                              double (*smem)[BX / tl::kWarp])
{
    __shared__ bool last;
    const int tid = threadIdx.x;
    if (tid == 0) {
        __threadfence();
        last = atomicAdd(rs.ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (!last) return;
    __threadfence();
    double t[N];
#pragma unroll
    for (int r = 0; r < N; ++r) t[r] = 0.0;
    for (int b = tid; b < nstrips; b += BX) {
#pragma unroll
        for (int r = 0; r < N; ++r) t[r] += __ldcg(&rs.partials[(long)b * N + r]);
    }
    __syncthreads();
    tl::block_sum<N, BX>(t, smem);
    if (tid == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) {
            rs.out_dev[r] = t[r];
            if (rs.out_host) rs.out_host[r] = t[r];
        }
        fin(t);
        *rs.ticket = 0u;
    }
}

// The pending reflective halo of u (depth uhd; u is not modified by the
// sweep) for column k of strip rows j0 .. j1-1: the cells mirrored from this
// column's interior cells (2d/c_kernels/omp3/local_halos.c:66-149 pattern).
__device__ __forceinline__ void strip_u_halo(const Geo& g, const Faces& fc, int uhd, double* u, int k, int j0, int j1)
{
    const int x = g.x;
    for (int d = 0; d < uhd; ++d) {
        if (fc.b && j0 == g.hd) u[k + (long)(g.hd - 1 - d) * x] = u[k + (long)(g.hd + d) * x];
        if (fc.t && j1 == g.y - g.hd) u[k + (long)(g.y - g.hd + d) * x] = u[k + (long)(g.y - g.hd - 1 - d) * x];
    }
    if (fc.l && k == g.hd)
        for (int j = j0; j < j1; ++j)
            for (int d = 0; d < uhd; ++d) u[(long)j * x + g.hd - 1 - d] = u[(long)j * x + g.hd + d];
    if (fc.r && k == x - g.hd - 1)
        for (int j = j0; j < j1; ++j)
            for (int d = 0; d < uhd; ++d) u[(long)j * x + x - g.hd + d] = u[(long)j * x + x - g.hd - 1 - d];
}

// ------------------------------------------------------------ w sweep ----
// Stage rows of the w sweep: kRowsT rows of p and r with a two-column ring
// on each side (columns k0-2 .. k0+129: the box starts on a 16-byte boundary
// for an even halo depth), kx with one extra column, ky; each array at a
// 128-byte aligned offset. Strip rows j0-1 .. j1 (the rows below and above
// included) are staged: stage b of a strip holds rows j0-1+kRowsT*b ...
constexpr int kRowsT = 4;
constexpr int kStagesT = 3;
static_assert((BX * sizeof(double)) % 16 == 0 && ((BX + 4) * sizeof(double)) % 16 == 0 &&
                  ((BX + 2) * sizeof(double)) % 16 == 0,
              "TMA boxes of the 2D sweeps must be multiples of 16 bytes wide");
struct RowsT {
    alignas(128) double P[kRowsT][BX + 4];
    alignas(128) double R[kRowsT][BX + 4];
    alignas(128) double KX[kRowsT][BX + 2];
    alignas(128) double KY[kRowsT][BX];
};
struct Tma2Maps {
    CUtensorMap p, r, kx, ky;
};
constexpr size_t kTmaRowsBytes = kStagesT * sizeof(RowsT) + kStagesT * 8 + 128;   // + barriers + alignment

__device__ __forceinline__ int w_stages(int j0, int j1) { return (j1 - j0 + 2 + kRowsT - 1) / kRowsT; }

// CG sweep 1, persistent and TMA-fed (k_cg_w_fused semantics):
//   [p = beta p + r]   (FUSE_P; cg.c:146-164, the previous step's calc_p)
//   w = A p ; pw = sum(w*p)   (cg.c:88-113)
// With REFLECT the depth-1 reflective halo of the new p is written into
// p_out; with u_halo the pending reflective halo of u (depth uhd, u is not
// modified here). p_out == p_in's buffer when !FUSE_P. `err`: the bounded
// barrier waits' flag.
template <bool FUSE_P, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(BX, kStreamBlocksPerSm) k_cg_w_stream(
    Geo g, Faces fc, Scalar beta, const __grid_constant__ Tma2Maps maps, double* p_out, double* __restrict__ w,
    double* u_halo, int uhd, ReduceSlots rs, const int* __restrict__ done, Finish fin, int* err)
{
    extern __shared__ __align__(128) unsigned char ws_raw[];
    __shared__ double red[1][BX / tl::kWarp];
    unsigned char* base = ws_raw + ((128 - (tl::smem_addr(ws_raw) & 127)) & 127);
    RowsT* ring = reinterpret_cast<RowsT*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesT * sizeof(RowsT));
    const int tx = threadIdx.x, lane = tx & 31;
    const int gx = strips_x(g), nstrips = strips_total(g);
    const int x = g.x;
    if (tx == 0) {
        for (int q = 0; q < kStagesT; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    if (!TL2D_PDL_LATE) pdl_launch_next();
    if (gate_closed(done)) return;
    const double bt = FUSE_P ? beta.get() : 0.0;

    // producer cursor (thread 0): next stage to issue, as (strip, stage of strip)
    int p_sid = blockIdx.x, p_b = 0, p_np = 0;
    unsigned issued = 0;
    if (tx == 0 && p_sid < nstrips) {
        const StripAt ps(g, gx, p_sid);
        p_np = w_stages(ps.j0, ps.j1);
    }
    auto issue_next = [&]() {
        const StripAt ps(g, gx, p_sid);
        const int slot = (int)(issued % kStagesT);
        RowsT& S = ring[slot];
        unsigned long long* bar = &bars[slot];
        const int y0 = ps.j0 - 1 + p_b * kRowsT;
        constexpr unsigned kBytes = sizeof(double) * kRowsT * ((FUSE_P ? 2 : 1) * (BX + 4) + (BX + 2) + BX);
        tl::mbar_expect_tx(bar, kBytes);
        tl::tma_load_3d(&S.P[0][0], &maps.p, ps.k0 - 2, y0, 0, bar);
        if (FUSE_P) tl::tma_load_3d(&S.R[0][0], &maps.r, ps.k0 - 2, y0, 0, bar);
        tl::tma_load_3d(&S.KX[0][0], &maps.kx, ps.k0, y0, 0, bar);
        tl::tma_load_3d(&S.KY[0][0], &maps.ky, ps.k0, y0, 0, bar);
        ++issued;
        if (++p_b == p_np) {
            p_sid += gridDim.x;
            p_b = 0;
            if (p_sid < nstrips) {
                const StripAt nx(g, gx, p_sid);
                p_np = w_stages(nx.j0, nx.j1);
            }
        }
    };

    unsigned q = 0;   // consumer: global stage index of this block's stream
    for (int sid = blockIdx.x; sid < nstrips; sid += gridDim.x) {
        const StripAt st(g, gx, sid);
        const int k = st.k0 + tx;
        const bool active = k < x - g.hd;
        const int kk = active ? k : x - g.hd - 1;   // lanes past the interior load valid cells, store nothing
        const bool at_l = kk == g.hd, at_r = kk == x - g.hd - 1;
        const bool edge_l = at_l || lane == 0, edge_r = at_r || lane == 31;
        const int ck = kk - st.k0;            // column of k in the kx / ky boxes
        const int cl = ck + 1, cc = ck + 2, cr = ck + 3;   // columns of k-1, k, k+1 in the p / r boxes
        // reflective halo cells of the new p this thread writes: below / above
        // the strip's first / last interior row, left / right of its column
        const bool hb = REFLECT && active && fc.b && st.j0 == g.hd;
        const bool ht = REFLECT && active && fc.t && st.j1 == g.y - g.hd;
        const bool hl = REFLECT && active && fc.l && k == g.hd;
        const bool hr = REFLECT && active && fc.r && k == x - g.hd - 1;
        if (u_halo && active) strip_u_halo(g, fc, uhd, u_halo, k, st.j0, st.j1);
        const int np = w_stages(st.j0, st.j1);
        double acc[1] = {0.0};
        // carried row values: pd (row below), pc (row c) with its left / right
        // neighbour candidates, kx at c and c+1, ky at c
        double pd = 0.0, pc = 0.0, lc = 0.0, rc = 0.0, kxc = 0.0, kxrc = 0.0, kyc = 0.0;
        long i = k + (long)st.j0 * x;
        for (int b = 0; b < np; ++b, ++q) {
            __syncthreads();   // every thread is past stage q-1: its slot is free
            if (tx == 0)
                while (p_sid < nstrips && issued < q + kStagesT) issue_next();
            tl::mbar_wait(&bars[q % kStagesT], (q / kStagesT) & 1u, err);
            const RowsT& S = ring[q % kStagesT];
#pragma unroll
            for (int u = 0; u < kRowsT; ++u) {
                const int jr = st.j0 - 1 + b * kRowsT + u;   // the row arriving from this stage
                if (jr > st.j1) break;
                // rows outside the interior keep p_in's values; interior rows are fused
                const bool halo_row = jr == g.hd - 1 || jr == g.y - g.hd;
                auto val = [&](int col, bool raw) -> double {
                    return (FUSE_P && !raw) ? bt * S.P[u][col] + S.R[u][col] : S.P[u][col];
                };
                const double fu = val(cc, halo_row);
                const double lu = edge_l ? val(cl, halo_row || at_l) : 0.0;
                const double ru = edge_r ? val(cr, halo_row || at_r) : 0.0;
                const double kxu = S.KX[u][ck];
                const double kxru = edge_r ? S.KX[u][ck + 1] : 0.0;
                const double kyu = S.KY[u][ck];
                if (jr == st.j0 - 1) {
                    pd = fu;
                } else if (jr == st.j0) {
                    pc = fu;
                    if (st.j0 == g.hd && REFLECT && fc.b) pd = pc;
                    lc = lu;
                    rc = ru;
                    kxc = kxu;
                    kxrc = kxru;
                    kyc = kyu;
                } else {
                    const int j = jr - 1;   // the row computed now
                    const double pu = (jr == g.y - g.hd && REFLECT && fc.t) ? pc : fu;
                    double pl = __shfl_up_sync(kFull, pc, 1);
                    double pr = __shfl_down_sync(kFull, pc, 1);
                    double kxr = __shfl_down_sync(kFull, kxc, 1);
                    if (at_l) pl = (REFLECT && fc.l) ? pc : lc;
                    else if (lane == 0) pl = lc;
                    if (at_r) pr = (REFLECT && fc.r) ? pc : rc;
                    else if (lane == 31) pr = rc;
                    if (edge_r) kxr = kxrc;
                    const double v = smvp(kxc, kxr, kyc, kyu, pc, pl, pr, pd, pu);
                    if (active) {
                        w[i] = v;
                        acc[0] += v * pc;
                        if (FUSE_P) p_out[i] = pc;
                        if (hb && j == st.j0) p_out[i - x] = pc;
                        if (ht && j == st.j1 - 1) p_out[i + x] = pc;
                        if (hl) p_out[i - 1] = pc;
                        if (hr) p_out[i + 1] = pc;
                    }
                    i += x;
                    pd = pc;
                    pc = pu;
                    lc = lu;
                    rc = ru;
                    kxc = kxu;
                    kxrc = kxru;
                    kyc = kyu;
                }
            }
        }
        strip_partial<1>(acc, rs, sid, red);
    }
    // every issued stage was waited for: no copy in flight
    if (TL2D_PDL_LATE) pdl_launch_next();
    strips_finish<1>(rs, nstrips, fin, red);
}

// ---------------------------------------------------------- u/r sweep ----
// Stage rows of the u/r update: kRowsU rows of u, p, r, w (BX columns from
// the strip's first column, 16-byte aligned for an even halo depth).
constexpr int kRowsU = 4;
constexpr int kStagesU = 3;
struct RowsU {
    alignas(128) double U[kRowsU][BX];
    alignas(128) double P[kRowsU][BX];
    alignas(128) double R[kRowsU][BX];
    alignas(128) double W[kRowsU][BX];
};
struct TmaUrMaps {
    CUtensorMap u, p, r, w;
};
constexpr size_t kTmaUrBytes = kStagesU * sizeof(RowsU) + kStagesU * 8 + 128;

__device__ __forceinline__ int ur_stages(int j0, int j1) { return (j1 - j0 + kRowsU - 1) / kRowsU; }

// CG sweep 2, persistent and TMA-fed (k_cg_ur_fused semantics):
//   u += alpha p ; r -= alpha w ; rrn = sum(r*r)   (cg.c:116-143)
template <typename Finish>
static __global__ void __launch_bounds__(BX, kStreamBlocksPerSm) k_cg_ur_stream(
    Geo g, Scalar alpha, const __grid_constant__ TmaUrMaps maps, double* __restrict__ u, double* __restrict__ r,
    ReduceSlots rs, const int* __restrict__ done, Finish fin, int* err)
{
    extern __shared__ __align__(128) unsigned char us_raw[];
    __shared__ double red[1][BX / tl::kWarp];
    unsigned char* base = us_raw + ((128 - (tl::smem_addr(us_raw) & 127)) & 127);
    RowsU* ring = reinterpret_cast<RowsU*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesU * sizeof(RowsU));
    const int tx = threadIdx.x;
    const int gx = strips_x(g), nstrips = strips_total(g);
    if (tx == 0) {
        for (int q = 0; q < kStagesU; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    pdl_wait();
    if (!TL2D_PDL_LATE) pdl_launch_next();
    if (gate_closed(done)) return;
    const double a = alpha.get();

    int p_sid = blockIdx.x, p_b = 0, p_np = 0;
    unsigned issued = 0;
    if (tx == 0 && p_sid < nstrips) {
        const StripAt ps(g, gx, p_sid);
        p_np = ur_stages(ps.j0, ps.j1);
    }
    auto issue_next = [&]() {
        const StripAt ps(g, gx, p_sid);
        const int slot = (int)(issued % kStagesU);
        RowsU& S = ring[slot];
        unsigned long long* bar = &bars[slot];
        const int y0 = ps.j0 + p_b * kRowsU;
        tl::mbar_expect_tx(bar, 4u * sizeof(double) * kRowsU * BX);
        tl::tma_load_3d(&S.U[0][0], &maps.u, ps.k0, y0, 0, bar);
        tl::tma_load_3d(&S.P[0][0], &maps.p, ps.k0, y0, 0, bar);
        tl::tma_load_3d(&S.R[0][0], &maps.r, ps.k0, y0, 0, bar);
        tl::tma_load_3d(&S.W[0][0], &maps.w, ps.k0, y0, 0, bar);
        ++issued;
        if (++p_b == p_np) {
            p_sid += gridDim.x;
            p_b = 0;
            if (p_sid < nstrips) {
                const StripAt nx(g, gx, p_sid);
                p_np = ur_stages(nx.j0, nx.j1);
            }
        }
    };

    unsigned q = 0;
    for (int sid = blockIdx.x; sid < nstrips; sid += gridDim.x) {
        const StripAt st(g, gx, sid);
        const int k = st.k0 + tx;
        const bool active = k < g.x - g.hd;
        const int np = ur_stages(st.j0, st.j1);
        double acc[1] = {0.0};
        long i = k + (long)st.j0 * g.x;
        for (int b = 0; b < np; ++b, ++q) {
            __syncthreads();   // every thread is past stage q-1: its slot is free
            if (tx == 0)
                while (p_sid < nstrips && issued < q + kStagesU) issue_next();
            tl::mbar_wait(&bars[q % kStagesU], (q / kStagesU) & 1u, err);
            const RowsU& S = ring[q % kStagesU];
#pragma unroll
            for (int t = 0; t < kRowsU; ++t) {
                const int j = st.j0 + b * kRowsU + t;
                if (j >= st.j1) break;
                if (active) {
                    u[i] = S.U[t][tx] + a * S.P[t][tx];
                    const double rn = S.R[t][tx] - a * S.W[t][tx];
                    r[i] = rn;
                    acc[0] += rn * rn;
                }
                i += g.x;
            }
        }
        strip_partial<1>(acc, rs, sid, red);
    }
    if (TL2D_PDL_LATE) pdl_launch_next();
    strips_finish<1>(rs, nstrips, fin, red);
}

}  // namespace tl2d
