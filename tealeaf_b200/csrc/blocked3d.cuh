// blocked3d.cuh -- temporally blocked Chebyshev trips and PPCG inner steps
// (3D, FP64, one chunk with six external faces).
//
// Between two norm evaluations a Chebyshev trip (3d/c_kernels/omp3/
// cheby_solver.c:62-99) and a PPCG inner step (ppcg_solver.c:29-73) are
// local 7-point updates with no global reduction, so L of them (L <= kTB3)
// run in one launch. A block owns an x-y region of kRX x kRY columns (the
// tile of kTX3 x kTY3 columns plus a kTB3-column margin) and a segment of
// kBZ3 z-planes, and streams up z as a wavefront: at step s the region's
// plane s is loaded (level 0), and level l (1 <= l <= L) advances plane
// s - l by one step, so every plane passes through all L steps while only a
// few planes per level are live. Each thread owns one column (x, y) and
// keeps, per level, the stencil field of the three planes around the one it
// advances in registers (the z-neighbours); x-neighbours come by warp shuffle
// (a warp is a region row) and y-neighbours through one shared-memory plane
// per level and plane parity. One barrier per step separates the steps.
// Each level's valid columns shrink by one per side and its valid planes by
// one at each end of the segment (the segment loads L planes beyond each
// end), so the tile's columns and the segment's planes are valid after L
// steps. The domain boundary is the depth-1 reflective halo applied on the
// fly (a neighbour outside the interior is the cell itself).
//
// Every cell goes through exactly the operations of the one-step kernels
// (k3_cheby_trip, k3_ppcg_step) in the same order, so the results are
// bit-identical. A norm the last step needs is not reduced here:
// k3_norm2_fin sums the stored residual with the one-step kernels'
// partition and order.
//
// Chebyshev (MODE 0), carried fields A = u, B = p, state (u_{n-1}, p_{n-1})
// with the add pending:   S = A + B ;  B = a_n B + b_n (u0 - A S) ;  A = S
// (or, with add_end, state (u_n, p_n): S = A for the first trip and the last
// trip's add applied on write-back, the order of run_cheby_solver_iterate)
// PPCG (MODE 1), A = sd, B = r, fold index pp:
//   S = pp == 0 ? B / theta : a_{pp-1} A + b_{pp-1} B ;  B -= A S ;  u += S ;  A = S
#pragma once

#include "kernels3d.cuh"

#include <type_traits>

namespace tl3d {

constexpr int kRX = 32;                  // region columns: one warp per region row
constexpr int kRY = 16;                  // region rows
constexpr int kB3Threads = kRX * kRY;    // 512
#ifndef TL3D_TB
#define TL3D_TB 2
#endif
constexpr int kTB3 = TL3D_TB;            // margin: the most steps one launch takes
constexpr int kTX3 = kRX - 2 * kTB3;     // tile columns
constexpr int kTY3 = kRY - 2 * kTB3;     // tile rows
#ifndef TL3D_BZ
#define TL3D_BZ 64
#endif
constexpr int kBZ3 = TL3D_BZ;            // output planes per block
static_assert(kTX3 > 0 && kTY3 > 0, "the margin must leave a tile");

struct Blocked3Args {
    int steps;            // L <= kTB3
    int first;            // Chebyshev: coefficient index of the first trip; PPCG: pp of the first step
    int wr_last;          // Chebyshev: write w and r of the last trip
    double theta;         // PPCG fold of pp == 0
    const double* alphas;
    const double* betas;
    int add_end = 0;      // Chebyshev: each trip ends with its u += p (the kernel-interface calls' order)
                          // instead of starting with the previous trip's
};

template <int MODE>
static __global__ void __launch_bounds__(kB3Threads, 1) k3_blocked(Geo g, Blocked3Args a,
                                                                   const double* __restrict__ A_in,
                                                                   const double* __restrict__ B_in, double* A_out,
                                                                   double* __restrict__ B_out,
                                                                   const double* __restrict__ u0,
                                                                   double* __restrict__ u, double* __restrict__ w,
                                                                   double* __restrict__ r,
                                                                   const double* __restrict__ kx,
                                                                   const double* __restrict__ ky,
                                                                   const double* __restrict__ kz,
                                                                   const int* __restrict__ done)
{
    __shared__ double sp[kTB3][2][kRY][kRX];   // level l's stencil field, plane parity, region
    if (gate_closed(done)) return;
    const int x = g.x, hd = g.hd;
    const long xy = g.xy();
    const int ilo = hd, ihi = g.x - hd, jlo = hd, jhi = g.y - hd, zlo = hd, zhi = g.z - hd;
    const int H = a.steps;
    const int cx = threadIdx.x, cy = threadIdx.y;
    const int gx = hd + blockIdx.x * kTX3 - kTB3 + cx;   // grid column and row of this thread
    const int gy = hd + blockIdx.y * kTY3 - kTB3 + cy;
    const bool colin = gx >= ilo && gx < ihi && gy >= jlo && gy < jhi;
    const int mx = max(max(kTB3 - cx, cx - (kTB3 + kTX3 - 1)), 0);
    const int my = max(max(kTB3 - cy, cy - (kTB3 + kTY3 - 1)), 0);
    const bool in_tile = colin && mx == 0 && my == 0;
    const bool at_l = gx == ilo, at_r = gx == ihi - 1, at_b = gy == jlo, at_t = gy == jhi - 1;
    const int Z0 = zlo + blockIdx.z * kBZ3, Z1 = min(Z0 + kBZ3, zhi);   // output planes [Z0, Z1)
    const long col = gx + (long)gy * x;   // index of (gx, gy) in plane 0 (used only when colin)

    // per level l < kTB3: stencil field of planes z-1, z, z+1 around the plane
    // level l + 1 advances next; B of that plane (bp) and of the newest (bn)
    double win[kTB3][3], bp[kTB3], bn[kTB3];
    double uacc[kTB3 + 1];   // PPCG: u of the tile plane at level l (plane s - l), its adds so far
#pragma unroll
    for (int l = 0; l < kTB3; ++l) {
        win[l][0] = win[l][1] = win[l][2] = 0.0;
        bp[l] = bn[l] = 0.0;
    }
#pragma unroll
    for (int q = 0; q <= kTB3; ++q) uacc[q] = 0.0;

    // the launch's coefficients: Chebyshev trip l (alphas / betas[first + l]);
    // PPCG fold of step l (pp = first + l: B / theta at pp == 0, else
    // alphas / betas[pp - 1])
    double ca[kTB3], cb[kTB3];
#pragma unroll
    for (int l = 0; l < kTB3; ++l) {
        ca[l] = cb[l] = 0.0;
        const int n = MODE == 0 ? a.first + l : a.first + l - 1;
        if (l < H && n >= 0) {
            ca[l] = a.alphas[n];
            cb[l] = a.betas[n];
        }
    }
    auto fold = [&](int l, double av, double bv) {
        if (a.first + l == 0) return bv / a.theta;
        return ca[l] * av + cb[l] * bv;
    };

    const int s_begin = max(Z0 - H, zlo);
    const int s_end = Z1 + H;   // steps s_begin .. s_end - 1 (level H reaches plane Z1 - 1 at s_end - 1)
    for (int s = s_begin; s < s_end; ++s) {
        // every global load of the step first, so that their latencies overlap:
        // plane s of A, B (and u) for level 0, the coefficients of plane s - l
        // for level l
        const bool act0 = s < min(Z1 + H, zhi);
        double av = 0.0, bv = 0.0, uv = 0.0;
        if (act0 && colin) {
            const long i = col + (long)s * xy;
            av = A_in[i];
            bv = B_in[i];
            if (MODE == 1 && in_tile && s >= Z0 && s < Z1) uv = u[i];
        }
        double kxc[kTB3], kyc[kTB3], kyu[kTB3], kzc[kTB3], kzf[kTB3], cc[kTB3];
        bool act[kTB3];
#pragma unroll
        for (int l = 1; l <= kTB3; ++l) {
            const int z = s - l;
            act[l - 1] = l <= H && z >= max(Z0 - H + l, zlo) && z < min(Z1 + H - l, zhi);
            kxc[l - 1] = kyc[l - 1] = kyu[l - 1] = kzc[l - 1] = kzf[l - 1] = cc[l - 1] = 0.0;
            if (act[l - 1] && colin) {
                const long i = col + (long)z * xy;
                kxc[l - 1] = kx[i];
                kyc[l - 1] = ky[i];
                kyu[l - 1] = ky[i + x];
                kzc[l - 1] = kz[i];
                kzf[l - 1] = kz[i + xy];
                if (MODE == 0) cc[l - 1] = u0[i];
            }
        }
        __syncthreads();   // the previous step's planes are written and read
        if (MODE == 1) {   // every plane in flight moves up one level
#pragma unroll
            for (int l = kTB3; l > 0; --l) uacc[l] = uacc[l - 1];
        }
        // level 0: plane s enters
        {
            const double sv = MODE == 0 ? (a.add_end ? av : av + bv) : fold(0, av, bv);
            if (MODE == 1) uacc[0] = uv + sv;
            win[0][0] = win[0][1];
            win[0][1] = win[0][2];
            win[0][2] = sv;
            bp[0] = bn[0];
            bn[0] = bv;
            if (act0) sp[0][s & 1][cy][cx] = sv;
        }
        // levels 1 .. H: level l advances plane s - l with the trip / step l - 1
#pragma unroll
        for (int l = 1; l <= kTB3; ++l) {
            if (l > H) break;
            const int z = s - l;
            if (!act[l - 1]) {
                if (l < H) {   // keep the window in step with the planes
                    win[l][0] = win[l][1];
                    win[l][1] = win[l][2];
                    win[l][2] = 0.0;
                    bp[l] = bn[l];
                    bn[l] = 0.0;
                }
                continue;
            }
            const double* W = win[l - 1];
            const double c = W[1];
            double lf = __shfl_up_sync(kFull3, c, 1);
            double rt = __shfl_down_sync(kFull3, c, 1);
            double dn = cy > 0 ? sp[l - 1][z & 1][cy - 1][cx] : 0.0;
            double up = cy < kRY - 1 ? sp[l - 1][z & 1][cy + 1][cx] : 0.0;
            double bk = W[0], fr = W[2];
            if (at_l) lf = c;
            if (at_r) rt = c;
            if (at_b) dn = c;
            if (at_t) up = c;
            if (z == zlo) bk = c;
            if (z == zhi - 1) fr = c;
            const long i = col + (long)z * xy;   // meaningful when colin
            double kxr = __shfl_down_sync(kFull3, kxc[l - 1], 1);
            if (at_r && colin) kxr = kx[i + 1];
            const double v = smvp(kxc[l - 1], kxr, kyc[l - 1], kyu[l - 1], kzc[l - 1], kzf[l - 1], c, lf, rt, dn,
                                  up, bk, fr);
            const double bz = bp[l - 1];   // B of plane z at level l - 1
            double bnew, snew = 0.0;
            if (MODE == 0) {
                const double res = cc[l - 1] - v;
                bnew = ca[l - 1] * bz + cb[l - 1] * res;
                if (l == H && a.wr_last && in_tile && z >= Z0 && z < Z1) {
                    w[i] = v;
                    r[i] = res;
                }
                if (l < H) snew = c + bnew;
            } else {
                bnew = bz - v;
                if (l < H) snew = fold(l, c, bnew);
                if (l < H) uacc[l] += snew;
            }
            if (l < H) {
                win[l][0] = win[l][1];
                win[l][1] = win[l][2];
                win[l][2] = snew;
                bp[l] = bn[l];
                bn[l] = bnew;
                sp[l][z & 1][cy][cx] = snew;
            } else if (in_tile && z >= Z0 && z < Z1) {
                // the tile's plane after H steps: A = S of step H - 1, B, the reflective halo of A
                A_out[i] = (MODE == 0 && a.add_end) ? c + bnew : c;   // halo: u before the last add
                B_out[i] = bnew;
                if (MODE == 1) u[i] = uacc[l];
                if (at_l) A_out[i - 1] = c;
                if (at_r) A_out[i + 1] = c;
                if (at_b) A_out[i - x] = c;
                if (at_t) A_out[i + x] = c;
                if (z == zlo) A_out[i - xy] = c;
                if (z == zhi - 1) A_out[i + xy] = c;
            }
        }
    }
}

// ------------------------------------------------------ TMA-staged form --
// The same wavefront with the region planes brought in by TMA and two region
// rows per thread: a block of 32 x 12 threads owns a 32 x 24-column region (a
// 28 x 20 tile plus the kTB3 margin), thread row t holding rows 2t and 2t+1,
// whose y-neighbour within the pair comes from registers. One thread issues
// the six kRX x kRYT boxes of plane p (A, B, C = u0 or u, kx, ky, kz; from
// grid column hd + bx kTX3 - kTB3, row hd + by kTYT3 - kTB3) into a ring of
// kRing3 planes on one shared-memory barrier per slot, kPf3 planes ahead of
// the plane that enters, so the steps read every operand from shared memory.
// Boxes start on a 16-byte boundary when the halo depth, the margin and the
// row length are even; cells outside the array read as zero, and, as in
// k3_blocked, only cells inside the interior and the margin are used. The
// ring also stages the plane after the last interior one for its kz (the
// front face coefficient of the last plane). The launch's step count is a
// template parameter (HS = a.steps), so the level loop is straight-line
// code. Every wait is bounded (err); every issued plane is waited for.
constexpr int kTYT = 12;                  // thread rows of the staged kernel
constexpr int kRYT = 2 * kTYT;            // region rows: two per thread
constexpr int kTYT3 = kRYT - 2 * kTB3;    // tile rows
constexpr int kB3TThreads = kRX * kTYT;   // 384
constexpr int kPf3 = 2;                   // planes issued ahead
constexpr int kRing3 = kTB3 + 1 + kPf3;   // planes s - kTB3 .. s + kPf3
struct Region3 {
    alignas(128) double f[6][kRYT][kRX];   // A, B, C, kx, ky, kz
};
static_assert(sizeof(Region3) % 128 == 0, "ring slots start on 128-byte boundaries");
struct Blocked3Maps {
    CUtensorMap a, b, c, kx, ky, kz;
};
constexpr size_t kBlocked3TmaBytes = kRing3 * sizeof(Region3) + kRing3 * 8 + 128;

template <int MODE, int HS>
static __global__ void __launch_bounds__(kB3TThreads, 1) k3_blocked_tma(Geo g, Blocked3Args a,
                                                                        const __grid_constant__ Blocked3Maps maps,
                                                                        double* A_out, double* __restrict__ B_out,
                                                                        double* __restrict__ u,
                                                                        double* __restrict__ w,
                                                                        double* __restrict__ r,
                                                                        const int* __restrict__ done, int* err)
{
    __shared__ double sp[kTB3][2][kRYT][kRX];   // level l's stencil field, plane parity, region
    extern __shared__ __align__(128) unsigned char b3_raw[];
    if (gate_closed(done)) return;
    unsigned char* base = b3_raw + ((128 - (tl::smem_addr(b3_raw) & 127)) & 127);
    Region3* ring = reinterpret_cast<Region3*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kRing3 * sizeof(Region3));
    const int x = g.x, hd = g.hd;
    const long xy = g.xy();
    const int ilo = hd, ihi = g.x - hd, jlo = hd, jhi = g.y - hd, zlo = hd, zhi = g.z - hd;
    constexpr int H = HS;   // steps of this launch (a.steps)
    const int cx = threadIdx.x, ty = threadIdx.y;
    const bool leader = cx == 0 && ty == 0;
    const int xs = hd + blockIdx.x * kTX3 - kTB3, ys = hd + blockIdx.y * kTYT3 - kTB3;   // region origin
    const int gx = xs + cx;
    const int mx = max(max(kTB3 - cx, cx - (kTB3 + kTX3 - 1)), 0);
    const bool at_l = gx == ilo, at_r = gx == ihi - 1;
    bool colin[2], in_tile[2], at_b[2], at_t[2];
    long col[2];
#pragma unroll
    for (int k = 0; k < 2; ++k) {
        const int ry = 2 * ty + k, gy = ys + ry;
        const int my = max(max(kTB3 - ry, ry - (kTB3 + kTYT3 - 1)), 0);
        colin[k] = gx >= ilo && gx < ihi && gy >= jlo && gy < jhi;
        in_tile[k] = colin[k] && mx == 0 && my == 0;
        at_b[k] = gy == jlo;
        at_t[k] = gy == jhi - 1;
        col[k] = gx + (long)gy * x;
    }
    const int Z0 = zlo + blockIdx.z * kBZ3, Z1 = min(Z0 + kBZ3, zhi);

    // per level l < kTB3 and row k: stencil field of the three planes around
    // the plane level l + 1 advances next; B of that plane (bp) and the newest (bn)
    double win[kTB3][3][2], bp[kTB3][2], bn[kTB3][2];
    double uacc[kTB3 + 1][2];   // PPCG: u of the tile plane at level l (plane s - l), its adds so far
#pragma unroll
    for (int l = 0; l < kTB3; ++l)
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            win[l][0][k] = win[l][1][k] = win[l][2][k] = 0.0;
            bp[l][k] = bn[l][k] = 0.0;
        }
#pragma unroll
    for (int q = 0; q <= kTB3; ++q) uacc[q][0] = uacc[q][1] = 0.0;
    double ca[kTB3], cb[kTB3];
#pragma unroll
    for (int l = 0; l < kTB3; ++l) {
        ca[l] = cb[l] = 0.0;
        const int n = MODE == 0 ? a.first + l : a.first + l - 1;
        if (l < H && n >= 0) {
            ca[l] = a.alphas[n];
            cb[l] = a.betas[n];
        }
    }
    auto fold = [&](int l, double av, double bv) {
        if (a.first + l == 0) return bv / a.theta;
        return ca[l] * av + cb[l] * bv;
    };

    const int s_begin = max(Z0 - H, zlo);
    const int s_end = Z1 + H;
    const int load_end = min(Z1 + H, zhi + 1);   // planes staged: s_begin .. load_end - 1
    auto issue = [&](int p) {
        const int q = (p - s_begin) % kRing3;
        Region3& R = ring[q];
        unsigned long long* bar = &bars[q];
        tl::mbar_expect_tx(bar, (unsigned)sizeof(Region3));
        tl::tma_load_3d(&R.f[0][0][0], &maps.a, xs, ys, p, bar);
        tl::tma_load_3d(&R.f[1][0][0], &maps.b, xs, ys, p, bar);
        tl::tma_load_3d(&R.f[2][0][0], &maps.c, xs, ys, p, bar);
        tl::tma_load_3d(&R.f[3][0][0], &maps.kx, xs, ys, p, bar);
        tl::tma_load_3d(&R.f[4][0][0], &maps.ky, xs, ys, p, bar);
        tl::tma_load_3d(&R.f[5][0][0], &maps.kz, xs, ys, p, bar);
    };
    if (leader) {
        for (int q = 0; q < kRing3; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (leader)
        for (int p = s_begin; p < s_begin + kPf3 && p < load_end; ++p) issue(p);

    // does the region reach a domain face in x or y (then neighbours there are reflected)?
    const bool touches = xs <= ilo || xs + kRX > ihi - 1 || ys <= jlo || ys + kRYT > jhi - 1;
    int qs = 0;          // ring slot of plane s
    unsigned ph = 0;     // barrier phase of that slot's current use
    for (int s = s_begin; s < s_end; ++s) {
        if (s < load_end) tl::mbar_wait(&bars[qs], ph, err);
        __syncthreads();   // the previous step's planes are read: the slot of plane s - kTB3 - 1 is free
        if (leader && s + kPf3 < load_end) issue(s + kPf3);
        if (MODE == 1) {   // every plane in flight moves up one level
#pragma unroll
            for (int l = kTB3; l > 0; --l) {
                uacc[l][0] = uacc[l - 1][0];
                uacc[l][1] = uacc[l - 1][1];
            }
        }
        // level 0: plane s enters
        {
            const bool act0 = s < min(Z1 + H, zhi);
            const Region3& R = ring[qs];
#pragma unroll
            for (int k = 0; k < 2; ++k) {
                const int ry = 2 * ty + k;
                double av = 0.0, bv = 0.0, uv = 0.0;
                if (act0 && colin[k]) {
                    av = R.f[0][ry][cx];
                    bv = R.f[1][ry][cx];
                    if (MODE == 1 && in_tile[k] && s >= Z0 && s < Z1) uv = R.f[2][ry][cx];
                }
                const double sv = MODE == 0 ? (a.add_end ? av : av + bv) : fold(0, av, bv);
                if (MODE == 1) uacc[0][k] = uv + sv;
                win[0][0][k] = win[0][1][k];
                win[0][1][k] = win[0][2][k];
                win[0][2][k] = sv;
                bp[0][k] = bn[0][k];
                bn[0][k] = bv;
                if (act0) sp[0][s & 1][ry][cx] = sv;
            }
        }
        auto levels = [&](auto reflect) {
            constexpr bool REFLECT = decltype(reflect)::value;
#pragma unroll
            for (int l = 1; l <= kTB3; ++l) {
                if (l > H) break;
                const int z = s - l;
                const bool act = z >= max(Z0 - H + l, zlo) && z < min(Z1 + H - l, zhi);
                if (!act) {
                    if (l < H) {
#pragma unroll
                        for (int k = 0; k < 2; ++k) {
                            win[l][0][k] = win[l][1][k];
                            win[l][1][k] = win[l][2][k];
                            win[l][2][k] = 0.0;
                            bp[l][k] = bn[l][k];
                            bn[l][k] = 0.0;
                        }
                    }
                    continue;
                }
                const int qz = qs - l < 0 ? qs - l + kRing3 : qs - l;              // slot of plane z
                const int qf = qs - l + 1 < 0 ? qs - l + 1 + kRing3 : qs - l + 1;  // slot of plane z + 1
                const Region3& R = ring[qz];
                const Region3& F = ring[qf];
                const double c0 = win[l - 1][1][0], c1 = win[l - 1][1][1];
                double snew[2];
#pragma unroll
                for (int k = 0; k < 2; ++k) {
                    const int ry = 2 * ty + k;
                    const double c = k == 0 ? c0 : c1;
                    double lf = __shfl_up_sync(kFull3, c, 1);
                    double rt = __shfl_down_sync(kFull3, c, 1);
                    double dn = k == 1 ? c0 : (ry > 0 ? sp[l - 1][z & 1][ry - 1][cx] : 0.0);
                    double up = k == 0 ? c1 : (ry < kRYT - 1 ? sp[l - 1][z & 1][ry + 1][cx] : 0.0);
                    double bk = win[l - 1][0][k], fr = win[l - 1][2][k];
                    if (REFLECT) {
                        if (at_l) lf = c;
                        if (at_r) rt = c;
                        if (at_b[k]) dn = c;
                        if (at_t[k]) up = c;
                    }
                    if (z == zlo) bk = c;
                    if (z == zhi - 1) fr = c;
                    const double kxc = R.f[3][ry][cx];
                    const double kxr = cx + 1 < kRX ? R.f[3][ry][cx + 1] : 0.0;
                    const double kyc = R.f[4][ry][cx];
                    const double kyu = ry + 1 < kRYT ? R.f[4][ry + 1][cx] : 0.0;
                    const double kzc = R.f[5][ry][cx];
                    const double kzf = F.f[5][ry][cx];
                    const double cc = MODE == 0 ? R.f[2][ry][cx] : 0.0;
                    const double v = smvp(kxc, kxr, kyc, kyu, kzc, kzf, c, lf, rt, dn, up, bk, fr);
                    const double bz = bp[l - 1][k];
                    const long i = col[k] + (long)z * xy;
                    double bnew;
                    snew[k] = 0.0;
                    if (MODE == 0) {
                        const double res = cc - v;
                        bnew = ca[l - 1] * bz + cb[l - 1] * res;
                        if (l == H && a.wr_last && in_tile[k] && z >= Z0 && z < Z1) {
                            w[i] = v;
                            r[i] = res;
                        }
                        if (l < H) snew[k] = c + bnew;
                    } else {
                        bnew = bz - v;
                        if (l < H) snew[k] = fold(l, c, bnew);
                        if (l < H) uacc[l][k] += snew[k];
                    }
                    if (l < H) {
                        bp[l][k] = bn[l][k];
                        bn[l][k] = bnew;
                        sp[l][z & 1][ry][cx] = snew[k];
                    } else if (in_tile[k] && z >= Z0 && z < Z1) {
                        A_out[i] = (MODE == 0 && a.add_end) ? c + bnew : c;   // halo: u before the last add
                        B_out[i] = bnew;
                        if (MODE == 1) u[i] = uacc[l][k];
                        if (REFLECT) {
                            if (at_l) A_out[i - 1] = c;
                            if (at_r) A_out[i + 1] = c;
                            if (at_b[k]) A_out[i - x] = c;
                            if (at_t[k]) A_out[i + x] = c;
                        }
                        if (z == zlo) A_out[i - xy] = c;
                        if (z == zhi - 1) A_out[i + xy] = c;
                    }
                }
                if (l < H) {   // the window moves after both rows used level l - 1's planes
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        win[l][0][k] = win[l][1][k];
                        win[l][1][k] = win[l][2][k];
                        win[l][2][k] = snew[k];
                    }
                }
            }
        };
        if (touches) levels(std::true_type());
        else levels(std::false_type());
        if (++qs == kRing3) {
            qs = 0;
            ph ^= 1u;
        }
    }
    // every issued plane was waited for (planes s_begin .. load_end - 1 at their steps)
}

inline dim3 blocked3_tma_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, kTX3), tl::ceil_div(g.y - 2 * g.hd, kTYT3),
                tl::ceil_div(g.z - 2 * g.hd, kBZ3));
}

// sum(b^2) over the interior with the partition and order of the one-step
// fused sweeps (k3_cheby_trip, k3_ppcg_step: grid gh, the halo-duty z-plane
// of blocks adding nothing), then `fin`; skipped once the loop has ended.
template <typename Finish>
static __global__ void __launch_bounds__(NT) k3_norm2_fin(Geo g, const double* __restrict__ b, ReduceSlots rs,
                                                         const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    if (blockIdx.z + 1 < gridDim.z) {
        const PencilC s(g);
        if (s.active) {
            const long xy = g.xy();
            long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
            for (int ii = s.i0; ii < s.i1; ++ii, i += xy) acc[0] += b[i] * b[i];
        }
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count(), fin);
}

// `fin` alone (a block of trips without a norm); skipped once the loop has ended.
template <typename Finish>
static __global__ void k3_finish_only(const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done) || threadIdx.x != 0) return;
    const double t[1] = {0.0};
    fin(t);
}

inline dim3 blocked3_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, kTX3), tl::ceil_div(g.y - 2 * g.hd, kTY3),
                tl::ceil_div(g.z - 2 * g.hd, kBZ3));
}

}  // namespace tl3d
