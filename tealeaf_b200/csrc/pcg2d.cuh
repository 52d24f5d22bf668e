// pcg2d.cuh -- Jacobi-preconditioned CG sweeps (2D, FP64).
//
// The reference documents a `tl_preconditioner_type` with a diagonal Jacobi
// (jac_diag) and a block Jacobi of block size 4 (jac_block) (README.md:127-133);
// its C kernel suites parse `preconditioner_on` and ignore it, and its cuda 3D
// kernel forms only the diagonal one at initialisation (mi = 1 / diag(A),
// z = mi r; 3d/c_kernels/cuda/cg_solver.cuknl:93-100). Here both are
// complete preconditioned CGs of the device-resident driver:
//
//   init:  z = M^-1 r, p = z (with its depth-1 reflective halo), rro = r.z
//   trip:  [p = beta p + z] w = A p, pw = p.w   (the CG w sweep, z folded)
//          alpha = rro / pw, u += alpha p, r -= alpha w, z = M^-1 r,
//          r.r (the stop test) and r.z;  beta = r.z / rro, rro = r.z
//
// M: jac_diag the diagonal of A, 1 + (kx_i+1 + kx_i) + (ky_i+x + ky_i);
// jac_block the tridiagonal part of A inside blocks of 4 rows along y that
// start at the first interior row (couplings -ky between vertical neighbours;
// the last block of a column may be shorter), solved per column by Thomas'
// algorithm. M is factored once per solve into the chunk's mi field (which
// the reference allocates for its preconditioner and whose cuda kernel holds
// 1 / diag(A) there): jac_diag mi = 1 / diag(A), jac_block the inverse pivots
// g_q = 1 / (d_q + ky_q c_q-1), c_q = -ky_q+1 g_q. Applying M^-1 then takes
// multiplications only (jac_block: y_q = (r_q + ky_q y_q-1) g_q forward,
// z_q = y_q - c_q z_q+1 back). z is an internal buffer of the suite.
//
// Algorithmic bytes per cell and iteration: the w sweep 48 (z, p_old, kx, ky
// -> p, w), the u/r/z sweep 64 for jac_diag (u, p, r, w, mi -> u, r, z) and
// 72 for jac_block (+ ky): 112 / 120 against plain CG's 96. The element-wise
// operations follow the oracle's restatement (oracle/tl_oracle.c,
// o2_precond_factor, o2_precond) in order, so z is bit-identical to it.
#pragma once

#include "kernels2d.cuh"

namespace tl2d {

enum { kPrecondNone = 0, kPrecondDiag = 1, kPrecondBlock = 2 };

// Factor of the column block at i0 = k + jb x (rows jb .. jb+m-1, m <= BS)
// into mi: jac_diag 1 / diag(A), jac_block the inverse pivots.
template <int BS>
__device__ __forceinline__ void precond_factor(const double* __restrict__ kx, const double* __restrict__ ky,
                                               double* __restrict__ mi, long i0, int x, int m)
{
    double c = 0.0;
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        if (q < m) {
            const long i = i0 + (long)q * x;
            const double d = 1.0 + (kx[i + 1] + kx[i]) + (ky[i + x] + ky[i]);
            const double g = q == 0 ? 1.0 / d : 1.0 / (d + ky[i] * c);
            mi[i] = g;
            c = -ky[i + x] * g;
        }
    }
}

// z = M^-1 r for the column block at i0 (rows jb .. jb+m-1), rv its residual.
template <int BS>
__device__ __forceinline__ void precond_apply(const double* __restrict__ ky, const double* __restrict__ mi, long i0,
                                              int x, int m, const double (&rv)[BS], double (&zv)[BS])
{
    if (BS == 1) {
        zv[0] = mi[i0] * rv[0];
        return;
    }
    double g[BS], kyn[BS], yv[BS];
    double kyc = ky[i0];
#pragma unroll
    for (int q = 0; q < BS; ++q) {
        if (q < m) {
            const long i = i0 + (long)q * x;
            g[q] = mi[i];
            kyn[q] = ky[i + x];
            yv[q] = q == 0 ? rv[0] * g[0] : (rv[q] + kyc * yv[q - 1]) * g[q];
            kyc = kyn[q];
        }
    }
    double zn = 0.0;
#pragma unroll
    for (int q = BS - 1; q >= 0; --q) {
        if (q < m) {
            if (q == m - 1) {
                zn = yv[q];
            } else {
                const double c = -kyn[q] * g[q];
                zn = yv[q] - c * zn;
            }
            zv[q] = zn;
        }
    }
}

// PCG start after cg_init: the factor of M into mi, z = M^-1 r, p = z with
// its depth-1 reflective halo, sum(r z) -> fin. Strips of g.rows rows (a
// multiple of BS).
template <int BS, typename Finish>
static __global__ void __launch_bounds__(BX) k_pcg_init(Geo g, Faces fc, const double* __restrict__ r,
                                                       const double* __restrict__ kx, const double* __restrict__ ky,
                                                       double* __restrict__ mi, double* __restrict__ z,
                                                       double* __restrict__ p, ReduceSlots rs, Finish fin)
{
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        const int x = g.x;
        for (int jb = s.j0; jb < s.j1; jb += BS) {
            const int m = min(BS, s.j1 - jb);
            const long i0 = s.k + (long)jb * x;
            double rv[BS], zv[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) rv[q] = q < m ? r[i0 + (long)q * x] : 0.0;
            precond_factor<BS>(kx, ky, mi, i0, x, m);
            precond_apply<BS>(ky, mi, i0, x, m, rv, zv);
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                if (q < m) {
                    const long i = i0 + (long)q * x;
                    z[i] = zv[q];
                    p[i] = zv[q];
                    reflect_store(p, g, fc, 1, s.k, jb + q, zv[q]);
                    acc[0] += rv[q] * zv[q];
                }
            }
        }
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// PCG sweep 2: u += alpha p ; r -= alpha w ; z = M^-1 r ; sums r.r, r.z -> fin.
template <int BS, typename Finish>
static __global__ void __launch_bounds__(BX) k_pcg_ur(Geo g, Scalar alpha, double* __restrict__ u,
                                                     const double* __restrict__ p, double* __restrict__ r,
                                                     const double* __restrict__ w, const double* __restrict__ ky,
                                                     const double* __restrict__ mi, double* __restrict__ z,
                                                     ReduceSlots rs, const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    Strip s(g);
    double acc[2] = {0.0, 0.0};
    if (s.active) {
        const double a = alpha.get();
        const int x = g.x;
        for (int jb = s.j0; jb < s.j1; jb += BS) {
            const int m = min(BS, s.j1 - jb);
            const long i0 = s.k + (long)jb * x;
            double rv[BS], zv[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                rv[q] = 0.0;
                if (q < m) {
                    const long i = i0 + (long)q * x;
                    u[i] += a * p[i];
                    const double rn = r[i] - a * w[i];
                    r[i] = rn;
                    rv[q] = rn;
                    acc[0] += rn * rn;
                }
            }
            precond_apply<BS>(ky, mi, i0, x, m, rv, zv);
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                if (q < m) {
                    z[i0 + (long)q * x] = zv[q];
                    acc[1] += rv[q] * zv[q];
                }
            }
        }
    }
    tl::grid_sum<2, BX>(acc, rs, block_id(), block_count(), fin);
}

// k_pcg_ur with its operands brought in by TMA: stages of kPcgRows = 4 rows
// (one jac_block block, four jac_diag ones) of the strip's u, p, r, w, mi and,
// for jac_block, ky (BX-column boxes from the strip's first column, 16-byte
// aligned for an even halo depth), in a 3-stage ring on shared-memory
// barriers; every wait bounded (err). The same strips, rows, order and
// arithmetic as k_pcg_ur: the same results, partial sums included.
constexpr int kPcgRows = 4;
constexpr int kPcgStages = 3;
struct PcgRows {
    alignas(128) double U[kPcgRows][BX];
    alignas(128) double P[kPcgRows][BX];
    alignas(128) double R[kPcgRows][BX];
    alignas(128) double W[kPcgRows][BX];
    alignas(128) double MI[kPcgRows][BX];
    alignas(128) double KY[kPcgRows][BX];
};
struct PcgMaps {
    CUtensorMap u, p, r, w, mi, ky;
};
constexpr size_t kPcgTmaBytes = kPcgStages * sizeof(PcgRows) + kPcgStages * 8 + 128;

template <int BS, typename Finish>
static __global__ void __launch_bounds__(BX, 3) k_pcg_ur_tma(Geo g, Scalar alpha, const __grid_constant__ PcgMaps maps,
                                                            double* __restrict__ u, double* __restrict__ r,
                                                            double* __restrict__ z, ReduceSlots rs,
                                                            const int* __restrict__ done, Finish fin, int* err)
{
    static_assert(kPcgRows % BS == 0, "a stage holds whole preconditioner blocks");
    extern __shared__ __align__(128) unsigned char tp_raw[];
    if (gate_closed(done)) return;
    unsigned char* base = tp_raw + ((128 - (tl::smem_addr(tp_raw) & 127)) & 127);
    PcgRows* ring = reinterpret_cast<PcgRows*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kPcgStages * sizeof(PcgRows));
    Strip s(g);
    double acc[2] = {0.0, 0.0};
    const int tx = threadIdx.x;
    const int k0 = g.hd + blockIdx.x * BX;
    const int np = (s.j1 - s.j0 + kPcgRows - 1) / kPcgRows;
    auto issue = [&](int b) {
        PcgRows& S = ring[b % kPcgStages];
        unsigned long long* bar = &bars[b % kPcgStages];
        const int y0 = s.j0 + b * kPcgRows;
        tl::mbar_expect_tx(bar, (BS > 1 ? 6u : 5u) * sizeof(double) * kPcgRows * BX);
        tl::tma_load_3d(&S.U[0][0], &maps.u, k0, y0, 0, bar);
        tl::tma_load_3d(&S.P[0][0], &maps.p, k0, y0, 0, bar);
        tl::tma_load_3d(&S.R[0][0], &maps.r, k0, y0, 0, bar);
        tl::tma_load_3d(&S.W[0][0], &maps.w, k0, y0, 0, bar);
        tl::tma_load_3d(&S.MI[0][0], &maps.mi, k0, y0, 0, bar);
        if (BS > 1) tl::tma_load_3d(&S.KY[0][0], &maps.ky, k0, y0, 0, bar);
    };
    if (tx == 0) {
        for (int q = 0; q < kPcgStages; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (tx == 0)
        for (int b = 0; b < kPcgStages - 1 && b < np; ++b) issue(b);
    const double a = alpha.get();
    const int x = g.x;
    for (int b = 0; b < np; ++b) {
        __syncthreads();   // every thread is past stage b-1: its slot is free
        if (tx == 0 && b + kPcgStages - 1 < np) issue(b + kPcgStages - 1);
        tl::mbar_wait(&bars[b % kPcgStages], (unsigned)(b / kPcgStages) & 1u, err);
        const PcgRows& S = ring[b % kPcgStages];
#pragma unroll
        for (int q0 = 0; q0 < kPcgRows; q0 += BS) {
            const int jb = s.j0 + b * kPcgRows + q0;
            if (jb >= s.j1) break;
            const int m = min(BS, s.j1 - jb);
            const long i0 = s.k + (long)jb * x;
            double rv[BS], zv[BS];
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                rv[q] = 0.0;
                if (q < m && s.active) {
                    u[i0 + (long)q * x] = S.U[q0 + q][tx] + a * S.P[q0 + q][tx];
                    const double rn = S.R[q0 + q][tx] - a * S.W[q0 + q][tx];
                    r[i0 + (long)q * x] = rn;
                    rv[q] = rn;
                    acc[0] += rn * rn;
                }
            }
            if (BS == 1) {
                zv[0] = S.MI[q0][tx] * rv[0];
            } else {
                // precond_apply's recurrences on the staged rows (ky of row q+1 is in the block)
                double yv[BS];
#pragma unroll
                for (int q = 0; q < BS; ++q)
                    if (q < m) yv[q] = q == 0 ? rv[0] * S.MI[q0][tx] : (rv[q] + S.KY[q0 + q][tx] * yv[q - 1]) * S.MI[q0 + q][tx];
                double zn = 0.0;
#pragma unroll
                for (int q = BS - 1; q >= 0; --q) {
                    if (q < m) {
                        if (q == m - 1) {
                            zn = yv[q];
                        } else {
                            const double c = -S.KY[q0 + q + 1][tx] * S.MI[q0 + q][tx];
                            zn = yv[q] - c * zn;
                        }
                        zv[q] = zn;
                    }
                }
            }
#pragma unroll
            for (int q = 0; q < BS; ++q) {
                if (q < m && s.active) {
                    z[i0 + (long)q * x] = zv[q];
                    acc[1] += rv[q] * zv[q];
                }
            }
        }
    }
    // every issued stage was waited for: no copy in flight
    tl::grid_sum<2, BX>(acc, rs, block_id(), block_count(), fin);
}

}  // namespace tl2d
