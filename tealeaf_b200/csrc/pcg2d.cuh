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

}  // namespace tl2d
