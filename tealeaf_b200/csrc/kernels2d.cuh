// kernels2d.cuh -- device kernels of the 2D suite (included by suite2d.cu
// and driver2d.cu; every kernel has internal linkage in each includer).
//
// Kernel shapes: interior sweeps run one thread per column (BX = 128 columns
// per block, one warp = 256 contiguous bytes per load) and walk Geo::rows
// rows (4-32, chosen per mesh so the grid fills the SMs) down the column,
// carrying the vertical neighbours of the stencil in registers,
// so each field is read from DRAM once per sweep. Reductions are fused into
// the sweep that produces their operands and finished by one last-block pass
// (common.cuh).
//
// Floating point: includers are compiled with -fmad=false so each + - * / is
// one IEEE operation in the reference's expression order.
#pragma once

#include "common.cuh"
#include "solver_common.cuh"
#include "tma.cuh"
#include "tealeaf_b200_2d.h"
using tl::ReduceSlots;

// Types have external linkage (identical in every includer); kernels are
// static, so each includer has its own copies.
namespace tl2d {

using tl::ChebyCoef;
using tl::DevParams;
using tl::DevState;
using tl::FinCgInit;
using tl::FinCgUr;
using tl::FinCgW;
using tl::FinPcgUr;
using tl::FinChebyBlock;
using tl::FinChebyTrip;
using tl::FinPpcgNorm;
using tl::FinPpcgW;
using tl::gate_closed;
using tl::PpcgCoef;
using tl::Scalar;

// Tuning of the fused sweeps: rows unrolled per thread and the minimum blocks
// per SM the register allocation must allow (__launch_bounds__).
#ifndef TL2D_UNROLL
#define TL2D_UNROLL 4
#endif
#ifndef TL2D_MINB
#define TL2D_MINB 16
#endif
#define TL2D_STR(x) #x
#define TL2D_PRAGMA_UNROLL(n) _Pragma(TL2D_STR(unroll n))

constexpr int BX = 128;   // threads (columns) per block of an interior sweep
constexpr int ROWS = 8;   // default rows per thread of an interior sweep (Geo::rows)
constexpr int FB = 256;   // threads per block of full-array kernels

struct Geo {
    int x, y, hd;
    int rows = ROWS;   // rows per thread of every interior sweep (chosen per chunk)
};

// ----------------------------------------------------------------- kernels

__device__ __forceinline__ double coef_w(int coefficient, double density)
{
    return coefficient == TL_CONDUCTIVITY ? density : 1.0 / density;
}

__device__ __forceinline__ double face(double r, double wa, double wb)
{
    return r * (wa + wb) / (2.0 * wa * wb);
}

// 5-point operator in the reference operand order (2d/shared.h:49-54):
// c = centre, l/r = x-1/x+1, d/u = y-1/y+1; kxc = kx[i], kxr = kx[i+1],
// kyc = ky[i], kyu = ky[i+x].
__device__ __forceinline__ double smvp(double kxc, double kxr, double kyc, double kyu,
                                       double c, double l, double r, double d, double u)
{
    return (1.0 + (kxr + kxc) + (kyu + kyc)) * c - (kxr * r + kxc * l) - (kyu * u + kyc * d);
}

__device__ __forceinline__ int block_id() { return blockIdx.x + blockIdx.y * gridDim.x; }
__device__ __forceinline__ int block_count() { return gridDim.x * gridDim.y; }

// Column-strip coordinates of an interior sweep.
struct Strip {
    int k, j0, j1;
    bool active;
    __device__ Strip(const Geo& g) : Strip(g, blockIdx.x, blockIdx.y) {}
    __device__ Strip(const Geo& g, int bx, int by)
    {
        k = g.hd + bx * BX + threadIdx.x;
        j0 = g.hd + by * g.rows;
        j1 = min(j0 + g.rows, g.y - g.hd);
        active = k < g.x - g.hd;
    }
};

// The CG u/r sweep walks the strips in the reverse of the w sweep's order
// (last strip first, each strip from its last row up), so that it starts on
// the rows the w sweep touched last, still in L2, and ends on the rows the
// next w sweep starts on. Each strip's partial sum keeps its slot, so the
// reduction order over strips is unchanged. 0: forward order.
#ifndef TL2D_UR_REVERSE
#define TL2D_UR_REVERSE 1
#endif
__device__ __forceinline__ int ur_bx() { return TL2D_UR_REVERSE ? gridDim.x - 1 - blockIdx.x : blockIdx.x; }
__device__ __forceinline__ int ur_by() { return TL2D_UR_REVERSE ? gridDim.y - 1 - blockIdx.y : blockIdx.y; }

// w = A p and pw = sum(w*p)   (cg.c:88-113)
static __global__ void __launch_bounds__(BX) k_cg_calc_w(Geo g, const double* __restrict__ p, double* __restrict__ w,
                                                  const double* __restrict__ kx, const double* __restrict__ ky,
                                                  ReduceSlots rs)
{
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        const int x = g.x;
        long i = s.k + (long)s.j0 * x;
        double pd = p[i - x], pc = p[i], kyc = ky[i];
#pragma unroll 4
        for (int j = s.j0; j < s.j1; ++j, i += x) {
            const double pu = p[i + x], kyu = ky[i + x];
            const double v = smvp(kx[i], kx[i + 1], kyc, kyu, pc, p[i - 1], p[i + 1], pd, pu);
            w[i] = v;
            acc[0] += v * pc;
            pd = pc;
            pc = pu;
            kyc = kyu;
        }
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count());
}

// u += alpha p; r -= alpha w; rrn = sum(r*r)   (cg.c:116-143)
static __global__ void __launch_bounds__(BX) k_cg_calc_ur(Geo g, double alpha, double* __restrict__ u,
                                                   const double* __restrict__ p, double* __restrict__ r,
                                                   const double* __restrict__ w, ReduceSlots rs)
{
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
        for (int j = s.j0; j < s.j1; ++j, i += g.x) {
            u[i] += alpha * p[i];
            const double rn = r[i] - alpha * w[i];
            r[i] = rn;
            acc[0] += rn * rn;
        }
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count());
}

// p = beta p + r   (cg.c:146-164)
static __global__ void __launch_bounds__(BX) k_cg_calc_p(Geo g, double beta, double* __restrict__ p,
                                                  const double* __restrict__ r)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) p[i] = beta * p[i] + r[i];
}

// Chebyshev sweep (cheby.c:26-85): w = A u; r = u0 - w;
// p = r/theta (INIT) or alpha p + beta r. u itself is updated by k_add_p.
template <bool INIT>
static __global__ void __launch_bounds__(BX) k_cheby_sweep(Geo g, double alpha, double beta, double theta,
                                                    const double* __restrict__ u, const double* __restrict__ u0,
                                                    double* __restrict__ p, double* __restrict__ r,
                                                    double* __restrict__ w, const double* __restrict__ kx,
                                                    const double* __restrict__ ky)
{
    Strip s(g);
    if (!s.active) return;
    const int x = g.x;
    long i = s.k + (long)s.j0 * x;
    double ud = u[i - x], uc = u[i], kyc = ky[i];
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += x) {
        const double uu = u[i + x], kyu = ky[i + x];
        const double v = smvp(kx[i], kx[i + 1], kyc, kyu, uc, u[i - 1], u[i + 1], ud, uu);
        w[i] = v;
        const double rr = u0[i] - v;
        r[i] = rr;
        p[i] = INIT ? rr / theta : alpha * p[i] + beta * rr;
        ud = uc;
        uc = uu;
        kyc = kyu;
    }
}

// u += p on the interior (cheby_calc_u, cheby.c:8-24)
static __global__ void __launch_bounds__(BX) k_add_p(Geo g, double* __restrict__ u, const double* __restrict__ p)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) u[i] += p[i];
}

// sd = r / theta   (ppcg.c:9-26)
static __global__ void __launch_bounds__(BX) k_ppcg_init(Geo g, double theta, const double* __restrict__ r,
                                                  double* __restrict__ sd)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) sd[i] = r[i] / theta;
}

// r -= A sd; u += sd   (ppcg.c:41-50)
static __global__ void __launch_bounds__(BX) k_ppcg_inner_a(Geo g, double* __restrict__ u, double* __restrict__ r,
                                                     const double* __restrict__ kx, const double* __restrict__ ky,
                                                     const double* __restrict__ sd)
{
    Strip s(g);
    if (!s.active) return;
    const int x = g.x;
    long i = s.k + (long)s.j0 * x;
    double sdd = sd[i - x], sdc = sd[i], kyc = ky[i];
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += x) {
        const double sdu = sd[i + x], kyu = ky[i + x];
        const double v = smvp(kx[i], kx[i + 1], kyc, kyu, sdc, sd[i - 1], sd[i + 1], sdd, sdu);
        r[i] -= v;
        u[i] += sdc;
        sdd = sdc;
        sdc = sdu;
        kyc = kyu;
    }
}

// sd = alpha sd + beta r   (ppcg.c:52-60)
static __global__ void __launch_bounds__(BX) k_ppcg_inner_b(Geo g, double alpha, double beta, double* __restrict__ sd,
                                                     const double* __restrict__ r)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) sd[i] = alpha * sd[i] + beta * r[i];
}

// u0 = u on the interior   (solver_methods.c:9-25)
static __global__ void __launch_bounds__(BX) k_copy_u(Geo g, double* __restrict__ u0, const double* __restrict__ u)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) u0[i] = u[i];
}

// r = u0 - A u   (solver_methods.c:28-48)
static __global__ void __launch_bounds__(BX) k_residual(Geo g, const double* __restrict__ u, const double* __restrict__ u0,
                                                 double* __restrict__ r, const double* __restrict__ kx,
                                                 const double* __restrict__ ky)
{
    Strip s(g);
    if (!s.active) return;
    const int x = g.x;
    long i = s.k + (long)s.j0 * x;
    double ud = u[i - x], uc = u[i], kyc = ky[i];
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += x) {
        const double uu = u[i + x], kyu = ky[i + x];
        r[i] = u0[i] - smvp(kx[i], kx[i + 1], kyc, kyu, uc, u[i - 1], u[i + 1], ud, uu);
        ud = uc;
        uc = uu;
        kyc = kyu;
    }
}

// sum(b*b) over the interior   (solver_methods.c:51-71)
static __global__ void __launch_bounds__(BX) k_norm2(Geo g, const double* __restrict__ b, ReduceSlots rs)
{
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
        for (int j = s.j0; j < s.j1; ++j, i += g.x) acc[0] += b[i] * b[i];
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count());
}

// energy = u / density   (solver_methods.c:74-90)
static __global__ void __launch_bounds__(BX) k_finalise(Geo g, double* __restrict__ energy,
                                                 const double* __restrict__ density, const double* __restrict__ u)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) energy[i] = u[i] / density[i];
}

// vol, mass, ie, temp   (field_summary.c:8-45)
static __global__ void __launch_bounds__(BX) k_field_summary(Geo g, const double* __restrict__ volume,
                                                      const double* __restrict__ density,
                                                      const double* __restrict__ energy0,
                                                      const double* __restrict__ u, ReduceSlots rs)
{
    Strip s(g);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (s.active) {
        long i = s.k + (long)s.j0 * g.x;
        for (int j = s.j0; j < s.j1; ++j, i += g.x) {
            const double cv = volume[i];
            const double cm = cv * density[i];
            acc[0] += cv;
            acc[1] += cm;
            acc[2] += cm * energy0[i];
            acc[3] += cm * u[i];
        }
    }
    tl::grid_sum<4, BX>(acc, rs, block_id(), block_count());
}

// Jacobi sweep (jacobi.c:78-101): reads r (a copy of u), writes u, L1 change.
static __global__ void __launch_bounds__(BX) k_jacobi_iterate(Geo g, const double* __restrict__ kx,
                                                       const double* __restrict__ ky,
                                                       const double* __restrict__ u0, double* __restrict__ u,
                                                       const double* __restrict__ r, ReduceSlots rs)
{
    Strip s(g);
    double acc[1] = {0.0};
    if (s.active) {
        const int x = g.x;
        long i = s.k + (long)s.j0 * x;
        for (int j = s.j0; j < s.j1; ++j, i += x) {
            const double kxc = kx[i], kxr = kx[i + 1], kyc = ky[i], kyu = ky[i + x];
            const double v = (u0[i] + (kxr * r[i + 1] + kxc * r[i - 1]) + (kyu * r[i + x] + kyc * r[i - x]))
                           / (1.0 + (kxc + kxr) + (kyc + kyu));
            u[i] = v;
            acc[0] += fabs(v - r[i]);
        }
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count());
}

// ---- full-array kernels (thread per cell) --------------------------------

// cg_init fused (cg.c:9-85), p written to both p buffers: u = e*rho everywhere; face coefficients on
// [hd, n-1); w = A u, r = u - w, p = r on the interior with rro = sum(r*p);
// p = r = 0 elsewhere and w = conductivity on the rest of [1, n-1).
// Coefficients and neighbour values are recomputed from density/energy with
// the reference expressions, so they equal the stored ones bit for bit.
template <typename Finish>
static __global__ void __launch_bounds__(FB) k_cg_init(Geo g, int coefficient, double rx, double ry,
                                                const double* __restrict__ density,
                                                const double* __restrict__ energy, double* __restrict__ u,
                                                double* __restrict__ p, double* __restrict__ p2,
                                                double* __restrict__ r,
                                                double* __restrict__ w, double* __restrict__ kx,
                                                double* __restrict__ ky, ReduceSlots rs, Finish fin)
{
    const int x = g.x, y = g.y, hd = g.hd;
    const int k = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * (FB / 32) + (threadIdx.x >> 5);
    double acc[1] = {0.0};
    if (k < x && j < y) {
        const long i = k + (long)j * x;
        const double rho = density[i];
        const double uc = energy[i] * rho;
        u[i] = uc;
        const bool interior = k >= hd && k < x - hd && j >= hd && j < y - hd;
        const bool ring = k >= 1 && k < x - 1 && j >= 1 && j < y - 1;
        const bool kzone = k >= hd && k < x - 1 && j >= hd && j < y - 1;
        double wc = 0.0;
        if (ring) wc = coef_w(coefficient, rho);
        double kxc = 0.0, kyc = 0.0;
        if (kzone) {
            kxc = face(rx, coef_w(coefficient, density[i - 1]), wc);
            kyc = face(ry, coef_w(coefficient, density[i - x]), wc);
            kx[i] = kxc;
            ky[i] = kyc;
        }
        if (interior) {
            // kx[i+1] / ky[i+x] are computed only inside [hd, n-1); with a one-cell
            // halo the last column/row keeps whatever the array held (cg.c:56-62).
            const double kxr = (k + 1 < x - 1) ? face(rx, wc, coef_w(coefficient, density[i + 1])) : kx[i + 1];
            const double kyu = (j + 1 < y - 1) ? face(ry, wc, coef_w(coefficient, density[i + x])) : ky[i + x];
            const double ul = energy[i - 1] * density[i - 1];
            const double ur = energy[i + 1] * density[i + 1];
            const double ud = energy[i - x] * density[i - x];
            const double uu = energy[i + x] * density[i + x];
            const double v = smvp(kxc, kxr, kyc, kyu, uc, ul, ur, ud, uu);
            w[i] = v;
            const double rr = uc - v;
            r[i] = rr;
            p[i] = rr;
            if (p2) p2[i] = rr;
            acc[0] = rr * rr;
        } else {
            p[i] = 0.0;
            if (p2) p2[i] = 0.0;
            r[i] = 0.0;
            if (ring) w[i] = wc;
        }
    }
    tl::grid_sum<1, FB>(acc, rs, block_id(), block_count(), fin);
}

// jacobi_init (jacobi.c:10-57): u0 = u = e*rho on [1, n-1); kx, ky on [hd, n-1).
static __global__ void __launch_bounds__(FB) k_jacobi_init(Geo g, int coefficient, double rx, double ry,
                                                    const double* __restrict__ density,
                                                    const double* __restrict__ energy, double* __restrict__ u0,
                                                    double* __restrict__ u, double* __restrict__ kx,
                                                    double* __restrict__ ky)
{
    const int x = g.x, y = g.y, hd = g.hd;
    const int k = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * (FB / 32) + (threadIdx.x >> 5);
    if (k >= x || j >= y) return;
    const long i = k + (long)j * x;
    if (k >= 1 && k < x - 1 && j >= 1 && j < y - 1) {
        const double t = energy[i] * density[i];
        u0[i] = t;
        u[i] = t;
    }
    if (k >= hd && k < x - 1 && j >= hd && j < y - 1) {
        const double c = coef_w(coefficient, density[i]);
        const double l = coef_w(coefficient, density[i - 1]);
        const double d = coef_w(coefficient, density[i - x]);
        kx[i] = rx * (l + c) / (2.0 * l * c);
        ky[i] = ry * (d + c) / (2.0 * d * c);
    }
}

// set_chunk_data (set_chunk_data.c:10-53): vertices, cell centres, volumes, areas.
static __global__ void k_set_chunk_data_axes(int x, int y, int hd, double x_min, double y_min, double dx, double dy,
                                      double* vertex_x, double* vertex_y, double* cell_x, double* cell_y)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= x) vertex_x[t] = x_min + dx * (double)(t - hd);
    if (t <= y) vertex_y[t] = y_min + dy * (double)(t - hd);
    if (t < x) cell_x[t] = 0.5 * ((x_min + dx * (double)(t - hd)) + (x_min + dx * (double)(t + 1 - hd)));
    if (t < y) cell_y[t] = 0.5 * ((y_min + dy * (double)(t - hd)) + (y_min + dy * (double)(t + 1 - hd)));
}

static __global__ void k_set_chunk_data_cells(long n, double dx, double dy, double* volume, double* x_area,
                                       double* y_area)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        volume[i] = dx * dy;
        x_area[i] = dy;
        y_area[i] = dx;
    }
}

// set_chunk_state (set_chunk_state.c:9-84): the last state that covers a cell wins.
static __global__ void __launch_bounds__(FB) k_set_chunk_state(Geo g, const double* __restrict__ vertex_x,
                                                        const double* __restrict__ vertex_y,
                                                        const double* __restrict__ cell_x,
                                                        const double* __restrict__ cell_y,
                                                        double* __restrict__ density, double* __restrict__ energy0,
                                                        double* __restrict__ u, int num_states,
                                                        const State* __restrict__ states)
{
    const int x = g.x, y = g.y;
    const int k = blockIdx.x * 32 + (threadIdx.x & 31);
    const int j = blockIdx.y * (FB / 32) + (threadIdx.x >> 5);
    if (k >= x || j >= y) return;
    const long i = k + (long)j * x;
    double e = states[0].energy, d = states[0].density;
    for (int s = 1; s < num_states; ++s) {
        const State st = states[s];
        bool hit = false;
        if (st.geometry == TL_GEOM_RECTANGULAR) {
            hit = vertex_x[k + 1] >= st.x_min && vertex_x[k] < st.x_max && vertex_y[j + 1] >= st.y_min &&
                  vertex_y[j] < st.y_max;
        } else if (st.geometry == TL_GEOM_CIRCULAR) {
            const double ax = cell_x[k] - st.x_min, ay = cell_y[j] - st.y_min;
            hit = sqrt(ax * ax + ay * ay) <= st.radius;
        } else if (st.geometry == TL_GEOM_POINT) {
            hit = vertex_x[k] == st.x_min && vertex_y[j] == st.y_min;
        }
        if (hit) {
            e = st.energy;
            d = st.density;
        }
    }
    energy0[i] = e;
    density[i] = d;
    if (k >= 1 && k < x - 1 && j >= 1 && j < y - 1) u[i] = e * d;
}

// Reflective halo update of up to six fields (local_halos.c:21-149): for each
// external face, copy `depth` interior layers outwards, interior span only.
struct HaloArgs {
    double* f[TL_NUM_FIELDS];
    int nf;
    int ext[4];  // left, right, bottom, top are external
};

static __global__ void k_local_halos(Geo g, int depth, HaloArgs a)
{
    const int x = g.x, y = g.y, hd = g.hd;
    const int ny = y - 2 * hd, nx = x - 2 * hd;
    const long per_field = (long)depth * (2L * ny + 2L * nx);
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (t >= per_field || blockIdx.y >= (unsigned)a.nf) return;
    double* f = a.f[blockIdx.y];
    long q = t;
    const int d = (int)(q % depth);
    q /= depth;
    if (q < ny) {  // left
        if (!a.ext[0]) return;
        const long row = (long)(hd + q) * x;
        f[row + (hd - d - 1)] = f[row + (hd + d)];
        return;
    }
    q -= ny;
    if (q < ny) {  // right
        if (!a.ext[1]) return;
        const long row = (long)(hd + q) * x;
        f[row + (x - hd + d)] = f[row + (x - hd - 1 - d)];
        return;
    }
    q -= ny;
    if (q < nx) {  // bottom
        if (!a.ext[2]) return;
        const long kk = hd + q;
        f[kk + (long)(hd - d - 1) * x] = f[kk + (long)(hd + d) * x];
        return;
    }
    q -= nx;
    if (q < nx) {  // top
        if (!a.ext[3]) return;
        const long kk = hd + q;
        f[kk + (long)(y - hd + d) * x] = f[kk + (long)(y - hd - 1 - d) * x];
    }
}

// MPI face buffers (pack_halos.c:4-207): pack copies a face of the field into
// a contiguous staging buffer, unpack scatters the buffer into the halo.
static __global__ void k_pack(Geo g, int depth, int face, int pack, double* __restrict__ field, double* __restrict__ buf)
{
    const int x = g.x, y = g.y, hd = g.hd;
    const int nx = x - 2 * hd, ny = y - 2 * hd;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long fi, bi;
    if (face == TL_CHUNK_LEFT || face == TL_CHUNK_RIGHT) {
        if (t >= (long)ny * depth) return;
        const int jj = hd + (int)(t / depth), c = (int)(t % depth);
        int kk;
        if (face == TL_CHUNK_LEFT) kk = pack ? hd + c : hd - depth + c;
        else kk = pack ? x - hd - depth + c : x - hd + c;
        fi = (long)jj * x + kk;
        bi = c + (long)(jj - hd) * depth;
    } else {
        if (t >= (long)nx * depth) return;
        const int kk = hd + (int)(t % nx), c = (int)(t / nx);
        int jj;
        if (face == TL_CHUNK_BOTTOM) jj = pack ? hd + c : hd - depth + c;
        else jj = pack ? y - hd - depth + c : y - hd + c;
        fi = (long)jj * x + kk;
        bi = (kk - hd) + (long)c * nx;
    }
    if (pack) buf[bi] = field[fi];
    else field[fi] = buf[bi];
}


// External faces whose depth-1 halo is reflected (left, right, bottom, top).
struct Faces {
    int l, r, b, t;
};

// ===================================================================
// Fused kernels: each absorbs the operations the reference performs between
// two sweeps (the p update of the previous CG step, the reflective halo of
// the stencil operand, the "u += p" of the previous Chebyshev step, the sd
// update of the previous PPCG inner step), so one pass over memory does what
// the reference does in two or three. Values that the reference would read
// from a freshly reflected halo are taken from the mirrored interior cell
// directly, and the reflected values are also written to the halo cells, so
// memory ends in the state the reference leaves it in.
// ===================================================================


// Halo store of value v of interior cell (k, j) into the mirrored cells of
// the external faces closer than `depth` (local_halos.c:66-149 pattern).
__device__ __forceinline__ void reflect_store(double* f, const Geo& g, const Faces& fc, int depth, int k, int j,
                                             double v)
{
    const long row = (long)j * g.x;
    if (fc.l && k - g.hd < depth) f[row + (2 * g.hd - 1 - k)] = v;
    if (fc.r && (g.x - g.hd - 1 - k) < depth) f[row + (2 * (g.x - g.hd) - 1 - k)] = v;
    if (fc.b && j - g.hd < depth) f[(long)(2 * g.hd - 1 - j) * g.x + k] = v;
    if (fc.t && (g.y - g.hd - 1 - j) < depth) f[(long)(2 * (g.y - g.hd) - 1 - j) * g.x + k] = v;
}

// Halo duty: the extra block row of a fused sweep writes reflective halo
// cells, so the row loop of the other blocks stays free of scattered stores.
// For every external face and layer d < depth: dst[mirror] = val(source),
// source = the interior cell d layers in (local_halos.c:66-149 pattern).
// `val` must read only data the sweep does not modify.
template <typename Val>
__device__ __forceinline__ void halo_duty(const Geo& g, const Faces& fc, int depth, double* __restrict__ dst,
                                          Val val)
{
    const int x = g.x, hd = g.hd;
    const long nx = g.x - 2 * hd, ny = g.y - 2 * hd;
    const long per = (long)depth * (2 * ny + 2 * nx);
    for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < per; t += (long)gridDim.x * blockDim.x) {
        const int d = (int)(t % depth);
        long q = t / depth;
        if (q < ny) {
            const long row = (long)(hd + q) * x;
            if (fc.l) dst[row + (hd - 1 - d)] = val(row + (hd + d));
        } else if ((q -= ny) < ny) {
            const long row = (long)(hd + q) * x;
            if (fc.r) dst[row + (x - hd + d)] = val(row + (x - hd - 1 - d));
        } else if ((q -= ny) < nx) {
            const long col = hd + q;
            if (fc.b) dst[col + (long)(hd - 1 - d) * x] = val(col + (long)(hd + d) * x);
        } else {
            q -= nx;
            const long col = hd + q;
            if (fc.t) dst[col + (long)(g.y - hd + d) * x] = val(col + (long)(g.y - hd - 1 - d) * x);
        }
    }
}

constexpr unsigned kFull = 0xffffffffu;

// Column-strip coordinates with the column clamped for lanes past the
// interior (they load valid cells, feed the warp shuffles, store nothing).
struct StripC {
    int k, kk, j0, j1, lane;
    bool active, at_l, at_r;
    __device__ StripC(const Geo& g)
    {
        k = g.hd + blockIdx.x * BX + threadIdx.x;
        active = k < g.x - g.hd;
        kk = active ? k : g.x - g.hd - 1;
        j0 = g.hd + blockIdx.y * g.rows;
        j1 = min(j0 + g.rows, g.y - g.hd);
        lane = threadIdx.x & 31;
        at_l = kk == g.hd;
        at_r = kk == g.x - g.hd - 1;
    }
};

// CG sweep 1 (grid: interior blocks + one halo-duty block row):
//   [p = beta p + r]   (FUSE_P; cg.c:146-164, the previous step's calc_p)
//   w = A p ; pw = sum(w*p)   (cg.c:88-113)
// With REFLECT the depth-1 reflective halo of p is taken from the mirrored
// interior cell and written into p_out's halo; with u_halo the pending
// reflective halo of u (depth uhd, u is not modified here) is written too.
// p is read from p_in, the new p written to p_out (a second buffer, since
// neighbours still read the old p; p_out == p_in when !FUSE_P).
template <bool FUSE_P, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(BX, TL2D_MINB) k_cg_w_fused(Geo g, Faces fc, Scalar beta,
                                                          const double* __restrict__ p_in, double* p_out,
                                                          const double* __restrict__ r, double* __restrict__ w,
                                                          const double* __restrict__ kx,
                                                          const double* __restrict__ ky, double* u_halo, int uhd,
                                                          ReduceSlots rs, const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    const double bt = FUSE_P ? beta.get() : 0.0;
    auto cur = [&](long idx) { return FUSE_P ? bt * p_in[idx] + r[idx] : p_in[idx]; };
    if (blockIdx.y + 1 < gridDim.y) {
        const StripC s(g);
        const int x = g.x;
        long i = s.kk + (long)s.j0 * x;
        double pc = cur(i);
        double pd = (s.j0 == g.hd) ? ((REFLECT && fc.b) ? pc : p_in[i - x]) : cur(i - x);
        double kyc = ky[i];
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += x) {
            const bool at_t = j == g.y - g.hd - 1;
            const double pu = at_t ? ((REFLECT && fc.t) ? pc : p_in[i + x]) : cur(i + x);
            const double kyu = ky[i + x];
            const double kxc = kx[i];
            double pl = __shfl_up_sync(kFull, pc, 1);
            double pr = __shfl_down_sync(kFull, pc, 1);
            double kxr = __shfl_down_sync(kFull, kxc, 1);
            if (s.at_l) pl = (REFLECT && fc.l) ? pc : p_in[i - 1];
            else if (s.lane == 0) pl = cur(i - 1);
            if (s.at_r) pr = (REFLECT && fc.r) ? pc : p_in[i + 1];
            else if (s.lane == 31) pr = cur(i + 1);
            if (s.at_r || s.lane == 31) kxr = kx[i + 1];
            const double v = smvp(kxc, kxr, kyc, kyu, pc, pl, pr, pd, pu);
            if (s.active) {
                w[i] = v;
                acc[0] += v * pc;
                if (FUSE_P) p_out[i] = pc;
            }
            pd = pc;
            pc = pu;
            kyc = kyu;
        }
    } else {
        if (REFLECT) halo_duty(g, fc, 1, p_out, cur);
        if (u_halo) halo_duty(g, fc, uhd, u_halo, [&](long idx) { return u_halo[idx]; });
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// Rows of the CG w sweep fed by TMA (tma.cuh): kRowsT rows of a block's strip
// of p and r with a two-column ring on each side (columns k0-2 .. k0+129: the
// box starts on a 16-byte boundary for an even halo depth), kx with one
// extra column, ky; each array at a 128-byte aligned offset.
#ifndef TL2D_TMA_ROWS
#define TL2D_TMA_ROWS 4
#endif
#ifndef TL2D_TMA_STAGES
#define TL2D_TMA_STAGES 3
#endif
constexpr int kRowsT = TL2D_TMA_ROWS;
constexpr int kStagesT = TL2D_TMA_STAGES;   // rows of stages b and b+1 are read while the rest are in flight
// TMA alignment: strip starts hd + BX bx and the boxes' widths keep every x
// start and every box row a multiple of 16 bytes for an even halo depth.
static_assert((BX * sizeof(double)) % 16 == 0 && ((BX + 4) * sizeof(double)) % 16 == 0 &&
                  ((BX + 2) * sizeof(double)) % 16 == 0,
              "TMA boxes of the 2D sweeps must be multiples of 16 bytes wide");
static_assert(kStagesT >= 3, "row block b reads stages b and b+1 while a later one is in flight");
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

// k_cg_w_fused with its operand rows brought in by TMA. The same strips,
// rows in the same order per thread and the same arithmetic, so the same
// results (partial sums included). Stage b holds rows j0-1+4b .. j0+2+4b;
// rows j0+4b .. j0+4b+3 read stages b and b+1. `err`: the bounded barrier
// waits' flag.
template <bool FUSE_P, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(BX, 4) k_cg_w_fused_tma(Geo g, Faces fc, Scalar beta,
                                                                      const __grid_constant__ Tma2Maps maps,
                                                                      const double* __restrict__ p_in, double* p_out,
                                                                      const double* __restrict__ r,
                                                                      double* __restrict__ w, double* u_halo,
                                                                      int uhd, ReduceSlots rs,
                                                                      const int* __restrict__ done, Finish fin,
                                                                      int* err)
{
    extern __shared__ __align__(128) unsigned char t2_raw[];
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    const double bt = FUSE_P ? beta.get() : 0.0;
    auto cur = [&](long idx) { return FUSE_P ? bt * p_in[idx] + r[idx] : p_in[idx]; };
    if (blockIdx.y + 1 < gridDim.y) {
        unsigned char* base = t2_raw + ((128 - (tl::smem_addr(t2_raw) & 127)) & 127);
        RowsT* ring = reinterpret_cast<RowsT*>(base);
        unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesT * sizeof(RowsT));
        const StripC s(g);
        const int x = g.x, tx = threadIdx.x;
        const int k0 = g.hd + blockIdx.x * BX;
        const int jb = s.j0 - 1;                              // first row of stage 0
        const int np = (s.j1 - s.j0 + 2 + kRowsT - 1) / kRowsT;   // stages: rows j0-1 .. j1
        constexpr unsigned kP = sizeof(double) * kRowsT * (BX + 4);
        constexpr unsigned kK = sizeof(double) * kRowsT * ((BX + 2) + BX);
        auto issue = [&](int b) {
            RowsT& S = ring[b % kStagesT];
            unsigned long long* bar = &bars[b % kStagesT];
            const int y0 = jb + b * kRowsT;
            tl::mbar_expect_tx(bar, kP * (FUSE_P ? 2u : 1u) + kK);
            tl::tma_load_3d(&S.P[0][0], &maps.p, k0 - 2, y0, 0, bar);
            if (FUSE_P) tl::tma_load_3d(&S.R[0][0], &maps.r, k0 - 2, y0, 0, bar);
            tl::tma_load_3d(&S.KX[0][0], &maps.kx, k0, y0, 0, bar);
            tl::tma_load_3d(&S.KY[0][0], &maps.ky, k0, y0, 0, bar);
        };
        if (tx == 0) {
            for (int q = 0; q < kStagesT; ++q) tl::mbar_init(&bars[q], 1);
            tl::mbar_fence_init();
        }
        __syncthreads();
        if (tx == 0)
            for (int b = 0; b < kStagesT - 1 && b < np; ++b) issue(b);
        // row j of the strip: stage (j - jb) / 4, row (j - jb) % 4
        auto raw = [&](int j, int dx) -> double {
            const int t = j - jb;
            return ring[(t / kRowsT) % kStagesT].P[t % kRowsT][tx + 2 + dx];
        };
        auto fused = [&](int j, int dx) -> double {
            const int t = j - jb;
            const RowsT& S = ring[(t / kRowsT) % kStagesT];
            return FUSE_P ? bt * S.P[t % kRowsT][tx + 2 + dx] + S.R[t % kRowsT][tx + 2 + dx]
                          : S.P[t % kRowsT][tx + 2 + dx];
        };
        double pc = 0.0, pd = 0.0, kyc = 0.0;
        long i = s.kk + (long)s.j0 * x;
        for (int b = 0; b * kRowsT < s.j1 - s.j0; ++b) {
            __syncthreads();   // every thread is past rows of block b-1: stage b-1 is free
            if (tx == 0 && b + kStagesT - 1 < np) issue(b + kStagesT - 1);
            tl::mbar_wait(&bars[b % kStagesT], (unsigned)(b / kStagesT) & 1u, err);
            if (b + 1 < np) tl::mbar_wait(&bars[(b + 1) % kStagesT], (unsigned)((b + 1) / kStagesT) & 1u, err);
            if (b == 0) {
                pc = fused(s.j0, 0);
                pd = (s.j0 == g.hd) ? ((REFLECT && fc.b) ? pc : raw(s.j0 - 1, 0)) : fused(s.j0 - 1, 0);
                kyc = ring[0].KY[1][tx];
            }
#pragma unroll
            for (int u = 0; u < kRowsT; ++u) {
                const int j = s.j0 + b * kRowsT + u;
                if (j >= s.j1) break;
                const int t = j - jb, tu = t + 1;
                const RowsT& S = ring[(t / kRowsT) % kStagesT];
                const RowsT& U = ring[(tu / kRowsT) % kStagesT];
                const bool at_t = j == g.y - g.hd - 1;
                const double pu = at_t ? ((REFLECT && fc.t) ? pc : raw(j + 1, 0)) : fused(j + 1, 0);
                const double kyu = U.KY[tu % kRowsT][tx];
                const double kxc = S.KX[t % kRowsT][tx];
                double pl = __shfl_up_sync(kFull, pc, 1);
                double pr = __shfl_down_sync(kFull, pc, 1);
                double kxr = __shfl_down_sync(kFull, kxc, 1);
                if (s.at_l) pl = (REFLECT && fc.l) ? pc : raw(j, -1);
                else if (s.lane == 0) pl = fused(j, -1);
                if (s.at_r) pr = (REFLECT && fc.r) ? pc : raw(j, 1);
                else if (s.lane == 31) pr = fused(j, 1);
                if (s.at_r || s.lane == 31) kxr = S.KX[t % kRowsT][tx + 1];
                const double v = smvp(kxc, kxr, kyc, kyu, pc, pl, pr, pd, pu);
                if (s.active) {
                    w[i] = v;
                    acc[0] += v * pc;
                    if (FUSE_P) p_out[i] = pc;
                }
                pd = pc;
                pc = pu;
                kyc = kyu;
                i += x;
            }
        }
        // every issued stage was waited for (the last rows read stage np-1): no copy in flight
    } else {
        if (REFLECT) halo_duty(g, fc, 1, p_out, cur);
        if (u_halo) halo_duty(g, fc, uhd, u_halo, [&](long idx) { return u_halo[idx]; });
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// CG sweep 2: u += alpha p ; r -= alpha w ; rrn = sum(r*r)  (cg.c:116-143)
template <typename Finish>
static __global__ void __launch_bounds__(BX, TL2D_MINB) k_cg_ur_fused(Geo g, Scalar alpha, double* __restrict__ u,
                                                           const double* __restrict__ p, double* __restrict__ r,
                                                           const double* __restrict__ w, ReduceSlots rs,
                                                           const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    const int bx = ur_bx(), by = ur_by();
    Strip s(g, bx, by);
    double acc[1] = {0.0};
    if (s.active) {
        const double a = alpha.get();
        const int j_first = TL2D_UR_REVERSE ? s.j1 - 1 : s.j0;
        const long step = TL2D_UR_REVERSE ? -(long)g.x : (long)g.x;
        long i = s.k + (long)j_first * g.x;
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int n = 0; n < s.j1 - s.j0; ++n, i += step) {
            u[i] += a * p[i];
            const double rn = r[i] - a * w[i];
            r[i] = rn;
            acc[0] += rn * rn;
        }
    }
    tl::grid_sum<1, BX>(acc, rs, bx + by * gridDim.x, block_count(), fin);
}

// k_cg_ur_fused with its operands brought in by TMA: stages of kRowsU rows
// of the block's strip of u, p, r, w (128-column boxes starting at the strip's
// first column, even for an even halo depth). Same strips, rows in the same
// order per thread (TL2D_UR_REVERSE), same arithmetic: the same results,
// partial sums included.
// 4-row stages, 4 deep (66 KB per block, 3 blocks per SM): measured faster
// than 3 deep at 4 blocks per SM (130.0 against 134.6 us at 4096^2), and than
// 2-row x 5 and 8-row x 3 and 6-row x 3 rings.
#ifndef TL2D_TMA_ROWS_U
#define TL2D_TMA_ROWS_U 4
#endif
#ifndef TL2D_TMA_STAGES_U
#define TL2D_TMA_STAGES_U 4
#endif
constexpr int kRowsU = TL2D_TMA_ROWS_U;
constexpr int kStagesU = TL2D_TMA_STAGES_U;
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

template <typename Finish>
static __global__ void __launch_bounds__(BX, 4) k_cg_ur_fused_tma(Geo g, Scalar alpha,
                                                               const __grid_constant__ TmaUrMaps maps,
                                                               double* __restrict__ u, double* __restrict__ r,
                                                               ReduceSlots rs, const int* __restrict__ done,
                                                               Finish fin, int* err)
{
    extern __shared__ __align__(128) unsigned char tu_raw[];
    if (gate_closed(done)) return;
    unsigned char* base = tu_raw + ((128 - (tl::smem_addr(tu_raw) & 127)) & 127);
    RowsU* ring = reinterpret_cast<RowsU*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesU * sizeof(RowsU));
    const int bx = ur_bx(), by = ur_by();
    Strip s(g, bx, by);
    double acc[1] = {0.0};
    const int tx = threadIdx.x;
    const int k0 = g.hd + bx * BX;
    const int np = (s.j1 - s.j0 + kRowsU - 1) / kRowsU;
    // stage b holds rows y0(b) .. y0(b) + kRowsU - 1 (the last stage of the
    // strip may run past j1; those rows are loaded and not used)
    auto stage_y0 = [&](int b) { return s.j0 + (TL2D_UR_REVERSE ? np - 1 - b : b) * kRowsU; };
    auto issue = [&](int b) {
        RowsU& S = ring[b % kStagesU];
        unsigned long long* bar = &bars[b % kStagesU];
        const int y0 = stage_y0(b);
        tl::mbar_expect_tx(bar, 4u * sizeof(double) * kRowsU * BX);
        tl::tma_load_3d(&S.U[0][0], &maps.u, k0, y0, 0, bar);
        tl::tma_load_3d(&S.P[0][0], &maps.p, k0, y0, 0, bar);
        tl::tma_load_3d(&S.R[0][0], &maps.r, k0, y0, 0, bar);
        tl::tma_load_3d(&S.W[0][0], &maps.w, k0, y0, 0, bar);
    };
    if (tx == 0) {
        for (int q = 0; q < kStagesU; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (tx == 0)
        for (int b = 0; b < kStagesU - 1 && b < np; ++b) issue(b);
    const double a = alpha.get();
    for (int b = 0; b < np; ++b) {
        __syncthreads();   // every thread is past stage b-1: its slot is free
        if (tx == 0 && b + kStagesU - 1 < np) issue(b + kStagesU - 1);
        tl::mbar_wait(&bars[b % kStagesU], (unsigned)(b / kStagesU) & 1u, err);
        const RowsU& S = ring[b % kStagesU];
        const int y0 = stage_y0(b);
#pragma unroll
        for (int q = 0; q < kRowsU; ++q) {
            const int t = TL2D_UR_REVERSE ? kRowsU - 1 - q : q;   // rows in the order of k_cg_ur_fused
            const int j = y0 + t;
            if (j >= s.j1) continue;
            if (s.active) {
                const long i = s.k + (long)j * g.x;
                u[i] = S.U[t][tx] + a * S.P[t][tx];
                const double rn = S.R[t][tx] - a * S.W[t][tx];
                r[i] = rn;
                acc[0] += rn * rn;
            }
        }
    }
    tl::grid_sum<1, BX>(acc, rs, bx + by * gridDim.x, block_count(), fin);
}

// p = beta p + r in place, with the depth-1 halo of p (and of u unless u is
// null) written from the final values (the end of a device-resident CG phase: the last trip's
// calc_p and halo update, cg_driver.c:116-123 + halo_update_driver).
static __global__ void __launch_bounds__(BX) k_cg_close(Geo g, Faces fc, Scalar beta, int apply_p, double* __restrict__ p,
                                                 const double* __restrict__ r, double* __restrict__ u)
{
    Strip s(g);
    if (!s.active) return;
    const double bt = beta.get();
    long i = s.k + (long)s.j0 * g.x;
    for (int j = s.j0; j < s.j1; ++j, i += g.x) {
        const double pn = apply_p ? bt * p[i] + r[i] : p[i];
        p[i] = pn;
        reflect_store(p, g, fc, 1, s.k, j, pn);
        if (u) reflect_store(u, g, fc, 1, s.k, j, u[i]);
    }
}

// --------------------------------------------------------- Chebyshev ----

// One Chebyshev trip (cheby.c:57-85) with the previous trip's u += p folded
// in (ADD: u_n = u_{n-1} + p_{n-1}, read at the stencil points from u_in and
// p_in): w = A u_n ; r = u0 - w ; p_n = alpha p_{n-1} + beta r. Writes u_n to
// u_out and p_n to p_out (second buffers: neighbours read the old values),
// w and r when `write_wr` applies, and reduces sum(r*r). With REFLECT the
// depth-1 halo of u_n is taken from the mirrored cells and written by the
// halo-duty block row (grid: interior blocks + one row).
template <bool ADD, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(BX, TL2D_MINB) k_cheby_trip(Geo g, Faces fc, ChebyCoef coef, int write_wr_always,
                                                          const double* __restrict__ u_in,
                                                          const double* __restrict__ p_in, double* u_out,
                                                          double* __restrict__ p_out, const double* __restrict__ u0,
                                                          double* __restrict__ w, double* __restrict__ r,
                                                          const double* __restrict__ kx,
                                                          const double* __restrict__ ky, ReduceSlots rs,
                                                          const int* __restrict__ done, Finish fin, DevParams prm)
{
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    double a, b;
    coef.get(a, b);
    // w and r are only observable on the trips that take the norm, and on
    // the last trip of the loop (their values stay in memory afterwards).
    const bool wr = write_wr_always || !coef.st ||
                    (coef.st->nch >= coef.st->est && ((coef.st->trip + 1) % 10) == 0) ||
                    (coef.st->trip + 1 >= prm.max_iters);
    auto cur = [&](long idx) { return ADD ? u_in[idx] + p_in[idx] : u_in[idx]; };
    if (blockIdx.y + 1 < gridDim.y) {
        const StripC s(g);
        const int x = g.x;
        long i = s.kk + (long)s.j0 * x;
        double uc = cur(i);
        double ud = (s.j0 == g.hd) ? ((REFLECT && fc.b) ? uc : u_in[i - x]) : cur(i - x);
        double kyc = ky[i];
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += x) {
            const bool at_t = j == g.y - g.hd - 1;
            const double uu = at_t ? ((REFLECT && fc.t) ? uc : u_in[i + x]) : cur(i + x);
            const double kyu = ky[i + x];
            const double kxc = kx[i];
            double ul = __shfl_up_sync(kFull, uc, 1);
            double ur = __shfl_down_sync(kFull, uc, 1);
            double kxr = __shfl_down_sync(kFull, kxc, 1);
            if (s.at_l) ul = (REFLECT && fc.l) ? uc : u_in[i - 1];
            else if (s.lane == 0) ul = cur(i - 1);
            if (s.at_r) ur = (REFLECT && fc.r) ? uc : u_in[i + 1];
            else if (s.lane == 31) ur = cur(i + 1);
            if (s.at_r || s.lane == 31) kxr = kx[i + 1];
            const double v = smvp(kxc, kxr, kyc, kyu, uc, ul, ur, ud, uu);
            const double rr = u0[i] - v;
            if (s.active) {
                const double pn = a * p_in[i] + b * rr;
                if (wr) {
                    w[i] = v;
                    r[i] = rr;
                }
                acc[0] += rr * rr;
                p_out[i] = pn;
                if (ADD) u_out[i] = uc;
            }
            ud = uc;
            uc = uu;
            kyc = kyu;
        }
    } else if (REFLECT) {
        halo_duty(g, fc, 1, ADD ? u_out : const_cast<double*>(u_in), cur);
    }
    tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

// u += p in place with the depth-1 halo of u written from the final values
// (closing the pending "u += p" of the last Chebyshev trip, cheby.c:8-24,
// and the halo update that followed it).
static __global__ void __launch_bounds__(BX) k_add_p_close(Geo g, Faces fc, double* __restrict__ u,
                                                    const double* __restrict__ p)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
    for (int j = s.j0; j < s.j1; ++j, i += g.x) {
        const double un = u[i] + p[i];
        u[i] = un;
        reflect_store(u, g, fc, 1, s.k, j, un);
    }
}

// --------------------------------------------------------------- PPCG ----

// One PPCG inner step (ppcg.c:29-61) with the previous step's sd update folded
// in: FOLD 0: sd = sd_in (as stored); FOLD 1: sd = r_in / theta (ppcg_init,
// ppcg.c:9-26); FOLD 2: sd = a_prev sd_in + b_prev r_in. Then, with the
// depth-1 reflective halo of sd: r = r_in - A sd ; u += sd. sd goes to
// sd_out, r to r_out (second buffers: neighbours read the old values); the
// halo-duty block row writes sd_out's halo; NORM reduces sum(r*r) of the new r.
template <int FOLD, bool NORM, typename Finish>
static __global__ void __launch_bounds__(BX, TL2D_MINB) k_ppcg_step(Geo g, Faces fc, double theta, PpcgCoef coef, int pp_prev,
                                                         const double* __restrict__ sd_in,
                                                         double* __restrict__ sd_out,
                                                         const double* __restrict__ r_in, double* __restrict__ r_out,
                                                         double* __restrict__ u, const double* __restrict__ kx,
                                                         const double* __restrict__ ky, ReduceSlots rs,
                                                         const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    double a = 0.0, b = 0.0;
    if (FOLD == 2) coef.get(pp_prev, a, b);
    auto cur = [&](long idx) {
        if (FOLD == 0) return sd_in[idx];
        if (FOLD == 1) return r_in[idx] / theta;
        return a * sd_in[idx] + b * r_in[idx];
    };
    if (blockIdx.y + 1 < gridDim.y) {
        const StripC s(g);
        const int x = g.x;
        long i = s.kk + (long)s.j0 * x;
        double sc = cur(i);
        double sdn = (s.j0 == g.hd) ? (fc.b ? sc : sd_in[i - x]) : cur(i - x);
        double kyc = ky[i];
TL2D_PRAGMA_UNROLL(TL2D_UNROLL)
        for (int j = s.j0; j < s.j1; ++j, i += x) {
            const bool at_t = j == g.y - g.hd - 1;
            const double su = at_t ? (fc.t ? sc : sd_in[i + x]) : cur(i + x);
            const double kyu = ky[i + x];
            const double kxc = kx[i];
            double sl = __shfl_up_sync(kFull, sc, 1);
            double sr = __shfl_down_sync(kFull, sc, 1);
            double kxr = __shfl_down_sync(kFull, kxc, 1);
            if (s.at_l) sl = fc.l ? sc : sd_in[i - 1];
            else if (s.lane == 0) sl = cur(i - 1);
            if (s.at_r) sr = fc.r ? sc : sd_in[i + 1];
            else if (s.lane == 31) sr = cur(i + 1);
            if (s.at_r || s.lane == 31) kxr = kx[i + 1];
            const double v = smvp(kxc, kxr, kyc, kyu, sc, sl, sr, sdn, su);
            if (s.active) {
                const double rn = r_in[i] - v;
                r_out[i] = rn;
                u[i] += sc;
                sd_out[i] = sc;
                if (NORM) acc[0] += rn * rn;
            }
            sdn = sc;
            sc = su;
            kyc = kyu;
        }
    } else {
        halo_duty(g, fc, 1, sd_out, cur);
    }
    if (NORM) tl::grid_sum<1, BX>(acc, rs, block_id(), block_count(), fin);
}

}  // namespace tl2d
