// suite2d.cu -- B200 (sm_100a) TeaLeaf 2D kernel suite behind the reference
// kernel interface (2d/kernel_interface.h:13-71).
//
// Data layout in HBM: every field is one cudaMalloc'd slice of a per-chunk
// slab, x*y FP64 values, index k + j*x (x fastest, halo included), exactly
// the layout the reference kernels index (2d/shared.h:49-54). Slices start on
// 256-byte boundaries.
//
// Kernel shapes: interior sweeps run one thread per column (128 columns per
// block, one warp = 256 contiguous bytes per load) and walk ROWS rows down
// the column, carrying the vertical neighbours of the stencil in registers,
// so each field is read from DRAM once per sweep. Reductions are fused into
// the sweep that produces their operands (p.w into w = Ap, r.r into the
// u/r update) and finished by one last-block pass (common.cuh), which also
// writes the scalar straight into mapped pinned host memory.
//
// Floating point: this file is compiled with -fmad=false so each + - * / is
// one IEEE operation in the reference's expression order; element-wise
// results equal the reference's strict-IEEE build bit for bit, and dot
// products differ only by summation order.
#include "common.cuh"
#include "tealeaf_b200_2d.h"

#include <cuda_runtime.h>
#include <vector>

using tl::ReduceSlots;

namespace {

constexpr int BX = 128;   // threads (columns) per block of an interior sweep
constexpr int ROWS = 8;   // rows per thread of an interior sweep
constexpr int FB = 256;   // threads per block of full-array kernels

struct Geo {
    int x, y, hd;
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
    __device__ Strip(const Geo& g)
    {
        k = g.hd + blockIdx.x * BX + threadIdx.x;
        j0 = g.hd + blockIdx.y * ROWS;
        j1 = min(j0 + ROWS, g.y - g.hd);
        active = k < g.x - g.hd;
    }
};

// w = A p and pw = sum(w*p)   (cg.c:88-113)
__global__ void __launch_bounds__(BX) k_cg_calc_w(Geo g, const double* __restrict__ p, double* __restrict__ w,
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
__global__ void __launch_bounds__(BX) k_cg_calc_ur(Geo g, double alpha, double* __restrict__ u,
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
__global__ void __launch_bounds__(BX) k_cg_calc_p(Geo g, double beta, double* __restrict__ p,
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
__global__ void __launch_bounds__(BX) k_cheby_sweep(Geo g, double alpha, double beta, double theta,
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
__global__ void __launch_bounds__(BX) k_add_p(Geo g, double* __restrict__ u, const double* __restrict__ p)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) u[i] += p[i];
}

// sd = r / theta   (ppcg.c:9-26)
__global__ void __launch_bounds__(BX) k_ppcg_init(Geo g, double theta, const double* __restrict__ r,
                                                  double* __restrict__ sd)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) sd[i] = r[i] / theta;
}

// r -= A sd; u += sd   (ppcg.c:41-50)
__global__ void __launch_bounds__(BX) k_ppcg_inner_a(Geo g, double* __restrict__ u, double* __restrict__ r,
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
__global__ void __launch_bounds__(BX) k_ppcg_inner_b(Geo g, double alpha, double beta, double* __restrict__ sd,
                                                     const double* __restrict__ r)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) sd[i] = alpha * sd[i] + beta * r[i];
}

// u0 = u on the interior   (solver_methods.c:9-25)
__global__ void __launch_bounds__(BX) k_copy_u(Geo g, double* __restrict__ u0, const double* __restrict__ u)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) u0[i] = u[i];
}

// r = u0 - A u   (solver_methods.c:28-48)
__global__ void __launch_bounds__(BX) k_residual(Geo g, const double* __restrict__ u, const double* __restrict__ u0,
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
__global__ void __launch_bounds__(BX) k_norm2(Geo g, const double* __restrict__ b, ReduceSlots rs)
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
__global__ void __launch_bounds__(BX) k_finalise(Geo g, double* __restrict__ energy,
                                                 const double* __restrict__ density, const double* __restrict__ u)
{
    Strip s(g);
    if (!s.active) return;
    long i = s.k + (long)s.j0 * g.x;
#pragma unroll 4
    for (int j = s.j0; j < s.j1; ++j, i += g.x) energy[i] = u[i] / density[i];
}

// vol, mass, ie, temp   (field_summary.c:8-45)
__global__ void __launch_bounds__(BX) k_field_summary(Geo g, const double* __restrict__ volume,
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
__global__ void __launch_bounds__(BX) k_jacobi_iterate(Geo g, const double* __restrict__ kx,
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

// cg_init fused (cg.c:9-85): u = e*rho everywhere; face coefficients on
// [hd, n-1); w = A u, r = u - w, p = r on the interior with rro = sum(r*p);
// p = r = 0 elsewhere and w = conductivity on the rest of [1, n-1).
// Coefficients and neighbour values are recomputed from density/energy with
// the reference expressions, so they equal the stored ones bit for bit.
__global__ void __launch_bounds__(FB) k_cg_init(Geo g, int coefficient, double rx, double ry,
                                                const double* __restrict__ density,
                                                const double* __restrict__ energy, double* __restrict__ u,
                                                double* __restrict__ p, double* __restrict__ r,
                                                double* __restrict__ w, double* __restrict__ kx,
                                                double* __restrict__ ky, ReduceSlots rs)
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
            acc[0] = rr * rr;
        } else {
            p[i] = 0.0;
            r[i] = 0.0;
            if (ring) w[i] = wc;
        }
    }
    tl::grid_sum<1, FB>(acc, rs, block_id(), block_count());
}

// jacobi_init (jacobi.c:10-57): u0 = u = e*rho on [1, n-1); kx, ky on [hd, n-1).
__global__ void __launch_bounds__(FB) k_jacobi_init(Geo g, int coefficient, double rx, double ry,
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
__global__ void k_set_chunk_data_axes(int x, int y, int hd, double x_min, double y_min, double dx, double dy,
                                      double* vertex_x, double* vertex_y, double* cell_x, double* cell_y)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t <= x) vertex_x[t] = x_min + dx * (double)(t - hd);
    if (t <= y) vertex_y[t] = y_min + dy * (double)(t - hd);
    if (t < x) cell_x[t] = 0.5 * ((x_min + dx * (double)(t - hd)) + (x_min + dx * (double)(t + 1 - hd)));
    if (t < y) cell_y[t] = 0.5 * ((y_min + dy * (double)(t - hd)) + (y_min + dy * (double)(t + 1 - hd)));
}

__global__ void k_set_chunk_data_cells(long n, double dx, double dy, double* volume, double* x_area,
                                       double* y_area)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        volume[i] = dx * dy;
        x_area[i] = dy;
        y_area[i] = dx;
    }
}

// set_chunk_state (set_chunk_state.c:9-84): the last state that covers a cell wins.
__global__ void __launch_bounds__(FB) k_set_chunk_state(Geo g, const double* __restrict__ vertex_x,
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

__global__ void k_local_halos(Geo g, int depth, HaloArgs a)
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
__global__ void k_pack(Geo g, int depth, int face, int pack, double* __restrict__ field, double* __restrict__ buf)
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

}  // namespace

// ===================================================================== host

struct TlSuite2D {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    Geo g{0, 0, 0};
    void* slab = nullptr;
    size_t slab_bytes = 0;
    ReduceSlots rs{};
    double* h_out = nullptr;          // mapped pinned result slots
    long partial_capacity = 0;        // doubles
    State* d_states = nullptr;
    int d_states_cap = 0;
    double* d_comm = nullptr;         // pack/unpack staging
    long d_comm_cap = 0;
    tl::Profiler prof;                // per-kernel device time (off by default)
};

// Launch on the suite stream, bracketed by profiler events when enabled.
#define TL_LAUNCH(s, name, ...)                \
    do {                                       \
        (s)->prof.begin((s)->stream, name);    \
        __VA_ARGS__;                           \
        (s)->prof.end((s)->stream);            \
        TL_LAUNCHED(name);                     \
    } while (0)

namespace {

TlSuite2D* suite_of(Chunk* chunk)
{
    if (!chunk || !chunk->ext || !chunk->ext->suite) {
        tl::fail(1, "chunk has no B200 suite state (run_kernel_initialise not called)");
        return nullptr;
    }
    return chunk->ext->suite;
}

dim3 interior_grid(const Geo& g) { return dim3(tl::ceil_div(g.x - 2 * g.hd, BX), tl::ceil_div(g.y - 2 * g.hd, ROWS)); }
dim3 full_grid(const Geo& g) { return dim3(tl::ceil_div(g.x, 32), tl::ceil_div(g.y, FB / 32)); }

// Waits for the stream and returns the published sums.
bool fetch(TlSuite2D* s, int n, double* out)
{
    if (!TL_CUDA(cudaStreamSynchronize(s->stream))) return false;
    if (s->prof.on) s->prof.resolve();
    for (int i = 0; i < n; ++i) out[i] = s->h_out[i];
    return true;
}

bool check_geometry(Chunk* chunk, Settings* settings)
{
    if (chunk->x < 2 * settings->halo_depth + 1 || chunk->y < 2 * settings->halo_depth + 1 ||
        settings->halo_depth < 1) {
        tl::fail(2, "invalid chunk extents x=%d y=%d halo_depth=%d", chunk->x, chunk->y, settings->halo_depth);
        return false;
    }
    return true;
}

}  // namespace

// The reference host's logger (2d/shared.c:25-51), used when the host provides it.
extern "C" void print_and_log(Settings* settings, const char* format, ...) __attribute__((weak));

extern "C" {

// ---------------------------------------------------------------- extras --
void tl2d_set_error_mode(int mode) { tl::error_state().mode = mode; }
void tl2d_set_device(int device) { TL_CUDA(cudaSetDevice(device)); }
int tl2d_get_error(char* msg, int msg_len) { return tl::take_error(msg, msg_len); }
void* tl2d_stream(Chunk* chunk)
{
    TlSuite2D* s = suite_of(chunk);
    return s ? (void*)s->stream : nullptr;
}

void tl2d_profile_enable(Chunk* chunk, int on)
{
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    s->prof.resolve();
    s->prof.on = on != 0;
}

void tl2d_profile_reset(Chunk* chunk)
{
    TlSuite2D* s = suite_of(chunk);
    if (s) s->prof.reset();
}

int tl2d_profile_read(Chunk* chunk, int index, char* name, int name_len, long long* calls, double* ms)
{
    TlSuite2D* s = suite_of(chunk);
    if (!s || index < 0 || index >= tl::Profiler::kMaxKernels || !s->prof.names[index]) return 0;
    s->prof.resolve();
    if (name && name_len > 0) snprintf(name, (size_t)name_len, "%s", s->prof.names[index]);
    if (calls) *calls = s->prof.calls[index];
    if (ms) *ms = s->prof.ms[index];
    return 1;
}

// -------------------------------------------------- initialisation kernels --
// 2d/kernel_interface.h:17 -- allocates and zeroes every field on the device
// and the four host coefficient arrays (kernel_initialise.c:27-70).
void run_kernel_initialise(Chunk* chunk, Settings* settings)
{
    if (tl::failed() || !check_geometry(chunk, settings)) return;
    if (!chunk->ext) {
        tl::fail(3, "chunk->ext is NULL (the host allocates ChunkExtension, 2d/chunk.c:29)");
        return;
    }
    TlSuite2D* s = new TlSuite2D();
    chunk->ext->suite = s;
    TL_CUDA(cudaGetDevice(&s->device));
    TL_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device));
    if (!TL_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking))) return;
    s->g = Geo{chunk->x, chunk->y, settings->halo_depth};
    const long x = chunk->x, y = chunk->y, n = x * y;

    struct Req { FieldBufferType* dst; long count; };
    Req reqs[] = {
        {&chunk->density0, n}, {&chunk->density, n}, {&chunk->energy0, n}, {&chunk->energy, n},
        {&chunk->u, n}, {&chunk->u0, n}, {&chunk->p, n}, {&chunk->r, n}, {&chunk->mi, n},
        {&chunk->w, n}, {&chunk->kx, n}, {&chunk->ky, n}, {&chunk->sd, n}, {&chunk->volume, n},
        {&chunk->x_area, (x + 1) * y}, {&chunk->y_area, x * (y + 1)},
        {&chunk->cell_x, x}, {&chunk->cell_y, y}, {&chunk->cell_dx, x}, {&chunk->cell_dy, y},
        {&chunk->vertex_dx, x + 1}, {&chunk->vertex_dy, y + 1},
        {&chunk->vertex_x, x + 1}, {&chunk->vertex_y, y + 1},
    };
    // Reduction partials: one slot set per block of the largest reduction launch.
    const dim3 gi = interior_grid(s->g), gf = full_grid(s->g);
    const long blocks = std::max<long>((long)gi.x * gi.y, (long)gf.x * gf.y);
    s->partial_capacity = blocks * tl::kMaxSums;

    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t bytes = 0;
    for (const Req& r : reqs) bytes += align((size_t)r.count * sizeof(double));
    bytes += align((size_t)s->partial_capacity * sizeof(double)) + align(tl::kMaxSums * sizeof(double)) + 256;
    if (!TL_CUDA(cudaMalloc(&s->slab, bytes))) return;
    s->slab_bytes = bytes;
    TL_CUDA(cudaMemsetAsync(s->slab, 0, bytes, s->stream));
    char* cur = (char*)s->slab;
    for (const Req& r : reqs) {
        *r.dst = (double*)cur;
        cur += align((size_t)r.count * sizeof(double));
    }
    s->rs.partials = (double*)cur;
    cur += align((size_t)s->partial_capacity * sizeof(double));
    s->rs.out_dev = (double*)cur;
    cur += align(tl::kMaxSums * sizeof(double));
    s->rs.ticket = (unsigned int*)cur;
    if (!TL_CUDA(cudaHostAlloc((void**)&s->h_out, tl::kMaxSums * sizeof(double), cudaHostAllocMapped))) return;
    double* dev_view = nullptr;
    if (!TL_CUDA(cudaHostGetDevicePointer((void**)&dev_view, s->h_out, 0))) return;
    s->rs.out_host = dev_view;

    const int mi = settings->max_iters > 0 ? settings->max_iters : 1;
    chunk->cg_alphas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cg_betas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cheby_alphas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cheby_betas = (double*)calloc((size_t)mi, sizeof(double));
    TL_CUDA(cudaStreamSynchronize(s->stream));
    if (print_and_log && settings->tea_out_fp)
        print_and_log(settings, "Performing this solve with the B200 (sm_100a) %s solver\n",
                      settings->solver_name ? settings->solver_name : "");
}

// 2d/kernel_interface.h:19 (kernel_initialise.c:73-110)
void run_kernel_finalise(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (!chunk || !chunk->ext || !chunk->ext->suite) return;
    TlSuite2D* s = chunk->ext->suite;
    cudaStreamSynchronize(s->stream);
    cudaFree(s->slab);
    cudaFreeHost(s->h_out);
    if (s->d_states) cudaFree(s->d_states);
    if (s->d_comm) cudaFree(s->d_comm);
    cudaStreamDestroy(s->stream);
    free(chunk->cg_alphas);
    free(chunk->cg_betas);
    free(chunk->cheby_alphas);
    free(chunk->cheby_betas);
    chunk->cg_alphas = chunk->cg_betas = chunk->cheby_alphas = chunk->cheby_betas = nullptr;
    delete s;
    chunk->ext->suite = nullptr;
}

// 2d/kernel_interface.h:13 (set_chunk_data.c:10-53)
void run_set_chunk_data(Chunk* chunk, Settings* settings)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    const double x_min = settings->grid_x_min + settings->dx * (double)chunk->left;
    const double y_min = settings->grid_y_min + settings->dy * (double)chunk->bottom;
    const int m = std::max(chunk->x, chunk->y) + 1;
    TL_LAUNCH(s, "k_set_chunk_data_axes", k_set_chunk_data_axes<<<tl::ceil_div(m, 256), 256, 0, s->stream>>>(
        chunk->x, chunk->y, settings->halo_depth, x_min, y_min, settings->dx, settings->dy, chunk->vertex_x,
        chunk->vertex_y, chunk->cell_x, chunk->cell_y));
    const long n = (long)chunk->x * chunk->y;
    TL_LAUNCH(s, "k_set_chunk_data_cells", k_set_chunk_data_cells<<<s->sm_count * 8, 256, 0, s->stream>>>(n, settings->dx, settings->dy, chunk->volume,
                                                                   chunk->x_area, chunk->y_area));
}

// 2d/kernel_interface.h:15 (set_chunk_state.c:9-84); states is a host array.
void run_set_chunk_state(Chunk* chunk, Settings* settings, State* states)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    const int ns = settings->num_states;
    if (ns < 1 || !states) {
        tl::fail(4, "run_set_chunk_state needs at least one state");
        return;
    }
    if (ns > s->d_states_cap) {
        if (s->d_states) cudaFree(s->d_states);
        if (!TL_CUDA(cudaMalloc(&s->d_states, sizeof(State) * ns))) return;
        s->d_states_cap = ns;
    }
    TL_CUDA(cudaMemcpyAsync(s->d_states, states, sizeof(State) * ns, cudaMemcpyHostToDevice, s->stream));
    TL_LAUNCH(s, "k_set_chunk_state", k_set_chunk_state<<<full_grid(s->g), FB, 0, s->stream>>>(s->g, chunk->vertex_x, chunk->vertex_y, chunk->cell_x,
                                                            chunk->cell_y, chunk->density, chunk->energy0,
                                                            chunk->u, ns, s->d_states));
    TL_CUDA(cudaStreamSynchronize(s->stream));  // the host may free `states` on return
}

// ------------------------------------------------------ solver-wide kernels --
// 2d/kernel_interface.h:23 (local_halos.c:21-64)
void run_local_halos(Chunk* chunk, Settings* settings, int depth)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    if (depth < 1 || depth > settings->halo_depth) {
        tl::fail(5, "halo depth %d outside [1, %d]", depth, settings->halo_depth);
        return;
    }
    HaloArgs a{};
    // reference update order: density, p, energy0, energy1, u, sd (local_halos.c:40-45)
    const int order[TL_NUM_FIELDS] = {TL_FIELD_DENSITY, TL_FIELD_P, TL_FIELD_ENERGY0,
                                      TL_FIELD_ENERGY1, TL_FIELD_U, TL_FIELD_SD};
    FieldBufferType fields[TL_NUM_FIELDS] = {chunk->density, chunk->energy0, chunk->energy,
                                             chunk->u, chunk->p, chunk->sd};
    for (int o = 0; o < TL_NUM_FIELDS; ++o)
        if (settings->fields_to_exchange[order[o]]) a.f[a.nf++] = fields[order[o]];
    if (a.nf == 0) return;
    for (int f = 0; f < 4; ++f) a.ext[f] = chunk->neighbours[f] == TL_EXTERNAL_FACE;
    const long per = (long)depth * (2L * (s->g.y - 2 * s->g.hd) + 2L * (s->g.x - 2 * s->g.hd));
    TL_LAUNCH(s, "k_local_halos", k_local_halos<<<dim3(tl::ceil_div(per, 256), a.nf), 256, 0, s->stream>>>(s->g, depth, a));
}

// 2d/kernel_interface.h:25 (pack_halos.c:179-207). `buffer` may be host or
// device memory (the reference host passes its malloc'd MPI buffers).
void run_pack_or_unpack(Chunk* chunk, Settings* settings, int depth, int face, bool pack, FieldBufferType field,
                        double* buffer)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    if (face < 0 || face > 3) {
        tl::fail(6, "Incorrect face provided: %d.", face);
        return;
    }
    const int nx = s->g.x - 2 * s->g.hd, ny = s->g.y - 2 * s->g.hd;
    const long len = (long)depth * ((face == TL_CHUNK_LEFT || face == TL_CHUNK_RIGHT) ? ny : nx);
    if (len > s->d_comm_cap) {
        if (s->d_comm) cudaFree(s->d_comm);
        if (!TL_CUDA(cudaMalloc(&s->d_comm, sizeof(double) * len))) return;
        s->d_comm_cap = len;
    }
    (void)settings;
    if (!pack)
        TL_CUDA(cudaMemcpyAsync(s->d_comm, buffer, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL_LAUNCH(s, "k_pack", k_pack<<<tl::ceil_div(len, 256), 256, 0, s->stream>>>(s->g, depth, face, pack ? 1 : 0, field, s->d_comm));
    if (pack)
        TL_CUDA(cudaMemcpyAsync(buffer, s->d_comm, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// 2d/kernel_interface.h:28 (store_energy.c:4-15): energy = energy0, full array.
void run_store_energy(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->energy, chunk->energy0, sizeof(double) * (size_t)chunk->x * chunk->y,
                            cudaMemcpyDeviceToDevice, s->stream));
}

// 2d/kernel_interface.h:30 (field_summary.c:8-45)
void run_field_summary(Chunk* chunk, Settings* settings, double* vol, double* mass, double* ie, double* temp)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_field_summary", k_field_summary<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->volume, chunk->density, chunk->energy0,
                                                              chunk->u, s->rs));
    double o[4];
    if (!fetch(s, 4, o)) return;
    *vol += o[0];
    *mass += o[1];
    *ie += o[2];
    *temp += o[3];
}

// ------------------------------------------------------------- CG kernels --
// 2d/kernel_interface.h:35 (cg.c:9-85)
void run_cg_init(Chunk* chunk, Settings* settings, double rx, double ry, double* rro)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    if (settings->coefficient != TL_CONDUCTIVITY && settings->coefficient != TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL_LAUNCH(s, "k_cg_init", k_cg_init<<<full_grid(s->g), FB, 0, s->stream>>>(s->g, settings->coefficient, rx, ry, chunk->density,
                                                    chunk->energy, chunk->u, chunk->p, chunk->r, chunk->w,
                                                    chunk->kx, chunk->ky, s->rs));
    double o;
    if (fetch(s, 1, &o)) *rro += o;
}

// 2d/kernel_interface.h:38 (cg.c:88-113)
void run_cg_calc_w(Chunk* chunk, Settings* settings, double* pw)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cg_calc_w", k_cg_calc_w<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->p, chunk->w, chunk->kx, chunk->ky, s->rs));
    double o;
    if (fetch(s, 1, &o)) *pw += o;
}

// 2d/kernel_interface.h:40 (cg.c:116-143)
void run_cg_calc_ur(Chunk* chunk, Settings* settings, double alpha, double* rrn)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cg_calc_ur", k_cg_calc_ur<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, alpha, chunk->u, chunk->p, chunk->r, chunk->w,
                                                           s->rs));
    double o;
    if (fetch(s, 1, &o)) *rrn += o;
}

// 2d/kernel_interface.h:42 (cg.c:146-164)
void run_cg_calc_p(Chunk* chunk, Settings* settings, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cg_calc_p", k_cg_calc_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, beta, chunk->p, chunk->r));
}

// ------------------------------------------------------- Chebyshev kernels --
// 2d/kernel_interface.h:46 (cheby.c:26-54)
void run_cheby_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cheby_sweep<init>", k_cheby_sweep<true><<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, 0.0, 0.0, chunk->theta, chunk->u,
                                                                   chunk->u0, chunk->p, chunk->r, chunk->w,
                                                                   chunk->kx, chunk->ky));
    TL_LAUNCH(s, "k_add_p", k_add_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->p));
}

// 2d/kernel_interface.h:48 (cheby.c:57-85)
void run_cheby_iterate(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cheby_sweep", k_cheby_sweep<false><<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, alpha, beta, 0.0, chunk->u, chunk->u0,
                                                                    chunk->p, chunk->r, chunk->w, chunk->kx,
                                                                    chunk->ky));
    TL_LAUNCH(s, "k_add_p", k_add_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->p));
}

// ---------------------------------------------------------- Jacobi kernels --
// 2d/kernel_interface.h:52 (jacobi.c:10-57)
void run_jacobi_init(Chunk* chunk, Settings* settings, double rx, double ry)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    if (settings->coefficient < TL_CONDUCTIVITY && settings->coefficient < TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL_LAUNCH(s, "k_jacobi_init", k_jacobi_init<<<full_grid(s->g), FB, 0, s->stream>>>(s->g, settings->coefficient, rx, ry, chunk->density,
                                                        chunk->energy, chunk->u0, chunk->u, chunk->kx, chunk->ky));
}

// 2d/kernel_interface.h:54 (jacobi.c:60-101). The L1 change is ASSIGNED to
// *error, as the reference kernel does (jacobi.c:100).
void run_jacobi_iterate(Chunk* chunk, Settings* settings, double* error)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->r, chunk->u, sizeof(double) * (size_t)chunk->x * chunk->y,
                            cudaMemcpyDeviceToDevice, s->stream));
    TL_LAUNCH(s, "k_jacobi_iterate", k_jacobi_iterate<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->kx, chunk->ky, chunk->u0, chunk->u,
                                                               chunk->r, s->rs));
    double o;
    if (fetch(s, 1, &o)) *error = o;
}

// ------------------------------------------------------------ PPCG kernels --
// 2d/kernel_interface.h:58 (ppcg.c:9-26)
void run_ppcg_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_ppcg_init", k_ppcg_init<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->theta, chunk->r, chunk->sd));
}

// 2d/kernel_interface.h:60 (ppcg.c:29-61)
void run_ppcg_inner_iteration(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_ppcg_inner_a", k_ppcg_inner_a<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->r, chunk->kx, chunk->ky,
                                                             chunk->sd));
    TL_LAUNCH(s, "k_ppcg_inner_b", k_ppcg_inner_b<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, alpha, beta, chunk->sd, chunk->r));
}

// ---------------------------------------------------------- shared kernels --
// 2d/kernel_interface.h:64 (solver_methods.c:9-25)
void run_copy_u(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_copy_u", k_copy_u<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u0, chunk->u));
}

// 2d/kernel_interface.h:66 (solver_methods.c:28-48)
void run_calculate_residual(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_residual", k_residual<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->u0, chunk->r, chunk->kx,
                                                         chunk->ky));
}

// 2d/kernel_interface.h:68 (solver_methods.c:51-71)
void run_calculate_2norm(Chunk* chunk, Settings* settings, FieldBufferType buffer, double* norm)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_norm2", k_norm2<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, buffer, s->rs));
    double o;
    if (fetch(s, 1, &o)) *norm += o;
}

// 2d/kernel_interface.h:70 (solver_methods.c:74-90)
void run_finalise(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_finalise", k_finalise<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->energy, chunk->density, chunk->u));
}

// ------------------------------------------------- host-buffer staging (new) --
static FieldBufferType field_by_id(Chunk* c, int id)
{
    switch (id) {
        case TL2D_DENSITY0: return c->density0;
        case TL2D_DENSITY: return c->density;
        case TL2D_ENERGY0: return c->energy0;
        case TL2D_ENERGY: return c->energy;
        case TL2D_U: return c->u;
        case TL2D_U0: return c->u0;
        case TL2D_P: return c->p;
        case TL2D_R: return c->r;
        case TL2D_MI: return c->mi;
        case TL2D_W: return c->w;
        case TL2D_KX: return c->kx;
        case TL2D_KY: return c->ky;
        case TL2D_SD: return c->sd;
        case TL2D_VOLUME: return c->volume;
        default: return nullptr;
    }
}

void tl2d_upload_field(Chunk* chunk, Settings* settings, int field_id, const double* host, long long count)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    FieldBufferType f = field_by_id(chunk, field_id);
    if (!f || count != (long long)chunk->x * chunk->y) {
        tl::fail(8, "upload: bad field id %d or count %lld", field_id, count);
        return;
    }
    TL_CUDA(cudaMemcpyAsync(f, host, sizeof(double) * count, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

void tl2d_download_field(Chunk* chunk, Settings* settings, int field_id, double* host, long long count)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    FieldBufferType f = field_by_id(chunk, field_id);
    if (!f || count != (long long)chunk->x * chunk->y) {
        tl::fail(8, "download: bad field id %d or count %lld", field_id, count);
        return;
    }
    TL_CUDA(cudaMemcpyAsync(host, f, sizeof(double) * count, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

}  // extern "C"
