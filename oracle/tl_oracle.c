/*
 * tl_oracle.c -- CPU restatement of the TeaLeaf solver path (TEST INFRASTRUCTURE).
 *
 * This is the checker, never the product: only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it. It restates, in plain serial C, the
 * arithmetic of the reference omp3 kernels and the host drivers that sequence
 * them, so that the B200 suite can be compared element by element on small
 * grids and solve by solve on seeded problems.
 *
 * Parity pins (see tests/test_oracle_pins.py): the restatement reproduces
 *   - the reference's own known answers (2d/tea.problems, 3d/tea.problems);
 *   - per-step iteration counts and field summaries of the reference omp3
 *     program compiled in this repository (oracle/_ref, golden fixtures in
 *     tests/golden/).
 *
 * Index convention (2d/shared.h:49-54): index = k + j*x (+ i*x*y in 3D), with
 * x, y, z the allocated extents including halo_depth cells on each side.
 * Floating point: compiled with -ffp-contract=off so every + - * / is one
 * IEEE-rounded operation, in the same order as the reference expressions.
 */
#include <float.h>
#include <math.h>
#include <stdbool.h>
#include <stdlib.h>
#include <string.h>

#define O_CONDUCTIVITY 1
#define O_RECIP_CONDUCTIVITY 2
#define O_JACOBI 0
#define O_CG 1
#define O_CHEBY 2
#define O_PPCG 3

/* Interior loop helpers: rows/columns [lo, hi). */
#define FOR2(j0, j1, k0, k1) for (int j = (j0); j < (j1); ++j) for (int k = (k0); k < (k1); ++k)
#define FOR3(i0, i1, j0, j1, k0, k1) \
    for (int i = (i0); i < (i1); ++i) for (int j = (j0); j < (j1); ++j) for (int k = (k0); k < (k1); ++k)

/* ======================================================================== */
/* 2D kernels                                                                */
/* ======================================================================== */

/* 5-point operator, reference SMVP macro 2d/shared.h:49-54 (same operand order). */
static inline double op2(const double* a, const double* kx, const double* ky, int i, int x)
{
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + x] + ky[i])) * a[i]
         - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
         - (ky[i + x] * a[i + x] + ky[i] * a[i - x]);
}

static inline double conductivity(int coefficient, double density)
{
    return coefficient == O_CONDUCTIVITY ? density : 1.0 / density;
}

/* Face coefficient between two cells, 2d/c_kernels/omp3/cg.c:56-62. */
static inline double face_coef(double r, double wa, double wb)
{
    return r * (wa + wb) / (2.0 * wa * wb);
}

/* set_chunk_data, 2d/c_kernels/omp3/set_chunk_data.c:10-53 */
void o2_set_chunk_data(int x, int y, int hd, double x_min, double y_min, double dx, double dy,
                       double* vx, double* vy, double* cx, double* cy,
                       double* volume, double* x_area, double* y_area)
{
    for (int k = 0; k < x + 1; ++k) vx[k] = x_min + dx * (k - hd);
    for (int j = 0; j < y + 1; ++j) vy[j] = y_min + dy * (j - hd);
    for (int k = 0; k < x; ++k) cx[k] = 0.5 * (vx[k] + vx[k + 1]);
    for (int j = 0; j < y; ++j) cy[j] = 0.5 * (vy[j] + vy[j + 1]);
    for (int n = 0; n < x * y; ++n) { volume[n] = dx * dy; x_area[n] = dy; y_area[n] = dx; }
}

/* set_chunk_state, 2d/c_kernels/omp3/set_chunk_state.c:9-84.
 * states: num_states records of {density, energy, x_min, y_min, x_max, y_max, radius, geometry}. */
typedef struct { double density, energy, x_min, y_min, z_min, x_max, y_max, z_max, radius; int geometry; } OState;

void o2_set_chunk_state(int x, int y, const double* vx, const double* vy, const double* cx, const double* cy,
                        double* density, double* energy0, double* u, int num_states, const OState* st)
{
    for (int n = 0; n < x * y; ++n) { energy0[n] = st[0].energy; density[n] = st[0].density; }
    for (int s = 1; s < num_states; ++s) {
        FOR2(0, y, 0, x) {
            bool hit = false;
            if (st[s].geometry == 0) {
                hit = vx[k + 1] >= st[s].x_min && vx[k] < st[s].x_max &&
                      vy[j + 1] >= st[s].y_min && vy[j] < st[s].y_max;
            } else if (st[s].geometry == 1) {
                double ddx = cx[k] - st[s].x_min, ddy = cy[j] - st[s].y_min;
                hit = sqrt(ddx * ddx + ddy * ddy) <= st[s].radius;
            } else if (st[s].geometry == 2) {
                hit = vx[k] == st[s].x_min && vy[j] == st[s].y_min;
            }
            if (hit) { energy0[k + j * x] = st[s].energy; density[k + j * x] = st[s].density; }
        }
    }
    FOR2(1, y - 1, 1, x - 1) u[k + j * x] = energy0[k + j * x] * density[k + j * x];
}

/* Reflective halo of one field on external faces, 2d/c_kernels/omp3/local_halos.c:66-149.
 * nb: int[4] neighbours (left, right, bottom, top), -1 = external. */
void o2_halo_field(int x, int y, int hd, int depth, const int* nb, double* f)
{
    if (nb[0] == -1) FOR2(hd, y - hd, 0, depth) f[j * x + (hd - k - 1)] = f[j * x + (hd + k)];
    if (nb[1] == -1) FOR2(hd, y - hd, 0, depth) f[j * x + (x - hd + k)] = f[j * x + (x - hd - 1 - k)];
    if (nb[3] == -1) for (int d = 0; d < depth; ++d) for (int k = hd; k < x - hd; ++k)
        f[k + (y - hd + d) * x] = f[k + (y - hd - 1 - d) * x];
    if (nb[2] == -1) for (int d = 0; d < depth; ++d) for (int k = hd; k < x - hd; ++k)
        f[k + (hd - d - 1) * x] = f[k + (hd + d) * x];
}

/* cg_init, 2d/c_kernels/omp3/cg.c:9-85; returns the accumulated r.p */
double o2_cg_init(int x, int y, int hd, int coefficient, double rx, double ry,
                  const double* density, const double* energy,
                  double* u, double* p, double* r, double* w, double* kx, double* ky)
{
    FOR2(0, y, 0, x) { int i = k + j * x; p[i] = 0.0; r[i] = 0.0; u[i] = energy[i] * density[i]; }
    FOR2(1, y - 1, 1, x - 1) { int i = k + j * x; w[i] = conductivity(coefficient, density[i]); }
    FOR2(hd, y - 1, hd, x - 1) {
        int i = k + j * x;
        kx[i] = face_coef(rx, w[i - 1], w[i]);
        ky[i] = face_coef(ry, w[i - x], w[i]);
    }
    double acc = 0.0;
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        w[i] = op2(u, kx, ky, i, x);
        r[i] = u[i] - w[i];
        p[i] = r[i];
        acc += r[i] * p[i];
    }
    return acc;
}

/* cg_calc_w, cg.c:88-113 */
double o2_cg_calc_w(int x, int y, int hd, const double* p, double* w, const double* kx, const double* ky)
{
    double acc = 0.0;
    FOR2(hd, y - hd, hd, x - hd) { int i = k + j * x; w[i] = op2(p, kx, ky, i, x); acc += w[i] * p[i]; }
    return acc;
}

/* cg_calc_ur, cg.c:116-143 */
double o2_cg_calc_ur(int x, int y, int hd, double alpha, double* u, const double* p, double* r, const double* w)
{
    double acc = 0.0;
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        u[i] += alpha * p[i];
        r[i] -= alpha * w[i];
        acc += r[i] * r[i];
    }
    return acc;
}

/* cg_calc_p, cg.c:146-164 */
void o2_cg_calc_p(int x, int y, int hd, double beta, double* p, const double* r)
{
    FOR2(hd, y - hd, hd, x - hd) { int i = k + j * x; p[i] = beta * p[i] + r[i]; }
}

/* cheby_init + cheby_calc_u, 2d/c_kernels/omp3/cheby.c:8-54 */
void o2_cheby_init(int x, int y, int hd, double theta, double* u, const double* u0, double* p, double* r,
                   double* w, const double* kx, const double* ky)
{
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        w[i] = op2(u, kx, ky, i, x);
        r[i] = u0[i] - w[i];
        p[i] = r[i] / theta;
    }
    FOR2(hd, y - hd, hd, x - hd) u[k + j * x] += p[k + j * x];
}

/* cheby_iterate, cheby.c:57-85 */
void o2_cheby_iterate(int x, int y, int hd, double alpha, double beta, double* u, const double* u0,
                      double* p, double* r, double* w, const double* kx, const double* ky)
{
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        w[i] = op2(u, kx, ky, i, x);
        r[i] = u0[i] - w[i];
        p[i] = alpha * p[i] + beta * r[i];
    }
    FOR2(hd, y - hd, hd, x - hd) u[k + j * x] += p[k + j * x];
}

/* ppcg_init, 2d/c_kernels/omp3/ppcg.c:9-26 */
void o2_ppcg_init(int x, int y, int hd, double theta, const double* r, double* sd)
{
    FOR2(hd, y - hd, hd, x - hd) sd[k + j * x] = r[k + j * x] / theta;
}

/* ppcg_inner_iteration, ppcg.c:29-61 */
void o2_ppcg_inner(int x, int y, int hd, double alpha, double beta, double* u, double* r,
                   const double* kx, const double* ky, double* sd)
{
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        double smvp = op2(sd, kx, ky, i, x);
        r[i] -= smvp;
        u[i] += sd[i];
    }
    FOR2(hd, y - hd, hd, x - hd) { int i = k + j * x; sd[i] = alpha * sd[i] + beta * r[i]; }
}

/* jacobi_init, 2d/c_kernels/omp3/jacobi.c:10-57 */
void o2_jacobi_init(int x, int y, int hd, int coefficient, double rx, double ry, const double* density,
                    const double* energy, double* u0, double* u, double* kx, double* ky)
{
    FOR2(1, y - 1, 1, x - 1) { int i = k + j * x; double t = energy[i] * density[i]; u0[i] = t; u[i] = t; }
    FOR2(hd, y - 1, hd, x - 1) {
        int i = k + j * x;
        double c = conductivity(coefficient, density[i]);
        double l = conductivity(coefficient, density[i - 1]);
        double d = conductivity(coefficient, density[i - x]);
        kx[i] = rx * (l + c) / (2.0 * l * c);
        ky[i] = ry * (d + c) / (2.0 * d * c);
    }
}

/* jacobi_iterate, jacobi.c:60-101; returns the L1 change (assigned, not accumulated) */
double o2_jacobi_iterate(int x, int y, int hd, const double* kx, const double* ky, const double* u0,
                         double* u, double* r)
{
    for (int n = 0; n < x * y; ++n) r[n] = u[n];
    double err = 0.0;
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        u[i] = (u0[i] + (kx[i + 1] * r[i + 1] + kx[i] * r[i - 1]) + (ky[i + x] * r[i + x] + ky[i] * r[i - x]))
             / (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + x]));
        err += fabs(u[i] - r[i]);
    }
    return err;
}

/* solver_methods.c:9-91 */
void o2_copy_u(int x, int y, int hd, double* u0, const double* u)
{
    FOR2(hd, y - hd, hd, x - hd) u0[k + j * x] = u[k + j * x];
}
void o2_calculate_residual(int x, int y, int hd, const double* u, const double* u0, double* r,
                           const double* kx, const double* ky)
{
    FOR2(hd, y - hd, hd, x - hd) { int i = k + j * x; r[i] = u0[i] - op2(u, kx, ky, i, x); }
}
double o2_calculate_2norm(int x, int y, int hd, const double* b)
{
    double acc = 0.0;
    FOR2(hd, y - hd, hd, x - hd) acc += b[k + j * x] * b[k + j * x];
    return acc;
}
void o2_finalise(int x, int y, int hd, double* energy, const double* density, const double* u)
{
    FOR2(hd, y - hd, hd, x - hd) energy[k + j * x] = u[k + j * x] / density[k + j * x];
}
/* field_summary.c:8-45; out[4] = {vol, mass, ie, temp} accumulated */
void o2_field_summary(int x, int y, int hd, const double* volume, const double* density,
                      const double* energy0, const double* u, double* out)
{
    double v = 0.0, m = 0.0, ie = 0.0, t = 0.0;
    FOR2(hd, y - hd, hd, x - hd) {
        int i = k + j * x;
        double cv = volume[i], cm = cv * density[i];
        v += cv; m += cm; ie += cm * energy0[i]; t += cm * u[i];
    }
    out[0] += v; out[1] += m; out[2] += ie; out[3] += t;
}

/* ======================================================================== */
/* 3D kernels (3d/c_kernels/omp3)                                           */
/* ======================================================================== */

/* 7-point operator, 3d/shared.h:52-58 */
static inline double op3(const double* a, const double* kx, const double* ky, const double* kz,
                         long i, int x, long xy)
{
    return (1.0 + (kx[i + 1] + kx[i]) + (ky[i + x] + ky[i]) + (kz[i + xy] + kz[i])) * a[i]
         - (kx[i + 1] * a[i + 1] + kx[i] * a[i - 1])
         - (ky[i + x] * a[i + x] + ky[i] * a[i - x])
         - (kz[i + xy] * a[i + xy] + kz[i] * a[i - xy]);
}
#define I3(k, j, i) ((long)(i) * xy + (long)(j) * x + (k))

void o3_set_chunk_data(int x, int y, int z, int hd, double x_min, double y_min, double z_min,
                       double dx, double dy, double dz, double* vx, double* vy, double* vz,
                       double* cx, double* cy, double* cz, double* volume, double* x_area,
                       double* y_area, double* z_area)
{
    for (int k = 0; k < x + 1; ++k) vx[k] = x_min + dx * (k - hd);
    for (int j = 0; j < y + 1; ++j) vy[j] = y_min + dy * (j - hd);
    for (int i = 0; i < z + 1; ++i) vz[i] = z_min + dz * (i - hd);
    for (int k = 0; k < x; ++k) cx[k] = 0.5 * (vx[k] + vx[k + 1]);
    for (int j = 0; j < y; ++j) cy[j] = 0.5 * (vy[j] + vy[j + 1]);
    for (int i = 0; i < z; ++i) cz[i] = 0.5 * (vz[i] + vz[i + 1]);
    long n = (long)x * y * z;
    for (long q = 0; q < n; ++q) {
        volume[q] = dx * dy * dz; x_area[q] = dy * dz; y_area[q] = dx * dz; z_area[q] = dx * dy;
    }
}

/* 3d/c_kernels/omp3/set_chunk_state.c:9-98 (cuboid 0, spherical 1, point 2) */
void o3_set_chunk_state(int x, int y, int z, const double* vx, const double* vy, const double* vz,
                        const double* cx, const double* cy, const double* cz, double* density,
                        double* energy0, double* u, int num_states, const OState* st)
{
    long xy = (long)x * y, n = xy * z;
    for (long q = 0; q < n; ++q) { energy0[q] = st[0].energy; density[q] = st[0].density; }
    for (int s = 1; s < num_states; ++s) {
        FOR3(0, z, 0, y, 0, x) {
            bool hit = false;
            if (st[s].geometry == 0) {
                hit = vx[k + 1] >= st[s].x_min && vx[k] < st[s].x_max &&
                      vy[j + 1] >= st[s].y_min && vy[j] < st[s].y_max &&
                      vz[i + 1] >= st[s].z_min && vz[i] < st[s].z_max;
            } else if (st[s].geometry == 1) {
                double a = cx[k] - st[s].x_min, b = cy[j] - st[s].y_min, c = cz[i] - st[s].z_min;
                hit = sqrt(a * a + b * b + c * c) <= st[s].radius;
            } else if (st[s].geometry == 2) {
                hit = vx[k] == st[s].x_min && vy[j] == st[s].y_min && vz[i] == st[s].z_min;
            }
            if (hit) { energy0[I3(k, j, i)] = st[s].energy; density[I3(k, j, i)] = st[s].density; }
        }
    }
    FOR3(1, z - 1, 1, y - 1, 1, x - 1) u[I3(k, j, i)] = energy0[I3(k, j, i)] * density[I3(k, j, i)];
}

/* 3d/c_kernels/omp3/local_halos.c: faces left,right,bottom,top,back,front; nb int[6] */
void o3_halo_field(int x, int y, int z, int hd, int depth, const int* nb, double* f)
{
    long xy = (long)x * y;
    if (nb[0] == -1) FOR3(hd, z - hd, hd, y - hd, 0, depth) f[I3(hd - k - 1, j, i)] = f[I3(hd + k, j, i)];
    if (nb[1] == -1) FOR3(hd, z - hd, hd, y - hd, 0, depth) f[I3(x - hd + k, j, i)] = f[I3(x - hd - 1 - k, j, i)];
    if (nb[3] == -1) FOR3(hd, z - hd, 0, depth, hd, x - hd) f[I3(k, y - hd + j, i)] = f[I3(k, y - hd - 1 - j, i)];
    if (nb[2] == -1) FOR3(hd, z - hd, 0, depth, hd, x - hd) f[I3(k, hd - j - 1, i)] = f[I3(k, hd + j, i)];
    if (nb[5] == -1) FOR3(0, depth, hd, y - hd, hd, x - hd) f[I3(k, j, z - hd + i)] = f[I3(k, j, z - hd - 1 - i)];
    if (nb[4] == -1) FOR3(0, depth, hd, y - hd, hd, x - hd) f[I3(k, j, hd - i - 1)] = f[I3(k, j, hd + i)];
}

/* 3d/c_kernels/omp3/cg_solver.c:9-102 */
double o3_cg_init(int x, int y, int z, int hd, int coefficient, double rx, double ry, double rz,
                  const double* density, const double* energy, double* u, double* p, double* r,
                  double* w, double* kx, double* ky, double* kz)
{
    long xy = (long)x * y;
    FOR3(0, z, 0, y, 0, x) { long q = I3(k, j, i); p[q] = 0.0; r[q] = 0.0; u[q] = energy[q] * density[q]; }
    FOR3(1, z - 1, 1, y - 1, 1, x - 1) { long q = I3(k, j, i); w[q] = conductivity(coefficient, density[q]); }
    FOR3(hd, z - 1, hd, y - 1, hd, x - 1) {
        long q = I3(k, j, i);
        kx[q] = face_coef(rx, w[q - 1], w[q]);
        ky[q] = face_coef(ry, w[q - x], w[q]);
        kz[q] = face_coef(rz, w[q - xy], w[q]);
    }
    double acc = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        w[q] = op3(u, kx, ky, kz, q, x, xy);
        r[q] = u[q] - w[q];
        p[q] = r[q];
        acc += r[q] * p[q];
    }
    return acc;
}

double o3_cg_calc_w(int x, int y, int z, int hd, const double* p, double* w, const double* kx,
                    const double* ky, const double* kz)
{
    long xy = (long)x * y;
    double acc = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        w[q] = op3(p, kx, ky, kz, q, x, xy);
        acc += w[q] * p[q];
    }
    return acc;
}

double o3_cg_calc_ur(int x, int y, int z, int hd, double alpha, double* u, const double* p, double* r,
                     const double* w)
{
    long xy = (long)x * y;
    double acc = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        u[q] += alpha * p[q];
        r[q] -= alpha * w[q];
        acc += r[q] * r[q];
    }
    return acc;
}

void o3_cg_calc_p(int x, int y, int z, int hd, double beta, double* p, const double* r)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) { long q = I3(k, j, i); p[q] = beta * p[q] + r[q]; }
}

void o3_cheby_init(int x, int y, int z, int hd, double theta, double* u, const double* u0, double* p,
                   double* r, double* w, const double* kx, const double* ky, const double* kz)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        w[q] = op3(u, kx, ky, kz, q, x, xy);
        r[q] = u0[q] - w[q];
        p[q] = r[q] / theta;
    }
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) u[I3(k, j, i)] += p[I3(k, j, i)];
}

void o3_cheby_iterate(int x, int y, int z, int hd, double alpha, double beta, double* u, const double* u0,
                      double* p, double* r, double* w, const double* kx, const double* ky, const double* kz)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        w[q] = op3(u, kx, ky, kz, q, x, xy);
        r[q] = u0[q] - w[q];
        p[q] = alpha * p[q] + beta * r[q];
    }
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) u[I3(k, j, i)] += p[I3(k, j, i)];
}

void o3_ppcg_init(int x, int y, int z, int hd, double theta, const double* r, double* sd)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) sd[I3(k, j, i)] = r[I3(k, j, i)] / theta;
}

void o3_ppcg_inner(int x, int y, int z, int hd, double alpha, double beta, double* u, double* r,
                   const double* kx, const double* ky, const double* kz, double* sd)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        double smvp = op3(sd, kx, ky, kz, q, x, xy);
        r[q] -= smvp;
        u[q] += sd[q];
    }
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) { long q = I3(k, j, i); sd[q] = alpha * sd[q] + beta * r[q]; }
}

void o3_jacobi_init(int x, int y, int z, int hd, int coefficient, double rx, double ry, double rz,
                    const double* density, const double* energy, double* u0, double* u,
                    double* kx, double* ky, double* kz)
{
    long xy = (long)x * y;
    FOR3(1, z - 1, 1, y - 1, 1, x - 1) { long q = I3(k, j, i); double t = energy[q] * density[q]; u0[q] = t; u[q] = t; }
    FOR3(hd, z - 1, hd, y - 1, hd, x - 1) {
        long q = I3(k, j, i);
        double c = conductivity(coefficient, density[q]);
        double l = conductivity(coefficient, density[q - 1]);
        double d = conductivity(coefficient, density[q - x]);
        double b = conductivity(coefficient, density[q - xy]);
        kx[q] = rx * (l + c) / (2.0 * l * c);
        ky[q] = ry * (d + c) / (2.0 * d * c);
        kz[q] = rz * (b + c) / (2.0 * b * c);
    }
}

double o3_jacobi_iterate(int x, int y, int z, int hd, const double* kx, const double* ky, const double* kz,
                         const double* u0, double* u, double* r)
{
    long xy = (long)x * y, n = xy * z;
    for (long q = 0; q < n; ++q) r[q] = u[q];
    double err = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        u[q] = (u0[q] + (kx[q + 1] * r[q + 1] + kx[q] * r[q - 1]) + (ky[q + x] * r[q + x] + ky[q] * r[q - x])
                + (kz[q + xy] * r[q + xy] + kz[q] * r[q - xy]))
             / (1.0 + (kx[q] + kx[q + 1]) + (ky[q] + ky[q + x]) + (kz[q] + kz[q + xy]));
        err += fabs(u[q] - r[q]);
    }
    return err;
}

void o3_copy_u(int x, int y, int z, int hd, double* u0, const double* u)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) u0[I3(k, j, i)] = u[I3(k, j, i)];
}
void o3_calculate_residual(int x, int y, int z, int hd, const double* u, const double* u0, double* r,
                           const double* kx, const double* ky, const double* kz)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) { long q = I3(k, j, i); r[q] = u0[q] - op3(u, kx, ky, kz, q, x, xy); }
}
double o3_calculate_2norm(int x, int y, int z, int hd, const double* b)
{
    long xy = (long)x * y;
    double acc = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) acc += b[I3(k, j, i)] * b[I3(k, j, i)];
    return acc;
}
void o3_finalise(int x, int y, int z, int hd, double* energy, const double* density, const double* u)
{
    long xy = (long)x * y;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) energy[I3(k, j, i)] = u[I3(k, j, i)] / density[I3(k, j, i)];
}
void o3_field_summary(int x, int y, int z, int hd, const double* volume, const double* density,
                      const double* energy0, const double* u, double* out)
{
    long xy = (long)x * y;
    double v = 0.0, m = 0.0, ie = 0.0, t = 0.0;
    FOR3(hd, z - hd, hd, y - hd, hd, x - hd) {
        long q = I3(k, j, i);
        double cv = volume[q], cm = cv * density[q];
        v += cv; m += cm; ie += cm * energy0[q]; t += cm * u[q];
    }
    out[0] += v; out[1] += m; out[2] += ie; out[3] += t;
}

/* ======================================================================== */
/* Host maths of the drivers                                                */
/* ======================================================================== */

static double sign_of(double a, double b) { return b < 0 ? -fabs(a) : fabs(a); }

/* Eigenvalues of a symmetric tridiagonal matrix by the implicit QL method
 * with shifts (the published "tqli" algorithm; the reference adapts the
 * Numerical Recipes routine, 2d/drivers/eigenvalue_driver.c:71-121).
 * d: diagonal (n), overwritten by eigenvalues; e: sub-diagonal with e[i]
 * coupling rows i-1 and i (e[0] unused). Returns 0, or -1 after 30 sweeps. */
int o_tridiag_eigenvalues(double* d, double* e, int n)
{
    for (int i = 0; i < n - 1; ++i) e[i] = e[i + 1];
    e[n - 1] = 0.0;
    for (int l = 0; l < n; ++l) {
        int sweeps = 0;
        int m;
        for (;;) {
            for (m = l; m < n - 1; ++m) {
                double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) + dd == dd) break;
            }
            if (m == l) break;
            if (sweeps++ == 30) return -1;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = sqrt((g * g) + 1.0);
            g = d[m] - d[l] + e[l] / (g + sign_of(r, g));
            double s = 1.0, c = 1.0, p = 0.0;
            int i;
            for (i = m - 1; i >= l; --i) {
                double f = s * e[i];
                double b = c * e[i];
                r = sqrt(f * f + g * g);
                e[i + 1] = r;
                if (r == 0.0) { d[i + 1] -= p; e[m] = 0.0; continue; }
                s = f / r;
                c = g / r;
                g = d[i + 1] - p;
                r = (d[i] - g) * s + 2.0 * c * b;
                p = s * r;
                d[i + 1] = g + p;
                g = c * r - b;
            }
            d[l] = d[l] - p;
            e[l] = g;
            e[m] = 0.0;
        }
    }
    return 0;
}

/* Lanczos bounds from CG coefficients, eigenvalue_driver.c:11-67.
 * Returns 0, -1 (tqli failure) or -2 (negative eigenvalue). */
int o_eigenvalue_bounds(const double* cg_alphas, const double* cg_betas, int n, double* eigmin, double* eigmax)
{
    double* d = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    double* e = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
    for (int i = 0; i < n; ++i) {
        d[i] = 1.0 / cg_alphas[i];
        if (i > 0) d[i] += cg_betas[i - 1] / cg_alphas[i - 1];
        if (i < n - 1) e[i + 1] = sqrt(cg_betas[i]) / cg_alphas[i];
    }
    int rc = o_tridiag_eigenvalues(d, e, n);
    double lo = DBL_MAX, hi = DBL_MIN;
    for (int i = 0; i < n; ++i) { lo = d[i] < lo ? d[i] : lo; hi = d[i] > hi ? d[i] : hi; }
    free(d); free(e);
    if (rc) return -1;
    if (lo < 0.0 || hi < 0.0) return -2;
    *eigmin = lo * 0.95;
    *eigmax = hi * 1.05;
    return 0;
}

/* Chebyshev coefficient tables, cheby_driver.c:163-183 */
void o_cheby_coefs(double eigmin, double eigmax, int n, double* theta, double* alphas, double* betas)
{
    *theta = (eigmax + eigmin) / 2.0;
    double delta = (eigmax - eigmin) / 2.0;
    double sigma = *theta / delta;
    double rho_old = 1.0 / sigma;
    for (int i = 0; i < n; ++i) {
        double rho_new = 1.0 / (2.0 * sigma - rho_old);
        alphas[i] = rho_new * rho_old;
        betas[i] = 2.0 * rho_new / delta;
        rho_old = rho_new;
    }
}

/* cheby_calc_est_iterations, cheby_driver.c:146-160 (single-precision logs as in the reference) */
int o_cheby_est_iterations(double eigmin, double eigmax, double error, double bb)
{
    double cn = eigmax / eigmin;
    double it_alpha = DBL_EPSILON * bb / (4.0 * error);
    double gamm = (sqrt(cn) - 1.0) / (sqrt(cn) + 1.0);
    return (int)roundf(logf(it_alpha) / (2.0 * logf(gamm)));
}

/* ======================================================================== */
/* Whole-run drivers (2d/diffuse.c + 2d/drivers, 3d equivalents)            */
/* ======================================================================== */

typedef struct {
    int dims;               /* 2 or 3 */
    int nx, ny, nz;         /* interior cells */
    int halo_depth;
    double xmin, ymin, zmin, xmax, ymax, zmax;
    double dt_init, eps, eps_lim;
    int max_iters, end_step, solver, coefficient, presteps, ppcg_inner_steps;
    int error_switch, check_result, summary_frequency;
    int preconditioner;     /* CG only: 0 none, 1 jac_diag, 2 jac_block (2D) */
} OSettings;

typedef struct {
    int total_iters, cg_iters, cheby_iters, ppcg_iters, jacobi_iters, est_iters;
    double error, eigmin, eigmax, exact_error;
    double vol, mass, ie, temp;
} OStep;

/* Field storage for one chunk. */
typedef struct {
    int dims, x, y, z, hd;
    long n;
    double *density, *energy0, *energy, *u, *u0, *p, *r, *w, *kx, *ky, *kz, *sd, *mi, *volume;
    double *vx, *vy, *vz, *cx, *cy, *cz, *xa, *ya, *za;
    double *cg_alphas, *cg_betas, *cheby_alphas, *cheby_betas;
    double theta, eigmin, eigmax;
    int nb[6];
    bool flags[6];          /* fields_to_exchange: density, energy0, energy1, u, p, sd */
} OChunk;

static double* zalloc(long n) { return (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double)); }

static void oc_halo(OChunk* c, int depth)
{
    bool any = false;
    for (int f = 0; f < 6; ++f) any |= c->flags[f];
    if (!any) return;
    /* update order of local_halos.c:36-45 (independent fields, order immaterial) */
    double* fld[6] = {c->density, c->energy0, c->energy, c->u, c->p, c->sd};
    for (int f = 0; f < 6; ++f) {
        if (!c->flags[f]) continue;
        if (c->dims == 2) o2_halo_field(c->x, c->y, c->hd, depth, c->nb, fld[f]);
        else o3_halo_field(c->x, c->y, c->z, c->hd, depth, c->nb, fld[f]);
    }
}
static void oc_reset_flags(OChunk* c) { for (int f = 0; f < 6; ++f) c->flags[f] = false; }

static double oc_calc_w(OChunk* c)
{
    return c->dims == 2 ? o2_cg_calc_w(c->x, c->y, c->hd, c->p, c->w, c->kx, c->ky)
                        : o3_cg_calc_w(c->x, c->y, c->z, c->hd, c->p, c->w, c->kx, c->ky, c->kz);
}
static double oc_calc_ur(OChunk* c, double alpha)
{
    return c->dims == 2 ? o2_cg_calc_ur(c->x, c->y, c->hd, alpha, c->u, c->p, c->r, c->w)
                        : o3_cg_calc_ur(c->x, c->y, c->z, c->hd, alpha, c->u, c->p, c->r, c->w);
}
static void oc_calc_p(OChunk* c, double beta)
{
    if (c->dims == 2) o2_cg_calc_p(c->x, c->y, c->hd, beta, c->p, c->r);
    else o3_cg_calc_p(c->x, c->y, c->z, c->hd, beta, c->p, c->r);
}
static double oc_2norm(OChunk* c, const double* b)
{
    return c->dims == 2 ? o2_calculate_2norm(c->x, c->y, c->hd, b) : o3_calculate_2norm(c->x, c->y, c->z, c->hd, b);
}
static void oc_residual(OChunk* c)
{
    if (c->dims == 2) o2_calculate_residual(c->x, c->y, c->hd, c->u, c->u0, c->r, c->kx, c->ky);
    else o3_calculate_residual(c->x, c->y, c->z, c->hd, c->u, c->u0, c->r, c->kx, c->ky, c->kz);
}

/* cg_init_driver, 2d/drivers/cg_driver.c:30-62 */
static double oc_cg_init_driver(OChunk* c, const OSettings* s, double rx, double ry, double rz)
{
    double rro = c->dims == 2
        ? o2_cg_init(c->x, c->y, c->hd, s->coefficient, rx, ry, c->density, c->energy, c->u, c->p, c->r, c->w, c->kx, c->ky)
        : o3_cg_init(c->x, c->y, c->z, c->hd, s->coefficient, rx, ry, rz, c->density, c->energy, c->u, c->p, c->r,
                     c->w, c->kx, c->ky, c->kz);
    oc_reset_flags(c);
    c->flags[3] = c->flags[4] = true;
    oc_halo(c, 1);
    if (c->dims == 2) o2_copy_u(c->x, c->y, c->hd, c->u0, c->u);
    else o3_copy_u(c->x, c->y, c->z, c->hd, c->u0, c->u);
    return rro;
}

/* cg_main_step_driver, cg_driver.c:65-124 */
static void oc_cg_main_step(OChunk* c, int tt, double* rro, double* error)
{
    double pw = oc_calc_w(c);
    double alpha = *rro / pw;
    c->cg_alphas[tt] = alpha;
    double rrn = oc_calc_ur(c, alpha);
    double beta = rrn / *rro;
    c->cg_betas[tt] = beta;
    oc_calc_p(c, beta);
    *error = rrn;
    *rro = rrn;
}

/* Solver convergence value: 2D tests rrn, 3D sqrt(rrn) (3d/drivers/cg_solver_driver.c:24-25). */
static void oc_post_trip(OChunk* c, double* error)
{
    if (c->dims == 3) *error = sqrt(*error);
}

static int oc_cg(OChunk* c, const OSettings* s, double rx, double ry, double rz, double* error, OStep* st)
{
    double rro = oc_cg_init_driver(c, s, rx, ry, rz);
    int tt;
    for (tt = 0; tt < s->max_iters; ++tt) {
        oc_cg_main_step(c, tt, &rro, error);
        oc_halo(c, 1);
        oc_post_trip(c, error);
        if (fabs(*error) < s->eps) break;
    }
    st->cg_iters = tt;
    st->total_iters = tt;
    return 0;
}

/* Jacobi preconditioners of CG (2D). The reference C ports only parse
 * preconditioner_on (2d/parse_config.c:136-138) and their kernels ignore it;
 * the README documents jac_diag and jac_block with a block size of 4
 * (README.md:127-133), and the reference's cuda 3D kernel stores the
 * diagonal one as mi = 1 / diag(A) and applies z = mi r
 * (3d/c_kernels/cuda/cg_solver.cuknl:93-100).
 * diag(A) = 1 + (kx_i+1 + kx_i) + (ky_i+x + ky_i). jac_block: M is the
 * tridiagonal part of A within blocks of 4 rows along y that start at the
 * first interior row (the last block of a column may be shorter), with
 * coupling -ky_i between rows i-x and i, solved by Thomas' algorithm; mi
 * holds the inverse pivots g_q = 1 / (d_q + ky_q c_q-1) (c_q-1 = -ky_q g_q-1,
 * g_0 = 1 / d_0), so applying M^-1 takes multiplications only:
 *   forward  y_0 = r_0 g_0,  y_q = (r_q + ky_q y_q-1) g_q
 *   back     z_m-1 = y_m-1,  z_q = y_q - c_q z_q+1,  c_q = -ky_q+1 g_q.
 * Factor once per solve (o2_precond_factor), apply per trip (o2_precond). */
void o2_precond_factor(int x, int y, int hd, int type, const double* kx, const double* ky, double* mi)
{
    const int bs = type == 2 ? 4 : 1;
    for (int k = hd; k < x - hd; ++k) {
        for (int jb = hd; jb < y - hd; jb += bs) {
            const int m = (y - hd - jb) < bs ? (y - hd - jb) : bs;
            double c = 0.0;
            for (int q = 0; q < m; ++q) {
                const long i = k + (long)(jb + q) * x;
                const double d = 1.0 + (kx[i + 1] + kx[i]) + (ky[i + x] + ky[i]);
                const double g = q == 0 ? 1.0 / d : 1.0 / (d + ky[i] * c);
                mi[i] = g;
                c = -ky[i + x] * g;
            }
        }
    }
}

void o2_precond(int x, int y, int hd, int type, const double* ky, const double* mi, const double* r, double* z)
{
    const int bs = type == 2 ? 4 : 1;
    for (int k = hd; k < x - hd; ++k) {
        for (int jb = hd; jb < y - hd; jb += bs) {
            const int m = (y - hd - jb) < bs ? (y - hd - jb) : bs;
            if (type == 1) {
                const long i = k + (long)jb * x;
                z[i] = mi[i] * r[i];
                continue;
            }
            double yv[4];
            for (int q = 0; q < m; ++q) {
                const long i = k + (long)(jb + q) * x;
                yv[q] = q == 0 ? r[i] * mi[i] : (r[i] + ky[i] * yv[q - 1]) * mi[i];
            }
            double zn = yv[m - 1];
            z[k + (long)(jb + m - 1) * x] = zn;
            for (int q = m - 2; q >= 0; --q) {
                const long i = k + (long)(jb + q) * x;
                const double c = -ky[i + x] * mi[i];
                zn = yv[q] - c * zn;
                z[i] = zn;
            }
        }
    }
}

static double o2_dot_interior(int x, int y, int hd, const double* a, const double* b)
{
    double s = 0.0;
    for (int j = hd; j < y - hd; ++j)
        for (int k = hd; k < x - hd; ++k) s += a[k + (long)j * x] * b[k + (long)j * x];
    return s;
}

/* Preconditioned CG (2D): cg_driver.c's loop with z = M^-1 r (M factored
 * into the chunk's mi field, which the reference allocates for its
 * preconditioner; z in sd, unused by CG):
 * after cg_init, z = M^-1 r, p = z (depth-1 reflective halo), rro = r.z; per
 * trip pw = p.w, alpha = rro / pw, u += alpha p, r -= alpha w, z = M^-1 r,
 * beta = r.z / rro, p = beta p + z, rro = r.z; the stop test is on r.r, the
 * error of the unpreconditioned CG, so eps means the same for both. */
static int oc_pcg(OChunk* c, const OSettings* s, double rx, double ry, double rz, double* error, OStep* st)
{
    if (c->dims != 2) return -4;
    oc_cg_init_driver(c, s, rx, ry, rz);
    double* z = c->sd;
    o2_precond_factor(c->x, c->y, c->hd, s->preconditioner, c->kx, c->ky, c->mi);
    o2_precond(c->x, c->y, c->hd, s->preconditioner, c->ky, c->mi, c->r, z);
    for (int j = c->hd; j < c->y - c->hd; ++j)
        for (int k = c->hd; k < c->x - c->hd; ++k) c->p[k + (long)j * c->x] = z[k + (long)j * c->x];
    oc_reset_flags(c);
    c->flags[3] = c->flags[4] = true;
    oc_halo(c, 1);
    double rro = o2_dot_interior(c->x, c->y, c->hd, c->r, z);
    int tt;
    for (tt = 0; tt < s->max_iters; ++tt) {
        const double pw = oc_calc_w(c);
        const double alpha = rro / pw;
        c->cg_alphas[tt] = alpha;
        const double rrn = oc_calc_ur(c, alpha);
        o2_precond(c->x, c->y, c->hd, s->preconditioner, c->ky, c->mi, c->r, z);
        const double rzn = o2_dot_interior(c->x, c->y, c->hd, c->r, z);
        const double beta = rzn / rro;
        c->cg_betas[tt] = beta;
        o2_cg_calc_p(c->x, c->y, c->hd, beta, c->p, z);
        rro = rzn;
        *error = rrn;
        oc_halo(c, 1);
        if (fabs(*error) < s->eps) break;
    }
    st->cg_iters = tt;
    st->total_iters = tt;
    return 0;
}

static bool oc_switch(const OSettings* s, int n_inner, int tt, double error)
{
    return n_inner || (s->error_switch ? (error < s->eps_lim) && (tt > 20)
                                       : (tt > s->presteps) && (error < 1.0));
}

/* cheby_driver, 2d/drivers/cheby_driver.c:11-143 */
static int oc_cheby(OChunk* c, const OSettings* s, double rx, double ry, double rz, double* error, OStep* st)
{
    double rro = oc_cg_init_driver(c, s, rx, ry, rz);
    int est = 0, nch = 0, tt;
    for (tt = 0; tt < s->max_iters; ++tt) {
        if (!oc_switch(s, nch, tt, *error)) {
            oc_cg_main_step(c, tt, &rro, error);
        } else {
            ++nch;
            bool norm = true;
            if (nch == 1) {
                int rc = o_eigenvalue_bounds(c->cg_alphas, c->cg_betas, tt, &c->eigmin, &c->eigmax);
                if (rc) return rc;
                o_cheby_coefs(c->eigmin, c->eigmax, s->max_iters - tt, &c->theta, c->cheby_alphas, c->cheby_betas);
                double bb = oc_2norm(c, c->u0);
                if (c->dims == 2) o2_cheby_init(c->x, c->y, c->hd, c->theta, c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky);
                else o3_cheby_init(c->x, c->y, c->z, c->hd, c->theta, c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky, c->kz);
                oc_reset_flags(c);
                c->flags[3] = true;
                oc_halo(c, 1);
                /* first main step always takes the norm */
                if (c->dims == 2)
                    o2_cheby_iterate(c->x, c->y, c->hd, c->cheby_alphas[nch], c->cheby_betas[nch], c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky);
                else
                    o3_cheby_iterate(c->x, c->y, c->z, c->hd, c->cheby_alphas[nch], c->cheby_betas[nch], c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky, c->kz);
                *error = oc_2norm(c, c->r);
                est = o_cheby_est_iterations(c->eigmin, c->eigmax, *error, bb);
                norm = false;
            } else {
                norm = (nch >= est) && ((tt + 1) % 10 == 0);
                if (c->dims == 2)
                    o2_cheby_iterate(c->x, c->y, c->hd, c->cheby_alphas[nch], c->cheby_betas[nch], c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky);
                else
                    o3_cheby_iterate(c->x, c->y, c->z, c->hd, c->cheby_alphas[nch], c->cheby_betas[nch], c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky, c->kz);
                if (norm) *error = oc_2norm(c, c->r);
            }
        }
        oc_halo(c, 1);
        oc_post_trip(c, error);
        if (fabs(*error) < s->eps) break;
    }
    st->cg_iters = tt - nch + 1;
    st->cheby_iters = nch;
    st->est_iters = est;
    st->total_iters = tt;
    st->eigmin = c->eigmin;
    st->eigmax = c->eigmax;
    return 0;
}

/* ppcg_driver, 2d/drivers/ppcg_driver.c:10-189 */
static int oc_ppcg(OChunk* c, const OSettings* s, double rx, double ry, double rz, double* error, OStep* st)
{
    double rro = oc_cg_init_driver(c, s, rx, ry, rz);
    int npp = 0, tt;
    for (tt = 0; tt < s->max_iters; ++tt) {
        if (!oc_switch(s, npp, tt, *error)) {
            oc_cg_main_step(c, tt, &rro, error);
        } else {
            ++npp;
            if (npp == 1) {
                int rc = o_eigenvalue_bounds(c->cg_alphas, c->cg_betas, tt, &c->eigmin, &c->eigmax);
                if (rc) return rc;
                o_cheby_coefs(c->eigmin, c->eigmax, s->ppcg_inner_steps, &c->theta, c->cheby_alphas, c->cheby_betas);
                oc_residual(c);
                oc_reset_flags(c);
                c->flags[4] = true;
                oc_halo(c, 1);
            }
            double pw = oc_calc_w(c);
            double alpha = rro / pw;
            (void)oc_calc_ur(c, alpha);
            /* inner iterations, ppcg_driver.c:152-189 */
            if (c->dims == 2) o2_ppcg_init(c->x, c->y, c->hd, c->theta, c->r, c->sd);
            else o3_ppcg_init(c->x, c->y, c->z, c->hd, c->theta, c->r, c->sd);
            oc_reset_flags(c);
            c->flags[5] = true;
            for (int pp = 0; pp < s->ppcg_inner_steps; ++pp) {
                oc_halo(c, 1);
                if (c->dims == 2)
                    o2_ppcg_inner(c->x, c->y, c->hd, c->cheby_alphas[pp], c->cheby_betas[pp], c->u, c->r, c->kx, c->ky, c->sd);
                else
                    o3_ppcg_inner(c->x, c->y, c->z, c->hd, c->cheby_alphas[pp], c->cheby_betas[pp], c->u, c->r, c->kx, c->ky, c->kz, c->sd);
            }
            oc_reset_flags(c);
            c->flags[4] = true;
            double rrn = oc_2norm(c, c->r);
            double beta = rrn / rro;
            oc_calc_p(c, beta);
            *error = rrn;
            rro = rrn;
        }
        oc_halo(c, 1);
        oc_post_trip(c, error);
        if (fabs(*error) < s->eps) break;
    }
    st->cg_iters = tt - npp + 1;
    st->ppcg_iters = npp;
    st->total_iters = tt;
    st->eigmin = c->eigmin;
    st->eigmax = c->eigmax;
    return 0;
}

/* jacobi_driver, 2d/drivers/jacobi_driver.c:7-83 */
static int oc_jacobi(OChunk* c, const OSettings* s, double rx, double ry, double rz, double* error, OStep* st)
{
    if (c->dims == 2) {
        o2_jacobi_init(c->x, c->y, c->hd, s->coefficient, rx, ry, c->density, c->energy, c->u0, c->u, c->kx, c->ky);
        o2_copy_u(c->x, c->y, c->hd, c->u0, c->u);
    } else {
        o3_jacobi_init(c->x, c->y, c->z, c->hd, s->coefficient, rx, ry, rz, c->density, c->energy, c->u0, c->u, c->kx, c->ky, c->kz);
        o3_copy_u(c->x, c->y, c->z, c->hd, c->u0, c->u);
    }
    oc_reset_flags(c);
    c->flags[3] = true;
    int tt;
    for (tt = 0; tt < s->max_iters; ++tt) {
        *error = c->dims == 2 ? o2_jacobi_iterate(c->x, c->y, c->hd, c->kx, c->ky, c->u0, c->u, c->r)
                              : o3_jacobi_iterate(c->x, c->y, c->z, c->hd, c->kx, c->ky, c->kz, c->u0, c->u, c->r);
        if (tt % 50 == 0) {
            oc_halo(c, 1);
            oc_residual(c);
            *error += oc_2norm(c, c->r);
        }
        oc_halo(c, 1);
        oc_post_trip(c, error);
        if (fabs(*error) < s->eps) break;
    }
    st->jacobi_iters = tt;
    st->total_iters = tt;
    return 0;
}

static void oc_summary(OChunk* c, double* out)
{
    out[0] = out[1] = out[2] = out[3] = 0.0;
    if (c->dims == 2) o2_field_summary(c->x, c->y, c->hd, c->volume, c->density, c->energy0, c->u, out);
    else o3_field_summary(c->x, c->y, c->z, c->hd, c->volume, c->density, c->energy0, c->u, out);
}

/* initialise_application (2d/initialise.c:11-31) for one chunk with every
 * face external (NO_MPI, 1 rank): allocation, mesh, states, halos, store_energy. */
static void oc_setup(OChunk* c, const OSettings* s, const OState* states, int num_states, double* dxyz)
{
    memset(c, 0, sizeof(*c));
    c->dims = s->dims;
    c->hd = s->halo_depth;
    c->x = s->nx + 2 * c->hd;
    c->y = s->ny + 2 * c->hd;
    c->z = s->dims == 3 ? s->nz + 2 * c->hd : 1;
    c->n = (long)c->x * c->y * c->z;
    for (int f = 0; f < 6; ++f) c->nb[f] = -1;
    c->density = zalloc(c->n); c->energy0 = zalloc(c->n); c->energy = zalloc(c->n); c->u = zalloc(c->n);
    c->u0 = zalloc(c->n); c->p = zalloc(c->n); c->r = zalloc(c->n); c->w = zalloc(c->n); c->kx = zalloc(c->n);
    c->ky = zalloc(c->n); c->kz = zalloc(c->n); c->sd = zalloc(c->n); c->mi = zalloc(c->n); c->volume = zalloc(c->n);
    c->xa = zalloc(c->n + c->y * c->z); c->ya = zalloc(c->n + c->x * c->z); c->za = zalloc(c->n + c->x * c->y);
    c->vx = zalloc(c->x + 1); c->vy = zalloc(c->y + 1); c->vz = zalloc(c->z + 1);
    c->cx = zalloc(c->x); c->cy = zalloc(c->y); c->cz = zalloc(c->z);
    c->cg_alphas = zalloc(s->max_iters); c->cg_betas = zalloc(s->max_iters);
    c->cheby_alphas = zalloc(s->max_iters); c->cheby_betas = zalloc(s->max_iters);

    double dx = (s->xmax - s->xmin) / (double)s->nx;
    double dy = (s->ymax - s->ymin) / (double)s->ny;
    double dz = s->dims == 3 ? (s->zmax - s->zmin) / (double)s->nz : 1.0;
    dxyz[0] = dx; dxyz[1] = dy; dxyz[2] = dz;
    if (s->dims == 2) {
        o2_set_chunk_data(c->x, c->y, c->hd, s->xmin, s->ymin, dx, dy, c->vx, c->vy, c->cx, c->cy, c->volume, c->xa, c->ya);
        o2_set_chunk_state(c->x, c->y, c->vx, c->vy, c->cx, c->cy, c->density, c->energy0, c->u, num_states, states);
    } else {
        o3_set_chunk_data(c->x, c->y, c->z, c->hd, s->xmin, s->ymin, s->zmin, dx, dy, dz, c->vx, c->vy, c->vz,
                          c->cx, c->cy, c->cz, c->volume, c->xa, c->ya, c->za);
        o3_set_chunk_state(c->x, c->y, c->z, c->vx, c->vy, c->vz, c->cx, c->cy, c->cz, c->density, c->energy0,
                           c->u, num_states, states);
    }
    oc_reset_flags(c);
    c->flags[0] = c->flags[1] = c->flags[2] = true;
    oc_halo(c, 2);
    memcpy(c->energy, c->energy0, sizeof(double) * (size_t)c->n);   /* store_energy */
}

static void oc_free(OChunk* c)
{
    double* f[] = {c->density, c->energy0, c->energy, c->u, c->u0, c->p, c->r, c->w, c->kx, c->ky, c->kz,
                   c->sd, c->mi, c->volume, c->xa, c->ya, c->za, c->vx, c->vy, c->vz, c->cx, c->cy, c->cz,
                   c->cg_alphas, c->cg_betas, c->cheby_alphas, c->cheby_betas};
    for (size_t k = 0; k < sizeof(f) / sizeof(f[0]); ++k) free(f[k]);
}

/* One solve() (2d/diffuse.c:22-80): halos, the solver driver,
 * solve_finished_driver, field summary. */
static int oc_step(OChunk* c, const OSettings* s, const double* dxyz, OStep* st)
{
    memset(st, 0, sizeof(*st));
    double dt = s->dt_init;
    double rx = dt / (dxyz[0] * dxyz[0]), ry = dt / (dxyz[1] * dxyz[1]), rz = dt / (dxyz[2] * dxyz[2]);
    oc_reset_flags(c);
    c->flags[2] = c->flags[0] = true;
    oc_halo(c, 2);
    double error = 1e+10;
    int rc;
    switch (s->solver) {
        case O_JACOBI: rc = oc_jacobi(c, s, rx, ry, rz, &error, st); break;
        case O_CG: rc = s->preconditioner ? oc_pcg(c, s, rx, ry, rz, &error, st) : oc_cg(c, s, rx, ry, rz, &error, st); break;
        case O_CHEBY: rc = oc_cheby(c, s, rx, ry, rz, &error, st); break;
        case O_PPCG: rc = oc_ppcg(c, s, rx, ry, rz, &error, st); break;
        default: rc = -3;
    }
    if (rc) return rc;
    st->error = error;
    /* solve_finished_driver, 2d/drivers/solve_finished_driver.c:7-43 */
    if (s->check_result) {
        oc_residual(c);
        st->exact_error = oc_2norm(c, c->r);
    }
    if (c->dims == 2) o2_finalise(c->x, c->y, c->hd, c->energy, c->density, c->u);
    else o3_finalise(c->x, c->y, c->z, c->hd, c->energy, c->density, c->u);
    c->flags[2] = true;
    oc_halo(c, 1);
    double out[4];
    oc_summary(c, out);
    st->vol = out[0]; st->mass = out[1]; st->ie = out[2]; st->temp = out[3];
    return 0;
}

/* Runs initialise_application + end_step x solve() (2d/initialise.c:11-31,
 * 2d/diffuse.c:10-80). One chunk, every face external (NO_MPI, 1 rank).
 * steps_out[end_step]; energy_out (nullable) receives the final energy field
 * (x*y[*z] values). Returns 0, or a negative driver failure code. */
int oracle_run(const OSettings* s, const OState* states, int num_states, OStep* steps_out, double* energy_out)
{
    OChunk cc;
    OChunk* c = &cc;
    double dxyz[3];
    oc_setup(c, s, states, num_states, dxyz);
    int rc = 0;
    for (int tt = 0; tt < s->end_step && rc == 0; ++tt) rc = oc_step(c, s, dxyz, &steps_out[tt]);
    if (energy_out) memcpy(energy_out, c->energy, sizeof(double) * (size_t)c->n);
    oc_free(c);
    return rc;
}

/* ======================================================================== */
/* FP64 CPU adjoint of the 3D CG timestep (the B200 suite's adjoint3d.cu     */
/* restated serially; the reference has no adjoint). Test infrastructure.    */
/* ======================================================================== */

/* A lam = rhs from lam = 0 by CG (the operator of o3_cg_calc_w with the
 * reflective depth-1 halo of p each trip), to r.r <= tol^2 rhs.rhs. */
static int oa_solve(OChunk* c, const double* rhs, double* lam, double tol, int max_iters)
{
    const long n = c->n;
    const int hd = c->hd;
    double gg = 0.0;
    for (int i3 = 0; i3 < c->z; ++i3)
        for (int j = 0; j < c->y; ++j)
            for (int k = 0; k < c->x; ++k) {
                const long i = k + (long)j * c->x + (long)i3 * c->x * c->y;
                const int in = k >= hd && k < c->x - hd && j >= hd && j < c->y - hd && i3 >= hd && i3 < c->z - hd;
                const double v = in ? rhs[i] : 0.0;
                c->r[i] = v;
                c->p[i] = v;
                gg += v * v;
            }
    memset(lam, 0, sizeof(double) * (size_t)n);
    if (gg == 0.0) return 0;
    double rro = gg;
    int tt;
    for (tt = 0; tt < max_iters; ++tt) {
        o3_halo_field(c->x, c->y, c->z, hd, 1, c->nb, c->p);
        const double pw = o3_cg_calc_w(c->x, c->y, c->z, hd, c->p, c->w, c->kx, c->ky, c->kz);
        const double alpha = rro / pw;
        const double rrn = o3_cg_calc_ur(c->x, c->y, c->z, hd, alpha, lam, c->p, c->r, c->w);
        const double beta = rrn / rro;
        o3_cg_calc_p(c->x, c->y, c->z, hd, beta, c->p, c->r);
        rro = rrn;
        if (rrn < tol * tol * gg) { ++tt; break; }
    }
    return tt;
}

/* grad_c -= dk/drho_c sum_{interior nb} r_axis (lam_c - lam_nb)(u_c - u_nb) */
static void oa_face_grad(OChunk* c, int coefficient, double rx, double ry, double rz, const double* lam,
                         const double* u, double* grad)
{
    const int x = c->x, y = c->y, z = c->z, hd = c->hd;
    const long xy = (long)x * y;
    for (int i3 = hd; i3 < z - hd; ++i3)
        for (int j = hd; j < y - hd; ++j)
            for (int k = hd; k < x - hd; ++k) {
                const long i = k + (long)j * x + (long)i3 * xy;
                const double rho = c->density[i];
                const double w = coefficient == O_CONDUCTIVITY ? rho : 1.0 / rho;
                const double dwdrho = coefficient == O_CONDUCTIVITY ? 1.0 : -w * w;
                const double dk = -dwdrho / (2.0 * w * w);
                double sx = 0.0, sy = 0.0, sz = 0.0;
                if (k > hd) sx += (lam[i] - lam[i - 1]) * (u[i] - u[i - 1]);
                if (k < x - hd - 1) sx += (lam[i] - lam[i + 1]) * (u[i] - u[i + 1]);
                if (j > hd) sy += (lam[i] - lam[i - x]) * (u[i] - u[i - x]);
                if (j < y - hd - 1) sy += (lam[i] - lam[i + x]) * (u[i] - u[i + x]);
                if (i3 > hd) sz += (lam[i] - lam[i - xy]) * (u[i] - u[i - xy]);
                if (i3 < z - hd - 1) sz += (lam[i] - lam[i + xy]) * (u[i] - u[i + xy]);
                grad[i] -= dk * (rx * sx + ry * sy + rz * sz);
            }
}

/* J = sum over cells whose centre is in box[6] of volume*density*u after
 * end_step CG timesteps, and dJ/dlog(density) of every interior cell
 * (grad_out: nx*ny*nz, x fastest). Every forward solution is kept (small
 * meshes only). Returns 0 or a negative code. */
int oracle_adjoint3d(const OSettings* s, const OState* states, int num_states, const double* box, double adj_tol,
                     double* J_out, double* grad_out)
{
    if (s->dims != 3 || s->solver != O_CG) return -10;
    OChunk cc;
    OChunk* c = &cc;
    double dxyz[3];
    oc_setup(c, s, states, num_states, dxyz);
    const long n = c->n;
    const int N = s->end_step, hd = c->hd, x = c->x, y = c->y, z = c->z;
    const long xy = (long)x * y;
    double* e0 = zalloc(n);
    memcpy(e0, c->energy, sizeof(double) * (size_t)n);
    double* us = zalloc(n * (long)N);
    int rc = 0;
    for (int tt = 0; tt < N && rc == 0; ++tt) {
        OStep st;
        rc = oc_step(c, s, dxyz, &st);
        memcpy(us + n * (long)tt, c->u, sizeof(double) * (size_t)n);
    }
    double* rhs = zalloc(n);
    double* grad = zalloc(n);
    double* lam = zalloc(n);
    double J = 0.0;
    const double* uN = us + n * (long)(N - 1);
    for (int i3 = hd; i3 < z - hd; ++i3)
        for (int j = hd; j < y - hd; ++j)
            for (int k = hd; k < x - hd; ++k) {
                const double cxv = s->xmin + dxyz[0] * (k - hd + 0.5);
                const double cyv = s->ymin + dxyz[1] * (j - hd + 0.5);
                const double czv = s->zmin + dxyz[2] * (i3 - hd + 0.5);
                if (cxv < box[0] || cxv > box[1] || cyv < box[2] || cyv > box[3] || czv < box[4] || czv > box[5])
                    continue;
                const long i = k + (long)j * x + (long)i3 * xy;
                rhs[i] = c->volume[i] * c->density[i];
                grad[i] = c->volume[i] * uN[i];
                J += rhs[i] * uN[i];
            }
    const double dt = s->dt_init;
    const double rx = dt / (dxyz[0] * dxyz[0]), ry = dt / (dxyz[1] * dxyz[1]), rz = dt / (dxyz[2] * dxyz[2]);
    for (int step = N; step >= 1 && rc == 0; --step) {
        oa_solve(c, rhs, lam, adj_tol, s->max_iters);
        oa_face_grad(c, s->coefficient, rx, ry, rz, lam, us + n * (long)(step - 1), grad);
        memcpy(rhs, lam, sizeof(double) * (size_t)n);
    }
    const long nx = x - 2 * hd, ny = y - 2 * hd;
    for (int i3 = hd; i3 < z - hd; ++i3)
        for (int j = hd; j < y - hd; ++j)
            for (int k = hd; k < x - hd; ++k) {
                const long i = k + (long)j * x + (long)i3 * xy;
                grad_out[(k - hd) + (j - hd) * nx + (i3 - hd) * nx * ny] = c->density[i] * (grad[i] + lam[i] * e0[i]);
            }
    *J_out = J;
    free(e0); free(us); free(rhs); free(grad); free(lam);
    oc_free(c);
    return rc;
}

/* J of oracle_adjoint3d after end_step CG timesteps with density[cell] (an
 * interior index, x fastest) multiplied by exp(log_scale) before the first
 * step; for central differences on the CPU. */
int oracle_objective3d(const OSettings* s, const OState* states, int num_states, const double* box, long cell,
                       double log_scale, double* J_out)
{
    if (s->dims != 3) return -10;
    OChunk cc;
    OChunk* c = &cc;
    double dxyz[3];
    oc_setup(c, s, states, num_states, dxyz);
    const int hd = c->hd, x = c->x, y = c->y, z = c->z;
    const long xy = (long)x * y, nx = x - 2 * hd, ny = y - 2 * hd;
    if (cell >= 0) {
        const long k = cell % nx, j = (cell / nx) % ny, i3 = cell / (nx * ny);
        c->density[(k + hd) + (j + hd) * x + (i3 + hd) * xy] *= exp(log_scale);
    }
    int rc = 0;
    for (int tt = 0; tt < s->end_step && rc == 0; ++tt) {
        OStep st;
        rc = oc_step(c, s, dxyz, &st);
    }
    double J = 0.0;
    for (int i3 = hd; i3 < z - hd; ++i3)
        for (int j = hd; j < y - hd; ++j)
            for (int k = hd; k < x - hd; ++k) {
                const double cxv = s->xmin + dxyz[0] * (k - hd + 0.5);
                const double cyv = s->ymin + dxyz[1] * (j - hd + 0.5);
                const double czv = s->zmin + dxyz[2] * (i3 - hd + 0.5);
                if (cxv < box[0] || cxv > box[1] || cyv < box[2] || cyv > box[3] || czv < box[4] || czv > box[5])
                    continue;
                const long i = k + (long)j * x + (long)i3 * xy;
                J += c->volume[i] * c->density[i] * c->u[i];
            }
    *J_out = J;
    oc_free(c);
    return rc;
}
