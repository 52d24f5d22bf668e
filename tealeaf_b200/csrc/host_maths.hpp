// host_maths.hpp -- host-side maths of the reference solver drivers, shared
// by the 2D and 3D device-resident drivers: Lanczos eigenvalue bounds from the
// CG coefficients, the Chebyshev coefficient tables and the Chebyshev
// iteration estimate (computed on the host, as the reference does, so the
// single-precision logf/roundf of the estimate match it exactly).
#pragma once

#include "common.cuh"

#include <cfloat>
#include <cmath>
#include <vector>

namespace tl {

// Eigenvalues of a symmetric tridiagonal matrix, implicit QL with shifts
// (published "tqli"; the reference adapts it, 2d/drivers/eigenvalue_driver.c:71-121).
inline bool tridiag_ql(std::vector<double>& d, std::vector<double>& e)
{
    const int n = (int)d.size();
    for (int i = 0; i < n - 1; ++i) e[i] = e[i + 1];
    e[n - 1] = 0.0;
    for (int l = 0; l < n; ++l) {
        int sweeps = 0, m;
        for (;;) {
            for (m = l; m < n - 1; ++m) {
                const double dd = fabs(d[m]) + fabs(d[m + 1]);
                if (fabs(e[m]) + dd == dd) break;
            }
            if (m == l) break;
            if (sweeps++ == 30) return false;
            double g = (d[l + 1] - d[l]) / (2.0 * e[l]);
            double r = sqrt((g * g) + 1.0);
            g = d[m] - d[l] + e[l] / (g + (g < 0 ? -fabs(r) : fabs(r)));
            double s = 1.0, c = 1.0, p = 0.0;
            for (int i = m - 1; i >= l; --i) {
                const double f = s * e[i];
                const double b = c * e[i];
                r = sqrt(f * f + g * g);
                e[i + 1] = r;
                if (r == 0.0) {
                    d[i + 1] -= p;
                    e[m] = 0.0;
                    continue;
                }
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
    return true;
}

// eigenvalue_driver_initialise (2d/drivers/eigenvalue_driver.c:11-67)
template <typename ChunkT>
bool eigen_bounds(ChunkT* chunk, int n)
{
    std::vector<double> d(n > 0 ? n : 1, 0.0), e(n > 0 ? n : 1, 0.0);
    for (int i = 0; i < n; ++i) {
        d[i] = 1.0 / chunk->cg_alphas[i];
        if (i > 0) d[i] += chunk->cg_betas[i - 1] / chunk->cg_alphas[i - 1];
        if (i < n - 1) e[i + 1] = sqrt(chunk->cg_betas[i]) / chunk->cg_alphas[i];
    }
    if (!tridiag_ql(d, e)) {
        tl::fail(30, "Too many iterations in TQLI routine");
        return false;
    }
    double lo = DBL_MAX, hi = DBL_MIN;
    for (int i = 0; i < n; ++i) {
        lo = d[i] < lo ? d[i] : lo;
        hi = d[i] > hi ? d[i] : hi;
    }
    if (lo < 0.0 || hi < 0.0) {
        tl::fail(31, "Calculated negative eigenvalues.");
        return false;
    }
    chunk->eigmin = lo * 0.95;
    chunk->eigmax = hi * 1.05;
    return true;
}

// cheby_coef_driver (2d/drivers/cheby_driver.c:163-183)
template <typename ChunkT>
void cheby_coefs(ChunkT* chunk, int count)
{
    chunk->theta = (chunk->eigmax + chunk->eigmin) / 2.0;
    const double delta = (chunk->eigmax - chunk->eigmin) / 2.0;
    const double sigma = chunk->theta / delta;
    double rho_old = 1.0 / sigma;
    for (int i = 0; i < count; ++i) {
        const double rho_new = 1.0 / (2.0 * sigma - rho_old);
        chunk->cheby_alphas[i] = rho_new * rho_old;
        chunk->cheby_betas[i] = 2.0 * rho_new / delta;
        rho_old = rho_new;
    }
}

// cheby_calc_est_iterations (2d/drivers/cheby_driver.c:146-160)
template <typename ChunkT>
int cheby_est(const ChunkT* chunk, double error, double bb)
{
    const double cn = chunk->eigmax / chunk->eigmin;
    const double it_alpha = DBL_EPSILON * bb / (4.0 * error);
    const double gamm = (sqrt(cn) - 1.0) / (sqrt(cn) + 1.0);
    return (int)roundf(logf(it_alpha) / (2.0 * logf(gamm)));
}

}  // namespace tl
