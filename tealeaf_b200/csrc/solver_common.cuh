// solver_common.cuh -- state of the device-resident solver loops, shared by
// the 2D and 3D suites: scalar operands that live on the host or the device,
// the loop control block, and the "finishers" that the last block of a
// reduction runs to form the next scalars (alpha = rro/pw, beta = rrn/rro,
// the Chebyshev/PPCG bookkeeping) and to take the stop decision.
#pragma once

#include "common.cuh"

namespace tl __attribute__((visibility("hidden"))) {

constexpr int kCgItersForEigenvalues = 20;   // 2d/shared.h:42
constexpr double kErrorSwitchMax = 1.0;      // 2d/shared.h:43

// Scalar operand: a host value, or a device location (device-resident driver).
struct Scalar {
    double v;
    const double* dev;
    __device__ __forceinline__ double get() const { return dev ? *dev : v; }
};

// Control block of the device-resident solver loops (device memory).
struct DevState {
    double rro, pw, rrn, alpha, beta, error;
    double theta;
    int trip;     // completed trips of the solver loop (the reference's tt)
    int done;     // the loop has ended
    int reason;   // 1 converged, 2 switch to Chebyshev/PPCG, 3 max_iters
    int nch;      // Chebyshev trips done (next coefficient index)
    int est;      // Chebyshev iteration estimate
    int pad;
};

// Read-only parameters of a solve.
struct DevParams {
    double eps, eps_lim;
    int max_iters, presteps, error_switch, switch_enabled, dims3;
};

// Stop test of the solver loops: 2D tests the error itself, 3D its square
// root (3d/drivers/cg_solver_driver.c:24-25); the switch from CG to
// Chebyshev/PPCG is evaluated for the next trip (2d/drivers/cheby_driver.c:30-32).
__device__ __forceinline__ void end_of_trip(DevState* st, const DevParams& prm, double error, int* host_mirror)
{
    const double e = prm.dims3 ? sqrt(error) : error;
    st->error = e;
    const int tt = st->trip;
    st->trip = tt + 1;
    int reason = 0;
    if (fabs(e) < prm.eps) reason = 1;
    else if (tt + 1 >= prm.max_iters) reason = 3;
    else if (prm.switch_enabled) {
        const bool sw = prm.error_switch ? (e < prm.eps_lim) && (tt + 1 > kCgItersForEigenvalues)
                                         : (tt + 1 > prm.presteps) && (e < kErrorSwitchMax);
        if (sw) reason = 2;
    }
    if (reason) {
        st->done = 1;
        st->reason = reason;
    }
    if (host_mirror) {
        host_mirror[0] = st->done;
        host_mirror[1] = st->trip;
        host_mirror[2] = st->reason;
    }
}

// Finishers (thread 0 of the last block, with the grid totals).
struct FinCgInit {         // rro of cg_init_driver (cg_driver.c:30-62) starts the loop state
    DevState* st;
    int* host_mirror;
    __device__ void operator()(const double* t) const
    {
        st->rro = t[0];
        st->trip = 0;
        st->done = 0;
        st->reason = 0;
        st->nch = 0;
        st->error = 1e10;
        if (host_mirror) {
            host_mirror[0] = 0;
            host_mirror[1] = 0;
            host_mirror[2] = 0;
        }
    }
};

struct FinCgW {            // alpha = rro / pw; cg_alphas[tt] = alpha  (cg_driver.c:87-93)
    DevState* st;
    double* cg_alphas;
    __device__ void operator()(const double* t) const
    {
        st->pw = t[0];
        const double a = st->rro / t[0];
        st->alpha = a;
        if (cg_alphas) cg_alphas[st->trip] = a;
    }
};

struct FinCgUr {           // beta = rrn / rro; rro = error = rrn  (cg_driver.c:104-123)
    DevState* st;
    double* cg_betas;
    DevParams prm;
    int* host_mirror;
    __device__ void operator()(const double* t) const
    {
        const double rrn = t[0];
        const double b = rrn / st->rro;
        st->beta = b;
        cg_betas[st->trip] = b;
        st->rro = rrn;
        st->rrn = rrn;
        end_of_trip(st, prm, rrn, host_mirror);
    }
};

struct FinPcgUr {          // preconditioned CG: t = (r.r, r.z); beta = r.z / rro, rro = r.z, error = r.r
    DevState* st;
    double* cg_betas;
    DevParams prm;
    int* host_mirror;
    __device__ void operator()(const double* t) const
    {
        const double b = t[1] / st->rro;
        st->beta = b;
        cg_betas[st->trip] = b;
        st->rro = t[1];
        st->rrn = t[0];
        end_of_trip(st, prm, t[0], host_mirror);
    }
};

__device__ __forceinline__ bool gate_closed(const int* done) { return done && *(volatile const int*)done; }

// Chebyshev coefficients of the current trip: host values, or the device
// tables indexed by the trip counter.
struct ChebyCoef {
    double alpha, beta;
    const double* alphas;   // device tables (device-resident driver) or null
    const double* betas;
    const DevState* st;
    __device__ __forceinline__ void get(double& a, double& b) const
    {
        if (alphas) {
            const int n = st->nch;
            a = alphas[n];
            b = betas[n];
        } else {
            a = alpha;
            b = beta;
        }
    }
};

struct FinChebyTrip {      // end of one Chebyshev trip of the device-resident loop
    DevState* st;
    DevParams prm;
    int* host_mirror;
    int force_norm;        // the first trip always takes the norm (cheby_driver.c:49-50)
    __device__ void operator()(const double* t) const
    {
        const bool norm = force_norm || (st->nch >= st->est && ((st->trip + 1) % 10) == 0);
        st->nch += 1;
        end_of_trip(st, prm, norm ? t[0] : st->error, host_mirror);
    }
};

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


// PPCG inner-step coefficients: host values or device tables [pp].
struct PpcgCoef {
    double alpha, beta;
    const double* alphas;
    const double* betas;
    __device__ __forceinline__ void get(int pp, double& a, double& b) const
    {
        if (alphas) {
            a = alphas[pp];
            b = betas[pp];
        } else {
            a = alpha;
            b = beta;
        }
    }
};

struct FinPpcgW {          // alpha = rro / pw  (ppcg_driver.c:100)
    DevState* st;
    __device__ void operator()(const double* t) const
    {
        st->pw = t[0];
        st->alpha = st->rro / t[0];
    }
};

struct FinPpcgNorm {       // beta = rrn / rro ; error = rro = rrn  (ppcg_driver.c:131-149)
    DevState* st;
    DevParams prm;
    int* host_mirror;
    __device__ void operator()(const double* t) const
    {
        const double rrn = t[0];
        st->beta = rrn / st->rro;
        st->rro = rrn;
        st->rrn = rrn;
        st->nch += 1;
        end_of_trip(st, prm, rrn, host_mirror);
    }
};

// Field summary in the reference's summation order (2d field_summary.c:8-45,
// 3d field_summary.c:8-49: one serial loop, x fastest, then y, then z), so
// vol, mass and ie come out bit-identical to the reference's and temp
// differs only by the solution itself. A serial sum cannot be reassociated,
// so each of the four sums is one dependent chain of adds: warp w < 4 (lane
// 0) advances sum w through a shared-memory tile of per-cell terms while
// the producer warps form the next tile's terms (volume, volume * density,
// mass * energy0, mass * u) from coalesced loads. One block; the chains'
// add latency bounds it (a few ns per cell). For 2D pass z = 1, hdz = 0.
constexpr int kSumTile = 1024;              // cells per tile
constexpr int kSumProducers = 256;          // producer threads (8 warps)
constexpr int kSumThreads = 128 + kSumProducers;
constexpr size_t kSumSmem = 2 * 4 * kSumTile * sizeof(double);

static __global__ void __launch_bounds__(kSumThreads) k_field_summary_ordered(int x, int y, int z, int hd, int hdz,
                                                                             const double* __restrict__ volume,
                                                                             const double* __restrict__ density,
                                                                             const double* __restrict__ energy0,
                                                                             const double* __restrict__ u,
                                                                             double* out_dev, double* out_host)
{
    extern __shared__ double terms[];   // [2 buffers][4 sums][kSumTile]
    const int nx = x - 2 * hd, ny = y - 2 * hd, nz = z - 2 * hdz;
    const long n = (long)nx * ny * nz;
    const long ntiles = (n + kSumTile - 1) / kSumTile;
    const long xy = (long)x * y;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int pt = (int)threadIdx.x - 128;   // producer thread id (< 0: a chain warp)

    auto produce = [&](long t) {
        double* dst = terms + (t & 1) * 4 * kSumTile;
        const long base = t * kSumTile;
        for (int m = pt; m < kSumTile; m += kSumProducers) {
            const long c = base + m;
            if (c >= n) break;
            const long r = c / nx;
            const long idx = (long)(hdz + r / ny) * xy + (long)(hd + r % ny) * x + (hd + c % nx);
            const double cv = volume[idx];
            const double cm = cv * density[idx];
            dst[m] = cv;
            dst[kSumTile + m] = cm;
            dst[2 * kSumTile + m] = cm * energy0[idx];
            dst[3 * kSumTile + m] = cm * u[idx];
        }
    };

    double acc = 0.0;
    if (pt >= 0 && ntiles > 0) produce(0);
    __syncthreads();
    for (long t = 0; t < ntiles; ++t) {
        if (pt >= 0) {
            if (t + 1 < ntiles) produce(t + 1);
        } else if (lane == 0) {
            const double* src = terms + (t & 1) * 4 * kSumTile + warp * kSumTile;
            const int cnt = (int)min((long)kSumTile, n - t * kSumTile);
            if (cnt == kSumTile) {
#pragma unroll 16
                for (int m = 0; m < kSumTile; ++m) acc += src[m];
            } else {
                for (int m = 0; m < cnt; ++m) acc += src[m];
            }
        }
        __syncthreads();
    }
    if (pt < 0 && lane == 0) {
        out_dev[warp] = acc;
        if (out_host) out_host[warp] = acc;
    }
}

// Launches k_field_summary_ordered on `st`, raising its dynamic shared
// memory limit on the current device first (a summary is rare; the call is
// repeated so every device a process uses is covered).
static inline void launch_field_summary_ordered(cudaStream_t st, int x, int y, int z, int hd, int hdz,
                                                const double* volume, const double* density,
                                                const double* energy0, const double* u, double* out_dev,
                                                double* out_host)
{
    cudaFuncSetAttribute(k_field_summary_ordered, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSumSmem);
    k_field_summary_ordered<<<1, kSumThreads, kSumSmem, st>>>(x, y, z, hd, hdz, volume, density, energy0, u,
                                                              out_dev, out_host);
}

}  // namespace tl
