// kernels3d.cuh -- device kernels of the 3D suite (included by suite3d.cu
// and driver3d.cu; kernels are static in each includer).
//
// Interior sweeps: blocks of 32 (x) x 4 (y) threads, each thread walking
// ZR cells up a z-pencil with the z-neighbours of the 7-point stencil carried
// in registers; x-neighbours come from the same warp's lines (L1) and
// y-neighbours from the neighbouring warps of the block (L1/L2), so each
// field streams from DRAM once per sweep. Index k + j*x + i*x*y, halo
// included (3d/shared.h:52-58). Includers are compiled with -fmad=false.
#pragma once

#include "common.cuh"
#include "tma.cuh"
#include "solver_common.cuh"
#include "tealeaf_b200_3d.h"

using tl::ReduceSlots;

namespace tl3d {

using tl::ChebyCoef;
using tl::DevParams;
using tl::DevState;
using tl::FinCgInit;
using tl::FinCgUr;
using tl::FinCgW;
using tl::FinChebyBlock;
using tl::FinChebyTrip;
using tl::FinPpcgNorm;
using tl::FinPpcgW;
using tl::gate_closed;
using tl::PpcgCoef;
using tl::Scalar;

#ifndef TL3D_UNROLL
#define TL3D_UNROLL 4
#endif
#ifndef TL3D_MINB
#define TL3D_MINB 4
#endif
#define TL3D_STR(x) #x
#define TL3D_PRAGMA_UNROLL(n) _Pragma(TL3D_STR(unroll n))
constexpr unsigned kFull3 = 0xffffffffu;

constexpr int BX = 32;   // x threads per block of an interior sweep
constexpr int BY = 8;    // y threads per block
#ifndef TL3D_ZR
#define TL3D_ZR 16
#endif
constexpr int ZR = TL3D_ZR;   // default z cells per thread (Geo::zr)
constexpr int NT = BX * BY;
constexpr int FBX = 32, FBY = 8;   // full-array kernels

struct Geo {
    int x, y, z, hd;
    int zr = ZR;   // z cells per thread of the interior sweeps (chosen per chunk)
    __host__ __device__ long xy() const { return (long)x * y; }
};

// External faces whose depth-1 halo is reflected.
struct Faces {
    int l, r, b, t, k, f;   // left, right, bottom, top, back, front
};

__device__ __forceinline__ double coef_w(int coefficient, double density)
{
    return coefficient == TL3_CONDUCTIVITY ? density : 1.0 / density;
}

__device__ __forceinline__ double face(double r, double wa, double wb) { return r * (wa + wb) / (2.0 * wa * wb); }

// 7-point operator in the reference operand order (3d/shared.h:52-58).
__device__ __forceinline__ double smvp(double kxc, double kxr, double kyc, double kyu, double kzc, double kzf,
                                       double c, double l, double r, double d, double u, double b, double f)
{
    return (1.0 + (kxr + kxc) + (kyu + kyc) + (kzf + kzc)) * c - (kxr * r + kxc * l) - (kyu * u + kyc * d) -
           (kzf * f + kzc * b);
}

__device__ __forceinline__ int block_id() { return blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z); }
__device__ __forceinline__ int block_count() { return gridDim.x * gridDim.y * gridDim.z; }

struct Pencil {
    int k, j, i0, i1;
    bool active;
    __device__ Pencil(const Geo& g) : Pencil(g, blockIdx.x, blockIdx.y, blockIdx.z) {}
    __device__ Pencil(const Geo& g, int bx, int by, int bz)
    {
        k = g.hd + bx * BX + threadIdx.x;
        j = g.hd + by * BY + threadIdx.y;
        i0 = g.hd + bz * g.zr;
        i1 = min(i0 + g.zr, g.z - g.hd);
        active = k < g.x - g.hd && j < g.y - g.hd;
    }
};

// The CG u/r sweep walks the pencils in the reverse of the w sweep's order
// (last block first, each pencil from its last plane down), so that it
// starts on the planes the w sweep touched last, still in L2, and ends on
// the planes the next w sweep starts on. Each block's partial sum keeps the
// slot of its pencils, so the reduction order over blocks is unchanged.
// 0: forward order.
#ifndef TL3D_UR_REVERSE
#define TL3D_UR_REVERSE 1
#endif
__device__ __forceinline__ int ur3_b(unsigned b, unsigned n) { return TL3D_UR_REVERSE ? (int)(n - 1 - b) : (int)b; }

// Pencil with the cell clamped into the interior for lanes past it (they
// load valid cells and feed the x-neighbour shuffles, but store nothing).
struct PencilC {
    int k, j, i0, i1, lane;
    bool active, rowok, at_l, at_r, at_b, at_t;
    __device__ PencilC(const Geo& g)
    {
        const int k0 = g.hd + blockIdx.x * BX + threadIdx.x;
        const int j0 = g.hd + blockIdx.y * BY + threadIdx.y;
        rowok = j0 < g.y - g.hd;
        active = rowok && k0 < g.x - g.hd;
        k = min(k0, g.x - g.hd - 1);
        j = min(j0, g.y - g.hd - 1);
        i0 = g.hd + blockIdx.z * g.zr;
        i1 = min(i0 + g.zr, g.z - g.hd);
        lane = threadIdx.x;
        at_l = k == g.hd;
        at_r = k == g.x - g.hd - 1;
        at_b = j == g.hd;
        at_t = j == g.y - g.hd - 1;
    }
};

// Halo duty of the extra z-plane of blocks: reflective halo cells of the
// external faces, dst[mirror] = val(source) for layers d < depth (3D
// local_halos.c pattern). `val` reads only data the sweep does not modify.
template <typename Val>
__device__ __forceinline__ void halo_duty3(const Geo& g, const Faces& fc, int depth, double* __restrict__ dst, Val val)
{
    const int x = g.x, y = g.y, z = g.z, hd = g.hd;
    const long nx = x - 2 * hd, ny = y - 2 * hd, nz = z - 2 * hd;
    const long xy = g.xy();
    const long lr = nz * ny * depth, tb = nz * nx * depth, fb = ny * nx * depth;
    const long nthreads = (long)gridDim.x * gridDim.y * blockDim.x * blockDim.y;
    const long t0 = ((long)blockIdx.y * gridDim.x + blockIdx.x) * (blockDim.x * blockDim.y) +
                    threadIdx.y * blockDim.x + threadIdx.x;
    for (long t = t0; t < 2 * (lr + tb + fb); t += nthreads) {
        long q = t;
        int face;
        if (q < 2 * lr) face = (int)(q / lr), q %= lr;
        else if ((q -= 2 * lr) < 2 * tb) face = 2 + (int)(q / tb), q %= tb;
        else q -= 2 * tb, face = 4 + (int)(q / fb), q %= fb;
        const int d = (int)(q % depth);
        q /= depth;
        if (face < 2) {
            const int jj = hd + (int)(q % ny), ii = hd + (int)(q / ny);
            const long base = (long)ii * xy + (long)jj * x;
            if (face == 0 && fc.l) dst[base + (hd - 1 - d)] = val(base + (hd + d));
            if (face == 1 && fc.r) dst[base + (x - hd + d)] = val(base + (x - hd - 1 - d));
        } else if (face < 4) {
            const int kk = hd + (int)(q % nx), ii = hd + (int)(q / nx);
            const long base = (long)ii * xy + kk;
            if (face == 2 && fc.b) dst[base + (long)(hd - 1 - d) * x] = val(base + (long)(hd + d) * x);
            if (face == 3 && fc.t) dst[base + (long)(y - hd + d) * x] = val(base + (long)(y - hd - 1 - d) * x);
        } else {
            const int kk = hd + (int)(q % nx), jj = hd + (int)(q / nx);
            const long base = (long)jj * x + kk;
            if (face == 4 && fc.k) dst[base + (long)(hd - 1 - d) * xy] = val(base + (long)(hd + d) * xy);
            if (face == 5 && fc.f) dst[base + (long)(z - hd + d) * xy] = val(base + (long)(z - hd - 1 - d) * xy);
        }
    }
}

// Operand planes of the fused sweeps, staged in shared memory: the block's
// BX x BY cells of the two operand arrays A, B with a one-cell ring (x and y
// neighbours), and the face coefficients kx (one extra column), ky (one extra
// row) and kz of one z-plane.
struct Plane3 {
    double A[BY + 2][BX + 2];
    double B[BY + 2][BX + 2];
    double kx[BY][BX + 1];
    double ky[BY + 1][BX];
    double kz[BY][BX];
};
constexpr int kStages3 = 4;   // ring of planes: plane ii is computed while ii+1 .. ii+3 are in flight

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem)
{
    const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;\n" ::"n"(N) : "memory"); }

// Fused stencil walker. The operand of a cell is comb(A, B) in the interior
// and A (as stored) in the halo; the depth-1 reflective halo of an external
// face is applied on the fly with REFLECT. Each thread copies its cell (and,
// at the block edges, the ring cells, the extra kx column and ky row) of
// planes i0 .. i1 into a ring of kStages3 shared planes with asynchronous
// copies (cp.async; the waits are the hardware's wait_group), so three planes
// are in flight while one is computed from shared memory. Addresses are
// clamped into the array, so edge blocks load valid memory for cells they do
// not use. All threads of the block must call it (uniform pencil length).
// body(ii, i, centre, smvp).
template <bool REFLECT, typename Comb, typename Body>
__device__ __forceinline__ void walkc(const Geo& g, const Faces& fc, const PencilC& s, const double* __restrict__ A,
                                      const double* __restrict__ B, const double* __restrict__ kx,
                                      const double* __restrict__ ky, const double* __restrict__ kz, Comb comb,
                                      Body body)
{
    __shared__ Plane3 ring[kStages3];
    const int x = g.x, y = g.y;
    const long xy = g.xy();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const int zlast = g.z - g.hd - 1;
    const int kb = g.hd + blockIdx.x * BX, jb = g.hd + blockIdx.y * BY;   // block origin
    auto gi = [&](int k, int j, int iz) {
        k = min(max(k, 0), x - 1);
        j = min(max(j, 0), y - 1);
        return (long)k + (long)j * x + (long)iz * xy;
    };
    // asynchronous copies of plane iz into ring slot st (coefficients only for computed planes)
    auto issue = [&](int iz, int st, bool coef) {
        Plane3& P = ring[st];
        const int k = kb + tx, j = jb + ty;
        auto ab = [&](int yy, int xx, long idx) {
            cp_async8(&P.A[yy][xx], A + idx);
            if (B) cp_async8(&P.B[yy][xx], B + idx);
        };
        ab(ty + 1, tx + 1, gi(k, j, iz));
        if (tx == 0) ab(ty + 1, 0, gi(k - 1, j, iz));
        if (tx == BX - 1) ab(ty + 1, BX + 1, gi(k + 1, j, iz));
        if (ty == 0) ab(0, tx + 1, gi(k, j - 1, iz));
        if (ty == BY - 1) ab(BY + 1, tx + 1, gi(k, j + 1, iz));
        cp_async8(&P.kz[ty][tx], kz + gi(k, j, iz));
        if (coef) {
            cp_async8(&P.kx[ty][tx], kx + gi(k, j, iz));
            if (tx == BX - 1) cp_async8(&P.kx[ty][BX], kx + gi(k + 1, j, iz));
            cp_async8(&P.ky[ty][tx], ky + gi(k, j, iz));
            if (ty == BY - 1) cp_async8(&P.ky[BY][tx], ky + gi(k, j + 1, iz));
        }
    };
    const int np = s.i1 - s.i0 + 1;   // planes i0 .. i1 (i1: the last plane's front neighbour)
    for (int q = 0; q < kStages3 - 1; ++q) {
        if (q < np) issue(s.i0 + q, q, s.i0 + q < s.i1);
        cp_async_commit();
    }
    long i = s.k + (long)s.j * x + (long)s.i0 * xy;
    double bk = (s.i0 == g.hd) ? 0.0 : comb(A[i - xy], B ? B[i - xy] : 0.0);
    const bool bk_reflect = s.i0 == g.hd;
#pragma unroll 1
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
        const int q = ii - s.i0;
        cp_async_wait<kStages3 - 3>();   // planes ii and ii+1 have landed (this thread's copies)
        __syncthreads();                 // ... everyone's; slot of plane ii-1 is free
        if (q + kStages3 - 1 < np) issue(ii + kStages3 - 1, (q + kStages3 - 1) % kStages3, ii + kStages3 - 1 < s.i1);
        cp_async_commit();
        const Plane3& P = ring[q % kStages3];
        const Plane3& F = ring[(q + 1) % kStages3];
        const int cx = tx + 1, cy = ty + 1;
        auto cell = [&](const Plane3& S, int yy, int xx) { return comb(S.A[yy][xx], B ? S.B[yy][xx] : 0.0); };
        const double c = cell(P, cy, cx);
        if (ii == s.i0 && bk_reflect) bk = (REFLECT && fc.k) ? c : A[i - xy];
        const double l = s.at_l ? ((REFLECT && fc.l) ? c : P.A[cy][cx - 1]) : cell(P, cy, cx - 1);
        const double r = s.at_r ? ((REFLECT && fc.r) ? c : P.A[cy][cx + 1]) : cell(P, cy, cx + 1);
        const double d = s.at_b ? ((REFLECT && fc.b) ? c : P.A[cy - 1][cx]) : cell(P, cy - 1, cx);
        const double u = s.at_t ? ((REFLECT && fc.t) ? c : P.A[cy + 1][cx]) : cell(P, cy + 1, cx);
        const double fr = ii == zlast ? ((REFLECT && fc.f) ? c : F.A[cy][cx]) : cell(F, cy, cx);
        const double v = smvp(P.kx[ty][tx], P.kx[ty][tx + 1], P.ky[ty][tx], P.ky[ty + 1][tx], P.kz[ty][tx],
                              F.kz[ty][tx], c, l, r, d, u, bk, fr);
        body(ii, i, c, v);
        bk = c;
    }
    cp_async_wait<0>();
    __syncthreads();
}

// The operand planes of walkc fed by TMA (tma.cuh), each array one box of a
// tensor map at a 128-byte aligned offset: A and B with columns kb-2 ..
// kb+33 (the box must start on a 16-byte boundary; kb = hd + 32 bx is even
// for an even halo depth) and rows jb-1 .. jb+8, kx with one extra column, ky
// with one extra row, kz.
struct PlaneT {
    alignas(128) double A[BY + 2][BX + 4];
    alignas(128) double B[BY + 2][BX + 4];
    alignas(128) double kx[BY][BX + 2];
    alignas(128) double ky[BY + 1][BX];
    alignas(128) double kz[BY][BX];
};

// Tensor maps of one fused sweep: the operand arrays (box (BX+4) x (BY+2) x 1)
// and the face coefficients (boxes (BX+2) x BY, BX x (BY+1), BX x BY).
struct Tma3Maps {
    CUtensorMap a, b, kx, ky, kz;
};

#ifndef TL3D_TMA_STAGES
#define TL3D_TMA_STAGES 4
#endif
constexpr int kStagesT3 = TL3D_TMA_STAGES;   // walkt's ring of planes (walkc keeps kStages3)
static_assert(kStagesT3 >= 3, "plane ii is read with ii+1 while a later one is in flight");
constexpr size_t kTmaRingBytes = kStagesT3 * sizeof(PlaneT) + kStagesT3 * 8 + 128;   // + barriers + alignment
// TMA alignment: boxes start at x = hd - 2 + BX bx (operands) or hd + BX bx
// (coefficients), so BX must keep them even and every box row 16-byte wide.
static_assert(BX % 2 == 0 && ((BX + 4) * sizeof(double)) % 16 == 0 && ((BX + 2) * sizeof(double)) % 16 == 0 &&
                  (BX * sizeof(double)) % 16 == 0,
              "TMA boxes of the 3D sweeps must start and extend on 16-byte boundaries");

// walkc with the planes brought in by TMA: one thread issues the plane's
// boxes on the slot's shared-memory barrier; every thread waits (bounded) for
// planes ii and ii+1, then computes exactly as walkc. All threads of the
// block must call it.
template <bool REFLECT, typename Comb, typename Body>
__device__ __forceinline__ void walkt(const Geo& g, const Faces& fc, const PencilC& s, const Tma3Maps& m,
                                      bool has_b, const double* __restrict__ A, const double* __restrict__ B,
                                      unsigned char* raw, int* err, Comb comb, Body body)
{
    unsigned char* base = raw + ((128 - (tl::smem_addr(raw) & 127)) & 127);
    PlaneT* ring = reinterpret_cast<PlaneT*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesT3 * sizeof(PlaneT));
    const int x = g.x;
    const long xy = g.xy();
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = tx == 0 && ty == 0;
    const int zlast = g.z - g.hd - 1;
    const int kb = g.hd + blockIdx.x * BX, jb = g.hd + blockIdx.y * BY;   // block origin
    constexpr unsigned kAB = sizeof(double) * (BY + 2) * (BX + 4);
    constexpr unsigned kKZ = sizeof(double) * BY * BX;
    constexpr unsigned kKXY = sizeof(double) * (BY * (BX + 2) + (BY + 1) * BX);
    auto issue = [&](int iz, int st, bool coef) {
        PlaneT& P = ring[st];
        tl::mbar_expect_tx(&bars[st], kAB * (has_b ? 2u : 1u) + kKZ + (coef ? kKXY : 0u));
        tl::tma_load_3d(&P.A[0][0], &m.a, kb - 2, jb - 1, iz, &bars[st]);
        if (has_b) tl::tma_load_3d(&P.B[0][0], &m.b, kb - 2, jb - 1, iz, &bars[st]);
        tl::tma_load_3d(&P.kz[0][0], &m.kz, kb, jb, iz, &bars[st]);
        if (coef) {
            tl::tma_load_3d(&P.kx[0][0], &m.kx, kb, jb, iz, &bars[st]);
            tl::tma_load_3d(&P.ky[0][0], &m.ky, kb, jb, iz, &bars[st]);
        }
    };
    const int np = s.i1 - s.i0 + 1;   // planes i0 .. i1 (i1: the last plane's front neighbour)
    if (leader) {
        for (int q = 0; q < kStagesT3; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (leader)
        for (int q = 0; q < kStagesT3 - 1 && q < np; ++q) issue(s.i0 + q, q, s.i0 + q < s.i1);
    long i = s.k + (long)s.j * x + (long)s.i0 * xy;
    double bk = (s.i0 == g.hd) ? 0.0 : comb(A[i - xy], B ? B[i - xy] : 0.0);
    const bool bk_reflect = s.i0 == g.hd;
#pragma unroll 1
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
        const int q = ii - s.i0;
        __syncthreads();   // every thread is past plane ii-1: its slot is free
        if (leader && q + kStagesT3 - 1 < np)
            issue(ii + kStagesT3 - 1, (q + kStagesT3 - 1) % kStagesT3, ii + kStagesT3 - 1 < s.i1);
        tl::mbar_wait(&bars[q % kStagesT3], (unsigned)(q / kStagesT3) & 1u, err);
        tl::mbar_wait(&bars[(q + 1) % kStagesT3], (unsigned)((q + 1) / kStagesT3) & 1u, err);
        const PlaneT& P = ring[q % kStagesT3];
        const PlaneT& F = ring[(q + 1) % kStagesT3];
        const int cx = tx + 2, cy = ty + 1;
        auto cell = [&](const PlaneT& S, int yy, int xx) { return comb(S.A[yy][xx], has_b ? S.B[yy][xx] : 0.0); };
        const double c = cell(P, cy, cx);
        if (ii == s.i0 && bk_reflect) bk = (REFLECT && fc.k) ? c : A[i - xy];
        const double l = s.at_l ? ((REFLECT && fc.l) ? c : P.A[cy][cx - 1]) : cell(P, cy, cx - 1);
        const double r = s.at_r ? ((REFLECT && fc.r) ? c : P.A[cy][cx + 1]) : cell(P, cy, cx + 1);
        const double d = s.at_b ? ((REFLECT && fc.b) ? c : P.A[cy - 1][cx]) : cell(P, cy - 1, cx);
        const double u = s.at_t ? ((REFLECT && fc.t) ? c : P.A[cy + 1][cx]) : cell(P, cy + 1, cx);
        const double fr = ii == zlast ? ((REFLECT && fc.f) ? c : F.A[cy][cx]) : cell(F, cy, cx);
        const double v = smvp(P.kx[ty][tx], P.kx[ty][tx + 1], P.ky[ty][tx], P.ky[ty + 1][tx], P.kz[ty][tx],
                              F.kz[ty][tx], c, l, r, d, u, bk, fr);
        body(ii, i, c, v);
        bk = c;
    }
    __syncthreads();   // every issued plane has been waited for: no copy is in flight
}

__device__ __forceinline__ void reflect_store(double* f, const Geo& g, const Faces& fc, int depth, int k, int j,
                                             int i, double v)
{
    const long xy = g.xy();
    const long base = (long)i * xy + (long)j * g.x;
    if (fc.l && k - g.hd < depth) f[base + (2 * g.hd - 1 - k)] = v;
    if (fc.r && (g.x - g.hd - 1 - k) < depth) f[base + (2 * (g.x - g.hd) - 1 - k)] = v;
    if (fc.b && j - g.hd < depth) f[(long)i * xy + (long)(2 * g.hd - 1 - j) * g.x + k] = v;
    if (fc.t && (g.y - g.hd - 1 - j) < depth) f[(long)i * xy + (long)(2 * (g.y - g.hd) - 1 - j) * g.x + k] = v;
    if (fc.k && i - g.hd < depth) f[(long)(2 * g.hd - 1 - i) * xy + (long)j * g.x + k] = v;
    if (fc.f && (g.z - g.hd - 1 - i) < depth) f[(long)(2 * (g.z - g.hd) - 1 - i) * xy + (long)j * g.x + k] = v;
}

// Generic stencil walker: CUR(idx) gives the operand value at an interior
// cell; halo neighbours come from `raw` (memory) unless REFLECT mirrors them
// on an external face. Calls body(i, centre, smvp) for every cell.
template <bool REFLECT, typename Cur, typename Body>
__device__ __forceinline__ void walk(const Geo& g, const Faces& fc, const Pencil& s, const double* __restrict__ raw,
                                     const double* __restrict__ kx, const double* __restrict__ ky,
                                     const double* __restrict__ kz, Cur cur, Body body)
{
    const int x = g.x, k = s.k, j = s.j;
    const long xy = g.xy();
    const bool at_l = k == g.hd, at_r = k == g.x - g.hd - 1;
    const bool at_b = j == g.hd, at_t = j == g.y - g.hd - 1;
    long i = k + (long)j * x + (long)s.i0 * xy;
    double c = cur(i);
    double bk = (s.i0 == g.hd) ? ((REFLECT && fc.k) ? c : raw[i - xy]) : cur(i - xy);
    double kzc = kz[i];
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
        const bool at_f = ii == g.z - g.hd - 1;
        const double fr = at_f ? ((REFLECT && fc.f) ? c : raw[i + xy]) : cur(i + xy);
        const double l = at_l ? ((REFLECT && fc.l) ? c : raw[i - 1]) : cur(i - 1);
        const double r = at_r ? ((REFLECT && fc.r) ? c : raw[i + 1]) : cur(i + 1);
        const double d = at_b ? ((REFLECT && fc.b) ? c : raw[i - x]) : cur(i - x);
        const double u = at_t ? ((REFLECT && fc.t) ? c : raw[i + x]) : cur(i + x);
        const double kzf = kz[i + xy];
        const double v = smvp(kx[i], kx[i + 1], ky[i], ky[i + x], kzc, kzf, c, l, r, d, u, bk, fr);
        body(ii, i, c, v);
        bk = c;
        c = fr;
        kzc = kzf;
    }
}

// ------------------------------------------------------ CG (cg_solver.c) --

// [p = beta p + r] ; depth-1 reflective halo of p ; w = A p ; pw = sum(w p)
// (3d/c_kernels/omp3/cg_solver.c:105-193). Grid: interior blocks plus one
// z-plane of halo-duty blocks (the reflected halo of p_out, and the pending
// halo of u when u_halo is given; u is read-only here).
template <bool FUSE_P, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(NT, TL3D_MINB) k3_cg_w(Geo g, Faces fc, Scalar beta,
                                                               const double* __restrict__ p_in, double* p_out,
                                                               const double* __restrict__ r, double* __restrict__ w,
                                                               const double* __restrict__ kx,
                                                               const double* __restrict__ ky,
                                                               const double* __restrict__ kz, double* u_halo, int uhd,
                                                               ReduceSlots rs, const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    const double bt = FUSE_P ? beta.get() : 0.0;
    auto cur = [&](long idx) { return FUSE_P ? bt * p_in[idx] + r[idx] : p_in[idx]; };
    if (blockIdx.z + 1 < gridDim.z) {
        const PencilC s(g);
        walkc<REFLECT>(g, fc, s, p_in, FUSE_P ? r : nullptr, kx, ky, kz,
                       [&](double pa, double rb) { return FUSE_P ? bt * pa + rb : pa; },
                       [&](int, long i, double c, double v) {
            if (s.active) {
                w[i] = v;
                acc[0] += v * c;
                if (FUSE_P) p_out[i] = c;
            }
        });
    } else {
        if (REFLECT) halo_duty3(g, fc, 1, p_out, cur);
        if (u_halo) halo_duty3(g, fc, uhd, u_halo, [&](long idx) { return u_halo[idx]; });
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count(), fin);
}

// k3_cg_w with the operand planes brought in by TMA (walkt); the same
// arithmetic, so the same results. `err`: the bounded barrier waits' flag.
template <bool FUSE_P, bool REFLECT, typename Finish>
static __global__ void __launch_bounds__(NT, TL3D_MINB) k3_cg_w_tma(Geo g, Faces fc, Scalar beta,
                                                                   const __grid_constant__ Tma3Maps maps,
                                                                   const double* __restrict__ p_in, double* p_out,
                                                                   const double* __restrict__ r,
                                                                   double* __restrict__ w, double* u_halo, int uhd,
                                                                   ReduceSlots rs, const int* __restrict__ done,
                                                                   Finish fin, int* err)
{
    extern __shared__ __align__(128) unsigned char t3_raw[];
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    const double bt = FUSE_P ? beta.get() : 0.0;
    auto cur = [&](long idx) { return FUSE_P ? bt * p_in[idx] + r[idx] : p_in[idx]; };
    if (blockIdx.z + 1 < gridDim.z) {
        const PencilC s(g);
        walkt<REFLECT>(g, fc, s, maps, FUSE_P, p_in, FUSE_P ? r : nullptr, t3_raw, err,
                       [&](double pa, double rb) { return FUSE_P ? bt * pa + rb : pa; },
                       [&](int, long i, double c, double v) {
            if (s.active) {
                w[i] = v;
                acc[0] += v * c;
                if (FUSE_P) p_out[i] = c;
            }
        });
    } else {
        if (REFLECT) halo_duty3(g, fc, 1, p_out, cur);
        if (u_halo) halo_duty3(g, fc, uhd, u_halo, [&](long idx) { return u_halo[idx]; });
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count(), fin);
}

// u += alpha p ; r -= alpha w ; rrn = sum(r r)  (cg_solver.c:134-160)
template <typename Finish>
static __global__ void __launch_bounds__(NT, 8) k3_cg_ur(Geo g, Scalar alpha, double* __restrict__ u,
                                                                const double* __restrict__ p, double* __restrict__ r,
                                                                const double* __restrict__ w, ReduceSlots rs,
                                                                const int* __restrict__ done, Finish fin)
{
    if (gate_closed(done)) return;
    const int bx = ur3_b(blockIdx.x, gridDim.x), by = ur3_b(blockIdx.y, gridDim.y), bz = ur3_b(blockIdx.z, gridDim.z);
    Pencil s(g, bx, by, bz);
    double acc[1] = {0.0};
    if (s.active) {
        const double a = alpha.get();
        const long xy = g.xy();
        const long step = TL3D_UR_REVERSE ? -xy : xy;
        long i = s.k + (long)s.j * g.x + (long)(TL3D_UR_REVERSE ? s.i1 - 1 : s.i0) * xy;
        TL3D_PRAGMA_UNROLL(TL3D_UNROLL)
        for (int n = 0; n < s.i1 - s.i0; ++n, i += step) {
            u[i] += a * p[i];
            const double rn = r[i] - a * w[i];
            r[i] = rn;
            acc[0] += rn * rn;
        }
    }
    tl::grid_sum<1, NT>(acc, rs, bx + gridDim.x * (by + gridDim.y * bz), block_count(), fin);
}

// k3_cg_ur with its operands brought in by TMA: stages of kPlanesU z-planes of
// the block's 32 x 8 columns of u, p, r, w. Same pencils, planes in the same
// order per thread (TL3D_UR_REVERSE), same arithmetic: the same results,
// partial sums included.
#ifndef TL3D_TMA_PLANES_U
#define TL3D_TMA_PLANES_U 2
#endif
#ifndef TL3D_TMA_STAGES_U
#define TL3D_TMA_STAGES_U 4   // 4 deep (65.5 KB, 3 blocks per SM): 132.9 against 135.9 us for 3 deep at 256^3
#endif
constexpr int kPlanesU = TL3D_TMA_PLANES_U;
constexpr int kStagesU3 = TL3D_TMA_STAGES_U;
struct PlanesU {
    alignas(128) double U[kPlanesU][BY][BX];
    alignas(128) double P[kPlanesU][BY][BX];
    alignas(128) double R[kPlanesU][BY][BX];
    alignas(128) double W[kPlanesU][BY][BX];
};
struct Tma3UrMaps {
    CUtensorMap u, p, r, w;
};
constexpr size_t kTmaUr3Bytes = kStagesU3 * sizeof(PlanesU) + kStagesU3 * 8 + 128;

template <typename Finish>
static __global__ void __launch_bounds__(NT, 4) k3_cg_ur_tma(Geo g, Scalar alpha,
                                                          const __grid_constant__ Tma3UrMaps maps,
                                                          double* __restrict__ u, double* __restrict__ r,
                                                          ReduceSlots rs, const int* __restrict__ done, Finish fin,
                                                          int* err)
{
    extern __shared__ __align__(128) unsigned char u3_raw[];
    if (gate_closed(done)) return;
    unsigned char* base = u3_raw + ((128 - (tl::smem_addr(u3_raw) & 127)) & 127);
    PlanesU* ring = reinterpret_cast<PlanesU*>(base);
    unsigned long long* bars = reinterpret_cast<unsigned long long*>(base + kStagesU3 * sizeof(PlanesU));
    const int bx = ur3_b(blockIdx.x, gridDim.x), by = ur3_b(blockIdx.y, gridDim.y), bz = ur3_b(blockIdx.z, gridDim.z);
    Pencil s(g, bx, by, bz);
    double acc[1] = {0.0};
    const int tx = threadIdx.x, ty = threadIdx.y;
    const bool leader = tx == 0 && ty == 0;
    const int kb = g.hd + bx * BX, jb = g.hd + by * BY;
    const int np = (s.i1 - s.i0 + kPlanesU - 1) / kPlanesU;
    // stage b holds planes z0(b) .. z0(b) + kPlanesU - 1 (the pencil's last
    // stage may run past i1; those planes are loaded and not used)
    auto stage_z0 = [&](int b) { return s.i0 + (TL3D_UR_REVERSE ? np - 1 - b : b) * kPlanesU; };
    auto issue = [&](int b) {
        PlanesU& S = ring[b % kStagesU3];
        unsigned long long* bar = &bars[b % kStagesU3];
        const int z0 = stage_z0(b);
        tl::mbar_expect_tx(bar, 4u * sizeof(double) * kPlanesU * BY * BX);
        tl::tma_load_3d(&S.U[0][0][0], &maps.u, kb, jb, z0, bar);
        tl::tma_load_3d(&S.P[0][0][0], &maps.p, kb, jb, z0, bar);
        tl::tma_load_3d(&S.R[0][0][0], &maps.r, kb, jb, z0, bar);
        tl::tma_load_3d(&S.W[0][0][0], &maps.w, kb, jb, z0, bar);
    };
    if (leader) {
        for (int q = 0; q < kStagesU3; ++q) tl::mbar_init(&bars[q], 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (leader)
        for (int b = 0; b < kStagesU3 - 1 && b < np; ++b) issue(b);
    const double a = alpha.get();
    const long xy = g.xy();
    for (int b = 0; b < np; ++b) {
        __syncthreads();   // every thread is past stage b-1: its slot is free
        if (leader && b + kStagesU3 - 1 < np) issue(b + kStagesU3 - 1);
        tl::mbar_wait(&bars[b % kStagesU3], (unsigned)(b / kStagesU3) & 1u, err);
        const PlanesU& S = ring[b % kStagesU3];
        const int z0 = stage_z0(b);
#pragma unroll
        for (int q = 0; q < kPlanesU; ++q) {
            const int t = TL3D_UR_REVERSE ? kPlanesU - 1 - q : q;   // planes in the order of k3_cg_ur
            const int ii = z0 + t;
            if (ii >= s.i1) continue;
            if (s.active) {
                const long i = s.k + (long)s.j * g.x + (long)ii * xy;
                u[i] = S.U[t][ty][tx] + a * S.P[t][ty][tx];
                const double rn = S.R[t][ty][tx] - a * S.W[t][ty][tx];
                r[i] = rn;
                acc[0] += rn * rn;
            }
        }
    }
    tl::grid_sum<1, NT>(acc, rs, bx + gridDim.x * (by + gridDim.y * bz), block_count(), fin);
}

// p = beta p + r (APPLY_P) and the depth-1 halos of p and (unless null) u.
static __global__ void __launch_bounds__(NT) k3_cg_close(Geo g, Faces fc, Scalar beta, int apply_p,
                                                        double* __restrict__ p, const double* __restrict__ r,
                                                        double* __restrict__ u)
{
    Pencil s(g);
    if (!s.active) return;
    const double bt = beta.get();
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
        const double pn = apply_p ? bt * p[i] + r[i] : p[i];
        p[i] = pn;
        reflect_store(p, g, fc, 1, s.k, s.j, ii, pn);
        if (u) reflect_store(u, g, fc, 1, s.k, s.j, ii, u[i]);
    }
}

// Chebyshev trip (3d/c_kernels/omp3/cheby_solver.c:62-99) with the previous
// trip's u += p folded in (ADD), or the init sweep (INIT: p = r / theta).
// With REFLECT the halo-duty z-plane writes the reflected halo of u_n.
// TMA: operand planes by walkt (maps of u_in, p_in, kx, ky, kz; err: the
// bounded waits' flag), else by walkc; the same results either way.
template <bool ADD, bool REFLECT, bool INIT, typename Finish, bool TMA = false>
static __global__ void __launch_bounds__(NT, TL3D_MINB) k3_cheby_trip(Geo g, Faces fc, ChebyCoef coef, double theta,
                                                                     int write_wr_always,
                                                                     const double* __restrict__ u_in,
                                                                     const double* __restrict__ p_in, double* u_out,
                                                                     double* p_out, const double* __restrict__ u0,
                                                                     double* __restrict__ w, double* __restrict__ r,
                                                                     const double* __restrict__ kx,
                                                                     const double* __restrict__ ky,
                                                                     const double* __restrict__ kz, ReduceSlots rs,
                                                                     const int* __restrict__ done, Finish fin,
                                                                     DevParams prm,
                                                                     const __grid_constant__ Tma3Maps maps,
                                                                     int* err)
{
    extern __shared__ __align__(128) unsigned char ct_raw[];
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    double a = 0.0, b = 0.0;
    if (!INIT) coef.get(a, b);
    const bool wr = INIT || write_wr_always || !coef.st ||
                    (coef.st->nch >= coef.st->est && ((coef.st->trip + 1) % 10) == 0) ||
                    (coef.st->trip + 1 >= prm.max_iters);
    auto cur = [&](long idx) { return ADD ? u_in[idx] + p_in[idx] : u_in[idx]; };
    if (blockIdx.z + 1 < gridDim.z) {
        const PencilC s(g);
        auto comb = [&](double ua, double pb) { return ADD ? ua + pb : ua; };
        auto body = [&](int, long i, double c, double v) {
            if (s.active) {
                const double rr = u0[i] - v;
                const double pn = INIT ? rr / theta : a * p_in[i] + b * rr;
                if (wr) {
                    w[i] = v;
                    r[i] = rr;
                }
                acc[0] += rr * rr;
                p_out[i] = pn;
                if (ADD) u_out[i] = c;
            }
        };
        if constexpr (TMA) walkt<REFLECT>(g, fc, s, maps, ADD, u_in, ADD ? p_in : nullptr, ct_raw, err, comb, body);
        else walkc<REFLECT>(g, fc, s, u_in, ADD ? p_in : nullptr, kx, ky, kz, comb, body);
    } else if (REFLECT) {
        halo_duty3(g, fc, 1, ADD ? u_out : const_cast<double*>(u_in), cur);
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count(), fin);
}

// u += p with the depth-1 halo of u written from the final values (APPLY),
// or u += p on the interior only (cheby_calc_u, cheby_solver.c:8-24).
template <bool CLOSE>
static __global__ void __launch_bounds__(NT) k3_add_p(Geo g, Faces fc, double* __restrict__ u,
                                                     const double* __restrict__ p)
{
    Pencil s(g);
    if (!s.active) return;
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
        const double un = u[i] + p[i];
        u[i] = un;
        if (CLOSE) reflect_store(u, g, fc, 1, s.k, s.j, ii, un);
    }
}

// PPCG inner step (3d/c_kernels/omp3/ppcg_solver.c:29-73) with the previous
// step's sd update folded in (FOLD 1: sd = r/theta; FOLD 2: a sd + b r); the
// halo-duty z-plane writes the reflected halo of sd_out.
// TMA as in k3_cheby_trip (maps of sd_in, r_in, kx, ky, kz).
template <int FOLD, bool NORM, typename Finish, bool TMA = false>
static __global__ void __launch_bounds__(NT, TL3D_MINB) k3_ppcg_step(Geo g, Faces fc, double theta, PpcgCoef coef,
                                                                    int pp_prev, const double* __restrict__ sd_in,
                                                                    double* __restrict__ sd_out,
                                                                    const double* __restrict__ r_in,
                                                                    double* __restrict__ r_out,
                                                                    double* __restrict__ u,
                                                                    const double* __restrict__ kx,
                                                                    const double* __restrict__ ky,
                                                                    const double* __restrict__ kz, ReduceSlots rs,
                                                                    const int* __restrict__ done, Finish fin,
                                                                    const __grid_constant__ Tma3Maps maps, int* err)
{
    extern __shared__ __align__(128) unsigned char ps_raw[];
    if (gate_closed(done)) return;
    double acc[1] = {0.0};
    double a = 0.0, b = 0.0;
    if (FOLD == 2) coef.get(pp_prev, a, b);
    auto cur = [&](long idx) {
        if (FOLD == 0) return sd_in[idx];
        if (FOLD == 1) return r_in[idx] / theta;
        return a * sd_in[idx] + b * r_in[idx];
    };
    if (blockIdx.z + 1 < gridDim.z) {
        const PencilC s(g);
        auto comb = [&](double sa, double rb) {
            if (FOLD == 0) return sa;
            if (FOLD == 1) return rb / theta;
            return a * sa + b * rb;
        };
        auto body = [&](int, long i, double c, double v) {
            if (s.active) {
                const double rn = r_in[i] - v;
                r_out[i] = rn;
                u[i] += c;
                sd_out[i] = c;
                if (NORM) acc[0] += rn * rn;
            }
        };
        if constexpr (TMA)
            walkt<true>(g, fc, s, maps, FOLD != 0, sd_in, FOLD == 0 ? nullptr : r_in, ps_raw, err, comb, body);
        else walkc<true>(g, fc, s, sd_in, FOLD == 0 ? nullptr : r_in, kx, ky, kz, comb, body);
    } else {
        halo_duty3(g, fc, 1, sd_out, cur);
    }
    if (NORM) tl::grid_sum<1, NT>(acc, rs, block_id(), block_count(), fin);
}

// sd = alpha sd + beta r (the second loop of ppcg_inner_iteration)
static __global__ void __launch_bounds__(NT) k3_ppcg_sd(Geo g, double alpha, double beta, double* __restrict__ sd,
                                                       const double* __restrict__ r)
{
    Pencil s(g);
    if (!s.active) return;
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) sd[i] = alpha * sd[i] + beta * r[i];
}

// r -= A sd ; u += sd (the first loop of ppcg_inner_iteration, halo as stored)
static __global__ void __launch_bounds__(NT) k3_ppcg_inner_a(Geo g, double* __restrict__ u, double* __restrict__ r,
                                                            const double* __restrict__ kx, const double* __restrict__ ky,
                                                            const double* __restrict__ kz, const double* __restrict__ sd)
{
    Pencil s(g);
    if (!s.active) return;
    Faces none{0, 0, 0, 0, 0, 0};
    walk<false>(g, none, s, sd, kx, ky, kz, [&](long idx) { return sd[idx]; },
                [&](int, long i, double c, double v) {
                    r[i] -= v;
                    u[i] += c;
                });
}

// ------------------------------------------------- shared solver methods --

static __global__ void __launch_bounds__(NT) k3_ppcg_init(Geo g, double theta, const double* __restrict__ r,
                                                         double* __restrict__ sd)
{
    Pencil s(g);
    if (!s.active) return;
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) sd[i] = r[i] / theta;
}

static __global__ void __launch_bounds__(NT) k3_copy_u(Geo g, double* __restrict__ u0, const double* __restrict__ u)
{
    Pencil s(g);
    if (!s.active) return;
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) u0[i] = u[i];
}

static __global__ void __launch_bounds__(NT) k3_residual(Geo g, const double* __restrict__ u,
                                                        const double* __restrict__ u0, double* __restrict__ r,
                                                        const double* __restrict__ kx, const double* __restrict__ ky,
                                                        const double* __restrict__ kz)
{
    Pencil s(g);
    if (!s.active) return;
    Faces none{0, 0, 0, 0, 0, 0};
    walk<false>(g, none, s, u, kx, ky, kz, [&](long idx) { return u[idx]; },
                [&](int, long i, double, double v) { r[i] = u0[i] - v; });
}

static __global__ void __launch_bounds__(NT) k3_norm2(Geo g, const double* __restrict__ b, ReduceSlots rs)
{
    Pencil s(g);
    double acc[1] = {0.0};
    if (s.active) {
        const long xy = g.xy();
        long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
        for (int ii = s.i0; ii < s.i1; ++ii, i += xy) acc[0] += b[i] * b[i];
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count());
}

static __global__ void __launch_bounds__(NT) k3_finalise(Geo g, double* __restrict__ energy,
                                                        const double* __restrict__ density, const double* __restrict__ u)
{
    Pencil s(g);
    if (!s.active) return;
    const long xy = g.xy();
    long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
    for (int ii = s.i0; ii < s.i1; ++ii, i += xy) energy[i] = u[i] / density[i];
}

static __global__ void __launch_bounds__(NT) k3_field_summary(Geo g, const double* __restrict__ volume,
                                                             const double* __restrict__ density,
                                                             const double* __restrict__ energy0,
                                                             const double* __restrict__ u, ReduceSlots rs)
{
    Pencil s(g);
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    if (s.active) {
        const long xy = g.xy();
        long i = s.k + (long)s.j * g.x + (long)s.i0 * xy;
        for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
            const double cv = volume[i];
            const double cm = cv * density[i];
            acc[0] += cv;
            acc[1] += cm;
            acc[2] += cm * energy0[i];
            acc[3] += cm * u[i];
        }
    }
    tl::grid_sum<4, NT>(acc, rs, block_id(), block_count());
}

// Jacobi sweep (3d/c_kernels/omp3/jacobi_solver.c:69-115), r holds the old u.
static __global__ void __launch_bounds__(NT) k3_jacobi_iterate(Geo g, const double* __restrict__ kx,
                                                              const double* __restrict__ ky,
                                                              const double* __restrict__ kz,
                                                              const double* __restrict__ u0, double* __restrict__ u,
                                                              const double* __restrict__ r, ReduceSlots rs)
{
    Pencil s(g);
    double acc[1] = {0.0};
    if (s.active) {
        const int x = g.x;
        const long xy = g.xy();
        long i = s.k + (long)s.j * x + (long)s.i0 * xy;
        for (int ii = s.i0; ii < s.i1; ++ii, i += xy) {
            const double v = (u0[i] + (kx[i + 1] * r[i + 1] + kx[i] * r[i - 1]) +
                              (ky[i + x] * r[i + x] + ky[i] * r[i - x]) + (kz[i + xy] * r[i + xy] + kz[i] * r[i - xy])) /
                             (1.0 + (kx[i] + kx[i + 1]) + (ky[i] + ky[i + x]) + (kz[i] + kz[i + xy]));
            u[i] = v;
            acc[0] += fabs(v - r[i]);
        }
    }
    tl::grid_sum<1, NT>(acc, rs, block_id(), block_count());
}

// ------------------------------------------------- full-array kernels ----

struct Cell {
    int k, j, i;
    bool in;
    __device__ Cell(const Geo& g)
    {
        k = blockIdx.x * FBX + threadIdx.x;
        j = blockIdx.y * FBY + threadIdx.y;
        i = blockIdx.z;
        in = k < g.x && j < g.y;
    }
};

// cg_solver_init fused (3d/c_kernels/omp3/cg_solver.c:9-102), p written to
// both p buffers; coefficients and neighbour values recomputed with the
// reference expressions.
template <typename Finish>
static __global__ void __launch_bounds__(FBX* FBY) k3_cg_init(Geo g, int coefficient, double rx, double ry, double rz,
                                                             const double* __restrict__ density,
                                                             const double* __restrict__ energy, double* __restrict__ u,
                                                             double* __restrict__ p, double* __restrict__ p2,
                                                             double* __restrict__ r, double* __restrict__ w,
                                                             double* __restrict__ kx, double* __restrict__ ky,
                                                             double* __restrict__ kz, ReduceSlots rs, Finish fin)
{
    const Cell c(g);
    const int x = g.x, y = g.y, z = g.z, hd = g.hd;
    const long xy = g.xy();
    double acc[1] = {0.0};
    if (c.in) {
        const int k = c.k, j = c.j, ii = c.i;
        const long i = k + (long)j * x + (long)ii * xy;
        const double rho = density[i];
        const double uc = energy[i] * rho;
        u[i] = uc;
        const bool interior = k >= hd && k < x - hd && j >= hd && j < y - hd && ii >= hd && ii < z - hd;
        const bool ring = k >= 1 && k < x - 1 && j >= 1 && j < y - 1 && ii >= 1 && ii < z - 1;
        const bool kzone = k >= hd && k < x - 1 && j >= hd && j < y - 1 && ii >= hd && ii < z - 1;
        double wc = 0.0;
        if (ring) wc = coef_w(coefficient, rho);
        double kxc = 0.0, kyc = 0.0, kzc = 0.0;
        if (kzone) {
            kxc = face(rx, coef_w(coefficient, density[i - 1]), wc);
            kyc = face(ry, coef_w(coefficient, density[i - x]), wc);
            kzc = face(rz, coef_w(coefficient, density[i - xy]), wc);
            kx[i] = kxc;
            ky[i] = kyc;
            kz[i] = kzc;
        }
        if (interior) {
            const double kxr = (k + 1 < x - 1) ? face(rx, wc, coef_w(coefficient, density[i + 1])) : kx[i + 1];
            const double kyu = (j + 1 < y - 1) ? face(ry, wc, coef_w(coefficient, density[i + x])) : ky[i + x];
            const double kzf = (ii + 1 < z - 1) ? face(rz, wc, coef_w(coefficient, density[i + xy])) : kz[i + xy];
            const double v = smvp(kxc, kxr, kyc, kyu, kzc, kzf, uc, energy[i - 1] * density[i - 1],
                                  energy[i + 1] * density[i + 1], energy[i - x] * density[i - x],
                                  energy[i + x] * density[i + x], energy[i - xy] * density[i - xy],
                                  energy[i + xy] * density[i + xy]);
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
    tl::grid_sum<1, FBX * FBY>(acc, rs, block_id(), block_count(), fin);
}

// jacobi_solver_init (3d/c_kernels/omp3/jacobi_solver.c:9-66)
static __global__ void __launch_bounds__(FBX* FBY) k3_jacobi_init(Geo g, int coefficient, double rx, double ry,
                                                                 double rz, const double* __restrict__ density,
                                                                 const double* __restrict__ energy,
                                                                 double* __restrict__ u0, double* __restrict__ u,
                                                                 double* __restrict__ kx, double* __restrict__ ky,
                                                                 double* __restrict__ kz)
{
    const Cell c(g);
    if (!c.in) return;
    const int x = g.x, y = g.y, z = g.z, hd = g.hd, k = c.k, j = c.j, ii = c.i;
    const long xy = g.xy();
    const long i = k + (long)j * x + (long)ii * xy;
    if (k >= 1 && k < x - 1 && j >= 1 && j < y - 1 && ii >= 1 && ii < z - 1) {
        const double t = energy[i] * density[i];
        u0[i] = t;
        u[i] = t;
    }
    if (k >= hd && k < x - 1 && j >= hd && j < y - 1 && ii >= hd && ii < z - 1) {
        const double cc = coef_w(coefficient, density[i]);
        const double l = coef_w(coefficient, density[i - 1]);
        const double d = coef_w(coefficient, density[i - x]);
        const double b = coef_w(coefficient, density[i - xy]);
        kx[i] = rx * (l + cc) / (2.0 * l * cc);
        ky[i] = ry * (d + cc) / (2.0 * d * cc);
        kz[i] = rz * (b + cc) / (2.0 * b * cc);
    }
}

// set_chunk_data (3d/c_kernels/omp3/set_chunk_data.c:8-74)
static __global__ void k3_set_chunk_data_axes(Geo g, double x_min, double y_min, double z_min, double dx, double dy,
                                             double dz, double* vx, double* vy, double* vz, double* cx, double* cy,
                                             double* cz)
{
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    const int hd = g.hd;
    if (t <= g.x) vx[t] = x_min + dx * (double)(t - hd);
    if (t <= g.y) vy[t] = y_min + dy * (double)(t - hd);
    if (t <= g.z) vz[t] = z_min + dz * (double)(t - hd);
    if (t < g.x) cx[t] = 0.5 * ((x_min + dx * (double)(t - hd)) + (x_min + dx * (double)(t + 1 - hd)));
    if (t < g.y) cy[t] = 0.5 * ((y_min + dy * (double)(t - hd)) + (y_min + dy * (double)(t + 1 - hd)));
    if (t < g.z) cz[t] = 0.5 * ((z_min + dz * (double)(t - hd)) + (z_min + dz * (double)(t + 1 - hd)));
}

static __global__ void k3_set_chunk_data_cells(long n, double dx, double dy, double dz, double* volume,
                                              double* x_area, double* y_area, double* z_area)
{
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        volume[i] = dx * dy * dz;
        x_area[i] = dy * dz;
        y_area[i] = dx * dz;
        z_area[i] = dx * dy;
    }
}

// set_chunk_state (3d/c_kernels/omp3/set_chunk_state.c:9-98): last state wins.
static __global__ void __launch_bounds__(FBX* FBY) k3_set_chunk_state(Geo g, const double* __restrict__ vx,
                                                                     const double* __restrict__ vy,
                                                                     const double* __restrict__ vz,
                                                                     const double* __restrict__ cx,
                                                                     const double* __restrict__ cy,
                                                                     const double* __restrict__ cz,
                                                                     double* __restrict__ density,
                                                                     double* __restrict__ energy0,
                                                                     double* __restrict__ u, int num_states,
                                                                     const State* __restrict__ states)
{
    const Cell c(g);
    if (!c.in) return;
    const int k = c.k, j = c.j, ii = c.i;
    const long i = k + (long)j * g.x + (long)ii * g.xy();
    double e = states[0].energy, d = states[0].density;
    for (int s = 1; s < num_states; ++s) {
        const State st = states[s];
        bool hit = false;
        if (st.geometry == TL3_GEOM_CUBOID) {
            hit = vx[k + 1] >= st.x_min && vx[k] < st.x_max && vy[j + 1] >= st.y_min && vy[j] < st.y_max &&
                  vz[ii + 1] >= st.z_min && vz[ii] < st.z_max;
        } else if (st.geometry == TL3_GEOM_SPHERICAL) {
            const double ax = cx[k] - st.x_min, ay = cy[j] - st.y_min, az = cz[ii] - st.z_min;
            hit = sqrt(ax * ax + ay * ay + az * az) <= st.radius;
        } else if (st.geometry == TL3_GEOM_POINT) {
            hit = vx[k] == st.x_min && vy[j] == st.y_min && vz[ii] == st.z_min;
        }
        if (hit) {
            e = st.energy;
            d = st.density;
        }
    }
    energy0[i] = e;
    density[i] = d;
    if (k >= 1 && k < g.x - 1 && j >= 1 && j < g.y - 1 && ii >= 1 && ii < g.z - 1) u[i] = e * d;
}

// Reflective halo update of up to six fields (3d/c_kernels/omp3/local_halos.c).
struct HaloArgs3 {
    double* f[TL3_NUM_FIELDS];
    int nf;
    int ext[6];
};

static __global__ void k3_local_halos(Geo g, int depth, HaloArgs3 a)
{
    const int x = g.x, y = g.y, z = g.z, hd = g.hd;
    const long nx = x - 2 * hd, ny = y - 2 * hd, nz = z - 2 * hd;
    const long xy = g.xy();
    const long lr = nz * ny * depth, tb = nz * nx * depth, fb = ny * nx * depth;
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    if (blockIdx.y >= (unsigned)a.nf || t >= 2 * (lr + tb + fb)) return;
    double* f = a.f[blockIdx.y];
    long q = t;
    int face;
    if (q < 2 * lr) face = (int)(q / lr), q %= lr;
    else if ((q -= 2 * lr) < 2 * tb) face = 2 + (int)(q / tb), q %= tb;
    else q -= 2 * tb, face = 4 + (int)(q / fb), q %= fb;
    if (!a.ext[face]) return;
    const int d = (int)(q % depth);
    q /= depth;
    if (face < 2) {           // left / right: q over (ii, jj)
        const int jj = hd + (int)(q % ny), ii = hd + (int)(q / ny);
        const long base = (long)ii * xy + (long)jj * x;
        if (face == 0) f[base + (hd - d - 1)] = f[base + (hd + d)];
        else f[base + (x - hd + d)] = f[base + (x - hd - 1 - d)];
    } else if (face < 4) {    // bottom / top: q over (ii, kk)
        const int kk = hd + (int)(q % nx), ii = hd + (int)(q / nx);
        const long base = (long)ii * xy + kk;
        if (face == 2) f[base + (long)(hd - d - 1) * x] = f[base + (long)(hd + d) * x];
        else f[base + (long)(y - hd + d) * x] = f[base + (long)(y - hd - 1 - d) * x];
    } else {                  // back / front: q over (jj, kk)
        const int kk = hd + (int)(q % nx), jj = hd + (int)(q / nx);
        const long base = (long)jj * x + kk;
        if (face == 4) f[base + (long)(hd - d - 1) * xy] = f[base + (long)(hd + d) * xy];
        else f[base + (long)(z - hd + d) * xy] = f[base + (long)(z - hd - 1 - d) * xy];
    }
}

// MPI face buffers (3d/c_kernels/omp3/pack_halos.c): pack/unpack one face.
static __global__ void k3_pack(Geo g, int depth, int face, int pack, double* __restrict__ field,
                               double* __restrict__ buf)
{
    const int x = g.x, y = g.y, z = g.z, hd = g.hd;
    const long nx = x - 2 * hd, ny = y - 2 * hd, nz = z - 2 * hd;
    const long xy = g.xy();
    const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
    long fi, bi;
    if (face == TL3_CHUNK_LEFT || face == TL3_CHUNK_RIGHT) {
        if (t >= nz * ny * depth) return;
        const int c = (int)(t % depth), jj = hd + (int)((t / depth) % ny), ii = hd + (int)(t / (depth * ny));
        int kk;
        if (face == TL3_CHUNK_LEFT) kk = pack ? hd + c : hd - depth + c;
        else kk = pack ? x - hd - depth + c : x - hd + c;
        fi = (long)ii * xy + (long)jj * x + kk;
        bi = c + (long)(jj - hd) * depth + (long)(ii - hd) * depth * ny;
    } else if (face == TL3_CHUNK_BOTTOM || face == TL3_CHUNK_TOP) {
        if (t >= nz * nx * depth) return;
        const int kk = hd + (int)(t % nx), c = (int)((t / nx) % depth), ii = hd + (int)(t / (nx * depth));
        int jj;
        if (face == TL3_CHUNK_BOTTOM) jj = pack ? hd + c : hd - depth + c;
        else jj = pack ? y - hd - depth + c : y - hd + c;
        fi = (long)ii * xy + (long)jj * x + kk;
        bi = (kk - hd) + (long)c * nx + (long)(ii - hd) * depth * nx;
    } else {
        if (t >= ny * nx * depth) return;
        const int kk = hd + (int)(t % nx), jj = hd + (int)((t / nx) % ny), c = (int)(t / (nx * ny));
        int ii;
        if (face == TL3_CHUNK_BACK) ii = pack ? hd + c : hd - depth + c;
        else ii = pack ? z - hd - depth + c : z - hd + c;
        fi = (long)ii * xy + (long)jj * x + kk;
        bi = (kk - hd) + (long)(jj - hd) * nx + (long)c * nx * ny;
    }
    if (pack) buf[bi] = field[fi];
    else field[fi] = buf[bi];
}

// r = u over the full array (the first loop of jacobi_solver_iterate),
// skipped once a device-resident loop has ended.
static __global__ void k3_copy_full(long n, double* __restrict__ dst, const double* __restrict__ src,
                                   const int* __restrict__ done)
{
    if (gate_closed(done)) return;
    for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
        dst[i] = src[i];
}

}  // namespace tl3d
