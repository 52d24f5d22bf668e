// suite2d_impl.hpp -- host-side state of one 2D chunk, shared by the
// kernel-interface layer (suite2d.cu) and the device-resident driver
// (driver2d.cu).
#pragma once

#include "blocked2d.cuh"

#include <cuda_runtime.h>

#include <algorithm>
#include <vector>

// Buffers that alternate between two slices (fused sweeps read the old values
// at stencil neighbours while writing the new ones). The Chunk always points
// at the current slice; the suite keeps the other.
enum AltField { ALT_P = 0, ALT_U = 1, ALT_R = 2, ALT_SD = 3, ALT_COUNT = 4 };

struct TlSuite2D {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    tl2d::Geo g{0, 0, 0};
    void* slab = nullptr;
    size_t slab_bytes = 0;
    tl::ReduceSlots rs{};
    double* h_out = nullptr;          // mapped pinned result slots
    long partial_capacity = 0;        // doubles
    State* d_states = nullptr;
    int d_states_cap = 0;
    double* d_comm = nullptr;         // pack/unpack staging
    long d_comm_cap = 0;
    double* alt[ALT_COUNT] = {nullptr, nullptr, nullptr, nullptr};
    tl::Profiler prof;                // per-kernel device time (off by default)

    // Operations the reference host requested that have not been run yet:
    // a CG p update and reflective halo updates (depth per field, 0 = none).
    // They are absorbed by the next sweep that can fuse them, or flushed.
    struct {
        bool calc_p = false;
        double beta = 0.0;
        int halo[TL_NUM_FIELDS] = {0, 0, 0, 0, 0, 0};
    } pend;

    // Device-resident driver state.
    tl2d::DevState* d_state = nullptr;
    int* h_mirror = nullptr;          // mapped: done, trip, reason
    int* d_mirror = nullptr;          // device view of h_mirror
    double* d_cg_alphas = nullptr;    // device coefficient tables [max_iters]
    double* d_cg_betas = nullptr;
    double* d_cheby_alphas = nullptr;
    double* d_cheby_betas = nullptr;
    int table_len = 0;

    // Device-resident driver: Chebyshev trips / PPCG inner steps temporally
    // blocked in shared memory (blocked2d.cuh); off = one launch per step.
    bool temporal_blocking = true;

    // Device-resident CG: Jacobi preconditioner (pcg2d.cuh), 0 none,
    // 1 jac_diag, 2 jac_block; settings->preconditioner selects jac_diag.
    int precond = 0;

    // Kernel-interface PPCG inner steps deferred for the blocked kernel:
    // run_ppcg_init opens the queue, run_ppcg_inner_iteration appends its
    // coefficients (absorbing the depth-1 halo update of sd before it), and
    // the next other entry point runs them (flush).
    struct {
        bool active = false;
        std::vector<double> a, b;
    } pq;

    // Kernel-interface Chebyshev trips deferred for the blocked kernel the
    // same way: run_cheby_iterate appends its coefficients (absorbing the
    // depth-1 halo update of u before it), the next other entry point runs
    // them.
    struct {
        bool active = false;
        std::vector<double> a, b;
    } cq;

    // FP32 buffers of the iterative-refinement form (mixed2d.cu), on first use.
    void* mx_slab = nullptr;
    size_t mx_bytes = 0;

    // CG w sweep fed by TMA where the layout allows (tl2d_set_tma); tensor
    // maps encoded once per array.
    bool tma = true;
    struct TmaEntry {
        const void* ptr;
        int kind;
        CUtensorMap map;
    };
    TmaEntry tma_cache[48];
    int tma_n = 0;
    int tma_next = 0;
};

// Index of the int, in the mapped mirror words, that the bounded TMA barrier
// waits set when one gives up.
constexpr int kTmaErrWord2 = 15;

// Launch on the suite stream, bracketed by profiler events when enabled.
#define TL_LAUNCH(s, name, ...)                \
    do {                                       \
        (s)->prof.begin((s)->stream, name);    \
        __VA_ARGS__;                           \
        (s)->prof.end((s)->stream);            \
        TL_LAUNCHED(name);                     \
    } while (0)

namespace tl2d {

TlSuite2D* suite_of(Chunk* chunk);
// Interior sweeps: BX columns x g.rows rows per block. Every interior
// reduction uses this one partition, so the kernel-interface path and the
// device-resident driver add the same partial sums in the same order.
inline dim3 interior_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, BX), tl::ceil_div(g.y - 2 * g.hd, g.rows));
}
inline dim3 full_grid(const Geo& g) { return dim3(tl::ceil_div(g.x, 32), tl::ceil_div(g.y, FB / 32)); }
// Interior grid plus the halo-duty block row of the fused sweeps.
inline dim3 fused_grid(const Geo& g)
{
    dim3 d = interior_grid(g);
    d.y += 1;
    return d;
}
// Rows per thread of the interior sweeps: the grid is cut into whole waves
// of resident blocks (sm_count * min_blocks) so no SM idles in a partial
// last wave; the fewest waves whose strips are at most TL2D_MAX_ROWS rows
// (longer strips: fewer per-strip ring fills, boundary re-reads and
// reduction partials; `max_rows`). At least 2 rows. `min_blocks`: resident
// blocks per SM of the kernels the grid is cut for.
#ifndef TL2D_MAX_ROWS
#define TL2D_MAX_ROWS 128
#endif
inline int choose_rows(int nx, int ny, int sm_count, int min_blocks = TL2D_MINB, int max_rows = TL2D_MAX_ROWS)
{
    const long slots = (long)sm_count * min_blocks;
    const long bx = tl::ceil_div(nx, BX);
    for (long waves = 1;; ++waves) {
        const long strips = std::max(1L, waves * slots / bx);   // strips per column band
        const int rows = std::max(2, tl::ceil_div(ny, strips));
        if (rows <= max_rows) return rows;
    }
}
// Waits for the stream and returns the published sums.
bool fetch(TlSuite2D* s, int n, double* out);
// Runs every pending operation (p update, then halo updates).
void flush(TlSuite2D* s, Chunk* chunk);
// External faces of the chunk (neighbours == EXTERNAL_FACE).
Faces faces_of(const Chunk* chunk);
// The chunk's pointer to an alternating field, and the swap after a fused sweep.
FieldBufferType* field_slot(Chunk* chunk, AltField f);
void swap_alt(TlSuite2D* s, Chunk* chunk, AltField f);


// A cached tensor map: (ptr, kind) -> map, encoded by `encode` on a miss; a
// full cache recycles its entries in turn (arrays of released buffers).
template <typename Encode>
inline const CUtensorMap* tma_lookup(TlSuite2D* s, const void* ptr, int kind, Encode encode)
{
    for (int i = 0; i < s->tma_n; ++i)
        if (s->tma_cache[i].ptr == ptr && s->tma_cache[i].kind == kind) return &s->tma_cache[i].map;
    const int cap = (int)(sizeof(s->tma_cache) / sizeof(s->tma_cache[0]));
    const int slot = s->tma_n < cap ? s->tma_n : (s->tma_next++ % cap);
    CUtensorMap m;
    if (!encode(&m)) return nullptr;
    TlSuite2D::TmaEntry& e = s->tma_cache[slot];
    e.map = m;
    e.ptr = ptr;
    e.kind = kind;
    if (s->tma_n < cap) ++s->tma_n;
    return &e.map;
}

// Tensor map of a chunk array for k_cg_w_fused_tma: kind 0 operand rows (box
// (BX+4) x kRowsT), 1 kx ((BX+2) x kRowsT), 2 ky (BX x kRowsT); for
// k_cg_ur_fused_tma: kind 3 (BX x kRowsU).
inline const CUtensorMap* tma_map(TlSuite2D* s, const double* ptr, int kind)
{
    static const unsigned box[4] = {BX + 4, BX + 2, BX, BX};
    return tma_lookup(s, ptr, kind, [&](CUtensorMap* m) {
        return tl::tma_encode_3d(m, ptr, s->g.x, s->g.y, 1, box[kind], kind == 3 ? kRowsU : kRowsT, 1);
    });
}

// The boxes start at x = hd - 2 + 128 bx: an even halo depth and an even row
// length keep every start and stride on a 16-byte boundary.
inline bool tma_usable(const TlSuite2D* s) { return s->tma && s->g.hd % 2 == 0 && s->g.x % 2 == 0; }

inline bool tma_failed(const TlSuite2D* s) { return s->h_mirror && s->h_mirror[kTmaErrWord2] != 0; }

// The fused CG w sweep (k_cg_w_fused semantics), by TMA where possible.
// Internal linkage, like the kernels it launches: each translation unit has
// its own kernel copies, so each keeps its own record of the raised
// shared-memory limit.
template <bool F, bool R, typename Finish>
static void launch_cg_w2(TlSuite2D* s, Chunk* chunk, dim3 grid, const Faces& fc, Scalar beta, const double* p_in,
                  double* p_out, const double* r, double* w, double* u_halo, int uhd, const int* done, Finish fin)
{
    if (tma_usable(s)) {
        const CUtensorMap* a = tma_map(s, p_in, 0);
        const CUtensorMap* b = F ? tma_map(s, r, 0) : a;
        const CUtensorMap* kx = tma_map(s, chunk->kx, 1);
        const CUtensorMap* ky = tma_map(s, chunk->ky, 2);
        if (a && b && kx && ky) {
            const Tma2Maps m{*a, *b, *kx, *ky};
            static unsigned attr_set = 0;   // devices on which the shared-memory size was raised
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k_cg_w_fused_tma<F, R, Finish>,
                                             cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaRowsBytes));
                attr_set |= 1u << (s->device & 31);
            }
            TL_LAUNCH(s, "k_cg_w_fused", (k_cg_w_fused_tma<F, R><<<grid, BX, kTmaRowsBytes, s->stream>>>(
                                             s->g, fc, beta, m, p_in, p_out, r, w, u_halo, uhd, s->rs, done, fin,
                                             s->d_mirror + kTmaErrWord2)));
            return;
        }
    }
    TL_LAUNCH(s, "k_cg_w_fused", (k_cg_w_fused<F, R><<<grid, BX, 0, s->stream>>>(
                                     s->g, fc, beta, p_in, p_out, r, w, chunk->kx, chunk->ky, u_halo, uhd, s->rs,
                                     done, fin)));
}

// The fused CG u/r update (k_cg_ur_fused semantics), by TMA where possible
// (internal linkage as launch_cg_w2).
template <typename Finish>
static void launch_cg_ur2(TlSuite2D* s, dim3 grid, Scalar alpha, double* u, const double* p, double* r, const double* w,
                   const int* done, Finish fin)
{
    if (tma_usable(s)) {
        const CUtensorMap* mu = tma_map(s, u, 3);
        const CUtensorMap* mp = tma_map(s, p, 3);
        const CUtensorMap* mr = tma_map(s, r, 3);
        const CUtensorMap* mw = tma_map(s, w, 3);
        if (mu && mp && mr && mw) {
            const TmaUrMaps m{*mu, *mp, *mr, *mw};
            static unsigned attr_set = 0;   // devices on which the shared-memory size was raised
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k_cg_ur_fused_tma<Finish>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kTmaUrBytes));
                attr_set |= 1u << (s->device & 31);
            }
            TL_LAUNCH(s, "k_cg_ur_fused", (k_cg_ur_fused_tma<<<grid, BX, kTmaUrBytes, s->stream>>>(
                                              s->g, alpha, m, u, r, s->rs, done, fin, s->d_mirror + kTmaErrWord2)));
            return;
        }
    }
    TL_LAUNCH(s, "k_cg_ur_fused", (k_cg_ur_fused<<<grid, BX, 0, s->stream>>>(s->g, alpha, u, p, r, w, s->rs, done,
                                                                            fin)));
}
// Region boxes (kTW x kTH cells, kind 4) of the TMA-staged blocked kernels.
inline const CUtensorMap* blocked_map(TlSuite2D* s, const double* ptr)
{
    return tma_lookup(s, ptr, 4, [&](CUtensorMap* m) {
        return tl::tma_encode_3d(m, ptr, s->g.x, s->g.y, 1, kTW, kTH, 1);
    });
}

// The region boxes of the staged Chebyshev kernel start at X0 - TB =
// hd - TB + TX bx: an even halo depth minus the margin, an even tile width and
// an even row length keep them on 16-byte boundaries.
inline bool blocked_tma_usable(const TlSuite2D* s)
{
    return s->tma && (s->g.hd - Blk<0>::TB) % 2 == 0 && Blk<0>::TX % 2 == 0 && s->g.x % 2 == 0;
}

// One temporally blocked launch of L <= TB Chebyshev trips (MODE 0, C = u0)
// or PPCG inner steps (MODE 1, C = u): for Chebyshev the persistent
// TMA-staged kernel where the alignment rules allow, else k_blocked
// (bit-identical results). Internal linkage as launch_cg_w2.
template <int MODE>
static void launch_blocked(TlSuite2D* s, const char* name, const BlockedArgs& a, const double* A_in,
                           const double* B_in, double* A_out, double* B_out, const double* C, double* u, double* w,
                           double* r, const double* kx, const double* ky, const int* done)
{
    static unsigned attr_set = 0;   // devices on which the shared-memory sizes were raised
    if (!(attr_set & (1u << (s->device & 31)))) {
        TL_CUDA(cudaFuncSetAttribute(k_blocked<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)blocked_smem<MODE>()));
        if constexpr (MODE == 0)
            TL_CUDA(cudaFuncSetAttribute(k_blocked_tma<MODE>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)kBlockedTmaBytes));
        attr_set |= 1u << (s->device & 31);
    }
    const dim3 gb = blocked_grid<MODE>(s->g);
    if constexpr (MODE == 0) {
        if (blocked_tma_usable(s)) {
            const CUtensorMap* ma = blocked_map(s, A_in);
            const CUtensorMap* mb = blocked_map(s, B_in);
            const CUtensorMap* mc = blocked_map(s, C);
            const CUtensorMap* mx = blocked_map(s, kx);
            const CUtensorMap* my = blocked_map(s, ky);
            if (ma && mb && mc && mx && my) {
                const BlockedMaps m{*ma, *mb, *mc, *mx, *my};
                const long tiles = (long)gb.x * gb.y;
                const unsigned grid = (unsigned)std::min<long>(tiles, s->sm_count);
                TL_LAUNCH(s, name, (k_blocked_tma<MODE><<<grid, kTBThreads, kBlockedTmaBytes, s->stream>>>(
                                       s->g, a, m, A_out, B_out, u, w, r, done, s->d_mirror + kTmaErrWord2)));
                return;
            }
        }
    }
    TL_LAUNCH(s, name, (k_blocked<MODE><<<gb, kTBThreads, blocked_smem<MODE>(), s->stream>>>(
                           s->g, a, A_in, B_in, A_out, B_out, MODE == 0 ? C : nullptr, u, w, r, kx, ky, done)));
}

}  // namespace tl2d
