// suite3d_impl.hpp -- host-side state of one 3D chunk, shared by the
// kernel-interface layer (suite3d.cu) and the device-resident driver
// (driver3d.cu). Same design as the 2D suite (suite2d_impl.hpp).
#pragma once

#include "blocked3d.cuh"
#include "kernels3d.cuh"

#include <cuda_runtime.h>

#include <vector>

enum AltField3 { ALT3_P = 0, ALT3_U = 1, ALT3_R = 2, ALT3_SD = 3, ALT3_COUNT = 4 };

struct TlSuite3D {
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    tl3d::Geo g{0, 0, 0, 0};
    void* slab = nullptr;
    size_t slab_bytes = 0;
    tl::ReduceSlots rs{};
    double* h_out = nullptr;
    long partial_capacity = 0;
    State* d_states = nullptr;
    int d_states_cap = 0;
    double* d_comm = nullptr;
    long d_comm_cap = 0;
    double* alt[ALT3_COUNT] = {nullptr, nullptr, nullptr, nullptr};
    tl::Profiler prof;
    struct {
        bool calc_p = false;
        double beta = 0.0;
        int halo[TL3_NUM_FIELDS] = {0, 0, 0, 0, 0, 0};
    } pend;
    tl::DevState* d_state = nullptr;
    int* h_mirror = nullptr;
    int* d_mirror = nullptr;
    double* d_cg_alphas = nullptr;
    double* d_cg_betas = nullptr;
    double* d_cheby_alphas = nullptr;
    double* d_cheby_betas = nullptr;
    int table_len = 0;
    bool tma = true;   // feed the CG w sweep by TMA where the layout allows (tl3d_set_tma)
    bool temporal_blocking = true;   // Chebyshev / PPCG blocks (tl3d_set_temporal_blocking)
    // Chebyshev trips / PPCG inner steps of the run_* path deferred while the
    // reference drivers' call pattern holds, then run temporally blocked
    struct Queue {
        bool active = false;
        std::vector<double> a, b;
    };
    Queue cq, pq;
    struct TmaEntry {
        const double* ptr;
        int kind;
        CUtensorMap map;
    };
    TmaEntry tma_cache[40];
    int tma_n = 0;
    int tma_next = 0;
};

// Index of the int, in the mapped mirror words, that the bounded TMA barrier
// waits set when one gives up.
constexpr int kTmaErrWord = 15;

#define TL3_LAUNCH(s, name, ...)               \
    do {                                       \
        (s)->prof.begin((s)->stream, name);    \
        __VA_ARGS__;                           \
        (s)->prof.end((s)->stream);            \
        TL_LAUNCHED(name);                     \
    } while (0)

namespace tl3d {

TlSuite3D* suite_of(Chunk* chunk);

inline dim3 interior_grid(const Geo& g)
{
    return dim3(tl::ceil_div(g.x - 2 * g.hd, BX), tl::ceil_div(g.y - 2 * g.hd, BY), tl::ceil_div(g.z - 2 * g.hd, g.zr));
}
// z cells per thread of the interior sweeps: the grid should be whole waves
// both for the staged stencil sweeps (TL3D_MINB blocks per SM) and for the
// pointwise ones (8 per SM); longer pencils carry less prologue (one extra
// staged plane per pencil).
inline int choose_zr(int nx, int ny, int nz, int sm_count)
{
    const long bxy = (long)tl::ceil_div(nx, BX) * tl::ceil_div(ny, BY);
    int best = ZR;
    double best_score = -1.0;
    for (int zr = 4; zr <= 32; ++zr) {
        const long blocks = bxy * tl::ceil_div(nz, zr);
        auto eff = [&](long slots) {
            const long waves = (blocks + slots - 1) / slots;
            return (double)blocks / (double)(waves * slots);
        };
        const double score = eff((long)sm_count * TL3D_MINB) * eff((long)sm_count * 8) * zr / (zr + 1.0);
        if (score > best_score + 1e-12) {
            best_score = score;
            best = zr;
        }
    }
    return best;
}
inline dim3 full_grid(const Geo& g) { return dim3(tl::ceil_div(g.x, FBX), tl::ceil_div(g.y, FBY), g.z); }
// Interior grid plus the halo-duty z-plane of the fused sweeps.
inline dim3 fused_grid(const Geo& g)
{
    dim3 d = interior_grid(g);
    d.z += 1;
    return d;
}
inline dim3 interior_block() { return dim3(BX, BY); }
inline dim3 full_block() { return dim3(FBX, FBY); }
bool fetch(TlSuite3D* s, int n, double* out);
void flush(TlSuite3D* s, Chunk* chunk);
Faces faces_of(const Chunk* chunk);
double** field_slot(Chunk* chunk, AltField3 f);
void swap_alt(TlSuite3D* s, Chunk* chunk, AltField3 f);


// Tensor map of a chunk array for walkt: kind 0 operand (box (BX+4) x (BY+2)),
// 1 kx (BX+2) x BY, 2 ky BX x (BY+1), 3 kz BX x BY; for k3_cg_ur_tma kind 4
// BX x BY x kPlanesU; for k3_blocked_tma kind 5 kRX x kRYT; encoded once per
// array.
inline const CUtensorMap* tma_map(TlSuite3D* s, const double* ptr, int kind)
{
    for (int i = 0; i < s->tma_n; ++i)
        if (s->tma_cache[i].ptr == ptr && s->tma_cache[i].kind == kind) return &s->tma_cache[i].map;
    // a full cache recycles its entries in turn (arrays of released buffers)
    const int cap = (int)(sizeof(s->tma_cache) / sizeof(s->tma_cache[0]));
    const int slot = s->tma_n < cap ? s->tma_n : (s->tma_next++ % cap);
    static const unsigned box[6][3] = {{BX + 4, BY + 2, 1}, {BX + 2, BY, 1}, {BX, BY + 1, 1}, {BX, BY, 1},
                                       {BX, BY, kPlanesU}, {kRX, kRYT, 1}};
    CUtensorMap m;
    if (!tl::tma_encode_3d(&m, ptr, s->g.x, s->g.y, s->g.z, box[kind][0], box[kind][1], box[kind][2]))
        return nullptr;
    TlSuite3D::TmaEntry& e = s->tma_cache[slot];
    e.map = m;
    e.ptr = ptr;
    e.kind = kind;
    if (s->tma_n < cap) ++s->tma_n;
    return &e.map;
}

// The TMA boxes start at x = hd - 2 + 32 bx: an even halo depth and an even
// row length keep every start and stride on a 16-byte boundary.
inline bool tma_usable(const TlSuite3D* s) { return s->tma && s->g.hd % 2 == 0 && s->g.x % 2 == 0; }

inline bool tma_failed(const TlSuite3D* s) { return s->h_mirror && s->h_mirror[kTmaErrWord] != 0; }

// One launch of the temporally blocked Chebyshev (MODE 0) / PPCG (MODE 1)
// steps: region planes by TMA where the boxes can start on 16-byte
// boundaries (even halo depth, margin and row length), else per-thread
// loads; the same results either way. Internal linkage, like the kernels.
template <int MODE, int HS>
static void launch_blocked3_tma(TlSuite3D* s, const char* name, const Blocked3Args& a, const Blocked3Maps& m,
                                double* A_out, double* B_out, double* u, double* w, double* r, const int* done)
{
    static unsigned set = 0;   // devices on which the shared-memory size was raised
    if (!(set & (1u << (s->device & 31)))) {
        TL_CUDA(cudaFuncSetAttribute(k3_blocked_tma<MODE, HS>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                     (int)kBlocked3TmaBytes));
        set |= 1u << (s->device & 31);
    }
    TL3_LAUNCH(s, name, (k3_blocked_tma<MODE, HS><<<blocked3_tma_grid(s->g), dim3(kRX, kTYT), kBlocked3TmaBytes,
                                                    s->stream>>>(s->g, a, m, A_out, B_out, u, w, r, done,
                                                                 s->d_mirror + kTmaErrWord)));
}

template <int MODE>
static void launch_blocked3(TlSuite3D* s, Chunk* chunk, const Blocked3Args& a, const double* A_in,
                            const double* B_in, double* A_out, double* B_out, const double* u0, double* u, double* w,
                            double* r, const int* done)
{
    const char* name = MODE == 0 ? "k3_blocked<cheby>" : "k3_blocked<ppcg>";
    if (tma_usable(s) && kTB3 % 2 == 0 && a.steps >= 1 && a.steps <= 2) {
        const CUtensorMap* ma = tma_map(s, A_in, 5);
        const CUtensorMap* mb = tma_map(s, B_in, 5);
        const CUtensorMap* mc = tma_map(s, MODE == 0 ? u0 : u, 5);
        const CUtensorMap* mx = tma_map(s, chunk->vec_kx, 5);
        const CUtensorMap* my = tma_map(s, chunk->vec_ky, 5);
        const CUtensorMap* mz = tma_map(s, chunk->vec_kz, 5);
        if (ma && mb && mc && mx && my && mz) {
            const Blocked3Maps m{*ma, *mb, *mc, *mx, *my, *mz};
            if (a.steps == 1) launch_blocked3_tma<MODE, 1>(s, name, a, m, A_out, B_out, u, w, r, done);
            else launch_blocked3_tma<MODE, 2>(s, name, a, m, A_out, B_out, u, w, r, done);
            return;
        }
    }
    TL3_LAUNCH(s, name, (k3_blocked<MODE><<<blocked3_grid(s->g), dim3(kRX, kRY), 0, s->stream>>>(
                            s->g, a, A_in, B_in, A_out, B_out, u0, u, w, r, chunk->vec_kx, chunk->vec_ky,
                            chunk->vec_kz, done)));
}

// The fused CG w sweep (k3_cg_w semantics), by TMA where possible.
// Internal linkage, like the kernels it launches: each translation unit has
// its own kernel copies, so each keeps its own record of the raised
// shared-memory limit.
template <bool F, bool R, typename Finish>
static void launch_cg_w3(TlSuite3D* s, Chunk* chunk, dim3 grid, const Faces& fc, Scalar beta, const double* p_in,
                  double* p_out, const double* r, double* w, double* u_halo, int uhd, const int* done, Finish fin)
{
    const dim3 bl = interior_block();
    if (tma_usable(s)) {
        const CUtensorMap* a = tma_map(s, p_in, 0);
        const CUtensorMap* b = F ? tma_map(s, r, 0) : a;
        const CUtensorMap* kx = tma_map(s, chunk->vec_kx, 1);
        const CUtensorMap* ky = tma_map(s, chunk->vec_ky, 2);
        const CUtensorMap* kz = tma_map(s, chunk->vec_kz, 3);
        if (a && b && kx && ky && kz) {
            const Tma3Maps m{*a, *b, *kx, *ky, *kz};
            static unsigned attr_set = 0;   // devices on which the shared-memory size was raised
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k3_cg_w_tma<F, R, Finish>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kTmaRingBytes));
                attr_set |= 1u << (s->device & 31);
            }
            TL3_LAUNCH(s, "k3_cg_w", (k3_cg_w_tma<F, R><<<grid, bl, kTmaRingBytes, s->stream>>>(
                                         s->g, fc, beta, m, p_in, p_out, r, w, u_halo, uhd, s->rs, done, fin,
                                         s->d_mirror + kTmaErrWord)));
            return;
        }
    }
    TL3_LAUNCH(s, "k3_cg_w", (k3_cg_w<F, R><<<grid, bl, 0, s->stream>>>(s->g, fc, beta, p_in, p_out, r, w,
                                                                      chunk->vec_kx, chunk->vec_ky, chunk->vec_kz,
                                                                      u_halo, uhd, s->rs, done, fin)));
}

// The fused CG u/r update (k3_cg_ur semantics), by TMA where possible
// (internal linkage as launch_cg_w3).
template <typename Finish>
static void launch_cg_ur3(TlSuite3D* s, dim3 grid, Scalar alpha, double* u, const double* p, double* r,
                          const double* w, const int* done, Finish fin)
{
    const dim3 bl = interior_block();
    if (tma_usable(s)) {
        const CUtensorMap* mu = tma_map(s, u, 4);
        const CUtensorMap* mp = tma_map(s, p, 4);
        const CUtensorMap* mr = tma_map(s, r, 4);
        const CUtensorMap* mw = tma_map(s, w, 4);
        if (mu && mp && mr && mw) {
            const Tma3UrMaps m{*mu, *mp, *mr, *mw};
            static unsigned attr_set = 0;   // devices on which the shared-memory size was raised
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k3_cg_ur_tma<Finish>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kTmaUr3Bytes));
                attr_set |= 1u << (s->device & 31);
            }
            TL3_LAUNCH(s, "k3_cg_ur", (k3_cg_ur_tma<<<grid, bl, kTmaUr3Bytes, s->stream>>>(
                                          s->g, alpha, m, u, r, s->rs, done, fin, s->d_mirror + kTmaErrWord)));
            return;
        }
    }
    TL3_LAUNCH(s, "k3_cg_ur", (k3_cg_ur<<<grid, bl, 0, s->stream>>>(s->g, alpha, u, p, r, w, s->rs, done, fin)));
}

// Tensor maps of a stencil sweep over operands a (and b) with the chunk's
// coefficients; false when the layout or an encoding rules TMA out.
static bool sweep_maps(TlSuite3D* s, Chunk* chunk, const double* a, const double* b, Tma3Maps* m)
{
    if (!tma_usable(s)) return false;
    const CUtensorMap* ma = tma_map(s, a, 0);
    const CUtensorMap* mb = b ? tma_map(s, b, 0) : ma;
    const CUtensorMap* kx = tma_map(s, chunk->vec_kx, 1);
    const CUtensorMap* ky = tma_map(s, chunk->vec_ky, 2);
    const CUtensorMap* kz = tma_map(s, chunk->vec_kz, 3);
    if (!(ma && mb && kx && ky && kz)) return false;
    *m = Tma3Maps{*ma, *mb, *kx, *ky, *kz};
    return true;
}

// Raises a TMA-fed kernel's dynamic shared-memory limit once per device
// (`set`: the caller's record of devices done).
template <typename Kernel>
static void raise_ring_smem(TlSuite3D* s, Kernel kernel, unsigned& set)
{
    if (set & (1u << (s->device & 31))) return;
    TL_CUDA(cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTmaRingBytes));
    set |= 1u << (s->device & 31);
}
}  // namespace tl3d
