// batch2d.cu -- many independent 2D timesteps in one persistent launch.
//
// A batch holds `count` initialised chunks of different sizes (each with its
// own tea.in settings). One batched timestep runs, for every problem, the
// reference's solve() (2d/diffuse.c:22-80) with the CG solve replaced by the
// refinement CG of refine2d.cuh (FP32 vectors and coefficients, FP32
// arithmetic in the sweeps, FP64 dot products, scalars and solution, FP64
// residual replacement) stopped
// when the FP64 residual satisfies the problem's own r.r < eps:
//
//   per problem: energy/density halos, cg_init, u0 = u, T-layout setup
//   ONE persistent cooperative kernel: the CG iterations of all problems
//   per problem: energy = u / density, energy halo
//
// captured once into a CUDA graph and replayed for every timestep.
//
// The persistent kernel starts every problem with its own group of blocks,
// sized by the problem's estimated work (cells x (nx + ny), CG's iteration
// count growing with the grid's side) and at least one block. Each problem
// walks its phases -- w = A p, then the u/r update, then (when the problem
// asked for one) the FP64 fold and residual -- with its tiles handed out by
// an atomic counter per problem; a block whose problem has no tile left in
// its open phase takes one from the problem with the most tiles left, so no
// block idles at a problem's phase boundary while other problems have work,
// and the largest problems get the whole grid once the small ones have
// converged. A block holds at most one tile and never waits while holding
// it; only a block that finds no tile anywhere polls, bounded by a clock
// limit (a timeout sets an error word and the blocks return). Per-problem
// dot products are reduced deterministically: each tile writes its block
// sum, and the block finishing the problem's last tile of the phase sums
// the problem's tile partials in tile order and runs the CG scalar update
// (alpha, beta, replacement and stop decisions) for it, then opens the
// problem's next phase.
//
// tile_rows (and the persistent grid size the groups share) come from the
// autotuner (tl2d_batch_tune): it times a few iterations of the real batch
// with each candidate and keeps the fastest.
#include "refine2d.cuh"
#include "suite2d_impl.hpp"

#include <algorithm>
#include <cmath>
#include <type_traits>
#include <vector>

using namespace tl2d;
using namespace tl2d::rf;

namespace {

// Arithmetic of the batch's FP32 sweeps (dot products and scalars are FP64
// either way): FP32 (TL2D_BATCH_MATH_F32 1; 785 against 846 ms for the
// 64-problem step, the same iterations) or FP64 on the FP32 values (0).
#ifndef TL2D_BATCH_MATH_F32
#define TL2D_BATCH_MATH_F32 1
#endif
using BatchM = std::conditional_t<TL2D_BATCH_MATH_F32 != 0, float, double>;

constexpr int kBatchMinB = 8;                    // resident blocks per SM of the persistent kernel
constexpr long long kWaitLimit = 4000000000LL;   // default: SM clocks a phase wait may take (~2 s)

enum { BF_KX = 0, BF_KY, BF_P0, BF_P1, BF_W, BF_R, BF_XS, BF_COUNT };

struct BProb {
    Lay L;
    int tx, ty;      // tiles per row / column
    int tile0;       // first global tile of this problem
    int g0, gsize;   // the problem's group: blocks g0 .. g0 + gsize - 1
    int gx, hd;      // FP64 chunk arrays: row length, halo depth
    float* f[BF_COUNT];
    double* u;
    const double* u0;
    const double* kx;
    const double* ky;
};

struct BCtl {
    int err;          // a block found no tile to work on for longer than the limit
    int iters;        // most iterations any problem ran
    long long limit;  // SM clocks a block may go without a tile before it gives up (kept across steps)
};

// Per-problem schedule of the persistent kernel. One 64-bit word holds the
// open phase (high half) and the tiles handed out in it (low half): a block
// takes tile t with one atomic add and holds a tile of that phase exactly
// when t < tiles per phase. The block completing the phase's last tile runs
// the phase's scalar update, writes the next phase's kind and iteration and
// opens it by swapping in (phase + 1) << 32; a finished problem's low half
// is kClosed, so every later draw comes back void. A block never waits
// while it holds a tile: when its problem has no tile left in the open
// phase it takes one from the problem with the most tiles left, and only
// when no problem has one does it poll (bounded by the clock limit).
enum { PH_W = 0, PH_UR = 1, PH_FOLD = 2, PH_RESID = 3, PH_DONE = 4 };
constexpr unsigned kClosed = 0x40000000u;
struct PCtl {
    unsigned long long word;   // open phase << 32 | tiles handed out in it
    int kind;                  // kind of the open phase
    int it;                    // CG iteration of the open phase
};

__device__ __forceinline__ unsigned long long vol_read64(const unsigned long long* p)
{
    return *(volatile const unsigned long long*)p;
}

// Block sum of this thread's values; returns true in every thread of the
// block that completed problem b's last tile of the phase, with the
// problem's totals (fixed-order sum of its tile partials) in tot (thread 0).
template <int N>
__device__ bool tile_done(double (&v)[N], int t, const BProb& P, unsigned* ticket, double* partials,
                          double (&tot)[N])
{
    __shared__ double smem[N][BX / tl::kWarp];
    __shared__ bool last;
    __syncthreads();
    tl::block_sum<N, BX>(v, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) partials[(long)t * 2 + r] = v[r];
        __threadfence();
        last = atomicAdd(ticket, 1u) == (unsigned)(P.tx * P.ty - 1);
    }
    __syncthreads();
    if (!last) return false;
    __threadfence();
    double s[N];
#pragma unroll
    for (int r = 0; r < N; ++r) s[r] = 0.0;
    const int nt = P.tx * P.ty;
    // partials k = tid, tid + BX, ... added in that order; four loads in flight
    for (int k0 = threadIdx.x; k0 < nt; k0 += 4 * BX) {
        double q[4][N];
#pragma unroll
        for (int u = 0; u < 4; ++u)
#pragma unroll
            for (int r = 0; r < N; ++r)
                q[u][r] = k0 + u * BX < nt ? __ldcg(&partials[(long)(P.tile0 + k0 + u * BX) * 2 + r]) : 0.0;
#pragma unroll
        for (int u = 0; u < 4; ++u)
            if (k0 + u * BX < nt)
#pragma unroll
                for (int r = 0; r < N; ++r) s[r] += q[u][r];
    }
    __syncthreads();
    tl::block_sum<N, BX>(s, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) tot[r] = s[r];
        *ticket = 0u;
    }
    return true;
}

// Warp 0: the unfinished problem with the most tiles not yet handed out in
// its open phase (the lowest index among equals); -1 when every problem has
// finished, -2 when none has a tile to hand out right now.
__device__ int find_work(const BProb* __restrict__ P, PCtl* pc, int np)
{
    const int lane = threadIdx.x & 31;
    int best = 0, who = -1;
    bool live = false;
    for (int b = lane; b < np; b += 32) {
        const unsigned lo = (unsigned)vol_read64(&pc[b].word);
        if (lo >= kClosed) continue;
        live = true;
        const unsigned nt = (unsigned)(P[b].tx * P[b].ty);
        if (lo < nt && (int)(nt - lo) > best) {
            best = (int)(nt - lo);
            who = b;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const int ob = __shfl_down_sync(0xffffffffu, best, o);
        const int ow = __shfl_down_sync(0xffffffffu, who, o);
        if (ob > best || (ob == best && ow >= 0 && (who < 0 || ow < who))) {
            best = ob;
            who = ow;
        }
    }
    who = __shfl_sync(0xffffffffu, who, 0);
    live = __any_sync(0xffffffffu, live);
    return who >= 0 ? who : (live ? -2 : -1);
}

// Thread 0: draws a tile of problem b; true with its index in t and the
// phase in g when one was left in the open phase.
__device__ __forceinline__ bool draw(const BProb* __restrict__ P, PCtl* pc, int b, int& t, unsigned& g)
{
    const unsigned nt = (unsigned)(P[b].tx * P[b].ty);
    const unsigned long long old = atomicAdd(&pc[b].word, 1ull);
    if ((unsigned)old >= nt) return false;
    t = (int)(unsigned)old;
    g = (unsigned)(old >> 32);
    return true;
}

__global__ void __launch_bounds__(BX, kBatchMinB) k_batch_cg(const BProb* __restrict__ P, int np,
                                                             const int* __restrict__ block_prob, MxState* st,
                                                             unsigned* tickets, double* partials, PCtl* pc,
                                                             BCtl* ctl, int max_iters)
{
    __shared__ int sh_go, sh_b, sh_t, sh_kind, sh_it;
    __shared__ unsigned sh_g;
    __shared__ double sh_coef;
    int b = block_prob[blockIdx.x];
    long long idle0 = clock64();
    for (;;) {
        if (threadIdx.x < 32) {
            int go = 0, t = 0;   // 1: a tile of problem b, 0: none right now, -1: leave
            unsigned g = 0;
            if (threadIdx.x == 0 && (unsigned)vol_read64(&pc[b].word) < (unsigned)(P[b].tx * P[b].ty))
                go = draw(P, pc, b, t, g) ? 1 : 0;
            go = __shfl_sync(0xffffffffu, go, 0);
            if (go == 0) {
                const int nb = find_work(P, pc, np);
                if (threadIdx.x == 0) {
                    if (nb == -1) {
                        go = -1;
                    } else if (nb >= 0 && draw(P, pc, nb, t, g)) {
                        go = 1;
                        b = nb;
                    }
                }
            }
            if (threadIdx.x == 0) {
                if (go == 1) {
                    __threadfence();   // the phase's kind, scalars and fields are those its opener published
                    idle0 = clock64();
                    const int kind = vol_read(&pc[b].kind);
                    sh_kind = kind;
                    sh_it = vol_read(&pc[b].it);
                    sh_coef = kind == PH_W ? __ldcg(&st[b].beta) : kind == PH_UR ? __ldcg(&st[b].alpha) : 0.0;
                } else if (go == 0) {
                    if (vol_read(&ctl->err)) {
                        go = -1;
                    } else if (clock64() - idle0 > ctl->limit) {
                        atomicExch(&ctl->err, 1);
                        go = -1;
                    } else {
                        __nanosleep(64);
                    }
                }
                sh_go = go;
                sh_b = b;
                sh_t = t;
                sh_g = g;
            }
        }
        __syncthreads();
        const int go = sh_go, lt = sh_t, kind = sh_kind, it = sh_it;
        const unsigned g = sh_g;
        const double coef = sh_coef;
        b = sh_b;
        __syncthreads();   // sh_* are rewritten by the next pass
        if (go < 0) return;
        if (go == 0) continue;
        const BProb& Q = P[b];
        const int tx = lt % Q.tx, ty = lt / Q.tx;
        double v[2] = {0.0, 0.0};
        if (kind == PH_W) {
            float* pin = Q.f[it == 0 ? BF_P0 : (((it - 1) & 1) ? BF_P1 : BF_P0)];
            float* pout = Q.f[(it & 1) ? BF_P1 : BF_P0];
            v[0] = it == 0 ? rf_w_tile<float, false, true, BatchM>(Q.L, tx, ty, 0.0, pin, pin, Q.f[BF_R],
                                                                    Q.f[BF_W], Q.f[BF_KX], Q.f[BF_KY])
                           : rf_w_tile<float, true, true, BatchM>(Q.L, tx, ty, coef, pin, pout, Q.f[BF_R],
                                                                   Q.f[BF_W], Q.f[BF_KX], Q.f[BF_KY]);
        } else if (kind == PH_UR) {
            v[0] = rf_ur_tile<float, true, BatchM>(Q.L, tx, ty, coef, Q.f[BF_XS], Q.f[(it & 1) ? BF_P1 : BF_P0],
                                                   Q.f[BF_R], Q.f[BF_W]);
        } else if (kind == PH_FOLD) {
            rf_fold_tile<float, true>(Q.L, tx, ty, Q.gx, Q.hd, Q.u, Q.f[BF_XS]);
        } else {
            rf_resid_tile<float, true>(Q.L, tx, ty, Q.gx, Q.hd, Q.u, Q.u0, Q.kx, Q.ky, Q.f[BF_R], v);
        }
        double tot[2];
        if (tile_done<2>(v, Q.tile0 + lt, Q, &tickets[b], partials, tot) && threadIdx.x == 0) {
            // the phase is complete: its scalar update, then open the next phase
            int next = PH_W, nit = it;
            if (kind == PH_W) {
                FinMxW{&st[b]}(tot);
                next = PH_UR;
            } else if (kind == PH_UR) {
                FinMxUr{&st[b], nullptr}(tot);
                if (st[b].upd) next = PH_FOLD;
                else nit = it + 1;
            } else if (kind == PH_FOLD) {
                next = PH_RESID;
            } else {
                FinMxRes{&st[b], nullptr}(tot);
                nit = it + 1;
                if (st[b].done) next = PH_DONE;
            }
            if (next == PH_W && nit >= max_iters) next = PH_DONE;
            if (next == PH_DONE) atomicMax(&ctl->iters, nit);
            pc[b].it = nit;
            pc[b].kind = next;
            __threadfence();
            atomicExch(&pc[b].word, ((unsigned long long)(g + 1u) << 32) | (next == PH_DONE ? kClosed : 0u));
        }
    }
}

// Clears the per-problem tile tickets and schedules (a step that gave up may
// have left them mid-phase) and the step's control words; the clock limit is
// kept. A problem the setup already converged starts closed.
__global__ void k_batch_reset(const MxState* st, int np, BCtl* ctl, unsigned* tickets, PCtl* pc)
{
    for (int b = threadIdx.x; b < np; b += blockDim.x) {
        const bool done = st[b].done != 0;
        tickets[b] = 0u;
        pc[b].word = done ? kClosed : 0ull;
        pc[b].kind = done ? PH_DONE : PH_W;
        pc[b].it = 0;
    }
    if (threadIdx.x == 0) {
        ctl->err = 0;
        ctl->iters = 0;
    }
}

}  // namespace

// ------------------------------------------------------------------ batch --

struct TlBatch {
    int count = 0;
    int device = 0;
    int sm_count = 148;
    cudaStream_t stream = nullptr;
    std::vector<Chunk*> chunks;
    std::vector<Settings*> settings;
    std::vector<TlSuite2D*> suites;
    std::vector<Lay> lay;
    void* slab = nullptr;            // FP32 arrays of every problem
    size_t slab_bytes = 0;
    std::vector<size_t> field_off;   // per problem: offset of its first FP32 array
    std::vector<size_t> field_bytes; // per problem: bytes of one FP32 array
    BProb* d_prob = nullptr;
    int* d_block_prob = nullptr;     // problem of every block of the persistent grid
    PCtl* d_pctl = nullptr;          // per-problem schedules
    MxState* d_st = nullptr;
    unsigned* d_tickets = nullptr;
    double* d_partials = nullptr;
    BCtl* d_ctl = nullptr;
    tl::ReduceSlots rs{};
    long rs_capacity = 0;
    DevState* d_scratch_state = nullptr;
    int max_tiles = 0;               // capacity of the tile tables
    int ntiles = 0;
    int tile_rows = 0;
    int grid_blocks = 0;             // blocks the groups share (co-resident limit at most)
    int launch_blocks = 0;           // blocks launched: the sum of the group sizes
    int max_grid = 0;
    int max_iters = 0;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    bool graph_ok = false;
};

namespace {

void batch_free(TlBatch* B)
{
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    void* ptrs[] = {B->slab, B->d_prob, B->d_block_prob, B->d_pctl, B->d_st, B->d_tickets, B->d_partials, B->d_ctl,
                    B->rs.partials, B->rs.ticket, B->rs.out_dev, B->d_scratch_state};
    for (void* p : ptrs)
        if (p) cudaFree(p);
    if (B->stream) cudaStreamDestroy(B->stream);
    delete B;
}

// Splits the grid_blocks blocks into one group per problem, in proportion
// to the estimated work cells x (nx + ny) (CG's iteration count grows with
// the grid's side), at least one block and at most one per tile of the
// problem's finest tiling; lays out the tiles for tile_rows and uploads the
// problem and block tables. tile_rows > 0: that height for every problem;
// kAdaptiveRows: per problem the height that gives its group about one tile
// per block per phase (between 2 and 64 rows).
constexpr int kAdaptiveRows = -1;

bool batch_layout(TlBatch* B, int tile_rows)
{
    const int n = B->count;
    std::vector<double> work(n);
    std::vector<long> cap(n);
    double total = 0.0;
    for (int b = 0; b < n; ++b) {
        Lay L = B->lay[b];
        work[b] = (double)L.nx * L.ny * (double)(L.nx + L.ny);
        total += work[b];
        L.rows = tile_rows > 0 ? tile_rows : 2;
        const dim3 t = lay_tiles<float>(L);
        cap[b] = (long)t.x * t.y;
    }
    if (B->grid_blocks < n) {
        tl::fail(62, "batch: %d problems need at least %d blocks, the grid has %d", n, n, B->grid_blocks);
        return false;
    }
    std::vector<int> size(n);
    long used = 0;
    for (int b = 0; b < n; ++b) {
        size[b] = (int)std::min<long>(cap[b], std::max<long>(1, (long)(B->grid_blocks * work[b] / total)));
        used += size[b];
    }
    while (used > B->grid_blocks) {   // the one-block minimum overshot: trim the largest groups
        int k = (int)(std::max_element(size.begin(), size.end()) - size.begin());
        --size[k];
        --used;
    }
    while (used < B->grid_blocks) {   // hand the rest to the most loaded groups per block
        int k = -1;
        double best = 0.0;
        for (int b = 0; b < n; ++b)
            if (size[b] < cap[b] && work[b] / size[b] > best) {
                best = work[b] / size[b];
                k = b;
            }
        if (k < 0) break;
        ++size[k];
        ++used;
    }
    std::vector<BProb> P(n);
    std::vector<int> bp;
    int tiles = 0;
    for (int b = 0; b < n; ++b) {
        Lay L = B->lay[b];
        if (tile_rows == kAdaptiveRows) {
            L.rows = 64;
            const long tx = lay_tiles<float>(L).x;
            L.rows = (int)std::min<long>(64, std::max<long>(2, (L.ny * tx + size[b] - 1) / size[b]));
        } else {
            L.rows = tile_rows;
        }
        B->lay[b] = L;
        const dim3 t = lay_tiles<float>(L);
        BProb& Q = P[b];
        Q.L = L;
        Q.tx = (int)t.x;
        Q.ty = (int)t.y;
        Q.tile0 = tiles;
        tiles += Q.tx * Q.ty;
        Q.g0 = (int)bp.size();
        Q.gsize = std::min(size[b], Q.tx * Q.ty);
        for (int k = 0; k < Q.gsize; ++k) bp.push_back(b);
        Q.gx = B->suites[b]->g.x;
        Q.hd = B->suites[b]->g.hd;
        char* base = (char*)B->slab + B->field_off[b];
        for (int k = 0; k < BF_COUNT; ++k) Q.f[k] = (float*)(base + B->field_bytes[b] * k);
        Chunk* c = B->chunks[b];
        Q.u = c->u;
        Q.u0 = c->u0;
        Q.kx = c->kx;
        Q.ky = c->ky;
    }
    if (tiles > B->max_tiles) {
        tl::fail(62, "batch: %d tiles exceed the table capacity %d", tiles, B->max_tiles);
        return false;
    }
    B->ntiles = tiles;
    B->tile_rows = tile_rows;
    B->launch_blocks = (int)bp.size();
    if (!TL_CUDA(cudaMemcpyAsync(B->d_prob, P.data(), sizeof(BProb) * P.size(), cudaMemcpyHostToDevice, B->stream)))
        return false;
    if (!TL_CUDA(cudaMemcpyAsync(B->d_block_prob, bp.data(), sizeof(int) * bp.size(), cudaMemcpyHostToDevice,
                                 B->stream)))
        return false;
    return TL_CUDA(cudaStreamSynchronize(B->stream));
}

void launch_halos(TlBatch* B, int b, int depth, std::initializer_list<double*> fields)
{
    TlSuite2D* s = B->suites[b];
    Chunk* c = B->chunks[b];
    HaloArgs a{};
    for (double* f : fields) a.f[a.nf++] = f;
    for (int f = 0; f < 4; ++f) a.ext[f] = c->neighbours[f] == TL_EXTERNAL_FACE;
    const long per = (long)depth * (2L * (s->g.y - 2 * s->g.hd) + 2L * (s->g.x - 2 * s->g.hd));
    k_local_halos<<<dim3(tl::ceil_div(per, 256), a.nf), 256, 0, B->stream>>>(s->g, depth, a);
}

// Everything of one batched timestep, issued on B->stream (capturable).
// iter_cap limits the iterations of the persistent kernel; finish = run the
// per-problem finalise (a full timestep) or stop after the solve (tuning).
void issue_step(TlBatch* B, int iter_cap, bool finish)
{
    for (int b = 0; b < B->count; ++b) {
        TlSuite2D* s = B->suites[b];
        Chunk* c = B->chunks[b];
        Settings* st = B->settings[b];
        const double dt = c->dt_init < st->dt_init ? c->dt_init : st->dt_init;
        const double rx = dt / (st->dx * st->dx), ry = dt / (st->dy * st->dy);
        launch_halos(B, b, 2, {c->density, c->energy});
        k_cg_init<<<full_grid(s->g), FB, 0, B->stream>>>(s->g, st->coefficient, rx, ry, c->density, c->energy, c->u,
                                                          c->p, nullptr, c->r, c->w, c->kx, c->ky, B->rs,
                                                          FinCgInit{B->d_scratch_state, nullptr});
        k_copy_u<<<interior_grid(s->g), BX, 0, B->stream>>>(s->g, c->u0, c->u);
        char* base = (char*)B->slab + B->field_off[b];
        float* f[BF_COUNT];
        for (int k = 0; k < BF_COUNT; ++k) f[k] = (float*)(base + B->field_bytes[b] * k);
        k_rf_init<float><<<B->sm_count, 256, 0, B->stream>>>(
            s->g.x, s->g.hd, B->lay[b], c->r, c->u0, c->kx, c->ky, f[BF_KX], f[BF_KY], f[BF_R], f[BF_P0], f[BF_P1],
            f[BF_W], f[BF_XS], B->rs, FinMxInit{&B->d_st[b], 0.0, st->eps, st->max_iters, nullptr});
    }
    k_batch_reset<<<1, 128, 0, B->stream>>>(B->d_st, B->count, B->d_ctl, B->d_tickets, B->d_pctl);
    void* args[] = {&B->d_prob, &B->count, &B->d_block_prob, &B->d_st, &B->d_tickets, &B->d_partials, &B->d_pctl,
                    &B->d_ctl, &iter_cap};
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = dim3(B->launch_blocks);
    cfg.blockDim = dim3(BX);
    cfg.stream = B->stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaLaunchKernelExC(&cfg, (const void*)k_batch_cg, args);
    if (!finish) return;
    for (int b = 0; b < B->count; ++b) {
        TlSuite2D* s = B->suites[b];
        Chunk* c = B->chunks[b];
        k_finalise<<<interior_grid(s->g), BX, 0, B->stream>>>(s->g, c->energy, c->density, c->u);
        launch_halos(B, b, 1, {c->energy});
    }
}

bool check_ctl(TlBatch* B, BCtl* out)
{
    BCtl h{};
    if (!TL_CUDA(cudaMemcpyAsync(&h, B->d_ctl, sizeof(BCtl), cudaMemcpyDeviceToHost, B->stream))) return false;
    if (!TL_CUDA(cudaStreamSynchronize(B->stream))) return false;
    if (h.err) {
        tl::fail(63, "batch: a phase wait of the persistent kernel timed out");
        return false;
    }
    if (out) *out = h;
    return true;
}

void drop_graph(TlBatch* B)
{
    if (B->exec) cudaGraphExecDestroy(B->exec);
    if (B->graph) cudaGraphDestroy(B->graph);
    B->exec = nullptr;
    B->graph = nullptr;
    B->graph_ok = false;
}

}  // namespace

extern "C" {

TlBatch* tl2d_batch_create(Chunk** chunks, Settings** settings, int count, int tile_rows, int grid_blocks)
{
    if (tl::failed()) return nullptr;
    if (!chunks || !settings || count < 1) {
        tl::fail(60, "tl2d_batch_create: need count >= 1 chunks and settings");
        return nullptr;
    }
    TlBatch* B = new TlBatch();
    B->count = count;
    TL_CUDA(cudaGetDevice(&B->device));
    TL_CUDA(cudaDeviceGetAttribute(&B->sm_count, cudaDevAttrMultiProcessorCount, B->device));
    if (!TL_CUDA(cudaStreamCreateWithFlags(&B->stream, cudaStreamNonBlocking))) {
        batch_free(B);
        return nullptr;
    }
    long max_full = 1;
    size_t total = 0;
    for (int b = 0; b < count; ++b) {
        TlSuite2D* s = suite_of(chunks[b]);
        if (!s) {
            batch_free(B);
            return nullptr;
        }
        const Faces fc = faces_of(chunks[b]);
        if (settings[b]->num_chunks_per_rank != 1 || !(fc.l && fc.r && fc.b && fc.t) ||
            (settings[b]->coefficient != TL_CONDUCTIVITY && settings[b]->coefficient != TL_RECIP_CONDUCTIVITY)) {
            tl::fail(61, "tl2d_batch_create: problem %d needs one chunk, four external faces, a valid coefficient", b);
            batch_free(B);
            return nullptr;
        }
        TL_CUDA(cudaStreamSynchronize(s->stream));
        B->chunks.push_back(chunks[b]);
        B->settings.push_back(settings[b]);
        B->suites.push_back(s);
        const int nx = s->g.x - 2 * s->g.hd, ny = s->g.y - 2 * s->g.hd;
        B->lay.push_back(make_lay<float>(nx, ny, 2));
        const size_t fbytes = ((size_t)B->lay.back().cells() * sizeof(float) + 255) & ~(size_t)255;
        B->field_off.push_back(total);
        B->field_bytes.push_back(fbytes);
        total += fbytes * BF_COUNT;
        const dim3 gf = full_grid(s->g);
        max_full = std::max<long>(max_full, (long)gf.x * gf.y);
        B->max_iters = std::max(B->max_iters, settings[b]->max_iters);
    }
    // tile tables sized for the shortest tiles (2 rows)
    long tiles = 0;
    for (int b = 0; b < count; ++b) {
        const dim3 t = lay_tiles<float>(B->lay[b]);
        tiles += (long)t.x * t.y;
    }
    B->max_tiles = (int)tiles;
    B->rs_capacity = std::max<long>(max_full, B->sm_count) * tl::kMaxSums;
    bool ok = TL_CUDA(cudaMalloc(&B->slab, total)) && TL_CUDA(cudaMalloc(&B->d_prob, sizeof(BProb) * count)) &&
              TL_CUDA(cudaMalloc(&B->d_pctl, sizeof(PCtl) * count)) &&
              TL_CUDA(cudaMalloc(&B->d_st, sizeof(MxState) * count)) &&
              TL_CUDA(cudaMalloc(&B->d_tickets, sizeof(unsigned) * count)) &&
              TL_CUDA(cudaMalloc(&B->d_partials, sizeof(double) * 2 * tiles)) &&
              TL_CUDA(cudaMalloc(&B->d_ctl, sizeof(BCtl))) &&
              TL_CUDA(cudaMalloc(&B->rs.partials, sizeof(double) * B->rs_capacity)) &&
              TL_CUDA(cudaMalloc(&B->rs.ticket, 256)) && TL_CUDA(cudaMalloc(&B->rs.out_dev, 256)) &&
              TL_CUDA(cudaMalloc(&B->d_scratch_state, sizeof(DevState)));
    if (!ok) {
        batch_free(B);
        return nullptr;
    }
    B->slab_bytes = total;
    B->rs.out_host = nullptr;
    TL_CUDA(cudaMemsetAsync(B->rs.ticket, 0, 256, B->stream));
    TL_CUDA(cudaMemsetAsync(B->d_tickets, 0, sizeof(unsigned) * count, B->stream));
    TL_CUDA(cudaMemsetAsync(B->d_ctl, 0, sizeof(BCtl), B->stream));
    static const long long default_limit = kWaitLimit;
    TL_CUDA(cudaMemcpyAsync(&B->d_ctl->limit, &default_limit, sizeof(long long), cudaMemcpyHostToDevice, B->stream));
    int per_sm = 0;
    TL_CUDA(cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_batch_cg, BX, 0));
    B->max_grid = std::max(1, per_sm) * B->sm_count;
    B->grid_blocks = grid_blocks > 0 ? std::min(grid_blocks, B->max_grid) : B->max_grid;
    if (!TL_CUDA(cudaMalloc(&B->d_block_prob, sizeof(int) * B->max_grid))) {
        batch_free(B);
        return nullptr;
    }
    if (!batch_layout(B, tile_rows != 0 ? tile_rows : 16)) {
        batch_free(B);
        return nullptr;
    }
    return B;
}

void tl2d_batch_destroy(TlBatch* B)
{
    if (!B) return;
    cudaStreamSynchronize(B->stream);
    batch_free(B);
}

// Autotuner: times `trial_iters` iterations of the batch's own CG (setup
// included, energy untouched; 0: the whole solve) for each tile height in
// {adaptive (-1), 4, 8, 16, 32, 64}
// and each persistent grid of {2, 4, 6, 8} blocks per SM (within the
// co-residency limit), and keeps the fastest. Returns 0 or an error code;
// the choice is readable with tl2d_batch_config.
int tl2d_batch_tune(TlBatch* B, int trial_iters, double* best_ms)
{
    if (tl::failed()) return tl::error_state().code;
    if (!B || trial_iters < 0) {
        tl::fail(64, "tl2d_batch_tune: batch and trial_iters >= 0 are required");
        return 64;
    }
    const int iters = trial_iters > 0 ? trial_iters : B->max_iters;   // 0: the whole solve
    drop_graph(B);
    const int rows_c[] = {kAdaptiveRows, 4, 8, 16, 32, 64};
    const int per_sm_c[] = {2, 4, 6, 8};
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    double best = 1e300;
    int best_rows = B->tile_rows, best_grid = B->grid_blocks;
    for (int k : per_sm_c) {
        const int grid = std::min(B->max_grid, k * B->sm_count);
        B->grid_blocks = grid;
        for (int rows : rows_c) {
            if (!batch_layout(B, rows)) break;   // the adaptive heights depend on the grid
            for (int rep = 0; rep < 2; ++rep) {   // first run warms up
                cudaEventRecord(e0, B->stream);
                issue_step(B, iters, false);
                cudaEventRecord(e1, B->stream);
                if (!check_ctl(B, nullptr)) break;
            }
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            if (ms < best) {
                best = ms;
                best_rows = rows;
                best_grid = grid;
            }
        }
        if (tl::failed() || grid == B->max_grid) break;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (tl::failed()) return tl::error_state().code;
    B->grid_blocks = best_grid;
    batch_layout(B, best_rows);
    if (best_ms) *best_ms = best;
    return tl::failed() ? tl::error_state().code : 0;
}

void tl2d_batch_config(TlBatch* B, int* tile_rows, int* grid_blocks)
{
    if (!B) return;
    if (tile_rows) *tile_rows = B->tile_rows;
    if (grid_blocks) *grid_blocks = B->grid_blocks;
}

// One timestep of every problem of the batch (a CUDA graph replay after the
// first call). Per-problem outcomes through tl2d_batch_results.
int tl2d_batch_step(TlBatch* B, TlBatchStats* stats)
{
    if (tl::failed()) return tl::error_state().code;
    if (!B) {
        tl::fail(64, "tl2d_batch_step: null batch");
        return 64;
    }
    TlBatchStats local{};
    TlBatchStats* out = stats ? stats : &local;
    *out = TlBatchStats{};
    for (TlSuite2D* s : B->suites) TL_CUDA(cudaStreamSynchronize(s->stream));
    if (!B->exec && !B->graph_ok) {
        cudaGraph_t g = nullptr;
        cudaError_t e = cudaStreamBeginCapture(B->stream, cudaStreamCaptureModeThreadLocal);
        if (e == cudaSuccess) {
            issue_step(B, B->max_iters, true);
            e = cudaStreamEndCapture(B->stream, &g);
        }
        if (e == cudaSuccess && g) e = cudaGraphInstantiate(&B->exec, g, 0);
        if (e == cudaSuccess) {
            B->graph = g;
            B->graph_ok = true;
        } else {
            cudaGetLastError();   // capture unsupported here: the same launches run directly
            if (g) cudaGraphDestroy(g);
            B->exec = nullptr;
        }
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, B->stream);
    if (B->exec) TL_CUDA(cudaGraphLaunch(B->exec, B->stream));
    else issue_step(B, B->max_iters, true);
    cudaEventRecord(e1, B->stream);
    TL_CUDA(cudaGetLastError());
    BCtl ctl{};
    const bool ok = check_ctl(B, &ctl);
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (!ok) return tl::error_state().code;
    std::vector<MxState> st(B->count);
    TL_CUDA(cudaMemcpy(st.data(), B->d_st, sizeof(MxState) * B->count, cudaMemcpyDeviceToHost));
    out->problems = B->count;
    for (const MxState& m : st) {
        out->converged += m.reason == 1 ? 1 : 0;
        out->max_iterations = std::max(out->max_iterations, m.trip);
        out->total_iterations += m.trip;
    }
    out->kernel_iterations = ctl.iters;
    out->tile_rows = B->tile_rows;
    out->grid_blocks = B->grid_blocks;
    out->graph = B->exec ? 1 : 0;
    out->device_ms = ms;
    return tl::failed() ? tl::error_state().code : 0;
}

// How long (SM clocks) a phase wait of the persistent kernel may take
// before it gives up; cycles <= 0 restores the default (about 2 s). The
// limit lives in device memory, so captured graphs pick it up.
int tl2d_batch_set_wait_limit(TlBatch* B, long long cycles)
{
    if (!B) {
        tl::fail(64, "tl2d_batch_set_wait_limit: null batch");
        return 64;
    }
    const long long v = cycles > 0 ? cycles : kWaitLimit;
    if (!TL_CUDA(cudaMemcpyAsync(&B->d_ctl->limit, &v, sizeof(long long), cudaMemcpyHostToDevice, B->stream)) ||
        !TL_CUDA(cudaStreamSynchronize(B->stream)))
        return tl::error_state().code;
    return 0;
}

// Per-problem CG iterations and final FP64 residual r.r of the last step.
int tl2d_batch_results(TlBatch* B, int* iterations, double* rr, int* converged)
{
    if (!B) return 64;
    std::vector<MxState> st(B->count);
    if (!TL_CUDA(cudaMemcpy(st.data(), B->d_st, sizeof(MxState) * B->count, cudaMemcpyDeviceToHost)))
        return tl::error_state().code;
    for (int b = 0; b < B->count; ++b) {
        if (iterations) iterations[b] = st[b].trip;
        if (rr) rr[b] = st[b].rtrue;
        if (converged) converged[b] = st[b].reason == 1 ? 1 : 0;
    }
    return 0;
}

}  // extern "C"
