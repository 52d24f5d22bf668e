// batch2d.cu -- many independent 2D timesteps in one persistent launch.
//
// A batch holds `count` initialised chunks of different sizes (each with its
// own tea.in settings). One batched timestep runs, for every problem, the
// reference's solve() (2d/diffuse.c:22-80) with the CG solve replaced by the
// refinement CG of refine2d.cuh (FP32 vectors and coefficients, FP64
// arithmetic, dot products and solution, FP64 residual replacement) stopped
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
// count growing with the grid's side) and at least one block. Tiles are
// handed out per problem by a monotonic counter whose index names both the
// phase -- w = A p, then the u/r update, then (when the problem asked for
// one) the FP64 fold and residual -- and the tile; a block whose index lies
// in a later phase waits (bounded by a clock limit: a timeout sets an error
// word and every block returns) until the phases before it completed.
// Problems therefore advance at their own pace, and a block whose problem
// converged moves to the unfinished problem with the most cells per block
// working on it, so the long tail of the largest problems gets the whole
// grid. Per-problem dot products are reduced deterministically: each tile
// writes its block sum, and the block finishing the problem's last tile of
// the phase sums the problem's tile partials in tile order and runs the CG
// scalar update (alpha, beta, replacement and stop decisions) for it.
//
// tile_rows (and the persistent grid size the groups share) come from the
// autotuner (tl2d_batch_tune): it times a few iterations of the real batch
// with each candidate and keeps the fastest.
#include "refine2d.cuh"
#include "suite2d_impl.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

using namespace tl2d;
using namespace tl2d::rf;

namespace {

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
    int err;          // a phase wait timed out
    int iters;        // most iterations any problem ran
    long long limit;  // SM clocks a phase wait may take before it gives up (kept across steps)
};

// Per-problem schedule of the persistent kernel. Tiles are handed out by a
// monotonic counter: index t is tile t % nt of phase t / nt, so a block that
// takes an index knows which phase it belongs to and waits (bounded) until
// the phases before it have completed; the block that completes a phase's
// last tile runs the phase's scalar update, sets the next phase's kind and
// then advances gen.
enum { PH_W = 0, PH_UR = 1, PH_FOLD = 2, PH_RESID = 3, PH_DONE = 4 };
struct PCtl {
    unsigned next;    // tile indices handed out
    unsigned gen;     // phases completed
    int kind;         // kind of phase `gen`
    int it;           // CG iteration of phase `gen`
    int helpers;      // blocks that have worked on the problem
    int pad;
};

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
    for (int k = threadIdx.x; k < nt; k += BX)
#pragma unroll
        for (int r = 0; r < N; ++r) s[r] += *(volatile double*)&partials[(long)(P.tile0 + k) * 2 + r];
    __syncthreads();
    tl::block_sum<N, BX>(s, smem);
    if (threadIdx.x == 0) {
#pragma unroll
        for (int r = 0; r < N; ++r) tot[r] = s[r];
        *ticket = 0u;
    }
    return true;
}

// The not-converged problem with the most cells per block that has worked
// on it (warp 0 scans; lane 0 counts itself in and returns it), or -1.
__device__ int pick_problem(const BProb* __restrict__ P, PCtl* pc, int np)
{
    const int lane = threadIdx.x & 31;
    double best = -1.0;
    int who = -1;
    for (int b = lane; b < np; b += 32) {
        if (vol_read(&pc[b].kind) == PH_DONE) continue;
        const double score = (double)P[b].L.nx * P[b].L.ny / (double)(vol_read(&pc[b].helpers) + 1);
        if (score > best) {
            best = score;
            who = b;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
        const double ob = __shfl_down_sync(0xffffffffu, best, o);
        const int ow = __shfl_down_sync(0xffffffffu, who, o);
        if (ob > best) {
            best = ob;
            who = ow;
        }
    }
    if (lane == 0 && who >= 0) atomicAdd(&pc[who].helpers, 1);
    return who;
}

__global__ void __launch_bounds__(BX, kBatchMinB) k_batch_cg(const BProb* __restrict__ P, int np,
                                                             const int* __restrict__ block_prob, MxState* st,
                                                             unsigned* tickets, double* partials, PCtl* pc,
                                                             BCtl* ctl, int max_iters)
{
    __shared__ int sh_b, sh_go;
    __shared__ unsigned sh_t;
    int b = block_prob[blockIdx.x];
    for (;;) {
        // a problem to work on: the block's own, then the most loaded one left
        if (threadIdx.x < 32) {
            int nb = b;
            if (vol_read(&pc[b].kind) == PH_DONE) nb = pick_problem(P, pc, np);
            if (threadIdx.x == 0) sh_b = nb;
        }
        __syncthreads();
        b = sh_b;
        if (b < 0) return;
        const BProb& Q = P[b];
        const unsigned nt = (unsigned)(Q.tx * Q.ty);
        // take a tile index and wait until its phase is the current one
        if (threadIdx.x == 0) {
            const unsigned t = atomicAdd(&pc[b].next, 1u);
            const unsigned phase = t / nt;
            int go = 1;   // 1: work, 0: the problem ended, -1: error
            const long long t0 = clock64();
            while (*(volatile unsigned*)&pc[b].gen < phase) {
                if (vol_read(&pc[b].kind) == PH_DONE) {
                    go = 0;
                    break;
                }
                if (vol_read(&ctl->err)) {
                    go = -1;
                    break;
                }
                if (clock64() - t0 > ctl->limit) {
                    atomicExch(&ctl->err, 1);
                    go = -1;
                    break;
                }
                __nanosleep(64);
            }
            __threadfence();
            if (go == 1 && vol_read(&pc[b].kind) == PH_DONE) go = 0;
            sh_t = t % nt;
            sh_go = go;
        }
        __syncthreads();
        const int go = sh_go;
        const int lt = (int)sh_t;
        __syncthreads();   // sh_* are rewritten by the next pass
        if (go < 0) return;
        if (go == 0) continue;
        const int tx = lt % Q.tx, ty = lt / Q.tx;
        const int kind = vol_read(&pc[b].kind), it = vol_read(&pc[b].it);
        double v[2] = {0.0, 0.0};
        if (kind == PH_W) {
            float* pin = Q.f[it == 0 ? BF_P0 : (((it - 1) & 1) ? BF_P1 : BF_P0)];
            float* pout = Q.f[(it & 1) ? BF_P1 : BF_P0];
            v[0] = it == 0 ? rf_w_tile<float, false>(Q.L, tx, ty, 0.0, pin, pin, Q.f[BF_R], Q.f[BF_W], Q.f[BF_KX],
                                                      Q.f[BF_KY])
                           : rf_w_tile<float, true>(Q.L, tx, ty, st[b].beta, pin, pout, Q.f[BF_R], Q.f[BF_W],
                                                     Q.f[BF_KX], Q.f[BF_KY]);
        } else if (kind == PH_UR) {
            v[0] = rf_ur_tile<float>(Q.L, tx, ty, st[b].alpha, Q.f[BF_XS], Q.f[(it & 1) ? BF_P1 : BF_P0], Q.f[BF_R],
                                     Q.f[BF_W]);
        } else if (kind == PH_FOLD) {
            rf_fold_tile<float>(Q.L, tx, ty, Q.gx, Q.hd, Q.u, Q.f[BF_XS]);
        } else {
            rf_resid_tile<float>(Q.L, tx, ty, Q.gx, Q.hd, Q.u, Q.u0, Q.kx, Q.ky, Q.f[BF_R], v);
        }
        double tot[2];
        if (tile_done<2>(v, Q.tile0 + lt, Q, &tickets[b], partials, tot) && threadIdx.x == 0) {
            // the phase is complete: its scalar update, then the next phase
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
            atomicAdd(&pc[b].gen, 1u);
        }
    }
}

// Clears the per-problem tile tickets and schedules (a step whose wait gave
// up may have left them mid-phase) and the step's control words; the clock
// limit is kept. A problem the setup already converged starts done.
__global__ void k_batch_reset(const BProb* __restrict__ P, const MxState* st, int np, BCtl* ctl,
                              unsigned* tickets, PCtl* pc)
{
    for (int b = threadIdx.x; b < np; b += blockDim.x) {
        tickets[b] = 0u;
        pc[b].next = 0u;
        pc[b].gen = 0u;
        pc[b].kind = st[b].done ? PH_DONE : PH_W;
        pc[b].it = 0;
        pc[b].helpers = P[b].gsize;
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
    k_batch_reset<<<1, 128, 0, B->stream>>>(B->d_prob, B->d_st, B->count, B->d_ctl, B->d_tickets, B->d_pctl);
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
