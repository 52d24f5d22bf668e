// suite2d.cu -- B200 (sm_100a) TeaLeaf 2D kernel suite behind the reference
// kernel interface (2d/kernel_interface.h:13-71).
//
// Data layout in HBM: every field is one cudaMalloc'd slice of a per-chunk
// slab, x*y FP64 values, index k + j*x (x fastest, halo included), exactly
// the layout the reference kernels index (2d/shared.h:49-54). Slices start on
// 256-byte boundaries.
//
// The kernels are in kernels2d.cuh. Reductions finish in one last-block pass
// that writes the scalar straight into mapped pinned host memory, so a
// run_* that returns a dot product costs one kernel and one stream sync.
//
// Deferred operations: run_cg_calc_p and run_local_halos return at once and
// record what was asked; the next sweep that can fuse it does the work
// (calc_w absorbs the p update and the reflective halo of p, calc_ur the
// halo of u), every other entry point first runs what is pending. A CG
// iteration of the reference drivers (calc_w, calc_ur, calc_p, halo(u,p))
// therefore costs two sweeps and 96 bytes per cell instead of four launches
// and 104 bytes. Because a fused p update reads the old p at the stencil
// neighbours, p alternates between two device buffers: chunk->p always points
// at the current one (the reference host reads chunk->p at every call).
//
// Floating point: this file is compiled with -fmad=false so each + - * / is
// one IEEE operation in the reference's expression order; element-wise
// results equal the reference's strict-IEEE build bit for bit, and dot
// products differ only by summation order.
#include "blocked2d.cuh"
#include "suite2d_impl.hpp"

#include <cuda_runtime.h>
#include <algorithm>
#include <cstring>

using namespace tl2d;
using tl::ReduceSlots;

bool tl_noalloc_prepare();   // noalloc2d.cu: reserves the allocation-free 2-norm's static scratch



// ================================================================= helpers

namespace tl2d {

TlSuite2D* suite_of(Chunk* chunk)
{
    if (!chunk || !chunk->ext || !chunk->ext->suite) {
        tl::fail(1, "chunk has no B200 suite state (run_kernel_initialise not called)");
        return nullptr;
    }
    return chunk->ext->suite;
}

bool fetch(TlSuite2D* s, int n, double* out)
{
    if (!TL_CUDA(cudaStreamSynchronize(s->stream))) return false;
    if (s->prof.on) s->prof.resolve();
    for (int i = 0; i < n; ++i) out[i] = s->h_out[i];
    return true;
}

Faces faces_of(const Chunk* chunk)
{
    const int* nb = chunk->neighbours;
    return Faces{nb[TL_CHUNK_LEFT] == TL_EXTERNAL_FACE, nb[TL_CHUNK_RIGHT] == TL_EXTERNAL_FACE,
                 nb[TL_CHUNK_BOTTOM] == TL_EXTERNAL_FACE, nb[TL_CHUNK_TOP] == TL_EXTERNAL_FACE};
}

FieldBufferType* field_slot(Chunk* chunk, AltField f)
{
    switch (f) {
        case ALT_P: return &chunk->p;
        case ALT_U: return &chunk->u;
        case ALT_R: return &chunk->r;
        default: return &chunk->sd;
    }
}

void swap_alt(TlSuite2D* s, Chunk* chunk, AltField f)
{
    FieldBufferType* slot = field_slot(chunk, f);
    double* cur = *slot;
    *slot = s->alt[f];
    s->alt[f] = cur;
}

static void launch_halos(TlSuite2D* s, Chunk* chunk, int depth, const int* which)
{
    // reference update order: density, p, energy0, energy1, u, sd (local_halos.c:40-45)
    const int order[TL_NUM_FIELDS] = {TL_FIELD_DENSITY, TL_FIELD_P, TL_FIELD_ENERGY0,
                                      TL_FIELD_ENERGY1, TL_FIELD_U, TL_FIELD_SD};
    FieldBufferType fields[TL_NUM_FIELDS] = {chunk->density, chunk->energy0, chunk->energy,
                                             chunk->u, chunk->p, chunk->sd};
    HaloArgs a{};
    for (int o = 0; o < TL_NUM_FIELDS; ++o)
        if (which[order[o]] == depth) a.f[a.nf++] = fields[order[o]];
    if (a.nf == 0) return;
    for (int f = 0; f < 4; ++f) a.ext[f] = chunk->neighbours[f] == TL_EXTERNAL_FACE;
    const long per = (long)depth * (2L * (s->g.y - 2 * s->g.hd) + 2L * (s->g.x - 2 * s->g.hd));
    TL_LAUNCH(s, "k_local_halos", k_local_halos<<<dim3(tl::ceil_div(per, 256), a.nf), 256, 0, s->stream>>>(s->g, depth, a));
}

// Runs the deferred PPCG inner steps (ppcg.c:9-61 as the reference drivers
// call them: sd = r / theta, then per step a depth-1 halo of sd and
// r -= A sd, u += sd, sd = a sd + b r): temporally blocked launches of up to
// Blk<1>::TB steps (the fold of each step at its start, sd reflected on the fly)
// and the last step's sd update, with the same results as one launch per
// call. With no step queued only sd = r / theta runs.
static void run_ppcg_queue(TlSuite2D* s, Chunk* chunk)
{
    s->pq.active = false;
    const int n = (int)s->pq.a.size();
    if (n == 0) {
        TL_LAUNCH(s, "k_ppcg_init",
                  k_ppcg_init<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->theta, chunk->r, chunk->sd));
        return;
    }
    TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, s->pq.a.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                            s->stream));
    TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, s->pq.b.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                            s->stream));
    // An even number of launches leaves r and sd in the buffers the chunk
    // pointed at: the host reads those pointers before its calls (e.g. the r
    // it passes to run_calculate_2norm), so a flush must not move them. An
    // odd count gets a closing zero-step launch, which copies the interior of
    // both and writes the depth-1 halo of sd (r's halo is left as the
    // one-step path leaves it: untouched).
    constexpr int TB = Blk<1>::TB;
    const int launches = (n + TB - 1) / TB;
    for (int q = 0; q < launches + (launches & 1); ++q) {
        const int pp0 = q * TB;
        const BlockedArgs a{std::max(0, std::min(TB, n - pp0)), std::min(pp0, n), 0, chunk->theta,
                            s->d_cheby_alphas, s->d_cheby_betas};
        launch_blocked<1>(s, "k_blocked<ppcg>", a, chunk->sd, chunk->r, s->alt[ALT_SD], s->alt[ALT_R], chunk->u,
                          chunk->u, nullptr, nullptr, chunk->kx, chunk->ky, nullptr);
        swap_alt(s, chunk, ALT_SD);
        swap_alt(s, chunk, ALT_R);
    }
    TL_LAUNCH(s, "k_ppcg_inner_b", k_ppcg_inner_b<<<interior_grid(s->g), BX, 0, s->stream>>>(
                                       s->g, s->pq.a[n - 1], s->pq.b[n - 1], chunk->sd, chunk->r));
    s->pq.a.clear();
    s->pq.b.clear();
}

// Runs the deferred Chebyshev trips (cheby.c:57-85 as the reference drivers
// call them: per trip a depth-1 halo of u, then w = A u, r = u0 - w,
// p = alpha p + beta r, u += p): temporally blocked launches of up to Blk<0>::TB
// trips, each trip ending with its u += p and u reflected on the fly; the
// last launch also writes w and r, and leaves u's halo as the call-by-call
// sequence does (mirroring u before the last add). The launches alternate
// buffers and the host holds the chunk's pointers, so their number is made
// even (a launch of two or more trips is split); a single trip runs as the
// one-step kernels. The same results as one launch per call.
static void run_cheby_queue(TlSuite2D* s, Chunk* chunk)
{
    s->cq.active = false;
    const int n = (int)s->cq.a.size();
    if (n == 0) return;
    std::vector<int> sizes;
    constexpr int TB = Blk<0>::TB;
    for (int left = n; left > 0; left -= TB) sizes.push_back(std::min(TB, left));
    if (sizes.size() % 2 == 1) {
        for (int q = (int)sizes.size() - 1; q >= 0; --q) {
            if (sizes[q] >= 2) {
                sizes[q] -= 1;
                sizes.insert(sizes.begin() + q + 1, 1);
                break;
            }
        }
    }
    if (sizes.size() % 2 == 1) {   // one trip: the absorbed halo update, then the one-step kernels
        int which[TL_NUM_FIELDS] = {0};
        which[TL_FIELD_U] = 1;
        launch_halos(s, chunk, 1, which);
        TL_LAUNCH(s, "k_cheby_sweep",
                  k_cheby_sweep<false><<<interior_grid(s->g), BX, 0, s->stream>>>(
                      s->g, s->cq.a[0], s->cq.b[0], 0.0, chunk->u, chunk->u0, chunk->p, chunk->r, chunk->w,
                      chunk->kx, chunk->ky));
        TL_LAUNCH(s, "k_add_p", k_add_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->p));
    } else {
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, s->cq.a.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                                s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, s->cq.b.data(), sizeof(double) * n, cudaMemcpyHostToDevice,
                                s->stream));
        int first = 0;
        for (size_t q = 0; q < sizes.size(); ++q) {
            const int steps = sizes[q];
            const BlockedArgs a{steps, first, first + steps == n ? 1 : 0, 0.0, s->d_cheby_alphas,
                                s->d_cheby_betas, 1};
            launch_blocked<0>(s, "k_blocked<cheby>", a, chunk->u, chunk->p, s->alt[ALT_U], s->alt[ALT_P], chunk->u0,
                              nullptr, chunk->w, chunk->r, chunk->kx, chunk->ky, nullptr);
            swap_alt(s, chunk, ALT_U);
            swap_alt(s, chunk, ALT_P);
            first += steps;
        }
    }
    s->cq.a.clear();
    s->cq.b.clear();
}

// Runs whichever deferred queue is open.
static void run_queues(TlSuite2D* s, Chunk* chunk)
{
    if (s->pq.active) run_ppcg_queue(s, chunk);
    if (s->cq.active) run_cheby_queue(s, chunk);
}

void flush(TlSuite2D* s, Chunk* chunk)
{
    run_queues(s, chunk);
    if (s->pend.calc_p) {
        TL_LAUNCH(s, "k_cg_calc_p",
                  k_cg_calc_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, s->pend.beta, chunk->p, chunk->r));
        s->pend.calc_p = false;
    }
    for (int d = 1; d <= s->g.hd; ++d) launch_halos(s, chunk, d, s->pend.halo);
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
}

}  // namespace tl2d

namespace {

bool check_geometry(Chunk* chunk, Settings* settings)
{
    if (chunk->x < 2 * settings->halo_depth + 1 || chunk->y < 2 * settings->halo_depth + 1 ||
        settings->halo_depth < 1) {
        tl::fail(2, "invalid chunk extents x=%d y=%d halo_depth=%d", chunk->x, chunk->y, settings->halo_depth);
        return false;
    }
    return true;
}

// Suite of a chunk with every deferred operation run (entry points that
// cannot fuse them).
TlSuite2D* ready(Chunk* chunk)
{
    if (tl::failed()) return nullptr;
    TlSuite2D* s = suite_of(chunk);
    if (s) flush(s, chunk);
    return s;
}

}  // namespace

// The bounded barrier wait of the TMA-fed sweeps, on a barrier that nothing
// completes: no copy is issued and nothing arrives, so the wait runs out
// after `polls` polls, and the give-up is recorded in `err` exactly as a
// sweep records it. Thread 0 waits; the block holds no copy in flight.
__global__ void k_bounded_wait_check(long polls, int* err)
{
    __shared__ __align__(8) unsigned long long bar;
    if (threadIdx.x == 0) {
        tl::mbar_init(&bar, 1);
        tl::mbar_fence_init();
    }
    __syncthreads();
    if (threadIdx.x == 0) tl::mbar_wait_limited(&bar, 0u, err, polls);
}

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

void tl2d_set_temporal_blocking(Chunk* chunk, int on)
{
    TlSuite2D* s = suite_of(chunk);
    if (s) s->temporal_blocking = on != 0;
}
void tl2d_set_tma(Chunk* chunk, int on)
{
    TlSuite2D* s = suite_of(chunk);
    if (s) s->tma = on != 0;
}
void tl2d_flush(Chunk* chunk) { ready(chunk); }

int tl2d_set_preconditioner(Chunk* chunk, int type)
{
    TlSuite2D* s = suite_of(chunk);
    if (!s) return tl::error_state().code;
    if (type < 0 || type > 2) {
        tl::fail(37, "tl2d_set_preconditioner: type %d is not 0 (none), 1 (jac_diag) or 2 (jac_block)", type);
        return 37;
    }
    s->precond = type;
    return 0;
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

int tl2d_check_bounded_wait(Chunk* chunk, long long polls)
{
    TlSuite2D* s = ready(chunk);
    if (!s) return tl::error_state().code;
    if (polls < 1 || polls > tl::kTmaSpinLimit) {
        tl::fail(36, "tl2d_check_bounded_wait: polls must be in [1, %ld]", tl::kTmaSpinLimit);
        return 36;
    }
    k_bounded_wait_check<<<1, 32, 0, s->stream>>>((long)polls, s->d_mirror + kTmaErrWord2);
    if (!TL_LAUNCHED("k_bounded_wait_check") || !TL_CUDA(cudaStreamSynchronize(s->stream))) return tl::error_state().code;
    if (tma_failed(s)) {
        tl::fail(35, "a bounded barrier wait gave up after %lld polls (wait check on a barrier nothing completes)",
                 polls);
        return 35;
    }
    return 0;
}

long long tl2d_launch_count(Chunk* chunk)
{
    TlSuite2D* s = suite_of(chunk);
    return s ? s->prof.launches : -1;
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
// Strips are cut for 8 resident blocks per SM: two whole waves of the
// TMA-fed CG sweeps (4 per SM) at 4096^2 (111-row strips), whose per-wave
// ring fill and tail then weigh half as much as with one wave of the
// 16-per-SM per-thread-load sweeps (measured: w sweep 143 against 148 us).
#ifndef TL2D_ROWS_BLOCKS
#define TL2D_ROWS_BLOCKS 8
#endif
    s->g.rows = choose_rows(chunk->x - 2 * settings->halo_depth, chunk->y - 2 * settings->halo_depth, s->sm_count,
                            TL2D_ROWS_BLOCKS);
    s->precond = settings->preconditioner ? 1 : 0;
    const long x = chunk->x, y = chunk->y, n = x * y;
    const long mi = settings->max_iters > 0 ? settings->max_iters : 1;

    struct Req { double** dst; long count; };
    Req reqs[] = {
        {&chunk->density0, n}, {&chunk->density, n}, {&chunk->energy0, n}, {&chunk->energy, n},
        {&chunk->u, n}, {&chunk->u0, n}, {&chunk->p, n}, {&chunk->r, n}, {&chunk->mi, n},
        {&chunk->w, n}, {&chunk->kx, n}, {&chunk->ky, n}, {&chunk->sd, n}, {&chunk->volume, n},
        {&chunk->x_area, (x + 1) * y}, {&chunk->y_area, x * (y + 1)},
        {&chunk->cell_x, x}, {&chunk->cell_y, y}, {&chunk->cell_dx, x}, {&chunk->cell_dy, y},
        {&chunk->vertex_dx, x + 1}, {&chunk->vertex_dy, y + 1},
        {&chunk->vertex_x, x + 1}, {&chunk->vertex_y, y + 1},
        {&s->alt[ALT_P], n}, {&s->alt[ALT_U], n}, {&s->alt[ALT_R], n}, {&s->alt[ALT_SD], n},
        {&s->d_cg_alphas, mi}, {&s->d_cg_betas, mi}, {&s->d_cheby_alphas, mi}, {&s->d_cheby_betas, mi},
    };
    s->table_len = (int)mi;
    // Reduction partials: one slot set per block of the largest reduction launch.
    const dim3 gh = fused_grid(s->g), gi = interior_grid(s->g), gf = full_grid(s->g);
    const long blocks = std::max<long>({(long)gh.x * gh.y, (long)gi.x * gi.y, (long)gf.x * gf.y});
    s->partial_capacity = blocks * tl::kMaxSums;

    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t bytes = 0;
    for (const Req& r : reqs) bytes += align((size_t)r.count * sizeof(double));
    bytes += align((size_t)s->partial_capacity * sizeof(double)) + align(tl::kMaxSums * sizeof(double)) + 256;
    bytes += align(sizeof(DevState));
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
    cur += 256;
    s->d_state = (DevState*)cur;
    if (!TL_CUDA(cudaHostAlloc((void**)&s->h_out, tl::kMaxSums * sizeof(double) + 64, cudaHostAllocMapped))) return;
    double* dev_view = nullptr;
    if (!TL_CUDA(cudaHostGetDevicePointer((void**)&dev_view, s->h_out, 0))) return;
    s->rs.out_host = dev_view;
    s->h_mirror = (int*)(s->h_out + tl::kMaxSums);
    memset(s->h_mirror, 0, 64);
    s->d_mirror = (int*)(dev_view + tl::kMaxSums);

    chunk->cg_alphas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cg_betas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cheby_alphas = (double*)calloc((size_t)mi, sizeof(double));
    chunk->cheby_betas = (double*)calloc((size_t)mi, sizeof(double));
    TL_CUDA(cudaStreamSynchronize(s->stream));
    tl_noalloc_prepare();
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
    if (s->mx_slab) cudaFree(s->mx_slab);
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
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    const double x_min = settings->grid_x_min + settings->dx * (double)chunk->left;
    const double y_min = settings->grid_y_min + settings->dy * (double)chunk->bottom;
    const int m = std::max(chunk->x, chunk->y) + 1;
    TL_LAUNCH(s, "k_set_chunk_data_axes",
              k_set_chunk_data_axes<<<tl::ceil_div(m, 256), 256, 0, s->stream>>>(
                  chunk->x, chunk->y, settings->halo_depth, x_min, y_min, settings->dx, settings->dy,
                  chunk->vertex_x, chunk->vertex_y, chunk->cell_x, chunk->cell_y));
    const long n = (long)chunk->x * chunk->y;
    TL_LAUNCH(s, "k_set_chunk_data_cells",
              k_set_chunk_data_cells<<<s->sm_count * 8, 256, 0, s->stream>>>(n, settings->dx, settings->dy,
                                                                           chunk->volume, chunk->x_area,
                                                                           chunk->y_area));
}

// 2d/kernel_interface.h:15 (set_chunk_state.c:9-84); states is a host array.
void run_set_chunk_state(Chunk* chunk, Settings* settings, State* states)
{
    TlSuite2D* s = ready(chunk);
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
    TL_LAUNCH(s, "k_set_chunk_state",
              k_set_chunk_state<<<full_grid(s->g), FB, 0, s->stream>>>(
                  s->g, chunk->vertex_x, chunk->vertex_y, chunk->cell_x, chunk->cell_y, chunk->density,
                  chunk->energy0, chunk->u, ns, s->d_states));
    TL_CUDA(cudaStreamSynchronize(s->stream));  // the host may free `states` on return
}

// ------------------------------------------------------ solver-wide kernels --
// 2d/kernel_interface.h:23 (local_halos.c:21-64): recorded, run by the next
// sweep that can fuse it or by the next flush.
void run_local_halos(Chunk* chunk, Settings* settings, int depth)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    if (depth < 1 || depth > settings->halo_depth) {
        tl::fail(5, "halo depth %d outside [1, %d]", depth, settings->halo_depth);
        return;
    }
    for (int f = 0; f < TL_NUM_FIELDS; ++f)
        if (settings->fields_to_exchange[f]) s->pend.halo[f] = std::max(s->pend.halo[f], depth);
}

// 2d/kernel_interface.h:25 (pack_halos.c:179-207). `buffer` may be host or
// device memory (the reference host passes its malloc'd MPI buffers).
void run_pack_or_unpack(Chunk* chunk, Settings* settings, int depth, int face, bool pack, FieldBufferType field,
                        double* buffer)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
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
    if (!pack)
        TL_CUDA(cudaMemcpyAsync(s->d_comm, buffer, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL_LAUNCH(s, "k_pack",
              k_pack<<<tl::ceil_div(len, 256), 256, 0, s->stream>>>(s->g, depth, face, pack ? 1 : 0, field, s->d_comm));
    if (pack)
        TL_CUDA(cudaMemcpyAsync(buffer, s->d_comm, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// 2d/kernel_interface.h:28 (store_energy.c:4-15): energy = energy0, full array.
void run_store_energy(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->energy, chunk->energy0, sizeof(double) * (size_t)chunk->x * chunk->y,
                            cudaMemcpyDeviceToDevice, s->stream));
}

// 2d/kernel_interface.h:30 (field_summary.c:8-45): the reference's serial
// summation order, so the totals match its rounding.
void run_field_summary(Chunk* chunk, Settings* settings, double* vol, double* mass, double* ie, double* temp)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_field_summary_ordered",
              tl::launch_field_summary_ordered(s->stream, s->g.x, s->g.y, 1, s->g.hd, 0, chunk->volume,
                                               chunk->density, chunk->energy0, chunk->u, s->rs.out_dev,
                                               s->rs.out_host));
    double o[4];
    if (!fetch(s, 4, o)) return;
    *vol += o[0];
    *mass += o[1];
    *ie += o[2];
    *temp += o[3];
}

// New: the same four totals from a parallel tree reduction (one sweep at
// full bandwidth; differs from the reference's serial order by rounding).
void tl2d_field_summary_fast(Chunk* chunk, Settings* settings, double* vol, double* mass, double* ie, double* temp)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_field_summary",
              k_field_summary<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->volume, chunk->density,
                                                                        chunk->energy0, chunk->u, s->rs));
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
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    if (settings->coefficient != TL_CONDUCTIVITY && settings->coefficient != TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL_LAUNCH(s, "k_cg_init",
              k_cg_init<<<full_grid(s->g), FB, 0, s->stream>>>(
                  s->g, settings->coefficient, rx, ry, chunk->density, chunk->energy, chunk->u, chunk->p,
                  s->alt[ALT_P], chunk->r, chunk->w, chunk->kx, chunk->ky, s->rs, tl::NoFinish()));
    double o;
    if (fetch(s, 1, &o)) *rro += o;
}

// 2d/kernel_interface.h:38 (cg.c:88-113). Absorbs a pending p update, a
// pending depth-1 halo of p and a pending halo of u: one sweep reads old p
// and r, writes the new p (to the second p buffer) with its reflected halo,
// w = A p and p.w; the halo-duty block row writes the halos (u is read-only here).
void run_cg_calc_w(Chunk* chunk, Settings* settings, double* pw)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);   // deferred steps precede everything recorded after them
    if (s->pend.halo[TL_FIELD_P] > 1) flush(s, chunk);
    const bool fuse = s->pend.calc_p;
    const bool refl = s->pend.halo[TL_FIELD_P] == 1;
    const int ud = s->pend.halo[TL_FIELD_U];
    double* u_halo = ud > 0 ? chunk->u : nullptr;
    const Faces fc = faces_of(chunk);
    const Scalar beta{s->pend.beta, nullptr};
    const dim3 gr = fused_grid(s->g);
    double* p_out = fuse ? s->alt[ALT_P] : chunk->p;
#define W2(F, R)                                                                                                    \
    launch_cg_w2<F, R>(s, chunk, gr, fc, beta, chunk->p, p_out, chunk->r, chunk->w, u_halo, ud, nullptr,            \
                       tl::NoFinish())
    if (fuse && refl) W2(true, true);
    else if (fuse) W2(true, false);
    else if (refl) W2(false, true);
    else W2(false, false);
#undef W2
    if (fuse) swap_alt(s, chunk, ALT_P);
    s->pend.calc_p = false;
    s->pend.halo[TL_FIELD_P] = 0;
    s->pend.halo[TL_FIELD_U] = 0;
    double o;
    if (fetch(s, 1, &o)) *pw += o;
}

// 2d/kernel_interface.h:40 (cg.c:116-143). A halo of u still pending here
// (a host that did not call calc_w first) is run before u changes.
void run_cg_calc_ur(Chunk* chunk, Settings* settings, double alpha, double* rrn)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);
    if (s->pend.calc_p || s->pend.halo[TL_FIELD_U]) flush(s, chunk);
    launch_cg_ur2(s, interior_grid(s->g), Scalar{alpha, nullptr}, chunk->u, chunk->p, chunk->r, chunk->w, nullptr,
                  tl::NoFinish());
    double o;
    if (fetch(s, 1, &o)) *rrn += o;
}

// 2d/kernel_interface.h:42 (cg.c:146-164): recorded; run by the next calc_w
// (fused) or the next flush.
void run_cg_calc_p(Chunk* chunk, Settings* settings, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);
    if (s->pend.calc_p || s->pend.halo[TL_FIELD_P]) flush(s, chunk);
    s->pend.calc_p = true;
    s->pend.beta = beta;
}

// ------------------------------------------------------- Chebyshev kernels --
// 2d/kernel_interface.h:46 (cheby.c:26-54)
void run_cheby_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cheby_sweep<init>",
              k_cheby_sweep<true><<<interior_grid(s->g), BX, 0, s->stream>>>(
                  s->g, 0.0, 0.0, chunk->theta, chunk->u, chunk->u0, chunk->p, chunk->r, chunk->w, chunk->kx,
                  chunk->ky));
    TL_LAUNCH(s, "k_add_p", k_add_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->p));
}

// 2d/kernel_interface.h:48 (cheby.c:57-85). With temporal blocking on and
// four external faces, a call preceded by nothing but the depth-1 halo update
// of u is queued (run_cheby_queue); otherwise it runs at once.
void run_cheby_iterate(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    const Faces fc = faces_of(chunk);
    if (s->temporal_blocking && fc.l && fc.r && fc.b && fc.t && !s->pq.active && !s->pend.calc_p &&
        s->pend.halo[TL_FIELD_U] <= 1 && (long)s->cq.a.size() < s->table_len) {
        bool other = false;
        for (int f = 0; f < TL_NUM_FIELDS; ++f) other |= f != TL_FIELD_U && s->pend.halo[f] != 0;
        if (!other) {
            s->pend.halo[TL_FIELD_U] = 0;   // the blocked trips reflect u on the fly and write its halo
            s->cq.active = true;
            s->cq.a.push_back(alpha);
            s->cq.b.push_back(beta);
            return;
        }
    }
    s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_cheby_sweep",
              k_cheby_sweep<false><<<interior_grid(s->g), BX, 0, s->stream>>>(
                  s->g, alpha, beta, 0.0, chunk->u, chunk->u0, chunk->p, chunk->r, chunk->w, chunk->kx,
                  chunk->ky));
    TL_LAUNCH(s, "k_add_p", k_add_p<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->p));
}

// ---------------------------------------------------------- Jacobi kernels --
// 2d/kernel_interface.h:52 (jacobi.c:10-57)
void run_jacobi_init(Chunk* chunk, Settings* settings, double rx, double ry)
{
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    if (settings->coefficient < TL_CONDUCTIVITY && settings->coefficient < TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL_LAUNCH(s, "k_jacobi_init",
              k_jacobi_init<<<full_grid(s->g), FB, 0, s->stream>>>(s->g, settings->coefficient, rx, ry,
                                                                  chunk->density, chunk->energy, chunk->u0,
                                                                  chunk->u, chunk->kx, chunk->ky));
}

// 2d/kernel_interface.h:54 (jacobi.c:60-101). The L1 change is ASSIGNED to
// *error, as the reference kernel does (jacobi.c:100).
void run_jacobi_iterate(Chunk* chunk, Settings* settings, double* error)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->r, chunk->u, sizeof(double) * (size_t)chunk->x * chunk->y,
                            cudaMemcpyDeviceToDevice, s->stream));
    TL_LAUNCH(s, "k_jacobi_iterate",
              k_jacobi_iterate<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->kx, chunk->ky, chunk->u0,
                                                                         chunk->u, chunk->r, s->rs));
    double o;
    if (fetch(s, 1, &o)) *error = o;
}

// ------------------------------------------------------------ PPCG kernels --
// 2d/kernel_interface.h:58 (ppcg.c:9-26)
void run_ppcg_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    const Faces fc = faces_of(chunk);
    if (s->temporal_blocking && fc.l && fc.r && fc.b && fc.t) {
        s->pq.active = true;   // sd = r / theta runs with the first queued step
        s->pq.a.clear();
        s->pq.b.clear();
        return;
    }
    TL_LAUNCH(s, "k_ppcg_init",
              k_ppcg_init<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->theta, chunk->r, chunk->sd));
}

// 2d/kernel_interface.h:60 (ppcg.c:29-61)
void run_ppcg_inner_iteration(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
    if (!s) return;
    // queued only in the reference drivers' pattern: a depth-1 halo update of
    // sd (and nothing else) requested right before the step
    if (s->pq.active && !s->pend.calc_p && s->pend.halo[TL_FIELD_SD] == 1 && (long)s->pq.a.size() < s->table_len) {
        bool other = false;
        for (int f = 0; f < TL_NUM_FIELDS; ++f) other |= f != TL_FIELD_SD && s->pend.halo[f] != 0;
        if (!other) {
            s->pend.halo[TL_FIELD_SD] = 0;   // the blocked steps reflect sd on the fly and write its halo
            s->pq.a.push_back(alpha);
            s->pq.b.push_back(beta);
            return;
        }
    }
    s = ready(chunk);   // runs the queue, if any, and the pending operations
    if (!s) return;
    TL_LAUNCH(s, "k_ppcg_inner_a",
              k_ppcg_inner_a<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->r, chunk->kx,
                                                                       chunk->ky, chunk->sd));
    TL_LAUNCH(s, "k_ppcg_inner_b",
              k_ppcg_inner_b<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, alpha, beta, chunk->sd, chunk->r));
}

// ---------------------------------------------------------- shared kernels --
// 2d/kernel_interface.h:64 (solver_methods.c:9-25)
void run_copy_u(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_copy_u", k_copy_u<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u0, chunk->u));
}

// 2d/kernel_interface.h:66 (solver_methods.c:28-48)
void run_calculate_residual(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_residual",
              k_residual<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->u, chunk->u0, chunk->r, chunk->kx,
                                                                   chunk->ky));
}

// 2d/kernel_interface.h:68 (solver_methods.c:51-71)
void run_calculate_2norm(Chunk* chunk, Settings* settings, FieldBufferType buffer, double* norm)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    TL_LAUNCH(s, "k_norm2", k_norm2<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, buffer, s->rs));
    double o;
    if (fetch(s, 1, &o)) *norm += o;
}

// 2d/kernel_interface.h:70 (solver_methods.c:74-90)
void run_finalise(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite2D* s = ready(chunk);
    if (!s) return;
    if (tma_failed(s)) {
        tl::fail(35, "a TMA row load of the w sweep did not complete (bounded barrier wait gave up)");
        return;
    }
    TL_LAUNCH(s, "k_finalise",
              k_finalise<<<interior_grid(s->g), BX, 0, s->stream>>>(s->g, chunk->energy, chunk->density, chunk->u));
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
    TlSuite2D* s = ready(chunk);
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
    TlSuite2D* s = ready(chunk);
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
