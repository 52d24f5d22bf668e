// suite3d.cu -- B200 (sm_100a) TeaLeaf 3D kernel suite behind the reference
// 3D kernel interface (3d/kernel_interface.h:9-65).
//
// Same structure as the 2D suite: fields are slices of one device slab
// (x*y*z FP64 values each, index k + j*x + i*x*y, 256-byte aligned slices);
// reductions finish in one last-block pass into mapped pinned memory;
// run_cg_solver_calc_p and run_local_halos are deferred and absorbed by the
// next sweep that can fuse them (calc_w takes the p update and the halo of p,
// calc_ur the halo of u), so a CG iteration of the reference 3D drivers costs
// two sweeps and 104 bytes per cell. p alternates between two buffers;
// chunk->vec_p always points at the current one.
#include "suite3d_impl.hpp"

#include <algorithm>
#include <vector>
#include <cstring>

using namespace tl3d;
using tl::ReduceSlots;

namespace tl3d {

TlSuite3D* suite_of(Chunk* chunk)
{
    if (!chunk || !chunk->ext || !chunk->ext->suite) {
        tl::fail(1, "chunk has no B200 suite state (run_kernel_initialise not called)");
        return nullptr;
    }
    return chunk->ext->suite;
}

bool fetch(TlSuite3D* s, int n, double* out)
{
    if (!TL_CUDA(cudaStreamSynchronize(s->stream))) return false;
    if (s->prof.on) s->prof.resolve();
    for (int i = 0; i < n; ++i) out[i] = s->h_out[i];
    return true;
}

Faces faces_of(const Chunk* chunk)
{
    const int* nb = chunk->neighbours;
    return Faces{nb[TL3_CHUNK_LEFT] == TL3_EXTERNAL_FACE,  nb[TL3_CHUNK_RIGHT] == TL3_EXTERNAL_FACE,
                 nb[TL3_CHUNK_BOTTOM] == TL3_EXTERNAL_FACE, nb[TL3_CHUNK_TOP] == TL3_EXTERNAL_FACE,
                 nb[TL3_CHUNK_BACK] == TL3_EXTERNAL_FACE,   nb[TL3_CHUNK_FRONT] == TL3_EXTERNAL_FACE};
}

double** field_slot(Chunk* chunk, AltField3 f)
{
    switch (f) {
        case ALT3_P: return &chunk->vec_p;
        case ALT3_U: return &chunk->vec_u;
        case ALT3_R: return &chunk->vec_r;
        default: return &chunk->vec_sd;
    }
}

void swap_alt(TlSuite3D* s, Chunk* chunk, AltField3 f)
{
    double** slot = field_slot(chunk, f);
    double* cur = *slot;
    *slot = s->alt[f];
    s->alt[f] = cur;
}

static void launch_halos(TlSuite3D* s, Chunk* chunk, int depth, const int* which)
{
    const int order[TL3_NUM_FIELDS] = {TL3_FIELD_DENSITY, TL3_FIELD_P, TL3_FIELD_ENERGY0,
                                       TL3_FIELD_ENERGY1, TL3_FIELD_U, TL3_FIELD_SD};
    double* fields[TL3_NUM_FIELDS] = {chunk->density, chunk->energy0, chunk->energy,
                                      chunk->vec_u, chunk->vec_p, chunk->vec_sd};
    HaloArgs3 a{};
    for (int o = 0; o < TL3_NUM_FIELDS; ++o)
        if (which[order[o]] == depth) a.f[a.nf++] = fields[order[o]];
    if (a.nf == 0) return;
    for (int f = 0; f < 6; ++f) a.ext[f] = chunk->neighbours[f] == TL3_EXTERNAL_FACE;
    const Geo& g = s->g;
    const long nx = g.x - 2 * g.hd, ny = g.y - 2 * g.hd, nz = g.z - 2 * g.hd;
    const long per = 2L * depth * (nz * ny + nz * nx + ny * nx);
    TL3_LAUNCH(s, "k3_local_halos",
               k3_local_halos<<<dim3(tl::ceil_div(per, 256), a.nf), 256, 0, s->stream>>>(g, depth, a));
}

// Launch sizes of up to kTB3 steps for n queued steps, made an even count
// (the launches alternate buffers while the host holds the chunk's
// pointers): a two-step launch is split when the count is odd. n >= 2.
static std::vector<int> even_blocks(int n)
{
    std::vector<int> sizes;
    for (int left = n; left > 0; left -= kTB3) sizes.push_back(std::min(kTB3, left));
    if (sizes.size() % 2 == 1) {
        for (int q = (int)sizes.size() - 1; q >= 0; --q) {
            if (sizes[q] >= 2) {
                sizes[q] -= 1;
                sizes.insert(sizes.begin() + q + 1, 1);
                break;
            }
        }
    }
    return sizes;
}

static void upload_queue(TlSuite3D* s, const TlSuite3D::Queue& q)
{
    const size_t n = q.a.size();
    TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, q.a.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
    TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, q.b.data(), sizeof(double) * n, cudaMemcpyHostToDevice, s->stream));
}

// Runs the deferred PPCG inner steps (ppcg_solver.c:8-73 as the reference
// drivers call them: sd = r / theta, then per step a depth-1 halo of sd and
// r -= A sd, u += sd, sd = a sd + b r): temporally blocked launches (the fold
// of each step at its start, sd reflected on the fly and its halo written)
// and the last step's sd update, with the same results as one launch per
// call; an even number of launches (the sd and r buffers alternate). One
// step runs as the one-step kernels, and with none queued sd = r / theta
// alone.
static void run_ppcg_queue(TlSuite3D* s, Chunk* chunk)
{
    s->pq.active = false;
    const int n = (int)s->pq.a.size();
    const dim3 gr = interior_grid(s->g), bl = interior_block();
    if (n <= 1) {
        TL3_LAUNCH(s, "k3_ppcg_init", k3_ppcg_init<<<gr, bl, 0, s->stream>>>(s->g, chunk->theta, chunk->vec_r,
                                                                              chunk->vec_sd));
        if (n == 1) {   // the absorbed halo update, then the step
            int which[TL3_NUM_FIELDS] = {0};
            which[TL3_FIELD_SD] = 1;
            launch_halos(s, chunk, 1, which);
            TL3_LAUNCH(s, "k3_ppcg_inner_a", k3_ppcg_inner_a<<<gr, bl, 0, s->stream>>>(
                                                 s->g, chunk->vec_u, chunk->vec_r, chunk->vec_kx, chunk->vec_ky,
                                                 chunk->vec_kz, chunk->vec_sd));
            TL3_LAUNCH(s, "k3_ppcg_sd", k3_ppcg_sd<<<gr, bl, 0, s->stream>>>(s->g, s->pq.a[0], s->pq.b[0],
                                                                              chunk->vec_sd, chunk->vec_r));
        }
    } else {
        upload_queue(s, s->pq);
        int pp0 = 0;
        for (int steps : even_blocks(n)) {
            const Blocked3Args a{steps, pp0, 0, chunk->theta, s->d_cheby_alphas, s->d_cheby_betas};
            launch_blocked3<1>(s, chunk, a, chunk->vec_sd, chunk->vec_r, s->alt[ALT3_SD], s->alt[ALT3_R], nullptr,
                               chunk->vec_u, nullptr, nullptr, nullptr);
            swap_alt(s, chunk, ALT3_SD);
            swap_alt(s, chunk, ALT3_R);
            pp0 += steps;
        }
        TL3_LAUNCH(s, "k3_ppcg_sd", k3_ppcg_sd<<<gr, bl, 0, s->stream>>>(s->g, s->pq.a[n - 1], s->pq.b[n - 1],
                                                                          chunk->vec_sd, chunk->vec_r));
    }
    s->pq.a.clear();
    s->pq.b.clear();
}

// The one-step Chebyshev trip of the run_* path (cheby_solver.c:62-99: w = A u,
// r = u0 - w, p = alpha p + beta r, then u += p).
static void cheby_trip_one_step(TlSuite3D* s, Chunk* chunk, double alpha, double beta)
{
    const dim3 gf = fused_grid(s->g), gr = interior_grid(s->g), bl = interior_block();
    const Faces none{0, 0, 0, 0, 0, 0};
    const tl::ChebyCoef coef{alpha, beta, nullptr, nullptr, nullptr};
    tl::DevParams prm{};
    TL3_LAUNCH(s, "k3_cheby_trip",
               (k3_cheby_trip<false, false, false><<<gf, bl, 0, s->stream>>>(
                   s->g, none, coef, 0.0, 1, chunk->vec_u, chunk->vec_p, chunk->vec_u, chunk->vec_p, chunk->vec_u0,
                   chunk->vec_w, chunk->vec_r, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs, nullptr,
                   tl::NoFinish(), prm, Tma3Maps{}, nullptr)));
    TL3_LAUNCH(s, "k3_add_p", k3_add_p<false><<<gr, bl, 0, s->stream>>>(s->g, none, chunk->vec_u, chunk->vec_p));
}

// Runs the deferred Chebyshev trips (cheby_solver.c:62-99 as the reference
// drivers call them: per trip a depth-1 halo of u, then the trip ending with
// its u += p): temporally blocked launches, each trip's add at its end and u
// reflected on the fly; the last launch also writes w and r and leaves u's
// halo as the call-by-call sequence does (mirroring u before the last add).
// An even number of launches (the u and p buffers alternate); a single trip
// runs as the one-step kernels. The same results as one launch per call.
static void run_cheby_queue(TlSuite3D* s, Chunk* chunk)
{
    s->cq.active = false;
    const int n = (int)s->cq.a.size();
    if (n == 1) {   // the absorbed halo update, then the one-step kernels
        int which[TL3_NUM_FIELDS] = {0};
        which[TL3_FIELD_U] = 1;
        launch_halos(s, chunk, 1, which);
        cheby_trip_one_step(s, chunk, s->cq.a[0], s->cq.b[0]);
    } else if (n > 1) {
        upload_queue(s, s->cq);
        int first = 0;
        for (int steps : even_blocks(n)) {
            const Blocked3Args a{steps, first, first + steps == n ? 1 : 0, 0.0, s->d_cheby_alphas,
                                 s->d_cheby_betas, 1};
            launch_blocked3<0>(s, chunk, a, chunk->vec_u, chunk->vec_p, s->alt[ALT3_U], s->alt[ALT3_P],
                               chunk->vec_u0, nullptr, chunk->vec_w, chunk->vec_r, nullptr);
            swap_alt(s, chunk, ALT3_U);
            swap_alt(s, chunk, ALT3_P);
            first += steps;
        }
    }
    s->cq.a.clear();
    s->cq.b.clear();
}

// Runs whichever deferred queue is open.
static void run_queues(TlSuite3D* s, Chunk* chunk)
{
    if (s->pq.active) run_ppcg_queue(s, chunk);
    if (s->cq.active) run_cheby_queue(s, chunk);
}

void flush(TlSuite3D* s, Chunk* chunk)
{
    run_queues(s, chunk);
    if (s->pend.calc_p) {
        TL3_LAUNCH(s, "k3_cg_close",
                   k3_cg_close<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                       s->g, Faces{0, 0, 0, 0, 0, 0}, Scalar{s->pend.beta, nullptr}, 1, chunk->vec_p, chunk->vec_r,
                       nullptr));
        s->pend.calc_p = false;
    }
    for (int d = 1; d <= s->g.hd; ++d) launch_halos(s, chunk, d, s->pend.halo);
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
}

}  // namespace tl3d

namespace {

TlSuite3D* ready(Chunk* chunk)
{
    if (tl::failed()) return nullptr;
    TlSuite3D* s = suite_of(chunk);
    if (s) flush(s, chunk);
    return s;
}

double* field_by_id(Chunk* c, int id)
{
    switch (id) {
        case TL3D_DENSITY0: return c->density0;
        case TL3D_DENSITY: return c->density;
        case TL3D_ENERGY0: return c->energy0;
        case TL3D_ENERGY: return c->energy;
        case TL3D_U: return c->vec_u;
        case TL3D_U0: return c->vec_u0;
        case TL3D_P: return c->vec_p;
        case TL3D_R: return c->vec_r;
        case TL3D_MI: return c->vec_mi;
        case TL3D_W: return c->vec_w;
        case TL3D_KX: return c->vec_kx;
        case TL3D_KY: return c->vec_ky;
        case TL3D_SD: return c->vec_sd;
        case TL3D_VOLUME: return c->volume;
        case TL3D_KZ: return c->vec_kz;
        default: return nullptr;
    }
}

}  // namespace

extern "C" {

void tl3d_set_error_mode(int mode) { tl::error_state().mode = mode; }
void tl3d_set_device(int device) { TL_CUDA(cudaSetDevice(device)); }
int tl3d_get_error(char* msg, int msg_len) { return tl::take_error(msg, msg_len); }
void* tl3d_stream(Chunk* chunk)
{
    TlSuite3D* s = suite_of(chunk);
    return s ? (void*)s->stream : nullptr;
}
void tl3d_profile_enable(Chunk* chunk, int on)
{
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    s->prof.resolve();
    s->prof.on = on != 0;
}
void tl3d_profile_reset(Chunk* chunk)
{
    TlSuite3D* s = suite_of(chunk);
    if (s) s->prof.reset();
}
void tl3d_set_tma(Chunk* chunk, int on)
{
    TlSuite3D* s = suite_of(chunk);
    if (s) s->tma = on != 0;
}
void tl3d_set_temporal_blocking(Chunk* chunk, int on)
{
    TlSuite3D* s = suite_of(chunk);
    if (s) s->temporal_blocking = on != 0;
}
void tl3d_flush(Chunk* chunk) { ready(chunk); }
long long tl3d_launch_count(Chunk* chunk)
{
    TlSuite3D* s = suite_of(chunk);
    return s ? s->prof.launches : -1;
}

int tl3d_profile_read(Chunk* chunk, int index, char* name, int name_len, long long* calls, double* ms)
{
    TlSuite3D* s = suite_of(chunk);
    if (!s || index < 0 || index >= tl::Profiler::kMaxKernels || !s->prof.names[index]) return 0;
    s->prof.resolve();
    if (name && name_len > 0) snprintf(name, (size_t)name_len, "%s", s->prof.names[index]);
    if (calls) *calls = s->prof.calls[index];
    if (ms) *ms = s->prof.ms[index];
    return 1;
}

// 3d/kernel_interface.h:13 (3d/c_kernels/omp3/kernel_init_chunk.c:28-108)
void run_kernel_initialise(Chunk* chunk, Settings* settings)
{
    if (tl::failed()) return;
    const int hd = settings->halo_depth;
    if (hd < 1 || chunk->x < 2 * hd + 1 || chunk->y < 2 * hd + 1 || chunk->z < 2 * hd + 1) {
        tl::fail(2, "invalid chunk extents x=%d y=%d z=%d halo_depth=%d", chunk->x, chunk->y, chunk->z, hd);
        return;
    }
    if (!chunk->ext) {
        tl::fail(3, "chunk->ext is NULL (the host allocates chunk_extension_t, 3d/chunk.c:37)");
        return;
    }
    TlSuite3D* s = new TlSuite3D();
    chunk->ext->suite = s;
    TL_CUDA(cudaGetDevice(&s->device));
    TL_CUDA(cudaDeviceGetAttribute(&s->sm_count, cudaDevAttrMultiProcessorCount, s->device));
    if (!TL_CUDA(cudaStreamCreateWithFlags(&s->stream, cudaStreamNonBlocking))) return;
    s->g = Geo{chunk->x, chunk->y, chunk->z, hd};
    s->g.zr = choose_zr(chunk->x - 2 * hd, chunk->y - 2 * hd, chunk->z - 2 * hd, s->sm_count);
    const long x = chunk->x, y = chunk->y, z = chunk->z, n = x * y * z;
    const long mi = settings->max_iters > 0 ? settings->max_iters : 1;
    struct Req { double** dst; long count; };
    Req reqs[] = {
        {&chunk->density0, n}, {&chunk->density, n}, {&chunk->energy0, n}, {&chunk->energy, n},
        {&chunk->vec_u, n}, {&chunk->vec_u0, n}, {&chunk->vec_p, n}, {&chunk->vec_r, n}, {&chunk->vec_mi, n},
        {&chunk->vec_w, n}, {&chunk->vec_kx, n}, {&chunk->vec_ky, n}, {&chunk->vec_kz, n}, {&chunk->vec_sd, n},
        {&chunk->vec_z, n}, {&chunk->volume, n},
        {&chunk->x_area, (x + 1) * y * z}, {&chunk->y_area, x * (y + 1) * z}, {&chunk->z_area, x * y * (z + 1)},
        {&chunk->cell_x, x}, {&chunk->cell_y, y}, {&chunk->cell_z, z},
        {&chunk->cell_dx, x}, {&chunk->cell_dy, y}, {&chunk->cell_dz, z},
        {&chunk->vertex_dx, x + 1}, {&chunk->vertex_dy, y + 1}, {&chunk->vertex_dz, z + 1},
        {&chunk->vertex_x, x + 1}, {&chunk->vertex_y, y + 1}, {&chunk->vertex_z, z + 1},
        {&s->alt[ALT3_P], n}, {&s->alt[ALT3_U], n}, {&s->alt[ALT3_R], n}, {&s->alt[ALT3_SD], n},
        {&s->d_cg_alphas, mi}, {&s->d_cg_betas, mi}, {&s->d_cheby_alphas, mi}, {&s->d_cheby_betas, mi},
    };
    s->table_len = (int)mi;
    const dim3 gi = fused_grid(s->g), gf = full_grid(s->g);
    const long blocks = std::max<long>((long)gi.x * gi.y * gi.z, (long)gf.x * gf.y * gf.z);
    s->partial_capacity = blocks * tl::kMaxSums;
    auto align = [](size_t b) { return (b + 255) & ~(size_t)255; };
    size_t bytes = 0;
    for (const Req& r : reqs) bytes += align((size_t)r.count * sizeof(double));
    bytes += align((size_t)s->partial_capacity * sizeof(double)) + align(tl::kMaxSums * sizeof(double)) + 256;
    bytes += align(sizeof(tl::DevState));
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
    s->d_state = (tl::DevState*)cur;
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
}

void run_kernel_finalise(Chunk* chunk, Settings* settings)
{
    (void)settings;
    if (!chunk || !chunk->ext || !chunk->ext->suite) return;
    TlSuite3D* s = chunk->ext->suite;
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

// 3d/kernel_interface.h:9 (3d/c_kernels/omp3/set_chunk_data.c:8-74)
void run_set_chunk_data(Chunk* chunk, Settings* settings)
{
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    const double x_min = settings->grid_x_min + settings->dx * (double)chunk->left;
    const double y_min = settings->grid_y_min + settings->dy * (double)chunk->bottom;
    const double z_min = settings->grid_z_min + settings->dz * (double)chunk->back;
    const int m = std::max(chunk->x, std::max(chunk->y, chunk->z)) + 1;
    TL3_LAUNCH(s, "k3_set_chunk_data_axes",
               k3_set_chunk_data_axes<<<tl::ceil_div(m, 256), 256, 0, s->stream>>>(
                   s->g, x_min, y_min, z_min, settings->dx, settings->dy, settings->dz, chunk->vertex_x,
                   chunk->vertex_y, chunk->vertex_z, chunk->cell_x, chunk->cell_y, chunk->cell_z));
    TL3_LAUNCH(s, "k3_set_chunk_data_cells",
               k3_set_chunk_data_cells<<<s->sm_count * 8, 256, 0, s->stream>>>(
                   s->g.xy() * s->g.z, settings->dx, settings->dy, settings->dz, chunk->volume, chunk->x_area,
                   chunk->y_area, chunk->z_area));
}

// 3d/kernel_interface.h:11 (3d/c_kernels/omp3/set_chunk_state.c:9-98)
void run_set_chunk_state(Chunk* chunk, Settings* settings, State* states)
{
    TlSuite3D* s = ready(chunk);
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
    TL3_LAUNCH(s, "k3_set_chunk_state",
               k3_set_chunk_state<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                   s->g, chunk->vertex_x, chunk->vertex_y, chunk->vertex_z, chunk->cell_x, chunk->cell_y,
                   chunk->cell_z, chunk->density, chunk->energy0, chunk->vec_u, ns, s->d_states));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// 3d/kernel_interface.h:17: recorded, run by the next fusing sweep or flush.
void run_local_halos(Chunk* chunk, Settings* settings, int depth)
{
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    if (depth < 1 || depth > settings->halo_depth) {
        tl::fail(5, "halo depth %d outside [1, %d]", depth, settings->halo_depth);
        return;
    }
    for (int f = 0; f < TL3_NUM_FIELDS; ++f)
        if (settings->fields_to_exchange[f]) s->pend.halo[f] = std::max(s->pend.halo[f], depth);
}

// 3d/kernel_interface.h:19 (3d/c_kernels/omp3/pack_halos.c)
void run_pack_or_unpack(Chunk* chunk, Settings* settings, int depth, int face, bool pack, double* field,
                        double* buffer)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    if (face < 0 || face > 5) {
        tl::fail(6, "Incorrect face provided: %d.", face);
        return;
    }
    const Geo& g = s->g;
    const long nx = g.x - 2 * g.hd, ny = g.y - 2 * g.hd, nz = g.z - 2 * g.hd;
    const long len = (long)depth * (face < 2 ? nz * ny : face < 4 ? nz * nx : ny * nx);
    if (len > s->d_comm_cap) {
        if (s->d_comm) cudaFree(s->d_comm);
        if (!TL_CUDA(cudaMalloc(&s->d_comm, sizeof(double) * len))) return;
        s->d_comm_cap = len;
    }
    if (!pack)
        TL_CUDA(cudaMemcpyAsync(s->d_comm, buffer, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL3_LAUNCH(s, "k3_pack", k3_pack<<<tl::ceil_div(len, 256), 256, 0, s->stream>>>(g, depth, face, pack ? 1 : 0,
                                                                                     field, s->d_comm));
    if (pack)
        TL_CUDA(cudaMemcpyAsync(buffer, s->d_comm, sizeof(double) * len, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// 3d/kernel_interface.h:22 (3d/c_kernels/omp3/store_energy.c)
void run_store_energy(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->energy, chunk->energy0, sizeof(double) * (size_t)(s->g.xy() * s->g.z),
                            cudaMemcpyDeviceToDevice, s->stream));
}

// 3d/kernel_interface.h:24 (3d/c_kernels/omp3/field_summary.c:8-49): the
// reference's serial summation order.
void run_field_summary(Chunk* chunk, Settings* settings, double* vol, double* mass, double* ie, double* temp)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL3_LAUNCH(s, "k_field_summary_ordered",
               tl::launch_field_summary_ordered(s->stream, s->g.x, s->g.y, s->g.z, s->g.hd, s->g.hd, chunk->volume,
                                                chunk->density, chunk->energy0, chunk->vec_u, s->rs.out_dev,
                                                s->rs.out_host));
    double o[4];
    if (!fetch(s, 4, o)) return;
    *vol += o[0];
    *mass += o[1];
    *ie += o[2];
    *temp += o[3];
}

// New: tree-reduced field summary (full bandwidth, different rounding).
void tl3d_field_summary_fast(Chunk* chunk, Settings* settings, double* vol, double* mass, double* ie, double* temp)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL3_LAUNCH(s, "k3_field_summary",
               k3_field_summary<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                   s->g, chunk->volume, chunk->density, chunk->energy0, chunk->vec_u, s->rs));
    double o[4];
    if (!fetch(s, 4, o)) return;
    *vol += o[0];
    *mass += o[1];
    *ie += o[2];
    *temp += o[3];
}

// 3d/kernel_interface.h:29 (3d/c_kernels/omp3/cg_solver.c:9-102)
void run_cg_solver_init(Chunk* chunk, Settings* settings, double rx, double ry, double rz, double* rro)
{
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    if (settings->coefficient != TL3_CONDUCTIVITY && settings->coefficient != TL3_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL3_LAUNCH(s, "k3_cg_init",
               k3_cg_init<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                   s->g, settings->coefficient, rx, ry, rz, chunk->density, chunk->energy, chunk->vec_u,
                   chunk->vec_p, s->alt[ALT3_P], chunk->vec_r, chunk->vec_w, chunk->vec_kx, chunk->vec_ky,
                   chunk->vec_kz, s->rs, tl::NoFinish()));
    double o;
    if (fetch(s, 1, &o)) *rro += o;
}

// 3d/kernel_interface.h:32 (cg_solver.c:105-131), absorbing a pending p
// update, a pending depth-1 halo of p and a pending halo of u.
void run_cg_solver_calc_w(Chunk* chunk, Settings* settings, double* pw)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);   // deferred steps precede everything recorded after them
    if (s->pend.halo[TL3_FIELD_P] > 1) flush(s, chunk);
    const bool fuse = s->pend.calc_p;
    const bool refl = s->pend.halo[TL3_FIELD_P] == 1;
    const int ud = s->pend.halo[TL3_FIELD_U];
    double* u_halo = ud > 0 ? chunk->vec_u : nullptr;
    const Faces fc = faces_of(chunk);
    const Scalar beta{s->pend.beta, nullptr};
    const dim3 gr = fused_grid(s->g), bl = interior_block();
    double* p_out = fuse ? s->alt[ALT3_P] : chunk->vec_p;
#define W3(F, R)                                                                                                   \
    launch_cg_w3<F, R>(s, chunk, gr, fc, beta, chunk->vec_p, p_out, chunk->vec_r, chunk->vec_w, u_halo, ud, nullptr, \
                       tl::NoFinish())
    if (fuse && refl) W3(true, true);
    else if (fuse) W3(true, false);
    else if (refl) W3(false, true);
    else W3(false, false);
#undef W3
    if (fuse) swap_alt(s, chunk, ALT3_P);
    s->pend.calc_p = false;
    s->pend.halo[TL3_FIELD_P] = 0;
    s->pend.halo[TL3_FIELD_U] = 0;
    double o;
    if (fetch(s, 1, &o)) *pw += o;
}

// 3d/kernel_interface.h:34 (cg_solver.c:134-160); a halo of u still pending
// here is run before u changes.
void run_cg_solver_calc_ur(Chunk* chunk, Settings* settings, double alpha, double* rrn)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);
    if (s->pend.calc_p || s->pend.halo[TL3_FIELD_U]) flush(s, chunk);
    launch_cg_ur3(s, interior_grid(s->g), Scalar{alpha, nullptr}, chunk->vec_u, chunk->vec_p, chunk->vec_r,
                  chunk->vec_w, nullptr, tl::NoFinish());
    double o;
    if (fetch(s, 1, &o)) *rrn += o;
}

// 3d/kernel_interface.h:36 (cg_solver.c:163-193): recorded.
void run_cg_solver_calc_p(Chunk* chunk, Settings* settings, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    run_queues(s, chunk);
    if (s->pend.calc_p || s->pend.halo[TL3_FIELD_P]) flush(s, chunk);
    s->pend.calc_p = true;
    s->pend.beta = beta;
}

// 3d/kernel_interface.h:40 (3d/c_kernels/omp3/cheby_solver.c:27-59)
void run_cheby_solver_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    const dim3 gf = fused_grid(s->g), gr = interior_grid(s->g), bl = interior_block();
    const Faces none{0, 0, 0, 0, 0, 0};
    const tl::ChebyCoef coef{0.0, 0.0, nullptr, nullptr, nullptr};
    tl::DevParams prm{};
    TL3_LAUNCH(s, "k3_cheby_trip<init>",
               (k3_cheby_trip<false, false, true><<<gf, bl, 0, s->stream>>>(
                   s->g, none, coef, chunk->theta, 1, chunk->vec_u, chunk->vec_p, chunk->vec_u, chunk->vec_p,
                   chunk->vec_u0, chunk->vec_w, chunk->vec_r, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs,
                   nullptr, tl::NoFinish(), prm, Tma3Maps{}, nullptr)));
    TL3_LAUNCH(s, "k3_add_p", k3_add_p<false><<<gr, bl, 0, s->stream>>>(s->g, none, chunk->vec_u, chunk->vec_p));
}

// 3d/kernel_interface.h:42 (cheby_solver.c:62-99)
// With temporal blocking on and all six faces external, trips called in the
// reference drivers' pattern (a depth-1 halo update of u and nothing else
// pending before each) are deferred and run temporally blocked when any other
// run_* call needs the device state (run_cheby_queue); otherwise the trip
// runs at once.
void run_cheby_solver_iterate(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    const Faces fc = faces_of(chunk);
    if (s->temporal_blocking && fc.l && fc.r && fc.b && fc.t && fc.k && fc.f && !s->pq.active && !s->pend.calc_p &&
        s->pend.halo[TL3_FIELD_U] <= 1 && (long)s->cq.a.size() < s->table_len) {
        bool other = false;
        for (int f = 0; f < TL3_NUM_FIELDS; ++f) other |= f != TL3_FIELD_U && s->pend.halo[f] != 0;
        if (!other) {
            s->pend.halo[TL3_FIELD_U] = 0;   // the blocked trips reflect u on the fly and write its halo
            s->cq.active = true;
            s->cq.a.push_back(alpha);
            s->cq.b.push_back(beta);
            return;
        }
    }
    s = ready(chunk);
    if (!s) return;
    cheby_trip_one_step(s, chunk, alpha, beta);
}

// 3d/kernel_interface.h:46 (3d/c_kernels/omp3/jacobi_solver.c:9-66)
void run_jacobi_solver_init(Chunk* chunk, Settings* settings, double rx, double ry, double rz)
{
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    if (settings->coefficient < TL3_CONDUCTIVITY && settings->coefficient < TL3_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL3_LAUNCH(s, "k3_jacobi_init",
               k3_jacobi_init<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                   s->g, settings->coefficient, rx, ry, rz, chunk->density, chunk->energy, chunk->vec_u0,
                   chunk->vec_u, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz));
}

// 3d/kernel_interface.h:48 (jacobi_solver.c:69-115); the L1 change is assigned.
void run_jacobi_solver_iterate(Chunk* chunk, Settings* settings, double* error)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL_CUDA(cudaMemcpyAsync(chunk->vec_r, chunk->vec_u, sizeof(double) * (size_t)(s->g.xy() * s->g.z),
                            cudaMemcpyDeviceToDevice, s->stream));
    TL3_LAUNCH(s, "k3_jacobi_iterate",
               k3_jacobi_iterate<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                   s->g, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, chunk->vec_u0, chunk->vec_u, chunk->vec_r,
                   s->rs));
    double o;
    if (fetch(s, 1, &o)) *error = o;
}

// 3d/kernel_interface.h:52 (3d/c_kernels/omp3/ppcg_solver.c:8-26)
void run_ppcg_init(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    const Faces fc = faces_of(chunk);
    if (s->temporal_blocking && fc.l && fc.r && fc.b && fc.t && fc.k && fc.f) {
        s->pq.active = true;   // sd = r / theta runs with the first queued step
        s->pq.a.clear();
        s->pq.b.clear();
        return;
    }
    TL3_LAUNCH(s, "k3_ppcg_init", k3_ppcg_init<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                                      s->g, chunk->theta, chunk->vec_r, chunk->vec_sd));
}

// 3d/kernel_interface.h:54 (ppcg_solver.c:29-73)
void run_ppcg_inner_iteration(Chunk* chunk, Settings* settings, double alpha, double beta)
{
    (void)settings;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    // queued only in the reference drivers' pattern: a depth-1 halo update of
    // sd (and nothing else) requested right before the step
    if (s->pq.active && !s->pend.calc_p && s->pend.halo[TL3_FIELD_SD] == 1 && (long)s->pq.a.size() < s->table_len) {
        bool other = false;
        for (int f = 0; f < TL3_NUM_FIELDS; ++f) other |= f != TL3_FIELD_SD && s->pend.halo[f] != 0;
        if (!other) {
            s->pend.halo[TL3_FIELD_SD] = 0;   // the blocked steps reflect sd on the fly and write its halo
            s->pq.a.push_back(alpha);
            s->pq.b.push_back(beta);
            return;
        }
    }
    s = ready(chunk);   // runs the queue, if any, and the pending operations
    if (!s) return;
    const dim3 gr = interior_grid(s->g), bl = interior_block();
    TL3_LAUNCH(s, "k3_ppcg_inner_a", k3_ppcg_inner_a<<<gr, bl, 0, s->stream>>>(
                                         s->g, chunk->vec_u, chunk->vec_r, chunk->vec_kx, chunk->vec_ky,
                                         chunk->vec_kz, chunk->vec_sd));
    TL3_LAUNCH(s, "k3_ppcg_sd",
               k3_ppcg_sd<<<gr, bl, 0, s->stream>>>(s->g, alpha, beta, chunk->vec_sd, chunk->vec_r));
}

// 3d/kernel_interface.h:58 (3d/c_kernels/omp3/solver_methods.c:9-28)
void run_solver_copy_u(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL3_LAUNCH(s, "k3_copy_u", k3_copy_u<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                                   s->g, chunk->vec_u0, chunk->vec_u));
}

// 3d/kernel_interface.h:60 (solver_methods.c:31-56)
void run_calculate_residual(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL3_LAUNCH(s, "k3_residual", k3_residual<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                                     s->g, chunk->vec_u, chunk->vec_u0, chunk->vec_r, chunk->vec_kx, chunk->vec_ky,
                                     chunk->vec_kz));
}

// 3d/kernel_interface.h:62 (solver_methods.c:59-82)
void run_calculate_2norm(Chunk* chunk, Settings* settings, double* buffer, double* norm)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    TL3_LAUNCH(s, "k3_norm2",
               k3_norm2<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(s->g, buffer, s->rs));
    double o;
    if (fetch(s, 1, &o)) *norm += o;
}

// 3d/kernel_interface.h:64 (solver_methods.c:85-108)
void run_solver_finalise(Chunk* chunk, Settings* settings)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    if (tma_failed(s)) {
        tl::fail(35, "a TMA plane load of the w sweep did not complete (bounded barrier wait gave up)");
        return;
    }
    TL3_LAUNCH(s, "k3_finalise", k3_finalise<<<interior_grid(s->g), interior_block(), 0, s->stream>>>(
                                     s->g, chunk->energy, chunk->density, chunk->vec_u));
}

void tl3d_upload_field(Chunk* chunk, Settings* settings, int field_id, const double* host, long long count)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    double* f = field_by_id(chunk, field_id);
    if (!f || count != (long long)(s->g.xy() * s->g.z)) {
        tl::fail(8, "upload: bad field id %d or count %lld", field_id, count);
        return;
    }
    TL_CUDA(cudaMemcpyAsync(f, host, sizeof(double) * count, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

void tl3d_download_field(Chunk* chunk, Settings* settings, int field_id, double* host, long long count)
{
    (void)settings;
    TlSuite3D* s = ready(chunk);
    if (!s) return;
    double* f = field_by_id(chunk, field_id);
    if (!f || count != (long long)(s->g.xy() * s->g.z)) {
        tl::fail(8, "download: bad field id %d or count %lld", field_id, count);
        return;
    }
    TL_CUDA(cudaMemcpyAsync(host, f, sizeof(double) * count, cudaMemcpyDefault, s->stream));
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

}  // extern "C"
