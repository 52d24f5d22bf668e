// driver3d.cu -- device-resident timestep for the 3D suite.
//
// tl3d_solve_step runs one solve() (3d/diffuse.c:21-81) with the solver loops
// of 3d/drivers/{cg,cheby,ppcg}_solver_driver.c kept on the GPU, exactly as
// the 2D driver does (driver2d.cu), with the 3D stop test: after every trip
// the error is replaced by its square root before it is compared with eps
// (3d/drivers/cg_solver_driver.c:24-25) -- including the Chebyshev trips that
// do not recompute the norm, whose stale error is square-rooted again
// (3d/drivers/cheby_solver_driver.c:70-71). Jacobi is driven from the host
// through the suite's own kernel-interface entry points.
#include "blocked3d.cuh"
#include "host_maths.hpp"
#include "suite3d_impl.hpp"

#include <algorithm>

using namespace tl3d;
using tl::cheby_coefs;
using tl::cheby_est;
using tl::eigen_bounds;

extern "C" void print_and_log(Settings* settings, const char* format, ...) __attribute__((weak));

namespace {

constexpr int kBatch = 16;

struct Run3 {
    TlSuite3D* s;
    Chunk* chunk;
    Settings* settings;
    DevParams prm;
    Faces fc;
    dim3 gi, bl;
    dim3 gh;   // fused sweeps: interior + halo-duty z-plane
    DevState host_state;

    const int* done() const { return &s->d_state->done; }

    DevState read_state()
    {
        TL_CUDA(cudaMemcpyAsync(&host_state, s->d_state, sizeof(DevState), cudaMemcpyDeviceToHost, s->stream));
        TL_CUDA(cudaStreamSynchronize(s->stream));
        if (s->prof.on) s->prof.resolve();
        return host_state;
    }
    void write_state(const DevState& st)
    {
        host_state = st;
        s->h_mirror[0] = st.done;
        s->h_mirror[1] = st.trip;
        s->h_mirror[2] = st.reason;
        TL_CUDA(cudaMemcpyAsync(s->d_state, &host_state, sizeof(DevState), cudaMemcpyHostToDevice, s->stream));
        TL_CUDA(cudaStreamSynchronize(s->stream));
    }

    template <typename F>
    DevState loop(int first_trip, F&& launch_trip)
    {
        cudaEvent_t ev[2];
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
        int t = first_trip, batch = 0;
        bool pending_prev = false;
        while (t < prm.max_iters && !tl::failed()) {
            const int end = std::min(prm.max_iters, t + kBatch);
            for (; t < end; ++t) launch_trip(t);
            cudaEventRecord(ev[batch & 1], s->stream);
            if (pending_prev) {
                cudaEventSynchronize(ev[(batch + 1) & 1]);
                if (*(volatile int*)&s->h_mirror[0]) break;
            }
            pending_prev = true;
            ++batch;
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        return read_state();
    }

    // Launches blocks of trips: block(t) launches the block starting at trip t
    // and returns its length; batches of about kBatch trips, the done word of
    // the previous batch looked at while the current one runs. Returns the
    // state read back and, in `starts`, the first trip of every block launched.
    template <typename F>
    DevState loop_blocks(int first_trip, F&& block, std::vector<int>& starts)
    {
        cudaEvent_t ev[2];
        cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
        cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
        int t = first_trip, batch = 0;
        bool pending_prev = false;
        while (t < prm.max_iters && !tl::failed()) {
            const int end = std::min(prm.max_iters, t + kBatch);
            while (t < end) {
                starts.push_back(t);
                t += block(t);
            }
            cudaEventRecord(ev[batch & 1], s->stream);
            if (pending_prev) {
                cudaEventSynchronize(ev[(batch + 1) & 1]);
                if (*(volatile int*)&s->h_mirror[0]) break;
            }
            pending_prev = true;
            ++batch;
        }
        cudaEventDestroy(ev[0]);
        cudaEventDestroy(ev[1]);
        return read_state();
    }

    bool blocking() const { return s->temporal_blocking && fc.l && fc.r && fc.b && fc.t && fc.k && fc.f; }

    template <int MODE>
    void launch_blocked(const Blocked3Args& a, const double* A_in, const double* B_in, double* A_out, double* B_out,
                        const double* u0, double* u, double* w, double* r)
    {
        launch_blocked3<MODE>(s, chunk, a, A_in, B_in, A_out, B_out, u0, u, w, r, done());
    }

    double norm(const double* b)
    {
        TL3_LAUNCH(s, "k3_norm2", k3_norm2<<<gi, bl, 0, s->stream>>>(s->g, b, s->rs));
        double o = 0.0;
        fetch(s, 1, &o);
        return o;
    }

    void copy(double* dst, const double* src)
    {
        TL_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)(s->g.xy() * s->g.z), cudaMemcpyDeviceToDevice,
                                s->stream));
    }

    // cg_solver_main_step_driver trips until the loop ends; closes the phase.
    DevState cg_phase(int from, bool fresh)
    {
        double* buf[2] = {chunk->vec_p, s->alt[ALT3_P]};
        tl::FinCgW fin_w{s->d_state, s->d_cg_alphas};
        tl::FinCgUr fin_ur{s->d_state, s->d_cg_betas, prm, s->d_mirror};
        const Scalar beta{0.0, &s->d_state->beta}, alpha{0.0, &s->d_state->alpha};
        int cur = 0;
        auto trip = [&](int t) {
            if (fresh && t == from) {
                launch_cg_w3<false, false>(s, chunk, gh, fc, beta, buf[cur], buf[cur], chunk->vec_r, chunk->vec_w,
                                           nullptr, 0, done(), fin_w);
            } else {
                launch_cg_w3<true, true>(s, chunk, gh, fc, beta, buf[cur], buf[cur ^ 1], chunk->vec_r, chunk->vec_w,
                                         nullptr, 0, done(), fin_w);
                cur ^= 1;
            }
            launch_cg_ur3(s, gi, alpha, chunk->vec_u, buf[cur], chunk->vec_r, chunk->vec_w, done(), fin_ur);
        };
        DevState st = loop(from, trip);
        const int ran = st.trip - from;
        const int flips = fresh ? std::max(0, ran - 1) : ran;
        if (buf[flips & 1] != chunk->vec_p) swap_alt(s, chunk, ALT3_P);
        TL3_LAUNCH(s, "k3_cg_close", k3_cg_close<<<gi, bl, 0, s->stream>>>(s->g, fc, beta, 1, chunk->vec_p,
                                                                            chunk->vec_r, chunk->vec_u));
        if (st.trip > 0) {
            TL_CUDA(cudaMemcpyAsync(chunk->cg_alphas, s->d_cg_alphas, sizeof(double) * st.trip,
                                    cudaMemcpyDeviceToHost, s->stream));
            TL_CUDA(cudaMemcpyAsync(chunk->cg_betas, s->d_cg_betas, sizeof(double) * st.trip,
                                    cudaMemcpyDeviceToHost, s->stream));
        }
        TL_CUDA(cudaStreamSynchronize(s->stream));
        return st;
    }

    // cheby_solver_driver after the switch at trip tt (3d/drivers/cheby_solver_driver.c:11-154).
    DevState cheby_phase(int tt, TlStepStats3* stats)
    {
        if (!eigen_bounds(chunk, tt)) return host_state;
        const int count = prm.max_iters - tt;
        cheby_coefs(chunk, count);
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, chunk->cheby_alphas, sizeof(double) * count,
                                cudaMemcpyHostToDevice, s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, chunk->cheby_betas, sizeof(double) * count,
                                cudaMemcpyHostToDevice, s->stream));
        const double bb = norm(chunk->vec_u0);
        const Faces none{0, 0, 0, 0, 0, 0};
        tl::DevParams pc = prm;
        pc.switch_enabled = 0;
        TL3_LAUNCH(s, "k3_cheby_trip<init>",
                   (k3_cheby_trip<false, false, true><<<gh, bl, 0, s->stream>>>(
                       s->g, none, tl::ChebyCoef{0.0, 0.0, nullptr, nullptr, nullptr}, chunk->theta, 1, chunk->vec_u,
                       chunk->vec_p, chunk->vec_u, chunk->vec_p, chunk->vec_u0, chunk->vec_w, chunk->vec_r,
                       chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs, nullptr, tl::NoFinish(), pc, Tma3Maps{},
                       nullptr)));
        copy(s->alt[ALT3_U], chunk->vec_u);
        copy(s->alt[ALT3_P], chunk->vec_p);
        DevState st = host_state;
        st.nch = 1;
        st.est = 0;
        st.done = 0;
        st.reason = 0;
        write_state(st);
        double* ub[2] = {chunk->vec_u, s->alt[ALT3_U]};
        double* pb[2] = {chunk->vec_p, s->alt[ALT3_P]};
        tl::ChebyCoef coef{0.0, 0.0, s->d_cheby_alphas, s->d_cheby_betas, s->d_state};
        int cur = 0;
        auto trip = [&](int, int force) {
            tl::FinChebyTrip fin{s->d_state, pc, s->d_mirror, force};
            Tma3Maps m{};
            if (sweep_maps(s, chunk, ub[cur], pb[cur], &m)) {
                static unsigned set = 0;
                raise_ring_smem(s, k3_cheby_trip<true, true, false, tl::FinChebyTrip, true>, set);
                TL3_LAUNCH(s, "k3_cheby_trip",
                           (k3_cheby_trip<true, true, false, tl::FinChebyTrip, true><<<gh, bl, kTmaRingBytes,
                                                                                       s->stream>>>(
                               s->g, fc, coef, 0.0, force, ub[cur], pb[cur], ub[cur ^ 1], pb[cur ^ 1], chunk->vec_u0,
                               chunk->vec_w, chunk->vec_r, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs, done(),
                               fin, pc, m, s->d_mirror + kTmaErrWord)));
            } else {
                TL3_LAUNCH(s, "k3_cheby_trip", (k3_cheby_trip<true, true, false><<<gh, bl, 0, s->stream>>>(
                               s->g, fc, coef, 0.0, force, ub[cur], pb[cur], ub[cur ^ 1], pb[cur ^ 1], chunk->vec_u0,
                               chunk->vec_w, chunk->vec_r, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs, done(),
                               fin, pc, Tma3Maps{}, nullptr)));
            }
            cur ^= 1;
        };
        trip(tt, 1);
        st = read_state();
        const double error = s->h_out[0];
        const int est = cheby_est(chunk, error, bb);
        if (stats) stats->est_iters = est;
        int flips = 1;   // buffer flips of the launches that ran
        if (!st.done) {
            st.est = est;
            write_state(st);
            if (blocking()) {
                // trip t takes the norm when nch >= est and (t + 1) % 10 == 0
                // (FinChebyTrip); a block ends at such a trip, at max_iters or
                // after kTB3 trips
                auto is_norm = [&](int t) { return t - tt + 1 >= est && ((t + 1) % 10) == 0; };
                std::vector<int> starts;
                st = loop_blocks(tt + 1, [&](int t) {
                    int L = 1;
                    while (!(is_norm(t + L - 1) || L == kTB3 || t + L >= prm.max_iters)) ++L;
                    const int last = t + L - 1;
                    const int nrm = is_norm(last) ? 1 : 0;
                    const Blocked3Args a{L, t - tt + 1, (nrm || last + 1 >= prm.max_iters) ? 1 : 0, 0.0,
                                         s->d_cheby_alphas, s->d_cheby_betas};
                    launch_blocked<0>(a, ub[cur], pb[cur], ub[cur ^ 1], pb[cur ^ 1], chunk->vec_u0, nullptr,
                                      chunk->vec_w, chunk->vec_r);
                    const tl::FinChebyBlock fin{s->d_state, pc, s->d_mirror, L, nrm};
                    if (nrm)
                        TL3_LAUNCH(s, "k3_norm2_fin", (k3_norm2_fin<<<gh, bl, 0, s->stream>>>(s->g, chunk->vec_r,
                                                                                             s->rs, done(), fin)));
                    else
                        TL3_LAUNCH(s, "k3_finish_only", (k3_finish_only<<<1, 32, 0, s->stream>>>(done(), fin)));
                    cur ^= 1;
                    return L;
                }, starts);
                for (int t0 : starts) flips += t0 < st.trip ? 1 : 0;
            } else {
                st = loop(tt + 1, [&](int t) { trip(t, 0); });
                flips = st.nch - 1;
            }
        }
        const int trips = st.nch - 1;
        if (ub[flips & 1] != chunk->vec_u) swap_alt(s, chunk, ALT3_U);
        if (pb[flips & 1] != chunk->vec_p) swap_alt(s, chunk, ALT3_P);
        TL3_LAUNCH(s, "k3_add_p<close>", k3_add_p<true><<<gi, bl, 0, s->stream>>>(s->g, fc, chunk->vec_u, chunk->vec_p));
        TL_CUDA(cudaStreamSynchronize(s->stream));
        if (stats) stats->cheby_iters = trips;
        return st;
    }

    // ppcg_solver_driver after the switch at trip tt (3d/drivers/ppcg_solver_driver.c:9-190).
    DevState ppcg_phase(int tt, TlStepStats3* stats)
    {
        if (!eigen_bounds(chunk, tt)) return host_state;
        const int ni = settings->ppcg_inner_steps;
        cheby_coefs(chunk, ni);
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, chunk->cheby_alphas, sizeof(double) * ni,
                                cudaMemcpyHostToDevice, s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, chunk->cheby_betas, sizeof(double) * ni, cudaMemcpyHostToDevice,
                                s->stream));
        TL3_LAUNCH(s, "k3_residual", k3_residual<<<gi, bl, 0, s->stream>>>(s->g, chunk->vec_u, chunk->vec_u0,
                                                                            chunk->vec_r, chunk->vec_kx,
                                                                            chunk->vec_ky, chunk->vec_kz));
        copy(s->alt[ALT3_R], chunk->vec_r);
        copy(s->alt[ALT3_SD], chunk->vec_sd);
        DevState st = host_state;
        st.done = 0;
        st.reason = 0;
        st.nch = 0;
        write_state(st);
        double* pb[2] = {chunk->vec_p, s->alt[ALT3_P]};
        double* rb[2] = {chunk->vec_r, s->alt[ALT3_R]};
        double* sb[2] = {chunk->vec_sd, s->alt[ALT3_SD]};
        int pc = 0, rc = 0, sc = 0;
        const Scalar beta{0.0, &s->d_state->beta}, alpha{0.0, &s->d_state->alpha};
        const tl::PpcgCoef coef{0.0, 0.0, s->d_cheby_alphas, s->d_cheby_betas};
        tl::DevParams pp_prm = prm;
        pp_prm.switch_enabled = 0;
        tl::FinPpcgW fin_w{s->d_state};
        tl::FinPpcgNorm fin_n{s->d_state, pp_prm, s->d_mirror};
        const bool blocked = blocking();
        const int inner_flips = blocked ? (ni + kTB3 - 1) / kTB3 : ni;   // r/sd buffer flips per outer trip
        auto trip = [&](int t) {
            if (t == tt) {
                launch_cg_w3<false, false>(s, chunk, gh, fc, beta, pb[pc], pb[pc], rb[rc], chunk->vec_w, nullptr, 0,
                                           done(), fin_w);
            } else {
                launch_cg_w3<true, true>(s, chunk, gh, fc, beta, pb[pc], pb[pc ^ 1], rb[rc], chunk->vec_w, nullptr,
                                         0, done(), fin_w);
                pc ^= 1;
            }
            launch_cg_ur3(s, gi, alpha, chunk->vec_u, pb[pc], rb[rc], chunk->vec_w, done(), tl::NoFinish());
            if (blocked) {
                for (int pp0 = 0; pp0 < ni; pp0 += kTB3) {
                    const int L = std::min(kTB3, ni - pp0);
                    const Blocked3Args a{L, pp0, 0, chunk->theta, s->d_cheby_alphas, s->d_cheby_betas};
                    launch_blocked<1>(a, sb[sc], rb[rc], sb[sc ^ 1], rb[rc ^ 1], nullptr, chunk->vec_u, nullptr,
                                      nullptr);
                    sc ^= 1;
                    rc ^= 1;
                    if (pp0 + L == ni)
                        TL3_LAUNCH(s, "k3_norm2_fin", (k3_norm2_fin<<<gh, bl, 0, s->stream>>>(s->g, rb[rc], s->rs,
                                                                                             done(), fin_n)));
                }
                return;
            }
            for (int pp = 0; pp < ni; ++pp) {
                const bool last = pp == ni - 1;
#define STEP3(FOLD, NORM, FIN)                                                                                    \
    do {                                                                                                          \
        Tma3Maps m{};                                                                                             \
        if (sweep_maps(s, chunk, sb[sc], rb[rc], &m)) {                                                           \
            static unsigned set = 0;                                                                              \
            raise_ring_smem(s, k3_ppcg_step<FOLD, NORM, decltype(FIN), true>, set);                               \
            TL3_LAUNCH(s, "k3_ppcg_step",                                                                         \
                       (k3_ppcg_step<FOLD, NORM, decltype(FIN), true><<<gh, bl, kTmaRingBytes, s->stream>>>(       \
                           s->g, fc, chunk->theta, coef, pp - 1, sb[sc], sb[sc ^ 1], rb[rc], rb[rc ^ 1],         \
                           chunk->vec_u, chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs, done(), FIN, m,     \
                           s->d_mirror + kTmaErrWord)));                                                          \
        } else {                                                                                                  \
            TL3_LAUNCH(s, "k3_ppcg_step", (k3_ppcg_step<FOLD, NORM><<<gh, bl, 0, s->stream>>>(                    \
                                              s->g, fc, chunk->theta, coef, pp - 1, sb[sc], sb[sc ^ 1], rb[rc],  \
                                              rb[rc ^ 1], chunk->vec_u, chunk->vec_kx, chunk->vec_ky,           \
                                              chunk->vec_kz, s->rs, done(), FIN, Tma3Maps{}, nullptr)));          \
        }                                                                                                         \
    } while (0)
                if (pp == 0 && last) STEP3(1, true, fin_n);
                else if (pp == 0) STEP3(1, false, tl::NoFinish());
                else if (last) STEP3(2, true, fin_n);
                else STEP3(2, false, tl::NoFinish());
#undef STEP3
                sc ^= 1;
                rc ^= 1;
            }
        };
        st = loop(tt, trip);
        const int outer = st.nch;
        const int pflips = std::max(0, outer - 1);
        const int rflips = outer * inner_flips;
        if (pb[pflips & 1] != chunk->vec_p) swap_alt(s, chunk, ALT3_P);
        if (rb[rflips & 1] != chunk->vec_r) swap_alt(s, chunk, ALT3_R);
        if (sb[rflips & 1] != chunk->vec_sd) swap_alt(s, chunk, ALT3_SD);
        if (outer > 0) {
            TL3_LAUNCH(s, "k3_ppcg_sd", k3_ppcg_sd<<<gi, bl, 0, s->stream>>>(s->g, chunk->cheby_alphas[ni - 1],
                                                                              chunk->cheby_betas[ni - 1],
                                                                              chunk->vec_sd, chunk->vec_r));
            TL3_LAUNCH(s, "k3_cg_close", k3_cg_close<<<gi, bl, 0, s->stream>>>(s->g, fc, beta, 1, chunk->vec_p,
                                                                                chunk->vec_r, nullptr));
        }
        TL_CUDA(cudaStreamSynchronize(s->stream));
        if (stats) stats->ppcg_iters = outer;
        return st;
    }
};

// solve_finished_driver (3d/drivers/solve_finished_driver.c:7-44)
void solve_finished(Run3& R, TlStepStats3* st_out)
{
    TlSuite3D* s = R.s;
    Chunk* chunk = R.chunk;
    Settings* settings = R.settings;
    bool* flags = settings->fields_to_exchange;
    flush(s, chunk);
    if (settings->check_result) {
        TL3_LAUNCH(s, "k3_residual", k3_residual<<<R.gi, R.bl, 0, s->stream>>>(
                                         s->g, chunk->vec_u, chunk->vec_u0, chunk->vec_r, chunk->vec_kx,
                                         chunk->vec_ky, chunk->vec_kz));
        st_out->exact_error = R.norm(chunk->vec_r);
    }
    TL3_LAUNCH(s, "k3_finalise", k3_finalise<<<R.gi, R.bl, 0, s->stream>>>(s->g, chunk->energy, chunk->density,
                                                                            chunk->vec_u));
    flags[TL3_FIELD_ENERGY1] = true;
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) s->pend.halo[f] = flags[f] ? 1 : 0;
    flush(s, chunk);
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// jacobi_solver_driver (3d/drivers/jacobi_solver_driver.c:7-86)
double jacobi_loop(Chunk* chunk, Settings* settings, double rx, double ry, double rz, int* iters)
{
    bool* flags = settings->fields_to_exchange;
    run_jacobi_solver_init(chunk, settings, rx, ry, rz);
    run_solver_copy_u(chunk, settings);
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) flags[f] = false;
    flags[TL3_FIELD_U] = true;
    double error = 1e10;
    int tt;
    for (tt = 0; tt < settings->max_iters && !tl::failed(); ++tt) {
        run_jacobi_solver_iterate(chunk, settings, &error);
        if (tt % 50 == 0) {
            run_local_halos(chunk, settings, 1);
            run_calculate_residual(chunk, settings);
            run_calculate_2norm(chunk, settings, chunk->vec_r, &error);
        }
        run_local_halos(chunk, settings, 1);
        error = sqrt(error);
        if (fabs(error) < settings->eps) break;
    }
    *iters = tt;
    return error;
}

}  // namespace

extern "C" {

void tl3d_solve_step(Chunk* chunk, Settings* settings, int tt, TlStepStats3* stats)
{
    (void)tt;
    if (tl::failed()) return;
    TlSuite3D* s = suite_of(chunk);
    if (!s) return;
    if (settings->max_iters > s->table_len) {
        tl::fail(32, "max_iters %d exceeds the %d the chunk was initialised with", settings->max_iters, s->table_len);
        return;
    }
    if (settings->num_chunks_per_rank != 1) {
        tl::fail(34, "the device-resident driver solves one chunk per rank (num_chunks_per_rank=%d)",
                 settings->num_chunks_per_rank);
        return;
    }
    const Faces fc = faces_of(chunk);
    if (!(fc.l && fc.r && fc.b && fc.t && fc.k && fc.f)) {   // no remote halo exchange inside the device loop
        tl::fail(34, "the device-resident driver solves a chunk whose six faces are external (a decomposed mesh "
                     "runs through run_*)");
        return;
    }
    flush(s, chunk);
    TlStepStats3 local{};
    TlStepStats3* st_out = stats ? stats : &local;
    *st_out = TlStepStats3{};
    Run3 R{s, chunk, settings, {}, faces_of(chunk), interior_grid(s->g), interior_block(), fused_grid(s->g), {}};
    R.prm.eps = settings->eps;
    R.prm.eps_lim = settings->eps_lim;
    R.prm.max_iters = settings->max_iters;
    R.prm.presteps = settings->presteps;
    R.prm.error_switch = settings->error_switch ? 1 : 0;
    R.prm.switch_enabled = (settings->solver == TL3_CHEBY_SOLVER || settings->solver == TL3_PPCG_SOLVER) ? 1 : 0;
    R.prm.dims3 = 1;
    bool* flags = settings->fields_to_exchange;

    // solve(): dt, rx, ry, rz (3d/diffuse.c:27-36)
    const double dt = chunk->dt_init < settings->dt_init ? chunk->dt_init : settings->dt_init;
    const double rx = dt / (settings->dx * settings->dx);
    const double ry = dt / (settings->dy * settings->dy);
    const double rz = dt / (settings->dz * settings->dz);
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
    s->pend.halo[TL3_FIELD_ENERGY1] = s->pend.halo[TL3_FIELD_DENSITY] = 2;
    flush(s, chunk);

    if (settings->solver == TL3_JACOBI_SOLVER) {
        int it = 0;
        const double error = jacobi_loop(chunk, settings, rx, ry, rz, &it);
        st_out->jacobi_iters = it;
        st_out->total_iters = it;
        st_out->error = error;
        solve_finished(R, st_out);
        if (print_and_log && settings->tea_out_fp) print_and_log(settings, "Jacobi: \t\t%d iterations\n", it);
        return;
    }
    if (settings->coefficient != TL3_CONDUCTIVITY && settings->coefficient != TL3_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    // cg_solver_init_driver (3d/drivers/cg_solver_driver.c:31-63)
    TL3_LAUNCH(s, "k3_cg_init", k3_cg_init<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                                    s->g, settings->coefficient, rx, ry, rz, chunk->density, chunk->energy,
                                    chunk->vec_u, chunk->vec_p, s->alt[ALT3_P], chunk->vec_r, chunk->vec_w,
                                    chunk->vec_kx, chunk->vec_ky, chunk->vec_kz, s->rs,
                                    tl::FinCgInit{s->d_state, s->d_mirror}));
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
    s->pend.halo[TL3_FIELD_U] = s->pend.halo[TL3_FIELD_P] = 1;
    flush(s, chunk);
    TL3_LAUNCH(s, "k3_copy_u", k3_copy_u<<<R.gi, R.bl, 0, s->stream>>>(s->g, chunk->vec_u0, chunk->vec_u));
    R.read_state();

    DevState st = R.cg_phase(0, true);
    double error = st.error;
    if (st.reason == 2 && settings->solver == TL3_CHEBY_SOLVER) {
        st = R.cheby_phase(st.trip, st_out);
        error = st.error;
        for (int f = 0; f < TL3_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL3_FIELD_U] = true;
    } else if (st.reason == 2 && settings->solver == TL3_PPCG_SOLVER) {
        st = R.ppcg_phase(st.trip, st_out);
        error = st.error;
        for (int f = 0; f < TL3_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL3_FIELD_P] = true;
    } else {
        for (int f = 0; f < TL3_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL3_FIELD_U] = flags[TL3_FIELD_P] = true;
    }
    if (tl::failed()) return;
    if (tma_failed(s)) {
        tl::fail(35, "a TMA plane load of the w sweep did not complete (bounded barrier wait gave up)");
        return;
    }
    const int tt_exit = st.reason == 1 ? st.trip - 1 : st.trip;
    st_out->total_iters = tt_exit;
    if (settings->solver == TL3_CHEBY_SOLVER) st_out->cg_iters = tt_exit - st_out->cheby_iters + 1;
    else if (settings->solver == TL3_PPCG_SOLVER) st_out->cg_iters = tt_exit - st_out->ppcg_iters + 1;
    else st_out->cg_iters = tt_exit;
    st_out->error = error;
    st_out->eigmin = chunk->eigmin;
    st_out->eigmax = chunk->eigmax;
    solve_finished(R, st_out);
    if (print_and_log && settings->tea_out_fp) {
        print_and_log(settings, "CG: \t\t\t%d iterations\n", st_out->cg_iters);
        if (settings->solver == TL3_CHEBY_SOLVER)
            print_and_log(settings, "Cheby: \t\t\t%d iterations (%d estimated)\n", st_out->cheby_iters,
                          st_out->est_iters);
        if (settings->solver == TL3_PPCG_SOLVER)
            print_and_log(settings, "PPCG: \t\t\t%d iterations (%d inner iterations per)\n", st_out->ppcg_iters,
                          settings->ppcg_inner_steps);
    }
}

}  // extern "C"
