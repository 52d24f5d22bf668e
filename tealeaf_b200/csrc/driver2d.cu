// driver2d.cu -- device-resident timestep for the 2D suite.
//
// tl2d_solve_step runs one solve() (2d/diffuse.c:22-80) with the solver loops
// of 2d/drivers/{cg,cheby,ppcg,jacobi}_driver.c kept on the GPU: the scalars
// (alpha = rro/pw, beta = rrn/rro, the Chebyshev/PPCG coefficients by trip),
// the stop test and the CG-to-Chebyshev/PPCG switch are evaluated by the last
// block of each reduction, and the host only launches trips in batches and
// looks at a mapped "done" word once per batch. Everything the host needs on
// the way is computed on the host exactly as the reference drivers do: the
// Lanczos eigenvalue bounds (tridiagonal QL), the Chebyshev tables and the
// iteration estimate (single-precision logf/roundf, as cheby_driver.c:146-160).
//
// The fused sweeps of kernels2d.cuh do the CG iteration in 96 B/cell, a
// Chebyshev trip in 56-72 B/cell and a PPCG inner step in 64 B/cell. Memory
// ends each solve in the state the reference leaves it in: pending updates
// and halo reflections are closed at the end of every phase, following the
// reference's halo flags (e.g. the halo of u is not refreshed during PPCG).
//
// diffuse_overload (2d/application.h:9-11) runs every timestep this way.
#include "blocked2d.cuh"
#include "host_maths.hpp"
#include "pcg2d.cuh"
#include "suite2d_impl.hpp"

#include <cfloat>
#include <cmath>
#include <vector>

using namespace tl2d;
using tl::cheby_coefs;
using tl::cheby_est;
using tl::eigen_bounds;

extern "C" void print_and_log(Settings* settings, const char* format, ...) __attribute__((weak));
extern "C" void field_summary_driver(Chunk* chunks, Settings* settings, bool is_solve_finished) __attribute__((weak));

namespace {

constexpr int kBatch = 16;   // solver-loop trips launched between looks at the done word

// ------------------------------------------------------------- the driver --

struct Run {
    TlSuite2D* s;
    Chunk* chunk;
    Settings* settings;
    DevParams prm;
    Faces fc;
    dim3 gi;               // interior sweeps
    dim3 gh;               // fused sweeps: interior + halo-duty block row
    DevState host_state;   // last copy read back

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

    // Launches trips through `launch_trip(t)` in batches, looking at the done
    // word of the previous batch while the current one runs; returns when the
    // loop has ended (state read back).
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

    bool blocking() const
    {
        return s->temporal_blocking && fc.l && fc.r && fc.b && fc.t;
    }

    // ------------------------------------------------------------- CG phase
    // Trips `from`.. of cg_main_step_driver (2d/drivers/cg_driver.c:65-124)
    // until the loop ends; `fresh`: the first trip follows cg_init (nothing
    // pending). Closes the phase: last p update and the halo of u and p.
    DevState cg_phase(int from, bool fresh)
    {
        FinCgUr fin_ur{s->d_state, s->d_cg_betas, prm, s->d_mirror};
        const Scalar alpha{0.0, &s->d_state->alpha};
        return cg_trips(from, fresh, chunk->r, [&](double* p) {
            launch_cg_ur2(s, gi, alpha, chunk->u, p, chunk->r, chunk->w, done(), fin_ur);
        });
    }

    // The CG loop with `fold` the field of the p update p = beta p + fold (r
    // for CG, z for the preconditioned CG) and ur(p) launching the second
    // sweep of a trip on the current p buffer.
    template <typename Ur>
    DevState cg_trips(int from, bool fresh, const double* fold, Ur&& ur)
    {
        double* buf[2] = {chunk->p, s->alt[ALT_P]};
        FinCgW fin_w{s->d_state, s->d_cg_alphas};
        const Scalar beta{0.0, &s->d_state->beta};
        // parity of the current p buffer: trip t (t > from or !fresh) writes buf[(t - from + base) & 1]
        int cur = 0;
        auto trip = [&](int t) {
            if (fresh && t == from) {
                launch_cg_w2<false, false>(s, chunk, gh, fc, beta, buf[cur], buf[cur], fold, chunk->w, nullptr,
                                           0, done(), fin_w);
            } else {
                launch_cg_w2<true, true>(s, chunk, gh, fc, beta, buf[cur], buf[cur ^ 1], fold, chunk->w,
                                         nullptr, 0, done(), fin_w);
                cur ^= 1;
            }
            ur(buf[cur]);
        };
        DevState st = loop(from, trip);
        // Trips from..st.trip-1 ran; the fused ones flipped the current buffer.
        const int ran = st.trip - from;
        const int flips = fresh ? std::max(0, ran - 1) : ran;
        double* pcur = buf[flips & 1];
        if (pcur != chunk->p) swap_alt(s, chunk, ALT_P);
        TL_LAUNCH(s, "k_cg_close", (k_cg_close<<<gi, BX, 0, s->stream>>>(s->g, fc, beta, 1, chunk->p, fold,
                                                                           chunk->u)));
        // host copies of the CG coefficients (the reference drivers keep them on the host)
        if (st.trip > 0) {
            TL_CUDA(cudaMemcpyAsync(chunk->cg_alphas, s->d_cg_alphas, sizeof(double) * st.trip,
                                    cudaMemcpyDeviceToHost, s->stream));
            TL_CUDA(cudaMemcpyAsync(chunk->cg_betas, s->d_cg_betas, sizeof(double) * st.trip,
                                    cudaMemcpyDeviceToHost, s->stream));
        }
        TL_CUDA(cudaStreamSynchronize(s->stream));
        return st;
    }

    // ------------------------------------------------- preconditioned CG
    // After cg_init, the halo of u and p and copy_u: M factored into the
    // chunk's mi field, z = M^-1 r, p = z, rro = r.z, then the CG loop with z
    // folded into p and the u/r/z sweep (pcg2d.cuh). z is held in the suite's
    // second sd buffer (unused by CG).
    template <int BS>
    DevState pcg_phase()
    {
        Geo gb = s->g;
        gb.rows = (gb.rows + BS - 1) / BS * BS;   // strips of whole blocks
        const dim3 gbi = interior_grid(gb);
        double* z = s->alt[ALT_SD];
        TL_LAUNCH(s, "k_pcg_init", (k_pcg_init<BS><<<gbi, BX, 0, s->stream>>>(
                                       gb, fc, chunk->r, chunk->kx, chunk->ky, chunk->mi, z, chunk->p, s->rs,
                                       FinCgInit{s->d_state, s->d_mirror})));
        read_state();
        FinPcgUr fin_ur{s->d_state, s->d_cg_betas, prm, s->d_mirror};
        const Scalar alpha{0.0, &s->d_state->alpha};
        if (tma_usable(s)) {
            static unsigned attr_set = 0;   // devices on which the shared-memory size was raised
            if (!(attr_set & (1u << (s->device & 31)))) {
                TL_CUDA(cudaFuncSetAttribute(k_pcg_ur_tma<BS, FinPcgUr>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)kPcgTmaBytes));
                attr_set |= 1u << (s->device & 31);
            }
        }
        return cg_trips(0, true, z, [&](double* p) {
            const CUtensorMap *mu = nullptr, *mp = nullptr, *mr = nullptr, *mw = nullptr, *mm = nullptr, *my = nullptr;
            if (tma_usable(s)) {
                mu = tma_map(s, chunk->u, 3);
                mp = tma_map(s, p, 3);
                mr = tma_map(s, chunk->r, 3);
                mw = tma_map(s, chunk->w, 3);
                mm = tma_map(s, chunk->mi, 3);
                my = tma_map(s, chunk->ky, 3);
            }
            if (mu && mp && mr && mw && mm && my) {
                const PcgMaps m{*mu, *mp, *mr, *mw, *mm, *my};
                TL_LAUNCH(s, "k_pcg_ur", (k_pcg_ur_tma<BS><<<gbi, BX, kPcgTmaBytes, s->stream>>>(
                                             gb, alpha, m, chunk->u, chunk->r, z, s->rs, done(), fin_ur,
                                             s->d_mirror + kTmaErrWord2)));
            } else {
                TL_LAUNCH(s, "k_pcg_ur", (k_pcg_ur<BS><<<gbi, BX, 0, s->stream>>>(gb, alpha, chunk->u, p, chunk->r,
                                                                                  chunk->w, chunk->ky, chunk->mi, z,
                                                                                  s->rs, done(), fin_ur)));
            }
        });
    }

    double norm(const double* b)
    {
        TL_LAUNCH(s, "k_norm2", k_norm2<<<gi, BX, 0, s->stream>>>(s->g, b, s->rs));
        double o = 0.0;
        fetch(s, 1, &o);
        return o;
    }

    void copy(double* dst, const double* src)
    {
        TL_CUDA(cudaMemcpyAsync(dst, src, sizeof(double) * (size_t)s->g.x * s->g.y, cudaMemcpyDeviceToDevice,
                                s->stream));
    }

    // --------------------------------------------------------- Chebyshev
    // 2d/drivers/cheby_driver.c:11-143 after the switch at trip `tt`.
    DevState cheby_phase(int tt, TlStepStats* stats)
    {
        if (!eigen_bounds(chunk, tt)) return host_state;
        const int count = prm.max_iters - tt;
        cheby_coefs(chunk, count);
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, chunk->cheby_alphas, sizeof(double) * count,
                                cudaMemcpyHostToDevice, s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, chunk->cheby_betas, sizeof(double) * count,
                                cudaMemcpyHostToDevice, s->stream));
        const double bb = norm(chunk->u0);
        // cheby_init (cheby.c:26-54) without its final u += p, which the next trip folds in
        TL_LAUNCH(s, "k_cheby_sweep<init>",
                  k_cheby_sweep<true><<<gi, BX, 0, s->stream>>>(s->g, 0.0, 0.0, chunk->theta, chunk->u, chunk->u0,
                                                               chunk->p, chunk->r, chunk->w, chunk->kx, chunk->ky));
        copy(s->alt[ALT_U], chunk->u);
        copy(s->alt[ALT_P], chunk->p);
        DevState st = host_state;
        st.nch = 1;
        st.est = 0;
        st.done = 0;
        st.reason = 0;
        write_state(st);
        double* ub[2] = {chunk->u, s->alt[ALT_U]};
        double* pb[2] = {chunk->p, s->alt[ALT_P]};
        ChebyCoef coef{0.0, 0.0, s->d_cheby_alphas, s->d_cheby_betas, s->d_state};
        DevParams pc = prm;
        pc.switch_enabled = 0;   // already switched
        int cur = 0;
        auto trip = [&](int t, int force) {
            FinChebyTrip fin{s->d_state, pc, s->d_mirror, force};
            TL_LAUNCH(s, "k_cheby_trip", (k_cheby_trip<true, true><<<gh, BX, 0, s->stream>>>(
                          s->g, fc, coef, force, ub[cur], pb[cur], ub[cur ^ 1], pb[cur ^ 1], chunk->u0, chunk->w,
                          chunk->r, chunk->kx, chunk->ky, s->rs, done(), fin, pc)));
            cur ^= 1;
            (void)t;
        };
        // first Chebyshev trip: always takes the norm, then the estimate
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
                // after Blk<0>::TB trips
                auto is_norm = [&](int t) { return t - tt + 1 >= est && ((t + 1) % 10) == 0; };
                std::vector<int> starts;
                st = loop_blocks(tt + 1, [&](int t) {
                    int L = 1;
                    while (!(is_norm(t + L - 1) || L == Blk<0>::TB || t + L >= prm.max_iters)) ++L;
                    const int last = t + L - 1;
                    const int norm = is_norm(last) ? 1 : 0;
                    BlockedArgs a{L, t - tt + 1, (norm || last + 1 >= prm.max_iters) ? 1 : 0, 0.0, s->d_cheby_alphas,
                                  s->d_cheby_betas};
                    launch_blocked<0>(s, "k_blocked<cheby>", a, ub[cur], pb[cur], ub[cur ^ 1], pb[cur ^ 1],
                                      chunk->u0, nullptr, chunk->w, chunk->r, chunk->kx, chunk->ky, done());
                    const FinChebyBlock fin{s->d_state, pc, s->d_mirror, L, norm};
                    if (norm)
                        TL_LAUNCH(s, "k_norm2_fin", (k_norm2_fin<<<gi, BX, 0, s->stream>>>(s->g, chunk->r, s->rs,
                                                                                            done(), fin)));
                    else
                        TL_LAUNCH(s, "k_finish_only", (k_finish_only<<<1, 32, 0, s->stream>>>(done(), fin)));
                    cur ^= 1;
                    return L;
                }, starts);
                for (int t0 : starts) flips += t0 < st.trip ? 1 : 0;
            } else {
                st = loop(tt + 1, [&](int t) { trip(t, 0); });
                flips = st.nch - 1;
            }
        }
        const int trips = st.nch - 1;           // Chebyshev trips run
        if (ub[flips & 1] != chunk->u) swap_alt(s, chunk, ALT_U);
        if (pb[flips & 1] != chunk->p) swap_alt(s, chunk, ALT_P);
        TL_LAUNCH(s, "k_add_p_close", k_add_p_close<<<gi, BX, 0, s->stream>>>(s->g, fc, chunk->u, chunk->p));
        TL_CUDA(cudaStreamSynchronize(s->stream));
        if (stats) stats->cheby_iters = trips;
        return st;
    }

    // --------------------------------------------------------------- PPCG
    // 2d/drivers/ppcg_driver.c:10-189 after the switch at trip `tt`.
    DevState ppcg_phase(int tt, TlStepStats* stats)
    {
        if (!eigen_bounds(chunk, tt)) return host_state;
        const int ni = settings->ppcg_inner_steps;
        cheby_coefs(chunk, ni);
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_alphas, chunk->cheby_alphas, sizeof(double) * ni,
                                cudaMemcpyHostToDevice, s->stream));
        TL_CUDA(cudaMemcpyAsync(s->d_cheby_betas, chunk->cheby_betas, sizeof(double) * ni, cudaMemcpyHostToDevice,
                                s->stream));
        // ppcg_init_driver: r = u0 - A u (the halo of p is already in place)
        TL_LAUNCH(s, "k_residual", k_residual<<<gi, BX, 0, s->stream>>>(s->g, chunk->u, chunk->u0, chunk->r,
                                                                          chunk->kx, chunk->ky));
        copy(s->alt[ALT_R], chunk->r);
        copy(s->alt[ALT_SD], chunk->sd);
        DevState st = host_state;
        st.done = 0;
        st.reason = 0;
        st.nch = 0;
        write_state(st);
        double* pb[2] = {chunk->p, s->alt[ALT_P]};
        double* rb[2] = {chunk->r, s->alt[ALT_R]};
        double* sb[2] = {chunk->sd, s->alt[ALT_SD]};
        int pc = 0, rc = 0, sc = 0;
        const Scalar beta{0.0, &s->d_state->beta}, alpha{0.0, &s->d_state->alpha};
        const PpcgCoef coef{0.0, 0.0, s->d_cheby_alphas, s->d_cheby_betas};
        DevParams pp_prm = prm;
        pp_prm.switch_enabled = 0;   // already switched
        FinPpcgW fin_w{s->d_state};
        FinPpcgNorm fin_n{s->d_state, pp_prm, s->d_mirror};
        const bool blocked = blocking();
        constexpr int TB = Blk<1>::TB;
        const int inner_flips = blocked ? (ni + TB - 1) / TB : ni;   // r/sd buffer flips per outer trip
        auto trip = [&](int t) {
            if (t == tt) {
                launch_cg_w2<false, false>(s, chunk, gh, fc, beta, pb[pc], pb[pc], rb[rc], chunk->w, nullptr, 0,
                                           done(), fin_w);
            } else {
                launch_cg_w2<true, true>(s, chunk, gh, fc, beta, pb[pc], pb[pc ^ 1], rb[rc], chunk->w, nullptr, 0,
                                         done(), fin_w);
                pc ^= 1;
            }
            launch_cg_ur2(s, gi, alpha, chunk->u, pb[pc], rb[rc], chunk->w, done(), tl::NoFinish());
            if (blocked) {
                for (int pp0 = 0; pp0 < ni; pp0 += TB) {
                    const int L = std::min(TB, ni - pp0);
                    const bool last = pp0 + L == ni;
                    BlockedArgs a{L, pp0, 0, chunk->theta, s->d_cheby_alphas, s->d_cheby_betas};
                    launch_blocked<1>(s, "k_blocked<ppcg>", a, sb[sc], rb[rc], sb[sc ^ 1], rb[rc ^ 1], chunk->u,
                                      chunk->u, nullptr, nullptr, chunk->kx, chunk->ky, done());
                    sc ^= 1;
                    rc ^= 1;
                    if (last)
                        TL_LAUNCH(s, "k_norm2_fin", (k_norm2_fin<<<gi, BX, 0, s->stream>>>(s->g, rb[rc], s->rs,
                                                                                            done(), fin_n)));
                }
                return;
            }
            for (int pp = 0; pp < ni; ++pp) {
                const bool last = pp == ni - 1;
                if (pp == 0 && last)
                    TL_LAUNCH(s, "k_ppcg_step", (k_ppcg_step<1, true><<<gh, BX, 0, s->stream>>>(
                                  s->g, fc, chunk->theta, coef, 0, sb[sc], sb[sc ^ 1], rb[rc], rb[rc ^ 1], chunk->u,
                                  chunk->kx, chunk->ky, s->rs, done(), fin_n)));
                else if (pp == 0)
                    TL_LAUNCH(s, "k_ppcg_step", (k_ppcg_step<1, false><<<gh, BX, 0, s->stream>>>(
                                  s->g, fc, chunk->theta, coef, 0, sb[sc], sb[sc ^ 1], rb[rc], rb[rc ^ 1], chunk->u,
                                  chunk->kx, chunk->ky, s->rs, done(), tl::NoFinish())));
                else if (last)
                    TL_LAUNCH(s, "k_ppcg_step", (k_ppcg_step<2, true><<<gh, BX, 0, s->stream>>>(
                                  s->g, fc, chunk->theta, coef, pp - 1, sb[sc], sb[sc ^ 1], rb[rc], rb[rc ^ 1],
                                  chunk->u, chunk->kx, chunk->ky, s->rs, done(), fin_n)));
                else
                    TL_LAUNCH(s, "k_ppcg_step", (k_ppcg_step<2, false><<<gh, BX, 0, s->stream>>>(
                                  s->g, fc, chunk->theta, coef, pp - 1, sb[sc], sb[sc ^ 1], rb[rc], rb[rc ^ 1],
                                  chunk->u, chunk->kx, chunk->ky, s->rs, done(), tl::NoFinish())));
                sc ^= 1;
                rc ^= 1;
            }
        };
        st = loop(tt, trip);
        const int outer = st.nch;               // PPCG trips run
        const int pflips = std::max(0, outer - 1);
        const int rflips = outer * inner_flips;
        if (pb[pflips & 1] != chunk->p) swap_alt(s, chunk, ALT_P);
        if (rb[rflips & 1] != chunk->r) swap_alt(s, chunk, ALT_R);
        if (sb[rflips & 1] != chunk->sd) swap_alt(s, chunk, ALT_SD);
        // close: the last sd update of the last inner step, the last p update
        // and the halo of p (the halo of u is not refreshed during PPCG).
        if (outer > 0) {
            TL_LAUNCH(s, "k_ppcg_inner_b",
                      k_ppcg_inner_b<<<gi, BX, 0, s->stream>>>(s->g, chunk->cheby_alphas[ni - 1],
                                                               chunk->cheby_betas[ni - 1], chunk->sd, chunk->r));
            TL_LAUNCH(s, "k_cg_close", (k_cg_close<<<gi, BX, 0, s->stream>>>(s->g, fc, beta, 1, chunk->p, chunk->r,
                                                                               nullptr)));
        }
        TL_CUDA(cudaStreamSynchronize(s->stream));
        if (stats) stats->ppcg_iters = outer;
        return st;
    }
};

// solve_finished_driver (2d/drivers/solve_finished_driver.c:7-43)
void solve_finished(Run& R, TlStepStats* st_out)
{
    TlSuite2D* s = R.s;
    Chunk* chunk = R.chunk;
    Settings* settings = R.settings;
    bool* flags = settings->fields_to_exchange;
    flush(s, chunk);
    if (settings->check_result) {
        TL_LAUNCH(s, "k_residual", k_residual<<<R.gi, BX, 0, s->stream>>>(s->g, chunk->u, chunk->u0, chunk->r,
                                                                            chunk->kx, chunk->ky));
        st_out->exact_error = R.norm(chunk->r);
    }
    TL_LAUNCH(s, "k_finalise", k_finalise<<<R.gi, BX, 0, s->stream>>>(s->g, chunk->energy, chunk->density, chunk->u));
    flags[TL_FIELD_ENERGY1] = true;
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = flags[f] ? 1 : 0;
    flush(s, chunk);
    TL_CUDA(cudaStreamSynchronize(s->stream));
}

// jacobi_driver (2d/drivers/jacobi_driver.c:7-83), driven from the host
// through the suite's own kernel-interface entry points (Jacobi is not a
// performance path; its stop test needs a host round trip every trip).
double jacobi_loop(Chunk* chunk, Settings* settings, double rx, double ry, int* iters)
{
    bool* flags = settings->fields_to_exchange;
    run_jacobi_init(chunk, settings, rx, ry);
    run_copy_u(chunk, settings);
    for (int f = 0; f < TL_NUM_FIELDS; ++f) flags[f] = false;
    flags[TL_FIELD_U] = true;
    double error = 1e10;
    int tt;
    for (tt = 0; tt < settings->max_iters && !tl::failed(); ++tt) {
        run_jacobi_iterate(chunk, settings, &error);
        if (tt % 50 == 0) {
            run_local_halos(chunk, settings, 1);
            run_calculate_residual(chunk, settings);
            run_calculate_2norm(chunk, settings, chunk->r, &error);
        }
        run_local_halos(chunk, settings, 1);
        if (fabs(error) < settings->eps) break;
    }
    *iters = tt;
    return error;
}

}  // namespace

extern "C" {

void tl2d_solve_step(Chunk* chunk, Settings* settings, int tt, TlStepStats* stats)
{
    if (tl::failed()) return;
    TlSuite2D* s = suite_of(chunk);
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
    if (!(fc.l && fc.r && fc.b && fc.t)) {   // no remote halo exchange inside the device loop
        tl::fail(34, "the device-resident driver solves a chunk whose four faces are external (a decomposed mesh "
                     "runs through run_*)");
        return;
    }
    flush(s, chunk);
    TlStepStats local{};
    TlStepStats* st_out = stats ? stats : &local;
    *st_out = TlStepStats{};
    Run R{s, chunk, settings, {}, faces_of(chunk), interior_grid(s->g), fused_grid(s->g), {}};
    R.prm.eps = settings->eps;
    R.prm.eps_lim = settings->eps_lim;
    R.prm.max_iters = settings->max_iters;
    R.prm.presteps = settings->presteps;
    R.prm.error_switch = settings->error_switch ? 1 : 0;
    R.prm.switch_enabled = (settings->solver == TL_CHEBY_SOLVER || settings->solver == TL_PPCG_SOLVER) ? 1 : 0;
    R.prm.dims3 = 0;
    bool* flags = settings->fields_to_exchange;

    // solve(): dt, rx, ry (2d/diffuse.c:28-35)
    const double dt = chunk->dt_init < settings->dt_init ? chunk->dt_init : settings->dt_init;
    const double rx = dt / (settings->dx * settings->dx);
    const double ry = dt / (settings->dy * settings->dy);
    // halo of energy and density, depth 2 (2d/diffuse.c:38-41)
    int h2[TL_NUM_FIELDS] = {0};
    h2[TL_FIELD_ENERGY1] = h2[TL_FIELD_DENSITY] = 2;
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = h2[f];
    flush(s, chunk);

    double error = 1e10;
    DevState st{};
    if (settings->solver == TL_JACOBI_SOLVER) {
        int it = 0;
        error = jacobi_loop(chunk, settings, rx, ry, &it);
        st_out->jacobi_iters = it;
        st_out->total_iters = it;
        st_out->error = error;
        solve_finished(R, st_out);
        if (print_and_log && settings->tea_out_fp) print_and_log(settings, "Jacobi: \t\t%d iterations\n", it);
        return;
    }
    // cg_init_driver: cg_init, halo(u, p) depth 1, copy_u (2d/drivers/cg_driver.c:30-62)
    if (settings->coefficient != TL_CONDUCTIVITY && settings->coefficient != TL_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return;
    }
    TL_LAUNCH(s, "k_cg_init", k_cg_init<<<full_grid(s->g), FB, 0, s->stream>>>(
                                  s->g, settings->coefficient, rx, ry, chunk->density, chunk->energy, chunk->u,
                                  chunk->p, s->alt[ALT_P], chunk->r, chunk->w, chunk->kx, chunk->ky, s->rs,
                                  FinCgInit{s->d_state, s->d_mirror}));
    int h1[TL_NUM_FIELDS] = {0};
    h1[TL_FIELD_U] = h1[TL_FIELD_P] = 1;
    for (int f = 0; f < TL_NUM_FIELDS; ++f) s->pend.halo[f] = h1[f];
    flush(s, chunk);
    TL_LAUNCH(s, "k_copy_u", k_copy_u<<<R.gi, BX, 0, s->stream>>>(s->g, chunk->u0, chunk->u));
    R.read_state();

    if (settings->solver == TL_CG_SOLVER && s->precond == kPrecondDiag) st = R.pcg_phase<1>();
    else if (settings->solver == TL_CG_SOLVER && s->precond == kPrecondBlock) st = R.pcg_phase<4>();
    else st = R.cg_phase(0, true);
    error = st.error;
    if (st.reason == 2 && settings->solver == TL_CHEBY_SOLVER) {
        const int tt_sw = st.trip;
        st = R.cheby_phase(tt_sw, st_out);
        st_out->cg_iters = tt_sw;
        error = st.error;
        for (int f = 0; f < TL_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL_FIELD_U] = true;
    } else if (st.reason == 2 && settings->solver == TL_PPCG_SOLVER) {
        const int tt_sw = st.trip;
        st = R.ppcg_phase(tt_sw, st_out);
        st_out->cg_iters = tt_sw;
        error = st.error;
        for (int f = 0; f < TL_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL_FIELD_P] = true;
    } else {
        // converged or capped during CG
        st_out->cg_iters = st.reason == 1 ? st.trip - 1 : st.trip;
        for (int f = 0; f < TL_NUM_FIELDS; ++f) flags[f] = false;
        flags[TL_FIELD_U] = flags[TL_FIELD_P] = true;
    }
    if (tl::failed()) return;
    if (tma_failed(s)) {
        tl::fail(35, "a TMA row load of the w sweep did not complete (bounded barrier wait gave up)");
        return;
    }
    // the reference's printed iteration count is the loop index at exit
    const int tt_exit = st.reason == 1 ? st.trip - 1 : st.trip;
    st_out->total_iters = tt_exit;
    if (settings->solver == TL_CHEBY_SOLVER) st_out->cg_iters = tt_exit - st_out->cheby_iters + 1;
    if (settings->solver == TL_PPCG_SOLVER) st_out->cg_iters = tt_exit - st_out->ppcg_iters + 1;
    st_out->error = error;
    st_out->eigmin = chunk->eigmin;
    st_out->eigmax = chunk->eigmax;

    solve_finished(R, st_out);

    if (print_and_log && settings->tea_out_fp) {
        if (settings->solver == TL_CG_SOLVER) {
            print_and_log(settings, "CG: \t\t\t%d iterations\n", st_out->cg_iters);
        } else if (settings->solver == TL_CHEBY_SOLVER) {
            print_and_log(settings, "CG: \t\t\t%d iterations\n", st_out->cg_iters);
            print_and_log(settings, "Cheby: \t\t\t%d iterations (%d estimated)\n", st_out->cheby_iters,
                          st_out->est_iters);
        } else {
            print_and_log(settings, "CG: \t\t\t%d iterations\n", st_out->cg_iters);
            print_and_log(settings, "PPCG: \t\t\t%d iterations (%d inner iterations per)\n", st_out->ppcg_iters,
                          settings->ppcg_inner_steps);
        }
    }
    (void)tt;
}

// 2d/application.h:9-11: replaces diffuse() (2d/diffuse.c:10-19).
void diffuse_overload(Chunk* chunks, Settings* settings)
{
    if (print_and_log && settings->tea_out_fp)
        print_and_log(settings, "This implementation overloads the diffuse function.\n");
    for (int tt = 0; tt < settings->end_step && !tl::failed(); ++tt) {
        if (print_and_log && settings->tea_out_fp) print_and_log(settings, "\nTimestep %d\n", tt + 1);
        for (int cc = 0; cc < settings->num_chunks_per_rank; ++cc) tl2d_solve_step(&chunks[cc], settings, tt, nullptr);
        if (settings->summary_frequency > 0 && tt % settings->summary_frequency == 0 && field_summary_driver)
            field_summary_driver(chunks, settings, false);
    }
    if (field_summary_driver) field_summary_driver(chunks, settings, true);
}

}  // extern "C"
