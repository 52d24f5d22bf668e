// adjoint3d.cu -- hand-written adjoint of the 3D implicit timestep.
//
// The forward timestep (3d/diffuse.c:21-81 with the CG solver,
// 3d/drivers/cg_solver_driver.c) is, for density rho (constant in time) and
// energy e_n:
//
//   w = 1/rho (recip conductivity) or rho (conductivity)        cg_solver.c:9-102
//   k_f = r (w_a + w_b) / (2 w_a w_b) on the face f between cells a, b
//   A u = u + sum_f k_f (u_a - u_b)(e_a - e_b)   (7-point operator, reflective
//                                                 boundary: boundary terms vanish)
//   u0_n = e_n rho ;  A u_n = u0_n ;  e_{n+1} = u_n / rho   (so u0_{n+1} = u_n)
//
// For a functional J(u_N, rho) the Lagrangian L = J - sum_n l_n.(A u_n - u_{n-1})
// gives, with A symmetric, the adjoint recursion
//
//   A l_N = dJ/du_N ;  A l_n = l_{n+1}   (n = N-1 .. 1)
//
// solved by the forward CG sweeps (k3_cg_w, k3_cg_ur), and the gradient
//
//   dJ/drho_c = dJ/drho_c|explicit + l_1,c e_0,c
//               - sum_n sum_{f at c} (dk_f/drho_c) (l_a - l_b)(u_a - u_b),
//   dk_f/drho_c = -r / (2 w_c^2) dw_c/drho_c   (r/2 for recip conductivity).
//
// tl3d_solve_step_backward is the backward of one timestep (adjoint solve +
// face-coefficient gradient); tl3d_adjoint_gradient runs N forward timesteps,
// keeps the energy every `every` steps, and walks back segment by segment,
// recomputing the segment's forward solutions from its checkpoint. J is the
// field summary's temperature restricted to a box (3d/c_kernels/omp3/
// field_summary.c:8-49: sum of volume * density * u over cells whose centre
// lies in the box), and the result is dJ/d(log rho) = rho dJ/drho per cell.
#include "suite3d_impl.hpp"

#include <algorithm>
#include <cmath>
#include <vector>

using namespace tl3d;

namespace {

constexpr int kBatch = 16;

struct Box {   // interior index ranges [lo, hi) of the cells whose centre is in the box
    int k0, k1, j0, j1, i0, i1;
};

// J = sum_box V rho u ; g = dJ/du = V rho 1_box (zero elsewhere, halo
// included) ; grad = explicit dJ/drho = V u 1_box.
static __global__ void __launch_bounds__(FBX* FBY) k3a_objective(Geo g, Box b, const double* __restrict__ volume,
                                                                 const double* __restrict__ density,
                                                                 const double* __restrict__ u, double* __restrict__ gu,
                                                                 double* __restrict__ grad, ReduceSlots rs)
{
    const Cell c(g);
    double acc[1] = {0.0};
    if (c.in) {
        const long i = c.k + (long)c.j * g.x + (long)c.i * g.xy();
        const int kk = c.k - g.hd, jj = c.j - g.hd, ii = c.i - g.hd;
        const bool in = kk >= b.k0 && kk < b.k1 && jj >= b.j0 && jj < b.j1 && ii >= b.i0 && ii < b.i1;
        double gv = 0.0, gr = 0.0;
        if (in) {
            gv = volume[i] * density[i];
            gr = volume[i] * u[i];
            acc[0] = gv * u[i];
        }
        gu[i] = gv;
        grad[i] = gr;
    }
    tl::grid_sum<1, FBX * FBY>(acc, rs, block_id(), block_count());
}

// Start of an adjoint solve A l = rhs from l = 0: r = p = rhs, l = 0 (whole
// array); rro = rhs.rhs over the interior.
template <typename Finish>
static __global__ void __launch_bounds__(FBX* FBY) k3a_prep(Geo g, const double* __restrict__ rhs, double* __restrict__ r,
                                                            double* __restrict__ p, double* __restrict__ lam,
                                                            ReduceSlots rs, Finish fin)
{
    const Cell c(g);
    double acc[1] = {0.0};
    if (c.in) {
        const long i = c.k + (long)c.j * g.x + (long)c.i * g.xy();
        const bool interior = c.k >= g.hd && c.k < g.x - g.hd && c.j >= g.hd && c.j < g.y - g.hd &&
                              c.i >= g.hd && c.i < g.z - g.hd;
        const double v = interior ? rhs[i] : 0.0;
        r[i] = v;
        p[i] = v;
        lam[i] = 0.0;
        acc[0] = v * v;
    }
    tl::grid_sum<1, FBX * FBY>(acc, rs, block_id(), block_count(), fin);
}

// grad_c -= dk/drho_c * sum over interior neighbours of r_axis (l_c - l_nb)(u_c - u_nb)
static __global__ void __launch_bounds__(FBX* FBY) k3a_face_grad(Geo g, int coefficient, double rx, double ry,
                                                                 double rz, const double* __restrict__ density,
                                                                 const double* __restrict__ lam,
                                                                 const double* __restrict__ u,
                                                                 double* __restrict__ grad)
{
    const Cell c(g);
    if (!c.in) return;
    const int hd = g.hd;
    if (c.k < hd || c.k >= g.x - hd || c.j < hd || c.j >= g.y - hd || c.i < hd || c.i >= g.z - hd) return;
    const long x = g.x, xy = g.xy();
    const long i = c.k + (long)c.j * x + (long)c.i * xy;
    const double rho = density[i];
    const double w = coef_w(coefficient, rho);
    const double dwdrho = coefficient == TL3_CONDUCTIVITY ? 1.0 : -w * w;
    const double dk = -dwdrho / (2.0 * w * w);
    const double lc = lam[i], uc = u[i];
    auto term = [&](long j) { return (lc - lam[j]) * (uc - u[j]); };
    double sx = 0.0, sy = 0.0, sz = 0.0;
    if (c.k > hd) sx += term(i - 1);
    if (c.k < g.x - hd - 1) sx += term(i + 1);
    if (c.j > hd) sy += term(i - x);
    if (c.j < g.y - hd - 1) sy += term(i + x);
    if (c.i > hd) sz += term(i - xy);
    if (c.i < g.z - hd - 1) sz += term(i + xy);
    grad[i] -= dk * (rx * sx + ry * sy + rz * sz);
}

// out[interior, x fastest] = rho (grad + l_1 e_0)
static __global__ void __launch_bounds__(FBX* FBY) k3a_finish(Geo g, const double* __restrict__ density,
                                                              const double* __restrict__ grad,
                                                              const double* __restrict__ lam1,
                                                              const double* __restrict__ e0, double* __restrict__ out)
{
    const Cell c(g);
    if (!c.in) return;
    const int hd = g.hd;
    if (c.k < hd || c.k >= g.x - hd || c.j < hd || c.j >= g.y - hd || c.i < hd || c.i >= g.z - hd) return;
    const long i = c.k + (long)c.j * g.x + (long)c.i * g.xy();
    const long nx = g.x - 2 * hd, ny = g.y - 2 * hd;
    const long o = (c.k - hd) + (c.j - hd) * nx + (c.i - hd) * nx * ny;
    out[o] = density[i] * (grad[i] + lam1[i] * e0[i]);
}

template <typename F>
void batched(TlSuite3D* s, int max_trips, F&& launch_trip)
{
    cudaEvent_t ev[2];
    cudaEventCreateWithFlags(&ev[0], cudaEventDisableTiming);
    cudaEventCreateWithFlags(&ev[1], cudaEventDisableTiming);
    int t = 0, batch = 0;
    bool pending_prev = false;
    while (t < max_trips && !tl::failed()) {
        const int end = std::min(max_trips, t + kBatch);
        for (; t < end; ++t) launch_trip(t);
        cudaEventRecord(ev[batch & 1], s->stream);
        if (pending_prev) {
            cudaEventSynchronize(ev[(batch + 1) & 1]);
            if (*(volatile int*)&s->h_mirror[0]) break;
        }
        pending_prev = true;
        ++batch;
    }
    cudaStreamSynchronize(s->stream);
    cudaEventDestroy(ev[0]);
    cudaEventDestroy(ev[1]);
}

size_t field_bytes(const TlSuite3D* s) { return sizeof(double) * (size_t)(s->g.xy() * s->g.z); }

void copy_field(TlSuite3D* s, double* dst, const double* src)
{
    TL_CUDA(cudaMemcpyAsync(dst, src, field_bytes(s), cudaMemcpyDeviceToDevice, s->stream));
}

// CG solve A lam = rhs from lam = 0 to r.r <= rel_tol^2 rhs.rhs with the
// forward sweeps; clobbers the chunk's p, r, w. Returns the iterations.
int adjoint_solve(TlSuite3D* s, Chunk* chunk, const double* rhs, double* lam, double rel_tol, int max_iters)
{
    const Faces fc = faces_of(chunk);
    const dim3 gi = interior_grid(s->g), gh = fused_grid(s->g), bl = interior_block();
    s->h_mirror[0] = 0;
    TL3_LAUNCH(s, "k3a_prep", (k3a_prep<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                                  s->g, rhs, chunk->vec_r, chunk->vec_p, lam, s->rs,
                                  tl::FinCgInit{s->d_state, s->d_mirror})));
    double gg = 0.0;
    if (!fetch(s, 1, &gg)) return 0;
    if (gg == 0.0) return 0;
    for (int f = 0; f < TL3_NUM_FIELDS; ++f) s->pend.halo[f] = 0;
    s->pend.halo[TL3_FIELD_P] = 1;
    flush(s, chunk);
    DevParams prm{};
    prm.eps = rel_tol * rel_tol * gg;
    prm.max_iters = max_iters;
    double* buf[2] = {chunk->vec_p, s->alt[ALT3_P]};
    tl::FinCgW fin_w{s->d_state, s->d_cg_alphas};
    tl::FinCgUr fin_ur{s->d_state, s->d_cg_betas, prm, s->d_mirror};
    const Scalar beta{0.0, &s->d_state->beta}, alpha{0.0, &s->d_state->alpha};
    const int* done = &s->d_state->done;
    int cur = 0;
    batched(s, max_iters, [&](int t) {
        if (t == 0) {
            launch_cg_w3<false, false>(s, chunk, gh, fc, beta, buf[cur], buf[cur], chunk->vec_r, chunk->vec_w,
                                       nullptr, 0, done, fin_w);
        } else {
            launch_cg_w3<true, true>(s, chunk, gh, fc, beta, buf[cur], buf[cur ^ 1], chunk->vec_r, chunk->vec_w,
                                     nullptr, 0, done, fin_w);
            cur ^= 1;
        }
        launch_cg_ur3(s, gi, alpha, lam, buf[cur], chunk->vec_r, chunk->vec_w, done, fin_ur);
    });
    DevState st{};
    TL_CUDA(cudaMemcpy(&st, s->d_state, sizeof(DevState), cudaMemcpyDeviceToHost));
    const int flips = std::max(0, st.trip - 1);
    if (buf[flips & 1] != chunk->vec_p) swap_alt(s, chunk, ALT3_P);
    return st.trip;
}

void face_grad(TlSuite3D* s, Chunk* chunk, Settings* settings, const double* lam, const double* u, double* grad)
{
    const double dt = chunk->dt_init < settings->dt_init ? chunk->dt_init : settings->dt_init;
    const double rx = dt / (settings->dx * settings->dx);
    const double ry = dt / (settings->dy * settings->dy);
    const double rz = dt / (settings->dz * settings->dz);
    TL3_LAUNCH(s, "k3a_face_grad", k3a_face_grad<<<full_grid(s->g), full_block(), 0, s->stream>>>(
                                       s->g, settings->coefficient, rx, ry, rz, chunk->density, lam, u, grad));
}

bool check_chunk(TlSuite3D* s, Chunk* chunk, Settings* settings)
{
    if (!s) return false;
    const Faces fc = faces_of(chunk);
    if (settings->num_chunks_per_rank != 1 || !(fc.l && fc.r && fc.b && fc.t && fc.k && fc.f)) {
        tl::fail(52, "the adjoint needs one chunk with six external faces");
        return false;
    }
    if (settings->solver != TL3_CG_SOLVER) {
        tl::fail(53, "the adjoint differentiates the CG timestep (solver %d given)", settings->solver);
        return false;
    }
    if (settings->coefficient != TL3_CONDUCTIVITY && settings->coefficient != TL3_RECIP_CONDUCTIVITY) {
        tl::fail(7, "Coefficient %d is not valid.", settings->coefficient);
        return false;
    }
    return true;
}

}  // namespace

extern "C" int tl3d_solve_step_backward(Chunk* chunk, Settings* settings, const double* g_u, const double* u,
                                        double* lam, double* grad, double rel_tol, int* iterations)
{
    if (tl::failed()) return tl::error_state().code;
    TlSuite3D* s = suite_of(chunk);
    if (!check_chunk(s, chunk, settings)) return tl::error_state().code;
    if (!g_u || !u || !lam || !grad || !(rel_tol > 0.0)) {
        tl::fail(51, "tl3d_solve_step_backward: null field or non-positive rel_tol");
        return 51;
    }
    flush(s, chunk);
    const int it = adjoint_solve(s, chunk, g_u, lam, rel_tol, settings->max_iters);
    face_grad(s, chunk, settings, lam, u, grad);
    TL_CUDA(cudaStreamSynchronize(s->stream));
    if (iterations) *iterations = it;
    return tl::failed() ? tl::error_state().code : 0;
}

extern "C" int tl3d_adjoint_gradient(Chunk* chunk, Settings* settings, int steps, int every, const double* box,
                                     double rel_tol, double* dj_dlogrho, TlAdjointStats* stats)
{
    if (tl::failed()) return tl::error_state().code;
    TlSuite3D* s = suite_of(chunk);
    if (!check_chunk(s, chunk, settings)) return tl::error_state().code;
    if (steps < 1 || every < 1 || !box || !dj_dlogrho || !(rel_tol > 0.0)) {
        tl::fail(51, "tl3d_adjoint_gradient: steps >= 1, every >= 1, box, output and rel_tol > 0 are required");
        return 51;
    }
    TlAdjointStats local{};
    TlAdjointStats* out = stats ? stats : &local;
    *out = TlAdjointStats{};
    flush(s, chunk);
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, s->stream);

    // box -> interior index ranges (cell centre in [lo, hi] per axis)
    const Geo g = s->g;
    const int nx = g.x - 2 * g.hd, ny = g.y - 2 * g.hd, nz = g.z - 2 * g.hd;
    auto range = [](double lo, double hi, double mn, double d, int n, int& a, int& b) {
        a = n;
        b = 0;
        for (int c = 0; c < n; ++c) {
            const double x = mn + d * (c + 0.5);
            if (x >= lo && x <= hi) {
                a = std::min(a, c);
                b = std::max(b, c + 1);
            }
        }
        if (a >= b) a = b = 0;
    };
    Box bx{};
    range(box[0], box[1], settings->grid_x_min, settings->dx, nx, bx.k0, bx.k1);
    range(box[2], box[3], settings->grid_y_min, settings->dy, ny, bx.j0, bx.j1);
    range(box[4], box[5], settings->grid_z_min, settings->dz, nz, bx.i0, bx.i1);

    // device storage: segment checkpoints of energy, the segment's solutions,
    // the adjoint field, its right-hand side, the gradient, the final energy
    const int nseg = (steps + every - 1) / every;
    const size_t fb = (field_bytes(s) + 255) & ~(size_t)255;
    const int nfields = nseg + every + 4;
    char* slab = nullptr;
    if (!TL_CUDA(cudaMalloc(&slab, fb * (size_t)nfields))) return tl::error_state().code;
    auto fld = [&](int k) { return (double*)(slab + fb * (size_t)k); };
    double* ckpt0 = fld(0);                  // energy at steps 0, every, 2 every, ...
    double* useg0 = fld(nseg);               // u_n of the current segment
    double* lam = fld(nseg + every);
    double* rhs = fld(nseg + every + 1);
    double* grad = fld(nseg + every + 2);
    double* efinal = fld(nseg + every + 3);
    auto ckpt = [&](int sgi) { return ckpt0 + (fb / sizeof(double)) * (size_t)sgi; };
    auto useg = [&](int k) { return useg0 + (fb / sizeof(double)) * (size_t)k; };

    TlStepStats3 st3{};
    auto forward = [&](int n) {   // timestep n (1-based)
        tl3d_solve_step(chunk, settings, n - 1, &st3);
        out->forward_steps += 1;
        out->forward_iters += st3.total_iters;
    };

    // 1. forward run with checkpoints; the last segment's solutions are kept
    const int last_start = (nseg - 1) * every;
    for (int n = 1; n <= steps && !tl::failed(); ++n) {
        if ((n - 1) % every == 0) copy_field(s, ckpt((n - 1) / every), chunk->energy);
        forward(n);
        if (n > last_start) copy_field(s, useg(n - last_start - 1), chunk->vec_u);
    }
    out->checkpoints = nseg;
    copy_field(s, efinal, chunk->energy);

    // 2. objective and the adjoint's starting right-hand side
    TL3_LAUNCH(s, "k3a_objective", k3a_objective<<<full_grid(g), full_block(), 0, s->stream>>>(
                                       g, bx, chunk->volume, chunk->density, useg(steps - last_start - 1), rhs, grad,
                                       s->rs));
    double J = 0.0;
    fetch(s, 1, &J);
    out->J = J;

    // 3. backward, segment by segment
    for (int sgi = nseg - 1; sgi >= 0 && !tl::failed(); --sgi) {
        const int start = sgi * every, end = std::min(steps, start + every);
        if (sgi != nseg - 1) {
            copy_field(s, chunk->energy, ckpt(sgi));
            for (int n = start + 1; n <= end && !tl::failed(); ++n) {
                forward(n);
                copy_field(s, useg(n - start - 1), chunk->vec_u);
            }
        }
        for (int n = end; n > start && !tl::failed(); --n) {
            out->adjoint_iters += adjoint_solve(s, chunk, rhs, lam, rel_tol, settings->max_iters);
            face_grad(s, chunk, settings, lam, useg(n - start - 1), grad);
            if (n > 1) copy_field(s, rhs, lam);
        }
    }

    // 4. dJ/dlog rho = rho (grad + l_1 e_0); restore the final state
    double* dout = rhs;   // reuse: interior values, x fastest
    TL3_LAUNCH(s, "k3a_finish", k3a_finish<<<full_grid(g), full_block(), 0, s->stream>>>(g, chunk->density, grad, lam,
                                                                                        ckpt(0), dout));
    TL_CUDA(cudaMemcpyAsync(dj_dlogrho, dout, sizeof(double) * (size_t)nx * ny * nz, cudaMemcpyDeviceToHost,
                            s->stream));
    copy_field(s, chunk->energy, efinal);
    cudaEventRecord(e1, s->stream);
    TL_CUDA(cudaStreamSynchronize(s->stream));
    float ms = 0.f;
    cudaEventElapsedTime(&ms, e0, e1);
    out->device_ms = ms;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(slab);
    if (tma_failed(s)) tl::fail(35, "a TMA plane load of the w sweep did not complete (bounded barrier wait gave up)");
    return tl::failed() ? tl::error_state().code : 0;
}
