/*
 * tealeaf_b200_3d.h -- C ABI of the B200 (sm_100a) TeaLeaf 3D kernel suite.
 *
 * libtealeaf_b200_3d.so is a drop-in kernel suite for the unchanged TeaLeaf
 * 3D host (main.c, diffuse.c, drivers/, chunk.c built with -DNO_MPI). It
 * exports the 21 functions of the reference 3D kernel interface with the same
 * names, argument meaning and accumulate/synchronous result semantics
 * (3d/kernel_interface.h:9-65), and the entry points marked "new" below.
 *
 * The Chunk / Settings / State structs restate the reference layouts field
 * for field (3d/chunk.h:7-102, 3d/settings.h:63-126, 3d/settings.h:137-150);
 * a test compares every offset against the reference headers. The host
 * includes the suite's chunk_extension_t from build/chunk_extension.h
 * (3d/chunk.h:5, copied by 3d/Makefile:38): one opaque pointer. 3D fields are
 * plain double* device pointers the host never dereferences.
 *
 * Results are ACCUMULATED (*out += value) and valid on return, except
 * run_jacobi_solver_iterate, which assigns (3d jacobi_solver.c). Errors
 * print and exit(1) like the reference die(), unless
 * tl3d_set_error_mode(TL_ERRMODE_RECORD) was called.
 */
#ifndef TEALEAF_B200_3D_H
#define TEALEAF_B200_3D_H

#include <stdbool.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- suite-owned extension point (same text as suite/3d/chunk_extension.h) */
#ifndef TL_B200_CHUNK_EXTENSION_3D
#define TL_B200_CHUNK_EXTENSION_3D
struct TlSuite3D;
typedef struct chunk_extension_t
{
    struct TlSuite3D* suite;
} chunk_extension_t;
#endif

/* ---- constants shared with the host (3d/shared.h:21-44) ------------------ */
#define TL3_NUM_FIELDS 6
#define TL3_CHUNK_LEFT 0
#define TL3_CHUNK_RIGHT 1
#define TL3_CHUNK_BOTTOM 2
#define TL3_CHUNK_TOP 3
#define TL3_CHUNK_BACK 4
#define TL3_CHUNK_FRONT 5
#define TL3_EXTERNAL_FACE (-1)
#define TL3_FIELD_DENSITY 0
#define TL3_FIELD_ENERGY0 1
#define TL3_FIELD_ENERGY1 2
#define TL3_FIELD_U 3
#define TL3_FIELD_P 4
#define TL3_FIELD_SD 5
#define TL3_CONDUCTIVITY 1
#define TL3_RECIP_CONDUCTIVITY 2
/* solver_e (3d/settings.h:47-53), geometry_e (3d/settings.h:129-134) */
#define TL3_JACOBI_SOLVER 0
#define TL3_CG_SOLVER 1
#define TL3_CHEBY_SOLVER 2
#define TL3_PPCG_SOLVER 3
#define TL3_GEOM_CUBOID 0
#define TL3_GEOM_SPHERICAL 1
#define TL3_GEOM_POINT 2

struct profile;

/* 3d/settings.h:63-126 */
typedef struct Settings
{
    struct profile* kernel_profile;
    struct profile* application_profile;
    struct profile* wallclock_profile;
    FILE* tea_out_fp;
    int rank;
    int end_step;
    int presteps;
    int max_iters;
    int coefficient;
    int ppcg_inner_steps;
    int summary_frequency;
    int halo_depth;
    int num_states;
    int num_chunks;
    int num_chunks_per_rank;
    int num_ranks;
    bool* fields_to_exchange;   /* host bool[TL3_NUM_FIELDS] */
    bool is_offload;
    bool error_switch;
    bool check_result;
    bool preconditioner;
    double eps;
    double dt_init;
    double end_time;
    double eps_lim;
    char* tea_in_filename;
    char* tea_out_filename;
    char* test_problem_filename;
    int solver;                 /* solver_e */
    int kernel_language;        /* kernel_language_e */
    int grid_x_cells;
    int grid_y_cells;
    int grid_z_cells;
    double grid_x_min;
    double grid_y_min;
    double grid_z_min;
    double grid_x_max;
    double grid_y_max;
    double grid_z_max;
    double dx;
    double dy;
    double dz;
} Settings;

/* 3d/settings.h:137-150 */
typedef struct State
{
    bool defined;
    double density;
    double energy;
    double x_min;
    double y_min;
    double z_min;
    double x_max;
    double y_max;
    double z_max;
    double radius;
    int geometry;               /* geometry_e */
} State;

/* 3d/chunk.h:7-102 */
typedef struct Chunk
{
    double dt_init;
    int* neighbours;            /* host int[6] */
    double* left_send;
    double* left_recv;
    double* right_send;
    double* right_recv;
    double* top_send;
    double* top_recv;
    double* bottom_send;
    double* bottom_recv;
    double* front_send;
    double* front_recv;
    double* back_send;
    double* back_recv;
    int lr_page;
    int tb_page;
    int fb_page;
    int left;
    int right;
    int bottom;
    int top;
    int back;
    int front;
    int x;                      /* cells incl. halo */
    int y;
    int z;
    double* density0;
    double* density;
    double* energy0;
    double* energy;
    double* vec_u;
    double* vec_u0;
    double* vec_p;
    double* vec_r;
    double* vec_mi;
    double* vec_w;
    double* vec_kx;
    double* vec_ky;
    double* vec_kz;
    double* vec_sd;
    double* vec_z;
    double* cell_x;
    double* cell_y;
    double* cell_z;
    double* cell_dx;
    double* cell_dy;
    double* cell_dz;
    double* vertex_dx;
    double* vertex_dy;
    double* vertex_dz;
    double* vertex_x;
    double* vertex_y;
    double* vertex_z;
    double* volume;
    double* x_area;
    double* y_area;
    double* z_area;
    double theta;
    double eigmin;
    double eigmax;
    double* cg_alphas;          /* host arrays of max_iters */
    double* cg_betas;
    double* cheby_alphas;
    double* cheby_betas;
    struct chunk_extension_t* ext;
} Chunk;

/* ---- reference kernel interface (3d/kernel_interface.h:9-65) ------------- */
void run_set_chunk_data(Chunk* chunk, Settings* settings);                      /* :9 */
void run_set_chunk_state(Chunk* chunk, Settings* settings, State* states);      /* :11 */
void run_kernel_initialise(Chunk* chunk, Settings* settings);                   /* :13 */
void run_local_halos(Chunk* chunk, Settings* settings, int depth);              /* :17 */
void run_pack_or_unpack(Chunk* chunk, Settings* settings, int depth,            /* :19 */
        int face, bool pack, double* field, double* buffer);
void run_store_energy(Chunk* chunk, Settings* settings);                        /* :22 */
void run_field_summary(Chunk* chunk, Settings* settings,                        /* :24 */
        double* vol, double* mass, double* ie, double* temp);
void run_cg_solver_init(Chunk* chunk, Settings* settings,                       /* :29 */
        double rx, double ry, double rz, double* rro);
void run_cg_solver_calc_w(Chunk* chunk, Settings* settings, double* pw);        /* :32 */
void run_cg_solver_calc_ur(Chunk* chunk, Settings* settings,                    /* :34 */
        double alpha, double* rrn);
void run_cg_solver_calc_p(Chunk* chunk, Settings* settings, double beta);       /* :36 */
void run_cheby_solver_init(Chunk* chunk, Settings* settings);                   /* :40 */
void run_cheby_solver_iterate(Chunk* chunk, Settings* settings,                 /* :42 */
        double alpha, double beta);
void run_jacobi_solver_init(Chunk* chunk, Settings* settings,                   /* :46 */
        double rx, double ry, double rz);
void run_jacobi_solver_iterate(Chunk* chunk, Settings* settings, double* error);/* :48 */
void run_ppcg_init(Chunk* chunk, Settings* settings);                           /* :52 */
void run_ppcg_inner_iteration(Chunk* chunk, Settings* settings,                 /* :54 */
        double alpha, double beta);
void run_solver_copy_u(Chunk* chunk, Settings* settings);                       /* :58 */
void run_calculate_residual(Chunk* chunk, Settings* settings);                  /* :60 */
void run_calculate_2norm(Chunk* chunk, Settings* settings,                      /* :62 */
        double* buffer, double* norm);
void run_solver_finalise(Chunk* chunk, Settings* settings);                     /* :64 */

/* ---- new entry points (no reference counterpart) ------------------------- */
/* Frees what run_kernel_initialise allocated (the 3D interface has no finalise). */
void run_kernel_finalise(Chunk* chunk, Settings* settings);

#define TL3_ERRMODE_EXIT 0
#define TL3_ERRMODE_RECORD 1
void tl3d_set_error_mode(int mode);
int tl3d_get_error(char* msg, int msg_len);
void tl3d_set_device(int device);
void* tl3d_stream(Chunk* chunk);
void tl3d_profile_enable(Chunk* chunk, int on);
void tl3d_profile_reset(Chunk* chunk);
int tl3d_profile_read(Chunk* chunk, int index, char* name, int name_len,
        long long* calls, double* ms);
/* Kernel launches issued for this chunk since initialisation (counted
 * whether or not the profile is enabled); -1 for an unknown chunk. */
long long tl3d_launch_count(Chunk* chunk);
/* No counterpart in the reference. Feed the CG w sweep's operand planes by
 * TMA tile loads (1, the default, where the halo depth and row length are
 * even; results are bit-identical) or by per-thread asynchronous copies (0). */
void tl3d_set_tma(Chunk* chunk, int on);
/* No counterpart in the reference. Run Chebyshev trips and PPCG inner steps
 * temporally blocked in shared memory (1, the default; results are
 * bit-identical; used when all six faces are external) or one launch per
 * trip / step (0): in the device-resident driver, and through
 * run_cheby_solver_iterate / run_ppcg_inner_iteration, whose calls in the
 * reference drivers' pattern are deferred and run blocked when another
 * run_* call needs the device state. */
void tl3d_set_temporal_blocking(Chunk* chunk, int on);
/* No counterpart in the reference. Runs every operation the suite has
 * deferred for this chunk (a CG p update, halo updates, queued Chebyshev
 * trips or PPCG inner steps), as every run_* call
 * that touches device data does first; call it before reading the chunk's
 * device fields by other means. Asynchronous on the chunk's stream. */
void tl3d_flush(Chunk* chunk);

/* Field ids for the host-buffer staging calls (x*y*z values each). */
#define TL3D_DENSITY0 0
#define TL3D_DENSITY 1
#define TL3D_ENERGY0 2
#define TL3D_ENERGY 3
#define TL3D_U 4
#define TL3D_U0 5
#define TL3D_P 6
#define TL3D_R 7
#define TL3D_MI 8
#define TL3D_W 9
#define TL3D_KX 10
#define TL3D_KY 11
#define TL3D_SD 12
#define TL3D_VOLUME 13
#define TL3D_KZ 14
void tl3d_upload_field(Chunk* chunk, Settings* settings, int field_id,
        const double* host, long long count);
void tl3d_download_field(Chunk* chunk, Settings* settings, int field_id,
        double* host, long long count);

/* Per-timestep statistics of the device-resident driver (same layout as 2D). */
typedef struct TlStepStats3
{
    int cg_iters;
    int cheby_iters;
    int ppcg_iters;
    int jacobi_iters;
    int est_iters;
    int total_iters;
    double error;
    double eigmin;
    double eigmax;
    double exact_error;
} TlStepStats3;

/* The four field-summary totals from a parallel tree reduction: one sweep at
 * full bandwidth instead of run_field_summary's serial reference order, so
 * the last bits differ from the reference (accumulated like run_field_summary). */
void tl3d_field_summary_fast(Chunk* chunk, Settings* settings,
        double* vol, double* mass, double* ie, double* temp);

/* One timestep of solve() (3d/diffuse.c:21-81) on the device-resident path.
 * The chunk must be undivided (six external faces: the loop holds no remote
 * halo exchange); a chunk with a neighbour reports error 34. */
void tl3d_solve_step(Chunk* chunk, Settings* settings, int tt, TlStepStats3* stats);

/* Adjoint of the implicit CG timestep: no counterpart in the reference.
 * Backward of one timestep u = A(rho)^-1 u0: solves A lam = g_u with the
 * forward CG sweeps (A is symmetric) to lam-residual <= rel_tol * ||g_u||, then
 * accumulates into grad (dJ/drho) the face-coefficient term
 * -sum_f dk_f/drho_c (lam_a - lam_b)(u_a - u_b). g_u, u (this step's forward
 * solution), lam and grad are device arrays in the chunk layout. The chunk's
 * p, r and w are overwritten. One chunk, six external faces, CG solver.
 * Returns 0, or an error code (message from tl3d_get_error). */
int tl3d_solve_step_backward(Chunk* chunk, Settings* settings, const double* g_u, const double* u,
        double* lam, double* grad, double rel_tol, int* iterations);

/* Statistics of tl3d_adjoint_gradient. */
typedef struct TlAdjointStats
{
    double J;               /* the functional at the final step */
    double device_ms;       /* device time of the whole call */
    int forward_steps;      /* timesteps run forward, recomputation included */
    int forward_iters;      /* CG iterations of those timesteps */
    int adjoint_iters;      /* CG iterations of the adjoint solves */
    int checkpoints;        /* energy checkpoints kept */
} TlAdjointStats;

/* Gradient of J = sum over the cells whose centre lies in the box
 * {box[0] <= x <= box[1], box[2] <= y <= box[3], box[4] <= z <= box[5]} of
 * volume * density * u after `steps` timesteps (the field summary's
 * temperature restricted to the box), with respect to log(density) of every
 * interior cell. Runs the timesteps forward from the chunk's current state
 * (tl3d_solve_step, settings->eps as the forward stop), keeps the energy
 * every `every` steps, then walks back segment by segment, recomputing each
 * segment's forward solutions from its checkpoint, with the adjoint solves
 * stopped at rel_tol. dj_dlogrho: host array of nx*ny*nz values, x fastest.
 * The chunk ends in its state after the forward steps. */
int tl3d_adjoint_gradient(Chunk* chunk, Settings* settings, int steps, int every, const double* box,
        double rel_tol, double* dj_dlogrho, TlAdjointStats* stats);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* TEALEAF_B200_3D_H */
