/*
 * tealeaf_b200_2d.h -- C ABI of the B200 (sm_100a) TeaLeaf 2D kernel suite.
 *
 * libtealeaf_b200_2d.so is a drop-in kernel suite for the unchanged TeaLeaf
 * 2D host (main.c, diffuse.c, drivers/, chunk.c built with -DNO_MPI). It
 * exports the 23 functions of the reference kernel interface with the same
 * names, argument meaning and accumulate/synchronous result semantics
 * (2d/kernel_interface.h:13-71), the optional diffuse_overload hook
 * (2d/application.h:9-11), and a few additional entry points marked "new"
 * below.
 *
 * The Chunk / Settings / State structs below restate the reference layouts
 * field for field (2d/chunk.h:10-79, 2d/settings.h:69-150) so the library
 * reads the host's structs at the host's offsets; a test compares every
 * offset against the reference headers. FieldBufferType and ChunkExtension
 * are the suite's own choice (tealeaf_b200/suite/2d/chunk_extension.h):
 * field buffers are device pointers the host never dereferences.
 *
 * Result semantics (2d/drivers/cg_driver.c:35,72,88): every double* result
 * is ACCUMULATED (*out += value) and valid when the call returns.
 * Error semantics: by default a CUDA or argument error prints a message and
 * calls exit(1), as the reference die() does (2d/shared.c:97-111);
 * tl2d_set_error_mode(TL_ERRMODE_RECORD) makes calls record the error and
 * return instead (read it with tl2d_get_error).
 */
#ifndef TEALEAF_B200_2D_H
#define TEALEAF_B200_2D_H

#include <stdbool.h>
#include <stdio.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Every function below is exported even when the library is built with
 * hidden default visibility. */
#if defined(__GNUC__)
#pragma GCC visibility push(default)
#endif

/* ---- suite-owned extension point (same text as suite/2d/chunk_extension.h) */
#ifndef TL_B200_CHUNK_EXTENSION_2D
#define TL_B200_CHUNK_EXTENSION_2D
typedef double* FieldBufferType;
struct TlSuite2D;
typedef struct ChunkExtension
{
    struct TlSuite2D* suite;
} ChunkExtension;
#endif

/* ---- constants shared with the host (2d/shared.h:22-43) ------------------ */
#define TL_NUM_FIELDS 6
#define TL_CHUNK_LEFT 0
#define TL_CHUNK_RIGHT 1
#define TL_CHUNK_BOTTOM 2
#define TL_CHUNK_TOP 3
#define TL_EXTERNAL_FACE (-1)
#define TL_FIELD_DENSITY 0
#define TL_FIELD_ENERGY0 1
#define TL_FIELD_ENERGY1 2
#define TL_FIELD_U 3
#define TL_FIELD_P 4
#define TL_FIELD_SD 5
#define TL_CONDUCTIVITY 1
#define TL_RECIP_CONDUCTIVITY 2
#define TL_CG_ITERS_FOR_EIGENVALUES 20
#define TL_ERROR_SWITCH_MAX 1.0
/* Solver enum values (2d/settings.h:50-56) and Geometry (2d/settings.h:131-136). */
#define TL_JACOBI_SOLVER 0
#define TL_CG_SOLVER 1
#define TL_CHEBY_SOLVER 2
#define TL_PPCG_SOLVER 3
#define TL_GEOM_RECTANGULAR 0
#define TL_GEOM_CIRCULAR 1
#define TL_GEOM_POINT 2

/* ---- host structs: layout restated from 2d/settings.h:69-128 ------------- */
struct Profile;

typedef struct Settings
{
    struct Profile* kernel_profile;
    struct Profile* application_profile;
    struct Profile* wallclock_profile;
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
    bool* fields_to_exchange;   /* host bool[TL_NUM_FIELDS] */
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
    int solver;                 /* enum Solver */
    char* solver_name;
    int kernel_language;        /* enum Kernel_Language */
    int grid_x_cells;
    int grid_y_cells;
    double grid_x_min;
    double grid_y_min;
    double grid_x_max;
    double grid_y_max;
    double dx;
    double dy;
} Settings;

/* 2d/settings.h:139-150 */
typedef struct State
{
    bool defined;
    double density;
    double energy;
    double x_min;
    double y_min;
    double x_max;
    double y_max;
    double radius;
    int geometry;               /* enum Geometry */
} State;

/* 2d/chunk.h:10-79 */
typedef struct Chunk
{
    double dt_init;
    int* neighbours;            /* host int[4] */
    double* left_send;
    double* left_recv;
    double* right_send;
    double* right_recv;
    double* top_send;
    double* top_recv;
    double* bottom_send;
    double* bottom_recv;
    int left;
    int right;
    int bottom;
    int top;
    int x;                      /* cells incl. halo: x_cells + 2*halo_depth */
    int y;
    FieldBufferType density0;
    FieldBufferType density;
    FieldBufferType energy0;
    FieldBufferType energy;
    FieldBufferType u;
    FieldBufferType u0;
    FieldBufferType p;
    FieldBufferType r;
    FieldBufferType mi;
    FieldBufferType w;
    FieldBufferType kx;
    FieldBufferType ky;
    FieldBufferType sd;
    FieldBufferType cell_x;
    FieldBufferType cell_y;
    FieldBufferType cell_dx;
    FieldBufferType cell_dy;
    FieldBufferType vertex_dx;
    FieldBufferType vertex_dy;
    FieldBufferType vertex_x;
    FieldBufferType vertex_y;
    FieldBufferType volume;
    FieldBufferType x_area;
    FieldBufferType y_area;
    double theta;
    double eigmin;
    double eigmax;
    double* cg_alphas;          /* host arrays of max_iters (drivers write them) */
    double* cg_betas;
    double* cheby_alphas;
    double* cheby_betas;
    struct ChunkExtension* ext;
} Chunk;

/* ---- reference kernel interface (2d/kernel_interface.h:13-71) ------------ */
/* Initialisation kernels */
void run_set_chunk_data(Chunk* chunk, Settings* settings);                 /* :13 */
void run_set_chunk_state(Chunk* chunk, Settings* settings, State* states); /* :15 */
void run_kernel_initialise(Chunk* chunk, Settings* settings);              /* :17 */
void run_kernel_finalise(Chunk* chunk, Settings* settings);                /* :19 */
/* Solver-wide kernels */
void run_local_halos(Chunk* chunk, Settings* settings, int depth);         /* :23 */
void run_pack_or_unpack(Chunk* chunk, Settings* settings, int depth,       /* :25 */
        int face, bool pack, FieldBufferType field, double* buffer);
void run_store_energy(Chunk* chunk, Settings* settings);                   /* :28 */
void run_field_summary(Chunk* chunk, Settings* settings,                   /* :30 */
        double* vol, double* mass, double* ie, double* temp);
/* CG solver kernels */
void run_cg_init(Chunk* chunk, Settings* settings,                         /* :35 */
        double rx, double ry, double* rro);
void run_cg_calc_w(Chunk* chunk, Settings* settings, double* pw);          /* :38 */
void run_cg_calc_ur(Chunk* chunk, Settings* settings,                      /* :40 */
        double alpha, double* rrn);
void run_cg_calc_p(Chunk* chunk, Settings* settings, double beta);         /* :42 */
/* Chebyshev solver kernels */
void run_cheby_init(Chunk* chunk, Settings* settings);                     /* :46 */
void run_cheby_iterate(Chunk* chunk, Settings* settings,                   /* :48 */
        double alpha, double beta);
/* Jacobi solver kernels */
void run_jacobi_init(Chunk* chunk, Settings* settings, double rx, double ry); /* :52 */
void run_jacobi_iterate(Chunk* chunk, Settings* settings, double* error);  /* :54 */
/* PPCG solver kernels */
void run_ppcg_init(Chunk* chunk, Settings* settings);                      /* :58 */
void run_ppcg_inner_iteration(Chunk* chunk, Settings* settings,            /* :60 */
        double alpha, double beta);
/* Shared solver kernels */
void run_copy_u(Chunk* chunk, Settings* settings);                         /* :64 */
void run_calculate_residual(Chunk* chunk, Settings* settings);             /* :66 */
void run_calculate_2norm(Chunk* chunk, Settings* settings,                 /* :68 */
        FieldBufferType buffer, double* norm);
void run_finalise(Chunk* chunk, Settings* settings);                       /* :70 */

/* ---- optional host hook (2d/application.h:9-11, 2d/main.c:32-36) -------- */
/* Device-resident replacement of diffuse() (2d/diffuse.c:10-19): runs every
 * timestep with the solver loops kept on the GPU (scalars alpha/beta/rro
 * formed on the device, one host synchronisation per batch of iterations)
 * and finishes with the host's field_summary_driver(…, true) when the host
 * provides it. */
void diffuse_overload(Chunk* chunk, Settings* settings);

/* ---- new entry points (no reference counterpart) ------------------------- */
#define TL_ERRMODE_EXIT 0
#define TL_ERRMODE_RECORD 1
/* Error behaviour: TL_ERRMODE_EXIT (default, like die()) or TL_ERRMODE_RECORD. */
void tl2d_set_error_mode(int mode);
/* Returns the first recorded error code (0: none) and its message; clears it. */
int tl2d_get_error(char* msg, int msg_len);
/* Selects the CUDA device for the chunks initialised afterwards on this thread. */
void tl2d_set_device(int device);
/* The cudaStream_t every kernel of this chunk is issued on (as void*). */
void* tl2d_stream(Chunk* chunk);

/* No counterpart in the reference. Run Chebyshev trips and PPCG inner steps
 * temporally blocked in shared memory (1, the default; results are
 * bit-identical) or one launch per step (0): in the device-resident driver
 * (tl2d_solve_step), and through the kernel interface, where consecutive
 * run_cheby_iterate / run_ppcg_inner_iteration calls (each preceded only by
 * the drivers' depth-1 halo update) are deferred and run as blocked launches
 * when the next other entry point is called. The same switch selects the
 * blocked preconditioner of the refinement form's PPCG (tl2d_refine_solve_step;
 * its fields are bit-identical, its r.z is summed over another partition). */
void tl2d_set_temporal_blocking(Chunk* chunk, int on);

/* Jacobi preconditioner of the device-resident CG (tl2d_solve_step with the
 * CG solver): 0 none, 1 jac_diag, 2 jac_block (tridiagonal blocks of 4 rows
 * along y). The reference documents both as tl_preconditioner_type
 * (README.md:127-133) but its C kernels ignore `preconditioner_on`; here
 * settings->preconditioner at run_kernel_initialise selects jac_diag and
 * this call any of the three. The stop test stays r.r < eps. The run_*
 * kernel interface is unpreconditioned, as in the reference. Returns 0, or
 * 37 for another type. */
int tl2d_set_preconditioner(Chunk* chunk, int type);

/* No counterpart in the reference. Feed the CG w sweep's operand rows by TMA
 * tile loads (1, the default, where the halo depth and row length are even;
 * results are bit-identical) or by per-thread loads (0). */
void tl2d_set_tma(Chunk* chunk, int on);

/* No counterpart in the reference. Runs every operation the suite has
 * deferred for this chunk (a CG p update, halo updates, queued PPCG inner
 * steps), as every run_* call that touches device data does first. Call it
 * before reading the chunk's device fields by other means (own kernels, or
 * an allocation-free entry point given a field pointer). Asynchronous on the
 * chunk's stream. */
void tl2d_flush(Chunk* chunk);

/* Per-kernel device-time profile (CUDA events around every launch on the
 * chunk's stream, resolved at the next synchronisation): enable/disable,
 * reset, and read entry `index` (returns 0 past the last entry). */
void tl2d_profile_enable(Chunk* chunk, int on);
void tl2d_profile_reset(Chunk* chunk);
int tl2d_profile_read(Chunk* chunk, int index, char* name, int name_len,
        long long* calls, double* ms);
/* Kernel launches issued for this chunk since initialisation (counted
 * whether or not the profile is enabled); -1 for an unknown chunk. */
long long tl2d_launch_count(Chunk* chunk);

/* Field ids for the host-buffer staging calls. */
#define TL2D_DENSITY0 0
#define TL2D_DENSITY 1
#define TL2D_ENERGY0 2
#define TL2D_ENERGY 3
#define TL2D_U 4
#define TL2D_U0 5
#define TL2D_P 6
#define TL2D_R 7
#define TL2D_MI 8
#define TL2D_W 9
#define TL2D_KX 10
#define TL2D_KY 11
#define TL2D_SD 12
#define TL2D_VOLUME 13
#define TL2D_NUM_IDS 14
/* Copies a full x*y field between a host buffer and the chunk (blocking;
 * pinned host memory gives full PCIe/NVLink-C2C bandwidth). */
void tl2d_upload_field(Chunk* chunk, Settings* settings, int field_id,
        const double* host, long long count);
void tl2d_download_field(Chunk* chunk, Settings* settings, int field_id,
        double* host, long long count);

/* Per-timestep statistics of the device-resident driver. */
typedef struct TlStepStats
{
    int cg_iters;       /* CG iterations (CG solver, or presteps of Cheby/PPCG) */
    int cheby_iters;
    int ppcg_iters;     /* outer PPCG iterations */
    int jacobi_iters;
    int est_iters;      /* Chebyshev estimate */
    int total_iters;    /* loop trips of the solver loop (tt at exit) */
    double error;
    double eigmin;
    double eigmax;
    double exact_error; /* ||u0 - A u||^2 after the solve (check_result) */
} TlStepStats;

/* Allocation-free 2-norm: no counterpart in the reference. Adds the sum of
 * squares of the interior of `field` (a device array of x*y values, halo
 * included, index k + j*x) to the device double *norm_dev, like
 * run_calculate_2norm does for a host double; the sum equals that entry
 * point's up to rounding (the block partials are added in another tree).
 * For callers that cannot allocate device memory, or cannot
 * take the device-wide synchronisation a cudaMalloc/cudaFree implies (e.g. a
 * host whose memory is held by its own pool allocator): the reduction scratch
 * is a static device array of 65536 block partials (about 512 KiB) that every
 * GPU loading the library holds until exit, so this call allocates nothing.
 * Interiors needing more than 65536 blocks of 128 x 8 cells (beyond about
 * 8192 x 8192) are rejected with an error before any launch. Asynchronous on
 * `stream` (a cudaStream_t, NULL for the default stream). The array's address
 * is looked up once per device (cudaGetSymbolAddress) and cached; under CUDA's
 * lazy module loading that look-up is also when the driver reserves the
 * array. run_kernel_initialise does it, so a host that initialises a chunk
 * first has the array in place; a caller without a chunk should make its
 * first call before it gives the rest of device memory to its pool and
 * before any stream capture, or set CUDA_MODULE_LOADING=EAGER. All calls share the one
 * array: calls that overlap on the GPU race and must be serialised. Returns 0,
 * or an error code with the message available from tl2d_get_error. */
int tl2d_calculate_2norm_noalloc(const double* field, int x, int y, int halo_depth,
        double* norm_dev, void* stream);

/* Drives the bounded barrier wait that every TMA-fed sweep uses to expiry,
 * without a GPU fault: one block waits on a shared-memory barrier that no copy
 * and no thread completes, gives up after `polls` polls (1 .. 2^26) and
 * records that in the chunk's wait-error word, as a sweep whose tile load
 * never completed would. Returns 35 with the message from tl2d_get_error
 * (set tl2d_set_error_mode(1) first, or the error exits like die()); every
 * later solve on the chunk then reports error 35 as well, until the chunk is
 * finalised. No counterpart in the reference: its failures are die() calls
 * (2d/shared.c:97-111); this exists to test the error path of the waits. */
int tl2d_check_bounded_wait(Chunk* chunk, long long polls);

/* The four field-summary totals from a parallel tree reduction: one sweep at
 * full bandwidth instead of run_field_summary's serial reference order, so
 * the last bits differ from the reference (accumulated like run_field_summary). */
void tl2d_field_summary_fast(Chunk* chunk, Settings* settings,
        double* vol, double* mass, double* ie, double* temp);

/* One timestep of solve() (2d/diffuse.c:22-80) on the device-resident path.
 * The chunk must be undivided (four external faces: the loop holds no remote
 * halo exchange); a chunk with a neighbour reports error 34. */
void tl2d_solve_step(Chunk* chunk, Settings* settings, int tt, TlStepStats* stats);

/* Statistics of one iterative-refinement timestep. */
typedef struct TlRefineStats
{
    int iterations;        /* CG iterations; for PPCG the CG trips plus the outer PPCG steps */
    int residual_updates;  /* FP64 residual recomputations */
    int converged;         /* 1 when rel_residual <= rel_tol */
    int cg_trips;          /* PPCG: CG trips before the switch (CG: equal to iterations) */
    double rel_residual;   /* ||u0 - A u||_2 / ||u0||_2 in FP64 at exit */
    double device_ms;      /* device time of the whole timestep on the chunk stream */
} TlRefineStats;

/* Iterative-refinement timestep: no counterpart in the reference. Runs the
 * timestep of solve() (2d/diffuse.c:22-80: halos, cg_init, u0 = u, solve,
 * finalise) with the solve run to the relative FP64 residual
 * ||u0 - A u||_2 / ||u0||_2 <= rel_tol. precision 32: vectors and operator
 * coefficients stored in FP32, the stencil and vector updates in FP32
 * arithmetic, FP64 dot products and scalars, the solution accumulated in FP64
 * with the residual recomputed in FP64 (reliable updates); precision 64: the
 * same iteration with FP64 storage and arithmetic. The solve is
 * CG, or PPCG when settings->solver is TL_PPCG_SOLVER (2d/drivers/ppcg_driver.c:
 * CG trips to the reference's switch test, Lanczos eigenvalue bounds and
 * Chebyshev coefficients in FP64 from the FP64 CG scalars, outer steps with
 * settings->ppcg_inner_steps inner steps). Needs one chunk with four external
 * faces; at most settings->max_iters iterations. Returns 0, or an error code
 * with the message available from tl2d_get_error. */
int tl2d_refine_solve_step(Chunk* chunk, Settings* settings, int tt, double rel_tol,
        int precision, TlRefineStats* stats);

/* Batched timesteps: no counterpart in the reference. A batch holds `count`
 * initialised chunks of any sizes (each one chunk with four external faces,
 * with its own settings). tl2d_batch_step runs one solve() of every problem
 * (halos, cg_init, u0 = u, the solve, finalise, energy halo) with the CG
 * solve of all problems in one persistent cooperative kernel: FP32 vectors
 * and coefficients, FP32 arithmetic in the sweeps, FP64 dot products,
 * scalars and solution, FP64 residual replacement, each problem stopped when its FP64 residual gives
 * r.r < its settings->eps (the reference's 2D stop test). The whole timestep
 * is captured once into a CUDA graph and replayed. */
typedef struct TlBatch TlBatch;

typedef struct TlBatchStats
{
    int problems;
    int converged;          /* problems whose FP64 residual met eps */
    int max_iterations;     /* CG iterations of the slowest problem */
    int total_iterations;   /* summed over the problems */
    int kernel_iterations;  /* iterations the persistent kernel ran */
    int tile_rows;          /* tile height in use */
    int grid_blocks;        /* persistent grid in use */
    int graph;              /* 1 when the step ran as a CUDA graph replay */
    double device_ms;       /* device time of the whole batched timestep */
} TlBatchStats;

/* tile_rows, grid_blocks: 0 for the defaults (16; the co-residency limit);
 * tile_rows -1: per-problem heights (see tl2d_batch_tune). */
TlBatch* tl2d_batch_create(Chunk** chunks, Settings** settings, int count, int tile_rows, int grid_blocks);
void tl2d_batch_destroy(TlBatch* batch);
/* Autotuner: times trial_iters iterations of the batch (0: the whole solve)
 * for each tile height in {-1 = per problem, about one tile per block of the
 * grid, 8..64 rows; 4, 8, 16, 32, 64} and persistent grid of {2,4,6,8} blocks
 * per SM and keeps
 * the fastest (best_ms: its time). Leaves the energy fields unchanged. */
int tl2d_batch_tune(TlBatch* batch, int trial_iters, double* best_ms);
void tl2d_batch_config(TlBatch* batch, int* tile_rows, int* grid_blocks);
int tl2d_batch_step(TlBatch* batch, TlBatchStats* stats);
/* Per problem of the last step: CG iterations, FP64 r.r, converged flag
 * (arrays of count; any may be NULL). */
int tl2d_batch_results(TlBatch* batch, int* iterations, double* rr, int* converged);
/* How many SM clocks a phase wait of the persistent kernel may take
 * before it gives up (cycles <= 0: the default, about 2 s). A wait that gives
 * up makes every block return and tl2d_batch_step report error 63; the
 * batch's fields are then invalid until the next step. No counterpart in the
 * reference (its MPI barriers do not time out). */
int tl2d_batch_set_wait_limit(TlBatch* batch, long long cycles);

#if defined(__GNUC__)
#pragma GCC visibility pop
#endif

#ifdef __cplusplus
}
#endif

#endif /* TEALEAF_B200_2D_H */
