/*
 * Test harness around the reference TeaLeaf host code (checker only).
 *
 * This file is test infrastructure. It replaces the reference's `main`
 * (2d/main.c:9-59, 3d/main.c) with a loop that times every timestep and
 * reports the per-step field summary, which the reference itself only
 * computes and never prints (2d/drivers/field_summary_driver.c:8-54).
 *
 * It is compiled against the reference's own headers and linked with the
 * reference's host/driver objects plus ONE kernel suite: either the
 * reference omp3 suite (the oracle) or the B200 suite (to prove the B200
 * library is a drop-in behind the unchanged `kernel_interface.h`).
 *
 * Output (stdout, the master rank), besides the reference's own log lines:
 *   TLSTEP <step> <vol> <mass> <ie> <temp> <seconds>
 * with %.17e values (summed over ranks), one line per timestep, and a final
 *   TLDONE <total solve seconds>
 *
 * Build: oracle/build_ref.py (-DTL3D selects the 3D host).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

#include "chunk.h"
#include "settings.h"
#include "application.h"
#include "comms.h"
#include "drivers/drivers.h"
#include "kernel_interface.h"

/* `solve` is a global of the reference timestep loop (2d/diffuse.c:22). */
void solve(Chunk* chunks, Settings* settings, int tt, double* wallclock_prev);

static double now_seconds(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1.0e-9 * (double)ts.tv_nsec;
}

int main(int argc, char** argv)
{
    if (argc < 2) {
        fprintf(stderr, "usage: %s tea.in [max_iters_override [warm_steps warm_cap]]\n", argv[0]);
        return 2;
    }

    initialise_comms(argc, argv);

    Settings* settings = (Settings*)malloc(sizeof(Settings));
    set_default_settings(settings);
    strncpy(settings->tea_in_filename, argv[1], 255);
    settings->tea_in_filename[255] = '\0';
    initialise_ranks(settings);

    Chunk* chunks = NULL;
    initialise_application(&chunks, settings);

    /* Optional cap used for the bounded CPU-baseline samples; the first
     * warm_steps timesteps (warm-up, not timed by the caller) may use a
     * smaller cap of their own. */
    int cap = settings->max_iters, warm_steps = 0, warm_cap = 0;
    if (argc >= 3) {
        cap = atoi(argv[2]);
    }
    if (argc >= 5) {
        warm_steps = atoi(argv[3]);
        warm_cap = atoi(argv[4]);
    }
    settings->max_iters = cap;

    double wallclock_prev = 0.0;
    double total = 0.0;
    for (int tt = 0; tt < settings->end_step; ++tt) {
        settings->max_iters = (tt < warm_steps && warm_cap > 0) ? warm_cap : cap;
        double t0 = now_seconds();
        solve(chunks, settings, tt, &wallclock_prev);
        double t1 = now_seconds();
        total += t1 - t0;

        double vol = 0.0, mass = 0.0, ie = 0.0, temp = 0.0;
        run_field_summary(&chunks[0], settings, &vol, &mass, &ie, &temp);
        /* the mesh's summary on several ranks (field_summary_driver.c:28-31) */
        sum_over_ranks(settings, &vol);
        sum_over_ranks(settings, &mass);
        sum_over_ranks(settings, &ie);
        sum_over_ranks(settings, &temp);
        if (settings->rank == MASTER) {
            printf("TLSTEP %d %.17e %.17e %.17e %.17e %.9f\n",
                   tt + 1, vol, mass, ie, temp, t1 - t0);
            fflush(stdout);
        }
    }
    if (settings->rank == MASTER) {
        printf("TLDONE %.9f\n", total);
        fflush(stdout);
    }

#ifndef TL3D
    kernel_finalise_driver(chunks, settings);
#endif
    finalise_comms();
    return 0;
}
