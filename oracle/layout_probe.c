/*
 * Struct-layout probe (test infrastructure).
 *
 * Prints "<struct>.<field> <offset> <size>" and "<struct> sizeof <n>" for the
 * structs that cross the kernel-suite boundary: Chunk (2d/chunk.h:10-79,
 * 3d/chunk.h), Settings (2d/settings.h:69-128, 3d/settings.h) and State
 * (2d/settings.h:139-150). Compiled once against the reference headers (the
 * golden layout) and once against include/tealeaf_b200_{2d,3d}.h, so a test
 * can prove the B200 library reads the host's structs at the same offsets.
 */
#include <stddef.h>
#include <stdio.h>

#ifdef TL_PROBE_B200
#  ifdef TL3D
#    include "tealeaf_b200_3d.h"
#  else
#    include "tealeaf_b200_2d.h"
#  endif
#else
#  include "chunk.h"
#  include "settings.h"
#endif

#define F(S, f) printf(#S "." #f " %zu %zu\n", offsetof(S, f), sizeof(((S*)0)->f))

int main(void)
{
    F(Chunk, dt_init); F(Chunk, neighbours);
    F(Chunk, left_send); F(Chunk, left_recv); F(Chunk, right_send); F(Chunk, right_recv);
    F(Chunk, top_send); F(Chunk, top_recv); F(Chunk, bottom_send); F(Chunk, bottom_recv);
#ifdef TL3D
    F(Chunk, front_send); F(Chunk, front_recv); F(Chunk, back_send); F(Chunk, back_recv);
    F(Chunk, lr_page); F(Chunk, tb_page); F(Chunk, fb_page);
#endif
    F(Chunk, left); F(Chunk, right); F(Chunk, bottom); F(Chunk, top);
#ifdef TL3D
    F(Chunk, back); F(Chunk, front);
#endif
    F(Chunk, x); F(Chunk, y);
#ifdef TL3D
    F(Chunk, z);
#endif
    F(Chunk, density0); F(Chunk, density); F(Chunk, energy0); F(Chunk, energy);
#ifdef TL3D
    F(Chunk, vec_u); F(Chunk, vec_u0); F(Chunk, vec_p); F(Chunk, vec_r); F(Chunk, vec_mi);
    F(Chunk, vec_w); F(Chunk, vec_kx); F(Chunk, vec_ky); F(Chunk, vec_kz); F(Chunk, vec_sd);
    F(Chunk, vec_z);
    F(Chunk, cell_x); F(Chunk, cell_y); F(Chunk, cell_z);
    F(Chunk, cell_dx); F(Chunk, cell_dy); F(Chunk, cell_dz);
    F(Chunk, vertex_dx); F(Chunk, vertex_dy); F(Chunk, vertex_dz);
    F(Chunk, vertex_x); F(Chunk, vertex_y); F(Chunk, vertex_z);
    F(Chunk, volume); F(Chunk, x_area); F(Chunk, y_area); F(Chunk, z_area);
#else
    F(Chunk, u); F(Chunk, u0); F(Chunk, p); F(Chunk, r); F(Chunk, mi); F(Chunk, w);
    F(Chunk, kx); F(Chunk, ky); F(Chunk, sd);
    F(Chunk, cell_x); F(Chunk, cell_y); F(Chunk, cell_dx); F(Chunk, cell_dy);
    F(Chunk, vertex_dx); F(Chunk, vertex_dy); F(Chunk, vertex_x); F(Chunk, vertex_y);
    F(Chunk, volume); F(Chunk, x_area); F(Chunk, y_area);
#endif
    F(Chunk, theta); F(Chunk, eigmin); F(Chunk, eigmax);
    F(Chunk, cg_alphas); F(Chunk, cg_betas); F(Chunk, cheby_alphas); F(Chunk, cheby_betas);
    F(Chunk, ext);
    printf("Chunk sizeof %zu\n", sizeof(Chunk));

    F(Settings, kernel_profile); F(Settings, application_profile); F(Settings, wallclock_profile);
    F(Settings, tea_out_fp); F(Settings, rank); F(Settings, end_step); F(Settings, presteps);
    F(Settings, max_iters); F(Settings, coefficient); F(Settings, ppcg_inner_steps);
    F(Settings, summary_frequency); F(Settings, halo_depth); F(Settings, num_states);
    F(Settings, num_chunks); F(Settings, num_chunks_per_rank); F(Settings, num_ranks);
    F(Settings, fields_to_exchange); F(Settings, is_offload); F(Settings, error_switch);
    F(Settings, check_result); F(Settings, preconditioner); F(Settings, eps);
    F(Settings, dt_init); F(Settings, end_time); F(Settings, eps_lim);
    F(Settings, tea_in_filename); F(Settings, tea_out_filename); F(Settings, test_problem_filename);
    F(Settings, solver);
#ifndef TL3D
    F(Settings, solver_name);
#endif
    F(Settings, kernel_language);
    F(Settings, grid_x_cells); F(Settings, grid_y_cells);
#ifdef TL3D
    F(Settings, grid_z_cells);
#endif
    F(Settings, grid_x_min); F(Settings, grid_y_min);
#ifdef TL3D
    F(Settings, grid_z_min);
#endif
    F(Settings, grid_x_max); F(Settings, grid_y_max);
#ifdef TL3D
    F(Settings, grid_z_max);
#endif
    F(Settings, dx); F(Settings, dy);
#ifdef TL3D
    F(Settings, dz);
#endif
    printf("Settings sizeof %zu\n", sizeof(Settings));

    F(State, defined); F(State, density); F(State, energy);
    F(State, x_min); F(State, y_min);
#ifdef TL3D
    F(State, z_min);
#endif
    F(State, x_max); F(State, y_max);
#ifdef TL3D
    F(State, z_max);
#endif
    F(State, radius); F(State, geometry);
    printf("State sizeof %zu\n", sizeof(State));
    return 0;
}
