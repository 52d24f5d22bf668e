/* Checker probe (test infrastructure): prints the reference's own
 * decomposition of a mesh over N ranks, one chunk per rank, by calling its
 * decompose_field (2d/initialise.c:34-134; 3d/initialise.c:34-174 with
 * -DTL3D) once per rank, as each MPI rank would.
 *
 *   decompose2d X Y N     ->  per rank: r left right bottom top nb_l nb_r nb_b nb_t
 *   decompose3d X Y Z N   ->  per rank: r left right bottom top back nb_l nb_r nb_b nb_t nb_k nb_f
 *
 * (3D `front` is not printed: the reference computes it from itself,
 * 3d/initialise.c, and no kernel reads it.) A failed decomposition ends in
 * the reference's own die().
 *
 * Build: oracle/build_ref.py (linked with the reference host objects).
 */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "chunk.h"
#include "settings.h"

void decompose_field(Settings* settings, Chunk* chunks);

int main(int argc, char** argv)
{
#ifdef TL3D
    const int nargs = 5;
#else
    const int nargs = 4;
#endif
    if (argc != nargs) {
        fprintf(stderr, "usage: %s cells... ranks\n", argv[0]);
        return 2;
    }
    Settings* settings = (Settings*)calloc(1, sizeof(Settings));
    set_default_settings(settings);
    settings->grid_x_cells = atoi(argv[1]);
    settings->grid_y_cells = atoi(argv[2]);
#ifdef TL3D
    settings->grid_z_cells = atoi(argv[3]);
#endif
    const int n = atoi(argv[nargs - 1]);
    settings->num_ranks = n;
    settings->num_chunks_per_rank = 1;
    for (int r = 0; r < n; ++r) {
        Chunk chunk;
        memset(&chunk, 0, sizeof(chunk));
        settings->rank = r;
        decompose_field(settings, &chunk);
        printf("%d %d %d %d %d", r, chunk.left, chunk.right, chunk.bottom, chunk.top);
#ifdef TL3D
        printf(" %d", chunk.back);
        const int faces = 6;
#else
        const int faces = 4;
#endif
        for (int f = 0; f < faces; ++f) printf(" %d", chunk.neighbours[f]);
        printf("\n");
    }
    return 0;
}
