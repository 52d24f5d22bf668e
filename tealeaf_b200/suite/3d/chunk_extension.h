/*
 * B200 kernel-suite extension point for the 3D TeaLeaf host.
 *
 * The 3D host includes "build/chunk_extension.h" (3d/chunk.h:5); the
 * reference make copies every header of the suite directory into build/
 * (3d/Makefile:38). 3D fields are plain `double*` in the host's Chunk; here
 * they are device pointers that the host never dereferences.
 *
 * chunk_extension_t holds one opaque pointer to the suite's per-chunk state,
 * filled by run_kernel_initialise. The host allocates the struct itself
 * (3d/chunk.c:37) and never reads it.
 */
#ifndef TL_B200_CHUNK_EXTENSION_3D
#define TL_B200_CHUNK_EXTENSION_3D

struct TlSuite3D;

typedef struct chunk_extension_t
{
    struct TlSuite3D* suite;
} chunk_extension_t;

#endif
