/*
 * B200 kernel-suite extension point for the 2D TeaLeaf host.
 *
 * The host includes this file from the kernel-suite directory
 * (2d/chunk.h:7 with -I$(KERNELS_PATH), 2d/Makefile:40-41). It fixes
 *   - FieldBufferType: a device pointer (cudaMalloc'd FP64 field, x fastest),
 *     never dereferenced by the host;
 *   - struct ChunkExtension: one opaque pointer to the suite's per-chunk
 *     state, filled by run_kernel_initialise. The host allocates the struct
 *     itself (2d/chunk.c:29) and never reads it.
 */
#ifndef TL_B200_CHUNK_EXTENSION_2D
#define TL_B200_CHUNK_EXTENSION_2D

typedef double* FieldBufferType;

struct TlSuite2D;

typedef struct ChunkExtension
{
    struct TlSuite2D* suite;
} ChunkExtension;

#endif
