/*
 * Storage for the CUDA built-in index variables used when the reference's
 * kernels run as host functions (test infrastructure; see oracle/Makefile).
 * The reference translation units see these as `extern const` (the form
 * curand_kernel.h uses for host compiles); this file owns them and the
 * harness sets them before every emulated thread.
 */
#include <vector_types.h>

uint3 threadIdx;
uint3 blockIdx;
dim3 blockDim;
dim3 gridDim;

extern "C" void qmb_ref_set_thread(unsigned block, unsigned thread, unsigned block_dim,
                                   unsigned grid_dim) {
    blockIdx.x = block;
    blockIdx.y = blockIdx.z = 0;
    threadIdx.x = thread;
    threadIdx.y = threadIdx.z = 0;
    blockDim.x = block_dim;
    blockDim.y = blockDim.z = 1;
    gridDim.x = grid_dim;
    gridDim.y = gridDim.z = 1;
}
