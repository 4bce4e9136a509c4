/* Force-included (g++ -include) when the reference's CUDA sources are compiled
 * for the host by oracle/Makefile.  Kernels become plain host functions; the
 * built-in index variables are declared the way curand_kernel.h declares them
 * for host compiles, and oracle/ref_harness.cpp defines them and sets them
 * before each emulated thread.  Test infrastructure only. */
#pragma once
#include <cstdint>
#include <vector_types.h>
extern const uint3 threadIdx;
extern const uint3 blockIdx;
extern const dim3 blockDim;
extern const dim3 gridDim;
