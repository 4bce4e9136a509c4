/*
 * Compiles the reference's exact_diagonalization/utils.cu, unmodified and
 * from where it lies, under the data model it was written for.  The reference
 * targets MSVC on Windows (LLP64: `long` is 32 bits).  Its bit loops
 * `for (long unsigned int i = 1 << 31; ...)` (utils.cu:19, :53, :730) rely on
 * that: under LP64 `1 << 31` sign-extends into a 64-bit `unsigned long` and
 * the rank / orbit loops test several bits at once.  Every header utils.cu
 * includes is pulled in first (all are include-guarded), then `long` is
 * mapped away so `long unsigned int` reads `unsigned int`; no other `long`
 * token follows in utils.cu.  Test infrastructure only.
 */
#include "exact_diagonalization/utils.h"
#include "utils/misc_funcs_gpu.h"
#include <thrust/complex.h>
#include <cooperative_groups.h>
#include <stdio.h>
#define long
#include "exact_diagonalization/utils.cu"
#undef long
