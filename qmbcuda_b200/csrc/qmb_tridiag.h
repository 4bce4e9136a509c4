// qmb_tridiag.h -- FP64 symmetric tridiagonal eigensolver for the Lanczos
// matrix T (diagonal a[0..m-1], off-diagonal e[0..m-2]).  Replaces the
// reference's FormTriMat + cusolverDnXsyevd call (exact_diagonalization/
// lanczos.cu:17-28,245-259; cuda_wrappers/CudaWrappers.cu:174-265).
#pragma once
#include <vector>

namespace qmb {

// Lowest eigenvalue by Sturm-sequence bisection (the count of negative
// pivots of T - x I equals the number of eigenvalues below x), to full
// double precision.
double tridiag_min_eig(const double* a, const double* e, int m);

// k-th smallest eigenvalue (k = 0 is the lowest), same method.
double tridiag_eig(const double* a, const double* e, int m, int k);

// Unit eigenvector for eigenvalue theta by inverse iteration with a
// partially pivoted tridiagonal LU of T - theta I; sign fixed so that the
// first component is >= 0.
void tridiag_eigvec(const double* a, const double* e, int m, double theta, double* v);

// tridiag_eigvec with caller-provided workspace (work: 4*m doubles, iwork: m
// ints); performs no heap allocation.
void tridiag_eigvec_ws(const double* a, const double* e, int m, double theta, double* v,
                       double* work, int* iwork);

}  // namespace qmb
