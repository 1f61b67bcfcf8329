// Small dense symmetric eigensolver used inside the batched Rayleigh-Ritz
// steps (local GHEP, level-3 HEP).  Cyclic Jacobi rotations (Jacobi's method
// as given in Golub & Van Loan, "Matrix Computations", section 8.5) executed
// by one warp on a matrix in shared memory, followed by an ascending sort.
#pragma once

#include "pmf_common.cuh"

namespace pmf {

// A: n x n symmetric, row-major with leading dimension lda (destroyed; on
// return its diagonal holds the eigenvalues in the original order).
// V: n x n eigenvector matrix (columns), lda.  w: n sorted eigenvalues; V is
// permuted to match.  n <= 32.  Must be called by all 32 lanes of one warp.
__device__ inline void warp_jacobi_eigh(double* A, double* V, double* w, int n, int lda, int max_sweeps = 30) {
  const int l = threadIdx.x & 31;
  for (int i = 0; i < n; ++i)
    if (l < n) V[i * lda + l] = (i == l) ? 1.0 : 0.0;
  __syncwarp();
  double norm = 0.0;
  if (l < n)
    for (int j = 0; j < n; ++j) norm += A[l * lda + j] * A[l * lda + j];
  norm = warp_sum(norm);
  const double tiny = 1e-300;
  for (int sweep = 0; sweep < max_sweeps; ++sweep) {
    double off = 0.0;
    if (l < n)
      for (int j = 0; j < n; ++j)
        if (j != l) off += A[l * lda + j] * A[l * lda + j];
    off = warp_sum(off);
    if (off <= 1e-30 * norm || off < tiny) break;
    for (int p = 0; p < n - 1; ++p) {
      for (int q = p + 1; q < n; ++q) {
        const double apq = A[p * lda + q];
        const double app = A[p * lda + p];
        const double aqq = A[q * lda + q];
        if (fabs(apq) <= 1e-18 * sqrt(fabs(app * aqq)) || fabs(apq) < tiny) continue;
        const double theta = (aqq - app) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double s = t * c;
        __syncwarp();
        if (l < n) {  // columns p, q
          const double akp = A[l * lda + p], akq = A[l * lda + q];
          A[l * lda + p] = c * akp - s * akq;
          A[l * lda + q] = s * akp + c * akq;
        }
        __syncwarp();
        if (l < n) {  // rows p, q
          const double apk = A[p * lda + l], aqk = A[q * lda + l];
          A[p * lda + l] = c * apk - s * aqk;
          A[q * lda + l] = s * apk + c * aqk;
        }
        __syncwarp();
        if (l < n) {
          const double vkp = V[l * lda + p], vkq = V[l * lda + q];
          V[l * lda + p] = c * vkp - s * vkq;
          V[l * lda + q] = s * vkp + c * vkq;
        }
        __syncwarp();
      }
    }
  }
  // ascending selection sort of eigenvalues, permuting columns of V
  if (l < n) w[l] = A[l * lda + l];
  __syncwarp();
  for (int i = 0; i < n - 1; ++i) {
    int best = i;
    double bv = w[i];
    for (int j = i + 1; j < n; ++j)
      if (w[j] < bv) {
        bv = w[j];
        best = j;
      }
    __syncwarp();
    if (best != i) {
      if (l < n) {
        const double a = V[l * lda + i];
        V[l * lda + i] = V[l * lda + best];
        V[l * lda + best] = a;
      }
      if (l == 0) {
        const double a = w[i];
        w[i] = w[best];
        w[best] = a;
      }
    }
    __syncwarp();
  }
}

// Cheap deterministic pseudo-random number in [-1, 1) (splitmix64 finaliser).
__device__ __forceinline__ double hash_uniform(unsigned long long a) {
  a += 0x9E3779B97F4A7C15ull;
  a = (a ^ (a >> 30)) * 0xBF58476D1CE4E5B9ull;
  a = (a ^ (a >> 27)) * 0x94D049BB133111EBull;
  a ^= a >> 31;
  return (double)(a >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

}  // namespace pmf
