// Small dense symmetric eigensolver used inside the batched Rayleigh-Ritz
// steps (local GHEP, level-3 HEP): Jacobi's method with the parallel
// round-robin ("chess tournament") ordering of Brent & Luk (1985), executed by
// one warp on a matrix in shared memory, followed by an ascending sort.
#pragma once

#include "pmf_common.cuh"

namespace pmf {

// A: n x n symmetric, row-major, leading dimension lda (destroyed).
// V: n x n eigenvectors (columns).  w: n eigenvalues, ascending; V permuted
// to match.  n <= 32.  scratch: unused (kept for call-site compatibility).
// Must be called by all 32 lanes of one warp.
//
// Each round, lane k < n_even/2 computes the rotation of pair k; the
// parameters reach every lane by warp shuffles, and each lane then rotates
// its own column (row pass) and its own row (column pass) for all pairs with
// the loads of a group of pairs issued before any dependent arithmetic.
// Sweeps stop when every off-diagonal entry is below 1e-14 ||A||_F.
__device__ inline void warp_jacobi_eigh(double* A, double* V, double* w, int n, int lda, double* scratch,
                                        int max_sweeps = 20) {
  (void)scratch;
  const int l = threadIdx.x & 31;
  for (int i = 0; i < n; ++i)
    if (l < n) V[i * lda + l] = (i == l) ? 1.0 : 0.0;
  __syncwarp();
  const int ne = n + (n & 1);
  const int half = ne >> 1;
  double fro = 0.0;
  if (l < n)
    for (int j = 0; j < n; ++j) fro += A[l * lda + j] * A[l * lda + j];
  fro = sqrt(warp_sum(fro));
  for (int sweep = 0; sweep < max_sweeps && n > 1; ++sweep) {
    int bad = 0;
    if (l < n)
      for (int j = 0; j < n; ++j)
        if (j != l && fabs(A[l * lda + j]) > 1e-14 * fro) bad = 1;
    if (!__any_sync(0xffffffffu, bad)) break;
    for (int round = 0; round < ne - 1; ++round) {
      int p = 0, q = 0;
      double c = 1.0, s = 0.0;
      if (l < half) {
        const int pa = l, pb = ne - 1 - l;
        p = pa == 0 ? 0 : ((pa - 1 + round) % (ne - 1)) + 1;
        q = ((pb - 1 + round) % (ne - 1)) + 1;
        if (p > q) {
          const int t = p;
          p = q;
          q = t;
        }
        if (q < n) {
          const double apq = A[p * lda + q];
          const double app = A[p * lda + p];
          const double aqq = A[q * lda + q];
          if (fabs(apq) > 1e-300 && fabs(apq) > 1e-18 * sqrt(fabs(app * aqq))) {
            // tan of the rotation angle from single-precision arithmetic: an
            // approximate angle still shrinks a_pq, and (c, s) below are made
            // exactly orthonormal in FP64 from whatever t is used.
            const double theta = (aqq - app) * (0.5 / apq);
            double t;
            if (fabs(theta) < 1e18) {
              const float th = (float)theta;
              t = (double)(copysignf(1.0f, th) / (fabsf(th) + sqrtf(fmaf(th, th, 1.0f))));
            } else {
              t = 0.5 / theta;
            }
            c = rsqrt(fma(t, t, 1.0));
            s = t * c;
          }
        } else {
          q = p;  // dummy partner: no rotation
        }
      }
      __syncwarp();
      // row pass (J^T A): lane = column l; pairs in groups of 4
      for (int k0 = 0; k0 < half; k0 += 4) {
        int pk[4], qk[4];
        double ck[4], sk[4], ap[4], aq[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int src = min(k0 + u, half - 1);
          pk[u] = __shfl_sync(0xffffffffu, p, src);
          qk[u] = __shfl_sync(0xffffffffu, q, src);
          ck[u] = __shfl_sync(0xffffffffu, c, src);
          sk[u] = __shfl_sync(0xffffffffu, s, src);
          if (k0 + u >= half) sk[u] = 0.0;
        }
        if (l < n) {
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (sk[u] != 0.0) {
              ap[u] = A[pk[u] * lda + l];
              aq[u] = A[qk[u] * lda + l];
            }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (sk[u] != 0.0) {
              A[pk[u] * lda + l] = ck[u] * ap[u] - sk[u] * aq[u];
              A[qk[u] * lda + l] = sk[u] * ap[u] + ck[u] * aq[u];
            }
        }
      }
      __syncwarp();
      // column pass (A J, V J): lane = row l
      for (int k0 = 0; k0 < half; k0 += 4) {
        int pk[4], qk[4];
        double ck[4], sk[4], ap[4], aq[4], vp[4], vq[4];
#pragma unroll
        for (int u = 0; u < 4; ++u) {
          const int src = min(k0 + u, half - 1);
          pk[u] = __shfl_sync(0xffffffffu, p, src);
          qk[u] = __shfl_sync(0xffffffffu, q, src);
          ck[u] = __shfl_sync(0xffffffffu, c, src);
          sk[u] = __shfl_sync(0xffffffffu, s, src);
          if (k0 + u >= half) sk[u] = 0.0;
        }
        if (l < n) {
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (sk[u] != 0.0) {
              ap[u] = A[l * lda + pk[u]];
              aq[u] = A[l * lda + qk[u]];
              vp[u] = V[l * lda + pk[u]];
              vq[u] = V[l * lda + qk[u]];
            }
#pragma unroll
          for (int u = 0; u < 4; ++u)
            if (sk[u] != 0.0) {
              A[l * lda + pk[u]] = ck[u] * ap[u] - sk[u] * aq[u];
              A[l * lda + qk[u]] = sk[u] * ap[u] + ck[u] * aq[u];
              V[l * lda + pk[u]] = ck[u] * vp[u] - sk[u] * vq[u];
              V[l * lda + qk[u]] = sk[u] * vp[u] + ck[u] * vq[u];
            }
        }
      }
      __syncwarp();
    }
  }
  // ascending sort of eigenvalues (rank by counting), permuting columns of V
  // through A, which is no longer needed once its diagonal has been read
  const double d = l < n ? A[l * lda + l] : 0.0;
  int rank = 0;
  for (int j = 0; j < n; ++j) {
    const double dj = __shfl_sync(0xffffffffu, d, j);
    if (l < n && (dj < d || (dj == d && j < l))) ++rank;
  }
  if (l < n) w[rank] = d;
  __syncwarp();
  if (l < n)
    for (int j = 0; j < n; ++j) A[l * lda + j] = V[l * lda + j];
  __syncwarp();
  for (int j = 0; j < n; ++j) {
    const int rj = __shfl_sync(0xffffffffu, rank, j);
    if (l < n) V[l * lda + rj] = A[l * lda + j];
  }
  __syncwarp();
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
