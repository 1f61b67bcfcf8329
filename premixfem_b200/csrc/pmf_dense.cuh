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

// Same method executed by a whole CTA (blockDim.x >= 32): the lanes of warp 0
// compute the round's rotations, then every thread applies a share of the
// row rotations (J^T A), and after a barrier a share of the column
// rotations (A J) and of V J.  All threads must call it; ip (>= 32 ints) and
// dp (>= 32 doubles) are shared-memory scratch.  Rotations are computed in
// FP64 (quadratic convergence); sweeps stop when every off-diagonal entry is
// below tol ||A||_F.
__device__ inline void cta_jacobi_eigh(double* A, double* V, double* w, int n, int lda, int* ip, double* dp,
                                       double tol = 1e-14, int max_sweeps = 20) {
  const int t = threadIdx.x, T = blockDim.x;
  for (int e = t; e < n * n; e += T) V[(e / n) * lda + (e % n)] = (e / n == e % n) ? 1.0 : 0.0;
  if (t < 32) {
    double f = 0.0;
    for (int i = t; i < n; i += 32)
      for (int j = 0; j < n; ++j) f += A[i * lda + j] * A[i * lda + j];
    f = warp_sum(f);
    if (t == 0) dp[31] = sqrt(f);
  }
  __syncthreads();
  const double fro = dp[31];
  const int ne = n + (n & 1);
  const int half = ne >> 1;
  int* rp = ip;
  int* rq = ip + 16;
  double* rc = dp;
  double* rs = dp + 16;
  for (int sweep = 0; sweep < max_sweeps && n > 1; ++sweep) {
    int bad = 0;
    for (int e = t; e < n * n; e += T) {
      const int i = e / n, j = e % n;
      if (i != j && fabs(A[i * lda + j]) > tol * fro) bad = 1;
    }
    if (!__syncthreads_or(bad)) break;
    for (int round = 0; round < ne - 1; ++round) {
      if (t < half) {
        const int pa = t, pb = ne - 1 - t;
        int p = pa == 0 ? 0 : ((pa - 1 + round) % (ne - 1)) + 1;
        int q = ((pb - 1 + round) % (ne - 1)) + 1;
        if (p > q) {
          const int x = p;
          p = q;
          q = x;
        }
        double c = 1.0, s = 0.0;
        if (q < n) {
          const double apq = A[p * lda + q];
          const double app = A[p * lda + p];
          const double aqq = A[q * lda + q];
          if (fabs(apq) > 1e-300 && fabs(apq) > 1e-18 * sqrt(fabs(app * aqq))) {
            const double theta = (aqq - app) / (2.0 * apq);
            const double tt = (theta >= 0.0 ? 1.0 : -1.0) / (fabs(theta) + sqrt(theta * theta + 1.0));
            c = 1.0 / sqrt(tt * tt + 1.0);
            s = tt * c;
          }
        } else {
          q = p;
        }
        rp[t] = p;
        rq[t] = q;
        rc[t] = c;
        rs[t] = s;
      }
      __syncthreads();
      for (int e = t; e < half * n; e += T) {  // rows p, q
        const int k = e / n, col = e % n;
        const double s = rs[k];
        if (s == 0.0) continue;
        const int p = rp[k], q = rq[k];
        const double c = rc[k];
        const double a1 = A[p * lda + col], a2 = A[q * lda + col];
        A[p * lda + col] = c * a1 - s * a2;
        A[q * lda + col] = s * a1 + c * a2;
      }
      __syncthreads();
      for (int e = t; e < half * n; e += T) {  // columns p, q and V
        const int k = e / n, row = e % n;
        const double s = rs[k];
        if (s == 0.0) continue;
        const int p = rp[k], q = rq[k];
        const double c = rc[k];
        const double a1 = A[row * lda + p], a2 = A[row * lda + q];
        A[row * lda + p] = c * a1 - s * a2;
        A[row * lda + q] = s * a1 + c * a2;
        const double v1 = V[row * lda + p], v2 = V[row * lda + q];
        V[row * lda + p] = c * v1 - s * v2;
        V[row * lda + q] = s * v1 + c * v2;
      }
      __syncthreads();
    }
  }
  // ascending order: rank of each diagonal entry, then permute V's columns through A
  for (int l = t; l < n; l += T) {
    const double d = A[l * lda + l];
    int rank = 0;
    for (int j = 0; j < n; ++j) {
      const double dj = A[j * lda + j];
      if (dj < d || (dj == d && j < l)) ++rank;
    }
    ip[l] = rank;
  }
  __syncthreads();
  for (int l = t; l < n; l += T) w[ip[l]] = A[l * lda + l];
  __syncthreads();
  for (int e = t; e < n * n; e += T) A[(e / n) * lda + (e % n)] = V[(e / n) * lda + (e % n)];
  __syncthreads();
  for (int e = t; e < n * n; e += T) {
    const int row = e / n, j = e % n;
    V[row * lda + ip[j]] = A[row * lda + j];
  }
  __syncthreads();
}

// Cheap deterministic pseudo-random number in [-1, 1) (splitmix64 finaliser).
__device__ __forceinline__ double hash_uniform(unsigned long long a) {
  a += 0x9E3779B97F4A7C15ull;
  a = (a ^ (a >> 30)) * 0xBF58476D1CE4E5B9ull;
  a = (a ^ (a >> 27)) * 0x94D049BB133111EBull;
  a ^= a >> 31;
  return (double)(a >> 11) * (2.0 / 9007199254740992.0) - 1.0;
}

// Lowest m eigenpairs of a symmetric q x q matrix (q <= 32, m <= 16), by the
// whole CTA (blockDim.x >= 256, multiple of 32):
//   1. Householder tridiagonalisation T = Q^T A Q (Golub & Van Loan, Alg. 8.3.1);
//   2. eigenvalues by Sturm-count multisection: warp w owns eigenvalue j = w
//      (+8, ...), its 32 lanes evaluate the Sturm count at 32 interior points
//      of the current bracket, so every round shrinks the bracket 33-fold;
//   3. eigenvectors of T by inverse iteration (tridiagonal LU with partial
//      pivoting, three steps), then modified Gram-Schmidt in ascending order;
//   4. back-transformation by the stored reflectors.
// A (destroyed), V (q x m eigenvectors, columns, ld lda), w (m eigenvalues,
// ascending).  sc: shared scratch of >= 4 * 32 * 33 + 8 * 32 doubles.
__device__ inline double sturm_count(const double* d, const double* e2, int q, double x, double pivmin) {
  int cnt = 0;
  double t = d[0] - x;
  if (fabs(t) < pivmin) t = -pivmin;
  if (t < 0.0) ++cnt;
  for (int i = 1; i < q; ++i) {
    t = (d[i] - x) - e2[i - 1] / t;
    if (fabs(t) < pivmin) t = -pivmin;
    if (t < 0.0) ++cnt;
  }
  return (double)cnt;
}

static __device__ __noinline__ void cta_sym_lowest(double* A, double* V, double* w, int q, int m, int lda, double* sc) {
  const int t = threadIdx.x, T = blockDim.x;
  const int lane = t & 31, wid = t >> 5, nw = T >> 5;
  double* Hv = sc;                // reflectors, row k holds v_k (length q)
  double* Z = sc + 32 * 33;       // eigenvectors of T, column j at Z[i*33 + j]
  double* pv = Z + 32 * 33;       // p / w work vector
  double* dg = pv + 64;           // diagonal of T
  double* of = dg + 32;           // off-diagonal e_i = T[i+1][i]
  double* e2 = of + 32;           // e_i^2
  double* beta = e2 + 32;         // reflector coefficients
  double* misc = beta + 32;       // scalars
  // ---- 1. tridiagonalisation
  for (int k = 0; k + 2 < q; ++k) {
    const int n1 = q - k - 1;
    if (wid == 0) {
      double x = lane < n1 ? A[(k + 1 + lane) * lda + k] : 0.0;
      double nrm2 = warp_sum(x * x);
      const double x0 = __shfl_sync(0xffffffffu, x, 0);
      const double nrm = sqrt(nrm2);
      double b = 0.0, alpha = x0;
      if (nrm2 > 1e-300) {
        alpha = x0 >= 0.0 ? -nrm : nrm;
        const double v0 = x0 - alpha;
        const double vv = nrm2 - x0 * x0 + v0 * v0;
        b = vv > 0.0 ? 2.0 / vv : 0.0;
        if (lane < n1) Hv[k * 33 + lane] = lane == 0 ? v0 : x;
      } else if (lane < n1) {
        Hv[k * 33 + lane] = 0.0;
      }
      if (lane == 0) {
        beta[k] = b;
        misc[0] = alpha;
      }
    }
    __syncthreads();
    const double b = beta[k];
    if (b != 0.0) {
      // p = b * A_trail v
      for (int i = t; i < n1; i += T) {
        double acc = 0.0;
        for (int j = 0; j < n1; ++j) acc += A[(k + 1 + i) * lda + (k + 1 + j)] * Hv[k * 33 + j];
        pv[i] = b * acc;
      }
      __syncthreads();
      if (wid == 0) {
        double pvv = 0.0;
        for (int i = lane; i < n1; i += 32) pvv += pv[i] * Hv[k * 33 + i];
        pvv = warp_sum(pvv);
        if (lane == 0) misc[1] = 0.5 * b * pvv;
      }
      __syncthreads();
      const double K = misc[1];
      for (int i = t; i < n1; i += T) pv[32 + i] = pv[i] - K * Hv[k * 33 + i];  // w = p - K v
      __syncthreads();
      for (int e = t; e < n1 * n1; e += T) {
        const int i = e / n1, j = e % n1;
        A[(k + 1 + i) * lda + (k + 1 + j)] -= Hv[k * 33 + i] * pv[32 + j] + pv[32 + i] * Hv[k * 33 + j];
      }
    }
    if (t == 0) A[(k + 1) * lda + k] = misc[0];
    __syncthreads();
  }
  for (int i = t; i < q; i += T) {
    dg[i] = A[i * lda + i];
    const double ei = i + 1 < q ? A[(i + 1) * lda + i] : 0.0;
    of[i] = ei;
    e2[i] = ei * ei;
  }
  __syncthreads();
  // ---- 2. multisection for the m lowest eigenvalues
  if (t == 0) {
    double lo = 1e300, hi = -1e300, emax = 0.0;
    for (int i = 0; i < q; ++i) {
      const double r = (i > 0 ? fabs(of[i - 1]) : 0.0) + (i + 1 < q ? fabs(of[i]) : 0.0);
      lo = fmin(lo, dg[i] - r);
      hi = fmax(hi, dg[i] + r);
      emax = fmax(emax, fabs(dg[i]) + r);
    }
    const double pad = 1e-14 * fmax(emax, 1e-300);
    misc[2] = lo - pad;
    misc[3] = hi + pad;
    misc[4] = fmax(emax, 1e-300) * 2.3e-16 * 2.3e-16 + 1e-300;  // pivmin
    misc[5] = emax;
  }
  __syncthreads();
  const double pivmin = misc[4], emax = misc[5];
  for (int j = wid; j < m; j += nw) {
    double lo = misc[2], hi = misc[3];
    for (int round = 0; round < 16; ++round) {
      if (hi - lo <= 1e-14 * fmax(fabs(lo), fabs(hi)) + 1e-17 * emax) break;
      const double x = lo + (hi - lo) * (double)(lane + 1) / 33.0;
      const double cnt = sturm_count(dg, e2, q, x, pivmin);
      const unsigned ge = __ballot_sync(0xffffffffu, cnt >= (double)(j + 1));
      const int p = ge ? __ffs(ge) - 1 : 32;  // first point with count >= j+1
      const double nlo = p == 0 ? lo : lo + (hi - lo) * (double)p / 33.0;
      const double nhi = p == 32 ? hi : lo + (hi - lo) * (double)(p + 1) / 33.0;
      lo = nlo;
      hi = nhi;
    }
    if (lane == 0) w[j] = 0.5 * (lo + hi);
  }
  __syncthreads();
  // ---- 3. inverse iteration on T for each eigenvalue (one thread per eigenvector)
  if (t < m) {
    const int j = t;
    // shift slightly below the eigenvalue so that the factorisation is nonsingular
    const double lam = w[j] - 4e-15 * fmax(emax, 1e-300) * (1 + j);
    double z[32], dl[32], du[32], du2[32], dd[32];
    int piv[32];
    for (int i = 0; i < q; ++i) z[i] = hash_uniform(0x5bd1e995ull * (j + 1) + i);
    // LU of (T - lam I) with partial pivoting (tridiagonal: dgttrf pattern)
    for (int i = 0; i < q; ++i) {
      dd[i] = dg[i] - lam;
      dl[i] = i + 1 < q ? of[i] : 0.0;
      du[i] = i + 1 < q ? of[i] : 0.0;
      du2[i] = 0.0;
    }
    for (int i = 0; i + 1 < q; ++i) {
      if (fabs(dd[i]) >= fabs(dl[i])) {
        piv[i] = 0;
        double f = dd[i] != 0.0 ? dl[i] / dd[i] : 0.0;
        dl[i] = f;
        dd[i + 1] -= f * du[i];
      } else {
        piv[i] = 1;
        const double f = dd[i] / dl[i];
        dd[i] = dl[i];
        dl[i] = f;
        const double tmp = du[i];
        du[i] = dd[i + 1];
        dd[i + 1] = tmp - f * dd[i + 1];
        if (i + 2 < q) {
          du2[i] = du[i + 1];
          du[i + 1] = -f * du[i + 1];
        }
      }
    }
    const double tiny = 1e-300 + 1e-16 * fmax(emax, 1e-300) * 1e-3;
    for (int i = 0; i < q; ++i)
      if (fabs(dd[i]) < tiny) dd[i] = dd[i] < 0 ? -tiny : tiny;
    for (int itr = 0; itr < 3; ++itr) {
      // forward: apply L^-1 with pivots
      for (int i = 0; i + 1 < q; ++i) {
        if (piv[i]) {
          const double tmp = z[i];
          z[i] = z[i + 1];
          z[i + 1] = tmp - dl[i] * z[i];
        } else {
          z[i + 1] -= dl[i] * z[i];
        }
      }
      // backward: U z = y (U has diagonals dd, du, du2)
      for (int i = q - 1; i >= 0; --i) {
        double s = z[i];
        if (i + 1 < q) s -= du[i] * z[i + 1];
        if (i + 2 < q) s -= du2[i] * z[i + 2];
        z[i] = s / dd[i];
      }
      double nrm = 0.0;
      for (int i = 0; i < q; ++i) nrm += z[i] * z[i];
      nrm = 1.0 / sqrt(fmax(nrm, 1e-300));
      for (int i = 0; i < q; ++i) z[i] *= nrm;
    }
    for (int i = 0; i < q; ++i) Z[i * 33 + j] = z[i];
  }
  __syncthreads();
  // modified Gram-Schmidt in ascending order (warp 0, lanes over components)
  if (wid == 0) {
    for (int j = 0; j < m; ++j) {
      double zj = lane < q ? Z[lane * 33 + j] : 0.0;
      for (int i = 0; i < j; ++i) {
        const double zi = lane < q ? Z[lane * 33 + i] : 0.0;
        const double d = warp_sum(zi * zj);
        zj -= d * zi;
      }
      const double nrm = sqrt(fmax(warp_sum(zj * zj), 1e-300));
      if (lane < q) Z[lane * 33 + j] = zj / nrm;
      __syncwarp();
    }
  }
  __syncthreads();
  // ---- 4. back-transformation: y = P_0 P_1 ... P_{q-3} z
  for (int k = q - 3; k >= 0; --k) {
    const double b = beta[k];
    if (b != 0.0) {
      const int n1 = q - k - 1;
      if (t < m) {
        double d = 0.0;
        for (int i = 0; i < n1; ++i) d += Hv[k * 33 + i] * Z[(k + 1 + i) * 33 + t];
        pv[t] = b * d;
      }
      __syncthreads();
      for (int e = t; e < m * n1; e += T) {
        const int j = e / n1, i = e % n1;
        Z[(k + 1 + i) * 33 + j] -= pv[j] * Hv[k * 33 + i];
      }
    }
    __syncthreads();
  }
  for (int e = t; e < q * m; e += T) {
    const int i = e / m, j = e % m;
    V[i * lda + j] = Z[i * 33 + j];
  }
  __syncthreads();
}

}  // namespace pmf
