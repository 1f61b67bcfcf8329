// Level-2 local generalized eigenproblems (_PC_setup_lv2_eigen,
// src/PreMixFEM_3D.c:224-421): per subdomain, the smallest en_lv1 eigenpairs
// of A_i^N v = lambda M_i v, A_i^N the subdomain-Neumann 7-point matrix and
// M_i the diagonal "mass" of the selected variant (MOD / MEAN / DIAG).
//
// SLEPc's shift-and-invert Krylov-Schur is replaced by a batched LOBPCG
// (Knyazev 2001) in one persistent launch: each CTA owns a subdomain at a
// time; its block vectors live in a private global work slab that stays in
// L2.  The preconditioner is IC(0) of (A_i^N + sigma M_i) applied with the
// same hyperplane wavefront as the level-1 solves; the basis [X W P] is
// M-orthonormalised by SVQB (Stathopoulos & Wu 2002) and the Rayleigh-Ritz
// projection is always formed and solved in FP64.  Vectors are stored in T
// (float for the mixed-precision setup, double for the plain form); a final
// FP64 Rayleigh-Ritz polish fixes the returned eigenvalues and the
// M-normalisation (v^T M v = 1, the GHEP normalisation SLEPc returns).
#include <algorithm>

#include "pmf_dense.cuh"
#include "pmf_kernels.h"

namespace pmf {

#define LB_LD 32     // leading dimension of the small matrices
#define LB_CH 32     // cell chunk of the Gram tiles
#define LB_THREADS 256

struct LbSmem {
  double GM[LB_LD * LB_LD];
  double GA[LB_LD * LB_LD];
  double U[LB_LD * LB_LD];
  double Q[LB_LD * LB_LD];
  double H[LB_LD * LB_LD];
  double V[LB_LD * LB_LD];
  double Y[LB_LD * LB_LD];
  double w[LB_LD], th[LB_LD], dsc[LB_LD], lam[LB_LD], res[LB_LD];
  double stile[LB_LD * (LB_CH + 1)];
  double ttile[LB_LD * (LB_CH + 1)];
  double red[LB_LD * 33];
  double scal[4];
  int ival[4];
};

// Column stride of the block vectors: max_cells rounded up to 64 so every
// column (and the FP64 polish buffer laid over W|P) starts 256-byte aligned.
__host__ __device__ inline int lb_ld(int max_cells) { return (max_cells + 63) & ~63; }

size_t lobpcg_work_bytes(int max_cells, int m, int prec_bytes) {
  const size_t ld = lb_ld(max_cells);
  return (size_t)6 * m * ld * prec_bytes + (size_t)3 * ld * sizeof(double);
}

__device__ __forceinline__ double avg_k(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

// G[a][b] = sum_cl wgt[cl] * S[a][cl] * T[b][cl], a < na, b < nb; S, T column-major
// with column stride nc.  All threads of the CTA must call it.
template <typename TS, typename TT>
__device__ void cta_gram(const TS* S, int na, const TT* Tm, int nb, const double* wgt, int ncells, int ld,
                         double* G, LbSmem& sm) {
  const int t = threadIdx.x;
  const bool own = t < 256;
  const int a0 = 2 * (t >> 4), b0 = 2 * (t & 15);
  double acc00 = 0, acc01 = 0, acc10 = 0, acc11 = 0;
  for (int c0 = 0; c0 < ncells; c0 += LB_CH) {
    const int ch = min(LB_CH, ncells - c0);
    for (int e = t; e < LB_LD * LB_CH; e += blockDim.x) {
      const int a = e / LB_CH, cl = e % LB_CH;
      double sv = 0.0, tv = 0.0;
      if (cl < ch) {
        if (a < na) sv = (double)S[(long long)a * ld + c0 + cl] * (wgt ? wgt[c0 + cl] : 1.0);
        if (a < nb) tv = (double)Tm[(long long)a * ld + c0 + cl];
      }
      sm.stile[a * (LB_CH + 1) + cl] = sv;
      sm.ttile[a * (LB_CH + 1) + cl] = tv;
    }
    __syncthreads();
    if (own && a0 < na && b0 < nb) {
#pragma unroll 8
      for (int cl = 0; cl < LB_CH; ++cl) {
        const double s0 = sm.stile[a0 * (LB_CH + 1) + cl], s1 = sm.stile[(a0 + 1) * (LB_CH + 1) + cl];
        const double t0 = sm.ttile[b0 * (LB_CH + 1) + cl], t1 = sm.ttile[(b0 + 1) * (LB_CH + 1) + cl];
        acc00 += s0 * t0;
        acc01 += s0 * t1;
        acc10 += s1 * t0;
        acc11 += s1 * t1;
      }
    }
    __syncthreads();
  }
  if (own) {
    if (a0 < na && b0 < nb) G[a0 * LB_LD + b0] = acc00;
    if (a0 < na && b0 + 1 < nb) G[a0 * LB_LD + b0 + 1] = acc01;
    if (a0 + 1 < na && b0 < nb) G[(a0 + 1) * LB_LD + b0] = acc10;
    if (a0 + 1 < na && b0 + 1 < nb) G[(a0 + 1) * LB_LD + b0 + 1] = acc11;
  }
  __syncthreads();
}

// C[n1 x n3] = A[n1 x n2] * B[n2 x n3] (small, ld LB_LD), optional transpose of A.
__device__ void cta_small_gemm(const double* A, bool transA, const double* B, double* C, int n1, int n2, int n3) {
  for (int e = threadIdx.x; e < n1 * n3; e += blockDim.x) {
    const int i = e / n3, j = e % n3;
    double acc = 0.0;
    for (int l = 0; l < n2; ++l) acc += (transA ? A[l * LB_LD + i] : A[i * LB_LD + l]) * B[l * LB_LD + j];
    C[i * LB_LD + j] = acc;
  }
  __syncthreads();
}

// Rayleigh-Ritz on a basis with Gram matrices GM (M) and GA (A), size nS.
// Produces Y (nS x m): coefficients of the m lowest Ritz vectors, M-orthonormal,
// and their Ritz values in sm.lam.  Returns the kept rank q (>= m on success).
__device__ int cta_rayleigh_ritz(LbSmem& sm, int nS, int m, double drop) {
  // symmetrise the Grams
  for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
    const int a = e / nS, b = e % nS;
    if (a < b) {
      const double vm = 0.5 * (sm.GM[a * LB_LD + b] + sm.GM[b * LB_LD + a]);
      sm.GM[a * LB_LD + b] = sm.GM[b * LB_LD + a] = vm;
      const double va = 0.5 * (sm.GA[a * LB_LD + b] + sm.GA[b * LB_LD + a]);
      sm.GA[a * LB_LD + b] = sm.GA[b * LB_LD + a] = va;
    }
  }
  __syncthreads();
  if (threadIdx.x < nS) sm.dsc[threadIdx.x] = 1.0 / sqrt(fmax(sm.GM[threadIdx.x * LB_LD + threadIdx.x], 1e-300));
  __syncthreads();
  for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
    const int a = e / nS, b = e % nS;
    sm.H[a * LB_LD + b] = sm.GM[a * LB_LD + b] * sm.dsc[a] * sm.dsc[b];
  }
  __syncthreads();
  if (threadIdx.x < 32) warp_jacobi_eigh(sm.H, sm.U, sm.w, nS, LB_LD);
  __syncthreads();
  if (threadIdx.x == 0) {
    int q = 0;
    const double wmax = sm.w[nS - 1];
    for (int c = 0; c < nS; ++c)
      if (sm.w[c] > drop * wmax) ++q;
    sm.ival[0] = q;
  }
  __syncthreads();
  const int q = sm.ival[0];
  // Q = D U_kept w^-1/2  (kept = last q columns)
  for (int e = threadIdx.x; e < nS * q; e += blockDim.x) {
    const int a = e / q, c = e % q, cc = nS - q + c;
    sm.Q[a * LB_LD + c] = sm.dsc[a] * sm.U[a * LB_LD + cc] / sqrt(sm.w[cc]);
  }
  __syncthreads();
  // H = Q^T GA Q
  cta_small_gemm(sm.GA, false, sm.Q, sm.V, nS, nS, q);  // V = GA Q
  cta_small_gemm(sm.Q, true, sm.V, sm.H, q, nS, q);     // H = Q^T V
  for (int e = threadIdx.x; e < q * q; e += blockDim.x) {
    const int a = e / q, b = e % q;
    if (a < b) {
      const double v = 0.5 * (sm.H[a * LB_LD + b] + sm.H[b * LB_LD + a]);
      sm.H[a * LB_LD + b] = sm.H[b * LB_LD + a] = v;
    }
  }
  __syncthreads();
  if (threadIdx.x < 32) warp_jacobi_eigh(sm.H, sm.V, sm.th, q, LB_LD);
  __syncthreads();
  const int mm = min(m, q);
  cta_small_gemm(sm.Q, false, sm.V, sm.Y, nS, q, mm);  // Y = Q V[:, :m]
  if (threadIdx.x < mm) sm.lam[threadIdx.x] = sm.th[threadIdx.x];
  __syncthreads();
  return q;
}

template <typename T>
__device__ __forceinline__ void neumann_apply_col(const Grid& g, const SubInfo& S, const double* tx, const double* ty,
                                                  const double* tz, const double* dN, const T* v, T* out,
                                                  int ncells) {
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny;
  for (int cl = threadIdx.x; cl < ncells; cl += blockDim.x) {
    const int i = cl % nx, tt = cl / nx, j = tt % ny, k = tt / ny;
    const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + (S.x0 + i);
    double a = dN[cl] * (double)v[cl];
    if (i > 0) a -= tx[cg] * (double)v[cl - 1];
    if (i < nx - 1) a -= tx[cg + 1] * (double)v[cl + 1];
    if (j > 0) a -= ty[cg] * (double)v[cl - nx];
    if (j < ny - 1) a -= ty[cg + g.M] * (double)v[cl + nx];
    if (k > 0) a -= tz[cg] * (double)v[cl - nxny];
    if (k < nz - 1) a -= tz[cg + g.MN] * (double)v[cl + nxny];
    out[cl] = (T)a;
  }
}

template <typename T>
__global__ void __launch_bounds__(512) k_lobpcg(LobpcgArgs a, unsigned char* work, size_t work_stride, T* phi,
                                                 double* evals, int* iters, int* status, int* ks, double eb) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbSmem& sm = *reinterpret_cast<LbSmem*>(smraw);
  double* u = reinterpret_cast<double*>(smraw + sizeof(LbSmem));
  const Grid g = a.g;
  const int m = a.m, k = a.k;
  unsigned char* wb = work + (size_t)blockIdx.x * work_stride;
  const int ld = a.ld;

  for (int s = blockIdx.x; s < a.nsub; s += gridDim.x) {
    const SubInfo S = a.subs[s];
    const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
    T* X = reinterpret_cast<T*>(wb);
    T* W = X + (size_t)m * ld;
    T* P = W + (size_t)m * ld;
    T* AX = P + (size_t)m * ld;
    T* AW = AX + (size_t)m * ld;
    T* AP = AW + (size_t)m * ld;
    double* Md = reinterpret_cast<double*>(AP + (size_t)m * ld);
    double* dN = Md + ld;
    double* invD = dN + ld;

    // ---- mass diagonal (src/PreMixFEM_3D.c:243-346) and Neumann diagonal
    double ratio = 0.0;
    for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
      const int i = cl % nx, tt = cl / nx, j = tt % ny, kk = tt / ny;
      const int ex = S.x0 + i, ey = S.y0 + j, ez = S.z0 + kk;
      const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
      double dn = a.db[cg];
      if (i > 0) dn += a.tx[cg];
      if (i < nx - 1) dn += a.tx[cg + 1];
      if (j > 0) dn += a.ty[cg];
      if (j < ny - 1) dn += a.ty[cg + g.M];
      if (kk > 0) dn += a.tz[cg];
      if (kk < nz - 1) dn += a.tz[cg + g.MN];
      double mv;
      if (a.eg_op == 1) {  // EIG_OP_MEAN (:332-333)
        mv = a.kx[cg] + a.ky[cg] + a.kz[cg];
      } else if (a.eg_op == 2) {  // EIG_OP_DIAG: diag(A_i^N)
        mv = dn;
      } else {  // EIG_OP_MOD with the reference's x-direction accumulation (:258-320)
        mv = 0.0;
        if (i == 0 && ex >= 1) mv += 2.0 * avg_k(a.kx[cg - 1], a.kx[cg]) / a.Hx / a.Hx;
        if (ex + 1 != g.M) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / a.Hx / a.Hx;
        if (ey >= 1) mv += 2.0 * avg_k(a.ky[cg - g.M], a.ky[cg]) / a.Hy / a.Hy;
        if (ey + 1 != g.N) mv += 2.0 * avg_k(a.ky[cg], a.ky[cg + g.M]) / a.Hy / a.Hy;
        if (ez >= 1) mv += 2.0 * avg_k(a.kz[cg - g.MN], a.kz[cg]) / a.Hz / a.Hz;
        if (ez + 1 != g.P) mv += 2.0 * avg_k(a.kz[cg], a.kz[cg + g.MN]) / a.Hz / a.Hz;
        if (i + 1 < nx) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / a.Hx / a.Hx;
        // Dirichlet extension: 2 t_b per boundary face
        if (a.db[cg] != 0.0) {
          if (a.dirichlet_mask & 1 && ex == 0) mv += 2.0 * (2.0 * a.kx[cg]) / a.Hx / a.Hx;
          if (a.dirichlet_mask & 2 && ex == g.M - 1) mv += 2.0 * (2.0 * a.kx[cg]) / a.Hx / a.Hx;
          if (a.dirichlet_mask & 4 && ey == 0) mv += 2.0 * (2.0 * a.ky[cg]) / a.Hy / a.Hy;
          if (a.dirichlet_mask & 8 && ey == g.N - 1) mv += 2.0 * (2.0 * a.ky[cg]) / a.Hy / a.Hy;
          if (a.dirichlet_mask & 16 && ez == 0) mv += 2.0 * (2.0 * a.kz[cg]) / a.Hz / a.Hz;
          if (a.dirichlet_mask & 32 && ez == g.P - 1) mv += 2.0 * (2.0 * a.kz[cg]) / a.Hz / a.Hz;
        }
        mv = mv * a.meas;
      }
      Md[cl] = mv;
      dN[cl] = dn;
      ratio = fmax(ratio, dn / mv);
    }
    // block max of dN / M: a scale for the eigenvalues (>= lambda_max / 2)
    {
      for (int o = 16; o > 0; o >>= 1) ratio = fmax(ratio, __shfl_xor_sync(0xffffffffu, ratio, o));
      if ((threadIdx.x & 31) == 0) sm.red[threadIdx.x >> 5] = ratio;
      __syncthreads();
      if (threadIdx.x == 0) {
        double r = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) r = fmax(r, sm.red[w]);
        sm.scal[0] = r > 0 ? r : 1.0;
      }
      __syncthreads();
    }
    const double lscale = sm.scal[0];
    const double sigma = a.sigma_rel * lscale;

    // ---- IC(0) pivots of A^N + sigma M (wavefront, natural order)
    {
      const int t = threadIdx.x, jj = t % ny, kk = t / ny;
      const int nplanes = nx + ny + nz - 2;
      for (int d = 0; d < nplanes; ++d) {
        const int i = d - jj - kk;
        if (t < ny * nz && i >= 0 && i < nx) {
          const int cl = (kk * ny + jj) * nx + i;
          const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + i);
          double sacc = 0.0;
          if (kk > 0) sacc += a.tz[cg] * a.tz[cg] / u[cl - nxny];
          if (jj > 0) sacc += a.ty[cg] * a.ty[cg] / u[cl - nx];
          if (i > 0) sacc += a.tx[cg] * a.tx[cg] / u[cl - 1];
          double D = dN[cl] + sigma * Md[cl] - sacc;
          if (!(D > 0.0)) D = dN[cl] + sigma * Md[cl];
          u[cl] = D;
          invD[cl] = 1.0 / D;
        }
        __syncthreads();
      }
    }

    // ---- initial block
    for (int e = threadIdx.x; e < m * nc; e += blockDim.x) {
      const int j = e / nc, cl = e % nc;
      double v;
      if (a.xinit) {
        const int i = cl % nx, tt = cl / nx, jj = tt % ny, kk = tt / ny;
        const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + i);
        v = a.xinit[cg * m + j];
      } else {
        v = hash_uniform(a.seed ^ ((unsigned long long)s << 32) ^ (unsigned long long)e);
      }
      X[(size_t)j * ld + cl] = (T)v;
    }
    __syncthreads();
    for (int j = 0; j < m; ++j) neumann_apply_col(g, S, a.tx, a.ty, a.tz, dN, X + (size_t)j * ld, AX + (size_t)j * ld, nc);
    __syncthreads();
    const double drop = sizeof(T) == 4 ? 1e-9 : 1e-13;
    cta_gram(X, m, X, m, Md, nc, ld, sm.GM, sm);
    cta_gram(X, m, AX, m, (const double*)nullptr, nc, ld, sm.GA, sm);
    cta_rayleigh_ritz(sm, m, m, drop);
    // X <- X Y, AX <- AX Y (per cell, in place)
    for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
      double xr[LB_LD], ar[LB_LD];
      for (int b = 0; b < m; ++b) {
        xr[b] = (double)X[(size_t)b * ld + cl];
        ar[b] = (double)AX[(size_t)b * ld + cl];
      }
      for (int j = 0; j < m; ++j) {
        double xn = 0.0, an = 0.0;
        for (int b = 0; b < m; ++b) {
          xn += xr[b] * sm.Y[b * LB_LD + j];
          an += ar[b] * sm.Y[b * LB_LD + j];
        }
        X[(size_t)j * ld + cl] = (T)xn;
        AX[(size_t)j * ld + cl] = (T)an;
      }
    }
    __syncthreads();

    bool hasP = false;
    int it = 0;
    bool conv = false;
    for (; it < a.max_it; ++it) {
      // residuals R = AX - M X Lambda (into W), ||R_j||_{M^-1}
      double racc[LB_LD];
      for (int j = 0; j < m; ++j) racc[j] = 0.0;
      for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
        const double mv = Md[cl];
        for (int j = 0; j < m; ++j) {
          const double r = (double)AX[(size_t)j * ld + cl] - sm.lam[j] * mv * (double)X[(size_t)j * ld + cl];
          W[(size_t)j * ld + cl] = (T)r;
          racc[j] += r * r / mv;
        }
      }
      for (int j = 0; j < m; ++j) {
        const double v = warp_sum(racc[j]);
        if ((threadIdx.x & 31) == 0) sm.red[j * 33 + (threadIdx.x >> 5)] = v;
      }
      __syncthreads();
      if (threadIdx.x < m) {
        double v = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v += sm.red[threadIdx.x * 33 + w];
        sm.res[threadIdx.x] = sqrt(v) / lscale;
      }
      __syncthreads();
      conv = true;
      for (int j = 0; j < k; ++j)
        if (!(sm.res[j] <= a.tol)) conv = false;
      if (conv) break;
      // W = T R: IC(0) solve of (A^N + sigma M) per column
      for (int j = 0; j < m; ++j) {
        T* Wj = W + (size_t)j * ld;
        for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) u[cl] = (double)Wj[cl];
        __syncthreads();
        const int t = threadIdx.x, jj = t % ny, kk = t / ny;
        const bool line = t < ny * nz;
        const long long base = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + S.x0;
        const int nplanes = nx + ny + nz - 2;
        for (int d = 0; d < nplanes; ++d) {
          const int i = d - jj - kk;
          if (line && i >= 0 && i < nx) {
            const int cl = (kk * ny + jj) * nx + i;
            const long long cg = base + i;
            double sacc = u[cl];
            if (kk > 0) sacc += a.tz[cg] * u[cl - nxny];
            if (jj > 0) sacc += a.ty[cg] * u[cl - nx];
            if (i > 0) sacc += a.tx[cg] * u[cl - 1];
            u[cl] = sacc * invD[cl];
          }
          __syncthreads();
        }
        for (int d = nplanes - 1; d >= 0; --d) {
          const int i = d - jj - kk;
          if (line && i >= 0 && i < nx) {
            const int cl = (kk * ny + jj) * nx + i;
            const long long cg = base + i;
            double sacc = 0.0;
            if (i < nx - 1) sacc += a.tx[cg + 1] * u[cl + 1];
            if (jj < ny - 1) sacc += a.ty[cg + g.M] * u[cl + nx];
            if (kk < nz - 1) sacc += a.tz[cg + g.MN] * u[cl + nxny];
            u[cl] = u[cl] + sacc * invD[cl];
          }
          __syncthreads();
        }
        for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) Wj[cl] = (T)u[cl];
        __syncthreads();
      }
      for (int j = 0; j < m; ++j)
        neumann_apply_col(g, S, a.tx, a.ty, a.tz, dN, W + (size_t)j * ld, AW + (size_t)j * ld, nc);
      __syncthreads();
      const int nS = hasP ? 3 * m : 2 * m;
      cta_gram(X, nS, X, nS, Md, nc, ld, sm.GM, sm);
      cta_gram(X, nS, AX, nS, (const double*)nullptr, nc, ld, sm.GA, sm);
      const int q = cta_rayleigh_ritz(sm, nS, m, drop);
      if (q < m) {  // basis collapsed: restart without P
        hasP = false;
        continue;
      }
      // X <- S Y, P <- [W P] Y_WP, same for AX / AP (per cell, in place)
      for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
        double xr[3 * 10];
        for (int b = 0; b < nS; ++b) xr[b] = (double)X[(size_t)b * ld + cl];
        for (int j = 0; j < m; ++j) {
          double pn = 0.0;
          for (int b = m; b < nS; ++b) pn += xr[b] * sm.Y[b * LB_LD + j];
          double xn = pn;
          for (int b = 0; b < m; ++b) xn += xr[b] * sm.Y[b * LB_LD + j];
          X[(size_t)j * ld + cl] = (T)xn;
          P[(size_t)j * ld + cl] = (T)pn;
        }
        for (int b = 0; b < nS; ++b) xr[b] = (double)AX[(size_t)b * ld + cl];
        for (int j = 0; j < m; ++j) {
          double pn = 0.0;
          for (int b = m; b < nS; ++b) pn += xr[b] * sm.Y[b * LB_LD + j];
          double xn = pn;
          for (int b = 0; b < m; ++b) xn += xr[b] * sm.Y[b * LB_LD + j];
          AX[(size_t)j * ld + cl] = (T)xn;
          AP[(size_t)j * ld + cl] = (T)pn;
        }
      }
      __syncthreads();
      hasP = true;
    }

    // ---- final FP64 Rayleigh-Ritz polish on X (A X recomputed in FP64 into the W/P slab)
    double* AX64 = reinterpret_cast<double*>(W);
    {
      for (int j = 0; j < m; ++j) {
        const T* v = X + (size_t)j * ld;
        double* o = AX64 + (size_t)j * ld;
        for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
          const int i = cl % nx, tt = cl / nx, jj = tt % ny, kk = tt / ny;
          const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + i);
          double av = dN[cl] * (double)v[cl];
          if (i > 0) av -= a.tx[cg] * (double)v[cl - 1];
          if (i < nx - 1) av -= a.tx[cg + 1] * (double)v[cl + 1];
          if (jj > 0) av -= a.ty[cg] * (double)v[cl - nx];
          if (jj < ny - 1) av -= a.ty[cg + g.M] * (double)v[cl + nx];
          if (kk > 0) av -= a.tz[cg] * (double)v[cl - nxny];
          if (kk < nz - 1) av -= a.tz[cg + g.MN] * (double)v[cl + nxny];
          o[cl] = av;
        }
      }
      __syncthreads();
      cta_gram(X, m, X, m, Md, nc, ld, sm.GM, sm);
      cta_gram(X, m, AX64, m, (const double*)nullptr, nc, ld, sm.GA, sm);
      cta_rayleigh_ritz(sm, m, m, 1e-14);
    }
    // adaptive count (:369-383) and output
    if (threadIdx.x == 0) {
      int num = k;
      for (int j = 0; j < k; ++j)
        if (sm.lam[j] >= eb) {
          num = j + 1;
          break;
        }
      sm.ival[1] = num;
      ks[s] = num;
      iters[s] = it;
      status[s] = conv ? 0 : 1;
    }
    __syncthreads();
    const int num = sm.ival[1];
    if (threadIdx.x < k) evals[(long long)s * k + threadIdx.x] = sm.lam[threadIdx.x];
    for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
      const int i = cl % nx, tt = cl / nx, jj = tt % ny, kk = tt / ny;
      const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + i);
      double xr[LB_LD];
      for (int b = 0; b < m; ++b) xr[b] = (double)X[(size_t)b * ld + cl];
      for (int j = 0; j < a.kmax; ++j) {
        double v = 0.0;
        if (j < num)
          for (int b = 0; b < m; ++b) v += xr[b] * sm.Y[b * LB_LD + j];
        phi[cg * a.kmax + j] = (T)v;
      }
    }
    __syncthreads();
  }
}

template <typename T>
void launch_lobpcg(const LobpcgArgs& a_in, int nblocks, void* work, T* phi, double* evals, int* iters, int* status,
                   int* ks, double eb, int max_cells, int max_lines, cudaStream_t st) {
  LobpcgArgs a = a_in;
  a.ld = lb_ld(max_cells);
  const int threads = std::max(LB_THREADS, ((max_lines + 31) / 32) * 32);
  const size_t smem = sizeof(LbSmem) + (size_t)max_cells * sizeof(double);
  cudaFuncSetAttribute(k_lobpcg<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const size_t stride = (lobpcg_work_bytes(max_cells, a.m, sizeof(T)) + 255) & ~(size_t)255;
  k_lobpcg<T><<<nblocks, threads, smem, st>>>(a, (unsigned char*)work, stride, phi, evals, iters, status, ks, eb);
}
template void launch_lobpcg<float>(const LobpcgArgs&, int, void*, float*, double*, int*, int*, int*, double, int, int,
                                   cudaStream_t);
template void launch_lobpcg<double>(const LobpcgArgs&, int, void*, double*, double*, int*, int*, int*, double, int,
                                    int, cudaStream_t);

}  // namespace pmf
