// Level-2 local generalized eigenproblems (_PC_setup_lv2_eigen,
// src/PreMixFEM_3D.c:224-421): per subdomain, the smallest en_lv1 eigenpairs
// of A_i^N v = lambda M_i v, A_i^N the subdomain-Neumann 7-point matrix and
// M_i the diagonal "mass" of the selected variant (MOD / MEAN / DIAG).
//
// SLEPc's shift-and-invert Krylov-Schur is replaced by a batched LOBPCG
// (Knyazev 2001) in one persistent launch: each CTA owns one subdomain at a
// time and keeps its block vectors in a private global slab (L2-resident).
// Preconditioner: IC(0) of (A_i^N + sigma M_i), applied as a hyperplane
// wavefront with its coefficients and all active vectors held in shared
// memory (FP32: it only shapes the search directions).  The basis [X W P]
// is orthonormalised in the M inner product (Cholesky QR, SVQB of Stathopoulos
// & Wu 2002 when it is nearly dependent) and the Rayleigh-Ritz projection is
// formed and solved in FP64: the Grams and the basis update run on the FP64
// tensor cores (mma.sync m8n8k4), the projected eigenproblem by Householder
// tridiagonalisation and multisection.  Converged vectors are soft-locked.
// X, W, P are stored in T (float for the mixed-precision setup, double for
// the plain form); their A-images are always FP64, so the projection stays
// consistent without recomputation.  A final FP64 Rayleigh-Ritz fixes the
// returned eigenvalues and the normalisation v^T M v = 1 (the GHEP
// normalisation SLEPc returns).
#include <algorithm>
#include <cstddef>
#include <cstdio>
#include <cstdlib>

#include "pmf_bulk.cuh"
#include "pmf_dense.cuh"
#include "pmf_kernels.h"
#include "tune.h"

namespace pmf {

#define LB_LD 32  // leading dimension of the small matrices
#define LB_CH 32  // cell chunk of the Gram tiles
#define LB_MM 10  // largest block size m (3m <= 32)
#define LB_THREADS 256

struct __align__(16) LbSmall {
  double w[32], th[32], dsc[32], lam[32], res[32], jac[64], scal[8];
  int ival[8], act[32], ival2[32];
};
struct LbMats {
  double GM[LB_LD * LB_LD], GA[LB_LD * LB_LD], U[LB_LD * LB_LD], Q[LB_LD * LB_LD], H[LB_LD * LB_LD],
      V[LB_LD * LB_LD], Y[LB_LD * LB_LD];
  double stile[LB_LD * (LB_CH + 1)], ttile[LB_LD * (LB_CH + 1)], atile[LB_LD * (LB_CH + 1)];
  double red[32 * 33];
};

__host__ __device__ inline int lb_ld(int max_cells) { return (max_cells + 63) & ~63; }

size_t lobpcg_work_bytes(int max_cells, int m, int prec_bytes) {
  const size_t ld = lb_ld(max_cells);
  // X, W, P in the storage precision; their A-images always FP64; M, Neumann diagonals
  return (size_t)3 * m * ld * prec_bytes + (size_t)3 * m * ld * sizeof(double) + (size_t)3 * ld * sizeof(double) +
         (size_t)4 * ld * sizeof(float);  // + IC(0) sweep coefficients (batched solver)
}

__device__ __forceinline__ double avg_k(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

// Four consecutive cells of a column (16-byte aligned for float, 2 x 16 bytes for double).
__device__ __forceinline__ void ld4(const float* p, double v[4]) {
  const float4 f = *reinterpret_cast<const float4*>(p);
  v[0] = f.x;
  v[1] = f.y;
  v[2] = f.z;
  v[3] = f.w;
}
__device__ __forceinline__ void ld4(const double* p, double v[4]) {
  const double2 a = *reinterpret_cast<const double2*>(p);
  const double2 b = *reinterpret_cast<const double2*>(p + 2);
  v[0] = a.x;
  v[1] = a.y;
  v[2] = b.x;
  v[3] = b.y;
}
__device__ __forceinline__ void st4(float* p, const double v[4]) {
  *reinterpret_cast<float4*>(p) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
}
__device__ __forceinline__ void st4(double* p, const double v[4]) {
  *reinterpret_cast<double2*>(p) = make_double2(v[0], v[1]);
  *reinterpret_cast<double2*>(p + 2) = make_double2(v[2], v[3]);
}

// u[b][cl] = (float) src[(j0 + b) * ld + cl] for b < nb, cl < nc (vectorised copy into shared memory).
template <typename T>
__device__ __forceinline__ void load_cols_to_smem(const T* src, size_t ld, int nb, int nc, float* u, int ldc) {
  const int ng = nc >> 2;
  for (int e = threadIdx.x; e < nb * ng; e += blockDim.x) {
    const int b = e / ng, cl = (e % ng) * 4;
    double v[4];
    ld4(src + (size_t)b * ld + cl, v);
    *reinterpret_cast<float4*>(u + (size_t)b * ldc + cl) = make_float4((float)v[0], (float)v[1], (float)v[2], (float)v[3]);
  }
  for (int e = threadIdx.x; e < nb * (nc - 4 * ng); e += blockDim.x) {
    const int b = e / (nc - 4 * ng), cl = 4 * ng + e % (nc - 4 * ng);
    u[(size_t)b * ldc + cl] = (float)src[(size_t)b * ld + cl];
  }
}
template <typename T>
__device__ __forceinline__ void store_cols_from_smem(T* dst, size_t ld, int nb, int nc, const float* u, int ldc) {
  const int ng = nc >> 2;
  for (int e = threadIdx.x; e < nb * ng; e += blockDim.x) {
    const int b = e / ng, cl = (e % ng) * 4;
    const float4 f = *reinterpret_cast<const float4*>(u + (size_t)b * ldc + cl);
    const double v[4] = {f.x, f.y, f.z, f.w};
    st4(dst + (size_t)b * ld + cl, v);
  }
  for (int e = threadIdx.x; e < nb * (nc - 4 * ng); e += blockDim.x) {
    const int b = e / (nc - 4 * ng), cl = 4 * ng + e % (nc - 4 * ng);
    dst[(size_t)b * ld + cl] = (T)u[(size_t)b * ldc + cl];
  }
}

// Column c of a segmented block [A0 (n0 cols) | A1 (n1 cols) | A2 (n2 cols)], stride ld.
template <typename T>
struct Seg3 {
  const T* b[3];
  int n[3];
  int ld;
  __device__ __forceinline__ const T* col(int c) const {
    if (c < n[0]) return b[0] + (size_t)c * ld;
    c -= n[0];
    if (c < n[1]) return b[1] + (size_t)c * ld;
    return b[2] + (size_t)(c - n[1]) * ld;
  }
  __device__ __forceinline__ int total() const { return n[0] + n[1] + n[2]; }
};

// G[a][b] = sum_cl wgt[cl] * S_a[cl] * T_b[cl] (a, b < 32), register-tiled 2x2 per thread.
// Tiles of 32 cells are staged through shared memory; the next tile is loaded
// into registers while the current one is multiplied (one tile of prefetch).
template <typename TS, typename TT>
__device__ void cta_gram(const Seg3<TS>& S, const Seg3<TT>& Tm, const double* wgt, int ncells, double* G,
                         LbMats& mt) {
  const int t = threadIdx.x;
  const bool own = t < 256;
  const int na = S.total(), nb = Tm.total();
  const int a0 = 2 * (t >> 4), b0 = 2 * (t & 15);
  const int lc = t & 31, ab = (t >> 5) & 7;
  const TS* sp[4];
  const TT* tp[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int a = ab + 8 * r;
    sp[r] = (own && a < na) ? S.col(a) : nullptr;
    tp[r] = (own && a < nb) ? Tm.col(a) : nullptr;
  }
  double sv[4], tv[4];
  auto load = [&](int c0) {
    const int c = c0 + lc;
    const bool in = c < ncells;
    const double wv = (in && wgt) ? wgt[c] : 1.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      sv[r] = (in && sp[r]) ? (double)sp[r][c] * wv : 0.0;
      tv[r] = (in && tp[r]) ? (double)tp[r][c] : 0.0;
    }
  };
  load(0);
  double acc00 = 0, acc01 = 0, acc10 = 0, acc11 = 0;
  for (int c0 = 0; c0 < ncells; c0 += LB_CH) {
    if (own) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        mt.stile[(ab + 8 * r) * (LB_CH + 1) + lc] = sv[r];
        mt.ttile[(ab + 8 * r) * (LB_CH + 1) + lc] = tv[r];
      }
    }
    __syncthreads();
    if (c0 + LB_CH < ncells) load(c0 + LB_CH);
    if (own && a0 < na && b0 < nb) {
#pragma unroll 8
      for (int cl = 0; cl < LB_CH; ++cl) {
        const double s0 = mt.stile[a0 * (LB_CH + 1) + cl], s1 = mt.stile[(a0 + 1) * (LB_CH + 1) + cl];
        const double t0 = mt.ttile[b0 * (LB_CH + 1) + cl], t1 = mt.ttile[(b0 + 1) * (LB_CH + 1) + cl];
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

// Both Rayleigh-Ritz Grams in one pass over the cells:
//   GM[a][b] = sum_cl wgt[cl] S_a[cl] S_b[cl],   GA[a][b] = sum_cl S_a[cl] AS_b[cl].
// Same tiling and one-tile register prefetch as cta_gram.
template <typename TS, typename TA>
__device__ void cta_gram2(const Seg3<TS>& S, const Seg3<TA>& AS, const double* wgt, int ncells, double* GM,
                          double* GA, LbMats& mt) {
  const int t = threadIdx.x;
  const bool own = t < 256;
  const int ns = S.total();
  const int a0 = 2 * (t >> 4), b0 = 2 * (t & 15);
  const int lc = t & 31, ab = (t >> 5) & 7;
  const TS* sp[4];
  const TA* ap[4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int a = ab + 8 * r;
    sp[r] = (own && a < ns) ? S.col(a) : nullptr;
    ap[r] = (own && a < ns) ? AS.col(a) : nullptr;
  }
  double sv[4], av[4], wv;
  auto load = [&](int c0) {
    const int c = c0 + lc;
    const bool in = c < ncells;
    wv = in ? wgt[c] : 0.0;
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      sv[r] = (in && sp[r]) ? (double)sp[r][c] : 0.0;
      av[r] = (in && ap[r]) ? (double)ap[r][c] : 0.0;
    }
  };
  load(0);
  double m00 = 0, m01 = 0, m10 = 0, m11 = 0, g00 = 0, g01 = 0, g10 = 0, g11 = 0;
  const bool act = own && a0 < ns && b0 < ns;
  for (int c0 = 0; c0 < ncells; c0 += LB_CH) {
    if (own) {
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int row = (ab + 8 * r) * (LB_CH + 1) + lc;
        mt.stile[row] = sv[r] * wv;
        mt.ttile[row] = sv[r];
        mt.atile[row] = av[r];
      }
    }
    __syncthreads();
    if (c0 + LB_CH < ncells) load(c0 + LB_CH);
    if (act) {
#pragma unroll 4
      for (int cl = 0; cl < LB_CH; ++cl) {
        const double w0 = mt.stile[a0 * (LB_CH + 1) + cl], w1 = mt.stile[(a0 + 1) * (LB_CH + 1) + cl];
        const double s0 = mt.ttile[a0 * (LB_CH + 1) + cl], s1 = mt.ttile[(a0 + 1) * (LB_CH + 1) + cl];
        const double t0 = mt.ttile[b0 * (LB_CH + 1) + cl], t1 = mt.ttile[(b0 + 1) * (LB_CH + 1) + cl];
        const double q0 = mt.atile[b0 * (LB_CH + 1) + cl], q1 = mt.atile[(b0 + 1) * (LB_CH + 1) + cl];
        m00 += w0 * t0;
        m01 += w0 * t1;
        m10 += w1 * t0;
        m11 += w1 * t1;
        g00 += s0 * q0;
        g01 += s0 * q1;
        g10 += s1 * q0;
        g11 += s1 * q1;
      }
    }
    __syncthreads();
  }
  if (act) {
    GM[a0 * LB_LD + b0] = m00;
    GA[a0 * LB_LD + b0] = g00;
    if (b0 + 1 < ns) {
      GM[a0 * LB_LD + b0 + 1] = m01;
      GA[a0 * LB_LD + b0 + 1] = g01;
    }
    if (a0 + 1 < ns) {
      GM[(a0 + 1) * LB_LD + b0] = m10;
      GA[(a0 + 1) * LB_LD + b0] = g10;
    }
    if (a0 + 1 < ns && b0 + 1 < ns) {
      GM[(a0 + 1) * LB_LD + b0 + 1] = m11;
      GA[(a0 + 1) * LB_LD + b0 + 1] = g11;
    }
  }
  __syncthreads();
}

// FP64 tensor-core MMA, D(8x8) += A(8x4) * B(4x8) (PTX mma.sync m8n8k4 f64).
// Fragments: lane l holds A[l/4][l%4], B[l%4][l/4], C/D[l/4][2(l%4)], C/D[l/4][2(l%4)+1].
__device__ __forceinline__ void dmma884(double& d0, double& d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// Both Rayleigh-Ritz Grams on the FP64 tensor cores:
//   GM = (w S)^T S,  GA = S^T (A S),  S = [X W P] (ns <= 32 columns).
// Warp w takes cells 4w + 32i; for each group of 4 cells lane l loads basis
// row 8t + l/4 at cell l%4, which is at once its A fragment (row of S^T) and
// its B fragment (column of S / AS): no shared-memory staging.  The per-warp
// partial tiles are reduced in a fixed order through shared memory, so the
// result is deterministic.  red: >= 8 * 32 * 32 doubles.
template <typename TS, typename TA, int NT>
__device__ __noinline__ void cta_gram2_mma(const Seg3<TS> S, const Seg3<TA> AS, const double* wgt, int ncells,
                                           double* GM, double* GA, double* red) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int r = lane >> 2, cq = lane & 3;
  const int ns = S.total();
  const int nt = (ns + 7) >> 3;
  const TS* sp[NT];
  const TA* ap[NT];
#pragma unroll
  for (int ta = 0; ta < NT; ++ta) {
    const int a = 8 * ta + r;
    sp[ta] = (ta < nt && a < ns) ? S.col(a) : nullptr;
    ap[ta] = (ta < nt && a < ns) ? AS.col(a) : nullptr;
  }
  // Only the tiles ta <= tb are accumulated (both Grams are symmetric); the
  // reduction mirrors them.  NT is the exact tile count when nt == NT (the
  // batched solver dispatches on it); tiles past nt load zeros.
  constexpr int NP = NT * (NT + 1) / 2;
  double cm[NP][2], ca[NP][2];
#pragma unroll
  for (int p = 0; p < NP; ++p) cm[p][0] = cm[p][1] = ca[p][0] = ca[p][1] = 0.0;
  // Each warp step covers 8 cells (two k-steps of 4): lane l reads cells
  // c0 + l%4 and c0 + 4 + l%4, so a column's two loads fill whole 32-byte
  // sectors, and the next step's 16 loads per lane are in flight during the MMAs.
  double s[NT], as[NT], s2[NT], as2[NT], wv, wv2;
  auto load = [&](int c0) {
    const int c = c0 + cq, c2 = c0 + 4 + cq;
    const bool in = c < ncells, in2 = c2 < ncells;
    wv = in ? wgt[c] : 0.0;
    wv2 = in2 ? wgt[c2] : 0.0;
#pragma unroll
    for (int ta = 0; ta < NT; ++ta) {
      s[ta] = (in && sp[ta]) ? (double)sp[ta][c] : 0.0;
      as[ta] = (in && ap[ta]) ? (double)ap[ta][c] : 0.0;
      s2[ta] = (in2 && sp[ta]) ? (double)sp[ta][c2] : 0.0;
      as2[ta] = (in2 && ap[ta]) ? (double)ap[ta][c2] : 0.0;
    }
  };
  load(8 * w);
  for (int c0 = 8 * w; c0 < ncells; c0 += 8 * nwarp) {
    double cs[NT], cas[NT], cs2[NT], cas2[NT];
#pragma unroll
    for (int ta = 0; ta < NT; ++ta) {
      cs[ta] = s[ta];
      cas[ta] = as[ta];
      cs2[ta] = s2[ta];
      cas2[ta] = as2[ta];
    }
    const double cw = wv, cw2 = wv2;
    if (c0 + 8 * nwarp < ncells) load(c0 + 8 * nwarp);  // next step in flight during the MMAs
#pragma unroll
    for (int ta = 0; ta < NT; ++ta) {
      const double ws = cs[ta] * cw, ws2 = cs2[ta] * cw2;
#pragma unroll
      for (int tb = ta; tb < NT; ++tb) {
        const int p = ta * NT - ta * (ta - 1) / 2 + (tb - ta);
        dmma884(cm[p][0], cm[p][1], ws, cs[tb]);
        dmma884(ca[p][0], ca[p][1], cs[ta], cas[tb]);
        dmma884(cm[p][0], cm[p][1], ws2, cs2[tb]);
        dmma884(ca[p][0], ca[p][1], cs2[ta], cas2[tb]);
      }
    }
  }
  // deterministic cross-warp reduction, one Gram at a time
#pragma unroll 1
  for (int which = 0; which < 2; ++which) {
    __syncthreads();
#pragma unroll
    for (int ta = 0; ta < NT; ++ta)
#pragma unroll
      for (int tb = ta; tb < NT; ++tb) {
        const int p = ta * NT - ta * (ta - 1) / 2 + (tb - ta);
        if (tb < nt) {
          const int row = 8 * ta + r, col = 8 * tb + 2 * cq;
          red[(w * 32 + row) * 32 + col] = which ? ca[p][0] : cm[p][0];
          red[(w * 32 + row) * 32 + col + 1] = which ? ca[p][1] : cm[p][1];
        }
      }
    __syncthreads();
    double* G = which ? GA : GM;
    for (int e = threadIdx.x; e < ns * ns; e += blockDim.x) {
      int a = e / ns, b = e % ns;
      if ((a >> 3) > (b >> 3)) {  // below the accumulated block triangle: the mirror
        const int x = a;
        a = b;
        b = x;
      }
      double v = 0.0;
      for (int ww = 0; ww < nwarp; ++ww) v += red[(ww * 32 + a) * 32 + b];
      G[(e / ns) * LB_LD + (e % ns)] = v;
    }
  }
  __syncthreads();
}

// In-place basis update on the FP64 tensor cores:
//   B0[:, j] <- sum_b S_b Y[b][j]            (b < ns, S = [B0 | B1 | B2])
//   B2[:, j] <- sum_{b >= m0} S_b Y[b][j]    (the new search direction)
// for j < m (m <= 8 NJ).  Warp w handles groups of 8 cells; lane l's A fragment
// is S_{k0 + l%4} at cell 8g + l/4 and its B fragments come from Y.  Every warp
// reads all ns columns of its 8 cells before writing them.
//
// Each lane resolves its NK column addresses (b = 4 kk + l%4 in [B0 | B1 | B2])
// once, and for NJ = 1 keeps its Y fragments in registers, so that a group
// costs NK predicated loads, 2 NK MMAs and the stores: no per-load selection
// among the three blocks and no loop bounds known only at run time.  Columns
// b >= ns load as zero and meet zero rows of Y (NK k-steps always run).
template <typename T, int NK, int NJ, int STAGES>
__device__ __noinline__ void cta_update_mma(T* B0, T* B1, T* B2, int m0, int n1, int n2, int m, const double* Y,
                                            int ncells, size_t ld) {
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nwarp = blockDim.x >> 5;
  const int r = lane >> 2, cq = lane & 3;
  const int ns = m0 + n1 + n2;
  const int ngrp = (ncells + 7) >> 3;
  const T* colp[NK];
  double yx[NK], yq[NK];  // Y fragments of tile 0 (NJ = 1)
#pragma unroll
  for (int kk = 0; kk < NK; ++kk) {
    const int b = 4 * kk + cq;
    colp[kk] = b >= ns        ? nullptr
               : b < m0      ? B0 + (size_t)b * ld
               : b < m0 + n1 ? B1 + (size_t)(b - m0) * ld
                             : B2 + (size_t)(b - m0 - n1) * ld;
    const double y = (NJ == 1 && b < ns && r < m) ? Y[b * LB_LD + r] : 0.0;
    yx[kk] = y;
    yq[kk] = b >= m0 ? y : 0.0;
  }
  // STAGES groups ahead are loading while group gi is multiplied.
  double av[NK], an[NK], an2[NK];
  auto load = [&](int gi, double* dst) {
    const int cell = 8 * gi + r;
    const bool in = cell < ncells;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) dst[kk] = (in && colp[kk]) ? (double)colp[kk][cell] : 0.0;
  };
  if (w < ngrp) load(w, an);
  if (STAGES > 1 && w + nwarp < ngrp) load(w + nwarp, an2);
  for (int gi = w; gi < ngrp; gi += nwarp) {
    const int cell = 8 * gi + r;
    const bool in = cell < ncells;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) {
      av[kk] = an[kk];
      if (STAGES > 1) an[kk] = an2[kk];
    }
    if (STAGES > 1) {
      if (gi + 2 * nwarp < ngrp) load(gi + 2 * nwarp, an2);
    } else {
      if (gi + nwarp < ngrp) load(gi + nwarp, an);
    }
    double dx[NJ][2], dp[NJ][2];
#pragma unroll
    for (int tj = 0; tj < NJ; ++tj) dx[tj][0] = dx[tj][1] = dp[tj][0] = dp[tj][1] = 0.0;
#pragma unroll
    for (int kk = 0; kk < NK; ++kk) {
#pragma unroll
      for (int tj = 0; tj < NJ; ++tj) {
        double y = yx[kk], yp = yq[kk];
        if (NJ > 1) {
          const int bb = 4 * kk + cq, jj = 8 * tj + r;
          y = (bb < ns && jj < m) ? Y[bb * LB_LD + jj] : 0.0;
          yp = bb >= m0 ? y : 0.0;
        }
        dmma884(dx[tj][0], dx[tj][1], av[kk], y);
        dmma884(dp[tj][0], dp[tj][1], av[kk], yp);
      }
    }
    // D fragment: rows = cells 8gi + r, columns j = 8tj + 2cq + {0, 1}
#pragma unroll
    for (int tj = 0; tj < NJ; ++tj) {
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int j = 8 * tj + 2 * cq + h;
        if (in && j < m) {
          B0[(size_t)j * ld + cell] = (T)dx[tj][h];
          B2[(size_t)j * ld + cell] = (T)dp[tj][h];
        }
      }
    }
  }
}

// The same update on the CUDA cores, one cell per thread (FP64 arithmetic):
// each thread loads the ns values of its cell (independent, coalesced loads:
// consecutive threads on consecutive cells), then accumulates both outputs
// with Y broadcast from shared memory, and writes them.  Every value of a
// cell is read before the cell is written, as in cta_update_mma.
template <typename T, int MM>
__device__ __noinline__ void cta_update_cc(T* B0, T* B1, T* B2, int m0, int n1, int n2, int m, const double* Y,
                                           int ncells, size_t ld) {
  const int ns = m0 + n1 + n2;
  for (int cell = threadIdx.x; cell < ncells; cell += blockDim.x) {
    double sv[3 * MM];
#pragma unroll
    for (int b = 0; b < 3 * MM; ++b) {
      double v = 0.0;
      if (b < ns) {
        if (b < m0)
          v = (double)B0[(size_t)b * ld + cell];
        else if (b < m0 + n1)
          v = (double)B1[(size_t)(b - m0) * ld + cell];
        else
          v = (double)B2[(size_t)(b - m0 - n1) * ld + cell];
      }
      sv[b] = v;
    }
    double ax[MM], ap[MM];
#pragma unroll
    for (int j = 0; j < MM; ++j) ax[j] = ap[j] = 0.0;
#pragma unroll
    for (int b = 0; b < 3 * MM; ++b) {
      if (b < ns) {
#pragma unroll
        for (int j = 0; j < MM; ++j) {
          const double y = Y[b * LB_LD + j];
          ax[j] += sv[b] * y;
          if (b >= m0) ap[j] += sv[b] * y;
        }
      }
    }
#pragma unroll
    for (int j = 0; j < MM; ++j)
      if (j < m) {
        B0[(size_t)j * ld + cell] = (T)ax[j];
        B2[(size_t)j * ld + cell] = (T)ap[j];
      }
  }
}

// out[b] = A32 u_b for nb vectors staged in shared memory: A32 is the subdomain
// Neumann operator with its off-diagonal couplings rounded to FP32 (the sweep
// coefficients), applied in FP64 arithmetic and stored in FP64.  For FP32
// basis vectors this gives A-images that are exactly consistent with the
// stored vectors (a fixed operator, no drift); the final FP64 Rayleigh-Ritz
// uses the true operator.
__device__ void smem_neumann64(const float* u, int ldc, int nb, int nx, int ny, int nz, const float* ctx,
                               const float* cty, const float* ctz, const double* dN, double* out, size_t ld) {
  // cell-major: a cell's position, couplings and diagonal are read once for all nb columns
  const int nxny = nx * ny, nc = nxny * nz;
  for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
    const int i = cl % nx, tt = cl / nx, j = tt % ny, k = tt / ny;
    const double d = dN[cl];
    const double cxm = i > 0 ? (double)ctx[cl] : 0.0, cxp = i < nx - 1 ? (double)ctx[cl + 1] : 0.0;
    const double cym = j > 0 ? (double)cty[cl] : 0.0, cyp = j < ny - 1 ? (double)cty[cl + nx] : 0.0;
    const double czm = k > 0 ? (double)ctz[cl] : 0.0, czp = k < nz - 1 ? (double)ctz[cl + nxny] : 0.0;
    for (int b = 0; b < nb; ++b) {
      const float* ub = u + (size_t)b * ldc;
      double v = d * (double)ub[cl];
      if (i > 0) v -= cxm * (double)ub[cl - 1];
      if (i < nx - 1) v -= cxp * (double)ub[cl + 1];
      if (j > 0) v -= cym * (double)ub[cl - nx];
      if (j < ny - 1) v -= cyp * (double)ub[cl + nx];
      if (k > 0) v -= czm * (double)ub[cl - nxny];
      if (k < nz - 1) v -= czp * (double)ub[cl + nxny];
      out[(size_t)b * ld + cl] = v;
    }
  }
}

// C[n1 x n3] = op(A)[n1 x n2] * B[n2 x n3] (small, ld LB_LD).
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
// Produces Y (nS x m) holding the coefficients of the m lowest Ritz vectors
// (M-orthonormal) and their Ritz values in sm.lam.  Returns the kept rank.
//
// The basis is first scaled to unit M-norm (D = diag(GM)^-1/2).  Normally the
// scaled Gram is factored by Cholesky, L L^T = D GM D, and Q = D L^-T; if a
// pivot falls below `drop` the basis is nearly dependent and SVQB takes over
// (eigendecomposition of D GM D, directions with eigenvalue <= drop * max
// dropped).  Then H = Q^T GA Q is diagonalised and Y = Q V[:, :m].
// Phase timer for diagnostics: thread 0 accumulates clock64() deltas.
struct PhaseClock {
  long long* p;
  long long t0;
  __device__ void start() {
    if (p && threadIdx.x == 0) t0 = clock64();
  }
  __device__ void lap(int ph) {
    if (p && threadIdx.x == 0) {
      const long long t1 = clock64();
      p[ph] += t1 - t0;
      t0 = t1;
    }
  }
};

// sc: scratch of the tridiagonal eigensolver (>= 2 400 doubles); null: mt.stile and the tiles after it.  The
// phase-batched Rayleigh-Ritz passes mt.GM: GM, GA and U are dead by then, so its shared memory ends at stile.
__device__ int cta_rayleigh_ritz(LbSmall& sm, LbMats& mt, int nS, int m, double drop, double jtol,
                                 PhaseClock* pc = nullptr, double* sc = nullptr);
__device__ int cta_rayleigh_ritz(LbSmall& sm, LbMats& mt, int nS, int m, double drop, double jtol, PhaseClock* pc,
                                 double* sc) {
  for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
    const int a = e / nS, b = e % nS;
    if (a < b) {
      const double vm = 0.5 * (mt.GM[a * LB_LD + b] + mt.GM[b * LB_LD + a]);
      mt.GM[a * LB_LD + b] = mt.GM[b * LB_LD + a] = vm;
      const double va = 0.5 * (mt.GA[a * LB_LD + b] + mt.GA[b * LB_LD + a]);
      mt.GA[a * LB_LD + b] = mt.GA[b * LB_LD + a] = va;
    }
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    double mx = 0.0;
    for (int a = 0; a < nS; ++a) mx = fmax(mx, mt.GM[a * LB_LD + a]);
    sm.scal[1] = mx;
  }
  __syncthreads();
  if (threadIdx.x < nS) {
    const double gaa = mt.GM[threadIdx.x * LB_LD + threadIdx.x];
    sm.dsc[threadIdx.x] = gaa > 1e-28 * sm.scal[1] ? 1.0 / sqrt(gaa) : 0.0;
  }
  __syncthreads();
  for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
    const int a = e / nS, b = e % nS;
    const double v = mt.GM[a * LB_LD + b] * sm.dsc[a] * sm.dsc[b];
    mt.H[a * LB_LD + b] = v;
    mt.U[a * LB_LD + b] = v;
  }
  __syncthreads();
  if (pc) pc->lap(8);
  // Cholesky of the scaled Gram (warp 0, right-looking, lower factor in U)
  if (threadIdx.x < 32) {
    const int l = threadIdx.x;
    int ok = 1;
    for (int j = 0; j < nS; ++j) {
      const double d = mt.U[j * LB_LD + j];
      if (!(d > drop) || sm.dsc[j] == 0.0) {
        ok = 0;
        break;
      }
      const double ljj = sqrt(d);
      __syncwarp();
      if (l == 0) mt.U[j * LB_LD + j] = ljj;
      if (l > j && l < nS) mt.U[l * LB_LD + j] /= ljj;
      __syncwarp();
      if (l > j && l < nS) {
        const double lij = mt.U[l * LB_LD + j];
        for (int kk = j + 1; kk <= l; ++kk) mt.U[l * LB_LD + kk] -= lij * mt.U[kk * LB_LD + j];
      }
      __syncwarp();
    }
    if (l == 0) sm.ival[4] = ok;
  }
  __syncthreads();
  if (pc) pc->lap(9);
  int q;
  if (sm.ival[4]) {
    // Q = D L^-T: lane c solves L x = e_c (forward substitution), Q[a][c] = D_a x[c -> row a]
    if (threadIdx.x < nS) {
      const int c = threadIdx.x;
      for (int i = 0; i < nS; ++i) {
        double s = (i == c) ? 1.0 : 0.0;
        for (int kk = c; kk < i; ++kk) s -= mt.U[i * LB_LD + kk] * mt.V[kk * LB_LD + c];
        mt.V[i * LB_LD + c] = i < c ? 0.0 : s / mt.U[i * LB_LD + i];
      }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
      const int a = e / nS, c = e % nS;
      mt.Q[a * LB_LD + c] = sm.dsc[a] * mt.V[c * LB_LD + a];  // (L^-1)^T
    }
    __syncthreads();
    q = nS;
  } else {
    cta_jacobi_eigh(mt.H, mt.U, sm.w, nS, LB_LD, sm.ival2, sm.jac, jtol);
    if (threadIdx.x == 0) {
      int qq = 0;
      const double wmax = sm.w[nS - 1];
      for (int c = 0; c < nS; ++c)
        if (sm.w[c] > drop * wmax && sm.w[c] > 0.0) ++qq;
      sm.ival[0] = qq;
    }
    __syncthreads();
    q = sm.ival[0];
    for (int e = threadIdx.x; e < nS * q; e += blockDim.x) {
      const int a = e / q, c = e % q, cc = nS - q + c;
      mt.Q[a * LB_LD + c] = sm.dsc[a] * mt.U[a * LB_LD + cc] / sqrt(sm.w[cc]);
    }
    __syncthreads();
  }
  if (pc) pc->lap(10);
  cta_small_gemm(mt.GA, false, mt.Q, mt.V, nS, nS, q);  // V = GA Q
  cta_small_gemm(mt.Q, true, mt.V, mt.H, q, nS, q);     // H = Q^T GA Q
  for (int e = threadIdx.x; e < q * q; e += blockDim.x) {
    const int a = e / q, b = e % q;
    if (a < b) {
      const double v = 0.5 * (mt.H[a * LB_LD + b] + mt.H[b * LB_LD + a]);
      mt.H[a * LB_LD + b] = mt.H[b * LB_LD + a] = v;
    }
  }
  __syncthreads();
  if (pc) pc->lap(11);
  // only the lowest min(m, q) eigenpairs of H are needed
  cta_sym_lowest(mt.H, mt.V, sm.th, q, min(m, q), LB_LD, sc ? sc : mt.stile);
  (void)jtol;
  if (pc) pc->lap(12);
  const int mm = min(m, q);
  cta_small_gemm(mt.Q, false, mt.V, mt.Y, nS, q, mm);  // Y = Q V[:, :m]
  if (threadIdx.x < mm) sm.lam[threadIdx.x] = sm.th[threadIdx.x];
  __syncthreads();
  if (pc) pc->lap(13);
  return q;
}

// Cell size, Dirichlet faces and the box of the subdomain's problem: the
// solver's own for a single problem, the problem table's for a batch.
struct EigGeom {
  double Hx, Hy, Hz, meas;
  int dmask, M, N, z0, z1;
};
__device__ __forceinline__ EigGeom eig_geom(const ProbInfo* probs, const Grid& g, double Hx, double Hy, double Hz,
                                            double meas, int dmask, const SubInfo& S) {
  EigGeom e;
  if (probs) {
    const ProbInfo& p = probs[S.prob];
    e.Hx = p.Hx;
    e.Hy = p.Hy;
    e.Hz = p.Hz;
    e.meas = p.meas;
    e.dmask = p.dmask;
    e.M = p.M;
    e.N = p.N;
    e.z0 = p.z0;
    e.z1 = p.z0 + p.P;
  } else {
    e.Hx = Hx;
    e.Hy = Hy;
    e.Hz = Hz;
    e.meas = meas;
    e.dmask = dmask;
    e.M = g.M;
    e.N = g.N;
    e.z0 = 0;
    e.z1 = g.P;
  }
  return e;
}
__device__ __forceinline__ bool touches_dirichlet(const EigGeom& e, const SubInfo& S) {
  const int dm = e.dmask;
  return ((dm & 1) && S.x0 == 0) || ((dm & 2) && S.x0 + S.nx == e.M) || ((dm & 4) && S.y0 == 0) ||
         ((dm & 8) && S.y0 + S.ny == e.N) || ((dm & 16) && S.z0 == e.z0) || ((dm & 32) && S.z0 + S.nz == e.z1);
}

// out = A^N v on the subdomain (FP64 arithmetic, stored as TO).
template <typename TI, typename TO>
__device__ __forceinline__ void neumann_apply_col(const Grid& g, const SubInfo& S, const double* tx, const double* ty,
                                                  const double* tz, const double* dN, const TI* v, TO* out,
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
    out[cl] = (TO)a;
  }
}

// Per-subdomain iteration state of the phase-batched solver (global memory).
struct EbState {
  double lam[LB_MM];
  double lscale, best;
  int act[LB_MM];
  int nact, np, nS, hasP, done, conv, stag, it, last_improve, restart;
};

template <typename T>
__global__ void __launch_bounds__(LB_THREADS) k_lobpcg(LobpcgArgs a, unsigned char* work, size_t work_stride, T* phi,
                                                double* evals, int* iters, int* status, int* ks, double eb) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbSmall& sm = *reinterpret_cast<LbSmall*>(smraw);
  const int ldc = a.ldc;
  float* ctx = reinterpret_cast<float*>(smraw + sizeof(LbSmall));
  float* cty = ctx + ldc;
  float* ctz = cty + ldc;
  float* cinv = ctz + ldc;
  unsigned char* uni = smraw + sizeof(LbSmall) + (size_t)16 * ldc;
  LbMats& mt = *reinterpret_cast<LbMats*>(uni);
  float* u = reinterpret_cast<float*>(uni);
  double* Dtmp = reinterpret_cast<double*>(uni);
  const Grid g = a.g;
  const int m = a.m, k = a.k, mb = a.mb;
  unsigned char* wb = work + (size_t)blockIdx.x * work_stride;
  const int ld = a.ld;
  PhaseClock pc{a.prof ? a.prof + (size_t)blockIdx.x * 16 : nullptr, 0};
  pc.start();

  const int count = (a.sub_list && a.nlist) ? *a.nlist : a.nsub;
  __shared__ int s_next;
  for (int idx = blockIdx.x;; idx += gridDim.x) {
    if (a.queue) {  // dynamic schedule: take the next unclaimed subdomain
      __syncthreads();
      if (threadIdx.x == 0) s_next = atomicAdd(a.queue, 1);
      __syncthreads();
      idx = s_next;
    }
    if (idx >= count) break;
    const int s = a.sub_list ? a.sub_list[idx] : idx;
    const SubInfo S = a.subs[s];
    const EigGeom eg = eig_geom(a.probs, g, a.Hx, a.Hy, a.Hz, a.meas, a.dirichlet_mask, S);
    const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
    unsigned char* wbs = a.mode ? a.slab + (size_t)s * a.slab_stride : wb;
    T* X = reinterpret_cast<T*>(wbs);
    T* W = X + (size_t)m * ld;
    T* P = W + (size_t)m * ld;
    double* AX = reinterpret_cast<double*>(P + (size_t)m * ld);
    double* AW = AX + (size_t)m * ld;
    double* AP = AW + (size_t)m * ld;
    double* Md = reinterpret_cast<double*>(AP + (size_t)m * ld);
    double* dN = Md + ld;
    double* dN32 = dN + ld;  // diagonal matching the FP32-rounded couplings (FP32 storage)

    bool hasP = false;
    int it = 0;
    bool conv = false;
    if (a.mode == 2) {  // final phase of the batched solver: the state comes from the slab
      const EbState* es = reinterpret_cast<const EbState*>(a.state) + s;
      it = es->it;
      conv = es->conv != 0;
      if (threadIdx.x == 0) sm.ival[6] = es->stag;
      __syncthreads();
    } else {
    // ---- mass diagonal (src/PreMixFEM_3D.c:243-346), Neumann diagonal, sweep coefficients
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
        if (i == 0 && ex >= 1) mv += 2.0 * avg_k(a.kx[cg - 1], a.kx[cg]) / eg.Hx / eg.Hx;
        if (ex + 1 != g.M) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / eg.Hx / eg.Hx;
        if (ey >= 1) mv += 2.0 * avg_k(a.ky[cg - g.M], a.ky[cg]) / eg.Hy / eg.Hy;
        if (ey + 1 != g.N) mv += 2.0 * avg_k(a.ky[cg], a.ky[cg + g.M]) / eg.Hy / eg.Hy;
        if (ez >= 1) mv += 2.0 * avg_k(a.kz[cg - g.MN], a.kz[cg]) / eg.Hz / eg.Hz;
        if (ez + 1 != g.P) mv += 2.0 * avg_k(a.kz[cg], a.kz[cg + g.MN]) / eg.Hz / eg.Hz;
        if (i + 1 < nx) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / eg.Hx / eg.Hx;
        // Dirichlet extension: 2 t_b per boundary face
        if (eg.dmask & 1 && ex == 0) mv += 2.0 * (2.0 * a.kx[cg]) / eg.Hx / eg.Hx;
        if (eg.dmask & 2 && ex == eg.M - 1) mv += 2.0 * (2.0 * a.kx[cg]) / eg.Hx / eg.Hx;
        if (eg.dmask & 4 && ey == 0) mv += 2.0 * (2.0 * a.ky[cg]) / eg.Hy / eg.Hy;
        if (eg.dmask & 8 && ey == eg.N - 1) mv += 2.0 * (2.0 * a.ky[cg]) / eg.Hy / eg.Hy;
        if (eg.dmask & 16 && ez == eg.z0) mv += 2.0 * (2.0 * a.kz[cg]) / eg.Hz / eg.Hz;
        if (eg.dmask & 32 && ez == eg.z1 - 1) mv += 2.0 * (2.0 * a.kz[cg]) / eg.Hz / eg.Hz;
        mv = mv * eg.meas;
      }
      Md[cl] = mv;
      dN[cl] = dn;
      {
        double d32 = a.db[cg];
        if (i > 0) d32 += (double)(float)a.tx[cg];
        if (i < nx - 1) d32 += (double)(float)a.tx[cg + 1];
        if (j > 0) d32 += (double)(float)a.ty[cg];
        if (j < ny - 1) d32 += (double)(float)a.ty[cg + g.M];
        if (kk > 0) d32 += (double)(float)a.tz[cg];
        if (kk < nz - 1) d32 += (double)(float)a.tz[cg + g.MN];
        dN32[cl] = d32;
      }
      ctx[cl] = i > 0 ? (float)a.tx[cg] : 0.0f;
      cty[cl] = j > 0 ? (float)a.ty[cg] : 0.0f;
      ctz[cl] = kk > 0 ? (float)a.tz[cg] : 0.0f;
      ratio = fmax(ratio, dn / mv);
    }
    for (int o = 16; o > 0; o >>= 1) ratio = fmax(ratio, __shfl_xor_sync(0xffffffffu, ratio, o));
    if ((threadIdx.x & 31) == 0) mt.red[threadIdx.x >> 5] = ratio;
    __syncthreads();
    if (threadIdx.x == 0) {
      double r = 0.0;
      for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) r = fmax(r, mt.red[wi]);
      sm.scal[0] = r > 0 ? r : 1.0;
    }
    __syncthreads();
    const double lscale = sm.scal[0];
    const double sigma = a.sigma_rel * lscale;

    // ---- IC(0) pivots of A^N + sigma M (wavefront, natural order, FP64)
    const int t = threadIdx.x, jj = t % ny, kk = t / ny;
    const bool line = t < ny * nz;
    const int nplanes = nx + ny + nz - 2;
    for (int d = 0; d < nplanes; ++d) {
      const int i = d - jj - kk;
      if (line && i >= 0 && i < nx) {
        const int cl = (kk * ny + jj) * nx + i;
        double sacc = 0.0;
        if (kk > 0) sacc += (double)ctz[cl] * (double)ctz[cl] / Dtmp[cl - nxny];
        if (jj > 0) sacc += (double)cty[cl] * (double)cty[cl] / Dtmp[cl - nx];
        if (i > 0) sacc += (double)ctx[cl] * (double)ctx[cl] / Dtmp[cl - 1];
        double D = dN[cl] + sigma * Md[cl] - sacc;
        if (!(D > 0.0)) D = dN[cl] + sigma * Md[cl];
        Dtmp[cl] = D;
        cinv[cl] = (float)(1.0 / D);
      }
      __syncthreads();
    }

    // ---- initial block, A X, first Rayleigh-Ritz
    for (int e = threadIdx.x; e < m * nc; e += blockDim.x) {
      const int j = e / nc, cl = e % nc;
      double v;
      if (a.xinit_patch && j < a.xinit_k) {
        const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
        v = a.xinit_patch[((size_t)s * 4096 + (kz_ * 16 + jy) * 16 + i) * 16 + j];
      } else if (a.xinit) {
        const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
        const long long cg = ((long long)(S.z0 + kz_) * g.N + (S.y0 + jy)) * g.M + (S.x0 + i);
        v = a.xinit[cg * m + j];
      } else {
        v = hash_uniform(a.seed ^ ((unsigned long long)s << 32) ^ (unsigned long long)e);
      }
      X[(size_t)j * ld + cl] = (T)v;
    }
    __syncthreads();
    if (sizeof(T) == 8) {
      for (int j = 0; j < m; ++j)
        neumann_apply_col(g, S, a.tx, a.ty, a.tz, dN, X + (size_t)j * ld, AX + (size_t)j * ld, nc);
      __syncthreads();
    } else {
      for (int j0 = 0; j0 < m; j0 += mb) {
        const int nb = min(mb, m - j0);
        load_cols_to_smem(X + (size_t)j0 * ld, ld, nb, nc, u, ldc);
        __syncthreads();
        smem_neumann64(u, ldc, nb, nx, ny, nz, ctx, cty, ctz, dN32, AX + (size_t)j0 * ld, ld);
        __syncthreads();
      }
    }
    const double drop = sizeof(T) == 4 ? 1e-9 : 1e-13;
    {
      Seg3<T> sx{{X, X, X}, {m, 0, 0}, ld};
      Seg3<double> sax{{AX, AX, AX}, {m, 0, 0}, ld};
      cta_gram2(sx, sax, Md, nc, mt.GM, mt.GA, mt);
    }
    cta_rayleigh_ritz(sm, mt, m, m, drop, 1e-12);
    for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
      double xr[LB_MM], ar[LB_MM];
#pragma unroll
      for (int b = 0; b < LB_MM; ++b) {
        xr[b] = b < m ? (double)X[(size_t)b * ld + cl] : 0.0;
        ar[b] = b < m ? (double)AX[(size_t)b * ld + cl] : 0.0;
      }
#pragma unroll
      for (int j = 0; j < LB_MM; ++j)
        if (j < m) {
          double xn = 0.0, an = 0.0;
#pragma unroll
          for (int b = 0; b < LB_MM; ++b)
            if (b < m) {
              xn += xr[b] * mt.Y[b * LB_LD + j];
              an += ar[b] * mt.Y[b * LB_LD + j];
            }
          X[(size_t)j * ld + cl] = (T)xn;
          AX[(size_t)j * ld + cl] = an;
        }
    }
    __syncthreads();

    if (threadIdx.x == 0) {
      sm.scal[2] = 1e300;
      sm.ival[5] = 0;
      sm.ival[6] = 0;
    }
    __syncthreads();
    pc.lap(0);
    if (a.mode == 1) {  // set-up phase of the batched solver: keep coefficients and state
      EbState* es = reinterpret_cast<EbState*>(a.state) + s;
      float* gc = reinterpret_cast<float*>(dN32 + ld);
      for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
        gc[cl] = ctx[cl];
        gc[(size_t)ld + cl] = cty[cl];
        gc[(size_t)2 * ld + cl] = ctz[cl];
        gc[(size_t)3 * ld + cl] = cinv[cl];
      }
      if (threadIdx.x < m) es->lam[threadIdx.x] = sm.lam[threadIdx.x];
      if (threadIdx.x == 0) {
        es->lscale = lscale;
        es->best = 1e300;
        es->last_improve = 0;
        es->hasP = 0;
        es->done = 0;
        es->conv = 0;
        es->stag = 0;
        es->it = 0;
        es->restart = 0;
        es->nact = 0;
        es->np = 0;
        es->nS = m;
      }
      continue;
    }
    for (; it < a.max_it; ++it) {
      // ---- residuals R = AX - M X Lambda (into W) and ||R_j||_{M^-1}
      double racc[LB_MM];
#pragma unroll
      for (int j = 0; j < LB_MM; ++j) racc[j] = 0.0;
      {
        const int ng = nc >> 2;
        for (int gi = threadIdx.x; gi < ng; gi += blockDim.x) {
          const int cl = gi * 4;
          double mv[4];
          ld4(Md + cl, mv);
#pragma unroll
          for (int j = 0; j < LB_MM; ++j)
            if (j < m) {
              double ax[4], xv[4], r[4];
              ld4(AX + (size_t)j * ld + cl, ax);
              ld4(X + (size_t)j * ld + cl, xv);
#pragma unroll
              for (int q = 0; q < 4; ++q) {
                r[q] = ax[q] - sm.lam[j] * mv[q] * xv[q];
                racc[j] += r[q] * r[q] / mv[q];
              }
              st4(W + (size_t)j * ld + cl, r);
            }
        }
        for (int cl = 4 * ng + threadIdx.x; cl < nc; cl += blockDim.x) {
          const double mv = Md[cl];
#pragma unroll
          for (int j = 0; j < LB_MM; ++j)
            if (j < m) {
              const double r = (double)AX[(size_t)j * ld + cl] - sm.lam[j] * mv * (double)X[(size_t)j * ld + cl];
              W[(size_t)j * ld + cl] = (T)r;
              racc[j] += r * r / mv;
            }
        }
      }
#pragma unroll
      for (int j = 0; j < LB_MM; ++j)
        if (j < m) {
          const double v = warp_sum(racc[j]);
          if ((threadIdx.x & 31) == 0) mt.red[j * 33 + (threadIdx.x >> 5)] = v;
        }
      __syncthreads();
      if (threadIdx.x < m) {
        double v = 0.0;
        for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) v += mt.red[threadIdx.x * 33 + wi];
        // residual scale: lscale (the largest diag(A_N)/M), or, with a relative
        // floor f, max(|lambda_j|, f lscale) as an eigenvalue-relative test
        const double rs = a.rel_floor > 0.0 ? fmax(fabs(sm.lam[threadIdx.x]), a.rel_floor * lscale) : lscale;
        sm.res[threadIdx.x] = sqrt(v) / rs;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        int na = 0, cv = 1;
        double worst = 0.0;
        for (int j = 0; j < m; ++j) {
          const bool done_j = sm.res[j] <= a.tol;
          if (j < k) worst = fmax(worst, sm.res[j]);
          if (j < k && !done_j) cv = 0;
          if (!done_j || j >= k) sm.act[na++] = j;  // soft locking of converged wanted vectors
        }
        // rounding floor: no halving of the worst wanted residual in 12 iterations
        // while within 10 x tol -> accept (status 2)
        if (!cv) {
          if (worst < 0.5 * sm.scal[2]) {
            sm.scal[2] = worst;
            sm.ival[5] = it;
          } else if (it - sm.ival[5] >= 12 && worst <= 10.0 * a.tol) {
            cv = 1;
            sm.ival[6] = 1;
          }
        }
        sm.ival[2] = na;
        sm.ival[3] = cv;
      }
      __syncthreads();
      conv = sm.ival[3] != 0;
      pc.lap(1);
      if (conv) break;
      const int nact = sm.ival[2];
      // compact the active residuals to the front of W (act[] is increasing)
      for (int c = 0; c < nact; ++c) {
        const int src = sm.act[c];
        if (src != c)
          for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) W[(size_t)c * ld + cl] = W[(size_t)src * ld + cl];
        __syncthreads();
      }
      // ---- W = T R: IC(0) sweeps, mb vectors per wavefront, FP32 in shared memory
      for (int j0 = 0; j0 < nact; j0 += mb) {
        const int nb = min(mb, nact - j0);
        load_cols_to_smem(W + (size_t)j0 * ld, ld, nb, nc, u, ldc);
        __syncthreads();
        for (int d = 0; d < nplanes; ++d) {
          const int i = d - jj - kk;
          if (line && i >= 0 && i < nx) {
            const int cl = (kk * ny + jj) * nx + i;
            const float cz_ = ctz[cl], cy_ = cty[cl], cx_ = ctx[cl], ci = cinv[cl];
#pragma unroll 4
            for (int b = 0; b < nb; ++b) {
              float* ub = u + b * ldc;
              float sacc = ub[cl];
              if (kk > 0) sacc += cz_ * ub[cl - nxny];
              if (jj > 0) sacc += cy_ * ub[cl - nx];
              if (i > 0) sacc += cx_ * ub[cl - 1];
              ub[cl] = sacc * ci;
            }
          }
          __syncthreads();
        }
        for (int d = nplanes - 1; d >= 0; --d) {
          const int i = d - jj - kk;
          if (line && i >= 0 && i < nx) {
            const int cl = (kk * ny + jj) * nx + i;
            const float cxp = i < nx - 1 ? ctx[cl + 1] : 0.0f;
            const float cyp = jj < ny - 1 ? cty[cl + nx] : 0.0f;
            const float czp = kk < nz - 1 ? ctz[cl + nxny] : 0.0f;
            const float ci = cinv[cl];
#pragma unroll 4
            for (int b = 0; b < nb; ++b) {
              float* ub = u + b * ldc;
              float sacc = 0.0f;
              if (i < nx - 1) sacc += cxp * ub[cl + 1];
              if (jj < ny - 1) sacc += cyp * ub[cl + nx];
              if (kk < nz - 1) sacc += czp * ub[cl + nxny];
              ub[cl] = ub[cl] + sacc * ci;
            }
          }
          __syncthreads();
        }
        if (sizeof(T) == 4) smem_neumann64(u, ldc, nb, nx, ny, nz, ctx, cty, ctz, dN32, AW + (size_t)j0 * ld, ld);
        store_cols_from_smem(W + (size_t)j0 * ld, ld, nb, nc, u, ldc);
        __syncthreads();
      }
      pc.lap(2);
      if (sizeof(T) == 8) {  // FP64 A-images of the new directions
        for (int j = 0; j < nact; ++j)
          neumann_apply_col(g, S, a.tx, a.ty, a.tz, dN, W + (size_t)j * ld, AW + (size_t)j * ld, nc);
        __syncthreads();
      }
      pc.lap(3);
      const int np = hasP ? m : 0;
      const int nS = m + nact + np;
      {
        Seg3<T> sS{{X, W, P}, {m, nact, np}, ld};
        Seg3<double> sA{{AX, AW, AP}, {m, nact, np}, ld};
        if (nS <= 24)
          cta_gram2_mma<T, double, 3>(sS, sA, Md, nc, mt.GM, mt.GA, mt.U);
        else
          cta_gram2_mma<T, double, 4>(sS, sA, Md, nc, mt.GM, mt.GA, mt.U);
      }
      pc.lap(4);
      pc.lap(5);
      const int q = cta_rayleigh_ritz(sm, mt, nS, m, drop, 1e-11, &pc);
      if (q < m) {  // basis collapsed: restart without P
        hasP = false;
        continue;
      }
      // ---- X <- S Y, P <- [W P] Y_WP, same for AX / AP (per cell, in place)
      // X <- S Y, P <- [W P] Y_WP and the same combination of the FP64 A-images, on the
      // FP64 tensor cores
      cta_update_mma<T, 8, 2, 1>(X, W, P, m, nact, np, m, mt.Y, nc, ld);
      pc.lap(14);
      if (sizeof(T) == 8) {
        cta_update_mma<double, 8, 2, 1>(AX, AW, AP, m, nact, np, m, mt.Y, nc, ld);
        __syncthreads();
      } else {
        // FP32 storage rounds X and P: their A-images are recomputed from the stored values
        __syncthreads();
        for (int blk = 0; blk < 2; ++blk) {
          const T* src = blk ? P : X;
          double* dst = blk ? AP : AX;
          for (int j0 = 0; j0 < m; j0 += mb) {
            const int nb = min(mb, m - j0);
            load_cols_to_smem(src + (size_t)j0 * ld, ld, nb, nc, u, ldc);
            __syncthreads();
            smem_neumann64(u, ldc, nb, nx, ny, nz, ctx, cty, ctz, dN32, dst + (size_t)j0 * ld, ld);
            __syncthreads();
          }
        }
      }
      hasP = true;
      pc.lap(6);
    }
    }  // mode != 2

    // ---- final FP64 Rayleigh-Ritz on X (A X recomputed in FP64 over the W|P slab)
    double* AX64 = AX;
    for (int j = 0; j < m; ++j)
      neumann_apply_col(g, S, a.tx, a.ty, a.tz, dN, X + (size_t)j * ld, AX64 + (size_t)j * ld, nc);
    __syncthreads();
    {
      Seg3<T> sx{{X, X, X}, {m, 0, 0}, ld};
      Seg3<double> sax{{AX64, AX64, AX64}, {m, 0, 0}, ld};
      cta_gram2(sx, sax, Md, nc, mt.GM, mt.GA, mt);
    }
    cta_rayleigh_ritz(sm, mt, m, m, 1e-14, 1e-14);
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
      status[s] = conv ? (sm.ival[6] ? 2 : 0) : 1;
    }
    __syncthreads();
    const int num = sm.ival[1];
    if (threadIdx.x < k) evals[(long long)s * k + threadIdx.x] = sm.lam[threadIdx.x];
    // FP32 storage: on a subdomain that touches no Dirichlet face, the lowest
    // eigenvector of A_i^N v = lambda M_i v is exactly the constant (A_i^N 1 = 0),
    // but FP32 iterations only reach it to ~1e-6.  Write the exact M-normalised
    // constant instead, so that the coarse spaces contain the global null vector
    // of a pure-Neumann operator exactly and its coarse pivot stays negligible.
    bool snap = false;
    double cval = 0.0;
    if (sizeof(T) == 4 && num >= 1) {
      const bool touches = touches_dirichlet(eg, S);
      if (!touches) {
        double msum = 0.0, vsum = 0.0;
        for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
          double v0 = 0.0;
          for (int b = 0; b < m; ++b) v0 += (double)X[(size_t)b * ld + cl] * mt.Y[b * LB_LD];
          msum += Md[cl];
          vsum += Md[cl] * v0;
        }
        msum = block_sum(msum, sm.res);
        vsum = block_sum(vsum, sm.res);
        snap = msum > 0.0;
        cval = snap ? copysign(1.0 / sqrt(msum), vsum) : 0.0;
      }
    }
    for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
      const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
      const long long cg = ((long long)(S.z0 + kz_) * g.N + (S.y0 + jy)) * g.M + (S.x0 + i);
      double xr[LB_MM];
#pragma unroll
      for (int b = 0; b < LB_MM; ++b) xr[b] = b < m ? (double)X[(size_t)b * ld + cl] : 0.0;
      for (int j = 0; j < a.kmax; ++j) {
        double v = 0.0;
        if (j < num) {
#pragma unroll
          for (int b = 0; b < LB_MM; ++b)
            if (b < m) v += xr[b] * mt.Y[b * LB_LD + j];
        }
        if (snap && j == 0) v = cval;
        phi[cg * a.kmax + j] = (T)v;
      }
    }
    __syncthreads();
    pc.lap(7);
  }
}

template <typename T>
void launch_lobpcg(const LobpcgArgs& a_in, int nblocks, void* work, T* phi, double* evals, int* iters, int* status,
                   int* ks, double eb, int max_cells, int max_lines, cudaStream_t st) {
  LobpcgArgs a = a_in;
  a.ld = lb_ld(max_cells);
  a.ldc = (max_cells + 3) & ~3;
  const size_t fixed = sizeof(LbSmall) + (size_t)16 * a.ldc;
  const size_t limit = 227 * 1024 - 256;  // leave room for the kernel's static shared memory
  const size_t avail = limit > fixed ? limit - fixed : 0;
  int mb = (int)std::min<size_t>(a.m, avail / ((size_t)4 * a.ldc));
  if (mb < 1) mb = 1;
  a.mb = mb;
  const size_t uni = std::max(std::max(sizeof(LbMats), (size_t)mb * 4 * a.ldc), (size_t)8 * a.ldc);
  const size_t smem = fixed + uni;
  const int threads = LB_THREADS;  // one x-line per thread: callers guarantee ny*nz <= 256
  (void)max_lines;
  cudaFuncSetAttribute(k_lobpcg<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  const size_t stride = (lobpcg_work_bytes(max_cells, a.m, sizeof(T)) + 255) & ~(size_t)255;
  if (a.queue) cudaMemsetAsync(a.queue, 0, sizeof(int), st);
  { note_launch(); k_lobpcg<T><<<nblocks, threads, smem, st>>>(a, (unsigned char*)work, stride, phi, evals, iters, status, ks, eb); }
}
template void launch_lobpcg<float>(const LobpcgArgs&, int, void*, float*, double*, int*, int*, int*, double, int, int,
                                   cudaStream_t);
template void launch_lobpcg<double>(const LobpcgArgs&, int, void*, double*, double*, int*, int*, int*, double, int,
                                    int, cudaStream_t);


// ============================================================================
// Phase-batched LOBPCG.  The iteration of k_lobpcg, one launch per phase over
// every active subdomain, the block vectors of all subdomains resident in HBM
// (per-subdomain slabs: X, W, P, their FP64 A-images, M, the Neumann
// diagonals and the IC(0) sweep coefficients).  Set-up and the final
// Rayleigh-Ritz are k_lobpcg's own code (modes 1 and 2).  Each phase is a
// separate grid (subdomain x cell chunk or column batch), so many more warps
// per SM are in flight than in the one-CTA-per-SM persistent kernel; partial
// sums are reduced in a fixed order, so results do not depend on scheduling.

namespace {

constexpr int EB_CHUNK = 1024;  // cells per Gram / residual / update chunk

template <typename T>
struct EbSlab {
  T *X, *W, *P;
  double *AX, *AW, *AP, *Md, *dN, *dN32;
  float *ctx, *cty, *ctz, *cinv;
  __device__ EbSlab(unsigned char* base, int m, int ld) {
    X = reinterpret_cast<T*>(base);
    W = X + (size_t)m * ld;
    P = W + (size_t)m * ld;
    AX = reinterpret_cast<double*>(P + (size_t)m * ld);
    AW = AX + (size_t)m * ld;
    AP = AW + (size_t)m * ld;
    Md = AP + (size_t)m * ld;
    dN = Md + ld;
    dN32 = dN + ld;
    ctx = reinterpret_cast<float*>(dN32 + ld);
    cty = ctx + ld;
    ctz = cty + ld;
    cinv = ctz + ld;
  }
};

struct EbArgs {
  Grid g;
  const SubInfo* subs;
  const int* list;
  int m, k, ld, ldc, mb, nchunk, max_it;
  double tol, rel_floor;
  unsigned char* slab;
  size_t slab_stride;
  EbState* state;
  double* Ybuf;
  double* gpart;
  double* rpart;
  int* nactive;
  int* alist;  // subdomains still iterating, compacted by k_eb_control
  unsigned long long* colcells;  // sum over active subdomain-iterations of (basis columns x cells)
  const double *tx, *ty, *tz;
  const ProbInfo* probs;  // a batch's problem table, or null
};

// Phase kernels index the compacted active list; the control kernel the full list.
__device__ __forceinline__ int eb_sub(const EbArgs& a, int idx) { return a.alist[idx]; }

// Partial ||AX_j - lambda_j M X_j||^2_{M^-1} over one chunk of cells.
// All m columns at once: a full chunk gives each thread four consecutive cells
// (vector loads, every column's loads in flight together); the per-column
// sums are reduced per warp by shuffles and across the warps in a fixed order.
template <typename T>
__global__ void __launch_bounds__(256) k_eb_resid(EbArgs a, int use_alist) {
  __shared__ double red[32][LB_MM];
  const int s = use_alist ? a.alist[blockIdx.y] : (a.list ? a.list[blockIdx.y] : (int)blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK, c1 = min(nc, c0 + EB_CHUNK);
  double* out = a.rpart + ((size_t)s * a.nchunk + blockIdx.x) * LB_MM;
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  const int m = a.m;
  double lam[LB_MM], acc[LB_MM];
#pragma unroll
  for (int j = 0; j < LB_MM; ++j) {
    lam[j] = j < m ? es.lam[j] : 0.0;
    acc[j] = 0.0;
  }
  if (c1 - c0 == 4 * (int)blockDim.x) {
    const int cl = c0 + 4 * threadIdx.x;  // 16-byte aligned: c0 and ld are multiples of 4
    double md[4];
    ld4(sl.Md + cl, md);
#pragma unroll
    for (int j = 0; j < LB_MM; ++j) {
      if (j < m) {
        double ax[4], xv[4];
        ld4(sl.AX + (size_t)j * a.ld + cl, ax);
        ld4(sl.X + (size_t)j * a.ld + cl, xv);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double r = ax[q] - lam[j] * md[q] * xv[q];
          acc[j] += r * r / md[q];
        }
      }
    }
  } else {
    for (int cl = c0 + threadIdx.x; cl < c1; cl += blockDim.x) {
      const double mv = sl.Md[cl];
#pragma unroll
      for (int j = 0; j < LB_MM; ++j) {
        if (j < m) {
          const double r = sl.AX[(size_t)j * a.ld + cl] - lam[j] * mv * (double)sl.X[(size_t)j * a.ld + cl];
          acc[j] += r * r / mv;
        }
      }
    }
  }
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < LB_MM; ++j) {
    const double v = warp_sum(acc[j]);
    if (lane == 0) red[w][j] = v;
  }
  __syncthreads();
  if (threadIdx.x < m) {
    double v = 0.0;
    for (int q = 0; q < nw; ++q) v += red[q][threadIdx.x];
    out[threadIdx.x] = v;
  }
}

// Convergence, soft locking and the rounding-floor test of k_lobpcg, one
// thread per subdomain.
__global__ void k_eb_control(EbArgs a, int nlist, int it) {
  const int idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= nlist) return;
  const int s = a.list ? a.list[idx] : idx;
  EbState& es = a.state[s];
  if (es.done) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int nch = (nc + EB_CHUNK - 1) / EB_CHUNK;
  const int m = a.m, k = a.k;
  int na = 0, cv = 1;
  double worst = 0.0;
  for (int j = 0; j < m; ++j) {
    double v = 0.0;
    for (int c = 0; c < nch; ++c) v += a.rpart[((size_t)s * a.nchunk + c) * LB_MM + j];
    const double rs = a.rel_floor > 0.0 ? fmax(fabs(es.lam[j]), a.rel_floor * es.lscale) : es.lscale;
    const double res = sqrt(v) / rs;
    const bool done_j = res <= a.tol;
    if (j < k) worst = fmax(worst, res);
    if (j < k && !done_j) cv = 0;
    if (!done_j || j >= k) es.act[na++] = j;
  }
  if (!cv) {
    if (worst < 0.5 * es.best) {
      es.best = worst;
      es.last_improve = it;
    } else if (it - es.last_improve >= 12 && worst <= 10.0 * a.tol) {
      cv = 1;
      es.stag = 1;
    }
  }
  if (cv) {
    es.done = 1;
    es.conv = 1;
    es.it = it;
    return;
  }
  es.nact = na;
  es.np = es.hasP ? m : 0;
  es.nS = m + na + es.np;
  es.it = it + 1;  // iterations counted if the iteration limit ends the solve
  a.alist[atomicAdd(a.nactive, 1)] = s;  // order is irrelevant: subdomains are independent
  atomicAdd(a.nactive + 1, na);          // active columns: the preconditioner's work
  atomicAdd(a.nactive + 2, es.nS);       // basis columns: the Gram's and the update's work
  if (a.colcells) atomicAdd(a.colcells, (unsigned long long)es.nS * (unsigned long long)nc);
}

// W_c = T (AX_a - lambda_a M X_a) for active columns c (a = act[c]) of one
// column batch: IC(0) sweeps of A^N + sigma M in shared memory (FP32), and in
// FP32 storage the FP64 A-image with the FP32-rounded couplings.
//
// Shared memory: a 16-byte header (mbarrier, flag), the four coefficient
// arrays at the slab's pitch ld (one bulk copy of 16 ld bytes, which lands
// while the threads form the residuals), then the nb columns at pitch ldc.
// The residuals are formed four cells at a time with vector loads, two groups
// of four per thread in flight.  Thread 0's wait for the copy is bounded; a
// copy that does not land sets nactive[3] and the CTA writes nothing.
template <typename T>
__global__ void __launch_bounds__(256) k_eb_precond(EbArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  const int s = eb_sub(a, blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done) return;
  const int c0 = blockIdx.x * a.mb;
  const int nb = min(a.mb, es.nact - c0);
  if (nb <= 0) return;
  const SubInfo S = a.subs[s];
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
  const int ldc = a.ldc, ld = a.ld;
  uint64_t* bar = reinterpret_cast<uint64_t*>(smraw);
  int* flag = reinterpret_cast<int*>(smraw + 8);
  float* ctx = reinterpret_cast<float*>(smraw + 16);
  float* cty = ctx + ld;
  float* ctz = cty + ld;
  float* cinv = ctz + ld;
  float* u = cinv + ld;
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, ld);
  if (threadIdx.x == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    const uint32_t bytes = (uint32_t)(16 * (size_t)ld);  // ctx, cty, ctz, cinv: contiguous in the slab
    mbar_arrive_expect_tx(bar, bytes);
    bulk_g2s(ctx, sl.ctx, bytes, bar);
  }
  {
    const int ng = nc >> 2, tot = nb * ng, bd = blockDim.x;
    auto resid4 = [&](int e, float4& o) {
      const int b = e / ng, cl = 4 * (e - b * ng);
      const int col = es.act[c0 + b];
      const double lam = es.lam[col];
      double ax[4], xv[4], md[4];
      ld4(sl.AX + (size_t)col * ld + cl, ax);
      ld4(sl.X + (size_t)col * ld + cl, xv);
      ld4(sl.Md + cl, md);
      o.x = (float)(T)(ax[0] - lam * md[0] * xv[0]);
      o.y = (float)(T)(ax[1] - lam * md[1] * xv[1]);
      o.z = (float)(T)(ax[2] - lam * md[2] * xv[2]);
      o.w = (float)(T)(ax[3] - lam * md[3] * xv[3]);
      return b * ldc + cl;
    };
    for (int e = threadIdx.x; e < tot; e += 2 * bd) {
      float4 o0, o1;
      const int d0 = resid4(e, o0);
      const int d1 = e + bd < tot ? resid4(e + bd, o1) : -1;
      *reinterpret_cast<float4*>(u + d0) = o0;
      if (d1 >= 0) *reinterpret_cast<float4*>(u + d1) = o1;
    }
    const int tail = nc - 4 * ng;  // cells past the last group of four
    for (int e = threadIdx.x; e < nb * tail; e += bd) {
      const int b = e / tail, cl = 4 * ng + e % tail;
      const int col = es.act[c0 + b];
      const double r = sl.AX[(size_t)col * ld + cl] - es.lam[col] * sl.Md[cl] * (double)sl.X[(size_t)col * ld + cl];
      u[(size_t)b * ldc + cl] = (float)(T)r;
    }
  }
  if (threadIdx.x == 0) {
    const bool ok = mbar_wait_bounded(bar);
    *flag = ok ? 0 : 1;
    if (!ok) atomicOr(a.nactive + 3, 1);
  }
  __syncthreads();
  if (*flag) return;
  const int t = threadIdx.x, jj = t % ny, kk = t / ny;
  const bool line = t < ny * nz;
  const int nplanes = nx + ny + nz - 2;
  for (int d = 0; d < nplanes; ++d) {
    const int i = d - jj - kk;
    if (line && i >= 0 && i < nx) {
      const int cl = (kk * ny + jj) * nx + i;
      const float cz_ = ctz[cl], cy_ = cty[cl], cx_ = ctx[cl], ci = cinv[cl];
#pragma unroll 4
      for (int b = 0; b < nb; ++b) {
        float* ub = u + b * ldc;
        float sacc = ub[cl];
        if (kk > 0) sacc += cz_ * ub[cl - nxny];
        if (jj > 0) sacc += cy_ * ub[cl - nx];
        if (i > 0) sacc += cx_ * ub[cl - 1];
        ub[cl] = sacc * ci;
      }
    }
    __syncthreads();
  }
  for (int d = nplanes - 1; d >= 0; --d) {
    const int i = d - jj - kk;
    if (line && i >= 0 && i < nx) {
      const int cl = (kk * ny + jj) * nx + i;
      const float cxp = i < nx - 1 ? ctx[cl + 1] : 0.0f;
      const float cyp = jj < ny - 1 ? cty[cl + nx] : 0.0f;
      const float czp = kk < nz - 1 ? ctz[cl + nxny] : 0.0f;
      const float ci = cinv[cl];
#pragma unroll 4
      for (int b = 0; b < nb; ++b) {
        float* ub = u + b * ldc;
        float sacc = 0.0f;
        if (i < nx - 1) sacc += cxp * ub[cl + 1];
        if (jj < ny - 1) sacc += cyp * ub[cl + nx];
        if (kk < nz - 1) sacc += czp * ub[cl + nxny];
        ub[cl] = ub[cl] + sacc * ci;
      }
    }
    __syncthreads();
  }
  if (sizeof(T) == 4) smem_neumann64(u, ldc, nb, nx, ny, nz, ctx, cty, ctz, sl.dN32, sl.AW + (size_t)c0 * ld, ld);
  store_cols_from_smem(sl.W + (size_t)c0 * ld, ld, nb, nc, u, ldc);
}

// FP64 A-images: out_j = A v_j for columns j of the block chosen by `which`
// (0: W -> AW, FP64 operator; 1: X -> AX and P -> AP, FP32-rounded couplings).
template <typename T>
__global__ void __launch_bounds__(256) k_eb_aimg(EbArgs a, int which) {
  const int s = eb_sub(a, blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done || (which == 1 && es.restart)) return;
  const int col = blockIdx.x;
  const SubInfo S = a.subs[s];
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
  const int ld = a.ld;
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, ld);
  if (which == 0) {
    if (col >= es.nact) return;
    neumann_apply_col(a.g, S, a.tx, a.ty, a.tz, sl.dN, sl.W + (size_t)col * ld, sl.AW + (size_t)col * ld, nc);
    return;
  }
  const bool isP = col >= a.m;
  const int j = isP ? col - a.m : col;
  const T* v = (isP ? sl.P : sl.X) + (size_t)j * ld;
  double* out = (isP ? sl.AP : sl.AX) + (size_t)j * ld;
  // cell coordinates advanced incrementally (no division per cell)
  const int sti = blockDim.x % nx, stl = blockDim.x / nx;
  int i = threadIdx.x % nx, jj = (threadIdx.x / nx) % ny, kk = threadIdx.x / nxny;
  for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
    if (cl != (int)threadIdx.x) {
      i += sti;
      int dl = stl;
      if (i >= nx) {
        i -= nx;
        ++dl;
      }
      jj += dl;
      while (jj >= ny) {
        jj -= ny;
        ++kk;
      }
    }
    double r = sl.dN32[cl] * (double)(float)v[cl];
    if (i > 0) r -= (double)sl.ctx[cl] * (double)(float)v[cl - 1];
    if (i < nx - 1) r -= (double)sl.ctx[cl + 1] * (double)(float)v[cl + 1];
    if (jj > 0) r -= (double)sl.cty[cl] * (double)(float)v[cl - nx];
    if (jj < ny - 1) r -= (double)sl.cty[cl + nx] * (double)(float)v[cl + nx];
    if (kk > 0) r -= (double)sl.ctz[cl] * (double)(float)v[cl - nxny];
    if (kk < nz - 1) r -= (double)sl.ctz[cl + nxny] * (double)(float)v[cl + nxny];
    out[cl] = r;
  }
}

// Partial Grams (w S)^T S and S^T (A S), S = [X W P], over one chunk of cells.
template <typename T>
__global__ void __launch_bounds__(256, 2) k_eb_gram(EbArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* red = reinterpret_cast<double*>(smraw);
  const int s = eb_sub(a, blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int cn = min(nc - c0, EB_CHUNK);
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  double* G = a.gpart + ((size_t)s * a.nchunk + blockIdx.x) * 2 * LB_LD * LB_LD;
  Seg3<T> sS{{sl.X + c0, sl.W + c0, sl.P + c0}, {a.m, es.nact, es.np}, a.ld};
  Seg3<double> sA{{sl.AX + c0, sl.AW + c0, sl.AP + c0}, {a.m, es.nact, es.np}, a.ld};
  if (es.nS <= 16)  // the exact tile count: no zero tiles multiplied
    cta_gram2_mma<T, double, 2>(sS, sA, sl.Md + c0, cn, G, G + LB_LD * LB_LD, red);
  else if (es.nS <= 24)
    cta_gram2_mma<T, double, 3>(sS, sA, sl.Md + c0, cn, G, G + LB_LD * LB_LD, red);
  else
    cta_gram2_mma<T, double, 4>(sS, sA, sl.Md + c0, cn, G, G + LB_LD * LB_LD, red);
}

// Rayleigh-Ritz on the chunk-summed Grams (k_lobpcg's cta_rayleigh_ritz).
__global__ void __launch_bounds__(256) k_eb_rr(EbArgs a, double drop) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbSmall& sm = *reinterpret_cast<LbSmall*>(smraw);
  LbMats& mt = *reinterpret_cast<LbMats*>(smraw + sizeof(LbSmall));
  const int s = eb_sub(a, blockIdx.x);
  EbState& es = a.state[s];
  if (es.done) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int nch = (nc + EB_CHUNK - 1) / EB_CHUNK;
  const int nS = es.nS, m = a.m;
  for (int e = threadIdx.x; e < nS * nS; e += blockDim.x) {
    const int r = e / nS, c = e % nS;
    double gm = 0.0, ga = 0.0;
    for (int q = 0; q < nch; ++q) {
      const double* G = a.gpart + ((size_t)s * a.nchunk + q) * 2 * LB_LD * LB_LD;
      gm += G[r * LB_LD + c];
      ga += G[LB_LD * LB_LD + r * LB_LD + c];
    }
    mt.GM[r * LB_LD + c] = gm;
    mt.GA[r * LB_LD + c] = ga;
  }
  if (threadIdx.x < LB_MM) sm.lam[threadIdx.x] = threadIdx.x < m ? es.lam[threadIdx.x] : 0.0;
  if (threadIdx.x == 0) sm.scal[0] = es.lscale;
  __syncthreads();
  const int q = cta_rayleigh_ritz(sm, mt, nS, m, drop, 1e-11, nullptr, mt.GM);
  double* Y = a.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int e = threadIdx.x; e < nS * m; e += blockDim.x) {
    const int r = e / m, c = e % m;
    Y[r * LB_LD + c] = mt.Y[r * LB_LD + c];
  }
  if (threadIdx.x < m) es.lam[threadIdx.x] = sm.lam[threadIdx.x];
  if (threadIdx.x == 0) {
    es.restart = q < m ? 1 : 0;  // basis collapsed: no update, next iteration without P
    es.hasP = q < m ? 0 : 1;
  }
}

// X <- S Y, P <- [W P] Y_WP (and the FP64 A-images in FP64 storage), per chunk.
// NK / NJ: k-steps and 8-column tiles of the tensor-core update (6 / 1 for m <= 8);
// ST: groups of 8 cells each warp has loading while it multiplies one (1 or 2).
template <typename T, int NK, int NJ, int ST>
__global__ void __launch_bounds__(256, (NJ == 1 && ST == 1) ? 3 : 2) k_eb_update(EbArgs a) {
  __shared__ double Ys[LB_LD * LB_LD];
  const int s = eb_sub(a, blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done || es.restart) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int cn = min(nc - c0, EB_CHUNK);
  const double* Y = a.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int e = threadIdx.x; e < es.nS * LB_LD; e += blockDim.x) Ys[e] = Y[e];
  __syncthreads();
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  const int m = a.m;
  cta_update_mma<T, NK, NJ, ST>(sl.X + c0, sl.W + c0, sl.P + c0, m, es.nact, es.np, m, Ys, cn, a.ld);
  if (sizeof(T) == 8)
    cta_update_mma<double, NK, NJ, ST>(sl.AX + c0, sl.AW + c0, sl.AP + c0, m, es.nact, es.np, m, Ys, cn, a.ld);
}

// k_eb_update with the CUDA-core update (m <= 8 block columns)
template <typename T>
__global__ void __launch_bounds__(256, 2) k_eb_update_cc(EbArgs a) {
  __shared__ double Ys[LB_LD * LB_LD];
  const int s = eb_sub(a, blockIdx.y);
  const EbState& es = a.state[s];
  if (es.done || es.restart) return;
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int cn = min(nc - c0, EB_CHUNK);
  const double* Y = a.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int e = threadIdx.x; e < es.nS * LB_LD; e += blockDim.x) Ys[e] = Y[e];
  __syncthreads();
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  const int m = a.m;
  cta_update_cc<T, 8>(sl.X + c0, sl.W + c0, sl.P + c0, m, es.nact, es.np, m, Ys, cn, a.ld);
  if (sizeof(T) == 8)
    cta_update_cc<double, 8>(sl.AX + c0, sl.AW + c0, sl.AP + c0, m, es.nact, es.np, m, Ys, cn, a.ld);
}

// ---- final phase (k_lobpcg mode 2 as phase kernels over every subdomain of
// the list): FP64 A-images of X, Grams of X, the FP64 Rayleigh-Ritz with the
// adaptive count (:369-383) and the output of the k_i wanted vectors.  Run at
// full occupancy instead of one register-heavy CTA per SM.  After this phase
// the state's nact / np / best hold the kept count, the snap flag and the
// value of the snapped constant vector.
__device__ __forceinline__ int eb_full(const EbArgs& a, int idx) { return a.list ? a.list[idx] : idx; }

template <typename T>
__global__ void __launch_bounds__(256) k_eb_fin_aimg(EbArgs a) {
  const int s = eb_full(a, blockIdx.y);
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  const int col = blockIdx.x;
  neumann_apply_col(a.g, S, a.tx, a.ty, a.tz, sl.dN, sl.X + (size_t)col * a.ld, sl.AX + (size_t)col * a.ld, nc);
}

template <typename T>
__global__ void __launch_bounds__(256, 2) k_eb_fin_gram(EbArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  double* red = reinterpret_cast<double*>(smraw);
  const int s = eb_full(a, blockIdx.y);
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int cn = min(nc - c0, EB_CHUNK);
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  double* G = a.gpart + ((size_t)s * a.nchunk + blockIdx.x) * 2 * LB_LD * LB_LD;
  Seg3<T> sS{{sl.X + c0, sl.X + c0, sl.X + c0}, {a.m, 0, 0}, a.ld};
  Seg3<double> sA{{sl.AX + c0, sl.AX + c0, sl.AX + c0}, {a.m, 0, 0}, a.ld};
  if (a.m <= 8)
    cta_gram2_mma<T, double, 1>(sS, sA, sl.Md + c0, cn, G, G + LB_LD * LB_LD, red);
  else
    cta_gram2_mma<T, double, 2>(sS, sA, sl.Md + c0, cn, G, G + LB_LD * LB_LD, red);
}

template <typename T>
__global__ void __launch_bounds__(256) k_eb_fin_rr(EbArgs a, double eb, int dmask, double* evals, int* iters,
                                                   int* status, int* ks) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbSmall& sm = *reinterpret_cast<LbSmall*>(smraw);
  LbMats& mt = *reinterpret_cast<LbMats*>(smraw + sizeof(LbSmall));
  const int s = eb_full(a, blockIdx.x);
  EbState& es = a.state[s];
  const SubInfo S = a.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int nch = (nc + EB_CHUNK - 1) / EB_CHUNK;
  const int m = a.m, k = a.k;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int r = e / m, c = e % m;
    double gm = 0.0, ga = 0.0;
    for (int q = 0; q < nch; ++q) {
      const double* G = a.gpart + ((size_t)s * a.nchunk + q) * 2 * LB_LD * LB_LD;
      gm += G[r * LB_LD + c];
      ga += G[LB_LD * LB_LD + r * LB_LD + c];
    }
    mt.GM[r * LB_LD + c] = gm;
    mt.GA[r * LB_LD + c] = ga;
  }
  if (threadIdx.x < LB_MM) sm.lam[threadIdx.x] = threadIdx.x < m ? es.lam[threadIdx.x] : 0.0;
  if (threadIdx.x == 0) sm.scal[0] = es.lscale;
  __syncthreads();
  cta_rayleigh_ritz(sm, mt, m, m, 1e-14, 1e-14);
  if (threadIdx.x == 0) {
    int num = k;
    for (int j = 0; j < k; ++j)
      if (sm.lam[j] >= eb) {
        num = j + 1;
        break;
      }
    sm.ival[1] = num;
    ks[s] = num;
    iters[s] = es.it;
    status[s] = es.conv ? (es.stag ? 2 : 0) : 1;
  }
  __syncthreads();
  const int num = sm.ival[1];
  if (threadIdx.x < k) evals[(long long)s * k + threadIdx.x] = sm.lam[threadIdx.x];
  double* Y = a.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
    const int r = e / m, c = e % m;
    Y[r * LB_LD + c] = mt.Y[r * LB_LD + c];
  }
  // FP32 storage, subdomain touching no Dirichlet face: the lowest vector is
  // the constant; write it exactly (M-normalised, sign of the computed one)
  bool snap = false;
  double cval = 0.0;
  if (sizeof(T) == 4 && num >= 1) {
    const bool touches = touches_dirichlet(eig_geom(a.probs, a.g, 0.0, 0.0, 0.0, 0.0, dmask, S), S);
    if (!touches) {
      EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
      double msum = 0.0, vsum = 0.0;
      for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
        double v0 = 0.0;
        for (int b = 0; b < m; ++b) v0 += (double)sl.X[(size_t)b * a.ld + cl] * mt.Y[b * LB_LD];
        msum += sl.Md[cl];
        vsum += sl.Md[cl] * v0;
      }
      msum = block_sum(msum, sm.res);
      vsum = block_sum(vsum, sm.res);
      snap = msum > 0.0;
      cval = snap ? copysign(1.0 / sqrt(msum), vsum) : 0.0;
    }
  }
  if (threadIdx.x == 0) {
    es.nact = num;
    es.np = snap ? 1 : 0;
    es.best = cval;
  }
}

template <typename T>
__global__ void __launch_bounds__(256) k_eb_fin_out(EbArgs a, int kmax, T* phi) {
  __shared__ double Ys[LB_LD * LB_LD];
  const int s = eb_full(a, blockIdx.y);
  const EbState& es = a.state[s];
  const SubInfo S = a.subs[s];
  const int nx = S.nx, ny = S.ny, nc = nx * ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int c1 = min(nc, c0 + EB_CHUNK);
  const double* Y = a.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int e = threadIdx.x; e < a.m * LB_LD; e += blockDim.x) Ys[e] = Y[e];
  __syncthreads();
  const int m = a.m, num = es.nact;
  const bool snap = es.np != 0;
  const double cval = es.best;
  EbSlab<T> sl(a.slab + (size_t)s * a.slab_stride, a.m, a.ld);
  for (int cl = c0 + threadIdx.x; cl < c1; cl += blockDim.x) {
    const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
    const long long cg = ((long long)(S.z0 + kz_) * a.g.N + (S.y0 + jy)) * a.g.M + (S.x0 + i);
    double xr[LB_MM];
#pragma unroll
    for (int b = 0; b < LB_MM; ++b) xr[b] = b < m ? (double)sl.X[(size_t)b * a.ld + cl] : 0.0;
    for (int j = 0; j < kmax; ++j) {
      double v = 0.0;
      if (j < num) {
#pragma unroll
        for (int b = 0; b < LB_MM; ++b)
          if (b < m) v += xr[b] * Ys[b * LB_LD + j];
      }
      if (snap && j == 0) v = cval;
      phi[cg * kmax + j] = (T)v;
    }
  }
}

// ---- set-up phase (k_lobpcg mode 1 as phase kernels over every subdomain of
// the list): mass and Neumann diagonals, FP32 sweep coefficients, IC(0) pivots
// of A^N + sigma M and the initial block (one CTA per subdomain), the
// A-images of the block, its Grams, the first Rayleigh-Ritz with the state
// initialisation, and the rotation of X and A X by the Ritz coefficients.
template <typename T>
__global__ void __launch_bounds__(256) k_eb_init_a(EbArgs e, LobpcgArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ double red[32];
  const int ldc = e.ldc;
  double* Dtmp = reinterpret_cast<double*>(smraw);
  float* ctx = reinterpret_cast<float*>(Dtmp + ldc);
  float* cty = ctx + ldc;
  float* ctz = cty + ldc;
  const int s = eb_full(e, blockIdx.x);
  EbState& es = e.state[s];
  const SubInfo S = e.subs[s];
  const Grid g = e.g;
  const EigGeom eg = eig_geom(a.probs, g, a.Hx, a.Hy, a.Hz, a.meas, a.dirichlet_mask, S);
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
  const int m = e.m, ld = e.ld;
  EbSlab<T> sl(e.slab + (size_t)s * e.slab_stride, m, ld);
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
      if (i == 0 && ex >= 1) mv += 2.0 * avg_k(a.kx[cg - 1], a.kx[cg]) / eg.Hx / eg.Hx;
      if (ex + 1 != g.M) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / eg.Hx / eg.Hx;
      if (ey >= 1) mv += 2.0 * avg_k(a.ky[cg - g.M], a.ky[cg]) / eg.Hy / eg.Hy;
      if (ey + 1 != g.N) mv += 2.0 * avg_k(a.ky[cg], a.ky[cg + g.M]) / eg.Hy / eg.Hy;
      if (ez >= 1) mv += 2.0 * avg_k(a.kz[cg - g.MN], a.kz[cg]) / eg.Hz / eg.Hz;
      if (ez + 1 != g.P) mv += 2.0 * avg_k(a.kz[cg], a.kz[cg + g.MN]) / eg.Hz / eg.Hz;
      if (i + 1 < nx) mv += 2.0 * avg_k(a.kx[cg], a.kx[cg + 1]) / eg.Hx / eg.Hx;
      if (eg.dmask & 1 && ex == 0) mv += 2.0 * (2.0 * a.kx[cg]) / eg.Hx / eg.Hx;
      if (eg.dmask & 2 && ex == eg.M - 1) mv += 2.0 * (2.0 * a.kx[cg]) / eg.Hx / eg.Hx;
      if (eg.dmask & 4 && ey == 0) mv += 2.0 * (2.0 * a.ky[cg]) / eg.Hy / eg.Hy;
      if (eg.dmask & 8 && ey == eg.N - 1) mv += 2.0 * (2.0 * a.ky[cg]) / eg.Hy / eg.Hy;
      if (eg.dmask & 16 && ez == eg.z0) mv += 2.0 * (2.0 * a.kz[cg]) / eg.Hz / eg.Hz;
      if (eg.dmask & 32 && ez == eg.z1 - 1) mv += 2.0 * (2.0 * a.kz[cg]) / eg.Hz / eg.Hz;
      mv = mv * eg.meas;
    }
    sl.Md[cl] = mv;
    sl.dN[cl] = dn;
    double d32 = a.db[cg];
    if (i > 0) d32 += (double)(float)a.tx[cg];
    if (i < nx - 1) d32 += (double)(float)a.tx[cg + 1];
    if (j > 0) d32 += (double)(float)a.ty[cg];
    if (j < ny - 1) d32 += (double)(float)a.ty[cg + g.M];
    if (kk > 0) d32 += (double)(float)a.tz[cg];
    if (kk < nz - 1) d32 += (double)(float)a.tz[cg + g.MN];
    sl.dN32[cl] = d32;
    const float fx = i > 0 ? (float)a.tx[cg] : 0.0f, fy = j > 0 ? (float)a.ty[cg] : 0.0f,
                fz = kk > 0 ? (float)a.tz[cg] : 0.0f;
    ctx[cl] = fx;
    cty[cl] = fy;
    ctz[cl] = fz;
    sl.ctx[cl] = fx;
    sl.cty[cl] = fy;
    sl.ctz[cl] = fz;
    ratio = fmax(ratio, dn / mv);
  }
  for (int o = 16; o > 0; o >>= 1) ratio = fmax(ratio, __shfl_xor_sync(0xffffffffu, ratio, o));
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = ratio;
  __syncthreads();
  double r = 0.0;
  for (int wi = 0; wi < (int)(blockDim.x >> 5); ++wi) r = fmax(r, red[wi]);
  const double lscale = r > 0 ? r : 1.0;
  const double sigma = a.sigma_rel * lscale;
  // IC(0) pivots of A^N + sigma M (wavefront, natural order, FP64)
  const int t = threadIdx.x, jj = t % ny, kk = t / ny;
  const bool line = t < ny * nz;
  const int nplanes = nx + ny + nz - 2;
  for (int d = 0; d < nplanes; ++d) {
    const int i = d - jj - kk;
    if (line && i >= 0 && i < nx) {
      const int cl = (kk * ny + jj) * nx + i;
      double sacc = 0.0;
      if (kk > 0) sacc += (double)ctz[cl] * (double)ctz[cl] / Dtmp[cl - nxny];
      if (jj > 0) sacc += (double)cty[cl] * (double)cty[cl] / Dtmp[cl - nx];
      if (i > 0) sacc += (double)ctx[cl] * (double)ctx[cl] / Dtmp[cl - 1];
      double D = sl.dN[cl] + sigma * sl.Md[cl] - sacc;
      if (!(D > 0.0)) D = sl.dN[cl] + sigma * sl.Md[cl];
      Dtmp[cl] = D;
      sl.cinv[cl] = (float)(1.0 / D);
    }
    __syncthreads();
  }
  // initial block: the learned patch columns, a given block, or random
  for (int q = threadIdx.x; q < m * nc; q += blockDim.x) {
    const int j = q / nc, cl = q % nc;
    double v;
    if (a.xinit_patch && j < a.xinit_k) {
      const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
      v = a.xinit_patch[((size_t)s * 4096 + (kz_ * 16 + jy) * 16 + i) * 16 + j];
    } else if (a.xinit) {
      const int i = cl % nx, tt = cl / nx, jy = tt % ny, kz_ = tt / ny;
      const long long cg = ((long long)(S.z0 + kz_) * g.N + (S.y0 + jy)) * g.M + (S.x0 + i);
      v = a.xinit[cg * m + j];
    } else {
      v = hash_uniform(a.seed ^ ((unsigned long long)s << 32) ^ (unsigned long long)q);
    }
    sl.X[(size_t)j * ld + cl] = (T)v;
  }
  if (threadIdx.x == 0) es.lscale = lscale;
}

// A X of the initial block: FP64 operator in FP64 storage; in FP32 storage the
// FP32-rounded couplings and diagonal, as the lock-step A-images use them.
template <typename T>
__global__ void __launch_bounds__(256) k_eb_init_aimg(EbArgs e) {
  const int s = eb_full(e, blockIdx.y);
  const SubInfo S = e.subs[s];
  const int nx = S.nx, ny = S.ny, nz = S.nz, nxny = nx * ny, nc = nxny * nz;
  const int ld = e.ld, col = blockIdx.x;
  EbSlab<T> sl(e.slab + (size_t)s * e.slab_stride, e.m, ld);
  if (sizeof(T) == 8) {
    neumann_apply_col(e.g, S, e.tx, e.ty, e.tz, sl.dN, sl.X + (size_t)col * ld, sl.AX + (size_t)col * ld, nc);
    return;
  }
  const T* v = sl.X + (size_t)col * ld;
  double* out = sl.AX + (size_t)col * ld;
  for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
    const int i = cl % nx, tt = cl / nx, j = tt % ny, k = tt / ny;
    double r = sl.dN32[cl] * (double)(float)v[cl];
    if (i > 0) r -= (double)sl.ctx[cl] * (double)(float)v[cl - 1];
    if (i < nx - 1) r -= (double)sl.ctx[cl + 1] * (double)(float)v[cl + 1];
    if (j > 0) r -= (double)sl.cty[cl] * (double)(float)v[cl - nx];
    if (j < ny - 1) r -= (double)sl.cty[cl + nx] * (double)(float)v[cl + nx];
    if (k > 0) r -= (double)sl.ctz[cl] * (double)(float)v[cl - nxny];
    if (k < nz - 1) r -= (double)sl.ctz[cl + nxny] * (double)(float)v[cl + nxny];
    out[cl] = r;
  }
}

__global__ void __launch_bounds__(256) k_eb_init_rr(EbArgs e, double drop) {
  extern __shared__ __align__(16) unsigned char smraw[];
  LbSmall& sm = *reinterpret_cast<LbSmall*>(smraw);
  LbMats& mt = *reinterpret_cast<LbMats*>(smraw + sizeof(LbSmall));
  const int s = eb_full(e, blockIdx.x);
  EbState& es = e.state[s];
  const SubInfo S = e.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int nch = (nc + EB_CHUNK - 1) / EB_CHUNK;
  const int m = e.m;
  for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
    const int r = q / m, c = q % m;
    double gm = 0.0, ga = 0.0;
    for (int h = 0; h < nch; ++h) {
      const double* G = e.gpart + ((size_t)s * e.nchunk + h) * 2 * LB_LD * LB_LD;
      gm += G[r * LB_LD + c];
      ga += G[LB_LD * LB_LD + r * LB_LD + c];
    }
    mt.GM[r * LB_LD + c] = gm;
    mt.GA[r * LB_LD + c] = ga;
  }
  if (threadIdx.x < LB_MM) sm.lam[threadIdx.x] = 0.0;
  if (threadIdx.x == 0) sm.scal[0] = es.lscale;
  __syncthreads();
  cta_rayleigh_ritz(sm, mt, m, m, drop, 1e-12);
  double* Y = e.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int q = threadIdx.x; q < m * m; q += blockDim.x) {
    const int r = q / m, c = q % m;
    Y[r * LB_LD + c] = mt.Y[r * LB_LD + c];
  }
  if (threadIdx.x < m) es.lam[threadIdx.x] = sm.lam[threadIdx.x];
  if (threadIdx.x == 0) {
    es.best = 1e300;
    es.last_improve = 0;
    es.hasP = 0;
    es.done = 0;
    es.conv = 0;
    es.stag = 0;
    es.it = 0;
    es.restart = 0;
    es.nact = 0;
    es.np = 0;
    es.nS = m;
  }
}

// X <- X Y and A X <- (A X) Y, cell by cell (in place: every cell's m values
// are read before any is written).
template <typename T>
__global__ void __launch_bounds__(256) k_eb_init_rot(EbArgs e) {
  __shared__ double Ys[LB_LD * LB_LD];
  const int s = eb_full(e, blockIdx.y);
  const SubInfo S = e.subs[s];
  const int nc = S.nx * S.ny * S.nz;
  const int c0 = blockIdx.x * EB_CHUNK;
  if (c0 >= nc) return;
  const int c1 = min(nc, c0 + EB_CHUNK);
  const double* Y = e.Ybuf + (size_t)s * LB_LD * LB_LD;
  for (int q = threadIdx.x; q < e.m * LB_LD; q += blockDim.x) Ys[q] = Y[q];
  __syncthreads();
  const int m = e.m, ld = e.ld;
  EbSlab<T> sl(e.slab + (size_t)s * e.slab_stride, m, ld);
  for (int cl = c0 + threadIdx.x; cl < c1; cl += blockDim.x) {
    double xr[LB_MM], ar[LB_MM];
#pragma unroll
    for (int b = 0; b < LB_MM; ++b) {
      xr[b] = b < m ? (double)sl.X[(size_t)b * ld + cl] : 0.0;
      ar[b] = b < m ? sl.AX[(size_t)b * ld + cl] : 0.0;
    }
#pragma unroll
    for (int j = 0; j < LB_MM; ++j)
      if (j < m) {
        double xn = 0.0, an = 0.0;
#pragma unroll
        for (int b = 0; b < LB_MM; ++b)
          if (b < m) {
            xn += xr[b] * Ys[b * LB_LD + j];
            an += ar[b] * Ys[b * LB_LD + j];
          }
        sl.X[(size_t)j * ld + cl] = (T)xn;
        sl.AX[(size_t)j * ld + cl] = an;
      }
  }
}

}  // namespace

size_t lobpcg_batched_slab_bytes(int max_cells, int m, int prec_bytes) {
  return (lobpcg_work_bytes(max_cells, m, prec_bytes) + 255) & ~(size_t)255;
}
size_t lobpcg_batched_state_bytes() { return sizeof(EbState); }
int lobpcg_batched_nchunk(int max_cells) { return (max_cells + EB_CHUNK - 1) / EB_CHUNK; }

template <typename T>
int launch_lobpcg_batched(const LobpcgArgs& a_in, const EbBuffers& b, const int* list, int nlist, T* phi,
                          double* evals, int* iters, int* status, int* ks, double eb, int max_cells, int max_lines,
                          cudaStream_t st) {
  if (nlist <= 0) return 0;
  // set-up phase: k_lobpcg mode 1 into the per-subdomain slabs
  LobpcgArgs a = a_in;
  a.slab = b.slab;
  a.slab_stride = b.slab_stride;
  a.state = b.state;
  a.sub_list = list;
  a.nlist = nullptr;
  a.nsub = list ? nlist : a_in.nsub;
  const int ctas = 148;
  EbArgs e;
  e.g = a.g;
  e.subs = a.subs;
  e.list = list;
  e.m = a.m;
  e.k = a.k;
  e.ld = lb_ld(max_cells);
  e.ldc = (max_cells + 3) & ~3;
  e.nchunk = b.nchunk;
  e.max_it = a.max_it;
  e.tol = a.tol;
  e.rel_floor = a.rel_floor;
  e.slab = b.slab;
  e.slab_stride = b.slab_stride;
  e.state = reinterpret_cast<EbState*>(b.state);
  e.Ybuf = b.Ybuf;
  e.gpart = b.gpart;
  e.rpart = b.rpart;
  e.nactive = b.nactive;
  e.alist = b.alist;
  e.colcells = b.colcells;
  if (b.colcells) cudaMemsetAsync(b.colcells, 0, sizeof(unsigned long long), st);
  e.tx = a.tx;
  e.ty = a.ty;
  e.tz = a.tz;
  e.probs = a.probs;
  if (a.init_batched) {
    const size_t init_smem = (size_t)20 * e.ldc;  // FP64 pivots + three FP32 coupling arrays
    const size_t rr_smem0 = sizeof(LbSmall) + sizeof(LbMats);
    const size_t gram_smem0 = (size_t)8 * 32 * 32 * sizeof(double);
    cudaFuncSetAttribute(k_eb_init_a<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)init_smem);
    cudaFuncSetAttribute(k_eb_init_rr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rr_smem0);
    cudaFuncSetAttribute(k_eb_fin_gram<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem0);
    { note_launch(); k_eb_init_a<T><<<nlist, 256, init_smem, st>>>(e, a); }
    { note_launch(); k_eb_init_aimg<T><<<dim3(a.m, nlist), 256, 0, st>>>(e); }
    { note_launch(); k_eb_fin_gram<T><<<dim3(e.nchunk, nlist), 256, gram_smem0, st>>>(e); }
    { note_launch(); k_eb_init_rr<<<nlist, 256, rr_smem0, st>>>(e, sizeof(T) == 4 ? 1e-9 : 1e-13); }
    { note_launch(); k_eb_init_rot<T><<<dim3(e.nchunk, nlist), 256, 0, st>>>(e); }
  } else {
    a.mode = 1;
    launch_lobpcg<T>(a, std::min(ctas, nlist), nullptr, phi, evals, iters, status, ks, eb, max_cells, max_lines, st);
  }
  // column batch of the preconditioner: the built-in one keeps coefficients + mb
  // vectors within ~113 KB (2 CTAs per SM); the online tuner also tries all m
  // columns in one CTA (fewer barriers per column, 1 CTA per SM) and one column.
  // coef: the 16-byte header and the four coefficient arrays at pitch ld.
  const size_t coef = (size_t)16 * e.ld + 16;
  e.mb = (int)std::max<size_t>(1, std::min<size_t>(a.m, (113 * 1024 - coef) / ((size_t)4 * e.ldc)));
  int mb_c[3], nmb = 0;
  mb_c[nmb++] = e.mb;
  if (a.m != e.mb && coef + (size_t)4 * e.ldc * a.m <= 220 * 1024) mb_c[nmb++] = a.m;
  if (e.mb != 1) mb_c[nmb++] = 1;
  size_t pre_smem_max = 0;
  for (int q = 0; q < nmb; ++q) pre_smem_max = std::max(pre_smem_max, coef + (size_t)4 * e.ldc * mb_c[q]);
  const size_t gram_smem = (size_t)8 * 32 * 32 * sizeof(double);
  const size_t rr_smem = sizeof(LbSmall) + offsetof(LbMats, stile);  // k_eb_rr stops at the tiles: 3 CTAs / SM
  cudaFuncSetAttribute(k_eb_precond<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)pre_smem_max);
  // basis update tiles: <6,1> (3 CTAs per SM) is the built-in for m <= 8, <8,2> the alternative;
  // candidates 2 / 3 are the same tiles with two groups of cells loading ahead per warp
  // candidate 4 (m <= 8): the CUDA-core update, one cell per thread
  const int nupd = a.m <= 8 ? 5 : 2;
  char kpre[96], kupd[96];
  snprintf(kpre, sizeof(kpre), "eb_precond|%s|m%d|c%d", sizeof(T) == 4 ? "f32" : "f64", a.m, e.ldc);
  snprintf(kupd, sizeof(kupd), "eb_update|%s|m%d|c%d|cc", sizeof(T) == 4 ? "f32" : "f64", a.m, e.ldc);
  cudaEvent_t tev[4];
  for (auto& x : tev) cudaEventCreate(&x);
  int prev_pc = -1, prev_uc = -1, prev_cols = 0, prev_ns = 0;
  // time per unit of work of the previous iteration's launches, read after the
  // iteration's own synchronisation (no extra host waits)
  auto report_prev = [&]() {
    if (prev_pc < 0) return;
    float ms = 0.0f;
    if (cudaEventElapsedTime(&ms, tev[0], tev[1]) == cudaSuccess && prev_cols > 0)
      tune_online_report(kpre, nmb, prev_pc, 1e3f * ms / (float)prev_cols);
    if (cudaEventElapsedTime(&ms, tev[2], tev[3]) == cudaSuccess && prev_ns > 0)
      tune_online_report(kupd, nupd, prev_uc, 1e3f * ms / (float)prev_ns);
    prev_pc = -1;
  };
  cudaFuncSetAttribute(k_eb_gram<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem);
  cudaFuncSetAttribute(k_eb_rr, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)rr_smem);
  const double drop = sizeof(T) == 4 ? 1e-9 : 1e-13;
  // optional phase timing (b.phase_ms, or PMF_PROFILE_EIGEN): device time per phase
  const bool prof = b.phase_ms != nullptr || getenv("PMF_PROFILE_EIGEN") != nullptr;
  cudaEvent_t pev[9];
  float ptot[8] = {0};
  if (prof)
    for (auto& x : pev) cudaEventCreate(&x);
  auto mark = [&](int i) {
    if (prof) cudaEventRecord(pev[i], st);
  };
  mark(0);
  int nact = nlist, lockstep = 0;
  cudaMemsetAsync(b.nactive + 3, 0, sizeof(int), st);  // set by a preconditioner copy that never landed
  for (int it = 0; it < a.max_it; ++it) {
    // residual norms of the subdomains still iterating (all of them at it = 0)
    mark(1);
    { note_launch(); k_eb_resid<T><<<dim3(e.nchunk, nact), 256, 0, st>>>(e, it > 0 ? 1 : 0); }
    cudaMemsetAsync(b.nactive, 0, 3 * sizeof(int), st);
    { note_launch(); k_eb_control<<<(nlist + 127) / 128, 128, 0, st>>>(e, nlist, it); }
    cudaMemcpyAsync(b.h_nactive, b.nactive, 4 * sizeof(int), cudaMemcpyDeviceToHost, st);
    mark(2);
    if (cudaStreamSynchronize(st) != cudaSuccess) return 76;
    report_prev();
    if (prof) {
      float ms;
      cudaEventElapsedTime(&ms, pev[1], pev[2]);
      ptot[0] += ms;
    }
    if (b.h_nactive[3]) return 76;  // a bounded wait in the preconditioner ran out
    nact = b.h_nactive[0];
    if (nact == 0) break;
    ++lockstep;
    const int pc = tune_online_pick(kpre, nmb), uc = tune_online_pick(kupd, nupd);
    EbArgs ep = e;
    ep.mb = mb_c[pc];
    const dim3 gchunk(e.nchunk, nact), gpre((a.m + ep.mb - 1) / ep.mb, nact);
    mark(2);
    cudaEventRecord(tev[0], st);
    { note_launch(); k_eb_precond<T><<<gpre, 256, coef + (size_t)4 * e.ldc * ep.mb, st>>>(ep); }
    cudaEventRecord(tev[1], st);
    if (sizeof(T) == 8) { note_launch(); k_eb_aimg<T><<<dim3(a.m, nact), 256, 0, st>>>(e, 0); }
    mark(3);
    { note_launch(); k_eb_gram<T><<<gchunk, 256, gram_smem, st>>>(e); }
    mark(4);
    { note_launch(); k_eb_rr<<<nact, 256, rr_smem, st>>>(e, drop); }
    mark(5);
    note_launch();
    cudaEventRecord(tev[2], st);
    if (a.m <= 8 && uc == 4)
      k_eb_update_cc<T><<<gchunk, 256, 0, st>>>(e);
    else if (a.m <= 8 && uc == 0)
      k_eb_update<T, 6, 1, 1><<<gchunk, 256, 0, st>>>(e);
    else if (a.m <= 8 && uc == 2)
      k_eb_update<T, 6, 1, 2><<<gchunk, 256, 0, st>>>(e);
    else if (uc == 3 || (a.m > 8 && uc == 1))
      k_eb_update<T, 8, 2, 2><<<gchunk, 256, 0, st>>>(e);
    else
      k_eb_update<T, 8, 2, 1><<<gchunk, 256, 0, st>>>(e);
    cudaEventRecord(tev[3], st);
    prev_pc = pc;
    prev_uc = uc;
    prev_cols = b.h_nactive[1];
    prev_ns = b.h_nactive[2];
    mark(6);
    if (sizeof(T) == 4) { note_launch(); k_eb_aimg<T><<<dim3(2 * a.m, nact), 256, 0, st>>>(e, 1); }
    mark(7);
    if (prof) {
      cudaEventSynchronize(pev[7]);
      float ms;
      for (int q = 2; q < 7; ++q) {
        cudaEventElapsedTime(&ms, pev[q], pev[q + 1]);
        ptot[q - 1] += ms;
      }
    }
  }
  if (cudaStreamSynchronize(st) != cudaSuccess) return 76;
  {
    int fl = 0;  // the last iteration's preconditioner
    if (cudaMemcpy(&fl, b.nactive + 3, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess || fl) return 76;
  }
  report_prev();
  for (auto& x : tev) cudaEventDestroy(x);
  if (prof) {
    if (b.phase_ms) {
      for (int q = 0; q < 6; ++q) b.phase_ms[q] += ptot[q];
      b.phase_ms[6] += lockstep;
    }
    if (getenv("PMF_PROFILE_EIGEN"))
      fprintf(stderr,
              "[premixfem_b200] batched LOBPCG ms: resid+control %.2f precond %.2f gram %.2f rr %.2f update %.2f "
              "a-images %.2f (%d lockstep iterations)\n",
              ptot[0], ptot[1], ptot[2], ptot[3], ptot[4], ptot[5], lockstep);
    for (auto& x : pev) cudaEventDestroy(x);
  }
  // final phase: FP64 Rayleigh-Ritz, adaptive count, output
  if (a.final_batched) {
    const size_t fin_rr_smem = sizeof(LbSmall) + sizeof(LbMats);
    cudaFuncSetAttribute(k_eb_fin_rr<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)fin_rr_smem);
    cudaFuncSetAttribute(k_eb_fin_gram<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)gram_smem);
    { note_launch(); k_eb_fin_aimg<T><<<dim3(a.m, nlist), 256, 0, st>>>(e); }
    { note_launch(); k_eb_fin_gram<T><<<dim3(e.nchunk, nlist), 256, gram_smem, st>>>(e); }
    { note_launch(); k_eb_fin_rr<T><<<nlist, 256, fin_rr_smem, st>>>(e, eb, a.dirichlet_mask, evals, iters, status, ks); }
    { note_launch(); k_eb_fin_out<T><<<dim3(e.nchunk, nlist), 256, 0, st>>>(e, a.kmax, phi); }
    return cudaGetLastError() == cudaSuccess ? 0 : 76;
  }
  // final phase as one persistent launch: k_lobpcg mode 2
  a.mode = 2;
  launch_lobpcg<T>(a, std::min(ctas, nlist), nullptr, phi, evals, iters, status, ks, eb, max_cells, max_lines, st);
  return cudaGetLastError() == cudaSuccess ? 0 : 76;
}
template int launch_lobpcg_batched<float>(const LobpcgArgs&, const EbBuffers&, const int*, int, float*, double*, int*,
                                          int*, int*, double, int, int, cudaStream_t);
template int launch_lobpcg_batched<double>(const LobpcgArgs&, const EbBuffers&, const int*, int, double*, double*,
                                           int*, int*, int*, double, int, int, cudaStream_t);

}  // namespace pmf
