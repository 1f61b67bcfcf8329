// The global coarse problem of -use_2level (_PC_setup_lv2_c,
// src/PreMixFEM_3D.c:423-735, factorised there by SuperLU_dist at :714-728,
// and applied by _PC_apply_vec_lv2_2level, :1481-1537) as a banded FP64
// Cholesky factorisation.
//
// A2 = Phi^T A Phi couples a subdomain's k dofs to its six face neighbours
// only.  Numbered in subdomain-grid order with the axis of most subdomains
// slowest, it is banded with half-bandwidth b = k * n0 * n1 + k - 1 (n0, n1
// the two smaller subdomain counts): 1 541 for the 256^3 workload (24 576
// unknowns), 4 103 for 512 x 512 x 256 (131 072 unknowns).
//
// Storage: w x w tiles (w = 64) of the lower band, T[I][d] = tile (I, I - d),
// d = 0 .. B with B = ceil((b + w - 1) / w) - the tile bandwidth; rows are
// padded to NS * B tiles with identity.
//
// Factorisation (right-looking, tiled): for each tile column K, POTRF of the
// diagonal tile (one CTA), TRSM of the B tiles below it (one CTA each), and
// the SYRK / GEMM update of the B(B+1)/2 trailing tiles (one CTA each).  A
// pivot at or below tol x max|diag(A2)| is a null direction: its column of L
// is zeroed and it is kept out of the solve, as the oracle's semidefinite
// Cholesky does (the singular coarse matrices of pure-Neumann problems).
//
// Solve: in superblocks of B tiles L is block bidiagonal, so with the
// inverses X_m of the diagonal superblocks (computed once, null rows zeroed)
//   forward   y_m = X_m (c_m - L_{m,m-1} y_{m-1}),
//   backward  x_m = X_m^T (y_m - L_{m+1,m}^T x_{m+1}),
// dense matrix-vector products streaming each superblock once: a warp per row
// forward; backward (transposed products) one CTA per 64 x 64 tile writing
// column partial sums, added per column in a fixed order by a second launch.
#include <algorithm>
#include <vector>

#include "pmf_kernels.h"

namespace pmf {

namespace {
constexpr int W = 64;          // tile size
constexpr int kTileThreads = 256;

__device__ __forceinline__ double* tile_ptr(double* T, int B, int I, int d) {
  return T + ((long long)I * (B + 1) + d) * (W * W);
}
__device__ __forceinline__ const double* tile_ptr(const double* T, int B, int I, int d) {
  return T + ((long long)I * (B + 1) + d) * (W * W);
}
// superblock inverse tile (i, j), j <= i, of superblock m
__device__ __forceinline__ double* xtile(double* X, int B, int m, int i, int j) {
  return X + (((long long)m * B + i) * B + j) * (W * W);
}
__device__ __forceinline__ const double* xtile(const double* X, int B, int m, int i, int j) {
  return X + (((long long)m * B + i) * B + j) * (W * W);
}
}  // namespace

// A2 (+ shift) in tile-band storage.  perm[g] = natural coarse dof of grid
// dof g (-1: padding); identity rows for padding and for unused basis
// columns (j >= k_s).
__global__ void k_cband_assemble(const SubInfo* subs, int kmax, const double* blk, const int* perm, int NTp, int B,
                                 double shift, double* T) {
  const long long total = (long long)NTp * (B + 1) * W * W;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const long long t = e / (W * W);
    const int rc = (int)(e % (W * W)), r = rc / W, c = rc % W;
    const int I = (int)(t / (B + 1)), d = (int)(t % (B + 1));
    const int J = I - d;
    double v = 0.0;
    if (J >= 0 && !(d == 0 && c > r)) {
      const long long gi = (long long)I * W + r, gj = (long long)J * W + c;
      const int ni = perm[gi], nj = perm[gj];
      if (ni < 0 || nj < 0) {
        v = gi == gj ? 1.0 : 0.0;
      } else {
        const int si = ni / kmax, ai = ni % kmax, sj = nj / kmax, aj = nj % kmax;
        const SubInfo& S = subs[si];
        if (ai >= S.k || aj >= subs[sj].k) {
          v = gi == gj ? 1.0 : 0.0;
        } else if (si == sj) {
          v = blk[(((long long)si * 7) * kmax + ai) * kmax + aj];
          if (gi == gj) v += shift;
        } else {
          for (int f = 0; f < 6; ++f)
            if (S.nb[f] == sj) v = blk[(((long long)si * 7 + 1 + f) * kmax + ai) * kmax + aj];
        }
      }
    }
    T[e] = v;
  }
}

// max |diagonal| of the assembled matrix (the null-pivot scale), one CTA
__global__ void k_cband_diag_max(const double* T, int NTp, int B, double* out) {
  __shared__ double red[32];
  double m = 0.0;
  for (long long i = threadIdx.x; i < (long long)NTp * W; i += blockDim.x) {
    const int I = (int)(i / W), r = (int)(i % W);
    m = fmax(m, fabs(tile_ptr(T, B, I, 0)[r * W + r]));
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, red[w]);
    *out = v > 0.0 ? v : 1.0;
  }
}

// Cholesky of the diagonal tile K in shared memory; null pivots flagged.
__global__ void __launch_bounds__(kTileThreads) k_cband_potrf(double* T, int B, int K, const double* scale,
                                                                double tol, int* nullf, int* nnull) {
  __shared__ double a[W][W + 1];
  double* tk = tile_ptr(T, B, K, 0);
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) a[e / W][e % W] = tk[e];
  __syncthreads();
  const double thr = tol * (*scale);
  __shared__ int isnull;
  for (int k = 0; k < W; ++k) {
    if (threadIdx.x == 0) {
      const double d = a[k][k];
      isnull = !(d > thr);
      a[k][k] = isnull ? 1.0 : sqrt(d);
      nullf[K * W + k] = isnull;
      if (isnull) atomicAdd(nnull, 1);
    }
    __syncthreads();
    const double p = a[k][k];
    for (int i = k + 1 + threadIdx.x; i < W; i += blockDim.x) a[i][k] = isnull ? 0.0 : a[i][k] / p;
    __syncthreads();
    // trailing update of the lower triangle
    const int m = W - k - 1;
    for (int e = threadIdx.x; e < m * m; e += blockDim.x) {
      const int i = k + 1 + e / m, j = k + 1 + e % m;
      if (j <= i) a[i][j] -= a[i][k] * a[j][k];
    }
    __syncthreads();
  }
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
    const int i = e / W, j = e % W;
    tk[e] = j <= i ? a[i][j] : 0.0;
  }
}

// Tiles below the diagonal tile K: L(I, K) = A(I, K) L(K, K)^-T, one CTA per
// tile; columns of null pivots are zero.
__global__ void __launch_bounds__(kTileThreads) k_cband_trsm(double* T, int B, int K, int NTp, const int* nullf) {
  const int I = K + 1 + blockIdx.x;
  if (I >= NTp || I - K > B) return;
  extern __shared__ double cb_sm[];
  double(*L)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm);
  double(*X)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm + W * (W + 1));
  const double* lk = tile_ptr(T, B, K, 0);
  double* ti = tile_ptr(T, B, I, I - K);
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
    L[e / W][e % W] = lk[e];
    X[e / W][e % W] = ti[e];
  }
  __syncthreads();
  // row r of X solves x L^T = a: x_c = (a_c - sum_{c' < c} x_c' L[c][c']) / L[c][c]
  if (threadIdx.x < W) {
    const int r = threadIdx.x;
    for (int c = 0; c < W; ++c) {
      double s = X[r][c];
      for (int c2 = 0; c2 < c; ++c2) s -= X[r][c2] * L[c][c2];
      X[r][c] = nullf[K * W + c] ? 0.0 : s / L[c][c];
    }
  }
  __syncthreads();
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) ti[e] = X[e / W][e % W];
}

// Trailing update A(I, J) -= L(I, K) L(J, K)^T for K < J <= I <= K + B, one CTA
// per tile pair; each thread computes a 4 x 4 block of the 64 x 64 tile.
__global__ void __launch_bounds__(kTileThreads) k_cband_syrk(double* T, int B, int K, int NTp) {
  // blockIdx.x -> (dI, dJ), 1 <= dJ <= dI <= B, in row order of the lower triangle
  int dI = 1, rem = blockIdx.x;
  while (rem >= dI) {
    rem -= dI;
    ++dI;
  }
  const int dJ = rem + 1;
  const int I = K + dI, J = K + dJ;
  if (I >= NTp || dI > B) return;
  extern __shared__ double cb_sm[];
  double(*A)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm);
  double(*Bt)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm + W * (W + 1));
  const double* li = tile_ptr(T, B, I, I - K);
  const double* lj = tile_ptr(T, B, J, J - K);
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
    A[e / W][e % W] = li[e];
    Bt[e / W][e % W] = lj[e];
  }
  __syncthreads();
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;  // 16 x 16 threads, 4 x 4 outputs each
  double acc[4][4] = {};
  for (int k = 0; k < W; ++k) {
    double av[4], bv[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      av[q] = A[tr + 16 * q][k];
      bv[q] = Bt[tc + 16 * q][k];
    }
#pragma unroll
    for (int q = 0; q < 4; ++q)
#pragma unroll
      for (int p = 0; p < 4; ++p) acc[q][p] += av[q] * bv[p];
  }
  double* cij = tile_ptr(T, B, I, I - J);
  const bool diag = I == J;
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int r = tr + 16 * q, c = tc + 16 * p;
      if (!diag || c <= r) cij[r * W + c] -= acc[q][p];
    }
}

// Superblock inverses, step i (tile row i of every superblock): for each
// superblock m and tile column j <= i,
//   X(i, j) = L(i, i)^-1 (delta_ij I - sum_{k=j}^{i-1} L(i, k) X(k, j)),
// with L(i, k) the band tile (mB + i, i - k).  One CTA per (m, j).  After the
// last step, rows of null dofs are zeroed by k_cband_xnull.
__global__ void __launch_bounds__(kTileThreads) k_cband_xinv(const double* T, double* X, int B, int i) {
  const int m = blockIdx.x / (i + 1), j = blockIdx.x % (i + 1);
  const int Ig = m * B + i;
  extern __shared__ double cb_sm[];
  double(*R)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm);
  double(*L)[W + 1] = reinterpret_cast<double(*)[W + 1]>(cb_sm + W * (W + 1));
  const int tr = threadIdx.x / 16, tc = threadIdx.x % 16;
  double acc[4][4] = {};
  for (int k = j; k < i; ++k) {
    const double* lik = tile_ptr(T, B, Ig, i - k);
    const double* xkj = xtile(X, B, m, k, j);
    __syncthreads();
    for (int e = threadIdx.x; e < W * W; e += blockDim.x) {
      L[e / W][e % W] = lik[e];
      R[e / W][e % W] = xkj[e];
    }
    __syncthreads();
    for (int kk = 0; kk < W; ++kk) {
      double av[4], bv[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        av[q] = L[tr + 16 * q][kk];
        bv[q] = R[kk][tc + 16 * q];
      }
#pragma unroll
      for (int q = 0; q < 4; ++q)
#pragma unroll
        for (int p = 0; p < 4; ++p) acc[q][p] += av[q] * bv[p];
    }
  }
  __syncthreads();
  // R = delta_ij I - acc, then solve L(i, i) Y = R column by column
#pragma unroll
  for (int q = 0; q < 4; ++q)
#pragma unroll
    for (int p = 0; p < 4; ++p) {
      const int r = tr + 16 * q, c = tc + 16 * p;
      R[r][c] = (i == j && r == c ? 1.0 : 0.0) - acc[q][p];
    }
  const double* lii = tile_ptr(T, B, Ig, 0);
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) L[e / W][e % W] = lii[e];
  __syncthreads();
  if (threadIdx.x < W) {
    const int c = threadIdx.x;
    for (int r = 0; r < W; ++r) {
      double s = R[r][c];
      for (int r2 = 0; r2 < r; ++r2) s -= L[r][r2] * R[r2][c];
      R[r][c] = s / L[r][r];
    }
  }
  __syncthreads();
  double* xo = xtile(X, B, m, i, j);
  for (int e = threadIdx.x; e < W * W; e += blockDim.x) xo[e] = R[e / W][e % W];
}

__global__ void k_cband_xnull(double* X, int B, int NS, const int* nullf) {
  const long long rows = (long long)NS * B * W;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < rows;
       g += (long long)gridDim.x * blockDim.x) {
    if (!nullf[g]) continue;
    const int m = (int)(g / ((long long)B * W)), lr = (int)(g % ((long long)B * W));
    const int i = lr / W, r = lr % W;
    for (int j = 0; j <= i; ++j) {
      double* x = xtile(X, B, m, i, j) + r * W;
      for (int c = 0; c < W; ++c) x[c] = 0.0;
    }
  }
}

// ---- solve -------------------------------------------------------------------
// grid-order vector from the natural coarse vector (padding 0), and back
__global__ void k_cband_gather(const int* perm, long long n, const double* c, double* v, const int* done) {
  if (done && *done) return;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int p = perm[g];
    v[g] = p >= 0 ? c[p] : 0.0;
  }
}
__global__ void k_cband_scatter(const int* perm, long long n, const double* v, double* out, const int* done) {
  if (done && *done) return;
  for (long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x; g < n; g += (long long)gridDim.x * blockDim.x) {
    const int p = perm[g];
    if (p >= 0) out[p] = v[g];
  }
}

// forward, part 1: t_m = c_m - L_{m,m-1} y_{m-1} (one warp per row of superblock m)
__global__ void k_cband_fwd_off(const double* T, int B, int m, const double* c, const double* y, double* t,
                                const int* done) {
  if (done && *done) return;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= B * W) return;
  const long long g = (long long)m * B * W + row;
  double s = 0.0;
  if (m > 0) {
    const int I = m * B + row / W, r = row % W;
    // tiles (I, J) with J in superblock m-1 and I - J <= B
    for (int J = max((m - 1) * B, I - B); J < m * B; ++J) {
      const double* tl = tile_ptr(T, B, I, I - J) + r * W;
      const double* yy = y + (long long)J * W;
      for (int q = lane; q < W; q += 32) s += tl[q] * yy[q];
    }
  }
  s = warp_sum(s);
  if (lane == 0) t[g] = c[g] - s;
}
// forward, part 2: y_m = X_m t_m
__global__ void k_cband_fwd_diag(const double* X, int B, int m, const double* t, double* y, const int* done) {
  if (done && *done) return;
  const int row = (blockIdx.x * blockDim.x + threadIdx.x) >> 5, lane = threadIdx.x & 31;
  if (row >= B * W) return;
  const int i = row / W, r = row % W;
  const double* tt = t + (long long)m * B * W;
  double s = 0.0;
  for (int j = 0; j <= i; ++j) {
    const double* x = xtile(X, B, m, i, j) + r * W;
    for (int q = lane; q < W; q += 32) s += x[q] * tt[j * W + q];
  }
  s = warp_sum(s);
  if (lane == 0) y[(long long)m * B * W + row] = s;
}
// backward, part 1: t_m = y_m - L_{m+1,m}^T x_{m+1}.  One CTA per tile (I, J) of
// L_{m+1,m} (J in superblock m, I in m+1, inside the band): 64 columns x 4 groups
// of 16 rows, the tile's column sums into part[(I - (m+1)B) B + (J - mB)];
// k_cband_bwd_off_sum adds them per column in a fixed order.
__global__ void __launch_bounds__(256) k_cband_bwd_off_part(const double* T, int B, int m, int NS, const double* x,
                                                           double* part, const int* done) {
  if (done && *done) return;
  if (m + 1 >= NS) return;
  const int il = blockIdx.x / B, jl = blockIdx.x % B;
  const int I = (m + 1) * B + il, J = m * B + jl;
  const int c = threadIdx.x & (W - 1), rg = threadIdx.x >> 6;
  __shared__ double red[4][W];
  double s = 0.0;
  if (I - J <= B) {
    const double* tl = tile_ptr(T, B, I, I - J);
    const double* xx = x + (long long)I * W;
    for (int r = rg * 16; r < rg * 16 + 16; ++r) s += tl[r * W + c] * xx[r];
  }
  red[rg][c] = s;
  __syncthreads();
  if (rg == 0) part[((long long)il * B + jl) * W + c] = ((red[0][c] + red[1][c]) + red[2][c]) + red[3][c];
}
__global__ void k_cband_bwd_off_sum(int B, int m, int NS, const double* y, const double* part, double* t,
                                    const int* done) {
  if (done && *done) return;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;  // one thread per column of superblock m
  if (col >= B * W) return;
  const long long g = (long long)m * B * W + col;
  double s = 0.0;
  if (m + 1 < NS) {
    const int jl = col / W, c = col % W, J = m * B + jl;
    for (int il = 0; il < B; ++il)
      if ((m + 1) * B + il - J <= B) s += part[((long long)il * B + jl) * W + c];
  }
  t[g] = y[g] - s;
}
// backward, part 2: x_m = X_m^T t_m, the same way over the tiles (i, j >= ... i) of X_m
__global__ void __launch_bounds__(256) k_cband_bwd_diag_part(const double* X, int B, int m, const double* t,
                                                            double* part, const int* done) {
  if (done && *done) return;
  const int i = blockIdx.x / B, j = blockIdx.x % B;
  if (i < j) return;
  const int c = threadIdx.x & (W - 1), rg = threadIdx.x >> 6;
  __shared__ double red[4][W];
  const double* xt = xtile(X, B, m, i, j);
  const double* tt = t + (long long)m * B * W + (long long)i * W;
  double s = 0.0;
  for (int r = rg * 16; r < rg * 16 + 16; ++r) s += xt[r * W + c] * tt[r];
  red[rg][c] = s;
  __syncthreads();
  if (rg == 0) part[((long long)i * B + j) * W + c] = ((red[0][c] + red[1][c]) + red[2][c]) + red[3][c];
}
__global__ void k_cband_bwd_diag_sum(int B, int m, const double* part, double* x, const int* done) {
  if (done && *done) return;
  const int col = blockIdx.x * blockDim.x + threadIdx.x;
  if (col >= B * W) return;
  const int j = col / W, c = col % W;
  double s = 0.0;
  for (int i = j; i < B; ++i) s += part[((long long)i * B + j) * W + c];
  x[(long long)m * B * W + col] = s;
}

// ---------------------------------------------------------------------------
// host side
int cband_plan(const std::vector<SubInfo>& subs, const int grid[3], int kmax, CBandPlan* p) {
  // subdomain grid coordinates from the boxes
  const int nsub = (int)subs.size();
  std::vector<int> xs, ys, zs;
  for (const SubInfo& S : subs) {
    xs.push_back(S.x0);
    ys.push_back(S.y0);
    zs.push_back(S.z0);
  }
  auto uniq = [](std::vector<int>& v) {
    std::sort(v.begin(), v.end());
    v.erase(std::unique(v.begin(), v.end()), v.end());
  };
  uniq(xs);
  uniq(ys);
  uniq(zs);
  const int n[3] = {(int)xs.size(), (int)ys.size(), (int)zs.size()};
  if (n[0] != grid[0] || n[1] != grid[1] || n[2] != grid[2]) return 62;
  // axis order: the axis with the most subdomains slowest
  int ax[3] = {0, 1, 2};
  std::sort(ax, ax + 3, [&](int a, int b) { return n[a] < n[b] || (n[a] == n[b] && a < b); });
  p->nc = (long long)nsub * kmax;
  p->b = (long long)kmax * n[ax[0]] * n[ax[1]] + kmax - 1;
  p->B = (int)((p->b + W - 1) / W);
  const long long NT = (p->nc + W - 1) / W;
  p->NS = (int)((NT + p->B - 1) / p->B);
  p->NTp = (long long)p->NS * p->B;
  p->perm.assign((size_t)p->NTp * W, -1);
  for (int s = 0; s < nsub; ++s) {
    const SubInfo& S = subs[s];
    const int c[3] = {(int)(std::lower_bound(xs.begin(), xs.end(), S.x0) - xs.begin()),
                      (int)(std::lower_bound(ys.begin(), ys.end(), S.y0) - ys.begin()),
                      (int)(std::lower_bound(zs.begin(), zs.end(), S.z0) - zs.begin())};
    const long long gidx = ((long long)c[ax[2]] * n[ax[1]] + c[ax[1]]) * n[ax[0]] + c[ax[0]];
    for (int a = 0; a < kmax; ++a) p->perm[(size_t)(gidx * kmax + a)] = s * kmax + a;
  }
  p->tile_bytes = (size_t)W * W * sizeof(double);
  p->T_bytes = (size_t)p->NTp * (p->B + 1) * p->tile_bytes;
  p->X_bytes = (size_t)p->NS * p->B * p->B * p->tile_bytes;
  return 0;
}

void launch_cband_factor(const SubInfo* subs, int kmax, const double* blk, const int* d_perm, const CBandPlan& p,
                         double shift, double tol, double* T, double* X, int* nullf, int* nnull, double* scale,
                         cudaStream_t st) {
  const int B = p.B, NTp = (int)p.NTp;
  {
    const long long total = (long long)NTp * (B + 1) * W * W;
    const int nb = (int)std::min<long long>((total + 255) / 256, 148 * 64);
    note_launch();
    k_cband_assemble<<<nb, 256, 0, st>>>(subs, kmax, blk, d_perm, NTp, B, shift, T);
  }
  note_launch();
  k_cband_diag_max<<<1, 1024, 0, st>>>(T, NTp, B, scale);
  const int sm2 = 2 * W * (W + 1) * (int)sizeof(double);  // two padded tiles
  cudaFuncSetAttribute(k_cband_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2);
  cudaFuncSetAttribute(k_cband_syrk, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2);
  cudaFuncSetAttribute(k_cband_xinv, cudaFuncAttributeMaxDynamicSharedMemorySize, sm2);
  for (int K = 0; K < NTp; ++K) {
    note_launch();
    k_cband_potrf<<<1, kTileThreads, 0, st>>>(T, B, K, scale, tol, nullf, nnull);
    const int nI = std::min(B, NTp - 1 - K);
    if (nI <= 0) continue;
    note_launch();
    k_cband_trsm<<<nI, kTileThreads, sm2, st>>>(T, B, K, NTp, nullf);
    note_launch();
    k_cband_syrk<<<B * (B + 1) / 2, kTileThreads, sm2, st>>>(T, B, K, NTp);
  }
  for (int i = 0; i < B; ++i) {
    note_launch();
    k_cband_xinv<<<p.NS * (i + 1), kTileThreads, sm2, st>>>(T, X, B, i);
  }
  note_launch();
  k_cband_xnull<<<256, 256, 0, st>>>(X, B, p.NS, nullf);
}

void launch_cband_solve(const int* d_perm, const CBandPlan& p, const double* T, const double* X, const double* c,
                        double* out, double* v, double* y, double* t, double* part, const int* done,
                        cudaStream_t st) {
  const int B = p.B, NS = p.NS;
  const long long n = p.NTp * W;
  const int rows = B * W;
  { note_launch(); k_cband_gather<<<256, 256, 0, st>>>(d_perm, n, c, v, done); }
  for (int m = 0; m < NS; ++m) {
    { note_launch(); k_cband_fwd_off<<<(rows * 32 + 255) / 256, 256, 0, st>>>(T, B, m, v, y, t, done); }
    { note_launch(); k_cband_fwd_diag<<<(rows * 32 + 255) / 256, 256, 0, st>>>(X, B, m, t, y, done); }
  }
  // backward into v (the gathered right-hand side is no longer needed)
  for (int m = NS - 1; m >= 0; --m) {
    if (m + 1 < NS) { note_launch(); k_cband_bwd_off_part<<<B * B, 256, 0, st>>>(T, B, m, NS, v, part, done); }
    { note_launch(); k_cband_bwd_off_sum<<<(rows + 127) / 128, 128, 0, st>>>(B, m, NS, y, part, t, done); }
    { note_launch(); k_cband_bwd_diag_part<<<B * B, 256, 0, st>>>(X, B, m, t, part, done); }
    { note_launch(); k_cband_bwd_diag_sum<<<(rows + 127) / 128, 128, 0, st>>>(B, m, part, v, done); }
  }
  { note_launch(); k_cband_scatter<<<256, 256, 0, st>>>(d_perm, n, v, out, done); }
}

}  // namespace pmf
