// Coarse-space kernels (FP64): level-2 Galerkin assembly, batched dense SPD
// inverses, the level-3 eigenproblem and the small coarse products used by the
// cycle executor.
#include <cooperative_groups.h>

#include <algorithm>
#include <cstdio>

#include "pmf_dense.cuh"
#include "pmf_kernels.h"
#include "tune.h"

namespace pmf {

// ---------------------------------------------------------------------------
// out = base - A2 v with A2 = Phi^T A Phi stored as 7 kmax x kmax blocks per
// subdomain row (diagonal + six face neighbours).
__global__ void k_a2_mult(const SubInfo* subs, int nsub, int kmax, const double* blk, const double* v,
                          const double* base, double* out, const int* done) {
  if (done && *done) return;
  const long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (row >= (long long)nsub * kmax) return;
  const int s = (int)(row / kmax), i = (int)(row % kmax);
  const SubInfo& S = subs[s];
  double acc = 0.0;
  for (int b = 0; b < 7; ++b) {
    const int nb = b == 0 ? s : S.nb[b - 1];
    if (nb < 0) continue;
    const double* B = blk + (((long long)s * 7 + b) * kmax + i) * kmax;
    const double* vv = v + (long long)nb * kmax;
    for (int j = 0; j < kmax; ++j) acc += B[j] * vv[j];
  }
  out[row] = (base ? base[row] : 0.0) - acc;
}
void launch_a2_mult(const SubInfo* subs, int nsub, int kmax, const double* blk, const double* v, const double* base,
                    double* out, const int* done, cudaStream_t st) {
  long long n = (long long)nsub * kmax;
  { note_launch(); k_a2_mult<<<(int)((n + 255) / 256), 256, 0, st>>>(subs, nsub, kmax, blk, v, base, out, done); }
}

// Batched dense GEMV, one warp per row.
__global__ void k_block_gemv(int nrank, int nr, const double* inv, const double* in, double* out, int accumulate,
                             const int* done) {
  if (done && *done) return;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= (long long)nrank * nr) return;
  const long long r = row / nr;
  const double* A = inv + row * nr;
  const double* x = in + r * nr;
  double acc = 0.0;
  for (int j = lane; j < nr; j += 32) acc += A[j] * x[j];
  acc = warp_sum(acc);
  if (lane == 0) out[row] = accumulate ? out[row] + acc : acc;
}
void launch_block_gemv(int nrank, int nr, const double* inv, const double* in, double* out, int accumulate,
                       const int* done, cudaStream_t st) {
  long long threads = (long long)nrank * nr * 32;
  { note_launch(); k_block_gemv<<<(int)((threads + 255) / 256), 256, 0, st>>>(nrank, nr, inv, in, out, accumulate, done); }
}

// d[r][j] = sum_i V[r][i][j] c[r][i]  (Psi^T r = V^T Phi^T r, per rank)
__global__ void k_lv3_restrict(int nrank, int nr, int en2, const double* V, const double* c, double* d,
                               const int* done) {
  if (done && *done) return;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= (long long)nrank * en2) return;
  const long long r = row / en2;
  const int j = (int)(row % en2);
  const double* Vr = V + r * nr * en2;
  const double* cr = c + r * nr;
  double acc = 0.0;
  for (int i = lane; i < nr; i += 32) acc += Vr[(long long)i * en2 + j] * cr[i];
  acc = warp_sum(acc);
  if (lane == 0) d[row] = acc;
}
void launch_lv3_restrict(int nrank, int nr, int en2, const double* V, const double* c, double* d, const int* done,
                         cudaStream_t st) {
  long long threads = (long long)nrank * en2 * 32;
  { note_launch(); k_lv3_restrict<<<(int)((threads + 255) / 256), 256, 0, st>>>(nrank, nr, en2, V, c, d, done); }
}

// dz[r][i] = sum_j V[r][i][j] w[r][j]
__global__ void k_lv3_prolong(int nrank, int nr, int en2, const double* V, const double* w, double* dz,
                              const int* done) {
  if (done && *done) return;
  const long long row = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (row >= (long long)nrank * nr) return;
  const long long r = row / nr;
  const double* Vi = V + row * en2;
  const double* wr = w + r * en2;
  double acc = 0.0;
  for (int j = 0; j < en2; ++j) acc += Vi[j] * wr[j];
  dz[row] = acc;
}
void launch_lv3_prolong(int nrank, int nr, int en2, const double* V, const double* w, double* dz, const int* done,
                        cudaStream_t st) {
  long long n = (long long)nrank * nr;
  { note_launch(); k_lv3_prolong<<<(int)((n + 255) / 256), 256, 0, st>>>(nrank, nr, en2, V, w, dz, done); }
}

// ---- the same products over ranks of different sizes (RankLayout) ----------
__device__ __forceinline__ int rank_nr(const RankLayout& L, int r) { return (L.first[r + 1] - L.first[r]) * L.kmax; }
__device__ __forceinline__ long long rank_dof0(const RankLayout& L, int r) { return (long long)L.first[r] * L.kmax; }
// the rank whose range [off[r], off[r+1]) holds e (binary search)
__device__ __forceinline__ int rank_of(const long long* off, int nrank, long long e) {
  int lo = 0, hi = nrank - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (off[mid] <= e)
      lo = mid;
    else
      hi = mid - 1;
  }
  return lo;
}

// out[g] = sum_j inv_r[i][j] in[dof0_r + j] for coarse dof g = dof0_r + i, one warp per dof
__global__ void k_block_gemv_r(RankLayout L, long long ncoarse, const double* inv, const double* in, double* out,
                               const int* done) {
  if (done && *done) return;
  const long long g = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (g >= ncoarse) return;
  const int r = L.dof_rank[g];
  const int nr = rank_nr(L, r);
  const long long d0 = rank_dof0(L, r);
  const double* A = inv + L.off2[r] + (g - d0) * nr;
  const double* x = in + d0;
  double acc = 0.0;
  for (int j = lane; j < nr; j += 32) acc += A[j] * x[j];
  acc = warp_sum(acc);
  if (lane == 0) out[g] = acc;
}
void launch_block_gemv_r(const RankLayout& L, long long ncoarse, const double* inv, const double* in, double* out,
                         const int* done, cudaStream_t st) {
  const long long threads = ncoarse * 32;
  { note_launch(); k_block_gemv_r<<<(int)((threads + 255) / 256), 256, 0, st>>>(L, ncoarse, inv, in, out, done); }
}
__global__ void k_lv3_restrict_r(RankLayout L, int nrank, int en2, const double* V, const double* c, double* d,
                                 const int* done) {
  if (done && *done) return;
  const long long row = (blockIdx.x * (long long)blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (row >= (long long)nrank * en2) return;
  const int r = (int)(row / en2), j = (int)(row % en2);
  const int nr = rank_nr(L, r);
  const double* Vr = V + L.offv[r];
  const double* cr = c + rank_dof0(L, r);
  double acc = 0.0;
  for (int i = lane; i < nr; i += 32) acc += Vr[(long long)i * en2 + j] * cr[i];
  acc = warp_sum(acc);
  if (lane == 0) d[row] = acc;
}
void launch_lv3_restrict_r(const RankLayout& L, int nrank, int en2, const double* V, const double* c, double* d,
                           const int* done, cudaStream_t st) {
  const long long threads = (long long)nrank * en2 * 32;
  { note_launch(); k_lv3_restrict_r<<<(int)((threads + 255) / 256), 256, 0, st>>>(L, nrank, en2, V, c, d, done); }
}
__global__ void k_lv3_prolong_r(RankLayout L, long long ncoarse, int en2, const double* V, const double* w, double* dz,
                                const int* done) {
  if (done && *done) return;
  const long long g = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (g >= ncoarse) return;
  const int r = L.dof_rank[g];
  const double* Vi = V + L.offv[r] + (g - rank_dof0(L, r)) * en2;
  const double* wr = w + (long long)r * en2;
  double acc = 0.0;
  for (int j = 0; j < en2; ++j) acc += Vi[j] * wr[j];
  dz[g] = acc;
}
void launch_lv3_prolong_r(const RankLayout& L, long long ncoarse, int en2, const double* V, const double* w,
                          double* dz, const int* done, cudaStream_t st) {
  { note_launch(); k_lv3_prolong_r<<<(int)((ncoarse + 255) / 256), 256, 0, st>>>(L, ncoarse, en2, V, w, dz, done); }
}

__global__ void k_axpy(long long n, double a, const double* x, double* y, const int* done) {
  if (done && *done) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] += a * x[i];
}
__global__ void k_copy(long long n, const double* x, double* y, const int* done) {
  if (done && *done) return;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    y[i] = x[i];
}
void launch_axpy(long long n, double a, const double* x, double* y, const int* done, cudaStream_t st) {
  { note_launch(); k_axpy<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(n, a, x, y, done); }
}
void launch_copy(long long n, const double* x, double* y, const int* done, cudaStream_t st) {
  { note_launch(); k_copy<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(n, x, y, done); }
}

// ---------------------------------------------------------------------------
// Galerkin blocks of Phi^T A Phi (_PC_setup_lv2_J, src/PreMixFEM_3D.c:756-890).
// Warp i of the CTA for subdomain s computes row i of:
//   blk[s][0]   = Phi_s^T A_s Phi_s, A_s the principal submatrix of A on s
//                 (interior faces in difference form, globally interior
//                 boundary faces and Dirichlet terms on the diagonal);
//   blk[s][1+f] = -sum_{face f} t phi_s,i(c) phi_nb,j(c')  (neighbour coupling);
//   gface[s][f] =  sum_{face f} t phi_s,i(c) phi_s,j(c)    (boundary-face part of
//                 the diagonal block, removed again for rank-Neumann matrices).
template <typename T, int KM>
__global__ void k_galerkin(Grid g, const SubInfo* subs, int kmax, const double* tx, const double* ty,
                           const double* tz, const double* diag, const T* phi, double* blk, double* gface) {
  const int s = blockIdx.x;
  const SubInfo S = subs[s];
  const int wid = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (wid >= kmax) return;
  const int i = wid;
  const int nx = S.nx, ny = S.ny, nz = S.nz, ncells = nx * ny * nz;
  double acc[KM];
#pragma unroll
  for (int j = 0; j < KM; ++j) acc[j] = 0.0;
  for (int cl = lane; cl < ncells; cl += 32) {
    const int ii = cl % nx, tt = cl / nx, jj = tt % ny, kk = tt / ny;
    const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + ii);
    const double pi = (double)phi[cg * kmax + i];
    if (pi == 0.0) continue;
    const double dg = diag[cg];
    const double t_xm = ii > 0 ? tx[cg] : 0.0, t_xp = ii < nx - 1 ? tx[cg + 1] : 0.0;
    const double t_ym = jj > 0 ? ty[cg] : 0.0, t_yp = jj < ny - 1 ? ty[cg + g.M] : 0.0;
    const double t_zm = kk > 0 ? tz[cg] : 0.0, t_zp = kk < nz - 1 ? tz[cg + g.MN] : 0.0;
#pragma unroll
    for (int j = 0; j < KM; ++j) {
      if (j >= kmax) break;
      double a = dg * (double)phi[cg * kmax + j];
      if (ii > 0) a -= t_xm * (double)phi[(cg - 1) * kmax + j];
      if (ii < nx - 1) a -= t_xp * (double)phi[(cg + 1) * kmax + j];
      if (jj > 0) a -= t_ym * (double)phi[(cg - g.M) * kmax + j];
      if (jj < ny - 1) a -= t_yp * (double)phi[(cg + g.M) * kmax + j];
      if (kk > 0) a -= t_zm * (double)phi[(cg - g.MN) * kmax + j];
      if (kk < nz - 1) a -= t_zp * (double)phi[(cg + g.MN) * kmax + j];
      acc[j] += pi * a;
    }
  }
#pragma unroll
  for (int j = 0; j < KM; ++j) {
    if (j >= kmax) break;
    const double v = warp_sum(acc[j]);
    if (lane == 0) blk[(((long long)s * 7 + 0) * kmax + i) * kmax + j] = v;
  }
  // faces x-, x+, y-, y+, z-, z+
  for (int f = 0; f < 6; ++f) {
    const int axis = f >> 1, hi = f & 1;
    bool exists;
    int na, nb;  // face extents
    if (axis == 0) {
      exists = hi ? (S.x0 + nx < g.M) : (S.x0 > 0);
      na = ny;
      nb = nz;
    } else if (axis == 1) {
      exists = hi ? (S.y0 + ny < g.N) : (S.y0 > 0);
      na = nx;
      nb = nz;
    } else {
      exists = hi ? (S.z0 + nz < g.P) : (S.z0 > 0);
      na = nx;
      nb = ny;
    }
    double ag[KM], ac[KM];
#pragma unroll
    for (int j = 0; j < KM; ++j) ag[j] = ac[j] = 0.0;
    if (exists) {
      for (int idx = lane; idx < na * nb; idx += 32) {
        const int a = idx % na, b = idx / na;
        int ii, jj, kk;
        if (axis == 0) {
          ii = hi ? nx - 1 : 0;
          jj = a;
          kk = b;
        } else if (axis == 1) {
          ii = a;
          jj = hi ? ny - 1 : 0;
          kk = b;
        } else {
          ii = a;
          jj = b;
          kk = hi ? nz - 1 : 0;
        }
        const long long cg = ((long long)(S.z0 + kk) * g.N + (S.y0 + jj)) * g.M + (S.x0 + ii);
        const long long off = axis == 0 ? 1 : (axis == 1 ? g.M : g.MN);
        const long long cn = hi ? cg + off : cg - off;
        const double* tt = axis == 0 ? tx : (axis == 1 ? ty : tz);
        const double t = hi ? tt[cn] : tt[cg];
        const double pi = (double)phi[cg * kmax + i];
#pragma unroll
        for (int j = 0; j < KM; ++j) {
          if (j >= kmax) break;
          ag[j] += t * pi * (double)phi[cg * kmax + j];
          ac[j] -= t * pi * (double)phi[cn * kmax + j];
        }
      }
    }
#pragma unroll
    for (int j = 0; j < KM; ++j) {
      if (j >= kmax) break;
      const double vg = warp_sum(ag[j]);
      const double vc = warp_sum(ac[j]);
      if (lane == 0) {
        gface[(((long long)s * 6 + f) * kmax + i) * kmax + j] = vg;
        blk[(((long long)s * 7 + 1 + f) * kmax + i) * kmax + j] = vc;
      }
    }
  }
}

template <typename T>
void launch_galerkin(const Grid& g, const SubInfo* subs, int nsub, int kmax, const double* tx, const double* ty,
                     const double* tz, const double* diag, const T* phi, double* blk, double* gface,
                     cudaStream_t st) {
  const int threads = 32 * kmax;
  if (kmax <= 4)
    { note_launch(); k_galerkin<T, 4><<<nsub, threads, 0, st>>>(g, subs, kmax, tx, ty, tz, diag, phi, blk, gface); }
  else if (kmax <= 8)
    { note_launch(); k_galerkin<T, 8><<<nsub, threads, 0, st>>>(g, subs, kmax, tx, ty, tz, diag, phi, blk, gface); }
  else
    { note_launch(); k_galerkin<T, 16><<<nsub, threads, 0, st>>>(g, subs, kmax, tx, ty, tz, diag, phi, blk, gface); }
}
template void launch_galerkin<float>(const Grid&, const SubInfo*, int, int, const double*, const double*,
                                     const double*, const double*, const float*, double*, double*, cudaStream_t);
template void launch_galerkin<double>(const Grid&, const SubInfo*, int, int, const double*, const double*,
                                      const double*, const double*, const double*, double*, double*, cudaStream_t);

// Dense per-rank coarse matrices.  mode 0: the rank's principal block of
// Phi^T A Phi (level-2 matrix of _PC_setup_lv2_J); mode 1: the rank-Neumann
// matrix of _PC_setup_lv3_eigen (:938-1076), i.e. without the boundary-face
// terms of faces that leave the rank.  Padded dofs (j >= k_s) are identity.
__global__ void k_assemble_dense(const SubInfo* subs, int nrank, int spr, int kmax, const double* blk,
                                 const double* gface, int mode, double* dense) {
  const long long nr = (long long)spr * kmax;
  const long long total = (long long)nrank * nr * nr;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = (int)(e / (nr * nr));
    const long long rem = e % (nr * nr);
    const int row = (int)(rem / nr), col = (int)(rem % nr);
    const int a = row / kmax, i = row % kmax, b = col / kmax, j = col % kmax;
    const int s = r * spr + a, s2 = r * spr + b;
    const SubInfo& S = subs[s];
    double v = 0.0;
    if (i >= S.k || j >= subs[s2].k) {
      v = (row == col) ? 1.0 : 0.0;
    } else if (a == b) {
      v = blk[(((long long)s * 7) * kmax + i) * kmax + j];
      if (mode == 1)
        for (int f = 0; f < 6; ++f)
          if (S.nb[f] >= 0 && subs[S.nb[f]].rank != r) v -= gface[(((long long)s * 6 + f) * kmax + i) * kmax + j];
    } else {
      for (int f = 0; f < 6; ++f)
        if (S.nb[f] == s2) v = blk[(((long long)s * 7 + 1 + f) * kmax + i) * kmax + j];
    }
    dense[e] = v;
  }
}
__global__ void k_assemble_dense_r(const SubInfo* subs, int nrank, RankLayout L, long long total, const double* blk,
                                   const double* gface, int mode, double* dense) {
  const int kmax = L.kmax;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < total;
       e += (long long)gridDim.x * blockDim.x) {
    const int r = rank_of(L.off2, nrank, e);
    const long long nr = rank_nr(L, r);
    const long long rem = e - L.off2[r];
    const int row = (int)(rem / nr), col = (int)(rem % nr);
    const int a = row / kmax, i = row % kmax, b = col / kmax, j = col % kmax;
    const int s = L.first[r] + a, s2 = L.first[r] + b;
    const SubInfo& S = subs[s];
    double v = 0.0;
    if (i >= S.k || j >= subs[s2].k) {
      v = (row == col) ? 1.0 : 0.0;
    } else if (a == b) {
      v = blk[(((long long)s * 7) * kmax + i) * kmax + j];
      if (mode == 1)
        for (int f = 0; f < 6; ++f)
          if (S.nb[f] >= 0 && subs[S.nb[f]].rank != r) v -= gface[(((long long)s * 6 + f) * kmax + i) * kmax + j];
    } else {
      for (int f = 0; f < 6; ++f)
        if (S.nb[f] == s2) v = blk[(((long long)s * 7 + 1 + f) * kmax + i) * kmax + j];
    }
    dense[e] = v;
  }
}
void launch_assemble_dense_r(const SubInfo* subs, int nrank, const RankLayout& L, long long total, const double* blk,
                             const double* gface, int mode, double* dense, cudaStream_t st) {
  const int nb = (int)std::min<long long>((total + 255) / 256, 148 * 32);
  { note_launch(); k_assemble_dense_r<<<nb, 256, 0, st>>>(subs, nrank, L, total, blk, gface, mode, dense); }
}
__global__ void k_add_diag_r(RankLayout L, double* dense, double mu, int relative) {
  const int r = blockIdx.x;
  const int n = rank_nr(L, r);
  double* A = dense + L.off2[r];
  __shared__ double mx;
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, fabs(A[(long long)i * n + i]));
    mx = relative ? m * mu : mu;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) A[(long long)i * n + i] += mx;
}
void launch_add_diag_r(const RankLayout& L, int nrank, double* dense, double mu, int relative, cudaStream_t st) {
  { note_launch(); k_add_diag_r<<<nrank, 256, 0, st>>>(L, dense, mu, relative); }
}

void launch_assemble_dense(const SubInfo* subs, int nsub, int nrank, int spr, int kmax, const double* blk,
                           const double* gface, int mode, double* dense, cudaStream_t st) {
  (void)nsub;
  long long total = (long long)nrank * spr * kmax * spr * kmax;
  int nb = (int)std::min<long long>((total + 255) / 256, 148 * 32);
  { note_launch(); k_assemble_dense<<<nb, 256, 0, st>>>(subs, nrank, spr, kmax, blk, gface, mode, dense); }
}

// In-place Gauss-Jordan inverse of SPD matrices (one CTA per matrix).
// Pivots <= tol * max diag are null directions: that row/column is dropped
// (zero in the result), which equals inverting the matrix with the index
// removed -- the same treatment as the semidefinite Cholesky of the oracle.
__global__ void k_spd_inverse(int n, double* a_all, double tol, int* nnull) {
  double* a = a_all + (long long)blockIdx.x * n * n;
  extern __shared__ double sh[];
  double* colk = sh;
  double* rowk = sh + n;
  __shared__ double red[32];
  __shared__ int nul;
  double mx = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) mx = fmax(mx, fabs(a[(long long)i * n + i]));
  // block max via shared reduction
  {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
    if (lane == 0) red[wid] = mx;
    __syncthreads();
    if (threadIdx.x == 0) {
      double m = 0.0;
      for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) m = fmax(m, red[w]);
      red[0] = m;
      nul = 0;
    }
    __syncthreads();
  }
  const double scale = red[0] > 0 ? red[0] : 1.0;
  for (int k = 0; k < n; ++k) {
    const double piv = a[(long long)k * n + k];
    const bool isnull = !(piv > tol * scale);
    for (int i = threadIdx.x; i < n; i += blockDim.x) {
      colk[i] = a[(long long)i * n + k];
      rowk[i] = isnull ? 0.0 : (i == k ? 1.0 : a[(long long)k * n + i]) / piv;
    }
    __syncthreads();
    if (isnull) {
      for (int i = threadIdx.x; i < n; i += blockDim.x) {
        a[(long long)k * n + i] = 0.0;
        a[(long long)i * n + k] = 0.0;
      }
      if (threadIdx.x == 0) nul += 1;
    } else {
      // rank-1 update, one warp per row (no index division in the inner loop)
      const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
      for (int i = threadIdx.x >> 5; i < n; i += nw) {
        double* row = a + (long long)i * n;
        if (i == k) {
          for (int j = lane; j < n; j += 32) row[j] = rowk[j];
        } else {
          const double ci = colk[i];
          for (int j = lane; j < n; j += 32) row[j] = (j == k ? 0.0 : row[j]) - ci * rowk[j];
        }
      }
    }
    __syncthreads();
  }
  {
    const int lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    for (int i = threadIdx.x >> 5; i < n; i += nw)
      for (int j = i + 1 + lane; j < n; j += 32) {
        const double v = 0.5 * (a[(long long)i * n + j] + a[(long long)j * n + i]);
        a[(long long)i * n + j] = v;
        a[(long long)j * n + i] = v;
      }
  }
  if (threadIdx.x == 0 && nnull) atomicAdd(nnull, nul);
}
// The same Gauss-Jordan inverse by a cluster of kSpdCl CTAs per matrix, for
// n <= 32 * NM.  CTA c of the cluster owns rows [c R, c R + R), R = ceil(n /
// kSpdCl); warp w holds rows c R + w + 16 s (s < RW) in registers, lane l the
// columns l + 32 m.  Per pivot the owning warp publishes the scaled pivot row
// in its CTA's shared memory, one cluster barrier makes it visible, and every
// CTA copies it through distributed shared memory and updates its rows.  The
// arithmetic per element is that of k_spd_inverse, so the results agree bit
// for bit.
constexpr int kSpdCl = 8;
constexpr int kSpdWarps = 16;

template <int NM, int RW>
__global__ void __launch_bounds__(kSpdWarps * 32, 1)
    k_spd_inverse_cl(int n, double* a_all, double tol, int* nnull) {
  namespace cg = cooperative_groups;
  cg::cluster_group cluster = cg::this_cluster();
  const int crank = (int)cluster.block_rank();
  const int mat = blockIdx.x / kSpdCl;
  double* a = a_all + (long long)mat * n * n;
  const int R = (n + kSpdCl - 1) / kSpdCl;
  const int r0 = crank * R;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  __shared__ double pub[2][NM * 32];  // published pivot rows (read by the whole cluster)
  __shared__ double prow[NM * 32];    // local copy of the current pivot row
  __shared__ int pnull[2];
  __shared__ double cmax[kSpdWarps];
  __shared__ double smax;
  double v[RW][NM];
  int rows[RW];
#pragma unroll
  for (int s = 0; s < RW; ++s) {
    const int i = r0 + w + kSpdWarps * s;
    rows[s] = (w + kSpdWarps * s < R && i < n) ? i : -1;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      const int j = lane + 32 * m;
      v[s][m] = (rows[s] >= 0 && j < n) ? a[(long long)i * n + j] : 0.0;
    }
  }
  // scale = max |a_ii| over the whole matrix
  double mx = 0.0;
#pragma unroll
  for (int s = 0; s < RW; ++s)
#pragma unroll
    for (int m = 0; m < NM; ++m)
      if (rows[s] >= 0 && lane + 32 * m == rows[s]) mx = fmax(mx, fabs(v[s][m]));
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) cmax[w] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m2 = 0.0;
    for (int q = 0; q < kSpdWarps; ++q) m2 = fmax(m2, cmax[q]);
    smax = m2;
  }
  cluster.sync();
  if (threadIdx.x == 0) {
    double m2 = 0.0;
    for (int c = 0; c < kSpdCl; ++c) m2 = fmax(m2, *cluster.map_shared_rank(&smax, c));
    cmax[0] = m2 > 0 ? m2 : 1.0;
  }
  cluster.sync();  // every CTA has read the others' maxima before smax is reused
  const double scale = cmax[0];
  int nul = 0;
  for (int k = 0; k < n; ++k) {
    const int o = k / R, ok = k - o * R;
    const int ow = ok % kSpdWarps, os = ok / kSpdWarps;
    const int km = k >> 5, kl = k & 31;
    if (crank == o && w == ow) {  // owner warp: publish row k scaled by its pivot
#pragma unroll
      for (int s = 0; s < RW; ++s)
        if (s == os) {
          double pv = 0.0;
#pragma unroll
          for (int m = 0; m < NM; ++m)
            if (m == km) pv = v[s][m];
          const double piv = __shfl_sync(0xffffffffu, pv, kl);
          const bool isnull = !(piv > tol * scale);
#pragma unroll
          for (int m = 0; m < NM; ++m) {
            const int j = lane + 32 * m;
            pub[k & 1][j] = isnull ? 0.0 : (j == k ? 1.0 : v[s][m]) / piv;
          }
          if (lane == 0) pnull[k & 1] = isnull ? 1 : 0;
        }
    }
    cluster.sync();
    {
      const double* src = cluster.map_shared_rank(&pub[k & 1][0], o);
      for (int j = threadIdx.x; j < NM * 32; j += blockDim.x) prow[j] = src[j];
    }
    const bool isnull = *cluster.map_shared_rank(&pnull[k & 1], o) != 0;
    __syncthreads();
    if (isnull) {
      if (crank == o && threadIdx.x == 0) ++nul;
#pragma unroll
      for (int s = 0; s < RW; ++s) {
        if (rows[s] < 0) continue;
#pragma unroll
        for (int m = 0; m < NM; ++m)
          if (rows[s] == k || (m == km && lane == kl)) v[s][m] = 0.0;
      }
    } else {
#pragma unroll
      for (int s = 0; s < RW; ++s) {
        if (rows[s] < 0) continue;
        if (rows[s] == k) {
#pragma unroll
          for (int m = 0; m < NM; ++m) v[s][m] = prow[lane + 32 * m];
        } else {
          double cv = 0.0;
#pragma unroll
          for (int m = 0; m < NM; ++m)
            if (m == km) cv = v[s][m];
          const double ci = __shfl_sync(0xffffffffu, cv, kl);
#pragma unroll
          for (int m = 0; m < NM; ++m) {
            const int j = lane + 32 * m;
            v[s][m] = (j == k ? 0.0 : v[s][m]) - ci * prow[j];
          }
        }
      }
    }
  }
  // rows back to global memory, then the symmetrisation of k_spd_inverse by the
  // owner of the lower row index of each pair
#pragma unroll
  for (int s = 0; s < RW; ++s)
    if (rows[s] >= 0)
#pragma unroll
      for (int m = 0; m < NM; ++m) {
        const int j = lane + 32 * m;
        if (j < n) a[(long long)rows[s] * n + j] = v[s][m];
      }
  cluster.sync();
#pragma unroll
  for (int s = 0; s < RW; ++s) {
    const int i = rows[s];
    if (i < 0) continue;
#pragma unroll
    for (int m = 0; m < NM; ++m) {
      const int j = lane + 32 * m;
      if (j > i && j < n) {
        const double sv = 0.5 * (v[s][m] + a[(long long)j * n + i]);
        a[(long long)i * n + j] = sv;
        a[(long long)j * n + i] = sv;
      }
    }
  }
  if (threadIdx.x == 0 && nnull && nul) atomicAdd(nnull, nul);
}

template <int NM, int RW>
static bool spd_inverse_cl(int nb, int n, double* a, double tol, int* nnull, cudaStream_t st) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3(nb * kSpdCl);
  cfg.blockDim = dim3(kSpdWarps * 32);
  cfg.dynamicSmemBytes = 0;
  cfg.stream = st;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeClusterDimension;
  attr[0].val.clusterDim.x = kSpdCl;
  attr[0].val.clusterDim.y = 1;
  attr[0].val.clusterDim.z = 1;
  cfg.attrs = attr;
  cfg.numAttrs = 1;
  if (cudaLaunchKernelEx(&cfg, k_spd_inverse_cl<NM, RW>, n, a, tol, nnull) != cudaSuccess) {
    (void)cudaGetLastError();  // cluster launch refused: the caller falls back to one CTA per matrix
    return false;
  }
  note_launch();
  return true;
}

// The same Gauss-Jordan inverse spread over the whole GPU, for matrices too
// large for one cluster, in panels of kGjPB pivots.  Eliminating the pivots P
// of a panel turns [A_PP A_PR; A_RP A_RR] into
//   A_PP <- Z = A_PP^-1,  A_PR <- Z A_PR,  A_RP <- -A_RP Z,  A_RR <- A_RR - A_RP Z A_PR,
// which is what the pivots one at a time give in exact arithmetic; Z comes
// from the pivot-by-pivot Gauss-Jordan of the diagonal block with
// k_spd_inverse's arithmetic and null-pivot rule (a pivot at or below
// tol x max|diag| drops its row and column), so a null pivot zeroes its row
// and column of the result as before.  Per panel: k_gjb_diag (one CTA per
// matrix), k_gjb_rows (R = Z A_PR), k_gjb_update (the rank-kGjPB update of
// every element outside the panel: 64 x 64 tiles, 2 n^2 kGjPB flops per
// panel), k_gjb_cols (A_RP) and k_gjb_prow (A_PR, A_PP).  Matrix b has order
// nv[b] (or n) and starts at off[b] (or b n^2); panels past a matrix's order
// leave it alone.
struct GjShape {
  const int* nv;         // per matrix order, or null (all n)
  const long long* off;  // per matrix offset, or null (b n^2)
  int n;
  __device__ int ord(int b) const { return nv ? nv[b] : n; }
  __device__ long long at(int b) const { return off ? off[b] : (long long)b * n * n; }
};
constexpr int kGjPB = 64;  // pivots per panel
constexpr int kGjT = 64;   // tile edge of the update
constexpr int kGjLd = kGjPB + 1;

__global__ void k_gj_scale(GjShape sh, const double* a_all, double* scale) {
  const int nb = sh.ord(blockIdx.x);
  const double* a = a_all + sh.at(blockIdx.x);
  __shared__ double red[32];
  double mx = 0.0;
  for (int i = threadIdx.x; i < nb; i += blockDim.x) mx = fmax(mx, fabs(a[(long long)i * nb + i]));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) mx = fmax(mx, __shfl_xor_sync(0xffffffffu, mx, o));
  if (lane == 0) red[wid] = mx;
  __syncthreads();
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int w = 0; w < (int)((blockDim.x + 31) >> 5); ++w) m = fmax(m, red[w]);
    scale[blockIdx.x] = m > 0 ? m : 1.0;
  }
}

// Z = inverse of the panel's diagonal block, pivot by pivot in shared memory.
__global__ void __launch_bounds__(256) k_gjb_diag(GjShape sh, const double* a_all, int k0, double tol,
                                                  const double* scale, double* zbuf, int* nnull) {
  const int b = blockIdx.x;
  const int n = sh.ord(b);
  if (k0 >= n) return;
  const int pb = min(kGjPB, n - k0);
  const double* a = a_all + sh.at(b);
  __shared__ double z[kGjPB][kGjLd];
  __shared__ double colk[kGjPB], rowk[kGjPB];
  const int tid = threadIdx.x, bd = blockDim.x;
  for (int e = tid; e < pb * pb; e += bd) {
    const int i = e / pb, j = e % pb;
    z[i][j] = a[(long long)(k0 + i) * n + k0 + j];
  }
  __syncthreads();
  const double thr = tol * scale[b];
  int nul = 0;
  for (int kk = 0; kk < pb; ++kk) {
    const double piv = z[kk][kk];
    const bool isnull = !(piv > thr);
    for (int i = tid; i < pb; i += bd) {
      colk[i] = z[i][kk];
      rowk[i] = isnull ? 0.0 : (i == kk ? 1.0 : z[kk][i]) / piv;
    }
    __syncthreads();
    for (int e = tid; e < pb * pb; e += bd) {
      const int i = e / pb, j = e % pb;
      if (isnull) {
        if (i == kk || j == kk) z[i][j] = 0.0;
      } else if (i == kk) {
        z[i][j] = rowk[j];
      } else {
        z[i][j] = (j == kk ? 0.0 : z[i][j]) - colk[i] * rowk[j];
      }
    }
    __syncthreads();
    nul += isnull ? 1 : 0;
  }
  double* zb = zbuf + (long long)b * kGjPB * kGjPB;
  for (int e = tid; e < pb * pb; e += bd) zb[(e / pb) * kGjPB + e % pb] = z[e / pb][e % pb];
  if (tid == 0 && nnull && nul) atomicAdd(nnull, nul);
}

// R[c][j] = sum_c' Z[c][c'] A[k0 + c'][j] for the columns j outside the panel; 64 columns per CTA.
__global__ void __launch_bounds__(256) k_gjb_rows(GjShape sh, const double* a_all, int k0, const double* zbuf,
                                                  double* rbuf) {
  const int b = blockIdx.y;
  const int n = sh.ord(b);
  const int j0 = blockIdx.x * kGjT;
  if (k0 >= n || j0 >= n) return;
  const int pb = min(kGjPB, n - k0);
  const double* a = a_all + sh.at(b);
  extern __shared__ double gj_sm[];
  double* zs = gj_sm;                 // [kGjPB][kGjLd]
  double* as = gj_sm + kGjPB * kGjLd;  // [kGjPB][kGjT + 1]
  const double* zb = zbuf + (long long)b * kGjPB * kGjPB;
  const int tid = threadIdx.x;
  for (int e = tid; e < pb * pb; e += blockDim.x) zs[(e / pb) * kGjLd + e % pb] = zb[(e / pb) * kGjPB + e % pb];
  for (int e = tid; e < pb * kGjT; e += blockDim.x) {
    const int c = e / kGjT, jj = e % kGjT, j = j0 + jj;
    as[c * (kGjT + 1) + jj] = j < n ? a[(long long)(k0 + c) * n + j] : 0.0;
  }
  __syncthreads();
  double* rb = rbuf + (long long)b * kGjPB * sh.n;
  const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int c = ty + 16 * r;
    if (c >= pb) continue;
    double acc[4] = {0.0, 0.0, 0.0, 0.0};
    for (int q = 0; q < pb; ++q) {
      const double zv = zs[c * kGjLd + q];
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) acc[s2] += zv * as[q * (kGjT + 1) + tx + 16 * s2];
    }
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) {
      const int j = j0 + tx + 16 * s2;
      if (j < n && (j < k0 || j >= k0 + pb)) rb[(long long)c * sh.n + j] = acc[s2];
    }
  }
}

// A[i][j] -= sum_c A[i][k0 + c] R[c][j] for i, j outside the panel; one 64 x 64 tile per CTA.
__global__ void __launch_bounds__(256) k_gjb_update(GjShape sh, double* a_all, int k0, const double* rbuf,
                                                    int ntile) {
  const int b = blockIdx.y;
  const int n = sh.ord(b);
  const int i0 = (blockIdx.x / ntile) * kGjT, j0 = (blockIdx.x % ntile) * kGjT;
  if (k0 >= n || i0 >= n || j0 >= n) return;
  const int pb = min(kGjPB, n - k0);
  double* a = a_all + sh.at(b);
  extern __shared__ double gj_sm[];
  double* ls = gj_sm;                 // [kGjT][kGjLd]: A[i0 + ii][k0 + c]
  double* rs = gj_sm + kGjT * kGjLd;  // [kGjPB][kGjT + 1]: R[c][j0 + jj]
  const double* rb = rbuf + (long long)b * kGjPB * sh.n;
  const int tid = threadIdx.x;
  for (int e = tid; e < kGjT * pb; e += blockDim.x) {
    const int ii = e / pb, c = e % pb, i = i0 + ii;
    ls[ii * kGjLd + c] = i < n ? a[(long long)i * n + k0 + c] : 0.0;
  }
  for (int e = tid; e < pb * kGjT; e += blockDim.x) {
    const int c = e / kGjT, jj = e % kGjT, j = j0 + jj;
    rs[c * (kGjT + 1) + jj] = (j < n && (j < k0 || j >= k0 + pb)) ? rb[(long long)c * sh.n + j] : 0.0;
  }
  __syncthreads();
  const int tx = tid & 15, ty = tid >> 4;
  double acc[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r)
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) acc[r][s2] = 0.0;
  for (int c = 0; c < pb; ++c) {
    double lv[4], rv[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) lv[r] = ls[(ty + 16 * r) * kGjLd + c];
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) rv[s2] = rs[c * (kGjT + 1) + tx + 16 * s2];
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int s2 = 0; s2 < 4; ++s2) acc[r][s2] += lv[r] * rv[s2];
  }
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i >= n || (i >= k0 && i < k0 + pb)) continue;
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) {
      const int j = j0 + tx + 16 * s2;
      if (j < n && (j < k0 || j >= k0 + pb)) a[(long long)i * n + j] -= acc[r][s2];
    }
  }
}

// A[i][k0 + c] = -sum_c' A[i][k0 + c'] Z[c'][c] for the rows i outside the panel; 64 rows per CTA.
__global__ void __launch_bounds__(256) k_gjb_cols(GjShape sh, double* a_all, int k0, const double* zbuf) {
  const int b = blockIdx.y;
  const int n = sh.ord(b);
  const int i0 = blockIdx.x * kGjT;
  if (k0 >= n || i0 >= n) return;
  const int pb = min(kGjPB, n - k0);
  double* a = a_all + sh.at(b);
  extern __shared__ double gj_sm[];
  double* zs = gj_sm;                 // [kGjPB][kGjLd]
  double* ls = gj_sm + kGjPB * kGjLd;  // [kGjT][kGjLd]
  const double* zb = zbuf + (long long)b * kGjPB * kGjPB;
  const int tid = threadIdx.x;
  for (int e = tid; e < pb * pb; e += blockDim.x) zs[(e / pb) * kGjLd + e % pb] = zb[(e / pb) * kGjPB + e % pb];
  for (int e = tid; e < kGjT * pb; e += blockDim.x) {
    const int ii = e / pb, c = e % pb, i = i0 + ii;
    ls[ii * kGjLd + c] = i < n ? a[(long long)i * n + k0 + c] : 0.0;
  }
  __syncthreads();
  const int tx = tid & 15, ty = tid >> 4;
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = i0 + ty + 16 * r;
    if (i >= n || (i >= k0 && i < k0 + pb)) continue;
#pragma unroll
    for (int s2 = 0; s2 < 4; ++s2) {
      const int c = tx + 16 * s2;
      if (c >= pb) continue;
      double acc = 0.0;
      for (int q = 0; q < pb; ++q) acc += ls[(ty + 16 * r) * kGjLd + q] * zs[q * kGjLd + c];
      a[(long long)i * n + k0 + c] = -acc;
    }
  }
}

// the panel's rows: A[k0 + c][j] = R[c][j] outside the panel, Z[c][j - k0] inside
__global__ void k_gjb_prow(GjShape sh, double* a_all, int k0, const double* zbuf, const double* rbuf) {
  const int b = blockIdx.y;
  const int n = sh.ord(b);
  if (k0 >= n) return;
  const int pb = min(kGjPB, n - k0);
  double* a = a_all + sh.at(b);
  const double* zb = zbuf + (long long)b * kGjPB * kGjPB;
  const double* rb = rbuf + (long long)b * kGjPB * sh.n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < (long long)pb * n;
       e += (long long)gridDim.x * blockDim.x) {
    const int c = (int)(e / n), j = (int)(e % n);
    a[(long long)(k0 + c) * n + j] =
        (j >= k0 && j < k0 + pb) ? zb[c * kGjPB + (j - k0)] : rb[(long long)c * sh.n + j];
  }
}

__global__ void k_gj_sym(GjShape sh, double* a_all) {
  const int b = blockIdx.y;
  const int n = sh.ord(b);
  double* a = a_all + sh.at(b);
  const long long nn = (long long)n * n;
  for (long long e = blockIdx.x * (long long)blockDim.x + threadIdx.x; e < nn; e += (long long)gridDim.x * blockDim.x) {
    const int i = (int)(e / n), j = (int)(e % n);
    if (j > i) {
      const double v = 0.5 * (a[e] + a[(long long)j * n + i]);
      a[e] = v;
      a[(long long)j * n + i] = v;
    }
  }
}
// nb matrices of orders <= n; returns false when the scratch could not be allocated
static bool gj_inverse(int nb, GjShape sh, double* a, double tol, int* nnull, cudaStream_t st) {
  const int n = sh.n;
  double* scr = nullptr;
  const size_t bytes = sizeof(double) * (size_t)nb * (1 + (size_t)kGjPB * kGjPB + (size_t)kGjPB * n);
  if (cudaMallocAsync((void**)&scr, bytes, st) != cudaSuccess) {
    (void)cudaGetLastError();
    return false;
  }
  double* scale = scr;
  double* zbuf = scr + nb;
  double* rbuf = zbuf + (size_t)nb * kGjPB * kGjPB;
  const int sm_rows = (int)(sizeof(double) * (kGjPB * kGjLd + kGjPB * (kGjT + 1)));
  const int sm_upd = (int)(sizeof(double) * (kGjT * kGjLd + kGjPB * (kGjT + 1)));
  const int sm_cols = (int)(sizeof(double) * (kGjPB * kGjLd + kGjT * kGjLd));
  cudaFuncSetAttribute(k_gjb_rows, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_rows);
  cudaFuncSetAttribute(k_gjb_update, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_upd);
  cudaFuncSetAttribute(k_gjb_cols, cudaFuncAttributeMaxDynamicSharedMemorySize, sm_cols);
  { note_launch(); k_gj_scale<<<nb, 256, 0, st>>>(sh, a, scale); }
  const int nt = (n + kGjT - 1) / kGjT;
  const int gp = (int)std::max<long long>(1, std::min<long long>(((long long)kGjPB * n + 255) / 256, 64));
  for (int k0 = 0; k0 < n; k0 += kGjPB) {
    { note_launch(); k_gjb_diag<<<nb, 256, 0, st>>>(sh, a, k0, tol, scale, zbuf, nnull); }
    { note_launch(); k_gjb_rows<<<dim3(nt, nb), 256, sm_rows, st>>>(sh, a, k0, zbuf, rbuf); }
    { note_launch(); k_gjb_update<<<dim3(nt * nt, nb), 256, sm_upd, st>>>(sh, a, k0, rbuf, nt); }
    { note_launch(); k_gjb_cols<<<dim3(nt, nb), 256, sm_cols, st>>>(sh, a, k0, zbuf); }
    { note_launch(); k_gjb_prow<<<dim3(gp, nb), 256, 0, st>>>(sh, a, k0, zbuf, rbuf); }
  }
  const long long nn = (long long)n * n;
  const int gx = (int)std::max<long long>(1, std::min<long long>((nn + 255) / 256, (148 * 8 + nb - 1) / nb));
  { note_launch(); k_gj_sym<<<dim3(gx, nb), 256, 0, st>>>(sh, a); }
  cudaFreeAsync(scr, st);
  return true;
}

void launch_spd_inverse_r(const RankLayout& L, int nrank, int nr_max, double* dense, double tol, int* nnull,
                          cudaStream_t st) {
  // the per-rank orders as an int array next to the layout: nr_r = (first[r+1] - first[r]) x kmax
  int* nv = nullptr;
  if (cudaMallocAsync((void**)&nv, sizeof(int) * nrank, st) != cudaSuccess) {
    (void)cudaGetLastError();
    return;
  }
  std::vector<int> h_first(nrank + 1), h_nv(nrank);
  cudaMemcpyAsync(h_first.data(), L.first, sizeof(int) * (nrank + 1), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  for (int r = 0; r < nrank; ++r) h_nv[r] = (h_first[r + 1] - h_first[r]) * L.kmax;
  cudaMemcpyAsync(nv, h_nv.data(), sizeof(int) * nrank, cudaMemcpyHostToDevice, st);
  GjShape sh{nv, L.off2, nr_max};
  gj_inverse(nrank, sh, dense, tol, nnull, st);
  cudaFreeAsync(nv, st);
  cudaStreamSynchronize(st);  // the host vector must outlive the copy
}

// The cluster inverse for one of its three widths (false: the shape does not fit it, or the launch was refused).
static bool spd_inverse_cluster(int nb, int n, double* a, double tol, int* nnull, cudaStream_t st) {
  const int R = (n + kSpdCl - 1) / kSpdCl;
  if (n <= 128 && R <= kSpdWarps) return spd_inverse_cl<4, 1>(nb, n, a, tol, nnull, st);
  if (n > 128 && n <= 256 && R <= 2 * kSpdWarps) return spd_inverse_cl<8, 2>(nb, n, a, tol, nnull, st);
  if (n > 256 && n <= 384 && R <= 3 * kSpdWarps) return spd_inverse_cl<12, 3>(nb, n, a, tol, nnull, st);
  return false;
}

void launch_spd_inverse(int nb, int n, double* a, double tol, int* nnull, cudaStream_t st) {
  if (n <= 384) {
    // up to 384 unknowns both the cluster inverse and the panel Gauss-Jordan apply: the tuner times
    // them on a scratch copy of the matrices (the inverse works in place; no null counts while tuning)
    int choice = 0;
    if (n > 64 && tune_enabled()) {
      double* scr = nullptr;  // allocated only when the key is tuned (the candidates run on it)
      const size_t bytes = sizeof(double) * (size_t)nb * n * n;
      char key[64];
      snprintf(key, sizeof(key), "spd_inverse|n%d|b%d", n, nb);
      choice = tune_choose(key, 2, [&](int c) {
        if (!scr && cudaMallocAsync((void**)&scr, bytes, st) != cudaSuccess) {
          (void)cudaGetLastError();
          scr = nullptr;
          return false;
        }
        cudaMemcpyAsync(scr, a, bytes, cudaMemcpyDeviceToDevice, st);
        return c == 0 ? spd_inverse_cluster(nb, n, scr, tol, nullptr, st)
                      : gj_inverse(nb, GjShape{nullptr, nullptr, n}, scr, tol, nullptr, st);
      }, st);
      if (scr) cudaFreeAsync(scr, st);
    }
    if (choice == 1 && gj_inverse(nb, GjShape{nullptr, nullptr, n}, a, tol, nnull, st)) return;
    if (spd_inverse_cluster(nb, n, a, tol, nnull, st)) return;
  }
  if (n > 384 && gj_inverse(nb, GjShape{nullptr, nullptr, n}, a, tol, nnull, st)) return;
  const int smem = 2 * n * sizeof(double);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_spd_inverse, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  { note_launch(); k_spd_inverse<<<nb, 1024, smem, st>>>(n, a, tol, nnull); }
}

// ---------------------------------------------------------------------------
// Level-3 HEP (_PC_setup_lv3_eigen, :1086-1115): smallest en2 eigenpairs of
// each rank's dense rank-Neumann matrix.  SLEPc's shift-and-invert Krylov-
// Schur is replaced by block inverse subspace iteration with the precomputed
// (A + mu I)^-1, SVQB orthonormalisation and a Rayleigh-Ritz step on A; the
// eigenvectors come out orthonormal in the 2-norm as SLEPc returns them.
// work: 3 * nr * p doubles per rank.
#define PMF_L3_MAXP 32

// Out[i * p + c] = sum_l M[i][l] Xs[l * ldx + c] (- shift[c] Xs[i * ldx + c]) for c < q, with the
// block Xs staged in shared memory: one warp per row, lanes along l (coalesced
// row reads), eight column accumulators per pass, warp reductions.
__device__ void cta_rows_mm(const double* __restrict__ M, int nr, const double* Xs, int ldx, int q, double* Out,
                            int p, const double* shift) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int i = wid; i < nr; i += nw) {
    const double* row = M + (long long)i * nr;
    for (int c0 = 0; c0 < q; c0 += 8) {
      double acc[8];
#pragma unroll
      for (int c = 0; c < 8; ++c) acc[c] = 0.0;
      for (int l = lane; l < nr; l += 32) {
        const double mv = row[l];
        const double* xr = Xs + l * ldx + c0;
#pragma unroll
        for (int c = 0; c < 8; ++c)
          if (c0 + c < q) acc[c] += mv * xr[c];
      }
#pragma unroll
      for (int c = 0; c < 8; ++c) {
        const double v = warp_sum(acc[c]);
        if (lane == 0 && c0 + c < q)
          Out[(long long)i * p + c0 + c] = shift ? v - shift[c0 + c] * Xs[i * ldx + c0 + c] : v;
      }
    }
  }
}

// Xs[l * ldx + c] = X[l * p + c], c < q
__device__ __forceinline__ void cta_stage_block(const double* X, int nr, int p, int q, double* Xs, int ldx) {
  for (int e = threadIdx.x; e < nr * q; e += blockDim.x) {
    const int l = e / q, c = e - l * q;
    Xs[l * ldx + c] = X[(long long)l * p + c];
  }
  __syncthreads();
}

__global__ void __launch_bounds__(512) k_dense_smallest_eig(RankLayout L, int en2, int p, const double* A_all,
                                                             const double* inv_all, double* V_all, double* evals_all,
                                                             int* iters, double tol, int max_it, double* work_all,
                                                             int ldx) {
  extern __shared__ double xs[];  // nr x ldx staging block when ldx > 0
  const int r = blockIdx.x;
  const int nr = rank_nr(L, r);
  const double* A = A_all + L.off2[r];
  const double* inv = inv_all + L.off2[r];
  double* X = work_all + L.offw[r];
  double* Y = X + (long long)nr * p;
  double* AY = Y + (long long)nr * p;
  __shared__ double G[PMF_L3_MAXP * PMF_L3_MAXP], U[PMF_L3_MAXP * PMF_L3_MAXP], w[PMF_L3_MAXP],
      C[PMF_L3_MAXP * PMF_L3_MAXP], dsc[PMF_L3_MAXP], jac[64];
  __shared__ int ijac[32];
  __shared__ int keep, conv;
  __shared__ double anorm;
  const int tid = threadIdx.x, nt = blockDim.x;
  // scale of A: max |diag|
  if (tid == 0) {
    double m = 0.0;
    for (int i = 0; i < nr; ++i) m = fmax(m, fabs(A[(long long)i * nr + i]));
    anorm = m > 0 ? m : 1.0;
  }
  for (long long e = tid; e < (long long)nr * p; e += nt)
    X[e] = hash_uniform(((unsigned long long)r << 40) ^ (unsigned long long)e);
  __syncthreads();
  int it = 0;
  for (; it < max_it; ++it) {
    // Y = inv X
    if (ldx > 0) {
      cta_stage_block(X, nr, p, p, xs, ldx);
      cta_rows_mm(inv, nr, xs, ldx, p, Y, p, nullptr);
    } else {
      for (long long e = tid; e < (long long)nr * p; e += nt) {
        const int i = (int)(e / p), j = (int)(e % p);
        const double* row = inv + (long long)i * nr;
        double acc = 0.0;
        for (int l = 0; l < nr; ++l) acc += row[l] * X[(long long)l * p + j];
        Y[e] = acc;
      }
    }
    __syncthreads();
    // SVQB: G = Y^T Y, D^-1/2 G D^-1/2 = U w U^T, X = Y D^-1/2 U w^-1/2 (kept columns)
    for (int e = tid; e < p * p; e += nt) {
      const int a = e / p, b = e % p;
      double acc = 0.0;
      for (int l = 0; l < nr; ++l) acc += Y[(long long)l * p + a] * Y[(long long)l * p + b];
      G[a * PMF_L3_MAXP + b] = acc;
    }
    __syncthreads();
    if (tid < p) dsc[tid] = 1.0 / sqrt(fmax(G[tid * PMF_L3_MAXP + tid], 1e-300));
    __syncthreads();
    for (int e = tid; e < p * p; e += nt) {
      const int a = e / p, b = e % p;
      G[a * PMF_L3_MAXP + b] *= dsc[a] * dsc[b];
    }
    __syncthreads();
    cta_jacobi_eigh(G, U, w, p, PMF_L3_MAXP, ijac, jac);
    if (tid == 0) {
      int kk = 0;
      const double wmax = w[p - 1];
      for (int c = p - 1; c >= 0; --c)
        if (w[c] > 1e-12 * wmax) ++kk;
      keep = kk;
    }
    __syncthreads();
    const int q = keep;  // kept columns are the last q (largest w)
    for (int e = tid; e < p * q; e += nt) {
      const int a = e / q, c = e % q;
      const int cc = p - q + c;
      C[a * PMF_L3_MAXP + c] = dsc[a] * U[a * PMF_L3_MAXP + cc] / sqrt(w[cc]);
    }
    __syncthreads();
    for (long long e = tid; e < (long long)nr * q; e += nt) {
      const int i = (int)(e / q), c = (int)(e % q);
      double acc = 0.0;
      for (int a = 0; a < p; ++a) acc += Y[(long long)i * p + a] * C[a * PMF_L3_MAXP + c];
      X[(long long)i * p + c] = acc;
    }
    __syncthreads();
    // AY = A X (q columns), H = X^T A X
    if (ldx > 0) {
      cta_stage_block(X, nr, p, q, xs, ldx);
      cta_rows_mm(A, nr, xs, ldx, q, AY, p, nullptr);
    } else {
      for (long long e = tid; e < (long long)nr * q; e += nt) {
        const int i = (int)(e / q), c = (int)(e % q);
        const double* row = A + (long long)i * nr;
        double acc = 0.0;
        for (int l = 0; l < nr; ++l) acc += row[l] * X[(long long)l * p + c];
        AY[(long long)i * p + c] = acc;
      }
    }
    __syncthreads();
    for (int e = tid; e < q * q; e += nt) {
      const int a = e / q, b = e % q;
      double acc = 0.0;
      for (int l = 0; l < nr; ++l) acc += X[(long long)l * p + a] * AY[(long long)l * p + b];
      G[a * PMF_L3_MAXP + b] = acc;
    }
    __syncthreads();
    for (int e = tid; e < q * q; e += nt) {  // symmetrise
      const int a = e / q, b = e % q;
      if (a < b) {
        const double v = 0.5 * (G[a * PMF_L3_MAXP + b] + G[b * PMF_L3_MAXP + a]);
        G[a * PMF_L3_MAXP + b] = v;
        G[b * PMF_L3_MAXP + a] = v;
      }
    }
    __syncthreads();
    cta_jacobi_eigh(G, U, w, q, PMF_L3_MAXP, ijac, jac);
    // X <- X U (through Y as scratch)
    for (long long e = tid; e < (long long)nr * q; e += nt) {
      const int i = (int)(e / q), c = (int)(e % q);
      double ax = 0.0;
      for (int a = 0; a < q; ++a) ax += X[(long long)i * p + a] * U[a * PMF_L3_MAXP + c];
      Y[(long long)i * p + c] = ax;
    }
    __syncthreads();
    for (long long e = tid; e < (long long)nr * q; e += nt) {
      const int i = (int)(e / q), c = (int)(e % q);
      X[(long long)i * p + c] = Y[(long long)i * p + c];
    }
    __syncthreads();
    // recompute AY for the Ritz vectors and the residuals of the wanted ones
    if (ldx > 0) {
      cta_stage_block(X, nr, p, q, xs, ldx);
      cta_rows_mm(A, nr, xs, ldx, q, AY, p, w);
    } else {
      for (long long e = tid; e < (long long)nr * q; e += nt) {
        const int i = (int)(e / q), c = (int)(e % q);
        const double* row = A + (long long)i * nr;
        double acc = 0.0;
        for (int l = 0; l < nr; ++l) acc += row[l] * X[(long long)l * p + c];
        AY[(long long)i * p + c] = acc - w[c] * X[(long long)i * p + c];
      }
    }
    __syncthreads();
    if (tid == 0) conv = 1;
    __syncthreads();
    for (int c = tid; c < min(en2, q); c += nt) {
      double rr = 0.0;
      for (int l = 0; l < nr; ++l) rr += AY[(long long)l * p + c] * AY[(long long)l * p + c];
      if (sqrt(rr) > tol * anorm) conv = 0;
    }
    if (q < en2 && tid == 0) conv = 0;
    __syncthreads();
    // pad dropped columns with fresh random directions for the next sweep
    for (long long e = tid; e < (long long)nr * (p - q); e += nt) {
      const int i = (int)(e / (p - q)), c = q + (int)(e % (p - q));
      X[(long long)i * p + c] = hash_uniform(((unsigned long long)(r + 7) << 44) ^ ((unsigned long long)it << 32) ^
                                             (unsigned long long)e);
    }
    __syncthreads();
    if (conv) break;
  }
  double* V = V_all + L.offv[r];
  for (long long e = tid; e < (long long)nr * en2; e += nt) {
    const int i = (int)(e / en2), j = (int)(e % en2);
    V[e] = X[(long long)i * p + j];
  }
  if (tid < en2) evals_all[(long long)r * en2 + tid] = w[tid];
  if (tid == 0) iters[r] = it + 1;
}

// The same iteration for ranks whose block does not fit in shared memory, in
// phases over all ranks: the two dense products of an iteration (Y = inv X
// and AY = A X) spread over CTAs of 32 rows each, the projected problems
// (SVQB of Y, Rayleigh-Ritz on A) one CTA per rank.  The Ritz vectors' images
// are rotated with the vectors (A (X U) = (A X) U) instead of recomputed, so an
// iteration streams each rank's two matrices once.  A converged rank's
// kernels return at once; the host checks every 8 iterations whether all
// ranks have converged.
struct L3Rank {
  double anorm;
  double w[PMF_L3_MAXP];
  int q, conv, it;
};
constexpr int kL3Rows = 32;    // rows per CTA of the products
constexpr int kL3Tile = 256;   // l-values per shared-memory tile of the block
constexpr int kL3Cols = 16;    // columns the product kernel holds in registers

__global__ void k_l3_init(RankLayout L, int p, const double* A_all, double* work_all, L3Rank* st) {
  const int r = blockIdx.x;
  const int nr = rank_nr(L, r);
  const double* A = A_all + L.off2[r];
  double* X = work_all + L.offw[r];
  __shared__ double red[32];
  double m = 0.0;
  for (int i = threadIdx.x; i < nr; i += blockDim.x) m = fmax(m, fabs(A[(long long)i * nr + i]));
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_xor_sync(0xffffffffu, m, o));
  if (lane == 0) red[wid] = m;
  __syncthreads();
  if (threadIdx.x == 0) {
    double v = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); ++w) v = fmax(v, red[w]);
    st[r].anorm = v > 0 ? v : 1.0;
    for (int c = 0; c < PMF_L3_MAXP; ++c) st[r].w[c] = 0.0;
    st[r].q = p;
    st[r].conv = 0;
    st[r].it = 0;
  }
  for (long long e = threadIdx.x; e < (long long)nr * p; e += blockDim.x)
    X[e] = hash_uniform(((unsigned long long)r << 40) ^ (unsigned long long)e);
}

// Out = M In for the rank's first `cols` columns (cols = p, or the kept count q): block src/dst of the
// rank's workspace (0 X, 1 Y, 2 AY), 32 rows per CTA, 8 warps x 4 rows, lanes along the row.
__global__ void __launch_bounds__(256) k_l3_mm(RankLayout L, int p, const double* M_all, double* work_all, int src,
                                               int dst, int use_q, const L3Rank* st) {
  const int r = blockIdx.y;
  if (st[r].conv) return;
  const int nr = rank_nr(L, r);
  const int i0 = blockIdx.x * kL3Rows;
  if (i0 >= nr) return;
  const int cols = use_q ? st[r].q : p;
  const double* M = M_all + L.off2[r];
  const double* In = work_all + L.offw[r] + (long long)src * nr * p;
  double* Out = work_all + L.offw[r] + (long long)dst * nr * p;
  __shared__ double xs[kL3Tile][kL3Cols + 1];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  double acc[4][kL3Cols];
#pragma unroll
  for (int a = 0; a < 4; ++a)
#pragma unroll
    for (int c = 0; c < kL3Cols; ++c) acc[a][c] = 0.0;
  for (int l0 = 0; l0 < nr; l0 += kL3Tile) {
    for (int e = threadIdx.x; e < kL3Tile * kL3Cols; e += blockDim.x) {
      const int l = e / kL3Cols, c = e % kL3Cols;
      xs[l][c] = (l0 + l < nr && c < cols) ? In[(long long)(l0 + l) * p + c] : 0.0;
    }
    __syncthreads();
    const int lend = min(kL3Tile, nr - l0);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      const int i = i0 + wid * 4 + a;
      if (i >= nr) continue;
      const double* row = M + (long long)i * nr + l0;
      for (int l = lane; l < lend; l += 32) {
        const double mv = row[l];
#pragma unroll
        for (int c = 0; c < kL3Cols; ++c) acc[a][c] += mv * xs[l][c];
      }
    }
    __syncthreads();
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const int i = i0 + wid * 4 + a;
#pragma unroll
    for (int c = 0; c < kL3Cols; ++c) {
      const double v = warp_sum(acc[a][c]);
      if (lane == 0 && i < nr && c < cols) Out[(long long)i * p + c] = v;
    }
  }
}

// SVQB of Y: G = Y^T Y, D^-1/2 G D^-1/2 = U w U^T, X = Y D^-1/2 U w^-1/2 on the kept columns (q).
__global__ void __launch_bounds__(512) k_l3_svqb(RankLayout L, int p, double* work_all, L3Rank* st) {
  const int r = blockIdx.x;
  if (st[r].conv) return;
  const int nr = rank_nr(L, r);
  double* X = work_all + L.offw[r];
  const double* Y = X + (long long)nr * p;
  __shared__ double G[PMF_L3_MAXP * PMF_L3_MAXP], U[PMF_L3_MAXP * PMF_L3_MAXP], w[PMF_L3_MAXP],
      C[PMF_L3_MAXP * PMF_L3_MAXP], dsc[PMF_L3_MAXP], jac[64];
  __shared__ int ijac[32];
  __shared__ int keep;
  const int tid = threadIdx.x, nt = blockDim.x;
  for (int e = tid; e < p * p; e += nt) {
    const int a = e / p, b = e % p;
    double acc = 0.0;
    for (int l = 0; l < nr; ++l) acc += Y[(long long)l * p + a] * Y[(long long)l * p + b];
    G[a * PMF_L3_MAXP + b] = acc;
  }
  __syncthreads();
  if (tid < p) dsc[tid] = 1.0 / sqrt(fmax(G[tid * PMF_L3_MAXP + tid], 1e-300));
  __syncthreads();
  for (int e = tid; e < p * p; e += nt) {
    const int a = e / p, b = e % p;
    G[a * PMF_L3_MAXP + b] *= dsc[a] * dsc[b];
  }
  __syncthreads();
  cta_jacobi_eigh(G, U, w, p, PMF_L3_MAXP, ijac, jac);
  if (tid == 0) {
    int kk = 0;
    const double wmax = w[p - 1];
    for (int c = p - 1; c >= 0; --c)
      if (w[c] > 1e-12 * wmax) ++kk;
    keep = kk;
    st[r].q = kk;
  }
  __syncthreads();
  const int q = keep;  // kept columns are the last q (largest w)
  for (int e = tid; e < p * q; e += nt) {
    const int a = e / q, c = e % q;
    const int cc = p - q + c;
    C[a * PMF_L3_MAXP + c] = dsc[a] * U[a * PMF_L3_MAXP + cc] / sqrt(w[cc]);
  }
  __syncthreads();
  for (long long e = tid; e < (long long)nr * q; e += nt) {
    const int i = (int)(e / q), c = (int)(e % q);
    double acc = 0.0;
    for (int a = 0; a < p; ++a) acc += Y[(long long)i * p + a] * C[a * PMF_L3_MAXP + c];
    X[(long long)i * p + c] = acc;
  }
}

// Rayleigh-Ritz on A: H = X^T AY, H = U w U^T, X <- X U, AY <- AY U, residual test of the wanted pairs;
// columns dropped by the SVQB get fresh random directions for the next iteration.
__global__ void __launch_bounds__(512) k_l3_rr(RankLayout L, int en2, int p, double* work_all, L3Rank* st,
                                               double tol, int it) {
  const int r = blockIdx.x;
  if (st[r].conv) return;
  const int nr = rank_nr(L, r);
  double* X = work_all + L.offw[r];
  double* Y = X + (long long)nr * p;
  double* AY = Y + (long long)nr * p;
  __shared__ double G[PMF_L3_MAXP * PMF_L3_MAXP], U[PMF_L3_MAXP * PMF_L3_MAXP], w[PMF_L3_MAXP], jac[64];
  __shared__ int ijac[32];
  __shared__ int conv;
  const int tid = threadIdx.x, nt = blockDim.x;
  const int q = st[r].q;
  for (int e = tid; e < q * q; e += nt) {
    const int a = e / q, b = e % q;
    double acc = 0.0;
    for (int l = 0; l < nr; ++l) acc += X[(long long)l * p + a] * AY[(long long)l * p + b];
    G[a * PMF_L3_MAXP + b] = acc;
  }
  __syncthreads();
  for (int e = tid; e < q * q; e += nt) {  // symmetrise
    const int a = e / q, b = e % q;
    if (a < b) {
      const double v = 0.5 * (G[a * PMF_L3_MAXP + b] + G[b * PMF_L3_MAXP + a]);
      G[a * PMF_L3_MAXP + b] = v;
      G[b * PMF_L3_MAXP + a] = v;
    }
  }
  __syncthreads();
  cta_jacobi_eigh(G, U, w, q, PMF_L3_MAXP, ijac, jac);
  // X <- X U and AY <- AY U, through Y
  for (long long e = tid; e < (long long)nr * q; e += nt) {
    const int i = (int)(e / q), c = (int)(e % q);
    double ax = 0.0;
    for (int a = 0; a < q; ++a) ax += X[(long long)i * p + a] * U[a * PMF_L3_MAXP + c];
    Y[(long long)i * p + c] = ax;
  }
  __syncthreads();
  for (long long e = tid; e < (long long)nr * q; e += nt) {
    const int i = (int)(e / q), c = (int)(e % q);
    X[(long long)i * p + c] = Y[(long long)i * p + c];
  }
  __syncthreads();
  for (long long e = tid; e < (long long)nr * q; e += nt) {
    const int i = (int)(e / q), c = (int)(e % q);
    double ay = 0.0;
    for (int a = 0; a < q; ++a) ay += AY[(long long)i * p + a] * U[a * PMF_L3_MAXP + c];
    Y[(long long)i * p + c] = ay;
  }
  __syncthreads();
  for (long long e = tid; e < (long long)nr * q; e += nt) {
    const int i = (int)(e / q), c = (int)(e % q);
    AY[(long long)i * p + c] = Y[(long long)i * p + c];
  }
  if (tid == 0) conv = q >= en2 ? 1 : 0;
  __syncthreads();
  const double thr = tol * st[r].anorm;
  for (int c = tid; c < min(en2, q); c += nt) {
    double rr = 0.0;
    for (int l = 0; l < nr; ++l) {
      const double v = AY[(long long)l * p + c] - w[c] * X[(long long)l * p + c];
      rr += v * v;
    }
    if (sqrt(rr) > thr) conv = 0;
  }
  __syncthreads();
  if (tid < q) st[r].w[tid] = w[tid];
  if (tid == 0) {
    st[r].it = it + 1;
    st[r].conv = conv;
  }
  if (!conv)
    for (long long e = tid; e < (long long)nr * (p - q); e += nt) {
      const int i = (int)(e / (p - q)), c = q + (int)(e % (p - q));
      X[(long long)i * p + c] = hash_uniform(((unsigned long long)(r + 7) << 44) ^ ((unsigned long long)it << 32) ^
                                             (unsigned long long)e);
    }
}

__global__ void k_l3_count(const L3Rank* st, int nrank, int* left) {
  __shared__ int n;
  if (threadIdx.x == 0) n = 0;
  __syncthreads();
  for (int r = threadIdx.x; r < nrank; r += blockDim.x)
    if (!st[r].conv) atomicAdd(&n, 1);
  __syncthreads();
  if (threadIdx.x == 0) *left = n;
}

__global__ void k_l3_out(RankLayout L, int en2, int p, const double* work_all, const L3Rank* st, double* V_all,
                         double* evals_all, int* iters) {
  const int r = blockIdx.x;
  const int nr = rank_nr(L, r);
  const double* X = work_all + L.offw[r];
  double* V = V_all + L.offv[r];
  for (long long e = threadIdx.x; e < (long long)nr * en2; e += blockDim.x) {
    const int i = (int)(e / en2), j = (int)(e % en2);
    V[e] = X[(long long)i * p + j];
  }
  if (threadIdx.x < en2) evals_all[(long long)r * en2 + threadIdx.x] = st[r].w[threadIdx.x];
  if (threadIdx.x == 0) iters[r] = st[r].it;
}

void launch_dense_smallest_eig(const RankLayout& L, int nrank, int nr, int en2, int p, const double* A,
                               const double* inv, double* V, double* evals, int* iters, double tol, int max_it,
                               double* work, cudaStream_t st) {
  // stage the iteration block in shared memory (odd leading dimension: no bank conflicts) when it fits
  const int ldx = p | 1;
  const size_t smem = (size_t)nr * ldx * sizeof(double);
  L3Rank* rs = nullptr;
  int* left = nullptr;
  if (smem > 160 * 1024 && p <= kL3Cols && cudaMallocAsync((void**)&rs, sizeof(L3Rank) * nrank + 16, st) == cudaSuccess) {
    left = reinterpret_cast<int*>(rs + nrank);
    const int gx = (nr + kL3Rows - 1) / kL3Rows;
    { note_launch(); k_l3_init<<<nrank, 256, 0, st>>>(L, p, A, work, rs); }
    for (int it = 0; it < max_it; ++it) {
      { note_launch(); k_l3_mm<<<dim3(gx, nrank), 256, 0, st>>>(L, p, inv, work, 0, 1, 0, rs); }
      { note_launch(); k_l3_svqb<<<nrank, 512, 0, st>>>(L, p, work, rs); }
      { note_launch(); k_l3_mm<<<dim3(gx, nrank), 256, 0, st>>>(L, p, A, work, 0, 2, 1, rs); }
      { note_launch(); k_l3_rr<<<nrank, 512, 0, st>>>(L, en2, p, work, rs, tol, it); }
      if ((it + 1) % 8 == 0 || it + 1 == max_it) {
        int h = 1;
        { note_launch(); k_l3_count<<<1, 256, 0, st>>>(rs, nrank, left); }
        if (cudaMemcpyAsync(&h, left, sizeof(int), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
            cudaStreamSynchronize(st) != cudaSuccess)
          break;  // the caller's stream check reports the error
        if (h == 0) break;
      }
    }
    { note_launch(); k_l3_out<<<nrank, 256, 0, st>>>(L, en2, p, work, rs, V, evals, iters); }
    cudaFreeAsync(rs, st);
    return;
  }
  (void)cudaGetLastError();
  int ld = ldx;
  size_t sm = smem;
  if (sm > 160 * 1024) {
    ld = 0;
    sm = 0;
  } else {  // the kernel also holds ~26 KB of static shared memory
    cudaFuncSetAttribute(k_dense_smallest_eig, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
  }
  { note_launch(); k_dense_smallest_eig<<<nrank, 512, sm, st>>>(L, en2, p, A, inv, V, evals, iters, tol, max_it, work, ld); }
}

}  // namespace pmf
