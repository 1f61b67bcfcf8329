// Level-1 IC(0) block solves (_PC_apply_vec_lv1, src/PreMixFEM_3D.c:1429-1479)
// with the factor stored per subdomain and staged into shared memory by one
// TMA bulk copy.
//
// The preconditioner keeps, next to the natural-order operator arrays, a
// subdomain-blocked copy of what the sweeps read: for the cells of subdomain
// s in local order cl = i + nx*(j + ny*k), coef[coff[s] + cl] = {tx, ty, tz,
// 1/D} (the lower-face transmissibilities of the cell and its inverse IC(0)
// pivot; the couplings are not masked at the subdomain's faces).  One CTA
// solves one subdomain:
//
//   1. thread 0 starts a cp.async.bulk copy of the subdomain's coefficient
//      block (64 KB for 16^3 FP32 cells) into shared memory, completed on an
//      mbarrier;
//   2. meanwhile the threads stage the subdomain's residual x (and, when the
//      visit has an iterate, y) in shared memory with coalesced loads;
//   3. r = x - A y on the subdomain (the natural-order kernel's operations in
//      its order; the two kernels differ only where the compiler contracts a
//      multiply-add differently), then the forward and backward hyperplane
//      sweeps in shared memory, and the result is written out (y + IC^-1 r,
//      as the preconditioner's FP32 iterate or the FP64 result with the z.r
//      partial).
//
// With 16^3 FP32 subdomains a CTA uses 81 KB of shared memory (97 KB with an
// iterate), so two CTAs share an SM and one's copy overlaps the other's
// sweeps.  The only wait is
// thread 0's on the mbarrier, bounded by an iteration limit: if the copy had
// not landed by then the CTA records the failure in *err and returns without
// touching the data (the host turns the flag into an error code).
//
// Requirements (checked by the host before this kernel is chosen): every
// subdomain 16 cells wide in x with x0 a multiple of 4, M a multiple of 4
// (16-byte aligned rows), ny*nz <= 256 lines.
//
// k_ic_apply_stg (below) is the same solve with steps 2 and 3 reorganised so
// that every global load of a CTA is issued before any is used; the launch-
// shape tuner chooses between the two and the natural-order kernel per visit.
#include <stdint.h>

#include "pmf_bulk.cuh"
#include "pmf_kernels.h"

namespace pmf {

template <typename T>
struct Coef4;
template <>
struct Coef4<float> {
  typedef float4 type;
};
template <>
struct Coef4<double> {
  typedef double4 type;
};

namespace {

constexpr int kNX = 16;  // cells per x-line of the blocked kernel
}  // namespace

// Shared-memory layout of k_ic_apply_blk (bytes): header (mbarrier, flag,
// reduction scratch) 512, coefficients ldc x sizeof(V4), u ldc x sizeof(T),
// and, for visits with an iterate, the subdomain's y: ldc x sizeof(T).
template <typename T>
static size_t ic_blk_smem(int ldc, bool has_y) {
  typedef typename Coef4<T>::type V4;
  return 512 + (size_t)ldc * sizeof(V4) + (size_t)ldc * sizeof(T) * (has_y ? 2 : 1);
}

// The forward and backward IC(0) sweeps of one subdomain in shared memory:
// thread (j, k) = (t % ny, t / ny) owns the x-line (., j, k) and handles its
// cell i = d - j - k on hyperplane d.  Every thread of the CTA takes part in
// the barriers.
template <typename T, typename V4>
__device__ __forceinline__ void ic_blk_sweeps(const V4* cs, T* u, int t, int ny, int nz) {
  const int nxny = kNX * ny, nlines = ny * nz;
  // forward sweep (D + L) w = r: w_i = (r_i + sum_{lower j} t_ij w_j) / D_i, hyperplane i + j + k = d
  const int j = t % ny, k = t / ny;
  const bool line = t < nlines;
  const int base = (k * ny + j) * kNX;
  const int nplanes = kNX + ny + nz - 2;
  const int jk = j + k;
  for (int d = 0; d < nplanes; ++d) {
    const int i = d - jk;
    if (line && i >= 0 && i < kNX) {
      const int cl = base + i;
      const V4 c = cs[cl];
      T s = u[cl];
      if (k > 0) s += c.z * u[cl - nxny];
      if (j > 0) s += c.y * u[cl - kNX];
      if (i > 0) s += c.x * u[cl - 1];
      u[cl] = s * c.w;
    }
    __syncthreads();
  }
  // backward sweep (D + L^T) z = D w: z_i = w_i + (sum_{upper j} t_ij z_j) / D_i
  for (int d = nplanes - 1; d >= 0; --d) {
    const int i = d - jk;
    if (line && i >= 0 && i < kNX) {
      const int cl = base + i;
      T s = (T)0;
      if (i < kNX - 1) s += cs[cl + 1].x * u[cl + 1];
      if (j < ny - 1) s += cs[cl + kNX].y * u[cl + kNX];
      if (k < nz - 1) s += cs[cl + nxny].z * u[cl + nxny];
      u[cl] = u[cl] + s * cs[cl].w;
    }
    __syncthreads();
  }
}

// Work is cell-parallel except in the sweeps: thread t handles the cells
// cl = t + n * blockDim.x, consecutive threads on consecutive cells, so the
// shared-memory reads of the coefficients and of y are free of bank
// conflicts; blockDim.x is a multiple of 16, so a thread keeps its position i
// in the x-line and only steps through lines.  In the sweeps thread (j, k)
// owns the x-line (., j, k) and handles its cell i = d - j - k on hyperplane d.
template <typename T, bool HAS_Y, bool FINAL>
__global__ void __launch_bounds__(512, 2)
    k_ic_apply_blk(Grid g, const SubInfo* subs, const long long* coff, const typename Coef4<T>::type* coef,
                   const T* tx, const T* ty, const T* tz, const T* diag, const double* x, const T* yin, T* out_t,
                   double* out_d, double* part, const int* done, int* err, int ldc) {
  typedef typename Coef4<T>::type V4;
  if (done && *done) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  int* flag = reinterpret_cast<int*>(smem_raw + 8);
  double* red = reinterpret_cast<double*>(smem_raw + 256);
  V4* cs = reinterpret_cast<V4*>(smem_raw + 512);
  T* u = reinterpret_cast<T*>(cs + ldc);
  T* ys = u + ldc;  // HAS_Y only
  const SubInfo S = subs[blockIdx.x];
  const int ny = S.ny, nz = S.nz, nxny = kNX * ny, ncells = nxny * nz;
  const int t = threadIdx.x, bd = blockDim.x, lstep = bd / kNX;
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    const uint32_t bytes = (uint32_t)(ncells * sizeof(V4));
    mbar_arrive_expect_tx(bar, bytes);
    bulk_g2s(cs, coef + coff[blockIdx.x], bytes, bar);
  }
  const long long MN = (long long)g.M * g.N;
  const int i0 = t & (kNX - 1);
  // the subdomain's x (and y) into shared memory while the coefficients land
  {
    int line = t >> 4, j = line % ny, k = line / ny;
    for (int cl = t; cl < ncells; cl += bd) {
      const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0;
      u[cl] = (T)x[cg];
      if (HAS_Y) ys[cl] = yin[cg];
      j += lstep;
      while (j >= ny) {
        j -= ny;
        ++k;
      }
    }
  }
  if (t == 0) {
    long long spins = 0;
    bool ok = true;
    while (!mbar_try_wait(bar, 0)) {
      if (++spins > kBulkSpinLimit) {
        ok = false;
        break;
      }
    }
    if (!ok) {
      atomicOr(err, 1);
      // give the copy in flight a last bounded chance to land before the CTA exits
      for (long long s2 = 0; s2 < kBulkSpinLimit && !mbar_try_wait(bar, 0); ++s2) {
      }
    }
    *flag = ok ? 0 : 1;
  }
  __syncthreads();
  if (*flag) return;
  if (HAS_Y) {
    // r = x - A y in apply_A's order of operations: diagonal, x-, x+, y-, y+, z-, z+
    int line = t >> 4, j = line % ny, k = line / ny;
    const int i = i0;
    for (int cl = t; cl < ncells; cl += bd) {
      const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i;
      const V4 c = cs[cl];
      const T yc = ys[cl];
      T v = diag[cg] * yc;
      if (i > 0)
        v -= c.x * ys[cl - 1];
      else if (S.x0 > 0)
        v -= c.x * yin[cg - 1];
      if (i < kNX - 1)
        v -= cs[cl + 1].x * ys[cl + 1];
      else if (S.x0 + kNX < g.M)
        v -= tx[cg + 1] * yin[cg + 1];
      if (j > 0)
        v -= c.y * ys[cl - kNX];
      else if (S.y0 > 0)
        v -= c.y * yin[cg - g.M];
      if (j < ny - 1)
        v -= cs[cl + kNX].y * ys[cl + kNX];
      else if (S.y0 + ny < g.N)
        v -= ty[cg + g.M] * yin[cg + g.M];
      if (k > 0)
        v -= c.z * ys[cl - nxny];
      else if (S.z0 > 0)
        v -= c.z * yin[cg - MN];
      if (k < nz - 1)
        v -= cs[cl + nxny].z * ys[cl + nxny];
      else if (S.z0 + nz < g.P)
        v -= tz[cg + MN] * yin[cg + MN];
      u[cl] = u[cl] - v;
      j += lstep;
      while (j >= ny) {
        j -= ny;
        ++k;
      }
    }
    __syncthreads();
  }
  ic_blk_sweeps<T, V4>(cs, u, t, ny, nz);
  double dot = 0.0;
  {
    int line = t >> 4, j = line % ny, k = line / ny;
    for (int cl = t; cl < ncells; cl += bd) {
      const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0;
      T o = u[cl];
      if (HAS_Y) o += ys[cl];
      if (FINAL) {
        const double od = (double)o;
        out_d[cg] = od;
        dot += x[cg] * od;
      } else {
        out_t[cg] = o;
      }
      j += lstep;
      while (j >= ny) {
        j -= ny;
        ++k;
      }
    }
  }
  if (FINAL) {
    dot = block_sum(dot, red);
    if (t == 0) part[blockIdx.x] = dot;
  }
}

// k_ic_apply_blk with every global load of a CTA issued in one pass, before
// any of them is used.  Each thread holds PER = 4096 / BD cells at fixed
// compile-time positions (unrolled loops), so its loads of x, the iterate y
// and the diagonal, and its share of the subdomain's face halo (the iterate
// on the six neighbouring planes and the couplings across the three upper
// faces: 9 x 256 values) are all in flight together while the bulk copy of
// the factor lands.  The residual r = x - A y is then formed from shared
// memory and registers only, in the blocked kernel's order of operations, and
// the sweeps are the blocked kernel's.  Takes the blocked kernel's shapes with
// ny <= 16 and nz <= 16 (each face at most 256 cells).
namespace {
constexpr int kHalo = 256;  // entries per face of the staged halo
}  // namespace

template <typename T>
static size_t ic_stg_smem(int ldc, bool has_y) {
  return ic_blk_smem<T>(ldc, has_y) + (has_y ? (size_t)9 * kHalo * sizeof(T) : 0);
}

template <typename T, bool HAS_Y, bool FINAL, int BD>
__global__ void __launch_bounds__(BD, sizeof(T) == 4 ? 2 : 1)
    k_ic_apply_stg(Grid g, const SubInfo* subs, const long long* coff, const typename Coef4<T>::type* coef,
                   const T* tx, const T* ty, const T* tz, const T* diag, const double* x, const T* yin, T* out_t,
                   double* out_d, double* part, const int* done, int* err, int ldc) {
  typedef typename Coef4<T>::type V4;
  constexpr int PER = 4096 / BD, LSTEP = BD / kNX, HPER = (9 * kHalo + BD - 1) / BD;
  if (done && *done) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  int* flag = reinterpret_cast<int*>(smem_raw + 8);
  double* red = reinterpret_cast<double*>(smem_raw + 256);
  V4* cs = reinterpret_cast<V4*>(smem_raw + 512);
  T* u = reinterpret_cast<T*>(cs + ldc);
  T* ys = u + ldc;      // HAS_Y only
  T* hal = ys + ldc;    // HAS_Y only: faces x- y, x+ y, x+ tx, y- y, y+ y, y+ ty, z- y, z+ y, z+ tz
  const SubInfo S = subs[blockIdx.x];
  const int ny = S.ny, nz = S.nz, nxny = kNX * ny, nlines = ny * nz;
  const int t = threadIdx.x;
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    const uint32_t bytes = (uint32_t)(nxny * nz * sizeof(V4));
    mbar_arrive_expect_tx(bar, bytes);
    bulk_g2s(cs, coef + coff[blockIdx.x], bytes, bar);
  }
  const int i0 = t & (kNX - 1), line0 = t >> 4;
  // cell p of this thread: line line0 + p * LSTEP (if < nlines), position i0 in the line
  T xr[PER], yr[PER], dr[PER];
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int line = line0 + p * LSTEP;
    if (line < nlines) {
      const int j = line % ny, k = line / ny;
      const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0;
      xr[p] = (T)x[cg];
      if (HAS_Y) {
        yr[p] = yin[cg];
        dr[p] = diag[cg];
      }
    }
  }
  T hr[HPER];
  if (HAS_Y) {
#pragma unroll
    for (int q = 0; q < HPER; ++q) {
      const int h = t + q * BD;
      hr[q] = (T)0;
      if (h < 9 * kHalo) {
        const int f = h / kHalo, e = h % kHalo;
        long long cg = -1;
        const T* src = yin;
        if (f < 3) {  // x faces, entry = line k * ny + j
          const int j = e % ny, k = e / ny;
          const long long row = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M;
          if (e < nlines && f == 0 && S.x0 > 0) cg = row + S.x0 - 1;
          if (e < nlines && f > 0 && S.x0 + kNX < g.M) cg = row + S.x0 + kNX;
          if (f == 2) src = tx;
        } else if (f < 6) {  // y faces, entry = k * 16 + i
          const int i = e & (kNX - 1), k = e / kNX;
          if (k < nz && f == 3 && S.y0 > 0) cg = ((long long)(S.z0 + k) * g.N + (S.y0 - 1)) * g.M + S.x0 + i;
          if (k < nz && f > 3 && S.y0 + ny < g.N)
            cg = ((long long)(S.z0 + k) * g.N + (S.y0 + ny)) * g.M + S.x0 + i;
          if (f == 5) src = ty;
        } else {  // z faces, entry = j * 16 + i
          const int i = e & (kNX - 1), j = e / kNX;
          if (j < ny && f == 6 && S.z0 > 0) cg = ((long long)(S.z0 - 1) * g.N + (S.y0 + j)) * g.M + S.x0 + i;
          if (j < ny && f > 6 && S.z0 + nz < g.P)
            cg = ((long long)(S.z0 + nz) * g.N + (S.y0 + j)) * g.M + S.x0 + i;
          if (f == 8) src = tz;
        }
        if (cg >= 0) hr[q] = src[cg];
      }
    }
  }
#pragma unroll
  for (int p = 0; p < PER; ++p) {
    const int cl = t + p * BD;
    if (line0 + p * LSTEP < nlines) {
      u[cl] = xr[p];
      if (HAS_Y) ys[cl] = yr[p];
    }
  }
  if (HAS_Y) {
#pragma unroll
    for (int q = 0; q < HPER; ++q)
      if (t + q * BD < 9 * kHalo) hal[t + q * BD] = hr[q];
  }
  if (t == 0) *flag = mbar_wait_bounded(bar) ? 0 : 1;
  __syncthreads();
  if (*flag) {
    if (t == 0) atomicOr(err, 1);
    return;
  }
  if (HAS_Y) {
    // r = x - A y in apply_A's order of operations: diagonal, x-, x+, y-, y+, z-, z+
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int line = line0 + p * LSTEP;
      if (line < nlines) {
        const int j = line % ny, k = line / ny, i = i0, cl = t + p * BD;
        const V4 c = cs[cl];
        const T yc = ys[cl];
        T v = dr[p] * yc;
        if (i > 0)
          v -= c.x * ys[cl - 1];
        else if (S.x0 > 0)
          v -= c.x * hal[0 * kHalo + line];
        if (i < kNX - 1)
          v -= cs[cl + 1].x * ys[cl + 1];
        else if (S.x0 + kNX < g.M)
          v -= hal[2 * kHalo + line] * hal[1 * kHalo + line];
        if (j > 0)
          v -= c.y * ys[cl - kNX];
        else if (S.y0 > 0)
          v -= c.y * hal[3 * kHalo + k * kNX + i];
        if (j < ny - 1)
          v -= cs[cl + kNX].y * ys[cl + kNX];
        else if (S.y0 + ny < g.N)
          v -= hal[5 * kHalo + k * kNX + i] * hal[4 * kHalo + k * kNX + i];
        if (k > 0)
          v -= c.z * ys[cl - nxny];
        else if (S.z0 > 0)
          v -= c.z * hal[6 * kHalo + j * kNX + i];
        if (k < nz - 1)
          v -= cs[cl + nxny].z * ys[cl + nxny];
        else if (S.z0 + nz < g.P)
          v -= hal[8 * kHalo + j * kNX + i] * hal[7 * kHalo + j * kNX + i];
        u[cl] = u[cl] - v;
      }
    }
    __syncthreads();
  }
  ic_blk_sweeps<T, V4>(cs, u, t, ny, nz);
  double dot = 0.0;
  if (FINAL) {
    double xd[PER];
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int line = line0 + p * LSTEP;
      if (line < nlines) {
        const int j = line % ny, k = line / ny;
        xd[p] = x[((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0];
      }
    }
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int line = line0 + p * LSTEP;
      if (line < nlines) {
        const int j = line % ny, k = line / ny, cl = t + p * BD;
        const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0;
        T o = u[cl];
        if (HAS_Y) o += ys[cl];
        const double od = (double)o;
        out_d[cg] = od;
        dot += xd[p] * od;
      }
    }
    dot = block_sum(dot, red);
    if (t == 0) part[blockIdx.x] = dot;
  } else {
#pragma unroll
    for (int p = 0; p < PER; ++p) {
      const int line = line0 + p * LSTEP;
      if (line < nlines) {
        const int j = line % ny, k = line / ny, cl = t + p * BD;
        T o = u[cl];
        if (HAS_Y) o += ys[cl];
        out_t[((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0 + i0] = o;
      }
    }
  }
}

template <typename T>
__global__ void k_pack_ic_coef(Grid g, const SubInfo* subs, const long long* coff, const T* tx, const T* ty,
                               const T* tz, const T* inv, typename Coef4<T>::type* coef) {
  typedef typename Coef4<T>::type V4;
  const SubInfo S = subs[blockIdx.x];
  const int nxny = S.nx * S.ny, ncells = nxny * S.nz;
  V4* out = coef + coff[blockIdx.x];
  for (int cl = threadIdx.x; cl < ncells; cl += blockDim.x) {
    const int i = cl % S.nx, tt = cl / S.nx, j = tt % S.ny, k = tt / S.ny;
    const long long cg = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + (S.x0 + i);
    V4 c;
    c.x = tx[cg];
    c.y = ty[cg];
    c.z = tz[cg];
    c.w = inv[cg];
    out[cl] = c;
  }
}

template <typename T>
void launch_pack_ic_coef(const Grid& g, const SubInfo* subs, int nsub, const long long* coff, const T* tx,
                         const T* ty, const T* tz, const T* inv, void* coef, cudaStream_t st) {
  note_launch();
  k_pack_ic_coef<T><<<nsub, 256, 0, st>>>(g, subs, coff, tx, ty, tz, inv,
                                          reinterpret_cast<typename Coef4<T>::type*>(coef));
}

size_t ic_blk_coef_bytes(int prec_bytes) { return prec_bytes == 4 ? sizeof(float4) : sizeof(double4); }

template <typename T>
size_t ic_blk_smem_bytes(int max_cells) {
  return ic_blk_smem<T>(max_cells, true);
}

template <typename T>
void launch_ic_apply_blk(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const long long* coff,
                         const void* coef, const T* tx, const T* ty, const T* tz, const T* diag, const double* x,
                         const T* yin, T* out_t, double* out_d, double* part, const int* done, int* err,
                         cudaStream_t st, int threads) {
  typedef typename Coef4<T>::type V4;
  const int ldc = max_cells;
  const size_t smem = ic_blk_smem<T>(ldc, yin != nullptr);
  const bool fin = out_d != nullptr;
  const V4* c4 = reinterpret_cast<const V4*>(coef);
  threads = (threads == 256 || threads == 512) ? threads : 512;
#define PMF_BLK(HY, FN)                                                                                              \
  {                                                                                                                  \
    cudaFuncSetAttribute(k_ic_apply_blk<T, HY, FN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);        \
    note_launch();                                                                                                   \
    k_ic_apply_blk<T, HY, FN><<<nsub, threads, smem, st>>>(g, subs, coff, c4, tx, ty, tz, diag, x, yin, out_t,      \
                                                           out_d, part, done, err, ldc);                             \
  }
  if (yin) {
    if (fin) PMF_BLK(true, true) else PMF_BLK(true, false)
  } else {
    if (fin) PMF_BLK(false, true) else PMF_BLK(false, false)
  }
#undef PMF_BLK
}

template <typename T>
size_t ic_stg_smem_bytes(int max_cells) {
  return ic_stg_smem<T>(max_cells, true);
}

template <typename T>
void launch_ic_apply_stg(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const long long* coff,
                         const void* coef, const T* tx, const T* ty, const T* tz, const T* diag, const double* x,
                         const T* yin, T* out_t, double* out_d, double* part, const int* done, int* err,
                         cudaStream_t st) {
  typedef typename Coef4<T>::type V4;
  const int ldc = max_cells;
  const size_t smem = ic_stg_smem<T>(ldc, yin != nullptr);
  const bool fin = out_d != nullptr;
  const V4* c4 = reinterpret_cast<const V4*>(coef);
#define PMF_STG(HY, FN)                                                                                              \
  {                                                                                                                  \
    cudaFuncSetAttribute(k_ic_apply_stg<T, HY, FN, 512>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);   \
    note_launch();                                                                                                   \
    k_ic_apply_stg<T, HY, FN, 512><<<nsub, 512, smem, st>>>(g, subs, coff, c4, tx, ty, tz, diag, x, yin, out_t,     \
                                                            out_d, part, done, err, ldc);                            \
  }
  if (yin) {
    if (fin) PMF_STG(true, true) else PMF_STG(true, false)
  } else {
    if (fin) PMF_STG(false, true) else PMF_STG(false, false)
  }
#undef PMF_STG
}

#define PMF_INST(T)                                                                                                \
  template void launch_pack_ic_coef<T>(const Grid&, const SubInfo*, int, const long long*, const T*, const T*,   \
                                       const T*, const T*, void*, cudaStream_t);                                 \
  template size_t ic_blk_smem_bytes<T>(int);                                                                     \
  template void launch_ic_apply_blk<T>(const Grid&, const SubInfo*, int, int, const long long*, const void*,     \
                                       const T*, const T*, const T*, const T*, const double*, const T*, T*,      \
                                       double*, double*, const int*, int*, cudaStream_t, int);                   \
  template size_t ic_stg_smem_bytes<T>(int);                                                                     \
  template void launch_ic_apply_stg<T>(const Grid&, const SubInfo*, int, int, const long long*, const void*,     \
                                       const T*, const T*, const T*, const T*, const double*, const T*, T*,      \
                                       double*, double*, const int*, int*, cudaStream_t);
PMF_INST(float)
PMF_INST(double)
#undef PMF_INST

}  // namespace pmf
