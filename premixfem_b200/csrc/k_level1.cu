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
//   2. meanwhile every thread (one per x-line (j, k)) loads its line of the
//      residual x (FP64) and, when the visit has an iterate y, its line of y
//      and of the diagonal with 16-byte vector loads, and the threads on the
//      subdomain's faces load the neighbouring cells of y and the couplings
//      of the upper faces;
//   3. r = x - A y on the subdomain (the same operations in the same order as
//      the natural-order kernel, so the result is bit-identical), then the
//      forward and backward hyperplane sweeps in shared memory, and the line
//      is written out (y + IC^-1 r, as the preconditioner's FP32 iterate or
//      the FP64 result with the z.r partial).
//
// With 16^3 FP32 subdomains a CTA uses 89 KB of shared memory, so two CTAs
// share an SM and one's copy overlaps the other's sweeps.  The only wait is
// thread 0's on the mbarrier, bounded by an iteration limit: if the copy had
// not landed by then the CTA records the failure in *err and returns without
// touching the data (the host turns the flag into an error code).
//
// Requirements (checked by the host before this kernel is chosen): every
// subdomain 16 cells wide in x with x0 a multiple of 4, M a multiple of 4
// (16-byte aligned rows), ny*nz <= 256 lines.
#include <stdint.h>

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

constexpr int kNX = 16;                  // cells per x-line of the blocked kernel
constexpr long long kBulkSpinLimit = 1LL << 22;  // mbarrier polls before the CTA gives up

__device__ __forceinline__ uint32_t smem_u32(const void* p) {
  return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void mbar_init(uint64_t* b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void fence_mbar_init() {
  asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
__device__ __forceinline__ void mbar_arrive_expect_tx(uint64_t* b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
// global -> shared bulk copy (TMA engine); bytes a multiple of 16, both addresses 16-byte aligned
__device__ __forceinline__ void bulk_g2s(void* dst, const void* src, uint32_t bytes, uint64_t* b) {
  asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                   smem_u32(dst)),
               "l"(src), "r"(bytes), "r"(smem_u32(b))
               : "memory");
}
__device__ __forceinline__ bool mbar_try_wait(uint64_t* b, uint32_t parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
      : "=r"(ok)
      : "r"(smem_u32(b)), "r"(parity)
      : "memory");
  return ok != 0;
}

// 16 consecutive values with 16-byte loads / stores (16-byte aligned address)
__device__ __forceinline__ void load16(const float* p, float (&r)[kNX]) {
  const float4* q = reinterpret_cast<const float4*>(p);
#pragma unroll
  for (int v = 0; v < 4; ++v) {
    const float4 a = q[v];
    r[4 * v] = a.x;
    r[4 * v + 1] = a.y;
    r[4 * v + 2] = a.z;
    r[4 * v + 3] = a.w;
  }
}
__device__ __forceinline__ void load16(const double* p, double (&r)[kNX]) {
  const double2* q = reinterpret_cast<const double2*>(p);
#pragma unroll
  for (int v = 0; v < 8; ++v) {
    const double2 a = q[v];
    r[2 * v] = a.x;
    r[2 * v + 1] = a.y;
  }
}
__device__ __forceinline__ void store16(float* p, const float (&r)[kNX]) {
  float4* q = reinterpret_cast<float4*>(p);
#pragma unroll
  for (int v = 0; v < 4; ++v) q[v] = make_float4(r[4 * v], r[4 * v + 1], r[4 * v + 2], r[4 * v + 3]);
}
__device__ __forceinline__ void store16(double* p, const double (&r)[kNX]) {
  double2* q = reinterpret_cast<double2*>(p);
#pragma unroll
  for (int v = 0; v < 8; ++v) q[v] = make_double2(r[2 * v], r[2 * v + 1]);
}

}  // namespace

// Shared-memory layout of k_ic_apply_blk (bytes): header (mbarrier, flag,
// reduction scratch) 512, coefficients ldc x sizeof(V4), u ldc x sizeof(T),
// y faces 2 x 16 x (max_nz + max_ny) x sizeof(T), upper-face couplings
// 16 x (max_nz + max_ny) x sizeof(T).
template <typename T>
static size_t ic_blk_smem(int ldc, int max_ny, int max_nz) {
  typedef typename Coef4<T>::type V4;
  return 512 + (size_t)ldc * sizeof(V4) + (size_t)ldc * sizeof(T) + (size_t)3 * kNX * (max_nz + max_ny) * sizeof(T);
}

template <typename T, bool HAS_Y, bool FINAL>
__global__ void __launch_bounds__(256, (sizeof(T) == 4 ? 2 : 1))
    k_ic_apply_blk(Grid g, const SubInfo* subs, const long long* coff, const typename Coef4<T>::type* coef,
                   const T* tx, const T* ty, const T* tz, const T* diag, const double* x, const T* yin, T* out_t,
                   double* out_d, double* part, const int* done, int* err, int ldc, int fny, int fnz) {
  typedef typename Coef4<T>::type V4;
  if (done && *done) return;
  extern __shared__ __align__(128) unsigned char smem_raw[];
  uint64_t* bar = reinterpret_cast<uint64_t*>(smem_raw);
  int* flag = reinterpret_cast<int*>(smem_raw + 8);
  double* red = reinterpret_cast<double*>(smem_raw + 256);
  V4* cs = reinterpret_cast<V4*>(smem_raw + 512);
  T* u = reinterpret_cast<T*>(cs + ldc);
  T* yf = u + ldc;                   // y of the neighbouring cells: [face 0 y-][nz][16], [1 y+][nz][16],
                                     // [2 z-][ny][16], [3 z+][ny][16]
  T* tf = yf + 2 * kNX * (fnz + fny);  // couplings of the upper faces: [y+][nz][16], [z+][ny][16]
  const SubInfo S = subs[blockIdx.x];
  const int ny = S.ny, nz = S.nz, nxny = kNX * ny, ncells = nxny * nz, nlines = ny * nz;
  const int t = threadIdx.x;
  const int j = t % ny, k = t / ny;
  const bool line = t < nlines;
  if (t == 0) {
    mbar_init(bar, 1);
    fence_mbar_init();
    const uint32_t bytes = (uint32_t)(ncells * sizeof(V4));
    mbar_arrive_expect_tx(bar, bytes);
    bulk_g2s(cs, coef + coff[blockIdx.x], bytes, bar);
  }
  const long long MN = (long long)g.M * g.N;
  const long long cg0 = ((long long)(S.z0 + k) * g.N + (S.y0 + j)) * g.M + S.x0;
  double xr[kNX];
  T yr[kNX], dr[kNX];
  T yl = (T)0, yh = (T)0, txh = (T)0;
  if (line) {
    load16(x + cg0, xr);
    if (HAS_Y) {
      load16(yin + cg0, yr);
      load16(diag + cg0, dr);
      if (S.x0 > 0) yl = yin[cg0 - 1];
      if (S.x0 + kNX < g.M) {
        yh = yin[cg0 + kNX];
        txh = tx[cg0 + kNX];
      }
      T tmp[kNX], tmp2[kNX];
      if (j == 0 && S.y0 > 0) {
        load16(yin + cg0 - g.M, tmp);
#pragma unroll
        for (int i = 0; i < kNX; ++i) yf[k * kNX + i] = tmp[i];
      }
      if (j == ny - 1 && S.y0 + ny < g.N) {
        load16(yin + cg0 + g.M, tmp);
        load16(ty + cg0 + g.M, tmp2);
#pragma unroll
        for (int i = 0; i < kNX; ++i) {
          yf[(fnz + k) * kNX + i] = tmp[i];
          tf[k * kNX + i] = tmp2[i];
        }
      }
      if (k == 0 && S.z0 > 0) {
        load16(yin + cg0 - MN, tmp);
#pragma unroll
        for (int i = 0; i < kNX; ++i) yf[(2 * fnz + j) * kNX + i] = tmp[i];
      }
      if (k == nz - 1 && S.z0 + nz < g.P) {
        load16(yin + cg0 + MN, tmp);
        load16(tz + cg0 + MN, tmp2);
#pragma unroll
        for (int i = 0; i < kNX; ++i) {
          yf[(2 * fnz + fny + j) * kNX + i] = tmp[i];
          tf[(fnz + j) * kNX + i] = tmp2[i];
        }
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
  const int base = (k * ny + j) * kNX;  // local index of the line's first cell
  if (HAS_Y) {
    // r = x - A y in the natural-order kernel's order of operations (apply_A):
    // diagonal, x-, x+, y-, y+, z-, z+
    if (line) store16(u + base, yr);
    __syncthreads();
    T rr[kNX];
    if (line) {
#pragma unroll
      for (int i = 0; i < kNX; ++i) {
        const int cl = base + i;
        const V4 c = cs[cl];
        T v = dr[i] * yr[i];
        if (i > 0)
          v -= c.x * yr[i - 1];
        else if (S.x0 > 0)
          v -= c.x * yl;
        if (i < kNX - 1)
          v -= cs[cl + 1].x * yr[i + 1];
        else if (S.x0 + kNX < g.M)
          v -= txh * yh;
        if (j > 0)
          v -= c.y * u[cl - kNX];
        else if (S.y0 > 0)
          v -= c.y * yf[k * kNX + i];
        if (j < ny - 1)
          v -= cs[cl + kNX].y * u[cl + kNX];
        else if (S.y0 + ny < g.N)
          v -= tf[k * kNX + i] * yf[(fnz + k) * kNX + i];
        if (k > 0)
          v -= c.z * u[cl - nxny];
        else if (S.z0 > 0)
          v -= c.z * yf[(2 * fnz + j) * kNX + i];
        if (k < nz - 1)
          v -= cs[cl + nxny].z * u[cl + nxny];
        else if (S.z0 + nz < g.P)
          v -= tf[(fnz + j) * kNX + i] * yf[(2 * fnz + fny + j) * kNX + i];
        rr[i] = (T)xr[i] - v;
      }
    }
    __syncthreads();
    if (line) store16(u + base, rr);
  } else {
    if (line) {
      T rr[kNX];
#pragma unroll
      for (int i = 0; i < kNX; ++i) rr[i] = (T)xr[i];
      store16(u + base, rr);
    }
  }
  __syncthreads();
  // forward sweep (D + L) w = r: w_i = (r_i + sum_{lower j} t_ij w_j) / D_i, hyperplane i + j + k = d
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
  double dot = 0.0;
  if (line) {
    T o[kNX];
#pragma unroll
    for (int i = 0; i < kNX; ++i) {
      o[i] = u[base + i];
      if (HAS_Y) o[i] += yr[i];
    }
    if (FINAL) {
      double od[kNX];
#pragma unroll
      for (int i = 0; i < kNX; ++i) {
        od[i] = (double)o[i];
        dot += xr[i] * od[i];
      }
      store16(out_d + cg0, od);
    } else {
      store16(out_t + cg0, o);
    }
  }
  if (FINAL) {
    dot = block_sum(dot, red);
    if (t == 0) part[blockIdx.x] = dot;
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
size_t ic_blk_smem_bytes(int max_cells, int max_ny, int max_nz) {
  return ic_blk_smem<T>(max_cells, max_ny, max_nz);
}

template <typename T>
void launch_ic_apply_blk(const Grid& g, const SubInfo* subs, int nsub, int max_cells, int max_ny, int max_nz,
                         const long long* coff, const void* coef, const T* tx, const T* ty, const T* tz,
                         const T* diag, const double* x, const T* yin, T* out_t, double* out_d, double* part,
                         const int* done, int* err, cudaStream_t st) {
  typedef typename Coef4<T>::type V4;
  const int ldc = max_cells;
  const size_t smem = ic_blk_smem<T>(ldc, max_ny, max_nz);
  const bool fin = out_d != nullptr;
  const V4* c4 = reinterpret_cast<const V4*>(coef);
#define PMF_BLK(HY, FN)                                                                                              \
  {                                                                                                                  \
    cudaFuncSetAttribute(k_ic_apply_blk<T, HY, FN>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);        \
    note_launch();                                                                                                   \
    k_ic_apply_blk<T, HY, FN><<<nsub, 256, smem, st>>>(g, subs, coff, c4, tx, ty, tz, diag, x, yin, out_t, out_d,  \
                                                       part, done, err, ldc, max_ny, max_nz);                        \
  }
  if (yin) {
    if (fin) PMF_BLK(true, true) else PMF_BLK(true, false)
  } else {
    if (fin) PMF_BLK(false, true) else PMF_BLK(false, false)
  }
#undef PMF_BLK
}

#define PMF_INST(T)                                                                                                \
  template void launch_pack_ic_coef<T>(const Grid&, const SubInfo*, int, const long long*, const T*, const T*,   \
                                       const T*, const T*, void*, cudaStream_t);                                 \
  template size_t ic_blk_smem_bytes<T>(int, int, int);                                                           \
  template void launch_ic_apply_blk<T>(const Grid&, const SubInfo*, int, int, int, int, const long long*,        \
                                       const void*, const T*, const T*, const T*, const T*, const double*,       \
                                       const T*, T*, double*, double*, const int*, int*, cudaStream_t);
PMF_INST(float)
PMF_INST(double)
#undef PMF_INST

}  // namespace pmf
