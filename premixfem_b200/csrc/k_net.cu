// Kernels of the learned-initialisation network (layer table in pmf_net.h).
//
// Forward: every layer is one implicit GEMM, out[row][cout] = sum over
// (tap, cin) of in[gather(row, tap)][cin] * W[tap][cin][cout], computed on
// the BF16 tensor cores (mma.sync m16n8k16, FP32 accumulation) with the bias,
// skip addition, ReLU and the BF16 rounding fused in the epilogue.  A CTA owns
// 64 output voxels of one sample and all output channels; per tap it stages
// the 64 gathered input rows and the tap's weight slice in shared memory.
// Transposed (up2) layers order their rows by (sample, parity, coarse voxel)
// so that one tile uses one weight slice.
//
// Backward (training only, FP32 CUDA cores): the input gradient is a gather
// over the taps that touched each input voxel, fused with the skip-gradient
// addition and the ReLU mask of the input activation; the weight gradient is
// a tiled reduction over output rows with FP32 atomics per chunk.
#include <cuda_bf16.h>

#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <random>
#include <vector>

#include "pmf_kernels.h"
#include "pmf_net.h"
#include "tune.h"

namespace pmf {

const NetLayer kNetLayers[NET_LAYERS] = {
    // type     cin cout s_in s_out relu skip in out
    {NL_CONV3, 16, 32, 16, 16, 1, -1, 0, 1},
    {NL_DOWN2, 32, 64, 16, 8, 1, -1, 1, 2},
    {NL_CONV3, 64, 64, 8, 8, 1, -1, 2, 3},
    {NL_DOWN2, 64, 96, 8, 4, 1, -1, 3, 4},
    {NL_CONV3, 96, 96, 4, 4, 1, -1, 4, 5},
    {NL_UP2, 96, 64, 4, 8, 1, 3, 5, 6},
    {NL_UP2, 64, 32, 8, 16, 1, 1, 6, 7},
    {NL_CONV3, 32, 32, 16, 16, 1, -1, 7, 8},
    {NL_CONV1, 32, 16, 16, 16, 0, -1, 8, 9},
};
const NetActShape kNetActs[NET_ACTS] = {{16, 16}, {16, 32}, {8, 64}, {8, 64}, {4, 96},
                                        {4, 96},  {8, 64},  {16, 32}, {16, 32}, {16, 16}};

namespace {

__device__ __forceinline__ int cube(int s) { return s * s * s; }

// Input voxel read by output voxel o through tap t (-1: zero padding / not this tap).
__device__ __forceinline__ int in_vox(int type, int s_in, int s_out, int o, int t) {
  int x = o % s_out, y = (o / s_out) % s_out, z = o / (s_out * s_out);
  if (type == NL_CONV3) {
    x += t % 3 - 1;
    y += (t / 3) % 3 - 1;
    z += t / 9 - 1;
    if (x < 0 || y < 0 || z < 0 || x >= s_in || y >= s_in || z >= s_in) return -1;
    return (z * s_in + y) * s_in + x;
  }
  if (type == NL_DOWN2) return ((2 * z + (t >> 2)) * s_in + 2 * y + ((t >> 1) & 1)) * s_in + 2 * x + (t & 1);
  if (type == NL_CONV1) return o;
  const int par = (x & 1) | ((y & 1) << 1) | ((z & 1) << 2);
  if (par != t) return -1;
  return ((z >> 1) * s_in + (y >> 1)) * s_in + (x >> 1);
}

// Fine voxel of coarse voxel v (edge s_in) and parity d.
__device__ __forceinline__ int up_vox(int v, int d, int s_in) {
  const int x = v % s_in, y = (v / s_in) % s_in, z = v / (s_in * s_in), s = 2 * s_in;
  return ((2 * z + (d >> 2)) * s + 2 * y + ((d >> 1) & 1)) * s + 2 * x + (d & 1);
}

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void ldsm_x4(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void ldsm_x4_t(uint32_t addr, uint32_t& r0, uint32_t& r1, uint32_t& r2, uint32_t& r3) {
  asm volatile("ldmatrix.sync.aligned.m8n8.x4.trans.shared.b16 {%0,%1,%2,%3}, [%4];\n"
               : "=r"(r0), "=r"(r1), "=r"(r2), "=r"(r3)
               : "r"(addr));
}
__device__ __forceinline__ void mma_bf16(float* c, uint32_t a0, uint32_t a1, uint32_t a2, uint32_t a3, uint32_t b0,
                                         uint32_t b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a0), "r"(a1), "r"(a2), "r"(a3), "r"(b0), "r"(b1));
}

struct FwdArgs {
  int type, cin, cout, s_in, s_out, relu;
  const __nv_bfloat16* in;
  const __nv_bfloat16* W;
  const float* bias;
  const __nv_bfloat16* skip;
  __nv_bfloat16* out;
  float* outf;
};

__device__ __forceinline__ void cp_async16(void* dst, const void* src, bool valid) {
  // 16-byte global->shared copy; zero-filled when !valid (src-size 0)
  const unsigned d = (unsigned)__cvta_generic_to_shared(dst);
  const int n = valid ? 16 : 0;
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(d), "l"(src), "r"(n));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// ROWS output voxels of one sample per CTA (ROWS / (16 MT) warps, each MT
// 16-row tiles x all output channels, sharing the weight fragments); the
// gathered input rows and the weight slice of the next tap are copied with
// cp.async while the current tap is multiplied.
template <int NT, int ROWS, int MT>
__global__ void __launch_bounds__(ROWS * 2 / MT) k_net_fwd(FwdArgs a) {
  extern __shared__ __align__(16) unsigned char smraw[];
  __shared__ int rowout[ROWS];
  const int lda = a.cin + 8, ldb = a.cout + 8;
  __nv_bfloat16* As0 = reinterpret_cast<__nv_bfloat16*>(smraw);
  __nv_bfloat16* Bs0 = As0 + 2 * ROWS * lda;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int nthr = ROWS * 2 / MT;
  const int so3 = cube(a.s_out), si3 = cube(a.s_in);
  const long long r0 = (long long)blockIdx.x * ROWS;
  const int b = (int)(r0 / so3);
  const int rem0 = (int)(r0 % so3);
  const bool up = a.type == NL_UP2;
  const int d_tile = up ? rem0 / si3 : 0;
  for (int q = tid; q < ROWS; q += nthr) rowout[q] = up ? up_vox((rem0 + q) % si3, d_tile, a.s_in) : rem0 + q;
  __syncthreads();
  const int ntap = (up || a.type == NL_CONV1) ? 1 : net_taps(a.type);
  const int vin = a.cin >> 3, vout = a.cout >> 3;
  // Per-thread copy assignments, fixed for all taps: up to EA input-row
  // vectors and EB weight vectors, with their coordinates precomputed so the
  // per-tap gather needs no division.
  constexpr int NTHR = ROWS * 2 / MT;
  constexpr int EA = (ROWS * 12 + NTHR - 1) / NTHR;  // cin <= 96: 12 vectors per row
  constexpr int EB = (96 * 12 + NTHR - 1) / NTHR;
  int a_dst[EA], a_xyz[EA], a_src[EA];
  int b_dst[EB];
  const int sin = a.s_in;
#pragma unroll
  for (int j = 0; j < EA; ++j) {
    const int e = tid + j * nthr;
    a_dst[j] = -1;
    if (e < ROWS * vin) {
      const int rr = e / vin, cv = e % vin;
      a_dst[j] = rr * lda + cv * 8;
      if (up) {
        a_src[j] = ((rem0 + rr) % si3) * a.cin + cv * 8;
        a_xyz[j] = 0;
      } else {
        const int o = rowout[rr], so = a.s_out;
        int x = o % so, y = (o / so) % so, z = o / (so * so);
        if (a.type == NL_DOWN2) {
          x *= 2;
          y *= 2;
          z *= 2;
        }
        a_xyz[j] = x | (y << 10) | (z << 20);
        a_src[j] = ((z * sin + y) * sin + x) * a.cin + cv * 8;
      }
    }
  }
#pragma unroll
  for (int j = 0; j < EB; ++j) {
    const int e = tid + j * nthr;
    b_dst[j] = e < a.cin * vout ? (e / vout) * ldb + (e % vout) * 8 : -1;
  }
  const __nv_bfloat16* inb = a.in + (size_t)b * si3 * a.cin;
  auto stage = [&](int ti, int buf) {
    const int t = up ? d_tile : ti;
    __nv_bfloat16* As = As0 + buf * ROWS * lda;
    __nv_bfloat16* Bs = Bs0 + buf * a.cin * ldb;
    int dx = 0, dy = 0, dz = 0;
    if (a.type == NL_CONV3) {
      dx = t % 3 - 1;
      dy = (t / 3) % 3 - 1;
      dz = t / 9 - 1;
    } else if (a.type == NL_DOWN2) {
      dx = t & 1;
      dy = (t >> 1) & 1;
      dz = t >> 2;
    }
    const int off = ((dz * sin + dy) * sin + dx) * a.cin;
#pragma unroll
    for (int j = 0; j < EA; ++j) {
      if (a_dst[j] < 0) continue;
      bool ok = true;
      if (a.type == NL_CONV3) {
        const int x = (a_xyz[j] & 1023) + dx, y = ((a_xyz[j] >> 10) & 1023) + dy, z = (a_xyz[j] >> 20) + dz;
        ok = x >= 0 && y >= 0 && z >= 0 && x < sin && y < sin && z < sin;
      }
      const int src = ok ? a_src[j] + (up || a.type == NL_CONV1 ? 0 : off) : 0;
      cp_async16(As + a_dst[j], inb + src, ok);
    }
    const __nv_bfloat16* wt = a.W + (size_t)t * a.cin * a.cout;
#pragma unroll
    for (int j = 0; j < EB; ++j) {
      if (b_dst[j] < 0) continue;
      cp_async16(Bs + b_dst[j], wt + 8 * (tid + j * nthr), true);
    }
    cp_async_commit();
  };
  float acc[MT][NT][4];
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
    for (int n = 0; n < NT; ++n) acc[mt][n][0] = acc[mt][n][1] = acc[mt][n][2] = acc[mt][n][3] = 0.f;
  stage(0, 0);
  for (int ti = 0; ti < ntap; ++ti) {
    if (ti + 1 < ntap) {
      stage(ti + 1, (ti + 1) & 1);
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    const __nv_bfloat16* As = As0 + (ti & 1) * ROWS * lda;
    const __nv_bfloat16* Bs = Bs0 + (ti & 1) * a.cin * ldb;
    for (int kc = 0; kc < a.cin; kc += 16) {
      uint32_t af[MT][4];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
        ldsm_x4(smem_u32(As + ((warp * MT + mt) * 16 + (lane & 15)) * lda + kc + (lane >> 4) * 8), af[mt][0],
                af[mt][1], af[mt][2], af[mt][3]);
#pragma unroll
      for (int np = 0; np < NT / 2; ++np) {
        uint32_t b0, b1, b2, b3;
        ldsm_x4_t(smem_u32(Bs + (kc + (lane & 7) + ((lane >> 3) & 1) * 8) * ldb + np * 16 + (lane >> 4) * 8), b0, b1,
                  b2, b3);
#pragma unroll
        for (int mt = 0; mt < MT; ++mt) {
          mma_bf16(acc[mt][2 * np], af[mt][0], af[mt][1], af[mt][2], af[mt][3], b0, b1);
          mma_bf16(acc[mt][2 * np + 1], af[mt][0], af[mt][1], af[mt][2], af[mt][3], b2, b3);
        }
      }
    }
    __syncthreads();  // the buffer just read is refilled two taps later
  }
  // epilogue: bias, skip, ReLU, store
#pragma unroll
  for (int mt = 0; mt < MT; ++mt)
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const int rr = (warp * MT + mt) * 16 + (lane >> 2) + h * 8;
    const size_t rowbase = ((size_t)b * so3 + rowout[rr]) * a.cout;
#pragma unroll
    for (int n = 0; n < NT; ++n) {
      const int col = n * 8 + (lane & 3) * 2;
      float v0 = acc[mt][n][2 * h] + a.bias[col];
      float v1 = acc[mt][n][2 * h + 1] + a.bias[col + 1];
      if (a.skip) {
        const __nv_bfloat162 s2 = *reinterpret_cast<const __nv_bfloat162*>(a.skip + rowbase + col);
        v0 += __bfloat162float(s2.x);
        v1 += __bfloat162float(s2.y);
      }
      if (a.relu) {
        v0 = fmaxf(v0, 0.f);
        v1 = fmaxf(v1, 0.f);
      }
      if (a.outf) {
        *reinterpret_cast<float2*>(a.outf + rowbase + col) = make_float2(v0, v1);
      } else {
        *reinterpret_cast<__nv_bfloat162*>(a.out + rowbase + col) = __floats2bfloat162_rn(v0, v1);
      }
    }
  }
}

// ---- 3x3x3 convolutions of 16^3 patches on the tcgen05 tensor cores ---------------------------
// One CTA (four warps) per patch marches through the 16 output z-planes.  The
// input planes z-1, z, z+1 sit with a one-voxel zero halo in a ring of four
// shared-memory slots ([slot][cin/8][18][18][8 channels] BF16) while plane
// z+2 is copied in with cp.async; all 27 taps' weights stay resident in the
// UMMA K-major layout ([tap][k-step][2][cout/8][8][8]).  An output plane is
// two 128-row tiles (rows y x 8 x-positions, one per x half), and for tap
// (dx, dy, dz) a tile's A operand is just a window of the haloed plane: a
// no-swizzle K-major descriptor whose 8-row groups step by one haloed row
// (288 B) and whose two 8-channel groups step by one channel plane, so the
// im2col gather costs nothing.  One thread issues the 27 x cin/16 x 2
// tcgen05.mma (kind::f16, BF16 in, FP32 accumulation in TMEM, M = 128,
// N = cout) and commits them to the plane's mbarrier; the accumulators are
// double-buffered across planes so that the epilogue of plane z-1
// (tcgen05.ld, bias, ReLU, BF16 store) overlaps the MMAs of plane z.  Every
// wait is bounded; a wait that runs out sets *err and skips the stores.
// Every load is a plain per-CTA cp.async (single-GPU code).
namespace {
constexpr int kTcPl = 18 * 18;                 // positions of one haloed plane
constexpr long long kTcSpin = 1LL << 24;      // mbarrier polls before giving up

__device__ __forceinline__ void tc_mbar_init(uint64_t* b) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(b)) : "memory");
}
__device__ __forceinline__ bool tc_mbar_try(uint64_t* b, uint32_t ph) {
  uint32_t ok;
  asm volatile("{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n}"
               : "=r"(ok)
               : "r"(smem_u32(b)), "r"(ph)
               : "memory");
  return ok != 0;
}
// shared-memory matrix descriptor: no swizzle, K-major, sm_100 version bit
__device__ __forceinline__ uint64_t tc_desc(uint32_t saddr, uint32_t lbo, uint32_t sbo) {
  return (uint64_t)((saddr >> 4) & 0x3FFFu) | ((uint64_t)((lbo >> 4) & 0x3FFFu) << 16) |
         ((uint64_t)((sbo >> 4) & 0x3FFFu) << 32) | ((uint64_t)1 << 46);
}
// instruction descriptor of kind::f16: BF16 A and B (K-major), FP32 D, M x N
__host__ __device__ constexpr uint32_t tc_idesc(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}
template <int CIN, int COUT>
constexpr size_t tc_conv_smem() {
  return (size_t)27 * CIN * COUT * 2 + 4 * (CIN / 8) * kTcPl * 16 + 64;
}
}  // namespace

template <int CIN, int COUT>
__global__ void __launch_bounds__(128, 1) k_net_conv_tc(const __nv_bfloat16* in, const __nv_bfloat16* wpk,
                                                       const float* bias, __nv_bfloat16* out, int* err) {
  constexpr int VIN = CIN / 8, KS = CIN / 16;
  constexpr int WBYTES = 27 * CIN * COUT * 2;
  constexpr int SLOT = VIN * kTcPl * 16;
  constexpr int NCOL = 4 * COUT <= 32 ? 32 : (4 * COUT <= 64 ? 64 : (4 * COUT <= 128 ? 128 : 256));
  static_assert(CIN % 16 == 0 && COUT % 16 == 0 && 4 * COUT <= 256, "tile shape");
  extern __shared__ __align__(1024) unsigned char tc_sm[];
  unsigned char* slab = tc_sm + WBYTES;
  uint64_t* mbar = reinterpret_cast<uint64_t*>(slab + 4 * SLOT);
  uint32_t* taddr_s = reinterpret_cast<uint32_t*>(mbar + 2);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int b = blockIdx.x;
  const __nv_bfloat16* inb = in + (size_t)b * 4096 * CIN;
  const uint32_t wsa = smem_u32(tc_sm), sla = smem_u32(slab);
  for (int c = tid; c < WBYTES / 16; c += 128)
    cp_async16(tc_sm + c * 16, reinterpret_cast<const char*>(wpk) + c * 16, true);
  auto load_plane = [&](int zi) {
    unsigned char* base = slab + ((zi + 1) & 3) * SLOT;
    for (int e = tid; e < VIN * kTcPl; e += 128) {
      const int cg = e / kTcPl, pp = e % kTcPl, y = pp / 18 - 1, x = pp % 18 - 1;
      const bool ok = zi >= 0 && zi < 16 && y >= 0 && y < 16 && x >= 0 && x < 16;
      const __nv_bfloat16* src = ok ? inb + ((size_t)((zi * 16 + y) * 16 + x) * CIN + cg * 8) : inb;
      cp_async16(base + (cg * kTcPl + pp) * 16, src, ok);
    }
  };
  load_plane(-1);
  load_plane(0);
  cp_async_commit();
  load_plane(1);
  cp_async_commit();
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(taddr_s)),
                 "r"(NCOL));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::);
  }
  if (tid == 0) {
    tc_mbar_init(mbar);
    tc_mbar_init(mbar + 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  const uint32_t tmem = *taddr_s;
  constexpr uint32_t idesc = tc_idesc(128, COUT);
  bool ok = true;
  auto wait_mma = [&](int zz) {
    for (long long s = 0; !tc_mbar_try(mbar + (zz & 1), (uint32_t)((zz >> 1) & 1)); ++s)
      if (s > kTcSpin) {
        ok = false;
        break;
      }
  };
  auto epilogue = [&](int zz) {
    const uint32_t buf = (uint32_t)((zz & 1) * 2 * COUT);
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int m = 32 * warp + lane, y = m >> 3, x = 8 * h + (m & 7);
      __nv_bfloat16* op = out + ((size_t)b * 4096 + (zz * 16 + y) * 16 + x) * COUT;
#pragma unroll
      for (int c0 = 0; c0 < COUT; c0 += 16) {
        uint32_t r[16];
        const uint32_t ta = tmem + ((uint32_t)(32 * warp) << 16) + buf + (uint32_t)(h * COUT + c0);
        asm volatile(
            "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
            : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]),
              "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
            : "r"(ta));
        asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
        uint32_t pk[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          const float v0 = fmaxf(__uint_as_float(r[2 * q]) + bias[c0 + 2 * q], 0.f);
          const float v1 = fmaxf(__uint_as_float(r[2 * q + 1]) + bias[c0 + 2 * q + 1], 0.f);
          __nv_bfloat162 bb = __floats2bfloat162_rn(v0, v1);
          pk[q] = *reinterpret_cast<uint32_t*>(&bb);
        }
        uint4* dst = reinterpret_cast<uint4*>(op + c0);
        dst[0] = make_uint4(pk[0], pk[1], pk[2], pk[3]);
        dst[1] = make_uint4(pk[4], pk[5], pk[6], pk[7]);
      }
    }
  };
  for (int z = 0; z < 16; ++z) {
    cp_async_wait<0>();  // the weights and the planes up to z + 1 have landed
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
    __syncthreads();
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
    if (tid == 0) {
      const uint32_t dbuf = tmem + (uint32_t)((z & 1) * 2 * COUT);
      int cnt = 0;
      for (int t = 0; t < 27; ++t) {
        const int dx = t % 3 - 1, dy = (t / 3) % 3 - 1, dz = t / 9 - 1;
        const uint32_t pbase = sla + (uint32_t)(((z + dz + 1) & 3) * SLOT);
#pragma unroll
        for (int ks = 0; ks < KS; ++ks) {
          const uint64_t bd = tc_desc(wsa + (uint32_t)((t * KS + ks) * 16 * COUT * 2), (COUT / 8) * 128, 128);
#pragma unroll
          for (int h = 0; h < 2; ++h) {
            const uint32_t a0 = pbase + (uint32_t)(((2 * ks) * kTcPl + (1 + dy) * 18 + (1 + dx + 8 * h)) * 16);
            const uint64_t ad = tc_desc(a0, kTcPl * 16, 18 * 16);
            const uint32_t acc = cnt >= 2 ? 1u : 0u;  // each half's first MMA starts from zero
            asm volatile(
                "{\n\t.reg .pred p;\n\tsetp.ne.b32 p, %4, 0;\n\t"
                "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, {%5, %6, %7, %8}, p;\n\t}\n" ::"r"(
                    dbuf + (uint32_t)(h * COUT)),
                "l"(ad), "l"(bd), "r"(idesc), "r"(acc), "r"(0u), "r"(0u), "r"(0u), "r"(0u));
            ++cnt;
          }
        }
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(mbar + (z & 1)))
                   : "memory");
    }
    // plane z + 2 replaces plane z - 2, which the MMAs of plane z - 1 read last
    if (z >= 1) wait_mma(z - 1);
    if (z + 2 <= 16) load_plane(z + 2);
    cp_async_commit();
    if (z >= 1 && ok) {
      asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
      epilogue(z - 1);
    }
  }
  wait_mma(15);
  asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
  if (ok) epilogue(15);
  if (!ok) atomicOr(err, 1);
  asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(NCOL));
}

// W[tap][cin][cout] (BF16) -> [tap][cin/16][2][cout/8][8 n][8 k], the B operand of k_net_conv_tc
__global__ void k_net_pack_tc(int cin, int cout, const __nv_bfloat16* w16, __nv_bfloat16* wpk) {
  const int n = 27 * cin * cout;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const int co = i % cout, ci = (i / cout) % cin, t = i / (cin * cout);
    const int ks = ci / 16, k = ci % 16;
    const size_t blk = (size_t)(t * (cin / 16) + ks) * 16 * cout;
    wpk[blk + ((k / 8) * (cout / 8) + co / 8) * 64 + (co % 8) * 8 + k % 8] = w16[i];
  }
}

// layers k_net_conv_tc takes: 3x3x3 on 16^3 with ReLU, no skip, BF16 output
static bool conv_tc_layer(const NetLayer& L) {
  return L.type == NL_CONV3 && L.s_in == 16 && L.s_out == 16 && L.relu && L.skip < 0 &&
         ((L.cin == 16 && L.cout == 32) || (L.cin == 32 && L.cout == 32));
}

static void conv_tc_launch(const NetLayer& L, const __nv_bfloat16* in, const __nv_bfloat16* wpk, const float* bias,
                           __nv_bfloat16* out, int B, int* err, cudaStream_t st) {
  if (L.cin == 16) {
    constexpr size_t sm = tc_conv_smem<16, 32>();
    cudaFuncSetAttribute(k_net_conv_tc<16, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_net_conv_tc<16, 32><<<B, 128, sm, st>>>(in, wpk, bias, out, err);
  } else {
    constexpr size_t sm = tc_conv_smem<32, 32>();
    cudaFuncSetAttribute(k_net_conv_tc<32, 32>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm);
    k_net_conv_tc<32, 32><<<B, 128, sm, st>>>(in, wpk, bias, out, err);
  }
}

// ---- backward -------------------------------------------------------------------------------
struct DgradArgs {
  int type, cin, cout, s_in, s_out, B;
  const float* dz;                // pre-activation gradient of this layer's output [B][s_out^3][cout]
  const float* wt;                // W[tap][cout][cin] (FP32)
  const __nv_bfloat16* in_act;    // this layer's input activation (ReLU mask), may be null
  const float* add;               // gradient reaching the input through a skip, may be null
  float* din;                     // pre-activation gradient of the previous layer's output
};

__global__ void k_net_dgrad(DgradArgs a) {
  const int si3 = cube(a.s_in), so3 = cube(a.s_out);
  const long long total = (long long)a.B * si3 * a.cin;
  for (long long idx = blockIdx.x * (long long)blockDim.x + threadIdx.x; idx < total;
       idx += (long long)gridDim.x * blockDim.x) {
    const int ci = (int)(idx % a.cin);
    const int i = (int)((idx / a.cin) % si3);
    const int b = (int)(idx / ((long long)a.cin * si3));
    if (a.in_act && !(__bfloat162float(a.in_act[idx]) > 0.f)) {
      a.din[idx] = 0.f;
      continue;
    }
    const int x = i % a.s_in, y = (i / a.s_in) % a.s_in, z = i / (a.s_in * a.s_in);
    float s = 0.f;
    auto tap = [&](int o, int t) {
      const float* dzr = a.dz + ((size_t)b * so3 + o) * a.cout;
      const float* w = a.wt + (size_t)t * a.cout * a.cin + ci;
      for (int co = 0; co < a.cout; ++co) s += dzr[co] * w[(size_t)co * a.cin];
    };
    if (a.type == NL_CONV3) {
      for (int t = 0; t < 27; ++t) {
        const int ox = x - (t % 3 - 1), oy = y - ((t / 3) % 3 - 1), oz = z - (t / 9 - 1);
        if (ox < 0 || oy < 0 || oz < 0 || ox >= a.s_out || oy >= a.s_out || oz >= a.s_out) continue;
        tap((oz * a.s_out + oy) * a.s_out + ox, t);
      }
    } else if (a.type == NL_DOWN2) {
      tap(((z >> 1) * a.s_out + (y >> 1)) * a.s_out + (x >> 1), (x & 1) | ((y & 1) << 1) | ((z & 1) << 2));
    } else if (a.type == NL_CONV1) {
      tap(i, 0);
    } else {
      for (int d = 0; d < 8; ++d) tap(up_vox(i, d, a.s_in), d);
    }
    if (a.add) s += a.add[idx];
    a.din[idx] = s;
  }
}

struct WgradArgs {
  int type, cin, cout, s_in, s_out, B, rows_per_chunk;
  const __nv_bfloat16* in;  // layer input activation
  const float* dz;          // pre-activation gradient of the output
  float* gw;                // [tap][cin][cout], accumulated
};

// dW[t][ci][co] = sum over output rows of in[gather(row, t)][ci] * dz[row][co].
// blockIdx.y = tap, blockIdx.x = chunk of rows; 16 x 16 threads, each TA x TB outputs.
template <int TA, int TB>
__global__ void __launch_bounds__(256) k_net_wgrad(WgradArgs a) {
  constexpr int CIN = 16 * TA, COUT = 16 * TB, RT = 32;
  __shared__ float xs[RT][CIN + 1];
  __shared__ float zs[RT][COUT + 1];
  const int t = blockIdx.y;
  const bool up = a.type == NL_UP2;
  const int so3 = cube(a.s_out), si3 = cube(a.s_in);
  const long long nrows = (long long)a.B * (up ? si3 : so3);
  const long long rbeg = (long long)blockIdx.x * a.rows_per_chunk;
  const long long rend = min(nrows, rbeg + a.rows_per_chunk);
  const int tx = threadIdx.x & 15, ty = threadIdx.x >> 4;
  float acc[TA][TB];
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) acc[i][j] = 0.f;
  for (long long r0 = rbeg; r0 < rend; r0 += RT) {
    for (int e = threadIdx.x; e < RT * CIN; e += 256) {
      const int rr = e / CIN, c = e % CIN;
      const long long row = r0 + rr;
      float v = 0.f;
      if (row < rend) {
        int b, iv;
        if (up) {
          b = (int)(row / si3);
          iv = (int)(row % si3);
        } else {
          b = (int)(row / so3);
          iv = in_vox(a.type, a.s_in, a.s_out, (int)(row % so3), t);
        }
        if (iv >= 0) v = __bfloat162float(a.in[((size_t)b * si3 + iv) * CIN + c]);
      }
      xs[rr][c] = v;
    }
    for (int e = threadIdx.x; e < RT * COUT; e += 256) {
      const int rr = e / COUT, c = e % COUT;
      const long long row = r0 + rr;
      float v = 0.f;
      if (row < rend) {
        int b, o;
        if (up) {
          b = (int)(row / si3);
          o = up_vox((int)(row % si3), t, a.s_in);
        } else {
          b = (int)(row / so3);
          o = (int)(row % so3);
        }
        v = a.dz[((size_t)b * so3 + o) * COUT + c];
      }
      zs[rr][c] = v;
    }
    __syncthreads();
#pragma unroll 4
    for (int rr = 0; rr < RT; ++rr) {
      float xv[TA], zv[TB];
#pragma unroll
      for (int i = 0; i < TA; ++i) xv[i] = xs[rr][ty + 16 * i];
#pragma unroll
      for (int j = 0; j < TB; ++j) zv[j] = zs[rr][tx + 16 * j];
#pragma unroll
      for (int i = 0; i < TA; ++i)
#pragma unroll
        for (int j = 0; j < TB; ++j) acc[i][j] += xv[i] * zv[j];
    }
    __syncthreads();
  }
#pragma unroll
  for (int i = 0; i < TA; ++i)
#pragma unroll
    for (int j = 0; j < TB; ++j) atomicAdd(&a.gw[((size_t)t * CIN + ty + 16 * i) * COUT + tx + 16 * j], acc[i][j]);
}

__global__ void k_net_bgrad(const float* dz, long long rows, int cout, float* gb) {
  __shared__ double red[32];
  const int co = blockIdx.x;
  double s = 0.0;
  for (long long r = threadIdx.x; r < rows; r += blockDim.x) s += dz[r * cout + co];
  s = block_sum(s, red);
  if (threadIdx.x == 0) gb[co] = (float)s;
}

__global__ void k_net_adam(long long n, float* w, const float* g, float* m, float* v, float lr, float b1, float b2,
                           float eps, float wd, float bc1, float bc2) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const float gi = g[i] + wd * w[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    w[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + eps);
  }
}

// BF16 copy W16[t][ci][co] and FP32 transpose Wt[t][co][ci] of the master weights.
__global__ void k_net_refresh(int taps, int cin, int cout, const float* w, __nv_bfloat16* w16, float* wt) {
  const long long n = (long long)taps * cin * cout;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x) {
    const int co = (int)(i % cout), ci = (int)((i / cout) % cin), t = (int)(i / ((long long)cin * cout));
    w16[i] = __float2bfloat16_rn(w[i]);
    wt[((size_t)t * cout + co) * cin + ci] = w[i];
  }
}

// ---- subspace loss ----------------------------------------------------------------------------
constexpr int kLossK = 8;

__global__ void __launch_bounds__(256) k_net_loss(const float* y, const float* V, const float* Mw, int k, int B,
                                                  float* loss, float* dy) {
  __shared__ double red[32];
  __shared__ double G[kLossK * kLossK], H[kLossK * kLossK], C[kLossK * kLossK];
  const int b = blockIdx.x;
  const float* yb = y + (size_t)b * NET_VOX * NET_COUT;
  const float* vb = V + (size_t)b * NET_VOX * k;
  const float* mb = Mw + (size_t)b * NET_VOX;
  // G and H, one entry per pass over the patch (k <= 8: at most 128 passes)
  for (int e = 0; e < 2 * k * k; ++e) {
    const int i = (e % (k * k)) / k, j = e % k;
    const bool g = e < k * k;
    double s = 0.0;
    for (int v = threadIdx.x; v < NET_VOX; v += blockDim.x) {
      const float m = mb[v];
      if (m == 0.f) continue;
      s += (double)m * yb[(size_t)v * NET_COUT + i] * (g ? yb[(size_t)v * NET_COUT + j] : vb[(size_t)v * k + j]);
    }
    s = block_sum(s, red);
    if (threadIdx.x == 0) (g ? G : H)[i * kLossK + j] = s;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    // C = (G + eps I)^-1 H by Cholesky
    double tr = 0.0;
    for (int i = 0; i < k; ++i) tr += G[i * kLossK + i];
    const double eps = 1e-6 * tr / k + 1e-30;
    double L[kLossK * kLossK];
    for (int i = 0; i < k; ++i)
      for (int j = 0; j <= i; ++j) {
        double s = G[i * kLossK + j] + (i == j ? eps : 0.0);
        for (int q = 0; q < j; ++q) s -= L[i * kLossK + q] * L[j * kLossK + q];
        L[i * kLossK + j] = (i == j) ? sqrt(fmax(s, 1e-300)) : s / L[j * kLossK + j];
      }
    for (int c = 0; c < k; ++c) {
      double z[kLossK];
      for (int i = 0; i < k; ++i) {
        double s = H[i * kLossK + c];
        for (int q = 0; q < i; ++q) s -= L[i * kLossK + q] * z[q];
        z[i] = s / L[i * kLossK + i];
      }
      for (int i = k - 1; i >= 0; --i) {
        double s = z[i];
        for (int q = i + 1; q < k; ++q) s -= L[q * kLossK + i] * C[q * kLossK + c];
        C[i * kLossK + c] = s / L[i * kLossK + i];
      }
    }
  }
  __syncthreads();
  const float scale = -2.f / (float)(B * k);
  double lacc = 0.0;
  for (int v = threadIdx.x; v < NET_VOX; v += blockDim.x) {
    const float m = mb[v];
    float r[kLossK];
    for (int j = 0; j < k; ++j) {
      double p = 0.0;
      for (int i = 0; i < k; ++i) p += (double)yb[(size_t)v * NET_COUT + i] * C[i * kLossK + j];
      r[j] = vb[(size_t)v * k + j] - (float)p;
      lacc += (double)m * r[j] * r[j];
    }
    float* d = dy + ((size_t)b * NET_VOX + v) * NET_COUT;
    for (int i = 0; i < NET_COUT; ++i) {
      float s = 0.f;
      if (i < k)
        for (int j = 0; j < k; ++j) s += r[j] * (float)C[i * kLossK + j];
      d[i] = scale * m * s;
    }
  }
  lacc = block_sum(lacc, red);
  if (threadIdx.x == 0) loss[b] = (float)(lacc / k);
}

// ---- patches -------------------------------------------------------------------------------------
__global__ void k_net_features(Grid g, const SubInfo* subs, const double* kx, const double* ky, const double* kz,
                               int dmask, __nv_bfloat16* feats) {
  __shared__ double red[32];
  const SubInfo S = subs[blockIdx.x];
  const int nc = S.nx * S.ny * S.nz;
  double s = 0.0;
  for (int cl = threadIdx.x; cl < nc; cl += blockDim.x) {
    const int i = cl % S.nx, j = (cl / S.nx) % S.ny, q = cl / (S.nx * S.ny);
    const long long cg = ((long long)(S.z0 + q) * g.N + (S.y0 + j)) * g.M + (S.x0 + i);
    s += log(kx[cg]) + log(ky[cg]) + log(kz[cg]);
  }
  const double mean = block_sum(s, red) / (3.0 * nc);
  for (int v = threadIdx.x; v < NET_VOX; v += blockDim.x) {
    const int x = v % NET_S, y = (v / NET_S) % NET_S, z = v / (NET_S * NET_S);
    float f[NET_CIN];
#pragma unroll
    for (int c = 0; c < NET_CIN; ++c) f[c] = 0.f;
    if (x < S.nx && y < S.ny && z < S.nz) {
      const int ex = S.x0 + x, ey = S.y0 + y, ez = S.z0 + z;
      const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
      f[0] = (float)((log(kx[cg]) - mean) * 0.25);
      f[1] = (float)((log(ky[cg]) - mean) * 0.25);
      f[2] = (float)((log(kz[cg]) - mean) * 0.25);
      const bool dir = ((dmask & 1) && ex == 0) || ((dmask & 2) && ex == g.M - 1) || ((dmask & 4) && ey == 0) ||
                       ((dmask & 8) && ey == g.N - 1) || ((dmask & 16) && ez == 0) || ((dmask & 32) && ez == g.P - 1);
      f[3] = dir ? 1.f : 0.f;
      f[4] = 1.f;
    }
    __nv_bfloat16* o = feats + ((size_t)blockIdx.x * NET_VOX + v) * NET_CIN;
#pragma unroll
    for (int c = 0; c < NET_CIN; c += 2)
      *reinterpret_cast<__nv_bfloat162*>(o + c) = __floats2bfloat162_rn(f[c], f[c + 1]);
  }
}

__device__ __forceinline__ double harm(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

// Mass diagonal of the local eigenproblem (src/PreMixFEM_3D.c:243-346), the same
// expression, term for term, as the batched eigensolver's.
__global__ void k_net_targets(NetTargetArgs a) {
  const SubInfo S = a.subs[blockIdx.x];
  const Grid g = a.g;
  for (int v = threadIdx.x; v < NET_VOX; v += blockDim.x) {
    const int i = v % NET_S, j = (v / NET_S) % NET_S, kk = v / (NET_S * NET_S);
    float* Vo = a.V + ((size_t)blockIdx.x * NET_VOX + v) * a.k;
    if (!(i < S.nx && j < S.ny && kk < S.nz)) {
      for (int c = 0; c < a.k; ++c) Vo[c] = 0.f;
      a.Mw[(size_t)blockIdx.x * NET_VOX + v] = 0.f;
      continue;
    }
    const int nx = S.nx, ny = S.ny, nz = S.nz;
    const int ex = S.x0 + i, ey = S.y0 + j, ez = S.z0 + kk;
    const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
    double mv;
    if (a.eg_op == 1) {
      mv = a.kx[cg] + a.ky[cg] + a.kz[cg];
    } else if (a.eg_op == 2) {
      double dn = a.db[cg];
      if (i > 0) dn += a.tx[cg];
      if (i < nx - 1) dn += a.tx[cg + 1];
      if (j > 0) dn += a.ty[cg];
      if (j < ny - 1) dn += a.ty[cg + g.M];
      if (kk > 0) dn += a.tz[cg];
      if (kk < nz - 1) dn += a.tz[cg + g.MN];
      mv = dn;
    } else {
      mv = 0.0;
      if (i == 0 && ex >= 1) mv += 2.0 * harm(a.kx[cg - 1], a.kx[cg]) / a.Hx / a.Hx;
      if (ex + 1 != g.M) mv += 2.0 * harm(a.kx[cg], a.kx[cg + 1]) / a.Hx / a.Hx;
      if (ey >= 1) mv += 2.0 * harm(a.ky[cg - g.M], a.ky[cg]) / a.Hy / a.Hy;
      if (ey + 1 != g.N) mv += 2.0 * harm(a.ky[cg], a.ky[cg + g.M]) / a.Hy / a.Hy;
      if (ez >= 1) mv += 2.0 * harm(a.kz[cg - g.MN], a.kz[cg]) / a.Hz / a.Hz;
      if (ez + 1 != g.P) mv += 2.0 * harm(a.kz[cg], a.kz[cg + g.MN]) / a.Hz / a.Hz;
      if (i + 1 < nx) mv += 2.0 * harm(a.kx[cg], a.kx[cg + 1]) / a.Hx / a.Hx;
      const int dm = a.dirichlet_mask;
      if (dm & 1 && ex == 0) mv += 2.0 * (2.0 * a.kx[cg]) / a.Hx / a.Hx;
      if (dm & 2 && ex == g.M - 1) mv += 2.0 * (2.0 * a.kx[cg]) / a.Hx / a.Hx;
      if (dm & 4 && ey == 0) mv += 2.0 * (2.0 * a.ky[cg]) / a.Hy / a.Hy;
      if (dm & 8 && ey == g.N - 1) mv += 2.0 * (2.0 * a.ky[cg]) / a.Hy / a.Hy;
      if (dm & 16 && ez == 0) mv += 2.0 * (2.0 * a.kz[cg]) / a.Hz / a.Hz;
      if (dm & 32 && ez == g.P - 1) mv += 2.0 * (2.0 * a.kz[cg]) / a.Hz / a.Hz;
      mv *= a.meas;
    }
    a.Mw[(size_t)blockIdx.x * NET_VOX + v] = (float)mv;
    for (int c = 0; c < a.k; ++c)
      Vo[c] = a.phi_f32 ? reinterpret_cast<const float*>(a.phi)[cg * a.kmax + c]
                        : (float)reinterpret_cast<const double*>(a.phi)[cg * a.kmax + c];
  }
}

// Subdomains whose eigensolve did not converge (status 1), in index order.
__global__ void k_failed_list(const int* status, int nsub, int* list, int* count) {
  if (threadIdx.x != 0) return;
  int c = 0;
  for (int s = 0; s < nsub; ++s)
    if (status[s] == 1) list[c++] = s;
  *count = c;
}

}  // namespace

void launch_net_targets(const NetTargetArgs& a, cudaStream_t st) {
  { note_launch(); k_net_targets<<<a.nsub, 256, 0, st>>>(a); }
}

void launch_failed_list(const int* status, int nsub, int* list, int* count, cudaStream_t st) {
  { note_launch(); k_failed_list<<<1, 32, 0, st>>>(status, nsub, list, count); }
}

void launch_net_features(const Grid& g, const SubInfo* subs, int nsub, const double* kx, const double* ky,
                         const double* kz, int dirichlet_mask, __nv_bfloat16* feats, cudaStream_t st) {
  { note_launch(); k_net_features<<<nsub, 256, 0, st>>>(g, subs, kx, ky, kz, dirichlet_mask, feats); }
}

void launch_net_loss(const float* y, const float* V, const float* Mw, int B, int k, float* loss, float* dy,
                     cudaStream_t st) {
  { note_launch(); k_net_loss<<<B, 256, 0, st>>>(y, V, Mw, k, B, loss, dy); }
}

// ---- host side ---------------------------------------------------------------------------------
static size_t wcount(const NetLayer& L) { return (size_t)net_taps(L.type) * L.cin * L.cout; }
static size_t act_elems(int a) { return (size_t)kNetActs[a].s * kNetActs[a].s * kNetActs[a].s * kNetActs[a].c; }

Net::Net() {}

Net::~Net() {
  for (int l = 0; l < NET_LAYERS; ++l) {
    void* p[] = {w32_[l], b32_[l], w16_[l], wt_[l], wtc_[l], gw_[l], gb_[l], mw_[l], vw_[l], mb_[l], vb_[l]};
    for (void* q : p)
      if (q) cudaFree(q);
  }
  for (int a = 0; a < NET_ACTS; ++a) {
    if (a > 0 && act_[a]) cudaFree(act_[a]);
    if (dact_[a]) cudaFree(dact_[a]);
  }
  if (d_err_) cudaFree(d_err_);
}

int Net::take_error() {
  if (!d_err_) return 0;
  int f = 0;
  if (cudaMemcpy(&f, d_err_, sizeof(int), cudaMemcpyDeviceToHost) != cudaSuccess) {
    err = "reading the network's kernel flag failed";
    return 76;
  }
  if (!f) return 0;
  cudaMemset(d_err_, 0, sizeof(int));
  err = "a tensor-core convolution's wait for its MMAs ran out";
  return 76;
}

int Net::params() const {
  int n = 0;
  for (const NetLayer& L : kNetLayers) n += (int)wcount(L) + L.cout;
  return n;
}

int Net::alloc_params() {
  if (w32_[0]) return 0;
  for (int l = 0; l < NET_LAYERS; ++l) {
    const size_t nw = wcount(kNetLayers[l]), nb = kNetLayers[l].cout;
    bool ok = cudaMalloc(&w32_[l], nw * 4) == cudaSuccess && cudaMalloc(&b32_[l], nb * 4) == cudaSuccess &&
              cudaMalloc(&w16_[l], nw * 2) == cudaSuccess && cudaMalloc(&wt_[l], nw * 4) == cudaSuccess &&
              cudaMalloc(&gw_[l], nw * 4) == cudaSuccess && cudaMalloc(&gb_[l], nb * 4) == cudaSuccess &&
              cudaMalloc(&mw_[l], nw * 4) == cudaSuccess && cudaMalloc(&vw_[l], nw * 4) == cudaSuccess &&
              cudaMalloc(&mb_[l], nb * 4) == cudaSuccess && cudaMalloc(&vb_[l], nb * 4) == cudaSuccess;
    if (ok && conv_tc_layer(kNetLayers[l])) ok = cudaMalloc(&wtc_[l], nw * 2) == cudaSuccess;
    if (!ok) {
      err = "cudaMalloc of the network parameters failed";
      return 76;
    }
    cudaMemset(mw_[l], 0, nw * 4);
    cudaMemset(vw_[l], 0, nw * 4);
    cudaMemset(mb_[l], 0, nb * 4);
    cudaMemset(vb_[l], 0, nb * 4);
  }
  if (cudaMalloc(&d_err_, sizeof(int)) != cudaSuccess) {
    err = "cudaMalloc of the network parameters failed";
    return 76;
  }
  cudaMemset(d_err_, 0, sizeof(int));
  return 0;
}

void Net::refresh(int l, cudaStream_t st) {
  const NetLayer& L = kNetLayers[l];
  const long long n = (long long)wcount(L);
  { note_launch(); k_net_refresh<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(net_taps(L.type), L.cin, L.cout, w32_[l], w16_[l], wt_[l]); }
  if (wtc_[l]) { note_launch(); k_net_pack_tc<<<(int)std::min<long long>((n + 255) / 256, 4096), 256, 0, st>>>(L.cin, L.cout, w16_[l], wtc_[l]); }
}

int Net::set_weights(int l, const float* w, const float* b) {
  if (l < 0 || l >= NET_LAYERS) {
    err = "layer index out of range";
    return 62;
  }
  if (int e = alloc_params()) return e;
  const NetLayer& L = kNetLayers[l];
  if (w) cudaMemcpy(w32_[l], w, wcount(L) * 4, cudaMemcpyHostToDevice);
  if (b) cudaMemcpy(b32_[l], b, L.cout * 4, cudaMemcpyHostToDevice);
  refresh(l, 0);
  if (cudaDeviceSynchronize() != cudaSuccess) {
    err = "set_weights failed";
    return 76;
  }
  return 0;
}

int Net::get_weights(int l, float* w, float* b) const {
  if (l < 0 || l >= NET_LAYERS || !w32_[l]) return 62;
  if (w) cudaMemcpy(w, w32_[l], wcount(kNetLayers[l]) * 4, cudaMemcpyDeviceToHost);
  if (b) cudaMemcpy(b, b32_[l], kNetLayers[l].cout * 4, cudaMemcpyDeviceToHost);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 76;
}

int Net::get_grads(int l, float* gw, float* gb) const {
  if (l < 0 || l >= NET_LAYERS || !gw_[l]) return 62;
  if (gw) cudaMemcpy(gw, gw_[l], wcount(kNetLayers[l]) * 4, cudaMemcpyDeviceToHost);
  if (gb) cudaMemcpy(gb, gb_[l], kNetLayers[l].cout * 4, cudaMemcpyDeviceToHost);
  return cudaDeviceSynchronize() == cudaSuccess ? 0 : 76;
}

int Net::init(unsigned long long seed) {
  if (int e = alloc_params()) return e;
  std::mt19937_64 rng(seed);
  for (int l = 0; l < NET_LAYERS; ++l) {
    const NetLayer& L = kNetLayers[l];
    const int fan_in = (L.type == NL_UP2 ? 1 : net_taps(L.type)) * (l == 0 ? 5 : L.cin);
    std::normal_distribution<float> nd(0.f, std::sqrt((L.relu ? 2.f : 1.f) / fan_in));
    std::vector<float> w(wcount(L)), b(L.cout, 0.f);
    for (auto& x : w) x = nd(rng);
    if (int e = set_weights(l, w.data(), b.data())) return e;
  }
  step_ = 0;
  return 0;
}

static const char kMagic[8] = {'P', 'M', 'F', 'N', 'E', 'T', '0', '1'};

int Net::save(const char* path) const {
  FILE* f = fopen(path, "wb");
  if (!f) return 62;
  fwrite(kMagic, 1, 8, f);
  const int hdr[2] = {1, NET_LAYERS};
  fwrite(hdr, 4, 2, f);
  for (int l = 0; l < NET_LAYERS; ++l) {
    const NetLayer& L = kNetLayers[l];
    const int d[4] = {L.type, L.cin, L.cout, net_taps(L.type)};
    fwrite(d, 4, 4, f);
    std::vector<__nv_bfloat16> w(wcount(L));
    std::vector<float> b(L.cout);
    cudaMemcpy(w.data(), w16_[l], w.size() * 2, cudaMemcpyDeviceToHost);
    cudaMemcpy(b.data(), b32_[l], b.size() * 4, cudaMemcpyDeviceToHost);
    fwrite(w.data(), 2, w.size(), f);
    fwrite(b.data(), 4, b.size(), f);
  }
  const bool ok = fclose(f) == 0;
  return ok ? 0 : 76;
}

int Net::load(const char* path) {
  FILE* f = fopen(path, "rb");
  if (!f) {
    err = std::string("cannot open network weights ") + path;
    return 62;
  }
  auto fail = [&](const char* why) {
    fclose(f);
    err = std::string(path) + ": " + why;
    return 62;
  };
  char mg[8];
  int hdr[2];
  if (fread(mg, 1, 8, f) != 8 || memcmp(mg, kMagic, 8) != 0) return fail("not a weight file");
  if (fread(hdr, 4, 2, f) != 2 || hdr[0] != 1 || hdr[1] != NET_LAYERS) return fail("unsupported version or layout");
  if (int e = alloc_params()) {
    fclose(f);
    return e;
  }
  for (int l = 0; l < NET_LAYERS; ++l) {
    const NetLayer& L = kNetLayers[l];
    int d[4];
    if (fread(d, 4, 4, f) != 4 || d[0] != L.type || d[1] != L.cin || d[2] != L.cout || d[3] != net_taps(L.type))
      return fail("layer shapes differ from this build's network");
    std::vector<__nv_bfloat16> w(wcount(L));
    std::vector<float> w32(w.size()), b(L.cout);
    if (fread(w.data(), 2, w.size(), f) != w.size() || fread(b.data(), 4, b.size(), f) != b.size())
      return fail("truncated");
    for (size_t i = 0; i < w.size(); ++i) w32[i] = __bfloat162float(w[i]);
    if (int e = set_weights(l, w32.data(), b.data())) {
      fclose(f);
      return e;
    }
  }
  fclose(f);
  return 0;
}

int Net::ensure(int B) {
  if (B <= cap_) return 0;
  for (int a = 1; a < NET_ACTS; ++a) {
    if (act_[a]) cudaFree(act_[a]);
    if (dact_[a]) cudaFree(dact_[a]);
    act_[a] = nullptr;
    dact_[a] = nullptr;
  }
  for (int a = 1; a < NET_ACTS - 1; ++a)
    if (cudaMalloc(&act_[a], act_elems(a) * B * 2) != cudaSuccess) {
      err = "cudaMalloc of the network activations failed";
      cap_ = 0;
      return 76;
    }
  cap_ = B;
  return 0;
}

// One forward layer with ROWS-row tiles and MT 16-row m-tiles per warp.
template <int NT, int ROWS, int MT>
static bool fwd_launch_t(const FwdArgs& a, long long rows, cudaStream_t st) {
  const size_t smem = (2 * (size_t)ROWS * (a.cin + 8) + 2 * (size_t)a.cin * (a.cout + 8)) * 2;
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_net_fwd<NT, ROWS, MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  k_net_fwd<NT, ROWS, MT><<<(int)(rows / ROWS), ROWS * 2 / MT, smem, st>>>(a);
  return true;
}

template <int NT>
static bool fwd_launch_nt(int R, int MT, const FwdArgs& a, long long rows, cudaStream_t st) {
  if (R == 256 && MT == 2) return fwd_launch_t<NT, 256, 2>(a, rows, st);
  if (R == 128 && MT == 1) return fwd_launch_t<NT, 128, 1>(a, rows, st);
  if (R == 128 && MT == 2) return fwd_launch_t<NT, 128, 2>(a, rows, st);
  if (R == 64 && MT == 1) return fwd_launch_t<NT, 64, 1>(a, rows, st);
  return false;
}

static bool fwd_launch(int ntv, int R, int MT, const FwdArgs& a, long long rows, cudaStream_t st) {
  switch (ntv) {
    case 2: return fwd_launch_nt<2>(R, MT, a, rows, st);
    case 4: return fwd_launch_nt<4>(R, MT, a, rows, st);
    case 8: return fwd_launch_nt<8>(R, MT, a, rows, st);
    case 12: return fwd_launch_nt<12>(R, MT, a, rows, st);
  }
  return false;
}

int Net::forward(const __nv_bfloat16* x, int B, float* y, bool keep, cudaStream_t st) {
  if (!w32_[0]) {
    err = "network weights not initialised or loaded";
    return 73;
  }
  if (int e = ensure(B)) return e;
  x_ = x;
  for (int l = 0; l < NET_LAYERS; ++l) {
    const NetLayer& L = kNetLayers[l];
    FwdArgs a;
    a.type = L.type;
    a.cin = L.cin;
    a.cout = L.cout;
    a.s_in = L.s_in;
    a.s_out = L.s_out;
    a.relu = L.relu;
    a.in = L.in_act == 0 ? x : act_[L.in_act];
    a.W = w16_[l];
    a.bias = b32_[l];
    a.skip = L.skip >= 0 ? act_[L.skip] : nullptr;
    a.out = L.out_act == NET_ACTS - 1 ? nullptr : act_[L.out_act];
    a.outf = L.out_act == NET_ACTS - 1 ? y : nullptr;
    const long long rows = (long long)B * L.s_out * L.s_out * L.s_out;
    // tiles stay inside one sample (and one parity class for up2); candidate 0
    // is the built-in choice, the tuner may pick another for this layer and batch
    const int per = L.type == NL_UP2 ? L.s_in * L.s_in * L.s_in : L.s_out * L.s_out * L.s_out;
    static const int kTiles[4][2] = {{256, 2}, {128, 1}, {128, 2}, {64, 1}};
    int cand[5], nc = 0;
    const int def = per % 256 == 0 ? 0 : 3;
    cand[nc++] = def;
    for (int t = 0; t < 4; ++t)
      if (t != def && per % kTiles[t][0] == 0) cand[nc++] = t;
    const int ntv = L.cout / 8;
    if (ntv != 2 && ntv != 4 && ntv != 8 && ntv != 12) {
      err = "unsupported layer width";
      return 56;
    }
    // the tensor-core convolution (candidate index 4) where the layer fits it
    const bool tc = wtc_[l] && conv_tc_layer(L) && !a.outf;
    if (tc) cand[nc++] = 4;
    auto launch = [&](int c) -> bool {
      if (cand[c] == 4) {
        conv_tc_launch(L, a.in, wtc_[l], a.bias, a.out, B, d_err_, st);
        return true;
      }
      return fwd_launch(ntv, kTiles[cand[c]][0], kTiles[cand[c]][1], a, rows, st);
    };
    char key[96];
    snprintf(key, sizeof(key), tc ? "net_fwd|L%d|B%d|tc" : "net_fwd|L%d|B%d", l, B);
    const int c = tune_choose(key, nc, launch, st);
    note_launch();
    launch(c);
  }
  (void)keep;
  return 0;
}

int Net::backward(const float* dy, int B, cudaStream_t st) {
  if (B > cap_ || !x_) {
    err = "backward needs the activations of a forward pass of the same batch";
    return 73;
  }
  for (int a = 1; a < NET_ACTS - 1; ++a)
    if (!dact_[a] && cudaMalloc(&dact_[a], act_elems(a) * cap_ * 4) != cudaSuccess) {
      err = "cudaMalloc of the network gradients failed";
      return 76;
    }
  // dpre[l]: pre-activation gradient of layer l's output; layer 8's is dy.
  auto dpre = [&](int l) -> float* {
    return l == NET_LAYERS - 1 ? const_cast<float*>(dy) : dact_[kNetLayers[l].out_act];
  };
  for (int l = NET_LAYERS - 1; l >= 0; --l) {
    const NetLayer& L = kNetLayers[l];
    const __nv_bfloat16* in = L.in_act == 0 ? x_ : act_[L.in_act];
    cudaMemsetAsync(gw_[l], 0, wcount(L) * 4, st);
    // weight gradient
    WgradArgs w;
    w.type = L.type;
    w.cin = L.cin;
    w.cout = L.cout;
    w.s_in = L.s_in;
    w.s_out = L.s_out;
    w.B = B;
    w.rows_per_chunk = 2048;
    w.in = in;
    w.dz = dpre(l);
    w.gw = gw_[l];
    const long long rows = (long long)B * (L.type == NL_UP2 ? L.s_in * L.s_in * L.s_in : L.s_out * L.s_out * L.s_out);
    dim3 grid((unsigned)((rows + w.rows_per_chunk - 1) / w.rows_per_chunk), net_taps(L.type));
    const int ta = L.cin / 16, tb = L.cout / 16;
    note_launch();
    if (ta == 1 && tb == 2) k_net_wgrad<1, 2><<<grid, 256, 0, st>>>(w);
    else if (ta == 2 && tb == 4) k_net_wgrad<2, 4><<<grid, 256, 0, st>>>(w);
    else if (ta == 4 && tb == 4) k_net_wgrad<4, 4><<<grid, 256, 0, st>>>(w);
    else if (ta == 4 && tb == 6) k_net_wgrad<4, 6><<<grid, 256, 0, st>>>(w);
    else if (ta == 6 && tb == 6) k_net_wgrad<6, 6><<<grid, 256, 0, st>>>(w);
    else if (ta == 6 && tb == 4) k_net_wgrad<6, 4><<<grid, 256, 0, st>>>(w);
    else if (ta == 4 && tb == 2) k_net_wgrad<4, 2><<<grid, 256, 0, st>>>(w);
    else if (ta == 2 && tb == 2) k_net_wgrad<2, 2><<<grid, 256, 0, st>>>(w);
    else if (ta == 2 && tb == 1) k_net_wgrad<2, 1><<<grid, 256, 0, st>>>(w);
    else {
      err = "unsupported layer shape in backward";
      return 56;
    }
    const long long orows = (long long)B * L.s_out * L.s_out * L.s_out;
    { note_launch(); k_net_bgrad<<<L.cout, 256, 0, st>>>(dpre(l), orows, L.cout, gb_[l]); }
    if (l == 0) break;
    // gradient reaching the input activation, masked by its ReLU, plus skip gradients
    DgradArgs d;
    d.type = L.type;
    d.cin = L.cin;
    d.cout = L.cout;
    d.s_in = L.s_in;
    d.s_out = L.s_out;
    d.B = B;
    d.dz = dpre(l);
    d.wt = wt_[l];
    d.in_act = in;
    d.add = nullptr;
    for (int j = 0; j < NET_LAYERS; ++j)
      if (kNetLayers[j].skip == L.in_act) d.add = dpre(j);
    d.din = dact_[L.in_act];
    const long long tot = (long long)B * L.s_in * L.s_in * L.s_in * L.cin;
    { note_launch(); k_net_dgrad<<<(int)std::min<long long>((tot + 255) / 256, 1 << 20), 256, 0, st>>>(d); }
  }
  return 0;
}

void Net::adam(float lr, float b1, float b2, float eps, float wd, cudaStream_t st) {
  ++step_;
  const float bc1 = 1.f - powf(b1, (float)step_), bc2 = 1.f - powf(b2, (float)step_);
  for (int l = 0; l < NET_LAYERS; ++l) {
    const NetLayer& L = kNetLayers[l];
    const long long nw = (long long)wcount(L);
    { note_launch(); k_net_adam<<<(int)std::min<long long>((nw + 255) / 256, 4096), 256, 0, st>>>(nw, w32_[l], gw_[l], mw_[l], vw_[l], lr, b1, b2, eps, wd, bc1, bc2); }
    { note_launch(); k_net_adam<<<1, 256, 0, st>>>(L.cout, b32_[l], gb_[l], mb_[l], vb_[l], lr, b1, b2, eps, 0.f, bc1, bc2); }
    refresh(l, st);
  }
}

}  // namespace pmf
