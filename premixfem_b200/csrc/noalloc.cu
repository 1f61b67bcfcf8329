// pmf_residual_noalloc: r = b - A x and ||r||_2 for device vectors, with no
// memory allocation of any kind on the call path.
//
// Why it exists.  Every other entry point may allocate: pmf_apply_A and
// pmf_solve stage host vectors through solver-owned device buffers, and the
// reductions inside pmf_solve write per-block partial sums to cudaMalloc'd
// scratch.  Some callers cannot allow an allocation at the point where they
// need a residual:
//   * a caller whose device memory is fully reserved by its own pool (a
//     framework's caching allocator, or a solver service that pre-sizes all
//     memory at start-up), where cudaMalloc would fail or evict;
//   * a latency-critical loop (a convergence monitor called every Krylov
//     iteration) where cudaMalloc/cudaFree would synchronise the device;
//   * code that records a fixed sequence of launches for later replay and
//     must not see a new allocation appear between recordings.
// For these, the reduction scratch lives in a file-scope __device__ array in
// this translation unit, and the call only launches one kernel.
//
// Limits and rules (also in include/pmf_b200.h):
//   * the mesh may hold at most PMF_NOALLOC_MAX_CELLS cells (one block of
//     256 threads reduces 2048 cells; PMF_NOALLOC_MAX_BLOCKS partial sums fit
//     the scratch), larger meshes are rejected with error 62;
//   * the first call on each device resolves the scratch address with
//     cudaGetSymbolAddress (which may load this module and reserve its static
//     memory) and zeroes the ticket counter; make that first call, on every
//     device used, before any stream capture begins;
//   * the ticket counter must be zero when a call starts: it is zero when
//     the module loads, the first call on each device zeroes it again, and
//     every completed call returns it to zero.  The partial sums
//     need no initial value (each block writes its own slot first);
//   * calls on the same device share the scratch, so two calls that overlap
//     in time (different streams, different host threads, or the same solver
//     from two threads) race and give wrong results: serialise them, e.g. on
//     one stream.
#include <cuda_runtime.h>

#include <mutex>

#include "pmf_b200.h"
#include "pmf_common.cuh"
#include "pmf_kernels.h"
#include "solver.h"

namespace {

constexpr int kThreads = 256;
constexpr int kCellsPerThread = 8;
constexpr int kCellsPerBlock = kThreads * kCellsPerThread;  // 2048
constexpr int kMaxDevices = 64;

static_assert(PMF_NOALLOC_MAX_CELLS == (long long)PMF_NOALLOC_MAX_BLOCKS * kCellsPerBlock,
              "cell limit must match the scratch size");

struct NoAllocScratch {
  double partial[PMF_NOALLOC_MAX_BLOCKS];  // one FP64 partial sum per block (128 KiB)
  unsigned int ticket;                     // blocks finished in the current call; zero between calls
};

static __device__ __align__(256) NoAllocScratch g_noalloc_scratch;

// The same 7-point product, term for term, as the solver's y = A x.
__device__ __forceinline__ double stencil(const pmf::Grid& g, long long c, int ex, int ey, int ez, const double* tx,
                                          const double* ty, const double* tz, const double* diag, const double* x) {
  double v = diag[c] * x[c];
  if (ex > 0) v -= tx[c] * x[c - 1];
  if (ex < g.M - 1) v -= tx[c + 1] * x[c + 1];
  if (ey > 0) v -= ty[c] * x[c - g.M];
  if (ey < g.N - 1) v -= ty[c + g.M] * x[c + g.M];
  if (ez > 0) v -= tz[c] * x[c - g.MN];
  if (ez < g.P - 1) v -= tz[c + g.MN] * x[c + g.MN];
  return v;
}

// One launch: each block forms r on its 2048 cells and writes the sum of r^2
// to its slot; the last block to finish (by ticket) adds the slots in a fixed
// order, so the norm is deterministic for a given mesh size, and resets the
// ticket to zero.  No thread waits on another block.
__global__ void __launch_bounds__(kThreads) k_residual_noalloc(pmf::Grid g, const double* tx, const double* ty,
                                                               const double* tz, const double* diag,
                                                               const double* b, const double* x, double* r,
                                                               double* rnorm, NoAllocScratch* sc) {
  __shared__ double red[32];
  __shared__ bool last;
  const long long base = (long long)blockIdx.x * kCellsPerBlock;
  double v = 0.0;
#pragma unroll
  for (int i = 0; i < kCellsPerThread; ++i) {
    const long long c = base + i * kThreads + threadIdx.x;
    if (c < g.ncell) {
      const int ex = (int)(c % g.M);
      const int ey = (int)((c / g.M) % g.N);
      const int ez = (int)(c / g.MN);
      const double ri = b[c] - stencil(g, c, ex, ey, ez, tx, ty, tz, diag, x);
      r[c] = ri;
      v += ri * ri;
    }
  }
  v = pmf::block_sum(v, red);
  if (threadIdx.x == 0) {
    sc->partial[blockIdx.x] = v;
    __threadfence();
    const unsigned int t = atomicAdd(&sc->ticket, 1u);
    last = (t == gridDim.x - 1);
  }
  __syncthreads();
  if (!last) return;
  __threadfence();
  double s = 0.0;
  for (int i = threadIdx.x; i < (int)gridDim.x; i += kThreads) s += __ldcg(&sc->partial[i]);
  s = pmf::block_sum(s, red);
  if (threadIdx.x == 0) {
    *rnorm = sqrt(s);
    sc->ticket = 0u;
  }
}

std::mutex g_setup_mutex;
NoAllocScratch* g_scratch_ptr[kMaxDevices] = {nullptr};

// Once per device, with that device current.
int scratch_for_device(int dev, NoAllocScratch** out, const char** why) {
  if (dev < 0 || dev >= kMaxDevices) {
    *why = "device ordinal beyond the supported range";
    return 62;
  }
  std::lock_guard<std::mutex> lock(g_setup_mutex);
  if (!g_scratch_ptr[dev]) {
    void* p = nullptr;
    cudaError_t rc = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (rc != cudaSuccess || !p) {
      *why = rc != cudaSuccess ? cudaGetErrorString(rc) : "cudaGetSymbolAddress returned null";
      return 76;
    }
    NoAllocScratch* sc = (NoAllocScratch*)p;
    rc = cudaMemset(&sc->ticket, 0, sizeof(unsigned int));
    if (rc == cudaSuccess) rc = cudaDeviceSynchronize();
    if (rc != cudaSuccess) {
      *why = cudaGetErrorString(rc);
      return 76;
    }
    g_scratch_ptr[dev] = sc;
  }
  *out = g_scratch_ptr[dev];
  return 0;
}

}  // namespace

// handle access and error reporting shared with the other entry points (capi.cu)
pmf::Solver* pmf_internal_solver(pmf_solver* h);
int pmf_internal_fail(int code, const char* msg);

extern "C" int pmf_residual_noalloc(pmf_solver* s, const double* b, const double* x, double* r, double* rnorm,
                                    void* stream) {
  pmf::Solver* sv = pmf_internal_solver(s);
  if (!sv) return pmf_internal_fail(62, "null solver handle");
  if (sv->g.ncell > PMF_NOALLOC_MAX_CELLS)
    return pmf_internal_fail(62, "pmf_residual_noalloc: the mesh has more cells than PMF_NOALLOC_MAX_CELLS "
                                 "(33554432); use pmf_apply_A for larger meshes");
  if (!b || !x || !r || !rnorm) return pmf_internal_fail(62, "pmf_residual_noalloc: null vector");
  if (!sv->tx) return pmf_internal_fail(73, "pmf_residual_noalloc: operator not assembled (call pmf_setup)");
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess) return pmf_internal_fail(76, "pmf_residual_noalloc: cudaGetDevice failed");
  cudaPointerAttributes attr;
  if (cudaPointerGetAttributes(&attr, sv->tx) != cudaSuccess || attr.device != dev)
    return pmf_internal_fail(62, "pmf_residual_noalloc: the current device is not the solver's device");
  NoAllocScratch* sc = nullptr;
  const char* why = nullptr;
  if (int e = scratch_for_device(dev, &sc, &why)) return pmf_internal_fail(e, why);
  const int nblocks = (int)((sv->g.ncell + kCellsPerBlock - 1) / kCellsPerBlock);
  pmf::note_launch();
  k_residual_noalloc<<<nblocks, kThreads, 0, (cudaStream_t)stream>>>(sv->g, sv->tx, sv->ty, sv->tz, sv->diag, b, x, r,
                                                                     rnorm, sc);
  const cudaError_t rc = cudaGetLastError();
  if (rc != cudaSuccess) return pmf_internal_fail(76, cudaGetErrorString(rc));
  return 0;
}
