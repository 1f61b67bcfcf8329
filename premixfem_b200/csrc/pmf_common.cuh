// Shared definitions for the B200 PreMixFEM kernels.
//
// Grid layout: a mesh of M x N x P cells, natural order, x fastest:
//   cell id c = (ez * N + ey) * M + ex.
// Face transmissibilities are stored per cell for the cell's lower face in each
// direction: tx[c] couples (ex-1, ex), ty[c] couples (ey-1, ey), tz[c] couples
// (ez-1, ez); they are zero on the domain boundary.  diag[c] is the full
// diagonal of A (the six face terms plus any Dirichlet boundary term).
//
// Subdomains are axis-aligned boxes, grouped into "virtual ranks" exactly as
// the reference splits a DMDA box per MPI rank (src/PreMixFEM_3D.c:47-78).
// Coarse (level-2) degrees of freedom are padded to kmax per subdomain:
// coarse index = s * kmax + j.  Columns j >= k_s of a subdomain's basis are
// zero and the padded coarse rows are identity rows, so they never move.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#define PMF_MAX_K 16          // largest local eigen count supported
#define PMF_MAX_SUB_CELLS 8192 // largest subdomain (cells) for the shared-memory sweeps
#define PMF_MAX_LINES 1024     // ny * nz of a subdomain (one thread per x-line)

namespace pmf {

struct SubInfo {
  int x0, nx, y0, ny, z0, nz;  // box
  int rank;                    // virtual rank
  int k;                       // eigen vectors kept (eigen_num_lv1)
  int local;                   // index inside its rank
  int nb[6];                   // neighbour subdomain across x-, x+, y-, y+, z-, z+ (-1: none)
  int prob;                    // problem of a batch (0 for a single problem)
};

// One problem of a batch.  The problems of a batch share one mesh: problem q
// occupies the cells x < M, y < N of the layers z0 .. z0 + P - 1 of a mesh
// max(M) x max(N) x sum(P + 1); the other cells and one layer between
// consecutive problems hold zero permeability, which decouples them.
struct ProbInfo {
  int M, N, P, z0;              // the problem's mesh and first layer in the shared mesh
  double Hx, Hy, Hz, meas;      // cell size and volume
  double cx, cy, cz;            // |face|^2 / |cell| per direction
  int dmask;                    // Dirichlet faces (bit f: x-, x+, y-, y+, z-, z+)
  double dval[6];               // Dirichlet values
  long long c0, c1;             // cell range [c0, c1) of its layers in the shared mesh
  int s0, s1;                   // its subdomains [s0, s1)
};

struct Grid {
  int M, N, P;
  int MN;
  long long ncell;
};

__host__ __device__ inline int cell_id(const Grid& g, int ex, int ey, int ez) {
  return (ez * g.N + ey) * g.M + ex;
}

// ---------------------------------------------------------------------------
// reductions
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Block-wide sum; every thread gets the result.  `scratch` holds >= 32 doubles.
__device__ inline double block_sum(double v, double* scratch) {
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
  v = warp_sum(v);
  __syncthreads();
  if (lane == 0) scratch[wid] = v;
  __syncthreads();
  double t = 0.0;
  if (wid == 0) {
    t = lane < nw ? scratch[lane] : 0.0;
    t = warp_sum(t);
    if (lane == 0) scratch[0] = t;
  }
  __syncthreads();
  t = scratch[0];
  __syncthreads();
  return t;
}

template <typename T>
struct VecT;
template <>
struct VecT<float> {
  typedef float type;
};
template <>
struct VecT<double> {
  typedef double type;
};

}  // namespace pmf
