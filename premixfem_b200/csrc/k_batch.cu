// Preconditioned CG over a batch of independent problems (the reference's
// KSPCG, src/Expe_scal.c:100-119, run once per problem) in one set of launches:
// every problem keeps its own CG scalars (PcgState), and every CG kernel is a
// two-dimensional grid whose blockIdx.y is the problem, so the dot products
// are reduced per problem in a fixed order.  The preconditioner application
// in between is the shared three-level cycle of the whole batch (its
// operators are block diagonal over the problems); it runs while any problem
// is still iterating, and the CG kernels of a finished problem do nothing.
#include "pmf_kernels.h"

namespace pmf {

namespace {
constexpr int kBT = 256;  // threads of the CG kernels

// the cells of problem q handled by thread t of block b: c0 + b*kBT + t + k*nblk*kBT
struct ProbCells {
  long long c0, c1, stride;
};
__device__ __forceinline__ ProbCells prob_cells(const ProbInfo& p, int nblk) {
  return ProbCells{p.c0 + (long long)blockIdx.x * kBT + threadIdx.x, p.c1, (long long)nblk * kBT};
}
__device__ __forceinline__ double bfixed_sum(const double* part, int n, double* red) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  return block_sum(v, red);
}
}  // namespace

// r = b, x = 0, partial r.r per (problem, block)
__global__ void k_bpcg_start(const ProbInfo* probs, const double* b, double* x, double* r, double* part, int nblk) {
  __shared__ double red[32];
  const int q = blockIdx.y;
  const ProbCells pc = prob_cells(probs[q], nblk);
  double v = 0.0;
  for (long long c = pc.c0; c < pc.c1; c += pc.stride) {
    const double bc = b[c];
    x[c] = 0.0;
    r[c] = bc;
    v += bc * bc;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[(long long)q * nblk + blockIdx.x] = v;
}
__global__ void k_bpcg_start_fin(const double* part, int nblk, PcgState* st, double rtol, double atol, int max_it) {
  __shared__ double red[32];
  const int q = blockIdx.x;
  const double v = bfixed_sum(part + (long long)q * nblk, nblk, red);
  if (threadIdx.x == 0) {
    PcgState& s = st[q];
    const double dp = sqrt(v);
    s.dp = dp;
    s.rnorm0 = dp;
    s.ttol = fmax(rtol * dp, atol);  // KSPConvergedDefault
    s.its = 0;
    s.max_it = max_it;
    s.first = 1;
    s.beta = s.betaold = s.dpi = s.dpiold = s.alpha = 0.0;
    s.done = (!(dp == dp) || isinf(dp)) ? 4 : (dp <= s.ttol) ? 1 : 0;
  }
}

// beta = z.r of each problem from the per-subdomain partials of the final level-1 visit
__global__ void k_bpcg_beta_fin(const ProbInfo* probs, const double* part, PcgState* st) {
  __shared__ double red[32];
  const int q = blockIdx.x;
  PcgState& s = st[q];
  if (s.done) return;
  const double v = bfixed_sum(part + probs[q].s0, probs[q].s1 - probs[q].s0, red);
  if (threadIdx.x == 0) {
    s.beta = v;
    if (v == 0.0) {
      s.its += 1;
      s.done = 5;  // KSP_CONVERGED_ATOL
    }
  }
}

// p <- z (first) or z + (beta/betaold) p; w <- A p; partial p.w (the single-problem kernel per problem)
__global__ void k_bpcg_iter_a(Grid g, const ProbInfo* probs, const double* tx, const double* ty, const double* tz,
                              const double* diag, const double* z, const double* pin, double* pout, double* w,
                              double* part, const PcgState* st, int nblk) {
  __shared__ double red[32];
  const int q = blockIdx.y;
  const PcgState& s = st[q];
  if (s.done) return;
  const bool first = s.first != 0;
  const double b = first ? 0.0 : s.beta / s.betaold;
  const ProbCells pc = prob_cells(probs[q], nblk);
  double v = 0.0;
  for (long long c = pc.c0; c < pc.c1; c += pc.stride) {
    const int ex = (int)(c % g.M);
    const long long t = c / g.M;
    const int ey = (int)(t % g.N), ez = (int)(t / g.N);
#define PNEW(i) (first ? z[i] : z[i] + b * pin[i])
    const double pcv = PNEW(c);
    double a = diag[c] * pcv;
    if (ex > 0) a -= tx[c] * PNEW(c - 1);
    if (ex < g.M - 1) a -= tx[c + 1] * PNEW(c + 1);
    if (ey > 0) a -= ty[c] * PNEW(c - g.M);
    if (ey < g.N - 1) a -= ty[c + g.M] * PNEW(c + g.M);
    if (ez > 0) a -= tz[c] * PNEW(c - g.MN);
    if (ez < g.P - 1) a -= tz[c + g.MN] * PNEW(c + g.MN);
#undef PNEW
    pout[c] = pcv;
    w[c] = a;
    v += pcv * a;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[(long long)q * nblk + blockIdx.x] = v;
}
__global__ void k_bpcg_iter_a_fin(const double* part, int nblk, PcgState* st) {
  __shared__ double red[32];
  const int q = blockIdx.x;
  PcgState& s = st[q];
  if (s.done) return;
  const double dpi = bfixed_sum(part + (long long)q * nblk, nblk, red);
  if (threadIdx.x == 0) {
    s.dpiold = s.dpi;
    s.dpi = dpi;
    s.betaold = s.beta;
    const bool flip = !s.first && ((dpi > 0) != (s.dpiold > 0));
    s.first = 0;
    if (dpi == 0.0 || flip) {
      s.its += 1;
      s.done = 3;  // KSP_DIVERGED_INDEFINITE_MAT
    } else {
      s.alpha = s.beta / dpi;
    }
  }
}

// The same step one cell per thread: a (32 x 4)-thread CTA covers 32 x 4 cells of
// one layer of the shared mesh, whose problem is layer_prob[z] (separator
// layers: none); partial (z gy + y) gx + x, so problem q's partials are the
// contiguous range of its layers.
__global__ void __launch_bounds__(128) k_bpcg_iter_a1(Grid g, const int* layer_prob, const double* __restrict__ tx,
                                                     const double* __restrict__ ty, const double* __restrict__ tz,
                                                     const double* __restrict__ diag, const double* __restrict__ z,
                                                     const double* __restrict__ pin, double* pout, double* w,
                                                     double* part, const PcgState* st) {
  __shared__ double red[4];
  const int ez = blockIdx.z;
  const int q = layer_prob[ez];
  if (q < 0) return;
  const PcgState& s = st[q];
  if (s.done) return;
  const bool first = s.first != 0;
  const double b = first ? 0.0 : s.beta / s.betaold;
  const int ex = blockIdx.x * 32 + threadIdx.x, ey = blockIdx.y * 4 + threadIdx.y;
  double v = 0.0;
  if (ex < g.M && ey < g.N) {
    const long long c = ((long long)ez * g.N + ey) * g.M + ex;
#define PNEW(i) (first ? z[i] : z[i] + b * pin[i])
    const double pcv = PNEW(c);
    double a = diag[c] * pcv;
    if (ex > 0) a -= tx[c] * PNEW(c - 1);
    if (ex < g.M - 1) a -= tx[c + 1] * PNEW(c + 1);
    if (ey > 0) a -= ty[c] * PNEW(c - g.M);
    if (ey < g.N - 1) a -= ty[c + g.M] * PNEW(c + g.M);
    if (ez > 0) a -= tz[c] * PNEW(c - g.MN);
    if (ez < g.P - 1) a -= tz[c + g.MN] * PNEW(c + g.MN);
#undef PNEW
    pout[c] = pcv;
    w[c] = a;
    v = pcv * a;
  }
  v = warp_sum(v);
  if (threadIdx.x == 0) red[threadIdx.y] = v;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0)
    part[((long long)ez * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = ((red[0] + red[1]) + red[2]) + red[3];
}
__global__ void __launch_bounds__(1024) k_bpcg_iter_a1_fin(const ProbInfo* probs, const double* part, int per_layer,
                                                           PcgState* st) {
  __shared__ double red[32];
  const int q = blockIdx.x;
  PcgState& s = st[q];
  if (s.done) return;
  const ProbInfo pq = probs[q];
  const double* pp = part + (long long)pq.z0 * per_layer;
  const int n = pq.P * per_layer;
  double a8[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) a8[u] = 0.0;
  for (int i0 = threadIdx.x; i0 < n; i0 += 8 * blockDim.x) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) a8[u] += pp[i];
    }
  }
  const double dpi = block_sum(((a8[0] + a8[1]) + (a8[2] + a8[3])) + ((a8[4] + a8[5]) + (a8[6] + a8[7])), red);
  if (threadIdx.x == 0) {
    s.dpiold = s.dpi;
    s.dpi = dpi;
    s.betaold = s.beta;
    const bool flip = !s.first && ((dpi > 0) != (s.dpiold > 0));
    s.first = 0;
    if (dpi == 0.0 || flip) {
      s.its += 1;
      s.done = 3;  // KSP_DIVERGED_INDEFINITE_MAT
    } else {
      s.alpha = s.beta / dpi;
    }
  }
}

// x += alpha p, r -= alpha w, partial r.r
__global__ void k_bpcg_iter_b(const ProbInfo* probs, double* x, double* r, const double* p, const double* w,
                              double* part, const PcgState* st, int nblk) {
  __shared__ double red[32];
  const int q = blockIdx.y;
  const PcgState& s = st[q];
  if (s.done) return;
  const double a = s.alpha;
  const ProbCells pc = prob_cells(probs[q], nblk);
  double v = 0.0;
  for (long long c = pc.c0; c < pc.c1; c += pc.stride) {
    x[c] += a * p[c];
    const double rc = r[c] - a * w[c];
    r[c] = rc;
    v += rc * rc;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[(long long)q * nblk + blockIdx.x] = v;
}
__global__ void k_bpcg_iter_b_fin(const double* part, int nblk, PcgState* st) {
  __shared__ double red[32];
  const int q = blockIdx.x;
  PcgState& s = st[q];
  if (s.done) return;
  const double v = bfixed_sum(part + (long long)q * nblk, nblk, red);
  if (threadIdx.x == 0) {
    const double dp = sqrt(v);
    s.dp = dp;
    s.its += 1;
    if (!(dp == dp) || isinf(dp))
      s.done = 4;
    else if (dp <= s.ttol)
      s.done = 1;
    else if (s.its >= s.max_it)
      s.done = 2;
  }
}

// all_done = 1 when every problem has stopped (the shared preconditioner kernels test it)
__global__ void k_bpcg_all_done(const PcgState* st, int nprob, int* all_done) {
  __shared__ int any;
  if (threadIdx.x == 0) any = 0;
  __syncthreads();
  for (int q = threadIdx.x; q < nprob; q += blockDim.x)
    if (!st[q].done) any = 1;
  __syncthreads();
  if (threadIdx.x == 0) *all_done = any ? 0 : 1;
}

void launch_bpcg_start(const ProbInfo* probs, int nprob, const double* b, double* x, double* r, double* part,
                       PcgState* st, double rtol, double atol, int max_it, int* all_done, int nblk, cudaStream_t s) {
  { note_launch(); k_bpcg_start<<<dim3(nblk, nprob), kBT, 0, s>>>(probs, b, x, r, part, nblk); }
  { note_launch(); k_bpcg_start_fin<<<nprob, 256, 0, s>>>(part, nblk, st, rtol, atol, max_it); }
  { note_launch(); k_bpcg_all_done<<<1, 256, 0, s>>>(st, nprob, all_done); }
}
void launch_bpcg_beta(const ProbInfo* probs, int nprob, const double* part, PcgState* st, cudaStream_t s) {
  { note_launch(); k_bpcg_beta_fin<<<nprob, 256, 0, s>>>(probs, part, st); }
}
void launch_bpcg_iter_a(const Grid& g, const ProbInfo* probs, const int* layer_prob, int nprob, const double* tx,
                        const double* ty, const double* tz, const double* diag, const double* z, const double* pin,
                        double* pout, double* w, double* part, PcgState* st, int nblk, cudaStream_t s) {
  // one cell per thread (pcg_part_capacity(g) partials) where the grid fits, else the grid-stride form
  const dim3 grid((g.M + 31) / 32, (g.N + 3) / 4, g.P);
  if (layer_prob && grid.y <= 65535 && grid.z <= 65535) {
    { note_launch(); k_bpcg_iter_a1<<<grid, dim3(32, 4), 0, s>>>(g, layer_prob, tx, ty, tz, diag, z, pin, pout, w, part, st); }
    { note_launch(); k_bpcg_iter_a1_fin<<<nprob, 1024, 0, s>>>(probs, part, (int)(grid.x * grid.y), st); }
    return;
  }
  { note_launch(); k_bpcg_iter_a<<<dim3(nblk, nprob), kBT, 0, s>>>(g, probs, tx, ty, tz, diag, z, pin, pout, w, part, st, nblk); }
  { note_launch(); k_bpcg_iter_a_fin<<<nprob, 256, 0, s>>>(part, nblk, st); }
}
void launch_bpcg_iter_b(const ProbInfo* probs, int nprob, double* x, double* r, const double* p, const double* w,
                        double* part, PcgState* st, int* all_done, int nblk, cudaStream_t s) {
  { note_launch(); k_bpcg_iter_b<<<dim3(nblk, nprob), kBT, 0, s>>>(probs, x, r, p, w, part, st, nblk); }
  { note_launch(); k_bpcg_iter_b_fin<<<nprob, 256, 0, s>>>(part, nblk, st); }
  { note_launch(); k_bpcg_all_done<<<1, 256, 0, s>>>(st, nprob, all_done); }
}

}  // namespace pmf
