// Fine-grid kernels: operator assembly, stencil products, CG vector updates,
// level-1 IC(0) block solves and the level-2 restriction / prolongation.
#include <algorithm>

#include "pmf_kernels.h"

namespace pmf {

int cell_blocks(long long n) {
  long long b = (n + kCellThreads - 1) / kCellThreads;
  const long long cap = 148LL * 16;
  return (int)std::max(1LL, std::min(b, cap));
}

__device__ __forceinline__ void decode(long long c, const Grid& g, int& ex, int& ey, int& ez) {
  ex = (int)(c % g.M);
  long long t = c / g.M;
  ey = (int)(t % g.N);
  ez = (int)(t / g.N);
}

// ---------------------------------------------------------------------------
// PC_create_A (src/PreMixFEM_3D.c:1757-1824): interior faces get
// t = |f|^2/|K| * 2 / (1/k_L + 1/k_R), evaluated in the reference's order.
// Dirichlet faces (extension) add t_b = |f|^2/|K| * 2 k_cell to the diagonal
// and t_b * p_D to the right-hand side.
__device__ __forceinline__ double hmean(double a, double b) { return 2.0 / (1.0 / a + 1.0 / b); }

__global__ void k_assemble(AssembleArgs a, double* tx, double* ty, double* tz, double* diag, double* db,
                           double* bval) {
  const Grid g = a.g;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    decode(c, g, ex, ey, ez);
    // the cell's problem: its face coefficients, faces and Dirichlet data
    double cx = a.cx, cy = a.cy, cz = a.cz;
    int lo[3] = {0, 0, 0}, hi[3] = {g.M, g.N, g.P};
    bool dir_on[6];
    double dir_val[6];
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      dir_on[f] = a.dir_on[f] != 0;
      dir_val[f] = a.dir_val[f];
    }
    if (a.probs) {
      const int q = a.layer_prob[ez];
      if (q < 0 || ex >= a.probs[q].M || ey >= a.probs[q].N) {  // no problem: decoupled, zero row
        tx[c] = ty[c] = tz[c] = diag[c] = db[c] = bval[c] = 0.0;
        continue;
      }
      const ProbInfo& p = a.probs[q];
      cx = p.cx;
      cy = p.cy;
      cz = p.cz;
      hi[0] = p.M;
      hi[1] = p.N;
      lo[2] = p.z0;
      hi[2] = p.z0 + p.P;
#pragma unroll
      for (int f = 0; f < 6; ++f) {
        dir_on[f] = (p.dmask >> f) & 1;
        dir_val[f] = p.dval[f];
      }
    }
    const double txc = ex > lo[0] ? cx * hmean(a.kx[c - 1], a.kx[c]) : 0.0;
    const double tyc = ey > lo[1] ? cy * hmean(a.ky[c - g.M], a.ky[c]) : 0.0;
    const double tzc = ez > lo[2] ? cz * hmean(a.kz[c - g.MN], a.kz[c]) : 0.0;
    const double txn = ex < hi[0] - 1 ? cx * hmean(a.kx[c], a.kx[c + 1]) : 0.0;
    const double tyn = ey < hi[1] - 1 ? cy * hmean(a.ky[c], a.ky[c + g.M]) : 0.0;
    const double tzn = ez < hi[2] - 1 ? cz * hmean(a.kz[c], a.kz[c + g.MN]) : 0.0;
    double dbc = 0.0, bv = 0.0;
    const bool on[6] = {ex == lo[0], ex == hi[0] - 1, ey == lo[1], ey == hi[1] - 1, ez == lo[2], ez == hi[2] - 1};
    const double cf[6] = {cx, cx, cy, cy, cz, cz};
    const double kk[6] = {a.kx[c], a.kx[c], a.ky[c], a.ky[c], a.kz[c], a.kz[c]};
#pragma unroll
    for (int f = 0; f < 6; ++f) {
      if (dir_on[f] && on[f]) {
        const double tb = cf[f] * (2.0 * kk[f]);
        dbc += tb;
        bv += tb * dir_val[f];
      }
    }
    tx[c] = txc;
    ty[c] = tyc;
    tz[c] = tzc;
    double d = txc + tyc;
    d = d + tzc;
    d = d + txn;
    d = d + tyn;
    d = d + tzn;
    d = d + dbc;
    diag[c] = d;
    db[c] = dbc;
    bval[c] = bv;
  }
}

__global__ void k_zero_padding(Grid g, const ProbInfo* probs, const int* layer_prob, double* kx, double* ky,
                               double* kz) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    decode(c, g, ex, ey, ez);
    const int q = layer_prob[ez];
    if (q < 0 || ex >= probs[q].M || ey >= probs[q].N) kx[c] = ky[c] = kz[c] = 0.0;
  }
}
void launch_zero_padding(const Grid& g, const ProbInfo* probs, const int* layer_prob, double* kx, double* ky,
                         double* kz, cudaStream_t st) {
  { note_launch(); k_zero_padding<<<cell_blocks(g.ncell), kCellThreads, 0, st>>>(g, probs, layer_prob, kx, ky, kz); }
}

void launch_assemble(const AssembleArgs& a, double* tx, double* ty, double* tz, double* diag, double* db,
                     double* bval, cudaStream_t st) {
  { note_launch(); k_assemble<<<cell_blocks(a.g.ncell), kCellThreads, 0, st>>>(a, tx, ty, tz, diag, db, bval); }
}

__global__ void k_to_f32(const double* in, float* out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (float)in[i];
}
__global__ void k_to_f64(const float* in, double* out, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    out[i] = (double)in[i];
}
void launch_to_f32(const double* in, float* out, long long n, cudaStream_t st) {
  { note_launch(); k_to_f32<<<cell_blocks(n), kCellThreads, 0, st>>>(in, out, n); }
}
void launch_to_f64(const float* in, double* out, long long n, cudaStream_t st) {
  { note_launch(); k_to_f64<<<cell_blocks(n), kCellThreads, 0, st>>>(in, out, n); }
}

// ---------------------------------------------------------------------------
// 7-point stencil product A x, precision T.
template <typename T>
__device__ __forceinline__ T apply_A(const Grid& g, long long c, int ex, int ey, int ez, const T* tx, const T* ty,
                                     const T* tz, const T* diag, const T* x) {
  T v = diag[c] * x[c];
  if (ex > 0) v -= tx[c] * x[c - 1];
  if (ex < g.M - 1) v -= tx[c + 1] * x[c + 1];
  if (ey > 0) v -= ty[c] * x[c - g.M];
  if (ey < g.N - 1) v -= ty[c + g.M] * x[c + g.M];
  if (ez > 0) v -= tz[c] * x[c - g.MN];
  if (ez < g.P - 1) v -= tz[c + g.MN] * x[c + g.MN];
  return v;
}

__global__ void k_spmv(Grid g, const double* tx, const double* ty, const double* tz, const double* diag,
                       const double* x, double* y) {
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    decode(c, g, ex, ey, ez);
    y[c] = apply_A(g, c, ex, ey, ez, tx, ty, tz, diag, x);
  }
}

void launch_spmv(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                 const double* x, double* y, cudaStream_t st) {
  { note_launch(); k_spmv<<<cell_blocks(g.ncell), kCellThreads, 0, st>>>(g, tx, ty, tz, diag, x, y); }
}

// ---------------------------------------------------------------------------
// Deterministic reductions: each block writes one partial; a single block
// sums the partials in a fixed order.
__device__ __forceinline__ double fixed_sum(const double* part, int n, double* scratch) {
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) v += part[i];
  return block_sum(v, scratch);
}
// The same for long partial lists (the one-cell-per-thread CG step writes one
// per 128 cells): eight independent accumulators per thread keep eight loads
// in flight, summed in a fixed order.
__device__ __forceinline__ double fixed_sum_wide(const double* part, int n, double* scratch) {
  double a[8];
#pragma unroll
  for (int u = 0; u < 8; ++u) a[u] = 0.0;
  for (int i0 = threadIdx.x; i0 < n; i0 += 8 * blockDim.x) {
#pragma unroll
    for (int u = 0; u < 8; ++u) {
      const int i = i0 + u * blockDim.x;
      if (i < n) a[u] += part[i];
    }
  }
  const double v = ((a[0] + a[1]) + (a[2] + a[3])) + ((a[4] + a[5]) + (a[6] + a[7]));
  return block_sum(v, scratch);
}

__global__ void k_dot(const double* a, const double* b, long long n, double* part) {
  __shared__ double red[32];
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v += a[i] * b[i];
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
__global__ void k_fin_sum(const double* part, int n, double* out) {
  __shared__ double red[32];
  double v = fixed_sum(part, n, red);
  if (threadIdx.x == 0) *out = v;
}
void launch_dot(const double* a, const double* b, long long n, double* part, double* out, cudaStream_t st) {
  int nb = cell_blocks(n);
  { note_launch(); k_dot<<<nb, kCellThreads, 0, st>>>(a, b, n, part); }
  { note_launch(); k_fin_sum<<<1, 256, 0, st>>>(part, nb, out); }
}

// --- KSPSolve_CG (PETSc src/ksp/ksp/impls/cg/cg.c) with the unpreconditioned norm ---
__global__ void k_pcg_start(long long n, const double* b, double* x, double* r, double* part) {
  __shared__ double red[32];
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double bi = b[i];
    x[i] = 0.0;
    r[i] = bi;
    v += bi * bi;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
__global__ void k_pcg_start_fin(const double* part, int nb, PcgState* s, double rtol, double atol, int max_it) {
  __shared__ double red[32];
  const double v = fixed_sum(part, nb, red);
  if (threadIdx.x == 0) {
    const double dp = sqrt(v);
    s->dp = dp;
    s->rnorm0 = dp;
    s->ttol = fmax(rtol * dp, atol);  // KSPConvergedDefault: max(rtol*rnorm0, abstol)
    s->its = 0;
    s->max_it = max_it;
    s->first = 1;
    s->beta = s->betaold = s->dpi = s->dpiold = s->alpha = 0.0;
    // KSPConvergedDefault tests for NaN/Inf before the tolerance
    s->done = (!(dp == dp) || isinf(dp)) ? 4 : (dp <= s->ttol) ? 1 : 0;
  }
}
void launch_pcg_start(const Grid& g, const double* b, double* x, double* r, double* part, PcgState* s, double rtol,
                      double atol, int max_it, cudaStream_t st) {
  int nb = cell_blocks(g.ncell);
  { note_launch(); k_pcg_start<<<nb, kCellThreads, 0, st>>>(g.ncell, b, x, r, part); }
  { note_launch(); k_pcg_start_fin<<<1, 256, 0, st>>>(part, nb, s, rtol, atol, max_it); }
}

// beta = z.r (the dot is written per block by the preconditioner's last kernel
// or by k_dot); a zero beta ends the loop with done = 5 (KSP_CONVERGED_ATOL,
// as KSPSolve_CG reports it).
__global__ void k_pcg_beta_fin(const double* part, int nb, PcgState* s) {
  __shared__ double red[32];
  if (s->done) return;
  const double v = fixed_sum(part, nb, red);
  if (threadIdx.x == 0) {
    s->beta = v;
    if (v == 0.0) {
      s->its += 1;
      s->done = 5;
    }
  }
}
void launch_pcg_beta_fin(const double* part, int nparts, PcgState* s, cudaStream_t st) {
  { note_launch(); k_pcg_beta_fin<<<1, 256, 0, st>>>(part, nparts, s); }
}
void launch_pcg_beta(const double* r, const double* z, long long n, double* part, PcgState* s, cudaStream_t st) {
  int nb = cell_blocks(n);
  { note_launch(); k_dot<<<nb, kCellThreads, 0, st>>>(r, z, n, part); }
  { note_launch(); k_pcg_beta_fin<<<1, 256, 0, st>>>(part, nb, s); }
}

// Constant null space (-ksp_constant_null_space): PETSc's KSP_PCApply removes
// the operator's null space from every preconditioned residual of a left-
// preconditioned solve (MatNullSpaceRemove with a constant: z <- z - (sum z / n) 1),
// then CG takes beta = z.r of the projected z.  Two grid-stride passes: the
// per-block sums of z, then every block forms the mean from those partials in
// the same fixed order, shifts z and writes its partial of z.r.  Skipped once
// the solve is done, like the preconditioner kernels of a replayed graph chunk.
__global__ void k_null_sum(const double* z, long long n, double* zpart, const int* done) {
  __shared__ double red[32];
  if (*done) return;
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    v += z[i];
  v = block_sum(v, red);
  if (threadIdx.x == 0) zpart[blockIdx.x] = v;
}
__global__ void k_null_project(double* z, const double* r, long long n, const double* zpart, int nb, double* part,
                               const int* done) {
  __shared__ double red[32];
  if (*done) return;
  const double shift = fixed_sum(zpart, nb, red) / (-(double)n);
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double zi = z[i] + shift;
    z[i] = zi;
    v += zi * r[i];
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
void launch_pcg_null_beta(double* z, const double* r, long long n, double* part, double* zpart, PcgState* s,
                          cudaStream_t st) {
  const int nb = cell_blocks(n);
  { note_launch(); k_null_sum<<<nb, kCellThreads, 0, st>>>(z, n, zpart, &s->done); }
  { note_launch(); k_null_project<<<nb, kCellThreads, 0, st>>>(z, r, n, zpart, nb, part, &s->done); }
  { note_launch(); k_pcg_beta_fin<<<1, 256, 0, st>>>(part, nb, s); }
}

// p <- z (first) or z + (beta/betaold) p; w <- A p; partial p.w.
// In-place on p: the stencil reads p at neighbours, so p_new is formed from z
// and the old p of each neighbour on the fly, and written to pout != pin.
__global__ void k_pcg_iter_a(Grid g, const double* tx, const double* ty, const double* tz, const double* diag,
                             const double* z, const double* pin, double* pout, double* w, double* part,
                             const PcgState* s) {
  __shared__ double red[32];
  if (s->done) return;
  const bool first = s->first != 0;
  const double b = first ? 0.0 : s->beta / s->betaold;
  double v = 0.0;
  for (long long c = blockIdx.x * (long long)blockDim.x + threadIdx.x; c < g.ncell;
       c += (long long)gridDim.x * blockDim.x) {
    int ex, ey, ez;
    decode(c, g, ex, ey, ez);
#define PNEW(i) (first ? z[i] : z[i] + b * pin[i])
    const double pc = PNEW(c);
    double a = diag[c] * pc;
    if (ex > 0) a -= tx[c] * PNEW(c - 1);
    if (ex < g.M - 1) a -= tx[c + 1] * PNEW(c + 1);
    if (ey > 0) a -= ty[c] * PNEW(c - g.M);
    if (ey < g.N - 1) a -= ty[c + g.M] * PNEW(c + g.M);
    if (ez > 0) a -= tz[c] * PNEW(c - g.MN);
    if (ez < g.P - 1) a -= tz[c + g.MN] * PNEW(c + g.MN);
#undef PNEW
    pout[c] = pc;
    w[c] = a;
    v += pc * a;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
__global__ void __launch_bounds__(1024) k_pcg_iter_a_fin(const double* part, int nb, PcgState* s) {
  __shared__ double red[32];
  if (s->done) return;
  const double dpi = fixed_sum_wide(part, nb, red);
  if (threadIdx.x == 0) {
    s->dpiold = s->dpi;
    s->dpi = dpi;
    s->betaold = s->beta;
    const bool flip = !s->first && ((dpi > 0) != (s->dpiold > 0));
    s->first = 0;
    if (dpi == 0.0 || flip) {
      s->its += 1;
      s->done = 3;  // KSP_DIVERGED_INDEFINITE_MAT
    } else {
      s->alpha = s->beta / dpi;
    }
  }
}
// The same step as a 2.5-D march: a CTA owns a 32 x 16 tile of x-lines and a
// stretch of z-planes; the new p of the current plane sits in shared memory
// with a one-cell halo, the planes below and above in registers, so z and p
// are read once per cell (plus the tile halo) instead of at all seven stencil
// points.  The operator is evaluated in apply_A's order (same w bit for bit).
// One cell per thread: a (32 x 4)-thread CTA covers 32 x 4 cells of one z-plane,
// the grid covers the mesh, so no thread decodes a linear index and every load
// has the whole GPU's parallelism behind it; the seven-point stencil reads its
// neighbours through L1/L2.  Same arithmetic as k_pcg_iter_a, in the same
// order.  One partial of p.w per CTA.
constexpr int kP1X = 32, kP1Y = 4;
__global__ void __launch_bounds__(kP1X * kP1Y) k_pcg_iter_a1(Grid g, const double* __restrict__ tx,
                                                            const double* __restrict__ ty,
                                                            const double* __restrict__ tz,
                                                            const double* __restrict__ diag,
                                                            const double* __restrict__ z,
                                                            const double* __restrict__ pin, double* pout, double* w,
                                                            double* part, const PcgState* s) {
  __shared__ double red[kP1Y];
  if (s->done) return;
  const bool first = s->first != 0;
  const double b = first ? 0.0 : s->beta / s->betaold;
  const int ex = blockIdx.x * kP1X + threadIdx.x, ey = blockIdx.y * kP1Y + threadIdx.y, ez = blockIdx.z;
  double v = 0.0;
  if (ex < g.M && ey < g.N) {
    const long long c = ((long long)ez * g.N + ey) * g.M + ex;
#define PNEW(i) (first ? z[i] : z[i] + b * pin[i])
    const double pc = PNEW(c);
    double a = diag[c] * pc;
    if (ex > 0) a -= tx[c] * PNEW(c - 1);
    if (ex < g.M - 1) a -= tx[c + 1] * PNEW(c + 1);
    if (ey > 0) a -= ty[c] * PNEW(c - g.M);
    if (ey < g.N - 1) a -= ty[c + g.M] * PNEW(c + g.M);
    if (ez > 0) a -= tz[c] * PNEW(c - g.MN);
    if (ez < g.P - 1) a -= tz[c + g.MN] * PNEW(c + g.MN);
#undef PNEW
    pout[c] = pc;
    w[c] = a;
    v = pc * a;
  }
  v = warp_sum(v);
  if (threadIdx.x == 0) red[threadIdx.y] = v;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double t = 0.0;
    for (int i = 0; i < kP1Y; ++i) t += red[i];
    part[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = t;
  }
}

int pcg_part_capacity(const Grid& g) {
  const long long n1 = (long long)((g.M + kP1X - 1) / kP1X) * ((g.N + kP1Y - 1) / kP1Y) * g.P;
  return (int)std::max<long long>(cell_blocks(g.ncell), n1);
}

constexpr int kPaX = 32, kPaY = 16;
__global__ void __launch_bounds__(kPaX * kPaY) k_pcg_iter_a25(Grid g, const double* __restrict__ tx,
                                                             const double* __restrict__ ty,
                                                             const double* __restrict__ tz,
                                                             const double* __restrict__ diag,
                                                             const double* __restrict__ z,
                                                             const double* __restrict__ pin, double* pout,
                                                             double* w, double* part, const PcgState* s, int zc) {
  __shared__ double sp[kPaY + 2][kPaX + 2];
  __shared__ double red[32];
  if (s->done) return;
  const bool first = s->first != 0;
  const double b = first ? 0.0 : s->beta / s->betaold;
  const int lx = threadIdx.x % kPaX, ly = threadIdx.x / kPaX;
  const int ex = blockIdx.x * kPaX + lx, ey = blockIdx.y * kPaY + ly;
  const int zb = blockIdx.z * zc, ze = min(g.P, zb + zc);
  const bool in = ex < g.M && ey < g.N;
  auto pn = [&](long long c) { return first ? z[c] : z[c] + b * pin[c]; };
  const long long row = (long long)ey * g.M + ex;
  double pprev = 0.0, pcur = 0.0;
  if (in) {
    pcur = pn((long long)zb * g.MN + row);
    if (zb > 0) pprev = pn((long long)(zb - 1) * g.MN + row);
  }
  double v = 0.0;
  for (int ez = zb; ez < ze; ++ez) {
    const long long c = (long long)ez * g.MN + row;
    const double pnext = (in && ez + 1 < g.P) ? pn(c + g.MN) : 0.0;
    sp[ly + 1][lx + 1] = pcur;
    if (lx == 0) sp[ly + 1][0] = (in && ex > 0) ? pn(c - 1) : 0.0;
    if (lx == kPaX - 1) sp[ly + 1][kPaX + 1] = (in && ex + 1 < g.M) ? pn(c + 1) : 0.0;
    if (ly == 0) sp[0][lx + 1] = (in && ey > 0) ? pn(c - g.M) : 0.0;
    if (ly == kPaY - 1) sp[kPaY + 1][lx + 1] = (in && ey + 1 < g.N) ? pn(c + g.M) : 0.0;
    __syncthreads();
    if (in) {
      double a = diag[c] * pcur;
      if (ex > 0) a -= tx[c] * sp[ly + 1][lx];
      if (ex < g.M - 1) a -= tx[c + 1] * sp[ly + 1][lx + 2];
      if (ey > 0) a -= ty[c] * sp[ly][lx + 1];
      if (ey < g.N - 1) a -= ty[c + g.M] * sp[ly + 2][lx + 1];
      if (ez > 0) a -= tz[c] * pprev;
      if (ez < g.P - 1) a -= tz[c + g.MN] * pnext;
      pout[c] = pcur;
      w[c] = a;
      v += pcur * a;
    }
    __syncthreads();  // the next plane overwrites sp
    pprev = pcur;
    pcur = pnext;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[((long long)blockIdx.z * gridDim.y + blockIdx.y) * gridDim.x + blockIdx.x] = v;
}

int launch_pcg_iter_a_main(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                           const double* z, const double* pin, double* pout, double* w, double* part,
                           const PcgState* s, cudaStream_t st, int variant) {
  // variant 0: one cell per thread (pcg_part_capacity(g) partials, the size the caller's buffer holds);
  // 1: the 2.5-D march; 2: grid-stride.  Variants 1 and 2 use at most cell_blocks(ncell) partials.
  if (variant == 0) {
    const dim3 grid((g.M + kP1X - 1) / kP1X, (g.N + kP1Y - 1) / kP1Y, g.P);
    if (grid.y <= 65535 && grid.z <= 65535) {
      { note_launch(); k_pcg_iter_a1<<<grid, dim3(kP1X, kP1Y), 0, st>>>(g, tx, ty, tz, diag, z, pin, pout, w, part, s); }
      return (int)(grid.x * grid.y * grid.z);
    }
    variant = 1;
  }
  const int cap = cell_blocks(g.ncell);
  const int bx = (g.M + kPaX - 1) / kPaX, by = (g.N + kPaY - 1) / kPaY;
  const int per_z = std::max(1, cap / std::max(1, bx * by));
  const int zc = std::max(16, (g.P + per_z - 1) / per_z);
  const int bz = (g.P + zc - 1) / zc;
  const long long nb25 = (long long)bx * by * bz;
  if (variant == 1 && nb25 <= cap && by <= 65535 && bz <= 65535) {
    { note_launch(); k_pcg_iter_a25<<<dim3(bx, by, bz), kPaX * kPaY, 0, st>>>(g, tx, ty, tz, diag, z, pin, pout, w, part, s, zc); }
    return (int)nb25;
  }
  { note_launch(); k_pcg_iter_a<<<cap, kCellThreads, 0, st>>>(g, tx, ty, tz, diag, z, pin, pout, w, part, s); }
  return cap;
}

void launch_pcg_iter_a(const Grid& g, const double* tx, const double* ty, const double* tz, const double* diag,
                       const double* z, const double* pin, double* pout, double* w, double* part, PcgState* s,
                       cudaStream_t st, int variant) {
  const int nb = launch_pcg_iter_a_main(g, tx, ty, tz, diag, z, pin, pout, w, part, s, st, variant);
  { note_launch(); k_pcg_iter_a_fin<<<1, 1024, 0, st>>>(part, nb, s); }
}

// x += alpha p; r -= alpha w; partial r.r; then dp, its and the convergence test.
__global__ void k_pcg_iter_b(long long n, double* x, double* r, const double* p, const double* w, double* part,
                             const PcgState* s) {
  __shared__ double red[32];
  if (s->done) return;
  const double a = s->alpha;
  double v = 0.0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    x[i] += a * p[i];
    const double ri = r[i] - a * w[i];
    r[i] = ri;
    v += ri * ri;
  }
  v = block_sum(v, red);
  if (threadIdx.x == 0) part[blockIdx.x] = v;
}
__global__ void k_pcg_iter_b_fin(const double* part, int nb, PcgState* s) {
  __shared__ double red[32];
  if (s->done) return;
  const double v = fixed_sum(part, nb, red);
  if (threadIdx.x == 0) {
    const double dp = sqrt(v);
    s->dp = dp;
    s->its += 1;
    if (!(dp == dp) || isinf(dp))
      s->done = 4;
    else if (dp <= s->ttol)
      s->done = 1;
    else if (s->its >= s->max_it)
      s->done = 2;
  }
}
void launch_pcg_iter_b(long long n, double* x, double* r, const double* p, const double* w, double* part,
                       PcgState* s, cudaStream_t st) {
  int nb = cell_blocks(n);
  { note_launch(); k_pcg_iter_b<<<nb, kCellThreads, 0, st>>>(n, x, r, p, w, part, s); }
  { note_launch(); k_pcg_iter_b_fin<<<1, 256, 0, st>>>(part, nb, s); }
}

// ---------------------------------------------------------------------------
// Level 1: IC(0) of each subdomain's principal submatrix (PCICC, natural
// order, src/PreMixFEM_3D.c:200-215).  For the 7-point pattern the factor is
// (D + L) D^-1 (D + L^T) with D_i = a_ii - sum_{lower nb j} a_ij^2 / D_j.
//
// Both the factorisation and the solves run as hyperplane wavefronts inside
// one CTA per subdomain: thread (j, k) owns the x-line (., j, k) and handles
// its cell i = d - j - k on plane d; neighbours on the previous plane are
// read from shared memory after a barrier.
struct SubGeom {
  int x0, y0, z0, nx, ny, nz, nxny, ncells, nlines, nplanes;
};
__device__ __forceinline__ SubGeom sub_geom(const SubInfo& s) {
  SubGeom q;
  q.x0 = s.x0;
  q.y0 = s.y0;
  q.z0 = s.z0;
  q.nx = s.nx;
  q.ny = s.ny;
  q.nz = s.nz;
  q.nxny = s.nx * s.ny;
  q.ncells = q.nxny * s.nz;
  q.nlines = s.ny * s.nz;
  q.nplanes = s.nx + s.ny + s.nz - 2;
  return q;
}

__global__ void k_ic_factor(Grid g, const SubInfo* subs, const double* tx, const double* ty, const double* tz,
                            const double* diag, double* inv_d, int* bad) {
  extern __shared__ double Dsh[];
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  const int t = threadIdx.x;
  const int j = t % q.ny, k = t / q.ny;
  for (int d = 0; d < q.nplanes; ++d) {
    const int i = d - j - k;
    if (t < q.nlines && i >= 0 && i < q.nx) {
      const int cl = (k * q.ny + j) * q.nx + i;
      const long long cg = ((long long)(q.z0 + k) * g.N + (q.y0 + j)) * g.M + (q.x0 + i);
      double s = 0.0;
      if (k > 0) {
        const double a = tz[cg];
        s += a * a / Dsh[cl - q.nxny];
      }
      if (j > 0) {
        const double a = ty[cg];
        s += a * a / Dsh[cl - q.nx];
      }
      if (i > 0) {
        const double a = tx[cg];
        s += a * a / Dsh[cl - 1];
      }
      double D = diag[cg] - s;
      if (!(D > 0.0)) {
        atomicAdd(bad, 1);
        D = diag[cg];
      }
      Dsh[cl] = D;
      inv_d[cg] = 1.0 / D;
    }
    __syncthreads();
  }
}

void launch_ic_factor(const Grid& g, const SubInfo* subs, int nsub, int max_lines, const double* tx,
                      const double* ty, const double* tz, const double* diag, double* inv_d, int* bad,
                      cudaStream_t st) {
  // the caller guarantees ny*nz <= PMF_MAX_LINES and cells <= PMF_MAX_SUB_CELLS for every subdomain
  int threads = std::max(32, ((max_lines + 31) / 32) * 32);
  const int smem = PMF_MAX_SUB_CELLS * sizeof(double);
  cudaFuncSetAttribute(k_ic_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  { note_launch(); k_ic_factor<<<nsub, threads, smem, st>>>(g, subs, tx, ty, tz, diag, inv_d, bad); }
}

// Hyperplane sweeps of the IC(0) solve on a subdomain whose couplings (cx, cy,
// cz: lower-face transmissibility of each cell inside the subdomain, 0 on its
// boundary) and inverse pivots (ci) sit in shared memory next to the vector u.
template <typename T>
__device__ __forceinline__ void ic_sweeps_smem(const SubGeom& q, const T* cx, const T* cy, const T* cz, const T* ci,
                                               T* u) {
  const int t = threadIdx.x;
  const int j = t % q.ny, k = t / q.ny;
  const bool line = t < q.nlines;
  // forward: (D + L) w = r  ->  w_i = (r_i + sum t_ij w_j) / D_i
  for (int d = 0; d < q.nplanes; ++d) {
    const int i = d - j - k;
    if (line && i >= 0 && i < q.nx) {
      const int cl = (k * q.ny + j) * q.nx + i;
      T s = u[cl];
      if (k > 0) s += cz[cl] * u[cl - q.nxny];
      if (j > 0) s += cy[cl] * u[cl - q.nx];
      if (i > 0) s += cx[cl] * u[cl - 1];
      u[cl] = s * ci[cl];
    }
    __syncthreads();
  }
  // backward: (D + L^T) z = D w  ->  z_i = w_i + (sum_{upper j} t_ij z_j) / D_i
  for (int d = q.nplanes - 1; d >= 0; --d) {
    const int i = d - j - k;
    if (line && i >= 0 && i < q.nx) {
      const int cl = (k * q.ny + j) * q.nx + i;
      T s = (T)0;
      if (i < q.nx - 1) s += cx[cl + 1] * u[cl + 1];
      if (j < q.ny - 1) s += cy[cl + q.nx] * u[cl + q.nx];
      if (k < q.nz - 1) s += cz[cl + q.nxny] * u[cl + q.nxny];
      u[cl] = u[cl] + s * ci[cl];
    }
    __syncthreads();
  }
}

template <typename T, bool HAS_Y, bool FINAL>
__global__ void k_ic_apply(Grid g, const SubInfo* subs, const T* tx, const T* ty, const T* tz, const T* diag,
                           const T* inv_d, const double* x, const T* yin, T* out_t, double* out_d, double* part,
                           const int* done, int ldc) {
  if (done && *done) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  double* red = reinterpret_cast<double*>(smem_raw);
  T* u = reinterpret_cast<T*>(smem_raw + 32 * sizeof(double));
  T* cx = u + ldc;
  T* cy = cx + ldc;
  T* cz = cy + ldc;
  T* ci = cz + ldc;
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  // right-hand side r = x - A y on the subdomain (y read across subdomain faces)
  // and the subdomain's couplings / inverse pivots, in one coalesced pass
  for (int cl = threadIdx.x; cl < q.ncells; cl += blockDim.x) {
    const int i = cl % q.nx, tt = cl / q.nx, j = tt % q.ny, k = tt / q.ny;
    const int ex = q.x0 + i, ey = q.y0 + j, ez = q.z0 + k;
    const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
    const T txc = tx[cg], tyc = ty[cg], tzc = tz[cg];
    cx[cl] = i > 0 ? txc : (T)0;
    cy[cl] = j > 0 ? tyc : (T)0;
    cz[cl] = k > 0 ? tzc : (T)0;
    ci[cl] = inv_d[cg];
    T r = (T)x[cg];
    if (HAS_Y) r -= apply_A(g, cg, ex, ey, ez, tx, ty, tz, diag, yin);
    u[cl] = r;
  }
  __syncthreads();
  ic_sweeps_smem(q, cx, cy, cz, ci, u);
  double dot = 0.0;
  for (int cl = threadIdx.x; cl < q.ncells; cl += blockDim.x) {
    const int i = cl % q.nx, tt = cl / q.nx, j = tt % q.ny, k = tt / q.ny;
    const long long cg = ((long long)(q.z0 + k) * g.N + (q.y0 + j)) * g.M + (q.x0 + i);
    T o = u[cl];
    if (HAS_Y) o += yin[cg];
    if (FINAL) {
      const double od = (double)o;
      out_d[cg] = od;
      dot += x[cg] * od;
    } else {
      out_t[cg] = o;
    }
  }
  if (FINAL) {
    dot = block_sum(dot, red);
    if (threadIdx.x == 0) part[blockIdx.x] = dot;
  }
}

template <typename T>
void launch_ic_apply(const Grid& g, const SubInfo* subs, int nsub, int max_lines, int max_cells, const T* tx,
                     const T* ty, const T* tz, const T* diag, const T* inv_d, const double* x, const T* yin,
                     T* out_t, double* out_d, double* part, const int* done, cudaStream_t st, int threads) {
  threads = std::max(threads, std::max(64, ((max_lines + 31) / 32) * 32));
  const int ldc = (max_cells + 3) & ~3;
  size_t smem = 32 * sizeof(double) + (size_t)5 * ldc * sizeof(T);
  const bool fin = out_d != nullptr;
  if (smem > 48 * 1024) {
    if (yin) {
      cudaFuncSetAttribute(k_ic_apply<T, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(k_ic_apply<T, true, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    } else {
      cudaFuncSetAttribute(k_ic_apply<T, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
      cudaFuncSetAttribute(k_ic_apply<T, false, false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    }
  }
  if (yin) {
    if (fin)
      { note_launch(); k_ic_apply<T, true, true><<<nsub, threads, smem, st>>>(g, subs, tx, ty, tz, diag, inv_d, x, yin, out_t, out_d, part, done, ldc); }
    else
      { note_launch(); k_ic_apply<T, true, false><<<nsub, threads, smem, st>>>(g, subs, tx, ty, tz, diag, inv_d, x, yin, out_t, out_d, part, done, ldc); }
  } else {
    if (fin)
      { note_launch(); k_ic_apply<T, false, true><<<nsub, threads, smem, st>>>(g, subs, tx, ty, tz, diag, inv_d, x, yin, out_t, out_d, part, done, ldc); }
    else
      { note_launch(); k_ic_apply<T, false, false><<<nsub, threads, smem, st>>>(g, subs, tx, ty, tz, diag, inv_d, x, yin, out_t, out_d, part, done, ldc); }
  }
}

// ---------------------------------------------------------------------------
// Level-2 restriction c_s = Phi_s^T (x - A y)|_s  (VecMDot in
// _PC_apply_vec_lv2, src/PreMixFEM_3D.c:1564) fused with the residual update
// r = x - A y of PC_apply_vec (:1859-1926): the residual is never stored.
template <typename T, int KM, bool HAS_Y>
__global__ void k_resid_restrict(Grid g, const SubInfo* subs, int kmax, const T* tx, const T* ty, const T* tz,
                                 const T* diag, const T* phi, const double* x, const T* y, double* c,
                                 const int* done) {
  if (done && *done) return;
  __shared__ double red[KM][33];
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  double acc[KM];
#pragma unroll
  for (int j = 0; j < KM; ++j) acc[j] = 0.0;
  for (int cl = threadIdx.x; cl < q.ncells; cl += blockDim.x) {
    const int i = cl % q.nx, tt = cl / q.nx, jj = tt % q.ny, k = tt / q.ny;
    const int ex = q.x0 + i, ey = q.y0 + jj, ez = q.z0 + k;
    const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
    T r = (T)x[cg];
    if (HAS_Y) r -= apply_A(g, cg, ex, ey, ez, tx, ty, tz, diag, y);
    const T* ph = phi + cg * kmax;
#pragma unroll
    for (int j = 0; j < KM; ++j)
      if (j < kmax) acc[j] += (double)(ph[j] * r);
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
#pragma unroll
  for (int j = 0; j < KM; ++j) {
    double v = warp_sum(acc[j]);
    if (lane == 0) red[j][wid] = v;
  }
  __syncthreads();
  if (threadIdx.x < kmax) {
    double v = 0.0;
    for (int w = 0; w < nw; ++w) v += red[threadIdx.x][w];
    c[(long long)blockIdx.x * kmax + threadIdx.x] = v;
  }
}

template <typename T, int KM>
static void rr_dispatch(const Grid& g, const SubInfo* subs, int nsub, int kmax, const T* tx, const T* ty,
                        const T* tz, const T* diag, const T* phi, const double* x, const T* y, double* c,
                        const int* done, cudaStream_t st, int threads) {
  if (y)
    { note_launch(); k_resid_restrict<T, KM, true><<<nsub, threads, 0, st>>>(g, subs, kmax, tx, ty, tz, diag, phi, x, y, c, done); }
  else
    { note_launch(); k_resid_restrict<T, KM, false><<<nsub, threads, 0, st>>>(g, subs, kmax, tx, ty, tz, diag, phi, x, y, c, done); }
}

template <typename T>
void launch_resid_restrict(const Grid& g, const SubInfo* subs, int nsub, int kmax, const T* tx, const T* ty,
                           const T* tz, const T* diag, const T* phi, const double* x, const T* y, double* c,
                           const int* done, cudaStream_t st, int threads) {
  threads = (threads >= 32 && threads <= 1024 && threads % 32 == 0) ? threads : 256;
  if (kmax <= 4)
    rr_dispatch<T, 4>(g, subs, nsub, kmax, tx, ty, tz, diag, phi, x, y, c, done, st, threads);
  else if (kmax <= 8)
    rr_dispatch<T, 8>(g, subs, nsub, kmax, tx, ty, tz, diag, phi, x, y, c, done, st, threads);
  else
    rr_dispatch<T, 16>(g, subs, nsub, kmax, tx, ty, tz, diag, phi, x, y, c, done, st, threads);
}

// Prolongation y += Phi_s Z_s (VecMAXPY in _PC_apply_vec_lv2, :1578).
template <typename T, int KM>
__global__ void k_prolong(Grid g, const SubInfo* subs, int kmax, const T* phi, const double* Z, T* y,
                          const int* done) {
  if (done && *done) return;
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  T z[KM];
#pragma unroll
  for (int j = 0; j < KM; ++j) z[j] = j < kmax ? (T)Z[(long long)blockIdx.x * kmax + j] : (T)0;
  for (int cl = threadIdx.x; cl < q.ncells; cl += blockDim.x) {
    const int i = cl % q.nx, tt = cl / q.nx, jj = tt % q.ny, k = tt / q.ny;
    const long long cg = ((long long)(q.z0 + k) * g.N + (q.y0 + jj)) * g.M + (q.x0 + i);
    const T* ph = phi + cg * kmax;
    T v = y[cg];
#pragma unroll
    for (int j = 0; j < KM; ++j)
      if (j < kmax) v += ph[j] * z[j];
    y[cg] = v;
  }
}

template <typename T>
void launch_prolong(const Grid& g, const SubInfo* subs, int nsub, int kmax, const T* phi, const double* Z, T* y,
                    const int* done, cudaStream_t st, int threads) {
  threads = (threads >= 32 && threads <= 1024 && threads % 32 == 0) ? threads : 256;
  if (kmax <= 4)
    { note_launch(); k_prolong<T, 4><<<nsub, threads, 0, st>>>(g, subs, kmax, phi, Z, y, done); }
  else if (kmax <= 8)
    { note_launch(); k_prolong<T, 8><<<nsub, threads, 0, st>>>(g, subs, kmax, phi, Z, y, done); }
  else
    { note_launch(); k_prolong<T, 16><<<nsub, threads, 0, st>>>(g, subs, kmax, phi, Z, y, done); }
}

// ---------------------------------------------------------------------------
// Exact level-1 local solves (-use_full_Cholesky_lv1, src/PreMixFEM_3D.c:205-207,
// where the reference switches the local KSP from ICC(0) to a full Cholesky):
// banded Cholesky L L^T of every subdomain's principal block in natural
// order.  The lower bandwidth is b = nx*ny; column j of L holds L(j + d, j),
// d = 0..b, at band[boff[s] + j * ld + d] with ld = band_ld(b) (a multiple of
// 4, zero past the last row).
constexpr int kCholW = 8;  // panel width of the factorisation

__host__ __device__ inline int band_ld(int b) { return (b + 1 + 3) & ~3; }
int band_ld_host(int b) { return band_ld(b); }

// Blocked left-looking factorisation, one CTA per subdomain, FP64.  For each
// panel of kCholW columns: the panel rows (b + kCholW of them) start from A and
// subtract sum_q L(i, q) L(j0 + c, q) over the previous b columns (one thread
// per row, the multipliers staged in shared memory), then the panel is
// factored in shared memory and written out.  Non-positive pivots are counted
// in *bad (and replaced by 1 so that the factor stays finite).
__global__ void __launch_bounds__(256) k_band_chol_factor(Grid g, const SubInfo* subs, const double* tx,
                                                          const double* ty, const double* tz, const double* diag,
                                                          const long long* boff, double* band, int* bad) {
  extern __shared__ double chs[];
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  const int n = q.ncells, b = q.nxny, ld = band_ld(b);
  double* L = band + boff[blockIdx.x];
  double* P = chs;                     // (b + kCholW) x kCholW panel, P[r * kCholW + c]
  double* Mq = P + (b + kCholW) * kCholW;  // Mq[(qc - qlo) * kCholW + c] = L(j0 + c, qc)
  int nbad = 0;
  for (int j0 = 0; j0 < n; j0 += kCholW) {
    const int wc = min(kCholW, n - j0);
    const int rows = min(n - j0, b + wc);
    const int qlo = max(0, j0 - b);
    const int nq = j0 - qlo;
    for (int e = threadIdx.x; e < nq * kCholW; e += blockDim.x) {
      const int qq = e / kCholW, c = e - qq * kCholW;
      const int qc = qlo + qq, d = j0 + c - qc;
      Mq[e] = (c < wc && d <= b) ? L[(long long)qc * ld + d] : 0.0;
    }
    __syncthreads();
    for (int r = threadIdx.x; r < rows; r += blockDim.x) {
      const int i = j0 + r;
      const int ii = i % q.nx, tt = i / q.nx, jj = tt % q.ny, kk = tt / q.ny;
      const long long cg = ((long long)(q.z0 + kk) * g.N + (q.y0 + jj)) * g.M + (q.x0 + ii);
      double acc[kCholW];
#pragma unroll
      for (int c = 0; c < kCholW; ++c) {
        const int dd = i - (j0 + c);
        double a = 0.0;
        if (c < wc) {
          if (dd == 0)
            a = diag[cg];
          else if (dd == 1 && ii > 0)
            a = -tx[cg];
          else if (dd == q.nx && jj > 0)
            a = -ty[cg];
          else if (dd == q.nxny && kk > 0)
            a = -tz[cg];
        }
        acc[c] = a;
      }
      for (int qc = max(qlo, i - b); qc < j0; ++qc) {
        const double lv = L[(long long)qc * ld + (i - qc)];
        const double* m = Mq + (qc - qlo) * kCholW;
#pragma unroll
        for (int c = 0; c < kCholW; ++c) acc[c] -= lv * m[c];
      }
#pragma unroll
      for (int c = 0; c < kCholW; ++c) P[r * kCholW + c] = acc[c];
    }
    __syncthreads();
    for (int c = 0; c < wc; ++c) {
      if (threadIdx.x == 0) {
        double d = P[c * kCholW + c];
        if (!(d > 0.0)) {
          ++nbad;
          d = 1.0;
        }
        P[c * kCholW + c] = sqrt(d);
      }
      __syncthreads();
      const double piv = P[c * kCholW + c];
      for (int r = c + 1 + threadIdx.x; r < rows; r += blockDim.x) P[r * kCholW + c] /= piv;
      __syncthreads();
      for (int r = c + 1 + threadIdx.x; r < rows; r += blockDim.x) {
        const double lrc = P[r * kCholW + c];
        for (int c2 = c + 1; c2 < wc; ++c2)
          if (r >= c2) P[r * kCholW + c2] -= lrc * P[c2 * kCholW + c];
      }
      __syncthreads();
    }
    for (int e = threadIdx.x; e < wc * ld; e += blockDim.x) {
      const int c = e / ld, d = e - c * ld;
      L[(long long)(j0 + c) * ld + d] = (d <= b && c + d < rows) ? P[(c + d) * kCholW + c] : 0.0;
    }
    __syncthreads();
  }
  if (threadIdx.x == 0 && nbad) atomicAdd(bad, nbad);
}

void launch_band_chol_factor(const Grid& g, const SubInfo* subs, int nsub, int max_b, const double* tx,
                             const double* ty, const double* tz, const double* diag, const long long* boff,
                             double* band, int* bad, cudaStream_t st) {
  const int smem = (2 * max_b + kCholW) * kCholW * (int)sizeof(double);
  if (smem > 48 * 1024) cudaFuncSetAttribute(k_band_chol_factor, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);
  { note_launch(); k_band_chol_factor<<<nsub, 256, smem, st>>>(g, subs, tx, ty, tz, diag, boff, band, bad); }
}

// out = yin + (L L^T)^-1 (x - A yin), one warp per subdomain: the right-hand
// side goes to shared memory, then a column-oriented forward substitution
// (w_j = u_j / L_jj; u_{j+d} -= L(j+d, j) w_j across the lanes) and a dot-
// product backward substitution (z_j = (w_j - sum_d L(j+d, j) z_{j+d}) / L_jj).
template <typename T, bool HAS_Y, bool FINAL>
__global__ void __launch_bounds__(32) k_band_chol_apply(Grid g, const SubInfo* subs, const T* tx, const T* ty,
                                                        const T* tz, const T* diag, const long long* boff,
                                                        const T* band, const double* x, const T* yin, T* out_t,
                                                        double* out_d, double* part, const int* done) {
  if (done && *done) return;
  extern __shared__ __align__(16) unsigned char chu_raw[];
  T* u = reinterpret_cast<T*>(chu_raw);
  const SubGeom q = sub_geom(subs[blockIdx.x]);
  const int n = q.ncells, b = q.nxny, ld = band_ld(b);
  const T* L = band + boff[blockIdx.x];
  const int lane = threadIdx.x;
  for (int cl = lane; cl < n; cl += 32) {
    const int i = cl % q.nx, tt = cl / q.nx, j = tt % q.ny, k = tt / q.ny;
    const int ex = q.x0 + i, ey = q.y0 + j, ez = q.z0 + k;
    const long long cg = ((long long)ez * g.N + ey) * g.M + ex;
    T r = (T)x[cg];
    if (HAS_Y) r -= apply_A(g, cg, ex, ey, ez, tx, ty, tz, diag, yin);
    u[cl] = r;
  }
  __syncwarp();
  for (int j = 0; j < n; ++j) {
    const T* col = L + (long long)j * ld;
    const T wj = u[j] / col[0];
    const int dmax = min(b, n - 1 - j);
    __syncwarp();
    if (lane == 0) u[j] = wj;
#pragma unroll 4
    for (int d = 1 + lane; d <= dmax; d += 32) u[j + d] -= col[d] * wj;
    __syncwarp();
  }
  for (int j = n - 1; j >= 0; --j) {
    const T* col = L + (long long)j * ld;
    const int dmax = min(b, n - 1 - j);
    T sacc = (T)0;
#pragma unroll 4
    for (int d = 1 + lane; d <= dmax; d += 32) sacc += col[d] * u[j + d];
    sacc = warp_sum(sacc);
    if (lane == 0) u[j] = (u[j] - sacc) / col[0];
    __syncwarp();
  }
  double dot = 0.0;
  for (int cl = lane; cl < n; cl += 32) {
    const int i = cl % q.nx, tt = cl / q.nx, j = tt % q.ny, k = tt / q.ny;
    const long long cg = ((long long)(q.z0 + k) * g.N + (q.y0 + j)) * g.M + (q.x0 + i);
    T o = u[cl];
    if (HAS_Y) o += yin[cg];
    if (FINAL) {
      const double od = (double)o;
      out_d[cg] = od;
      dot += x[cg] * od;
    } else {
      out_t[cg] = o;
    }
  }
  if (FINAL) {
    dot = warp_sum(dot);
    if (lane == 0) part[blockIdx.x] = dot;
  }
}

template <typename T>
void launch_band_chol_apply(const Grid& g, const SubInfo* subs, int nsub, int max_cells, const T* tx, const T* ty,
                            const T* tz, const T* diag, const long long* boff, const T* band, const double* x,
                            const T* yin, T* out_t, double* out_d, double* part, const int* done, cudaStream_t st) {
  const int smem = max_cells * (int)sizeof(T);
  const bool fin = out_d != nullptr;
#define PMF_BCH(HY, FN)                                                                                        \
  {                                                                                                            \
    if (smem > 48 * 1024)                                                                                      \
      cudaFuncSetAttribute(k_band_chol_apply<T, HY, FN>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem);   \
    note_launch();                                                                                             \
    k_band_chol_apply<T, HY, FN><<<nsub, 32, smem, st>>>(g, subs, tx, ty, tz, diag, boff, band, x, yin, out_t, \
                                                         out_d, part, done);                                   \
  }
  if (yin) {
    if (fin) PMF_BCH(true, true) else PMF_BCH(true, false)
  } else {
    if (fin) PMF_BCH(false, true) else PMF_BCH(false, false)
  }
#undef PMF_BCH
}

#define PMF_INST(T)                                                                                              \
  template void launch_ic_apply<T>(const Grid&, const SubInfo*, int, int, int, const T*, const T*, const T*,      \
                                   const T*, const T*, const double*, const T*, T*, double*, double*, const int*, \
                                   cudaStream_t, int);                                                           \
  template void launch_resid_restrict<T>(const Grid&, const SubInfo*, int, int, const T*, const T*, const T*,     \
                                         const T*, const T*, const double*, const T*, double*, const int*,        \
                                         cudaStream_t, int);                                                      \
  template void launch_prolong<T>(const Grid&, const SubInfo*, int, int, const T*, const double*, T*, const int*, \
                                  cudaStream_t, int);                                                           \
  template void launch_band_chol_apply<T>(const Grid&, const SubInfo*, int, int, const T*, const T*, const T*,   \
                                          const T*, const long long*, const T*, const double*, const T*, T*,     \
                                          double*, double*, const int*, cudaStream_t);
PMF_INST(float)
PMF_INST(double)
#undef PMF_INST

}  // namespace pmf
