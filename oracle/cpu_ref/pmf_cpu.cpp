// CPU restatement (C++17 / OpenMP, FP64) of the three-level GMsFEM-preconditioned
// CG solve of the lumped RT0-P0 Darcy operator.  TEST INFRASTRUCTURE and the timed
// CPU baseline: the library never links or calls it.
//
// It follows src/PreMixFEM_3D.c of Laphet/PreMixFEM: operator (PC_create_A,
// :1757-1824), partition (_PC_setup_lv1_partition, :47-78), level 1 IC(0) of each
// subdomain's principal block (:80-222, applied :1429-1479), level 2 local GHEPs
// A_i^N v = lambda M_i v with the MOD / MEAN / DIAG mass (:224-421), per-rank
// Galerkin blocks Phi^T A Phi and their Cholesky factors (:737-916), level 3
// rank-Neumann HEP (:918-1175) and Psi^T A Psi + NIL I (:1177-1390), the V/W
// cycle with a full residual before every visit (:1840-1936) and PETSc's CG with
// the unpreconditioned norm and a zero initial guess.
//
// The reference's third-party solvers are replaced by published algorithms
// written here: SLEPc's Krylov-Schur on the local GHEPs by LOBPCG (Knyazev 2001)
// with SVQB orthonormalisation (Stathopoulos & Wu 2002) preconditioned by IC(0)
// of A^N + sigma M; the level-3 HEP and the Rayleigh-Ritz problems by
// Householder tridiagonalisation and the implicit symmetric QR step with a
// Wilkinson shift (Golub & Van Loan, Matrix Computations, Alg. 8.3.1-8.3.3),
// a level-3 HEP of more than 256 coarse unknowns by inverse subspace iteration
// for its smallest eigenpairs (Alg. 8.2.3 with a Rayleigh-Ritz step);
// MUMPS / SuperLU by a dense Cholesky factorisation that drops null pivots;
// CHOLMOD (-use_full_Cholesky_lv1) by a band Cholesky of each subdomain block
// (Golub & Van Loan, Alg. 4.3.5).  Adaptive eigenvector counts (-eb_lv1,
// -eb_lv2, :369-383 and :1100-1115) are kept as zero basis columns, which the
// null-pivot Cholesky factors and the level-3 right-hand sides then ignore.
// tests/test_cpu_ref.py checks it against the NumPy oracle (oracle/pmf_oracle.py).
#include <omp.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <random>
#include <vector>

namespace {

constexpr double NIL = 1.0e-12;  // src/PreMixFEM_3D.h:15

using Vec = std::vector<double>;

struct Box {
  int x0, nx, y0, ny, z0, nz, rank;
  int n() const { return nx * ny * nz; }
};

// Near-equal split, the first n % parts pieces one longer (src/PreMixFEM_3D.c:62-71).
void split(int n, int parts, std::vector<int>& st, std::vector<int>& len) {
  st.assign(parts, 0);
  len.assign(parts, 0);
  for (int i = 0; i < parts; ++i) len[i] = n / parts + ((n % parts) > i ? 1 : 0);
  for (int i = 1; i < parts; ++i) st[i] = st[i - 1] + len[i - 1];
}

struct Problem {
  int M = 0, N = 0, P = 0;
  long long n = 0, MN = 0;
  double Hx = 0, Hy = 0, Hz = 0, meas = 0;
  const double *kx = nullptr, *ky = nullptr, *kz = nullptr;
  Vec tx, ty, tz, diag, db, bval;
  int dir_on[6] = {0, 0, 0, 0, 0, 0};
  long long id(int x, int y, int z) const { return ((long long)z * N + y) * M + x; }
};

// ---- dense linear algebra (row-major n x n) ------------------------------------------

// Cholesky L L^T = A, lower factor in place.  A pivot <= rel_tol * max|diag| marks a
// null direction: its column of L is zero with a unit pivot, and solves zero it.
void chol_semidef(Vec& A, int n, std::vector<char>& null, double rel_tol = 1e-14) {
  double scale = 1e-300;
  for (int i = 0; i < n; ++i) scale = std::max(scale, std::fabs(A[(size_t)i * n + i]));
  null.assign(n, 0);
  for (int j = 0; j < n; ++j) {
    double* rj = &A[(size_t)j * n];
    double d = rj[j];
    for (int q = 0; q < j; ++q) d -= rj[q] * rj[q];
    if (d <= rel_tol * scale) {
      null[j] = 1;
      for (int i = j + 1; i < n; ++i) A[(size_t)i * n + j] = 0.0;
      rj[j] = 1.0;
      continue;
    }
    const double l = std::sqrt(d);
    rj[j] = l;
#pragma omp parallel for schedule(static) if (n - j > 256)
    for (int i = j + 1; i < n; ++i) {
      double* ri = &A[(size_t)i * n];
      double v = ri[j];
      for (int q = 0; q < j; ++q) v -= ri[q] * rj[q];
      ri[j] = v / l;
    }
  }
  for (int i = 0; i < n; ++i)
    for (int j = i + 1; j < n; ++j) A[(size_t)i * n + j] = 0.0;
}

void chol_solve(const Vec& L, const std::vector<char>& null, int n, double* b) {
  for (int i = 0; i < n; ++i) {
    const double* ri = &L[(size_t)i * n];
    double v = b[i];
    for (int q = 0; q < i; ++q) v -= ri[q] * b[q];
    b[i] = null[i] ? 0.0 : v / ri[i];
  }
  for (int i = n - 1; i >= 0; --i) {
    double v = b[i];
    for (int q = i + 1; q < n; ++q) v -= L[(size_t)q * n + i] * b[q];
    b[i] = null[i] ? 0.0 : v / L[(size_t)i * n + i];
  }
}

// Symmetric eigendecomposition A = Q diag(w) Q^T, w ascending, Q row-major with the
// eigenvectors in its columns.  Householder reduction to tridiagonal form with the
// reflections accumulated into Q, then implicit symmetric QR steps with the Wilkinson
// shift, chasing the bulge with Givens rotations, and deflation of negligible
// off-diagonal entries.
void sym_eig(Vec A, int n, Vec& w, Vec& Q) {
  Q.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; ++i) Q[(size_t)i * n + i] = 1.0;
  Vec v(n), p(n), wv(n);
  for (int k = 0; k + 2 < n; ++k) {
    const int m = n - k - 1;  // length of column k below the diagonal
    double sigma = 0.0;
    const double x0 = A[(size_t)(k + 1) * n + k];
    for (int i = 1; i < m; ++i) {
      const double xi = A[(size_t)(k + 1 + i) * n + k];
      sigma += xi * xi;
    }
    if (sigma == 0.0) continue;  // column already reduced
    const double mu = std::sqrt(x0 * x0 + sigma);
    const double v0 = x0 <= 0.0 ? x0 - mu : -sigma / (x0 + mu);
    const double beta = 2.0 * v0 * v0 / (sigma + v0 * v0);
    v[0] = 1.0;
    for (int i = 1; i < m; ++i) v[i] = A[(size_t)(k + 1 + i) * n + k] / v0;
    // p = beta A22 v, w = p - (beta p.v / 2) v, A22 -= v w^T + w v^T
    double pv = 0.0;
    for (int i = 0; i < m; ++i) {
      const double* ri = &A[(size_t)(k + 1 + i) * n + k + 1];
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += ri[j] * v[j];
      p[i] = beta * s;
      pv += p[i] * v[i];
    }
    for (int i = 0; i < m; ++i) wv[i] = p[i] - 0.5 * beta * pv * v[i];
    for (int i = 0; i < m; ++i) {
      double* ri = &A[(size_t)(k + 1 + i) * n + k + 1];
      for (int j = 0; j < m; ++j) ri[j] -= v[i] * wv[j] + wv[i] * v[j];
    }
    A[(size_t)(k + 1) * n + k] = A[(size_t)k * n + k + 1] = mu;
    for (int i = 1; i < m; ++i) A[(size_t)(k + 1 + i) * n + k] = A[(size_t)k * n + k + 1 + i] = 0.0;
    // Q <- Q H_k, H_k = I - beta v v^T acting on indices k+1 .. n-1
    for (int r = 0; r < n; ++r) {
      double* qr = &Q[(size_t)r * n + k + 1];
      double s = 0.0;
      for (int j = 0; j < m; ++j) s += qr[j] * v[j];
      s *= beta;
      for (int j = 0; j < m; ++j) qr[j] -= s * v[j];
    }
  }
  Vec d(n), e(n > 1 ? n - 1 : 1, 0.0);
  for (int i = 0; i < n; ++i) d[i] = A[(size_t)i * n + i];
  for (int i = 0; i + 1 < n; ++i) e[i] = A[(size_t)(i + 1) * n + i];
  const double eps = 2.2204460492503131e-16;
  int hi = n - 1, guard = 0;
  while (hi > 0 && guard < 60 * n) {
    if (std::fabs(e[hi - 1]) <= eps * (std::fabs(d[hi - 1]) + std::fabs(d[hi]))) {
      e[hi - 1] = 0.0;
      --hi;
      continue;
    }
    int lo = hi - 1;
    while (lo > 0 && std::fabs(e[lo - 1]) > eps * (std::fabs(d[lo - 1]) + std::fabs(d[lo]))) --lo;
    ++guard;
    // Wilkinson shift: the eigenvalue of the trailing 2x2 block nearer its last entry
    const double dd = 0.5 * (d[hi - 1] - d[hi]);
    const double den = dd + (dd >= 0.0 ? 1.0 : -1.0) * std::hypot(dd, e[hi - 1]);
    const double shift = d[hi] - (den != 0.0 ? e[hi - 1] * e[hi - 1] / den : 0.0);
    double x = d[lo] - shift, z = e[lo];
    for (int k = lo; k < hi; ++k) {
      const double r = std::hypot(x, z);
      const double c = r == 0.0 ? 1.0 : x / r, s = r == 0.0 ? 0.0 : z / r;
      if (k > lo) e[k - 1] = r;
      const double ak = d[k], ak1 = d[k + 1], bk = e[k];
      d[k] = c * c * ak + 2.0 * c * s * bk + s * s * ak1;
      d[k + 1] = s * s * ak - 2.0 * c * s * bk + c * c * ak1;
      e[k] = c * s * (ak1 - ak) + (c * c - s * s) * bk;
      if (k + 1 < hi) {
        z = s * e[k + 1];  // bulge at (k + 2, k)
        e[k + 1] = c * e[k + 1];
        x = e[k];
      }
      for (int r2 = 0; r2 < n; ++r2) {
        double* qr = &Q[(size_t)r2 * n];
        const double a0 = qr[k], a1 = qr[k + 1];
        qr[k] = c * a0 + s * a1;
        qr[k + 1] = -s * a0 + c * a1;
      }
    }
  }
  std::vector<int> ord(n);
  for (int i = 0; i < n; ++i) ord[i] = i;
  std::sort(ord.begin(), ord.end(), [&](int a, int b) { return d[a] < d[b]; });
  w.resize(n);
  Vec Q2((size_t)n * n);
  for (int j = 0; j < n; ++j) {
    w[j] = d[ord[j]];
    for (int i = 0; i < n; ++i) Q2[(size_t)i * n + j] = Q[(size_t)i * n + ord[j]];
  }
  Q.swap(Q2);
}

// The k smallest eigenpairs of a symmetric positive semidefinite A (n x n, row-major)
// by inverse subspace iteration: block p = min(n, k + 4), Y = (A + s I)^-1 X with a
// Cholesky factor (s = 1e-10 max diag, so that null directions stay solvable), an
// orthonormal basis of Y, Rayleigh-Ritz on it, until the k wanted residuals
// ||A v - t v|| fall below 1e-12 max diag.  w: k ascending values; V: n x k,
// eigenvector j in column j (V[i * k + j]).
void smallest_eig(const Vec& A, int n, int k, Vec& w, Vec& V) {
  const int p = std::min(n, k + 4);
  double dmax = 0.0;
  for (int i = 0; i < n; ++i) dmax = std::max(dmax, A[(size_t)i * n + i]);
  Vec L = A;
  for (int i = 0; i < n; ++i) L[(size_t)i * n + i] += 1e-10 * dmax;
  std::vector<char> nl;
  chol_semidef(L, n, nl);
  Vec X((size_t)n * p), Y((size_t)n * p), AY((size_t)n * p), th, Z;
  unsigned long long st = 0x2545F4914F6CDD1Dull;
  for (auto& v : X) {
    st = st * 6364136223846793005ull + 1442695040888963407ull;
    v = (double)(st >> 11) / 9007199254740992.0 - 0.5;
  }
  for (int it = 0; it < 300; ++it) {
#pragma omp parallel for schedule(static) if (n > 512)
    for (int c = 0; c < p; ++c) {
      Vec col(n);
      for (int i = 0; i < n; ++i) col[i] = X[(size_t)i * p + c];
      chol_solve(L, nl, n, col.data());
      for (int i = 0; i < n; ++i) Y[(size_t)i * p + c] = col[i];
    }
    for (int pass = 0; pass < 2; ++pass)  // modified Gram-Schmidt, twice
      for (int c = 0; c < p; ++c) {
        for (int b = 0; b < c; ++b) {
          double d = 0.0;
          for (int i = 0; i < n; ++i) d += Y[(size_t)i * p + b] * Y[(size_t)i * p + c];
          for (int i = 0; i < n; ++i) Y[(size_t)i * p + c] -= d * Y[(size_t)i * p + b];
        }
        double nn = 0.0;
        for (int i = 0; i < n; ++i) nn += Y[(size_t)i * p + c] * Y[(size_t)i * p + c];
        nn = nn > 0.0 ? 1.0 / std::sqrt(nn) : 0.0;
        for (int i = 0; i < n; ++i) Y[(size_t)i * p + c] *= nn;
      }
#pragma omp parallel for schedule(static) if (n > 512)
    for (int i = 0; i < n; ++i)
      for (int c = 0; c < p; ++c) {
        double v = 0.0;
        for (int q = 0; q < n; ++q) v += A[(size_t)i * n + q] * Y[(size_t)q * p + c];
        AY[(size_t)i * p + c] = v;
      }
    Vec H((size_t)p * p, 0.0);
    for (int a = 0; a < p; ++a)
      for (int b = 0; b < p; ++b) {
        double v = 0.0;
        for (int i = 0; i < n; ++i) v += Y[(size_t)i * p + a] * AY[(size_t)i * p + b];
        H[(size_t)a * p + b] = v;
      }
    for (int a = 0; a < p; ++a)
      for (int b = 0; b < a; ++b) H[(size_t)a * p + b] = H[(size_t)b * p + a] = 0.5 * (H[(size_t)a * p + b] + H[(size_t)b * p + a]);
    sym_eig(H, p, th, Z);
    double worst = 0.0;
    for (int i = 0; i < n; ++i) {
      double xr[64], ar[64];
      for (int j = 0; j < p; ++j) {
        double xv = 0.0, av = 0.0;
        for (int b = 0; b < p; ++b) {
          xv += Y[(size_t)i * p + b] * Z[(size_t)b * p + j];
          av += AY[(size_t)i * p + b] * Z[(size_t)b * p + j];
        }
        xr[j] = xv;
        ar[j] = av;
      }
      for (int j = 0; j < p; ++j) {
        X[(size_t)i * p + j] = xr[j];
        AY[(size_t)i * p + j] = ar[j] - th[j] * xr[j];  // residual, reusing AY
      }
    }
    for (int j = 0; j < k; ++j) {
      double r2 = 0.0;
      for (int i = 0; i < n; ++i) r2 += AY[(size_t)i * p + j] * AY[(size_t)i * p + j];
      worst = std::max(worst, std::sqrt(r2));
    }
    if (worst <= 1e-12 * dmax) break;
  }
  w.assign(th.begin(), th.begin() + k);
  V.assign((size_t)n * k, 0.0);
  for (int i = 0; i < n; ++i)
    for (int j = 0; j < k; ++j) V[(size_t)i * k + j] = X[(size_t)i * p + j];
}

// ---- operator (PC_create_A, :1757-1824) -------------------------------------------------
void assemble(Problem& p, const double dom[3], const int dir_on[6], const double dir_val[6]) {
  p.Hx = dom[0] / p.M;
  p.Hy = dom[1] / p.N;
  p.Hz = dom[2] / p.P;
  p.meas = p.Hx * p.Hy * p.Hz;
  const double fyz = p.Hy * p.Hz, fzx = p.Hz * p.Hx, fxy = p.Hx * p.Hy;
  const double cx = fyz * fyz / p.meas, cy = fzx * fzx / p.meas, cz = fxy * fxy / p.meas;
  const long long n = p.n, MN = p.MN;
  p.tx.assign(n, 0.0);
  p.ty.assign(n, 0.0);
  p.tz.assign(n, 0.0);
  p.db.assign(n, 0.0);
  p.bval.assign(n, 0.0);
  p.diag.assign(n, 0.0);
  for (int f = 0; f < 6; ++f) p.dir_on[f] = dir_on[f] ? 1 : 0;
#pragma omp parallel for schedule(static)
  for (int z = 0; z < p.P; ++z)
    for (int y = 0; y < p.N; ++y)
      for (int x = 0; x < p.M; ++x) {
        const long long c = p.id(x, y, z);
        if (x > 0) p.tx[c] = cx * (2.0 / (1.0 / p.kx[c - 1] + 1.0 / p.kx[c]));
        if (y > 0) p.ty[c] = cy * (2.0 / (1.0 / p.ky[c - p.M] + 1.0 / p.ky[c]));
        if (z > 0) p.tz[c] = cz * (2.0 / (1.0 / p.kz[c - MN] + 1.0 / p.kz[c]));
        double tb = 0.0, bv = 0.0;
        auto face = [&](int f, double t) {
          if (p.dir_on[f]) {
            tb += t;
            bv += t * dir_val[f];
          }
        };
        if (x == 0) face(0, cx * (2.0 * p.kx[c]));
        if (x == p.M - 1) face(1, cx * (2.0 * p.kx[c]));
        if (y == 0) face(2, cy * (2.0 * p.ky[c]));
        if (y == p.N - 1) face(3, cy * (2.0 * p.ky[c]));
        if (z == 0) face(4, cz * (2.0 * p.kz[c]));
        if (z == p.P - 1) face(5, cz * (2.0 * p.kz[c]));
        p.db[c] = tb;
        p.bval[c] = bv;
      }
  // diagonal in ADD_VALUES order: own low faces, then the ones the +x, +y, +z cells add
#pragma omp parallel for schedule(static)
  for (long long c = 0; c < n; ++c) {
    const int x = (int)(c % p.M), y = (int)((c / p.M) % p.N), z = (int)(c / MN);
    double d = p.tx[c] + p.ty[c];
    d = d + p.tz[c];
    if (x < p.M - 1) d += p.tx[c + 1];
    if (y < p.N - 1) d += p.ty[c + p.M];
    if (z < p.P - 1) d += p.tz[c + MN];
    p.diag[c] = d + p.db[c];
  }
}

void spmv(const Problem& p, const double* x, double* y) {
  const long long MN = p.MN;
#pragma omp parallel for schedule(static) collapse(2)
  for (int z = 0; z < p.P; ++z)
    for (int yy = 0; yy < p.N; ++yy) {
      const long long base = p.id(0, yy, z);
      for (int xx = 0; xx < p.M; ++xx) {
        const long long c = base + xx;
        double v = p.diag[c] * x[c];
        if (xx > 0) v -= p.tx[c] * x[c - 1];
        if (xx < p.M - 1) v -= p.tx[c + 1] * x[c + 1];
        if (yy > 0) v -= p.ty[c] * x[c - p.M];
        if (yy < p.N - 1) v -= p.ty[c + p.M] * x[c + p.M];
        if (z > 0) v -= p.tz[c] * x[c - MN];
        if (z < p.P - 1) v -= p.tz[c + MN] * x[c + MN];
        y[c] = v;
      }
    }
}

// ---- box-local operators (local cell index x-fastest) -----------------------------------
struct Local {
  const Problem* p;
  Box b;
};

// y = A_box v with the box's own diagonal dg (principal block or Neumann matrix).
void local_apply(const Local& L, const double* dg, const double* v, double* y) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  const int sxy = b.nx * b.ny;
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j) {
      const long long c0 = p.id(b.x0, b.y0 + j, b.z0 + k);
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const long long c = c0 + i;
        double a = dg[cl] * v[cl];
        if (i > 0) a -= p.tx[c] * v[cl - 1];
        if (i < b.nx - 1) a -= p.tx[c + 1] * v[cl + 1];
        if (j > 0) a -= p.ty[c] * v[cl - b.nx];
        if (j < b.ny - 1) a -= p.ty[c + p.M] * v[cl + b.nx];
        if (k > 0) a -= p.tz[c] * v[cl - sxy];
        if (k < b.nz - 1) a -= p.tz[c + p.MN] * v[cl + sxy];
        y[cl] = a;
      }
    }
}

// Diagonal of the principal block (neumann = false) or of the Neumann matrix: the
// principal block minus the transmissibilities of the faces leaving the box into the
// domain (:245-320); Dirichlet terms stay.
void local_diag(const Local& L, bool neumann, Vec& d) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  d.resize(b.n());
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j)
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const long long c = p.id(b.x0 + i, b.y0 + j, b.z0 + k);
        if (!neumann) {
          d[cl] = p.diag[c];
          continue;
        }
        double v = p.db[c];
        if (i > 0) v += p.tx[c];
        if (i < b.nx - 1) v += p.tx[c + 1];
        if (j > 0) v += p.ty[c];
        if (j < b.ny - 1) v += p.ty[c + p.M];
        if (k > 0) v += p.tz[c];
        if (k < b.nz - 1) v += p.tz[c + p.MN];
        d[cl] = v;
      }
}

// IC(0) of the box matrix with diagonal dg (+ shift * Ms), natural order; iD receives
// the reciprocal pivots.  For the 7-point pattern IC(0) keeps no fill, so
// D_i = a_ii - sum_{j<i} a_ij^2 / D_j and the factor is (D + L) D^-1 (D + L^T).  A
// non-positive pivot of the shifted matrix falls back to its diagonal (that factor only
// preconditions the eigensolver).
void ic0(const Local& L, const Vec& dg, const double* Ms, double shift, Vec& iD) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  const int sxy = b.nx * b.ny;
  iD.resize(b.n());
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j)
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const long long c = p.id(b.x0 + i, b.y0 + j, b.z0 + k);
        const double a = dg[cl] + (Ms ? shift * Ms[cl] : 0.0);
        double v = a;
        if (i > 0) v -= p.tx[c] * p.tx[c] * iD[cl - 1];
        if (j > 0) v -= p.ty[c] * p.ty[c] * iD[cl - b.nx];
        if (k > 0) v -= p.tz[c] * p.tz[c] * iD[cl - sxy];
        if (Ms && !(v > 0.0)) v = a;
        iD[cl] = 1.0 / v;
      }
}

// y = ((D + L) D^-1 (D + L^T))^-1 r on a box (iD = 1 / D); L holds the negated
// transmissibilities.
void ic0_solve(const Local& L, const Vec& iD, const double* r, double* y) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  const int sxy = b.nx * b.ny;
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j) {
      const long long c0 = p.id(b.x0, b.y0 + j, b.z0 + k);
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const long long c = c0 + i;
        double v = r[cl];
        if (i > 0) v += p.tx[c] * y[cl - 1];
        if (j > 0) v += p.ty[c] * y[cl - b.nx];
        if (k > 0) v += p.tz[c] * y[cl - sxy];
        y[cl] = v * iD[cl];
      }
    }
  cl = b.n() - 1;
  for (int k = b.nz - 1; k >= 0; --k)
    for (int j = b.ny - 1; j >= 0; --j) {
      const long long c0 = p.id(b.x0, b.y0 + j, b.z0 + k);
      for (int i = b.nx - 1; i >= 0; --i, --cl) {
        const long long c = c0 + i;
        double v = 0.0;
        if (i < b.nx - 1) v += p.tx[c + 1] * y[cl + 1];
        if (j < b.ny - 1) v += p.ty[c + p.M] * y[cl + b.nx];
        if (k < b.nz - 1) v += p.tz[c + p.MN] * y[cl + sxy];
        y[cl] += v * iD[cl];
      }
    }
}

// Exact Cholesky L L^T of a box's principal block with diagonal dg
// (-use_full_Cholesky_lv1, :205-207): natural order, half bandwidth hb = nx ny,
// band[i (hb + 1) + (i - j)] = L(i, j) for i - hb <= j <= i (band Cholesky,
// Golub & Van Loan Alg. 4.3.5, row by row).  Returns false on a non-positive pivot.
bool band_chol(const Local& L, const Vec& dg, Vec& band) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  const int n = b.n(), hb = b.nx * b.ny, w = hb + 1;
  band.assign((size_t)n * w, 0.0);
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j) {
      const long long c0 = p.id(b.x0, b.y0 + j, b.z0 + k);
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const long long c = c0 + i;
        double* row = &band[(size_t)cl * w];
        row[0] = dg[cl];
        if (i > 0) row[1] = -p.tx[c];
        if (j > 0) row[b.nx] = -p.ty[c];
        if (k > 0) row[hb] = -p.tz[c];
      }
    }
  for (int i = 0; i < n; ++i) {
    const int j0 = std::max(0, i - hb);
    double* Li = &band[(size_t)i * w];
    for (int j = j0; j <= i; ++j) {
      const double* Lj = &band[(size_t)j * w];
      double s = Li[i - j];
      for (int q = j0; q < j; ++q) s -= Li[i - q] * Lj[j - q];
      if (j < i) {
        Li[i - j] = s / Lj[0];
      } else {
        if (!(s > 0.0)) return false;
        Li[0] = std::sqrt(s);
      }
    }
  }
  return true;
}

// y = (L L^T)^-1 r with the band factor of band_chol.
void band_solve(const Vec& band, int n, int hb, const double* r, double* y) {
  const int w = hb + 1;
  for (int i = 0; i < n; ++i) {
    const double* Li = &band[(size_t)i * w];
    double s = r[i];
    for (int q = std::max(0, i - hb); q < i; ++q) s -= Li[i - q] * y[q];
    y[i] = s / Li[0];
  }
  for (int i = n - 1; i >= 0; --i) {
    const double* Li = &band[(size_t)i * w];
    const double yi = y[i] / Li[0];
    y[i] = yi;
    for (int q = std::max(0, i - hb); q < i; ++q) y[q] -= Li[i - q] * yi;
  }
}

// Mass diagonal M_i of the local GHEP (:243-346).  eg_op 0 (MOD) keeps the reference's
// x-direction accumulation: the face between local cells i-1 and i is added to cell i-1,
// so a cell counts its right face twice unless it ends its row, and its left face only
// when it starts the row.  1 (MEAN): kx + ky + kz.  2 (DIAG): the Neumann diagonal.
void mass_diag(const Local& L, int eg_op, const Vec& dN, Vec& Md) {
  const Problem& p = *L.p;
  const Box& b = L.b;
  Md.resize(b.n());
  auto hm = [](double a, double c) { return 2.0 / (1.0 / a + 1.0 / c); };
  int cl = 0;
  for (int k = 0; k < b.nz; ++k)
    for (int j = 0; j < b.ny; ++j)
      for (int i = 0; i < b.nx; ++i, ++cl) {
        const int ex = b.x0 + i, ey = b.y0 + j, ez = b.z0 + k;
        const long long c = p.id(ex, ey, ez);
        if (eg_op == 1) {
          Md[cl] = p.kx[c] + p.ky[c] + p.kz[c];
          continue;
        }
        if (eg_op == 2) {
          Md[cl] = dN[cl];
          continue;
        }
        double mv = 0.0;
        if (i == 0 && ex >= 1) mv += 2.0 * hm(p.kx[c - 1], p.kx[c]) / p.Hx / p.Hx;
        if (ex + 1 != p.M) mv += 2.0 * hm(p.kx[c], p.kx[c + 1]) / p.Hx / p.Hx;
        if (i + 1 < b.nx) mv += 2.0 * hm(p.kx[c], p.kx[c + 1]) / p.Hx / p.Hx;
        if (ey >= 1) mv += 2.0 * hm(p.ky[c - p.M], p.ky[c]) / p.Hy / p.Hy;
        if (ey + 1 != p.N) mv += 2.0 * hm(p.ky[c], p.ky[c + p.M]) / p.Hy / p.Hy;
        if (ez >= 1) mv += 2.0 * hm(p.kz[c - p.MN], p.kz[c]) / p.Hz / p.Hz;
        if (ez + 1 != p.P) mv += 2.0 * hm(p.kz[c], p.kz[c + p.MN]) / p.Hz / p.Hz;
        if (p.dir_on[0] && ex == 0) mv += 2.0 * (2.0 * p.kx[c]) / p.Hx / p.Hx;
        if (p.dir_on[1] && ex == p.M - 1) mv += 2.0 * (2.0 * p.kx[c]) / p.Hx / p.Hx;
        if (p.dir_on[2] && ey == 0) mv += 2.0 * (2.0 * p.ky[c]) / p.Hy / p.Hy;
        if (p.dir_on[3] && ey == p.N - 1) mv += 2.0 * (2.0 * p.ky[c]) / p.Hy / p.Hy;
        if (p.dir_on[4] && ez == 0) mv += 2.0 * (2.0 * p.kz[c]) / p.Hz / p.Hz;
        if (p.dir_on[5] && ez == p.P - 1) mv += 2.0 * (2.0 * p.kz[c]) / p.Hz / p.Hz;
        Md[cl] = mv * p.meas;
      }
}

// ---- local GHEP: LOBPCG -------------------------------------------------------------------
struct EigStat {
  int its = 0, converged = 0;
  Vec lam;  // the k lowest Ritz values of the last Rayleigh-Ritz step
};

// Smallest k eigenpairs of A^N v = lambda M v on a box; block size m = k + 2, soft
// locking of converged wanted columns.  Residual ||A x - lambda M x||_{M^-1} divided by
// max_i (A^N_ii / M_ii).  Xout: k M-orthonormal columns (column j at [j * n]).
EigStat lobpcg(const Local& L, int eg_op, int k, double tol, int max_it, double sigma_rel, double rel_floor,
               unsigned long long seed, Vec& Xout) {
  const int n = L.b.n();
  const int m = std::min(k + 2, n);
  constexpr int CH = 64;
  Vec dN, Md, D;
  local_diag(L, true, dN);
  mass_diag(L, eg_op, dN, Md);
  double lscale = 0.0;
  for (int i = 0; i < n; ++i) lscale = std::max(lscale, dN[i] / Md[i]);
  if (!(lscale > 0.0)) lscale = 1.0;
  ic0(L, dN, Md.data(), sigma_rel * lscale, D);
  Vec iMd(n);
  for (int i = 0; i < n; ++i) iMd[i] = 1.0 / Md[i];
  Vec X((size_t)n * m), AX((size_t)n * m), W((size_t)n * m), AW((size_t)n * m), P((size_t)n * m),
      AP((size_t)n * m), lam(m, 0.0);
  std::mt19937_64 rng(seed);
  std::uniform_real_distribution<double> U(-1.0, 1.0);
  for (auto& v : X) v = U(rng);
  for (int j = 0; j < m; ++j) local_apply(L, dN.data(), &X[(size_t)j * n], &AX[(size_t)j * n]);

  // Rayleigh-Ritz on the span of S: M-orthonormal basis by SVQB, then the projected
  // HEP; Y holds the coefficients of the m lowest Ritz vectors.  False when the basis
  // is numerically rank-deficient.
  auto rayleigh_ritz = [&](const std::vector<const double*>& S, const std::vector<const double*>& AS, Vec& Y) {
    const int ns = (int)S.size();
    Vec GM((size_t)ns * ns, 0.0), GA((size_t)ns * ns, 0.0), GB((size_t)ns * ns, 0.0);
    // chunks of CH cells keep the 2 ns vector pieces in L1 across the ns^2 / 2 products
    for (int i0 = 0; i0 < n; i0 += CH) {
      const int len = std::min(CH, n - i0);
      const double* mi = &Md[i0];
      for (int a = 0; a < ns; ++a)
        for (int b = 0; b <= a; ++b) {
          double gm = 0.0, ga = 0.0, gb = 0.0;
          const double *sa = S[a] + i0, *sb = S[b] + i0, *asa = AS[a] + i0, *asb = AS[b] + i0;
#pragma omp simd reduction(+ : gm, ga, gb)
          for (int i = 0; i < len; ++i) {
            gm += sa[i] * mi[i] * sb[i];
            ga += sa[i] * asb[i];
            gb += sb[i] * asa[i];
          }
          GM[(size_t)a * ns + b] += gm;
          GA[(size_t)a * ns + b] += ga;
          GB[(size_t)a * ns + b] += gb;
        }
    }
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b <= a; ++b) {
        GM[(size_t)b * ns + a] = GM[(size_t)a * ns + b];
        GA[(size_t)a * ns + b] = GA[(size_t)b * ns + a] = 0.5 * (GA[(size_t)a * ns + b] + GB[(size_t)a * ns + b]);
      }
    // unit M-norm scaling; a column whose M-norm is negligible against the
    // block's largest (search directions decay geometrically once X stops
    // moving) carries no direction and is left out (scale 0), as a clamped
    // scale would blow its rounding up into the projected matrix
    Vec dsc(ns), G2((size_t)ns * ns), ev, EV;
    double gmax = 0.0;
    for (int a = 0; a < ns; ++a) gmax = std::max(gmax, GM[(size_t)a * ns + a]);
    for (int a = 0; a < ns; ++a) {
      const double gaa = GM[(size_t)a * ns + a];
      dsc[a] = gaa > 1e-28 * gmax ? 1.0 / std::sqrt(gaa) : 0.0;
    }
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) G2[(size_t)a * ns + b] = GM[(size_t)a * ns + b] * dsc[a] * dsc[b];
    sym_eig(G2, ns, ev, EV);
    std::vector<int> keep;
    for (int c = 0; c < ns; ++c)
      if (ev[c] > 1e-13 * ev[ns - 1]) keep.push_back(c);
    const int q = (int)keep.size();
    if (q < m) return false;
    Vec Qc((size_t)ns * q);
    for (int a = 0; a < ns; ++a)
      for (int c = 0; c < q; ++c) Qc[(size_t)a * q + c] = dsc[a] * EV[(size_t)a * ns + keep[c]] / std::sqrt(ev[keep[c]]);
    Vec T((size_t)ns * q, 0.0), H((size_t)q * q, 0.0);
    for (int a = 0; a < ns; ++a)
      for (int b = 0; b < ns; ++b) {
        const double g = GA[(size_t)a * ns + b];
        for (int c = 0; c < q; ++c) T[(size_t)a * q + c] += g * Qc[(size_t)b * q + c];
      }
    for (int c = 0; c < q; ++c)
      for (int e = 0; e < q; ++e) {
        double v = 0.0;
        for (int a = 0; a < ns; ++a) v += Qc[(size_t)a * q + c] * T[(size_t)a * q + e];
        H[(size_t)c * q + e] = v;
      }
    for (int c = 0; c < q; ++c)
      for (int e = 0; e < c; ++e) H[(size_t)c * q + e] = H[(size_t)e * q + c] = 0.5 * (H[(size_t)c * q + e] + H[(size_t)e * q + c]);
    Vec th, Z;
    sym_eig(H, q, th, Z);
    Y.assign((size_t)ns * m, 0.0);
    for (int a = 0; a < ns; ++a)
      for (int j = 0; j < m; ++j) {
        double v = 0.0;
        for (int c = 0; c < q; ++c) v += Qc[(size_t)a * q + c] * Z[(size_t)c * q + j];
        Y[(size_t)a * m + j] = v;
      }
    for (int j = 0; j < m; ++j) lam[j] = th[j];
    return true;
  };
  // out[:, j] = sum_{a >= from} Y[a][j] S[a]
  auto combine = [&](const std::vector<const double*>& S, const Vec& Y, int from, Vec& out) {
    Vec t((size_t)n * m, 0.0);
    for (int i0 = 0; i0 < n; i0 += CH) {
      const int len = std::min(CH, n - i0);
      for (int j = 0; j < m; ++j) {
        double* tj = &t[(size_t)j * n + i0];
        for (int a = from; a < (int)S.size(); ++a) {
          const double y = Y[(size_t)a * m + j];
          const double* sa = S[a] + i0;
#pragma omp simd
          for (int i = 0; i < len; ++i) tj[i] += y * sa[i];
        }
      }
    }
    out.swap(t);
  };
  std::vector<const double*> S, AS;
  auto basis = [&](int na, bool withP) {
    S.clear();
    AS.clear();
    for (int j = 0; j < m; ++j) {
      S.push_back(&X[(size_t)j * n]);
      AS.push_back(&AX[(size_t)j * n]);
    }
    for (int c = 0; c < na; ++c) {
      S.push_back(&W[(size_t)c * n]);
      AS.push_back(&AW[(size_t)c * n]);
    }
    if (withP)
      for (int j = 0; j < m; ++j) {
        S.push_back(&P[(size_t)j * n]);
        AS.push_back(&AP[(size_t)j * n]);
      }
  };
  Vec Y;
  basis(0, false);
  if (rayleigh_ritz(S, AS, Y)) {
    Vec Xn, AXn;
    combine(S, Y, 0, Xn);
    combine(AS, Y, 0, AXn);
    X.swap(Xn);
    AX.swap(AXn);
  }
  EigStat st;
  bool hasP = false;
  Vec rcol(n);
  int it = 0;
  for (; it < max_it; ++it) {
    bool conv = true;
    int na = 0;
    for (int j = 0; j < m; ++j) {
      double s = 0.0;
      const double *axj = &AX[(size_t)j * n], *xj = &X[(size_t)j * n];
      const double lj = lam[j];
#pragma omp simd reduction(+ : s)
      for (int i = 0; i < n; ++i) {
        const double r = axj[i] - lj * Md[i] * xj[i];
        rcol[i] = r;
        s += r * r * iMd[i];
      }
      // residual scale: lscale, or max(|lambda_j|, rel_floor lscale) (eigenvalue-relative)
      const double rs = rel_floor > 0.0 ? std::max(std::fabs(lj), rel_floor * lscale) : lscale;
      const bool done = std::sqrt(s) / rs <= tol;
      if (j < k && !done) conv = false;
      if (!done || j >= k) {  // soft locking: converged wanted columns leave the search
        ic0_solve(L, D, rcol.data(), &W[(size_t)na * n]);
        ++na;
      }
    }
    if (conv) {
      st.converged = 1;
      break;
    }
    for (int c = 0; c < na; ++c) local_apply(L, dN.data(), &W[(size_t)c * n], &AW[(size_t)c * n]);
    bool withP = hasP;
    basis(na, withP);
    if (!rayleigh_ritz(S, AS, Y)) {
      if (!withP) break;
      withP = false;  // drop the search directions and retry on [X, W]
      basis(na, false);
      if (!rayleigh_ritz(S, AS, Y)) break;
    }
    Vec Pn, APn, Xn, AXn;
    combine(S, Y, m, Pn);
    combine(AS, Y, m, APn);
    combine(S, Y, 0, Xn);
    combine(AS, Y, 0, AXn);
    X.swap(Xn);
    AX.swap(AXn);
    P.swap(Pn);
    AP.swap(APn);
    hasP = true;
  }
  st.its = it;
  st.lam.assign(lam.begin(), lam.begin() + k);
  Xout.assign((size_t)n * k, 0.0);
  for (int j = 0; j < k; ++j) {
    double s = 0.0;
    for (int i = 0; i < n; ++i) s += X[(size_t)j * n + i] * Md[i] * X[(size_t)j * n + i];
    s = 1.0 / std::sqrt(s);
    for (int i = 0; i < n; ++i) Xout[(size_t)j * n + i] = X[(size_t)j * n + i] * s;
  }
  return st;
}

}  // namespace

extern "C" {

// Setup + PCG solve with the three-level preconditioner (FP64).
//   mesh[3] M N P; dom[3] domain lengths; kx, ky, kz cell permeabilities (ky / kz may be
//   null: isotropic); source per cell; dir_on[6] / dir_val[6] Dirichlet faces
//   x- x+ y- y+ z- z+ and their pressures.
//   iopt[20]: sd[3], vranks[3], en_lv1, en_lv2, si_lv1, si_lv2, use_W_cycle, max_it,
//             eig_max_it, eg_op, threads (<= 0: the OpenMP default), constant null
//             space (-ksp_constant_null_space: every preconditioned residual loses its
//             mean), no_shift_A_cc, use_2level, use_full_Cholesky_lv1, nrhs
//   dopt[6]:  rtol, eig_tol, eig_sigma (IC(0) shift of the eigensolver, x max A_ii/M_ii),
//             eig_rel_floor (> 0: eigen residual test relative to max(|lambda|, floor x
//             lscale)), eb_lv1, eb_lv2 (< 0: 1 / NIL, every subdomain keeps en_lv1 and
//             every rank en_lv2 vectors)
//   x_out[nrhs n]: solutions; info[12]: its, setup_s, solve_s (all right-hand
//             sides), threads, eig_its_mean, eig_its_max, eig_unconverged,
//             ||r_final||, ||r_0|| (its, ||r|| of the first right-hand side), level-3
//             size, its summed and the largest over the right-hand sides
//   source[nrhs n]: nrhs = iopt[19] right-hand sides solved after one set-up
// Returns 0, -1 for invalid arguments, -2 when a subdomain block of
// -use_full_Cholesky_lv1 is not positive definite.
int pmf_cpu_solve(const int* mesh, const double* dom, const double* kx, const double* ky, const double* kz,
                  const double* source, const int* dir_on, const double* dir_val, const int* iopt,
                  const double* dopt, double* x_out, double* info) {
  using clk = std::chrono::steady_clock;
  if (!mesh || !dom || !kx || !source || !dir_on || !dir_val || !iopt || !dopt || !x_out) return -1;
  const int sd[3] = {iopt[0], iopt[1], iopt[2]}, vr[3] = {iopt[3], iopt[4], iopt[5]};
  const int k = iopt[6], en2_in = iopt[7], si1 = std::max(1, iopt[8]), si2 = std::max(1, iopt[9]);
  const int wcycle = iopt[10], max_it = iopt[11], eig_max_it = iopt[12], eg_op = iopt[13], threads = iopt[14];
  const bool null_space = iopt[15] != 0, no_shift = iopt[16] != 0, two_level = iopt[17] != 0,
             full_chol = iopt[18] != 0;
  const int nrhs = iopt[19];
  const double rtol = dopt[0], eig_tol = dopt[1], eig_sigma = dopt[2], eig_rel_floor = dopt[3];
  const double eb1 = dopt[4] < 0.0 ? 1.0 / NIL : dopt[4], eb2 = dopt[5] < 0.0 ? 1.0 / NIL : dopt[5];
  for (int i = 0; i < 3; ++i)
    if (mesh[i] < 1 || sd[i] < 1 || vr[i] < 1 || mesh[i] < vr[i] * sd[i]) return -1;
  if (k < 1 || k > 64 || en2_in < 1 || eg_op < 0 || eg_op > 2 || nrhs < 1) return -1;
  if (threads > 0) omp_set_num_threads(threads);

  const auto t0 = clk::now();
  Problem p;
  p.M = mesh[0];
  p.N = mesh[1];
  p.P = mesh[2];
  p.MN = (long long)p.M * p.N;
  p.n = p.MN * p.P;
  p.kx = kx;
  p.ky = ky ? ky : kx;
  p.kz = kz ? kz : kx;
  assemble(p, dom, dir_on, dir_val);
  const long long n = p.n, MN = p.MN;

  // virtual-rank boxes (x-fastest) and their subdomains (x-fastest inside a rank)
  std::vector<Box> ranks, subs;
  {
    std::vector<int> rxs, rxl, rys, ryl, rzs, rzl;
    split(p.M, vr[0], rxs, rxl);
    split(p.N, vr[1], rys, ryl);
    split(p.P, vr[2], rzs, rzl);
    for (int kz2 = 0; kz2 < vr[2]; ++kz2)
      for (int ky2 = 0; ky2 < vr[1]; ++ky2)
        for (int kx2 = 0; kx2 < vr[0]; ++kx2) {
          const int r = (int)ranks.size();
          const Box rb{rxs[kx2], rxl[kx2], rys[ky2], ryl[ky2], rzs[kz2], rzl[kz2], r};
          ranks.push_back(rb);
          std::vector<int> sxs, sxl, sys, syl, szs, szl;
          split(rb.nx, sd[0], sxs, sxl);
          split(rb.ny, sd[1], sys, syl);
          split(rb.nz, sd[2], szs, szl);
          for (int cz = 0; cz < sd[2]; ++cz)
            for (int cy = 0; cy < sd[1]; ++cy)
              for (int cx = 0; cx < sd[0]; ++cx)
                subs.push_back(Box{rb.x0 + sxs[cx], sxl[cx], rb.y0 + sys[cy], syl[cy], rb.z0 + szs[cz], szl[cz], r});
        }
  }
  const int nsub = (int)subs.size(), nrank = (int)ranks.size(), spr = sd[0] * sd[1] * sd[2];
  for (const Box& b : subs)
    if (b.n() < k) return -1;
  // owner subdomain and local index of every cell
  std::vector<int> owner(n), lidx(n);
#pragma omp parallel for schedule(static)
  for (int s = 0; s < nsub; ++s) {
    const Box& b = subs[s];
    int cl = 0;
    for (int kk = 0; kk < b.nz; ++kk)
      for (int jj = 0; jj < b.ny; ++jj)
        for (int ii = 0; ii < b.nx; ++ii, ++cl) {
          const long long c = p.id(b.x0 + ii, b.y0 + jj, b.z0 + kk);
          owner[c] = s;
          lidx[c] = cl;
        }
  }

  // level 1 factors (IC(0), or the exact band Cholesky) and level 2 local
  // eigenvectors; the adaptive count (:369-383) keeps the first j + 1 vectors at
  // the first lambda_j >= eb_lv1 and zeroes the rest
  std::vector<Vec> lv1D(nsub), phi(nsub);
  std::vector<EigStat> est(nsub);
  std::vector<int> ks(nsub, k);
  int chol_fail = 0;
#pragma omp parallel for schedule(dynamic) reduction(+ : chol_fail)
  for (int s = 0; s < nsub; ++s) {
    const Local L{&p, subs[s]};
    Vec dg;
    local_diag(L, false, dg);
    if (full_chol)
      chol_fail += band_chol(L, dg, lv1D[s]) ? 0 : 1;
    else
      ic0(L, dg, nullptr, 0.0, lv1D[s]);
    est[s] = lobpcg(L, eg_op, k, eig_tol, eig_max_it, eig_sigma, eig_rel_floor, 0x9E3779B97F4A7C15ull ^ (unsigned long long)(s + 1),
                    phi[s]);
    for (int j = 0; j < k; ++j)
      if (est[s].lam[j] >= eb1) {
        ks[s] = j + 1;
        break;
      }
    const int ns = subs[s].n();
    std::fill(phi[s].begin() + (size_t)ks[s] * ns, phi[s].end(), 0.0);
  }
  if (chol_fail) return -2;

  // Galerkin blocks: blk[s][0] = Phi_s^T A Phi_s, blk[s][1 + f] = Phi_s^T A Phi_nb(s, f);
  // gface[s][f] = sum over face f of t phi_s phi_s^T (the Neumann correction across it).
  // Neighbouring subdomains share whole faces (the splits of a direction agree across
  // ranks), so one neighbour per face.
  const size_t kk2 = (size_t)k * k;
  std::vector<int> nbr((size_t)nsub * 6, -1);
  Vec blk((size_t)nsub * 7 * kk2, 0.0), gface((size_t)nsub * 6 * kk2, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int s = 0; s < nsub; ++s) {
    const Box& b = subs[s];
    const int ns = b.n();
    const Local L{&p, b};
    const double* ph = phi[s].data();
    Vec dg, y(ns);
    local_diag(L, false, dg);
    for (int j = 0; j < k; ++j) {
      local_apply(L, dg.data(), ph + (size_t)j * ns, y.data());
      for (int i = 0; i < k; ++i) {
        double v = 0.0;
        const double* pi = ph + (size_t)i * ns;
#pragma omp simd reduction(+ : v)
        for (int c = 0; c < ns; ++c) v += pi[c] * y[c];
        blk[((size_t)s * 7) * kk2 + (size_t)i * k + j] = v;
      }
    }
    for (int f = 0; f < 6; ++f) {
      const int dim = f / 2, hi = f % 2;
      const int lo0 = dim == 0 ? b.x0 : (dim == 1 ? b.y0 : b.z0);
      const int len = dim == 0 ? b.nx : (dim == 1 ? b.ny : b.nz);
      const int glen = dim == 0 ? p.M : (dim == 1 ? p.N : p.P);
      if (hi ? lo0 + len >= glen : lo0 == 0) continue;  // domain boundary
      const long long off = dim == 0 ? 1 : (dim == 1 ? p.M : MN);
      const double* tt = dim == 0 ? p.tx.data() : (dim == 1 ? p.ty.data() : p.tz.data());
      double* G = &gface[((size_t)s * 6 + f) * kk2];
      double* B = &blk[((size_t)s * 7 + 1 + f) * kk2];
      const int n1 = dim == 0 ? b.ny : b.nx, n2 = dim == 2 ? b.ny : b.nz;
      const int lc = hi ? len - 1 : 0;
      for (int u2 = 0; u2 < n2; ++u2)
        for (int u1 = 0; u1 < n1; ++u1) {
          const int ii = dim == 0 ? lc : u1;
          const int jj = dim == 0 ? u1 : (dim == 1 ? lc : u2);
          const int kk = dim == 2 ? lc : u2;
          const long long c = p.id(b.x0 + ii, b.y0 + jj, b.z0 + kk);
          const long long cn = hi ? c + off : c - off;
          const double t = hi ? tt[cn] : tt[c];
          const int cl = (kk * b.ny + jj) * b.nx + ii;
          const int s2 = owner[cn], cl2 = lidx[cn], ns2 = subs[s2].n();
          nbr[(size_t)s * 6 + f] = s2;
          const double* ph2 = phi[s2].data();
          for (int i = 0; i < k; ++i) {
            const double a = t * ph[(size_t)i * ns + cl];
            for (int j = 0; j < k; ++j) {
              G[i * k + j] += a * ph[(size_t)j * ns + cl];
              B[i * k + j] -= a * ph2[(size_t)j * ns2 + cl2];
            }
          }
        }
    }
  }

  // level 2: per-rank principal block of Phi^T A Phi and its factor; level 3: the
  // rank-Neumann form Phi^T A^N_rank Phi and its smallest en_lv2 eigenvectors
  const int nr = spr * k;
  const int en2 = std::min(en2_in, nr);
  std::vector<Vec> A2L(nrank), V3(nrank);
  std::vector<std::vector<char>> A2null(nrank);
  std::vector<int> num3(nrank, 0);
#pragma omp parallel for schedule(dynamic) if (nrank > 1)
  for (int r = 0; r < (two_level ? 0 : nrank); ++r) {
    Vec A((size_t)nr * nr, 0.0), AN((size_t)nr * nr, 0.0);
    for (int a = 0; a < spr; ++a) {
      const int s = r * spr + a;
      for (int i = 0; i < k; ++i)
        for (int j = 0; j < k; ++j) {
          const double v = blk[((size_t)s * 7) * kk2 + (size_t)i * k + j];
          double vn = v;
          for (int f = 0; f < 6; ++f) {
            const int s2 = nbr[(size_t)s * 6 + f];
            if (s2 >= 0 && subs[s2].rank != r) vn -= gface[((size_t)s * 6 + f) * kk2 + (size_t)i * k + j];
          }
          A[(size_t)(a * k + i) * nr + a * k + j] = v;
          AN[(size_t)(a * k + i) * nr + a * k + j] = vn;
        }
      for (int f = 0; f < 6; ++f) {
        const int s2 = nbr[(size_t)s * 6 + f];
        if (s2 < 0 || subs[s2].rank != r) continue;
        const int b2 = s2 - r * spr;
        for (int i = 0; i < k; ++i)
          for (int j = 0; j < k; ++j) {
            const double v = blk[((size_t)s * 7 + 1 + f) * kk2 + (size_t)i * k + j];
            A[(size_t)(a * k + i) * nr + b2 * k + j] = v;
            AN[(size_t)(a * k + i) * nr + b2 * k + j] = v;
          }
      }
    }
    chol_semidef(A, nr, A2null[r]);
    A2L[r].swap(A);
    // HEP on the rank's kept dofs only; adaptive count (:1100-1115) with eb_lv2
    std::vector<int> act;
    for (int a = 0; a < spr; ++a)
      for (int i = 0; i < ks[r * spr + a]; ++i) act.push_back(a * k + i);
    const int na = (int)act.size();
    Vec ANc((size_t)na * na), w, V;
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < na; ++j) ANc[(size_t)i * na + j] = AN[(size_t)act[i] * nr + act[j]];
    const int k3 = std::min(en2_in, na);
    int ldv = na;
    if (na > 256 && k3 + 4 <= 64) {  // the k3 smallest only: inverse subspace iteration
      smallest_eig(ANc, na, k3, w, V);
      ldv = k3;
    } else {
      sym_eig(ANc, na, w, V);
    }
    int num = k3;
    for (int j = 0; j < k3; ++j)
      if (w[j] >= eb2) {
        num = j + 1;
        break;
      }
    num3[r] = num;
    V3[r].assign((size_t)nr * en2, 0.0);
    for (int i = 0; i < na; ++i)
      for (int j = 0; j < num; ++j) V3[r][(size_t)act[i] * en2 + j] = V[(size_t)i * ldv + j];
  }

  // A3 = V^T (Phi^T A Phi) V + NIL I, assembled block by block (each thread owns the
  // rows of its rank), and its factor
  const int n3 = two_level ? 0 : nrank * en2;
  Vec A3((size_t)n3 * n3, 0.0);
#pragma omp parallel for schedule(dynamic)
  for (int r = 0; r < (two_level ? 0 : nrank); ++r) {
    Vec t(k);
    for (int a = 0; a < spr; ++a) {
      const int s = r * spr + a;
      for (int bb = 0; bb < 7; ++bb) {
        const int s2 = bb == 0 ? s : nbr[(size_t)s * 6 + bb - 1];
        if (s2 < 0) continue;
        const int r2 = subs[s2].rank, a2 = s2 - r2 * spr;
        const double* B = &blk[((size_t)s * 7 + bb) * kk2];
        for (int j2 = 0; j2 < en2; ++j2) {
          for (int i = 0; i < k; ++i) {
            double v = 0.0;
            for (int i2 = 0; i2 < k; ++i2) v += B[i * k + i2] * V3[r2][(size_t)(a2 * k + i2) * en2 + j2];
            t[i] = v;
          }
          for (int j = 0; j < en2; ++j) {
            double v = 0.0;
            for (int i = 0; i < k; ++i) v += V3[r][(size_t)(a * k + i) * en2 + j] * t[i];
            A3[(size_t)(r * en2 + j) * n3 + r2 * en2 + j2] += v;
          }
        }
      }
    }
  }
  if (!no_shift)  // :1361-1363
    for (int i = 0; i < n3; ++i) A3[(size_t)i * n3 + i] += NIL;
  std::vector<char> A3null;
  if (n3) chol_semidef(A3, n3, A3null);
  // -use_2level (:423-735): the global Phi^T A Phi over every subdomain, cross-rank
  // blocks included, + NIL I unless -no_shift_A_cc, in place of levels 2 and 3
  const int nc = two_level ? nsub * k : 0;
  Vec A2g((size_t)nc * nc, 0.0);
  std::vector<char> A2gnull;
  if (two_level) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < nsub; ++s)
      for (int bb = 0; bb < 7; ++bb) {
        const int s2 = bb == 0 ? s : nbr[(size_t)s * 6 + bb - 1];
        if (s2 < 0) continue;
        const double* B = &blk[((size_t)s * 7 + bb) * kk2];
        for (int i = 0; i < k; ++i)
          for (int j = 0; j < k; ++j) A2g[(size_t)(s * k + i) * nc + s2 * k + j] = B[i * k + j];
      }
    if (!no_shift)
      for (int i = 0; i < nc; ++i) A2g[(size_t)i * nc + i] += NIL;
    chol_semidef(A2g, nc, A2gnull);
  }
  int n3_kept = 0;
  for (int r = 0; r < nrank; ++r) n3_kept += num3[r];
  const auto t1 = clk::now();

  // ---- preconditioner: y = 0, then r = x - A y and y += B_l r for each visit
  std::vector<int> sched;  // 1, 2, 3: the levels; 4: the global 2-level coarse solve
  for (int i = 0; i < si1; ++i) sched.push_back(1);
  if (two_level) {  // :1918-1922
    sched.push_back(4);
  } else {
    for (int i = 0; i < si2; ++i) sched.push_back(2);
    sched.push_back(3);
    if (wcycle) {
      for (int i = 0; i < si2; ++i) sched.push_back(2);
      sched.push_back(3);
    }
    for (int i = 0; i < si2; ++i) sched.push_back(2);
  }
  for (int i = 0; i < si1; ++i) sched.push_back(1);
  Vec cvec((size_t)nsub * k), zvec((size_t)nsub * k), rres(n), ay(n), d3(n3);
  auto restrict_ = [&](const double* r) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < nsub; ++s) {
      const Box& b = subs[s];
      const int ns = b.n();
      const double* ph = phi[s].data();
      double acc[64];
      for (int j = 0; j < k; ++j) acc[j] = 0.0;
      int cl = 0;
      for (int kk = 0; kk < b.nz; ++kk)
        for (int jj = 0; jj < b.ny; ++jj) {
          const double* rr = r + p.id(b.x0, b.y0 + jj, b.z0 + kk);
          for (int ii = 0; ii < b.nx; ++ii, ++cl)
            for (int j = 0; j < k; ++j) acc[j] += ph[(size_t)j * ns + cl] * rr[ii];
        }
      for (int j = 0; j < k; ++j) cvec[(size_t)s * k + j] = acc[j];
    }
  };
  auto prolong = [&](double* y) {
#pragma omp parallel for schedule(static)
    for (int s = 0; s < nsub; ++s) {
      const Box& b = subs[s];
      const int ns = b.n();
      const double* ph = phi[s].data();
      const double* z = &zvec[(size_t)s * k];
      int cl = 0;
      for (int kk = 0; kk < b.nz; ++kk)
        for (int jj = 0; jj < b.ny; ++jj) {
          double* yy = y + p.id(b.x0, b.y0 + jj, b.z0 + kk);
          for (int ii = 0; ii < b.nx; ++ii, ++cl) {
            double v = 0.0;
            for (int j = 0; j < k; ++j) v += ph[(size_t)j * ns + cl] * z[j];
            yy[ii] += v;
          }
        }
    }
  };
  auto pc_apply = [&](const double* x, double* y) {
    std::fill(y, y + n, 0.0);
    bool first = true;
    for (int lvl : sched) {
      if (first) {  // y = 0: the residual is x itself
        std::copy(x, x + n, rres.begin());
        first = false;
      } else {
        spmv(p, y, ay.data());
#pragma omp parallel for schedule(static)
        for (long long i = 0; i < n; ++i) rres[i] = x[i] - ay[i];
      }
      if (lvl == 1) {
#pragma omp parallel for schedule(dynamic)
        for (int s = 0; s < nsub; ++s) {
          const Box& b = subs[s];
          const int ns = b.n();
          const Local L{&p, b};
          Vec rl(ns), yl(ns);
          int cl = 0;
          for (int kk = 0; kk < b.nz; ++kk)
            for (int jj = 0; jj < b.ny; ++jj) {
              const long long c0 = p.id(b.x0, b.y0 + jj, b.z0 + kk);
              for (int ii = 0; ii < b.nx; ++ii, ++cl) rl[cl] = rres[c0 + ii];
            }
          if (full_chol)
            band_solve(lv1D[s], ns, b.nx * b.ny, rl.data(), yl.data());
          else
            ic0_solve(L, lv1D[s], rl.data(), yl.data());
          cl = 0;
          for (int kk = 0; kk < b.nz; ++kk)
            for (int jj = 0; jj < b.ny; ++jj) {
              const long long c0 = p.id(b.x0, b.y0 + jj, b.z0 + kk);
              for (int ii = 0; ii < b.nx; ++ii, ++cl) y[c0 + ii] += yl[cl];
            }
        }
      } else if (lvl == 4) {
        restrict_(rres.data());
        std::copy(cvec.begin(), cvec.end(), zvec.begin());
        chol_solve(A2g, A2gnull, nc, zvec.data());
        prolong(y);
      } else if (lvl == 2) {
        restrict_(rres.data());
#pragma omp parallel for schedule(dynamic)
        for (int r = 0; r < nrank; ++r) {
          double* v = &zvec[(size_t)r * nr];
          std::copy(&cvec[(size_t)r * nr], &cvec[(size_t)r * nr] + nr, v);
          chol_solve(A2L[r], A2null[r], nr, v);
        }
        prolong(y);
      } else {
        restrict_(rres.data());
#pragma omp parallel for schedule(static)
        for (int r = 0; r < nrank; ++r)
          for (int j = 0; j < en2; ++j) {
            double v = 0.0;
            for (int i = 0; i < nr; ++i) v += V3[r][(size_t)i * en2 + j] * cvec[(size_t)r * nr + i];
            d3[(size_t)r * en2 + j] = v;
          }
        chol_solve(A3, A3null, n3, d3.data());
#pragma omp parallel for schedule(static)
        for (int r = 0; r < nrank; ++r)
          for (int i = 0; i < nr; ++i) {
            double v = 0.0;
            for (int j = 0; j < en2; ++j) v += V3[r][(size_t)i * en2 + j] * d3[(size_t)r * en2 + j];
            zvec[(size_t)r * nr + i] = v;
          }
        prolong(y);
      }
    }
  };

  // ---- PETSc KSPSolve_CG, unpreconditioned norm, zero initial guess, for each
  // right-hand side after the one set-up
  Vec r(n), z(n), pp(n), w(n);
  auto dot = [&](const double* a, const double* c) {
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long long i = 0; i < n; ++i) s += a[i] * c[i];
    return s;
  };
  // MatNullSpaceRemove of the constant null space: z <- z - (sum z / n) 1
  auto remove_constant = [&](double* v) {
    if (!null_space) return;
    double s = 0.0;
#pragma omp parallel for reduction(+ : s) schedule(static)
    for (long long i = 0; i < n; ++i) s += v[i];
    s = s / (-(double)n);
#pragma omp parallel for schedule(static)
    for (long long i = 0; i < n; ++i) v[i] += s;
  };
  auto cg = [&](const double* src, double* x_out, double& dp, double& r0) {
#pragma omp parallel for schedule(static)
  for (long long i = 0; i < n; ++i) {
    r[i] = src[i] + p.bval[i];
    x_out[i] = 0.0;
  }
  dp = std::sqrt(dot(r.data(), r.data()));
  r0 = dp;
  const double ttol = std::max(rtol * dp, 1e-50);
  int its = 0;
  if (dp > ttol) {
    pc_apply(r.data(), z.data());
    remove_constant(z.data());
    double beta = dot(z.data(), r.data()), betaold = 0.0, dpi = 0.0;
    for (int i = 0; i < max_it; ++i) {
      its = i + 1;
      if (beta == 0.0) break;
      if (i == 0) {
        std::copy(z.begin(), z.end(), pp.begin());
      } else {
        const double bb = beta / betaold;
#pragma omp parallel for schedule(static)
        for (long long q = 0; q < n; ++q) pp[q] = z[q] + bb * pp[q];
      }
      spmv(p, pp.data(), w.data());
      const double dpiold = dpi;
      dpi = dot(pp.data(), w.data());
      betaold = beta;
      if (dpi == 0.0 || (i > 0 && ((dpi > 0.0) != (dpiold > 0.0)))) break;
      const double a = beta / dpi;
#pragma omp parallel for schedule(static)
      for (long long q = 0; q < n; ++q) {
        x_out[q] += a * pp[q];
        r[q] -= a * w[q];
      }
      dp = std::sqrt(dot(r.data(), r.data()));
      if (!std::isfinite(dp) || dp <= ttol) break;
      pc_apply(r.data(), z.data());
      remove_constant(z.data());
      beta = dot(z.data(), r.data());
    }
  }
  return its;
  };
  double dp = 0.0, r0 = 0.0;
  int its = 0, its_sum = 0, its_max = 0;
  for (int q = nrhs - 1; q >= 0; --q) {  // the first right-hand side last: info[] reports it
    double dq, r0q;
    const int iq = cg(source + (size_t)q * n, x_out + (size_t)q * n, dq, r0q);
    its_sum += iq;
    its_max = std::max(its_max, iq);
    its = iq;
    dp = dq;
    r0 = r0q;
  }
  const auto t2 = clk::now();
  if (info) {
    double eit = 0.0;
    int emax = 0, eunc = 0;
    for (const EigStat& e : est) {
      eit += e.its;
      emax = std::max(emax, e.its);
      eunc += e.converged ? 0 : 1;
    }
    info[0] = its;
    info[1] = std::chrono::duration<double>(t1 - t0).count();
    info[2] = std::chrono::duration<double>(t2 - t1).count();
    info[3] = omp_get_max_threads();
    info[4] = eit / std::max(1, nsub);
    info[5] = emax;
    info[6] = eunc;
    info[7] = dp;
    info[8] = r0;
    info[9] = two_level ? 0 : n3_kept;
    info[10] = its_sum;
    info[11] = its_max;
  }
  return 0;
}

}  // extern "C"
