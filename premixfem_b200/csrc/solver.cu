// Solver orchestration: setup stages (_PC_setup, src/PreMixFEM_3D.c:1392-1427),
// the V/W-cycle executor (PC_apply_vec, :1840-1936) and the preconditioned CG
// loop (PETSc KSPCG as driven by src/Expe_scal.c:100-119).
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <sstream>

#include "pmf_net.h"
#include "solver.h"
#include "tune.h"

namespace pmf {

unsigned long long g_launches = 0;

// ---------------------------------------------------------------------------
// options
void OptionDB::parse(const std::string& s) {
  std::istringstream is(s);
  std::vector<std::string> tok;
  std::string t;
  while (is >> t) tok.push_back(t);
  for (size_t i = 0; i < tok.size(); ++i) {
    if (tok[i].size() > 1 && tok[i][0] == '-' && !(tok[i][1] >= '0' && tok[i][1] <= '9') && tok[i][1] != '.') {
      std::string v;
      if (i + 1 < tok.size()) {
        const std::string& n = tok[i + 1];
        const bool is_opt = n.size() > 1 && n[0] == '-' && !(n[1] >= '0' && n[1] <= '9') && n[1] != '.';
        if (!is_opt) {
          v = n;
          ++i;
        }
      }
      kv[tok[i - (v.empty() ? 0 : 1)].substr(1)] = v;
    }
  }
}
bool OptionDB::get_int(const char* name, int* v) const {
  auto it = kv.find(name);
  if (it == kv.end() || it->second.empty()) return false;
  *v = (int)strtol(it->second.c_str(), nullptr, 10);
  return true;
}
bool OptionDB::get_real(const char* name, double* v) const {
  auto it = kv.find(name);
  if (it == kv.end() || it->second.empty()) return false;
  *v = strtod(it->second.c_str(), nullptr);
  return true;
}
bool OptionDB::get_ints(const char* name, int* v, int n) const {
  auto it = kv.find(name);
  if (it == kv.end() || it->second.empty()) return false;
  std::string s = it->second;
  for (auto& ch : s)
    if (ch == ',') ch = ' ';
  std::istringstream is(s);
  int cnt = 0;
  while (cnt < n && (is >> v[cnt])) ++cnt;
  if (cnt == 1)
    for (int i = 1; i < n; ++i) v[i] = v[0];
  return cnt > 0;
}

// PC_init option semantics (src/PreMixFEM_3D.c:1662-1721).
int options_from_db(const OptionDB& db, Options* o, std::string* err) {
  int sd = 2;
  const bool has_sd = db.get_int("sd", &sd);
  if (has_sd && sd < 1) {
    *err = "Error in sub_domains (-sd must be >= 1)";
    return 62;  // PETSC_ERR_ARG_WRONG
  }
  if (sd == 1) sd = 2;  // :1718-1721
  o->sd[0] = o->sd[1] = o->sd[2] = sd;
  db.get_ints("pmf_sd", o->sd, 3);
  db.get_ints("pmf_vranks", o->vranks, 3);
  if (db.get_int("si_lv1", &o->si_lv1)) o->si_lv1 = std::max(1, o->si_lv1);
  if (db.get_int("si_lv2", &o->si_lv2)) o->si_lv2 = std::max(1, o->si_lv2);
  db.get_int("en_lv1", &o->en_lv1);
  db.get_int("en_lv2", &o->en_lv2);
  if (o->en_lv1 < 1 || o->en_lv2 < 1) {
    *err = "Error in max_eigen_num (-en_lv1/-en_lv2 must be >= 1)";
    return 62;
  }
  db.get_int("eg_op", &o->eg_op);
  if (o->eg_op < 0 || o->eg_op > 2) {
    *err = "Error in lv2_eigen_op (-eg_op must be 0, 1 or 2)";
    return 62;
  }
  db.get_real("eb_lv1", &o->eb_lv1);
  db.get_real("eb_lv2", &o->eb_lv2);
  o->use_W_cycle = db.has("use_W_cycle");
  o->no_shift_A_cc = db.has("no_shift_A_cc");
  o->use_full_Cholesky_lv1 = db.has("use_full_Cholesky_lv1");
  o->use_2level = db.has("use_2level");
  {
    // PETSc boolean option: the bare flag or true/yes/on/1 sets it, false/no/off/0 clears it
    auto itn = db.kv.find("ksp_constant_null_space");
    if (itn != db.kv.end()) {
      const std::string& v = itn->second;
      if (v.empty() || v == "1" || v == "true" || v == "yes" || v == "on")
        o->null_space = true;
      else if (v == "0" || v == "false" || v == "no" || v == "off")
        o->null_space = false;
      else {
        *err = "Error in -ksp_constant_null_space (true | false)";
        return 62;
      }
    }
  }
  db.get_real("ksp_rtol", &o->rtol);
  db.get_real("ksp_atol", &o->atol);
  db.get_int("ksp_max_it", &o->max_it);
  std::string prec;
  auto it = db.kv.find("pmf_precision");
  if (it != db.kv.end()) {
    if (it->second == "mixed" || it->second == "fp32")
      o->precision = 1;
    else if (it->second == "fp64" || it->second == "double")
      o->precision = 0;
    else {
      *err = "Error in -pmf_precision (fp64 | mixed)";
      return 62;
    }
  }
  db.get_int("pmf_eig_max_it", &o->eig_max_it);
  db.get_real("pmf_eig_tol", &o->eig_tol);
  db.get_real("pmf_eig_sigma", &o->eig_sigma);
  if (db.get_real("pmf_eig_rel_floor", &o->eig_rel_floor) && !(o->eig_rel_floor >= 0.0 && o->eig_rel_floor < 1.0)) {
    *err = "Error in -pmf_eig_rel_floor (0 <= f < 1)";
    return 62;
  }
  if (db.get_int("pmf_eig_guard", &o->eig_guard) && o->eig_guard < 0) {
    *err = "Error in -pmf_eig_guard (must be >= 0)";
    return 62;
  }
  db.get_int("pmf_pcg_chunk", &o->pcg_chunk);
  if (db.get_int("pmf_eig_ctas", &o->eig_ctas) && o->eig_ctas < 0) {
    *err = "Error in -pmf_eig_ctas (must be >= 0; 0: one per SM)";
    return 62;
  }
  db.get_int("pmf_eig_batched", &o->eig_batched);
  db.get_int("pmf_eig_final", &o->eig_final);
  db.get_int("pmf_eig_init", &o->eig_init);
  db.get_int("pmf_eig_profile", &o->eig_profile);
  o->eig_require_converged = db.has("pmf_eig_require_converged");
  {
    auto ite = db.kv.find("pmf_eig_precision");
    if (ite != db.kv.end()) {
      if (ite->second == "fp64" || ite->second == "double")
        o->eig_precision = 0;
      else if (ite->second == "fp32" || ite->second == "mixed")
        o->eig_precision = 1;
      else {
        *err = "Error in -pmf_eig_precision (fp64 | fp32)";
        return 62;
      }
    }
  }
  {
    auto itk = db.kv.find("pmf_lv1_kernel");
    if (itk != db.kv.end()) {
      if (itk->second == "auto")
        o->lv1_kernel = 0;
      else if (itk->second == "natural")
        o->lv1_kernel = 1;
      else if (itk->second == "blocked")
        o->lv1_kernel = 2;
      else if (itk->second == "staged")
        o->lv1_kernel = 3;
      else {
        *err = "Error in -pmf_lv1_kernel (auto | natural | blocked | staged)";
        return 62;
      }
    }
  }
  db.get_int("pmf_pcg_graph", &o->pcg_graph);
  db.get_int("pmf_autotune", &o->autotune);
  {
    auto it2 = db.kv.find("pmf_learned");
    if (it2 != db.kv.end()) {
      if (it2->second.empty()) {
        *err = "-pmf_learned needs the path of a network weight file";
        return 62;
      }
      o->learned_path = it2->second;
    }
  }
  if (db.get_real("pmf_learned_tol", &o->learned_tol) && !(o->learned_tol > 0.0)) {
    *err = "-pmf_learned_tol must be > 0";
    return 62;
  }
  if (db.get_int("pmf_learned_its", &o->learned_its) && o->learned_its < 1) {
    *err = "-pmf_learned_its must be >= 1";
    return 62;
  }
  return 0;
}

static void split(int n, int parts, std::vector<int>& start, std::vector<int>& len) {
  start.assign(parts, 0);
  len.assign(parts, 0);
  for (int i = 0; i < parts; ++i) len[i] = n / parts + ((n % parts) > i ? 1 : 0);
  for (int i = 1; i < parts; ++i) start[i] = start[i - 1] + len[i - 1];
}

// ---------------------------------------------------------------------------
// small setup kernels
__global__ void k_add_diag(int nb, int n, double* a, double mu_rel, int relative) {
  const int b = blockIdx.x;
  double* A = a + (long long)b * n * n;
  __shared__ double mx;
  if (threadIdx.x == 0) {
    double m = 0.0;
    for (int i = 0; i < n; ++i) m = fmax(m, fabs(A[(long long)i * n + i]));
    mx = relative ? m * mu_rel : mu_rel;
  }
  __syncthreads();
  for (int i = threadIdx.x; i < n; i += blockDim.x) A[(long long)i * n + i] += mx;
}

// A3 = V^T (Phi^T A Phi) V block (r, r2): sum over subdomains s of rank r and the
// block-sparse coupling to subdomains of rank r2.  Padded level-3 dofs are identity.
__global__ void k_build_a3(const SubInfo* subs, RankLayout L, int en2, const double* blk, const double* V,
                           const int* rank_nb, const int* ks3, double* A3, int n3, double nil) {
  const int r = blockIdx.x / 7, q = blockIdx.x % 7;
  const int r2 = q == 0 ? r : rank_nb[r * 6 + q - 1];
  if (r2 < 0) return;
  const int kmax = L.kmax;
  const int nsr = L.first[r + 1] - L.first[r];
  const double* Vr = V + L.offv[r];
  const double* Vr2 = V + L.offv[r2];
  for (int e = threadIdx.x; e < en2 * en2; e += blockDim.x) {
    const int j = e / en2, j2 = e % en2;
    double v = 0.0;
    if (j < ks3[r] && j2 < ks3[r2]) {
      for (int a = 0; a < nsr; ++a) {
        const int s = L.first[r] + a;
        const SubInfo& S = subs[s];
        for (int b = 0; b < 7; ++b) {
          const int nb = b == 0 ? s : S.nb[b - 1];
          if (nb < 0 || subs[nb].rank != r2) continue;
          const int la = subs[nb].local;
          const double* B = blk + ((long long)s * 7 + b) * kmax * kmax;
          for (int i = 0; i < kmax; ++i) {
            const double vi = Vr[((long long)a * kmax + i) * en2 + j];
            if (vi == 0.0) continue;
            double t = 0.0;
            for (int i2 = 0; i2 < kmax; ++i2) t += B[i * kmax + i2] * Vr2[((long long)la * kmax + i2) * en2 + j2];
            v += vi * t;
          }
        }
      }
      if (q == 0 && j == j2) v += nil;
    } else if (q == 0 && j == j2) {
      v = 1.0;
    }
    A3[(long long)(r * en2 + j) * n3 + (r2 * en2 + j2)] = v;
  }
}

// level-3 eigenvector columns beyond a rank's adaptive count are zero
__global__ void k_zero_v_cols(int nrank, RankLayout L, int en2, double* V, const int* ks3) {
  for (int r = blockIdx.x; r < nrank; r += gridDim.x) {
    const long long n = L.offv[r + 1] - L.offv[r];
    double* Vr = V + L.offv[r];
    for (long long e = threadIdx.x; e < n; e += blockDim.x)
      if ((int)(e % en2) >= ks3[r]) Vr[e] = 0.0;
  }
}

__global__ void k_zero_d(double* a, long long n) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n; i += (long long)gridDim.x * blockDim.x)
    a[i] = 0.0;
}

// ---------------------------------------------------------------------------
int Solver::check(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return 0;
  err = std::string(what) + ": " + cudaGetErrorString(e);
  return 76;  // PETSC_ERR_LIB
}

// The set-up's stream-ordered scratch (cudaMallocAsync / cudaFreeAsync in the
// coarse inverses and the level-3 eigensolves) comes from the device's default
// memory pool; by default the pool hands freed memory back to the driver at
// every synchronisation, so each set-up allocated it afresh, which stalled the
// set-up for up to half a second at times.  Keeping freed blocks in the pool
// (a per-process runtime attribute, not a device setting) makes them reusable.
static void keep_pool_memory() {
  int dev = 0;
  cudaMemPool_t pool;
  if (cudaGetDevice(&dev) == cudaSuccess && cudaDeviceGetDefaultMemPool(&pool, dev) == cudaSuccess) {
    uint64_t keep = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep);
  }
  (void)cudaGetLastError();
}

Solver::Solver(const double d[3], const int mesh[3], const Options& o) : opt(o) {
  for (int i = 0; i < 3; ++i) dom[i] = d[i];
  g.M = mesh[0];
  g.N = mesh[1];
  g.P = mesh[2];
  g.MN = g.M * g.N;
  g.ncell = (long long)g.M * g.N * g.P;
  H[0] = dom[0] / (double)g.M;  // :1707-1709
  H[1] = dom[1] / (double)g.N;
  H[2] = dom[2] / (double)g.P;
  keep_pool_memory();
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaMallocHost(&h_state, sizeof(PcgState));
}

// A batch of nprob problems (dom, mesh, sd: 3 values per problem) on one
// shared mesh: problem q's cells x < M_q, y < N_q of the layers
// z0_q .. z0_q + P_q - 1, one layer of zero permeability between problems.
Solver::Solver(int np, const double* doms, const int* meshes, const int* sds, const Options& o) : opt(o) {
  nprob = np;
  probs.assign(np, ProbInfo());
  bsd.assign(sds, sds + 3 * np);
  int M = 0, N = 0, P = 0;
  for (int q = 0; q < np; ++q) {
    ProbInfo& p = probs[q];
    p.M = meshes[3 * q];
    p.N = meshes[3 * q + 1];
    p.P = meshes[3 * q + 2];
    p.z0 = P;
    P += p.P + (q + 1 < np ? 1 : 0);
    M = std::max(M, p.M);
    N = std::max(N, p.N);
    p.Hx = doms[3 * q] / (double)p.M;  // :1707-1709
    p.Hy = doms[3 * q + 1] / (double)p.N;
    p.Hz = doms[3 * q + 2] / (double)p.P;
    p.meas = p.Hx * p.Hy * p.Hz;
    const double fyz = p.Hy * p.Hz, fzx = p.Hz * p.Hx, fxy = p.Hx * p.Hy;
    p.cx = fyz * fyz / p.meas;
    p.cy = fzx * fzx / p.meas;
    p.cz = fxy * fxy / p.meas;
    p.dmask = 0;
    for (double& v : p.dval) v = 0.0;
  }
  g.M = M;
  g.N = N;
  g.P = P;
  g.MN = M * N;
  g.ncell = (long long)M * N * P;
  for (ProbInfo& p : probs) {
    p.c0 = (long long)p.z0 * g.MN;
    p.c1 = (long long)(p.z0 + p.P) * g.MN;
  }
  for (int i = 0; i < 3; ++i) {
    dom[i] = doms[i];
    H[i] = probs[0].Hx;
  }
  H[1] = probs[0].Hy;
  H[2] = probs[0].Hz;
  keep_pool_memory();
  cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
  cudaEventCreate(&ev0);
  cudaEventCreate(&ev1);
  cudaMallocHost(&h_state, sizeof(PcgState));
}

int Solver::set_dirichlet_prob(int q, int face, double value) {
  if (q < 0 || q >= nprob || face < 0 || face > 5) {
    err = "batch Dirichlet face: problem index or face (0..5) out of range";
    return 62;
  }
  probs[q].dmask |= 1 << face;
  probs[q].dval[face] = value;
  return 0;
}

// Device copies of the problem table and of the layer -> problem map.
int Solver::upload_probs() {
  if (!nprob) return 0;
  if (!d_probs) {
    if (int e = dalloc((void**)&d_probs, sizeof(ProbInfo) * nprob, "batch problem table")) return e;
    if (int e = dalloc((void**)&d_layer_prob, sizeof(int) * g.P, "batch layer map")) return e;
  }
  layer_prob.assign(g.P, -1);
  for (int q = 0; q < nprob; ++q)
    for (int z = probs[q].z0; z < probs[q].z0 + probs[q].P; ++z) layer_prob[z] = q;
  cudaMemcpyAsync(d_probs, probs.data(), sizeof(ProbInfo) * nprob, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_layer_prob, layer_prob.data(), sizeof(int) * g.P, cudaMemcpyHostToDevice, st);
  return check(cudaStreamSynchronize(st), "batch problem table");
}

Solver::~Solver() {
  if (st) cudaStreamSynchronize(st);
  void* ptrs[] = {d_subs, kx,    ky,    kz,    tx,     ty,    tz,     diag,     db,       bval,    tx32,  ty32,
                  tz32,   diag32, inv32, inv64, phi,    blk,   gface,  A2inv,    AN,       ANinv,   V3,    A3inv,
                  d_eig1, d_eig3, d_ks,  d_iters, d_status, d_l3it, d_flag, d_rank_nb, eig_work, c,     dz,    Zacc,
                  d3,     w3,     y0,    y1,    vb,     vx,    r,      z,        p0,       p1,      w,     part,
                  state};
  for (void* p : ptrs)
    if (p) cudaFree(p);
  if (pcg_exec) cudaGraphExecDestroy(pcg_exec);
  if (bpcg_exec) cudaGraphExecDestroy(bpcg_exec);
  for (void* p : {(void*)bstate, (void*)d_all_done})
    if (p) cudaFree(p);
  if (h_bstate) cudaFreeHost(h_bstate);
  if (h_all_done) cudaFreeHost(h_all_done);
  for (void* p : {(void*)eb.slab, eb.state, (void*)eb.Ybuf, (void*)eb.gpart, (void*)eb.rpart, (void*)eb.nactive,
                  (void*)eb.alist, (void*)eb.colcells})
    if (p) cudaFree(p);
  if (eb.h_nactive) cudaFreeHost(eb.h_nactive);
  for (void* p : {(void*)cb_T, (void*)cb_X, (void*)cb_v, (void*)cb_y, (void*)cb_t, (void*)cb_part, (void*)cb_perm, (void*)cb_null,
                  (void*)cb_scale})
    if (p) cudaFree(p);
  for (void* p : {(void*)d_ks3, (void*)l3work, (void*)d_queue, net_x, (void*)net_y, (void*)d_fail_list, (void*)d_fail_count, (void*)d_iters_learned,
                  (void*)d_status_learned, (void*)d_boff, (void*)band64, (void*)band32})
    if (p) cudaFree(p);
  delete net;
  if (h_state) cudaFreeHost(h_state);
  if (ev0) cudaEventDestroy(ev0);
  if (ev1) cudaEventDestroy(ev1);
  for (auto& e : prof_ev)
    if (e) cudaEventDestroy(e);
  for (void* q : {(void*)d_coff, ic_coef, (void*)d_kerr, (void*)phi64, (void*)d_rl_first, (void*)d_rl_off,
                  (void*)d_rl_dof_rank, (void*)d_probs, (void*)d_layer_prob})
    if (q) cudaFree(q);
  if (st) cudaStreamDestroy(st);
}

int Solver::build_partition() {
  if (nprob) return build_partition_batch();
  const int px = opt.vranks[0], py = opt.vranks[1], pz = opt.vranks[2];
  const int sx = opt.sd[0], sy = opt.sd[1], sz = opt.sd[2];
  if (px < 1 || py < 1 || pz < 1 || sx < 1 || sy < 1 || sz < 1) {
    err = "virtual rank grid and subdomain counts must be positive";
    return 62;
  }
  rank_grid[0] = px;
  rank_grid[1] = py;
  rank_grid[2] = pz;
  std::vector<int> rxs, rxl, rys, ryl, rzs, rzl;
  split(g.M, px, rxs, rxl);
  split(g.N, py, rys, ryl);
  split(g.P, pz, rzs, rzl);
  nrank = px * py * pz;
  spr = sx * sy * sz;
  nsub = nrank * spr;
  subs.assign(nsub, SubInfo());
  const int GX = px * sx, GY = py * sy, GZ = pz * sz;
  std::vector<int> gmap((size_t)GX * GY * GZ, -1);
  max_cells = 0;
  max_lines = 0;
  for (int kz = 0; kz < pz; ++kz)
    for (int ky = 0; ky < py; ++ky)
      for (int kx_ = 0; kx_ < px; ++kx_) {
        const int rr = (kz * py + ky) * px + kx_;
        std::vector<int> xs, xl, ys, yl, zs, zl;
        split(rxl[kx_], sx, xs, xl);
        split(ryl[ky], sy, ys, yl);
        split(rzl[kz], sz, zs, zl);
        for (int cz = 0; cz < sz; ++cz)
          for (int cy = 0; cy < sy; ++cy)
            for (int cx = 0; cx < sx; ++cx) {
              const int loc = (cz * sy + cy) * sx + cx;
              const int s = rr * spr + loc;
              SubInfo& S = subs[s];
              S.x0 = rxs[kx_] + xs[cx];
              S.nx = xl[cx];
              S.y0 = rys[ky] + ys[cy];
              S.ny = yl[cy];
              S.z0 = rzs[kz] + zs[cz];
              S.nz = zl[cz];
              S.rank = rr;
              S.local = loc;
              S.k = opt.en_lv1;
              S.prob = 0;
              if (S.nx < 1 || S.ny < 1 || S.nz < 1) {
                err = "empty subdomain: too many subdomains or ranks for the mesh";
                return 62;
              }
              const int gx = kx_ * sx + cx, gy = ky * sy + cy, gz = kz * sz + cz;
              gmap[((size_t)gz * GY + gy) * GX + gx] = s;
              max_cells = std::max(max_cells, S.nx * S.ny * S.nz);
              max_lines = std::max(max_lines, S.ny * S.nz);
            }
      }
  for (int s = 0; s < nsub; ++s) {
    SubInfo& S = subs[s];
    const int kx_ = (S.rank % px), ky = (S.rank / px) % py, kz = S.rank / (px * py);
    const int cx = S.local % sx, cy = (S.local / sx) % sy, cz = S.local / (sx * sy);
    const int gx = kx_ * sx + cx, gy = ky * sy + cy, gz = kz * sz + cz;
    auto at = [&](int x, int y, int zz) -> int {
      if (x < 0 || y < 0 || zz < 0 || x >= GX || y >= GY || zz >= GZ) return -1;
      return gmap[((size_t)zz * GY + y) * GX + x];
    };
    S.nb[0] = at(gx - 1, gy, gz);
    S.nb[1] = at(gx + 1, gy, gz);
    S.nb[2] = at(gx, gy - 1, gz);
    S.nb[3] = at(gx, gy + 1, gz);
    S.nb[4] = at(gx, gy, gz - 1);
    S.nb[5] = at(gx, gy, gz + 1);
  }
  rank_first.assign(nrank + 1, 0);
  for (int r = 0; r <= nrank; ++r) rank_first[r] = r * spr;
  ragged = false;
  return partition_checks();
}

// A batch of problems: each problem is one virtual rank, split into its own
// subdomain grid (near-equal, as :47-78) inside its box of the shared mesh;
// subdomains only neighbour subdomains of their own problem.
int Solver::build_partition_batch() {
  nrank = nprob;
  rank_grid[0] = nprob;
  rank_grid[1] = rank_grid[2] = 1;
  subs.clear();
  rank_first.assign(nprob + 1, 0);
  max_cells = max_lines = 0;
  spr = 0;
  for (int q = 0; q < nprob; ++q) {
    ProbInfo& pq = probs[q];
    const int sx = bsd[3 * q], sy = bsd[3 * q + 1], sz = bsd[3 * q + 2];
    if (sx < 1 || sy < 1 || sz < 1 || sx > pq.M || sy > pq.N || sz > pq.P) {
      err = "batch problem " + std::to_string(q) + ": subdomain counts must be between 1 and the cells per axis";
      return 62;
    }
    std::vector<int> xs, xl, ys, yl, zs, zl;
    split(pq.M, sx, xs, xl);
    split(pq.N, sy, ys, yl);
    split(pq.P, sz, zs, zl);
    const int s0 = (int)subs.size();
    rank_first[q] = s0;
    pq.s0 = s0;
    for (int cz = 0; cz < sz; ++cz)
      for (int cy = 0; cy < sy; ++cy)
        for (int cx = 0; cx < sx; ++cx) {
          SubInfo S;
          S.x0 = xs[cx];
          S.nx = xl[cx];
          S.y0 = ys[cy];
          S.ny = yl[cy];
          S.z0 = pq.z0 + zs[cz];
          S.nz = zl[cz];
          S.rank = q;
          S.local = (cz * sy + cy) * sx + cx;
          S.k = opt.en_lv1;
          S.prob = q;
          auto at = [&](int x, int y, int z) {
            return (x < 0 || y < 0 || z < 0 || x >= sx || y >= sy || z >= sz) ? -1 : s0 + (z * sy + y) * sx + x;
          };
          S.nb[0] = at(cx - 1, cy, cz);
          S.nb[1] = at(cx + 1, cy, cz);
          S.nb[2] = at(cx, cy - 1, cz);
          S.nb[3] = at(cx, cy + 1, cz);
          S.nb[4] = at(cx, cy, cz - 1);
          S.nb[5] = at(cx, cy, cz + 1);
          max_cells = std::max(max_cells, S.nx * S.ny * S.nz);
          max_lines = std::max(max_lines, S.ny * S.nz);
          subs.push_back(S);
        }
    pq.s1 = (int)subs.size();
    spr = std::max(spr, pq.s1 - s0);
  }
  nsub = (int)subs.size();
  rank_first[nprob] = nsub;
  ragged = true;
  if (!opt.learned_path.empty() || opt.use_2level) {
    err = "a batch of problems runs neither -pmf_learned nor -use_2level";
    return 56;
  }
  return partition_checks();
}

// Limits every partition must meet, then the coarse sizes.
int Solver::partition_checks() {
  if (max_cells > PMF_MAX_SUB_CELLS || max_lines > 256) {
    err = "subdomain too large for the shared-memory sweeps (cells <= 8192, ny*nz <= 256)";
    return 62;
  }
  if (32 * 8 + 5 * (size_t)((max_cells + 3) & ~3) * (opt.precision == 1 ? 4 : 8) > 227 * 1024) {
    err = "subdomain too large for the shared-memory IC(0) sweep of this precision (FP64: <= 5600 cells)";
    return 62;
  }
  if (!opt.learned_path.empty()) {
    for (const SubInfo& S : subs)
      if (S.nx > NET_S || S.ny > NET_S || S.nz > NET_S) {
        err = "-pmf_learned needs subdomains of at most 16 x 16 x 16 cells";
        return 62;
      }
  }
  kmax = opt.en_lv1;
  if (kmax > 8 || opt.en_lv1 + opt.eig_guard > 10) {
    err = "en_lv1 must be <= 8 (block size en_lv1 + guard <= 10)";
    return 62;
  }
  for (const SubInfo& S : subs)
    if (kmax > S.nx * S.ny * S.nz) {
      err = "en_lv1 larger than a subdomain";
      return 62;
    }
  rank_sizes();
  if (!opt.use_2level && (nr > 4096 || n3 > 8192)) {
    err = "coarse blocks too large (subdomains per rank * en_lv1 <= 4096, ranks * en_lv2 <= 8192)";
    return 62;
  }
  return 0;
}

// Sizes of the per-rank coarse data from rank_first: nr is the largest rank's
// coarse order, en2 = min(en_lv2, the smallest rank's order), and the prefix
// sums of the dense blocks (nr_r^2), level-3 vectors (nr_r en2) and level-3
// work (3 nr_r p).
void Solver::rank_sizes() {
  nr = 0;
  nr_min = 1 << 30;
  for (int r = 0; r < nrank; ++r) {
    const int n = (rank_first[r + 1] - rank_first[r]) * kmax;
    nr = std::max(nr, n);
    nr_min = std::min(nr_min, n);
  }
  en2 = std::min(opt.en_lv2, nr_min);
  n3 = nrank * en2;
  l3p = std::min(nr_min, std::min(32, 2 * en2 + 4));
  tot2 = totv = totw = 0;
  for (int r = 0; r < nrank; ++r) {
    const long long n = (long long)(rank_first[r + 1] - rank_first[r]) * kmax;
    tot2 += n * n;
    totv += n * en2;
    totw += 3 * n * l3p;
  }
}

int Solver::rank_layout() {
  if (d_rl_first) return 0;
  std::vector<long long> off(3 * (size_t)(nrank + 1), 0);
  for (int r = 0; r < nrank; ++r) {
    const long long n = (long long)(rank_first[r + 1] - rank_first[r]) * kmax;
    off[r + 1] = off[r] + n * n;
    off[(nrank + 1) + r + 1] = off[(nrank + 1) + r] + n * en2;
    off[2 * (nrank + 1) + r + 1] = off[2 * (nrank + 1) + r] + 3 * n * l3p;
  }
  std::vector<int> dof_rank((size_t)nsub * kmax);
  for (int r = 0; r < nrank; ++r)
    for (long long g = (long long)rank_first[r] * kmax; g < (long long)rank_first[r + 1] * kmax; ++g) dof_rank[g] = r;
  int e = dalloc((void**)&d_rl_first, sizeof(int) * (nrank + 1), "rank layout");
  if (!e) e = dalloc((void**)&d_rl_off, sizeof(long long) * off.size(), "rank layout");
  if (!e) e = dalloc((void**)&d_rl_dof_rank, sizeof(int) * dof_rank.size(), "rank layout");
  if (e) return e;
  cudaMemcpyAsync(d_rl_first, rank_first.data(), sizeof(int) * (nrank + 1), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_rl_off, off.data(), sizeof(long long) * off.size(), cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_rl_dof_rank, dof_rank.data(), sizeof(int) * dof_rank.size(), cudaMemcpyHostToDevice, st);
  rl.first = d_rl_first;
  rl.off2 = d_rl_off;
  rl.offv = d_rl_off + (nrank + 1);
  rl.offw = d_rl_off + 2 * (nrank + 1);
  rl.dof_rank = d_rl_dof_rank;
  rl.kmax = kmax;
  // the host vectors must outlive the copies
  return check(cudaStreamSynchronize(st), "rank layout");
}

// cudaMalloc with its return code checked: on failure *p is null, err names
// the array and the PETSc-style code 76 comes back.
int Solver::dalloc(void** p, size_t bytes, const char* what) {
  *p = nullptr;
  const cudaError_t e = cudaMalloc(p, bytes);
  if (e == cudaSuccess) return 0;
  *p = nullptr;
  cudaGetLastError();  // clear the sticky-free allocation error
  err = std::string("cudaMalloc ") + what + " (" + std::to_string(bytes) + " bytes): " + cudaGetErrorString(e);
  return 76;  // PETSC_ERR_LIB
}

// The fine-grid arrays of the operator, the preconditioner and the CG loop.
// All or nothing: when one allocation fails, every array allocated here is
// freed and reset to null (so a later call retries from scratch) and the
// error is returned before any kernel can write through a null pointer.
int Solver::alloc_fine() {
  const size_t n = (size_t)g.ncell;
  const size_t pb = opt.precision == 1 ? 4 : 8;
  const int nparts = std::max(pcg_part_capacity(g), nsub) + 64;  // partial slots of the CG and level-1 kernels
  struct A {
    void** p;
    size_t bytes;
    const char* what;
  };
  std::vector<A> list = {{(void**)&tx, n * 8, "tx"},      {(void**)&ty, n * 8, "ty"},
                         {(void**)&tz, n * 8, "tz"},      {(void**)&diag, n * 8, "diag"},
                         {(void**)&db, n * 8, "db"},      {(void**)&bval, n * 8, "bval"},
                         {(void**)&inv64, n * 8, "inv64"}, {(void**)&vb, n * 8, "vb"},
                         {(void**)&vx, n * 8, "vx"},      {(void**)&r, n * 8, "r"},
                         {(void**)&z, n * 8, "z"},        {(void**)&p0, n * 8, "p0"},
                         {(void**)&p1, n * 8, "p1"},      {(void**)&w, n * 8, "w"},
                         {(void**)&y0, n * pb, "y0"},     {(void**)&y1, n * pb, "y1"},
                         {(void**)&phi, n * kmax * pb, "phi"},
                         {(void**)&part, (size_t)(nparts + cell_blocks(g.ncell)) * 8, "part"},
                         {(void**)&state, sizeof(PcgState), "state"}};
  if (opt.precision == 1) {
    list.push_back({(void**)&tx32, n * 4, "tx32"});
    list.push_back({(void**)&ty32, n * 4, "ty32"});
    list.push_back({(void**)&tz32, n * 4, "tz32"});
    list.push_back({(void**)&diag32, n * 4, "diag32"});
    list.push_back({(void**)&inv32, n * 4, "inv32"});
  }
  for (size_t i = 0; i < list.size(); ++i) {
    if (int e = dalloc(list[i].p, list[i].bytes, list[i].what)) {
      for (size_t j = 0; j < i; ++j) {
        cudaFree(*list[j].p);
        *list[j].p = nullptr;
      }
      zpart = nullptr;
      return e;
    }
  }
  zpart = part + nparts;
  return 0;
}

int Solver::set_kappa(const double* k0, const double* k1, const double* k2, bool on_device) {
  if (int e = build_partition()) return e;
  const size_t n = (size_t)g.ncell;
  if (!kx || !ky || !kz) {
    for (double** p : {&kx, &ky, &kz}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    int e = dalloc((void**)&kx, n * 8, "kappa x");
    if (!e) e = dalloc((void**)&ky, n * 8, "kappa y");
    if (!e) e = dalloc((void**)&kz, n * 8, "kappa z");
    if (e) {
      for (double** p : {&kx, &ky, &kz}) {
        if (*p) cudaFree(*p);
        *p = nullptr;
      }
      return e;
    }
  }
  const cudaMemcpyKind kind = on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
  cudaMemcpyAsync(kx, k0, n * 8, kind, st);
  cudaMemcpyAsync(ky, k1 ? k1 : k0, n * 8, kind, st);
  cudaMemcpyAsync(kz, k2 ? k2 : k0, n * 8, kind, st);
  if (nprob) {  // cells of no problem hold zero permeability, whatever the caller passed there
    if (int e = upload_probs()) return e;
    launch_zero_padding(g, d_probs, d_layer_prob, kx, ky, kz, st);
  }
  return check(cudaStreamSynchronize(st), "set_kappa");
}

int Solver::set_dirichlet(int face, double value) {
  if (nprob) {
    err = "a batch takes its Dirichlet faces per problem (pmf_batch_set_dirichlet)";
    return 73;
  }
  if (face < 0 || face > 5) {
    err = "Dirichlet face must be 0..5 (x-,x+,y-,y+,z-,z+)";
    return 62;
  }
  dir_on_[face] = 1;
  dir_val_[face] = value;
  return 0;
}

std::vector<int> Solver::schedule() const {
  std::vector<int> s;
  if (opt.use_2level) {  // :1918-1922: [1] * si1, global coarse solve, [1] * si1
    for (int i = 0; i < opt.si_lv1; ++i) s.push_back(1);
    s.push_back(4);
    for (int i = 0; i < opt.si_lv1; ++i) s.push_back(1);
    return s;
  }
  for (int i = 0; i < opt.si_lv1; ++i) s.push_back(1);
  for (int i = 0; i < opt.si_lv2; ++i) s.push_back(2);
  s.push_back(3);
  if (opt.use_W_cycle) {  // :1857-1894
    for (int i = 0; i < opt.si_lv2; ++i) s.push_back(2);
    s.push_back(3);
  }
  for (int i = 0; i < opt.si_lv2; ++i) s.push_back(2);
  for (int i = 0; i < opt.si_lv1; ++i) s.push_back(1);
  return s;
}

// Face transmissibilities, diagonal and Dirichlet terms of the operator on
// the solver stream (PC_create_A, src/PreMixFEM_3D.c:1757-1824).
void Solver::assemble_launch() {
  AssembleArgs aa;
  aa.g = g;
  aa.kx = kx;
  aa.ky = ky;
  aa.kz = kz;
  const double meas = H[0] * H[1] * H[2];
  const double fyz = H[1] * H[2], fzx = H[2] * H[0], fxy = H[0] * H[1];
  aa.cx = fyz * fyz / meas;
  aa.cy = fzx * fzx / meas;
  aa.cz = fxy * fxy / meas;
  for (int f = 0; f < 6; ++f) {
    aa.dir_on[f] = dir_on_[f];
    aa.dir_val[f] = dir_val_[f];
  }
  aa.probs = d_probs;
  aa.layer_prob = d_layer_prob;
  launch_assemble(aa, tx, ty, tz, diag, db, bval, st);
}

int Solver::assemble() {
  if (!kx) {
    err = "kappa not set";
    return 73;
  }
  if (!tx)
    if (int e = alloc_fine()) return e;
  assemble_launch();
  return check(cudaStreamSynchronize(st), "assemble");
}

int Solver::alloc_eb(int m, bool mixed) {
  const size_t stride = lobpcg_batched_slab_bytes(max_cells, m, mixed ? 4 : 8);
  if (eb.slab && eb.slab_stride == stride) return 0;
  if (pcg_exec) cudaGraphExecDestroy(pcg_exec);
  for (void* p : {(void*)eb.slab, eb.state, (void*)eb.Ybuf, (void*)eb.gpart, (void*)eb.rpart})
    if (p) cudaFree(p);
  eb.slab_stride = stride;
  eb.nchunk = lobpcg_batched_nchunk(max_cells);
  const size_t ns = (size_t)nsub;
  if (int e = check(cudaMalloc(&eb.slab, ns * stride), "cudaMalloc eigensolver slabs")) return e;
  if (int e = check(cudaMalloc(&eb.state, ns * lobpcg_batched_state_bytes()), "cudaMalloc eigensolver state")) return e;
  if (int e = check(cudaMalloc(&eb.Ybuf, ns * 32 * 32 * sizeof(double)), "cudaMalloc eigensolver Y")) return e;
  if (int e = check(cudaMalloc(&eb.gpart, ns * eb.nchunk * 2 * 32 * 32 * sizeof(double)), "cudaMalloc Grams"))
    return e;
  if (int e = check(cudaMalloc(&eb.rpart, ns * eb.nchunk * 10 * sizeof(double)), "cudaMalloc residuals")) return e;
  if (!eb.nactive)
    if (int e = dalloc((void**)&eb.nactive, 4 * sizeof(int), "eigensolver counters")) return e;
  if (!eb.colcells)
    if (int e = dalloc((void**)&eb.colcells, sizeof(unsigned long long), "eigensolver traffic counter")) return e;
  if (eb.alist) cudaFree(eb.alist);
  if (int e = dalloc((void**)&eb.alist, ns * sizeof(int), "eigensolver active list")) return e;
  if (!eb.h_nactive)
    if (int e = check(cudaMallocHost(&eb.h_nactive, 4 * sizeof(int)), "cudaMallocHost eigensolver counters"))
      return e;
  return 0;
}

// The batched local eigensolves over `list` (nullptr: every subdomain), with
// the phase-batched solver or the single persistent launch.
int Solver::run_eigen(LobpcgArgs& la, const int* list, int nlist, int eig_blocks, double eb1) {
  const bool e32 = eig32();
  // FP64 eigenvectors go to phi, or to phi64 when the preconditioner is FP32
  double* out64 = opt.precision == 1 ? phi64 : (double*)phi;
  if (!opt.eig_batched) {
    if (list) {
      la.sub_list = list;
      la.nlist = d_fail_count;
    }
    if (e32)
      launch_lobpcg<float>(la, eig_blocks, eig_work, (float*)phi, d_eig1, d_iters, d_status, d_ks, eb1, max_cells,
                           max_lines, st);
    else
      launch_lobpcg<double>(la, eig_blocks, eig_work, out64, d_eig1, d_iters, d_status, d_ks, eb1, max_cells,
                            max_lines, st);
    return 0;
  }
  if (int e = alloc_eb(la.m, e32)) return e;
  eb.phase_ms = opt.eig_profile ? eig_phase_ms : nullptr;
  int r;
  if (e32)
    r = launch_lobpcg_batched<float>(la, eb, list, nlist, (float*)phi, d_eig1, d_iters, d_status, d_ks, eb1,
                                     max_cells, max_lines, st);
  else
    r = launch_lobpcg_batched<double>(la, eb, list, nlist, out64, d_eig1, d_iters, d_status, d_ks, eb1, max_cells,
                                      max_lines, st);
  if (r) {
    err = "batched eigensolve: a CUDA call failed";
    return r;
  }
  unsigned long long cc = 0;
  cudaMemcpyAsync(&cc, eb.colcells, sizeof(cc), cudaMemcpyDeviceToHost, st);
  cudaStreamSynchronize(st);
  eig_colcells += cc;
  return 0;
}

// Local eigensolves from the network's initial blocks: one LOBPCG launch
// capped at learned_its iterations, then a second launch, from a random start
// with the full budget, over the subdomains the first one left unconverged
// (the list is built on the device, so no host round trip is needed).
int Solver::run_learned_eigen(LobpcgArgs& la, int eig_blocks, double eb1) {
  const bool mixed = opt.precision == 1;
  if (!net) {
    net = new Net();
    if (int e = net->load(opt.learned_path.c_str())) {
      err = net->err;
      delete net;
      net = nullptr;
      return e;
    }
  }
  const int chunk = std::min(nsub, 1024);
  if (!net_y) {
    if (int e = check(cudaMalloc(&net_y, (size_t)nsub * NET_VOX * NET_COUT * sizeof(float)), "cudaMalloc net output"))
      return e;
    if (int e = check(cudaMalloc(&net_x, (size_t)chunk * NET_VOX * NET_CIN * 2), "cudaMalloc net input")) return e;
    if (int e = dalloc((void**)&d_fail_list, sizeof(int) * nsub, "fallback list")) return e;
    if (int e = dalloc((void**)&d_fail_count, sizeof(int), "fallback count")) return e;
    if (int e = dalloc((void**)&d_iters_learned, sizeof(int) * nsub, "learned iterations")) return e;
    if (int e = dalloc((void**)&d_status_learned, sizeof(int) * nsub, "learned status")) return e;
  }
  int dmask = 0;
  for (int f = 0; f < 6; ++f)
    if (dir_on_[f]) dmask |= 1 << f;
  cudaEvent_t n0, n1;
  cudaEventCreate(&n0);
  cudaEventCreate(&n1);
  cudaEventRecord(n0, st);
  for (int c0 = 0; c0 < nsub; c0 += chunk) {
    const int cb = std::min(chunk, nsub - c0);
    launch_net_features(g, d_subs + c0, cb, kx, ky, kz, dmask, (__nv_bfloat16*)net_x, st);
    if (int e = net->forward((const __nv_bfloat16*)net_x, cb, net_y + (size_t)c0 * NET_VOX * NET_COUT, false, st)) {
      err = net->err;
      return e;
    }
  }
  cudaEventRecord(n1, st);
  LobpcgArgs l1 = la;
  l1.xinit_patch = net_y;
  l1.xinit_k = opt.en_lv1;
  l1.max_it = std::min(opt.learned_its, opt.eig_max_it);
  l1.tol = std::max(opt.learned_tol, la.tol);
  LobpcgArgs l2 = la;
  l2.sub_list = d_fail_list;
  l2.nlist = d_fail_count;
  if (int er = run_eigen(l1, nullptr, nsub, eig_blocks, eb1)) return er;
  cudaMemcpyAsync(d_iters_learned, d_iters, sizeof(int) * nsub, cudaMemcpyDeviceToDevice, st);
  cudaMemcpyAsync(d_status_learned, d_status, sizeof(int) * nsub, cudaMemcpyDeviceToDevice, st);
  launch_failed_list(d_status, nsub, d_fail_list, d_fail_count, st);
  if (opt.eig_batched) {
    int nfail = 0;
    cudaMemcpyAsync(eb.h_nactive, d_fail_count, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int er = check(cudaStreamSynchronize(st), "learned eigensolve")) return er;
    nfail = *eb.h_nactive;
    LobpcgArgs l3 = la;
    if (int er = run_eigen(l3, d_fail_list, nfail, eig_blocks, eb1)) return er;
  } else {
    if (int er = run_eigen(l2, nullptr, nsub, eig_blocks, eb1)) return er;
  }
  float ms = 0.f;
  cudaEventSynchronize(n1);
  cudaEventElapsedTime(&ms, n0, n1);
  net_ms = ms;
  if (int e = net->take_error()) {
    err = net->err;
    cudaEventDestroy(n0);
    cudaEventDestroy(n1);
    return e;
  }
  cudaEventDestroy(n0);
  cudaEventDestroy(n1);
  return 0;
}

int Solver::setup() {
  if (!kx) {
    err = "kappa not set (PC_init contract: the caller constructs kappa before setup)";
    return 73;  // PETSC_ERR_ARG_WRONGSTATE
  }
  if (opt.autotune >= 0) tune_set_enabled(opt.autotune == 1);
  if (int er = upload_probs()) return er;
  // stage events, destroyed on every return path
  struct StageEvents {
    cudaEvent_t ev[8];
    StageEvents() {
      for (auto& x : ev) cudaEventCreate(&x);
    }
    ~StageEvents() {
      for (auto& x : ev) cudaEventDestroy(x);
    }
  } evs;
  cudaEvent_t* e = evs.ev;
  const bool mixed = opt.precision == 1;
  if (!tx)
    if (int er = alloc_fine()) return er;
  if (!d_subs)
    if (int er = dalloc((void**)&d_subs, sizeof(SubInfo) * nsub, "subdomain table")) return er;
  cudaMemcpyAsync(d_subs, subs.data(), sizeof(SubInfo) * nsub, cudaMemcpyHostToDevice, st);
  cudaEventRecord(e[0], st);
  // operator (PC_create_A) and level 1
  assemble_launch();
  int dmask = 0;
  for (int f = 0; f < 6; ++f)
    if (dir_on_[f]) dmask |= 1 << f;
  if (!d_flag)
    if (int er = dalloc((void**)&d_flag, 4 * sizeof(int), "pivot flags")) return er;
  cudaMemsetAsync(d_flag, 0, 4 * sizeof(int), st);
  if (opt.use_full_Cholesky_lv1) {
    if (int er = setup_band_cholesky(mixed)) return er;
  } else {
    launch_ic_factor(g, d_subs, nsub, max_lines, tx, ty, tz, diag, inv64, d_flag, st);
  }
  {
    // a non-positive level-1 pivot (a cell with kappa <= 0, for instance)
    // stops the set-up here, before the eigensolves see the operator, as
    // PETSc's factorisation fails in KSPSetUp (src/PreMixFEM_3D.c:200-215)
    if (int er = check(cudaStreamSynchronize(st), "level-1 factorisation")) return er;
    int bad_pivots = 0;
    if (int er = check(cudaMemcpy(&bad_pivots, d_flag, sizeof(int), cudaMemcpyDeviceToHost), "pivot flag"))
      return er;
    if (bad_pivots) {
      err = std::to_string(bad_pivots) +
            (opt.use_full_Cholesky_lv1 ? " non-positive pivot(s) in the level-1 Cholesky factorisations"
                                       : " non-positive IC(0) pivot(s) in the level-1 factorisations");
      return 71;  // PETSC_ERR_MAT_LU_ZRPVT
    }
  }
  if (mixed) {
    launch_to_f32(tx, tx32, g.ncell, st);
    launch_to_f32(ty, ty32, g.ncell, st);
    launch_to_f32(tz, tz32, g.ncell, st);
    launch_to_f32(diag, diag32, g.ncell, st);
    launch_to_f32(inv64, inv32, g.ncell, st);
  }
  if (!opt.use_full_Cholesky_lv1) {
    if (int er = setup_ic_blocked(mixed)) return er;
    if (opt.lv1_kernel == 2 && !ic_blk_ok) {
      err = "-pmf_lv1_kernel blocked needs every subdomain 16 cells wide in x with x0 % 4 == 0, M % 4 == 0 and "
            "ny*nz <= 256";
      return 56;  // PETSC_ERR_SUP
    }
    if (opt.lv1_kernel == 3 && !ic_stg_ok) {
      err = "-pmf_lv1_kernel staged needs every subdomain 16 cells wide in x with x0 % 4 == 0, M % 4 == 0, "
            "ny <= 16 and nz <= 16";
      return 56;  // PETSC_ERR_SUP
    }
  }
  cudaEventRecord(e[1], st);
  // level-2 local eigenproblems
  if (!d_eig1 || !d_ks || !d_iters || !d_status) {
    for (void* q : {(void*)d_eig1, (void*)d_ks, (void*)d_iters, (void*)d_status})
      if (q) cudaFree(q);
    d_eig1 = nullptr;
    d_ks = d_iters = d_status = nullptr;
    if (int er = dalloc((void**)&d_eig1, sizeof(double) * nsub * opt.en_lv1, "local eigenvalues")) return er;
    if (int er = dalloc((void**)&d_ks, sizeof(int) * nsub, "local eigen counts")) return er;
    if (int er = dalloc((void**)&d_iters, sizeof(int) * nsub, "eigensolver iterations")) return er;
    if (int er = dalloc((void**)&d_status, sizeof(int) * nsub, "eigensolver status")) return er;
  }
  int dev = 0, nsm = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  const int eig_blocks = std::min(nsub, opt.eig_ctas > 0 ? opt.eig_ctas : nsm);
  LobpcgArgs la;
  la.g = g;
  la.subs = d_subs;
  la.nsub = nsub;
  la.k = opt.en_lv1;
  la.m = opt.en_lv1 + opt.eig_guard;
  la.kmax = kmax;
  la.eg_op = opt.eg_op;
  la.max_it = opt.eig_max_it;
  la.tol = opt.eig_tol > 0 ? opt.eig_tol : (eig32() ? 1e-6 : 1e-8);
  if (mixed && !eig32() && !phi64)
    if (int er = dalloc((void**)&phi64, sizeof(double) * (size_t)g.ncell * kmax, "FP64 eigenvectors")) return er;
  la.sigma_rel = opt.eig_sigma;
  la.seed = opt.seed;
  la.tx = tx;
  la.ty = ty;
  la.tz = tz;
  la.diag = diag;
  la.db = db;
  la.kx = kx;
  la.ky = ky;
  la.kz = kz;
  la.Hx = H[0];
  la.Hy = H[1];
  la.Hz = H[2];
  la.meas = H[0] * H[1] * H[2];
  la.xinit = nullptr;
  la.xinit_patch = nullptr;
  la.xinit_k = 0;
  la.sub_list = nullptr;
  la.nlist = nullptr;
  if (!d_queue)
    if (int er = dalloc((void**)&d_queue, sizeof(int), "eigensolver queue")) return er;
  la.queue = d_queue;
  la.mode = 0;
  la.rel_floor = opt.eig_rel_floor;
  la.final_batched = opt.eig_final;
  la.init_batched = opt.eig_init;
  la.slab = nullptr;
  la.slab_stride = 0;
  la.state = nullptr;
  la.dirichlet_mask = dmask;
  la.probs = d_probs;
  la.ld = 0;
  la.prof = nullptr;
  long long* d_prof = nullptr;
  const bool prof_eig = getenv("PMF_PROFILE_EIGEN") != nullptr;
  if (prof_eig) {
    if (int er = dalloc((void**)&d_prof, sizeof(long long) * 16 * eig_blocks, "eigensolver probe")) return er;
    cudaMemsetAsync(d_prof, 0, sizeof(long long) * 16 * eig_blocks, st);
    la.prof = d_prof;
  }
  const size_t need = ((lobpcg_work_bytes(max_cells, la.m, eig32() ? 4 : 8) + 255) & ~(size_t)255) * eig_blocks;
  if (eig_work_bytes < need) {
    if (eig_work) cudaFree(eig_work);
    if (int er = check(cudaMalloc(&eig_work, need), "cudaMalloc eigen work")) return er;
    eig_work_bytes = need;
  }
  const double eb1 = opt.eb_lv1 < 0 ? 1.0e12 : opt.eb_lv1;  // 1/NIL
  for (double& x : eig_phase_ms) x = 0.0;
  eig_colcells = 0;
  if (!opt.learned_path.empty()) {
    if (int er = run_learned_eigen(la, eig_blocks, eb1)) return er;
  } else {
    if (int er = run_eigen(la, nullptr, nsub, eig_blocks, eb1)) return er;
  }
  cudaEventRecord(e[2], st);
  if (int er = check(cudaStreamSynchronize(st), "local eigensolves")) return er;
  if (int er = check(cudaGetLastError(), "setup launch")) return er;
  if (prof_eig) {  // diagnostics: cycles per LOBPCG phase, summed over CTAs
    std::vector<long long> hp(16 * eig_blocks);
    cudaMemcpy(hp.data(), d_prof, sizeof(long long) * hp.size(), cudaMemcpyDeviceToHost);
    const char* names[15] = {"init",    "residual",  "precond",   "stencil",  "gram",     "pre_rr",   "update_aimg",
                             "final",   "rr_scale",  "rr_chol",   "rr_basis", "rr_proj",  "rr_jacobi", "rr_coef",
                             "update_mma"};
    long long tot[16] = {0}, mx = 0;
    for (int b = 0; b < eig_blocks; ++b) {
      long long sb = 0;
      for (int p = 0; p < 16; ++p) {
        tot[p] += hp[b * 16 + p];
        sb += hp[b * 16 + p];
      }
      mx = std::max(mx, sb);
    }
    fprintf(stderr, "[premixfem_b200] LOBPCG cycles per phase (sum over %d CTAs; slowest CTA %lld):", eig_blocks, mx);
    for (int p = 0; p < 15; ++p) fprintf(stderr, " %s=%lld", names[p], tot[p]);
    fprintf(stderr, "\n");
    cudaFree(d_prof);
  }
  ks.resize(nsub);
  eig_iters.resize(nsub);
  eig_status.resize(nsub);
  eig1.resize((size_t)nsub * opt.en_lv1);
  cudaMemcpy(ks.data(), d_ks, sizeof(int) * nsub, cudaMemcpyDeviceToHost);
  cudaMemcpy(eig_iters.data(), d_iters, sizeof(int) * nsub, cudaMemcpyDeviceToHost);
  if (!opt.learned_path.empty()) {
    // iterations from the learned start, plus the random restart where it was needed
    std::vector<int> it_l(nsub), st_l(nsub);
    cudaMemcpy(it_l.data(), d_iters_learned, sizeof(int) * nsub, cudaMemcpyDeviceToHost);
    cudaMemcpy(st_l.data(), d_status_learned, sizeof(int) * nsub, cudaMemcpyDeviceToHost);
    learned_used = 1;
    learned_fallbacks = 0;
    learned_iters = fallback_iters = 0;
    for (int s_ = 0; s_ < nsub; ++s_) {
      learned_iters += it_l[s_];
      if (st_l[s_] == 1) {
        ++learned_fallbacks;
        fallback_iters += eig_iters[s_];
        eig_iters[s_] += it_l[s_];
      }
    }
  }
  cudaMemcpy(eig_status.data(), d_status, sizeof(int) * nsub, cudaMemcpyDeviceToHost);
  cudaMemcpy(eig1.data(), d_eig1, sizeof(double) * eig1.size(), cudaMemcpyDeviceToHost);
  {
    // A local eigensolve that used its whole iteration budget keeps its last
    // Ritz block (status 1, counted by pmf_get_eigen_lv1); with
    // -pmf_eig_require_converged it is an error instead, as SLEPc's "cannot
    // find enough eigenvectors" is in the reference (src/PreMixFEM_3D.c:367)
    int nmax = 0;
    for (int s_ = 0; s_ < nsub; ++s_) nmax += eig_status[s_] == 1;
    if (nmax && opt.eig_require_converged) {
      err = "local eigensolver did not converge on " + std::to_string(nmax) + " of " + std::to_string(nsub) +
            " subdomains within -pmf_eig_max_it " + std::to_string(opt.eig_max_it) + " iterations";
      return 83;  // PETSC_ERR_USER
    }
  }
  for (int s = 0; s < nsub; ++s) subs[s].k = ks[s];
  cudaMemcpyAsync(d_subs, subs.data(), sizeof(SubInfo) * nsub, cudaMemcpyHostToDevice, st);
  // level-2 Galerkin (Phi^T A Phi) and per-rank inverses
  if (int er = rank_layout()) return er;
  if (!coarse_ok) {
    // all or nothing, as alloc_fine
    struct A {
      void** p;
      size_t bytes;
      const char* what;
    };
    const A list[] = {{(void**)&blk, sizeof(double) * nsub * 7 * kmax * kmax, "coarse blocks"},
                      {(void**)&gface, sizeof(double) * nsub * 6 * kmax * kmax, "coarse face blocks"},
                      {(void**)&A2inv, sizeof(double) * tot2, "level-2 inverses"},
                      {(void**)&AN, sizeof(double) * tot2, "rank-Neumann matrices"},
                      {(void**)&ANinv, sizeof(double) * tot2, "rank-Neumann inverses"},
                      {(void**)&V3, sizeof(double) * totv, "level-3 eigenvectors"},
                      {(void**)&d_eig3, sizeof(double) * nrank * en2, "level-3 eigenvalues"},
                      {(void**)&d_l3it, sizeof(int) * nrank, "level-3 iterations"},
                      {(void**)&A3inv, sizeof(double) * n3 * n3, "level-3 inverse"},
                      {(void**)&c, sizeof(double) * nsub * kmax, "coarse residual"},
                      {(void**)&dz, sizeof(double) * nsub * kmax, "coarse correction"},
                      {(void**)&Zacc, sizeof(double) * nsub * kmax, "coarse accumulator"},
                      {(void**)&d3, sizeof(double) * n3, "level-3 right-hand side"},
                      {(void**)&w3, sizeof(double) * n3, "level-3 solution"},
                      {(void**)&d_rank_nb, sizeof(int) * nrank * 6, "rank neighbours"}};
    const int nl = (int)(sizeof(list) / sizeof(list[0]));
    for (int i = 0; i < nl; ++i) {
      if (*list[i].p) cudaFree(*list[i].p);
      *list[i].p = nullptr;
    }
    for (int i = 0; i < nl; ++i) {
      if (int er = dalloc(list[i].p, list[i].bytes, list[i].what)) {
        for (int j = 0; j < i; ++j) {
          cudaFree(*list[j].p);
          *list[j].p = nullptr;
        }
        return er;
      }
    }
    coarse_ok = true;
  }
  if (mixed && !eig32()) launch_to_f32(phi64, (float*)phi, g.ncell * kmax, st);  // the basis the FP32 cycle uses
  if (mixed)
    launch_galerkin<float>(g, d_subs, nsub, kmax, tx, ty, tz, diag, (const float*)phi, blk, gface, st);
  else
    launch_galerkin<double>(g, d_subs, nsub, kmax, tx, ty, tz, diag, (const double*)phi, blk, gface, st);
  auto finish = [&]() -> int {
    if (int er = check(cudaStreamSynchronize(st), "coarse setup")) return er;
    if (int er = check(cudaGetLastError(), "coarse setup launch")) return er;
    float ms[5];
    for (int i = 0; i < 5; ++i) cudaEventElapsedTime(&ms[i], e[i], e[i + 1]);
    t_stages[ST_SU_LV1] += ms[0] * 1e-3;
    t_stages[ST_SU_LV2_1] += ms[1] * 1e-3;
    t_stages[ST_SU_LV2_2] += ms[2] * 1e-3;
    t_stages[ST_SU_LV3_1] += ms[3] * 1e-3;
    t_stages[ST_SU_LV3_2] += ms[4] * 1e-3;
    float tot;
    cudaEventElapsedTime(&tot, e[0], e[5]);
    t_stages[ST_SU] += tot * 1e-3;
    last_setup_ms = tot;
    // launch shapes of the preconditioner kernels (first set-up of a shape only)
    if (mixed)
      tune_pc<float>();
    else
      tune_pc<double>();
    if (int er = check(cudaStreamSynchronize(st), "launch-shape tuning")) return er;
    is_setup = true;
    return 0;
  };
  if (opt.use_2level) {
    // _PC_setup_lv2_c (:423-735): the global Galerkin matrix Phi^T A Phi over all
    // subdomains (+ NIL I unless -no_shift_A_cc), factorised by the banded
    // Cholesky in subdomain-grid order (k_coarse_band.cu)
    if (int er = setup_two_level()) return er;
    cudaEventRecord(e[3], st);
    cudaEventRecord(e[4], st);
    cudaEventRecord(e[5], st);
    eig3.clear();
    ks3.clear();
    l3_iters.clear();
    return finish();
  }
  launch_assemble_dense_r(d_subs, nrank, rl, tot2, blk, gface, 0, A2inv, st);
  if (ragged)
    launch_spd_inverse_r(rl, nrank, nr, A2inv, 1e-14, d_flag + 1, st);
  else
    launch_spd_inverse(nrank, nr, A2inv, 1e-14, d_flag + 1, st);
  cudaEventRecord(e[3], st);
  // level 3: rank-Neumann HEP
  launch_assemble_dense_r(d_subs, nrank, rl, tot2, blk, gface, 1, AN, st);
  cudaMemcpyAsync(ANinv, AN, sizeof(double) * tot2, cudaMemcpyDeviceToDevice, st);
  launch_add_diag_r(rl, nrank, ANinv, 1e-8, 1, st);
  if (ragged)
    launch_spd_inverse_r(rl, nrank, nr, ANinv, 1e-14, d_flag + 2, st);
  else
    launch_spd_inverse(nrank, nr, ANinv, 1e-14, d_flag + 2, st);
  if (!l3work) {
    if (int er = check(cudaMalloc(&l3work, sizeof(double) * totw), "cudaMalloc l3 work")) return er;
  }
  launch_dense_smallest_eig(rl, nrank, nr, en2, l3p, AN, ANinv, V3, d_eig3, d_l3it, opt.l3_tol, opt.l3_max_it, l3work,
                            st);
  if (int er = check(cudaStreamSynchronize(st), "level-3 eigensolve")) return er;
  eig3.resize((size_t)nrank * en2);
  l3_iters.resize(nrank);
  cudaMemcpy(eig3.data(), d_eig3, sizeof(double) * eig3.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(l3_iters.data(), d_l3it, sizeof(int) * nrank, cudaMemcpyDeviceToHost);
  const double eb2 = opt.eb_lv2 < 0 ? 1.0e12 : opt.eb_lv2;
  ks3.assign(nrank, en2);
  for (int rr = 0; rr < nrank; ++rr)
    for (int j = 0; j < en2; ++j)
      if (eig3[(size_t)rr * en2 + j] >= eb2) {  // :1100-1115
        ks3[rr] = j + 1;
        break;
      }
  std::vector<int> rnb((size_t)nrank * 6, -1);
  for (int rr = 0; rr < nrank && !nprob; ++rr) {
    const int px = rank_grid[0], py = rank_grid[1], pz = rank_grid[2];
    const int rx = rr % px, ry = (rr / px) % py, rz = rr / (px * py);
    auto at = [&](int x, int y, int zz) { return (x < 0 || y < 0 || zz < 0 || x >= px || y >= py || zz >= pz) ? -1 : (zz * py + y) * px + x; };
    rnb[rr * 6 + 0] = at(rx - 1, ry, rz);
    rnb[rr * 6 + 1] = at(rx + 1, ry, rz);
    rnb[rr * 6 + 2] = at(rx, ry - 1, rz);
    rnb[rr * 6 + 3] = at(rx, ry + 1, rz);
    rnb[rr * 6 + 4] = at(rx, ry, rz - 1);
    rnb[rr * 6 + 5] = at(rx, ry, rz + 1);
  }
  if (!d_ks3)
    if (int er = dalloc((void**)&d_ks3, sizeof(int) * nrank, "level-3 counts")) return er;
  cudaMemcpyAsync(d_ks3, ks3.data(), sizeof(int) * nrank, cudaMemcpyHostToDevice, st);
  cudaMemcpyAsync(d_rank_nb, rnb.data(), sizeof(int) * nrank * 6, cudaMemcpyHostToDevice, st);
  { note_launch(); k_zero_v_cols<<<std::min(nrank, 1024), 256, 0, st>>>(nrank, rl, en2, V3, d_ks3); }
  cudaEventRecord(e[4], st);
  { note_launch(); k_zero_d<<<256, 256, 0, st>>>(A3inv, (long long)n3 * n3); }
  { note_launch(); k_build_a3<<<nrank * 7, 64, 0, st>>>(d_subs, rl, en2, blk, V3, d_rank_nb, d_ks3, A3inv, n3,
                                       opt.no_shift_A_cc ? 0.0 : 1.0e-12); }
  launch_spd_inverse(1, n3, A3inv, 1e-14, d_flag + 3, st);
  cudaEventRecord(e[5], st);
  return finish();
}

// -use_2level: plan, allocate (once per plan) and factorise the banded
// global coarse matrix.  The factor and the superblock inverses take
// T_bytes + X_bytes of device memory (about 0.65 GB for 24 576 unknowns,
// 8.8 GB for 131 072); a device without room for them gets error 55.
int Solver::setup_two_level() {
  const int grid[3] = {opt.vranks[0] * opt.sd[0], opt.vranks[1] * opt.sd[1], opt.vranks[2] * opt.sd[2]};
  CBandPlan p;
  if (int e = cband_plan(subs, grid, kmax, &p)) {
    err = "-use_2level: the subdomains do not form a grid";
    return e;
  }
  const size_t vec = (size_t)p.NTp * 64 * sizeof(double);
  if (!cb_T || p.NTp != cband.NTp || p.B != cband.B) {
    for (void** q : {(void**)&cb_T, (void**)&cb_X, (void**)&cb_v, (void**)&cb_y, (void**)&cb_t, (void**)&cb_part,
                     (void**)&cb_perm, (void**)&cb_null, (void**)&cb_scale}) {
      if (*q) cudaFree(*q);
      *q = nullptr;
    }
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    const size_t need = p.T_bytes + p.X_bytes + 3 * vec + p.perm.size() * 8 + (256u << 20);
    if (need > freeb) {
      err = "-use_2level: not enough device memory for the banded coarse factor (" + std::to_string(need >> 20) +
            " MiB needed, " + std::to_string(freeb >> 20) + " MiB free)";
      return 55;  // PETSC_ERR_MEM
    }
    int e = dalloc((void**)&cb_T, p.T_bytes, "coarse band factor");
    if (!e) e = dalloc((void**)&cb_X, p.X_bytes, "coarse superblock inverses");
    if (!e) e = dalloc((void**)&cb_v, vec, "coarse work");
    if (!e) e = dalloc((void**)&cb_y, vec, "coarse work");
    if (!e) e = dalloc((void**)&cb_t, vec, "coarse work");
    if (!e) e = dalloc((void**)&cb_part, (size_t)p.B * p.B * 64 * sizeof(double), "coarse partial sums");
    if (!e) e = dalloc((void**)&cb_perm, p.perm.size() * sizeof(int), "coarse ordering");
    if (!e) e = dalloc((void**)&cb_null, p.perm.size() * sizeof(int), "coarse null flags");
    if (!e) e = dalloc((void**)&cb_scale, sizeof(double), "coarse scale");
    if (e) return e;
    cudaMemcpyAsync(cb_perm, p.perm.data(), p.perm.size() * sizeof(int), cudaMemcpyHostToDevice, st);
    // the plan's host vector must outlive the copy
    if (int er = check(cudaStreamSynchronize(st), "coarse ordering")) return er;
  }
  cband = p;
  launch_cband_factor(d_subs, kmax, blk, cb_perm, cband, opt.no_shift_A_cc ? 0.0 : 1.0e-12, 1e-14, cb_T, cb_X,
                      cb_null, d_flag + 1, cb_scale, st);
  return 0;
}

// -use_full_Cholesky_lv1 (src/PreMixFEM_3D.c:205-207): banded Cholesky factors
// of every subdomain block, FP64 (plus an FP32 copy for the mixed form).
int Solver::setup_band_cholesky(bool mixed) {
  std::vector<long long> off(nsub);
  long long len = 0;
  int mb = 0;
  for (int s = 0; s < nsub; ++s) {
    const SubInfo& S = subs[s];
    const int b = S.nx * S.ny;
    off[s] = len;
    len += (long long)S.nx * S.ny * S.nz * band_ld_host(b);
    mb = std::max(mb, b);
  }
  if ((2LL * mb + 8) * 8 * 8 > 227 * 1024) {
    err = "subdomain too wide for the banded Cholesky factorisation (nx*ny <= 1800)";
    return 62;
  }
  if (len != band_len) {
    if (band64) cudaFree(band64);
    if (band32) cudaFree(band32);
    band64 = nullptr;
    band32 = nullptr;
    size_t freeb = 0, totb = 0;
    cudaMemGetInfo(&freeb, &totb);
    const size_t need = (size_t)len * (8 + (mixed ? 4 : 0));
    if (need + (256u << 20) > freeb) {
      err = "not enough device memory for the level-1 Cholesky factors";
      return 55;  // PETSC_ERR_MEM
    }
    if (int er = check(cudaMalloc(&band64, sizeof(double) * len), "cudaMalloc Cholesky factors")) return er;
    band_len = len;
  }
  if (mixed && !band32)
    if (int er = check(cudaMalloc(&band32, sizeof(float) * len), "cudaMalloc Cholesky factors (FP32)")) return er;
  if (!d_boff)
    if (int er = dalloc((void**)&d_boff, sizeof(long long) * nsub, "Cholesky offsets")) return er;
  cudaMemcpyAsync(d_boff, off.data(), sizeof(long long) * nsub, cudaMemcpyHostToDevice, st);
  launch_band_chol_factor(g, d_subs, nsub, mb, tx, ty, tz, diag, d_boff, band64, d_flag, st);
  if (mixed) launch_to_f32(band64, band32, len, st);
  // the host vector must outlive the asynchronous copy
  return check(cudaStreamSynchronize(st), "level-1 Cholesky factorisation");
}

// The subdomain-blocked copy of the IC(0) factor for k_ic_apply_blk, when
// every subdomain fits that kernel (16 cells wide in x, 16-byte aligned
// rows, at most 256 x-lines); rebuilt by every set-up.
int Solver::setup_ic_blocked(bool mixed) {
  ic_blk_ok = max_lines <= 256;
  ic_stg_ok = true;
  for (const SubInfo& S : subs) {
    if (S.nx != 16) ic_blk_ok = false;
    if (S.ny > 16 || S.nz > 16) ic_stg_ok = false;
  }
  const size_t smem = mixed ? ic_blk_smem_bytes<float>(max_cells) : ic_blk_smem_bytes<double>(max_cells);
  if (smem > 227 * 1024) ic_blk_ok = false;
  const size_t smem_stg = mixed ? ic_stg_smem_bytes<float>(max_cells) : ic_stg_smem_bytes<double>(max_cells);
  ic_stg_ok = ic_stg_ok && ic_blk_ok && smem_stg <= 227 * 1024;
  if (!d_kerr) {
    if (int e = dalloc((void**)&d_kerr, sizeof(int), "kernel wait flag")) return e;
    cudaMemsetAsync(d_kerr, 0, sizeof(int), st);
  }
  if (!ic_blk_ok) return 0;
  if (!d_coff) {
    std::vector<long long> off(nsub);
    long long acc = 0;
    for (int s = 0; s < nsub; ++s) {
      off[s] = acc;
      acc += (long long)subs[s].nx * subs[s].ny * subs[s].nz;
    }
    if (int e = dalloc((void**)&d_coff, sizeof(long long) * nsub, "blocked factor offsets")) return e;
    if (int e = dalloc(&ic_coef, (size_t)acc * ic_blk_coef_bytes(mixed ? 4 : 8), "blocked IC(0) factor")) {
      cudaFree(d_coff);
      d_coff = nullptr;
      return e;
    }
    cudaMemcpyAsync(d_coff, off.data(), sizeof(long long) * nsub, cudaMemcpyHostToDevice, st);
    // the host vector must outlive the asynchronous copy
    if (int e = check(cudaStreamSynchronize(st), "blocked factor offsets")) return e;
  }
  if (mixed)
    launch_pack_ic_coef<float>(g, d_subs, nsub, d_coff, tx32, ty32, tz32, inv32, ic_coef, st);
  else
    launch_pack_ic_coef<double>(g, d_subs, nsub, d_coff, tx, ty, tz, inv64, ic_coef, st);
  return 0;
}

// A bounded wait inside a kernel ran out (the kernel recorded it and returned
// without computing): report it as a library failure.
int Solver::check_kernel_flag(const char* what) {
  if (!d_kerr) return 0;
  int f = 0;
  if (int e = check(cudaMemcpy(&f, d_kerr, sizeof(int), cudaMemcpyDeviceToHost), what)) return e;
  if (f) {
    cudaMemset(d_kerr, 0, sizeof(int));
    err = std::string(what) + ": a level-1 kernel's wait for its bulk copy ran out";
    return 76;
  }
  return 0;
}

// One level-1 visit: out = yin + IC^-1 (x - A yin) with the tuned kernel.
template <typename T>
void Solver::launch_lv1(const double* x, const T* yin, T* out_t, double* out_d, double* partial, const int* done) {
  const bool f32 = sizeof(T) == 4;
  const T* ttx = f32 ? (const T*)tx32 : (const T*)tx;
  const T* tty = f32 ? (const T*)ty32 : (const T*)ty;
  const T* ttz = f32 ? (const T*)tz32 : (const T*)tz;
  const T* tdg = f32 ? (const T*)diag32 : (const T*)diag;
  const int kind = yin ? 1 : 0;
  if (ic_variant[kind] == 2 && ic_stg_ok) {
    launch_ic_apply_stg<T>(g, d_subs, nsub, max_cells, d_coff, ic_coef, ttx, tty, ttz, tdg, x, yin, out_t, out_d,
                           partial, done, d_kerr, st);
  } else if (ic_variant[kind] >= 1 && ic_blk_ok) {
    launch_ic_apply_blk<T>(g, d_subs, nsub, max_cells, d_coff, ic_coef, ttx, tty, ttz, tdg, x, yin, out_t, out_d,
                           partial, done, d_kerr, st, ic_blk_threads[kind]);
  } else {
    const T* tinv = f32 ? (const T*)inv32 : (const T*)inv64;
    launch_ic_apply<T>(g, d_subs, nsub, max_lines, max_cells, ttx, tty, ttz, tdg, tinv, x, yin, out_t, out_d,
                       partial, done, st, ic_threads);
  }
}

// Threads per subdomain of the level-1 solve and of the level-2 restriction /
// prolongation, chosen by the launch-shape tuner on scratch buffers (the first
// set-up of a shape times every candidate; later set-ups reuse the choice).
template <typename T>
void Solver::tune_pc() {
  const bool f32 = sizeof(T) == 4;
  const T* ttx = f32 ? (const T*)tx32 : (const T*)tx;
  const T* tty = f32 ? (const T*)ty32 : (const T*)ty;
  const T* ttz = f32 ? (const T*)tz32 : (const T*)tz;
  const T* tdg = f32 ? (const T*)diag32 : (const T*)diag;
  const T* tinv = f32 ? (const T*)inv32 : (const T*)inv64;
  const T* tphi = (const T*)phi;
  T* ya = (T*)y0;
  T* yo = (T*)y1;
  cudaMemsetAsync(ya, 0, sizeof(T) * g.ncell, st);
  cudaMemsetAsync(z, 0, sizeof(double) * g.ncell, st);
  cudaMemsetAsync(Zacc, 0, sizeof(double) * nsub * kmax, st);
  const int old[8] = {ic_threads,    rr_threads,    pr_threads,        pcga_variant,
                      ic_variant[0], ic_variant[1], ic_blk_threads[0], ic_blk_threads[1]};
  char key[192];
  const char* prec = f32 ? "f32" : "f64";
  if (!opt.use_full_Cholesky_lv1) {
    const int base = std::max(64, ((max_lines + 31) / 32) * 32);
    std::vector<int> cand = {base};
    for (int t : {384, 512, 768, 1024})
      if (t > base) cand.push_back(t);
    // candidates per visit kind (first visit: no iterate; later visits: with
    // one): the natural-order kernel with each thread count, then the blocked
    // kernel with 512 and 256 threads (when every subdomain fits it) and its
    // staged form (when every subdomain also has ny, nz <= 16).  The natural
    // kernel's thread count is tuned on the visits with an iterate.
    const int nnat = (int)cand.size();
    const int nblk = ic_blk_ok ? (ic_stg_ok ? 3 : 2) : 0;
    const int blk_threads[2] = {512, 256};
    // The visits with an iterate are timed in the form the V-cycle's last
    // visit takes (FP64 result and the z.r partials, into p0 and part, which
    // hold nothing yet); the first visit writes the preconditioner's iterate.
    for (int kind = 1; kind >= 0; --kind) {
      snprintf(key, sizeof(key), "ic_apply|%s|n%d|c%d|l%d|b%d|y%d|f", prec, nsub, max_cells, max_lines, nblk, kind);
      const int ncand = kind == 1 ? nnat + nblk : 1 + nblk;
      T* o_t = kind ? nullptr : yo;
      double* o_d = kind ? p0 : nullptr;
      double* o_p = kind ? part : nullptr;
      const int ci = tune_choose(key, ncand, [&](int i) {
        const int nn = kind == 1 ? nnat : 1;
        if (i < nn)
          launch_ic_apply<T>(g, d_subs, nsub, max_lines, max_cells, ttx, tty, ttz, tdg, tinv, z, kind ? ya : nullptr,
                             o_t, o_d, o_p, nullptr, st, kind ? cand[i] : ic_threads);
        else if (i - nn < 2)
          launch_ic_apply_blk<T>(g, d_subs, nsub, max_cells, d_coff, ic_coef, ttx, tty, ttz, tdg, z,
                                 kind ? ya : nullptr, o_t, o_d, o_p, nullptr, d_kerr, st, blk_threads[i - nn]);
        else
          launch_ic_apply_stg<T>(g, d_subs, nsub, max_cells, d_coff, ic_coef, ttx, tty, ttz, tdg, z,
                                 kind ? ya : nullptr, o_t, o_d, o_p, nullptr, d_kerr, st);
        return true;
      }, st);
      const int nn = kind == 1 ? nnat : 1;
      ic_variant[kind] = ci < nn ? 0 : (ci - nn < 2 ? 1 : 2);
      if (ci >= nn && ci - nn < 2) ic_blk_threads[kind] = blk_threads[ci - nn];
      if (kind == 1) ic_threads = cand[std::min(ci, nnat - 1)];
      if (opt.lv1_kernel == 1) ic_variant[kind] = 0;
      if (opt.lv1_kernel == 2) ic_variant[kind] = 1;  // eligibility checked by setup()
      if (opt.lv1_kernel == 3) ic_variant[kind] = 2;
    }
  }
  const int rcand[3] = {256, 128, 512};
  snprintf(key, sizeof(key), "resid_restrict|%s|n%d|c%d|k%d", prec, nsub, max_cells, kmax);
  rr_threads = rcand[tune_choose(key, 3, [&](int i) {
    launch_resid_restrict<T>(g, d_subs, nsub, kmax, ttx, tty, ttz, tdg, tphi, z, ya, c, nullptr, st, rcand[i]);
    return true;
  }, st)];
  snprintf(key, sizeof(key), "prolong|%s|n%d|c%d|k%d", prec, nsub, max_cells, kmax);
  pr_threads = rcand[tune_choose(key, 3, [&](int i) {
    launch_prolong<T>(g, d_subs, nsub, kmax, tphi, Zacc, yo, nullptr, st, rcand[i]);
    return true;
  }, st)];
  // the CG step's fused p-update + operator kernel: 2.5-D march or grid-stride
  // (the main kernel alone is timed, in the state of a later iteration, whose
  // p = z + (beta/betaold) p reads the previous p; not done)
  {
    PcgState hs;
    memset(&hs, 0, sizeof(hs));
    hs.first = 0;
    hs.beta = hs.betaold = 1.0;
    hs.dpi = 1.0;
    cudaMemsetAsync(p0, 0, sizeof(double) * g.ncell, st);
    cudaMemcpyAsync(state, &hs, sizeof(hs), cudaMemcpyHostToDevice, st);
    cudaStreamSynchronize(st);
    snprintf(key, sizeof(key), "pcg_iter_a|M%d|N%d|P%d|p3", g.M, g.N, g.P);
    pcga_variant = tune_choose(key, 3, [&](int i) {
      launch_pcg_iter_a_main(g, tx, ty, tz, diag, z, p0, p1, w, part, state, st, i);
      return true;
    }, st);
  }
  if (pcg_exec && (old[0] != ic_threads || old[1] != rr_threads || old[2] != pr_threads || old[3] != pcga_variant ||
                   old[4] != ic_variant[0] || old[5] != ic_variant[1] || old[6] != ic_blk_threads[0] ||
                   old[7] != ic_blk_threads[1])) {
    cudaGraphExecDestroy(pcg_exec);  // captured with other launch shapes
    pcg_exec = nullptr;
    pcg_graph_x = nullptr;
  }
}

template <typename T>
void Solver::apply_impl(const double* x, double* out, double* partial, const int* done) {
  const bool f32 = sizeof(T) == 4;
  const T* ttx = f32 ? (const T*)tx32 : (const T*)tx;
  const T* tty = f32 ? (const T*)ty32 : (const T*)ty;
  const T* ttz = f32 ? (const T*)tz32 : (const T*)tz;
  const T* tdg = f32 ? (const T*)diag32 : (const T*)diag;
  const T* tphi = (const T*)phi;
  T* yb[2] = {(T*)y0, (T*)y1};
  const std::vector<int> sch = schedule();
  int cur = 0;
  bool y_zero = true, z_pend = false, c_valid = false;
  const long long ncoarse = (long long)nsub * kmax;
  for (size_t idx = 0; idx < sch.size(); ++idx) {
    const int v = sch[idx];
    const bool last = idx + 1 == sch.size();
    if (v == 1) {
      if (z_pend) {
        launch_prolong<T>(g, d_subs, nsub, kmax, tphi, Zacc, yb[cur], done, st, pr_threads);
        prof_mark(PROF_PROLONG);
        z_pend = false;
      }
      const T* yin = y_zero ? nullptr : yb[cur];
      const int lv1_slot = y_zero ? PROF_LV1_FIRST : PROF_LV1_Y;
      if (opt.use_full_Cholesky_lv1) {
        const T* tband = f32 ? (const T*)band32 : (const T*)band64;
        if (last)
          launch_band_chol_apply<T>(g, d_subs, nsub, max_cells, ttx, tty, ttz, tdg, d_boff, tband, x, yin, nullptr,
                                    out, partial, done, st);
        else {
          launch_band_chol_apply<T>(g, d_subs, nsub, max_cells, ttx, tty, ttz, tdg, d_boff, tband, x, yin,
                                    yb[1 - cur], nullptr, nullptr, done, st);
          cur = 1 - cur;
        }
      } else if (last)
        launch_lv1<T>(x, yin, nullptr, out, partial, done);
      else {
        launch_lv1<T>(x, yin, yb[1 - cur], nullptr, nullptr, done);
        cur = 1 - cur;
      }
      prof_mark(lv1_slot);
      y_zero = false;
      c_valid = false;
    } else {
      if (!c_valid) {
        if (z_pend) {
          launch_prolong<T>(g, d_subs, nsub, kmax, tphi, Zacc, yb[cur], done, st, pr_threads);
          prof_mark(PROF_PROLONG);
          z_pend = false;
        }
        launch_resid_restrict<T>(g, d_subs, nsub, kmax, ttx, tty, ttz, tdg, tphi, x, y_zero ? nullptr : yb[cur], c,
                                 done, st, rr_threads);
        prof_mark(PROF_RESTRICT);
        c_valid = true;
      }
      if (v == 2) {
        launch_block_gemv_r(rl, ncoarse, A2inv, c, dz, done, st);
      } else if (v == 4) {  // _PC_apply_vec_lv2_2level (:1481-1537)
        launch_cband_solve(cb_perm, cband, cb_T, cb_X, c, dz, cb_v, cb_y, cb_t, cb_part, done, st);
      } else {
        launch_lv3_restrict_r(rl, nrank, en2, V3, c, d3, done, st);
        launch_block_gemv(1, n3, A3inv, d3, w3, 0, done, st);
        launch_lv3_prolong_r(rl, ncoarse, en2, V3, w3, dz, done, st);
      }
      if (z_pend)
        launch_axpy(ncoarse, 1.0, dz, Zacc, done, st);
      else
        launch_copy(ncoarse, dz, Zacc, done, st);
      z_pend = true;
      const bool next_coarse = !last && sch[idx + 1] != 1;
      if (next_coarse)
        launch_a2_mult(d_subs, nsub, kmax, blk, dz, c, c, done, st);
      else
        c_valid = false;
      prof_mark(PROF_COARSE);
    }
  }
}

// PCG of every problem of the batch at once (KSPCG per problem, as Solver::solve
// for one): the CG steps are per-problem kernels over 2-D grids, the
// preconditioner the shared cycle, skipped once every problem has stopped.
// its, rnorm, reason: one entry per problem.
int Solver::solve_batch(const double* b_in, double* x_out, bool on_device, int* its, double* rnorm, int* reason) {
  if (!nprob) {
    err = "not a batch of problems";
    return 73;
  }
  if (!is_setup) {
    err = "setup not done";
    return 73;
  }
  if (opt.null_space) {
    err = "a batch solve has no constant null space option";
    return 56;
  }
  if (!bstate) {
    int e = dalloc((void**)&bstate, sizeof(PcgState) * nprob, "batch CG states");
    if (!e) e = dalloc((void**)&d_all_done, sizeof(int), "batch CG flag");
    if (!e) e = check(cudaMallocHost(&h_bstate, sizeof(PcgState) * nprob), "pinned batch CG states");
    if (!e) e = check(cudaMallocHost(&h_all_done, sizeof(int)), "pinned batch CG flag");
    if (e) return e;
  }
  const size_t n = (size_t)g.ncell;
  const double* bs = b_in;
  double* xs = x_out;
  if (!on_device) {
    cudaMemcpyAsync(vb, b_in, n * 8, cudaMemcpyHostToDevice, st);
    bs = vb;
    xs = vx;
  }
  // entries outside every problem stay zero in every CG vector
  for (double* v : {z, p0, p1, w, r, xs}) cudaMemsetAsync(v, 0, n * 8, st);
  const int nblk = bpcg_blocks();
  cudaEventRecord(ev0, st);
  launch_bpcg_start(d_probs, nprob, bs, xs, r, part, bstate, opt.rtol, opt.atol, opt.max_it, d_all_done, nblk, st);
  apply(r, z, part, d_all_done);
  launch_bpcg_beta(d_probs, nprob, part, bstate, st);
  double* pin = p0;
  double* pout = p1;
  const int chunk = std::max(2, opt.pcg_chunk & ~1);  // even: the p buffers return to their roles
  auto enqueue_chunk = [&]() {
    for (int c_ = 0; c_ < chunk; ++c_) {
      launch_bpcg_iter_a(g, d_probs, d_layer_prob, nprob, tx, ty, tz, diag, z, pin, pout, w, part, bstate, nblk, st);
      launch_bpcg_iter_b(d_probs, nprob, xs, r, pout, w, part, bstate, d_all_done, nblk, st);
      apply(r, z, part, d_all_done);
      launch_bpcg_beta(d_probs, nprob, part, bstate, st);
      std::swap(pin, pout);
    }
  };
  const bool use_graph = opt.pcg_graph != 0;
  if (use_graph && (!bpcg_exec || bpcg_graph_x != xs)) {
    if (bpcg_exec) cudaGraphExecDestroy(bpcg_exec);
    bpcg_exec = nullptr;
    const unsigned long long l0 = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
    cudaGraph_t graph = nullptr;
    if (int e = check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture")) return e;
    enqueue_chunk();
    if (int e = check(cudaStreamEndCapture(st, &graph), "graph capture")) return e;
    bpcg_graph_kernels = __atomic_load_n(&g_launches, __ATOMIC_RELAXED) - l0;
    __atomic_fetch_sub(&g_launches, bpcg_graph_kernels, __ATOMIC_RELAXED);  // captured, not launched
    const cudaError_t ie = cudaGraphInstantiate(&bpcg_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int e = check(ie, "graph instantiate")) return e;
    bpcg_graph_x = xs;
  }
  int guard = 0;
  for (;;) {
    if (use_graph) {
      if (int e = check(cudaGraphLaunch(bpcg_exec, st), "graph launch")) return e;
      __atomic_fetch_add(&g_launches, bpcg_graph_kernels, __ATOMIC_RELAXED);
    } else {
      enqueue_chunk();
    }
    cudaMemcpyAsync(h_all_done, d_all_done, sizeof(int), cudaMemcpyDeviceToHost, st);
    if (int e = check(cudaStreamSynchronize(st), "batch KSPSolve")) return e;
    if (int e = check(cudaGetLastError(), "batch KSPSolve launch")) return e;
    if (*h_all_done) break;
    if (++guard * chunk > opt.max_it + 8) break;
  }
  cudaEventRecord(ev1, st);
  cudaMemcpyAsync(h_bstate, bstate, sizeof(PcgState) * nprob, cudaMemcpyDeviceToHost, st);
  if (!on_device) cudaMemcpyAsync(x_out, xs, n * 8, cudaMemcpyDeviceToHost, st);
  int e = check(cudaStreamSynchronize(st), "batch KSPSolve");
  if (!e) e = check_kernel_flag("batch KSPSolve");
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  last_solve_ms = ms;
  last_its = 0;
  for (int q = 0; q < nprob; ++q) {
    const PcgState& s = h_bstate[q];
    if (its) its[q] = s.its;
    if (rnorm) rnorm[q] = s.dp;
    if (reason) reason[q] = s.done ? s.done : 2;
    last_its = std::max(last_its, s.its);
  }
  return e;
}

void Solver::prof_mark(int slot) {
  if (!prof_on || prof_n >= 64) return;
  cudaEventRecord(prof_ev[prof_n], st);
  prof_slot[prof_n++] = slot;
}

// One PCG iteration's kernels (CG p-update + A p, x/r update, the whole
// preconditioner application, beta) run `reps` times outside any graph, with
// an event after each launch group; ms[c] is the mean device time per
// iteration of class c, launches[c] its launch groups per iteration.  Runs on
// scratch: the solution and residual go to the host-staging buffers vx, vb and
// the CG scalars to the solver's state (reset here, rewritten by every solve).
int Solver::profile_iteration(int reps, double ms[PROF_SLOTS], int launches[PROF_SLOTS]) {
  if (!is_setup) {
    err = "setup not done";
    return 73;
  }
  for (int c_ = 0; c_ < PROF_SLOTS; ++c_) {
    ms[c_] = 0.0;
    launches[c_] = 0;
  }
  if (!prof_ev[0])
    for (auto& e : prof_ev)
      if (int er = check(cudaEventCreate(&e), "profile events")) return er;
  PcgState hs;
  memset(&hs, 0, sizeof(hs));
  hs.beta = hs.betaold = 1.0;
  hs.dpi = 1.0;  // a positive previous p.Ap: the indefinite test compares signs
  hs.max_it = 1 << 30;
  cudaMemcpyAsync(vb, r, sizeof(double) * g.ncell, cudaMemcpyDeviceToDevice, st);
  cudaMemsetAsync(vx, 0, sizeof(double) * g.ncell, st);
  cudaMemsetAsync(p0, 0, sizeof(double) * g.ncell, st);
  for (int rep = 0; rep < std::max(1, reps); ++rep) {
    *h_state = hs;
    cudaMemcpyAsync(state, h_state, sizeof(PcgState), cudaMemcpyHostToDevice, st);
    prof_n = 0;
    prof_on = true;
    prof_mark(-1);
    launch_pcg_iter_a(g, tx, ty, tz, diag, z, p0, p1, w, part, state, st, pcga_variant);
    prof_mark(PROF_CG_A);
    launch_pcg_iter_b(g.ncell, vx, vb, p1, w, part, state, st);
    prof_mark(PROF_CG_B);
    apply(vb, z, part, nullptr);
    if (opt.null_space)
      launch_pcg_null_beta(z, vb, g.ncell, part, zpart, state, st);
    else
      launch_pcg_beta_fin(part, nparts_apply(), state, st);
    prof_mark(PROF_BETA);
    prof_on = false;
    if (int er = check(cudaStreamSynchronize(st), "profile iteration")) return er;
    if (int er = check(cudaGetLastError(), "profile iteration launch")) return er;
    for (int i = 1; i < prof_n; ++i) {
      float t = 0.f;
      cudaEventElapsedTime(&t, prof_ev[i - 1], prof_ev[i]);
      const int c_ = prof_slot[i];
      if (c_ >= 0 && c_ < PROF_SLOTS) {
        ms[c_] += t;
        if (rep == 0) launches[c_] += 1;
      }
    }
  }
  for (int c_ = 0; c_ < PROF_SLOTS; ++c_) ms[c_] /= std::max(1, reps);
  return 0;
}

void Solver::apply(const double* x, double* out, double* partial, const int* done) {
  if (opt.precision == 1)
    apply_impl<float>(x, out, partial, done);
  else
    apply_impl<double>(x, out, partial, done);
}

int Solver::rhs(const double* source, double* out, bool on_device) {
  if (!tx) {
    err = "operator not assembled";
    return 73;
  }
  const size_t n = (size_t)g.ncell;
  cudaMemcpyAsync(vb, source, n * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
  launch_axpy(g.ncell, 1.0, bval, vb, nullptr, st);
  cudaMemcpyAsync(out, vb, n * 8, on_device ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st);
  return check(cudaStreamSynchronize(st), "rhs");
}

int Solver::apply_A(const double* x_in, double* y_out, bool on_device) {
  if (!tx) {
    err = "operator not assembled";
    return 73;
  }
  const size_t n = (size_t)g.ncell;
  const double* xs = x_in;
  double* ys = y_out;
  if (!on_device) {
    cudaMemcpyAsync(vx, x_in, n * 8, cudaMemcpyHostToDevice, st);
    xs = vx;
    ys = w;
  }
  launch_spmv(g, tx, ty, tz, diag, xs, ys, st);
  if (!on_device) cudaMemcpyAsync(y_out, ys, n * 8, cudaMemcpyDeviceToHost, st);
  return check(cudaStreamSynchronize(st), "apply_A");
}

int Solver::pc_apply(const double* x_in, double* y_out, bool on_device) {
  if (!is_setup) {
    err = "setup not done";
    return 73;
  }
  const size_t n = (size_t)g.ncell;
  const double* xs = x_in;
  double* ys = y_out;
  if (!on_device) {
    cudaMemcpyAsync(vx, x_in, n * 8, cudaMemcpyHostToDevice, st);
    xs = vx;
    ys = z;
  }
  cudaEventRecord(ev0, st);
  apply(xs, ys, part, nullptr);
  cudaEventRecord(ev1, st);
  if (!on_device) cudaMemcpyAsync(y_out, ys, n * 8, cudaMemcpyDeviceToHost, st);
  int e = check(cudaStreamSynchronize(st), "PC_apply_vec");
  if (!e) e = check(cudaGetLastError(), "PC_apply_vec launch");
  if (!e) e = check_kernel_flag("PC_apply_vec");
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  t_stages[ST_AV] += ms * 1e-3;
  return e;
}

int Solver::solve(const double* b_in, double* x_out, bool on_device, int* its, double* rnorm, int* reason) {
  if (nprob) {
    err = "a batch of problems is solved by pmf_batch_solve (one CG per problem)";
    return 73;
  }
  if (!is_setup) {
    err = "setup not done";
    return 73;
  }
  const size_t n = (size_t)g.ncell;
  const double* bs = b_in;
  double* xs = x_out;
  if (!on_device) {
    cudaMemcpyAsync(vb, b_in, n * 8, cudaMemcpyHostToDevice, st);
    bs = vb;
    xs = vx;
  }
  cudaEventRecord(ev0, st);
  launch_pcg_start(g, bs, xs, r, part, state, opt.rtol, opt.atol, opt.max_it, st);
  const int* done = &state->done;
  // beta = z.r from the preconditioner's partials, or of the projected z when
  // the operator carries the constant null space
  auto beta = [&]() {
    if (opt.null_space)
      launch_pcg_null_beta(z, r, g.ncell, part, zpart, state, st);
    else
      launch_pcg_beta_fin(part, nparts_apply(), state, st);
  };
  apply(r, z, part, done);
  beta();
  double* pin = p0;
  double* pout = p1;
  int guard = 0;
  const int chunk = std::max(1, opt.pcg_chunk);
  auto enqueue_chunk = [&]() {
    for (int c_ = 0; c_ < chunk; ++c_) {
      launch_pcg_iter_a(g, tx, ty, tz, diag, z, pin, pout, w, part, state, st, pcga_variant);
      launch_pcg_iter_b(g.ncell, xs, r, pout, w, part, state, st);
      apply(r, z, part, done);
      beta();
      std::swap(pin, pout);
    }
  };
  // A chunk of PCG iterations (each: p-update + A p, x/r update, the whole
  // preconditioner application, beta) as one CUDA graph: captured once per
  // solution buffer and replayed until the device-side `done` flag is set.
  // An even chunk returns the p buffers to their roles, so replays chain.
  const bool use_graph = opt.pcg_graph && chunk % 2 == 0;
  if (use_graph && (!pcg_exec || pcg_graph_x != xs || pcg_graph_ns != opt.null_space)) {
    if (pcg_exec) cudaGraphExecDestroy(pcg_exec);
    pcg_exec = nullptr;
    const unsigned long long l0 = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
    cudaGraph_t graph = nullptr;
    if (int e = check(cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal), "graph capture")) return e;
    enqueue_chunk();
    if (int e = check(cudaStreamEndCapture(st, &graph), "graph capture")) return e;
    const unsigned long long l1 = __atomic_load_n(&g_launches, __ATOMIC_RELAXED);
    pcg_graph_kernels = l1 - l0;
    __atomic_fetch_sub(&g_launches, pcg_graph_kernels, __ATOMIC_RELAXED);  // captured, not launched
    const cudaError_t ie = cudaGraphInstantiate(&pcg_exec, graph, 0);
    cudaGraphDestroy(graph);
    if (int e = check(ie, "graph instantiate")) return e;
    pcg_graph_x = xs;
    pcg_graph_ns = opt.null_space;
  }
  for (;;) {
    if (use_graph) {
      if (int e = check(cudaGraphLaunch(pcg_exec, st), "graph launch")) return e;
      __atomic_fetch_add(&g_launches, pcg_graph_kernels, __ATOMIC_RELAXED);
    } else {
      enqueue_chunk();
    }
    cudaMemcpyAsync(h_state, state, sizeof(PcgState), cudaMemcpyDeviceToHost, st);
    if (int e = check(cudaStreamSynchronize(st), "KSPSolve")) return e;
    if (int e = check(cudaGetLastError(), "KSPSolve launch")) return e;
    if (h_state->done) break;
    if (++guard > opt.max_it + 8) break;
  }
  cudaEventRecord(ev1, st);
  if (!on_device) cudaMemcpyAsync(x_out, xs, n * 8, cudaMemcpyDeviceToHost, st);
  int e = check(cudaStreamSynchronize(st), "KSPSolve");
  if (!e) e = check_kernel_flag("KSPSolve");
  float ms = 0;
  cudaEventElapsedTime(&ms, ev0, ev1);
  last_solve_ms = ms;
  last_its = h_state->its;
  if (its) *its = h_state->its;
  if (rnorm) *rnorm = h_state->dp;
  // the host guard stopped the loop before the device set a stop code: the
  // iteration budget is spent (KSP_DIVERGED_ITS)
  if (reason) *reason = h_state->done ? h_state->done : 2;
  return e;
}

}  // namespace pmf
