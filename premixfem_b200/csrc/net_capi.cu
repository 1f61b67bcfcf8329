// C ABI of the learned-initialisation network (training and inspection) and
// of the training-data gather from a set-up solver.  Every pointer argument
// except the file paths is device memory; work is enqueued on the legacy
// default stream.
#include <cuda_runtime.h>

#include <new>

#include "pmf_b200.h"
#include "pmf_net.h"
#include "solver.h"

struct pmf_net {
  pmf::Net n;
};

pmf::Solver* pmf_internal_solver(pmf_solver* h);
int pmf_internal_fail(int code, const char* msg);

static int net_fail(pmf_net* h, int code) { return code ? pmf_internal_fail(code, h->n.err.c_str()) : 0; }
static int launch_check(const char* what) {
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? 0 : pmf_internal_fail(76, (std::string(what) + ": " + cudaGetErrorString(e)).c_str());
}

extern "C" {

int pmf_net_create(unsigned long long seed, pmf_net** out) {
  if (!out) return pmf_internal_fail(62, "null output handle");
  pmf_net* h = new (std::nothrow) pmf_net;
  if (!h) return pmf_internal_fail(55, "out of host memory");
  if (int e = h->n.init(seed)) {
    const int r = net_fail(h, e);
    delete h;
    return r;
  }
  *out = h;
  return 0;
}

int pmf_net_load(const char* path, pmf_net** out) {
  if (!out || !path) return pmf_internal_fail(62, "null argument");
  pmf_net* h = new (std::nothrow) pmf_net;
  if (!h) return pmf_internal_fail(55, "out of host memory");
  if (int e = h->n.load(path)) {
    const int r = net_fail(h, e);
    delete h;
    return r;
  }
  *out = h;
  return 0;
}

int pmf_net_save(pmf_net* h, const char* path) {
  if (!h || !path) return pmf_internal_fail(62, "null argument");
  if (int e = h->n.save(path)) return pmf_internal_fail(e, "cannot write the weight file");
  return 0;
}

int pmf_net_destroy(pmf_net* h) {
  delete h;
  return 0;
}

int pmf_net_params(pmf_net* h) { return h ? h->n.params() : -62; }

int pmf_net_layer_info(int layer, int info[6]) {
  if (layer < 0 || layer >= pmf::NET_LAYERS || !info) return pmf_internal_fail(62, "layer index out of range");
  const pmf::NetLayer& L = pmf::kNetLayers[layer];
  info[0] = L.type;
  info[1] = L.cin;
  info[2] = L.cout;
  info[3] = L.s_in;
  info[4] = L.s_out;
  info[5] = pmf::net_taps(L.type);
  return 0;
}

int pmf_net_forward(pmf_net* h, const void* x, int B, float* y) {
  if (!h || !x || !y || B < 1) return pmf_internal_fail(62, "bad argument to pmf_net_forward");
  if (int e = h->n.forward((const __nv_bfloat16*)x, B, y, true, 0)) return net_fail(h, e);
  if (int e = launch_check("pmf_net_forward")) return e;
  if (int e = h->n.take_error()) return net_fail(h, e);
  return 0;
}

int pmf_net_backward(pmf_net* h, const float* dy, int B) {
  if (!h || !dy || B < 1) return pmf_internal_fail(62, "bad argument to pmf_net_backward");
  if (int e = h->n.backward(dy, B, 0)) return net_fail(h, e);
  return launch_check("pmf_net_backward");
}

int pmf_net_adam(pmf_net* h, float lr, float beta1, float beta2, float eps, float weight_decay) {
  if (!h) return pmf_internal_fail(62, "null network");
  h->n.adam(lr, beta1, beta2, eps, weight_decay, 0);
  return launch_check("pmf_net_adam");
}

int pmf_net_get_weights(pmf_net* h, int layer, float* w, float* b) {
  if (!h) return pmf_internal_fail(62, "null network");
  if (int e = h->n.get_weights(layer, w, b)) return pmf_internal_fail(e, "pmf_net_get_weights failed");
  return 0;
}

int pmf_net_set_weights(pmf_net* h, int layer, const float* w, const float* b) {
  if (!h) return pmf_internal_fail(62, "null network");
  if (int e = h->n.set_weights(layer, w, b)) return net_fail(h, e);
  return 0;
}

int pmf_net_get_grads(pmf_net* h, int layer, float* gw, float* gb) {
  if (!h) return pmf_internal_fail(62, "null network");
  if (int e = h->n.get_grads(layer, gw, gb)) return pmf_internal_fail(e, "pmf_net_get_grads failed");
  return 0;
}

int pmf_net_loss(const float* y, const float* V, const float* M, int B, int k, float* loss, float* dy) {
  if (!y || !V || !M || !loss || !dy || B < 1 || k < 1 || k > 8)
    return pmf_internal_fail(62, "bad argument to pmf_net_loss (k must be 1..8)");
  pmf::launch_net_loss(y, V, M, B, k, loss, dy, 0);
  return launch_check("pmf_net_loss");
}

int pmf_learned_patches(pmf_solver* h, void* feats, float* V, float* M) {
  pmf::Solver* s = pmf_internal_solver(h);
  if (!s) return pmf_internal_fail(62, "null solver handle");
  if (!s->is_setup) return pmf_internal_fail(73, "pmf_learned_patches needs a finished pmf_setup");
  for (const pmf::SubInfo& S : s->subs)
    if (S.nx > pmf::NET_S || S.ny > pmf::NET_S || S.nz > pmf::NET_S)
      return pmf_internal_fail(62, "pmf_learned_patches needs subdomains of at most 16^3 cells");
  int dmask = 0;
  for (int f = 0; f < 6; ++f)
    if (s->dir_on_[f]) dmask |= 1 << f;
  cudaStreamSynchronize(s->st);
  if (feats) pmf::launch_net_features(s->g, s->d_subs, s->nsub, s->kx, s->ky, s->kz, dmask, (__nv_bfloat16*)feats, 0);
  if (V && M) {
    pmf::NetTargetArgs a;
    a.g = s->g;
    a.subs = s->d_subs;
    a.nsub = s->nsub;
    a.k = s->opt.en_lv1;
    a.kmax = s->kmax;
    a.phi_f32 = s->opt.precision == 1;
    a.eg_op = s->opt.eg_op;
    a.dirichlet_mask = dmask;
    a.phi = s->phi;
    a.kx = s->kx;
    a.ky = s->ky;
    a.kz = s->kz;
    a.tx = s->tx;
    a.ty = s->ty;
    a.tz = s->tz;
    a.db = s->db;
    a.Hx = s->H[0];
    a.Hy = s->H[1];
    a.Hz = s->H[2];
    a.meas = s->H[0] * s->H[1] * s->H[2];
    a.V = V;
    a.Mw = M;
    pmf::launch_net_targets(a, 0);
  }
  if (cudaDeviceSynchronize() != cudaSuccess) return launch_check("pmf_learned_patches");
  return launch_check("pmf_learned_patches");
}

int pmf_get_learned_stats(pmf_solver* h, long long stats[4], double* net_ms) {
  pmf::Solver* s = pmf_internal_solver(h);
  if (!s || !stats) return pmf_internal_fail(62, "null argument");
  stats[0] = s->learned_used;
  stats[1] = s->learned_fallbacks;
  stats[2] = s->learned_iters;
  stats[3] = s->fallback_iters;
  if (net_ms) *net_ms = s->net_ms;
  return 0;
}

}  // extern "C"
