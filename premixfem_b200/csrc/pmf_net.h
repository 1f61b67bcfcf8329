// Learned initial blocks for the local eigensolves: a small 3-D convolutional
// encoder-decoder that maps a subdomain's log-permeability patch to k starting
// vectors for LOBPCG.  Weights are BF16 (FP32 master copies while training),
// activations BF16, accumulation FP32.
//
// Geometry: every sample is a 16^3 patch (a subdomain, zero-padded when it is
// smaller), channels-last: act[b][voxel][c], voxel = (z*16 + y)*16 + x.
//
// Layers (cin -> cout, patch edge in -> out):
//   0 conv3 16->32  16->16 relu        h1
//   1 down2 32->64  16->8  relu        h2
//   2 conv3 64->64   8->8  relu        h3
//   3 down2 64->96   8->4  relu        h4
//   4 conv3 96->96   4->4  relu        h5
//   5 up2   96->64   4->8  relu, +h3   u6
//   6 up2   64->32   8->16 relu, +h1   u7
//   7 conv3 32->32  16->16 relu        h8
//   8 conv1 32->16  16->16 linear      y (FP32; channels 0..k-1 used)
// conv3: 3x3x3, stride 1, zero padding 1; down2: 2x2x2, stride 2; up2:
// transposed 2x2x2, stride 2; conv1: 1x1x1.  Weights are stored
// W[tap][cin][cout] with tap = dz*9+dy*3+dx (conv3, d in {0,1,2} for offsets
// -1..1) or dz*4+dy*2+dx (down2/up2, d in {0,1}).  532 976 parameters.
#pragma once

#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <string>

#include "pmf_common.cuh"

namespace pmf {

constexpr int NET_S = 16;                       // patch edge
constexpr int NET_VOX = NET_S * NET_S * NET_S;  // 4096
constexpr int NET_CIN = 16;                     // input feature channels (5 used)
constexpr int NET_COUT = 16;                    // output channels (k used)
constexpr int NET_LAYERS = 9;
constexpr int NET_ACTS = 10;  // activations 0 (input) .. 9 (output)

enum NetLayerType { NL_CONV3 = 0, NL_DOWN2 = 1, NL_UP2 = 2, NL_CONV1 = 3 };

struct NetLayer {
  int type, cin, cout, s_in, s_out, relu, skip, in_act, out_act;
};

__host__ __device__ inline int net_taps(int type) {
  return type == NL_CONV3 ? 27 : (type == NL_CONV1 ? 1 : 8);
}

extern const NetLayer kNetLayers[NET_LAYERS];

struct NetActShape {
  int s, c;
};
extern const NetActShape kNetActs[NET_ACTS];

class Net {
 public:
  Net();
  ~Net();
  int init(unsigned long long seed);       // He-normal weights, zero biases
  int load(const char* path);              // BF16 weight file
  int save(const char* path) const;        // BF16 weight file
  int params() const;

  // y[b][4096][16] (FP32) for B input patches x[b][4096][16] (BF16).
  // keep = true keeps the activations for backward().
  int forward(const __nv_bfloat16* x, int B, float* y, bool keep, cudaStream_t st);
  // Gradients of the loss w.r.t. all weights and biases, given dL/dy (FP32,
  // same layout as y) for the batch of the last forward(keep = true).
  int backward(const float* dy, int B, cudaStream_t st);
  // One Adam step on the FP32 master weights; refreshes the BF16 copies.
  void adam(float lr, float beta1, float beta2, float eps, float weight_decay, cudaStream_t st);
  // Copy weights/biases (FP32) out or in, layer by layer (tests).
  int get_weights(int layer, float* w, float* b) const;
  int set_weights(int layer, const float* w, const float* b);
  int get_grads(int layer, float* gw, float* gb) const;
  // 76 (and err) when a tensor-core convolution's bounded wait ran out since the last call
  int take_error();

  std::string err;

 private:
  float* w32_[NET_LAYERS] = {};
  float* b32_[NET_LAYERS] = {};
  __nv_bfloat16* w16_[NET_LAYERS] = {};
  float* wt_[NET_LAYERS] = {};  // FP32 W[tap][cout][cin] for the input-gradient kernel
  __nv_bfloat16* wtc_[NET_LAYERS] = {};  // UMMA B-operand layout for k_net_conv_tc (its layers only)
  int* d_err_ = nullptr;                 // wait-ran-out flag of k_net_conv_tc
  float* gw_[NET_LAYERS] = {};
  float* gb_[NET_LAYERS] = {};
  float* mw_[NET_LAYERS] = {};
  float* vw_[NET_LAYERS] = {};
  float* mb_[NET_LAYERS] = {};
  float* vb_[NET_LAYERS] = {};
  long long step_ = 0;
  int cap_ = 0;  // batch capacity of the workspace
  __nv_bfloat16* act_[NET_ACTS] = {};
  float* dact_[NET_ACTS] = {};
  const __nv_bfloat16* x_ = nullptr;
  int ensure(int B);
  void refresh(int layer, cudaStream_t st);
  int alloc_params();
};

// Subdomain patches for the network and its training targets, from a set-up solver.
struct SubInfo;
// feats[s][4096][16] (BF16): log-permeability channels minus the patch mean /4,
// a Dirichlet-face indicator and an inside-the-subdomain indicator.
void launch_net_features(const Grid& g, const SubInfo* subs, int nsub, const double* kx, const double* ky,
                         const double* kz, int dirichlet_mask, __nv_bfloat16* feats, cudaStream_t st);
// Training targets of every subdomain: V[s][4096][k] (the local eigenvectors
// from a finished set-up, zero outside the subdomain) and Mw[s][4096] (the
// diagonal of the eigenproblem's mass matrix, zero outside), so that
// V_j^T diag(Mw) V_j = 1.
struct NetTargetArgs {
  Grid g;
  const SubInfo* subs;
  int nsub, k, kmax, phi_f32, eg_op, dirichlet_mask;
  const void* phi;
  const double *kx, *ky, *kz, *tx, *ty, *tz, *db;
  double Hx, Hy, Hz, meas;
  float* V;
  float* Mw;
};
void launch_net_targets(const NetTargetArgs& a, cudaStream_t st);
// list[0 .. *count-1] = subdomains with status 1 (eigensolve hit its iteration limit).
void launch_failed_list(const int* status, int nsub, int* list, int* count, cudaStream_t st);
// Subspace loss per sample: with G = Y^T M Y, H = Y^T M V (k x k) and C = G^-1 H,
// loss_b = ||V - Y C||_M^2 / k and dy = -2 M (V - Y C) C^T / (B k).
void launch_net_loss(const float* y, const float* V, const float* Mw, int B, int k, float* loss, float* dy,
                     cudaStream_t st);

}  // namespace pmf
