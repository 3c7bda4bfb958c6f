// Learned direction/strategy predictor: an 8 -> 32 -> 32 -> 3 MLP (ReLU,
// softmax cross-entropy, 1,443 FP32 parameters) with hand-written forward,
// backward and SGD kernels, and the per-device weight slot read by the
// persistent traversal kernel.
//
// No counterpart in the reference, whose switch is the fixed alpha/beta
// heuristic at bfs_adaptiveFQ_wb_async.cuh:946-1078; that heuristic stays as
// the fallback when no weights are installed.
//
// Packed parameter layout (floats), shared with the traversal kernel:
//   [feature mean 8][feature std 8][W1 32x8][b1 32][W2 32x32][b2 32][W3 3x32][b3 3]
// The normalisation constants are not trained; the 1,443 trainable
// parameters start at offset 16.
#include <math.h>
#include <string.h>

#include <mutex>
#include <vector>

#include "common.cuh"
#include "internal.hpp"

namespace xbfs {

constexpr int kIn = 8, kH = 32, kOut = 3;
constexpr int kOffW1 = 16;
constexpr int kOffB1 = kOffW1 + kH * kIn;
constexpr int kOffW2 = kOffB1 + kH;
constexpr int kOffB2 = kOffW2 + kH * kH;
constexpr int kOffW3 = kOffB2 + kH;
constexpr int kOffB3 = kOffW3 + kOut * kH;
constexpr int kPacked = kOffB3 + kOut;  // 16 + 1443
constexpr int kTrainable = kPacked - 16;
constexpr int kMlpBound = 8;  // per-feature sensitivity bound stored after the installed weights

static std::mutex g_mlp_mu;
static float* g_mlp_dev[64] = {nullptr};

const float* mlp_device_weights(int device) {
  if (device < 0 || device >= 64) return nullptr;
  std::lock_guard<std::mutex> lk(g_mlp_mu);
  return g_mlp_dev[device];
}

// ---------------------------------------------------------------------------
// Training kernels. One CTA of 32 x 32 threads processes a mini-batch: each
// warp owns samples (strided), lanes own hidden units. Gradients are
// accumulated per CTA in shared memory and written to a gradient buffer; SGD
// is a separate elementwise kernel. Everything is FP32.
// ---------------------------------------------------------------------------
struct MlpFwd {
  float x[kIn];
  float h1[kH];
  float h2[kH];
  float o[kOut];
};

__device__ void mlp_forward_warp(const float* w, const float* feat, float* h1, float* h2, float* out, int lane) {
  const float* mean = w;
  const float* sd = w + 8;
  float x[kIn];
#pragma unroll
  for (int i = 0; i < kIn; ++i) x[i] = (feat[i] - mean[i]) / sd[i];
  float a = w[kOffB1 + lane];
#pragma unroll
  for (int i = 0; i < kIn; ++i) a = fmaf(w[kOffW1 + lane * kIn + i], x[i], a);
  a = fmaxf(a, 0.f);
  h1[lane] = a;
  __syncwarp();
  float b = w[kOffB2 + lane];
  for (int i = 0; i < kH; ++i) b = fmaf(w[kOffW2 + lane * kH + i], h1[i], b);
  b = fmaxf(b, 0.f);
  h2[lane] = b;
  __syncwarp();
  for (int k = 0; k < kOut; ++k) {
    float t = warp_sum(w[kOffW3 + k * kH + lane] * b);
    if (lane == 0) out[k] = t + w[kOffB3 + k];
  }
  __syncwarp();
}

// logits for n samples (inference check against the CPU)
__global__ void k_mlp_logits(const float* w, const float* feats, int n, float* logits) {
  __shared__ float h1[32][kH], h2[32][kH], o[32][4];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int s = blockIdx.x * 32 + wid; s < n; s += gridDim.x * 32) {
    mlp_forward_warp(w, feats + (size_t)s * kIn, h1[wid], h2[wid], o[wid], lane);
    if (lane < kOut) logits[(size_t)s * kOut + lane] = o[wid][lane];
    __syncwarp();
  }
}

// Forward + backward of softmax cross-entropy over n samples; grad (size
// kTrainable, zeroed by the caller) receives the mean gradient, loss[0] the
// mean loss.
__global__ void k_mlp_grad(const float* w, const float* feats, const int* labels, int n, float* grad,
                           float* loss) {
  __shared__ float g[kTrainable];
  __shared__ float h1[32][kH], h2[32][kH], o[32][4], d2[32][kH];
  __shared__ float sloss;
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kTrainable; i += blockDim.x) g[i] = 0.f;
  if (threadIdx.x == 0) sloss = 0.f;
  __syncthreads();
  const float inv_n = 1.f / (float)n;
  for (int s = blockIdx.x * 32 + wid; s < n; s += gridDim.x * 32) {
    const float* f = feats + (size_t)s * kIn;
    mlp_forward_warp(w, f, h1[wid], h2[wid], o[wid], lane);
    // softmax
    const float m = fmaxf(o[wid][0], fmaxf(o[wid][1], o[wid][2]));
    const float e0 = expf(o[wid][0] - m), e1 = expf(o[wid][1] - m), e2 = expf(o[wid][2] - m);
    const float z = e0 + e1 + e2;
    const float pr[3] = {e0 / z, e1 / z, e2 / z};
    const int y = labels[s];
    if (lane == 0) atomicAdd(&sloss, -logf(fmaxf(pr[y], 1e-30f)) * inv_n);
    float dout[3];
    for (int k = 0; k < 3; ++k) dout[k] = (pr[k] - (k == y ? 1.f : 0.f)) * inv_n;
    // layer 3: dW3[k][lane] = dout[k] * h2[lane]; db3[k] = dout[k]
    const float hb = h2[wid][lane];
    for (int k = 0; k < 3; ++k) atomicAdd(&g[kOffW3 - 16 + k * kH + lane], dout[k] * hb);
    if (lane < 3) atomicAdd(&g[kOffB3 - 16 + lane], dout[lane]);
    // dh2[lane] = sum_k W3[k][lane] dout[k], through ReLU
    float dh2 = 0.f;
    for (int k = 0; k < 3; ++k) dh2 = fmaf(w[kOffW3 + k * kH + lane], dout[k], dh2);
    if (hb <= 0.f) dh2 = 0.f;
    d2[wid][lane] = dh2;
    __syncwarp();
    // layer 2: dW2[lane][i] = dh2[lane] * h1[i]; db2[lane] = dh2[lane]
    for (int i = 0; i < kH; ++i) atomicAdd(&g[kOffW2 - 16 + lane * kH + i], dh2 * h1[wid][i]);
    atomicAdd(&g[kOffB2 - 16 + lane], dh2);
    // dh1[lane] = sum_j W2[j][lane] dh2[j], through ReLU
    float dh1 = 0.f;
    for (int j = 0; j < kH; ++j) dh1 = fmaf(w[kOffW2 + j * kH + lane], d2[wid][j], dh1);
    if (h1[wid][lane] <= 0.f) dh1 = 0.f;
    // layer 1: dW1[lane][i] = dh1 * x[i]
    for (int i = 0; i < kIn; ++i) {
      const float xi = (f[i] - w[i]) / w[8 + i];
      atomicAdd(&g[kOffW1 - 16 + lane * kIn + i], dh1 * xi);
    }
    atomicAdd(&g[kOffB1 - 16 + lane], dh1);
    __syncwarp();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kTrainable; i += blockDim.x) atomicAdd(&grad[i], g[i]);
  if (threadIdx.x == 0) atomicAdd(loss, sloss);
}

__global__ void k_mlp_sgd(float* w, const float* grad, float lr, float momentum, float* vel) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < kTrainable; i += gridDim.x * blockDim.x) {
    float v = momentum * vel[i] + grad[i];
    vel[i] = v;
    w[16 + i] -= lr * v;
  }
}

}  // namespace xbfs

using namespace xbfs;

extern "C" {

int32_t xbfs_mlp_num_params(void) { return kPacked; }

xbfs_status xbfs_mlp_set_weights(int32_t device, const float* packed, int32_t n) {
  if (n != 0 && n != kPacked) return set_error(XBFS_ERR_INVALID_ARG, "expected %d floats, got %d", kPacked, n);
  if (device < 0 || device >= 64) return set_error(XBFS_ERR_INVALID_ARG, "bad device %d", device);
  DeviceGuard dg(device);
  std::lock_guard<std::mutex> lk(g_mlp_mu);
  if (!packed || n == 0) {
    if (g_mlp_dev[device]) cudaFree(g_mlp_dev[device]);
    g_mlp_dev[device] = nullptr;
    return XBFS_OK;
  }
  // The installed copy carries, after the packed weights, a per-feature
  // sensitivity bound of the network (path bound through the ReLU layers):
  //   P[i] = max over class pairs (a, b) of
  //          sum_k |W3[a][k] - W3[b][k]| * sum_j |W2[k][j]| * |W1[j][i]|,
  // so that moving the normalised features by d changes any logit
  // difference by at most sum_i P[i] * |d_i|. The traversal kernel reuses
  // its last decision while that bound stays below the decision's margin,
  // i.e. only where evaluating the network again would give the same class.
  std::vector<float> ext(kPacked + kMlpBound);
  memcpy(ext.data(), packed, kPacked * sizeof(float));
  const float* W1 = packed + kOffW1;
  const float* W2 = packed + kOffW2;
  const float* W3 = packed + kOffW3;
  for (int i = 0; i < kIn; ++i) {
    double h2[kH];  // sensitivity of each second-layer unit to feature i
    for (int k = 0; k < kH; ++k) {
      double t = 0;
      for (int j = 0; j < kH; ++j) t += fabs((double)W2[k * kH + j]) * fabs((double)W1[j * kIn + i]);
      h2[k] = t;
    }
    double worst = 0;
    for (int a = 0; a < kOut; ++a)
      for (int b = a + 1; b < kOut; ++b) {
        double t = 0;
        for (int k = 0; k < kH; ++k) t += fabs((double)W3[a * kH + k] - (double)W3[b * kH + k]) * h2[k];
        worst = t > worst ? t : worst;
      }
    ext[kPacked + i] = (float)(worst * (1.0 + 1e-5));  // rounded up
  }
  if (!g_mlp_dev[device])
    XBFS_CUDA_TRY(cudaMalloc(&g_mlp_dev[device], (kPacked + kMlpBound) * sizeof(float)));
  XBFS_CUDA_TRY(cudaMemcpy(g_mlp_dev[device], ext.data(), (kPacked + kMlpBound) * sizeof(float),
                           cudaMemcpyHostToDevice));
  return XBFS_OK;
}

// Logits of n samples (features n x 8, host) with packed weights (host).
xbfs_status xbfs_mlp_logits(int32_t device, const float* packed, const float* feats, int32_t n, float* logits) {
  if (!packed || !feats || !logits || n < 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(device);
  DevBuf dw, df, dl;
  xbfs_status st;
  if ((st = dw.ensure(kPacked * 4)) || (st = df.ensure((size_t)n * kIn * 4 + 4)) ||
      (st = dl.ensure((size_t)n * kOut * 4 + 4)))
    return st;
  XBFS_CUDA_TRY(cudaMemcpy(dw.p, packed, kPacked * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemcpy(df.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice));
  if (n > 0) k_mlp_logits<<<(n + 31) / 32 < 148 ? (n + 31) / 32 : 148, 1024>>>(dw.as<float>(), df.as<float>(), n, dl.as<float>());
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaMemcpy(logits, dl.p, (size_t)n * kOut * 4, cudaMemcpyDeviceToHost));
  return XBFS_OK;
}

// Mean loss and gradient (kTrainable floats) of softmax cross-entropy.
xbfs_status xbfs_mlp_grad(int32_t device, const float* packed, const float* feats, const int32_t* labels,
                          int32_t n, float* grad, float* loss) {
  if (!packed || !feats || !labels || !grad || !loss || n <= 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(device);
  DevBuf dw, df, dy, dg2, dls;
  xbfs_status st;
  if ((st = dw.ensure(kPacked * 4)) || (st = df.ensure((size_t)n * kIn * 4)) || (st = dy.ensure((size_t)n * 4)) ||
      (st = dg2.ensure(kTrainable * 4)) || (st = dls.ensure(4)))
    return st;
  XBFS_CUDA_TRY(cudaMemcpy(dw.p, packed, kPacked * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemcpy(df.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemcpy(dy.p, labels, (size_t)n * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemset(dg2.p, 0, kTrainable * 4));
  XBFS_CUDA_TRY(cudaMemset(dls.p, 0, 4));
  k_mlp_grad<<<(n + 31) / 32 < 148 ? (n + 31) / 32 : 148, 1024>>>(dw.as<float>(), df.as<float>(), dy.as<int>(), n,
                                                              dg2.as<float>(), dls.as<float>());
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaMemcpy(grad, dg2.p, kTrainable * 4, cudaMemcpyDeviceToHost));
  XBFS_CUDA_TRY(cudaMemcpy(loss, dls.p, 4, cudaMemcpyDeviceToHost));
  return XBFS_OK;
}

// Full-batch training on the device: `epochs` steps of SGD with momentum,
// weights updated in place (host array, kPacked floats). losses (nullable)
// receives the loss of every epoch.
xbfs_status xbfs_mlp_train(int32_t device, float* packed, const float* feats, const int32_t* labels, int32_t n,
                           int32_t epochs, float lr, float momentum, float* losses) {
  if (!packed || !feats || !labels || n <= 0 || epochs < 0) return set_error(XBFS_ERR_INVALID_ARG, "bad arguments");
  DeviceGuard dg(device);
  DevBuf dw, df, dy, dg2, dls, dv;
  xbfs_status st;
  if ((st = dw.ensure(kPacked * 4)) || (st = df.ensure((size_t)n * kIn * 4)) || (st = dy.ensure((size_t)n * 4)) ||
      (st = dg2.ensure(kTrainable * 4)) || (st = dls.ensure((size_t)(epochs + 1) * 4)) || (st = dv.ensure(kTrainable * 4)))
    return st;
  XBFS_CUDA_TRY(cudaMemcpy(dw.p, packed, kPacked * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemcpy(df.p, feats, (size_t)n * kIn * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemcpy(dy.p, labels, (size_t)n * 4, cudaMemcpyHostToDevice));
  XBFS_CUDA_TRY(cudaMemset(dv.p, 0, kTrainable * 4));
  XBFS_CUDA_TRY(cudaMemset(dls.p, 0, (size_t)(epochs + 1) * 4));
  const int grid = (n + 31) / 32 < 148 ? (n + 31) / 32 : 148;
  for (int e = 0; e < epochs; ++e) {
    XBFS_CUDA_TRY(cudaMemsetAsync(dg2.p, 0, kTrainable * 4));
    k_mlp_grad<<<grid, 1024>>>(dw.as<float>(), df.as<float>(), dy.as<int>(), n, dg2.as<float>(), dls.as<float>() + e);
    k_mlp_sgd<<<2, 1024>>>(dw.as<float>(), dg2.as<float>(), lr, momentum, dv.as<float>());
  }
  XBFS_CUDA_TRY(cudaGetLastError());
  XBFS_CUDA_TRY(cudaMemcpy(packed, dw.p, kPacked * 4, cudaMemcpyDeviceToHost));
  if (losses) XBFS_CUDA_TRY(cudaMemcpy(losses, dls.p, (size_t)epochs * 4, cudaMemcpyDeviceToHost));
  return XBFS_OK;
}

}  // extern "C"
