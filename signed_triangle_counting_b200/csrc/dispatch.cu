// Learned dispatcher: per-cell features, a small perceptron trained on the
// device from the counter's own per-cell timings, and the inference kernel
// that turns a model into dispatch tables on the device.
//
// A dispatch cell is (class of u's list, bucket |A'|, bucket |B|); a table
// maps every cell to MERGE, HASH or SEARCH.  All three give identical counts,
// so the model decides only speed.  It is trained by weighted softmax
// cross-entropy: the label of a cell is its fastest strategy under the timing
// recorder, its weight the cycles at stake (arcs x (slowest - fastest)
// cycles per arc), so cells that matter for the run time dominate the fit.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <string>
#include <vector>

#include "internal.h"
#include "stc_device.cuh"
#include "stc_gen.h"

namespace stc {

namespace {

constexpr int kTrainThreads = 256;
constexpr int kTrainWarps = kTrainThreads / 32;
constexpr uint32_t kMaxTrainSamples = 4096;
constexpr uint64_t kStreamMlpInit = 11;  // generator stream of the initial weights

// Parameter offsets (layout W1[hidden][in], b1[hidden], W2[out][hidden], b2[out]).
constexpr int kOffB1 = kMlpHidden * kMlpIn;
constexpr int kOffW2 = kOffB1 + kMlpHidden;
constexpr int kOffB2 = kOffW2 + kMlpOut * kMlpHidden;

// Bit width of a typical |N+(u)| of each class: warp lists hold up to 128
// entries (widths up to 8), block lists up to 1024, large up to 4096, giant
// lists more.
__host__ __device__ inline float class_log_degree(int cls) {
  return cls == kTableWarp ? 6.f : cls == kTableBlock ? 9.5f : cls == kTableLarge ? 12.f : 14.f;
}

__host__ __device__ inline void cell_features(uint32_t cell, float* f) {
  const int cls = (int)(cell >> 8);
  const float a = (float)((cell >> 4) & 15), b = (float)(cell & 15);
  const float lu = fmaxf(class_log_degree(cls), a);  // |A'| < |N+(u)|
  f[0] = a / 16.f;
  f[1] = b / 16.f;
  f[2] = (b - a) / 16.f;
  f[3] = lu / 16.f;
  f[4] = (lu - b) / 16.f;
  f[5] = cls == kTableGiant ? 0.f : 1.f;
}

// Logits z of features f; h receives the hidden activations.
__device__ __forceinline__ void mlp_forward(const float* p, const float* f, float* h, float* z) {
#pragma unroll
  for (int j = 0; j < kMlpHidden; j++) {
    float s = p[kOffB1 + j];
#pragma unroll
    for (int k = 0; k < kMlpIn; k++) s = fmaf(p[j * kMlpIn + k], f[k], s);
    h[j] = fmaxf(s, 0.f);
  }
#pragma unroll
  for (int o = 0; o < kMlpOut; o++) {
    float s = p[kOffB2 + o];
#pragma unroll
    for (int j = 0; j < kMlpHidden; j++) s = fmaf(p[kOffW2 + o * kMlpHidden + j], h[j], s);
    z[o] = s;
  }
}

// One thread per cell: the strategy of the largest logit (HASH excluded for
// the giant class, which stages no hash).
__global__ void k_mlp_tables(const float* __restrict__ params, uint8_t* __restrict__ tables) {
  __shared__ float p[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= kTableBytes) return;
  float f[kMlpIn], h[kMlpHidden], z[kMlpOut];
  cell_features(cell, f);
  mlp_forward(p, f, h, z);
  const bool giant = (cell >> 8) == kTableGiant;
  int best = 0;
  for (int o = 1; o < kMlpOut; o++) {
    if (giant && o == STC_STRATEGY_HASH - 1) continue;
    if (z[o] > z[best]) best = o;
  }
  tables[cell] = (uint8_t)(best + 1);
}

// Adds v, summed over the warp, to the warp's gradient row (lane 0 owns it;
// a fixed order, so training is deterministic).
__device__ __forceinline__ void grad_add(float* row, int idx, float v, unsigned lane) {
  v = warp_sum(v);
  if (lane == 0) row[idx] += v;
}

// Full-batch Adam in one CTA.  Each warp takes 32 samples at a time (one per
// lane) and reduces their gradient contributions with shuffles into its own
// row of `gpart`; the rows are summed in warp order for the update.
__global__ void __launch_bounds__(kTrainThreads)
    k_mlp_train(const float* __restrict__ X, const int32_t* __restrict__ y,
                const float* __restrict__ w, uint32_t S, uint32_t epochs, float lr, uint64_t seed,
                float* __restrict__ params_out, float* __restrict__ loss_out) {
  __shared__ float p[kMlpParams], m1[kMlpParams], m2[kMlpParams];
  __shared__ float gpart[kTrainWarps][kMlpParams];
  __shared__ float red[kTrainWarps];
  const unsigned lane = lane_id(), warp = threadIdx.x >> 5;
  for (int i = threadIdx.x; i < kMlpParams; i += kTrainThreads) {
    // Uniform in +-1/sqrt(fan_in) for weights, zero biases.
    const float u = (float)(stcgen::draw(seed, kStreamMlpInit, (uint64_t)i) >> 40) * 0x1p-24f;
    float v = 0.f;
    if (i < kOffB1) v = (2.f * u - 1.f) * rsqrtf((float)kMlpIn);
    else if (i >= kOffW2 && i < kOffB2) v = (2.f * u - 1.f) * rsqrtf((float)kMlpHidden);
    p[i] = v;
    m1[i] = 0.f;
    m2[i] = 0.f;
  }
  for (int i = threadIdx.x; i < kTrainWarps * kMlpParams; i += kTrainThreads) (&gpart[0][0])[i] = 0.f;
  // Total weight, for the loss normalisation.
  float ws = 0.f;
  for (uint32_t i = threadIdx.x; i < S; i += kTrainThreads) ws += w[i];
  ws = warp_sum(ws);
  if (lane == 0) red[warp] = ws;
  __syncthreads();
  float wsum = 0.f;
  for (int k = 0; k < kTrainWarps; k++) wsum += red[k];
  const float inv_w = wsum > 0.f ? 1.f / wsum : 0.f;
  __syncthreads();

  constexpr float kB1 = 0.9f, kB2 = 0.999f, kEps = 1e-8f;
  float b1t = 1.f, b2t = 1.f;
  float* row = gpart[warp];
  for (uint32_t ep = 0; ep <= epochs; ep++) {
    const bool last = ep == epochs;  // the last pass only measures the loss
    float loss = 0.f;
    for (uint32_t base = warp * 32; base < S; base += kTrainThreads) {
      const uint32_t i = base + lane;
      const bool valid = i < S;
      float f[kMlpIn], h[kMlpHidden], z[kMlpOut];
#pragma unroll
      for (int k = 0; k < kMlpIn; k++) f[k] = valid ? X[(size_t)i * kMlpIn + k] : 0.f;
      const int label = valid ? y[i] : 0;
      const float wi = valid ? w[i] * inv_w : 0.f;
      mlp_forward(p, f, h, z);
      const float zmax = fmaxf(z[0], fmaxf(z[1], z[2]));
      float e[kMlpOut], es = 0.f;
#pragma unroll
      for (int o = 0; o < kMlpOut; o++) {
        e[o] = expf(z[o] - zmax);
        es += e[o];
      }
      const float zl = label == 0 ? z[0] : label == 1 ? z[1] : z[2];
      loss += wi * (logf(es) - (zl - zmax));
      if (last) continue;
      float dz[kMlpOut];
#pragma unroll
      for (int o = 0; o < kMlpOut; o++) dz[o] = wi * (e[o] / es - (o == label ? 1.f : 0.f));
      float dh[kMlpHidden];
#pragma unroll
      for (int j = 0; j < kMlpHidden; j++) {
        float s = 0.f;
#pragma unroll
        for (int o = 0; o < kMlpOut; o++) s = fmaf(p[kOffW2 + o * kMlpHidden + j], dz[o], s);
        dh[j] = h[j] > 0.f ? s : 0.f;
      }
#pragma unroll
      for (int j = 0; j < kMlpHidden; j++) {
#pragma unroll
        for (int k = 0; k < kMlpIn; k++) grad_add(row, j * kMlpIn + k, dh[j] * f[k], lane);
        grad_add(row, kOffB1 + j, dh[j], lane);
      }
#pragma unroll
      for (int o = 0; o < kMlpOut; o++) {
#pragma unroll
        for (int j = 0; j < kMlpHidden; j++) grad_add(row, kOffW2 + o * kMlpHidden + j, dz[o] * h[j], lane);
        grad_add(row, kOffB2 + o, dz[o], lane);
      }
    }
    if (last) {
      loss = warp_sum(loss);
      if (lane == 0) red[warp] = loss;
      __syncthreads();
      if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < kTrainWarps; k++) t += red[k];
        if (loss_out) *loss_out = t;
      }
      break;
    }
    __syncthreads();
    b1t *= kB1;
    b2t *= kB2;
    for (int i = threadIdx.x; i < kMlpParams; i += kTrainThreads) {
      float g = 0.f;
      for (int k = 0; k < kTrainWarps; k++) {
        g += gpart[k][i];
        gpart[k][i] = 0.f;
      }
      m1[i] = kB1 * m1[i] + (1.f - kB1) * g;
      m2[i] = kB2 * m2[i] + (1.f - kB2) * g * g;
      const float mh = m1[i] / (1.f - b1t), vh = m2[i] / (1.f - b2t);
      p[i] -= lr * mh / (sqrtf(vh) + kEps);
    }
    __syncthreads();
  }
  for (int i = threadIdx.x; i < kMlpParams; i += kTrainThreads) params_out[i] = p[i];
}

}  // namespace

void dispatch_features(float* out) {
  for (uint32_t cell = 0; cell < kTableBytes; cell++) cell_features(cell, out + (size_t)cell * kMlpIn);
}

void load_dispatch_model(stc_ctx* c, const float* params) {
  if (!params) {
    c->model_loaded = false;
    return;
  }
  for (int i = 0; i < kMlpParams; i++)
    if (!std::isfinite(params[i])) fail(STC_ERR_INVALID_ARGUMENT, "model parameter is not finite");
  float* d_params = buffer<float>(c, B_DISPATCH_TRAIN, kMlpParams);
  uint8_t* d_tables = buffer<uint8_t>(c, B_DISPATCH, kTableBytes);
  STC_CUDA(cudaMemcpyAsync(d_params, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice,
                           c->stream));
  k_mlp_tables<<<(unsigned)(kTableBytes / 256), 256, 0, c->stream>>>(d_params, d_tables);
  STC_CUDA(cudaGetLastError());
  STC_CUDA(cudaStreamSynchronize(c->stream));
  c->model_loaded = true;
}

void train_dispatcher(stc_ctx* c, const float* features, const int32_t* labels,
                      const float* weights, uint32_t samples, uint32_t epochs, float lr,
                      uint64_t seed, float* params, float* loss) {
  if (!features || !labels || !weights || !params)
    fail(STC_ERR_INVALID_ARGUMENT, "null training array");
  if (samples == 0 || samples > kMaxTrainSamples)
    fail(STC_ERR_INVALID_ARGUMENT, "samples must be in [1, " + std::to_string(kMaxTrainSamples) + "]");
  if (epochs == 0 || epochs > 1000000) fail(STC_ERR_INVALID_ARGUMENT, "epochs must be in [1, 1e6]");
  if (!(lr > 0.f) || !std::isfinite(lr)) fail(STC_ERR_INVALID_ARGUMENT, "learning rate must be > 0");
  double wsum = 0.0;
  for (uint32_t i = 0; i < samples; i++) {
    if (labels[i] < 0 || labels[i] >= kMlpOut) fail(STC_ERR_INVALID_ARGUMENT, "label out of range");
    if (!(weights[i] >= 0.f) || !std::isfinite(weights[i]))
      fail(STC_ERR_INVALID_ARGUMENT, "weights must be finite and >= 0");
    for (int k = 0; k < kMlpIn; k++)
      if (!std::isfinite(features[(size_t)i * kMlpIn + k]))
        fail(STC_ERR_INVALID_ARGUMENT, "feature is not finite");
    wsum += weights[i];
  }
  if (!(wsum > 0.0)) fail(STC_ERR_INVALID_ARGUMENT, "total weight must be > 0");
  // Device layout: X[samples][kMlpIn], w[samples], y[samples], params, loss.
  const size_t nX = (size_t)samples * kMlpIn;
  float* base = buffer<float>(c, B_DISPATCH_TRAIN, nX + 2 * (size_t)samples + kMlpParams + 1);
  float* dX = base;
  float* dw = dX + nX;
  int32_t* dy = reinterpret_cast<int32_t*>(dw + samples);
  float* dp = reinterpret_cast<float*>(dy + samples);
  float* dl = dp + kMlpParams;
  cudaStream_t st = c->stream;
  STC_CUDA(cudaMemcpyAsync(dX, features, nX * sizeof(float), cudaMemcpyHostToDevice, st));
  STC_CUDA(cudaMemcpyAsync(dw, weights, samples * sizeof(float), cudaMemcpyHostToDevice, st));
  STC_CUDA(cudaMemcpyAsync(dy, labels, samples * sizeof(int32_t), cudaMemcpyHostToDevice, st));
  k_mlp_train<<<1, kTrainThreads, 0, st>>>(dX, dy, dw, samples, epochs, lr, seed, dp, dl);
  STC_CUDA(cudaGetLastError());
  float h_loss = 0.f;
  STC_CUDA(cudaMemcpyAsync(params, dp, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaMemcpyAsync(&h_loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  if (loss) *loss = h_loss;
  // The training buffer doubles as the model's parameter buffer: a loaded
  // model's tables are already on the device and stay valid.
}

}  // namespace stc
