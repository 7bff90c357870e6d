// Learned dispatcher: per-cell features, a small perceptron trained on the
// device from the counter's own per-cell timings, and the inference kernel
// that turns a model into dispatch tables on the device.
//
// A dispatch cell is (class of u's list, bucket |A'|, bucket |B|); a table
// maps every cell to a strategy (MERGE, HASH, SEARCH, SPLIT or HEAD).  All
// give identical counts,
// so the model decides only speed.  The model predicts, per strategy, the
// log2 of the SM cycles an arc of the cell costs, and a cell's table entry
// is the strategy of least predicted cost.  Training regresses the timing
// recorder's measured log2 cycles per arc (weighted squared error, L2 weight
// decay).  Log cost is close to linear in the log-bucketed lengths, which a
// ReLU network extends linearly beyond the cells it was trained on: that is
// what lets a model trained on small graphs place the HASH / SEARCH boundary
// for the long lists of a power-law graph it has not seen.
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

// Parameter offsets (layout W1[hidden][in], b1[hidden], W2[out][hidden], b2[out];
// outputs MERGE, HASH, SEARCH, SPLIT, HEAD).
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

// Outputs z (predicted log2 cycles per arc, one per strategy) of features f;
// h receives the hidden activations.
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

// A learned cell overrides the fixed table only where the model predicts the
// override at least this much cheaper (log2 of 1.05): the fixed thresholds
// stay the fallback wherever the model is unsure or extrapolating.
constexpr float kOverrideMargin = 0.0704f;

// One thread per cell: the strategy of least predicted cost, if the cell is
// in the model's support and that strategy beats the fixed table's choice by
// the margin, else the fixed choice.  The giant
// class stages no hash, so it never takes HASH or SPLIT (its fixed HASH
// cells run MERGE, and are compared as such).  HEAD is open only to the
// cells where the fixed table already holds it: the recorder times a HEAD
// arc's probes but not its share of the head side's sort and staging, so
// its costs are too low for the model to add HEAD cells; it may move a HEAD
// cell to a tail-side strategy.
__global__ void k_mlp_tables(const float* __restrict__ params, const uint8_t* __restrict__ fixed,
                             const uint8_t* __restrict__ support, uint8_t* __restrict__ tables) {
  __shared__ float p[kMlpParams];
  for (int i = threadIdx.x; i < kMlpParams; i += blockDim.x) p[i] = params[i];
  __syncthreads();
  const uint32_t cell = blockIdx.x * blockDim.x + threadIdx.x;
  if (cell >= kTableBytes) return;
  float f[kMlpIn], h[kMlpHidden], z[kMlpOut];
  cell_features(cell, f);
  mlp_forward(p, f, h, z);
  const bool giant = (cell >> 8) == kTableGiant;
  const bool head_ok = fixed[cell] == STC_STRATEGY_HEAD;
  auto staged_only = [](int o) { return o == STC_STRATEGY_HASH - 1 || o == STC_STRATEGY_SPLIT - 1; };
  int best = 0;
  for (int o = 1; o < kMlpOut; o++) {
    if (giant && staged_only(o)) continue;
    if (!head_ok && o == STC_STRATEGY_HEAD - 1) continue;
    if (z[o] < z[best]) best = o;
  }
  int fx = fixed[cell] - 1;
  if (giant && staged_only(fx)) fx = STC_STRATEGY_MERGE - 1;
  const bool trusted = support == nullptr || support[cell] != 0;
  tables[cell] = trusted && z[best] + kOverrideMargin < z[fx] ? (uint8_t)(best + 1) : fixed[cell];
}

// Adds v, summed over the warp, to the warp's gradient row (lane 0 owns it;
// a fixed order, so training is deterministic).
__device__ __forceinline__ void grad_add(float* row, int idx, float v, unsigned lane) {
  v = warp_sum(v);
  if (lane == 0) row[idx] += v;
}

// Full-batch Adam in one CTA.  Each warp takes 32 samples at a time (one per
// lane) and reduces their gradient contributions with shuffles into its own
// row of `gpart`; the rows are summed in warp order for the update.  The
// objective is sum_i w_i sum_o [T_io available] (z_io - T_io)^2 / sum_i w_i
// plus wd / 2 times the squared weights (the reported loss is the first term
// alone); targets are centred on their mean `mu` during training and `mu` is
// folded into the output biases at the end.
__global__ void __launch_bounds__(kTrainThreads)
    k_mlp_train(const float* __restrict__ X, const float* __restrict__ T,
                const float* __restrict__ w, uint32_t S, uint32_t epochs, float lr, float wd,
                uint64_t seed, float* __restrict__ params_out, float* __restrict__ loss_out) {
  __shared__ float p[kMlpParams], m1[kMlpParams], m2[kMlpParams];
  __shared__ float gpart[kTrainWarps][kMlpParams];
  __shared__ float red[3][kTrainWarps];
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
  // Total weight, and the mean of the available targets.
  float ws = 0.f, ts = 0.f, tn = 0.f;
  for (uint32_t i = threadIdx.x; i < S; i += kTrainThreads) {
    ws += w[i];
    for (int o = 0; o < kMlpOut; o++) {
      const float t = T[(size_t)i * kMlpOut + o];
      if (!isnan(t)) {
        ts += t;
        tn += 1.f;
      }
    }
  }
  ws = warp_sum(ws);
  ts = warp_sum(ts);
  tn = warp_sum(tn);
  if (lane == 0) {
    red[0][warp] = ws;
    red[1][warp] = ts;
    red[2][warp] = tn;
  }
  __syncthreads();
  float wsum = 0.f, tsum = 0.f, tcnt = 0.f;
  for (int k = 0; k < kTrainWarps; k++) {
    wsum += red[0][k];
    tsum += red[1][k];
    tcnt += red[2][k];
  }
  const float inv_w = wsum > 0.f ? 1.f / wsum : 0.f;
  const float mu = tcnt > 0.f ? tsum / tcnt : 0.f;
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
      float f[kMlpIn], h[kMlpHidden], z[kMlpOut], dz[kMlpOut];
#pragma unroll
      for (int k = 0; k < kMlpIn; k++) f[k] = valid ? X[(size_t)i * kMlpIn + k] : 0.f;
      const float wi = valid ? w[i] * inv_w : 0.f;
      mlp_forward(p, f, h, z);
#pragma unroll
      for (int o = 0; o < kMlpOut; o++) {
        const float t = valid ? T[(size_t)i * kMlpOut + o] : NAN;
        const float e = isnan(t) ? 0.f : z[o] - (t - mu);
        loss += wi * e * e;
        dz[o] = 2.f * wi * e;
      }
      if (last) continue;
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
      if (lane == 0) red[0][warp] = loss;
      __syncthreads();
      if (threadIdx.x == 0) {
        float t = 0.f;
        for (int k = 0; k < kTrainWarps; k++) t += red[0][k];
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
      const bool weight = i < kOffB1 || (i >= kOffW2 && i < kOffB2);
      if (weight) g += wd * p[i];
      m1[i] = kB1 * m1[i] + (1.f - kB1) * g;
      m2[i] = kB2 * m2[i] + (1.f - kB2) * g * g;
      const float mh = m1[i] / (1.f - b1t), vh = m2[i] / (1.f - b2t);
      p[i] -= lr * mh / (sqrtf(vh) + kEps);
    }
    __syncthreads();
  }
  __syncthreads();
  for (int i = threadIdx.x; i < kMlpParams; i += kTrainThreads)
    params_out[i] = i >= kOffB2 ? p[i] + mu : p[i];
}

}  // namespace

void dispatch_features(float* out) {
  for (uint32_t cell = 0; cell < kTableBytes; cell++) cell_features(cell, out + (size_t)cell * kMlpIn);
}

void load_dispatch_model(stc_ctx* c, const float* params, const uint8_t* support) {
  if (!params) {
    c->model_loaded = false;
    return;
  }
  for (int i = 0; i < kMlpParams; i++)
    if (!std::isfinite(params[i])) fail(STC_ERR_INVALID_ARGUMENT, "model parameter is not finite");
  CountConfig fixed_cfg;
  fixed_cfg.dispatch = STC_DISPATCH_FIXED;
  const uint8_t* d_fixed = dispatch_tables(c, fixed_cfg);
  // Parameters, then the support mask, in one staging buffer.
  float* d_params = buffer<float>(c, B_DISPATCH_TRAIN, kMlpParams + kTableBytes / sizeof(float));
  uint8_t* d_support = reinterpret_cast<uint8_t*>(d_params + kMlpParams);
  uint8_t* d_tables = buffer<uint8_t>(c, B_DISPATCH, kTableBytes);
  STC_CUDA(cudaMemcpyAsync(d_params, params, kMlpParams * sizeof(float), cudaMemcpyHostToDevice,
                           c->stream));
  if (support)
    STC_CUDA(cudaMemcpyAsync(d_support, support, kTableBytes, cudaMemcpyHostToDevice, c->stream));
  k_mlp_tables<<<(unsigned)(kTableBytes / 256), 256, 0, c->stream>>>(
      d_params, d_fixed, support ? d_support : nullptr, d_tables);
  STC_CUDA(cudaGetLastError());
  uint8_t h[kTableBytes];
  STC_CUDA(cudaMemcpyAsync(h, d_tables, kTableBytes, cudaMemcpyDeviceToHost, c->stream));
  STC_CUDA(cudaStreamSynchronize(c->stream));
  c->model_loaded = true;
  // Counts with these tables build the sign-split heads only if some cell
  // picks SPLIT.
  c->learned_uses_split = false;
  c->learned_uses_head = false;
  for (size_t i = 0; i < kTableBytes; i++) {
    c->learned_uses_split |= h[i] == STC_STRATEGY_SPLIT;
    c->learned_uses_head |= h[i] == STC_STRATEGY_HEAD;
  }
}

void train_dispatcher(stc_ctx* c, const float* features, const float* targets,
                      const float* weights, uint32_t samples, uint32_t epochs, float lr, float wd,
                      uint64_t seed, float* params, float* loss) {
  if (!features || !targets || !weights || !params)
    fail(STC_ERR_INVALID_ARGUMENT, "null training array");
  if (samples == 0 || samples > kMaxTrainSamples)
    fail(STC_ERR_INVALID_ARGUMENT, "samples must be in [1, " + std::to_string(kMaxTrainSamples) + "]");
  if (epochs == 0 || epochs > 1000000) fail(STC_ERR_INVALID_ARGUMENT, "epochs must be in [1, 1e6]");
  if (!(lr > 0.f) || !std::isfinite(lr)) fail(STC_ERR_INVALID_ARGUMENT, "learning rate must be > 0");
  if (!(wd >= 0.f) || !std::isfinite(wd)) fail(STC_ERR_INVALID_ARGUMENT, "weight decay must be >= 0");
  double wsum = 0.0;
  uint64_t available = 0;
  for (uint32_t i = 0; i < samples; i++) {
    if (!(weights[i] >= 0.f) || !std::isfinite(weights[i]))
      fail(STC_ERR_INVALID_ARGUMENT, "weights must be finite and >= 0");
    for (int k = 0; k < kMlpIn; k++)
      if (!std::isfinite(features[(size_t)i * kMlpIn + k]))
        fail(STC_ERR_INVALID_ARGUMENT, "feature is not finite");
    for (int o = 0; o < kMlpOut; o++) {
      const float t = targets[(size_t)i * kMlpOut + o];
      if (std::isnan(t)) continue;
      if (!std::isfinite(t)) fail(STC_ERR_INVALID_ARGUMENT, "target is infinite");
      available++;
    }
    wsum += weights[i];
  }
  if (!(wsum > 0.0)) fail(STC_ERR_INVALID_ARGUMENT, "total weight must be > 0");
  if (!available) fail(STC_ERR_INVALID_ARGUMENT, "no available target");
  // Device layout: X[samples][kMlpIn], T[samples][kMlpOut], w[samples], params, loss.
  const size_t nX = (size_t)samples * kMlpIn, nT = (size_t)samples * kMlpOut;
  float* base = buffer<float>(c, B_DISPATCH_TRAIN, nX + nT + samples + kMlpParams + 1);
  float* dX = base;
  float* dT = dX + nX;
  float* dw = dT + nT;
  float* dp = dw + samples;
  float* dl = dp + kMlpParams;
  cudaStream_t st = c->stream;
  STC_CUDA(cudaMemcpyAsync(dX, features, nX * sizeof(float), cudaMemcpyHostToDevice, st));
  STC_CUDA(cudaMemcpyAsync(dT, targets, nT * sizeof(float), cudaMemcpyHostToDevice, st));
  STC_CUDA(cudaMemcpyAsync(dw, weights, samples * sizeof(float), cudaMemcpyHostToDevice, st));
  k_mlp_train<<<1, kTrainThreads, 0, st>>>(dX, dT, dw, samples, epochs, lr, wd, seed, dp, dl);
  STC_CUDA(cudaGetLastError());
  float h_loss = 0.f;
  STC_CUDA(cudaMemcpyAsync(params, dp, kMlpParams * sizeof(float), cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaMemcpyAsync(&h_loss, dl, sizeof(float), cudaMemcpyDeviceToHost, st));
  STC_CUDA(cudaStreamSynchronize(st));
  if (loss) *loss = h_loss;
}

}  // namespace stc
