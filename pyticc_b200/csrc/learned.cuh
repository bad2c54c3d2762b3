// Learned sector-width proposer: per-sector features read from W_base, and a small
// MLP (8 -> 32 -> 32 -> 1, tanh) with hand-written forward, gradient and Adam kernels.
//
// The proposer maps local features of one fixed-step sector to log2 of how many aligned
// base sectors may be merged into one LDMD sector.  Features (all from the W_base values
// the propagation already uses; p^2 = W_mid,ii - 2 mu E):
//   0 asinh(max_i -p^2(E_max))          largest local open wavenumber squared
//   1 log10(min_i |p^2(E_max)| + 1e-12)  distance to a turning point, highest energy
//   2 log10(min_i |p^2(E_min)| + 1e-12)  same at the lowest energy
//   3 log10(max |W_end - W_start| / 2h)  first derivative of W (all elements)
//   4 log10(max |W_end - 2 W_mid + W_start| / h^2)   second derivative
//   5 log10(max_{i != j} |W_mid,ij|)     coupling strength
//   6 log10(h)                            base half-step
//   7 log10(max_i |p^2(E_max)| + 1e-12)  most strongly closed channel
// Features are max/min reductions, so they do not depend on the channel order.
#pragma once

#include "ticc_common.cuh"

namespace ticc {

constexpr int kFeat = 8;
constexpr int kHidden = 32;
constexpr int kOffW1 = 0;
constexpr int kOffB1 = kOffW1 + kHidden * kFeat;
constexpr int kOffW2 = kOffB1 + kHidden;
constexpr int kOffB2 = kOffW2 + kHidden * kHidden;
constexpr int kOffW3 = kOffB2 + kHidden;
constexpr int kOffB3 = kOffW3 + kHidden;
constexpr int kParams = kOffB3 + 1;  // 1377
constexpr int kFeatureThreads = 256;
constexpr int kMlpSamples = 128;     // samples (and threads) per gradient block
constexpr int kMlpPad = kHidden + 1;
constexpr size_t kMlpGradSmemBytes = sizeof(float) * (kParams + kMlpSamples * kFeat + 4 * kMlpSamples * kMlpPad + kMlpSamples + kMlpSamples);

__device__ __forceinline__ double block_reduce(double v, bool take_max, double* red) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  for (int o = 16; o > 0; o >>= 1) {
    const double u = __shfl_xor_sync(0xffffffffu, v, o);
    v = take_max ? fmax(v, u) : fmin(v, u);
  }
  __syncthreads();
  if (lane == 0) red[warp] = v;
  __syncthreads();
  if (threadIdx.x == 0) {
    for (int w = 1; w < nw; ++w) v = take_max ? fmax(v, red[w]) : fmin(v, red[w]);
    red[0] = v;
  }
  __syncthreads();
  return red[0];
}

// One CTA per sector.  Rows are visited warp by warp, columns lane by lane (coalesced).
__global__ void __launch_bounds__(kFeatureThreads) step_features_kernel(const double* __restrict__ Ws, long long ws_stride, const double* __restrict__ Wm, long long wm_stride, const double* __restrict__ We, long long we_stride, const double* __restrict__ h, int n, double two_mu_emax, double two_mu_emin, float* __restrict__ out) {
  __shared__ double red[kFeatureThreads / 32];
  const int s = blockIdx.x;
  const double* A = Ws + (long long)s * ws_stride;
  const double* B = Wm + (long long)s * wm_stride;
  const double* C = We + (long long)s * we_stride;
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5, nw = blockDim.x >> 5;
  double d1 = 0.0, d2 = 0.0, off = 0.0;
  for (int i = warp; i < n; i += nw) {
    const long long row = (long long)i * n;
    for (int j = lane; j < n; j += 32) {
      const double a = A[row + j], b = B[row + j], c = C[row + j];
      d1 = fmax(d1, fabs(c - a));
      d2 = fmax(d2, fabs(c - 2.0 * b + a));
      if (i != j) off = fmax(off, fabs(b));
    }
  }
  double open = -INFINITY, turn_hi = INFINITY, turn_lo = INFINITY, closed = 0.0;
  for (int i = threadIdx.x; i < n; i += blockDim.x) {
    const double w = B[(long long)i * n + i];
    const double p2 = w - two_mu_emax, q2 = w - two_mu_emin;
    open = fmax(open, -p2);
    turn_hi = fmin(turn_hi, fabs(p2));
    turn_lo = fmin(turn_lo, fabs(q2));
    closed = fmax(closed, fabs(p2));
  }
  d1 = block_reduce(d1, true, red);
  d2 = block_reduce(d2, true, red);
  off = block_reduce(off, true, red);
  open = block_reduce(open, true, red);
  turn_hi = block_reduce(turn_hi, false, red);
  turn_lo = block_reduce(turn_lo, false, red);
  closed = block_reduce(closed, true, red);
  if (threadIdx.x == 0) {
    const double hs = h[s];
    float* f = out + (long long)s * kFeat;
    f[0] = (float)asinh(open);
    f[1] = (float)log10(turn_hi + 1e-12);
    f[2] = (float)log10(turn_lo + 1e-12);
    f[3] = (float)log10(d1 / (2.0 * hs) + 1e-30);
    f[4] = (float)log10(d2 / (hs * hs) + 1e-30);
    f[5] = (float)log10(off + 1e-30);
    f[6] = (float)log10(hs);
    f[7] = (float)log10(closed + 1e-12);
  }
}

// Forward pass of one sample; x is already normalised.  h1/h2 receive the activations.
__device__ __forceinline__ float mlp_eval(const float* P, const float (&x)[kFeat], float (&h1)[kHidden], float (&h2)[kHidden]) {
#pragma unroll
  for (int k = 0; k < kHidden; ++k) {
    float s = P[kOffB1 + k];
#pragma unroll
    for (int f = 0; f < kFeat; ++f) s = fmaf(P[kOffW1 + k * kFeat + f], x[f], s);
    h1[k] = tanhf(s);
  }
#pragma unroll
  for (int k = 0; k < kHidden; ++k) {
    float s = P[kOffB2 + k];
#pragma unroll
    for (int j = 0; j < kHidden; ++j) s = fmaf(P[kOffW2 + k * kHidden + j], h1[j], s);
    h2[k] = tanhf(s);
  }
  float y = P[kOffB3];
#pragma unroll
  for (int k = 0; k < kHidden; ++k) y = fmaf(P[kOffW3 + k], h2[k], y);
  return y;
}

// norm = [mean (8), inverse scale (8)]
__device__ __forceinline__ void mlp_load_sample(const float* __restrict__ X, const float* __restrict__ norm, long long i, float (&x)[kFeat]) {
#pragma unroll
  for (int f = 0; f < kFeat; ++f) x[f] = (X[i * kFeat + f] - norm[f]) * norm[kFeat + f];
}

__global__ void __launch_bounds__(128) mlp_forward_kernel(const float* __restrict__ params, const float* __restrict__ norm, const float* __restrict__ X, int n, float* __restrict__ Y) {
  __shared__ float P[kParams];
  for (int p = threadIdx.x; p < kParams; p += blockDim.x) P[p] = params[p];
  __syncthreads();
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float x[kFeat], h1[kHidden], h2[kHidden];
  mlp_load_sample(X, norm, i, x);
  Y[i] = mlp_eval(P, x, h1, h2);
}

// Loss over the batch: sum_i w_i c_i (y_i - t_i)^2 * inv_wsum, c_i = over_weight when the
// network over-predicts (y > t: a too-wide sector), else 1.  Each block writes the
// gradient of its 128 samples to partials[block][*] and its loss to loss_partials[block];
// mlp_reduce_kernel sums them in a fixed order (deterministic).
__global__ void __launch_bounds__(kMlpSamples) mlp_partial_grad_kernel(const float* __restrict__ params, const float* __restrict__ norm, const float* __restrict__ X, const float* __restrict__ T, const float* __restrict__ Wt, int n, float over_weight, float inv_wsum, float* __restrict__ partials, float* __restrict__ loss_partials) {
  extern __shared__ float sm[];
  float* P = sm;
  float* Xs = P + kParams;
  float* H1 = Xs + kMlpSamples * kFeat;
  float* H2 = H1 + kMlpSamples * kMlpPad;
  float* D1 = H2 + kMlpSamples * kMlpPad;
  float* D2 = D1 + kMlpSamples * kMlpPad;
  float* D3 = D2 + kMlpSamples * kMlpPad;
  float* Ls = D3 + kMlpSamples;
  const int t = threadIdx.x;
  for (int p = t; p < kParams; p += kMlpSamples) P[p] = params[p];
  __syncthreads();
  const long long i = (long long)blockIdx.x * kMlpSamples + t;
  // activations and deltas live in this thread's row of shared memory (row stride 33:
  // threads reading the same column hit distinct banks)
  float* h1 = H1 + t * kMlpPad;
  float* h2 = H2 + t * kMlpPad;
  float* d1 = D1 + t * kMlpPad;
  float* d2 = D2 + t * kMlpPad;
  float x[kFeat];
  float g = 0.0f, loss = 0.0f;
  if (i < n) {
    mlp_load_sample(X, norm, i, x);
  } else {
#pragma unroll
    for (int f = 0; f < kFeat; ++f) x[f] = 0.0f;
  }
#pragma unroll 4
  for (int k = 0; k < kHidden; ++k) {
    float s = P[kOffB1 + k];
#pragma unroll
    for (int f = 0; f < kFeat; ++f) s = fmaf(P[kOffW1 + k * kFeat + f], x[f], s);
    h1[k] = tanhf(s);
  }
#pragma unroll 2
  for (int k = 0; k < kHidden; ++k) {
    float s = P[kOffB2 + k];
#pragma unroll 8
    for (int j = 0; j < kHidden; ++j) s = fmaf(P[kOffW2 + k * kHidden + j], h1[j], s);
    h2[k] = tanhf(s);
  }
  if (i < n) {
    float y = P[kOffB3];
#pragma unroll 8
    for (int k = 0; k < kHidden; ++k) y = fmaf(P[kOffW3 + k], h2[k], y);
    const float r = y - T[i];
    const float c = (r > 0.0f ? over_weight : 1.0f) * Wt[i] * inv_wsum;
    g = 2.0f * c * r;
    loss = c * r * r;
  }
#pragma unroll 8
  for (int k = 0; k < kHidden; ++k) d2[k] = g * P[kOffW3 + k] * (1.0f - h2[k] * h2[k]);
#pragma unroll 2
  for (int j = 0; j < kHidden; ++j) {
    float s = 0.0f;
#pragma unroll 8
    for (int k = 0; k < kHidden; ++k) s = fmaf(d2[k], P[kOffW2 + k * kHidden + j], s);
    d1[j] = s * (1.0f - h1[j] * h1[j]);
  }
#pragma unroll
  for (int f = 0; f < kFeat; ++f) Xs[t * kFeat + f] = x[f];
  D3[t] = g;
  Ls[t] = loss;
  __syncthreads();
  float* out = partials + (long long)blockIdx.x * kParams;
  for (int p = t; p < kParams; p += kMlpSamples) {
    float acc = 0.0f;
    if (p < kOffB1) {
      const int k = p / kFeat, f = p % kFeat;
      for (int s = 0; s < kMlpSamples; ++s) acc = fmaf(D1[s * kMlpPad + k], Xs[s * kFeat + f], acc);
    } else if (p < kOffW2) {
      const int k = p - kOffB1;
      for (int s = 0; s < kMlpSamples; ++s) acc += D1[s * kMlpPad + k];
    } else if (p < kOffB2) {
      const int k = (p - kOffW2) / kHidden, j = (p - kOffW2) % kHidden;
      for (int s = 0; s < kMlpSamples; ++s) acc = fmaf(D2[s * kMlpPad + k], H1[s * kMlpPad + j], acc);
    } else if (p < kOffW3) {
      const int k = p - kOffB2;
      for (int s = 0; s < kMlpSamples; ++s) acc += D2[s * kMlpPad + k];
    } else if (p < kOffB3) {
      const int k = p - kOffW3;
      for (int s = 0; s < kMlpSamples; ++s) acc = fmaf(D3[s], H2[s * kMlpPad + k], acc);
    } else {
      for (int s = 0; s < kMlpSamples; ++s) acc += D3[s];
    }
    out[p] = acc;
  }
  if (t == 0) {
    float l = 0.0f;
    for (int s = 0; s < kMlpSamples; ++s) l += Ls[s];
    loss_partials[blockIdx.x] = l;
  }
}

__global__ void mlp_reduce_kernel(const float* __restrict__ partials, const float* __restrict__ loss_partials, int n_blocks, float* __restrict__ grads, float* __restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < kParams) {
    float acc = 0.0f;
    for (int b = 0; b < n_blocks; ++b) acc += partials[(long long)b * kParams + p];
    grads[p] = acc;
  }
  if (p == 0) {
    float l = 0.0f;
    for (int b = 0; b < n_blocks; ++b) l += loss_partials[b];
    *loss = l;
  }
}

// Adam; moments = [m (kParams), v (kParams)].  step counts from 1.
__global__ void mlp_adam_kernel(float* __restrict__ params, const float* __restrict__ grads, float* __restrict__ moments, int step, float lr, float beta1, float beta2, float eps) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= kParams) return;
  const float g = grads[p];
  const float m = beta1 * moments[p] + (1.0f - beta1) * g;
  const float v = beta2 * moments[kParams + p] + (1.0f - beta2) * g * g;
  moments[p] = m;
  moments[kParams + p] = v;
  const float mhat = m / (1.0f - powf(beta1, (float)step));
  const float vhat = v / (1.0f - powf(beta2, (float)step));
  params[p] -= lr * mhat / (sqrtf(vhat) + eps);
}

inline int mlp_grad_blocks(int n) { return (n + kMlpSamples - 1) / kMlpSamples; }
inline size_t mlp_workspace_floats(int n) { return (size_t)mlp_grad_blocks(n) * (kParams + 1); }

}  // namespace ticc
