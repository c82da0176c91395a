// The learned schedule cost model's network: a 3-layer MLP
// in -> h1 -> h2 -> out (ReLU on the hidden layers, linear output), with
// hand-written forward, backward, masked-MSE loss, Adam and masked-argmin
// kernels. Sizes are tiny (48 -> 64 -> 64 -> K, K <= 1024), so every kernel is
// a plain one-thread-per-output loop; all reductions run in a fixed order, so
// training is bitwise reproducible.
//
// Parameter vector layout (fp32): W1[h1][in], b1[h1], W2[h2][h1], b2[h2],
// W3[out][h2], b3[out]. Activations are row-major [batch][width].
#include "common.cuh"

namespace dtc {
namespace {

constexpr int kThreads = 256;

inline unsigned blocks_for(int64_t n) {
  int64_t g = (n + kThreads - 1) / kThreads;
  if (g < 1) g = 1;
  if (g > (1 << 30)) g = 1 << 30;
  return (unsigned)g;
}

// Y[r][o] = b[o] + sum_i X[r][i] * W[o][i]; ReLU if relu.
__global__ void k_linear(const float* __restrict__ X, const float* __restrict__ W,
                         const float* __restrict__ b, float* __restrict__ Y, int32_t B, int I,
                         int O, int relu) {
  const int64_t n = (int64_t)B * O;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
    const int64_t r = t / O;
    const int o = (int)(t % O);
    const float* x = X + r * I;
    const float* w = W + (int64_t)o * I;
    float s = b[o];
    for (int i = 0; i < I; ++i) s = fmaf(x[i], w[i], s);
    Y[t] = relu ? fmaxf(s, 0.0f) : s;
  }
}

// Masked MSE over [B][O]: loss = sum m (y - t)^2 / sum m, dY = 2 m (y - t) / sum m.
// One block; each thread sums a fixed strided subset, then a fixed tree.
__global__ void k_mse(const float* __restrict__ Y, const float* __restrict__ T,
                      const float* __restrict__ Mk, int64_t n, float* __restrict__ dY,
                      float* __restrict__ loss) {
  __shared__ double sl[kThreads], sm[kThreads];
  double l = 0.0, m = 0.0;
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x) {
    const double d = (double)Y[i] - (double)T[i];
    l += (double)Mk[i] * d * d;
    m += (double)Mk[i];
  }
  sl[threadIdx.x] = l;
  sm[threadIdx.x] = m;
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s) {
      sl[threadIdx.x] += sl[threadIdx.x + s];
      sm[threadIdx.x] += sm[threadIdx.x + s];
    }
    __syncthreads();
  }
  const double msum = sm[0] > 0 ? sm[0] : 1.0;
  if (threadIdx.x == 0) *loss = (float)(sl[0] / msum);
  const float scale = (float)(2.0 / msum);
  for (int64_t i = threadIdx.x; i < n; i += blockDim.x)
    dY[i] = Mk[i] * scale * (Y[i] - T[i]);
}

// dW[o][i] = sum_r dY[r][o] X[r][i]; db[o] = sum_r dY[r][o] (thread i == I).
__global__ void k_grad_w(const float* __restrict__ dY, const float* __restrict__ X, int32_t B,
                         int I, int O, float* __restrict__ dW, float* __restrict__ db) {
  const int64_t n = (int64_t)O * (I + 1);
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
    const int o = (int)(t / (I + 1));
    const int i = (int)(t % (I + 1));
    float s = 0.0f;
    if (i < I) {
      for (int32_t r = 0; r < B; ++r) s = fmaf(dY[(int64_t)r * O + o], X[(int64_t)r * I + i], s);
      dW[(int64_t)o * I + i] = s;
    } else {
      for (int32_t r = 0; r < B; ++r) s += dY[(int64_t)r * O + o];
      db[o] = s;
    }
  }
}

// dX[r][i] = (H[r][i] > 0) * sum_o dY[r][o] W[o][i]  (H = ReLU output feeding the layer)
__global__ void k_grad_x(const float* __restrict__ dY, const float* __restrict__ W,
                         const float* __restrict__ H, int32_t B, int I, int O,
                         float* __restrict__ dX) {
  const int64_t n = (int64_t)B * I;
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < n; t += stride) {
    const int64_t r = t / I;
    const int i = (int)(t % I);
    float s = 0.0f;
    if (H[t] > 0.0f)
      for (int o = 0; o < O; ++o) s = fmaf(dY[r * O + o], W[(int64_t)o * I + i], s);
    dX[t] = s;
  }
}

__global__ void k_adam(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                       float* __restrict__ v, int64_t n, float lr, float b1, float b2, float eps,
                       float c1, float c2) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n; i += stride) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

// choice[r] = argmin over feasible o of Y[r][o] (lowest index on ties); -1 if none.
__global__ void k_argmin(const float* __restrict__ Y, const uint8_t* __restrict__ feas,
                         int feas_per_row, int32_t B, int O, int32_t* __restrict__ choice) {
  int64_t stride = (int64_t)gridDim.x * blockDim.x;
  for (int64_t r = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; r < B; r += stride) {
    const uint8_t* f = feas ? feas + (feas_per_row ? r * O : 0) : nullptr;
    int best = -1;
    float bv = 0.0f;
    for (int o = 0; o < O; ++o) {
      if (f && !f[o]) continue;
      const float y = Y[r * O + o];
      if (best < 0 || y < bv) { best = o; bv = y; }
    }
    choice[r] = best;
  }
}

struct Offs {
  int64_t W1, b1, W2, b2, W3, b3, total;
};

Offs offsets(const dtc_mlp_dims& d) {
  Offs o{};
  o.W1 = 0;
  o.b1 = o.W1 + (int64_t)d.h1 * d.in;
  o.W2 = o.b1 + d.h1;
  o.b2 = o.W2 + (int64_t)d.h2 * d.h1;
  o.W3 = o.b2 + d.h2;
  o.b3 = o.W3 + (int64_t)d.out * d.h2;
  o.total = o.b3 + d.out;
  return o;
}

bool dims_ok(const dtc_mlp_dims* d) {
  return d && d->in >= 1 && d->h1 >= 1 && d->h2 >= 1 && d->out >= 1 && d->in <= 4096 &&
         d->h1 <= 4096 && d->h2 <= 4096 && d->out <= 4096;
}

}  // namespace
}  // namespace dtc

using namespace dtc;

extern "C" {

int64_t dtc_mlp_num_params(const dtc_mlp_dims* dims) {
  return dims_ok(dims) ? offsets(*dims).total : -1;
}

dtc_status dtc_mlp_forward(const dtc_mlp_dims* dims, const float* d_params, const float* d_X,
                           int32_t batch, float* d_H1, float* d_H2, float* d_Y,
                           dtc_stream_t stream) {
  DTC_REQUIRE(dims_ok(dims), "bad MLP dimensions");
  DTC_REQUIRE(batch >= 0, "negative batch");
  DTC_REQUIRE(d_params && d_X && d_H1 && d_H2 && d_Y, "null device pointer");
  if (batch == 0) return DTC_OK;
  const dtc_mlp_dims& d = *dims;
  const Offs o = offsets(d);
  cudaStream_t st = (cudaStream_t)stream;
  k_linear<<<blocks_for((int64_t)batch * d.h1), kThreads, 0, st>>>(
      d_X, d_params + o.W1, d_params + o.b1, d_H1, batch, d.in, d.h1, 1);
  k_linear<<<blocks_for((int64_t)batch * d.h2), kThreads, 0, st>>>(
      d_H1, d_params + o.W2, d_params + o.b2, d_H2, batch, d.h1, d.h2, 1);
  k_linear<<<blocks_for((int64_t)batch * d.out), kThreads, 0, st>>>(
      d_H2, d_params + o.W3, d_params + o.b3, d_Y, batch, d.h2, d.out, 0);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

size_t dtc_mlp_backward_workspace_bytes(const dtc_mlp_dims* dims, int32_t batch) {
  if (!dims_ok(dims) || batch < 0) return 0;
  const size_t b = (size_t)(batch > 0 ? batch : 1);
  return align_up(b * dims->out * 4, 256) + align_up(b * dims->h2 * 4, 256) +
         align_up(b * dims->h1 * 4, 256);
}

dtc_status dtc_mlp_backward(const dtc_mlp_dims* dims, const float* d_params, const float* d_X,
                            const float* d_H1, const float* d_H2, const float* d_Y,
                            const float* d_target, const float* d_mask, int32_t batch,
                            float* d_grads, float* d_loss, void* d_workspace,
                            size_t workspace_bytes, dtc_stream_t stream) {
  DTC_REQUIRE(dims_ok(dims), "bad MLP dimensions");
  DTC_REQUIRE(batch >= 1, "batch must be >= 1");
  DTC_REQUIRE(d_params && d_X && d_H1 && d_H2 && d_Y && d_target && d_mask && d_grads && d_loss,
              "null device pointer");
  if (!d_workspace || workspace_bytes < dtc_mlp_backward_workspace_bytes(dims, batch)) {
    set_error("MLP backward workspace too small");
    return DTC_ERR_WORKSPACE_TOO_SMALL;
  }
  const dtc_mlp_dims& d = *dims;
  const Offs o = offsets(d);
  cudaStream_t st = (cudaStream_t)stream;
  char* ws = (char*)d_workspace;
  float* dY = (float*)ws;
  float* dH2 = (float*)(ws + align_up((size_t)batch * d.out * 4, 256));
  float* dH1 = (float*)((char*)dH2 + align_up((size_t)batch * d.h2 * 4, 256));
  k_mse<<<1, kThreads, 0, st>>>(d_Y, d_target, d_mask, (int64_t)batch * d.out, dY, d_loss);
  k_grad_w<<<blocks_for((int64_t)d.out * (d.h2 + 1)), kThreads, 0, st>>>(
      dY, d_H2, batch, d.h2, d.out, d_grads + o.W3, d_grads + o.b3);
  k_grad_x<<<blocks_for((int64_t)batch * d.h2), kThreads, 0, st>>>(dY, d_params + o.W3, d_H2,
                                                                    batch, d.h2, d.out, dH2);
  k_grad_w<<<blocks_for((int64_t)d.h2 * (d.h1 + 1)), kThreads, 0, st>>>(
      dH2, d_H1, batch, d.h1, d.h2, d_grads + o.W2, d_grads + o.b2);
  k_grad_x<<<blocks_for((int64_t)batch * d.h1), kThreads, 0, st>>>(dH2, d_params + o.W2, d_H1,
                                                                    batch, d.h1, d.h2, dH1);
  k_grad_w<<<blocks_for((int64_t)d.h1 * (d.in + 1)), kThreads, 0, st>>>(
      dH1, d_X, batch, d.in, d.h1, d_grads + o.W1, d_grads + o.b1);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

dtc_status dtc_mlp_adam(float* d_params, const float* d_grads, float* d_m, float* d_v, int64_t n,
                        float lr, float beta1, float beta2, float eps, int32_t step,
                        dtc_stream_t stream) {
  DTC_REQUIRE(d_params && d_grads && d_m && d_v, "null device pointer");
  DTC_REQUIRE(n >= 0 && step >= 1, "bad sizes");
  DTC_REQUIRE(beta1 >= 0.0f && beta1 < 1.0f && beta2 >= 0.0f && beta2 < 1.0f, "bad betas");
  const float c1 = 1.0f - powf(beta1, (float)step), c2 = 1.0f - powf(beta2, (float)step);
  k_adam<<<blocks_for(n), kThreads, 0, (cudaStream_t)stream>>>(d_params, d_grads, d_m, d_v, n, lr,
                                                               beta1, beta2, eps, c1, c2);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

dtc_status dtc_mlp_argmin(const float* d_Y, const uint8_t* d_feasible, int feasible_per_row,
                          int32_t batch, int32_t out, int32_t* d_choice, dtc_stream_t stream) {
  DTC_REQUIRE(d_Y && d_choice, "null device pointer");
  DTC_REQUIRE(batch >= 0 && out >= 1, "bad sizes");
  if (batch == 0) return DTC_OK;
  k_argmin<<<blocks_for(batch), kThreads, 0, (cudaStream_t)stream>>>(d_Y, d_feasible,
                                                                     feasible_per_row, batch, out,
                                                                     d_choice);
  DTC_CUDA(cudaGetLastError());
  return DTC_OK;
}

}  // extern "C"
