// mlp.cu -- the small networks of the learned parts, trained and run by this
// library's own kernels (no reference counterpart).
//
// One shape: in (<= 8) -> hidden (<= 64, ReLU) -> hidden (ReLU) -> 1.
// Parameters are fp32 for training, packed as
//   W1[h][in], b1[h], W2[h][h], b2[h], w3[h], b3
// and rounded to bf16 for inference (fp32 accumulation).  Losses: squared
// error (regression) or binary cross-entropy on the logit (classification),
// averaged over the batch.
//
// Training step on a batch of B samples (all resident in HBM):
//  1. mlpk_forward: a thread per sample, the parameters in shared memory;
//     keeps both hidden activations;
//  2. mlpk_backward: a thread per sample: the output gradient, then the
//     hidden-layer gradients (ReLU masks), kept per sample;
//  3. mlpk_grad: a thread per parameter, summing its gradient over the batch
//     in sample order (a fixed order: the gradients are deterministic);
//  4. mlpk_adam: Adam on the fp32 parameters.
// The gradients of step 3 are what the tests check against an FP64 CPU
// computation.
#include <cuda_bf16.h>

#include <vector>

#include "graph.cuh"

namespace ogb {

constexpr int kMlpMaxIn = 8, kMlpMaxH = 64;
constexpr int kMlpMaxParams = kMlpMaxH * kMlpMaxIn + kMlpMaxH + kMlpMaxH * kMlpMaxH + kMlpMaxH + kMlpMaxH + 1;

__host__ __device__ constexpr int mlp_nparams(int in, int h) { return h * in + h + h * h + h + h + 1; }

struct MlpOff {
  int w1, b1, w2, b2, w3, b3;
};
__host__ __device__ inline MlpOff mlp_off(int in, int h) {
  MlpOff o;
  o.w1 = 0;
  o.b1 = h * in;
  o.w2 = o.b1 + h;
  o.b2 = o.w2 + h * h;
  o.w3 = o.b2 + h;
  o.b3 = o.w3 + h;
  return o;
}

// Forward pass of one sample with parameters P (fp32, in shared memory or
// registers' reach); returns the output, and the activations when asked.
__device__ __forceinline__ float mlp_fwd(const float* P, const float* x, int in, int h, float* a1, float* a2) {
  const MlpOff o = mlp_off(in, h);
  float h1[kMlpMaxH], h2[kMlpMaxH];
  for (int i = 0; i < h; i++) {
    float s = P[o.b1 + i];
    for (int j = 0; j < in; j++) s = fmaf(P[o.w1 + i * in + j], x[j], s);
    h1[i] = fmaxf(s, 0.0f);
  }
  for (int i = 0; i < h; i++) {
    float s = P[o.b2 + i];
    for (int j = 0; j < h; j++) s = fmaf(P[o.w2 + i * h + j], h1[j], s);
    h2[i] = fmaxf(s, 0.0f);
  }
  float y = P[o.b3];
  for (int i = 0; i < h; i++) y = fmaf(P[o.w3 + i], h2[i], y);
  if (a1)
    for (int i = 0; i < h; i++) {
      a1[i] = h1[i];
      a2[i] = h2[i];
    }
  return y;
}

__global__ void __launch_bounds__(128) mlpk_forward(const float* __restrict__ X, const float* __restrict__ params,
                                                    int B, int in, int h, float* __restrict__ A1,
                                                    float* __restrict__ A2, float* __restrict__ Y) {
  __shared__ float P[kMlpMaxParams];
  const int np = mlp_nparams(in, h);
  for (int i = threadIdx.x; i < np; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    float x[kMlpMaxIn];
    for (int j = 0; j < in; j++) x[j] = X[(size_t)b * in + j];
    float a1[kMlpMaxH], a2[kMlpMaxH];
    Y[b] = mlp_fwd(P, x, in, h, a1, a2);
    for (int i = 0; i < h; i++) {
      A1[(size_t)b * h + i] = a1[i];
      A2[(size_t)b * h + i] = a2[i];
    }
  }
}

// dY = dLoss/dy (mean over the batch); D2 = dLoss/d(pre-activation 2);
// D1 = dLoss/d(pre-activation 1); Lb = per-sample loss.
__global__ void __launch_bounds__(128) mlpk_backward(const float* __restrict__ params, const float* __restrict__ T,
                                                     int B, int in, int h, int loss, const float* __restrict__ A1,
                                                     const float* __restrict__ A2, const float* __restrict__ Y,
                                                     float* __restrict__ dY, float* __restrict__ D1,
                                                     float* __restrict__ D2, float* __restrict__ Lb) {
  __shared__ float P[kMlpMaxParams];
  const int np = mlp_nparams(in, h);
  for (int i = threadIdx.x; i < np; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  const MlpOff o = mlp_off(in, h);
  const float invB = 1.0f / (float)B;
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const float y = Y[b], t = T[b];
    float dy, l;
    if (loss == 0) {
      dy = 2.0f * (y - t) * invB;
      l = (y - t) * (y - t);
    } else {
      const float p = 1.0f / (1.0f + expf(-y));
      dy = (p - t) * invB;
      l = fmaxf(y, 0.0f) - y * t + log1pf(expf(-fabsf(y)));
    }
    dY[b] = dy;
    Lb[b] = l;
    float d2[kMlpMaxH];
    for (int i = 0; i < h; i++) {
      d2[i] = (A2[(size_t)b * h + i] > 0.0f) ? dy * P[o.w3 + i] : 0.0f;
      D2[(size_t)b * h + i] = d2[i];
    }
    for (int j = 0; j < h; j++) {
      float s = 0.0f;
      for (int i = 0; i < h; i++) s = fmaf(P[o.w2 + i * h + j], d2[i], s);
      D1[(size_t)b * h + j] = (A1[(size_t)b * h + j] > 0.0f) ? s : 0.0f;
    }
  }
}

// A thread per parameter: its gradient summed over the batch in sample order.
__global__ void mlpk_grad(const float* __restrict__ X, int B, int in, int h, const float* __restrict__ A1,
                          const float* __restrict__ A2, const float* __restrict__ dY, const float* __restrict__ D1,
                          const float* __restrict__ D2, float* __restrict__ grad) {
  const int np = mlp_nparams(in, h);
  const MlpOff o = mlp_off(in, h);
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    float s = 0.0f;
    if (k < o.b1) {
      const int i = k / in, j = k % in;
      for (int b = 0; b < B; b++) s = fmaf(D1[(size_t)b * h + i], X[(size_t)b * in + j], s);
    } else if (k < o.w2) {
      const int i = k - o.b1;
      for (int b = 0; b < B; b++) s += D1[(size_t)b * h + i];
    } else if (k < o.b2) {
      const int i = (k - o.w2) / h, j = (k - o.w2) % h;
      for (int b = 0; b < B; b++) s = fmaf(D2[(size_t)b * h + i], A1[(size_t)b * h + j], s);
    } else if (k < o.w3) {
      const int i = k - o.b2;
      for (int b = 0; b < B; b++) s += D2[(size_t)b * h + i];
    } else if (k < o.b3) {
      const int i = k - o.w3;
      for (int b = 0; b < B; b++) s = fmaf(dY[b], A2[(size_t)b * h + i], s);
    } else {
      for (int b = 0; b < B; b++) s += dY[b];
    }
    grad[k] = s;
  }
}

__global__ void mlpk_adam(float* __restrict__ params, const float* __restrict__ grad, float* __restrict__ m,
                          float* __restrict__ v, int np, float lr, float b1, float b2, float eps, float c1, float c2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    const float g = grad[k];
    const float mk = b1 * m[k] + (1.0f - b1) * g;
    const float vk = b2 * v[k] + (1.0f - b2) * g * g;
    m[k] = mk;
    v[k] = vk;
    params[k] -= lr * (mk / c1) / (sqrtf(vk / c2) + eps);
  }
}

__global__ void mlpk_gather(const float* __restrict__ X, const float* __restrict__ T, const uint32_t* __restrict__ idx,
                            int B, int in, float* __restrict__ bx, float* __restrict__ bt) {
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < B; b += gridDim.x * blockDim.x) {
    const uint32_t i = idx[b];
    for (int j = 0; j < in; j++) bx[(size_t)b * in + j] = X[(size_t)i * in + j];
    bt[b] = T[i];
  }
}

__global__ void mlpk_sum(const float* __restrict__ x, int n, float* __restrict__ out) {
  __shared__ float s[256];
  float a = 0.0f;
  for (int i = threadIdx.x; i < n; i += blockDim.x) a += x[i];
  s[threadIdx.x] = a;
  __syncthreads();
  for (int o = 128; o; o >>= 1) {
    if ((int)threadIdx.x < o) s[threadIdx.x] += s[threadIdx.x + o];
    __syncthreads();
  }
  if (threadIdx.x == 0) *out = s[0];
}

// Inference with bf16 weights (rounded from fp32), fp32 accumulation.
__device__ __forceinline__ float mlp_fwd_bf16(const __nv_bfloat16* P, const float* x, int in, int h) {
  const MlpOff o = mlp_off(in, h);
  float h1[kMlpMaxH];
  for (int i = 0; i < h; i++) {
    float s = __bfloat162float(P[o.b1 + i]);
    for (int j = 0; j < in; j++) s = fmaf(__bfloat162float(P[o.w1 + i * in + j]), x[j], s);
    h1[i] = fmaxf(s, 0.0f);
  }
  float y = __bfloat162float(P[o.b3]);
  for (int i = 0; i < h; i++) {
    float s = __bfloat162float(P[o.b2 + i]);
    for (int j = 0; j < h; j++) s = fmaf(__bfloat162float(P[o.w2 + i * h + j]), h1[j], s);
    y = fmaf(__bfloat162float(P[o.w3 + i]), fmaxf(s, 0.0f), y);
  }
  return y;
}

__global__ void mlpk_to_bf16(const float* __restrict__ p, int n, __nv_bfloat16* __restrict__ q) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) q[i] = __float2bfloat16_rn(p[i]);
}

__global__ void __launch_bounds__(128) mlpk_infer(const float* __restrict__ X, const __nv_bfloat16* __restrict__ params,
                                                  int N, int in, int h, float* __restrict__ Y) {
  __shared__ __nv_bfloat16 P[kMlpMaxParams];
  const int np = mlp_nparams(in, h);
  for (int i = threadIdx.x; i < np; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (int b = blockIdx.x * blockDim.x + threadIdx.x; b < N; b += gridDim.x * blockDim.x) {
    float x[kMlpMaxIn];
    for (int j = 0; j < in; j++) x[j] = X[(size_t)b * in + j];
    Y[b] = mlp_fwd_bf16(P, x, in, h);
  }
}

// PageRank warm start: features log2(1 + in_degree), log2(1 + out_degree),
// the network predicts log2 of the vertex's unnormalized converged rank; the
// start vector is 2^prediction.
__global__ void __launch_bounds__(128) mlpk_pr_start(uint32_t V, const uint32_t* __restrict__ in_deg,
                                                     const uint32_t* __restrict__ out_deg,
                                                     const __nv_bfloat16* __restrict__ params, int h,
                                                     float* __restrict__ init) {
  __shared__ __nv_bfloat16 P[kMlpMaxParams];
  const int np = mlp_nparams(2, h);
  for (int i = threadIdx.x; i < np; i += blockDim.x) P[i] = params[i];
  __syncthreads();
  for (uint32_t v = blockIdx.x * blockDim.x + threadIdx.x; v < V; v += gridDim.x * blockDim.x) {
    float x[2] = {log2f(1.0f + (float)in_deg[v]), log2f(1.0f + (float)out_deg[v])};
    init[v] = exp2f(mlp_fwd_bf16(P, x, 2, h));
  }
}

// ------------------------------------------------------------ host ---------

static int check_shape(int in, int h) {
  if (in < 1 || in > kMlpMaxIn || h < 1 || h > kMlpMaxH) return fail(ERR_ARG, "mlp: shape %d -> %d unsupported", in, h);
  return OK;
}

int mlp_nparams_host(int in, int h) { return mlp_nparams(in, h); }

struct MlpScratch {
  DevBuf A1, A2, Y, dY, D1, D2, Lb, grad, params, m, v, lsum;
  int reserve(int B, int in, int h) {
    const size_t np = mlp_nparams(in, h);
    OGB_TRY(A1.alloc((size_t)B * h * 4));
    OGB_TRY(A2.alloc((size_t)B * h * 4));
    OGB_TRY(D1.alloc((size_t)B * h * 4));
    OGB_TRY(D2.alloc((size_t)B * h * 4));
    OGB_TRY(Y.alloc((size_t)B * 4));
    OGB_TRY(dY.alloc((size_t)B * 4));
    OGB_TRY(Lb.alloc((size_t)B * 4));
    OGB_TRY(grad.alloc(np * 4));
    OGB_TRY(params.alloc(np * 4));
    OGB_TRY(m.alloc(np * 4));
    OGB_TRY(v.alloc(np * 4));
    OGB_TRY(lsum.alloc(16));
    return OK;
  }
};

static void mlp_step_grads(MlpScratch& w, const float* X, const float* T, int B, int in, int h, int loss,
                           cudaStream_t s) {
  const int grid = std::max(1, std::min(sm_count() * 4, (B + 127) / 128));
  mlpk_forward<<<grid, 128, 0, s>>>(X, w.params.as<float>(), B, in, h, w.A1.as<float>(), w.A2.as<float>(),
                                    w.Y.as<float>());
  mlpk_backward<<<grid, 128, 0, s>>>(w.params.as<float>(), T, B, in, h, loss, w.A1.as<float>(), w.A2.as<float>(),
                                     w.Y.as<float>(), w.dY.as<float>(), w.D1.as<float>(), w.D2.as<float>(),
                                     w.Lb.as<float>());
  const int np = mlp_nparams(in, h);
  mlpk_grad<<<(np + 127) / 128, 128, 0, s>>>(X, B, in, h, w.A1.as<float>(), w.A2.as<float>(), w.dY.as<float>(),
                                             w.D1.as<float>(), w.D2.as<float>(), w.grad.as<float>());
}

int mlp_grad(int in, int h, int loss, const float* X, const float* T, int B, const float* params_host,
             float* grad_host, float* loss_host, cudaStream_t s) {
  OGB_TRY(check_shape(in, h));
  if (B < 1) return fail(ERR_ARG, "mlp: empty batch");
  MlpScratch w;
  OGB_TRY(w.reserve(B, in, h));
  const int np = mlp_nparams(in, h);
  OGB_CUDA(cudaMemcpyAsync(w.params.p, params_host, np * 4, cudaMemcpyHostToDevice, s));
  mlp_step_grads(w, X, T, B, in, h, loss, s);
  mlpk_sum<<<1, 256, 0, s>>>(w.Lb.as<float>(), B, w.lsum.as<float>());
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaMemcpyAsync(grad_host, w.grad.p, np * 4, cudaMemcpyDeviceToHost, s));
  float l = 0.f;
  OGB_CUDA(cudaMemcpyAsync(&l, w.lsum.p, 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  if (loss_host) *loss_host = l / (float)B;
  return OK;
}

// Adam over shuffled mini-batches (the sample order is shuffled once per
// epoch on the host from `seed`; the batches are gathered on the device).
int mlp_train(int in, int h, int loss, const float* X, const float* T, int N, int epochs, int batch, float lr,
              uint32_t seed, float* params_host, float* loss_hist, cudaStream_t s) {
  OGB_TRY(check_shape(in, h));
  if (N < 1 || batch < 1 || epochs < 0) return fail(ERR_ARG, "mlp_train: bad sizes");
  batch = std::min(batch, N);
  const int np = mlp_nparams(in, h);
  MlpScratch w;
  OGB_TRY(w.reserve(batch, in, h));
  DevBuf bx, bt, idx;
  OGB_TRY(bx.alloc((size_t)batch * in * 4));
  OGB_TRY(bt.alloc((size_t)batch * 4));
  OGB_TRY(idx.alloc((size_t)N * 4));
  OGB_CUDA(cudaMemcpyAsync(w.params.p, params_host, np * 4, cudaMemcpyHostToDevice, s));
  OGB_CUDA(cudaMemsetAsync(w.m.p, 0, np * 4, s));
  OGB_CUDA(cudaMemsetAsync(w.v.p, 0, np * 4, s));
  std::vector<uint32_t> order(N);
  uint64_t rs = seed * 0x9E3779B97F4A7C15ull + 1;
  auto rnd = [&rs]() {
    rs ^= rs << 13;
    rs ^= rs >> 7;
    rs ^= rs << 17;
    return rs;
  };
  int t = 0;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int e = 0; e < epochs; e++) {
    for (int i = 0; i < N; i++) order[i] = (uint32_t)i;
    for (int i = N - 1; i > 0; i--) std::swap(order[i], order[rnd() % (uint64_t)(i + 1)]);
    OGB_CUDA(cudaMemcpyAsync(idx.p, order.data(), (size_t)N * 4, cudaMemcpyHostToDevice, s));
    double esum = 0.0;
    int nb = 0;
    for (int b0 = 0; b0 + batch <= N; b0 += batch) {
      mlpk_gather<<<std::max(1, std::min(sm_count() * 4, (batch + 127) / 128)), 128, 0, s>>>(
          X, T, idx.as<uint32_t>() + b0, batch, in, bx.as<float>(), bt.as<float>());
      mlp_step_grads(w, bx.as<float>(), bt.as<float>(), batch, in, h, loss, s);
      t++;
      const float c1 = 1.0f - powf(b1, (float)t), c2 = 1.0f - powf(b2, (float)t);
      mlpk_adam<<<(np + 127) / 128, 128, 0, s>>>(w.params.as<float>(), w.grad.as<float>(), w.m.as<float>(),
                                                 w.v.as<float>(), np, lr, b1, b2, 1e-8f, c1, c2);
      if (loss_hist) {
        mlpk_sum<<<1, 256, 0, s>>>(w.Lb.as<float>(), batch, w.lsum.as<float>());
        float l = 0.f;
        OGB_CUDA(cudaMemcpyAsync(&l, w.lsum.p, 4, cudaMemcpyDeviceToHost, s));
        OGB_CUDA(cudaStreamSynchronize(s));
        esum += l / batch;
        nb++;
      }
    }
    OGB_CUDA(cudaGetLastError());
    if (loss_hist) loss_hist[e] = nb ? (float)(esum / nb) : 0.0f;
  }
  OGB_CUDA(cudaMemcpyAsync(params_host, w.params.p, np * 4, cudaMemcpyDeviceToHost, s));
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int mlp_infer(int in, int h, const float* params_host, const float* X, int N, float* Y, cudaStream_t s) {
  OGB_TRY(check_shape(in, h));
  const int np = mlp_nparams(in, h);
  DevBuf pf, pb;
  OGB_TRY(pf.alloc(np * 4));
  OGB_TRY(pb.alloc(np * 2 + 16));
  OGB_CUDA(cudaMemcpyAsync(pf.p, params_host, np * 4, cudaMemcpyHostToDevice, s));
  mlpk_to_bf16<<<(np + 255) / 256, 256, 0, s>>>(pf.as<float>(), np, pb.as<__nv_bfloat16>());
  if (N > 0)
    mlpk_infer<<<std::max(1, std::min(sm_count() * 8, (N + 127) / 128)), 128, 0, s>>>(
        X, pb.as<__nv_bfloat16>(), N, in, h, Y);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

int pr_warm_start(DevGraph& g, int h, const float* params_host, float* init, cudaStream_t s) {
  OGB_TRY(check_shape(2, h));
  const int np = mlp_nparams(2, h);
  DevBuf pf, pb;
  OGB_TRY(pf.alloc(np * 4));
  OGB_TRY(pb.alloc(np * 2 + 16));
  OGB_CUDA(cudaMemcpyAsync(pf.p, params_host, np * 4, cudaMemcpyHostToDevice, s));
  mlpk_to_bf16<<<(np + 255) / 256, 256, 0, s>>>(pf.as<float>(), np, pb.as<__nv_bfloat16>());
  mlpk_pr_start<<<sm_count() * 8, 128, 0, s>>>(g.V, g.inv.d_out_degree(), g.fwd.d_out_degree(),
                                               pb.as<__nv_bfloat16>(), h, init);
  OGB_CUDA(cudaGetLastError());
  OGB_CUDA(cudaStreamSynchronize(s));
  return OK;
}

}  // namespace ogb
