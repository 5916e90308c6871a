// Screening network: a small MLP 12 -> 256 -> 256 -> 256 -> 1 with GELU,
// trained and evaluated by hand-written kernels.  Weights are kept as FP32
// master copies for the optimiser and used in BF16 (rounded on load) by every
// product, with FP32 accumulation ("BF16 weights, FP32 accumulation").
// No counterpart in the reference (phoebe has no learned screening).
//
// Kernels: one tensor-core GEMM (tcgen05, 128 x 64 output tile per CTA)
// used for the forward products X W^T, the weight gradients dY^T X and the
// input gradients dY W; element-wise bias + GELU and its derivative; a
// mean-squared-error head; Adam.  GELU is the tanh form
// 0.5 x (1 + tanh(sqrt(2/pi)(x + 0.044715 x^3))).
//
// GEMM numerics: operands are staged in shared memory as BF16 hi + lo pairs.
// A weight operand keeps its hi part only (BF16 weights, exactly as rounded
// for the forward pass), so the product is A_hi W + A_lo W; two activation /
// gradient operands take hi*hi + hi*lo + lo*hi.  K is processed in 64-deep
// chunks, each accumulated in FP32 in tensor memory and added to FP32
// registers, so the tensor core's FP32 accumulation runs over 64 terms at a
// time.
#include <algorithm>
#include <cmath>
#include <cuda_bf16.h>
#include <string>
#include <vector>

#include "phx_internal.h"
#include "tc.cuh"
#include "tcgemm.cuh"

struct phx_mlp {
  phx_ctx* ctx = nullptr;
  int nin = 0, hidden = 0, layers = 0;  // layers = number of weight matrices (4)
  std::vector<int> dims;                // nin, hidden, hidden, hidden, 1
  std::vector<size_t> woff, boff;       // parameter offsets (floats)
  size_t nparam = 0;
  float* d_param = nullptr;             // FP32 master parameters
  float* d_grad = nullptr;
  float* d_m = nullptr;                 // Adam moments
  float* d_v = nullptr;
  long long step = 0;
  void* d_scratch = nullptr;            // activations of one batch
  size_t scratch_bytes = 0;
};

namespace {

__device__ __forceinline__ float bf16r(float x) { return __bfloat162float(__float2bfloat16_rn(x)); }

__device__ __forceinline__ float gelu(float x) {
  const float k = 0.7978845608028654f;  // sqrt(2/pi)
  return 0.5f * x * (1.f + tanhf(k * (x + 0.044715f * x * x * x)));
}
__device__ __forceinline__ float gelu_d(float x) {
  const float k = 0.7978845608028654f;
  const float u = k * (x + 0.044715f * x * x * x);
  const float t = tanhf(u);
  return 0.5f * (1.f + t) + 0.5f * x * (1.f - t * t) * k * (1.f + 3.f * 0.044715f * x * x);
}

// Z[b,n] += bias[n]; A = act ? GELU(Z) : Z
__global__ void bias_act_kernel(float* __restrict__ Z, float* __restrict__ Aout, const float* __restrict__ bias,
                                int B, int N, int act) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < (size_t)B * N; i += (size_t)gridDim.x * blockDim.x) {
    const float z = Z[i] + bf16r(bias[i % N]);
    Z[i] = z;
    Aout[i] = act ? gelu(z) : z;
  }
}

// dZ = dA * GELU'(Z)
__global__ void gelu_back_kernel(const float* __restrict__ Z, float* __restrict__ dA, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dA[i] *= gelu_d(Z[i]);
}

// bias gradient: db[n] = sum_b dZ[b,n]
__global__ void bias_grad_kernel(const float* __restrict__ dZ, float* __restrict__ db, int B, int N) {
  const int n = blockIdx.x * blockDim.x + threadIdx.x;
  if (n >= N) return;
  float s = 0.f;
  for (int b = 0; b < B; ++b) s += dZ[(size_t)b * N + n];
  db[n] += s;
}

// mean squared error on the output (B x 1): dY = 2 (y - t) / B, loss into *loss
__global__ void mse_kernel(const float* __restrict__ y, const float* __restrict__ t, float* __restrict__ dy, int B,
                           float* __restrict__ loss) {
  float s = 0.f;
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < B; i += gridDim.x * blockDim.x) {
    const float d = y[i] - t[i];
    dy[i] = 2.f * d / (float)B;
    s += d * d;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, s / (float)B);
}

__global__ void adam_kernel(float* __restrict__ p, const float* __restrict__ g, float* __restrict__ m,
                            float* __restrict__ v, size_t n, float lr, float b1, float b2, float eps, float c1,
                            float c2) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.f - b1) * gi;
    const float vi = b2 * v[i] + (1.f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
  }
}

template <bool TA, bool TB, bool RB>
int gemm(phx_ctx* ctx, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C, int ldc,
         int accumulate) {
  PHX_CUDA(ctx, (tcgemm::launch<TA, TB, RB, false>(M, N, K, A, lda, B, ldb, C, ldc, accumulate, 1.f, ctx->d_status,
                                                   ctx->stream)));
  return PHX_OK;
}

// a tensor-core GEMM that gave up waiting for its MMAs leaves a status bit
int check_status(phx_ctx* ctx) {
  int st = 0;
  PHX_CUDA(ctx, cudaMemcpy(&st, ctx->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (st) {
    cudaMemset(ctx->d_status, 0, sizeof(int));
    phx_set_error(ctx, PHX_ERR_CUDA, "screening network: a tensor-core GEMM gave up waiting (status " +
                                         std::to_string(st) + ")");
    return PHX_ERR_CUDA;
  }
  return PHX_OK;
}

int ew_grid(phx_ctx* ctx, size_t n) { return (int)std::min<size_t>((n + 255) / 256, (size_t)ctx->num_sms * 8); }

// activations of one batch: per layer Z (pre-activation) and A (output)
struct Acts {
  std::vector<float*> Z, A;   // A[0] = input
};

int reserve(phx_mlp* net, int B, Acts& acts, float** dA0, float** dA1, float** loss) {
  size_t per = 0;
  for (size_t l = 0; l < net->dims.size(); ++l) per += (size_t)B * net->dims[l];
  const size_t widest = (size_t)B * *std::max_element(net->dims.begin(), net->dims.end());
  const size_t bytes = sizeof(float) * (2 * per + 2 * widest + 64);
  if (net->scratch_bytes < bytes) {
    cudaFree(net->d_scratch);
    net->d_scratch = nullptr;
    net->scratch_bytes = 0;
    PHX_CUDA(net->ctx, cudaMalloc(&net->d_scratch, bytes));
    net->scratch_bytes = bytes;
  }
  float* p = static_cast<float*>(net->d_scratch);
  acts.Z.assign(net->dims.size(), nullptr);
  acts.A.assign(net->dims.size(), nullptr);
  for (size_t l = 0; l < net->dims.size(); ++l) {
    acts.Z[l] = p;
    p += (size_t)B * net->dims[l];
    acts.A[l] = p;
    p += (size_t)B * net->dims[l];
  }
  *dA0 = p;
  p += widest;
  *dA1 = p;
  p += widest;
  *loss = p;
  return PHX_OK;
}

// forward of B samples X (device, B x nin); output in acts.A.back()
int forward(phx_mlp* net, int B, const float* dX, Acts& acts) {
  phx_ctx* ctx = net->ctx;
  PHX_CUDA(ctx, cudaMemcpyAsync(acts.A[0], dX, sizeof(float) * B * net->nin, cudaMemcpyDeviceToDevice, ctx->stream));
  for (int l = 0; l < net->layers; ++l) {
    const int nin = net->dims[l], nout = net->dims[l + 1];
    // Z = A W^T with W (nout x nin) row-major: B(k=i, n=o) = W[o*nin + i]
    PHX_TRY((gemm<false, true, true>(ctx, B, nout, nin, acts.A[l], nin, net->d_param + net->woff[l], nin,
                                     acts.Z[l + 1], nout, 0)));
    bias_act_kernel<<<ew_grid(ctx, (size_t)B * nout), 256, 0, ctx->stream>>>(
        acts.Z[l + 1], acts.A[l + 1], net->d_param + net->boff[l], B, nout, l + 1 < net->layers);
    PHX_CUDA(ctx, cudaGetLastError());
  }
  return PHX_OK;
}

// gradients of the mean squared error of B samples (grad accumulated into d_grad)
int backward(phx_mlp* net, int B, const float* dT, Acts& acts, float* dA0, float* dA1, float* dloss) {
  phx_ctx* ctx = net->ctx;
  const int L = net->layers;
  mse_kernel<<<std::max(1, std::min(64, (B + 255) / 256)), 256, 0, ctx->stream>>>(acts.A[L], dT, dA0, B, dloss);
  PHX_CUDA(ctx, cudaGetLastError());
  float* dZ = dA0;   // output layer has no activation: dZ = dY
  for (int l = L - 1; l >= 0; --l) {
    const int nin = net->dims[l], nout = net->dims[l + 1];
    if (l + 1 < L) {
      gelu_back_kernel<<<ew_grid(ctx, (size_t)B * nout), 256, 0, ctx->stream>>>(acts.Z[l + 1], dZ, (size_t)B * nout);
      PHX_CUDA(ctx, cudaGetLastError());
    }
    // dW (nout x nin) += dZ^T A ; db += sum_b dZ
    PHX_TRY((gemm<true, false, false>(ctx, nout, nin, B, dZ, nout, acts.A[l], nin, net->d_grad + net->woff[l], nin,
                                      1)));
    bias_grad_kernel<<<(nout + 127) / 128, 128, 0, ctx->stream>>>(dZ, net->d_grad + net->boff[l], B, nout);
    PHX_CUDA(ctx, cudaGetLastError());
    if (l > 0) {
      // dA_prev (B x nin) = dZ W, W rounded to BF16 as in the forward
      float* dprev = dZ == dA0 ? dA1 : dA0;
      PHX_TRY((gemm<false, false, true>(ctx, B, nin, nout, dZ, nout, net->d_param + net->woff[l], nin, dprev, nin,
                                        0)));
      dZ = dprev;
    }
  }
  return PHX_OK;
}

}  // namespace

// Forward pass of B samples already on the device (dX (B, nin) -> dY (B)),
// in chunks of 65536 samples, on the network's stream (screened builder).
int phx_mlp_forward_device(phx_mlp* net, long long B, const float* dX, float* dY) {
  const long long chunk = 65536;
  for (long long b0 = 0; b0 < B; b0 += chunk) {
    const int nb = (int)std::min(chunk, B - b0);
    Acts acts;
    float *dA0, *dA1, *dl;
    PHX_TRY(reserve(net, nb, acts, &dA0, &dA1, &dl));
    PHX_TRY(forward(net, nb, dX + b0 * net->nin, acts));
    PHX_CUDA(net->ctx, cudaMemcpyAsync(dY + b0, acts.A.back(), sizeof(float) * nb, cudaMemcpyDeviceToDevice,
                                       net->ctx->stream));
  }
  return PHX_OK;
}
int phx_mlp_num_inputs(const phx_mlp* net) { return net ? net->nin : 0; }
phx_ctx* phx_mlp_context(const phx_mlp* net) { return net ? net->ctx : nullptr; }

extern "C" int phx_mlp_create(phx_ctx* ctx, int nin, int hidden, int depth, const float* params, phx_mlp** out) {
  PHX_ARG(ctx, ctx && out && nin > 0 && hidden > 0 && depth >= 1, "phx_mlp_create: bad arguments");
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  phx_mlp* net = new phx_mlp;
  net->ctx = ctx;
  net->nin = nin;
  net->hidden = hidden;
  net->layers = depth + 1;
  net->dims.push_back(nin);
  for (int i = 0; i < depth; ++i) net->dims.push_back(hidden);
  net->dims.push_back(1);
  size_t o = 0;
  for (int l = 0; l < net->layers; ++l) {
    net->woff.push_back(o);
    o += (size_t)net->dims[l + 1] * net->dims[l];
    net->boff.push_back(o);
    o += net->dims[l + 1];
  }
  net->nparam = o;
  cudaError_t e = cudaMalloc(&net->d_param, sizeof(float) * o);
  if (e == cudaSuccess) e = cudaMalloc(&net->d_grad, sizeof(float) * o);
  if (e == cudaSuccess) e = cudaMalloc(&net->d_m, sizeof(float) * o);
  if (e == cudaSuccess) e = cudaMalloc(&net->d_v, sizeof(float) * o);
  if (e == cudaSuccess) e = cudaMemset(net->d_m, 0, sizeof(float) * o);
  if (e == cudaSuccess) e = cudaMemset(net->d_v, 0, sizeof(float) * o);
  if (e == cudaSuccess && params) e = cudaMemcpy(net->d_param, params, sizeof(float) * o, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_mlp_create: ") + cudaGetErrorString(e));
    phx_mlp_destroy(net);
    return PHX_ERR_CUDA;
  }
  *out = net;
  return PHX_OK;
}

extern "C" int phx_mlp_destroy(phx_mlp* net) {
  if (!net) return PHX_OK;
  cudaFree(net->d_param);
  cudaFree(net->d_grad);
  cudaFree(net->d_m);
  cudaFree(net->d_v);
  cudaFree(net->d_scratch);
  delete net;
  return PHX_OK;
}

extern "C" long long phx_mlp_num_params(const phx_mlp* net) { return net ? (long long)net->nparam : 0; }

extern "C" int phx_mlp_get_params(phx_mlp* net, float* params) {
  PHX_ARG(net ? net->ctx : nullptr, net && params, "phx_mlp_get_params: bad arguments");
  PHX_CUDA(net->ctx, cudaMemcpy(params, net->d_param, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost));
  return PHX_OK;
}

extern "C" int phx_mlp_set_params(phx_mlp* net, const float* params) {
  PHX_ARG(net ? net->ctx : nullptr, net && params, "phx_mlp_set_params: bad arguments");
  PHX_CUDA(net->ctx, cudaMemcpy(net->d_param, params, sizeof(float) * net->nparam, cudaMemcpyHostToDevice));
  return PHX_OK;
}

extern "C" int phx_mlp_infer(phx_mlp* net, int B, const float* X, float* y) {
  PHX_ARG(net ? net->ctx : nullptr, net && X && y && B >= 0, "phx_mlp_infer: bad arguments");
  phx_ctx* ctx = net->ctx;
  if (B == 0) return PHX_OK;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int chunk = 65536;
  float* dX = nullptr;
  PHX_CUDA(ctx, cudaMalloc(&dX, sizeof(float) * (size_t)std::min(B, chunk) * net->nin));
  int rc = PHX_OK;
  for (int b0 = 0; b0 < B && rc == PHX_OK; b0 += chunk) {
    const int nb = std::min(chunk, B - b0);
    Acts acts;
    float *dA0, *dA1, *dl;
    rc = reserve(net, nb, acts, &dA0, &dA1, &dl);
    if (rc != PHX_OK) break;
    if (cudaMemcpyAsync(dX, X + (size_t)b0 * net->nin, sizeof(float) * nb * net->nin, cudaMemcpyHostToDevice,
                        ctx->stream) != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, "phx_mlp_infer: copy failed");
      rc = PHX_ERR_CUDA;
      break;
    }
    rc = forward(net, nb, dX, acts);
    if (rc != PHX_OK) break;
    if (cudaMemcpyAsync(y + b0, acts.A.back(), sizeof(float) * nb, cudaMemcpyDeviceToHost, ctx->stream) != cudaSuccess ||
        cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
      phx_set_error(ctx, PHX_ERR_CUDA, "phx_mlp_infer: copy back failed");
      rc = PHX_ERR_CUDA;
    }
  }
  cudaFree(dX);
  if (rc == PHX_OK) rc = check_status(ctx);
  return rc;
}

extern "C" int phx_mlp_grad(phx_mlp* net, int B, const float* X, const float* t, float* grad, float* loss) {
  PHX_ARG(net ? net->ctx : nullptr, net && X && t && grad && B > 0, "phx_mlp_grad: bad arguments");
  phx_ctx* ctx = net->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  float *dX = nullptr, *dT = nullptr;
  PHX_CUDA(ctx, cudaMalloc(&dX, sizeof(float) * (size_t)B * net->nin));
  int rc = PHX_OK;
  if (cudaMalloc(&dT, sizeof(float) * B) != cudaSuccess) {
    cudaFree(dX);
    phx_set_error(ctx, PHX_ERR_CUDA, "phx_mlp_grad: allocation failed");
    return PHX_ERR_CUDA;
  }
  Acts acts;
  float *dA0, *dA1, *dl;
  rc = reserve(net, B, acts, &dA0, &dA1, &dl);
  if (rc == PHX_OK) {
    cudaMemcpyAsync(dX, X, sizeof(float) * (size_t)B * net->nin, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemcpyAsync(dT, t, sizeof(float) * B, cudaMemcpyHostToDevice, ctx->stream);
    cudaMemsetAsync(net->d_grad, 0, sizeof(float) * net->nparam, ctx->stream);
    cudaMemsetAsync(dl, 0, sizeof(float), ctx->stream);
    rc = forward(net, B, dX, acts);
    if (rc == PHX_OK) rc = backward(net, B, dT, acts, dA0, dA1, dl);
    if (rc == PHX_OK) {
      cudaMemcpyAsync(grad, net->d_grad, sizeof(float) * net->nparam, cudaMemcpyDeviceToHost, ctx->stream);
      if (loss) cudaMemcpyAsync(loss, dl, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
      if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        phx_set_error(ctx, PHX_ERR_CUDA, "phx_mlp_grad: stream failed");
        rc = PHX_ERR_CUDA;
      }
    }
  }
  cudaFree(dX);
  cudaFree(dT);
  if (rc == PHX_OK) rc = check_status(ctx);
  return rc;
}

extern "C" int phx_mlp_train(phx_mlp* net, int n, const float* X, const float* t, int epochs, int batch, float lr,
                             unsigned long long seed, float* loss_per_epoch) {
  PHX_ARG(net ? net->ctx : nullptr, net && X && t && n > 0 && epochs >= 0 && batch > 0,
          "phx_mlp_train: bad arguments");
  phx_ctx* ctx = net->ctx;
  PHX_CUDA(ctx, cudaSetDevice(ctx->device));
  const int nin = net->nin;
  float *dX = nullptr, *dT = nullptr, *dXb = nullptr, *dTb = nullptr;
  cudaError_t e = cudaMalloc(&dX, sizeof(float) * (size_t)n * nin);
  if (e == cudaSuccess) e = cudaMalloc(&dT, sizeof(float) * n);
  if (e == cudaSuccess) e = cudaMalloc(&dXb, sizeof(float) * (size_t)batch * nin);
  if (e == cudaSuccess) e = cudaMalloc(&dTb, sizeof(float) * batch);
  if (e == cudaSuccess) e = cudaMemcpy(dX, X, sizeof(float) * (size_t)n * nin, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(dT, t, sizeof(float) * n, cudaMemcpyHostToDevice);
  int rc = PHX_OK;
  if (e != cudaSuccess) {
    phx_set_error(ctx, PHX_ERR_CUDA, std::string("phx_mlp_train: ") + cudaGetErrorString(e));
    rc = PHX_ERR_CUDA;
  }
  std::vector<int> perm(n);
  for (int i = 0; i < n; ++i) perm[i] = i;
  unsigned long long s = seed ? seed : 0x9E3779B97F4A7C15ull;
  auto next = [&]() {  // splitmix64
    s += 0x9E3779B97F4A7C15ull;
    unsigned long long z = s;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
  };
  std::vector<float> hx((size_t)batch * nin), ht(batch);
  std::vector<float> hX(X, X + (size_t)n * nin), hT(t, t + n);
  for (int ep = 0; ep < epochs && rc == PHX_OK; ++ep) {
    for (int i = n - 1; i > 0; --i) std::swap(perm[i], perm[next() % (unsigned long long)(i + 1)]);
    double lsum = 0.0;
    int nbat = 0;
    for (int b0 = 0; b0 + batch <= n && rc == PHX_OK; b0 += batch) {
      for (int j = 0; j < batch; ++j) {
        const int i = perm[b0 + j];
        std::copy(hX.begin() + (size_t)i * nin, hX.begin() + (size_t)(i + 1) * nin, hx.begin() + (size_t)j * nin);
        ht[j] = hT[i];
      }
      Acts acts;
      float *dA0, *dA1, *dl;
      rc = reserve(net, batch, acts, &dA0, &dA1, &dl);
      if (rc != PHX_OK) break;
      cudaMemcpyAsync(dXb, hx.data(), sizeof(float) * hx.size(), cudaMemcpyHostToDevice, ctx->stream);
      cudaMemcpyAsync(dTb, ht.data(), sizeof(float) * batch, cudaMemcpyHostToDevice, ctx->stream);
      cudaMemsetAsync(net->d_grad, 0, sizeof(float) * net->nparam, ctx->stream);
      cudaMemsetAsync(dl, 0, sizeof(float), ctx->stream);
      rc = forward(net, batch, dXb, acts);
      if (rc == PHX_OK) rc = backward(net, batch, dTb, acts, dA0, dA1, dl);
      if (rc != PHX_OK) break;
      ++net->step;
      const float b1 = 0.9f, b2 = 0.999f;
      const float c1 = 1.f - powf(b1, (float)net->step), c2 = 1.f - powf(b2, (float)net->step);
      adam_kernel<<<ew_grid(ctx, net->nparam), 256, 0, ctx->stream>>>(net->d_param, net->d_grad, net->d_m, net->d_v,
                                                                       net->nparam, lr, b1, b2, 1e-8f, c1, c2);
      float l = 0.f;
      cudaMemcpyAsync(&l, dl, sizeof(float), cudaMemcpyDeviceToHost, ctx->stream);
      if (cudaStreamSynchronize(ctx->stream) != cudaSuccess) {
        phx_set_error(ctx, PHX_ERR_CUDA, "phx_mlp_train: stream failed");
        rc = PHX_ERR_CUDA;
        break;
      }
      lsum += l;
      ++nbat;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = nbat ? (float)(lsum / nbat) : 0.f;
  }
  cudaFree(dX);
  cudaFree(dT);
  cudaFree(dXb);
  cudaFree(dTb);
  if (rc == PHX_OK) rc = check_status(ctx);
  return rc;
}
