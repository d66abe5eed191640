// Small fully connected network of the learned parameter chooser, trained and
// evaluated on the GPU with these kernels (no library GEMM).
//
// Shape: n_in -> H -> H -> H -> n_out, tanh hidden activations, linear output,
// FP32.  Parameters are one flat FP32 array: for each layer l, W_l (out x in,
// row-major) then b_l (out).  Loss: mean over samples and outputs of the
// squared error.  Optimiser: Adam (beta1 0.9, beta2 0.999, eps 1e-8).
//
// Kernels (all tiny; the whole net is < 10k parameters):
//  forward     one thread per (sample, unit) of a layer, activations kept for
//              the backward pass;
//  backward    output delta, then per layer: grad_W = delta^T a_prev (one
//              thread per weight, loop over the batch), grad_b = sum(delta),
//              delta_prev = (W^T delta) * (1 - a_prev^2);
//  adam        one thread per parameter.
#include <algorithm>
#include <cmath>
#include <random>
#include <vector>

#include "common.cuh"

namespace tb {

struct Mlp {
  int nin = 0, H = 0, nlayers = 0, nout = 0;  // nlayers = hidden layers
  std::vector<int> dims;                      // nin, H, ..., H, nout
  std::vector<size_t> woff, boff;             // per layer offsets into params
  size_t nparams = 0;
  DBuf<float> params, grads, m, v;
  DBuf<float> acts;    // activations: sum over layers of batch x dims[l]
  DBuf<float> deltas;  // same size
  DBuf<float> X, Y;    // batch inputs / targets
  DBuf<float> loss;    // per-sample squared error sums
  int64_t step = 0;
};

namespace {

constexpr int kT = 256;

__global__ void layer_forward(const float *__restrict__ in, int din, const float *__restrict__ W,
                              const float *__restrict__ b, float *__restrict__ out, int dout,
                              int64_t nb, int act_tanh) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nb * dout;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = idx / dout;
    const int o = (int)(idx % dout);
    const float *a = in + s * din;
    const float *w = W + (size_t)o * din;
    float z = b[o];
    for (int i = 0; i < din; i++) z = fmaf(w[i], a[i], z);
    out[idx] = act_tanh ? tanhf(z) : z;
  }
}

// delta_out = 2 (y - t) / (nb * nout); per-sample squared error to loss[s]
__global__ void output_delta(const float *__restrict__ y, const float *__restrict__ t, int nout,
                             int64_t nb, float *__restrict__ delta, float *__restrict__ loss) {
  for (int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; s < nb;
       s += (int64_t)gridDim.x * blockDim.x) {
    float l = 0.f;
    for (int o = 0; o < nout; o++) {
      const float d = y[s * nout + o] - t[s * nout + o];
      l += d * d;
      delta[s * nout + o] = 2.f * d / (float)(nb * nout);
    }
    loss[s] = l;
  }
}

// grad_W[o][i] = sum_s delta[s][o] * a_prev[s][i];  grad_b[o] = sum_s delta[s][o]
__global__ void layer_grad(const float *__restrict__ delta, int dout,
                           const float *__restrict__ aprev, int din, int64_t nb,
                           float *__restrict__ gW, float *__restrict__ gb) {
  const int64_t nw = (int64_t)dout * din;
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nw + dout;
       idx += (int64_t)gridDim.x * blockDim.x) {
    if (idx < nw) {
      const int o = (int)(idx / din), i = (int)(idx % din);
      float g = 0.f;
      for (int64_t s = 0; s < nb; s++) g = fmaf(delta[s * dout + o], aprev[s * din + i], g);
      gW[idx] = g;
    } else {
      const int o = (int)(idx - nw);
      float g = 0.f;
      for (int64_t s = 0; s < nb; s++) g += delta[s * dout + o];
      gb[o] = g;
    }
  }
}

// delta_prev[s][i] = (sum_o W[o][i] delta[s][o]) * (1 - a_prev^2)
__global__ void layer_backprop(const float *__restrict__ delta, int dout,
                               const float *__restrict__ W, const float *__restrict__ aprev,
                               int din, int64_t nb, float *__restrict__ dprev) {
  for (int64_t idx = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; idx < nb * din;
       idx += (int64_t)gridDim.x * blockDim.x) {
    const int64_t s = idx / din;
    const int i = (int)(idx % din);
    float g = 0.f;
    for (int o = 0; o < dout; o++) g = fmaf(W[(size_t)o * din + i], delta[s * dout + o], g);
    const float a = aprev[idx];
    dprev[idx] = g * (1.f - a * a);
  }
}

__global__ void adam_step(float *__restrict__ p, const float *__restrict__ g,
                          float *__restrict__ m, float *__restrict__ v, int64_t n, float lr,
                          float bc1, float bc2) {
  for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const float gi = g[i];
    const float mi = 0.9f * m[i] + 0.1f * gi;
    const float vi = 0.999f * v[i] + 0.001f * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] -= lr * (mi / bc1) / (sqrtf(vi / bc2) + 1e-8f);
  }
}

int grid(int64_t n) { return grid_for(n, kT, 148 * 8); }

size_t act_offset(const Mlp &N, int layer, int64_t nb) {
  size_t o = 0;
  for (int l = 0; l < layer; l++) o += (size_t)nb * N.dims[l];
  return o;
}

int forward(tapas_b200_ctx *ctx, Mlp &N, int64_t nb) {
  cudaStream_t s = ctx->stream;
  const int L = (int)N.dims.size() - 1;
  // layer 0 activations = inputs
  TB_CUDA(ctx, cudaMemcpyAsync(N.acts.p, N.X.p, sizeof(float) * nb * N.dims[0],
                               cudaMemcpyDeviceToDevice, s));
  for (int l = 0; l < L; l++) {
    float *in = N.acts.p + act_offset(N, l, nb);
    float *out = N.acts.p + act_offset(N, l + 1, nb);
    layer_forward<<<grid(nb * N.dims[l + 1]), kT, 0, s>>>(
        in, N.dims[l], N.params.p + N.woff[l], N.params.p + N.boff[l], out, N.dims[l + 1], nb,
        l + 1 < L ? 1 : 0);
    TB_LAUNCH_CHECK(ctx);
  }
  return TAPAS_B200_OK;
}

int backward(tapas_b200_ctx *ctx, Mlp &N, int64_t nb) {
  cudaStream_t s = ctx->stream;
  const int L = (int)N.dims.size() - 1;
  float *yout = N.acts.p + act_offset(N, L, nb);
  float *dout = N.deltas.p + act_offset(N, L, nb);
  output_delta<<<grid(nb), kT, 0, s>>>(yout, N.Y.p, N.nout, nb, dout, N.loss.p);
  TB_LAUNCH_CHECK(ctx);
  for (int l = L - 1; l >= 0; l--) {
    float *d = N.deltas.p + act_offset(N, l + 1, nb);
    float *aprev = N.acts.p + act_offset(N, l, nb);
    layer_grad<<<grid((int64_t)N.dims[l + 1] * N.dims[l] + N.dims[l + 1]), kT, 0, s>>>(
        d, N.dims[l + 1], aprev, N.dims[l], nb, N.grads.p + N.woff[l], N.grads.p + N.boff[l]);
    TB_LAUNCH_CHECK(ctx);
    if (l > 0) {
      layer_backprop<<<grid(nb * N.dims[l]), kT, 0, s>>>(
          d, N.dims[l + 1], N.params.p + N.woff[l], aprev, N.dims[l], nb,
          N.deltas.p + act_offset(N, l, nb));
      TB_LAUNCH_CHECK(ctx);
    }
  }
  return TAPAS_B200_OK;
}

int ensure_batch(tapas_b200_ctx *ctx, Mlp &N, int64_t nb) {
  cudaStream_t s = ctx->stream;
  size_t tot = 0;
  for (int d : N.dims) tot += (size_t)nb * d;
  TB_CUDA(ctx, N.acts.ensure(tot, s));
  TB_CUDA(ctx, N.deltas.ensure(tot, s));
  TB_CUDA(ctx, N.X.ensure((size_t)nb * N.nin, s));
  TB_CUDA(ctx, N.Y.ensure((size_t)nb * N.nout, s));
  TB_CUDA(ctx, N.loss.ensure((size_t)nb, s));
  return TAPAS_B200_OK;
}

Mlp *get(tapas_b200_ctx *ctx) { return ctx->mlp; }

}  // namespace

void mlp_release(tapas_b200_ctx *ctx) {
  if (!ctx->mlp) return;
  Mlp *N = ctx->mlp;
  N->params.release(); N->grads.release(); N->m.release(); N->v.release();
  N->acts.release(); N->deltas.release(); N->X.release(); N->Y.release(); N->loss.release();
  delete N;
  ctx->mlp = nullptr;
}

}  // namespace tb

using namespace tb;

extern "C" {

int tapas_b200_mlp_create(tapas_b200_ctx *ctx, int n_in, int n_hidden, int n_layers, int n_out,
                          uint64_t seed) {
  if (!ctx || n_in < 1 || n_hidden < 1 || n_layers < 1 || n_out < 1 || n_in > 4096 ||
      n_hidden > 4096 || n_layers > 16 || n_out > 4096) {
    set_error(ctx, "mlp_create: bad shape");
    return TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaSetDevice(ctx->device));
  mlp_release(ctx);
  Mlp *N = new Mlp();
  N->nin = n_in; N->H = n_hidden; N->nlayers = n_layers; N->nout = n_out;
  N->dims.push_back(n_in);
  for (int l = 0; l < n_layers; l++) N->dims.push_back(n_hidden);
  N->dims.push_back(n_out);
  size_t off = 0;
  for (size_t l = 0; l + 1 < N->dims.size(); l++) {
    N->woff.push_back(off);
    off += (size_t)N->dims[l] * N->dims[l + 1];
    N->boff.push_back(off);
    off += (size_t)N->dims[l + 1];
  }
  N->nparams = off;
  ctx->mlp = N;
  cudaStream_t s = ctx->stream;
  TB_CUDA(ctx, N->params.ensure(off, s));
  TB_CUDA(ctx, N->grads.ensure(off, s));
  TB_CUDA(ctx, N->m.ensure(off, s));
  TB_CUDA(ctx, N->v.ensure(off, s));
  // Xavier-uniform weights from a seeded host RNG, zero biases.
  std::vector<float> h(off, 0.f);
  std::mt19937_64 rng(seed);
  for (size_t l = 0; l + 1 < N->dims.size(); l++) {
    const int din = N->dims[l], dout = N->dims[l + 1];
    const float a = std::sqrt(6.f / (float)(din + dout));
    std::uniform_real_distribution<float> U(-a, a);
    for (size_t i = 0; i < (size_t)din * dout; i++) h[N->woff[l] + i] = U(rng);
  }
  TB_CUDA(ctx, cudaMemcpyAsync(N->params.p, h.data(), sizeof(float) * off,
                               cudaMemcpyHostToDevice, s));
  TB_CUDA(ctx, cudaMemsetAsync(N->m.p, 0, sizeof(float) * off, s));
  TB_CUDA(ctx, cudaMemsetAsync(N->v.p, 0, sizeof(float) * off, s));
  TB_CUDA(ctx, cudaStreamSynchronize(s));
  N->step = 0;
  return TAPAS_B200_OK;
}

int64_t tapas_b200_mlp_num_params(tapas_b200_ctx *ctx) {
  return (ctx && ctx->mlp) ? (int64_t)ctx->mlp->nparams : -1;
}

int tapas_b200_mlp_set_params(tapas_b200_ctx *ctx, const float *params) {
  if (!ctx || !ctx->mlp || !params) {
    set_error(ctx, "mlp_set_params: no network");
    return TAPAS_B200_ERR_STATE;
  }
  Mlp *N = ctx->mlp;
  TB_CUDA(ctx, cudaMemcpyAsync(N->params.p, params, sizeof(float) * N->nparams,
                               cudaMemcpyHostToDevice, ctx->stream));
  TB_CUDA(ctx, cudaMemsetAsync(N->m.p, 0, sizeof(float) * N->nparams, ctx->stream));
  TB_CUDA(ctx, cudaMemsetAsync(N->v.p, 0, sizeof(float) * N->nparams, ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  N->step = 0;
  return TAPAS_B200_OK;
}

int tapas_b200_mlp_get_params(tapas_b200_ctx *ctx, float *params) {
  if (!ctx || !ctx->mlp || !params) {
    set_error(ctx, "mlp_get_params: no network");
    return TAPAS_B200_ERR_STATE;
  }
  TB_CUDA(ctx, cudaMemcpyAsync(params, ctx->mlp->params.p, sizeof(float) * ctx->mlp->nparams,
                               cudaMemcpyDeviceToHost, ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TAPAS_B200_OK;
}

int tapas_b200_mlp_forward(tapas_b200_ctx *ctx, const float *X, int64_t n, float *Y) {
  if (!ctx || !ctx->mlp || !X || !Y || n <= 0) {
    set_error(ctx, "mlp_forward: no network or bad arguments");
    return TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaSetDevice(ctx->device));
  Mlp &N = *ctx->mlp;
  TB_TRY(ensure_batch(ctx, N, n));
  TB_CUDA(ctx, cudaMemcpyAsync(N.X.p, X, sizeof(float) * n * N.nin, cudaMemcpyHostToDevice,
                               ctx->stream));
  TB_TRY(forward(ctx, N, n));
  const int L = (int)N.dims.size() - 1;
  TB_CUDA(ctx, cudaMemcpyAsync(Y, N.acts.p + act_offset(N, L, n), sizeof(float) * n * N.nout,
                               cudaMemcpyDeviceToHost, ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  return TAPAS_B200_OK;
}

int tapas_b200_mlp_gradients(tapas_b200_ctx *ctx, const float *X, const float *Y, int64_t n,
                             float *grads, float *loss) {
  if (!ctx || !ctx->mlp || !X || !Y || n <= 0) {
    set_error(ctx, "mlp_gradients: no network or bad arguments");
    return TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaSetDevice(ctx->device));
  Mlp &N = *ctx->mlp;
  TB_TRY(ensure_batch(ctx, N, n));
  TB_CUDA(ctx, cudaMemcpyAsync(N.X.p, X, sizeof(float) * n * N.nin, cudaMemcpyHostToDevice,
                               ctx->stream));
  TB_CUDA(ctx, cudaMemcpyAsync(N.Y.p, Y, sizeof(float) * n * N.nout, cudaMemcpyHostToDevice,
                               ctx->stream));
  TB_TRY(forward(ctx, N, n));
  TB_TRY(backward(ctx, N, n));
  if (grads)
    TB_CUDA(ctx, cudaMemcpyAsync(grads, N.grads.p, sizeof(float) * N.nparams,
                                 cudaMemcpyDeviceToHost, ctx->stream));
  std::vector<float> l(n);
  TB_CUDA(ctx, cudaMemcpyAsync(l.data(), N.loss.p, sizeof(float) * n, cudaMemcpyDeviceToHost,
                               ctx->stream));
  TB_CUDA(ctx, cudaStreamSynchronize(ctx->stream));
  if (loss) {
    double t = 0;
    for (float v : l) t += v;
    *loss = (float)(t / (double)(n * N.nout));
  }
  return TAPAS_B200_OK;
}

int tapas_b200_mlp_train(tapas_b200_ctx *ctx, const float *X, const float *Y, int64_t n,
                         int epochs, int batch, float lr, uint64_t seed, float *loss_per_epoch) {
  if (!ctx || !ctx->mlp || !X || !Y || n <= 0 || epochs < 1 || batch < 1 || !(lr > 0)) {
    set_error(ctx, "mlp_train: no network or bad arguments");
    return TAPAS_B200_ERR_ARG;
  }
  TB_CUDA(ctx, cudaSetDevice(ctx->device));
  Mlp &N = *ctx->mlp;
  const int64_t nb = std::min<int64_t>(batch, n);
  TB_TRY(ensure_batch(ctx, N, nb));
  cudaStream_t s = ctx->stream;
  std::vector<int64_t> perm(n);
  for (int64_t i = 0; i < n; i++) perm[i] = i;
  std::mt19937_64 rng(seed);
  std::vector<float> bx((size_t)nb * N.nin), by((size_t)nb * N.nout), lb(nb);
  for (int ep = 0; ep < epochs; ep++) {
    std::shuffle(perm.begin(), perm.end(), rng);
    double eloss = 0;
    int64_t seen = 0;
    for (int64_t start = 0; start + nb <= n; start += nb) {
      for (int64_t k = 0; k < nb; k++) {
        const int64_t r = perm[start + k];
        for (int i = 0; i < N.nin; i++) bx[k * N.nin + i] = X[r * N.nin + i];
        for (int o = 0; o < N.nout; o++) by[k * N.nout + o] = Y[r * N.nout + o];
      }
      TB_CUDA(ctx, cudaMemcpyAsync(N.X.p, bx.data(), sizeof(float) * bx.size(),
                                   cudaMemcpyHostToDevice, s));
      TB_CUDA(ctx, cudaMemcpyAsync(N.Y.p, by.data(), sizeof(float) * by.size(),
                                   cudaMemcpyHostToDevice, s));
      TB_TRY(forward(ctx, N, nb));
      TB_TRY(backward(ctx, N, nb));
      N.step++;
      const float bc1 = 1.f - std::pow(0.9f, (float)N.step);
      const float bc2 = 1.f - std::pow(0.999f, (float)N.step);
      adam_step<<<grid((int64_t)N.nparams), kT, 0, s>>>(N.params.p, N.grads.p, N.m.p, N.v.p,
                                                        (int64_t)N.nparams, lr, bc1, bc2);
      TB_LAUNCH_CHECK(ctx);
      TB_CUDA(ctx, cudaMemcpyAsync(lb.data(), N.loss.p, sizeof(float) * nb,
                                   cudaMemcpyDeviceToHost, s));
      TB_CUDA(ctx, cudaStreamSynchronize(s));
      for (float v : lb) eloss += v;
      seen += nb;
    }
    if (loss_per_epoch) loss_per_epoch[ep] = (float)(eloss / (double)(seen * N.nout));
  }
  return TAPAS_B200_OK;
}

}  // extern "C"
