// mlp.cu - the learned planner's network: a 3-layer perceptron (in -> H ->
// H -> out, ReLU between), FP32 weights, trained on the GPU by these kernels
// (forward, backward, Adam) and run for planning in BF16 (weights and
// activations rounded to bfloat16, products accumulated in FP32).
//
// No counterpart in the reference (which has only the fixed from_bin /
// from_bin2 rules, bmpidx_create.cu:138-226); the layers are tiny (a batch of
// up to a few thousand rows of 32 features), so each kernel computes one
// output element per thread, coalesced over the batch.
//
// Parameters live in one device array, layer by layer: W1 [H x in], b1 [H],
// W2 [H x H], b2 [H], W3 [out x H], b3 [out] (row-major, W[j][i] multiplies
// input i into output j).
#include <cuda_bf16.h>
#include <math.h>
#include <string.h>
#include <vector>
#include "common.cuh"

struct mb_mlp {
  int device = 0;
  mb_mlp_config cfg{};
  uint32_t nparam = 0;
  float *p = nullptr;      // parameters
  float *g = nullptr;      // gradients
  float *m = nullptr;      // Adam first moments
  float *v = nullptr;      // Adam second moments
  uint64_t step = 0;
  // batch scratch
  uint32_t cap = 0;
  float *x = nullptr, *t = nullptr, *mk = nullptr, *h1 = nullptr, *h2 = nullptr, *y = nullptr, *dy = nullptr,
        *d2 = nullptr, *d1 = nullptr, *loss = nullptr;
  cudaStream_t st = nullptr;
};

namespace mb {
namespace {

struct Off {
  uint32_t w1, b1, w2, b2, w3, b3, n;
};
Off offsets(const mb_mlp_config &c) {
  Off o;
  o.w1 = 0;
  o.b1 = o.w1 + c.hidden * c.in;
  o.w2 = o.b1 + c.hidden;
  o.b2 = o.w2 + c.hidden * c.hidden;
  o.w3 = o.b2 + c.hidden;
  o.b3 = o.w3 + c.out * c.hidden;
  o.n = o.b3 + c.out;
  return o;
}

__device__ __forceinline__ float bf(float x) { return __bfloat162float(__float2bfloat16(x)); }

// y[r][j] = act(b[j] + sum_i W[j][i] x[r][i]); relu != 0 applies ReLU.  With
// BF16, W, b and x are rounded to bfloat16 and the products summed in FP32.
template <bool BF16>
__global__ void dense_fwd(const float *__restrict__ x, uint32_t n, uint32_t in, const float *__restrict__ W,
                          const float *__restrict__ b, uint32_t out, int relu, float *__restrict__ y) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (uint64_t)n * out) return;
  const uint32_t r = (uint32_t)(idx / out), j = (uint32_t)(idx % out);
  const float *xr = x + (uint64_t)r * in, *wj = W + (uint64_t)j * in;
  float s = BF16 ? bf(b[j]) : b[j];
  for (uint32_t i = 0; i < in; ++i) s += BF16 ? bf(wj[i]) * bf(xr[i]) : wj[i] * xr[i];
  if (relu && s < 0.f) s = 0.f;
  y[idx] = BF16 ? bf(s) : s;
}

// dy = 2 (y - t) mask / count and the masked squared error into loss[0].
__global__ void mse_grad(const float *__restrict__ y, const float *__restrict__ t, const float *__restrict__ mk,
                         uint64_t total, float inv_count, float *__restrict__ dy, float *__restrict__ loss) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  float e2 = 0.f;
  if (idx < total) {
    const float d = (y[idx] - t[idx]) * mk[idx];
    dy[idx] = 2.f * d * inv_count;
    e2 = d * d * inv_count;
  }
  for (int o = 16; o; o >>= 1) e2 += __shfl_down_sync(0xffffffffu, e2, o);
  if ((threadIdx.x & 31) == 0 && e2 != 0.f) atomicAdd(loss, e2);
}

// dW[j][i] = sum_r d[r][j] x[r][i]; db[j] = sum_r d[r][j].  One thread per
// weight (and per bias when i == in).
__global__ void dense_wgrad(const float *__restrict__ x, const float *__restrict__ d, uint32_t n, uint32_t in,
                            uint32_t out, float *__restrict__ dW, float *__restrict__ db) {
  const uint32_t idx = blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= out * (in + 1)) return;
  const uint32_t j = idx / (in + 1), i = idx % (in + 1);
  float s = 0.f;
  if (i < in)
    for (uint32_t r = 0; r < n; ++r) s += d[(uint64_t)r * out + j] * x[(uint64_t)r * in + i];
  else
    for (uint32_t r = 0; r < n; ++r) s += d[(uint64_t)r * out + j];
  if (i < in) dW[j * in + i] = s;
  else db[j] = s;
}

// dx[r][i] = (sum_j d[r][j] W[j][i]) * (h[r][i] > 0): the gradient through
// the layer into a ReLU output h.
__global__ void dense_xgrad(const float *__restrict__ d, uint32_t n, uint32_t out, const float *__restrict__ W,
                            uint32_t in, const float *__restrict__ h, float *__restrict__ dx) {
  const uint64_t idx = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (idx >= (uint64_t)n * in) return;
  const uint32_t r = (uint32_t)(idx / in), i = (uint32_t)(idx % in);
  float s = 0.f;
  for (uint32_t j = 0; j < out; ++j) s += d[(uint64_t)r * out + j] * W[(uint64_t)j * in + i];
  dx[idx] = h[idx] > 0.f ? s : 0.f;
}

// Adam (Kingma and Ba, 2015) with bias correction.
__global__ void adam_step(float *__restrict__ p, const float *__restrict__ g, float *__restrict__ m,
                          float *__restrict__ v, uint32_t n, float lr, float b1, float b2, float eps, float c1,
                          float c2) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  const float gi = g[i];
  const float mi = b1 * m[i] + (1.f - b1) * gi, vi = b2 * v[i] + (1.f - b2) * gi * gi;
  m[i] = mi;
  v[i] = vi;
  p[i] -= lr * (mi / c1) / (sqrtf(vi / c2) + eps);
}

inline unsigned blocks(uint64_t n, unsigned t = 256) { return (unsigned)((n + t - 1) / t); }

mb_status ensure(mb_mlp &M, uint32_t n) {
  if (n <= M.cap) return MB_OK;
  float **bufs[] = {&M.x, &M.t, &M.mk, &M.h1, &M.h2, &M.y, &M.dy, &M.d2, &M.d1};
  for (float **b : bufs) {
    cudaFree(*b);
    *b = nullptr;
  }
  const mb_mlp_config &c = M.cfg;
  const uint64_t sz[] = {(uint64_t)n * c.in, (uint64_t)n * c.out, (uint64_t)n * c.out, (uint64_t)n * c.hidden,
                         (uint64_t)n * c.hidden, (uint64_t)n * c.out, (uint64_t)n * c.out, (uint64_t)n * c.hidden,
                         (uint64_t)n * c.hidden};
  for (int i = 0; i < 9; ++i) MB_CUDA(cudaMalloc(bufs[i], sz[i] * 4));
  M.cap = n;
  return MB_OK;
}

// Forward pass over the n rows in M.x (activations kept for backward).
mb_status forward(mb_mlp &M, uint32_t n, bool bf16) {
  const mb_mlp_config &c = M.cfg;
  const Off o = offsets(c);
  auto fwd = bf16 ? dense_fwd<true> : dense_fwd<false>;
  fwd<<<blocks((uint64_t)n * c.hidden), 256, 0, M.st>>>(M.x, n, c.in, M.p + o.w1, M.p + o.b1, c.hidden, 1, M.h1);
  fwd<<<blocks((uint64_t)n * c.hidden), 256, 0, M.st>>>(M.h1, n, c.hidden, M.p + o.w2, M.p + o.b2, c.hidden, 1, M.h2);
  fwd<<<blocks((uint64_t)n * c.out), 256, 0, M.st>>>(M.h2, n, c.hidden, M.p + o.w3, M.p + o.b3, c.out, 0, M.y);
  MB_LAUNCH_CHECK("mlp forward");
  return MB_OK;
}

// Gradient of the masked mean squared error into M.g (after forward); the
// loss is added into M.loss (the caller zeroes it).  inv_count = 1 / the
// number of measured targets in the batch.
mb_status backward(mb_mlp &M, uint32_t n, float inv_count) {
  const mb_mlp_config &c = M.cfg;
  const Off o = offsets(c);
  const uint64_t tot = (uint64_t)n * c.out;
  mse_grad<<<blocks(tot), 256, 0, M.st>>>(M.y, M.t, M.mk, tot, inv_count, M.dy, M.loss);
  dense_wgrad<<<blocks(c.out * (c.hidden + 1)), 256, 0, M.st>>>(M.h2, M.dy, n, c.hidden, c.out, M.g + o.w3,
                                                                 M.g + o.b3);
  dense_xgrad<<<blocks((uint64_t)n * c.hidden), 256, 0, M.st>>>(M.dy, n, c.out, M.p + o.w3, c.hidden, M.h2, M.d2);
  dense_wgrad<<<blocks(c.hidden * (c.hidden + 1)), 256, 0, M.st>>>(M.h1, M.d2, n, c.hidden, c.hidden, M.g + o.w2,
                                                                    M.g + o.b2);
  dense_xgrad<<<blocks((uint64_t)n * c.hidden), 256, 0, M.st>>>(M.d2, n, c.hidden, M.p + o.w2, c.hidden, M.h1, M.d1);
  dense_wgrad<<<blocks(c.hidden * (c.in + 1)), 256, 0, M.st>>>(M.x, M.d1, n, c.in, c.hidden, M.g + o.w1,
                                                                M.g + o.b1);
  MB_LAUNCH_CHECK("mlp backward");
  return MB_OK;
}

float inv_count(const float *mask, uint64_t n) {
  uint64_t c = 0;
  for (uint64_t i = 0; i < n; ++i) c += mask[i] != 0.f;
  return c ? (float)(1.0 / (double)c) : 0.f;
}

// Rows idx[0..n) of the resident training set into the batch buffers.
__global__ void gather_rows(const float *__restrict__ X, const float *__restrict__ T, const float *__restrict__ MK,
                            const uint32_t *__restrict__ idx, uint32_t n, uint32_t in, uint32_t out,
                            float *__restrict__ x, float *__restrict__ t, float *__restrict__ mk) {
  const uint32_t r = blockIdx.x;
  if (r >= n) return;
  const uint64_t k = idx[r];
  for (uint32_t i = threadIdx.x; i < in; i += blockDim.x) x[(uint64_t)r * in + i] = X[k * in + i];
  for (uint32_t i = threadIdx.x; i < out; i += blockDim.x) {
    t[(uint64_t)r * out + i] = T[k * out + i];
    mk[(uint64_t)r * out + i] = MK[k * out + i];
  }
}

mb_status upload(mb_mlp &M, const float *x, const float *t, const float *mk, uint32_t n) {
  MB_CHECK(ensure(M, n));
  const mb_mlp_config &c = M.cfg;
  MB_CUDA(cudaMemcpyAsync(M.x, x, (size_t)n * c.in * 4, cudaMemcpyHostToDevice, M.st));
  if (t) MB_CUDA(cudaMemcpyAsync(M.t, t, (size_t)n * c.out * 4, cudaMemcpyHostToDevice, M.st));
  if (mk) MB_CUDA(cudaMemcpyAsync(M.mk, mk, (size_t)n * c.out * 4, cudaMemcpyHostToDevice, M.st));
  return MB_OK;
}

// Deterministic initial weights (He-uniform from a counter-based hash).
float init_weight(uint64_t seed, uint32_t i, uint32_t fan_in) {
  uint64_t z = seed * 0x9e3779b97f4a7c15ull + i + 1;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
  z ^= z >> 31;
  const double u = (double)(z >> 11) / 9007199254740992.0;  // [0, 1)
  const double lim = sqrt(6.0 / (double)fan_in);
  return (float)((2.0 * u - 1.0) * lim);
}

}  // namespace
}  // namespace mb

namespace mb {
bool mlp_shape(const mb_mlp *m, uint32_t *in, uint32_t *out) {
  if (!m) return false;
  *in = m->cfg.in, *out = m->cfg.out;
  return true;
}
}  // namespace mb

using namespace mb;

extern "C" mb_status mb_mlp_create(int device, const mb_mlp_config *cfg, mb_mlp **out) {
  if (!cfg || !out) return fail(MB_ERR_INVALID, "mb_mlp_create: NULL argument");
  *out = nullptr;
  if (cfg->in == 0 || cfg->hidden == 0 || cfg->out == 0 || cfg->in > 4096 || cfg->hidden > 4096 || cfg->out > 4096)
    return fail(MB_ERR_INVALID, "mb_mlp_create: sizes %u/%u/%u", cfg->in, cfg->hidden, cfg->out);
  MB_CUDA(cudaSetDevice(device));
  mb_mlp *M = new (std::nothrow) mb_mlp();
  if (!M) return fail(MB_ERR_OOM, "mb_mlp_create: host allocation");
  M->device = device;
  M->cfg = *cfg;
  const Off o = offsets(*cfg);
  M->nparam = o.n;
  std::vector<float> h(o.n, 0.f);
  for (uint32_t i = 0; i < cfg->hidden * cfg->in; ++i) h[o.w1 + i] = init_weight(cfg->seed, o.w1 + i, cfg->in);
  for (uint32_t i = 0; i < cfg->hidden * cfg->hidden; ++i) h[o.w2 + i] = init_weight(cfg->seed, o.w2 + i, cfg->hidden);
  for (uint32_t i = 0; i < cfg->out * cfg->hidden; ++i) h[o.w3 + i] = init_weight(cfg->seed, o.w3 + i, cfg->hidden);
  cudaError_t r = cudaStreamCreateWithFlags(&M->st, cudaStreamNonBlocking);
  float **arr[] = {&M->p, &M->g, &M->m, &M->v};
  for (float **a : arr)
    if (r == cudaSuccess) r = cudaMalloc(a, (size_t)o.n * 4);
  if (r == cudaSuccess) r = cudaMalloc(&M->loss, 4);
  if (r == cudaSuccess) r = cudaMemcpy(M->p, h.data(), (size_t)o.n * 4, cudaMemcpyHostToDevice);
  if (r == cudaSuccess) r = cudaMemset(M->m, 0, (size_t)o.n * 4);
  if (r == cudaSuccess) r = cudaMemset(M->v, 0, (size_t)o.n * 4);
  if (r == cudaSuccess) r = cudaMemset(M->g, 0, (size_t)o.n * 4);
  if (r != cudaSuccess) {
    mb_mlp_destroy(M);
    return cuda_fail(r, "mb_mlp_create");
  }
  *out = M;
  return MB_OK;
}

extern "C" mb_status mb_mlp_destroy(mb_mlp *M) {
  if (!M) return MB_OK;
  cudaSetDevice(M->device);
  if (M->st) cudaStreamSynchronize(M->st);
  float *bufs[] = {M->p, M->g, M->m, M->v, M->x, M->t, M->mk, M->h1, M->h2, M->y, M->dy, M->d2, M->d1, M->loss};
  for (float *b : bufs) cudaFree(b);
  if (M->st) cudaStreamDestroy(M->st);
  delete M;
  return MB_OK;
}

extern "C" uint32_t mb_mlp_nparams(const mb_mlp *M) { return M ? M->nparam : 0; }

extern "C" mb_status mb_mlp_get_params(mb_mlp *M, float *host) {
  if (!M || !host) return fail(MB_ERR_INVALID, "mb_mlp_get_params: NULL argument");
  MB_CUDA(cudaSetDevice(M->device));
  MB_CUDA(cudaMemcpyAsync(host, M->p, (size_t)M->nparam * 4, cudaMemcpyDeviceToHost, M->st));
  MB_CUDA(cudaStreamSynchronize(M->st));
  return MB_OK;
}

extern "C" mb_status mb_mlp_set_params(mb_mlp *M, const float *host) {
  if (!M || !host) return fail(MB_ERR_INVALID, "mb_mlp_set_params: NULL argument");
  MB_CUDA(cudaSetDevice(M->device));
  MB_CUDA(cudaMemcpyAsync(M->p, host, (size_t)M->nparam * 4, cudaMemcpyHostToDevice, M->st));
  MB_CUDA(cudaMemsetAsync(M->m, 0, (size_t)M->nparam * 4, M->st));
  MB_CUDA(cudaMemsetAsync(M->v, 0, (size_t)M->nparam * 4, M->st));
  MB_CUDA(cudaStreamSynchronize(M->st));
  M->step = 0;
  return MB_OK;
}

extern "C" mb_status mb_mlp_forward(mb_mlp *M, const float *x_host, uint32_t n, int bf16, float *y_host) {
  if (!M || (!x_host && n) || (!y_host && n)) return fail(MB_ERR_INVALID, "mb_mlp_forward: NULL argument");
  if (n == 0) return MB_OK;
  MB_CUDA(cudaSetDevice(M->device));
  MB_CHECK(upload(*M, x_host, nullptr, nullptr, n));
  MB_CHECK(forward(*M, n, bf16 != 0));
  MB_CUDA(cudaMemcpyAsync(y_host, M->y, (size_t)n * M->cfg.out * 4, cudaMemcpyDeviceToHost, M->st));
  MB_CUDA(cudaStreamSynchronize(M->st));
  return MB_OK;
}

extern "C" mb_status mb_mlp_gradients(mb_mlp *M, const float *x, const float *t, const float *mask, uint32_t n,
                                      float *grad_host, float *loss) {
  if (!M || !x || !t || !mask || !grad_host || n == 0) return fail(MB_ERR_INVALID, "mb_mlp_gradients: bad argument");
  MB_CUDA(cudaSetDevice(M->device));
  MB_CHECK(upload(*M, x, t, mask, n));
  MB_CHECK(forward(*M, n, false));
  MB_CUDA(cudaMemsetAsync(M->loss, 0, 4, M->st));
  MB_CHECK(backward(*M, n, inv_count(mask, (uint64_t)n * M->cfg.out)));
  MB_CUDA(cudaMemcpyAsync(grad_host, M->g, (size_t)M->nparam * 4, cudaMemcpyDeviceToHost, M->st));
  float l = 0;
  MB_CUDA(cudaMemcpyAsync(&l, M->loss, 4, cudaMemcpyDeviceToHost, M->st));
  MB_CUDA(cudaStreamSynchronize(M->st));
  if (loss) *loss = l;
  return MB_OK;
}

extern "C" mb_status mb_mlp_train(mb_mlp *M, const float *x, const float *t, const float *mask, uint32_t n,
                                  const mb_mlp_train_opts *o, float *final_loss) {
  NvtxRange nvtx_("mb_mlp_train");
  if (!M || !x || !t || !mask || !o || n == 0) return fail(MB_ERR_INVALID, "mb_mlp_train: bad argument");
  if (o->batch == 0 || o->epochs == 0) return fail(MB_ERR_INVALID, "mb_mlp_train: batch and epochs must be > 0");
  MB_CUDA(cudaSetDevice(M->device));
  const mb_mlp_config &c = M->cfg;
  const uint32_t B = o->batch < n ? o->batch : n;
  const uint32_t nb = n / B;  // whole batches per epoch (the remainder rotates with the shuffle)
  MB_CHECK(ensure(*M, B));
  // the training set stays resident for the whole run (freed on every exit)
  float *X = nullptr, *T = nullptr, *MK = nullptr;
  uint32_t *perm_d = nullptr;
  struct Frees {
    cudaStream_t st;
    void **p[4];
    ~Frees() {
      cudaStreamSynchronize(st);
      for (void **q : p) cudaFree(*q);
    }
  } frees{M->st, {(void **)&X, (void **)&T, (void **)&MK, (void **)&perm_d}};
  cudaError_t r = cudaMalloc(&X, (size_t)n * c.in * 4);
  if (r == cudaSuccess) r = cudaMalloc(&T, (size_t)n * c.out * 4);
  if (r == cudaSuccess) r = cudaMalloc(&MK, (size_t)n * c.out * 4);
  if (r == cudaSuccess) r = cudaMalloc(&perm_d, (size_t)n * 4);
  if (r == cudaSuccess) r = cudaMemcpyAsync(X, x, (size_t)n * c.in * 4, cudaMemcpyHostToDevice, M->st);
  if (r == cudaSuccess) r = cudaMemcpyAsync(T, t, (size_t)n * c.out * 4, cudaMemcpyHostToDevice, M->st);
  if (r == cudaSuccess) r = cudaMemcpyAsync(MK, mask, (size_t)n * c.out * 4, cudaMemcpyHostToDevice, M->st);
  std::vector<uint32_t> perm(n);
  std::vector<float> inv(nb);
  for (uint32_t i = 0; i < n; ++i) perm[i] = i;
  uint64_t rng = o->seed * 0x2545f4914f6cdd1dull + 1;
  float last = 0;
  for (uint32_t ep = 0; ep < o->epochs && r == cudaSuccess; ++ep) {
    for (uint32_t i = n - 1; i > 0; --i) {  // Fisher-Yates with a 64-bit LCG
      rng = rng * 6364136223846793005ull + 1442695040888963407ull;
      const uint32_t j = (uint32_t)((rng >> 33) % (i + 1));
      std::swap(perm[i], perm[j]);
    }
    for (uint32_t b = 0; b < nb; ++b) {  // measured targets per batch, for the means
      uint64_t cnt = 0;
      for (uint32_t k = b * B; k < (b + 1) * B; ++k)
        for (uint32_t i = 0; i < c.out; ++i) cnt += mask[(size_t)perm[k] * c.out + i] != 0.f;
      inv[b] = cnt ? (float)(1.0 / (double)cnt) : 0.f;
    }
    // the previous epoch's kernels read perm_d: wait before overwriting it
    r = cudaStreamSynchronize(M->st);
    if (r == cudaSuccess) r = cudaMemcpy(perm_d, perm.data(), (size_t)n * 4, cudaMemcpyHostToDevice);
    if (r == cudaSuccess) r = cudaMemsetAsync(M->loss, 0, 4, M->st);
    if (r != cudaSuccess) break;
    for (uint32_t b = 0; b < nb; ++b) {
      gather_rows<<<B, 64, 0, M->st>>>(X, T, MK, perm_d + (size_t)b * B, B, c.in, c.out, M->x, M->t, M->mk);
      MB_CHECK(forward(*M, B, false));
      MB_CHECK(backward(*M, B, inv[b]));
      ++M->step;
      const float c1 = 1.f - powf(o->beta1, (float)M->step), c2 = 1.f - powf(o->beta2, (float)M->step);
      adam_step<<<blocks(M->nparam), 256, 0, M->st>>>(M->p, M->g, M->m, M->v, M->nparam, o->lr, o->beta1, o->beta2,
                                                      1e-8f, c1, c2);
      MB_LAUNCH_CHECK("mlp train step");
    }
    float l = 0;
    r = cudaMemcpyAsync(&l, M->loss, 4, cudaMemcpyDeviceToHost, M->st);
    if (r == cudaSuccess) r = cudaStreamSynchronize(M->st);
    last = nb ? l / (float)nb : 0.f;
  }
  if (r != cudaSuccess) return cuda_fail(r, "mb_mlp_train");
  if (final_loss) *final_loss = last;
  return MB_OK;
}
