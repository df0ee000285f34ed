// mlp.cu -- the learned variant selector's network, trained and run on the
// GPU by the kernels below (no counterpart in the reference).
//
// MLP 16 -> 64 -> 64 -> K (ReLU, ReLU, logits), K = SPARSEP_NVARIANTS batch
// variants.  Weights are BF16 (round-to-nearest-even copies of FP32 master
// weights); every product is accumulated in FP32.  Parameters are one flat
// array: W1[64][16], b1[64], W2[64][64], b2[64], W3[K][64], b3[K].
//
// Training objective, per sample s (one matrix with its right-hand-side
// count), over the variants c that apply to it (t[s][c] > 0, the measured
// time): p = softmax(z) restricted to those c, regret r_c = t_c / min_c t_c - 1,
// soft target q = softmax(-r / tau) over the same c,
//   L_s = w_s * ( sum_c p_c r_c  +  lambda * sum_c -q_c log p_c ),
//   w_s = (min_c t_c * wscale)^alpha   (wscale = 1 / mean of min_c t_c),
// i.e. the expected relative slowdown of a pick drawn from p, plus a
// cross-entropy toward the near-best variants that keeps the gradient alive
// once p is sharp and leaves p's top probability meaningful as a confidence;
// alpha weighs matrices by their share of run time (0: all alike).  The loss
// is the mean over samples and
//   dL/dz_c = w_s ( p_c (r_c - sum_c' p_c' r_c') + lambda (p_c - q_c) ) / n.
//
// One CTA of 64 threads takes 64 samples, one thread per sample for the
// forward and backward passes (activations in shared memory, padded rows);
// then the CTA's threads split the parameters and each sums its parameters'
// gradient over the CTA's samples in sample order into a per-CTA slot.  A
// second kernel adds the slots in CTA order, so gradients are bit-identical
// from run to run.
#include <cuda_bf16.h>

#include <cstdio>
#include <new>

#include "fault.hpp"
#include "internal.hpp"
#include "sparsep.h"

namespace sparsep {
namespace mlp {

constexpr int F = SPARSEP_NFEATURES;
constexpr int H = 64;
constexpr int K = SPARSEP_NVARIANTS;
constexpr int OW1 = 0, OB1 = OW1 + H * F, OW2 = OB1 + H, OB2 = OW2 + H * H, OW3 = OB2 + H, OB3 = OW3 + K * H;
constexpr int NP = OB3 + K;
constexpr int S = 64;       // samples (threads) per CTA
constexpr int LD = S + 1;   // activation row stride (conflict-free across rows)
constexpr int ACT_ROWS = F + H + H + K + H + H;
constexpr size_t SMEM = sizeof(float) * ((size_t)NP + (size_t)ACT_ROWS * LD + S);

struct Acts {
  float *w, *x, *h1, *h2, *dz, *dh2, *dh1, *red;
};

__device__ __forceinline__ Acts carve(float *sm) {
  Acts a;
  a.w = sm;
  a.x = a.w + NP;
  a.h1 = a.x + F * LD;
  a.h2 = a.h1 + H * LD;
  a.dz = a.h2 + H * LD;
  a.dh2 = a.dz + K * LD;
  a.dh1 = a.dh2 + H * LD;
  a.red = a.dh1 + H * LD;
  return a;
}

template <bool GRAD>
__global__ void __launch_bounds__(S) fwd_bwd(const __nv_bfloat16 *__restrict__ wb, const float *__restrict__ xin,
                                             const float *__restrict__ tin, uint32_t n, float wscale, float alpha,
                                             float lambda, float tau, float *__restrict__ logits,
                                             float *__restrict__ gpart, float *__restrict__ lpart) {
  extern __shared__ float sm[];
  const Acts a = carve(sm);
  const int tid = threadIdx.x;
  const uint32_t s = blockIdx.x * S + tid;
  const bool valid = s < n;
  for (int p = tid; p < NP; p += S) a.w[p] = __bfloat162float(wb[p]);
  for (int f = 0; f < F; ++f) a.x[f * LD + tid] = valid ? xin[(size_t)s * F + f] : 0.f;
  __syncthreads();

  // forward
  for (int j = 0; j < H; ++j) {
    float acc = a.w[OB1 + j];
    for (int f = 0; f < F; ++f) acc += a.w[OW1 + j * F + f] * a.x[f * LD + tid];
    a.h1[j * LD + tid] = fmaxf(acc, 0.f);
  }
  for (int j = 0; j < H; ++j) {
    float acc = a.w[OB2 + j];
    for (int i = 0; i < H; ++i) acc += a.w[OW2 + j * H + i] * a.h1[i * LD + tid];
    a.h2[j * LD + tid] = fmaxf(acc, 0.f);
  }
  for (int c = 0; c < K; ++c) {
    float acc = a.w[OB3 + c];
    for (int j = 0; j < H; ++j) acc += a.w[OW3 + c * H + j] * a.h2[j * LD + tid];
    a.dz[c * LD + tid] = acc;  // logits, replaced by dL/dz below
    if (logits && valid) logits[(size_t)s * K + c] = acc;
  }
  if constexpr (!GRAD) return;

  // loss and dL/dz over the applicable variants
  float zmax = -3.0e38f, tb = 3.0e38f;
  bool any = false;
  for (int c = 0; c < K; ++c) {
    const float t = valid ? tin[(size_t)s * K + c] : 0.f;
    if (t > 0.f) {
      any = true;
      zmax = fmaxf(zmax, a.dz[c * LD + tid]);
      tb = fminf(tb, t);
    }
  }
  float sum = 0.f;
  for (int c = 0; c < K; ++c) {
    const float t = valid ? tin[(size_t)s * K + c] : 0.f;
    sum += t > 0.f ? expf(a.dz[c * LD + tid] - zmax) : 0.f;
  }
  const float lsum = logf(sum);
  float er = 0.f, qsum = 0.f;  // expected regret under p; soft-target normaliser
  for (int c = 0; c < K; ++c) {
    const float t = valid ? tin[(size_t)s * K + c] : 0.f;
    if (t > 0.f) {
      er += expf(a.dz[c * LD + tid] - zmax) / sum * (t / tb - 1.f);
      qsum += expf(-(t / tb - 1.f) / tau);
    }
  }
  float ce = 0.f;  // sum_c -q_c log p_c
  for (int c = 0; c < K; ++c) {
    const float t = valid ? tin[(size_t)s * K + c] : 0.f;
    if (t > 0.f) ce -= expf(-(t / tb - 1.f) / tau) / qsum * (a.dz[c * LD + tid] - zmax - lsum);
  }
  const float ws = any ? powf(tb * wscale, alpha) : 0.f;
  for (int c = 0; c < K; ++c) {
    const float t = valid ? tin[(size_t)s * K + c] : 0.f;
    float g = 0.f;
    if (any && t > 0.f) {
      const float p = expf(a.dz[c * LD + tid] - zmax) / sum, r = t / tb - 1.f;
      g = ws * (p * (r - er) + lambda * (p - expf(-r / tau) / qsum)) / (float)n;
    }
    a.dz[c * LD + tid] = g;
  }
  a.red[tid] = any ? ws * (er + lambda * ce) / (float)n : 0.f;

  // backward through the hidden layers
  for (int j = 0; j < H; ++j) {
    float acc = 0.f;
    for (int c = 0; c < K; ++c) acc += a.w[OW3 + c * H + j] * a.dz[c * LD + tid];
    a.dh2[j * LD + tid] = a.h2[j * LD + tid] > 0.f ? acc : 0.f;
  }
  for (int i = 0; i < H; ++i) {
    float acc = 0.f;
    for (int j = 0; j < H; ++j) acc += a.w[OW2 + j * H + i] * a.dh2[j * LD + tid];
    a.dh1[i * LD + tid] = a.h1[i * LD + tid] > 0.f ? acc : 0.f;
  }
  __syncthreads();

  // parameter gradients of this CTA's samples, summed in sample order
  float *g = gpart + (size_t)blockIdx.x * NP;
  for (int p = tid; p < NP; p += S) {
    const float *u, *v = nullptr;
    if (p < OB1) u = a.dh1 + (p / F) * LD, v = a.x + (p % F) * LD;
    else if (p < OW2) u = a.dh1 + (p - OB1) * LD;
    else if (p < OB2) u = a.dh2 + ((p - OW2) / H) * LD, v = a.h1 + ((p - OW2) % H) * LD;
    else if (p < OW3) u = a.dh2 + (p - OB2) * LD;
    else if (p < OB3) u = a.dz + ((p - OW3) / H) * LD, v = a.h2 + ((p - OW3) % H) * LD;
    else u = a.dz + (p - OB3) * LD;
    float acc = 0.f;
    if (v)
      for (int q = 0; q < S; ++q) acc += u[q] * v[q];
    else
      for (int q = 0; q < S; ++q) acc += u[q];
    g[p] = acc;
  }
  if (tid == 0) {
    float l = 0.f;
    for (int q = 0; q < S; ++q) l += a.red[q];
    lpart[blockIdx.x] = l;
  }
}

// grad[p] = sum over CTAs b (in order) of gpart[b][p]; loss likewise.
__global__ void reduce_parts(const float *__restrict__ gpart, const float *__restrict__ lpart, uint32_t nb,
                             float *__restrict__ grad, float *__restrict__ loss) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NP) {
    float acc = 0.f;
    for (uint32_t b = 0; b < nb; ++b) acc += gpart[(size_t)b * NP + p];
    grad[p] = acc;
  }
  if (p == NP && loss) {
    float acc = 0.f;
    for (uint32_t b = 0; b < nb; ++b) acc += lpart[b];
    *loss = acc;
  }
}

// Adam with decoupled weight decay on the FP32 master weights, then the BF16
// copy the forward pass reads.
__global__ void adam(float *__restrict__ w, __nv_bfloat16 *__restrict__ wb, const float *__restrict__ grad,
                     float *__restrict__ m, float *__restrict__ v, float lr, float b1, float b2, float eps, float wd,
                     float c1, float c2) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p >= NP) return;
  const float g = grad[p];
  const float mm = b1 * m[p] + (1.f - b1) * g;
  const float vv = b2 * v[p] + (1.f - b2) * g * g;
  m[p] = mm;
  v[p] = vv;
  const float wn = w[p] - lr * ((mm / c1) / (sqrtf(vv / c2) + eps) + wd * w[p]);
  w[p] = wn;
  wb[p] = __float2bfloat16_rn(wn);
}

__global__ void to_bf16(const float *__restrict__ w, __nv_bfloat16 *__restrict__ wb) {
  const int p = blockIdx.x * blockDim.x + threadIdx.x;
  if (p < NP) wb[p] = __float2bfloat16_rn(w[p]);
}

static int map_err(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  char msg[160];
  std::snprintf(msg, sizeof msg, "%s (%d)", cudaGetErrorString(e), (int)e);
  record_error(msg);
  return e == cudaErrorMemoryAllocation ? SPARSEP_ENOMEM : SPARSEP_EIO;
}

// Dynamic shared memory above 48 KB (set on the current device, every call).
static cudaError_t set_smem() {
  cudaError_t e = cudaFuncSetAttribute(fwd_bwd<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(fwd_bwd<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)SMEM);
  return e;
}

}  // namespace mlp
}  // namespace sparsep

using namespace sparsep::mlp;

struct sparsep_selector {
  __nv_bfloat16 *wb = nullptr;  // device weights
  float mean[SPARSEP_NFEATURES], stdev[SPARSEP_NFEATURES];
};

extern "C" {

uint32_t sparsep_mlp_nparams(void) { return NP; }

size_t sparsep_mlp_scratch_floats(uint32_t n) { return (size_t)((n + S - 1) / S) * (NP + 1); }

int sparsep_mlp_forward(const uint16_t *d_wb, const float *d_x, uint32_t n, float *d_logits, void *stream) {
  if (!d_wb || !d_x || !d_logits) return SPARSEP_EINVAL;
  if (!n) return SPARSEP_OK;
  if (int st = map_err(set_smem())) return st;
  fwd_bwd<false><<<(n + S - 1) / S, S, SMEM, static_cast<cudaStream_t>(stream)>>>(
      reinterpret_cast<const __nv_bfloat16 *>(d_wb), d_x, nullptr, n, 0.f, 0.f, 0.f, 1.f, d_logits, nullptr, nullptr);
  return map_err(cudaGetLastError());
}

int sparsep_mlp_loss_grad(const uint16_t *d_wb, const float *d_x, const float *d_t, uint32_t n, float wscale,
                          float alpha, float ce_weight, float tau, float *d_grad, float *d_loss, float *d_scratch,
                          void *stream) {
  if (!d_wb || !d_x || !d_t || !d_grad || !d_scratch || !n || !(tau > 0.f)) return SPARSEP_EINVAL;
  if (int st = map_err(set_smem())) return st;
  const uint32_t nb = (n + S - 1) / S;
  float *gpart = d_scratch, *lpart = d_scratch + (size_t)nb * NP;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  fwd_bwd<true><<<nb, S, SMEM, st>>>(reinterpret_cast<const __nv_bfloat16 *>(d_wb), d_x, d_t, n, wscale, alpha,
                                     ce_weight, tau, nullptr, gpart, lpart);
  if (int e = map_err(cudaGetLastError())) return e;
  reduce_parts<<<(NP + 1 + 255) / 256, 256, 0, st>>>(gpart, lpart, nb, d_grad, d_loss);
  return map_err(cudaGetLastError());
}

int sparsep_mlp_adam(float *d_w, uint16_t *d_wb, const float *d_grad, float *d_m, float *d_v, uint32_t step,
                     float lr, float beta1, float beta2, float eps, float weight_decay, void *stream) {
  if (!d_w || !d_wb || !d_grad || !d_m || !d_v || step == 0) return SPARSEP_EINVAL;
  const float c1 = 1.f - powf(beta1, (float)step), c2 = 1.f - powf(beta2, (float)step);
  adam<<<(NP + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_w, reinterpret_cast<__nv_bfloat16 *>(d_wb), d_grad, d_m, d_v, lr, beta1, beta2, eps, weight_decay, c1, c2);
  return map_err(cudaGetLastError());
}

int sparsep_mlp_to_bf16(const float *d_w, uint16_t *d_wb, void *stream) {
  if (!d_w || !d_wb) return SPARSEP_EINVAL;
  to_bf16<<<(NP + 255) / 256, 256, 0, static_cast<cudaStream_t>(stream)>>>(
      d_w, reinterpret_cast<__nv_bfloat16 *>(d_wb));
  return map_err(cudaGetLastError());
}

int sparsep_selector_create(const uint16_t *wb, const float *feat_mean, const float *feat_std,
                            sparsep_selector **out) {
  if (!wb || !feat_mean || !feat_std || !out) return SPARSEP_EINVAL;
  *out = nullptr;
  auto *s = new (std::nothrow) sparsep_selector();
  if (!s) return SPARSEP_ENOMEM;
  for (int i = 0; i < SPARSEP_NFEATURES; ++i) {
    s->mean[i] = feat_mean[i];
    s->stdev[i] = feat_std[i] > 0.f ? feat_std[i] : 1.f;
  }
  int st = map_err(sparsep::dev_malloc((void **)&s->wb, sizeof(__nv_bfloat16) * NP));
  if (!st) st = map_err(cudaMemcpy(s->wb, wb, sizeof(__nv_bfloat16) * NP, cudaMemcpyHostToDevice));
  if (st) {
    sparsep_selector_free(s);
    return st;
  }
  *out = s;
  return SPARSEP_OK;
}

void sparsep_selector_free(sparsep_selector *s) {
  if (!s) return;
  if (s->wb) sparsep::dev_free(s->wb);
  delete s;
}

// Logits (n x K) for raw features (n x 16): standardised here, scored on the
// GPU by the forward kernel.
int sparsep_selector_scores(sparsep_selector *s, const float *feats, uint32_t n, float *logits) {
  if (!s || !feats || !logits) return SPARSEP_EINVAL;
  if (!n) return SPARSEP_OK;
  float *hx = nullptr;
  try {
    hx = new float[(size_t)n * F];
  } catch (const std::bad_alloc &) {
    return SPARSEP_ENOMEM;
  }
  for (size_t q = 0; q < (size_t)n * F; ++q) hx[q] = (feats[q] - s->mean[q % F]) / s->stdev[q % F];
  float *dx = nullptr, *dl = nullptr;
  int st = map_err(sparsep::dev_malloc((void **)&dx, sizeof(float) * n * F));
  if (!st) st = map_err(sparsep::dev_malloc((void **)&dl, sizeof(float) * n * K));
  if (!st) st = map_err(cudaMemcpy(dx, hx, sizeof(float) * n * F, cudaMemcpyHostToDevice));
  if (!st) st = sparsep_mlp_forward(reinterpret_cast<const uint16_t *>(s->wb), dx, n, dl, nullptr);
  if (!st) st = map_err(cudaMemcpy(logits, dl, sizeof(float) * n * K, cudaMemcpyDeviceToHost));
  delete[] hx;
  if (dx) sparsep::dev_free(dx);
  if (dl) sparsep::dev_free(dl);
  return st;
}

}  // extern "C"
