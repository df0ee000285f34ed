// cg.cu -- conjugate gradient and power iteration on a plan: the iterative
// callers of the SpMV (no counterpart in the reference, whose programs run one
// SpMV).
//
// One CG iteration is the plan's SpMV q = A p followed by four small kernels:
//   dot   p . q                      (per-CTA partial sums)
//   fin   pq = sum of partials       (one CTA, fixed order)
//   xr    alpha = rr / pq;  x += alpha p;  r -= alpha q;  partials of r . r
//   beta  rr' = sum of partials; beta = rr' / rr; rr = rr';  p = r + beta p
// Every scalar stays on the device, so the iteration is captured once as a
// CUDA graph and replayed; the host reads the residual only every
// `check_every` iterations.  Reductions use a fixed grid and fixed orders, so
// a solve is bit-identical from run to run.  Dot products accumulate in
// double for both FP32 and FP64 vectors.
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <new>

#include "fault.hpp"
#include "internal.hpp"
#include "sparsep.h"

namespace sparsep {
namespace cg {

constexpr int NT = 256;   // threads per CTA of the vector kernels
constexpr int NB = 592;   // CTAs of the vector kernels (4 per SM of a B200)
enum { S_RR = 0, S_PQ = 1, S_BETA = 2, S_BB = 3, S_QQ = 4, S_NSC = 5 };

__device__ __forceinline__ double block_sum(double v, double *sm) {
  sm[threadIdx.x] = v;
  __syncthreads();
  for (int o = NT / 2; o > 0; o >>= 1) {
    if (threadIdx.x < o) sm[threadIdx.x] += sm[threadIdx.x + o];
    __syncthreads();
  }
  return sm[0];
}

// partials of a . b
template <typename T>
__global__ void __launch_bounds__(NT) dot(const T *__restrict__ a, const T *__restrict__ b, size_t n,
                                          double *__restrict__ part) {
  __shared__ double sm[NT];
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * NT + threadIdx.x; i < n; i += (size_t)NB * NT) s += (double)a[i] * (double)b[i];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// sc[slot] = sum of the NB partials, in order of the threads' strided sums
__global__ void __launch_bounds__(NT) finish(const double *__restrict__ part, double *__restrict__ sc, int slot) {
  __shared__ double sm[NT];
  double s = 0.0;
  for (int i = threadIdx.x; i < NB; i += NT) s += part[i];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) sc[slot] = s;
}

// r = b - q; p = r; partials of r . r
template <typename T>
__global__ void __launch_bounds__(NT) residual(const T *__restrict__ b, const T *__restrict__ q, T *__restrict__ r,
                                               T *__restrict__ p, size_t n, double *__restrict__ part) {
  __shared__ double sm[NT];
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * NT + threadIdx.x; i < n; i += (size_t)NB * NT) {
    const T v = b[i] - q[i];
    r[i] = v;
    p[i] = v;
    s += (double)v * (double)v;
  }
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// alpha = rr / pq (0 once converged); x += alpha p; r -= alpha q; partials of r . r
template <typename T>
__global__ void __launch_bounds__(NT) update_xr(T *__restrict__ x, T *__restrict__ r, const T *__restrict__ p,
                                                const T *__restrict__ q, size_t n, const double *__restrict__ sc,
                                                double *__restrict__ part) {
  __shared__ double sm[NT];
  const double pq = sc[S_PQ];
  const T alpha = (T)(pq != 0.0 ? sc[S_RR] / pq : 0.0);
  double s = 0.0;
  for (size_t i = (size_t)blockIdx.x * NT + threadIdx.x; i < n; i += (size_t)NB * NT) {
    x[i] += alpha * p[i];
    const T v = r[i] - alpha * q[i];
    r[i] = v;
    s += (double)v * (double)v;
  }
  s = block_sum(s, sm);
  if (threadIdx.x == 0) part[blockIdx.x] = s;
}

// rr' = sum of partials; beta = rr' / rr; rr = rr'
__global__ void __launch_bounds__(NT) finish_beta(const double *__restrict__ part, double *__restrict__ sc) {
  __shared__ double sm[NT];
  double s = 0.0;
  for (int i = threadIdx.x; i < NB; i += NT) s += part[i];
  s = block_sum(s, sm);
  if (threadIdx.x == 0) {
    const double rr = sc[S_RR];
    sc[S_BETA] = rr != 0.0 ? s / rr : 0.0;
    sc[S_RR] = s;
  }
}

// p = r + beta p
template <typename T>
__global__ void __launch_bounds__(NT) update_p(T *__restrict__ p, const T *__restrict__ r, size_t n,
                                               const double *__restrict__ sc) {
  const T beta = (T)sc[S_BETA];
  for (size_t i = (size_t)blockIdx.x * NT + threadIdx.x; i < n; i += (size_t)NB * NT) p[i] = r[i] + beta * p[i];
}

// power iteration: p = q / ||q|| with ||q||^2 in sc[slot] (p unchanged when q = 0);
// p and q may be the same vector
template <typename T>
__global__ void __launch_bounds__(NT) normalise(T *p, const T *q, size_t n, const double *__restrict__ sc, int slot) {
  const double qq = sc[slot];
  if (!(qq > 0.0)) return;
  const T inv = (T)(1.0 / std::sqrt(qq));
  for (size_t i = (size_t)blockIdx.x * NT + threadIdx.x; i < n; i += (size_t)NB * NT) p[i] = q[i] * inv;
}

}  // namespace cg
}  // namespace sparsep

using namespace sparsep::cg;

struct sparsep_cg {
  sparsep_plan *plan = nullptr;
  int dtype = 0;
  size_t n = 0, esize = 0;
  void *r = nullptr, *p = nullptr, *q = nullptr;
  double *part = nullptr, *sc = nullptr;
  cudaStream_t cap = nullptr;  // capture stream
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *graph_x = nullptr;  // x the captured iteration updates
};

static int cg_err(cudaError_t e) {
  if (e == cudaSuccess) return SPARSEP_OK;
  char msg[160];
  std::snprintf(msg, sizeof msg, "%s (%d)", cudaGetErrorString(e), (int)e);
  sparsep::record_error(msg);
  return e == cudaErrorMemoryAllocation ? SPARSEP_ENOMEM : SPARSEP_EIO;
}
#define CGK(x)                               \
  do {                                       \
    cudaError_t e_ = (x);                    \
    if (e_ != cudaSuccess) return cg_err(e_); \
  } while (0)

template <typename T>
static int iteration(sparsep_cg *c, T *x, cudaStream_t s) {
  if (int st = sparsep_execute_device(c->plan, c->p, c->q, s)) return st;
  const size_t n = c->n;
  dot<T><<<NB, NT, 0, s>>>((const T *)c->p, (const T *)c->q, n, c->part);
  finish<<<1, NT, 0, s>>>(c->part, c->sc, S_PQ);
  update_xr<T><<<NB, NT, 0, s>>>(x, (T *)c->r, (const T *)c->p, (const T *)c->q, n, c->sc, c->part);
  finish_beta<<<1, NT, 0, s>>>(c->part, c->sc);
  update_p<T><<<NB, NT, 0, s>>>((T *)c->p, (const T *)c->r, n, c->sc);
  return cg_err(cudaGetLastError());
}

template <typename T>
static int solve(sparsep_cg *c, const T *b, T *x, uint32_t max_iters, double tol, uint32_t check_every,
                 uint32_t *iters, double *rel, cudaStream_t s) {
  const size_t n = c->n;
  // r = b - A x; p = r; rr = r.r; bb = b.b
  if (int st = sparsep_execute_device(c->plan, x, c->q, s)) return st;
  residual<T><<<NB, NT, 0, s>>>(b, (const T *)c->q, (T *)c->r, (T *)c->p, n, c->part);
  finish<<<1, NT, 0, s>>>(c->part, c->sc, S_RR);
  dot<T><<<NB, NT, 0, s>>>(b, b, n, c->part);
  finish<<<1, NT, 0, s>>>(c->part, c->sc, S_BB);
  CGK(cudaGetLastError());
  if (!c->exec || c->graph_x != (void *)x) {
    if (c->exec) cudaGraphExecDestroy(c->exec);
    if (c->graph) cudaGraphDestroy(c->graph);
    c->exec = nullptr;
    c->graph = nullptr;
    CGK(cudaStreamBeginCapture(c->cap, cudaStreamCaptureModeThreadLocal));
    const int st = iteration<T>(c, x, c->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(c->cap, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    CGK(e);
    c->graph = g;
    CGK(cudaGraphInstantiate(&c->exec, c->graph, 0));
    c->graph_x = x;
  }
  double h[S_NSC];
  uint32_t it = 0;
  CGK(cudaMemcpyAsync(h, c->sc, sizeof h, cudaMemcpyDeviceToHost, s));
  CGK(cudaStreamSynchronize(s));
  const double bb = h[S_BB] > 0.0 ? h[S_BB] : 1.0;
  double r = std::sqrt(h[S_RR] / bb);
  const uint32_t every = check_every ? check_every : 1;
  while (r > tol && it < max_iters) {
    const uint32_t k = std::min(every, max_iters - it);
    for (uint32_t j = 0; j < k; ++j) CGK(cudaGraphLaunch(c->exec, s));
    it += k;
    CGK(cudaMemcpyAsync(h, c->sc, sizeof h, cudaMemcpyDeviceToHost, s));
    CGK(cudaStreamSynchronize(s));
    r = std::sqrt(h[S_RR] / bb);
  }
  if (iters) *iters = it;
  if (rel) *rel = r;
  return SPARSEP_OK;
}

// Power iteration: p_0 = x / ||x||; per iteration q = A p, lambda = p . q
// (the Rayleigh quotient, p having unit norm), p = q / ||q||.  The iteration is
// one captured graph (SpMV, two fixed-order dot products, the normalisation);
// the host reads lambda every check_every iterations and stops when two reads
// differ by at most rel_tol * |lambda|.  x receives the last p.
struct sparsep_power {
  sparsep_plan *plan = nullptr;
  int dtype = 0;
  size_t n = 0;
  void *q = nullptr;
  double *part = nullptr, *sc = nullptr;
  cudaStream_t cap = nullptr;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  void *graph_x = nullptr;
};

template <typename T>
static int power_step(sparsep_power *w, T *p, cudaStream_t s) {
  if (int st = sparsep_execute_device(w->plan, p, w->q, s)) return st;
  const T *q = static_cast<const T *>(w->q);
  dot<T><<<NB, NT, 0, s>>>(p, q, w->n, w->part);
  finish<<<1, NT, 0, s>>>(w->part, w->sc, S_PQ);
  dot<T><<<NB, NT, 0, s>>>(q, q, w->n, w->part);
  finish<<<1, NT, 0, s>>>(w->part, w->sc, S_QQ);
  normalise<T><<<NB, NT, 0, s>>>(p, q, w->n, w->sc, S_QQ);
  return cg_err(cudaGetLastError());
}

template <typename T>
static int power_run(sparsep_power *w, T *x, uint32_t max_iters, double tol, uint32_t check_every, double *lambda,
                     uint32_t *iters, cudaStream_t s) {
  // p_0 = x / ||x||, in place
  dot<T><<<NB, NT, 0, s>>>(x, x, w->n, w->part);
  finish<<<1, NT, 0, s>>>(w->part, w->sc, S_QQ);
  normalise<T><<<NB, NT, 0, s>>>(x, x, w->n, w->sc, S_QQ);
  CGK(cudaGetLastError());
  if (!w->exec || w->graph_x != (void *)x) {
    if (w->exec) cudaGraphExecDestroy(w->exec);
    if (w->graph) cudaGraphDestroy(w->graph);
    w->exec = nullptr;
    w->graph = nullptr;
    CGK(cudaStreamBeginCapture(w->cap, cudaStreamCaptureModeThreadLocal));
    const int st = power_step<T>(w, x, w->cap);
    cudaGraph_t g = nullptr;
    const cudaError_t e = cudaStreamEndCapture(w->cap, &g);
    if (st) {
      if (g) cudaGraphDestroy(g);
      return st;
    }
    CGK(e);
    w->graph = g;
    CGK(cudaGraphInstantiate(&w->exec, w->graph, 0));
    w->graph_x = x;
  }
  double h[S_NSC];
  uint32_t it = 0;
  double prev = 0.0, lam = 0.0;
  bool have_prev = false;
  const uint32_t every = check_every ? check_every : 1;
  while (it < max_iters) {
    const uint32_t k = std::min(every, max_iters - it);
    for (uint32_t j = 0; j < k; ++j) CGK(cudaGraphLaunch(w->exec, s));
    it += k;
    CGK(cudaMemcpyAsync(h, w->sc, sizeof h, cudaMemcpyDeviceToHost, s));
    CGK(cudaStreamSynchronize(s));
    lam = h[S_PQ];
    if (!(h[S_QQ] > 0.0)) break;  // A p = 0: lambda = 0 and nothing left to iterate
    if (have_prev && std::fabs(lam - prev) <= tol * std::fabs(lam)) break;
    prev = lam;
    have_prev = true;
  }
  if (lambda) *lambda = lam;
  if (iters) *iters = it;
  return SPARSEP_OK;
}

extern "C" {

int sparsep_cg_create(sparsep_plan *plan, sparsep_cg **out) {
  if (!plan || !out) return SPARSEP_EINVAL;
  *out = nullptr;
  sparsep_plan_info info;
  if (int st = sparsep_plan_get_info(plan, &info)) return st;
  if (info.nrows != info.ncols) return SPARSEP_EINVAL;
  if (info.dtype != SPARSEP_FP32 && info.dtype != SPARSEP_FP64) return SPARSEP_ENOSYS;
  auto *c = new (std::nothrow) sparsep_cg();
  if (!c) return SPARSEP_ENOMEM;
  c->plan = plan;
  c->dtype = info.dtype;
  c->n = info.nrows;
  c->esize = info.dtype == SPARSEP_FP32 ? 4 : 8;
  const size_t vb = (c->n + 64) * c->esize;
  int st = cg_err(sparsep::dev_malloc((void **)&c->r, vb));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&c->p, vb));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&c->q, vb));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&c->part, sizeof(double) * NB));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&c->sc, sizeof(double) * S_NSC));
  if (!st) st = cg_err(cudaStreamCreateWithFlags(&c->cap, cudaStreamNonBlocking));
  if (st) {
    sparsep_cg_free(c);
    return st;
  }
  *out = c;
  return SPARSEP_OK;
}

void sparsep_cg_free(sparsep_cg *c) {
  if (!c) return;
  if (c->exec) cudaGraphExecDestroy(c->exec);
  if (c->graph) cudaGraphDestroy(c->graph);
  for (void *d : {c->r, c->p, c->q, (void *)c->part, (void *)c->sc})
    if (d) sparsep::dev_free(d);
  if (c->cap) cudaStreamDestroy(c->cap);
  delete c;
}

int sparsep_cg_solve(sparsep_cg *c, const void *d_b, void *d_x, uint32_t max_iters, double rel_tol,
                     uint32_t check_every, uint32_t *iters, double *rel_residual, void *stream) {
  if (!c || !d_b || !d_x || !(rel_tol >= 0.0)) return SPARSEP_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (c->dtype == SPARSEP_FP32)
    return solve<float>(c, (const float *)d_b, (float *)d_x, max_iters, rel_tol, check_every, iters, rel_residual, s);
  return solve<double>(c, (const double *)d_b, (double *)d_x, max_iters, rel_tol, check_every, iters, rel_residual,
                       s);
}

int sparsep_power_create(sparsep_plan *plan, sparsep_power **out) {
  if (!plan || !out) return SPARSEP_EINVAL;
  *out = nullptr;
  sparsep_plan_info info;
  if (int st = sparsep_plan_get_info(plan, &info)) return st;
  if (info.nrows != info.ncols) return SPARSEP_EINVAL;
  if (info.dtype != SPARSEP_FP32 && info.dtype != SPARSEP_FP64) return SPARSEP_ENOSYS;
  auto *w = new (std::nothrow) sparsep_power();
  if (!w) return SPARSEP_ENOMEM;
  w->plan = plan;
  w->dtype = info.dtype;
  w->n = info.nrows;
  const size_t es = info.dtype == SPARSEP_FP32 ? 4 : 8;
  int st = cg_err(sparsep::dev_malloc((void **)&w->q, (w->n + 64) * es));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&w->part, sizeof(double) * NB));
  if (!st) st = cg_err(sparsep::dev_malloc((void **)&w->sc, sizeof(double) * S_NSC));
  if (!st) st = cg_err(cudaMemset(w->sc, 0, sizeof(double) * S_NSC));
  if (!st) st = cg_err(cudaStreamCreateWithFlags(&w->cap, cudaStreamNonBlocking));
  if (st) {
    sparsep_power_free(w);
    return st;
  }
  *out = w;
  return SPARSEP_OK;
}

void sparsep_power_free(sparsep_power *w) {
  if (!w) return;
  if (w->exec) cudaGraphExecDestroy(w->exec);
  if (w->graph) cudaGraphDestroy(w->graph);
  for (void *d : {w->q, (void *)w->part, (void *)w->sc})
    if (d) sparsep::dev_free(d);
  if (w->cap) cudaStreamDestroy(w->cap);
  delete w;
}

int sparsep_power_run(sparsep_power *w, void *d_x, uint32_t max_iters, double rel_tol, uint32_t check_every,
                      double *lambda, uint32_t *iters, void *stream) {
  if (!w || !d_x || !(rel_tol >= 0.0)) return SPARSEP_EINVAL;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  if (w->dtype == SPARSEP_FP32)
    return power_run<float>(w, (float *)d_x, max_iters, rel_tol, check_every, lambda, iters, s);
  return power_run<double>(w, (double *)d_x, max_iters, rel_tol, check_every, lambda, iters, s);
}

}  // extern "C"
