// mlp.cu -- C ABI of the control-variate network's tensor-core kernels
// (include/cubature/mlp.cuh, umma.cuh).
#include <cuda_bf16.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <memory>
#include <vector>

#include "capi_internal.h"
#include "cubature/mlp.cuh"

using namespace cubature;
using namespace cubature::capi;

namespace {

int* error_flag() {
  // one device flag per process and device, set by a kernel whose bounded
  // wait gave up
  static int* flags[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  dev &= 63;
  if (!flags[dev]) {
    if (cudaMalloc(&flags[dev], sizeof(int)) != cudaSuccess) return nullptr;
    cudaMemset(flags[dev], 0, sizeof(int));
  }
  return flags[dev];
}

template <int N, int EPI>
cudaError_t launch_gemm(dim3 grid, cudaStream_t s, const umma::GemmArgs& g,
                        const mlp::EpiArgs& ep) {
  static bool configured[64] = {};
  int dev = 0;
  cudaGetDevice(&dev);
  if (!configured[dev & 63]) {
    cudaError_t e = cudaFuncSetAttribute(mlp::k_gemm<N, EPI>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         mlp::kGemmSmem);
    if (e != cudaSuccess) return e;
    configured[dev & 63] = true;
  }
  mlp::k_gemm<N, EPI><<<grid, 128, mlp::kGemmSmem, s>>>(g, ep);
  return cudaGetLastError();
}

}  // namespace

int cub_mlp_gemm_bf16(int batch, int m, int n, int k, const void* d_a, long long lda,
                      const void* d_b, long long ldb, float* d_d, long long ldd, void* stream) {
  if (batch <= 0 || m <= 0 || m % umma::kTileM || k <= 0 || k % 16 || (n != 16 && n != 128) ||
      !d_a || !d_b || !d_d || lda < k || ldb < k || ldd < n || lda % 8 || ldb % 8) {
    set_error("cub_mlp_gemm_bf16: m % 128, k % 16, n in {16, 128}, lda/ldb % 8 required");
    return CUB_ERR_INVALID;
  }
  int* err = error_flag();
  if (!err) return cuda_error(cudaErrorMemoryAllocation, "error flag");
  cudaStream_t s = as_stream(stream);
  umma::GemmArgs g;
  g.a = static_cast<const __nv_bfloat16*>(d_a);
  g.b = static_cast<const __nv_bfloat16*>(d_b);
  g.lda = lda;
  g.ldb = ldb;
  g.batch_a = lda * m;
  g.batch_b = ldb * n;
  g.m = m;
  g.k = k;
  g.error = err;
  mlp::EpiArgs ep{};
  ep.out = d_d;
  ep.ld_out = ldd;
  ep.batch_out = ldd * m;
  const dim3 grid(m / umma::kTileM, 1, batch);
  cudaError_t e;
  if (n == 16) {
    e = launch_gemm<16, mlp::kEpiStore>(grid, s, g, ep);
  } else {
    e = launch_gemm<128, mlp::kEpiStore>(grid, s, g, ep);
  }
  if (e != cudaSuccess) return cuda_error(e, "k_gemm launch");
  int h_err = 0;
  if ((e = cudaMemcpyAsync(&h_err, err, sizeof(int), cudaMemcpyDeviceToHost, s)) != cudaSuccess ||
      (e = cudaStreamSynchronize(s)) != cudaSuccess)
    return cuda_error(e, "k_gemm");
  if (h_err) {
    cudaMemsetAsync(err, 0, sizeof(int), s);
    set_error("tensor-core GEMM: a bounded wait gave up");
    return CUB_ERR_TIMEOUT;
  }
  return 0;
}

// ---------------------------------------------------------------------------
// The networks: buffers, training and inference.
// ---------------------------------------------------------------------------
using mlp::Layout;
using bf16 = __nv_bfloat16;

struct cub_mlp {
  int device = 0, E = 0, S = 0, B = 0;
  cudaStream_t stream = nullptr;
  int* err = nullptr;
  int step = 0;
  bool have_data = false;
  std::vector<void*> bufs;
  float *P, *G, *Mm, *Vv, *part, *loss, *scale, *Y;
  bf16 *W0, *W1, *W1T, *W2, *W2T, *X, *XT, *XE, *XET;
  bf16 *Z1, *H1, *H1T, *Z2, *H2, *H2T, *Z3, *H3, *H3T;
  bf16 *dZ1, *dZ1T, *dZ2, *dZ2T, *dZ3, *dZ3T;

  template <class T>
  bool alloc(T** p, size_t n) {
    void* q = nullptr;
    if (cudaMalloc(&q, n * sizeof(T)) != cudaSuccess) return false;
    bufs.push_back(q);
    *p = static_cast<T*>(q);
    return true;
  }
  ~cub_mlp() {
    cudaSetDevice(device);
    if (stream) cudaStreamSynchronize(stream);
    for (void* q : bufs) cudaFree(q);
    if (stream) cudaStreamDestroy(stream);
  }
};

namespace {

// Uniform(-1/sqrt(fan_in), 1/sqrt(fan_in)) weights from a 64-bit LCG on
// the host, zero biases and zero padding columns of W0.
void init_params(std::vector<float>& p, int E, unsigned long long seed) {
  p.assign((size_t)E * Layout::kCount, 0.0f);
  unsigned long long x = seed * 6364136223846793005ull + 1442695040888963407ull;
  auto uni = [&x]() {
    x = x * 6364136223846793005ull + 1442695040888963407ull;
    return (double)(x >> 11) * (1.0 / 9007199254740992.0);
  };
  for (int e = 0; e < E; ++e) {
    float* q = p.data() + (size_t)e * Layout::kCount;
    const double a0 = 1.0 / std::sqrt((double)mlp::kIn), a = 1.0 / std::sqrt(128.0);
    for (int o = 0; o < 128; ++o)
      for (int i = 0; i < mlp::kIn; ++i) q[Layout::W0 + o * mlp::kInPad + i] = (float)((2 * uni() - 1) * a0);
    for (int i = 0; i < 128 * 128; ++i) q[Layout::W1 + i] = (float)((2 * uni() - 1) * a);
    for (int i = 0; i < 128 * 128; ++i) q[Layout::W2 + i] = (float)((2 * uni() - 1) * a);
    for (int i = 0; i < 128; ++i) q[Layout::W3 + i] = (float)((2 * uni() - 1) * a);
  }
}

int check(cudaError_t e, const char* what) { return e == cudaSuccess ? 0 : cuda_error(e, what); }

int refresh(cub_mlp* m) {
  mlp::k_refresh_weights<<<dim3(64, 1, m->E), 256, 0, m->stream>>>(m->P, m->W0, m->W1, m->W1T,
                                                                     m->W2, m->W2T);
  return check(cudaGetLastError(), "k_refresh_weights");
}

// Forward pass of `rows` rows (multiple of 128) starting at X (row-major,
// per-network stride batch_x): Z/H/HT of the three hidden layers.
int forward(cub_mlp* m, const bf16* X, long long batch_x, int rows) {
  const long long B = rows;
  const dim3 grid(rows / umma::kTileM, 1, m->E);
  umma::GemmArgs g{};
  g.error = m->err;
  g.m = rows;
  mlp::EpiArgs ep{};
  ep.batch_bias = Layout::kCount;
  ep.ld_act = 128;
  ep.batch_act = B * 128;
  ep.ld_t = B;
  ep.batch_t = 128 * B;
  const bf16* in[3] = {X, m->H1, m->H2};
  const bf16* w[3] = {m->W0, m->W1, m->W2};
  bf16* z[3] = {m->Z1, m->Z2, m->Z3};
  bf16* h[3] = {m->H1, m->H2, m->H3};
  bf16* ht[3] = {m->H1T, m->H2T, m->H3T};
  const int boff[3] = {Layout::B0, Layout::B1, Layout::B2};
  for (int l = 0; l < 3; ++l) {
    g.a = in[l];
    g.lda = l == 0 ? mlp::kInPad : 128;
    g.batch_a = l == 0 ? batch_x : B * 128;
    g.b = w[l];
    g.ldb = l == 0 ? mlp::kInPad : 128;
    g.batch_b = l == 0 ? 128 * mlp::kInPad : 128 * 128;
    g.k = l == 0 ? mlp::kInPad : 128;
    ep.bias = m->P + boff[l];
    ep.z = z[l];
    ep.h = h[l];
    ep.ht = ht[l];
    cudaError_t e = launch_gemm<128, mlp::kEpiForward>(grid, m->stream, g, ep);
    if (e != cudaSuccess) return cuda_error(e, "forward GEMM");
  }
  return 0;
}

// Forward + backward of minibatch b into G (no update); loss into m->loss.
int grad_step(cub_mlp* m, int b) {
  const long long B = m->B, S = m->S;
  const long long s0 = (long long)b * B;
  int rc = forward(m, m->X + s0 * mlp::kInPad, S * mlp::kInPad, m->B);
  if (rc) return rc;
  const int nblk = m->B / 128;
  const float inv = 1.0f / (float)m->B;
  mlp::k_output<<<dim3(nblk, 1, m->E), 128, 0, m->stream>>>(
      m->P, m->H3, m->Z3, m->Y + s0, S, inv, m->dZ3, m->dZ3T, m->part, B, B, m->scale, nullptr, 0);
  if ((rc = check(cudaGetLastError(), "k_output"))) return rc;
  mlp::k_reduce_output<<<dim3(1, 1, m->E), 160, 0, m->stream>>>(m->part, nblk, m->G, m->loss, inv);
  if ((rc = check(cudaGetLastError(), "k_reduce_output"))) return rc;
  umma::GemmArgs g{};
  g.error = m->err;
  mlp::EpiArgs ep{};
  ep.ld_act = 128;
  ep.batch_act = B * 128;
  ep.ld_t = B;
  ep.batch_t = 128 * B;
  const bf16* dzT[3] = {m->dZ1T, m->dZ2T, m->dZ3T};
  const bf16* hT[3] = {m->XT + s0, m->H1T, m->H2T};
  const int woff[3] = {Layout::W0, Layout::W1, Layout::W2};
  for (int l = 2; l >= 0; --l) {
    // weight gradient dW_l = dZ_{l+1}^T H_l
    g.a = dzT[l];
    g.lda = B;
    g.batch_a = 128 * B;
    g.b = hT[l];
    g.ldb = l == 0 ? S : B;
    g.batch_b = l == 0 ? mlp::kInPad * S : 128 * B;
    g.m = 128;
    g.k = m->B;
    ep.out = m->G + woff[l];
    ep.ld_out = l == 0 ? mlp::kInPad : 128;
    ep.batch_out = Layout::kCount;
    cudaError_t e = l == 0 ? launch_gemm<16, mlp::kEpiStore>(dim3(1, 1, m->E), m->stream, g, ep)
                           : launch_gemm<128, mlp::kEpiStore>(dim3(1, 1, m->E), m->stream, g, ep);
    if (e != cudaSuccess) return cuda_error(e, "weight-gradient GEMM");
    mlp::k_bias_grad<<<dim3(16, 1, m->E), 256, 0, m->stream>>>(dzT[l], B, m->G,
                                                                 woff[l] + (l == 0 ? 128 * 16 : 128 * 128));
    if ((rc = check(cudaGetLastError(), "k_bias_grad"))) return rc;
    if (l == 0) break;
    // dZ_l = (dZ_{l+1} W_l) * silu'(Z_l)
    g.a = l == 2 ? m->dZ3 : m->dZ2;
    g.lda = 128;
    g.batch_a = B * 128;
    g.b = l == 2 ? m->W2T : m->W1T;
    g.ldb = 128;
    g.batch_b = 128 * 128;
    g.m = m->B;
    g.k = 128;
    ep.zin = l == 2 ? m->Z2 : m->Z1;
    ep.dz = l == 2 ? m->dZ2 : m->dZ1;
    ep.dzt = l == 2 ? m->dZ2T : m->dZ1T;
    e = launch_gemm<128, mlp::kEpiBackward>(dim3(m->B / 128, 1, m->E), m->stream, g, ep);
    if (e != cudaSuccess) return cuda_error(e, "backward GEMM");
  }
  return 0;
}

int read_error(cub_mlp* m) {
  int h = 0;
  cudaError_t e = cudaMemcpyAsync(&h, m->err, sizeof(int), cudaMemcpyDeviceToHost, m->stream);
  if (e == cudaSuccess) e = cudaStreamSynchronize(m->stream);
  if (e != cudaSuccess) return cuda_error(e, "network kernels");
  if (h) {
    cudaMemsetAsync(m->err, 0, sizeof(int), m->stream);
    set_error("tensor-core GEMM: a bounded wait gave up");
    return CUB_ERR_TIMEOUT;
  }
  return 0;
}

}  // namespace

cub_mlp* cub_mlp_create(int device, int count, int samples, int batch, unsigned long long seed) {
  if (count <= 0 || batch <= 0 || batch % 128 || samples <= 0 || samples % batch) {
    set_error("cub_mlp_create: batch a multiple of 128 and samples a multiple of batch");
    return nullptr;
  }
  if (cudaSetDevice(device) != cudaSuccess) {
    set_error("cudaSetDevice failed");
    return nullptr;
  }
  auto* m = new cub_mlp;
  m->device = device;
  m->E = count;
  m->S = samples;
  m->B = batch;
  const size_t E = count, S = samples, B = batch, P = Layout::kCount;
  bool ok = cudaStreamCreateWithFlags(&m->stream, cudaStreamNonBlocking) == cudaSuccess &&
            m->alloc(&m->err, 1) && m->alloc(&m->P, E * P) && m->alloc(&m->G, E * P) &&
            m->alloc(&m->Mm, E * P) && m->alloc(&m->Vv, E * P) &&
            m->alloc(&m->part, E * (B / 128) * (128 + 2)) && m->alloc(&m->loss, E) &&
            m->alloc(&m->scale, E) && m->alloc(&m->Y, E * S) &&
            m->alloc(&m->W0, E * 128 * 16) && m->alloc(&m->W1, E * 128 * 128) &&
            m->alloc(&m->W1T, E * 128 * 128) && m->alloc(&m->W2, E * 128 * 128) &&
            m->alloc(&m->W2T, E * 128 * 128) && m->alloc(&m->X, E * S * 16) &&
            m->alloc(&m->XT, E * S * 16) && m->alloc(&m->XE, E * B * 16) &&
            m->alloc(&m->XET, E * B * 16);
  bf16** act[] = {&m->Z1, &m->H1, &m->H1T, &m->Z2, &m->H2, &m->H2T, &m->Z3, &m->H3,
                  &m->H3T, &m->dZ1, &m->dZ1T, &m->dZ2, &m->dZ2T, &m->dZ3, &m->dZ3T};
  for (bf16** a : act) ok = ok && m->alloc(a, E * B * 128);
  if (!ok) {
    set_error("cub_mlp_create: device allocation failed");
    delete m;
    return nullptr;
  }
  std::vector<float> p;
  init_params(p, count, seed);
  ok = cudaMemsetAsync(m->err, 0, sizeof(int), m->stream) == cudaSuccess &&
       cudaMemcpyAsync(m->P, p.data(), sizeof(float) * E * P, cudaMemcpyHostToDevice,
                       m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->G, 0, sizeof(float) * E * P, m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->Mm, 0, sizeof(float) * E * P, m->stream) == cudaSuccess &&
       cudaMemsetAsync(m->Vv, 0, sizeof(float) * E * P, m->stream) == cudaSuccess &&
       refresh(m) == 0 && cudaStreamSynchronize(m->stream) == cudaSuccess;
  if (!ok) {
    set_error("cub_mlp_create: initialisation failed");
    delete m;
    return nullptr;
  }
  return m;
}

void cub_mlp_destroy(cub_mlp* m) { delete m; }

int cub_mlp_set_data(cub_mlp* m, const double* d_x, const double* d_y) {
  if (!m || !d_x || !d_y) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  cudaSetDevice(m->device);
  const long long S = m->S;
  mlp::k_prep_inputs<<<dim3(64, 1, m->E), 256, 0, m->stream>>>(d_x, S, S * mlp::kIn, m->X, m->XT,
                                                                 S, S * mlp::kInPad,
                                                                 S * mlp::kInPad);
  mlp::k_scale_targets<<<dim3(1, 1, m->E), 256, 0, m->stream>>>(d_y, S, m->Y, m->scale);
  int rc = check(cudaGetLastError(), "set_data");
  if (!rc) rc = check(cudaStreamSynchronize(m->stream), "set_data");
  m->have_data = rc == 0;
  return rc;
}

int cub_mlp_params(cub_mlp* m, float* h_params, int set) {
  if (!m || !h_params) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  cudaSetDevice(m->device);
  const size_t bytes = sizeof(float) * (size_t)m->E * Layout::kCount;
  int rc = set ? check(cudaMemcpyAsync(m->P, h_params, bytes, cudaMemcpyHostToDevice, m->stream),
                       "params")
               : check(cudaMemcpyAsync(h_params, m->P, bytes, cudaMemcpyDeviceToHost, m->stream),
                       "params");
  if (!rc && set) rc = refresh(m);
  if (!rc) rc = check(cudaStreamSynchronize(m->stream), "params");
  return rc;
}

int cub_mlp_grad(cub_mlp* m, int b, float* h_loss, float* h_grads) {
  if (!m || !m->have_data || b < 0 || b >= m->S / m->B) {
    set_error("cub_mlp_grad: no data or minibatch out of range");
    return CUB_ERR_INVALID;
  }
  cudaSetDevice(m->device);
  int rc = grad_step(m, b);
  if (!rc) rc = read_error(m);
  if (!rc && h_loss)
    rc = check(cudaMemcpy(h_loss, m->loss, sizeof(float) * m->E, cudaMemcpyDeviceToHost), "loss");
  if (!rc && h_grads)
    rc = check(cudaMemcpy(h_grads, m->G, sizeof(float) * (size_t)m->E * Layout::kCount,
                          cudaMemcpyDeviceToHost),
               "grads");
  return rc;
}

int cub_mlp_train(cub_mlp* m, int epochs, float lr, float* h_loss) {
  if (!m || !m->have_data || epochs < 0 || !(lr > 0)) {
    set_error("cub_mlp_train: no data or bad arguments");
    return CUB_ERR_INVALID;
  }
  cudaSetDevice(m->device);
  const int nb = m->S / m->B;
  const long long n = (long long)m->E * Layout::kCount;
  const float b1 = 0.9f, b2 = 0.999f;
  for (int ep = 0; ep < epochs; ++ep) {
    for (int b = 0; b < nb; ++b) {
      int rc = grad_step(m, b);
      if (rc) return rc;
      ++m->step;
      const float c1 = 1.0f - std::pow(b1, (float)m->step), c2 = 1.0f - std::pow(b2, (float)m->step);
      mlp::k_adam<<<592, 256, 0, m->stream>>>(m->P, m->G, m->Mm, m->Vv, n, lr, b1, b2, 1e-8f, c1, c2);
      if ((rc = check(cudaGetLastError(), "k_adam")) || (rc = refresh(m))) return rc;
    }
    int rc = read_error(m);  // once per epoch
    if (rc) return rc;
  }
  if (h_loss)
    return check(cudaMemcpy(h_loss, m->loss, sizeof(float) * m->E, cudaMemcpyDeviceToHost), "loss");
  return 0;
}

int cub_mlp_eval(cub_mlp* m, long long n, const double* d_x, double* d_g) {
  if (!m || n <= 0 || !d_x || !d_g) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  cudaSetDevice(m->device);
  const long long B = m->B;
  for (long long c0 = 0; c0 < n; c0 += B) {
    const long long cnt = std::min(B, n - c0);
    // stale rows past cnt are evaluated and discarded
    mlp::k_prep_inputs<<<dim3(16, 1, m->E), 256, 0, m->stream>>>(
        d_x + c0 * mlp::kIn, cnt, n * mlp::kIn, m->XE, m->XET, B, B * mlp::kInPad,
        B * mlp::kInPad);
    int rc = check(cudaGetLastError(), "k_prep_inputs");
    if (rc || (rc = forward(m, m->XE, B * mlp::kInPad, m->B))) return rc;
    mlp::k_output<<<dim3(m->B / 128, 1, m->E), 128, 0, m->stream>>>(
        m->P, m->H3, m->Z3, nullptr, 0, 0.0f, nullptr, nullptr, nullptr, B, cnt, m->scale,
        d_g + c0, n);
    if ((rc = check(cudaGetLastError(), "k_output"))) return rc;
  }
  return read_error(m);
}

// ---------------------------------------------------------------------------
// Learned control variate: integral of f = integral of g + integral of
// (f - g), with g the network trained on f's values at rule nodes.
// ---------------------------------------------------------------------------
#include "cubature/engine.cuh"

namespace {

constexpr int kCvDim = 7;
using CvPT = detail::PointTable<kCvDim>;

// f at points x [E][S][7] for integral e's parameters -> y [E][S].
template <class F>
__global__ void k_eval_points(const GenzParams* params, const double* x, long long S, double* y) {
  const int e = blockIdx.z;
  const F f = F::load(params[e]);
  for (long long s = (long long)blockIdx.x * blockDim.x + threadIdx.x; s < S;
       s += (long long)gridDim.x * blockDim.x)
    y[e * S + s] = f(x + (e * S + s) * kCvDim);
}

// a f(x) + b g_p at the rule points of one region (g_p precomputed).
template <class F>
struct CvPoint {
  F f;
  double a, b;
  const double* g;
  __device__ __forceinline__ double operator()(const double* x, int p) const {
    const double gv = g[p];
    return a != 0.0 ? a * f(x) + b * gv : b * gv;
  }
};

// Rule and fourth difference of slots [0, n) for the integrand a f + b g:
// eight regions per block, 32 threads each.  A region stays active while
// its error exceeds its volume's share of the absolute budget,
// err > budget * volume (unit-cube volume 1), so that when every region is
// finished the total error is within the budget.
template <class F>
__global__ void __launch_bounds__(256) k_eval_cv(F f, double ca, double cb, const double* g,
                                                 RuleTables T, EngineArgs a, long long s0,
                                                 long long n, double budget) {
  __shared__ detail::GroupSmem<kCvDim> sm;
  sm.pt.fill(threadIdx.x, blockDim.x);
  __syncthreads();
  const int grp = threadIdx.x / 32, t = threadIdx.x % 32;
  const long long ngroups = 8ll * gridDim.x;
  for (long long base = 0; base < n; base += ngroups) {
    const long long local = base + (long long)grp * gridDim.x + blockIdx.x;
    const bool live = local < n;
    const long long slot = s0 + local;
    const int k = live ? a.rid[slot] : -1;
    double L[kCvDim], H[kCvDim];
#pragma unroll
    for (int d = 0; d < kCvDim; ++d) {
      L[d] = k >= 0 ? a.lo[(long long)d * a.cap + slot] : 0.0;
      H[d] = k >= 0 ? a.len[(long long)d * a.cap + slot] : 1.0;
    }
    const CvPoint<F> h{f, ca, cb, g + (k >= 0 ? local : 0) * CvPT::kPoints};
    const detail::RegionResult r =
        detail::eval_region_group<kCvDim, 32>(h, L, H, T, sm, grp, t, k >= 0);
    if (t == 0 && live) {
      if (k >= 0) {
        double vol = 1;
#pragma unroll
        for (int d = 0; d < kCvDim; ++d) vol *= H[d];
        a.avg[slot] = r.avg;
        a.err[slot] = r.err;
        a.axis[slot] = r.axis;
        a.active[slot] = r.err > budget * vol;
      } else {
        detail::store_padding(a, slot);
      }
    }
  }
}

// The network as a smooth function for integration: its bf16 weights with
// FP32 activations and FP32 arithmetic on the CUDA cores (the tensor-core
// path rounds every activation to bf16, a quantisation of ~2^-8 relative
// that no bisection resolves, so an adaptive rule cannot converge on it).
// One warp per node; the weights sit transposed in shared memory
// (W^T[in][out]: lanes read consecutive outputs).  g[r] for the nodes of
// slots [s0, s0 + n), row (s - s0) * npts + p.
constexpr int kSmoothSmem = (16 * 128 + 2 * 128 * 128 + 4 * 128 + 8 * 2 * 128) * 4;

__global__ void __launch_bounds__(256) k_cv_smooth(const float* P, const bf16* W0, const bf16* W1,
                                                   const bf16* W2, float scale, const double* lo,
                                                   const double* len, const int* rid,
                                                   long long cap, long long s0, long long n,
                                                   double* g) {
  extern __shared__ float fsm[];
  float* w0t = fsm;                 // [16][128]
  float* w1t = w0t + 16 * 128;      // [128][128]
  float* w2t = w1t + 128 * 128;     // [128][128]
  float* bias = w2t + 128 * 128;    // b0, b1, b2, w3
  float* buf = bias + 4 * 128;      // per warp: two rows of 128
  __shared__ CvPT pt;
  pt.fill(threadIdx.x, blockDim.x);
  for (int i = threadIdx.x; i < 128 * 128; i += blockDim.x) {
    const int o = i / 128, in = i % 128;
    w1t[in * 128 + o] = __bfloat162float(W1[i]);
    w2t[in * 128 + o] = __bfloat162float(W2[i]);
    if (i < 128 * 16) w0t[(i % 16) * 128 + i / 16] = __bfloat162float(W0[i]);
  }
  for (int j = threadIdx.x; j < 128; j += blockDim.x) {
    bias[j] = P[Layout::B0 + j];
    bias[128 + j] = P[Layout::B1 + j];
    bias[256 + j] = P[Layout::B2 + j];
    bias[384 + j] = P[Layout::W3 + j];
  }
  __syncthreads();
  const float b3 = P[Layout::B3];
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  float* ha = buf + warp * 256;
  float* hb = ha + 128;
  const long long nodes = n * CvPT::kPoints;
  const long long nwarps = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long r = (long long)blockIdx.x * (blockDim.x >> 5) + warp; r < nodes; r += nwarps) {
    const long long s = s0 + r / CvPT::kPoints;
    if (rid[s] < 0) {
      if (lane == 0) g[r] = 0.0;
      continue;
    }
    const uint2 e = pt.ent[(int)(r % CvPT::kPoints)];
    float xin[kCvDim];
#pragma unroll
    for (int i = 0; i < kCvDim; ++i) {
      const double x = fma(pt.ctab[(e.x >> (4 * i)) & 15u], len[(long long)i * cap + s],
                           lo[(long long)i * cap + s]);
      xin[i] = (float)(2.0 * x - 1.0);
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) {
      const int j = lane + 32 * q;
      float z = bias[j];
#pragma unroll
      for (int i = 0; i < kCvDim; ++i) z = fmaf(w0t[i * 128 + j], xin[i], z);
      ha[j] = mlp::silu(z);
    }
    __syncwarp();
    const float* wt[2] = {w1t, w2t};
    float* src = ha;
    float* dst = hb;
    for (int l = 0; l < 2; ++l) {
      float z[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) z[q] = bias[128 * (l + 1) + lane + 32 * q];
      for (int i = 0; i < 128; ++i) {
        const float h = src[i];
#pragma unroll
        for (int q = 0; q < 4; ++q) z[q] = fmaf(wt[l][i * 128 + lane + 32 * q], h, z[q]);
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) dst[lane + 32 * q] = mlp::silu(z[q]);
      __syncwarp();
      float* t = src;
      src = dst;
      dst = t;
    }
    float acc = 0;
#pragma unroll
    for (int q = 0; q < 4; ++q) acc = fmaf(bias[384 + lane + 32 * q], src[lane + 32 * q], acc);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(0xffffffffu, acc, o);
    if (lane == 0) g[r] = (double)scale * (double)(acc + b3);
    __syncwarp();
  }
}

// Evaluation hook of the engine's multi-launch driver: the rule over the
// current list for a f + b g, g from network net_k at every rule point.
template <class F>
struct CvHook {
  static constexpr bool kActive = true;
  cub_mlp* net;
  int net_k;
  F f;
  double ca, cb;
  double budget;  // absolute error budget of the integral
  RuleTables T;
  int sms;
  // growable scratch (shared by the hook's copies)
  struct Scratch {
    long long rows = 0;
    bf16 *X = nullptr, *Ha = nullptr, *Hb = nullptr;
    double* g = nullptr;
    void release() {
      cudaFree(X);
      cudaFree(Ha);
      cudaFree(Hb);
      cudaFree(g);
      X = Ha = Hb = nullptr;
      g = nullptr;
      rows = 0;
    }
  };
  Scratch* sc;

  // Node rows per chunk: the network's activations for 2^22 rows take
  // 2 x 1 GB, whatever the length of the list.
  static constexpr long long kRowsMax = 1ll << 22;

  int eval(const EngineArgs& a, long long n, cudaStream_t s) const {
    const long long per = kRowsMax / CvPT::kPoints;  // slots per chunk
    const long long cmax = std::min(n, per);
    const long long rmax = (cmax * CvPT::kPoints + 127) / 128 * 128;
    if (rmax > sc->rows) {
      cudaStreamSynchronize(s);
      sc->release();
      const long long r = std::max(rmax, 1ll << 16);
      if (cudaMalloc(&sc->g, sizeof(double) * r) != cudaSuccess) {
        set_error("control variate: scratch allocation failed");
        return kErrCuda;
      }
      sc->rows = r;
    }
    static bool configured[64] = {};
    int dev = 0;
    cudaGetDevice(&dev);
    if (!configured[dev & 63]) {
      if (cudaFuncSetAttribute(k_cv_smooth, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               kSmoothSmem) != cudaSuccess)
        return kErrCuda;
      configured[dev & 63] = true;
    }
    float scale = 1.0f;
    cudaMemcpyAsync(&scale, net->scale + net_k, sizeof(float), cudaMemcpyDeviceToHost, s);
    cudaStreamSynchronize(s);
    const long long P = Layout::kCount;
    for (long long s0 = 0; s0 < n; s0 += per) {
      const long long cn = std::min(per, n - s0);
      k_cv_smooth<<<(unsigned)sms, 256, kSmoothSmem, s>>>(
          net->P + net_k * P, net->W0 + (long long)net_k * 128 * 16,
          net->W1 + (long long)net_k * 128 * 128, net->W2 + (long long)net_k * 128 * 128, scale,
          a.lo, a.len, a.rid, a.cap, s0, cn, sc->g);
      if (cudaGetLastError() != cudaSuccess) return kErrCuda;
      const long long eb = std::min<long long>((cn + 7) / 8, (long long)sms * 8);
      k_eval_cv<F><<<(unsigned)std::max<long long>(eb, 1), 256, 0, s>>>(f, ca, cb, sc->g, T, a,
                                                                        s0, cn, budget);
      if (cudaGetLastError() != cudaSuccess) return kErrCuda;
    }
    return 0;
  }
};

double now_ms() {
  return std::chrono::duration<double, std::milli>(
             std::chrono::steady_clock::now().time_since_epoch())
      .count();
}

// The whole control-variate flow for one family (N = 7).
template <template <int> class Fam>
int cv_run(cub_ctx* ctx, int count, const GenzParams* h, double epsrel, double epsabs,
           const cub_cv_options& co, cub_result* out, cub_cv_stats* st) {
  using F = Fam<kCvDim>;
  Workspace& ws = *ctx->ws;
  const cudaStream_t s = ctx->stream;
  Options o;
  o.policy = kPolicyBreadth;
  o.max_slots = ws.auto_slots(kCvDim, o.policy);
  const RuleTables T = make_rule9_tables(kCvDim);
  int dev = 0;
  cudaGetDevice(&dev);
  const int sms = sm_count(dev);
  std::vector<double> er(count), ea(count);
  std::vector<Result> coarse(count), res(count);
  double t0 = now_ms();

  // 1. coarse plain run: the check of the result and the scale of the tolerances
  GenzParams* d_par = nullptr;
  if (cudaMalloc(&d_par, sizeof(GenzParams) * count) != cudaSuccess)
    return cuda_error(cudaErrorMemoryAllocation, "params");
  std::unique_ptr<GenzParams, decltype(&cudaFree)> par_guard(d_par, cudaFree);
  cudaMemcpyAsync(d_par, h, sizeof(GenzParams) * count, cudaMemcpyHostToDevice, s);
  for (int k = 0; k < count; ++k) {
    er[k] = std::max(co.coarse_epsrel, epsrel);
    ea[k] = epsabs;
  }
  {
    detail::ParamSource<F> src{d_par};
    const int rc = grouped_batch(count, o, [&](const std::vector<int>& idx, Result* g) {
      // groups of the batch run on consecutive parameter blocks
      detail::ParamSource<F> gs{d_par + idx[0]};
      (void)src;
      return run_batch<kCvDim>(ws, gs, (int)idx.size(), er.data(), ea.data(), o, g, s);
    }, coarse);
    if (rc != kOk && rc != kErrCapacity) return engine_status(ctx, rc);
  }
  st->ms_coarse = now_ms() - t0;

  // 2. training data: rule nodes of the initial grid (2^7 boxes), S per
  //    integral drawn with a seeded generator, and f there
  t0 = now_ms();
  const long long S = co.samples;
  std::vector<double> hx((size_t)count * S * kCvDim);
  unsigned long long rs = co.seed * 0x9E3779B97F4A7C15ull + 1;
  auto next = [&rs]() {
    rs = rs * 6364136223846793005ull + 1442695040888963407ull;
    return rs >> 17;
  };
  const double gen[5] = {kGenA1, kGenA2, kGenA3, kGenA4, kGenL};
  for (int e = 0; e < count; ++e)
    for (long long q = 0; q < S; ++q) {
      const int box = (int)(next() % 128), p = (int)(next() % CvPT::kPoints);
      const uint2 en = CvPT::entry(p);
      for (int i = 0; i < kCvDim; ++i) {
        const int c = (en.x >> (4 * i)) & 15;
        const double cf = c == 0 ? 0.5 : detail::coef(gen[(c - 1) >> 1], (c - 1) & 1);
        hx[((size_t)e * S + q) * kCvDim + i] = 0.5 * ((box >> i) & 1) + cf * 0.5;
      }
    }
  double *d_x = nullptr, *d_y = nullptr, *d_g = nullptr;
  if (cudaMalloc(&d_x, sizeof(double) * hx.size()) != cudaSuccess ||
      cudaMalloc(&d_y, sizeof(double) * count * S) != cudaSuccess ||
      cudaMalloc(&d_g, sizeof(double) * count * S) != cudaSuccess)
    return cuda_error(cudaErrorMemoryAllocation, "training data");
  std::unique_ptr<double, decltype(&cudaFree)> gx(d_x, cudaFree), gy(d_y, cudaFree),
      gg(d_g, cudaFree);
  cudaMemcpyAsync(d_x, hx.data(), sizeof(double) * hx.size(), cudaMemcpyHostToDevice, s);
  k_eval_points<F><<<dim3(32, 1, count), 256, 0, s>>>(d_par, d_x, S, d_y);
  if (cudaStreamSynchronize(s) != cudaSuccess) return cuda_error(cudaGetLastError(), "harvest");

  // 3. train the networks
  cub_mlp* net = cub_mlp_create(ctx->device, count, (int)S, co.batch, co.seed);
  if (!net) return CUB_ERR_CUDA;
  std::unique_ptr<cub_mlp, decltype(&cub_mlp_destroy)> net_guard(net, cub_mlp_destroy);
  int rc = cub_mlp_set_data(net, d_x, d_y);
  if (!rc) rc = cub_mlp_train(net, co.epochs, co.lr, nullptr);
  if (!rc) rc = cub_mlp_eval(net, S, d_x, d_g);
  if (rc) return rc;
  std::vector<double> hy((size_t)count * S), hg((size_t)count * S);
  cudaMemcpy(hy.data(), d_y, sizeof(double) * hy.size(), cudaMemcpyDeviceToHost);
  cudaMemcpy(hg.data(), d_g, sizeof(double) * hg.size(), cudaMemcpyDeviceToHost);
  st->ms_train = now_ms() - t0;

  // 4. per integral: residual and network integrals, or the plain method
  t0 = now_ms();
  typename CvHook<F>::Scratch scratch;
  st->fallbacks = 0;
  st->rejected = 0;
  double rho_sum = 0;
  std::vector<int> plain_idx;  // integrals the plain method integrates
  for (int k = 0; k < count; ++k) {
    double num = 0, den = 0;
    for (long long q = 0; q < S; ++q) {
      const double y = hy[(size_t)k * S + q], d = y - hg[(size_t)k * S + q];
      num += d * d;
      den += y * y;
    }
    const double rho = den > 0 ? std::sqrt(num / den) : 1.0;
    rho_sum += rho;
    const double tol = std::max(epsrel * std::fabs(coarse[k].value), epsabs);
    bool use_plain = !(rho <= co.rho_max) || coarse[k].status != 0;
    Result cv{};
    if (!use_plain) {
      const F f = F::load(h[k]);
      detail::SingleSource<F> dummy{f};
      const double half = 0.5 * tol, zero = 0.0;
      Result rr, rg;
      // a residual that does not converge within 2^20 regions (its error
      // estimate has not shrunk to the budget) stops there and the plain
      // method takes over
      Options oc = o;
      oc.max_slots = std::min<long long>(o.max_slots, 1ll << 20);
      CvHook<F> hr{net, k, f, 1.0, -1.0, half, T, sms, &scratch};
      CvHook<F> hgk{net, k, f, 0.0, 1.0, half, T, sms, &scratch};
      int r1 = run_batch<kCvDim>(ws, dummy, 1, &zero, &half, oc, &rr, s, nullptr, hr);
      int r2 = r1 == kOk ? run_batch<kCvDim>(ws, dummy, 1, &zero, &half, oc, &rg, s, nullptr, hgk)
                         : r1;
      if (r1 != kOk && r1 != kErrCapacity) {
        scratch.release();
        return engine_status(ctx, r1);
      }
      if (r2 != kOk && r2 != kErrCapacity) {
        scratch.release();
        return engine_status(ctx, r2);
      }
      if (r1 == kErrCapacity || r2 == kErrCapacity) rr.status = 1;
      st->regions_residual += rr.nregions;
      st->regions_network += rg.nregions;
      cv.value = rr.value + rg.value;
      cv.error = rr.error + rg.error;
      cv.nregions = rr.nregions + rg.nregions;
      cv.neval = rr.neval + rg.neval;
      cv.status = (rr.status || rg.status) ? 1 : 0;
      cv.iterations = rr.iterations + rg.iterations;
      cv.state = kStateDone;
      // the plain coarse run checks the result
      const bool agrees = std::fabs(cv.value - coarse[k].value) <=
                          3.0 * (coarse[k].error + cv.error) + 1e-300;
      if (cv.status != 0 || !agrees) {
        use_plain = true;
        st->rejected += 1;
      }
    }
    if (use_plain) {
      // integrated with the other fallbacks in one batch below
      st->fallbacks += 1;
      plain_idx.push_back(k);
      continue;
    }
    result_to_c(cv, &out[k]);
  }
  scratch.release();
  if (!plain_idx.empty()) {
    // the plain method on every integral that fell back, batched as
    // cub_integrate_batch would run them (groups on consecutive parameter
    // blocks of a staging copy)
    const int np = (int)plain_idx.size();
    GenzParams* d_sub = nullptr;
    if (cudaMalloc(&d_sub, sizeof(GenzParams) * np) != cudaSuccess)
      return cuda_error(cudaErrorMemoryAllocation, "fallback params");
    std::unique_ptr<GenzParams, decltype(&cudaFree)> sub_guard(d_sub, cudaFree);
    std::vector<GenzParams> hp;
    std::vector<double> per, pea;
    std::vector<Result> pres;
    const int rc = grouped_batch(np, o, [&](const std::vector<int>& idx, Result* g) {
      const int gn = (int)idx.size();
      hp.resize(gn);
      per.assign(gn, epsrel);
      pea.assign(gn, epsabs);
      for (int j = 0; j < gn; ++j) hp[j] = h[plain_idx[idx[j]]];
      if (cudaMemcpyAsync(d_sub, hp.data(), sizeof(GenzParams) * gn, cudaMemcpyHostToDevice, s) !=
          cudaSuccess)
        return (int)kErrCuda;
      detail::ParamSource<F> gs{d_sub};
      return run_batch<kCvDim>(ws, gs, gn, per.data(), pea.data(), o, g, s);
    }, pres, &ws);
    if (rc != kOk && rc != kErrCapacity) return engine_status(ctx, rc);
    for (int j = 0; j < np; ++j) result_to_c(pres[j], &out[plain_idx[j]]);
  }
  st->ms_integrate = now_ms() - t0;
  st->mean_residual_ratio = rho_sum / count;
  return 0;
}

}  // namespace

void cub_cv_default_options(cub_cv_options* o) {
  if (!o) return;
  o->samples = 8192;
  o->batch = 1024;
  o->epochs = 30;
  o->lr = 2e-3f;
  o->rho_max = 0.5;
  o->coarse_epsrel = 1e-3;
  o->seed = 1;
}

int cub_cv_integrate_batch(cub_ctx* ctx, int family, int count, const cub_genz_params* params,
                           double epsrel, double epsabs, const cub_cv_options* opt,
                           cub_result* out, cub_cv_stats* stats) {
  if (!ctx || !params || !out || count <= 0 || !(epsrel >= 0) || !(epsabs >= 0)) {
    set_error("invalid argument");
    return CUB_ERR_INVALID;
  }
  cub_cv_options co;
  cub_cv_default_options(&co);
  if (opt) co = *opt;
  if (co.batch <= 0 || co.batch % 128 || co.samples <= 0 || co.samples % co.batch) {
    set_error("cv options: batch a multiple of 128, samples a multiple of batch");
    return CUB_ERR_INVALID;
  }
  cub_cv_stats local{};
  cub_cv_stats* st = stats ? stats : &local;
  std::memset(st, 0, sizeof(*st));
  cudaError_t e = cudaSetDevice(ctx->device);
  if (e != cudaSuccess) return cuda_error(e, "cudaSetDevice");
  const GenzParams* h = reinterpret_cast<const GenzParams*>(params);
  switch (family) {
    case CUB_PRODUCT_PEAK: return cv_run<ProductPeak>(ctx, count, h, epsrel, epsabs, co, out, st);
    case CUB_GAUSSIAN: return cv_run<Gaussian>(ctx, count, h, epsrel, epsabs, co, out, st);
  }
  set_error("the control variate is built for the product-peak and Gaussian families");
  return CUB_ERR_UNSUPPORTED;
}
