// MLP surrogate for the binding-radius solve: sample generation with the
// device FP64 solver, hand-written training kernels (forward, backward,
// Adam), BF16 inference with a numrxnrate error check and exact fallback.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstring>
#include <random>
#include <string>
#include <vector>

#include "../../include/smoldyn_b200.h"
#include "devcommon.cuh"
#include "rxnparam.cuh"
#include "surrogate.h"

namespace smolb {

#define SCK(call)                                                              \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess) {                                                   \
      if (err) *err = std::string(#call) + ": " + cudaGetErrorString(e_);      \
      return -8;                                                               \
    }                                                                          \
  } while (0)

// domain of the reduced inputs
constexpr double kLogKappaLo = -5.5, kLogKappaHi = 3.1;  // a/s from ~1e-2 to ~1e2
constexpr double kRhoHi = 2.0;

struct Norm {
  float xs[3], xo[3];  // xn = (x - xo) * xs
  float ym[2], ys[2];  // yn = (y - ym) / ys
};

__device__ __forceinline__ float act(float z) { return tanhf(z); }

// Analytic reference for the reduced radius a/s at reduced rate kappa: the
// diffusion-limited radius kappa/(4 pi) (k = 4 pi D a) blended with the
// activation-limited one (3 kappa/(8 pi))^(1/3) (k dt = 4/3 pi a^3 with
// D dt / s^2 = 1/2).  The network fits the residual log10(a/s / approx),
// a narrow, smooth target.
__host__ __device__ __forceinline__ double log10_approx(double kappa) {
  const double aD = kappa / (4.0 * 3.14159265358979323846);
  const double aA = cbrt(3.0 * kappa / (8.0 * 3.14159265358979323846));
  return log10(cbrt(aD * aD * aD + aA * aA * aA));
}

// Exact samples: x = (log10 kappa, rho, rev), y = (log10 a/s, b/s) in units
// D = 1/2, dt = 1 (so s = 1 and k = kappa/2).  Non-finite solutions (rates a
// ratio < 1 placement cannot reach) are flagged with y0 = NaN.
__global__ void k_sur_samples(long long n, uint64_t seed, double *x, double *y) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const uint4 r = philox(make_uint4((uint32_t)i, (uint32_t)(i >> 32), 0x5A5A5A5Au, 1u),
                           make_uint2((uint32_t)seed, (uint32_t)(seed >> 32)));
    const double lk = kLogKappaLo + (kLogKappaHi - kLogKappaLo) * u01d(r.x);
    const bool rev = u01d(r.z) < 0.8;
    const double rho = rev ? kRhoHi * u01d(r.y) : 0.0;
    const double k = 0.5 * pow(10.0, lk);
    const double a = rxnp::bindingradius(k, 1.0, 0.5, rev ? rho : -1.0, rev ? 1 : 0);
    x[3 * i] = lk;
    x[3 * i + 1] = rho;
    x[3 * i + 2] = rev ? 1.0 : 0.0;
    const bool ok = isfinite(a) && a > 0;
    const double la = log10_approx(pow(10.0, lk));
    y[2 * i] = ok ? log10(a) - la : nan("");
    y[2 * i + 1] = ok ? (rev ? rho * a / pow(10.0, la) : 0.0) : nan("");
  }
}

constexpr int kTile = 128;  // samples per block tile in training
// Loss weight of each output.  Inference only uses output 0 (the binding
// radius; ratio placement fixes the unbinding radius as rho times it), so the
// second output is fitted with a tenth of the weight.
__constant__ float c_lossw[kMlpOut] = {1.0f, 0.1f};

// Forward + backward over one mini-batch; parameter gradients of the weighted
// mean squared error are accumulated into grad (zeroed by the caller), the
// summed loss into loss.  w is the parameter set the forward pass uses: the
// FP32 master copy, or in quantisation-aware steps its BF16-rounded copy (the
// gradient then updates the master copy: straight-through estimate).  Block: 256 threads, one tile of 128 samples at a time;
// thread t works on sample t/2, half t%2 of the 64 hidden units.
__global__ void __launch_bounds__(256) k_mlp_grad(const float *__restrict__ w, int n, const float *xn,
                                                  const float *tn, float *grad, float *loss, float inv_n) {
  extern __shared__ float sm[];
  float *H1 = sm;                     // [kTile][64]
  float *H2 = H1 + kTile * kMlpHid;   // [kTile][64] (later dZ2)
  float *X = H2 + kTile * kMlpHid;    // [kTile][3]
  float *D3 = X + kTile * kMlpIn;     // [kTile][2]
  float *G = D3 + kTile * kMlpOut;    // block gradient accumulator [kMlpNParam]
  for (int k = threadIdx.x; k < kMlpNParam; k += blockDim.x) G[k] = 0.f;
  const int t = threadIdx.x, smp = t >> 1, half = t & 1;
  float lsum = 0.f;
  for (int base = blockIdx.x * kTile; base < n; base += gridDim.x * kTile) {
    const int i = base + smp;
    const bool valid = i < n;
    __syncthreads();
    if (half == 0)
      for (int c = 0; c < kMlpIn; ++c) X[smp * kMlpIn + c] = valid ? xn[i * kMlpIn + c] : 0.f;
    __syncthreads();
    // layer 1
    for (int u = half * 32; u < half * 32 + 32; ++u) {
      float z = w[kMlpB1 + u];
      for (int c = 0; c < kMlpIn; ++c) z += w[kMlpW1 + u * kMlpIn + c] * X[smp * kMlpIn + c];
      H1[smp * kMlpHid + u] = act(z);
    }
    __syncthreads();
    // layer 2
    for (int u = half * 32; u < half * 32 + 32; ++u) {
      float z = w[kMlpB2 + u];
      const float *wr = w + kMlpW2 + u * kMlpHid;
      const float *h = H1 + smp * kMlpHid;
      for (int c = 0; c < kMlpHid; ++c) z += wr[c] * h[c];
      H2[smp * kMlpHid + u] = act(z);
    }
    __syncthreads();
    // output and its error
    {
      const int o = half;
      float z = w[kMlpB3 + o];
      for (int c = 0; c < kMlpHid; ++c) z += w[kMlpW3 + o * kMlpHid + c] * H2[smp * kMlpHid + c];
      const float e = valid ? (z - tn[i * kMlpOut + o]) : 0.f;
      lsum += c_lossw[o] * e * e;
      D3[smp * kMlpOut + o] = 2.f * c_lossw[o] * e * inv_n;
    }
    __syncthreads();
    // dW3, db3 (block partials)
    for (int k = t; k < kMlpOut * kMlpHid; k += blockDim.x) {
      const int o = k / kMlpHid, c = k % kMlpHid;
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += D3[b * kMlpOut + o] * H2[b * kMlpHid + c];
      G[kMlpW3 + k] += a;
    }
    if (t < kMlpOut) {
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += D3[b * kMlpOut + t];
      G[kMlpB3 + t] += a;
    }
    __syncthreads();
    // dZ2 = (W3^T d3) * (1 - H2^2), in place of H2
    for (int u = half * 32; u < half * 32 + 32; ++u) {
      float g = 0.f;
      for (int o = 0; o < kMlpOut; ++o) g += w[kMlpW3 + o * kMlpHid + u] * D3[smp * kMlpOut + o];
      const float h = H2[smp * kMlpHid + u];
      H2[smp * kMlpHid + u] = g * (1.f - h * h);
    }
    __syncthreads();
    // dW2[u][c] = sum_b dZ2[b][u] H1[b][c], db2
    for (int k = t; k < kMlpHid * kMlpHid; k += blockDim.x) {
      const int u = k / kMlpHid, c = k % kMlpHid;
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += H2[b * kMlpHid + u] * H1[b * kMlpHid + c];
      G[kMlpW2 + k] += a;
    }
    for (int u = t; u < kMlpHid; u += blockDim.x) {
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += H2[b * kMlpHid + u];
      G[kMlpB2 + u] += a;
    }
    __syncthreads();
    // dZ1 = (W2^T dZ2) * (1 - H1^2): each thread its half of the units
    float dz1[32];
    for (int q = 0; q < 32; ++q) {
      const int c = half * 32 + q;
      float g = 0.f;
      for (int u = 0; u < kMlpHid; ++u) g += w[kMlpW2 + u * kMlpHid + c] * H2[smp * kMlpHid + u];
      const float h = H1[smp * kMlpHid + c];
      dz1[q] = g * (1.f - h * h);
    }
    __syncthreads();
    for (int q = 0; q < 32; ++q) H1[smp * kMlpHid + half * 32 + q] = dz1[q];
    __syncthreads();
    // dW1, db1
    for (int k = t; k < kMlpHid * kMlpIn; k += blockDim.x) {
      const int u = k / kMlpIn, c = k % kMlpIn;
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += H1[b * kMlpHid + u] * X[b * kMlpIn + c];
      G[kMlpW1 + k] += a;
    }
    for (int u = t; u < kMlpHid; u += blockDim.x) {
      float a = 0.f;
      for (int b = 0; b < kTile; ++b) a += H1[b * kMlpHid + u];
      G[kMlpB1 + u] += a;
    }
  }
  __syncthreads();
  for (int k = threadIdx.x; k < kMlpNParam; k += blockDim.x)
    if (G[k] != 0.f) atomicAdd(&grad[k], G[k]);
  // loss: warp reduce then one atomic per warp
  for (int o = 16; o > 0; o >>= 1) lsum += __shfl_down_sync(0xffffffffu, lsum, o);
  if ((threadIdx.x & 31) == 0) atomicAdd(loss, lsum * inv_n);
}

// Adam step (Kingma & Ba 2015) with bias correction; also refreshes the
// BF16-rounded copy (as FP32 values) that quantisation-aware steps run on.
__global__ void k_adam(float *w, float *m, float *v, float *g, float *wq, int np, float lr, float b1,
                       float b2, float eps, float c1, float c2) {
  for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < np; k += gridDim.x * blockDim.x) {
    const float gk = g[k];
    m[k] = b1 * m[k] + (1.f - b1) * gk;
    v[k] = b2 * v[k] + (1.f - b2) * gk * gk;
    w[k] -= lr * (m[k] / c1) / (sqrtf(v[k] / c2) + eps);
    wq[k] = __bfloat162float(__float2bfloat16(w[k]));
    g[k] = 0.f;
  }
}

// Network forward for inference: BF16 weights, FP32 accumulation.
__device__ __forceinline__ void mlp_forward_bf16(const __nv_bfloat16 *w, const float x[3], float y[2]) {
  float h1[kMlpHid];
#pragma unroll 4
  for (int u = 0; u < kMlpHid; ++u) {
    float z = __bfloat162float(w[kMlpB1 + u]);
    for (int c = 0; c < kMlpIn; ++c) z += __bfloat162float(w[kMlpW1 + u * kMlpIn + c]) * x[c];
    h1[u] = act(z);
  }
  float o0 = __bfloat162float(w[kMlpB3]), o1 = __bfloat162float(w[kMlpB3 + 1]);
  for (int u = 0; u < kMlpHid; ++u) {
    float z = __bfloat162float(w[kMlpB2 + u]);
    for (int c = 0; c < kMlpHid; ++c) z += __bfloat162float(w[kMlpW2 + u * kMlpHid + c]) * h1[c];
    const float h = act(z);
    o0 += __bfloat162float(w[kMlpW3 + u]) * h;
    o1 += __bfloat162float(w[kMlpW3 + kMlpHid + u]) * h;
  }
  y[0] = o0;
  y[1] = o1;
}

// FP32-parameter forward (matches the training kernel; used for tests)
__global__ void k_mlp_forward(const float *w, int n, const float *xn, float *yn) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    float h1[kMlpHid];
    for (int u = 0; u < kMlpHid; ++u) {
      float z = w[kMlpB1 + u];
      for (int c = 0; c < kMlpIn; ++c) z += w[kMlpW1 + u * kMlpIn + c] * xn[i * kMlpIn + c];
      h1[u] = act(z);
    }
    float o0 = w[kMlpB3], o1 = w[kMlpB3 + 1];
    for (int u = 0; u < kMlpHid; ++u) {
      float z = w[kMlpB2 + u];
      for (int c = 0; c < kMlpHid; ++c) z += w[kMlpW2 + u * kMlpHid + c] * h1[c];
      const float h = act(z);
      o0 += w[kMlpW3 + u] * h;
      o1 += w[kMlpW3 + kMlpHid + u] * h;
    }
    yn[2 * i] = o0;
    yn[2 * i + 1] = o1;
  }
}

// Surrogate radii for n reactions; exact rxnp::pair_radii where the surrogate
// does not apply or its rate error estimate exceeds tol.
__global__ void k_sur_pair_radii(const __nv_bfloat16 *wg, Norm nm, long long n, const double *kf,
                                 const double *dsum, double dt, int same, int rev, int rparamt, double rparam,
                                 double tol, double *bind, double *unbind, unsigned long long *nfb) {
  __shared__ __nv_bfloat16 w[kMlpNParam];
  for (int k = threadIdx.x; k < kMlpNParam; k += blockDim.x) w[k] = wg[k];
  __syncthreads();
  const bool ratio = rev && rparamt == rxnp::kRPratio;
  const bool applies = (!rev || ratio) && rparam <= kRhoHi;
  int fb = 0;
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < n;
       i += (long long)gridDim.x * blockDim.x) {
    const double D = dsum[i];
    const double rate3 = same ? 2 * kf[i] : kf[i];
    bool exact = !applies || rate3 <= 0 || D <= 0 || dt <= 0;
    double a = 0, u = 0;
    if (!exact) {
      const double s = sqrt(2.0 * D * dt);
      const double lk = log10(rate3 / (D * s));
      if (lk < kLogKappaLo || lk > kLogKappaHi) {
        exact = true;
      } else {
        const float x[3] = {(float)((lk - nm.xo[0]) * nm.xs[0]), (float)((ratio ? rparam : 0.0) - nm.xo[1]) * nm.xs[1],
                            (float)(((ratio ? 1.0 : 0.0) - nm.xo[2]) * nm.xs[2])};
        float y[2];
        mlp_forward_bf16(w, x, y);
        a = s * pow(10.0, (double)(y[0] * nm.ys[0] + nm.ym[0]) + log10_approx(pow(10.0, lk)));
        // The tabulated per-step rate at the prediction and at a 0.1% larger
        // radius give the rate error and the local slope
        // g = dln(rate)/dln(a).  One secant step a *= (target/rate)^(1/g)
        // corrects the prediction; a third evaluation at the corrected radius
        // estimates its radius error as rate error / g.
        const double target = rate3 * dt;
        const double b0 = ratio ? rparam : -1.0;
        const double r0 = rxnp::numrxnrate(s, a, ratio ? b0 * a : -1.0);
        const double a1 = a * 1.001;
        const double r1 = rxnp::numrxnrate(s, a1, ratio ? b0 * a1 : -1.0);
        const double g = log(r1 / r0) / log(1.001);
        if (g > 0.1 && r0 > 0) a *= pow(target / r0, 1.0 / g);
        const double rc = rxnp::numrxnrate(s, a, ratio ? b0 * a : -1.0);
        const double rel = fabs(rc / target - 1.0) / fmax(g, 0.5);
        if (!(rel <= tol)) exact = true;
        else u = ratio ? rparam * a : 0.0;
      }
    }
    if (exact) {
      const rxnp::PairRadii pr = rxnp::pair_radii(kf[i], same, D, dt, rev, rparamt, rparam);
      a = pr.bindrad;
      u = pr.unbindrad;
      if (applies) fb++;
    }
    bind[i] = a;
    unbind[i] = u;
  }
  if (fb) atomicAdd(nfb, (unsigned long long)fb);
}

// ---------------------------------------------------------------------------
class SurrogateImpl {
 public:
  std::vector<float> w;  // FP32 master parameters
  Norm norm{};
  bool trained = false;
  double tol = 1e-3;
};

static int g_sm = 0;
static int sms() {
  if (!g_sm) {
    int dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&g_sm, cudaDevAttrMultiProcessorCount, dev);
    if (g_sm <= 0) g_sm = 148;
  }
  return g_sm;
}

Surrogate::Surrogate() : impl_(new SurrogateImpl) {
  // Glorot-uniform initialisation, fixed seed
  std::mt19937_64 g(12345);
  impl_->w.assign(kMlpNParam, 0.f);
  auto fill = [&](int off, int fan_in, int fan_out, int count) {
    const double lim = std::sqrt(6.0 / (fan_in + fan_out));
    std::uniform_real_distribution<double> U(-lim, lim);
    for (int k = 0; k < count; ++k) impl_->w[off + k] = (float)U(g);
  };
  fill(kMlpW1, kMlpIn, kMlpHid, kMlpHid * kMlpIn);
  fill(kMlpW2, kMlpHid, kMlpHid, kMlpHid * kMlpHid);
  fill(kMlpW3, kMlpHid, kMlpOut, kMlpOut * kMlpHid);
  Norm &nm = impl_->norm;
  nm.xo[0] = (float)(0.5 * (kLogKappaLo + kLogKappaHi));
  nm.xs[0] = (float)(2.0 / (kLogKappaHi - kLogKappaLo));
  nm.xo[1] = (float)(0.5 * kRhoHi);
  nm.xs[1] = (float)(2.0 / kRhoHi);
  nm.xo[2] = 0.5f;
  nm.xs[2] = 2.0f;
  nm.ym[0] = 0.f; nm.ys[0] = 1.f; nm.ym[1] = 0.f; nm.ys[1] = 1.f;
}
Surrogate::~Surrogate() { delete impl_; }
Surrogate::Surrogate(const Surrogate &o) : impl_(new SurrogateImpl(*o.impl_)) {}
bool Surrogate::trained() const { return impl_->trained; }
const std::vector<float> &Surrogate::params() const { return impl_->w; }
void Surrogate::set_tolerance(double t) { impl_->tol = t; }
int Surrogate::set_params(const std::vector<float> &p, std::string *err) {
  if ((int)p.size() != kMlpNParam) { if (err) *err = "wrong parameter count"; return -6; }
  impl_->w = p;
  return 0;
}

int Surrogate::samples(long long n, uint64_t seed, std::vector<double> *x, std::vector<double> *y,
                       std::string *err) {
  double *d = nullptr;
  SCK(cudaMalloc(&d, (size_t)n * 5 * sizeof(double)));
  k_sur_samples<<<sms() * 4, 128>>>(n, seed, d, d + 3 * n);
  SCK(cudaGetLastError());
  x->resize(3 * n);
  y->resize(2 * n);
  SCK(cudaMemcpy(x->data(), d, 3 * n * sizeof(double), cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(y->data(), d + 3 * n, 2 * n * sizeof(double), cudaMemcpyDeviceToHost));
  cudaFree(d);
  return 0;
}

static void normalise(const Norm &nm, long long n, const double *x, const double *y, std::vector<float> *xn,
                      std::vector<float> *tn) {
  xn->resize(3 * n);
  if (tn) tn->resize(2 * n);
  for (long long i = 0; i < n; ++i) {
    for (int c = 0; c < 3; ++c) (*xn)[3 * i + c] = (float)((x[3 * i + c] - nm.xo[c]) * nm.xs[c]);
    if (tn)
      for (int o = 0; o < 2; ++o) (*tn)[2 * i + o] = (float)((y[2 * i + o] - nm.ym[o]) / nm.ys[o]);
  }
}

int Surrogate::loss_grad(long long n, const double *x, const double *y, double *loss, std::vector<float> *grad,
                         std::string *err) {
  std::vector<float> xn, tn;
  normalise(impl_->norm, n, x, y, &xn, &tn);
  float *d = nullptr;
  const size_t np = kMlpNParam;
  SCK(cudaMalloc(&d, (np * 2 + 1 + 5 * n) * sizeof(float)));
  float *dw = d, *dg = d + np, *dl = d + 2 * np, *dx = dl + 1, *dt = dx + 3 * n;
  SCK(cudaMemcpy(dw, impl_->w.data(), np * sizeof(float), cudaMemcpyHostToDevice));
  SCK(cudaMemset(dg, 0, (np + 1) * sizeof(float)));
  SCK(cudaMemcpy(dx, xn.data(), 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dt, tn.data(), 2 * n * sizeof(float), cudaMemcpyHostToDevice));
  const size_t smem = (2 * kTile * kMlpHid + kTile * (kMlpIn + kMlpOut) + kMlpNParam) * sizeof(float);
  SCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int blocks = std::max(1, (int)std::min<long long>((n + kTile - 1) / kTile, sms() * 2));
  k_mlp_grad<<<blocks, 256, smem>>>(dw, (int)n, dx, dt, dg, dl, 1.0f / (float)n);
  SCK(cudaGetLastError());
  grad->resize(np);
  float l = 0;
  SCK(cudaMemcpy(grad->data(), dg, np * sizeof(float), cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
  *loss = l;
  cudaFree(d);
  return 0;
}

int Surrogate::forward(long long n, const double *x, double *y, std::string *err) {
  std::vector<float> xn;
  normalise(impl_->norm, n, x, nullptr, &xn, nullptr);
  float *d = nullptr;
  SCK(cudaMalloc(&d, (kMlpNParam + 5 * n) * sizeof(float)));
  float *dw = d, *dx = d + kMlpNParam, *dy = dx + 3 * n;
  SCK(cudaMemcpy(dw, impl_->w.data(), kMlpNParam * sizeof(float), cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dx, xn.data(), 3 * n * sizeof(float), cudaMemcpyHostToDevice));
  k_mlp_forward<<<sms() * 2, 128>>>(dw, (int)n, dx, dy);
  SCK(cudaGetLastError());
  std::vector<float> yn(2 * n);
  SCK(cudaMemcpy(yn.data(), dy, 2 * n * sizeof(float), cudaMemcpyDeviceToHost));
  for (long long i = 0; i < n; ++i)
    for (int o = 0; o < 2; ++o) y[2 * i + o] = yn[2 * i + o] * impl_->norm.ys[o] + impl_->norm.ym[o];
  cudaFree(d);
  return 0;
}

int Surrogate::train(long long nsamples, int epochs, int batch, double lr, uint64_t seed, SurrogateStats *st,
                     std::string *err) {
  const auto t0 = std::chrono::steady_clock::now();
  std::vector<double> x, y;
  if (samples(nsamples, seed, &x, &y, err)) return -8;
  // keep finite samples
  std::vector<double> xs, ys;
  xs.reserve(x.size());
  ys.reserve(y.size());
  for (long long i = 0; i < nsamples; ++i)
    if (std::isfinite(y[2 * i]) && std::isfinite(y[2 * i + 1])) {
      xs.insert(xs.end(), &x[3 * i], &x[3 * i + 3]);
      ys.insert(ys.end(), &y[2 * i], &y[2 * i + 2]);
    }
  const long long n = (long long)ys.size() / 2;
  if (n < 1000) { if (err) *err = "too few valid samples"; return -8; }
  // output standardisation
  Norm &nm = impl_->norm;
  for (int o = 0; o < 2; ++o) {
    double m = 0, v = 0;
    for (long long i = 0; i < n; ++i) m += ys[2 * i + o];
    m /= n;
    for (long long i = 0; i < n; ++i) v += (ys[2 * i + o] - m) * (ys[2 * i + o] - m);
    nm.ym[o] = (float)m;
    nm.ys[o] = (float)std::max(1e-6, std::sqrt(v / n));
  }
  std::vector<float> xn, tn;
  normalise(nm, n, xs.data(), ys.data(), &xn, &tn);
  const size_t np = kMlpNParam;
  float *d = nullptr;
  SCK(cudaMalloc(&d, (np * 5 + 1 + 5 * (size_t)n) * sizeof(float)));
  float *dw = d, *dm = d + np, *dv = d + 2 * np, *dg = d + 3 * np, *dwq = d + 4 * np, *dl = d + 5 * np,
        *dx = dl + 1, *dtn = dx + 3 * (size_t)n;
  SCK(cudaMemcpy(dw, impl_->w.data(), np * sizeof(float), cudaMemcpyHostToDevice));
  SCK(cudaMemset(dm, 0, np * 3 * sizeof(float)));
  SCK(cudaMemcpy(dx, xn.data(), 3 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dtn, tn.data(), 2 * (size_t)n * sizeof(float), cudaMemcpyHostToDevice));
  const size_t smem = (2 * kTile * kMlpHid + kTile * (kMlpIn + kMlpOut) + kMlpNParam) * sizeof(float);
  SCK(cudaFuncSetAttribute(k_mlp_grad, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
  const int bs = std::max(kTile, batch - batch % kTile);
  const long long nb = n / bs;
  const int blocks = bs / kTile;
  // Two phases, each with its own cosine learning-rate decay: FP32 training
  // over the first 4/5 of the epochs, then quantisation-aware steps (forward
  // and backward on the BF16-rounded weights inference uses) at a tenth of
  // the learning rate, which recovers most of the accuracy BF16 rounding
  // costs.
  const int qat_epochs = epochs >= 5 ? epochs / 5 : 0;
  const int phase_epochs[2] = {epochs - qat_epochs, qat_epochs};
  const double phase_lr[2] = {lr, 0.1 * lr};
  long long it = 0;
  SCK(cudaMemcpy(dwq, dw, np * sizeof(float), cudaMemcpyDeviceToDevice));
  for (int ph = 0; ph < 2; ++ph) {
    const long long total = (long long)phase_epochs[ph] * nb;
    const float *wfwd = ph == 0 ? dw : dwq;
    long long pit = 0;
    for (int ep = 0; ep < phase_epochs[ph]; ++ep) {
      for (long long b = 0; b < nb; ++b, ++it, ++pit) {
        const double frac = (double)pit / std::max<long long>(1, total);
        const double lr0 = phase_lr[ph];
        const float lrt = (float)(lr0 * 0.5 * (1.0 + std::cos(3.141592653589793 * frac)) + lr0 * 1e-3);
        SCK(cudaMemsetAsync(dl, 0, sizeof(float)));
        // the samples are in random order already; batches sweep them with an epoch offset
        const long long off = ((b + (long long)(ep + ph * phase_epochs[0]) * 7919) % nb) * bs;
        k_mlp_grad<<<blocks, 256, smem>>>(wfwd, bs, dx + 3 * off, dtn + 2 * off, dg, dl, 1.0f / (float)bs);
        const float c1 = 1.f - (float)std::pow(0.9, (double)(it + 1));
        const float c2 = 1.f - (float)std::pow(0.999, (double)(it + 1));
        k_adam<<<(int)((np + 255) / 256), 256>>>(dw, dm, dv, dg, dwq, (int)np, lrt, 0.9f, 0.999f, 1e-8f, c1, c2);
      }
    }
  }
  SCK(cudaGetLastError());
  // final loss over the first batches, on the BF16-rounded weights inference uses
  float l = 0;
  SCK(cudaMemset(dl, 0, sizeof(float)));
  SCK(cudaMemset(dg, 0, np * sizeof(float)));
  const long long ne = std::min<long long>(n, 65536) / kTile * kTile;
  k_mlp_grad<<<std::max(1, (int)(ne / kTile)), 256, smem>>>(dwq, (int)ne, dx, dtn, dg, dl, 1.0f / (float)ne);
  SCK(cudaMemcpy(&l, dl, sizeof(float), cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(impl_->w.data(), dw, np * sizeof(float), cudaMemcpyDeviceToHost));
  cudaFree(d);
  impl_->trained = true;
  if (st) {
    st->final_loss = l;
    st->samples = n;
    st->epochs = epochs;
    st->train_seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
  return 0;
}

int Surrogate::pair_radii(long long n, const double *kf, const double *dsum, double dt, int same, int rev,
                          int rparamt, double rparam, double *bind, double *unbind, long long *nfallback,
                          std::string *err) {
  if (n <= 0) return 0;
  std::vector<__nv_bfloat16> wb(kMlpNParam);
  for (int k = 0; k < kMlpNParam; ++k) wb[k] = __float2bfloat16(impl_->w[k]);
  if (rev && rparamt == rxnp::kRPnone) {  // default placement of a reversible pair
    rparamt = rxnp::kRPpgemmaxw;
    rparam = 0.2;
  }
  double *d = nullptr;
  __nv_bfloat16 *dwb = nullptr;
  unsigned long long *dfb = nullptr;
  SCK(cudaMalloc(&d, (size_t)n * 4 * sizeof(double)));
  SCK(cudaMalloc(&dwb, kMlpNParam * sizeof(__nv_bfloat16)));
  SCK(cudaMalloc(&dfb, sizeof(unsigned long long)));
  SCK(cudaMemcpy(d, kf, n * sizeof(double), cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(d + n, dsum, n * sizeof(double), cudaMemcpyHostToDevice));
  SCK(cudaMemcpy(dwb, wb.data(), kMlpNParam * sizeof(__nv_bfloat16), cudaMemcpyHostToDevice));
  SCK(cudaMemset(dfb, 0, sizeof(unsigned long long)));
  k_sur_pair_radii<<<sms() * 2, 128>>>(dwb, impl_->norm, n, d, d + n, dt, same, rev, rparamt, rparam, impl_->tol,
                                       d + 2 * n, d + 3 * n, dfb);
  SCK(cudaGetLastError());
  SCK(cudaMemcpy(bind, d + 2 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  SCK(cudaMemcpy(unbind, d + 3 * n, n * sizeof(double), cudaMemcpyDeviceToHost));
  unsigned long long fb = 0;
  SCK(cudaMemcpy(&fb, dfb, sizeof(fb), cudaMemcpyDeviceToHost));
  if (nfallback) *nfallback = (long long)fb;
  cudaFree(d);
  cudaFree(dwb);
  cudaFree(dfb);
  return 0;
}

}  // namespace smolb

// ---- C API ------------------------------------------------------------------
struct smolb_surrogate {
  smolb::Surrogate s;
};

ErrorCode smolb_record_error(const char *, ErrorCode, const std::string &);

smolb::Surrogate *smolb_surrogate_clone(surptr p) { return new smolb::Surrogate(p->s); }

extern "C" {

surptr smolgpuSurrogateNew(void) { return new smolb_surrogate(); }

enum ErrorCode smolgpuSurrogateFree(surptr sur) {
  delete sur;
  return ECok;
}

enum ErrorCode smolgpuSurrogateTrain(surptr sur, long long nsamples, int epochs, int batch, double lr,
                                     unsigned long long seed, double *final_loss, double *seconds) {
  if (!sur) return smolb_record_error(__func__, ECmissing, "missing surrogate");
  if (nsamples < 1000 || epochs < 1 || batch < 128 || !(lr > 0))
    return smolb_record_error(__func__, ECbounds, "nsamples>=1000, epochs>=1, batch>=128, lr>0 required");
  smolb::SurrogateStats st;
  std::string err;
  if (sur->s.train(nsamples, epochs, batch, lr, seed, &st, &err)) return smolb_record_error(__func__, ECerror, err);
  if (final_loss) *final_loss = st.final_loss;
  if (seconds) *seconds = st.train_seconds;
  return ECok;
}

enum ErrorCode smolgpuSurrogateSamples(surptr sur, long long n, unsigned long long seed, double *x, double *y) {
  if (!sur || !x || !y) return smolb_record_error(__func__, ECmissing, "missing argument");
  std::vector<double> xs, ys;
  std::string err;
  if (sur->s.samples(n, seed, &xs, &ys, &err)) return smolb_record_error(__func__, ECerror, err);
  memcpy(x, xs.data(), xs.size() * sizeof(double));
  memcpy(y, ys.data(), ys.size() * sizeof(double));
  return ECok;
}

enum ErrorCode smolgpuSurrogateForward(surptr sur, long long n, const double *x, double *y) {
  if (!sur || !x || !y) return smolb_record_error(__func__, ECmissing, "missing argument");
  std::string err;
  if (sur->s.forward(n, x, y, &err)) return smolb_record_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuSurrogateLossGrad(surptr sur, long long n, const double *x, const double *y, double *loss,
                                        float *grad) {
  if (!sur || !x || !y || !loss || !grad) return smolb_record_error(__func__, ECmissing, "missing argument");
  std::vector<float> g;
  std::string err;
  if (sur->s.loss_grad(n, x, y, loss, &g, &err)) return smolb_record_error(__func__, ECerror, err);
  memcpy(grad, g.data(), g.size() * sizeof(float));
  return ECok;
}

int smolgpuSurrogateParamCount(void) { return smolb::kMlpNParam; }

enum ErrorCode smolgpuSurrogateGetParams(surptr sur, float *params) {
  if (!sur || !params) return smolb_record_error(__func__, ECmissing, "missing argument");
  memcpy(params, sur->s.params().data(), smolb::kMlpNParam * sizeof(float));
  return ECok;
}

enum ErrorCode smolgpuSurrogateSetParams(surptr sur, const float *params) {
  if (!sur || !params) return smolb_record_error(__func__, ECmissing, "missing argument");
  std::string err;
  if (sur->s.set_params(std::vector<float>(params, params + smolb::kMlpNParam), &err))
    return smolb_record_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuSurrogateSetTolerance(surptr sur, double tol) {
  if (!sur) return smolb_record_error(__func__, ECmissing, "missing surrogate");
  sur->s.set_tolerance(tol);
  return ECok;
}

enum ErrorCode smolgpuSurrogatePairRadii(surptr sur, long long n, const double *kf, const double *dsum, double dt,
                                         int same, int rev, int rparamt, double rparam, double *bind,
                                         double *unbind, long long *nfallback) {
  if (!sur || !kf || !dsum || !bind || !unbind) return smolb_record_error(__func__, ECmissing, "missing argument");
  if (!sur->s.trained()) return smolb_record_error(__func__, ECerror, "surrogate not trained");
  std::string err;
  if (sur->s.pair_radii(n, kf, dsum, dt, same, rev, rparamt, rparam, bind, unbind, nfallback, &err))
    return smolb_record_error(__func__, ECerror, err);
  return ECok;
}

}  // extern "C"
