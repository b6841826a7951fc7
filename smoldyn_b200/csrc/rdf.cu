// Radial-distribution-function solver on the device: the numerical method
// that produced the rxnparam lookup tables (rxnparam.c:726-1114).
//
// A steady state alternates two operators on a radial profile g(r) of the
// partner density around one reactant (unit binding radius a, grid of n
// radii): one diffusion step of rms length s, a convolution with the radial
// Green's function plus a 1 + a2/r tail beyond the grid (rdfdiffuse,
// rxnparam.c:819-857), optionally the diffused image of the reverse
// reaction's source at the unbinding radius b (rdfreverserxn, 869-882), then
// absorption of probability `prob` of everything inside a (rdfabsorb,
// 784-802).  The absorbed amount per step converges to the reduced reaction
// rate tabulated in numrxnrate and numrxnrateprob.  A sweep (rdfmaketable,
// 920-1005; rdfmaketableprob, 1008-1114) solves 31 step lengths in order,
// each starting from the previous steady state.
//
// Layout: one thread-block cluster per sweep.  Every CTA of the cluster keeps
// the radii and full copies of both profiles in shared memory (6 n doubles);
// CTA `rank` computes the diffused values of its own slice of radii (one warp
// per radius, the lanes over the source radii with the trapezoid segments
// stitched across lanes by shuffles) and the slices are exchanged through
// distributed shared memory.  The diffusion step is n^2 Gaussian evaluations
// per iteration in FP64, so the sweep is bound by FP64 issue; pairs whose
// Gaussians underflow to zero skip the exponentials.
//
// Every CTA of a cluster runs the same number of iterations by construction:
// the loop decisions use only the flux published by CTA rank 0, read by all
// after a cluster barrier, and the iteration count is capped (100000, as in
// rxnparam.c:899).  Cluster barriers are the only waits.
#include <cooperative_groups.h>
#include <cuda_runtime.h>

#include <cmath>
#include <string>
#include <vector>

#include "../../include/smoldyn_b200.h"

ErrorCode smolb_record_error(const char *, ErrorCode, const std::string &);

namespace cg = cooperative_groups;

namespace smolb {
namespace {

constexpr double kPi = 3.14159265358979323846;
constexpr double kSqrt2Pi = 2.50662827462;  // the reference's literal (math2.h:14)
constexpr int kThreads = 512;  // block size limit; 256 when the sweeps need two waves of CTAs
constexpr int kMaxN = 4000;
constexpr int kMaxSteps = 64;
constexpr int kMaxIt = 100000;
constexpr double kMaxFlux = 1e7;
// exp(-x) is exactly 0 in FP64 for x > 745.2; pairs with (rr - r')^2 / 2
// above 750 contribute nothing and skip both exponentials.
constexpr double kZeroArg2 = 1500.0;
// exp(-(rr + r')^2/2) <= 2^-54 exp(-(rr - r')^2/2) once 2 rr r' >= 37.5, so
// the difference equals its first term exactly and the second is skipped.
constexpr double kSecondTerm = 40.0;
constexpr double kInvG1 = 1.0 / (4.0 * kPi * kSqrt2Pi);

struct RdfChain {
  const double *r;      // n radii: r[0] >= 0, the others > 0
  double *rdfa;         // n: trial profile in; profile after the last absorption out
  double *rdfd;         // n: profile after the last diffusion step out
  const double *steps;  // nsteps rms step lengths, solved in this order
  double *flux;         // nsteps steady-state fluxes (-1: no convergence)
  int *iters;           // nsteps iteration counts
  int nsteps;
  double a, b, prob;    // binding radius, unbinding radius (< 0: irreversible), probability
};

__device__ __forceinline__ double shell(double r0, double r1, double f0, double f1) {
  // 4 pi r^2 integral of the linear interpolant of (r0,f0)-(r1,f1) (rxnparam.c:771-776)
  return kPi * (f1 - f0) * (r1 + r0) * (r1 * r1 + r0 * r0) +
         4.0 * kPi / 3.0 * (r1 * f0 - r0 * f1) * (r1 * r1 + r1 * r0 + r0 * r0);
}

// Complementary error function by the Chebyshev fit of Numerical Recipes in
// C (2nd ed., section 6.2, "erfcc"; fractional error below 1.2e-7): the form
// the reference's tables were computed with (rxnparam.c:719-724).
__device__ double erfc_nr(double x) {
  const double z = fabs(x), t = 1.0 / (1.0 + 0.5 * z);
  double p = 0.17087277;
  p = -0.82215223 + t * p;
  p = 1.48851587 + t * p;
  p = -1.13520398 + t * p;
  p = 0.27886807 + t * p;
  p = -0.18628806 + t * p;
  p = 0.09678418 + t * p;
  p = 0.37409196 + t * p;
  p = 1.00002368 + t * p;
  const double v = t * exp(-z * z - 1.26551223 + t * p);
  return x >= 0.0 ? v : 2.0 - v;
}

// (g(r') - g(r)) times the radial Green's function between reduced radii rr
// and x (rxnparam.c:845): [e^{-(rr-x)^2/2} - e^{-(rr+x)^2/2}] / (4 pi sqrt(2 pi) rr x).
__device__ __forceinline__ double green_term(double rr, double irr, double x, double ix, double dg) {
  const double dm = rr - x;
  if (dm * dm > kZeroArg2) return 0.0;
  double e = exp(-dm * dm / 2.0);
  if (2.0 * rr * x < kSecondTerm) {
    const double sp = rr + x;
    e -= exp(-sp * sp / 2.0);
  }
  return dg * (irr * ix * e * kInvG1);
}

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

struct Shared {
  double *r, *rs, *irs, *fa, *fd, *term;
};

// Absorption (rxnparam.c:784-802) on this CTA's copy of `f`: the shells from
// the origin to the first grid point at or past a (points j0..jl), minus the
// last shell's upper-left triangle, times prob; points below jl keep 1-prob.
// Returns the flux in thread 0 (other threads: unspecified).
__device__ double absorb(const Shared &S, double *f, int j0, int jl, bool runs, double prob) {
  const int tid = threadIdx.x;
  if (runs)
    for (int j = j0 + tid; j <= jl; j += blockDim.x) {
      const double r0 = j == j0 ? 0.0 : S.r[j - 1], f0 = j == j0 ? f[0] : f[j - 1];
      S.term[j] = shell(r0, S.r[j], f0, f[j]);
    }
  __syncthreads();
  double sum = 0.0;
  if (tid < 32) {
    if (runs)
      for (int j = j0 + tid; j <= jl; j += 32) sum += S.term[j];
    sum = warp_sum(sum);
    const double r0 = !runs || jl == j0 ? 0.0 : S.r[jl - 1], r1 = runs ? S.r[jl] : 0.0,
                 f1 = runs ? f[jl] : f[0];
    sum -= shell(r0, r1, 0.0, f1);
    sum *= prob;
  } else {
    const int top = runs ? jl - 1 : j0 - 2;  // reference: rdf[j] for j <= (index after loop) - 2
    for (int k = tid - 32; k <= top; k += blockDim.x - 32) f[k] *= 1.0 - prob;
  }
  __syncthreads();
  return sum;
}

// One diffusion step of the profile fa into fd for this CTA's radii [lo, hi)
// (rxnparam.c:819-857), then the reverse-reaction source on the same radii
// when b >= 0 (rxnparam.c:869-882).
__device__ void diffuse_slice(const Shared &S, int n, int lo, int hi, int j0, double alpha, double step, double b,
                              double flux, double *s_a2) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarp = blockDim.x >> 5;
  const double g0 = 2.0 * kPi * kSqrt2Pi, g1 = 4.0 * kPi * kSqrt2Pi;
  if (warp == 0) {  // tail fit 1 + a2/r over the top 10% of the radii
    double beta = 0.0;
    for (int i = (int)(0.9 * n) + lane; i < n; i += 32) beta += (S.fa[i] - 1.0) / S.r[i];
    beta = warp_sum(beta);
    if (lane == 0) *s_a2 = beta / alpha / step;
  }
  __syncthreads();
  const double a2 = *s_a2;
  const double rlast = S.rs[n - 1];
  for (int i = lo + warp; i < hi; i += nwarp) {
    const double fai = S.fa[i];
    double acc = 0.0;
    if (i == 0 && S.r[0] == 0) {
      // r = 0: Green's function exp(-r'^2/2) / (2 pi sqrt(2 pi)) in reduced units
      double cx = 0.0, cf = 0.0;
      for (int base = 1; base < n; base += 32) {
        const int j = base + lane;
        double x = 0.0, f = 0.0;
        if (j < n) {
          x = S.rs[j];
          f = x * x > kZeroArg2 ? 0.0 : (S.fa[j] - fai) * (exp(-x * x / 2.0) / g0);
        }
        double px = __shfl_up_sync(0xffffffffu, x, 1), pf = __shfl_up_sync(0xffffffffu, f, 1);
        if (lane == 0) {
          px = cx;
          pf = cf;
        }
        if (j < n) acc += shell(px, x, pf, f);
        cx = __shfl_sync(0xffffffffu, x, 31);
        cf = __shfl_sync(0xffffffffu, f, 31);
      }
      acc = warp_sum(acc);
      if (lane == 0) {
        const double grn = exp(-rlast * rlast / 2.0) / g0;
        acc += (1.0 - fai) * (4.0 * kPi * rlast * grn + erfc_nr(rlast / sqrt(2.0)));
        S.fd[0] = acc + fai;
      }
    } else {
      const double rr = S.rs[i], irr = S.irs[i];
      double cx = 0.0, cf = (S.fa[0] - fai) * (exp(-rr * rr / 2.0) / g0);
      for (int base = j0; base < n; base += 64) {  // two points per lane: independent exponentials
        const int ja = base + 2 * lane, jb = ja + 1;
        double xa = 0.0, fa = 0.0, xb = 0.0, fb = 0.0;
        if (ja < n) {
          xa = S.rs[ja];
          fa = green_term(rr, irr, xa, S.irs[ja], S.fa[ja] - fai);
        }
        if (jb < n) {
          xb = S.rs[jb];
          fb = green_term(rr, irr, xb, S.irs[jb], S.fa[jb] - fai);
        }
        double px = __shfl_up_sync(0xffffffffu, xb, 1), pf = __shfl_up_sync(0xffffffffu, fb, 1);
        if (lane == 0) {
          px = cx;
          pf = cf;
        }
        if (ja < n) acc += shell(px, xa, pf, fa);
        if (jb < n) acc += shell(xa, xb, fa, fb);
        cx = __shfl_sync(0xffffffffu, xb, 31);
        cf = __shfl_sync(0xffffffffu, fb, 31);
      }
      acc = warp_sum(acc);
      if (lane == 0) {
        const double r1 = rlast;
        const double grn = 1.0 / rr / r1 *
                           (exp(-(rr - r1) * (rr - r1) / 2.0) - exp(-(rr + r1) * (rr + r1) / 2.0)) / g1;
        const double ed = erfc_nr((r1 - rr) / sqrt(2.0)), es = erfc_nr((r1 + rr) / sqrt(2.0));
        acc += (1.0 - fai) * (4.0 * kPi * r1 * grn + 1.0 / 2.0 * (ed + es)) + a2 / 2.0 / rr * (ed - es);
        S.fd[i] = acc + fai;
      }
    }
  }
  if (b >= 0) {
    __syncwarp();
    __syncthreads();
    const double k = 1.0 / (4.0 * kPi * kSqrt2Pi * step * step * step);
    const double bs = b / step;
    for (int i = lo + tid; i < hi; i += blockDim.x) {
      const double rr = S.rs[i];
      if (b == 0)
        S.fd[i] += flux * k * 2.0 * exp(-rr * rr / 2.0);
      else if (i == 0 && S.r[0] == 0)
        S.fd[i] += flux * k * 2.0 * exp(-bs * bs / 2.0);
      else
        S.fd[i] += flux * k / rr / bs * (exp(-(rr - bs) * (rr - bs) / 2.0) - exp(-(rr + bs) * (rr + bs) / 2.0));
    }
  }
}

// One cluster per sweep (chain).  Dynamic shared memory: 6 n doubles.
__global__ void __launch_bounds__(kThreads) k_rdf_sweep(const RdfChain *chains, int n, double eps) {
  cg::cluster_group cl = cg::this_cluster();
  const int cs = (int)cl.num_blocks(), rank = (int)cl.block_rank();
  const RdfChain ch = chains[blockIdx.x / cs];
  extern __shared__ double sm[];
  Shared S{sm, sm + n, sm + 2 * n, sm + 3 * n, sm + 4 * n, sm + 5 * n};
  __shared__ double s_a2, s_pub, s_alpha;
  __shared__ int s_j0, s_jl, s_runs;
  const int tid = threadIdx.x;
  const int lo = (int)((long long)n * rank / cs), hi = (int)((long long)n * (rank + 1) / cs);

  for (int i = tid; i < n; i += blockDim.x) {
    S.r[i] = ch.r[i];
    S.fa[i] = ch.rdfa[i];
  }
  __syncthreads();
  if (tid == 0) {
    const int j0 = S.r[0] == 0 ? 1 : 0;
    int jl = j0;
    while (jl < n - 1 && S.r[jl] < ch.a) ++jl;
    s_j0 = j0;
    s_jl = jl;
    s_runs = (ch.a > 0 && j0 < n) ? 1 : 0;
    double alpha = 0.0;
    for (int i = (int)(0.9 * n); i < n; ++i) alpha += 1.0 / S.r[i] / S.r[i];
    s_alpha = alpha;
  }
  __syncthreads();
  const int j0 = s_j0, jl = s_jl;
  const bool runs = s_runs != 0;
  const double alpha = s_alpha;
  double *pub0 = cl.map_shared_rank(&s_pub, 0);

  // diffusion of fa into fd over the whole cluster, then every CTA's fd is full
  auto diffuse_all = [&](double step, double bsrc, double flux) {
    diffuse_slice(S, n, lo, hi, j0, alpha, step, bsrc, flux, &s_a2);
    cl.sync();
    for (int q = 0; q < cs; ++q) {
      if (q == rank) continue;
      const double *remote = cl.map_shared_rank(S.fd, q);
      const int qlo = (int)((long long)n * q / cs), qhi = (int)((long long)n * (q + 1) / cs);
      for (int i = qlo + tid; i < qhi; i += blockDim.x) S.fd[i] = remote[i];
    }
    __syncthreads();
  };
  // absorption on this CTA's copy; every CTA continues with rank 0's flux
  auto absorb_all = [&](double *f) {
    const double v = absorb(S, f, j0, jl, runs, ch.prob);
    if (rank == 0 && tid == 0) s_pub = v;
    cl.sync();
    const double flux = *pub0;
    return flux;
  };

  bool failed = false;
  for (int k = 0; k < ch.nsteps; ++k) {
    if (failed) {
      if (rank == 0 && tid == 0) {
        ch.flux[k] = -1.0;
        ch.iters[k] = 0;
      }
      continue;
    }
    const double step = ch.steps[k];
    for (int i = tid; i < n; i += blockDim.x) {
      S.rs[i] = S.r[i] / step;
      S.irs[i] = S.rs[i] > 0 ? 1.0 / S.rs[i] : 0.0;
    }
    __syncthreads();
    // rxnparam.c:898-912
    diffuse_all(step, -1.0, 0.0);
    cl.sync();  // every CTA has copied the slices before fd is absorbed in place
    double flux = absorb_all(S.fd), fluxold = flux;
    int it = 0;
    while (it < 30 || (it < kMaxIt && flux < kMaxFlux && fabs((flux - fluxold) / (fluxold + 1e-20)) > eps)) {
      fluxold = flux;
      diffuse_all(step, ch.b, flux);
      for (int i = tid; i < n; i += blockDim.x) S.fa[i] = S.fd[i];
      __syncthreads();
      flux = absorb_all(S.fa);
      ++it;
    }
    if (it >= kMaxIt || flux >= kMaxFlux) {
      flux = -1.0;
      failed = true;
    }
    if (rank == 0 && tid == 0) {
      ch.flux[k] = flux;
      ch.iters[k] = it;
    }
  }
  if (rank == 0)
    for (int i = tid; i < n; i += blockDim.x) {
      ch.rdfa[i] = S.fa[i];
      ch.rdfd[i] = S.fd[i];
    }
  cl.sync();  // no CTA leaves while another may still read its shared memory
}

template <class T>
struct DevBuf {
  T *p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
  cudaError_t alloc(size_t count) { return cudaMalloc(&p, count * sizeof(T) + 16); }
};

// Launch the chains: the cluster size is the largest of 8, 4, 2, 1 that keeps
// the grid within one wave of the GPU and that the device can co-schedule.
int run_chains(std::vector<RdfChain> &chains, int n, double eps, cudaStream_t st, std::string *err) {
  if (chains.empty()) return 0;
  const size_t smem = (size_t)6 * n * sizeof(double);
  cudaError_t e = cudaFuncSetAttribute(k_rdf_sweep, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
  if (e != cudaSuccess) {
    *err = std::string("rdf solver: ") + cudaGetErrorString(e);
    return -1;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  DevBuf<RdfChain> dch;
  if ((e = dch.alloc(chains.size())) != cudaSuccess ||
      (e = cudaMemcpyAsync(dch.p, chains.data(), chains.size() * sizeof(RdfChain), cudaMemcpyHostToDevice, st)) !=
          cudaSuccess) {
    *err = std::string("rdf solver: ") + cudaGetErrorString(e);
    return -1;
  }
  // clusters above 8 CTAs need the non-portable opt-in; if the device
  // refuses it, sizes above 8 simply fail the occupancy check below
  if (cudaFuncSetAttribute(k_rdf_sweep, cudaFuncAttributeNonPortableClusterSizeAllowed, 1) != cudaSuccess)
    cudaGetLastError();
  const long long nch = (long long)chains.size();
  // Cluster size: the largest of 16, 8, 4, 2, 1 whose grid is resident in one
  // wave, either with 512 threads per CTA (one CTA per SM at this register
  // count) or with 256 (two CTAs per SM).  The larger cluster wins, 512
  // threads on a tie; beyond two sweeps per SM, single CTAs of 256 threads.
  int cs_one = 16;
  while (cs_one > 0 && nch * cs_one > sms) cs_one >>= 1;
  int cs_two = 16;
  while (cs_two > 1 && nch * cs_two > 2 * sms) cs_two >>= 1;
  int cs = cs_one >= cs_two ? cs_one : cs_two;
  const int threads = cs_one >= cs_two ? kThreads : kThreads / 2;
  for (;; cs >>= 1) {
    cudaLaunchConfig_t cfg = {};
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = cs;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.gridDim = dim3((unsigned)(nch * cs));
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    int nclusters = 0;
    e = cudaOccupancyMaxActiveClusters(&nclusters, k_rdf_sweep, &cfg);
    if ((e != cudaSuccess || nclusters < 1) && cs > 1) {
      cudaGetLastError();
      continue;
    }
    if (e != cudaSuccess || nclusters < 1) {
      *err = std::string("rdf solver: cannot schedule ") + (e != cudaSuccess ? cudaGetErrorString(e) : "a cluster");
      return -1;
    }
    const RdfChain *arg = dch.p;
    e = cudaLaunchKernelEx(&cfg, k_rdf_sweep, arg, n, eps);
    break;
  }
  if (e == cudaSuccess) e = cudaStreamSynchronize(st);
  if (e != cudaSuccess) {
    *err = std::string("rdf solver: ") + cudaGetErrorString(e);
    return -1;
  }
  return 0;
}

// Radial grid of the table sweeps (rxnparam.c:965-971): steps of dr from 0
// with the point at 1 replaced by the pair 0.9999, 1.0001; rmax 10 (mode
// 'i'), b+3 ('r'), 5 ('b').
bool table_grid(char mode, int n, double b, double *r) {
  const double dr = mode == 'i' ? 10.0 / n : mode == 'r' ? (b + 3.0) / n : 5.0 / n;
  int i = 1;
  r[0] = 0;
  while (r[i - 1] < 1 && i < n) {
    r[i] = r[i - 1] + dr;
    ++i;
  }
  if (r[i - 1] < 1 || i >= n) return false;
  r[i - 1] = 0.9999;
  r[i++] = 1.0001;
  for (; i < n; ++i) r[i] = r[i - 1] + dr;
  return true;
}

// Rows of a sweep (rxnparam.c:921-923, 996-1004): one row for 'i'; b = 1,
// e^0.2, ... e^3 for 'r'; b = 0, 0.1, ... 1 for 'b'.
std::vector<double> table_rows(char mode) {
  std::vector<double> b;
  if (mode == 'i') {
    b.push_back(-1);
  } else if (mode == 'r') {
    const double bincr = exp(0.2), bhi = exp(3.0);
    for (double v = exp(0.0); !(v > bhi * sqrt(bincr)); v *= bincr) b.push_back(v);
  } else {
    for (double v = 0; !(v > 1.0 + 0.1 / 2.0); v += 0.1) b.push_back(v);
  }
  return b;
}

// Step lengths of a sweep in order (rxnparam.c:921, 948-951, 987).
std::vector<double> table_steps(char dir) {
  double slo = exp(-3.0), shi = exp(3.0), sinc = exp(0.2), s;
  if (dir == 'd') {
    s = slo;
    slo = shi;
    shi = s;
    sinc = 1.0 / sinc;
  }
  std::vector<double> v;
  for (s = slo; slo < shi ? s < shi * sqrt(sinc) : s > shi * sqrt(sinc); s *= sinc) v.push_back(s);
  return v;
}

}  // namespace

int rdf_table_device(char mode, int n, double eps, char dir, int nprob, const double *probs, double *flux,
                     int *iters, int *nrows, std::string *err) {
  const std::vector<double> rows = table_rows(mode);
  const double one = 1.0;
  if (!probs) {
    probs = &one;
    nprob = 1;
  }
  std::vector<char> dirs;
  if (dir == 'a') {
    dirs = {'u', 'd'};
  } else {
    dirs = {dir};
  }
  const std::vector<double> su = table_steps('u'), sd = table_steps('d');
  const int ns = (int)su.size();
  if (ns != (int)sd.size() || ns > kMaxSteps) {
    *err = "rdf table: step sweep length";
    return -1;
  }
  const int nr = (int)rows.size();
  std::vector<double> hr((size_t)nr * n);
  for (int row = 0; row < nr; ++row)
    if (!table_grid(mode, n, rows[row], &hr[(size_t)row * n])) {
      *err = "rdf table: too few radial points to reach the binding radius";
      return -1;
    }
  // chain list: (row, prob, direction) with prob > 0
  struct Tag {
    int row, p, d;
  };
  std::vector<Tag> tags;
  for (int row = 0; row < nr; ++row)
    for (int p = 0; p < nprob; ++p)
      if (probs[p] != 0)
        for (int d = 0; d < (int)dirs.size(); ++d) tags.push_back({row, p, d});
  const size_t nch = tags.size();
  std::vector<double> ha(nch * n);
  for (size_t c = 0; c < nch; ++c) {
    const double *r = &hr[(size_t)tags[c].row * n];
    double *g = &ha[c * n];
    const double b = rows[tags[c].row];
    const char dc = dirs[tags[c].d];
    int i = 0;
    for (; i < n && r[i] < 1; ++i) g[i] = 0;
    if (dc == 'u' && mode == 'i')
      for (; i < n; ++i) g[i] = 1.0 - 1.0 / r[i];
    else if (dc == 'u' && mode == 'r')
      for (; i < n && r[i] < b; ++i) g[i] = 1.0 - (b - r[i]) / r[i] / (b - 1.0);
    for (; i < n; ++i) g[i] = 1.0;
  }
  cudaStream_t st = nullptr;
  DevBuf<double> dr, da, dd, dsu, dsd, dflux;
  DevBuf<int> dit;
  cudaError_t e;
  if ((e = dr.alloc(hr.size())) || (e = da.alloc(nch * n + 1)) || (e = dd.alloc(nch * n + 1)) ||
      (e = dsu.alloc(ns)) || (e = dsd.alloc(ns)) || (e = dflux.alloc(nch * ns + 1)) || (e = dit.alloc(nch * ns + 1)) ||
      (e = cudaMemcpyAsync(dr.p, hr.data(), hr.size() * sizeof(double), cudaMemcpyHostToDevice, st)) ||
      (nch && (e = cudaMemcpyAsync(da.p, ha.data(), ha.size() * sizeof(double), cudaMemcpyHostToDevice, st))) ||
      (e = cudaMemcpyAsync(dsu.p, su.data(), ns * sizeof(double), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(dsd.p, sd.data(), ns * sizeof(double), cudaMemcpyHostToDevice, st))) {
    *err = std::string("rdf table: ") + cudaGetErrorString(e);
    return -1;
  }
  std::vector<RdfChain> chains(nch);
  for (size_t c = 0; c < nch; ++c) {
    RdfChain &ch = chains[c];
    ch.r = dr.p + (size_t)tags[c].row * n;
    ch.rdfa = da.p + c * n;
    ch.rdfd = dd.p + c * n;
    ch.steps = dirs[tags[c].d] == 'u' ? dsu.p : dsd.p;
    ch.flux = dflux.p + c * ns;
    ch.iters = dit.p + c * ns;
    ch.nsteps = ns;
    ch.a = 1.0;
    ch.b = rows[tags[c].row];
    ch.prob = probs[tags[c].p];
  }
  if (run_chains(chains, n, eps, st, err)) return -1;
  std::vector<double> hf(nch * ns);
  std::vector<int> hi(nch * ns);
  if (nch && ((e = cudaMemcpy(hf.data(), dflux.p, hf.size() * sizeof(double), cudaMemcpyDeviceToHost)) ||
              (e = cudaMemcpy(hi.data(), dit.p, hi.size() * sizeof(int), cudaMemcpyDeviceToHost)))) {
    *err = std::string("rdf table: ") + cudaGetErrorString(e);
    return -1;
  }
  // assemble [row][prob][k]; 'a' averages the upward sweep (reversed) and
  // the downward sweep, in decreasing step order
  const size_t nout = (size_t)nr * nprob * ns;
  for (size_t o = 0; o < nout; ++o) {
    flux[o] = 0.0;
    if (iters) iters[o] = 0;
  }
  for (size_t c = 0; c < nch; ++c) {
    const size_t base = ((size_t)tags[c].row * nprob + tags[c].p) * ns;
    const bool up = dirs[tags[c].d] == 'u';
    for (int k = 0; k < ns; ++k) {
      const int ko = (dir == 'a' && up) ? ns - 1 - k : k;
      const double v = hf[c * ns + k];
      if (dir == 'a') {
        if (tags[c].d == 0) {
          flux[base + ko] = v;
        } else {
          const double u = flux[base + ko];
          flux[base + ko] = (u < 0 || v < 0) ? -1.0 : (u + v) / 2.0;
        }
      } else {
        flux[base + ko] = v;
      }
      if (iters) iters[base + ko] += hi[c * ns + k];
    }
  }
  if (nrows) *nrows = nr;
  return 0;
}

int rdf_steady_device(int nsolve, int n, const double *r, double *rdfa, double *rdfd, const double *step,
                      const double *a, const double *b, const double *prob, double eps, double *flux, int *iters,
                      std::string *err) {
  if (nsolve == 0) return 0;
  cudaStream_t st = nullptr;
  const size_t nn = (size_t)nsolve * n;
  DevBuf<double> dr, da, dd, ds, dflux;
  DevBuf<int> dit;
  cudaError_t e;
  if ((e = dr.alloc(nn)) || (e = da.alloc(nn)) || (e = dd.alloc(nn)) || (e = ds.alloc(nsolve)) ||
      (e = dflux.alloc(nsolve)) || (e = dit.alloc(nsolve)) ||
      (e = cudaMemcpyAsync(dr.p, r, nn * sizeof(double), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(da.p, rdfa, nn * sizeof(double), cudaMemcpyHostToDevice, st)) ||
      (e = cudaMemcpyAsync(ds.p, step, nsolve * sizeof(double), cudaMemcpyHostToDevice, st))) {
    *err = std::string("rdf steady state: ") + cudaGetErrorString(e);
    return -1;
  }
  std::vector<RdfChain> chains(nsolve);
  for (int c = 0; c < nsolve; ++c) {
    RdfChain &ch = chains[c];
    ch.r = dr.p + (size_t)c * n;
    ch.rdfa = da.p + (size_t)c * n;
    ch.rdfd = dd.p + (size_t)c * n;
    ch.steps = ds.p + c;
    ch.flux = dflux.p + c;
    ch.iters = dit.p + c;
    ch.nsteps = 1;
    ch.a = a[c];
    ch.b = b[c];
    ch.prob = prob[c];
  }
  if (run_chains(chains, n, eps, st, err)) return -1;
  std::vector<int> hit(nsolve);
  if ((e = cudaMemcpy(rdfa, da.p, nn * sizeof(double), cudaMemcpyDeviceToHost)) ||
      (rdfd && (e = cudaMemcpy(rdfd, dd.p, nn * sizeof(double), cudaMemcpyDeviceToHost))) ||
      (e = cudaMemcpy(flux, dflux.p, nsolve * sizeof(double), cudaMemcpyDeviceToHost)) ||
      (e = cudaMemcpy(hit.data(), dit.p, nsolve * sizeof(int), cudaMemcpyDeviceToHost))) {
    *err = std::string("rdf steady state: ") + cudaGetErrorString(e);
    return -1;
  }
  if (iters)
    for (int c = 0; c < nsolve; ++c) iters[c] = hit[c];
  return 0;
}

}  // namespace smolb

extern "C" {

enum ErrorCode smolgpuRdfTable(char mode, int n, double eps, char dir, int nprob, const double *probs, double *flux,
                               int *iters, int *nrows) {
  if (mode != 'i' && mode != 'r' && mode != 'b')
    return smolb_record_error(__func__, ECbounds, "mode must be 'i', 'r' or 'b'");
  if (dir != 'u' && dir != 'd' && dir != 'a')
    return smolb_record_error(__func__, ECbounds, "dir must be 'u', 'd' or 'a'");
  if (n < 10 || n > smolb::kMaxN) return smolb_record_error(__func__, ECbounds, "n must be in [10, 4000]");
  if (!(eps > 0)) return smolb_record_error(__func__, ECbounds, "eps must be > 0");
  if (probs && (nprob < 1 || nprob > 64)) return smolb_record_error(__func__, ECbounds, "nprob must be in [1, 64]");
  if (!flux) return smolb_record_error(__func__, ECmissing, "missing flux array");
  if (probs)
    for (int p = 0; p < nprob; ++p)
      if (!(probs[p] >= 0 && probs[p] <= 1))
        return smolb_record_error(__func__, ECbounds, "probabilities must be in [0, 1]");
  std::string err;
  if (smolb::rdf_table_device(mode, n, eps, dir, nprob, probs, flux, iters, nrows, &err))
    return smolb_record_error(__func__, ECerror, err);
  return ECok;
}

enum ErrorCode smolgpuRdfSteadyState(int nsolve, int n, const double *r, double *rdfa, double *rdfd,
                                     const double *step, const double *a, const double *b, const double *prob,
                                     double eps, double *flux, int *iters) {
  if (nsolve < 0 || nsolve > (1 << 20)) return smolb_record_error(__func__, ECbounds, "nsolve out of range");
  if (nsolve == 0) return ECok;
  if (n < 10 || n > smolb::kMaxN) return smolb_record_error(__func__, ECbounds, "n must be in [10, 4000]");
  if (!(eps > 0)) return smolb_record_error(__func__, ECbounds, "eps must be > 0");
  if (!r || !rdfa || !step || !a || !b || !prob || !flux)
    return smolb_record_error(__func__, ECmissing, "missing arrays");
  for (int c = 0; c < nsolve; ++c) {
    const double *rc = r + (size_t)c * n;
    if (!(rc[0] >= 0)) return smolb_record_error(__func__, ECbounds, "r[0] must be >= 0");
    for (int i = 1; i < n; ++i)
      if (!(rc[i] > 0)) return smolb_record_error(__func__, ECbounds, "radii after the first must be > 0");
    if (!(step[c] > 0)) return smolb_record_error(__func__, ECbounds, "step must be > 0");
    if (!(prob[c] >= 0 && prob[c] <= 1)) return smolb_record_error(__func__, ECbounds, "prob must be in [0, 1]");
  }
  std::string err;
  if (smolb::rdf_steady_device(nsolve, n, r, rdfa, rdfd, step, a, b, prob, eps, flux, iters, &err))
    return smolb_record_error(__func__, ECerror, err);
  return ECok;
}

}  // extern "C"
