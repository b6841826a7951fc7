// MLP surrogate for the binding / unbinding radius solve (host interface).
//
// The exact solve (bindingradius, rxnparam.c:558-584) finds a with
// numrxnrate(s, a, b) = k*dt by doubling and 15 bisections.  Because
// numrxnrate(s, a, b) = a^3 F(s/a, b/a), the reduced radius a/s depends only on
// the reduced rate kappa = k/(D*s) (s = sqrt(2*D*dt) the rms step, D the
// mutual diffusion coefficient) and on the unbinding parameter.  The surrogate
// is a 3->64->64->2 tanh network on
//   inputs  x = (log10 kappa, unbinding ratio rho in [0,2], reversible flag)
//   outputs y = (log10 (a/s)/A(kappa), (b/s)/A(kappa))
// with b = rho*a for ratio placement (0 if irreversible) and A(kappa) the
// analytic diffusion-/activation-limited radius (cbrt(aD^3 + aA^3), aD =
// kappa/(4 pi), aA = (3 kappa/(8 pi))^(1/3)), so the network fits a narrow
// residual.  It is trained on samples of the exact FP64 solver generated on
// the GPU, the last fifth of the epochs quantisation-aware (forward and
// backward on BF16-rounded weights).  Inference uses BF16 weights with FP32
// accumulation, then evaluates numrxnrate at the predicted radius and at a
// 0.1% larger one, takes one secant step in log a with the local slope
// g = dln(rate)/dln(a), and evaluates numrxnrate once more at the corrected
// radius: its rate error divided by g estimates the radius error; above the
// tolerance (default 1e-3) the exact solver runs for that instance instead.
// Three rate evaluations replace the exact solver's doubling and 15
// bisections (about 20 evaluations).
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace smolb {

constexpr int kMlpIn = 3, kMlpHid = 64, kMlpOut = 2;
// parameter layout: W1[64][3] b1[64] W2[64][64] b2[64] W3[2][64] b3[2]
constexpr int kMlpW1 = 0, kMlpB1 = kMlpW1 + kMlpHid * kMlpIn, kMlpW2 = kMlpB1 + kMlpHid,
              kMlpB2 = kMlpW2 + kMlpHid * kMlpHid, kMlpW3 = kMlpB2 + kMlpHid, kMlpB3 = kMlpW3 + kMlpOut * kMlpHid,
              kMlpNParam = kMlpB3 + kMlpOut;

struct SurrogateStats {
  double final_loss = 0;
  double train_seconds = 0;
  long long samples = 0;
  int epochs = 0;
};

class SurrogateImpl;

class Surrogate {
 public:
  Surrogate();
  ~Surrogate();
  Surrogate(const Surrogate &o);
  Surrogate &operator=(const Surrogate &) = delete;

  // Generate nsamples exact solver samples on the device and train.
  int train(long long nsamples, int epochs, int batch, double lr, uint64_t seed, SurrogateStats *st,
            std::string *err);
  bool trained() const;
  // Raw network on n inputs (x: n*3) -> y: n*2, FP32 parameters (training path).
  int forward(long long n, const double *x, double *y, std::string *err);
  // Mean squared loss and its gradient w.r.t. all parameters on one batch.
  int loss_grad(long long n, const double *x, const double *y, double *loss, std::vector<float> *grad,
                std::string *err);
  // Exact solver samples (x: n*3, y: n*2) generated on the device.
  int samples(long long n, uint64_t seed, std::vector<double> *x, std::vector<double> *y, std::string *err);
  const std::vector<float> &params() const;
  int set_params(const std::vector<float> &p, std::string *err);
  void set_tolerance(double tol);
  // Radii for a batch of bimolecular reactions (same semantics as
  // rxnp::pair_radii for irreversible and ratio placement; other placements
  // take the exact path).  *nfallback counts exact-solver fallbacks.
  int pair_radii(long long n, const double *kf, const double *dsum, double dt, int same, int rev, int rparamt,
                 double rparam, double *bind, double *unbind, long long *nfallback, std::string *err);

 private:
  SurrogateImpl *impl_;
};

}  // namespace smolb
