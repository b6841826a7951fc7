// Batched FP64 radius solve that allocates no device memory.
//
// Same work as smolgpuSolveRadii (bindingradius / unbindingradius,
// rxnparam.c:558-716, one thread per problem), but its inputs and outputs go
// through a fixed scratch array in static device memory instead of buffers
// from cudaMalloc.  It is for callers that cannot allocate: a rate update
// issued while an ensemble's steps run on another stream (cudaMalloc and
// cudaFree may synchronise the whole device and would stall those steps), and
// processes whose device memory is already spoken for (a simulation sized to
// fill HBM has no room left for per-call buffers).
//
// Rules of use:
// - at most kNoAllocMaxRadii problems per call; larger calls are rejected
//   with ECbounds before the device is touched;
// - the scratch is shared by every call on a device and keeps the last
//   call's contents, so calls that overlap on the GPU (two host threads, or a
//   call while an earlier one is still in flight) race on it and must be
//   serialised by the caller;
// - the first call on each device sets up the scratch address
//   (cudaGetSymbolAddress, with that device current).  With lazy module
//   loading (the CUDA 12 default) that call can load this library's device
//   code, which places the scratch in device memory and may synchronise, so
//   the first call belongs at set-up time: before HBM is filled and before
//   any stream capture.  The address is cached per device; a cudaDeviceReset
//   invalidates it, so the library must be reloaded after one;
// - the copies are synchronous cudaMemcpy and the kernel runs on the legacy
//   default stream, which waits for every blocking stream of the process:
//   the call overlaps only work on cudaStreamNonBlocking streams (the
//   engine's own streams are created that way).
// No scratch slot is read before the same call writes it (inputs are copied
// in, every output below n is written by the kernel), so nothing has to be
// cleared between calls.
#include <cuda_runtime.h>

#include <mutex>
#include <string>

#include "../../include/smoldyn_b200.h"

ErrorCode smolb_record_error(const char *, ErrorCode, const std::string &);

namespace smolb {

// defined in engine.cu
__global__ void k_solve_radii(int mode, long long n, const double *rate, double dt, const double *difc,
                              const double *b, int rel, double *out);

namespace {

constexpr long long kNoAllocMaxRadii = 65536;
constexpr int kMaxDevices = 64;

// rate | difc | b | out, each kNoAllocMaxRadii doubles (2 MiB in all).  In
// host code this name is only a stand-in for the device array: kernels get
// the address from cudaGetSymbolAddress below.
static __device__ __align__(256) double g_radii_scratch[4 * kNoAllocMaxRadii];

struct DeviceScratch {
  double *base = nullptr;
  int sms = 0;
};

std::mutex g_setup_mu;
DeviceScratch g_scratch[kMaxDevices];

// Set-up for the current device, done once: scratch address and SM count.
int device_scratch(DeviceScratch *out, std::string *err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { *err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return -1; }
  if (dev < 0 || dev >= kMaxDevices) { *err = "device index out of range"; return -1; }
  std::lock_guard<std::mutex> lock(g_setup_mu);
  DeviceScratch &d = g_scratch[dev];
  if (!d.base) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_radii_scratch);
    if (e != cudaSuccess) { *err = std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e); return -1; }
    int sms = 0;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) { *err = std::string("cudaDeviceGetAttribute: ") + cudaGetErrorString(e); return -1; }
    d.sms = sms > 0 ? sms : 148;
    d.base = static_cast<double *>(p);
  }
  *out = d;
  return 0;
}

}  // namespace
}  // namespace smolb

extern "C" enum ErrorCode smolgpuSolveRadiiNoAlloc(int mode, long long n, const double *rate, double dt,
                                                   const double *difc, const double *b, int rel, double *out) {
  using smolb::kNoAllocMaxRadii;
  if (n < 0) return smolb_record_error(__func__, ECbounds, "n must be >= 0");
  if (n > kNoAllocMaxRadii)
    return smolb_record_error(__func__, ECbounds,
                              "n = " + std::to_string(n) + " exceeds the scratch limit of " +
                                  std::to_string(kNoAllocMaxRadii) + " problems per call");
  if (n > 0 && !(rate && difc && b && out)) return smolb_record_error(__func__, ECmissing, "missing arrays");
  if (mode != 0 && mode != 1) return smolb_record_error(__func__, ECbounds, "mode must be 0 or 1");
  if (n == 0) return ECok;
  std::string err;
  smolb::DeviceScratch s;
  if (smolb::device_scratch(&s, &err)) return smolb_record_error(__func__, ECerror, err);
  double *d_rate = s.base, *d_difc = s.base + kNoAllocMaxRadii, *d_b = s.base + 2 * kNoAllocMaxRadii,
         *d_out = s.base + 3 * kNoAllocMaxRadii;
  const size_t bytes = (size_t)n * sizeof(double);
  cudaError_t e = cudaMemcpy(d_rate, rate, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_difc, difc, bytes, cudaMemcpyHostToDevice);
  if (e == cudaSuccess) e = cudaMemcpy(d_b, b, bytes, cudaMemcpyHostToDevice);
  if (e != cudaSuccess) return smolb_record_error(__func__, ECerror, std::string("copy in: ") + cudaGetErrorString(e));
  smolb::k_solve_radii<<<s.sms * 2, 128>>>(mode, n, d_rate, dt, d_difc, d_b, rel, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return smolb_record_error(__func__, ECerror, std::string("launch: ") + cudaGetErrorString(e));
  e = cudaMemcpy(out, d_out, bytes, cudaMemcpyDeviceToHost);
  if (e != cudaSuccess) return smolb_record_error(__func__, ECerror, std::string("copy out: ") + cudaGetErrorString(e));
  return ECok;
}
