// Allocation-free entry point: first-pass direct-summation potential of one
// small candidate with all device scratch in a fixed, file-scope array.
//
// Who needs it: callers that must not allocate device memory while they run
// -- a host framework whose caching allocator has reserved the device memory
// up front (a cudaMalloc behind its back can fail or fragment its pool), or
// a latency-bound loop that cannot tolerate an allocation (or an out-of-
// memory error) in the middle of a step.  pyfof_halo_potential serves the
// same computation but takes its scratch from the device memory pool on
// every call.
//
// The scratch array below is static device memory: every GPU that loads the
// library holds its kStaticMaxMembers-member capacity (about 42 KiB) until
// the process exits.  Host code cannot use the symbol itself as a device
// address; its address is looked up once per device with
// cudaGetSymbolAddress on the first call made on that device.  All calls
// share the one array:
// calls that overlap on the GPU race and must be serialised by the caller
// (the entry point itself synchronises the stream before it returns).
#include <cstring>
#include <mutex>

#include "context.cuh"
#include "unbind_direct.cuh"
#include "../../include/pyfof_b200.h"

namespace pyfof {

namespace {

constexpr int kStaticMaxMembers = 1000;  // the direct-summation limit
constexpr int kCap = 1024;

// Layout of the static scratch (all offsets multiples of 256 bytes).
struct StaticScratch {
  float q[3][kCap];
  float v[3][kCap];        // zero velocities: the potential needs none
  float w[kCap];
  int32_t pid[kCap];
  float phi[kCap];
  uint8_t keep[kCap];
  int64_t off[2];
  int32_t list[1];
  HaloResult res[1];
  int32_t flags[FLAG_COUNT];
};

static __device__ __align__(256) unsigned char g_static_scratch[sizeof(StaticScratch)];

struct DeviceSetup {
  bool done = false;
  StaticScratch *scratch = nullptr;  // device address of g_static_scratch
};
std::mutex g_setup_mu;
DeviceSetup g_setup[64];

// Once per device, with that device current: the scratch address and the
// kernel's dynamic shared-memory limit.
int32_t setup_device(int dev, StaticScratch **out) {
  std::lock_guard<std::mutex> lk(g_setup_mu);
  DeviceSetup &d = g_setup[dev];
  if (!d.done) {
    void *p = nullptr;
    PYFOF_CUDA(cudaGetSymbolAddress(&p, g_static_scratch));
    PYFOF_CUDA(cudaFuncSetAttribute(direct::ub_direct_kernel<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDirectSmem));
    PYFOF_CUDA(cudaFuncSetAttribute(direct::ub_direct_kernel<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kDirectSmem));
    d.scratch = static_cast<StaticScratch *>(p);
    d.done = true;
  }
  *out = d.scratch;
  return kOk;
}

}  // namespace

}  // namespace pyfof

using namespace pyfof;

extern "C" int32_t pyfof_halo_potential_direct_static(const float *q, const float *w, int32_t np,
                                                      double softening, double a_val, int32_t fp64,
                                                      float *phi, void *stream) {
  if (!q || !w || !phi || np <= 0) {
    set_error("pyfof_halo_potential_direct_static: invalid arguments");
    return kInvalid;
  }
  if (np > kStaticMaxMembers) {
    set_error("pyfof_halo_potential_direct_static: %d members exceed the static scratch limit of %d",
              np, kStaticMaxMembers);
    return kInvalid;
  }
  int dev = 0;
  PYFOF_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 64) {
    set_error("invalid device %d", dev);
    return kInvalid;
  }
  StaticScratch *S = nullptr;
  PYFOF_TRY(setup_device(dev, &S));
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const size_t nb = sizeof(float) * (size_t)np;
  for (int d = 0; d < 3; ++d) {
    PYFOF_CUDA(cudaMemcpyAsync(S->q[d], q + (size_t)d * np, nb, cudaMemcpyHostToDevice, s));
    PYFOF_CUDA(cudaMemsetAsync(S->v[d], 0, nb, s));
  }
  PYFOF_CUDA(cudaMemcpyAsync(S->w, w, nb, cudaMemcpyHostToDevice, s));
  // the previous call's contents stay in the array: reset what this call reads
  const int64_t off[2] = {0, np};
  const int32_t zero = 0;
  PYFOF_CUDA(cudaMemcpyAsync(S->off, off, sizeof(off), cudaMemcpyHostToDevice, s));
  PYFOF_CUDA(cudaMemcpyAsync(S->list, &zero, sizeof(zero), cudaMemcpyHostToDevice, s));
  PYFOF_CUDA(cudaMemsetAsync(S->flags, 0, sizeof(S->flags), s));
  Members m;
  for (int d = 0; d < 3; ++d) {
    m.q[d] = S->q[d];
    m.v[d] = S->v[d];
  }
  m.w = S->w;
  m.pid = S->pid;
  direct::DirectParams P;
  P.fac = a_val / (6.0 * 3.141592653589793238462643383279502884197);
  P.app = softening;
  P.b = 0.0f;
  P.nmin = 1;
  P.phi_only = 1;
  if (fp64)
    direct::ub_direct_kernel<true><<<1, direct::BLK, kDirectSmem, s>>>(m, S->off, S->list, P, S->res,
                                                                        S->keep, S->phi, S->flags);
  else
    direct::ub_direct_kernel<false><<<1, direct::BLK, kDirectSmem, s>>>(m, S->off, S->list, P, S->res,
                                                                         S->keep, S->phi, S->flags);
  PYFOF_CHECK_LAUNCH();
  int32_t err = 0;
  PYFOF_CUDA(cudaMemcpyAsync(phi, S->phi, nb, cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaMemcpyAsync(&err, &S->flags[FLAG_ERR], sizeof(err), cudaMemcpyDeviceToHost, s));
  PYFOF_CUDA(cudaStreamSynchronize(s));
  if (err) {
    set_error("pyfof_halo_potential_direct_static: non-finite potential");
    return err;
  }
  return kOk;
}
