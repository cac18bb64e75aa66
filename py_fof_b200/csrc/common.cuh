// Shared device/host helpers for the py_fof B200 library.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <cstdio>
#include <mutex>
#include <string>
#include <vector>

namespace pyfof {

// Reference error codes (py_fof/__init__.py:338-348, fof_fortran.f90:116-119).
enum : int32_t {
  kOk = 0,
  kInvalid = 1,      // invalid input or configuration
  kSpan = 2,         // candidate span exceeds the 15 Mpc limit
  kAlloc = 3,        // allocation failure
  kNonFinite = 4,    // NaN/Inf encountered
  kMass = 5,         // a particle mass is not positive and finite (the
                     // reference raises this in Python before its call,
                     // py_fof/__init__.py:259-260; here the device checks)
  kThreads = 10,     // n_threads > 256
  kCuda = 20,        // CUDA runtime failure (no reference counterpart)
};

void set_error(const char *fmt, ...);
std::string last_error();

#define PYFOF_CUDA(call)                                                        \
  do {                                                                          \
    cudaError_t e_ = (call);                                                    \
    if (e_ != cudaSuccess) {                                                    \
      ::pyfof::set_error("%s:%d %s: %s", __FILE__, __LINE__, #call,             \
                         cudaGetErrorString(e_));                               \
      return ::pyfof::kCuda;                                                    \
    }                                                                           \
  } while (0)

// Counts kernel launches (exposed through pyfof_get_stat("launches")) and
// checks the launch status.
extern std::atomic<int64_t> g_launches;
#define PYFOF_CHECK_LAUNCH()                                                   \
  do {                                                                         \
    ::pyfof::g_launches.fetch_add(1, std::memory_order_relaxed);               \
    PYFOF_CUDA(cudaGetLastError());                                            \
  } while (0)

#define PYFOF_TRY(expr)              \
  do {                               \
    int32_t r_ = (expr);             \
    if (r_ != ::pyfof::kOk) return r_; \
  } while (0)

inline int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }

constexpr int kNumSMs = 148;

// Per-call device allocator.  carve() takes memory from the device's
// stream-ordered pool (cudaMallocAsync on the call's stream; the pool keeps
// freed blocks cached, so steady-state calls do not reach the driver) and
// release() returns everything at the end of the call.
struct Arena {
  cudaStream_t stream = nullptr;
  std::vector<void *> ptrs;
  std::vector<size_t> sizes;
  size_t bytes = 0;      // held by this call
  size_t peak = 0;       // most held at once since the last reset
  size_t last_fail = 0;  // size of the last request that failed
  template <class T>
  T *carve(size_t count) {
    void *p = nullptr;
    size_t b = (count ? count : 1) * sizeof(T);
    if (cudaMallocAsync(&p, b, stream) != cudaSuccess) {
      cudaGetLastError();
      last_fail = b;
      return nullptr;
    }
    ptrs.push_back(p);
    sizes.push_back(b);
    bytes += b;
    if (bytes > peak) peak = bytes;
    return reinterpret_cast<T *>(p);
  }
  void release() { release_to(0); }
  // Blocks are freed in reverse order down to a mark taken earlier.
  size_t mark() const { return ptrs.size(); }
  void release_to(size_t m) {
    while (ptrs.size() > m) {
      cudaFreeAsync(ptrs.back(), stream);
      bytes -= sizes.back();
      ptrs.pop_back();
      sizes.pop_back();
    }
  }
};

// ---------------------------------------------------------------- device

// gfortran MODULO for real arguments: fmod, then add p when the remainder is
// non-zero and the operands' signs differ; +0 for a zero remainder.
__device__ __forceinline__ double fmodulo(double a, double p) {
  double r = fmod(a, p);
  if (r != 0.0) {
    if ((a < 0.0) != (p < 0.0)) r = __dadd_rn(r, p);
  } else {
    r = copysign(0.0, p);
  }
  return r;
}

// Unwrap a coordinate about an anchor: MODULO(x - anchor + half, L) - half,
// evaluated left to right in FP64 (fof_fortran.f90:525).
__device__ __forceinline__ double unwrap(double x, double anchor, double half, double L) {
  return __dadd_rn(fmodulo(__dadd_rn(__dadd_rn(x, -anchor), half), L), -half);
}

// Order-preserving maps between doubles and unsigned 64-bit integers, for
// exact atomic min/max of doubles.
__device__ __forceinline__ unsigned long long dbl_to_ord(double v) {
  unsigned long long b = (unsigned long long)__double_as_longlong(v);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__host__ __device__ inline double ord_to_dbl(unsigned long long o) {
  unsigned long long b = (o & 0x8000000000000000ull) ? (o & 0x7fffffffffffffffull) : ~o;
  double d;
  memcpy(&d, &b, sizeof(d));
  return d;
}

__device__ __forceinline__ unsigned lanemask_lt() {
  unsigned m;
  asm("mov.u32 %0, %%lanemask_lt;" : "=r"(m));
  return m;
}

// Particle coordinate accessor for (3,N) arrays in either Fortran order
// (AoS: x[3i+d]) or C order (SoA: x[d*N+i]).
struct Coords {
  const double *p;
  int64_t n;
  int32_t soa;
  __device__ __forceinline__ double get(int64_t i, int d) const {
    return soa ? p[d * n + i] : p[3 * i + d];
  }
};

}  // namespace pyfof
