// Per-device execution context: stream, scratch arenas, cached tables.
#pragma once

#include <map>
#include <memory>
#include <mutex>
#include <vector>

#include "common.cuh"

namespace pyfof {

struct GreenTable;  // unbinding Green's function cache entry (unbind_pm.cu)

// Green tables of one device, shared by all contexts of that device (they
// are read-only once built; building one holds the lock).
struct GreenCache {
  std::mutex mu;
  std::map<int64_t, std::shared_ptr<GreenTable>> tables;  // keyed by grid size and kind
};

// Device time of a launch group that repeats many times within one call
// (bracketed by begin/end on the stream); collect() adds up the completed
// pairs after a stream synchronisation.
struct GroupTimer {
  std::vector<cudaEvent_t> ev;
  size_t used = 0;
  double ms = 0.0;
  void begin(cudaStream_t s) { record(s); }
  void end(cudaStream_t s) { record(s); }
  void collect() {
    for (size_t i = 0; i + 1 < used; i += 2) {
      float t = 0.0f;
      if (cudaEventElapsedTime(&t, ev[i], ev[i + 1]) == cudaSuccess) ms += t;
    }
    used = 0;
  }
  void reset() { used = 0; ms = 0.0; }
  ~GroupTimer() { for (auto e : ev) cudaEventDestroy(e); }

 private:
  void record(cudaStream_t s) {
    if (used == ev.size()) {
      cudaEvent_t e;
      if (cudaEventCreate(&e) != cudaSuccess) return;
      ev.push_back(e);
    }
    cudaEventRecord(ev[used++], s);
  }
};

struct Context {
  static constexpr uint32_t kMagic = 0x50464f46u;
  uint32_t magic = kMagic;  // cleared on destruction (slot handle check)
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream (default)
  cudaStream_t aux_stream = nullptr;  // host-to-device copies of vp and mp
  // direct-summation unbinding, overlapping the particle-mesh halos (created
  // on first use); ev_fork/ev_join order it after and before `stream`
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  cudaEvent_t ev_alloc = nullptr, ev_inputs = nullptr, ev_masses = nullptr;
  // unbinding: members packed (stream) and their velocities packed on the
  // input stream; vel_wait is ev_vel while such a pack is pending, and
  // every kernel that reads member velocities is ordered after it
  // (wait_velocities)
  cudaEvent_t ev_pack = nullptr, ev_vel = nullptr, vel_wait = nullptr;
  Arena work;    // per-call device memory, released at the end of every call
  int32_t *d_flags = nullptr;  // device status words (error codes, counters)
  int32_t *h_flags = nullptr;  // pinned mirror
  std::mutex mu;
  std::shared_ptr<GreenCache> green;
  size_t pm_budget = (size_t)8 << 30;  // particle-mesh grid batch bytes
  int64_t last_peak_bytes = 0;         // device memory the last call held at most
  cudaEvent_t ev[12] = {};
  // timing of the last call's stages (ms), filled when timing is enabled
  bool timing = false;
  float stage_ms[16] = {};
  GroupTimer conv_timer;  // PM convolutions (the FFT kernels) of the last call
  // the PM pass loop's device idle time between passes (from the end of a
  // pass's last kernel to the first launch of the next, which waits for the
  // host to read the pass's results), and its pass count
  GroupTimer gap_timer;
  int64_t last_pm_passes = 0;
  bool side_timed = false;  // ev[9..11] hold this call's fork timing
  // statistics of the last call: PM solves and their algorithmic FFT bytes
  // (one read and one write of the padded (n+2) n^2 grid per transform, two
  // transforms per solve)
  int64_t last_pm_solves = 0;
  double last_pm_fft_bytes = 0.0;
  // statistics of the last call
  int64_t last_cells = 0, last_active = 0, last_candidates = 0, last_dense = 0;
  int64_t last_max_cell = 0;    // particles in the fullest cell
  int64_t last_cell_sorts = 0;  // 1: cell order by per-cell sorts, 0: by the radix sort
  int64_t last_direct = 0, last_pm = 0, last_valid = 0, last_tl_regions = 0;
  // host tables bound for the device: pinned, device-mapped staging that a
  // kernel reads (see upload); bump-allocated within a call and reset by
  // stage_reset at the start of the next one, when the previous call has
  // synchronised.  A buffer outgrown during a call is kept until the
  // context is destroyed (freeing pinned memory synchronises the device).
  uint8_t *h_stage = nullptr;
  size_t stage_cap = 0, stage_used = 0;
  std::vector<uint8_t *> stage_retired;
  void stage_reset() { stage_used = 0; }
  ~Context();
};

// Copies `bytes` of host memory to device memory in the order of stream s.
// A copy of more than a few KB from the host is a copy-engine transfer that
// queues behind the large input copies another stream has in flight (the
// velocities and masses, or another slot's inputs); so the bytes go into
// the context's pinned staging and a kernel reads them from there over the
// host link, which nothing queues behind.  Small copies stay
// cudaMemcpyAsync (the driver passes them inline).  `src` may be reused as
// soon as upload returns.
int32_t upload(Context &ctx, void *dst, const void *src, size_t bytes, cudaStream_t s);

// Orders stream s after the pending velocity pack of the call, if any.
inline cudaError_t wait_velocities(Context &ctx, cudaStream_t s) {
  return ctx.vel_wait ? cudaStreamWaitEvent(s, ctx.vel_wait, 0) : cudaSuccess;
}

// Returns the context of `device`, creating it on first use.
int32_t get_context(int device, Context **out);
void destroy_contexts();

}  // namespace pyfof
