// Per-device execution context: stream, scratch arenas, cached tables.
#pragma once

#include <map>
#include <memory>
#include <mutex>

#include "common.cuh"

namespace pyfof {

struct GreenTable;  // unbinding Green's function cache entry (unbind.cu)

struct Context {
  int device = 0;
  cudaStream_t stream = nullptr;      // stream all work is issued on
  cudaStream_t own_stream = nullptr;  // the context's own stream (default)
  Arena work;    // per-call device memory, released at the end of every call
  int32_t *d_flags = nullptr;  // device status words (error codes, counters)
  int32_t *h_flags = nullptr;  // pinned mirror
  std::mutex mu;
  std::map<int64_t, std::shared_ptr<GreenTable>> green;  // keyed by grid size and kind
  cudaEvent_t ev[8] = {};
  // timing of the last call's stages (ms), filled when timing is enabled
  bool timing = false;
  float stage_ms[16] = {};
  // statistics of the last call
  int64_t last_cells = 0, last_active = 0, last_candidates = 0, last_dense = 0;
  int64_t last_direct = 0, last_pm = 0, last_valid = 0, last_tl_regions = 0;
  ~Context();
};

// Returns the context of `device`, creating it on first use.
int32_t get_context(int device, Context **out);
void destroy_contexts();

}  // namespace pyfof
