// C-ABI of libpyfof_b200.so (declared in include/pyfof_b200.h), per-device
// contexts and error reporting.
#include <cstdarg>
#include <cstring>

#include "catalogue.cuh"
#include "context.cuh"
#include "fof.cuh"
#include "fof_internal.cuh"
#include "unbind_internal.cuh"
#include "../../include/pyfof_b200.h"

namespace pyfof {

std::atomic<int64_t> g_launches{0};

namespace {
thread_local std::string g_last_error;
std::mutex g_ctx_mu;
Context *g_ctx[64] = {};
int g_default_device = 0;
int g_bound_fp64 = 1;  // FP64 unbinding by default: direct sums bit-exact with the reference
int g_bound_per_halo = 0;
int g_timing = 0;
int64_t g_big_np = 0;
TileTable g_tiles;
int g_cell_order = 0;
}  // namespace

void set_error(const char *fmt, ...) {
  char buf[4096];
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(buf, sizeof(buf), fmt, ap);
  va_end(ap);
  g_last_error = buf;
}

std::string last_error() { return g_last_error; }

Context::~Context() {
  if (stream) {
    cudaStreamSynchronize(stream);
    work.release();
    cudaStreamSynchronize(stream);
  }
  if (own_stream) cudaStreamDestroy(own_stream);
  if (aux_stream) cudaStreamDestroy(aux_stream);
  if (side_stream) {
    cudaStreamSynchronize(side_stream);
    cudaStreamDestroy(side_stream);
  }
  if (ev_fork) cudaEventDestroy(ev_fork);
  if (ev_join) cudaEventDestroy(ev_join);
  if (ev_alloc) cudaEventDestroy(ev_alloc);
  if (ev_inputs) cudaEventDestroy(ev_inputs);
  if (ev_masses) cudaEventDestroy(ev_masses);
  if (ev_pack) cudaEventDestroy(ev_pack);
  if (ev_vel) cudaEventDestroy(ev_vel);
  for (auto &e : ev) if (e) cudaEventDestroy(e);
  if (d_flags) cudaFree(d_flags);
  if (h_flags) cudaFreeHost(h_flags);
  if (h_stage) cudaFreeHost(h_stage);
  for (uint8_t *p : stage_retired) cudaFreeHost(p);
}

// dst[i] = src[i], src in mapped host memory at a 16-byte aligned address
__global__ void upload_kernel(const uint8_t *__restrict__ src, uint8_t *__restrict__ dst, size_t bytes) {
  const size_t tid = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
  const size_t stride = (size_t)gridDim.x * blockDim.x;
  size_t done = 0;
  if ((reinterpret_cast<uintptr_t>(dst) & 15) == 0) {
    const size_t n16 = bytes / 16;
    for (size_t i = tid; i < n16; i += stride)
      reinterpret_cast<uint4 *>(dst)[i] = reinterpret_cast<const uint4 *>(src)[i];
    done = 16 * n16;
  }
  for (size_t i = done + tid; i < bytes; i += stride) dst[i] = src[i];
}

int32_t upload(Context &ctx, void *dst, const void *src, size_t bytes, cudaStream_t s) {
  constexpr size_t kInline = 4096;
  if (bytes == 0) return kOk;
  if (bytes <= kInline) {
    PYFOF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
    return kOk;
  }
  size_t off = (ctx.stage_used + 15) & ~(size_t)15;
  if (!ctx.h_stage || off + bytes > ctx.stage_cap) {
    size_t cap = std::max(2 * ctx.stage_cap, std::max(bytes, (size_t)1 << 20));
    cap = (cap + 4095) & ~(size_t)4095;
    uint8_t *p = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void **>(&p), cap, cudaHostAllocMapped | cudaHostAllocPortable) !=
        cudaSuccess) {
      // no pinned memory to be had: a plain copy (ordered, possibly queued)
      cudaGetLastError();
      PYFOF_CUDA(cudaMemcpyAsync(dst, src, bytes, cudaMemcpyHostToDevice, s));
      return kOk;
    }
    if (ctx.h_stage) ctx.stage_retired.push_back(ctx.h_stage);
    ctx.h_stage = p;
    ctx.stage_cap = cap;
    off = 0;
  }
  std::memcpy(ctx.h_stage + off, src, bytes);
  uint8_t *dsrc = nullptr;
  PYFOF_CUDA(cudaHostGetDevicePointer(reinterpret_cast<void **>(&dsrc), ctx.h_stage + off, 0));
  const unsigned grid = (unsigned)std::min<size_t>(bytes / 16 / 256 + 1, (size_t)kNumSMs * 2);
  upload_kernel<<<grid, 256, 0, s>>>(dsrc, reinterpret_cast<uint8_t *>(dst), bytes);
  PYFOF_CHECK_LAUNCH();
  ctx.stage_used = off + bytes;
  return kOk;
}

std::shared_ptr<GreenCache> g_green[64];

// A context of its own: streams, status words, events; the Green tables are
// shared by all contexts of a device.  Call with g_ctx_mu held.
static int32_t create_context(int device, Context **out) {
  if (device < 0 || device >= 64) {
    set_error("invalid device %d", device);
    return kInvalid;
  }
  int ndev = 0;
  PYFOF_CUDA(cudaGetDeviceCount(&ndev));
  if (device >= ndev) {
    set_error("device %d not present (%d devices)", device, ndev);
    return kInvalid;
  }
  PYFOF_CUDA(cudaSetDevice(device));
  Context *c = new Context();
  c->device = device;
  if (!g_green[device]) g_green[device] = std::make_shared<GreenCache>();
  c->green = g_green[device];
  auto fail = [&](cudaError_t e) {
    set_error("context creation: %s", cudaGetErrorString(e));
    delete c;
    return kCuda;
  };
  cudaError_t e;
  if ((e = cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  c->stream = c->own_stream;
  if ((e = cudaMalloc(&c->d_flags, sizeof(int32_t) * FLAG_COUNT)) != cudaSuccess) return fail(e);
  if ((e = cudaMallocHost(&c->h_flags, sizeof(int32_t) * FLAG_COUNT)) != cudaSuccess) return fail(e);
  for (auto &ev : c->ev)
    if ((e = cudaEventCreate(&ev)) != cudaSuccess) return fail(e);
  if ((e = cudaStreamCreateWithFlags(&c->aux_stream, cudaStreamNonBlocking)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&c->ev_alloc, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&c->ev_inputs, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&c->ev_masses, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&c->ev_pack, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  if ((e = cudaEventCreateWithFlags(&c->ev_vel, cudaEventDisableTiming)) != cudaSuccess) return fail(e);
  cudaMemPool_t pool;
  PYFOF_CUDA(cudaDeviceGetDefaultMemPool(&pool, device));
  uint64_t thr = UINT64_MAX;  // keep freed blocks cached in the pool
  PYFOF_CUDA(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr));
  c->work.stream = c->stream;
  *out = c;
  return kOk;
}

int32_t get_context(int device, Context **out) {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  if (device < 0 || device >= 64) {
    set_error("invalid device %d", device);
    return kInvalid;
  }
  if (!g_ctx[device]) PYFOF_TRY(create_context(device, &g_ctx[device]));
  *out = g_ctx[device];
  return kOk;
}

void destroy_contexts() {
  std::lock_guard<std::mutex> lk(g_ctx_mu);
  for (auto &c : g_ctx) {
    if (c) {
      cudaSetDevice(c->device);
      delete c;
      c = nullptr;
    }
  }
}

static int32_t validate(int32_t nhalo, int64_t total_np, const int32_t *np_halo,
                        int32_t n_threads) {
  if (n_threads > 256) {
    set_error("n_threads exceeds maximum supported slots (256)");
    return kThreads;
  }
  if (nhalo > 0 && !np_halo) {
    set_error("np_halo is null");
    return kInvalid;
  }
  int64_t s = 0;
  for (int32_t h = 0; h < nhalo; ++h) {
    if (np_halo[h] < 0) {
      set_error("np_halo[%d] < 0", h);
      return kInvalid;
    }
    s += np_halo[h];
  }
  if (nhalo > 0 && s != total_np) {
    set_error("sum(np_halo) != total_np");
    return kInvalid;
  }
  if (total_np >= (int64_t)INT32_MAX) {
    set_error("total_np must be below 2**31");
    return kInvalid;
  }
  return kOk;
}

// An allocation failure reports what the call held and what it asked for.
static void note_alloc_failure(Context &ctx, int32_t r) {
  if (r != kAlloc) return;
  size_t free_b = 0, total_b = 0;
  cudaMemGetInfo(&free_b, &total_b);
  // the largest blocks held, in allocation order
  std::string big;
  size_t thr = ctx.work.bytes / 50;
  for (size_t i = 0; i < ctx.work.sizes.size(); ++i)
    if (ctx.work.sizes[i] >= thr && big.size() < 200)
      big += " #" + std::to_string(i) + ":" + std::to_string(ctx.work.sizes[i] >> 20) + "MiB";
  big += " first:";
  for (size_t i = 0; i < ctx.work.sizes.size() && i < 40; ++i) big += " " + std::to_string(ctx.work.sizes[i]);
  big += " last:";
  for (size_t i = ctx.work.sizes.size() > 20 ? ctx.work.sizes.size() - 20 : 0; i < ctx.work.sizes.size(); ++i)
    big += " " + std::to_string(ctx.work.sizes[i]);
  set_error("%s (call holds %.3f GB in %zu blocks, failed request %.3f GB, device free %.3f of %.3f GB;%s)",
            last_error().c_str(), ctx.work.bytes / 1e9, ctx.work.sizes.size(), ctx.work.last_fail / 1e9,
            free_b / 1e9, total_b / 1e9, big.c_str());
}

// stage_ms: [0] linking kernel, [1] binning to candidates, [2] unbinding (or
// the plain ang_mom pass), [3] the whole call on the device
static void record_stage_times(Context &ctx) {
  for (float &t : ctx.stage_ms) t = 0.0f;
  cudaEventElapsedTime(&ctx.stage_ms[0], ctx.ev[0], ctx.ev[1]);
  cudaEventElapsedTime(&ctx.stage_ms[1], ctx.ev[2], ctx.ev[3]);
  cudaEventElapsedTime(&ctx.stage_ms[2], ctx.ev[3], ctx.ev[4]);
  cudaEventElapsedTime(&ctx.stage_ms[3], ctx.ev[2], ctx.ev[4]);
  ctx.stage_ms[4] = (float)ctx.conv_timer.ms;
  ctx.gap_timer.collect();
  ctx.stage_ms[11] = (float)ctx.gap_timer.ms;
  // from the fork of the direct-summation removal loops: their side stream,
  // and the particle-mesh halos on the call stream (0 when nothing forked)
  if (!ctx.side_timed || cudaEventElapsedTime(&ctx.stage_ms[12], ctx.ev[9], ctx.ev[10]) != cudaSuccess ||
      cudaEventElapsedTime(&ctx.stage_ms[13], ctx.ev[9], ctx.ev[11]) != cudaSuccess)
    ctx.stage_ms[12] = ctx.stage_ms[13] = 0.0f;
  // the part of "fof" before and after the (last region's) linking kernel
  cudaEventElapsedTime(&ctx.stage_ms[9], ctx.ev[2], ctx.ev[0]);
  cudaEventElapsedTime(&ctx.stage_ms[10], ctx.ev[1], ctx.ev[3]);
  cudaGetLastError();  // a region without linking leaves the link events unrecorded
}

// host-memory calls: [5] the position copy, [6] all input copies, [7] the
// output copy, [8] the whole call from the first copy to the last
static void record_copy_times(Context &ctx, bool side) {
  cudaEventElapsedTime(&ctx.stage_ms[5], ctx.ev[5], ctx.ev[6]);
  if (side) cudaEventElapsedTime(&ctx.stage_ms[6], ctx.ev[5], ctx.ev[8]);
  else ctx.stage_ms[6] = ctx.stage_ms[5];
  cudaEventElapsedTime(&ctx.stage_ms[7], ctx.ev[4], ctx.ev[7]);
  cudaEventElapsedTime(&ctx.stage_ms[8], ctx.ev[5], ctx.ev[7]);
  cudaGetLastError();
}

static int32_t run_common(Context &ctx, FofArgs &a) {
  ctx.timing = g_timing != 0;
  a.bound_fp64 = g_bound_fp64;
  a.bound_per_halo = g_bound_per_halo;
  a.big_np = g_big_np;
  a.tiles = g_tiles;
  a.cell_order = g_cell_order;
  int32_t r = fof_run(ctx, a);
  note_alloc_failure(ctx, r);
  cudaError_t e = cudaStreamSynchronize(ctx.stream);
  if (r == kOk && e != cudaSuccess) {
    set_error("CUDA failure: %s", cudaGetErrorString(e));
    r = kCuda;
  }
  if (ctx.timing && r == kOk) record_stage_times(ctx);
  ctx.work.release();
  cudaStreamSynchronize(ctx.stream);
  return r;
}

}  // namespace pyfof

using namespace pyfof;

extern "C" {

int32_t pyfof_version(void) { return PYFOF_B200_ABI_VERSION; }

int32_t pyfof_init(int32_t device) {
  Context *c;
  int32_t r = get_context(device, &c);
  if (r == kOk) g_default_device = device;
  return r;
}

int32_t pyfof_shutdown(void) {
  destroy_contexts();
  return kOk;
}

int32_t pyfof_last_error(char *buf, int64_t len) {
  if (!buf || len <= 0) return (int32_t)g_last_error.size();
  std::strncpy(buf, g_last_error.c_str(), (size_t)len - 1);
  buf[len - 1] = 0;
  return (int32_t)g_last_error.size();
}

int32_t pyfof_set_option(const char *key, int64_t value) {
  if (!key) return kInvalid;
  if (!std::strcmp(key, "unbind_fp64")) { g_bound_fp64 = value != 0; return kOk; }
  if (!std::strcmp(key, "unbind_per_halo")) { g_bound_per_halo = value != 0; return kOk; }
  if (!std::strcmp(key, "timing")) { g_timing = value != 0; return kOk; }
  if (!std::strcmp(key, "unbind_big_np")) { g_big_np = value; return kOk; }
  if (!std::strcmp(key, "cell_order")) {
    if (value < 0 || value > 2) {
      set_error("cell_order must be 0, 1 or 2");
      return kInvalid;
    }
    g_cell_order = (int)value;
    return kOk;
  }
  set_error("unknown option %s", key);
  return kInvalid;
}

int32_t pyfof_get_option(const char *key, int64_t *value) {
  if (!key || !value) return kInvalid;
  if (!std::strcmp(key, "unbind_fp64")) { *value = g_bound_fp64; return kOk; }
  if (!std::strcmp(key, "unbind_per_halo")) { *value = g_bound_per_halo; return kOk; }
  if (!std::strcmp(key, "timing")) { *value = g_timing; return kOk; }
  if (!std::strcmp(key, "unbind_big_np")) { *value = g_big_np; return kOk; }
  if (!std::strcmp(key, "cell_order")) { *value = g_cell_order; return kOk; }
  set_error("unknown option %s", key);
  return kInvalid;
}

// Tile table entries: "direct_threads" (index = size bucket 0..5, value 32,
// 64, 128 or 256), "pm_batch" (index = grid size n, value >= 0),
// "conv_waves" (index = grid size n, value 1..64).
static int *tile_slot(const char *key, int64_t index) {
  if (!key) return nullptr;
  if (!std::strcmp(key, "direct_threads"))
    return (index >= 0 && index < 6) ? &g_tiles.direct_threads[index] : nullptr;
  const int gi = kGridIndex((int)index);
  if (gi < 0 || index > 256) return nullptr;
  if (!std::strcmp(key, "pm_batch")) return &g_tiles.pm_batch[gi];
  if (!std::strcmp(key, "conv_waves")) return &g_tiles.conv_waves[gi];
  return nullptr;
}

int32_t pyfof_set_tile(const char *key, int64_t index, int64_t value) {
  int *slot = tile_slot(key, index);
  if (!slot) {
    set_error("unknown tile entry %s[%lld]", key ? key : "(null)", (long long)index);
    return kInvalid;
  }
  bool ok;
  if (!std::strcmp(key, "direct_threads")) ok = value == 32 || value == 64 || value == 128 || value == 256;
  else if (!std::strcmp(key, "pm_batch")) ok = value >= 0 && value <= (1 << 20);
  else ok = value >= 1 && value <= 64;
  if (!ok) {
    set_error("tile entry %s[%lld] out of range: %lld", key, (long long)index, (long long)value);
    return kInvalid;
  }
  *slot = (int)value;
  return kOk;
}

int32_t pyfof_get_tile(const char *key, int64_t index, int64_t *value) {
  int *slot = tile_slot(key, index);
  if (!slot || !value) {
    set_error("unknown tile entry %s[%lld]", key ? key : "(null)", (long long)index);
    return kInvalid;
  }
  *value = *slot;
  return kOk;
}

int32_t pyfof_host_alloc(int64_t bytes, void **ptr) {
  if (!ptr || bytes <= 0) {
    set_error("pyfof_host_alloc: invalid arguments");
    return kInvalid;
  }
  *ptr = nullptr;
  const cudaError_t e = cudaHostAlloc(ptr, (size_t)bytes, cudaHostAllocPortable);
  if (e != cudaSuccess) {
    cudaGetLastError();
    *ptr = nullptr;
    set_error("pinned host allocation of %lld bytes failed: %s", (long long)bytes, cudaGetErrorString(e));
    return kAlloc;
  }
  return kOk;
}

int32_t pyfof_host_free(void *ptr) {
  if (ptr) cudaFreeHost(ptr);
  cudaGetLastError();
  return kOk;
}

int32_t pyfof_set_stream(void *stream) {
  Context *c;
  PYFOF_TRY(get_context(g_default_device, &c));
  std::lock_guard<std::mutex> lk(c->mu);
  cudaStreamSynchronize(c->stream);
  if (!c->own_stream) PYFOF_CUDA(cudaStreamCreateWithFlags(&c->own_stream, cudaStreamNonBlocking));
  c->stream = stream ? (cudaStream_t)stream : c->own_stream;
  c->work.stream = c->stream;
  return kOk;
}

static int32_t context_stat(const Context *c, const char *key, int64_t *value) {
  if (!std::strcmp(key, "cells")) { *value = c->last_cells; return kOk; }
  if (!std::strcmp(key, "active")) { *value = c->last_active; return kOk; }
  if (!std::strcmp(key, "candidates")) { *value = c->last_candidates; return kOk; }
  if (!std::strcmp(key, "dense_cells")) { *value = c->last_dense; return kOk; }
  if (!std::strcmp(key, "vd_cells")) { *value = c->h_flags ? c->h_flags[FLAG_VD] : 0; return kOk; }
  if (!std::strcmp(key, "max_cell")) { *value = c->last_max_cell; return kOk; }
  if (!std::strcmp(key, "cell_sorts")) { *value = c->last_cell_sorts; return kOk; }
  if (!std::strcmp(key, "direct_halos")) { *value = c->last_direct; return kOk; }
  if (!std::strcmp(key, "pm_halos")) { *value = c->last_pm; return kOk; }
  if (!std::strcmp(key, "valid_halos")) { *value = c->last_valid; return kOk; }
  if (!std::strcmp(key, "refined_regions")) { *value = c->last_tl_regions; return kOk; }
  if (!std::strcmp(key, "pm_passes")) { *value = c->last_pm_passes; return kOk; }
  if (!std::strcmp(key, "pm_solves")) { *value = c->last_pm_solves; return kOk; }
  if (!std::strcmp(key, "pm_fft_bytes")) { *value = (int64_t)c->last_pm_fft_bytes; return kOk; }
  if (!std::strcmp(key, "peak_bytes")) { *value = c->last_peak_bytes; return kOk; }
  set_error("unknown statistic %s", key);
  return kInvalid;
}

int32_t pyfof_get_stat(const char *key, int64_t *value) {
  if (!key || !value) return kInvalid;
  if (!std::strcmp(key, "launches")) { *value = g_launches.load(); return kOk; }
  Context *c;
  PYFOF_TRY(get_context(g_default_device, &c));
  return context_stat(c, key, value);
}

int32_t pyfof_last_link_ms(float *ms) {
  Context *c;
  if (get_context(g_default_device, &c) != kOk || !ms) return kInvalid;
  *ms = c->stage_ms[0];
  return kOk;
}

int32_t pyfof_last_stage_ms(const char *stage, float *ms) {
  Context *c;
  if (!stage || !ms) {
    set_error("pyfof_last_stage_ms: null argument");
    return kInvalid;
  }
  if (get_context(g_default_device, &c) != kOk) return kInvalid;
  static const char *names[14] = {"link", "fof", "unbind", "call", "pm_fft",
                                  "h2d_positions", "h2d_inputs", "d2h", "host_call",
                                  "before_link", "after_link", "pm_gaps", "direct_loops",
                                  "pm_path"};
  for (int i = 0; i < 14; ++i)
    if (!std::strcmp(stage, names[i])) {
      *ms = c->stage_ms[i];
      return kOk;
    }
  set_error("unknown stage %s", stage);
  return kInvalid;
}

int32_t pyfof_halo_potential(const float *q, const float *w, int32_t np, double softening,
                             double a_val, double s_15_val, int64_t ng_val, int32_t fp64,
                             float *phi, int32_t *method) {
  if (!q || !w || !phi || !method || np <= 0) {
    set_error("invalid arguments");
    return kInvalid;
  }
  Context *cp;
  PYFOF_TRY(get_context(g_default_device, &cp));
  std::lock_guard<std::mutex> lk(cp->mu);
  PYFOF_CUDA(cudaSetDevice(cp->device));
  int32_t r = unbind_potential(*cp, q, w, np, softening, a_val, s_15_val, ng_val, fp64, phi, method);
  cudaStreamSynchronize(cp->stream);
  cp->work.release();
  cudaStreamSynchronize(cp->stream);
  return r;
}

// Host-memory call.  Positions are copied first on the call's stream; the
// velocities and masses follow on the context's second stream and are
// waited for only after the linking, so their copies overlap with it.
struct CatalogueOut {
  int32_t *members;
  int64_t *offsets;
  int64_t cap;
  int32_t *nfound;
};

static int32_t run_host(Context &ctx, const double *xp, const double *vp, const double *mp,
                        int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                        double L_Box, double linking_length, int32_t np_halo_min, int32_t bound_check,
                        int32_t verbose, double softening, double a_val, double b_val,
                        double s_15_val, int32_t n_threads, int64_t ng_val, double ng_global_val,
                        int32_t *in_halo, int32_t *halo_id, double *ang_mom, CatalogueOut *cat,
                        const pyfof_units_t *units, uint8_t *mask) {
  PYFOF_CUDA(cudaSetDevice(ctx.device));
  cudaStream_t s = ctx.stream;
  const size_t n = (size_t)total_np;
  const pyfof_units_t u = units ? *units : pyfof_units_t{1.0, 1.0, 1.0, 1.0};
  const bool fill_m = !mp && u.m_const != 1.0;  // a constant mass other than the unit one
  FofArgs a;
  double *xd = ctx.work.carve<double>(3 * n);
  double *vd = vp ? ctx.work.carve<double>(3 * n) : nullptr;
  double *md = (mp || fill_m) ? ctx.work.carve<double>(n) : nullptr;
  a.xp = xd;
  a.vp = vd;
  a.mp = md;
  a.in_halo = ctx.work.carve<int32_t>(n);
  a.halo_id = ctx.work.carve<int32_t>(n);
  if (!xd || (vp && !vd) || ((mp || fill_m) && !md) || !a.in_halo || !a.halo_id) {
    ctx.work.release();
    set_error("device allocation failed for %zu particles", n);
    return kAlloc;
  }
  const bool side = vp || mp || fill_m;
  // conversions to code units run on the stream of their copy; the masses
  // are converted after their check, inside the call
  ctx.timing = g_timing != 0;
  if (ctx.timing) cudaEventRecord(ctx.ev[5], s);
  PYFOF_CUDA(cudaMemcpyAsync(xd, xp, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, s));
  if (u.x_div != 1.0) PYFOF_TRY(divide_inplace(xd, (int64_t)(3 * n), u.x_div, s));
  if (ctx.timing) cudaEventRecord(ctx.ev[6], s);
  if (side) {
    // the other inputs follow the positions on the host link (the copies
    // share its bandwidth, so the positions, which the linking needs, go
    // first and the linking overlaps the rest); the buffers were allocated
    // in the order of stream s
    PYFOF_CUDA(cudaEventRecord(ctx.ev_alloc, s));
    PYFOF_CUDA(cudaStreamWaitEvent(ctx.aux_stream, ctx.ev_alloc, 0));
  }
  if (mp) {
    PYFOF_CUDA(cudaMemcpyAsync(md, mp, sizeof(double) * n, cudaMemcpyHostToDevice, ctx.aux_stream));
    a.m_div = u.m_div;
  } else if (fill_m) {
    PYFOF_TRY(fill_value(md, (int64_t)n, u.m_const, ctx.aux_stream));
  }
  if (mp || fill_m) {
    PYFOF_CUDA(cudaEventRecord(ctx.ev_masses, ctx.aux_stream));
    a.masses_ready = ctx.ev_masses;
  }
  if (vp) {
    PYFOF_CUDA(cudaMemcpyAsync(vd, vp, sizeof(double) * 3 * n, cudaMemcpyHostToDevice, ctx.aux_stream));
    if (u.v_mul != 1.0) PYFOF_TRY(multiply_inplace(vd, (int64_t)(3 * n), u.v_mul, ctx.aux_stream));
  }
  if (side) {
    if (ctx.timing) cudaEventRecord(ctx.ev[8], ctx.aux_stream);
    PYFOF_CUDA(cudaEventRecord(ctx.ev_inputs, ctx.aux_stream));
    a.inputs_ready = ctx.ev_inputs;
    a.input_stream = ctx.aux_stream;
  }
  PYFOF_CUDA(cudaMemsetAsync(a.in_halo, 0, sizeof(int32_t) * n, s));
  PYFOF_CUDA(cudaMemsetAsync(a.halo_id, 0, sizeof(int32_t) * n, s));
  a.soa = layout == PYFOF_LAYOUT_SOA ? 1 : 0;
  a.np_halo = np_halo;
  a.nhalo = nhalo;
  a.total_np = total_np;
  a.L_Box = L_Box;
  a.link = linking_length;
  a.np_halo_min = np_halo_min;
  a.bound_check = bound_check;
  a.verbose = verbose;
  a.softening = softening;
  a.a_val = a_val;
  a.b_val = b_val;
  a.s15 = s_15_val;
  a.n_threads = n_threads;
  a.ng = ng_val;
  a.ng_global = ng_global_val;
  a.ang_mom = ang_mom;
  a.bound_fp64 = g_bound_fp64;
  a.bound_per_halo = g_bound_per_halo;
  a.big_np = g_big_np;
  a.tiles = g_tiles;
  a.cell_order = g_cell_order;
  int32_t r = fof_run(ctx, a);
  if (r == kOk && cat) r = build_catalogue(ctx, a.halo_id, (int64_t)n, cat->members, cat->offsets, cat->cap,
                                           cat->nfound);
  note_alloc_failure(ctx, r);
  uint8_t *dmask = nullptr;
  if (r == kOk && mask) {
    dmask = ctx.work.carve<uint8_t>(n);
    if (!dmask) {
      set_error("device allocation failed for the membership mask");
      r = kAlloc;
    } else {
      r = member_mask(a.halo_id, (int64_t)n, dmask, s);
    }
  }
  if (r == kOk) {
    if (mask) {
      cudaMemcpyAsync(mask, dmask, n, cudaMemcpyDeviceToHost, s);
    } else {
      if (in_halo) cudaMemcpyAsync(in_halo, a.in_halo, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s);
      cudaMemcpyAsync(halo_id, a.halo_id, sizeof(int32_t) * n, cudaMemcpyDeviceToHost, s);
    }
    if (ctx.timing) cudaEventRecord(ctx.ev[7], s);
  }
  // an early failure may leave the side copies in flight: their buffers are
  // released in the order of stream s, after them
  if (side) {
    // everything the call queued on the input stream (its copies and the
    // velocity pack of the unbinding)
    cudaEventRecord(ctx.ev_inputs, ctx.aux_stream);
    cudaStreamWaitEvent(s, ctx.ev_inputs, 0);
  }
  cudaError_t e = cudaStreamSynchronize(s);
  if (r == kOk && e != cudaSuccess) {
    set_error("CUDA failure: %s", cudaGetErrorString(e));
    r = kCuda;
  }
  if (ctx.timing && r == kOk) {
    record_stage_times(ctx);
    record_copy_times(ctx, side);
  }
  ctx.last_peak_bytes = (int64_t)ctx.work.peak;
  ctx.work.peak = 0;
  ctx.work.release();
  cudaStreamSynchronize(s);
  return r;
}

// The checks and output conventions of pyfof_run around run_host; ctx null
// means the default device's context.
static int32_t run_host_checked(Context *ctx, const double *xp, const double *vp, const double *mp,
                                int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                                double L_Box, double linking_length, int32_t np_halo_min,
                                int32_t bound_check, int32_t verbose, double softening, double a_val,
                                double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                                double ng_global_val, int32_t *in_halo, int32_t *halo_id,
                                double *ang_mom, CatalogueOut *cat = nullptr,
                                const pyfof_units_t *units = nullptr, uint8_t *mask = nullptr) {
  // outputs are written in full on success and zeroed on every other path
  auto zero = [&]() {
    if (total_np > 0) {
      if (in_halo) std::memset(in_halo, 0, sizeof(int32_t) * (size_t)total_np);
      if (halo_id) std::memset(halo_id, 0, sizeof(int32_t) * (size_t)total_np);
      if (mask) std::memset(mask, 0, (size_t)total_np);
    }
    if (ang_mom && nhalo > 0) std::memset(ang_mom, 0, sizeof(double) * 3 * (size_t)nhalo);
  };
  int32_t r = validate(nhalo, total_np, np_halo, n_threads);
  if (r == kOk && (nhalo <= 0 || total_np <= 0)) {
    zero();
    if (cat) {
      *cat->nfound = 0;
      if (cat->cap >= 1) cat->offsets[0] = 0;
    }
    return kOk;
  }
  if (r == kOk && (!xp || !(halo_id || mask) || !ang_mom)) {
    set_error("null argument");
    r = kInvalid;
  }
  if (r == kOk && bound_check && !vp) {
    set_error("vp is required when bound_check is set");
    r = kInvalid;
  }
  if (r == kOk && !ctx) r = get_context(g_default_device, &ctx);
  if (r == kOk) {
    std::memset(ang_mom, 0, sizeof(double) * 3 * (size_t)nhalo);
    std::lock_guard<std::mutex> lk(ctx->mu);
    r = run_host(*ctx, xp, vp, mp, layout, np_halo, nhalo, total_np, L_Box, linking_length,
                 np_halo_min, bound_check, verbose, softening, a_val, b_val, s_15_val, n_threads,
                 ng_val, ng_global_val, in_halo, halo_id, ang_mom, cat, units, mask);
  }
  if (r != kOk) zero();
  return r;
}

int32_t pyfof_run(const double *xp, const double *vp, const double *mp, int32_t layout,
                  const int32_t *np_halo, int32_t nhalo, int64_t total_np, double L_Box,
                  double linking_length, int32_t np_halo_min, int32_t bound_check,
                  int32_t verbose, double softening, double a_val, double b_val,
                  double s_15_val, int32_t n_threads, int64_t ng_val, double ng_global_val,
                  int32_t *in_halo, int32_t *halo_id, double *ang_mom) {
  return run_host_checked(nullptr, xp, vp, mp, layout, np_halo, nhalo, total_np, L_Box,
                          linking_length, np_halo_min, bound_check, verbose, softening, a_val, b_val,
                          s_15_val, n_threads, ng_val, ng_global_val, in_halo, halo_id, ang_mom);
}

int32_t pyfof_run_device(const double *d_xp, const double *d_vp, const double *d_mp,
                         int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                         double L_Box, double linking_length, int32_t np_halo_min,
                         int32_t bound_check, int32_t verbose, double softening, double a_val,
                         double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                         double ng_global_val, int32_t *d_in_halo, int32_t *d_halo_id,
                         double *ang_mom) {
  if (ang_mom && nhalo > 0) std::memset(ang_mom, 0, sizeof(double) * 3 * (size_t)nhalo);
  int32_t r = validate(nhalo, total_np, np_halo, n_threads);
  if (r != kOk) return r;
  if (nhalo <= 0 || total_np <= 0) return kOk;
  if (!d_xp || !d_in_halo || !d_halo_id || !ang_mom) {
    set_error("null argument");
    return kInvalid;
  }
  if (bound_check && !d_vp) {
    set_error("vp is required when bound_check is set");
    return kInvalid;
  }
  Context *cp;
  PYFOF_TRY(get_context(g_default_device, &cp));
  Context &ctx = *cp;
  std::lock_guard<std::mutex> lk(ctx.mu);
  PYFOF_CUDA(cudaSetDevice(ctx.device));
  const size_t n = (size_t)total_np;
  PYFOF_CUDA(cudaMemsetAsync(d_in_halo, 0, sizeof(int32_t) * n, ctx.stream));
  PYFOF_CUDA(cudaMemsetAsync(d_halo_id, 0, sizeof(int32_t) * n, ctx.stream));
  FofArgs a;
  a.xp = d_xp;
  a.vp = d_vp;
  a.mp = d_mp;
  a.soa = layout == PYFOF_LAYOUT_SOA ? 1 : 0;
  a.np_halo = np_halo;
  a.nhalo = nhalo;
  a.total_np = total_np;
  a.L_Box = L_Box;
  a.link = linking_length;
  a.np_halo_min = np_halo_min;
  a.bound_check = bound_check;
  a.verbose = verbose;
  a.softening = softening;
  a.a_val = a_val;
  a.b_val = b_val;
  a.s15 = s_15_val;
  a.n_threads = n_threads;
  a.ng = ng_val;
  a.ng_global = ng_global_val;
  a.in_halo = d_in_halo;
  a.halo_id = d_halo_id;
  a.ang_mom = ang_mom;
  r = run_common(ctx, a);
  if (r != kOk) {
    cudaMemsetAsync(d_in_halo, 0, sizeof(int32_t) * n, ctx.stream);
    cudaMemsetAsync(d_halo_id, 0, sizeof(int32_t) * n, ctx.stream);
    cudaStreamSynchronize(ctx.stream);
    std::memset(ang_mom, 0, sizeof(double) * 3 * (size_t)nhalo);
  }
  return r;
}

int32_t pyfof_run_units(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                        const double *mp, int32_t layout, const int32_t *np_halo, int32_t nhalo,
                        int64_t total_np, double L_Box, double linking_length, int32_t np_halo_min,
                        int32_t bound_check, int32_t verbose, double softening, double a_val,
                        double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                        double ng_global_val, int32_t *in_halo, int32_t *halo_id, double *ang_mom) {
  if (slot && static_cast<Context *>(slot)->magic != Context::kMagic) {
    set_error("pyfof_run_units: not a slot");
    return kInvalid;
  }
  return run_host_checked(static_cast<Context *>(slot), xp, vp, mp, layout, np_halo, nhalo, total_np, L_Box,
                          linking_length, np_halo_min, bound_check, verbose, softening, a_val, b_val,
                          s_15_val, n_threads, ng_val, ng_global_val, in_halo, halo_id, ang_mom, nullptr,
                          units);
}

int32_t pyfof_run_mask(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                       const double *mp, int32_t layout, const int32_t *np_halo, int32_t nhalo,
                       int64_t total_np, double L_Box, double linking_length, int32_t np_halo_min,
                       int32_t bound_check, int32_t verbose, double softening, double a_val,
                       double b_val, double s_15_val, int32_t n_threads, int64_t ng_val,
                       double ng_global_val, uint8_t *in_halo, double *ang_mom) {
  if (slot && static_cast<Context *>(slot)->magic != Context::kMagic) {
    set_error("pyfof_run_mask: not a slot");
    return kInvalid;
  }
  if (!in_halo && total_np > 0 && nhalo > 0) {
    set_error("pyfof_run_mask: null in_halo");
    return kInvalid;
  }
  return run_host_checked(static_cast<Context *>(slot), xp, vp, mp, layout, np_halo, nhalo, total_np, L_Box,
                          linking_length, np_halo_min, bound_check, verbose, softening, a_val, b_val,
                          s_15_val, n_threads, ng_val, ng_global_val, nullptr, nullptr, ang_mom, nullptr,
                          units, in_halo);
}

int32_t pyfof_run_catalogue(void *slot, const pyfof_units_t *units, const double *xp, const double *vp,
                            const double *mp, int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                            double L_Box, double linking_length, int32_t np_halo_min, int32_t bound_check,
                            int32_t verbose, double softening, double a_val, double b_val, double s_15_val,
                            int32_t n_threads, int64_t ng_val, double ng_global_val, int32_t *halo_id,
                            double *ang_mom, int32_t *members, int64_t *offsets, int64_t offsets_cap,
                            int32_t *nhalo_found) {
  if (!members || !offsets || !nhalo_found || offsets_cap < 1) {
    set_error("pyfof_run_catalogue: null catalogue output");
    return kInvalid;
  }
  if (slot && static_cast<Context *>(slot)->magic != Context::kMagic) {
    set_error("pyfof_run_catalogue: not a slot");
    return kInvalid;
  }
  CatalogueOut cat{members, offsets, offsets_cap, nhalo_found};
  *nhalo_found = 0;
  return run_host_checked(static_cast<Context *>(slot), xp, vp, mp, layout, np_halo, nhalo, total_np, L_Box,
                          linking_length, np_halo_min, bound_check, verbose, softening, a_val, b_val,
                          s_15_val, n_threads, ng_val, ng_global_val, nullptr, halo_id, ang_mom, &cat,
                          units);
}

// ---------------------------------------------------------------- slots
// A slot is a context of its own (streams, scratch, status words) on one
// device; calls on different slots run concurrently on the GPU.

static bool valid_slot(void *slot) {
  return slot && static_cast<Context *>(slot)->magic == Context::kMagic;
}

int32_t pyfof_slot_create(int32_t device, int64_t pm_budget_bytes, void **slot) {
  if (!slot) {
    set_error("pyfof_slot_create: null handle pointer");
    return kInvalid;
  }
  *slot = nullptr;
  Context *c = nullptr;
  {
    std::lock_guard<std::mutex> lk(g_ctx_mu);
    PYFOF_TRY(create_context(device, &c));
  }
  if (pm_budget_bytes > 0) c->pm_budget = (size_t)pm_budget_bytes;
  *slot = c;
  return kOk;
}

int32_t pyfof_slot_destroy(void *slot) {
  if (!valid_slot(slot)) {
    set_error("pyfof_slot_destroy: not a slot");
    return kInvalid;
  }
  Context *c = static_cast<Context *>(slot);
  {
    std::lock_guard<std::mutex> lk(c->mu);
    cudaSetDevice(c->device);
  }
  c->magic = 0;
  delete c;
  return kOk;
}

int32_t pyfof_slot_run(void *slot, const double *xp, const double *vp, const double *mp,
                       int32_t layout, const int32_t *np_halo, int32_t nhalo, int64_t total_np,
                       double L_Box, double linking_length, int32_t np_halo_min, int32_t bound_check,
                       int32_t verbose, double softening, double a_val, double b_val, double s_15_val,
                       int32_t n_threads, int64_t ng_val, double ng_global_val, int32_t *in_halo,
                       int32_t *halo_id, double *ang_mom) {
  if (!valid_slot(slot)) {
    set_error("pyfof_slot_run: not a slot");
    return kInvalid;
  }
  return run_host_checked(static_cast<Context *>(slot), xp, vp, mp, layout, np_halo, nhalo, total_np,
                          L_Box, linking_length, np_halo_min, bound_check, verbose, softening, a_val,
                          b_val, s_15_val, n_threads, ng_val, ng_global_val, in_halo, halo_id, ang_mom);
}

int32_t pyfof_slot_stat(void *slot, const char *key, int64_t *value) {
  if (!valid_slot(slot) || !key || !value) {
    set_error("pyfof_slot_stat: invalid arguments");
    return kInvalid;
  }
  return context_stat(static_cast<Context *>(slot), key, value);
}

}  // extern "C"
