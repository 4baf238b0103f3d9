// Internal host-side state of one RBF-PUM transfer on one GPU.
#pragma once

#include <cstdint>
#include <cstring>
#include <memory>
#include <string>
#include <vector>

#include <cuda_runtime.h>

#include "../../include/pacman_b200.h"
#include "common.cuh"

namespace pacman_b200 {

// Error carried from the kernels' host wrappers to the C ABI.
struct Error {
  int code;
  std::string msg;
};

#define PB_CUDA(call)                                                          \
  do {                                                                         \
    cudaError_t e_ = (call);                                                   \
    if (e_ != cudaSuccess)                                                     \
      throw ::pacman_b200::Error{PACMAN_B200_ERR_CUDA,                         \
                                 std::string(#call) + ": " + cudaGetErrorString(e_)}; \
  } while (0)

// Stream-ordered device allocation owned by a plan.
struct DevMem {
  void *p = nullptr;
  size_t bytes = 0;
  cudaStream_t s = nullptr;
  DevMem() = default;
  DevMem(const DevMem &) = delete;
  DevMem &operator=(const DevMem &) = delete;
  DevMem(DevMem &&o) noexcept : p(o.p), bytes(o.bytes), s(o.s) {
    o.p = nullptr;
    o.bytes = 0;
  }
  DevMem &operator=(DevMem &&o) noexcept {
    if (this != &o) {
      release();
      p = o.p;
      bytes = o.bytes;
      s = o.s;
      o.p = nullptr;
      o.bytes = 0;
    }
    return *this;
  }
  ~DevMem() { release(); }
  void release() {
    if (p) cudaFreeAsync(p, s);
    p = nullptr;
    bytes = 0;
  }
  void alloc(size_t nbytes, cudaStream_t stream) {
    if (nbytes <= bytes && p) return;
    release();
    s = stream;
    if (nbytes == 0) nbytes = 16;
    cudaError_t e = cudaMallocAsync(&p, nbytes, stream);
    if (e != cudaSuccess) {
      cudaGetLastError();
      p = nullptr;
      throw Error{PACMAN_B200_ERR_NOMEM,
                  "device allocation of " + std::to_string(nbytes) + " bytes failed"};
    }
    bytes = nbytes;
  }
  template <typename T> T *as() const { return static_cast<T *>(p); }
};

struct DevGrid {
  GridView view{};
  DevMem start, items;
};

// Extra streams of a plan, created on first use on the plan's device: one per
// independent group of large patches (high priority) and one for the small
// patches (low priority: they fill the SMs the large-patch steps leave idle).
// Every use joins them back into the plan's stream with events before the
// call returns.
struct AuxStreams {
  static constexpr int kN = 8;      // slot groups of the large-patch engine (at most)
  static constexpr int kDefaultGroups = 4;  // without a tuned or given count
  static constexpr int kSmall = kN; // index of the small-patch stream
  cudaStream_t s[kN + 1] = {};
  cudaEvent_t ev[kN + 3] = {};      // per group, fork, small fork, small join
  bool made = false;
  void make() {
    if (made) return;
    int least = 0, greatest = 0;
    if (cudaDeviceGetStreamPriorityRange(&least, &greatest) != cudaSuccess)
      throw Error{PACMAN_B200_ERR_CUDA, "cudaDeviceGetStreamPriorityRange failed"};
    for (int i = 0; i <= kN; ++i) {
      if (cudaStreamCreateWithPriority(&s[i], cudaStreamNonBlocking,
                                       i == kSmall ? least : greatest) != cudaSuccess)
        throw Error{PACMAN_B200_ERR_CUDA, "cudaStreamCreateWithPriority failed"};
    }
    for (int i = 0; i < kN + 3; ++i) {
      if (cudaEventCreateWithFlags(&ev[i], cudaEventDisableTiming) != cudaSuccess)
        throw Error{PACMAN_B200_ERR_CUDA, "cudaEventCreateWithFlags failed"};
    }
    made = true;
  }
  AuxStreams() = default;
  AuxStreams(const AuxStreams &) = delete;
  AuxStreams &operator=(const AuxStreams &) = delete;
  ~AuxStreams() {
    for (int i = 0; i <= kN; ++i)
      if (s[i]) cudaStreamDestroy(s[i]);
    for (int i = 0; i < kN + 3; ++i)
      if (ev[i]) cudaEventDestroy(ev[i]);
  }
};

// Factorisations kept by an execute with PACMAN_B200_KEEP_FACTORS (defined
// in blocked.cuh; destroyed through destroy_factor_cache).
struct FactorCache;
void destroy_factor_cache(FactorCache *c);
struct FactorCacheDeleter {
  void operator()(FactorCache *c) const { destroy_factor_cache(c); }
};

struct Plan {
  int dim = 3;
  int64_t n = 0, m = 0;
  int device = 0;
  cudaStream_t stream = nullptr;
  bool own_stream = false;
  pacman_b200_options opts{};

  DevMem src4, tgt4;  // double4 AoS, zero padded
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  double radius = 0.0;
  int64_t ncand = 0;
  int K = 0;
  DevMem centers;  // double4[K]
  DevMem soff, sidx, toff, tidx;  // int64 offsets, int32 ids
  int64_t snnz = 0, tnnz = 0;
  std::vector<int> n_host, m_host;  // per patch sizes
  DevGrid cgrid;                    // grid of centres (weights)
  DevMem scratch;                   // solver workspace
  DevMem local;                     // per (patch, target) local values
  DevMem status;                    // per patch status words
  std::vector<int> patch_status;    // status words of the last execute (host copy)
  double ms_geometry = -1.0;         // device time of the geometry (read lazily)
  cudaEvent_t geom_ev[2] = {nullptr, nullptr};  // around the geometry, until read
  Plan() = default;
  Plan(const Plan &) = delete;
  Plan &operator=(const Plan &) = delete;
  ~Plan() {
    for (cudaEvent_t e : geom_ev)
      if (e) cudaEventDestroy(e);
  }
  int64_t dropped_axis_patches = 0;
  // State saved by an execute for the adjoint (pacman_b200_plan_adjoint).
  int saved_basis = -1, saved_F = 0;
  DevMem alpha;              // RBF coefficients, source-membership order x F
  DevMem beta;               // K x 4*8 polynomial coefficients
  DevMem act;                // K x 3 active axes
  DevMem src_t_off, src_t_pos;  // sources -> (patch, slot) transpose of the membership lists
  // Target shard (pacman_b200_plan_shard): the owned targets ascending, and
  // their count; m_owned < 0 for an unsharded plan.
  int shard_rank = 0, shard_world = 1;
  int64_t m_owned = -1;
  DevMem tlist;
  int64_t launches_geometry = 0;  // kernel launches of the geometry phase
  int64_t syncs_geometry = 0;     // host waits of the geometry phase
  int64_t launches = 0;           // kernel launches of the current execute
  AuxStreams aux;
  std::unique_ptr<FactorCache, FactorCacheDeleter> fcache;  // kept factorisations, or null
};

// Pinned host staging for the small host-to-device uploads of one call.  A
// copy from pageable memory first synchronises its stream, which would stall
// the host behind every queued kernel; copies from this arena do not.  The
// arena is reset at the start of each call (the previous call synchronised
// before returning), blocks outgrown in the middle of a call are released at
// the next reset.
class HostArena {
 public:
  static HostArena &get();
  void reset();
  void *alloc(size_t bytes);
  template <typename T> T *upload(const T *src, size_t count, void *dst, cudaStream_t st) {
    if (count == 0) return static_cast<T *>(dst);
    void *h = alloc(sizeof(T) * count);
    std::memcpy(h, src, sizeof(T) * count);
    PB_CUDA(cudaMemcpyAsync(dst, h, sizeof(T) * count, cudaMemcpyHostToDevice, st));
    return static_cast<T *>(dst);
  }
  ~HostArena();

 private:
  char *base_ = nullptr;
  size_t cap_ = 0, used_ = 0;
  std::vector<char *> retired_;
};

// Launch parameters of the patch solvers for the current device: the tuned
// file of its GPU model (tuning/<name>.conf beside the library) or the
// built-in defaults (tuning.cpp).
struct Tuning {
  int big_n_chol = 64;  // patches above this size use the tiled Cholesky (mixed)
  int int8_from = 4;    // first tile column updated on the int8 tensor cores
  int groups = 0;       // slot groups of the tiled engine (0: min(4, slots / 8))
  int back_stages = 3;  // ring depth of the one-field backward sweep (3 or 6)
  int sms = 148;
  std::string source = "built-in defaults";
};
const Tuning &tuning_for_current_device();
// The environment variable if set, else the tuned value.
int tuned_int(const char *env, int value);

// Launch counter of this library's own kernels on the calling thread.
int64_t &launch_counter();
inline void note_launch(int k = 1) { launch_counter() += k; }
// Counter of the calling thread's host waits for the device, and the waits
// themselves (every wait of a transfer goes through these).
int64_t &host_sync_counter();
inline cudaError_t host_sync(cudaStream_t s) {
  ++host_sync_counter();
  return cudaStreamSynchronize(s);
}
inline cudaError_t host_sync_event(cudaEvent_t e) {
  ++host_sync_counter();
  return cudaEventSynchronize(e);
}

// geometry.cu
void build_geometry(Plan &p, const double *src_dev, const double *tgt_dev);
// Device time of the plan's geometry phase: read from its events once the
// stream has passed them (callers have synchronised it), then cached.
double geometry_ms(Plan &p);
void pu_gather(Plan &p, const double *local, int F, double *out_dev);
// Packed double4 points with their exact bounding box, and the uniform cell
// grid over them (geometry.cu; used by nearest.cu).
void pack_points(const double *in_dev, int dim, int64_t n, DevMem &out4, double lo[3],
                 double hi[3], cudaStream_t st);
void build_point_grid(DevGrid &out, const double4 *pts, int64_t n, int dim, const double *lo,
                      const double *hi, double cell, cudaStream_t st);
// Finite-element NEAREST_NEAREST transfer (nearest.cu).
void fe_nearest(int dim, const double *src_dev, int64_t n, const double *vals_dev,
                const double *tgt_dev, int64_t m, double *out_dev, cudaStream_t st);
// Moving least squares transfer (mls.cu).
void mls_interpolate(int dim, const double *src_dev, int64_t n, const double *vals_dev,
                     const double *tgt_dev, int64_t m, double *out_dev, cudaStream_t st);
// Restricts the plan to target shard `rank` of `world` (shard.cu).
void shard_plan(Plan &p, int rank, int world);

// solve.cu
struct SolveReport {
  int64_t patches_fp32 = 0, patches_fp64 = 0, patches_fallback = 0, dropped = 0;
  double ms_factor = 0.0;     // device time of the factorisation launches
  double factor_flops = 0.0;  // their algorithmic FLOPs
  bool time_kernels = false;  // input: event-time the column-update launches
  // input: re-recorded by the large-patch engine where its steps stop filling
  // the GPU (the small patches start there), or null
  cudaEvent_t tail_event = nullptr;
  double ms_update = 0.0, update_flops = 0.0;
  int64_t update_launches = 0;
  // Per kind (0: FP64 steps k_col_step, 1: int8 steps k_col_step_ws): span
  // of device time with at least one launch of the kind running, FLOPs and
  // launch count (time_kernels only).
  double ms_kind[2] = {0.0, 0.0}, flops_kind[2] = {0.0, 0.0};
  int64_t launches_kind[2] = {0, 0};
  double mma_products_i8 = 0.0;
  // Events around each timed step launch, on the launching stream; resolved
  // by finish_kernel_timing once the solve has completed.
  struct TimedLaunch {
    cudaEvent_t e0, e1;
    int kind;
    double flops;
    double mma_products;  // int8 tile products (kind 1)
  };
  std::vector<TimedLaunch> timed;
  int64_t factors_reused = 0;  // patches solved from kept factorisations
};
// Turns the recorded launch events into the spans of SolveReport (ref: an
// event recorded on the solve's stream before any timed launch, complete).
void finish_kernel_timing(SolveReport &rep, cudaEvent_t ref);
void solve_patches(Plan &p, int basis, const double *vals_dev, int F, int precision,
                   double *local_dev, SolveReport &rep, bool save_state = false,
                   bool keep_factors = false);

// Extra inputs / outputs of the blocked engine beyond the forward transfer.
enum { kBigForward = 0, kBigForwardSave = 1, kBigAdjoint = 2 };
struct BigExtra {
  int mode = kBigForward;
  double *alpha_out = nullptr;  // forward + save
  double *beta_out = nullptr;
  int *act_out = nullptr;
  const double *h = nullptr;    // adjoint
  double *g_out = nullptr;
};

// adjoint.cu
void adjoint(Plan &p, const double *grad_out_dev, double *grad_values_dev,
             double *grad_targets_dev);

}  // namespace pacman_b200
