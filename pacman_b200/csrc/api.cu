// C ABI of the B200 RBF-PUM transfer (declared in include/pacman_b200.h).
//
// Each call validates its arguments like the reference's entry points
// (src/rbf_interface.cpp:109-128, src/pybindings/rbf_bindings.cpp:83-118),
// moves host inputs to the device on the call's stream, runs the geometry
// phase (geometry.cu), the patch solves (solve.cu, blocked.cu) and the
// partition-of-unity gather, and copies the result back when the caller
// passed a host pointer.  No exception crosses the ABI.
#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <string>

#include "plan.hpp"

struct pacman_b200_plan {
  pacman_b200::Plan p;
};

namespace pacman_b200 {

int64_t &launch_counter() {
  static thread_local int64_t c = 0;
  return c;
}

namespace {
thread_local std::string g_last_error;
}  // namespace

void set_last_error(const std::string &msg) { g_last_error = msg; }

HostArena &HostArena::get() {
  static thread_local HostArena arena;
  return arena;
}

void HostArena::reset() {
  for (char *b : retired_) cudaFreeHost(b);
  retired_.clear();
  used_ = 0;
}

void *HostArena::alloc(size_t bytes) {
  bytes = (bytes + 255) & ~size_t(255);
  if (used_ + bytes > cap_) {
    size_t cap = std::max<size_t>(cap_ * 2, std::max<size_t>(bytes, size_t(1) << 20));
    char *nb = nullptr;
    if (cudaHostAlloc(reinterpret_cast<void **>(&nb), cap, cudaHostAllocDefault) != cudaSuccess) {
      cudaGetLastError();
      throw Error{PACMAN_B200_ERR_NOMEM, "pinned host staging allocation failed"};
    }
    if (base_) retired_.push_back(base_);
    base_ = nb;
    cap_ = cap;
    used_ = 0;
  }
  void *p = base_ + used_;
  used_ += bytes;
  return p;
}

HostArena::~HostArena() {
  reset();
  if (base_) cudaFreeHost(base_);
}

namespace {

int fail(int code, const std::string &msg) {
  g_last_error = msg;
  return code;
}

// Keeps freed stream-ordered memory in the device pool between calls.
void tune_pool(int device) {
  static std::mutex mu;
  static bool done[64] = {false};
  std::lock_guard<std::mutex> lock(mu);
  if (device < 0 || device >= 64 || done[device]) return;
  cudaMemPool_t pool;
  if (cudaDeviceGetDefaultMemPool(&pool, device) == cudaSuccess) {
    uint64_t thr = UINT64_MAX;
    cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &thr);
  }
  cudaGetLastError();
  done[device] = true;
}

bool is_device_ptr(const void *ptr, int device) {
  if (!ptr) return false;
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, ptr) != cudaSuccess) {
    cudaGetLastError();
    return false;
  }
  if (at.type == cudaMemoryTypeManaged) return true;
  return at.type == cudaMemoryTypeDevice && at.device == device;
}

// Device view of a caller array: the pointer itself, or a staged copy.
struct InBuf {
  DevMem mem;
  const double *ptr = nullptr;
  void stage(const double *src, size_t count, int device, cudaStream_t st) {
    if (count == 0) {
      ptr = nullptr;
      return;
    }
    if (is_device_ptr(src, device)) {
      ptr = src;
      return;
    }
    mem.alloc(sizeof(double) * count, st);
    PB_CUDA(cudaMemcpyAsync(mem.p, src, sizeof(double) * count, cudaMemcpyHostToDevice, st));
    ptr = mem.as<double>();
  }
};

struct DeviceScope {
  int prev = -1;
  int dev = 0;
  explicit DeviceScope(int want) {
    PB_CUDA(cudaGetDevice(&prev));
    dev = (want >= 0) ? want : prev;
    if (dev != prev) PB_CUDA(cudaSetDevice(dev));
  }
  ~DeviceScope() {
    if (prev >= 0 && dev != prev) cudaSetDevice(prev);
  }
};

int check_basis(int32_t b) {
  if (b < PACMAN_B200_WENDLAND_C0 || b > PACMAN_B200_WENDLAND_C8)
    return fail(PACMAN_B200_ERR_INVALID,
                "Unsupported RBF function selector: " + std::to_string(b));
  return 0;
}

int check_opts(const pacman_b200_options &o) {
  if (o.nodes_per_cluster <= 0) return fail(PACMAN_B200_ERR_INVALID, "nodes_per_cluster must be > 0");
  if (!(o.relative_overlap > 0.0 && o.relative_overlap < 1.0))
    return fail(PACMAN_B200_ERR_INVALID, "relative_overlap must be in (0, 1)");
  if (!(o.support_radius > 0.0)) return fail(PACMAN_B200_ERR_INVALID, "support_radius must be > 0");
  if (o.precision != PACMAN_B200_FP64 && o.precision != PACMAN_B200_MIXED)
    return fail(PACMAN_B200_ERR_INVALID, "precision must be PACMAN_B200_FP64 or PACMAN_B200_MIXED");
  return 0;
}

int create_plan(int32_t dim, const double *src, int64_t n, const double *tgt, int64_t m,
                const pacman_b200_options *opts, pacman_b200_plan **out) {
  *out = nullptr;
  if (dim < 1 || dim > 3)
    return fail(PACMAN_B200_ERR_DIMENSION, "The dimension of the points can only be: 1, 2 or 3.");
  if (n < 0 || m < 0) return fail(PACMAN_B200_ERR_INVALID, "negative point count");
  if (src == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourcePoints is null but nSourcePoints > 0");
  if (tgt == nullptr && m > 0)
    return fail(PACMAN_B200_ERR_INVALID, "targetPoints is null but nTargetPoints > 0");
  if (n > 0x7fffffffll || m > 0x7fffffffll)
    return fail(PACMAN_B200_ERR_LIMIT, "point counts are limited to 2^31 - 1");
  pacman_b200_options o;
  pacman_b200_options_init(&o);
  if (opts) o = *opts;
  if (int rc = check_opts(o)) return rc;
  auto *h = new pacman_b200_plan();
  Plan &p = h->p;
  try {
    DeviceScope ds(o.device);
    tune_pool(ds.dev);
    HostArena::get().reset();
    p.device = ds.dev;
    p.dim = dim;
    p.n = n;
    p.m = m;
    p.opts = o;
    if (o.stream) {
      p.stream = static_cast<cudaStream_t>(o.stream);
    } else {
      PB_CUDA(cudaStreamCreateWithFlags(&p.stream, cudaStreamNonBlocking));
      p.own_stream = true;
    }
    if (n > 0) {
      InBuf s, t;
      s.stage(src, size_t(n) * dim, p.device, p.stream);
      t.stage(tgt, size_t(m) * dim, p.device, p.stream);
      const int64_t l0 = launch_counter();
      build_geometry(p, s.ptr, t.ptr);
      p.launches_geometry = launch_counter() - l0;
    }
  } catch (const Error &e) {
    delete h;
    return fail(e.code, e.msg);
  }
  *out = h;
  return 0;
}

int execute_plan(pacman_b200_plan *h, int32_t basis, const double *vals, int32_t F, double *out,
                 pacman_b200_stats *stats, uint32_t flags = 0) {
  if (!h) return fail(PACMAN_B200_ERR_INVALID, "plan is null");
  if (int rc = check_basis(basis)) return rc;
  Plan &p = h->p;
  if (F < 1 || F > 8) return fail(PACMAN_B200_ERR_INVALID, "n_fields must be in [1, 8]");
  if (vals == nullptr && p.n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourceValues is null but nSourcePoints > 0");
  if (out == nullptr && p.m > 0) return fail(PACMAN_B200_ERR_INVALID, "target_values is null");
  try {
    DeviceScope ds(p.device);
    HostArena::get().reset();
    cudaStream_t st = p.stream;
    cudaEvent_t e0, e1, e2;
    PB_CUDA(cudaEventCreate(&e0));
    PB_CUDA(cudaEventCreate(&e1));
    PB_CUDA(cudaEventCreate(&e2));
    PB_CUDA(cudaEventRecord(e0, st));
    const int64_t launches0 = launch_counter();
    p.saved_basis = -1;
    SolveReport rep;
    if (p.m > 0) {
      const bool out_dev = is_device_ptr(out, p.device);
      DevMem obuf;
      double *o = out;
      if (!out_dev) {
        obuf.alloc(sizeof(double) * size_t(p.m) * F, st);
        o = obuf.as<double>();
      }
      if (p.n == 0 || p.K == 0) {
        PB_CUDA(cudaMemsetAsync(o, 0, sizeof(double) * size_t(p.m) * F, st));
        PB_CUDA(cudaEventRecord(e1, st));
      } else {
        InBuf v;
        v.stage(vals, size_t(p.n) * F, p.device, st);
        p.local.alloc(sizeof(double) * size_t(std::max<int64_t>(p.tnnz, 1)) * F, st);
        rep.time_kernels = (flags & PACMAN_B200_TIME_KERNELS) != 0;
        solve_patches(p, basis, v.ptr, F, p.opts.precision, p.local.as<double>(), rep,
                      (flags & PACMAN_B200_SAVE_FOR_ADJOINT) != 0);
        PB_CUDA(cudaEventRecord(e1, st));
        pu_gather(p, p.local.as<double>(), F, o);
      }
      if (!out_dev)
        PB_CUDA(cudaMemcpyAsync(out, o, sizeof(double) * size_t(p.m) * F, cudaMemcpyDeviceToHost,
                                st));
    } else {
      PB_CUDA(cudaEventRecord(e1, st));
    }
    PB_CUDA(cudaEventRecord(e2, st));
    PB_CUDA(cudaEventSynchronize(e2));
    PB_CUDA(cudaGetLastError());
    if (flags & PACMAN_B200_SAVE_FOR_ADJOINT) {
      p.saved_basis = basis;
      p.saved_F = F;
    }
    if (stats) {
      float ms_solve = 0.f, ms_total = 0.f;
      cudaEventElapsedTime(&ms_solve, e0, e1);
      cudaEventElapsedTime(&ms_total, e0, e2);
      std::memset(stats, 0, sizeof(*stats));
      stats->radius = p.radius;
      stats->num_candidates = p.ncand;
      stats->num_patches = p.K;
      stats->sum_n = p.snnz;
      stats->sum_m = p.tnnz;
      int64_t mx = 0;
      for (int v : p.n_host) mx = std::max<int64_t>(mx, v);
      stats->max_n = mx;
      stats->patches_fp32 = rep.patches_fp32;
      stats->patches_fp64 = rep.patches_fp64;
      stats->patches_fallback = rep.patches_fallback;
      stats->dropped_axis_patches = rep.dropped;
      stats->ms_geometry = p.ms_geometry;
      stats->ms_solve = ms_solve;
      stats->ms_total = ms_total;
      stats->kernel_launches = launch_counter() - launches0 + p.launches_geometry;
      stats->ms_factor = rep.ms_factor;
      stats->factor_flops = rep.factor_flops;
      stats->ms_update = rep.ms_update;
      stats->update_flops = rep.update_flops;
      stats->update_launches = rep.update_launches;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

}  // namespace
}  // namespace pacman_b200

using namespace pacman_b200;

extern "C" {

void pacman_b200_options_init(pacman_b200_options *o) {
  if (!o) return;
  o->nodes_per_cluster = 50;
  o->relative_overlap = 0.15;
  o->support_radius = 0.1;
  o->precision = PACMAN_B200_FP64;
  o->device = -1;
  o->stream = nullptr;
}

const char *pacman_b200_last_error(void) { return g_last_error.c_str(); }
int32_t pacman_b200_abi_version(void) { return PACMAN_B200_ABI_VERSION; }

int pacman_b200_plan_create(int32_t dim, const double *src, int64_t n, const double *tgt,
                            int64_t m, const pacman_b200_options *opts, pacman_b200_plan **plan) {
  g_last_error.clear();
  if (!plan) return fail(PACMAN_B200_ERR_INVALID, "plan output pointer is null");
  return create_plan(dim, src, n, tgt, m, opts, plan);
}

int pacman_b200_plan_execute(pacman_b200_plan *plan, int32_t basis, const double *vals,
                             int32_t F, double *out, pacman_b200_stats *stats) {
  g_last_error.clear();
  return execute_plan(plan, basis, vals, F, out, stats);
}

int pacman_b200_plan_execute_ex(pacman_b200_plan *plan, int32_t basis, const double *vals,
                                int32_t F, double *out, uint32_t flags,
                                pacman_b200_stats *stats) {
  g_last_error.clear();
  return execute_plan(plan, basis, vals, F, out, stats, flags);
}

int pacman_b200_plan_adjoint(pacman_b200_plan *plan, const double *grad_out, double *grad_values,
                             double *grad_targets) {
  g_last_error.clear();
  if (!plan) return fail(PACMAN_B200_ERR_INVALID, "plan is null");
  Plan &p = plan->p;
  if (p.saved_basis < 0)
    return fail(PACMAN_B200_ERR_INVALID,
                "the adjoint needs a previous execute with PACMAN_B200_SAVE_FOR_ADJOINT");
  if (!grad_out && p.m > 0) return fail(PACMAN_B200_ERR_INVALID, "grad_target_values is null");
  try {
    DeviceScope ds(p.device);
    HostArena::get().reset();
    cudaStream_t st = p.stream;
    const int F = p.saved_F;
    InBuf g;
    g.stage(grad_out, size_t(p.m) * F, p.device, st);
    DevMem gv, gt;
    double *dv = grad_values, *dt = grad_targets;
    const bool hv = grad_values && !is_device_ptr(grad_values, p.device);
    const bool ht = grad_targets && !is_device_ptr(grad_targets, p.device);
    if (hv) {
      gv.alloc(sizeof(double) * std::max<int64_t>(p.n, 1) * F, st);
      dv = gv.as<double>();
    }
    if (ht) {
      gt.alloc(sizeof(double) * std::max<int64_t>(p.m, 1) * p.dim, st);
      dt = gt.as<double>();
    }
    adjoint(p, g.ptr, dv, dt);
    if (hv) PB_CUDA(cudaMemcpyAsync(grad_values, dv, sizeof(double) * p.n * F, cudaMemcpyDeviceToHost, st));
    if (ht) PB_CUDA(cudaMemcpyAsync(grad_targets, dt, sizeof(double) * p.m * p.dim, cudaMemcpyDeviceToHost, st));
    PB_CUDA(cudaStreamSynchronize(st));
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

void pacman_b200_plan_destroy(pacman_b200_plan *plan) {
  if (!plan) return;
  int prev = -1;
  cudaGetDevice(&prev);
  const int dev = plan->p.device;
  if (prev != dev) cudaSetDevice(dev);
  cudaStream_t st = plan->p.stream;
  const bool own = plan->p.own_stream;
  delete plan;  // frees device buffers stream-ordered on st
  if (own) {
    cudaStreamSynchronize(st);
    cudaStreamDestroy(st);
  }
  if (prev >= 0 && prev != dev) cudaSetDevice(prev);
  cudaGetLastError();
}

int pacman_b200_plan_info(const pacman_b200_plan *plan, double *radius, int64_t info[4]) {
  if (!plan) return fail(PACMAN_B200_ERR_INVALID, "plan is null");
  const Plan &p = plan->p;
  if (radius) *radius = p.radius;
  if (info) {
    info[0] = p.K;
    info[1] = p.ncand;
    info[2] = p.snnz;
    info[3] = p.tnnz;
  }
  return 0;
}

int pacman_b200_plan_centers(const pacman_b200_plan *plan, double *centers) {
  if (!plan || !centers) return fail(PACMAN_B200_ERR_INVALID, "null argument");
  const Plan &p = plan->p;
  try {
    DeviceScope ds(p.device);
    std::vector<double4> c(p.K);
    if (p.K)
      PB_CUDA(cudaMemcpyAsync(c.data(), p.centers.p, sizeof(double4) * p.K,
                              cudaMemcpyDeviceToHost, p.stream));
    PB_CUDA(cudaStreamSynchronize(p.stream));
    std::vector<double> h(size_t(p.K) * p.dim);
    for (int k = 0; k < p.K; ++k) {
      const double v[3] = {c[k].x, c[k].y, c[k].z};
      for (int d = 0; d < p.dim; ++d) h[size_t(k) * p.dim + d] = v[d];
    }
    if (!h.empty())
      PB_CUDA(cudaMemcpy(centers, h.data(), sizeof(double) * h.size(), cudaMemcpyDefault));
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_plan_patch_lists(const pacman_b200_plan *plan, int32_t which, int64_t *offsets,
                                 int32_t *indices) {
  if (!plan || !offsets) return fail(PACMAN_B200_ERR_INVALID, "null argument");
  if (which != 0 && which != 1) return fail(PACMAN_B200_ERR_INVALID, "which must be 0 or 1");
  const Plan &p = plan->p;
  try {
    DeviceScope ds(p.device);
    const DevMem &off = which == 0 ? p.soff : p.toff;
    const DevMem &idx = which == 0 ? p.sidx : p.tidx;
    const int64_t nnz = which == 0 ? p.snnz : p.tnnz;
    if (p.K > 0) {
      PB_CUDA(cudaMemcpyAsync(offsets, off.p, sizeof(int64_t) * (p.K + 1), cudaMemcpyDefault,
                              p.stream));
      if (nnz > 0 && indices)
        PB_CUDA(cudaMemcpyAsync(indices, idx.p, sizeof(int32_t) * nnz, cudaMemcpyDefault,
                                p.stream));
    } else {
      offsets[0] = 0;
    }
    PB_CUDA(cudaStreamSynchronize(p.stream));
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_plan_local_values(const pacman_b200_plan *plan, double *local) {
  if (!plan || !local) return fail(PACMAN_B200_ERR_INVALID, "null argument");
  const Plan &p = plan->p;
  if (!p.local.p) return fail(PACMAN_B200_ERR_INVALID, "plan has not been executed");
  try {
    DeviceScope ds(p.device);
    PB_CUDA(cudaMemcpyAsync(local, p.local.p, p.local.bytes, cudaMemcpyDefault, p.stream));
    PB_CUDA(cudaStreamSynchronize(p.stream));
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_rbf_interpolate(int32_t dim, int32_t basis, const double *src, int64_t n,
                                const double *vals, int32_t F, const double *tgt, int64_t m,
                                double *out, const pacman_b200_options *opts,
                                pacman_b200_stats *stats) {
  g_last_error.clear();
  if (int rc = check_basis(basis)) return rc;
  if (F < 1 || F > 8) return fail(PACMAN_B200_ERR_INVALID, "n_fields must be in [1, 8]");
  if (vals == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourceValues is null but nSourcePoints > 0");
  pacman_b200_plan *plan = nullptr;
  int rc = create_plan(dim, src, n, tgt, m, opts, &plan);
  if (rc) return rc;
  rc = execute_plan(plan, basis, vals, F, out, stats);
  pacman_b200_plan_destroy(plan);
  return rc;
}

}  // extern "C"
