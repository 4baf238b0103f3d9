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
#include <atomic>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "plan.hpp"

struct pacman_b200_plan {
  pacman_b200::Plan p;
};

namespace pacman_b200 {

int64_t &launch_counter() {
  static thread_local int64_t c = 0;
  return c;
}

int64_t &host_sync_counter() {
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
      const int64_t l0 = launch_counter(), h0 = host_sync_counter();
      build_geometry(p, s.ptr, t.ptr);
      p.launches_geometry = launch_counter() - l0;
      p.syncs_geometry = host_sync_counter() - h0;
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
    const int64_t launches0 = launch_counter(), syncs0 = host_sync_counter();
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
                      (flags & PACMAN_B200_SAVE_FOR_ADJOINT) != 0,
                      (flags & PACMAN_B200_KEEP_FACTORS) != 0);
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
    PB_CUDA(host_sync_event(e2));
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
      stats->ms_geometry = geometry_ms(p);
      stats->ms_solve = ms_solve;
      stats->ms_total = ms_total;
      stats->kernel_launches = launch_counter() - launches0 + p.launches_geometry;
      stats->host_syncs = host_sync_counter() - syncs0 + p.syncs_geometry;
      stats->ms_factor = rep.ms_factor;
      stats->factor_flops = rep.factor_flops;
      stats->ms_update = rep.ms_update;
      stats->update_flops = rep.update_flops;
      stats->update_launches = rep.update_launches;
      stats->ms_update_i8 = rep.ms_kind[1];
      stats->update_flops_i8 = rep.flops_kind[1];
      stats->update_launches_i8 = rep.launches_kind[1];
      stats->ms_update_f64 = rep.ms_kind[0];
      stats->update_flops_f64 = rep.flops_kind[0];
      stats->update_launches_f64 = rep.launches_kind[0];
      stats->mma_products_i8 = rep.mma_products_i8;
      stats->factors_reused = rep.factors_reused;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}


// ---------------------------------------------------------------------------
// Batched transfers.  Each problem keeps its own geometry (radius, centres,
// membership lists).  The patches of all problems with the same dimension and
// basis are then concatenated into one merged plan: points, centres and lists
// are copied side by side with the list entries shifted by the running point
// and membership counts, the source values are laid out with the group's
// largest field count (missing fields zero), and one solve covers every patch
// of the group.  The local values of problem i are then the merged local
// values from its first membership on, and its own partition-of-unity gather
// turns them into its targets' values.

__global__ void k_shift_i64(const int64_t *__restrict__ in, int64_t n, int64_t add,
                            int64_t *__restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = in[i] + add;
}

__global__ void k_shift_i32(const int *__restrict__ in, int64_t n, int add,
                            int *__restrict__ out) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < n;
       i += int64_t(gridDim.x) * blockDim.x)
    out[i] = in[i] + add;
}

// dst[r, f] = src[r, f] for the first `cols` fields of `rows` rows (row
// strides sf and df doubles): field-count changes between a problem's arrays
// and the merged layout.
__global__ void k_copy_fields(const double *__restrict__ src, int sf, double *__restrict__ dst,
                              int df, int cols, int64_t rows) {
  const int64_t n = rows * cols;
  for (int64_t e = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; e < n;
       e += int64_t(gridDim.x) * blockDim.x) {
    const int64_t r = e / cols;
    const int f = int(e - r * cols);
    dst[r * df + f] = src[r * sf + f];
  }
}

int shift_grid(int64_t n) {
  return int(std::max<int64_t>(1, std::min<int64_t>((n + 255) / 256, 148 * 8)));
}

void copy_fields(const double *src, int sf, double *dst, int df, int cols, int64_t rows,
                 cudaStream_t st) {
  if (rows <= 0) return;
  k_copy_fields<<<shift_grid(rows * cols), 256, 0, st>>>(src, sf, dst, df, cols, rows);
  note_launch();
}

int check_problem(const pacman_b200_problem &q, int32_t i) {
  const std::string at = "problem " + std::to_string(i) + ": ";
  if (q.dim < 1 || q.dim > 3)
    return fail(PACMAN_B200_ERR_DIMENSION,
                at + "The dimension of the points can only be: 1, 2 or 3.");
  if (int rc = check_basis(q.rbf_function)) return fail(rc, at + g_last_error);
  if (q.n_fields < 1 || q.n_fields > 8)
    return fail(PACMAN_B200_ERR_INVALID, at + "n_fields must be in [1, 8]");
  if (q.n_source < 0 || q.n_target < 0)
    return fail(PACMAN_B200_ERR_INVALID, at + "negative point count");
  if ((q.source_points == nullptr || q.source_values == nullptr) && q.n_source > 0)
    return fail(PACMAN_B200_ERR_INVALID, at + "source arrays are null but n_source > 0");
  if ((q.target_points == nullptr || q.target_values == nullptr) && q.n_target > 0)
    return fail(PACMAN_B200_ERR_INVALID, at + "target arrays are null but n_target > 0");
  return 0;
}

struct PlanHandle {
  pacman_b200_plan *h = nullptr;
  PlanHandle() = default;
  PlanHandle(const PlanHandle &) = delete;
  PlanHandle &operator=(const PlanHandle &) = delete;
  ~PlanHandle() {
    if (h) pacman_b200_plan_destroy(h);
  }
};

// Host threads that build the per-problem geometry of a batch, one stream
// each.  The plans keep those streams for their stream-ordered frees, so the
// streams live until release(), after the plans are gone.
struct GeometryWorkers {
  std::vector<cudaStream_t> streams;
  int run(const pacman_b200_problem *qs, int32_t count, const pacman_b200_options &o, int dev,
          std::vector<PlanHandle> &plans) {
    int nt = 8;
    if (const char *e = std::getenv("PACMAN_B200_BATCH_THREADS")) nt = std::atoi(e);
    nt = std::max(1, std::min<int>(nt, count));
    streams.assign(size_t(nt), nullptr);
    for (auto &s : streams) PB_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    std::atomic<int> next{0};
    std::atomic<bool> stop{false};
    std::vector<int> rcs(size_t(count), 0);
    std::vector<std::string> msgs(static_cast<size_t>(count));
    auto work = [&](int w) {
      cudaSetDevice(dev);
      pacman_b200_options ow = o;
      ow.stream = streams[size_t(w)];
      for (int i = next++; i < count && !stop; i = next++) {
        const pacman_b200_problem &q = qs[i];
        const int rc = create_plan(q.dim, q.source_points, q.n_source, q.target_points,
                                   q.n_target, &ow, &plans[size_t(i)].h);
        if (rc) {
          rcs[size_t(i)] = rc;
          msgs[size_t(i)] = g_last_error;
          stop = true;
        }
      }
    };
    std::vector<std::thread> th;
    for (int w = 1; w < nt; ++w) th.emplace_back(work, w);
    work(0);
    for (auto &t : th) t.join();
    for (int32_t i = 0; i < count; ++i)
      if (rcs[size_t(i)]) return fail(rcs[size_t(i)], "problem " + std::to_string(i) + ": " + msgs[size_t(i)]);
    return 0;
  }
  void release() {
    for (auto s : streams) {
      if (!s) continue;
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    streams.clear();
  }
  ~GeometryWorkers() { release(); }
};

// Solves the patches of the problems `ids` (same dim and basis) as one merged
// plan and writes every problem's target values.
void solve_group(const pacman_b200_problem *qs, const std::vector<int> &ids,
                 std::vector<PlanHandle> &plans, const pacman_b200_options &o, cudaStream_t st,
                 int device, SolveReport &rep) {
  HostArena::get().reset();  // the previous group has synchronised
  Plan g;
  g.device = device;
  g.stream = st;
  g.opts = o;
  g.dim = qs[ids[0]].dim;
  int Fg = 1;
  int64_t N = 0, M = 0, K = 0, snnz = 0, tnnz = 0;
  for (int i : ids) {
    const Plan &p = plans[i].h->p;
    Fg = std::max(Fg, int(qs[i].n_fields));
    N += p.n;
    M += p.m;
    K += p.K;
    snnz += p.snnz;
    tnnz += p.tnnz;
  }
  if (N > 0x7fffffffll || M > 0x7fffffffll || K > 0x7fffffffll || snnz > 0x7fffffffll ||
      tnnz > 0x7fffffffll)
    throw Error{PACMAN_B200_ERR_LIMIT,
                "a batch group is limited to 2^31 - 1 points, patches and memberships"};
  g.n = N;
  g.m = M;
  g.K = int(K);
  g.snnz = snnz;
  g.tnnz = tnnz;
  g.src4.alloc(sizeof(double4) * std::max<int64_t>(N, 1), st);
  g.tgt4.alloc(sizeof(double4) * std::max<int64_t>(M, 1), st);
  g.centers.alloc(sizeof(double4) * std::max<int64_t>(K, 1), st);
  g.soff.alloc(sizeof(int64_t) * (K + 1), st);
  g.toff.alloc(sizeof(int64_t) * (K + 1), st);
  g.sidx.alloc(sizeof(int) * std::max<int64_t>(snnz, 1), st);
  g.tidx.alloc(sizeof(int) * std::max<int64_t>(tnnz, 1), st);
  DevMem vals;
  vals.alloc(sizeof(double) * std::max<int64_t>(N, 1) * Fg, st);
  PB_CUDA(cudaMemsetAsync(vals.p, 0, sizeof(double) * std::max<int64_t>(N, 1) * Fg, st));
  g.n_host.reserve(size_t(K));
  g.m_host.reserve(size_t(K));
  std::vector<int64_t> toff_of(ids.size());
  int64_t n0 = 0, m0 = 0, k0 = 0, s0 = 0, t0 = 0;
  for (size_t u = 0; u < ids.size(); ++u) {
    const int i = ids[u];
    const Plan &p = plans[i].h->p;
    const pacman_b200_problem &q = qs[i];
    toff_of[u] = t0;
    if (p.n > 0) {
      InBuf v;
      v.stage(q.source_values, size_t(p.n) * q.n_fields, device, st);
      copy_fields(v.ptr, q.n_fields, vals.as<double>() + n0 * Fg, Fg, q.n_fields, p.n, st);
    }
    if (p.n > 0)
      PB_CUDA(cudaMemcpyAsync(g.src4.as<double4>() + n0, p.src4.p, sizeof(double4) * p.n,
                              cudaMemcpyDeviceToDevice, st));
    if (p.m > 0)
      PB_CUDA(cudaMemcpyAsync(g.tgt4.as<double4>() + m0, p.tgt4.p, sizeof(double4) * p.m,
                              cudaMemcpyDeviceToDevice, st));
    if (p.K > 0) {
      PB_CUDA(cudaMemcpyAsync(g.centers.as<double4>() + k0, p.centers.p, sizeof(double4) * p.K,
                              cudaMemcpyDeviceToDevice, st));
      k_shift_i64<<<shift_grid(p.K + 1), 256, 0, st>>>(p.soff.as<int64_t>(), p.K + 1, s0,
                                                       g.soff.as<int64_t>() + k0);
      k_shift_i64<<<shift_grid(p.K + 1), 256, 0, st>>>(p.toff.as<int64_t>(), p.K + 1, t0,
                                                       g.toff.as<int64_t>() + k0);
      note_launch(2);
      if (p.snnz > 0) {
        k_shift_i32<<<shift_grid(p.snnz), 256, 0, st>>>(p.sidx.as<int>(), p.snnz, int(n0),
                                                        g.sidx.as<int>() + s0);
        note_launch();
      }
      if (p.tnnz > 0) {
        k_shift_i32<<<shift_grid(p.tnnz), 256, 0, st>>>(p.tidx.as<int>(), p.tnnz, int(m0),
                                                        g.tidx.as<int>() + t0);
        note_launch();
      }
      g.n_host.insert(g.n_host.end(), p.n_host.begin(), p.n_host.end());
      g.m_host.insert(g.m_host.end(), p.m_host.begin(), p.m_host.end());
    }
    n0 += p.n;
    m0 += p.m;
    k0 += p.K;
    s0 += p.snnz;
    t0 += p.tnnz;
  }
  PB_CUDA(cudaGetLastError());
  g.local.alloc(sizeof(double) * std::max<int64_t>(tnnz, 1) * Fg, st);
  solve_patches(g, qs[ids[0]].rbf_function, vals.as<double>(), Fg, o.precision,
                g.local.as<double>(), rep, false);
  DevMem obuf, obuf2;
  for (size_t u = 0; u < ids.size(); ++u) {
    const int i = ids[u];
    Plan &p = plans[i].h->p;
    const pacman_b200_problem &q = qs[i];
    if (p.m == 0) continue;
    p.stream = st;  // the gather is ordered after the merged solve
    const bool out_dev = is_device_ptr(q.target_values, device);
    const bool direct = q.n_fields == Fg && out_dev;
    double *o = q.target_values;
    if (!direct) {
      obuf.alloc(sizeof(double) * size_t(p.m) * Fg, st);
      o = obuf.as<double>();
    }
    pu_gather(p, g.local.as<double>() + toff_of[u] * Fg, Fg, o);
    if (direct) continue;
    if (out_dev) {
      copy_fields(o, Fg, q.target_values, q.n_fields, q.n_fields, p.m, st);
      continue;
    }
    const double *h = o;
    if (q.n_fields != Fg) {
      obuf2.alloc(sizeof(double) * size_t(p.m) * q.n_fields, st);
      copy_fields(o, Fg, obuf2.as<double>(), q.n_fields, q.n_fields, p.m, st);
      h = obuf2.as<double>();
    }
    PB_CUDA(cudaMemcpyAsync(q.target_values, h, sizeof(double) * size_t(p.m) * q.n_fields,
                            cudaMemcpyDeviceToHost, st));
  }
  PB_CUDA(host_sync(st));
  g.stream = st;  // merged buffers are freed stream-ordered on the batch stream
}

int run_batch(const pacman_b200_problem *qs, int32_t count, const pacman_b200_options *opts,
              pacman_b200_stats *stats) {
  if (count < 0) return fail(PACMAN_B200_ERR_INVALID, "count must be >= 0");
  if (count > 0 && qs == nullptr) return fail(PACMAN_B200_ERR_INVALID, "problems is null");
  pacman_b200_options o;
  pacman_b200_options_init(&o);
  if (opts) o = *opts;
  if (int rc = check_opts(o)) return rc;
  for (int32_t i = 0; i < count; ++i)
    if (int rc = check_problem(qs[i], i)) return rc;
  if (stats) std::memset(stats, 0, sizeof(*stats));
  if (count == 0) return 0;
  cudaStream_t own = nullptr;
  try {
    DeviceScope ds(o.device);
    o.device = ds.dev;
    if (!o.stream) {
      PB_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
      o.stream = own;
    }
    cudaStream_t st = static_cast<cudaStream_t>(o.stream);
    cudaEvent_t e0, e1, e2;
    PB_CUDA(cudaEventCreate(&e0));
    PB_CUDA(cudaEventCreate(&e1));
    PB_CUDA(cudaEventCreate(&e2));
    PB_CUDA(cudaEventRecord(e0, st));
    const int64_t launches0 = launch_counter(), syncs0 = host_sync_counter();
    // Geometry per problem on a few host threads, each with its own stream:
    // the geometry phase waits on the device several times, and the threads
    // overlap those waits and the small launches of different problems.
    GeometryWorkers gw;  // declared first: its streams outlive the plans
    std::vector<PlanHandle> plans(static_cast<size_t>(count));
    int rc = gw.run(qs, count, o, ds.dev, plans);
    if (rc) {
      plans.clear();
      gw.release();
      cudaEventDestroy(e0);
      cudaEventDestroy(e1);
      cudaEventDestroy(e2);
      if (own) cudaStreamDestroy(own);
      return rc;
    }
    PB_CUDA(cudaEventRecord(e1, st));
    // Problems with targets but no patches get zeros; the rest are grouped by
    // (dim, basis) in first-seen order.
    std::vector<std::pair<int, int>> keys;
    std::vector<std::vector<int>> groups;
    for (int32_t i = 0; i < count; ++i) {
      const Plan &p = plans[i].h->p;
      const pacman_b200_problem &q = qs[i];
      if (p.m == 0) continue;
      if (p.n == 0 || p.K == 0) {
        const size_t bytes = sizeof(double) * size_t(p.m) * q.n_fields;
        if (is_device_ptr(q.target_values, ds.dev))
          PB_CUDA(cudaMemsetAsync(q.target_values, 0, bytes, st));
        else
          std::memset(q.target_values, 0, bytes);
        continue;
      }
      const std::pair<int, int> key(q.dim, q.rbf_function);
      size_t gi = 0;
      while (gi < keys.size() && keys[gi] != key) ++gi;
      if (gi == keys.size()) {
        keys.push_back(key);
        groups.emplace_back();
      }
      groups[gi].push_back(i);
    }
    SolveReport rep;
    for (const auto &ids : groups) solve_group(qs, ids, plans, o, st, ds.dev, rep);
    PB_CUDA(cudaEventRecord(e2, st));
    PB_CUDA(host_sync_event(e2));
    PB_CUDA(cudaGetLastError());
    if (stats) {
      float ms_solve = 0.f, ms_total = 0.f;
      cudaEventElapsedTime(&ms_solve, e1, e2);
      cudaEventElapsedTime(&ms_total, e0, e2);
      double rmax = 0.0;
      for (int32_t i = 0; i < count; ++i) {
        Plan &p = plans[i].h->p;
        rmax = std::max(rmax, p.radius);
        stats->num_candidates += p.ncand;
        stats->num_patches += p.K;
        stats->sum_n += p.snnz;
        stats->sum_m += p.tnnz;
        for (int v : p.n_host) stats->max_n = std::max<int64_t>(stats->max_n, v);
        stats->ms_geometry += geometry_ms(p);
      }
      stats->radius = rmax;
      stats->patches_fp32 = rep.patches_fp32;
      stats->patches_fp64 = rep.patches_fp64;
      stats->patches_fallback = rep.patches_fallback;
      stats->dropped_axis_patches = rep.dropped;
      stats->ms_solve = ms_solve;
      stats->ms_total = ms_total;
      stats->kernel_launches = launch_counter() - launches0;
      for (int32_t i = 0; i < count; ++i) stats->kernel_launches += plans[i].h->p.launches_geometry;
      stats->host_syncs = host_sync_counter() - syncs0;
      for (int32_t i = 0; i < count; ++i) stats->host_syncs += plans[i].h->p.syncs_geometry;
      stats->ms_factor = rep.ms_factor;
      stats->factor_flops = rep.factor_flops;
      stats->ms_update = rep.ms_update;
      stats->update_flops = rep.update_flops;
      stats->update_launches = rep.update_launches;
      stats->ms_update_i8 = rep.ms_kind[1];
      stats->update_flops_i8 = rep.flops_kind[1];
      stats->update_launches_i8 = rep.launches_kind[1];
      stats->ms_update_f64 = rep.ms_kind[0];
      stats->update_flops_f64 = rep.flops_kind[0];
      stats->update_launches_f64 = rep.launches_kind[0];
      stats->mma_products_i8 = rep.mma_products_i8;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaEventDestroy(e2);
    plans.clear();
    gw.release();
    if (own) {
      cudaStreamSynchronize(own);
      cudaStreamDestroy(own);
      own = nullptr;
    }
  } catch (const Error &e) {
    if (own) {
      cudaStreamSynchronize(own);
      cudaStreamDestroy(own);
    }
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
    PB_CUDA(host_sync(st));
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
    PB_CUDA(host_sync(p.stream));
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
    PB_CUDA(host_sync(p.stream));
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
    PB_CUDA(host_sync(p.stream));
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_plan_patch_status(const pacman_b200_plan *plan, int32_t *status) {
  if (!plan || !status) return fail(PACMAN_B200_ERR_INVALID, "null argument");
  const Plan &p = plan->p;
  if (p.K > 0 && p.patch_status.size() != size_t(p.K))
    return fail(PACMAN_B200_ERR_INVALID, "plan has not been executed");
  for (int k = 0; k < p.K; ++k) status[k] = p.patch_status[size_t(k)];
  return 0;
}

int pacman_b200_fe_interpolate(int32_t dim, int32_t method, const double *src, int64_t n,
                               const double *vals, const double *tgt, int64_t m, double *out,
                               int32_t *status, const pacman_b200_options *opts) {
  g_last_error.clear();
  if (src == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourcePoints is null but nSourcePoints > 0");
  if (tgt == nullptr && m > 0)
    return fail(PACMAN_B200_ERR_INVALID, "targetPoints is null but nTargetPoints > 0");
  if (vals == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourceValues is null but nSourcePoints > 0");
  if (dim < 1 || dim > 3)
    return fail(PACMAN_B200_ERR_DIMENSION, "The dimension of the points can only be: 1, 2 or 3.");
  if (method != PACMAN_B200_FE_NEAREST_NEAREST)
    return fail(PACMAN_B200_ERR_INVALID,
                "finite-element method " + std::to_string(method) +
                    " is not available in this engine (NEAREST_NEAREST = 0xF0 is)");
  if (n < 0 || m < 0) return fail(PACMAN_B200_ERR_INVALID, "negative point count");
  if (n > 0x7fffffffll || m > 0x7fffffffll)
    return fail(PACMAN_B200_ERR_LIMIT, "point counts are limited to 2^31 - 1");
  if (out == nullptr && m > 0) return fail(PACMAN_B200_ERR_INVALID, "target_values is null");
  pacman_b200_options o;
  pacman_b200_options_init(&o);
  if (opts) o = *opts;
  if (m == 0) return 0;
  cudaStream_t own = nullptr;
  try {
    DeviceScope ds(o.device);
    tune_pool(ds.dev);
    HostArena::get().reset();
    cudaStream_t st = static_cast<cudaStream_t>(o.stream);
    if (!st) {
      PB_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
      st = own;
    }
    {
      InBuf s, v, t;
      s.stage(src, size_t(n) * dim, ds.dev, st);
      v.stage(vals, size_t(n), ds.dev, st);
      t.stage(tgt, size_t(m) * dim, ds.dev, st);
      const bool out_dev = is_device_ptr(out, ds.dev);
      DevMem obuf;
      double *o_dev = out;
      if (!out_dev) {
        obuf.alloc(sizeof(double) * size_t(m), st);
        o_dev = obuf.as<double>();
      }
      fe_nearest(dim, s.ptr, n, v.ptr, t.ptr, m, o_dev, st);
      if (status) {  // TransferStatus::OUTSIDE everywhere
        if (is_device_ptr(status, ds.dev))
          PB_CUDA(cudaMemsetAsync(status, 0, sizeof(int32_t) * size_t(m), st));
        else
          std::memset(status, 0, sizeof(int32_t) * size_t(m));
      }
      if (!out_dev)
        PB_CUDA(cudaMemcpyAsync(out, o_dev, sizeof(double) * size_t(m), cudaMemcpyDeviceToHost,
                                st));
      PB_CUDA(host_sync(st));
    }
    if (own) {
      cudaStreamDestroy(own);
      own = nullptr;
    }
  } catch (const Error &e) {
    if (own) {
      cudaStreamSynchronize(own);
      cudaStreamDestroy(own);
    }
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_mls_interpolate(int32_t dim, const double *src, int64_t n, const double *vals,
                                const double *tgt, int64_t m, double *out,
                                const pacman_b200_options *opts) {
  g_last_error.clear();
  if (src == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourcePoints is null but nSourcePoints > 0");
  if (tgt == nullptr && m > 0)
    return fail(PACMAN_B200_ERR_INVALID, "targetPoints is null but nTargetPoints > 0");
  if (vals == nullptr && n > 0)
    return fail(PACMAN_B200_ERR_INVALID, "sourceValues is null but nSourcePoints > 0");
  if (dim < 1 || dim > 3)
    return fail(PACMAN_B200_ERR_DIMENSION, "The dimension of the points can only be: 1, 2 or 3.");
  if (n < 0 || m < 0) return fail(PACMAN_B200_ERR_INVALID, "negative point count");
  if (n > 0x7fffffffll || m > 0x7fffffffll)
    return fail(PACMAN_B200_ERR_LIMIT, "point counts are limited to 2^31 - 1");
  if (out == nullptr && m > 0) return fail(PACMAN_B200_ERR_INVALID, "target_values is null");
  pacman_b200_options o;
  pacman_b200_options_init(&o);
  if (opts) o = *opts;
  if (m == 0) return 0;
  cudaStream_t own = nullptr;
  try {
    DeviceScope ds(o.device);
    tune_pool(ds.dev);
    HostArena::get().reset();
    cudaStream_t st = static_cast<cudaStream_t>(o.stream);
    if (!st) {
      PB_CUDA(cudaStreamCreateWithFlags(&own, cudaStreamNonBlocking));
      st = own;
    }
    {
      InBuf s, v, t;
      s.stage(src, size_t(n) * dim, ds.dev, st);
      v.stage(vals, size_t(n), ds.dev, st);
      t.stage(tgt, size_t(m) * dim, ds.dev, st);
      const bool out_dev = is_device_ptr(out, ds.dev);
      DevMem obuf;
      double *o_dev = out;
      if (!out_dev) {
        obuf.alloc(sizeof(double) * size_t(m), st);
        o_dev = obuf.as<double>();
      }
      mls_interpolate(dim, s.ptr, n, v.ptr, t.ptr, m, o_dev, st);
      if (!out_dev)
        PB_CUDA(cudaMemcpyAsync(out, o_dev, sizeof(double) * size_t(m), cudaMemcpyDeviceToHost,
                                st));
      PB_CUDA(host_sync(st));
    }
    if (own) {
      cudaStreamDestroy(own);
      own = nullptr;
    }
  } catch (const Error &e) {
    if (own) {
      cudaStreamSynchronize(own);
      cudaStreamDestroy(own);
    }
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_plan_shard(pacman_b200_plan *plan, int32_t rank, int32_t world) {
  if (!plan) return fail(PACMAN_B200_ERR_INVALID, "plan is null");
  try {
    DeviceScope ds(plan->p.device);
    shard_plan(plan->p, rank, world);
  } catch (const Error &e) {
    return fail(e.code, e.msg);
  }
  return 0;
}

int pacman_b200_plan_owned_targets(const pacman_b200_plan *plan, int64_t *count, int32_t *owned) {
  if (!plan || !count) return fail(PACMAN_B200_ERR_INVALID, "null argument");
  const Plan &p = plan->p;
  const bool sharded = p.m_owned >= 0;
  *count = sharded ? p.m_owned : p.m;
  if (!owned || *count == 0) return 0;
  try {
    DeviceScope ds(p.device);
    if (sharded) {
      PB_CUDA(cudaMemcpyAsync(owned, p.tlist.p, sizeof(int32_t) * size_t(*count),
                              cudaMemcpyDefault, p.stream));
      PB_CUDA(host_sync(p.stream));
    } else {
      for (int64_t i = 0; i < *count; ++i) owned[i] = int32_t(i);
    }
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

int pacman_b200_rbf_interpolate_batch(const pacman_b200_problem *problems, int32_t count,
                                      const pacman_b200_options *opts,
                                      pacman_b200_stats *stats) {
  g_last_error.clear();
  return run_batch(problems, count, opts, stats);
}

}  // extern "C"
