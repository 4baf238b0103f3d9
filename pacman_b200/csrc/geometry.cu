// Geometry phase of the B200 RBF-PUM transfer: patch radius, centre cover,
// per-patch membership lists and the partition-of-unity gather.
//
// Replaces the ArborX BVH queries of the reference (src/rbf_pum/callbacks.hpp,
// clustering/clusters_radius.hpp, clustering/clustering.hpp, solver/solver.hpp
// :45-66 and :137-168) by uniform-grid searches over coalesced double4 points.
// Every predicate uses the exact arithmetic of common.cuh, so the radius, the
// centres and the sorted membership lists equal the CPU restatement's bit for
// bit.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>

#include "plan.hpp"

namespace pacman_b200 {
namespace {

constexpr int kThreads = 256;

inline int grid_for(int64_t n, int per_block = kThreads, int cap = 148 * 16) {
  int64_t b = (n + per_block - 1) / per_block;
  if (b < 1) b = 1;
  if (b > cap) b = cap;
  return int(b);
}

// ---------------------------------------------------------------------------
// Packing and bounding box
// ---------------------------------------------------------------------------

// Row-major [n x dim] doubles -> zero-padded double4; optional exact bbox via
// order-preserving 64-bit atomics (bb[0..2] min, bb[3..5] max).
__global__ void k_pack(const double *__restrict__ in, int dim, int64_t n, double4 *out,
                       unsigned long long *bb) {
  unsigned long long mn[3] = {~0ull, ~0ull, ~0ull}, mx[3] = {0ull, 0ull, 0ull};
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double c[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < dim; ++d) c[d] = in[i * dim + d];
    out[i] = make_double4(c[0], c[1], c[2], 0.0);
    if (bb) {
      for (int d = 0; d < 3; ++d) {
        const unsigned long long o = dbl_to_ordered(c[d]);
        mn[d] = o < mn[d] ? o : mn[d];
        mx[d] = o > mx[d] ? o : mx[d];
      }
    }
  }
  if (!bb) return;
  for (int d = 0; d < 3; ++d) {
    for (int s = 16; s > 0; s >>= 1) {
      const unsigned long long a = __shfl_xor_sync(0xffffffffu, mn[d], s);
      const unsigned long long b = __shfl_xor_sync(0xffffffffu, mx[d], s);
      mn[d] = a < mn[d] ? a : mn[d];
      mx[d] = b > mx[d] ? b : mx[d];
    }
  }
  if ((threadIdx.x & 31) == 0) {
    for (int d = 0; d < 3; ++d) {
      atomicMin(&bb[d], mn[d]);
      atomicMax(&bb[3 + d], mx[d]);
    }
  }
}

// ---------------------------------------------------------------------------
// FindRadius (src/rbf_pum/clustering/clusters_radius.hpp:22-125)
// ---------------------------------------------------------------------------

struct RadiusState {
  double samples[7][3];
  double proj[7][3];
  unsigned long long prefix[7];
  long long krem[7];
  double kth[7];
  double lo[3], hi[3];
  double radius;
  int nsamples;
  int dim;
};

__global__ void k_radius_samples(RadiusState *rs, const unsigned long long *bb, int dim,
                                 long long k) {
  if (threadIdx.x != 0 || blockIdx.x != 0) return;
  rs->dim = dim;
  rs->nsamples = 2 * dim + 1;
  double center[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    rs->lo[d] = d < dim ? ordered_to_dbl(bb[d]) : 0.0;
    rs->hi[d] = d < dim ? ordered_to_dbl(bb[3 + d]) : 0.0;
  }
  for (int d = 0; d < dim; ++d) center[d] = __ddiv_rn(__dadd_rn(rs->lo[d], rs->hi[d]), 2.0);
  for (int s = 0; s < 7; ++s)
    for (int d = 0; d < 3; ++d) rs->samples[s][d] = center[d];
  for (int a = 0; a < dim; ++a) {
    const double len = fabs(__dsub_rn(rs->hi[a], rs->lo[a]));
    double s_a = __dsub_rn(center[a], __dmul_rn(len, 0.25));
    rs->samples[a + 1][a] = s_a;
    s_a = __dadd_rn(s_a, __dmul_rn(len, 0.5));
    rs->samples[dim + a + 1][a] = s_a;
  }
  for (int s = 0; s < 7; ++s) {
    rs->prefix[s] = 0ull;
    rs->krem[s] = k;
  }
}

// Nearest source of each sample (lowest id on ties), in two exact passes with
// one sample per blockIdx.y: the minimum squared distance (its bit pattern is
// monotone for values >= 0), then the lowest id attaining it.
__device__ __forceinline__ unsigned long long warp_min_u64(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}

__global__ void k_nearest_dist(const double4 *__restrict__ pts, int64_t n, const RadiusState *rs,
                               unsigned long long *best_bits) {
  const int s = blockIdx.y;
  if (s >= rs->nsamples) return;
  const double sx = rs->samples[s][0], sy = rs->samples[s][1], sz = rs->samples[s][2];
  unsigned long long best = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = pts[i];
    const unsigned long long b =
        (unsigned long long)__double_as_longlong(sqdist3(sx, sy, sz, p.x, p.y, p.z));
    best = b < best ? b : best;
  }
  best = warp_min_u64(best);
  if ((threadIdx.x & 31) == 0) atomicMin(&best_bits[s], best);
}

__global__ void k_nearest_index(const double4 *__restrict__ pts, int64_t n, const RadiusState *rs,
                                const unsigned long long *best_bits, unsigned long long *best_id) {
  const int s = blockIdx.y;
  if (s >= rs->nsamples) return;
  const double sx = rs->samples[s][0], sy = rs->samples[s][1], sz = rs->samples[s][2];
  const unsigned long long target = best_bits[s];
  unsigned long long id = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = pts[i];
    const unsigned long long b =
        (unsigned long long)__double_as_longlong(sqdist3(sx, sy, sz, p.x, p.y, p.z));
    if (b == target && (unsigned long long)i < id) id = (unsigned long long)i;
  }
  id = warp_min_u64(id);
  if ((threadIdx.x & 31) == 0) atomicMin(&best_id[s], id);
}

__global__ void k_nearest_final(const unsigned long long *best_id, const double4 *pts,
                                RadiusState *rs) {
  const int s = threadIdx.x;
  if (s >= rs->nsamples) return;
  const double4 p = pts[best_id[s]];
  rs->proj[s][0] = p.x;
  rs->proj[s][1] = p.y;
  rs->proj[s][2] = p.z;
}

// One 8-bit radix-select pass over the squared distances (raw uint64 bits,
// monotone for values >= 0) from projected sample blockIdx.y to every source.
__global__ void k_knn_hist(const double4 *__restrict__ pts, int64_t n, const RadiusState *rs,
                           int pass, unsigned int *hist) {
  __shared__ unsigned int h[256];
  const int s = blockIdx.y;
  if (s >= rs->nsamples) return;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0u;
  __syncthreads();
  const int shift = 56 - 8 * pass;
  const unsigned long long hmask = pass == 0 ? 0ull : (~0ull << (64 - 8 * pass));
  const double sx = rs->proj[s][0], sy = rs->proj[s][1], sz = rs->proj[s][2];
  const unsigned long long pre = rs->prefix[s];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = pts[i];
    const unsigned long long key =
        (unsigned long long)__double_as_longlong(sqdist3(sx, sy, sz, p.x, p.y, p.z));
    if ((key & hmask) == pre) atomicAdd(&h[(key >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x) {
    const unsigned int v = h[i];
    if (v) atomicAdd(&hist[s * 256 + i], v);
  }
}

__global__ void k_knn_select(RadiusState *rs, unsigned int *hist, int pass) {
  const int s = threadIdx.x;
  if (s >= rs->nsamples) return;
  const int shift = 56 - 8 * pass;
  long long k = rs->krem[s];
  long long cum = 0;
  int d = 0;
  for (; d < 256; ++d) {
    const long long c = hist[s * 256 + d];
    if (cum + c >= k) break;
    cum += c;
  }
  if (d > 255) d = 255;
  rs->prefix[s] |= ((unsigned long long)d) << shift;
  rs->krem[s] = k - cum;
  for (int i = 0; i < 256; ++i) hist[s * 256 + i] = 0u;
  if (pass == 7) rs->kth[s] = __longlong_as_double((long long)rs->prefix[s]);
}

// Kokkos::sort of the per-sample maxima and the median pick
// (clusters_radius.hpp:121-124).
__global__ void k_radius_final(RadiusState *rs) {
  if (threadIdx.x != 0) return;
  double v[7];
  const int ns = rs->nsamples;
  for (int s = 0; s < ns; ++s) v[s] = rs->kth[s];
  for (int i = 1; i < ns; ++i) {
    const double x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
  rs->radius = __dsqrt_rn(v[rs->dim]);
}

// ---------------------------------------------------------------------------
// Uniform grids
// ---------------------------------------------------------------------------

struct GridSpec {
  double lo[3];
  double hi[3];  // inclusive upper bound of the grid domain
  double inv_h;
  int nc[3];
  int ncells;
};

GridSpec make_grid_spec(int dim, const double *bb_lo, const double *bb_hi, double radius,
                        int64_t npts) {
  GridSpec g{};
  const int64_t cap = std::max<int64_t>(std::min<int64_t>(npts * 2, int64_t(1) << 28), 1 << 12);
  double h = radius * (1.0 + 0x1p-20);
  for (int it = 0; it < 200; ++it) {
    int64_t tot = 1;
    bool ok = true;
    for (int d = 0; d < 3; ++d) {
      if (d >= dim) {
        g.nc[d] = 1;
        continue;
      }
      const double ext = (bb_hi[d] - bb_lo[d]) + 2.0 * h;
      const double c = std::floor(ext / h) + 1.0;
      if (!(c < 1.0e9)) {
        ok = false;
        break;
      }
      g.nc[d] = int(c);
      tot *= g.nc[d];
      if (tot > cap) {
        ok = false;
        break;
      }
    }
    if (ok) {
      g.ncells = int(tot);
      break;
    }
    h *= 1.25;
  }
  if (g.ncells == 0) throw Error{PACMAN_B200_ERR_LIMIT, "could not size the search grid"};
  for (int d = 0; d < 3; ++d) {
    g.lo[d] = d < dim ? bb_lo[d] - h : 0.0;
    g.hi[d] = d < dim ? bb_hi[d] + h : 0.0;
  }
  g.inv_h = 1.0 / h;
  return g;
}

__global__ void k_cell_keys(const double4 *__restrict__ pts, int64_t n, GridSpec g, int *keys,
                            int *ids) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const double4 p = pts[i];
    const double c[3] = {p.x, p.y, p.z};
    bool inside = true;
    for (int d = 0; d < 3; ++d)
      if (!(c[d] >= g.lo[d] && c[d] <= g.hi[d])) inside = false;
    int key = g.ncells;
    if (inside) {
      const int a = cell_coord(c[0], g.lo[0], g.inv_h, g.nc[0]);
      const int b = cell_coord(c[1], g.lo[1], g.inv_h, g.nc[1]);
      const int e = cell_coord(c[2], g.lo[2], g.inv_h, g.nc[2]);
      key = (a * g.nc[1] + b) * g.nc[2] + e;
    }
    keys[i] = key;
    ids[i] = int(i);
  }
}

// start[c] = first sorted position whose key >= c, for c in [0, ncells].
__global__ void k_cell_start(const int *skeys, int64_t n, int ncells, int *start) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= n;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int prev = (i == 0) ? -1 : skeys[i - 1];
    const int cur = (i == n) ? ncells + 1 : skeys[i];
    for (int c = prev + 1; c <= cur && c <= ncells; ++c) start[c] = int(i);
  }
}

void build_grid(DevGrid &out, const double4 *pts, int64_t n, int dim, const double *bb_lo,
                const double *bb_hi, double radius, cudaStream_t st) {
  const GridSpec g = make_grid_spec(dim, bb_lo, bb_hi, radius, n);
  DevMem keys, ids, skeys, tmp;
  const int64_t nn = std::max<int64_t>(n, 1);
  keys.alloc(sizeof(int) * nn, st);
  ids.alloc(sizeof(int) * nn, st);
  skeys.alloc(sizeof(int) * nn, st);
  out.items.alloc(sizeof(int) * nn, st);
  out.start.alloc(sizeof(int) * (size_t(g.ncells) + 2), st);
  if (n > 0) {
    k_cell_keys<<<grid_for(n), kThreads, 0, st>>>(pts, n, g, keys.as<int>(), ids.as<int>());
    note_launch();
    int end_bit = 1;
    while ((int64_t(1) << end_bit) <= g.ncells) ++end_bit;
    size_t tb = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<int>(), skeys.as<int>(),
                                            ids.as<int>(), out.items.as<int>(), int(n), 0,
                                            end_bit, st));
    tmp.alloc(tb, st);
    PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<int>(), skeys.as<int>(),
                                            ids.as<int>(), out.items.as<int>(), int(n), 0,
                                            end_bit, st));
    k_cell_start<<<grid_for(n + 1), kThreads, 0, st>>>(skeys.as<int>(), n, g.ncells,
                                                       out.start.as<int>());
    note_launch();
  } else {
    PB_CUDA(cudaMemsetAsync(out.start.p, 0, sizeof(int) * (size_t(g.ncells) + 1), st));
  }
  PB_CUDA(cudaGetLastError());
  GridView &v = out.view;
  for (int d = 0; d < 3; ++d) {
    v.lo[d] = g.lo[d];
    v.nc[d] = g.nc[d];
  }
  v.inv_h = g.inv_h;
  v.ncells = g.ncells;
  v.start = out.start.as<int>();
  v.items = out.items.as<int>();
}

// ---------------------------------------------------------------------------
// Centre cover (src/rbf_pum/clustering/clustering.hpp:127-271)
// ---------------------------------------------------------------------------

struct CandSpec {
  int dim;
  int shape[3];
  double dist[3];
  double lo[3];
  double r2;
  long long nb;
};

enum : unsigned char { kDead = 0, kAlive0 = 1, kSurvive = 2, kPending = 3 };

// Calls fn(point_id) for the points in the 3^3 cells around q that fall to
// this lane: the warp's 32 lanes split every cell's points between them.
template <typename Fn>
__device__ __forceinline__ void for_neighbors_lanes(const GridView &g, double qx, double qy,
                                                    double qz, int lane, Fn &&fn) {
  const int cx = cell_coord(qx, g.lo[0], g.inv_h, g.nc[0]);
  const int cy = cell_coord(qy, g.lo[1], g.inv_h, g.nc[1]);
  const int cz = cell_coord(qz, g.lo[2], g.inv_h, g.nc[2]);
  const int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.nc[0] - 1);
  const int y0 = max(cy - 1, 0), y1 = min(cy + 1, g.nc[1] - 1);
  const int z0 = max(cz - 1, 0), z1 = min(cz + 1, g.nc[2] - 1);
  for (int a = x0; a <= x1; ++a)
    for (int b = y0; b <= y1; ++b) {
      const int base = (a * g.nc[1] + b) * g.nc[2];
      const int s = g.start[base + z0];
      const int e = g.start[base + z1 + 1];
      for (int i = s + lane; i < e; i += 32) fn(g.items[i]);
    }
}

// Steps 5-8: candidate coordinates (row-major storage, last axis fastest),
// source and target emptiness tags (nearest within r, i.e. squared distance
// <= r*r), snap to the nearest source (lowest id on ties).
// One warp per candidate centre (dense blobs put thousands of sources in a
// candidate's 3^3 cells, too many for one thread): the lanes split the
// neighbourhood, the nearest source is the lexicographic minimum of (squared
// distance, index) over the warp, so the result does not depend on the split.
__global__ void k_candidates(CandSpec cs, GridView sg, const double4 *__restrict__ src,
                             GridView tg, const double4 *__restrict__ tgt, int has_targets,
                             double4 *cpos, unsigned char *state) {
  const int lane = threadIdx.x & 31;
  const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
  for (long long s = blockIdx.x * (long long)(blockDim.x >> 5) + (threadIdx.x >> 5); s < cs.nb;
       s += nw) {
    long long t = s;
    int coords[3] = {0, 0, 0};
    for (int a = cs.dim - 1; a >= 0; --a) {
      coords[a] = int(t % cs.shape[a]);
      t /= cs.shape[a];
    }
    double q[3] = {0.0, 0.0, 0.0};
    for (int a = 0; a < cs.dim; ++a) q[a] = __fma_rn(cs.dist[a], double(coords[a]), cs.lo[a]);
    double best = INFINITY;
    int bi = 0x7fffffff;
    for_neighbors_lanes(sg, q[0], q[1], q[2], lane, [&](int i) {
      const double4 p = src[i];
      const double d2 = sqdist3(q[0], q[1], q[2], p.x, p.y, p.z);
      if (d2 < best || (d2 == best && i < bi)) {
        best = d2;
        bi = i;
      }
    });
    for (int o = 16; o > 0; o >>= 1) {
      const double ob = __shfl_xor_sync(0xffffffffu, best, o);
      const int oi = __shfl_xor_sync(0xffffffffu, bi, o);
      if (ob < best || (ob == best && oi < bi)) {
        best = ob;
        bi = oi;
      }
    }
    bool alive = (bi != 0x7fffffff) && (best <= cs.r2);
    if (alive && has_targets) {
      bool any = false;
      for_neighbors_lanes(tg, q[0], q[1], q[2], lane, [&](int i) {
        if (!any) {
          const double4 p = tgt[i];
          any = sqdist3(q[0], q[1], q[2], p.x, p.y, p.z) <= cs.r2;
        }
      });
      alive = __any_sync(0xffffffffu, any);
    }
    if (lane == 0) {
      state[s] = alive ? kAlive0 : kDead;
      cpos[s] = alive ? src[bi] : make_double4(q[0], q[1], q[2], 0.0);
    }
  }
}

// Step 9 (order-dependent pruning, clustering.hpp:228-254), parallel form.
// Centre i dies if a later neighbour j > i (in the 26-offset table) is alive
// before the loop and closer than the threshold, or if an earlier neighbour
// j < i that survived its own turn is that close.  The first case is decided
// here; the second is recorded as a bit mask and resolved by k_prune_resolve.
__global__ void k_prune_mark(long long nb, int noff, const long long *__restrict__ offs,
                             double thr, const double4 *__restrict__ cpos,
                             const unsigned char *__restrict__ state0, unsigned char *state1,
                             unsigned int *mask) {
  for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < nb;
       i += (long long)gridDim.x * blockDim.x) {
    unsigned int m = 0u;
    unsigned char st = kDead;
    if (state0[i] == kAlive0) {
      const double4 c = cpos[i];
      bool fwd = false;
      for (int o = 0; o < noff; ++o) {
        const long long j = i + offs[o];
        if (j < 0 || j >= nb || state0[j] != kAlive0) continue;
        const double4 q = cpos[j];
        if (sqdist3(c.x, c.y, c.z, q.x, q.y, q.z) < thr) {
          if (j > i) fwd = true;
          else m |= 1u << o;
        }
      }
      st = fwd ? kDead : (m ? kPending : kSurvive);
    }
    state1[i] = st;
    mask[i] = m;
  }
}

// Resolves the pending centres in ascending-id order semantics: a pending
// centre dies iff one of its masked earlier neighbours survived.  Each sweep
// settles at least the smallest pending id, so nb + 1 sweeps always suffice.
__global__ void k_prune_resolve(long long nb, int noff, const long long *__restrict__ offs,
                                const unsigned int *__restrict__ mask, unsigned char *state1_,
                                int *status) {
  volatile unsigned char *state1 = state1_;
  for (long long sweep = 0; sweep <= nb; ++sweep) {
    int pending = 0;
    for (long long i = threadIdx.x; i < nb; i += blockDim.x) {
      if (state1[i] != kPending) continue;
      const unsigned int m = mask[i];
      bool any_alive = false, undecided = false;
      for (int o = 0; o < noff; ++o) {
        if (!(m & (1u << o))) continue;
        const unsigned char sj = state1[i + offs[o]];
        if (sj == kSurvive) any_alive = true;
        else if (sj == kPending) undecided = true;
      }
      if (any_alive) state1[i] = kDead;
      else if (!undecided) state1[i] = kSurvive;
      else pending = 1;
    }
    if (!__syncthreads_or(pending)) return;
  }
  if (threadIdx.x == 0) *status = 1;
}

// Step 10: re-tag surviving centres without a target within r.
__global__ void k_retag(long long nb, const double4 *__restrict__ cpos, unsigned char *state1,
                        GridView tg, const double4 *__restrict__ tgt, double r2,
                        unsigned char *flags) {
  for (long long s = blockIdx.x * (long long)blockDim.x + threadIdx.x; s < nb;
       s += (long long)gridDim.x * blockDim.x) {
    bool keep = state1[s] == kSurvive;
    if (keep && tgt) {
      const double4 c = cpos[s];
      bool any = false;
      for_neighbors(tg, c.x, c.y, c.z, [&](int i) {
        if (!any) {
          const double4 p = tgt[i];
          any = sqdist3(c.x, c.y, c.z, p.x, p.y, p.z) <= r2;
        }
      });
      keep = any;
    }
    flags[s] = keep ? 1 : 0;
  }
}

// ---------------------------------------------------------------------------
// Patch membership lists (solver.hpp:45-66): sqrt(d2) <= radius (ArborX
// sphere-point intersection), warp per patch.
// ---------------------------------------------------------------------------

template <bool kFill>
__global__ void k_members(int K, const double4 *__restrict__ centers, GridView g,
                          const double4 *__restrict__ pts, double radius, int *cnt,
                          const int64_t *__restrict__ off, int *idx) {
  const int lane = threadIdx.x & 31;
  const int warps = (blockDim.x >> 5) * gridDim.x;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
    const double4 c = centers[k];
    const int cx = cell_coord(c.x, g.lo[0], g.inv_h, g.nc[0]);
    const int cy = cell_coord(c.y, g.lo[1], g.inv_h, g.nc[1]);
    const int cz = cell_coord(c.z, g.lo[2], g.inv_h, g.nc[2]);
    const int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.nc[0] - 1);
    const int y0 = max(cy - 1, 0), y1 = min(cy + 1, g.nc[1] - 1);
    const int z0 = max(cz - 1, 0), z1 = min(cz + 1, g.nc[2] - 1);
    int64_t pos = kFill ? off[k] : 0;
    int total = 0;
    for (int a = x0; a <= x1; ++a)
      for (int b = y0; b <= y1; ++b) {
        const int base = (a * g.nc[1] + b) * g.nc[2];
        const int s = g.start[base + z0];
        const int e = g.start[base + z1 + 1];
        for (int i0 = s; i0 < e; i0 += 32) {
          const int i = i0 + lane;
          bool in = false;
          int id = 0;
          if (i < e) {
            id = g.items[i];
            const double4 p = pts[id];
            in = __dsqrt_rn(sqdist3(c.x, c.y, c.z, p.x, p.y, p.z)) <= radius;
          }
          const unsigned int bal = __ballot_sync(0xffffffffu, in);
          if (kFill && in) idx[pos + __popc(bal & ((1u << lane) - 1u))] = id;
          pos += __popc(bal);
          total += __popc(bal);
        }
      }
    if (!kFill && lane == 0) cnt[k] = total;
  }
}

__global__ void k_widen(const int *in, int64_t *out, int K) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < K) out[i] = in[i];
  if (i == K) out[K] = 0;
}

void build_lists(Plan &p, const GridView &g, const double4 *pts, double radius, DevMem &off,
                 DevMem &idx, int64_t &nnz, std::vector<int> &sizes) {
  cudaStream_t st = p.stream;
  const int K = p.K;
  DevMem cnt, cnt64, tmp, unsorted;
  cnt.alloc(sizeof(int) * (K + 1), st);
  cnt64.alloc(sizeof(int64_t) * (K + 1), st);
  off.alloc(sizeof(int64_t) * (K + 1), st);
  const int blocks = std::max(1, std::min((K + 7) / 8, 148 * 32));
  k_members<false><<<blocks, kThreads, 0, st>>>(K, p.centers.as<double4>(), g, pts, radius,
                                                cnt.as<int>(), nullptr, nullptr);
  note_launch();
  k_widen<<<(K + 1 + 255) / 256, 256, 0, st>>>(cnt.as<int>(), cnt64.as<int64_t>(), K);
  note_launch();
  size_t tb = 0;
  PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt64.as<int64_t>(), off.as<int64_t>(),
                                        K + 1, st));
  tmp.alloc(tb, st);
  PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp.p, tb, cnt64.as<int64_t>(), off.as<int64_t>(),
                                        K + 1, st));
  sizes.resize(K);
  PB_CUDA(cudaMemcpyAsync(&nnz, off.as<int64_t>() + K, sizeof(int64_t), cudaMemcpyDeviceToHost,
                          st));
  if (K > 0)
    PB_CUDA(cudaMemcpyAsync(sizes.data(), cnt.p, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  if (nnz > (int64_t(1) << 31) - 1)
    throw Error{PACMAN_B200_ERR_LIMIT, "more than 2^31 patch memberships"};
  unsorted.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  idx.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  k_members<true><<<blocks, kThreads, 0, st>>>(K, p.centers.as<double4>(), g, pts, radius,
                                               nullptr, off.as<int64_t>(), unsorted.as<int>());
  note_launch();
  if (nnz > 0) {
    size_t tb2 = 0;
    PB_CUDA(cub::DeviceSegmentedSort::SortKeys(nullptr, tb2, unsorted.as<int>(), idx.as<int>(),
                                               nnz, K, off.as<int64_t>(),
                                               off.as<int64_t>() + 1, st));
    DevMem tmp2;
    tmp2.alloc(tb2, st);
    PB_CUDA(cub::DeviceSegmentedSort::SortKeys(tmp2.p, tb2, unsorted.as<int>(), idx.as<int>(),
                                               nnz, K, off.as<int64_t>(),
                                               off.as<int64_t>() + 1, st));
    // tmp2 and unsorted are released stream-ordered: no wait needed.
  }
  PB_CUDA(cudaGetLastError());
}

// ---------------------------------------------------------------------------
// Partition-of-unity gather (solver.hpp:137-168 and :275-285): for each
// target, the centres within r in ascending order, Shepard-normalised
// Wendland C2 weights, and the weighted sum of the local values of the
// patches whose target list holds it (binary search in that sorted list).
// Deterministic and equal to the reference's serial patch-order accumulation.
// ---------------------------------------------------------------------------

constexpr int kMaxPatchesPerTarget = 64;

__device__ __forceinline__ int64_t find_sorted(const int *a, int64_t n, int v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && a[lo] == v) ? lo : -1;
}

__global__ void k_pu_gather(int64_t M, const int *__restrict__ tlist,
                            const double4 *__restrict__ tgt, GridView cg,
                            const double4 *__restrict__ centers, double r, double rinv,
                            const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                            const double *__restrict__ local, int F, double *out) {
  // M targets: all (tlist null) or those of a shard's list.
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < M;
       it += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = tlist ? tlist[it] : it;
    const double4 y = tgt[t];
    int ids[kMaxPatchesPerTarget];
    double ws[kMaxPatchesPerTarget];
    int cnt = 0;
    bool overflow = false;
    for_neighbors(cg, y.x, y.y, y.z, [&](int k) {
      const double4 c = centers[k];
      const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, c.x, c.y, c.z));
      if (d <= r) {
        if (cnt < kMaxPatchesPerTarget) {
          int j = cnt - 1;
          const double w = wendland<double>(kWendlandC2, d, rinv);
          while (j >= 0 && ids[j] > k) {
            ids[j + 1] = ids[j];
            ws[j + 1] = ws[j];
            --j;
          }
          ids[j + 1] = k;
          ws[j + 1] = w;
          ++cnt;
        } else {
          overflow = true;
        }
      }
    });
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    if (!overflow) {
      double sum = 0.0;
      for (int i = 0; i < cnt; ++i) sum = __dadd_rn(sum, ws[i]);
      for (int i = 0; i < cnt; ++i) {
        const int k = ids[i];
        const int64_t b = toff[k];
        const int64_t pos = find_sorted(tidx + b, toff[k + 1] - b, int(t));
        if (pos < 0) continue;
        const double wn = __ddiv_rn(ws[i], sum);
        for (int f = 0; f < F; ++f)
          acc[f] = __dadd_rn(acc[f], __dmul_rn(wn, local[(b + pos) * F + f]));
      }
    } else {
      // More than kMaxPatchesPerTarget centres: walk them in ascending order
      // by repeated selection (same arithmetic, fewer registers).
      double sum = 0.0;
      int last = -1;
      for (;;) {
        int nk = 0x7fffffff;
        double nd = 0.0;
        for_neighbors(cg, y.x, y.y, y.z, [&](int k) {
          if (k > last && k < nk) {
            const double4 c = centers[k];
            const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, c.x, c.y, c.z));
            if (d <= r) {
              nk = k;
              nd = d;
            }
          }
        });
        if (nk == 0x7fffffff) break;
        sum = __dadd_rn(sum, wendland<double>(kWendlandC2, nd, rinv));
        last = nk;
      }
      last = -1;
      for (;;) {
        int nk = 0x7fffffff;
        double nd = 0.0;
        for_neighbors(cg, y.x, y.y, y.z, [&](int k) {
          if (k > last && k < nk) {
            const double4 c = centers[k];
            const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, c.x, c.y, c.z));
            if (d <= r) {
              nk = k;
              nd = d;
            }
          }
        });
        if (nk == 0x7fffffff) break;
        last = nk;
        const int64_t b = toff[nk];
        const int64_t pos = find_sorted(tidx + b, toff[nk + 1] - b, int(t));
        if (pos < 0) continue;
        const double wn = __ddiv_rn(wendland<double>(kWendlandC2, nd, rinv), sum);
        for (int f = 0; f < F; ++f)
          acc[f] = __dadd_rn(acc[f], __dmul_rn(wn, local[(b + pos) * F + f]));
      }
    }
    for (int f = 0; f < F; ++f) out[t * F + f] = acc[f];
  }
}

int neighbor_offsets(int dim, const int *shape, long long *off) {
  // ZCurveNeighborOffsets, clustering.hpp:34-116 (3D table :96-102).
  if (dim == 1) {
    off[0] = -1;
    off[1] = 1;
    return 2;
  }
  if (dim == 2) {
    static const int o2[8][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1},
                                 {0, 1},   {1, -1}, {1, 0},  {1, 1}};
    for (int i = 0; i < 8; ++i) off[i] = o2[i][1] + (long long)o2[i][0] * shape[1];
    return 8;
  }
  static const int o3[26][3] = {{-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, 0},  {-1, 0, 1},
                                {-1, 0, -1},  {-1, 1, 0},  {-1, 1, 1},  {-1, 1, -1}, {0, -1, -1},
                                {0, -1, 0},   {0, -1, 1},  {0, 0, 1},   {0, 0, -1},  {0, 1, 0},
                                {0, 1, 1},    {0, 1, -1},  {1, -1, -1}, {1, -1, 0},  {1, -1, 1},
                                {1, 0, 0},    {1, 0, 1},   {1, 0, -1},  {1, 1, 0},   {1, 1, 1},
                                {1, 1, -1}};
  for (int i = 0; i < 26; ++i)
    off[i] = o3[i][2] + (long long)o3[i][1] * shape[2] + (long long)o3[i][0] * shape[2] * shape[1];
  return 26;
}

}  // namespace

// Full geometry phase on p.stream.  src_dev / tgt_dev are row-major device
// arrays of the caller's points.
void build_geometry(Plan &p, const double *src_dev, const double *tgt_dev) {
  cudaStream_t st = p.stream;
  const int dim = p.dim;
  const int64_t n = p.n, m = p.m;
  cudaEvent_t e0, e1;
  PB_CUDA(cudaEventCreate(&e0));
  PB_CUDA(cudaEventCreate(&e1));
  PB_CUDA(cudaEventRecord(e0, st));

  p.src4.alloc(sizeof(double4) * std::max<int64_t>(n, 1), st);
  p.tgt4.alloc(sizeof(double4) * std::max<int64_t>(m, 1), st);
  DevMem bb, rsm, pd, pi, hist;
  bb.alloc(sizeof(unsigned long long) * 6, st);
  unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
  PB_CUDA(cudaMemcpyAsync(bb.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_pack<<<grid_for(n), kThreads, 0, st>>>(src_dev, dim, n, p.src4.as<double4>(),
                                           bb.as<unsigned long long>());
  note_launch();
  if (m > 0) {
    k_pack<<<grid_for(m), kThreads, 0, st>>>(tgt_dev, dim, m, p.tgt4.as<double4>(), nullptr);
    note_launch();
  }

  // Patch radius.
  rsm.alloc(sizeof(RadiusState), st);
  const long long kk = std::min<long long>(p.opts.nodes_per_cluster, n);
  k_radius_samples<<<1, 1, 0, st>>>(rsm.as<RadiusState>(), bb.as<unsigned long long>(), dim, kk);
  note_launch();
  const int nb_near = grid_for(n, kThreads, 148 * 4);
  pd.alloc(sizeof(unsigned long long) * 7, st);
  pi.alloc(sizeof(unsigned long long) * 7, st);
  PB_CUDA(cudaMemsetAsync(pd.p, 0xff, sizeof(unsigned long long) * 7, st));
  PB_CUDA(cudaMemsetAsync(pi.p, 0xff, sizeof(unsigned long long) * 7, st));
  k_nearest_dist<<<dim3(nb_near, 2 * dim + 1), kThreads, 0, st>>>(
      p.src4.as<double4>(), n, rsm.as<RadiusState>(), pd.as<unsigned long long>());
  note_launch();
  k_nearest_index<<<dim3(nb_near, 2 * dim + 1), kThreads, 0, st>>>(
      p.src4.as<double4>(), n, rsm.as<RadiusState>(), pd.as<unsigned long long>(),
      pi.as<unsigned long long>());
  note_launch();
  k_nearest_final<<<1, 32, 0, st>>>(pi.as<unsigned long long>(), p.src4.as<double4>(),
                                    rsm.as<RadiusState>());
  note_launch();
  hist.alloc(sizeof(unsigned int) * 7 * 256, st);
  PB_CUDA(cudaMemsetAsync(hist.p, 0, sizeof(unsigned int) * 7 * 256, st));
  const int nb_hist = grid_for(n, kThreads, 148 * 4);
  for (int pass = 0; pass < 8; ++pass) {
    k_knn_hist<<<dim3(nb_hist, 2 * dim + 1), kThreads, 0, st>>>(p.src4.as<double4>(), n, rsm.as<RadiusState>(),
                                             pass, hist.as<unsigned int>());
    note_launch();
    k_knn_select<<<1, 32, 0, st>>>(rsm.as<RadiusState>(), hist.as<unsigned int>(), pass);
    note_launch();
  }
  k_radius_final<<<1, 32, 0, st>>>(rsm.as<RadiusState>());
  note_launch();
  PB_CUDA(cudaGetLastError());
  RadiusState rs;
  PB_CUDA(cudaMemcpyAsync(&rs, rsm.p, sizeof(rs), cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  for (int d = 0; d < 3; ++d) {
    p.lo[d] = rs.lo[d];
    p.hi[d] = rs.hi[d];
  }
  p.radius = rs.radius;
  if (std::getenv("PACMAN_B200_DEBUG")) {
    std::fprintf(stderr, "[pacman_b200] bbox lo %.17g %.17g %.17g hi %.17g %.17g %.17g\n",
                 rs.lo[0], rs.lo[1], rs.lo[2], rs.hi[0], rs.hi[1], rs.hi[2]);
    for (int s = 0; s < rs.nsamples; ++s)
      std::fprintf(stderr, "[pacman_b200] sample %d (%.17g %.17g %.17g) proj (%.17g %.17g %.17g) kth %.17g\n",
                   s, rs.samples[s][0], rs.samples[s][1], rs.samples[s][2], rs.proj[s][0],
                   rs.proj[s][1], rs.proj[s][2], rs.kth[s]);
    std::fprintf(stderr, "[pacman_b200] radius %.17g\n", rs.radius);
  }
  if (!(p.radius > 0.0) || !std::isfinite(p.radius))
    throw Error{PACMAN_B200_ERR_DEGENERATE, "degenerate patch radius (zero or non-finite)"};
  const double r = p.radius;
  const double r2 = r * r;

  // Candidate grid (clustering.hpp:142-203), host arithmetic as the reference.
  CandSpec cs{};
  cs.dim = dim;
  const double spacing = std::sqrt(4.0 / dim) * r * (1.0 - p.opts.relative_overlap);
  double min_d = 1.7976931348623157e308;
  long long nb = 1;
  for (int a = 0; a < 3; ++a) {
    cs.shape[a] = 1;
    cs.dist[a] = 0.0;
    cs.lo[a] = 0.0;
  }
  for (int a = 0; a < dim; ++a) {
    double edge = p.hi[a] - p.lo[a];
    edge = (edge < 0) ? -edge : edge;
    const double q = std::max(1.0, edge / spacing);
    if (!(q < 2.0e9)) throw Error{PACMAN_B200_ERR_LIMIT, "candidate centre grid too large"};
    cs.shape[a] = int(std::ceil(q));
    cs.dist[a] = edge / double(cs.shape[a]);
    if (cs.dist[a] < min_d) min_d = cs.dist[a];
    cs.shape[a] += 1;
    nb *= cs.shape[a];
    if (nb > 0x7fffffffll) throw Error{PACMAN_B200_ERR_LIMIT, "candidate centre grid exceeds int32"};
    cs.lo[a] = p.lo[a];
  }
  cs.r2 = r2;
  cs.nb = nb;
  p.ncand = nb;
  double thr = 0.4 * min_d;
  thr *= thr;

  DevGrid sgrid, tgrid;
  build_grid(sgrid, p.src4.as<double4>(), n, dim, p.lo, p.hi, r, st);
  build_grid(tgrid, p.tgt4.as<double4>(), m, dim, p.lo, p.hi, r, st);

  DevMem cpos, s0, s1, mask, offs, status, flags, tmp, nsel;
  cpos.alloc(sizeof(double4) * nb, st);
  s0.alloc(nb, st);
  s1.alloc(nb, st);
  flags.alloc(nb, st);
  mask.alloc(sizeof(unsigned int) * nb, st);
  offs.alloc(sizeof(long long) * 26, st);
  status.alloc(sizeof(int), st);
  PB_CUDA(cudaMemsetAsync(status.p, 0, sizeof(int), st));
  long long off_h[26];
  const int noff = neighbor_offsets(dim, cs.shape, off_h);
  PB_CUDA(cudaMemcpyAsync(offs.p, off_h, sizeof(long long) * noff, cudaMemcpyHostToDevice, st));
  k_candidates<<<grid_for(nb * 32), kThreads, 0, st>>>(cs, sgrid.view, p.src4.as<double4>(),
                                                  tgrid.view, p.tgt4.as<double4>(), m > 0 ? 1 : 0,
                                                  cpos.as<double4>(), s0.as<unsigned char>());
  note_launch();
  k_prune_mark<<<grid_for(nb), kThreads, 0, st>>>(nb, noff, offs.as<long long>(), thr,
                                                  cpos.as<double4>(), s0.as<unsigned char>(),
                                                  s1.as<unsigned char>(), mask.as<unsigned int>());
  note_launch();
  k_prune_resolve<<<1, 1024, 0, st>>>(nb, noff, offs.as<long long>(), mask.as<unsigned int>(),
                                      s1.as<unsigned char>(), status.as<int>());
  note_launch();
  k_retag<<<grid_for(nb), kThreads, 0, st>>>(nb, cpos.as<double4>(), s1.as<unsigned char>(),
                                             tgrid.view, m > 0 ? p.tgt4.as<double4>() : nullptr,
                                             r2, flags.as<unsigned char>());
  note_launch();
  // Step 11: stable compaction.
  p.centers.alloc(sizeof(double4) * nb, st);
  nsel.alloc(sizeof(int), st);
  size_t tb = 0;
  PB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, cpos.as<double4>(), flags.as<unsigned char>(),
                                     p.centers.as<double4>(), nsel.as<int>(), int(nb), st));
  tmp.alloc(tb, st);
  PB_CUDA(cub::DeviceSelect::Flagged(tmp.p, tb, cpos.as<double4>(), flags.as<unsigned char>(),
                                     p.centers.as<double4>(), nsel.as<int>(), int(nb), st));
  int K = 0, stat = 0;
  PB_CUDA(cudaMemcpyAsync(&K, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PB_CUDA(cudaMemcpyAsync(&stat, status.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  if (stat) throw Error{PACMAN_B200_ERR_LIMIT, "centre pruning did not settle"};
  p.K = K;

  // Membership lists: sources within r, targets within r - 1e-14
  // (solver.hpp:264-270).
  build_lists(p, sgrid.view, p.src4.as<double4>(), r, p.soff, p.sidx, p.snnz, p.n_host);
  build_lists(p, tgrid.view, p.tgt4.as<double4>(), r - kEps, p.toff, p.tidx, p.tnnz, p.m_host);

  // Grid of centres for the partition-of-unity weights.
  build_grid(p.cgrid, p.centers.as<double4>(), K, dim, p.lo, p.hi, r, st);
  PB_CUDA(cudaEventRecord(e1, st));
  // No wait here: the time is read after the execute's own final wait.
  p.geom_ev[0] = e0;
  p.geom_ev[1] = e1;
}

double geometry_ms(Plan &p) {
  if (p.geom_ev[0] && p.geom_ev[1] && cudaEventQuery(p.geom_ev[1]) == cudaSuccess) {
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, p.geom_ev[0], p.geom_ev[1]) == cudaSuccess) p.ms_geometry = ms;
    cudaEventDestroy(p.geom_ev[0]);
    cudaEventDestroy(p.geom_ev[1]);
    p.geom_ev[0] = p.geom_ev[1] = nullptr;
  }
  cudaGetLastError();
  return p.ms_geometry < 0.0 ? 0.0 : p.ms_geometry;
}

// Packed double4 copy of row-major points and their exact bounding box.
void pack_points(const double *in_dev, int dim, int64_t n, DevMem &out4, double lo[3],
                 double hi[3], cudaStream_t st) {
  out4.alloc(sizeof(double4) * std::max<int64_t>(n, 1), st);
  for (int d = 0; d < 3; ++d) lo[d] = hi[d] = 0.0;
  if (n == 0) return;
  DevMem bb;
  bb.alloc(sizeof(unsigned long long) * 6, st);
  unsigned long long init[6] = {~0ull, ~0ull, ~0ull, 0ull, 0ull, 0ull};
  PB_CUDA(cudaMemcpyAsync(bb.p, init, sizeof(init), cudaMemcpyHostToDevice, st));
  k_pack<<<grid_for(n), kThreads, 0, st>>>(in_dev, dim, n, out4.as<double4>(),
                                           bb.as<unsigned long long>());
  note_launch();
  unsigned long long h[6];
  PB_CUDA(cudaMemcpyAsync(h, bb.p, sizeof(h), cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  auto to_dbl = [](unsigned long long b) {
    b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
    double d;
    std::memcpy(&d, &b, sizeof(d));
    return d;
  };
  for (int d = 0; d < dim; ++d) {
    lo[d] = to_dbl(h[d]);
    hi[d] = to_dbl(h[3 + d]);
  }
}

void build_point_grid(DevGrid &out, const double4 *pts, int64_t n, int dim, const double *lo,
                      const double *hi, double cell, cudaStream_t st) {
  build_grid(out, pts, n, dim, lo, hi, cell, st);
}

void pu_gather(Plan &p, const double *local, int F, double *out_dev) {
  if (p.m == 0) return;
  const bool sharded = p.m_owned >= 0;
  if (p.K == 0 || sharded)  // a shard writes its own targets only: zeros elsewhere
    PB_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double) * p.m * F, p.stream));
  if (p.K == 0) return;
  const int64_t M = sharded ? p.m_owned : p.m;
  if (M == 0) return;
  const double r = p.radius;
  k_pu_gather<<<grid_for(M, 128, 148 * 64), 128, 0, p.stream>>>(
      M, sharded ? p.tlist.as<int>() : nullptr, p.tgt4.as<double4>(), p.cgrid.view,
      p.centers.as<double4>(), r, 1.0 / r, p.toff.as<int64_t>(), p.tidx.as<int>(), local, F,
      out_dev);
  note_launch();
  PB_CUDA(cudaGetLastError());
}

}  // namespace pacman_b200
