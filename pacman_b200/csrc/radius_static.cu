// Patch radius without any device allocation.
//
// Some callers of this library cannot allocate device memory: a coupled
// simulation code that reserves the whole GPU for its own pool allocator at
// start-up and hands out every buffer itself, so that an allocation made
// behind its back fails or breaks its accounting, or a solver running under
// a fixed device-memory budget in which a library may not grow its
// footprint.  This file gives them pacman_b200_patch_radius_noalloc: the same radius
// heuristic as the full transfer (sample points, nearest source, k-th
// nearest neighbour, median), computed with kernels whose working memory is
// one fixed file-scope __device__ array instead of cudaMallocAsync buffers.
//
// The array is small (kScratchBytes) and lives on every GPU that loads the
// library until the process exits.  Every call shares it and overwrites it:
// two calls that overlap on the GPU (different streams, or different host
// threads on the same device) race on it and must be serialised by the
// caller.  What has to start at zero or at an extreme is reset by each call.
#include <cstdint>
#include <cstring>
#include <cmath>
#include <string>

#include "../../include/pacman_b200.h"
#include "common.cuh"

namespace pacman_b200 {
// Message returned by pacman_b200_last_error() on this thread (api.cu).
void set_last_error(const std::string &msg);
}  // namespace pacman_b200

namespace pacman_b200 {
namespace {

// Scratch layout (bytes): bounding box 6 x u64, 7 samples x 3 coordinates,
// 7 projected samples x 3, 7 nearest squared-distance bit patterns, 7
// nearest ids, 7 radix prefixes, 7 remaining ranks, 7 k-th values, the
// radius, then 7 histograms of 256 u32 bins.
constexpr size_t kScratchBytes = 16384;

struct StaticRadiusState {
  unsigned long long bb[6];
  double samples[7][3];
  double proj[7][3];
  unsigned long long best_bits[7];
  unsigned long long best_id[7];
  unsigned long long prefix[7];
  long long krem[7];
  double kth[7];
  double radius;
  int nsamples;
  int dim;
  unsigned int hist[7][256];
};
static_assert(sizeof(StaticRadiusState) <= kScratchBytes, "scratch array too small");

static __device__ __align__(256) unsigned char g_radius_scratch[kScratchBytes];

constexpr int kThreads = 256;

__global__ void k_sr_reset(StaticRadiusState *st, int dim, long long k) {
  for (int i = threadIdx.x; i < 7 * 256; i += blockDim.x) (&st->hist[0][0])[i] = 0u;
  if (threadIdx.x < 7) {
    const int s = threadIdx.x;
    st->best_bits[s] = ~0ull;
    st->best_id[s] = ~0ull;
    st->prefix[s] = 0ull;
    st->krem[s] = k;
    st->kth[s] = 0.0;
  }
  if (threadIdx.x < 3) {
    st->bb[threadIdx.x] = ~0ull;
    st->bb[3 + threadIdx.x] = 0ull;
  }
  if (threadIdx.x == 0) {
    st->dim = dim;
    st->nsamples = 2 * dim + 1;
    st->radius = 0.0;
  }
}

__device__ __forceinline__ void load_point(const double *pts, int dim, int64_t i, double &x,
                                           double &y, double &z) {
  x = pts[i * dim];
  y = dim > 1 ? pts[i * dim + 1] : 0.0;
  z = dim > 2 ? pts[i * dim + 2] : 0.0;
}

__device__ __forceinline__ unsigned long long wmin(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w < v ? w : v;
  }
  return v;
}
__device__ __forceinline__ unsigned long long wmax(unsigned long long v) {
  for (int o = 16; o > 0; o >>= 1) {
    const unsigned long long w = __shfl_xor_sync(0xffffffffu, v, o);
    v = w > v ? w : v;
  }
  return v;
}

// Source bounding box by exact order-preserving 64-bit atomics.
__global__ void k_sr_bbox(const double *pts, int dim, int64_t n, StaticRadiusState *st) {
  unsigned long long mn0 = ~0ull, mn1 = ~0ull, mn2 = ~0ull, mx0 = 0ull, mx1 = 0ull, mx2 = 0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x, y, z;
    load_point(pts, dim, i, x, y, z);
    const unsigned long long ox = dbl_to_ordered(x), oy = dbl_to_ordered(y), oz = dbl_to_ordered(z);
    mn0 = ox < mn0 ? ox : mn0;
    mn1 = oy < mn1 ? oy : mn1;
    mn2 = oz < mn2 ? oz : mn2;
    mx0 = ox > mx0 ? ox : mx0;
    mx1 = oy > mx1 ? oy : mx1;
    mx2 = oz > mx2 ? oz : mx2;
  }
  mn0 = wmin(mn0);
  mn1 = wmin(mn1);
  mn2 = wmin(mn2);
  mx0 = wmax(mx0);
  mx1 = wmax(mx1);
  mx2 = wmax(mx2);
  if ((threadIdx.x & 31) == 0) {
    atomicMin(&st->bb[0], mn0);
    atomicMin(&st->bb[1], mn1);
    atomicMin(&st->bb[2], mn2);
    atomicMax(&st->bb[3], mx0);
    atomicMax(&st->bb[4], mx1);
    atomicMax(&st->bb[5], mx2);
  }
}

// Samples: bounding-box centre and centre -/+ a quarter of each extent
// (src/rbf_pum/clustering/clusters_radius.hpp:36-51).
__global__ void k_sr_samples(StaticRadiusState *st) {
  if (threadIdx.x != 0) return;
  const int dim = st->dim;
  double lo[3], hi[3], c[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < 3; ++d) {
    lo[d] = d < dim ? ordered_to_dbl(st->bb[d]) : 0.0;
    hi[d] = d < dim ? ordered_to_dbl(st->bb[3 + d]) : 0.0;
  }
  for (int d = 0; d < dim; ++d) c[d] = __ddiv_rn(__dadd_rn(lo[d], hi[d]), 2.0);
  for (int s = 0; s < 7; ++s)
    for (int d = 0; d < 3; ++d) st->samples[s][d] = c[d];
  for (int a = 0; a < dim; ++a) {
    const double len = fabs(__dsub_rn(hi[a], lo[a]));
    double s_a = __dsub_rn(c[a], __dmul_rn(len, 0.25));
    st->samples[a + 1][a] = s_a;
    s_a = __dadd_rn(s_a, __dmul_rn(len, 0.5));
    st->samples[dim + a + 1][a] = s_a;
  }
}

// Nearest source of sample blockIdx.y: minimum squared distance, then the
// lowest id attaining it.
template <bool kIndex>
__global__ void k_sr_nearest(const double *pts, int dim, int64_t n, StaticRadiusState *st) {
  const int s = blockIdx.y;
  if (s >= st->nsamples) return;
  const double sx = st->samples[s][0], sy = st->samples[s][1], sz = st->samples[s][2];
  const unsigned long long target = kIndex ? st->best_bits[s] : 0ull;
  unsigned long long best = ~0ull;
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x, y, z;
    load_point(pts, dim, i, x, y, z);
    const unsigned long long b =
        (unsigned long long)__double_as_longlong(sqdist3(sx, sy, sz, x, y, z));
    if (kIndex) {
      if (b == target && (unsigned long long)i < best) best = (unsigned long long)i;
    } else {
      best = b < best ? b : best;
    }
  }
  best = wmin(best);
  if ((threadIdx.x & 31) == 0) atomicMin(kIndex ? &st->best_id[s] : &st->best_bits[s], best);
}

__global__ void k_sr_project(const double *pts, int dim, int64_t n, StaticRadiusState *st) {
  const int s = threadIdx.x;
  if (s >= st->nsamples) return;
  const unsigned long long id = st->best_id[s];
  double x = st->samples[s][0], y = st->samples[s][1], z = st->samples[s][2];
  if (id < (unsigned long long)n) load_point(pts, dim, (int64_t)id, x, y, z);
  st->proj[s][0] = x;
  st->proj[s][1] = y;
  st->proj[s][2] = z;
}

// One 8-bit radix-select pass of the k-th smallest squared distance from
// projected sample blockIdx.y to every source.
__global__ void k_sr_hist(const double *pts, int dim, int64_t n, StaticRadiusState *st,
                          int pass) {
  __shared__ unsigned int h[256];
  const int s = blockIdx.y;
  if (s >= st->nsamples) return;
  for (int i = threadIdx.x; i < 256; i += blockDim.x) h[i] = 0u;
  __syncthreads();
  const int shift = 56 - 8 * pass;
  const unsigned long long hmask = pass == 0 ? 0ull : (~0ull << (64 - 8 * pass));
  const double sx = st->proj[s][0], sy = st->proj[s][1], sz = st->proj[s][2];
  const unsigned long long pre = st->prefix[s];
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x) {
    double x, y, z;
    load_point(pts, dim, i, x, y, z);
    const unsigned long long key =
        (unsigned long long)__double_as_longlong(sqdist3(sx, sy, sz, x, y, z));
    if ((key & hmask) == pre) atomicAdd(&h[(key >> shift) & 0xffu], 1u);
  }
  __syncthreads();
  for (int i = threadIdx.x; i < 256; i += blockDim.x)
    if (h[i]) atomicAdd(&st->hist[s][i], h[i]);
}

__global__ void k_sr_select(StaticRadiusState *st, int pass) {
  const int s = threadIdx.x;
  if (s >= st->nsamples) return;
  const int shift = 56 - 8 * pass;
  const long long k = st->krem[s];
  long long cum = 0;
  int d = 0;
  for (; d < 256; ++d) {
    const long long c = st->hist[s][d];
    if (cum + c >= k) break;
    cum += c;
  }
  if (d > 255) d = 255;
  st->prefix[s] |= ((unsigned long long)d) << shift;
  st->krem[s] = k - cum;
  for (int i = 0; i < 256; ++i) st->hist[s][i] = 0u;
  if (pass == 7) st->kth[s] = __longlong_as_double((long long)st->prefix[s]);
}

// Median of the sorted per-sample values (clusters_radius.hpp:121-124).
__global__ void k_sr_final(StaticRadiusState *st) {
  if (threadIdx.x != 0) return;
  double v[7];
  const int ns = st->nsamples;
  for (int s = 0; s < ns; ++s) v[s] = st->kth[s];
  for (int i = 1; i < ns; ++i) {
    const double x = v[i];
    int j = i - 1;
    while (j >= 0 && v[j] > x) {
      v[j + 1] = v[j];
      --j;
    }
    v[j + 1] = x;
  }
  st->radius = __dsqrt_rn(v[st->dim]);
}

int sr_fail(int code, const std::string &m) {
  set_last_error(m);
  return code;
}

// Device address of the scratch array in the CUDA context that is current on
// the calling thread.  A __device__ symbol's address belongs to one context:
// after cudaDeviceReset, or when the caller makes a context of its own
// current (driver API), an address cached from an earlier call would point
// into memory this call does not own.  So every call resolves it again; the
// lookup is cheap and allocates nothing.  The first call on a device also
// loads this file's kernels into the context.
int scratch_address(StaticRadiusState **out) {
  void *p = nullptr;
  const cudaError_t e = cudaGetSymbolAddress(&p, g_radius_scratch);
  if (e != cudaSuccess || !p) {
    cudaGetLastError();
    return sr_fail(PACMAN_B200_ERR_CUDA,
                   std::string("cudaGetSymbolAddress of the radius scratch failed: ") +
                       cudaGetErrorString(e));
  }
  *out = static_cast<StaticRadiusState *>(p);
  return 0;
}

}  // namespace
}  // namespace pacman_b200

using namespace pacman_b200;

extern "C" PACMAN_B200_API int pacman_b200_patch_radius_noalloc(
    int32_t dim, const double *source_points, int64_t n_source, int32_t nodes_per_cluster,
    void *stream, double *radius) {
  set_last_error(std::string());
  if (dim < 1 || dim > 3)
    return sr_fail(PACMAN_B200_ERR_DIMENSION,
                   "The dimension of the points can only be: 1, 2 or 3 (the scratch array holds "
                   "the state of at most 2*3+1 = 7 samples).");
  if (n_source < 1) return sr_fail(PACMAN_B200_ERR_INVALID, "n_source must be >= 1");
  if (n_source > 0x7fffffffll)
    return sr_fail(PACMAN_B200_ERR_LIMIT, "n_source is limited to 2^31 - 1 points");
  if (nodes_per_cluster < 1) return sr_fail(PACMAN_B200_ERR_INVALID, "nodes_per_cluster must be > 0");
  if (!source_points || !radius) return sr_fail(PACMAN_B200_ERR_INVALID, "null pointer argument");
  int device = 0;
  if (cudaGetDevice(&device) != cudaSuccess) {
    cudaGetLastError();
    return sr_fail(PACMAN_B200_ERR_CUDA, "no current CUDA device");
  }
  cudaPointerAttributes at{};
  if (cudaPointerGetAttributes(&at, source_points) != cudaSuccess ||
      !((at.type == cudaMemoryTypeDevice && at.device == device) ||
        at.type == cudaMemoryTypeManaged)) {
    cudaGetLastError();
    return sr_fail(PACMAN_B200_ERR_INVALID,
                   "source_points must be device memory of the current device (this entry point "
                   "allocates nothing, so it cannot stage host arrays)");
  }
  StaticRadiusState *st = nullptr;
  if (int rc = scratch_address(&st)) return rc;
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const long long k = nodes_per_cluster < n_source ? nodes_per_cluster : n_source;
  const int ns = 2 * dim + 1;
  int64_t b = (n_source + kThreads - 1) / kThreads;
  const int blocks = int(b < 1 ? 1 : (b > 148 * 4 ? 148 * 4 : b));
  k_sr_reset<<<1, 256, 0, s>>>(st, dim, k);
  k_sr_bbox<<<blocks, kThreads, 0, s>>>(source_points, dim, n_source, st);
  k_sr_samples<<<1, 32, 0, s>>>(st);
  k_sr_nearest<false><<<dim3(blocks, ns), kThreads, 0, s>>>(source_points, dim, n_source, st);
  k_sr_nearest<true><<<dim3(blocks, ns), kThreads, 0, s>>>(source_points, dim, n_source, st);
  k_sr_project<<<1, 32, 0, s>>>(source_points, dim, n_source, st);
  for (int pass = 0; pass < 8; ++pass) {
    k_sr_hist<<<dim3(blocks, ns), kThreads, 0, s>>>(source_points, dim, n_source, st, pass);
    k_sr_select<<<1, 32, 0, s>>>(st, pass);
  }
  k_sr_final<<<1, 32, 0, s>>>(st);
  double r_host = 0.0;
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(radius, &st->radius, sizeof(double), cudaMemcpyDefault, s);
  if (e == cudaSuccess)
    e = cudaMemcpyAsync(&r_host, &st->radius, sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    return sr_fail(PACMAN_B200_ERR_CUDA, std::string("radius kernels: ") + cudaGetErrorString(e));
  // The full transfer rejects the same radius (all sources coincide, or a
  // coordinate is not finite); so does this entry point, after writing it.
  if (!(r_host > 0.0) || !std::isfinite(r_host))
    return sr_fail(PACMAN_B200_ERR_DEGENERATE, "degenerate patch radius (zero or non-finite)");
  return 0;
}
