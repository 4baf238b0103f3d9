// Target sharding of one transfer over several GPUs (one process per GPU).
//
// The patch cover depends on every source and every target (a candidate
// centre without a target within r is dropped before the order-dependent
// pruning, clustering.hpp:204-254), so each rank builds the whole geometry.
// The targets are then cut into `world` contiguous ranges of their Morton
// order, balanced by the solve cost of the patches each range needs; a rank
// keeps only its targets in the patch target lists, solves the patches that
// still hold a target, and gathers its own targets.  Every patch solve and
// every gather is the one of the unsharded transfer, so the results are
// bit-identical; the other targets of the output are zero, and a sum over the
// ranks (one all-reduce) assembles the whole result exactly.
//
// The cut is computed on every rank from integer data only (costs, Morton
// keys, a stable radix sort, an integer scan), so all ranks agree on it.
#include <cub/cub.cuh>

#include <algorithm>

#include "plan.hpp"

namespace pacman_b200 {

namespace {

constexpr int kMortonBits = 21;  // per axis

// Solve cost of patch k spread over its targets: n^3 / m in units of 256.
__global__ void k_target_cost(int K, const int64_t *__restrict__ soff,
                              const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                              unsigned long long *cost) {
  const int lane = threadIdx.x & 31;
  const int warps = int(gridDim.x * blockDim.x) >> 5;
  for (int k = int(blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
    const int64_t t0 = toff[k], m = toff[k + 1] - t0;
    if (m == 0) continue;
    int64_t nk = soff[k + 1] - soff[k];
    if (nk > (int64_t(1) << 21)) nk = int64_t(1) << 21;  // n^3 stays below 2^63
    const unsigned long long n = static_cast<unsigned long long>(nk);
    unsigned long long share = (n * n * n / static_cast<unsigned long long>(m)) >> 8;
    if (share == 0) share = 1;
    for (int64_t i = lane; i < m; i += 32) atomicAdd(&cost[tidx[t0 + i]], share);
  }
}

// Morton key of every target over the source bounding box (clamped), one
// more unit of cost per target, and the identity permutation.
__global__ void k_morton(int64_t M, int dim, const double4 *__restrict__ tgt, double3 lo,
                         double3 scale, unsigned long long *key, unsigned long long *cost,
                         int *iota) {
  const double qmax = double((1u << kMortonBits) - 1);
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < M;
       t += int64_t(gridDim.x) * blockDim.x) {
    const double4 y = tgt[t];
    const double c[3] = {y.x, y.y, y.z}, l[3] = {lo.x, lo.y, lo.z}, s[3] = {scale.x, scale.y, scale.z};
    unsigned long long kk = 0;
    for (int a = 0; a < dim; ++a) {
      double q = __dmul_rn(__dsub_rn(c[a], l[a]), s[a]);
      if (!(q > 0.0)) q = 0.0;
      if (q > qmax) q = qmax;
      const unsigned long long v = static_cast<unsigned long long>(q);
      for (int b = 0; b < kMortonBits; ++b) kk |= ((v >> b) & 1ull) << (b * dim + a);
    }
    key[t] = kk;
    cost[t] += 1ull;
    iota[t] = int(t);
  }
}

__global__ void k_gather_cost(int64_t M, const int *__restrict__ order,
                              const unsigned long long *__restrict__ cost,
                              unsigned long long *sorted_cost) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < M;
       i += int64_t(gridDim.x) * blockDim.x)
    sorted_cost[i] = cost[order[i]];
}

// Position i of the Morton order goes to rank floor(P_{i-1} * world / total),
// P the inclusive prefix of the costs: contiguous ranges of equal cost.
__global__ void k_owned_flags(int64_t M, const int *__restrict__ order,
                              const unsigned long long *__restrict__ sorted_cost,
                              const unsigned long long *__restrict__ prefix,
                              unsigned long long total, int world, int rank, unsigned char *flag) {
  for (int64_t i = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; i < M;
       i += int64_t(gridDim.x) * blockDim.x) {
    const unsigned long long before = prefix[i] - sorted_cost[i];
    const unsigned long long r = before * static_cast<unsigned long long>(world) / total;
    const int ri = r < static_cast<unsigned long long>(world) ? int(r) : world - 1;
    flag[order[i]] = ri == rank ? 1 : 0;
  }
}

// Owned entries per patch target list (warp per patch).
__global__ void k_list_count(int K, const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                             const unsigned char *__restrict__ flag, int64_t *cnt) {
  const int lane = threadIdx.x & 31;
  const int warps = int(gridDim.x * blockDim.x) >> 5;
  for (int k = int(blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
    int c = 0;
    for (int64_t i = toff[k] + lane; i < toff[k + 1]; i += 32) c += flag[tidx[i]];
    for (int o = 16; o > 0; o >>= 1) c += __shfl_xor_sync(0xffffffffu, c, o);
    if (lane == 0) cnt[k] = c;
  }
  if (blockIdx.x == 0 && threadIdx.x == 0) cnt[K] = 0;
}

// The owned entries of every list, in their order (warp per patch).
__global__ void k_list_fill(int K, const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                            const unsigned char *__restrict__ flag,
                            const int64_t *__restrict__ noff, int *nidx, int *ncount) {
  const int lane = threadIdx.x & 31;
  const int warps = int(gridDim.x * blockDim.x) >> 5;
  for (int k = int(blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
    int64_t out = noff[k];
    for (int64_t b = toff[k]; b < toff[k + 1]; b += 32) {
      const int64_t i = b + lane;
      const int t = i < toff[k + 1] ? tidx[i] : 0;
      const bool keep = i < toff[k + 1] && flag[t];
      const unsigned mask = __ballot_sync(0xffffffffu, keep);
      if (keep) nidx[out + __popc(mask & ((1u << lane) - 1u))] = t;
      out += __popc(mask);
    }
    if (lane == 0) ncount[k] = int(noff[k + 1] - noff[k]);
  }
}

inline int blocks(int64_t n, int per = 256, int cap = 148 * 16) {
  return int(std::max<int64_t>(1, std::min<int64_t>((n + per - 1) / per, cap)));
}

}  // namespace

void shard_plan(Plan &p, int rank, int world) {
  if (p.m_owned >= 0) throw Error{PACMAN_B200_ERR_INVALID, "the plan is already sharded"};
  if (world < 1 || rank < 0 || rank >= world)
    throw Error{PACMAN_B200_ERR_INVALID, "shard rank must be in [0, world)"};
  cudaStream_t st = p.stream;
  const int64_t M = p.m;
  const int K = p.K;
  p.fcache.reset();  // kept factors were laid out for the unsharded target lists
  p.shard_rank = rank;
  p.shard_world = world;
  if (M == 0) {
    p.m_owned = 0;
    return;
  }
  DevMem cost, key, key2, iota, order, scost, prefix, flag, tmp, tmp2, nsel;
  cost.alloc(sizeof(unsigned long long) * M, st);
  PB_CUDA(cudaMemsetAsync(cost.p, 0, sizeof(unsigned long long) * M, st));
  if (K > 0) {
    k_target_cost<<<blocks(int64_t(K) * 32), 256, 0, st>>>(
        K, p.soff.as<int64_t>(), p.toff.as<int64_t>(), p.tidx.as<int>(),
        cost.as<unsigned long long>());
    note_launch();
  }
  key.alloc(sizeof(unsigned long long) * M, st);
  key2.alloc(sizeof(unsigned long long) * M, st);
  iota.alloc(sizeof(int) * M, st);
  order.alloc(sizeof(int) * M, st);
  double lo[3] = {0, 0, 0}, sc[3] = {0, 0, 0};
  for (int a = 0; a < p.dim; ++a) {
    lo[a] = p.lo[a];
    const double e = p.hi[a] - p.lo[a];
    sc[a] = e > 0.0 ? double((1u << kMortonBits) - 1) / e : 0.0;
  }
  k_morton<<<blocks(M), 256, 0, st>>>(M, p.dim, p.tgt4.as<double4>(),
                                      make_double3(lo[0], lo[1], lo[2]),
                                      make_double3(sc[0], sc[1], sc[2]),
                                      key.as<unsigned long long>(), cost.as<unsigned long long>(),
                                      iota.as<int>());
  note_launch();
  size_t tb = 0;
  const int end_bit = kMortonBits * p.dim;
  PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, key.as<unsigned long long>(),
                                          key2.as<unsigned long long>(), iota.as<int>(),
                                          order.as<int>(), M, 0, end_bit, st));
  tmp.alloc(tb, st);
  PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, key.as<unsigned long long>(),
                                          key2.as<unsigned long long>(), iota.as<int>(),
                                          order.as<int>(), M, 0, end_bit, st));
  scost.alloc(sizeof(unsigned long long) * M, st);
  prefix.alloc(sizeof(unsigned long long) * M, st);
  k_gather_cost<<<blocks(M), 256, 0, st>>>(M, order.as<int>(), cost.as<unsigned long long>(),
                                           scost.as<unsigned long long>());
  note_launch();
  tb = 0;
  PB_CUDA(cub::DeviceScan::InclusiveSum(nullptr, tb, scost.as<unsigned long long>(),
                                        prefix.as<unsigned long long>(), M, st));
  tmp2.alloc(tb, st);
  PB_CUDA(cub::DeviceScan::InclusiveSum(tmp2.p, tb, scost.as<unsigned long long>(),
                                        prefix.as<unsigned long long>(), M, st));
  unsigned long long total = 0;
  PB_CUDA(cudaMemcpyAsync(&total, prefix.as<unsigned long long>() + (M - 1), sizeof(total),
                          cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  if (total == 0 || total > ~0ull / static_cast<unsigned long long>(world))
    throw Error{PACMAN_B200_ERR_LIMIT, "target costs out of range for the shard cut"};
  flag.alloc(M, st);
  k_owned_flags<<<blocks(M), 256, 0, st>>>(M, order.as<int>(), scost.as<unsigned long long>(),
                                           prefix.as<unsigned long long>(), total, world, rank,
                                           flag.as<unsigned char>());
  note_launch();
  // Owned targets, ascending.
  p.tlist.alloc(sizeof(int) * M, st);
  nsel.alloc(sizeof(int), st);
  cub::CountingInputIterator<int> ids(0);
  tb = 0;
  PB_CUDA(cub::DeviceSelect::Flagged(nullptr, tb, ids, flag.as<unsigned char>(), p.tlist.as<int>(),
                                     nsel.as<int>(), int(M), st));
  DevMem tmp3;
  tmp3.alloc(tb, st);
  PB_CUDA(cub::DeviceSelect::Flagged(tmp3.p, tb, ids, flag.as<unsigned char>(), p.tlist.as<int>(),
                                     nsel.as<int>(), int(M), st));
  int owned = 0;
  PB_CUDA(cudaMemcpyAsync(&owned, nsel.p, sizeof(int), cudaMemcpyDeviceToHost, st));
  // Patch target lists restricted to the owned targets.
  if (K > 0) {
    DevMem cnt, noff, nidx, ncount, tmp4;
    cnt.alloc(sizeof(int64_t) * (K + 1), st);
    noff.alloc(sizeof(int64_t) * (K + 1), st);
    k_list_count<<<blocks(int64_t(K) * 32), 256, 0, st>>>(K, p.toff.as<int64_t>(), p.tidx.as<int>(),
                                                          flag.as<unsigned char>(),
                                                          cnt.as<int64_t>());
    note_launch();
    tb = 0;
    PB_CUDA(cub::DeviceScan::ExclusiveSum(nullptr, tb, cnt.as<int64_t>(), noff.as<int64_t>(),
                                          K + 1, st));
    tmp4.alloc(tb, st);
    PB_CUDA(cub::DeviceScan::ExclusiveSum(tmp4.p, tb, cnt.as<int64_t>(), noff.as<int64_t>(),
                                          K + 1, st));
    int64_t nnz = 0;
    PB_CUDA(cudaMemcpyAsync(&nnz, noff.as<int64_t>() + K, sizeof(int64_t), cudaMemcpyDeviceToHost,
                            st));
    PB_CUDA(host_sync(st));
    nidx.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
    ncount.alloc(sizeof(int) * K, st);
    k_list_fill<<<blocks(int64_t(K) * 32), 256, 0, st>>>(K, p.toff.as<int64_t>(), p.tidx.as<int>(),
                                                         flag.as<unsigned char>(),
                                                         noff.as<int64_t>(), nidx.as<int>(),
                                                         ncount.as<int>());
    note_launch();
    PB_CUDA(cudaMemcpyAsync(p.m_host.data(), ncount.p, sizeof(int) * K, cudaMemcpyDeviceToHost,
                            st));
    PB_CUDA(host_sync(st));
    std::swap(p.toff.p, noff.p);
    std::swap(p.toff.bytes, noff.bytes);
    std::swap(p.toff.s, noff.s);
    std::swap(p.tidx.p, nidx.p);
    std::swap(p.tidx.bytes, nidx.bytes);
    std::swap(p.tidx.s, nidx.s);
    p.tnnz = nnz;
  }
  PB_CUDA(host_sync(st));
  PB_CUDA(cudaGetLastError());
  p.m_owned = owned;
}

}  // namespace pacman_b200
