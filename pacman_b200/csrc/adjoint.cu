// Adjoint of the RBF-PUM transfer (no counterpart in the reference, which
// only evaluates the forward map, src/rbf_pum/solver/solver.hpp:217-286).
//
// For fixed geometry the transfer is linear in the source values:
//   out(t) = sum_k  wn_k(t) * local_k(t),   wn_k = w_k / S,  S = sum of w over
//   every centre within the patch radius,
//   local_k = E_k A_k^{-1} (I - Q_k P_k) b_k + V_k P_k b_k,  P = (Q^T Q)^{-1} Q^T.
// With A symmetric, the transpose applied to an upstream gradient G is, per
// patch, h = wn * G on its targets, z = A^{-1} E^T h and
//   g = z - Q' G'^{-1} (Q'^T z - V'^T h)   (centred monomials q' = [1, x - c]),
// summed over the patches that hold each source (solve.cu / blocked.cu do
// the per-patch part, kAdj / kBigAdjoint).  The gradient with respect to the
// target coordinates, at fixed membership, is
//   d out / d y = sum_k [ wn_k grad(local_k) + local_k (grad w_k - wn_k grad S) / S ],
//   grad(local_k)(y) = sum_j alpha_j phi'(|y - x_j| / rho) / rho (y - x_j) / |y - x_j|
//                      + beta_active,
// using the coefficients saved by the forward call.
#include <cub/cub.cuh>

#include <algorithm>
#include <vector>

#include "plan.hpp"
#include "poly.cuh"

namespace pacman_b200 {

void solve_adjoint(Plan &p, int basis, int F, const double *h, double *g_out, SolveReport &rep);

namespace {

constexpr int kMaxC = 64;  // centres held in registers per target (larger sets are re-scanned)

struct WeightTerm {
  int k;
  double w;
  double gx, gy, gz;  // gradient of w with respect to the target
};

// Centres within r of y in ascending order, with their C2 weights and
// weight gradients.  Returns the count (cnt > kMaxC: only the first kMaxC
// are stored and the caller re-scans).
__device__ int centre_terms(const GridView &cg, const double4 *centers, double4 y, double r,
                            double rinv, WeightTerm *out, int after, bool want_grad) {
  int cnt = 0;
  for_neighbors(cg, y.x, y.y, y.z, [&](int k) {
    if (k <= after) return;
    const double4 c = centers[k];
    const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, c.x, c.y, c.z));
    if (!(d <= r)) return;
    if (cnt < kMaxC) {
      WeightTerm t;
      t.k = k;
      t.w = wendland<double>(kWendlandC2, d, rinv);
      t.gx = t.gy = t.gz = 0.0;
      if (want_grad && d > 0.0) {
        const double s = wendland_dp(kWendlandC2, d * rinv) * rinv / d;
        t.gx = s * (y.x - c.x);
        t.gy = s * (y.y - c.y);
        t.gz = s * (y.z - c.z);
      }
      int j = cnt - 1;
      while (j >= 0 && out[j].k > k) {
        out[j + 1] = out[j];
        --j;
      }
      out[j + 1] = t;
    }
    ++cnt;
  });
  return cnt;
}

// S_t (and grad S_t) in ascending centre order, as the forward gather sums it.
__global__ void k_weight_sums(int64_t M, const double4 *__restrict__ tgt, GridView cg,
                              const double4 *__restrict__ centers, double r, double rinv,
                              double *wsum, double *wgrad) {
  WeightTerm terms[kMaxC];
  for (int64_t t = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; t < M;
       t += (int64_t)gridDim.x * blockDim.x) {
    const double4 y = tgt[t];
    double S = 0.0, gx = 0.0, gy = 0.0, gz = 0.0;
    int after = -1;
    for (;;) {
      const int cnt = centre_terms(cg, centers, y, r, rinv, terms, after, wgrad != nullptr);
      const int c = cnt < kMaxC ? cnt : kMaxC;
      for (int i = 0; i < c; ++i) {
        S = __dadd_rn(S, terms[i].w);
        gx += terms[i].gx;
        gy += terms[i].gy;
        gz += terms[i].gz;
      }
      if (cnt <= kMaxC) break;
      after = terms[kMaxC - 1].k;
    }
    wsum[t] = S;
    if (wgrad) {
      wgrad[3 * t] = gx;
      wgrad[3 * t + 1] = gy;
      wgrad[3 * t + 2] = gz;
    }
  }
}

// h = (w / S) * G per (patch, target), warp per patch.
__global__ void k_adj_h(int K, const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                        const double4 *__restrict__ tgt, const double4 *__restrict__ centers,
                        double rinv, const double *__restrict__ wsum, const double *__restrict__ gout,
                        int F, double *h) {
  const int lane = threadIdx.x & 31;
  const int warps = (blockDim.x >> 5) * gridDim.x;
  for (int k = (blockIdx.x * blockDim.x + threadIdx.x) >> 5; k < K; k += warps) {
    const double4 c = centers[k];
    for (int64_t e = toff[k] + lane; e < toff[k + 1]; e += 32) {
      const int t = tidx[e];
      const double4 y = tgt[t];
      const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, c.x, c.y, c.z));
      const double wn = __ddiv_rn(wendland<double>(kWendlandC2, d, rinv), wsum[t]);
      for (int f = 0; f < F; ++f) h[e * F + f] = __dmul_rn(wn, gout[int64_t(t) * F + f]);
    }
  }
}

// grad_values[i] = sum over the patches holding source i (ascending) of g.
__global__ void k_gather_sources(int64_t N, const int *__restrict__ off, const int *__restrict__ pos,
                                 const double *__restrict__ g, int F, double *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < N;
       i += (int64_t)gridDim.x * blockDim.x) {
    double acc[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) acc[f] = 0.0;
    for (int q = off[i]; q < off[i + 1]; ++q) {
      const int64_t e = pos[q];
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) acc[f] = __dadd_rn(acc[f], g[e * F + f]);
    }
    for (int f = 0; f < F; ++f) out[i * F + f] = acc[f];
  }
}

// Gradient of each patch's local interpolant at each of its targets
// (3 x F values per (patch, target)), warp per target, lanes over sources.
__global__ void __launch_bounds__(256)
    k_dlocal(int K, const double4 *__restrict__ src, const double4 *__restrict__ tgt,
             const int64_t *__restrict__ soff, const int *__restrict__ sidx,
             const int64_t *__restrict__ toff, const int *__restrict__ tidx,
             const double *__restrict__ alpha, const double *__restrict__ beta,
             const int *__restrict__ act, int basis, double rinv, int F, double *dloc) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  for (int k = blockIdx.x; k < K; k += gridDim.x) {
    const int64_t s0 = soff[k], t0 = toff[k];
    const int n = int(soff[k + 1] - s0), m = int(toff[k + 1] - t0);
    for (int i = warp; i < m; i += 8) {
      const double4 y = tgt[tidx[t0 + i]];
      double g[3][kMaxF];
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int f = 0; f < kMaxF; ++f) g[d][f] = 0.0;
      for (int j = lane; j < n; j += 32) {
        const double4 x = src[sidx[s0 + j]];
        const double dist = __dsqrt_rn(sqdist3(x.x, x.y, x.z, y.x, y.y, y.z));
        if (!(dist > 0.0)) continue;
        const double coef = wendland_dp(basis, dist * rinv) * rinv / dist;
        const double dx = coef * (y.x - x.x), dy = coef * (y.y - x.y), dz = coef * (y.z - x.z);
#pragma unroll
        for (int f = 0; f < kMaxF; ++f)
          if (f < F) {
            const double al = alpha[(s0 + j) * F + f];
            g[0][f] = __fma_rn(al, dx, g[0][f]);
            g[1][f] = __fma_rn(al, dy, g[1][f]);
            g[2][f] = __fma_rn(al, dz, g[2][f]);
          }
      }
#pragma unroll
      for (int d = 0; d < 3; ++d)
#pragma unroll
        for (int f = 0; f < kMaxF; ++f) g[d][f] = warp_sum(g[d][f]);
      if (lane == 0) {
        const double *b = beta + int64_t(k) * 4 * kMaxF;
        const int *ac = act + int64_t(k) * 3;
        for (int q = 0; q < 3; ++q)
          if (ac[q] >= 0)
            for (int f = 0; f < F; ++f) g[ac[q]][f] += b[4 * f + 1 + q];
        for (int d = 0; d < 3; ++d)
          for (int f = 0; f < F; ++f) dloc[(t0 + i) * 3 * F + d * F + f] = g[d][f];
      }
    }
  }
}

__device__ __forceinline__ int64_t find_sorted(const int *a, int64_t n, int v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = (lo + hi) >> 1;
    if (a[mid] < v) lo = mid + 1;
    else hi = mid;
  }
  return (lo < n && a[lo] == v) ? lo : -1;
}

// d (sum_f G_f out_f) / d y per target.
__global__ void k_target_grad(int64_t M, const int *__restrict__ tlist, int dim,
                              const double4 *__restrict__ tgt, GridView cg,
                              const double4 *__restrict__ centers, double r, double rinv,
                              const double *__restrict__ wsum, const double *__restrict__ wgrad,
                              const int64_t *__restrict__ toff, const int *__restrict__ tidx,
                              const double *__restrict__ local, const double *__restrict__ dloc,
                              const double *__restrict__ gout, int F, double *grad) {
  WeightTerm terms[kMaxC];
  // M targets: all (tlist null) or those of a shard's list.
  for (int64_t it = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; it < M;
       it += (int64_t)gridDim.x * blockDim.x) {
    const int64_t t = tlist ? tlist[it] : it;
    const double4 y = tgt[t];
    const double S = wsum[t];
    const double gS[3] = {wgrad[3 * t], wgrad[3 * t + 1], wgrad[3 * t + 2]};
    double acc[3] = {0.0, 0.0, 0.0};
    int after = -1;
    for (;;) {
      const int cnt = centre_terms(cg, centers, y, r, rinv, terms, after, true);
      const int c = cnt < kMaxC ? cnt : kMaxC;
      for (int i = 0; i < c; ++i) {
        const int k = terms[i].k;
        const int64_t b = toff[k];
        const int64_t pos = find_sorted(tidx + b, toff[k + 1] - b, int(t));
        if (pos < 0) continue;
        const double wn = terms[i].w / S;
        const double gw[3] = {terms[i].gx, terms[i].gy, terms[i].gz};
        for (int f = 0; f < F; ++f) {
          const double gf = gout[t * F + f];
          const double loc = local[(b + pos) * F + f];
          for (int d = 0; d < 3; ++d) {
            const double dwn = (gw[d] - wn * gS[d]) / S;
            acc[d] += gf * (dwn * loc + wn * dloc[(b + pos) * 3 * F + d * F + f]);
          }
        }
      }
      if (cnt <= kMaxC) break;
      after = terms[kMaxC - 1].k;
    }
    for (int d = 0; d < dim; ++d) grad[t * dim + d] = acc[d];
  }
}

__global__ void k_iota(int64_t n, int *out) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i < n;
       i += (int64_t)gridDim.x * blockDim.x)
    out[i] = int(i);
}

// off[c] = first sorted position whose key >= c, for c in [0, N].
__global__ void k_key_start(const int *skeys, int64_t nnz, int64_t N, int *off) {
  for (int64_t i = blockIdx.x * (int64_t)blockDim.x + threadIdx.x; i <= nnz;
       i += (int64_t)gridDim.x * blockDim.x) {
    const int64_t prev = (i == 0) ? -1 : skeys[i - 1];
    const int64_t cur = (i == nnz) ? N + 1 : skeys[i];
    for (int64_t c = prev + 1; c <= cur && c <= N; ++c) off[c] = int(i);
  }
}

inline int blocks_for(int64_t n, int per = 256, int cap = 148 * 32) {
  int64_t b = (n + per - 1) / per;
  return int(std::max<int64_t>(1, std::min<int64_t>(b, cap)));
}

// Sources -> positions in the membership lists, ascending patch order.
void build_source_transpose(Plan &p) {
  if (p.src_t_off.p) return;
  cudaStream_t st = p.stream;
  const int64_t nnz = p.snnz;
  DevMem keys, vals, skeys, tmp;
  keys.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  vals.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  skeys.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  p.src_t_pos.alloc(sizeof(int) * std::max<int64_t>(nnz, 1), st);
  p.src_t_off.alloc(sizeof(int) * (p.n + 1), st);
  if (nnz > 0) {
    PB_CUDA(cudaMemcpyAsync(keys.p, p.sidx.p, sizeof(int) * nnz, cudaMemcpyDeviceToDevice, st));
    k_iota<<<blocks_for(nnz), 256, 0, st>>>(nnz, vals.as<int>());
    note_launch();
    int end_bit = 1;
    while ((int64_t(1) << end_bit) <= p.n) ++end_bit;
    size_t tb = 0;
    PB_CUDA(cub::DeviceRadixSort::SortPairs(nullptr, tb, keys.as<int>(), skeys.as<int>(),
                                            vals.as<int>(), p.src_t_pos.as<int>(), int(nnz), 0,
                                            end_bit, st));
    tmp.alloc(tb, st);
    PB_CUDA(cub::DeviceRadixSort::SortPairs(tmp.p, tb, keys.as<int>(), skeys.as<int>(),
                                            vals.as<int>(), p.src_t_pos.as<int>(), int(nnz), 0,
                                            end_bit, st));
    k_key_start<<<blocks_for(nnz + 1), 256, 0, st>>>(skeys.as<int>(), nnz, p.n,
                                                     p.src_t_off.as<int>());
    note_launch();
  } else {
    PB_CUDA(cudaMemsetAsync(p.src_t_off.p, 0, sizeof(int) * (p.n + 1), st));
  }
  PB_CUDA(cudaGetLastError());
}

}  // namespace

void adjoint(Plan &p, const double *gout, double *grad_values, double *grad_targets) {
  if (p.saved_basis < 0)
    throw Error{PACMAN_B200_ERR_INVALID,
                "the adjoint needs a previous execute with PACMAN_B200_SAVE_FOR_ADJOINT"};
  cudaStream_t st = p.stream;
  const int F = p.saved_F;
  const int64_t N = p.n, M = p.m;
  if (grad_values) PB_CUDA(cudaMemsetAsync(grad_values, 0, sizeof(double) * N * F, st));
  if (grad_targets) PB_CUDA(cudaMemsetAsync(grad_targets, 0, sizeof(double) * M * p.dim, st));
  if (p.K == 0 || M == 0 || N == 0) {
    PB_CUDA(host_sync(st));
    return;
  }
  const double r = p.radius, rinv = 1.0 / r;
  DevMem wsum, wgrad;
  wsum.alloc(sizeof(double) * M, st);
  if (grad_targets) wgrad.alloc(sizeof(double) * 3 * M, st);
  k_weight_sums<<<blocks_for(M, 128, 148 * 64), 128, 0, st>>>(
      M, p.tgt4.as<double4>(), p.cgrid.view, p.centers.as<double4>(), r, rinv, wsum.as<double>(),
      grad_targets ? wgrad.as<double>() : nullptr);
  note_launch();
  if (grad_values) {
    DevMem h, g;
    h.alloc(sizeof(double) * std::max<int64_t>(p.tnnz, 1) * F, st);
    g.alloc(sizeof(double) * std::max<int64_t>(p.snnz, 1) * F, st);
    PB_CUDA(cudaMemsetAsync(g.p, 0, sizeof(double) * std::max<int64_t>(p.snnz, 1) * F, st));
    k_adj_h<<<std::max(1, std::min((p.K + 7) / 8, 148 * 32)), 256, 0, st>>>(
        p.K, p.toff.as<int64_t>(), p.tidx.as<int>(), p.tgt4.as<double4>(), p.centers.as<double4>(),
        rinv, wsum.as<double>(), gout, F, h.as<double>());
    note_launch();
    SolveReport rep;
    solve_adjoint(p, p.saved_basis, F, h.as<double>(), g.as<double>(), rep);
    build_source_transpose(p);
    k_gather_sources<<<blocks_for(N), 256, 0, st>>>(N, p.src_t_off.as<int>(), p.src_t_pos.as<int>(),
                                                    g.as<double>(), F, grad_values);
    note_launch();
  }
  if (grad_targets) {
    DevMem dloc;
    dloc.alloc(sizeof(double) * std::max<int64_t>(p.tnnz, 1) * 3 * F, st);
    k_dlocal<<<std::max(1, std::min(p.K, 148 * 16)), 256, 0, st>>>(
        p.K, p.src4.as<double4>(), p.tgt4.as<double4>(), p.soff.as<int64_t>(), p.sidx.as<int>(),
        p.toff.as<int64_t>(), p.tidx.as<int>(), p.alpha.as<double>(), p.beta.as<double>(),
        p.act.as<int>(), p.saved_basis, 1.0 / p.opts.support_radius, F, dloc.as<double>());
    note_launch();
    const bool sharded = p.m_owned >= 0;
    const int64_t Mg = sharded ? p.m_owned : M;
    if (Mg > 0) {
      k_target_grad<<<blocks_for(Mg, 128, 148 * 64), 128, 0, st>>>(
          Mg, sharded ? p.tlist.as<int>() : nullptr, p.dim, p.tgt4.as<double4>(), p.cgrid.view,
          p.centers.as<double4>(), r, rinv, wsum.as<double>(), wgrad.as<double>(),
          p.toff.as<int64_t>(), p.tidx.as<int>(), p.local.as<double>(), dloc.as<double>(), gout,
          F, grad_targets);
      note_launch();
    }
  }
  PB_CUDA(cudaGetLastError());
  PB_CUDA(host_sync(st));
}

}  // namespace pacman_b200
