// Per-patch solves of the B200 RBF-PUM transfer
// (src/rbf_pum/solver/solver.hpp:180-286 and solver/utils/*.hpp).
//
// One CTA per patch.  The patch's points, the Wendland matrix A (with the
// right-hand sides as extra columns) and all reductions live in shared
// memory when they fit; larger patches use a global workspace (the same code
// with a different base pointer) or the blocked engine of blocked.cu.
//
// Modes:
//   kLU    the reference algorithm: unpivoted Doolittle LU (KokkosBatched
//          SerialLU<Unblocked>, serial_solve.hpp:76-84) in FP64;
//   kChol  FP64 Cholesky of the symmetric positive definite A (half the flops),
//          with a per-patch breakdown flag that sends the patch back to kLU.
//
// The polynomial block (serial_ops.hpp:108-139, serial_solve.hpp:46-67) is
// solved from one reduction pass: the Gram matrix of the patch-centred
// monomials [1, x - c] gives the least-squares fit and, through its Cholesky
// factor times the change of basis back to [1, x], the singular values of the
// reference's uncentred Q for the condition test.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "blocked.cuh"
#include "patch.cuh"

namespace pacman_b200 {

constexpr int kSolveThreads = 256;
constexpr int kWarps = kSolveThreads / 32;

template <int MODE>
__global__ void __launch_bounds__(kSolveThreads)
    k_patch_solve(PatchArgs a, const int *__restrict__ plist, int np, int use_global) {
  extern __shared__ double smem[];
  __shared__ double red[kWarps][kRedVals];
  __shared__ double redf[kRedVals];
  __shared__ double beta_s[4 * kMaxF];
  __shared__ int act_s[3];
  __shared__ int flag_s;
  const int e = blockIdx.x;
  if (e >= np) return;
  const int k = plist[e];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t s0 = a.soff[k];
  const int n = int(a.soff[k + 1] - s0);
  const int64_t t0 = a.toff[k];
  const int m = int(a.toff[k + 1] - t0);
  const int F = a.F;
  const int lda = n + F;
  double *xs = smem;
  double *ys = xs + n;
  double *zs = ys + n;
  double *A = use_global ? (a.gA + a.gAoff[e]) : (zs + n);
  if (tid == 0) flag_s = 0;

  // Gather the patch (TeamFillB, team_ops.hpp:113-121).
  const double4 c = a.centers[k];
  const double shift[3] = {c.x, c.y, c.z};
  const int Fm = (MODE == kAdj) ? 0 : F;  // value moments only for the forward fit
  const int nred = 10 + 4 * Fm;
  for (int i = tid; i < n; i += kSolveThreads) {
    const int id = a.sidx[s0 + i];
    const double4 p = a.src[id];
    xs[i] = p.x;
    ys[i] = p.y;
    zs[i] = p.z;
    for (int f = 0; f < Fm; ++f) A[int64_t(i) * lda + n + f] = a.vals[int64_t(id) * F + f];
  }
  __syncthreads();
  // Moments of the centred monomials q = [1, x - c] (and q * b per field),
  // then the coordinate ranges: one thread per value, points in order.
  if (tid < nred + 6) {
    double v;
    if (tid < nred) {
      int i0, i1 = 0, f = -1;
      if (tid < 4) {
        i0 = tid;
      } else if (tid < 10) {
        const int pr[6][2] = {{1, 1}, {1, 2}, {1, 3}, {2, 2}, {2, 3}, {3, 3}};
        i0 = pr[tid - 4][0];
        i1 = pr[tid - 4][1];
      } else {
        f = (tid - 10) >> 2;
        i0 = (tid - 10) & 3;
      }
      v = 0.0;
      for (int i = 0; i < n; ++i) {
        const double q[4] = {1.0, xs[i] - shift[0], ys[i] - shift[1], zs[i] - shift[2]};
        const double w = (f >= 0) ? A[int64_t(i) * lda + n + f] : (tid < 4 ? 1.0 : q[i1]);
        v += q[i0] * w;
      }
    } else {
      const int d = (tid - nred) % 3;
      const bool is_max = tid - nred >= 3;
      const double *x = d == 0 ? xs : (d == 1 ? ys : zs);
      v = x[0];
      for (int i = 1; i < n; ++i) v = is_max ? fmax(v, x[i]) : fmin(v, x[i]);
    }
    redf[tid] = v;
  }
  __syncthreads();
  __shared__ int S_s[4], pv_s;
  __shared__ double R_s[4][4];
  if (tid == 0) {
    if (MODE == kAdj) {
      int S[4], pv;
      double R[4][4];
      const int dropped = poly_axes(redf, a.dim, shift, redf + nred, redf + nred + 3, S, pv, R);
      for (int i = 0; i < 4; ++i) {
        S_s[i] = S[i];
        for (int j = 0; j < 4; ++j) R_s[i][j] = R[i][j];
      }
      pv_s = pv;
      flag_s = dropped ? kStatusDropped : 0;
    } else {
      int act[3];
      const int dropped = poly_block(redf, F, a.dim, shift, beta_s, act);
      for (int d = 0; d < 3; ++d) act_s[d] = act[d];
      flag_s = dropped ? kStatusDropped : 0;
    }
  }
  __syncthreads();

  if (MODE == kAdj) {
    // Right-hand sides c = E^T h, E_ij = phi(|y_i - x_j|).
    for (int j = tid; j < n; j += kSolveThreads) {
      double cs[kMaxF];
#pragma unroll
      for (int f = 0; f < kMaxF; ++f) cs[f] = 0.0;
      for (int i = 0; i < m; ++i) {
        const double4 y = a.tgt[a.tidx[t0 + i]];
        const double ph =
            wendland<double>(a.basis, __dsqrt_rn(sqdist3(y.x, y.y, y.z, xs[j], ys[j], zs[j])), a.rinv);
#pragma unroll
        for (int f = 0; f < kMaxF; ++f)
          if (f < F) cs[f] = __fma_rn(ph, a.h[(t0 + i) * F + f], cs[f]);
      }
      for (int f = 0; f < F; ++f) A[int64_t(j) * lda + n + f] = cs[f];
    }
  } else {
    // Residual r = b - Q beta (serial_ops.hpp:149-185, gemv + vector sub).
    for (int i = tid; i < n; i += kSolveThreads) {
      const double pc[3] = {xs[i], ys[i], zs[i]};
      for (int f = 0; f < F; ++f) {
        double t = beta_s[4 * f];
        for (int j = 0; j < 3; ++j)
          if (act_s[j] >= 0) t = __fma_rn(pc[act_s[j]], beta_s[4 * f + 1 + j], t);
        A[int64_t(i) * lda + n + f] -= t;
      }
    }
  }
  // A_ij = phi(|x_i - x_j|) (TeamFillA, team_ops.hpp:35-52): warp per row,
  // upper triangle evaluated once and mirrored.
  for (int i = warp; i < n; i += kWarps) {
    const double xi = xs[i], yi = ys[i], zi = zs[i];
    for (int j = i + lane; j < n; j += 32) {
      const double d = __dsqrt_rn(sqdist3(xi, yi, zi, xs[j], ys[j], zs[j]));
      const double v = wendland<double>(a.basis, d, a.rinv);
      A[int64_t(i) * lda + j] = v;
      A[int64_t(j) * lda + i] = v;
    }
  }
  __syncthreads();

  // Factorisation with the right-hand sides as extra columns (the forward
  // substitution happens inside the elimination).
  if (MODE == kLU) {
    for (int p = 0; p < n; ++p) {
      const double piv = A[int64_t(p) * lda + p];
      for (int i = p + 1 + warp; i < n; i += kWarps) {
        double l = 0.0;
        if (lane == 0) {
          l = A[int64_t(i) * lda + p] / piv;
          A[int64_t(i) * lda + p] = l;
        }
        l = __shfl_sync(0xffffffffu, l, 0);
        double *ri = A + int64_t(i) * lda;
        const double *rp = A + int64_t(p) * lda;
        for (int j = p + 1 + lane; j < lda; j += 32) ri[j] = __fma_rn(-l, rp[j], ri[j]);
      }
      __syncthreads();
    }
  } else {
    double *lcol = xs;  // reuse after the assembly: xs is no longer needed here
    __shared__ double piv_s;
    (void)lcol;
    for (int p = 0; p < n; ++p) {
      if (tid == 0) {
        const double app = A[int64_t(p) * lda + p];
        if (!(app > 0.0)) flag_s |= kStatusBreakdown;
        piv_s = sqrt(app);
      }
      __syncthreads();
      const double d = piv_s;
      for (int i = p + tid; i < n; i += kSolveThreads) {
        double *ai = A + int64_t(i) * lda + p;
        *ai = (i == p) ? d : (*ai / d);
      }
      if (tid < F) A[int64_t(p) * lda + n + tid] /= d;
      __syncthreads();
      for (int i = p + 1 + warp; i < n; i += kWarps) {
        double *ri = A + int64_t(i) * lda;
        const double li = ri[p];
        for (int j = p + 1 + lane; j <= i; j += 32)
          ri[j] = __fma_rn(-li, A[int64_t(j) * lda + p], ri[j]);
        if (lane < F) ri[n + lane] = __fma_rn(-li, A[int64_t(p) * lda + n + lane], ri[n + lane]);
      }
      __syncthreads();
    }
  }
  // Back substitution, one warp per field: U alpha = y (LU) or L^T alpha = y.
  if (warp < F) {
    const int f = warp;
    for (int p = n - 1; p >= 0; --p) {
      double xp = 0.0;
      if (lane == 0) {
        xp = A[int64_t(p) * lda + n + f] / A[int64_t(p) * lda + p];
        A[int64_t(p) * lda + n + f] = xp;
      }
      xp = __shfl_sync(0xffffffffu, xp, 0);
      for (int i = lane; i < p; i += 32) {
        const double u = (MODE == kLU) ? A[int64_t(i) * lda + p] : A[int64_t(p) * lda + i];
        A[int64_t(i) * lda + n + f] = __fma_rn(-u, xp, A[int64_t(i) * lda + n + f]);
      }
      __syncwarp();
    }
  }
  __syncthreads();

  if (MODE == kAdj) {
    // g = z - Q' G'^{-1} (Q'^T z - V'^T h), centred monomials q' = [1, x - c].
    __shared__ double corr[4 * kMaxF];
    for (int f = 0; f < F; ++f) {
      double u[4] = {0, 0, 0, 0}, v[4] = {0, 0, 0, 0};
      for (int j = tid; j < n; j += kSolveThreads) {
        const double z = A[int64_t(j) * lda + n + f];
        const double q[4] = {1.0, xs[j] - shift[0], ys[j] - shift[1], zs[j] - shift[2]};
        for (int c2 = 0; c2 < 4; ++c2) u[c2] += q[c2] * z;
      }
      for (int i = tid; i < m; i += kSolveThreads) {
        const double4 y = a.tgt[a.tidx[t0 + i]];
        const double hv = a.h[(t0 + i) * F + f];
        const double q[4] = {1.0, y.x - shift[0], y.y - shift[1], y.z - shift[2]};
        for (int c2 = 0; c2 < 4; ++c2) v[c2] += q[c2] * hv;
      }
      for (int c2 = 0; c2 < 4; ++c2) {
        const double su = warp_sum(u[c2]), sv = warp_sum(v[c2]);
        if (lane == 0) {
          red[warp][c2] = su;
          red[warp][4 + c2] = sv;
        }
      }
      __syncthreads();
      if (tid == 0) {
        const int pv = pv_s;
        double rhs[4], x[4];
        for (int i = 0; i < pv; ++i) {
          double su = 0.0, sv = 0.0;
          for (int w = 0; w < kWarps; ++w) {
            su += red[w][S_s[i]];
            sv += red[w][4 + S_s[i]];
          }
          rhs[i] = su - sv;
        }
        gram_solve(R_s, pv, rhs, x);
        for (int c2 = 0; c2 < 4; ++c2) corr[4 * f + c2] = 0.0;
        for (int i = 0; i < pv; ++i) corr[4 * f + S_s[i]] = x[i];
      }
      __syncthreads();
    }
    int nonfinite = 0;
    for (int j = tid; j < n; j += kSolveThreads) {
      const double q[4] = {1.0, xs[j] - shift[0], ys[j] - shift[1], zs[j] - shift[2]};
      for (int f = 0; f < F; ++f) {
        double g = A[int64_t(j) * lda + n + f];
        for (int c2 = 0; c2 < 4; ++c2) g -= q[c2] * corr[4 * f + c2];
        if (!isfinite(g)) nonfinite = 1;
        a.g_out[(s0 + j) * F + f] = g;
      }
    }
    if (nonfinite) atomicOr(&flag_s, kStatusNonFinite);
    __syncthreads();
    if (tid == 0) a.status[k] = flag_s;
    return;
  }
  if (a.alpha_out) {
    for (int j = tid; j < n; j += kSolveThreads)
      for (int f = 0; f < F; ++f) a.alpha_out[(s0 + j) * F + f] = A[int64_t(j) * lda + n + f];
    if (tid < 4 * kMaxF) a.beta_out[int64_t(k) * 4 * kMaxF + tid] = beta_s[tid];
    if (tid < 3) a.act_out[int64_t(k) * 3 + tid] = act_s[tid];
  }

  // local = E alpha + V beta (solver.hpp:270-273), warp per target.
  int nonfinite = 0;
  for (int i = warp; i < m; i += kWarps) {
    const double4 y = a.tgt[a.tidx[t0 + i]];
    double s[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) s[f] = 0.0;
    for (int j = lane; j < n; j += 32) {
      const double d = __dsqrt_rn(sqdist3(y.x, y.y, y.z, xs[j], ys[j], zs[j]));
      const double ph = wendland<double>(a.basis, d, a.rinv);
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) s[f] = __fma_rn(ph, A[int64_t(j) * lda + n + f], s[f]);
    }
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) s[f] = warp_sum(s[f]);
    if (lane == 0) {
      const double yc[3] = {y.x, y.y, y.z};
      for (int f = 0; f < F; ++f) {
        double v = beta_s[4 * f];
        for (int j = 0; j < 3; ++j)
          if (act_s[j] >= 0) v = __fma_rn(yc[act_s[j]], beta_s[4 * f + 1 + j], v);
        const double out = s[f] + v;
        if (!isfinite(out)) nonfinite = 1;
        a.local[(t0 + i) * F + f] = out;
      }
    }
  }
  if (nonfinite) atomicOr(&flag_s, kStatusNonFinite);
  __syncthreads();
  if (tid == 0) a.status[k] = flag_s;
}

// Shared memory of one patch: 3n coordinates + n x (n + F) matrix.
static size_t smem_bytes(int n, int F, bool with_A) {
  size_t d = size_t(3) * n;
  if (with_A) d += size_t(n) * size_t(n + F);
  return d * sizeof(double);
}

static void launch(int mode, const PatchArgs &a, const int *plist, int np, int use_global,
                   size_t smem, cudaStream_t st) {
  if (np == 0) return;
  if (mode == kLU) {
    PB_CUDA(cudaFuncSetAttribute(k_patch_solve<kLU>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(smem)));
    k_patch_solve<kLU><<<np, kSolveThreads, smem, st>>>(a, plist, np, use_global);
    note_launch();
  } else if (mode == kAdj) {
    PB_CUDA(cudaFuncSetAttribute(k_patch_solve<kAdj>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_patch_solve<kAdj><<<np, kSolveThreads, smem, st>>>(a, plist, np, use_global);
    note_launch();
  } else {
    PB_CUDA(cudaFuncSetAttribute(k_patch_solve<kChol>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize, int(smem)));
    k_patch_solve<kChol><<<np, kSolveThreads, smem, st>>>(a, plist, np, use_global);
    note_launch();
  }
  PB_CUDA(cudaGetLastError());
}

// Runs one mode over a list of patches: buckets by size so the dynamic
// shared memory follows the bucket's largest patch; patches too large for
// shared memory use the global workspace.
static void run_list(Plan &p, PatchArgs a, int mode, const std::vector<int> &patches,
                     SolveReport &rep, cudaStream_t st, FactorCache *keep = nullptr) {
  if (patches.empty()) return;
  for (int k : patches) {
    const double n = p.n_host[k], m = p.m_host[k];
    rep.factor_flops += (mode == kLU ? 2.0 / 3.0 : 1.0 / 3.0) * n * n * n +
                        2.0 * n * n * a.F + 2.0 * m * n * a.F;
  }
  const int F = a.F;
  const size_t smem_cap = 200 * 1024;
  std::vector<int> order(patches);
  std::sort(order.begin(), order.end(),
            [&](int x, int y) { return p.n_host[x] < p.n_host[y]; });
  std::vector<int> small, big;
  for (int k : order) {
    if (smem_bytes(p.n_host[k], F, true) <= smem_cap) small.push_back(k);
    else big.push_back(k);
  }
  // Small: buckets of doubling size, each launched with its own shared memory.
  size_t pos = 0;
  std::vector<std::pair<size_t, size_t>> ranges;
  while (pos < small.size()) {
    const int n0 = p.n_host[small[pos]];
    int cap = 32;
    while (cap < n0) cap *= 2;
    size_t end = pos;
    while (end < small.size() && p.n_host[small[end]] <= cap &&
           smem_bytes(p.n_host[small[end]], F, true) <= smem_cap)
      ++end;
    ranges.emplace_back(pos, end);
    pos = end;
  }
  std::vector<int> host_list(small);
  host_list.insert(host_list.end(), big.begin(), big.end());
  DevMem list;
  list.alloc(sizeof(int) * host_list.size(), st);
  HostArena::get().upload(host_list.data(), host_list.size(), list.p, st);
  if (keep) {
    // Kept factors of the register kernel: N * N doubles per patch of the
    // launch's size class, in launch order.
    size_t tot = 0;
    keep->ranges.clear();
    for (auto &r : ranges) {
      int nmax = 0;
      for (size_t i = r.first; i < r.second; ++i) nmax = std::max(nmax, p.n_host[small[i]]);
      if (mode != kChol || nmax > 64) continue;
      SmallRange sr;
      sr.first = r.first;
      sr.count = int(r.second - r.first);
      sr.nmax = nmax;
      sr.fac_off = tot;
      tot += size_t(sr.count) * small_fac_doubles(nmax <= 32 ? 32 : 64);
      keep->ranges.push_back(sr);
    }
    keep->small_fac.alloc(sizeof(double) * std::max<size_t>(tot, 2), st);
  }
  size_t ri = 0;
  for (auto &r : ranges) {
    int nmax = 0;
    for (size_t i = r.first; i < r.second; ++i) nmax = std::max(nmax, p.n_host[small[i]]);
    if (mode == kChol && nmax <= 64) {
      PatchArgs b = a;
      if (keep) {
        b.fac = keep->small_fac.as<double>() + keep->ranges[ri++].fac_off;
        b.fac_mode = 1;
      }
      launch_small_chol(b, list.as<int>() + r.first, int(r.second - r.first), nmax, st);
    } else
      launch(mode, a, list.as<int>() + r.first, int(r.second - r.first), 0,
             smem_bytes(nmax, F, true), st);
  }
  if (!big.empty()) {
    std::vector<int64_t> offs(big.size());
    int64_t tot = 0;
    int nmax = 0;
    for (size_t i = 0; i < big.size(); ++i) {
      offs[i] = tot;
      const int64_t n = p.n_host[big[i]];
      tot += n * (n + F);
      nmax = std::max<int>(nmax, int(n));
    }
    DevMem goff, gA;
    goff.alloc(sizeof(int64_t) * big.size(), st);
    gA.alloc(sizeof(double) * size_t(tot), st);
    HostArena::get().upload(offs.data(), offs.size(), goff.p, st);
    PatchArgs b = a;
    b.gA = gA.as<double>();
    b.gAoff = goff.as<int64_t>();
    launch(mode, b, list.as<int>() + small.size(), int(big.size()), 1,
           smem_bytes(nmax, F, false), st);
  }
  if (keep) keep->small_list = std::move(list);  // freed with the plan's cache
}

// The register-kernel patches from kept factors.
static void run_small_cached(const FactorCache &c, PatchArgs a, cudaStream_t st) {
  for (const SmallRange &r : c.ranges) {
    PatchArgs b = a;
    b.fac = const_cast<double *>(c.small_fac.as<double>()) + r.fac_off;
    b.fac_mode = 2;
    launch_small_chol(b, c.small_list.as<int>() + r.first, r.count, r.nmax, st);
  }
}

void solve_big(Plan &p, int basis, const double *vals, int F, bool lu,
               const std::vector<int> &patches, double *local, int *status, SolveReport &rep,
               const BigExtra &extra, FactorCache *keep = nullptr);
void solve_big_cached(Plan &p, FactorCache &c, int basis, const double *vals, int F,
                      double *local, int *status, SolveReport &rep, const BigExtra &extra);

// Patches above this size use the blocked engine (blocked.cu): for the
// Cholesky path the tuned value (64 by default; the register kernels of
// small.cu take n <= 64), 128 for the LU and adjoint paths.
// PACMAN_B200_BIG_N overrides both.
static int big_threshold(int mode) {
  const char *e = std::getenv("PACMAN_B200_BIG_N");
  if (e) return std::max(1, std::atoi(e));
  return mode == kChol ? std::min(64, std::max(1, tuning_for_current_device().big_n_chol)) : 128;
}

static void solve_patches_impl(Plan &p, int basis, const double *vals_dev, int F, int precision,
                               double *local_dev, SolveReport &rep, bool save, bool keep_factors) {
  cudaStream_t st = p.stream;
  const int K = p.K;
  if (K == 0) return;
  const bool chol = precision != PACMAN_B200_FP64;
  const FactorCache *cached =
      (keep_factors && chol && p.fcache && p.fcache->basis == basis) ? p.fcache.get() : nullptr;
  FactorCache *keep = nullptr;
  if (keep_factors && !cached) {
    p.fcache.reset();
    if (chol) {
      p.fcache.reset(new FactorCache());
      p.fcache->basis = basis;
      keep = p.fcache.get();
    }
  }
  p.status.alloc(sizeof(int) * K, st);
  PB_CUDA(cudaMemsetAsync(p.status.p, 0, sizeof(int) * K, st));
  BigExtra ex;
  if (save) {
    p.alpha.alloc(sizeof(double) * std::max<int64_t>(p.snnz, 1) * F, st);
    p.beta.alloc(sizeof(double) * K * 4 * kMaxF, st);
    p.act.alloc(sizeof(int) * K * 3, st);
    PB_CUDA(cudaMemsetAsync(p.alpha.p, 0, sizeof(double) * std::max<int64_t>(p.snnz, 1) * F, st));
    PB_CUDA(cudaMemsetAsync(p.beta.p, 0, sizeof(double) * K * 4 * kMaxF, st));
    PB_CUDA(cudaMemsetAsync(p.act.p, 0xff, sizeof(int) * K * 3, st));
    ex.mode = kBigForwardSave;
    ex.alpha_out = p.alpha.as<double>();
    ex.beta_out = p.beta.as<double>();
    ex.act_out = p.act.as<int>();
  }
  PatchArgs a{};
  a.alpha_out = ex.alpha_out;
  a.beta_out = ex.beta_out;
  a.act_out = ex.act_out;
  a.src = p.src4.as<double4>();
  a.tgt = p.tgt4.as<double4>();
  a.vals = vals_dev;
  a.soff = p.soff.as<int64_t>();
  a.sidx = p.sidx.as<int>();
  a.toff = p.toff.as<int64_t>();
  a.tidx = p.tidx.as<int>();
  a.centers = p.centers.as<double4>();
  a.local = local_dev;
  a.status = p.status.as<int>();
  a.rinv = 1.0 / p.opts.support_radius;
  a.F = F;
  a.dim = p.dim;
  a.basis = basis;
  const int mode = precision == PACMAN_B200_FP64 ? kLU : kChol;
  const int nbig = big_threshold(mode);
  std::vector<int> small, big;
  for (int k = 0; k < K; ++k) {
    if (p.m_host[k] == 0) continue;  // no target: the patch contributes nothing
    (p.n_host[k] > nbig ? big : small).push_back(k);
  }
  cudaEvent_t ev0, ev1;
  PB_CUDA(cudaEventCreate(&ev0));
  PB_CUDA(cudaEventCreate(&ev1));
  PB_CUDA(cudaEventRecord(ev0, st));
  // Small patches on the low-priority stream, started where the large-patch
  // steps stop filling the GPU (the engine re-records the event there; with
  // no large patches it stays at this point of the plan's stream).
  p.aux.make();
  cudaStream_t ss = p.aux.s[AuxStreams::kSmall];
  rep.tail_event = p.aux.ev[AuxStreams::kN + 1];
  PB_CUDA(cudaEventRecord(rep.tail_event, st));
  if (cached) {
    // Kept factors: the small patches start at once (no factorisation steps
    // to wait for), the large ones run their sweeps on the group streams.
    PB_CUDA(cudaStreamWaitEvent(ss, rep.tail_event, 0));
    run_small_cached(*cached, a, ss);
    solve_big_cached(p, *p.fcache, basis, vals_dev, F, local_dev, p.status.as<int>(), rep, ex);
    for (const SmallRange &r : cached->ranges) rep.factors_reused += r.count;
  } else {
    solve_big(p, basis, vals_dev, F, mode == kLU, big, local_dev, p.status.as<int>(), rep, ex,
              keep);
    PB_CUDA(cudaStreamWaitEvent(ss, rep.tail_event, 0));
    run_list(p, a, mode, small, rep, ss, keep);
  }
  PB_CUDA(cudaEventRecord(p.aux.ev[AuxStreams::kN + 2], ss));
  PB_CUDA(cudaStreamWaitEvent(st, p.aux.ev[AuxStreams::kN + 2], 0));
  rep.tail_event = nullptr;
  std::vector<int> stat(K);
  PB_CUDA(cudaMemcpyAsync(stat.data(), p.status.p, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
  PB_CUDA(cudaEventRecord(ev1, st));
  PB_CUDA(host_sync(st));
  float ms = 0.f;
  PB_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
  rep.ms_factor += ms;
  finish_kernel_timing(rep, ev0);
  std::vector<int> redo_small, redo_big;
  std::vector<char> redo_mark(cached ? K : 0, 0);
  if (cached) {  // patches the factorising execute sent to the LU path
    for (int k : cached->redo_small) redo_mark[k] = 1;
    for (int k : cached->redo_big) redo_mark[k] = 2;
  }
  for (int k = 0; k < K; ++k) {
    if (p.m_host[k] == 0) continue;
    if (stat[k] & kStatusDropped) rep.dropped++;
    if ((mode == kChol && (stat[k] & (kStatusBreakdown | kStatusNonFinite | kStatusTimeout))) ||
        (cached && redo_mark[k]))
      (p.n_host[k] > nbig ? redo_big : redo_small).push_back(k);
  }
  if (keep) {
    keep->redo_small = redo_small;
    keep->redo_big = redo_big;
  }
  p.patch_status = stat;
  for (int k : redo_small) p.patch_status[k] |= kStatusResolved;
  for (int k : redo_big) p.patch_status[k] |= kStatusResolved;
  rep.patches_fp64 = int64_t(small.size() + big.size());
  if (!redo_small.empty() || !redo_big.empty()) {
    PB_CUDA(cudaEventRecord(ev0, st));
    run_list(p, a, kLU, redo_small, rep, st);
    solve_big(p, basis, vals_dev, F, true, redo_big, local_dev, p.status.as<int>(), rep, ex);
    PB_CUDA(cudaEventRecord(ev1, st));
    PB_CUDA(host_sync(st));
    PB_CUDA(cudaEventElapsedTime(&ms, ev0, ev1));
    rep.ms_factor += ms;
    rep.patches_fallback += int64_t(redo_small.size() + redo_big.size());
  }
  cudaEventDestroy(ev0);
  cudaEventDestroy(ev1);
}

void solve_patches(Plan &p, int basis, const double *vals_dev, int F, int precision,
                   double *local_dev, SolveReport &rep, bool save, bool keep_factors) {
  try {
    solve_patches_impl(p, basis, vals_dev, F, precision, local_dev, rep, save, keep_factors);
  } catch (...) {
    if (keep_factors) p.fcache.reset();  // a half-built cache is never reused
    throw;
  }
}

// Per-patch adjoint solves: g (per patch, source) from h (per patch, target).
void solve_adjoint(Plan &p, int basis, int F, const double *h, double *g_out, SolveReport &rep) {
  cudaStream_t st = p.stream;
  const int K = p.K;
  if (K == 0) return;
  p.status.alloc(sizeof(int) * K, st);
  PB_CUDA(cudaMemsetAsync(p.status.p, 0, sizeof(int) * K, st));
  PatchArgs a{};
  a.src = p.src4.as<double4>();
  a.tgt = p.tgt4.as<double4>();
  a.soff = p.soff.as<int64_t>();
  a.sidx = p.sidx.as<int>();
  a.toff = p.toff.as<int64_t>();
  a.tidx = p.tidx.as<int>();
  a.centers = p.centers.as<double4>();
  a.status = p.status.as<int>();
  a.rinv = 1.0 / p.opts.support_radius;
  a.F = F;
  a.dim = p.dim;
  a.basis = basis;
  a.h = h;
  a.g_out = g_out;
  const int nbig = big_threshold(kAdj);
  std::vector<int> small, big;
  for (int k = 0; k < K; ++k) {
    if (p.m_host[k] == 0) continue;  // h = 0 there: g = 0 (the caller zeroes g)
    (p.n_host[k] > nbig ? big : small).push_back(k);
  }
  run_list(p, a, kAdj, small, rep, p.stream);
  BigExtra ex;
  ex.mode = kBigAdjoint;
  ex.h = h;
  ex.g_out = g_out;
  solve_big(p, basis, nullptr, F, false, big, nullptr, p.status.as<int>(), rep, ex);
  // The adjoint has no second path: a pipeline wait that gave up is an error.
  std::vector<int> stat(K);
  PB_CUDA(cudaMemcpyAsync(stat.data(), p.status.p, sizeof(int) * K, cudaMemcpyDeviceToHost, st));
  PB_CUDA(host_sync(st));
  for (int k = 0; k < K; ++k)
    if (stat[k] & kStatusTimeout)
      throw Error{PACMAN_B200_ERR_CUDA, "adjoint: a pipeline wait timed out in patch " +
                                            std::to_string(k)};
}

}  // namespace pacman_b200
