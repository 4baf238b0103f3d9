// Register-resident Cholesky solver for the small patches (n <= 64) of the
// B200 RBF-PUM transfer, precision "mixed".
//
// Per patch (src/rbf_pum/solver/solver.hpp:180-286): A = phi(|x_i - x_j|),
// the polynomial block (serial_ops.hpp:108-139) and alpha = A^{-1}(b - Q beta),
// local = E alpha + V beta.  A team of (N/4)^2 threads holds the N x N matrix
// (N = 32 or 64, zero padded with an identity block) as 4 x 4 register blocks
// and eliminates it as L D L^T with the identity carried along (Gauss-Jordan
// on [A | I]): slot (i, s) holds A[i][s] until pivot s and L^{-1}[i][s]
// afterwards; one team barrier per pivot.  Then alpha = L^{-T} D^{-1} L^{-1} r
// by two team reductions.  The polynomial block (moments, condition test,
// least squares; poly.cuh) runs meanwhile on a separate warp.  For a plan
// that keeps its factorisations the eliminated blocks are stored after the
// elimination (fac_mode 1) and later loaded in place of assembly and
// elimination (fac_mode 2): N * N doubles per patch, thread-block order.
#include "patch.cuh"

namespace pacman_b200 {

namespace {

template <int N>
struct SmallCfg {
  static constexpr int kG = N / 4;                      // 4 x 4 blocks per side
  static constexpr int kTeam = kG * kG;                 // threads per patch
  static constexpr int kTeams = 256 / kTeam;            // patches per CTA
  static constexpr int kThreads = kTeams * kTeam + 32;  // + the polynomial warp
  static constexpr int kTPT = N / 16;                   // threads per target (evaluation)
};

template <int N>
struct SmallShared {
  double x[N], y[N], z[N];
  double b[kMaxF][N];  // values, then the residual r
  double w[kMaxF][N];  // D^{-1} L^{-1} r, then alpha
  double cv[2][N];     // the published pivot vector, double buffered
  double part[N / 4][N];
  double d[N];         // pivots of L D L^T
  double red[kRedVals];
  double beta[4 * kMaxF];
  int64_t s0, t0;
  int k, n, m, flag;
  int act[3];
};

__device__ __forceinline__ void team_sync(int id, int count) {
  asm volatile("bar.sync %0, %1;\n" ::"r"(id), "r"(count) : "memory");
}

// One reduced value of the polynomial pass: moments of the centred monomials
// q = [1, x - c] (ids 0..9), q * b_f (ids 10..nred-1), then min x,y,z and
// max x,y,z.  The points are summed in order.
template <int N>
__device__ double small_moment(const SmallShared<N> &S, int id, int nred, const double *shift) {
  const int n = S.n;
  if (id < nred) {
    int i0, i1 = 0, f = -1;
    if (id < 4) {
      i0 = id;
    } else if (id < 10) {
      const int pr[6][2] = {{1, 1}, {1, 2}, {1, 3}, {2, 2}, {2, 3}, {3, 3}};
      i0 = pr[id - 4][0];
      i1 = pr[id - 4][1];
    } else {
      f = (id - 10) >> 2;
      i0 = (id - 10) & 3;
    }
    double v = 0.0;
    for (int i = 0; i < n; ++i) {
      const double q[4] = {1.0, S.x[i] - shift[0], S.y[i] - shift[1], S.z[i] - shift[2]};
      const double w = (f >= 0) ? S.b[f][i] : (id < 4 ? 1.0 : q[i1]);
      v += q[i0] * w;
    }
    return v;
  }
  const int d = (id - nred) % 3;
  const bool is_max = id - nred >= 3;
  const double *x = d == 0 ? S.x : (d == 1 ? S.y : S.z);
  double v = x[0];
  for (int i = 1; i < n; ++i) v = is_max ? fmax(v, x[i]) : fmin(v, x[i]);
  return v;
}

// The polynomial block as a real call: its local arrays and spills stay out
// of the register allocation of the elimination.
__device__ __noinline__ int poly_block_call(const double *red, int F, int dim, const double *shift,
                                            double *beta, int *act) {
  return poly_block(red, F, dim, shift, beta, act);
}

template <int N>
__global__ void __launch_bounds__(SmallCfg<N>::kThreads)
    k_small_chol(PatchArgs a, const int *__restrict__ plist, int np) {
  using C = SmallCfg<N>;
  __shared__ SmallShared<N> sh[C::kTeams];
  const int tid = threadIdx.x;
  const int F = a.F;
  const int nred = 10 + 4 * F;
  const bool poly_warp = tid >= C::kTeams * C::kTeam;
  const int team = poly_warp ? 0 : tid / C::kTeam;
  const int lt = tid % C::kTeam;
  SmallShared<N> &S = sh[team];
  const int e = blockIdx.x * C::kTeams + team;
  const bool live = !poly_warp && e < np;

  // Gather the patch (TeamFillB, team_ops.hpp:113-121), zero padded to N.
  if (!poly_warp) {
    int k = 0, n = 0, m = 0;
    int64_t s0 = 0, t0 = 0;
    if (live) {
      k = plist[e];
      s0 = a.soff[k];
      n = int(a.soff[k + 1] - s0);
      t0 = a.toff[k];
      m = int(a.toff[k + 1] - t0);
    }
    if (lt == 0) {
      S.k = k;
      S.n = n;
      S.m = m;
      S.s0 = s0;
      S.t0 = t0;
      S.flag = 0;
    }
    if (lt < 4 * kMaxF) S.beta[lt] = 0.0;
    for (int i = lt; i < N; i += C::kTeam) {
      double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
      int id = 0;
      if (i < n) {
        id = a.sidx[s0 + i];
        p = a.src[id];
      }
      S.x[i] = p.x;
      S.y[i] = p.y;
      S.z[i] = p.z;
      for (int f = 0; f < F; ++f) S.b[f][i] = i < n ? a.vals[int64_t(id) * F + f] : 0.0;
    }
  }
  __syncthreads();

  if (poly_warp) {
    // Moments, condition test and least squares of every live patch.
    const int lane = tid & 31;
    for (int t = 0; t < C::kTeams; ++t) {
      SmallShared<N> &P = sh[t];
      if (P.n == 0) continue;
      const double4 c = a.centers[P.k];
      const double shift[3] = {c.x, c.y, c.z};
      for (int id = lane; id < nred + 6; id += 32) P.red[id] = small_moment(P, id, nred, shift);
    }
    __syncwarp();
    if (lane < C::kTeams && sh[lane].n > 0) {
      SmallShared<N> &P = sh[lane];
      const double4 c = a.centers[P.k];
      const double shift[3] = {c.x, c.y, c.z};
      int act[3];
      const int dropped = poly_block_call(P.red, F, a.dim, shift, P.beta, act);
      for (int d = 0; d < 3; ++d) P.act[d] = act[d];
      if (dropped) atomicOr(&P.flag, kStatusDropped);
    }
    __syncthreads();
    return;
  }

  // Assembly (TeamFillA, team_ops.hpp:35-52) and elimination in registers,
  // or the eliminated blocks of an earlier execute (fac_mode 2).
  const int n = S.n;
  const int bi = lt / C::kG, bs = lt % C::kG;
  const int bar = 1 + team;
  double *facp = (a.fac_mode != 0 && live) ? a.fac + size_t(e) * N * N + size_t(lt) * 16 : nullptr;
  double v[4][4];
  const bool load = a.fac_mode == 2;
  if (load && facp) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const double2 lo = *reinterpret_cast<const double2 *>(facp + 4 * r);
      const double2 hi = *reinterpret_cast<const double2 *>(facp + 4 * r + 2);
      v[r][0] = lo.x;
      v[r][1] = lo.y;
      v[r][2] = hi.x;
      v[r][3] = hi.y;
    }
  } else {
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int i = 4 * bi + r, s = 4 * bs + b;
        double val = 0.0;
        if (s <= i) {
          if (!load && i < n && s < n)
            val = wendland<double>(
                a.basis, __dsqrt_rn(sqdist3(S.x[i], S.y[i], S.z[i], S.x[s], S.y[s], S.z[s])),
                a.rinv);
          else
            val = (i == s) ? 1.0 : 0.0;
        }
        v[r][b] = val;
      }
  }
  bool bad = false;
  for (int p = 0; p < (load ? 0 : n); ++p) {
    double *c = S.cv[p & 1];
    const int pb = p >> 2, pr = p & 3;
    if (bi == pb) {  // row p: L^{-1}[p][s] for s < p, the pivot at s = p
#pragma unroll
      for (int b = 0; b < 4; ++b)
        if (4 * bs + b <= p) {
          double x = v[0][b];
          if (pr == 1) x = v[1][b];
          if (pr == 2) x = v[2][b];
          if (pr == 3) x = v[3][b];
          c[4 * bs + b] = x;
        }
    }
    if (bs == pb) {  // column p below the pivot
#pragma unroll
      for (int r = 0; r < 4; ++r)
        if (4 * bi + r > p) {
          double x = v[r][0];
          if (pr == 1) x = v[r][1];
          if (pr == 2) x = v[r][2];
          if (pr == 3) x = v[r][3];
          c[4 * bi + r] = x;
        }
    }
    team_sync(bar, C::kTeam);
    const double piv = c[p];
    bad |= !(piv > 0.0);
    const double inv = 1.0 / piv;
    double cs[4];
#pragma unroll
    for (int b = 0; b < 4; ++b) cs[b] = c[4 * bs + b];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = 4 * bi + r;
      if (i > p) {
        const double mlt = c[i] * inv;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int s = 4 * bs + b;
          if (s == p) v[r][b] = -mlt;
          else if (s <= i) v[r][b] = __fma_rn(-mlt, cs[b], v[r][b]);
        }
      }
    }
  }
  if (a.fac_mode == 1 && facp) {
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      *reinterpret_cast<double2 *>(facp + 4 * r) = make_double2(v[r][0], v[r][1]);
      *reinterpret_cast<double2 *>(facp + 4 * r + 2) = make_double2(v[r][2], v[r][3]);
    }
  }
  if (bi == bs) {
#pragma unroll
    for (int r = 0; r < 4; ++r) S.d[4 * bi + r] = v[r][r];
  }
  __syncthreads();  // the polynomial warp is done: beta and act are final

  // Residual r = b - Q beta (serial_ops.hpp:149-185).
  for (int e2 = lt; e2 < N * F; e2 += C::kTeam) {
    const int i = e2 % N, f = e2 / N;
    double r = 0.0;
    if (i < n) {
      const double pc[3] = {S.x[i], S.y[i], S.z[i]};
      double t = S.beta[4 * f];
      for (int j = 0; j < 3; ++j)
        if (S.act[j] >= 0) t = __fma_rn(pc[S.act[j]], S.beta[4 * f + 1 + j], t);
      r = S.b[f][i] - t;
    }
    S.b[f][i] = r;
  }
  team_sync(bar, C::kTeam);
  // alpha = L^{-T} D^{-1} L^{-1} r, L^{-1}[i][s] = slot (i, s) for s < i, 1 at s = i.
  for (int f = 0; f < F; ++f) {
    double pr4[4];
#pragma unroll
    for (int r = 0; r < 4; ++r) {
      const int i = 4 * bi + r;
      double s = 0.0;
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int sc = 4 * bs + b;
        const double y = sc < i ? v[r][b] : (sc == i ? 1.0 : 0.0);
        s = __fma_rn(y, S.b[f][sc], s);
      }
      pr4[r] = s;
    }
#pragma unroll
    for (int o = C::kG / 2; o > 0; o >>= 1)
#pragma unroll
      for (int r = 0; r < 4; ++r) pr4[r] += __shfl_xor_sync(0xffffffffu, pr4[r], o);
    if (bs == 0) {
#pragma unroll
      for (int r = 0; r < 4; ++r) S.w[f][4 * bi + r] = pr4[r] / S.d[4 * bi + r];
    }
    team_sync(bar, C::kTeam);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int sc = 4 * bs + b;
      double s = 0.0;
#pragma unroll
      for (int r = 0; r < 4; ++r) {
        const int i = 4 * bi + r;
        const double y = sc < i ? v[r][b] : (sc == i ? 1.0 : 0.0);
        s = __fma_rn(y, S.w[f][i], s);
      }
      S.part[bi][sc] = s;
    }
    team_sync(bar, C::kTeam);
    if (lt < N) {
      double s = 0.0;
      for (int q = 0; q < C::kG; ++q) s += S.part[q][lt];
      S.w[f][lt] = s;
    }
    team_sync(bar, C::kTeam);
  }
  if (a.alpha_out != nullptr && live) {  // teams past the end of the list hold no patch
    for (int e2 = lt; e2 < n * F; e2 += C::kTeam) {
      const int j = e2 / F, f = e2 % F;
      a.alpha_out[(S.s0 + j) * F + f] = S.w[f][j];
    }
    if (lt < 4 * kMaxF) a.beta_out[int64_t(S.k) * 4 * kMaxF + lt] = S.beta[lt];
    if (lt < 3) a.act_out[int64_t(S.k) * 3 + lt] = S.act[lt];
  }

  // local = E alpha + V beta (solver.hpp:270-273): kTPT threads per target,
  // 16 sources each.
  const int m = S.m;
  const int sub = lt % C::kTPT;
  bool nonfinite = false;
  for (int i = lt / C::kTPT; i < ((m + C::kTeam / C::kTPT - 1) / (C::kTeam / C::kTPT)) *
                                     (C::kTeam / C::kTPT);
       i += C::kTeam / C::kTPT) {
    double acc[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) acc[f] = 0.0;
    double4 y = make_double4(0.0, 0.0, 0.0, 0.0);
    if (i < m) {
      y = a.tgt[a.tidx[S.t0 + i]];
      const int j1 = min(n, 16 * sub + 16);
      for (int j = 16 * sub; j < j1; ++j) {
        const double ph = wendland<double>(
            a.basis, __dsqrt_rn(sqdist3(y.x, y.y, y.z, S.x[j], S.y[j], S.z[j])), a.rinv);
#pragma unroll
        for (int f = 0; f < kMaxF; ++f)
          if (f < F) acc[f] = __fma_rn(ph, S.w[f][j], acc[f]);
      }
    }
#pragma unroll
    for (int o = C::kTPT / 2; o > 0; o >>= 1)
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) acc[f] += __shfl_xor_sync(0xffffffffu, acc[f], o);
    if (i < m && sub == 0) {
      const double yc[3] = {y.x, y.y, y.z};
      for (int f = 0; f < F; ++f) {
        double vb = S.beta[4 * f];
        for (int d = 0; d < 3; ++d)
          if (S.act[d] >= 0) vb = __fma_rn(yc[S.act[d]], S.beta[4 * f + 1 + d], vb);
        const double out = acc[f] + vb;
        nonfinite |= !isfinite(out);
        a.local[(S.t0 + i) * F + f] = out;
      }
    }
  }
  if (nonfinite) atomicOr(&S.flag, kStatusNonFinite);
  if (lt == 0 && bad) atomicOr(&S.flag, kStatusBreakdown);
  team_sync(bar, C::kTeam);
  if (lt == 0 && live) a.status[S.k] = S.flag;
}

}  // namespace

void launch_small_chol(const PatchArgs &a, const int *plist, int np, int nmax, cudaStream_t st) {
  if (np == 0) return;
  if (nmax <= 32) {
    using C = SmallCfg<32>;
    k_small_chol<32><<<(np + C::kTeams - 1) / C::kTeams, C::kThreads, 0, st>>>(a, plist, np);
  } else {
    using C = SmallCfg<64>;
    k_small_chol<64><<<(np + C::kTeams - 1) / C::kTeams, C::kThreads, 0, st>>>(a, plist, np);
  }
  note_launch();
  PB_CUDA(cudaGetLastError());
}

}  // namespace pacman_b200
