// Blocked engine for large patches of the B200 RBF-PUM transfer.
//
// The reference solves each patch with one GPU thread running an unblocked
// LU in global memory (src/rbf_pum/solver/solver.hpp:422-490).  Here every
// patch above the shared-memory size gets an augmented matrix
//
//        [ A   r ]      A: n x n Wendland matrix (TeamFillA, team_ops.hpp:35-52)
//        [ E   0 ]      E: m x n evaluation matrix (TeamFillE, team_ops.hpp:78-97)
//                       r: n x F residuals b - Q beta (solver.hpp:451-468)
//
// stored in 64 x 64 tiles (A padded with an identity block).  Unpivoted
// elimination of the first n columns leaves the Schur complement
// S = -E A^{-1} r in the bottom-right block, i.e. minus the RBF part of the
// local interpolant (solver.hpp:474-478); no triangular solves and no
// separate evaluation pass are needed.  All large patches advance in lockstep,
// one 64-column pivot block per step:
//   k_diag    factor the diagonal tile (LU or Cholesky) and invert it,
//   k_trsm    apply the inverse to the panel tiles,
//   k_update  trailing update C -= A * op(B) of every remaining tile,
// with the tile products on the FP64 tensor cores (mma.sync m8n8k4 f64).
// Mode kLU is the reference's unpivoted LU; mode kChol uses the symmetry of A
// (lower tiles only, half the work) and flags non-positive pivots.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <vector>

#include "blocked.cuh"

namespace pacman_b200 {

// Tiles filled by the assembly of one slot: LU every (row, column) tile of
// the augmented matrix; Cholesky the lower A tiles, every E tile and the
// residual column (row t < T: t + 2 tiles, row t >= T: T + 1 tiles).
__device__ __forceinline__ void decode_assemble(bool lu, const BigSlot &sl, int l, int &ti,
                                                int &tj) {
  if (lu) {
    ti = l / (sl.T + 1);
    tj = l % (sl.T + 1);
    return;
  }
  int t = 0;
  for (;;) {
    const int len = (t < sl.T) ? t + 2 : sl.T + 1;
    if (l < len) {
      ti = t;
      tj = (t < sl.T) ? (l <= t ? l : sl.T) : l;
      return;
    }
    l -= len;
    ++t;
  }
}

// Panel tiles of step s.  LU: row panel (s, s+1..T) then column panel
// (s+1..R-1, s).  Cholesky: residual tile (s, T) then column panel.
__device__ __forceinline__ void decode_trsm(bool lu, const BigSlot &sl, int s, int l, int &ti,
                                            int &tj) {
  if (lu) {
    const int nrow = sl.T - s;
    if (l < nrow) {
      ti = s;
      tj = s + 1 + l;
    } else {
      ti = s + 1 + (l - nrow);
      tj = s;
    }
  } else if (l == 0) {
    ti = s;
    tj = sl.T;
  } else {
    ti = s + l;
    tj = s;
  }
}

// Trailing update in row strips: one CTA owns up to kStrip consecutive tiles
// of one tile row of step s, keeps the row's A tile in shared memory and
// prefetches the next B tile while the current product runs.
constexpr int kStrip = 4;

// Strip l of a slot at step s -> (row t, first list index j0, count).  The
// column list of row t is LU: s+1..T; Cholesky: s+1..min(t, T-1), then T.
__device__ __forceinline__ void decode_strip(bool lu, const BigSlot &sl, int s, int l, int &t,
                                             int &j0, int &count) {
  if (lu) {
    const int W = sl.T - s, cpr = (W + kStrip - 1) / kStrip;
    t = s + 1 + l / cpr;
    j0 = (l % cpr) * kStrip;
    count = min(kStrip, W - j0);
    return;
  }
  t = s + 1;
  for (;;) {
    const int len = (t < sl.T) ? (t - s + 1) : (sl.T - s);
    const int ch = (len + kStrip - 1) / kStrip;
    if (l < ch) {
      j0 = l * kStrip;
      count = min(kStrip, len - j0);
      return;
    }
    l -= ch;
    ++t;
  }
}

// ---------------------------------------------------------------------------
// Kernels
// ---------------------------------------------------------------------------




// Fills one 64 x 64 tile of an augmented matrix.
__global__ void __launch_bounds__(256)
    k_assemble(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre, int cnt,
               int lu) {
  __shared__ double rx[TB], ry[TB], rz[TB], cx[TB], cy[TB], cz[TB];
  const int q = find_slot(pre, cnt, blockIdx.x);
  const BigSlot sl = slots[q];
  struct {
    int ti, tj;
  } it;
  decode_assemble(lu != 0, sl, blockIdx.x - pre[q], it.ti, it.tj);
  const int tid = threadIdx.x;
  double *tile = a.W + sl.base + int64_t(it.ti) * TB * sl.ld + int64_t(it.tj) * TB;
  if (it.tj == sl.T) {  // residual columns: zero (the polynomial pass writes r)
    for (int e = tid; e < TB * TB; e += blockDim.x) tile[int64_t(e >> 6) * sl.ld + (e & 63)] = 0.0;
    return;
  }
  const bool erow = it.ti >= sl.T;
  const int64_t s0 = a.soff[sl.k], t0 = a.toff[sl.k];
  if (tid < TB) {
    const int gi = (erow ? it.ti - sl.T : it.ti) * TB + tid;
    double4 p = make_double4(0, 0, 0, 0);
    if (erow ? gi < sl.m : gi < sl.n) p = erow ? a.tgt[a.tidx[t0 + gi]] : a.src[a.sidx[s0 + gi]];
    rx[tid] = p.x;
    ry[tid] = p.y;
    rz[tid] = p.z;
  } else if (tid < 2 * TB) {
    const int gj = it.tj * TB + (tid - TB);
    double4 p = make_double4(0, 0, 0, 0);
    if (gj < sl.n) p = a.src[a.sidx[s0 + gj]];
    cx[tid - TB] = p.x;
    cy[tid - TB] = p.y;
    cz[tid - TB] = p.z;
  }
  __syncthreads();
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    const int gi = it.ti * TB + r, gj = it.tj * TB + c;
    double v;
    if (!erow) {
      if (gi < sl.n && gj < sl.n)
        v = wendland<double>(a.basis, __dsqrt_rn(sqdist3(rx[r], ry[r], rz[r], cx[c], cy[c], cz[c])),
                             a.rinv);
      else
        v = (gi == gj) ? 1.0 : 0.0;
    } else {
      const int ie = gi - sl.T * TB;
      v = (ie < sl.m && gj < sl.n)
              ? wendland<double>(a.basis,
                                 __dsqrt_rn(sqdist3(rx[r], ry[r], rz[r], cx[c], cy[c], cz[c])),
                                 a.rinv)
              : 0.0;
    }
    tile[int64_t(r) * sl.ld + c] = v;
  }
}

// Polynomial block and residual columns of one large patch (CTA per slot).
__global__ void __launch_bounds__(256) k_big_poly(BigArgs a, const BigSlot *__restrict__ slots) {
  __shared__ double red[8][kRedVals];
  __shared__ double redf[kRedVals];
  __shared__ double beta_s[4 * kMaxF];
  __shared__ int act_s[3];
  const BigSlot sl = slots[blockIdx.x];
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int F = a.F, n = sl.n;
  const int64_t s0 = a.soff[sl.k];
  const double4 c = a.centers[sl.k];
  const double shift[3] = {c.x, c.y, c.z};
  double acc[kRedVals - 6];
#pragma unroll
  for (int v = 0; v < kRedVals - 6; ++v) acc[v] = 0.0;
  double mn[3] = {INFINITY, INFINITY, INFINITY}, mx[3] = {-INFINITY, -INFINITY, -INFINITY};
  const int Fm = (a.mode == kBigAdjoint) ? 0 : F;
  const int nred = 10 + 4 * Fm;
  for (int i = tid; i < n; i += blockDim.x) {
    const int id = a.sidx[s0 + i];
    const double4 p = a.src[id];
    const double q[4] = {1.0, p.x - shift[0], p.y - shift[1], p.z - shift[2]};
    acc[0] += 1.0;
    acc[1] += q[1];
    acc[2] += q[2];
    acc[3] += q[3];
    acc[4] += q[1] * q[1];
    acc[5] += q[1] * q[2];
    acc[6] += q[1] * q[3];
    acc[7] += q[2] * q[2];
    acc[8] += q[2] * q[3];
    acc[9] += q[3] * q[3];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f)
      if (f < Fm) {
        const double b = a.vals[int64_t(id) * F + f];
#pragma unroll
        for (int cc = 0; cc < 4; ++cc) acc[10 + 4 * f + cc] += q[cc] * b;
      }
    const double pc[3] = {p.x, p.y, p.z};
#pragma unroll
    for (int d = 0; d < 3; ++d) {
      mn[d] = fmin(mn[d], pc[d]);
      mx[d] = fmax(mx[d], pc[d]);
    }
  }
#pragma unroll
  for (int v = 0; v < kRedVals - 6; ++v) {
    const double s = warp_sum(acc[v]);
    if (lane == 0 && v < nred) red[warp][v] = s;
  }
#pragma unroll
  for (int d = 0; d < 3; ++d) {
    double lo = mn[d], hi = mx[d];
    for (int o = 16; o > 0; o >>= 1) {
      lo = fmin(lo, __shfl_xor_sync(0xffffffffu, lo, o));
      hi = fmax(hi, __shfl_xor_sync(0xffffffffu, hi, o));
    }
    if (lane == 0) {
      red[warp][nred + d] = lo;
      red[warp][nred + 3 + d] = hi;
    }
  }
  __syncthreads();
  if (tid < nred + 6) {
    double s;
    if (tid < nred) {
      s = 0.0;
      for (int w = 0; w < 8; ++w) s += red[w][tid];
    } else if (tid < nred + 3) {
      s = INFINITY;
      for (int w = 0; w < 8; ++w) s = fmin(s, red[w][tid]);
    } else {
      s = -INFINITY;
      for (int w = 0; w < 8; ++w) s = fmax(s, red[w][tid]);
    }
    redf[tid] = s;
  }
  __syncthreads();
  {  // the padding rows of the residual column are zero (there is no assembly pass for it)
    double *rc = a.W + sl.base + int64_t(sl.T) * TB;
    for (int e = tid; e < (sl.T * TB - n) * F; e += blockDim.x)
      rc[int64_t(n + e / F) * sl.ld + e % F] = 0.0;
  }
  if (a.mode == kBigAdjoint) {
    if (tid < nred + 6) a.red_out[int64_t(sl.q) * kRedVals + tid] = redf[tid];
    return;
  }
  if (tid == 0) {
    int act[3];
    const int dropped = poly_block(redf, F, a.dim, shift, beta_s, act);
    for (int d = 0; d < 3; ++d) act_s[d] = act[d];
    a.status[sl.k] = dropped ? 1 : 0;
    for (int v = 0; v < 4 * kMaxF; ++v) a.beta[sl.q * 4 * kMaxF + v] = beta_s[v];
    for (int d = 0; d < 3; ++d) a.act[sl.q * 3 + d] = act[d];
    if (a.mode == kBigForwardSave) {
      for (int v = 0; v < 4 * kMaxF; ++v) a.beta_out[int64_t(sl.k) * 4 * kMaxF + v] = beta_s[v];
      for (int d = 0; d < 3; ++d) a.act_out[int64_t(sl.k) * 3 + d] = act[d];
    }
  }
  __syncthreads();
  double *rcol = a.W + sl.base + int64_t(sl.T) * TB;
  for (int i = tid; i < n; i += blockDim.x) {
    const int id = a.sidx[s0 + i];
    const double4 p = a.src[id];
    const double pc[3] = {p.x, p.y, p.z};
    for (int f = 0; f < F; ++f) {
      double t = beta_s[4 * f];
      for (int j = 0; j < 3; ++j)
        if (act_s[j] >= 0) t = __fma_rn(pc[act_s[j]], beta_s[4 * f + 1 + j], t);
      rcol[int64_t(i) * sl.ld + f] = a.vals[int64_t(id) * F + f] - t;
    }
  }
}

// Factors diagonal tile (s, s) of each listed slot in place: unpivoted LU
// (unit lower L below the diagonal, U on and above it) or Cholesky.
template <bool LU>
__global__ void __launch_bounds__(256) k_diag(BigArgs a, const BigSlot *__restrict__ slots, int s) {
  extern __shared__ double sm[];
  double *T = sm;                 // the tile
  __shared__ double piv;
  __shared__ int bad;
  const int slot = blockIdx.x;
  const BigSlot sl = slots[slot];
  const int tid = threadIdx.x;
  double *g = a.W + sl.base + int64_t(s) * TB * sl.ld + int64_t(s) * TB;
  load_tile(T, g, sl.ld, tid, blockDim.x);
  if (tid == 0) bad = 0;
  __syncthreads();
  for (int p = 0; p < TB; ++p) {
    if (LU) {
      const double d = T[p * LDS + p];
      for (int i = p + 1 + tid; i < TB; i += blockDim.x) T[i * LDS + p] /= d;
      __syncthreads();
      const int w = TB - 1 - p;
      for (int e = tid; e < w * w; e += blockDim.x) {
        const int i = p + 1 + e / w, j = p + 1 + e % w;
        T[i * LDS + j] = __fma_rn(-T[i * LDS + p], T[p * LDS + j], T[i * LDS + j]);
      }
      __syncthreads();
    } else {
      if (tid == 0) {
        const double app = T[p * LDS + p];
        if (!(app > 0.0)) bad = 1;
        piv = sqrt(app);
      }
      __syncthreads();
      const double d = piv;
      for (int i = p + tid; i < TB; i += blockDim.x) T[i * LDS + p] = (i == p) ? d : T[i * LDS + p] / d;
      __syncthreads();
      const int w = TB - 1 - p;
      for (int e = tid; e < w * w; e += blockDim.x) {
        const int i = p + 1 + e / w, j = p + 1 + e % w;
        if (j <= i) T[i * LDS + j] = __fma_rn(-T[i * LDS + p], T[j * LDS + p], T[i * LDS + j]);
      }
      __syncthreads();
    }
  }
  // The factors go back to the workspace, where the panel solves (k_trsm)
  // and the backward sweep read them.
  for (int idx = tid; idx < TB * TB / 2; idx += blockDim.x) {
    const int r = idx >> 5, c2 = idx & 31;
    *reinterpret_cast<double2 *>(g + int64_t(r) * sl.ld + 2 * c2) =
        *reinterpret_cast<const double2 *>(T + r * LDS + 2 * c2);
  }
  if (tid == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

__device__ __forceinline__ void load_inv(double *s, const double *g, int tid, int nt) {
  for (int idx = tid; idx < TB * TB / 2; idx += nt) {
    const int r = idx >> 5, c2 = idx & 31;
    *reinterpret_cast<double2 *>(s + r * LDS + 2 * c2) =
        *reinterpret_cast<const double2 *>(g + r * TB + 2 * c2);
  }
}

// Panel tiles of step s: row panel X := L^{-1} X (ti == s), column panel
// X := X U^{-1} (LU) or X := X L^{-T} (Cholesky), by triangular solves with
// the factors of the diagonal tile (s, s) as k_diag left them in the
// workspace (unit lower L below the diagonal, U on and above it, or the
// Cholesky factor below and on it): backward stable, unlike a product with
// the explicit inverse, whose error grows with the condition number of the
// diagonal tile.  Each of the 8 warps solves 8 rows of X (column panel) or 8
// columns (row panel, as rows of X^T against L^T) with warp_row_solve.
template <bool LU>
__global__ void __launch_bounds__(256)
    k_trsm(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre, int cnt,
           int s) {
  extern __shared__ double sm[];
  __shared__ double dinv[TB];
  double *sX = sm, *sU = sm + TB * LDS;
  const int q = find_slot(pre, cnt, blockIdx.x);
  const BigSlot sl = slots[q];
  struct {
    int slot, ti, tj;
  } it;
  it.slot = q;
  decode_trsm(LU, sl, s, blockIdx.x - pre[q], it.ti, it.tj);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double *X = a.W + sl.base + int64_t(it.ti) * TB * sl.ld + int64_t(it.tj) * TB;
  const double *D = a.W + sl.base + int64_t(s) * TB * sl.ld + int64_t(s) * TB;
  const bool left = it.ti == s;
  load_tile(sX, X, sl.ld, tid, blockDim.x);
  // The upper triangular operand of x U = c: U itself (LU column panel), or
  // the transpose of the lower factor (row panel: unit L; Cholesky: L).
  for (int e = tid; e < TB * TB; e += blockDim.x) {
    const int r = e >> 6, c = e & 63;
    const double v = D[int64_t(r) * sl.ld + c];
    if (LU && !left) sU[r * LDS + c] = c >= r ? v : 0.0;
    else if (LU) sU[c * LDS + r] = r > c ? v : (r == c ? 1.0 : 0.0);
    else sU[c * LDS + r] = r >= c ? v : 0.0;
  }
  __syncthreads();
  if (tid < TB) dinv[tid] = (LU && left) ? 1.0 : 1.0 / sU[tid * LDS + tid];
  __syncthreads();
  {
    const int r0 = 8 * warp;
    double lo[8], hi[8];
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) {
      lo[qq] = left ? sX[lane * LDS + r0 + qq] : sX[(r0 + qq) * LDS + lane];
      hi[qq] = left ? sX[(lane + 32) * LDS + r0 + qq] : sX[(r0 + qq) * LDS + 32 + lane];
    }
    warp_row_solve<8>(lo, hi, sU, dinv, lane);
#pragma unroll
    for (int qq = 0; qq < 8; ++qq) {
      if (left) {
        sX[lane * LDS + r0 + qq] = lo[qq];
        sX[(lane + 32) * LDS + r0 + qq] = hi[qq];
      } else {
        sX[(r0 + qq) * LDS + lane] = lo[qq];
        sX[(r0 + qq) * LDS + 32 + lane] = hi[qq];
      }
    }
  }
  __syncthreads();
  for (int idx = tid; idx < TB * TB / 2; idx += blockDim.x) {
    const int r = idx >> 5, c2 = idx & 31;
    *reinterpret_cast<double2 *>(X + int64_t(r) * sl.ld + 2 * c2) =
        *reinterpret_cast<const double2 *>(sX + r * LDS + 2 * c2);
  }
}

template <bool LU>
__global__ void __launch_bounds__(128, 2)
    k_update_strip(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre,
                   int cnt, int s) {
  extern __shared__ double sm[];
  double *sA = sm;
  double *sB[2] = {sm + TB * LDS, sm + 2 * TB * LDS};
  const int q = find_slot(pre, cnt, blockIdx.x);
  const BigSlot sl = slots[q];
  int t, j0, count;
  decode_strip(LU, sl, s, blockIdx.x - pre[q], t, j0, count);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  double *base = a.W + sl.base;
  const int ld = sl.ld;
  const int ncol = LU ? sl.T - s : ((t < sl.T) ? (t - s) : (sl.T - s - 1));
  auto column = [&](int j) { return LU ? s + 1 + j : (j < ncol ? s + 1 + j : sl.T); };
  auto bsrc = [&](int u) -> const double * {
    const bool bt = !LU && u < sl.T;
    return bt ? base + int64_t(u) * TB * ld + int64_t(s) * TB
              : base + int64_t(s) * TB * ld + int64_t(u) * TB;
  };
  async_tile(sA, base + int64_t(t) * TB * ld + int64_t(s) * TB, ld, tid, blockDim.x);
  async_tile(sB[0], bsrc(column(j0)), ld, tid, blockDim.x);
  cp_async_commit();
  for (int jj = 0; jj < count; ++jj) {
    const int u = column(j0 + jj);
    if (jj + 1 < count) {
      async_tile(sB[(jj + 1) & 1], bsrc(column(j0 + jj + 1)), ld, tid, blockDim.x);
      cp_async_commit();
    }
    double *C = base + int64_t(t) * TB * ld + int64_t(u) * TB;
    double acc[4][4][2];
    acc_load(acc, C, ld, wr, wc, lane);
    if (jj + 1 < count) cp_async_wait<1>();
    else cp_async_wait<0>();
    __syncthreads();
    if (!LU && u < sl.T) mma64<false, true>(sA, sB[jj & 1], acc, -1.0, wr, wc, lane);
    else mma64<false, false>(sA, sB[jj & 1], acc, -1.0, wr, wc, lane);
    acc_store(acc, C, ld, wr, wc, lane);
    __syncthreads();
  }
}

// local = V beta - S (S = -E alpha from the Schur complement).
__global__ void k_big_finish(BigArgs a, const BigSlot *__restrict__ slots) {
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F;
  const int64_t t0 = a.toff[sl.k];
  const double *beta = a.beta + sl.q * 4 * kMaxF;
  const int *act = a.act + sl.q * 3;
  const double *S = a.W + sl.base + int64_t(sl.T) * TB * sl.ld + int64_t(sl.T) * TB;
  int bad = 0;
  for (int i = threadIdx.x; i < sl.m; i += blockDim.x) {
    const double4 y = a.tgt[a.tidx[t0 + i]];
    const double yc[3] = {y.x, y.y, y.z};
    for (int f = 0; f < F; ++f) {
      double v = beta[4 * f];
      for (int j = 0; j < 3; ++j)
        if (act[j] >= 0) v = __fma_rn(yc[act[j]], beta[4 * f + 1 + j], v);
      const double out = v - S[int64_t(i) * sl.ld + f];
      if (!isfinite(out)) bad = 1;
      a.local[(t0 + i) * F + f] = out;
    }
  }
  if (bad) atomicOr(&a.status[sl.k], 2);
}


// Adjoint right-hand sides c = E^T h of one slot, in its residual column.
__global__ void __launch_bounds__(256) k_big_adj_rhs(BigArgs a, const BigSlot *__restrict__ slots) {
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F;
  const int64_t s0 = a.soff[sl.k], t0 = a.toff[sl.k];
  double *rcol = a.W + sl.base + int64_t(sl.T) * TB;
  for (int j = threadIdx.x; j < sl.n; j += blockDim.x) {
    const double4 x = a.src[a.sidx[s0 + j]];
    double cs[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) cs[f] = 0.0;
    for (int i = 0; i < sl.m; ++i) {
      const double4 y = a.tgt[a.tidx[t0 + i]];
      const double ph =
          wendland<double>(a.basis, __dsqrt_rn(sqdist3(y.x, y.y, y.z, x.x, x.y, x.z)), a.rinv);
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) cs[f] = __fma_rn(ph, a.h[(t0 + i) * F + f], cs[f]);
    }
    for (int f = 0; f < F; ++f) rcol[int64_t(j) * sl.ld + f] = cs[f];
  }
}

// Backward sweep after the elimination: the residual column holds
// y = L^{-1} r; solves U z = y (LU) or L^T z = y (Cholesky) tile row by tile
// row from the last, in place.  In forward-save mode z (the RBF coefficients
// alpha) is also written per (patch, source).
template <bool LU>
__global__ void __launch_bounds__(256) k_back_sweep(BigArgs a, const BigSlot *__restrict__ slots) {
  __shared__ double tile[TB][TB + 1];
  __shared__ double zt[TB][kMaxF];
  __shared__ double acc[TB][kMaxF];
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ld = sl.ld;
  double *W = a.W + sl.base;
  double *rcol = W + int64_t(sl.T) * TB;
  for (int s = sl.T - 1; s >= 0; --s) {
    for (int e = tid; e < TB * F; e += blockDim.x) {
      const int r = e / F, f = e % F;
      acc[r][f] = rcol[int64_t(s * TB + r) * ld + f];
    }
    for (int t = s + 1; t < sl.T; ++t) {
      const double *g = LU ? W + int64_t(s) * TB * ld + int64_t(t) * TB
                           : W + int64_t(t) * TB * ld + int64_t(s) * TB;
      __syncthreads();
      for (int e = tid; e < TB * TB; e += blockDim.x) tile[e >> 6][e & 63] = g[int64_t(e >> 6) * ld + (e & 63)];
      for (int e = tid; e < TB * F; e += blockDim.x) {
        const int r = e / F, f = e % F;
        zt[r][f] = rcol[int64_t(t * TB + r) * ld + f];
      }
      __syncthreads();
      const int o = tid & 63;
      for (int f = tid >> 6; f < F; f += 4) {
        double sum = 0.0;
        for (int c = 0; c < TB; ++c) sum = __fma_rn(LU ? tile[o][c] : tile[c][o], zt[c][f], sum);
        acc[o][f] -= sum;
      }
    }
    __syncthreads();
    const double *gd = W + int64_t(s) * TB * ld + int64_t(s) * TB;
    for (int e = tid; e < TB * TB; e += blockDim.x) tile[e >> 6][e & 63] = gd[int64_t(e >> 6) * ld + (e & 63)];
    __syncthreads();
    if (warp < F) {
      const int f = warp;
      for (int i = TB - 1; i >= 0; --i) {
        double sum = 0.0;
        for (int j = i + 1 + lane; j < TB; j += 32) sum = __fma_rn(LU ? tile[i][j] : tile[j][i], acc[j][f], sum);
        sum = warp_sum(sum);
        if (lane == 0) acc[i][f] = (acc[i][f] - sum) / tile[i][i];
        __syncwarp();
      }
    }
    __syncthreads();
    for (int e = tid; e < TB * F; e += blockDim.x) {
      const int r = e / F, f = e % F;
      rcol[int64_t(s * TB + r) * ld + f] = acc[r][f];
      const int j = s * TB + r;
      if (a.mode == kBigForwardSave && j < sl.n) a.alpha_out[(a.soff[sl.k] + j) * F + f] = acc[r][f];
    }
    __syncthreads();
  }
}

// Adjoint result of one slot: g = z - Q' G'^{-1} (Q'^T z - V'^T h).
__global__ void __launch_bounds__(256) k_big_adj_finish(BigArgs a, const BigSlot *__restrict__ slots) {
  __shared__ double red[8][8];
  __shared__ double corr[4 * kMaxF];
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int64_t s0 = a.soff[sl.k], t0 = a.toff[sl.k];
  const double4 c = a.centers[sl.k];
  const double shift[3] = {c.x, c.y, c.z};
  __shared__ int S_s[4], pv_s;
  __shared__ double R_s[4][4];
  if (tid == 0) {
    const double *redf = a.red_out + int64_t(sl.q) * kRedVals;
    int S[4], pv;
    double R[4][4];
    poly_axes(redf, a.dim, shift, redf + 10, redf + 13, S, pv, R);
    for (int i = 0; i < 4; ++i) {
      S_s[i] = S[i];
      for (int j = 0; j < 4; ++j) R_s[i][j] = R[i][j];
    }
    pv_s = pv;
  }
  __syncthreads();
  for (int f = 0; f < F; ++f) {
    double u[4] = {0, 0, 0, 0}, v[4] = {0, 0, 0, 0};
    for (int j = tid; j < sl.n; j += blockDim.x) {
      const double4 x = a.src[a.sidx[s0 + j]];
      const double z = a.zc[sl.zoff + int64_t(j) * F + f];
      const double q[4] = {1.0, x.x - shift[0], x.y - shift[1], x.z - shift[2]};
      for (int c2 = 0; c2 < 4; ++c2) u[c2] += q[c2] * z;
    }
    for (int i = tid; i < sl.m; i += blockDim.x) {
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
        for (int w = 0; w < 8; ++w) {
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
  int bad = 0;
  for (int j = tid; j < sl.n; j += blockDim.x) {
    const double4 x = a.src[a.sidx[s0 + j]];
    const double q[4] = {1.0, x.x - shift[0], x.y - shift[1], x.z - shift[2]};
    for (int f = 0; f < F; ++f) {
      double g = a.zc[sl.zoff + int64_t(j) * F + f];
      for (int c2 = 0; c2 < 4; ++c2) g -= q[c2] * corr[4 * f + c2];
      if (!isfinite(g)) bad = 1;
      a.g_out[(s0 + j) * F + f] = g;
    }
  }
  if (bad) atomicOr(&a.status[sl.k], 2);
}

// ---------------------------------------------------------------------------
// Host orchestration
// ---------------------------------------------------------------------------

static size_t slot_doubles(int n, int m) {
  const int T = (n + TB - 1) / TB, TE = (m + TB - 1) / TB;
  return size_t(T + TE) * TB * size_t(T + 1) * TB;
}

static int64_t count_assemble(bool lu, const BigSlot &q) {
  return lu ? int64_t(q.T + q.TE) * (q.T + 1) : int64_t(q.T) * (q.T + 3) / 2 + int64_t(q.TE) * (q.T + 1);
}
static int64_t count_trsm(bool lu, const BigSlot &q, int s) {
  const int R = q.T + q.TE;
  return lu ? int64_t(q.T - s) + (R - s - 1) : int64_t(R - s);
}
static int64_t ceil_div(int64_t a, int64_t b) { return (a + b - 1) / b; }
// sum_{L=1}^{W} ceil(L / kStrip)
static int64_t strip_sum(int64_t W) {
  const int64_t qq = W / kStrip, r = W % kStrip;
  return kStrip * qq * (qq + 1) / 2 + r * (qq + 1);
}
static int64_t count_strips(bool lu, const BigSlot &q, int s) {
  const int64_t R = q.T + q.TE, W = q.T - s;
  return lu ? (R - s - 1) * ceil_div(W, kStrip) : (strip_sum(W) - 1) + int64_t(q.TE) * ceil_div(W, kStrip);
}

static void set_smem_attributes() {
  static bool done = false;
  if (done) return;
  const int s3 = 3 * TB * LDS * sizeof(double), s2 = 2 * TB * LDS * sizeof(double);
  PB_CUDA(cudaFuncSetAttribute(k_diag<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s3));
  PB_CUDA(cudaFuncSetAttribute(k_trsm<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, s2));
  PB_CUDA(cudaFuncSetAttribute(k_update_strip<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               3 * TB * LDS * int(sizeof(double))));
  done = true;
}

// Solves the listed patches (each with m > 0) with the blocked engine.  The
// launches are queued on p.stream without host synchronisation; the
// workspace of each wave is released stream-ordered after its kernels, so the
// next wave reuses it.
void destroy_factor_cache(FactorCache *c) { delete c; }

int pipeline_wait_limit() {
  if (const char *e = std::getenv("PACMAN_B200_WAIT_LIMIT")) {
    const long v = std::strtol(e, nullptr, 10);
    if (v >= 1) return int(std::min<long>(v, 1l << 30));
  }
  return 1 << 22;
}

void solve_big(Plan &p, int basis, const double *vals, int F, bool lu,
               const std::vector<int> &patches, double *local, int *status, SolveReport &rep,
               const BigExtra &extra, FactorCache *keep) {
  if (patches.empty()) return;
  cudaStream_t st = p.stream;
  set_smem_attributes();
  size_t free_b = 0, total_b = 0;
  PB_CUDA(cudaMemGetInfo(&free_b, &total_b));
  size_t budget = std::max<size_t>(size_t(1) << 30, size_t(double(free_b) * 0.6)) / 8;
  // Largest patches first: the slots active at step s are then a prefix.
  std::vector<int> order(patches);
  std::stable_sort(order.begin(), order.end(),
                   [&](int x, int y) { return p.n_host[x] > p.n_host[y]; });
  BigArgs a{};
  a.src = p.src4.as<double4>();
  a.tgt = p.tgt4.as<double4>();
  a.vals = vals;
  a.soff = p.soff.as<int64_t>();
  a.sidx = p.sidx.as<int>();
  a.toff = p.toff.as<int64_t>();
  a.tidx = p.tidx.as<int>();
  a.centers = p.centers.as<double4>();
  a.status = status;
  a.local = local;
  a.rinv = 1.0 / p.opts.support_radius;
  a.F = F;
  a.dim = p.dim;
  a.basis = basis;
  a.mode = extra.mode;
  a.alpha_out = extra.alpha_out;
  a.beta_out = extra.beta_out;
  a.act_out = extra.act_out;
  a.h = extra.h;
  a.g_out = extra.g_out;
  a.wait_limit = pipeline_wait_limit();
  const bool adjoint = extra.mode == kBigAdjoint;
  if (adjoint) lu = false;
  if (!lu) chol_set_smem_attributes();
  // The Cholesky forward path evaluates local = E alpha + V beta from alpha
  // per (patch, source): alpha_out when saving, else a scratch array.
  DevMem dalpha;
  if (!lu && !adjoint) {
    if (extra.alpha_out != nullptr) {
      a.alpha_c = extra.alpha_out;
    } else {
      dalpha.alloc(sizeof(double) * size_t(p.snnz) * size_t(F), st);
      a.alpha_c = dalpha.as<double>();
    }
  }
  // The forward Cholesky of precision "mixed" runs its column updates on the
  // int8 tensor cores (k_col_step_ws); PACMAN_B200_INT8=0 keeps them in FP64.
  const char *i8env = std::getenv("PACMAN_B200_INT8");
  const bool oz = !lu && !adjoint && !(i8env && std::atoi(i8env) == 0);
  if (oz) {
    // sigma bounds every |L[r][c]| <= sqrt(A_rr) = sqrt(phi(0)) (1 for the
    // identity padding), with margin for rounding and for d_1 <= 127.
    const double phi0 = basis == 0x12 ? 3.0 : (basis == 0x14 ? 15.0 : 1.0);
    const double sigma = std::sqrt(std::max(phi0, 1.0)) * (128.0 / 127.0) * (1.0 + std::ldexp(1.0, -20));
    a.oz_mul = 128.0 / sigma;
    a.oz_sig2 = sigma * sigma;
  }
  if (lu || adjoint) keep = nullptr;  // only the mixed forward keeps its factors
  HostArena &arena = HostArena::get();
  size_t pos = 0;
  while (pos < order.size()) {
    if (keep && pos > 0) {
      // Kept waves stay allocated: size the next one by what is left.
      PB_CUDA(host_sync(st));
      PB_CUDA(cudaMemGetInfo(&free_b, &total_b));
      budget = std::max<size_t>(size_t(1) << 28, size_t(double(free_b) * 0.6)) / 8;
    }
    // One wave: as many patches as fit the workspace budget.
    std::vector<BigSlot> slots;
    size_t tot = 0;
    int64_t tot_inv = 0, tot_z = 0, tot_sl = 0;
    while (pos < order.size()) {
      const int k = order[pos];
      const int n = p.n_host[k], m = p.m_host[k];
      const int Tn = (n + TB - 1) / TB;
      const size_t d = slot_doubles(n, lu ? m : 0);
      const size_t dsl_doubles = oz ? (oz_slot_bytes(Tn) + 7) / 8 : 0;
      if (!slots.empty() && tot + size_t(tot_sl) / 8 + d + dsl_doubles > budget) break;
      BigSlot q{};
      q.base = int64_t(tot);
      q.T = (n + TB - 1) / TB;
      q.TE = lu ? (m + TB - 1) / TB : 0;
      q.inv = lu ? int64_t(slots.size()) * 2 * TB * TB : tot_inv;
      q.q = int(slots.size());
      q.zoff = tot_z;
      // Kept factors serve later executes with any field count: room for kMaxF.
      tot_z += int64_t(q.T) * TB * (keep ? kMaxF : F);
      q.sli = tot_sl;
      if (oz) tot_sl += int64_t(oz_slot_bytes(q.T));
      tot_inv += int64_t(q.T) * TB * TB;
      q.ld = (q.T + 1) * TB;
      q.k = k;
      q.n = n;
      q.m = m;
      slots.push_back(q);
      tot += d;
      ++pos;
      const double nn = n;
      rep.factor_flops += (lu ? 2.0 / 3.0 : 1.0 / 3.0) * nn * nn * nn + 2.0 * nn * nn * F +
                          2.0 * double(m) * nn * F;
    }
    const int ns = int(slots.size());
    const int steps = slots.front().T;
    // Prefix counts: assembly over all slots, then per step the trsm and
    // update counts over the active slots (a prefix of the sorted slots).
    std::vector<int> pre_asm(ns + 1, 0);
    for (int q = 0; q < ns; ++q) {
      const int64_t v = pre_asm[q] + count_assemble(lu, slots[q]);
      if (v > 0x7fffffffll) throw Error{PACMAN_B200_ERR_LIMIT, "too many tiles in one launch"};
      pre_asm[q + 1] = int(v);
    }
    // LU: per step the trsm and update-strip prefix counts over the active
    // slots (a prefix of the sorted slots); Cholesky: per slot group below.
    std::vector<int> cnt(steps), off(steps + 1, 0), pre;
    if (lu) {
      pre.reserve(size_t(steps) * 2 * (ns + 1));
      for (int s = 0; s < steps; ++s) {
        int c = 0;
        while (c < ns && slots[c].T > s) ++c;
        cnt[s] = c;
        off[s] = int(pre.size());
        int64_t acc = 0;
        pre.push_back(0);
        for (int q = 0; q < c; ++q) pre.push_back(int(acc += count_trsm(lu, slots[q], s)));
        acc = 0;
        pre.push_back(0);
        for (int q = 0; q < c; ++q) {
          acc += count_strips(lu, slots[q], s);
          if (acc > 0x7fffffffll) throw Error{PACMAN_B200_ERR_LIMIT, "too many tiles in one launch"};
          pre.push_back(int(acc));
        }
      }
      off[steps] = int(pre.size());
    }
    DevMem dW, dsmall;
    dW.alloc(sizeof(double) * tot, st);
    DevMem dzc, dsl;
    if (!lu) {
      dzc.alloc(sizeof(double) * size_t(tot_z), st);
      a.zc = dzc.as<double>();
    }
    a.slices = nullptr;
    a.dpart = nullptr;
    DevMem ddiag;
    if (oz && tot_sl > 0) {
      dsl.alloc(size_t(tot_sl), st);
      a.slices = dsl.as<uint8_t>();
      // The int8 steps' next diagonal tile: D' (TB x TB per slot), written by
      // the step's diagonal item and factored by k_diag_next.
      ddiag.alloc(sizeof(double) * TB * TB * size_t(ns), st);
      a.dpart = ddiag.as<double>();
    }
    const size_t n_inv = lu ? size_t(2) * TB * TB * ns : size_t(tot_inv);
    const size_t n_beta = size_t(4) * kMaxF * ns;
    const size_t n_red = size_t(kRedVals) * ns;
    const size_t bytes_small = sizeof(double) * (n_inv + n_beta + n_red) + sizeof(int) * 3 * ns +
                               sizeof(BigSlot) * ns + sizeof(int) * (pre_asm.size() + pre.size()) +
                               64;
    dsmall.alloc(bytes_small, st);
    char *cur = dsmall.as<char>();
    auto take = [&](size_t bytes) {
      char *r = cur;
      cur += (bytes + 15) & ~size_t(15);
      return r;
    };
    a.W = dW.as<double>();
    a.inv = reinterpret_cast<double *>(take(sizeof(double) * n_inv));
    a.beta = reinterpret_cast<double *>(take(sizeof(double) * n_beta));
    a.act = reinterpret_cast<int *>(take(sizeof(int) * 3 * ns));
    a.red_out = reinterpret_cast<double *>(take(sizeof(double) * n_red));
    BigSlot *ds = reinterpret_cast<BigSlot *>(take(sizeof(BigSlot) * ns));
    int *dpre_asm = reinterpret_cast<int *>(take(sizeof(int) * pre_asm.size()));
    int *dpre = reinterpret_cast<int *>(take(sizeof(int) * pre.size()));
    arena.upload(slots.data(), slots.size(), ds, st);
    arena.upload(pre_asm.data(), pre_asm.size(), dpre_asm, st);
    arena.upload(pre.data(), pre.size(), dpre, st);
    if (!lu) {
      // Interleaved groups of slots, each stepping in lockstep on its own
      // stream: the short diagonal and trsm launches and the tails of one
      // group's column updates overlap the other groups' work.
      // The tuned group count (PACMAN_B200_GROUPS, 1..8, overrides it).
      int G = std::min<int>(AuxStreams::kDefaultGroups, std::max(1, ns / 8));
      const int gt = tuned_int("PACMAN_B200_GROUPS", tuning_for_current_device().groups);
      if (gt > 0) G = std::min<int>(AuxStreams::kN, std::min(gt, ns));
      std::vector<std::vector<BigSlot>> gs(G);
      for (int q = 0; q < ns; ++q) gs[q % G].push_back(slots[q]);
      std::vector<CholPlan> gp(G);
      std::vector<DevMem> gmem(G);
      std::vector<BigSlot *> gds(G);
      std::vector<int *> gpre(G);
      for (int g = 0; g < G; ++g) {
        gp[g] = chol_prefix(gs[g]);
        const int ng = int(gs[g].size());
        const size_t b0 = (sizeof(BigSlot) * ng + 15) & ~size_t(15);
        gmem[g].alloc(b0 + sizeof(int) * gp[g].pre.size() + 64, st);
        gds[g] = gmem[g].as<BigSlot>();
        gpre[g] = reinterpret_cast<int *>(gmem[g].as<char>() + b0);
        arena.upload(gs[g].data(), gs[g].size(), gds[g], st);
        arena.upload(gp[g].pre.data(), gp[g].pre.size(), gpre[g], st);
      }
      p.aux.make();
      PB_CUDA(cudaEventRecord(p.aux.ev[AuxStreams::kN], st));
      for (int g = 0; g < G; ++g) {
        cudaStream_t sg = p.aux.s[g];
        PB_CUDA(cudaStreamWaitEvent(sg, p.aux.ev[AuxStreams::kN], 0));
        // The Wendland tiles are evaluated inside the step kernels; here only
        // the polynomial block and the residual column.
        const int ng = int(gs[g].size());
        k_big_poly<<<ng, 256, 0, sg>>>(a, gds[g]);
        note_launch();
        if (adjoint) {
          k_big_adj_rhs<<<ng, 256, 0, sg>>>(a, gds[g]);
          note_launch();
        }
        chol_launch_steps(a, gds[g], gs[g], gp[g], gpre[g], sg, rep,
                          g == 0 ? rep.tail_event : nullptr);
        // Each group sweeps and evaluates as soon as its own steps end, so
        // the sweeps overlap the other groups' last steps.
        chol_launch_finish(a, gds[g], int(gs[g].size()), adjoint, sg);
        if (adjoint) {
          k_big_adj_finish<<<int(gs[g].size()), 256, 0, sg>>>(a, gds[g]);
          note_launch();
        }
        PB_CUDA(cudaEventRecord(p.aux.ev[g], sg));
        PB_CUDA(cudaStreamWaitEvent(st, p.aux.ev[g], 0));
      }
      PB_CUDA(cudaGetLastError());
      if (keep) {
        CholWaveCache w;
        w.W = std::move(dW);
        w.small = std::move(dsmall);
        w.inv = a.inv;
        w.beta = a.beta;
        w.act = a.act;
        w.red = a.red_out;
        w.ns = ns;
        for (const BigSlot &q : slots) w.sum_T += q.T;
        w.ds = ds;
        keep->waves.push_back(std::move(w));
      }
      continue;
    }
    k_assemble<<<pre_asm[ns], 256, 0, st>>>(a, ds, dpre_asm, ns, 1);
    note_launch();
    k_big_poly<<<ns, 256, 0, st>>>(a, ds);
    note_launch();
    const size_t s3 = 3 * TB * LDS * sizeof(double), s2 = 2 * TB * LDS * sizeof(double);
    for (int s = 0; s < steps; ++s) {
      const int c = cnt[s];
      const int *pt = dpre + off[s];
      const int *pu = pt + c + 1;
      const int nt = pre[off[s] + c];
      const int nu = pre[off[s] + c + 1 + c];
      k_diag<true><<<c, 256, s3, st>>>(a, ds, s);
      if (nt) k_trsm<true><<<nt, 256, s2, st>>>(a, ds, pt, c, s);
      if (nu) k_update_strip<true><<<nu, 128, s3, st>>>(a, ds, pu, c, s);
      note_launch(1 + (nt ? 1 : 0) + (nu ? 1 : 0));
    }
    k_big_finish<<<ns, 128, 0, st>>>(a, ds);
    note_launch();
    if (extra.mode == kBigForwardSave) {
      k_back_sweep<true><<<ns, 256, 0, st>>>(a, ds);
      note_launch();
    }
    PB_CUDA(cudaGetLastError());
  }
}

// Large patches from kept factorisations, one launch each over all slots of
// a wave (largest first): the polynomial block and residual column
// (k_big_poly), the forward sweep from the kept tiles (k_chol_fwd), the
// backward sweep and the evaluation.
void solve_big_cached(Plan &p, FactorCache &c, int basis, const double *vals, int F,
                      double *local, int *status, SolveReport &rep, const BigExtra &extra) {
  if (c.waves.empty()) return;
  cudaStream_t st = p.stream;
  chol_set_smem_attributes();
  BigArgs a{};
  a.src = p.src4.as<double4>();
  a.tgt = p.tgt4.as<double4>();
  a.vals = vals;
  a.soff = p.soff.as<int64_t>();
  a.sidx = p.sidx.as<int>();
  a.toff = p.toff.as<int64_t>();
  a.tidx = p.tidx.as<int>();
  a.centers = p.centers.as<double4>();
  a.status = status;
  a.local = local;
  a.rinv = 1.0 / p.opts.support_radius;
  a.F = F;
  a.dim = p.dim;
  a.basis = basis;
  a.mode = extra.mode;
  a.alpha_out = extra.alpha_out;
  a.beta_out = extra.beta_out;
  a.act_out = extra.act_out;
  a.wait_limit = pipeline_wait_limit();
  DevMem dalpha;
  if (extra.alpha_out != nullptr) {
    a.alpha_c = extra.alpha_out;
  } else {
    dalpha.alloc(sizeof(double) * size_t(std::max<int64_t>(p.snnz, 1)) * size_t(F), st);
    a.alpha_c = dalpha.as<double>();
  }
  p.aux.make();
  for (CholWaveCache &w : c.waves) {
    DevMem dzc;
    dzc.alloc(sizeof(double) * size_t(w.sum_T) * TB * kMaxF, st);  // slot offsets for kMaxF
    a.zc = dzc.as<double>();
    a.W = w.W.as<double>();
    a.inv = w.inv;
    a.beta = w.beta;
    a.act = w.act;
    a.red_out = w.red;
    a.slices = nullptr;
    // On the high-priority stream, ahead of the small patches' kernel.
    cudaStream_t hs = p.aux.s[0];
    PB_CUDA(cudaEventRecord(p.aux.ev[AuxStreams::kN], st));
    PB_CUDA(cudaStreamWaitEvent(hs, p.aux.ev[AuxStreams::kN], 0));
    k_big_poly<<<w.ns, 256, 0, hs>>>(a, w.ds);
    note_launch();
    chol_launch_forward(a, w.ds, w.ns, hs);
    chol_launch_finish(a, w.ds, w.ns, false, hs);
    PB_CUDA(cudaEventRecord(p.aux.ev[0], hs));
    PB_CUDA(cudaStreamWaitEvent(st, p.aux.ev[0], 0));
    PB_CUDA(cudaGetLastError());
    rep.factors_reused += w.ns;
  }
}

}  // namespace pacman_b200
