// Left-looking blocked Cholesky for the large patches of the B200 RBF-PUM
// transfer (precision "mixed" and the adjoint).
//
// The reference factors each patch matrix with an unpivoted LU in one GPU
// thread (src/rbf_pum/solver/solver.hpp:422-490, KokkosBatched
// SerialLU<Unblocked>).  A is symmetric positive definite, so here it is
// factored as L L^T in 64 x 64 tiles, all large patches in lockstep, one tile
// column j per step and one launch per step (k_col_step):
//   C[i, j] = A[i, j] - sum_{p<j} L[i, p] L[j, p]^T for every i > j, with the
//   accumulator in registers for the whole K loop and the L panels streaming
//   through a cp.async pipeline; then L[i, j] = C X_j^T (X_j = L[j, j]^{-1},
//   formed one step earlier) and the forward substitution r_i -= L[i, j] y_j;
//   the CTA of row tile j + 1 also forms, factors and inverts the next
//   diagonal tile (X_{j+1}, y_{j+1} = X_{j+1} r_{j+1}).
// k_diag_chol does the diagonal tile of step 0.  Afterwards k_chol_back solves
// L^T alpha = y (with the kept tile inverses) and k_chol_eval evaluates
// local = E alpha + V beta (solver.hpp:270-273).  The tile products run on
// the FP64 tensor cores (mma.sync m8n8k4 f64).
#include <algorithm>
#include <cmath>
#include <vector>

#include "blocked.cuh"

namespace pacman_b200 {

constexpr int kKC = 32;                 // K chunk of the column update (doubles)
constexpr int kKLD = kKC + 4;           // shared row stride of a chunk: conflict-free fragments
constexpr int kStages = 2;              // cp.async pipeline depth (2 CTAs per SM)
constexpr int kColRows = 2 * TB;        // rows of one column-update CTA (two tiles)
constexpr int kColThreads = 256;
constexpr int kColStage = (kColRows + TB) * kKLD;  // doubles per pipeline stage
constexpr size_t kColSmem = size_t(kStages) * kColStage * sizeof(double);
constexpr size_t kDiagSmem = size_t(TB) * LDS * sizeof(double);

// acc += A B^T over one K chunk: A rows wr.., B rows wc.. (both K-contiguous).
__device__ __forceinline__ void mma_chunk_nt(const double *__restrict__ sA,
                                             const double *__restrict__ sB,
                                             double (&acc)[4][4][2], int wr, int wc, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int k0 = 0; k0 < kKC; k0 += 4) {
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) a[i] = sA[(wr + 8 * i + g) * kKLD + k0 + t];
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) b[jj] = sB[(wc + 8 * jj + g) * kKLD + k0 + t];
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) dmma(acc[i][jj][0], acc[i][jj][1], a[i], b[jj]);
  }
}

__device__ __forceinline__ void acc_neg(double (&acc)[4][4][2]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = -acc[i][jj][0], acc[i][jj][1] = -acc[i][jj][1];
}

// Inverse Cholesky factor X of one 64 x 64 tile D and y = X r (256 threads).  The tile is eliminated as L D L^T with the identity carried
// along (Gauss-Jordan on [A | I]): at pivot p every row i > p gets
// R_i -= (a_ip / a_pp) R_p, which leaves U = D L^T on the left and L^{-1} on
// the right.  Each thread owns a 4 x 4 block of registers; slot (i, s) holds
// A[i][s] until pivot s and L^{-1}[i][s] afterwards.  Per pivot the owners
// publish one vector (row p of L^{-1} left of the pivot, the pivot, column p
// of A below it) and all threads update their slots: one barrier per pivot.
// Only X = L_c^{-1} = D^{-1/2} L^{-1} is kept (the trsm, the forward and the
// backward substitution use nothing else).  Non-positive pivots set status 4.
// D: lower part at g (row stride ld, global or shared); r: the first F
// columns of the residual tile at rg (row stride rld), overwritten with y; X
// goes to gi (row stride TB).  Xs (TB x LDS), cv, dis and ys are shared
// scratch.  Returns true on a non-positive pivot.
__device__ bool diag_tile(const double *g, int ld, double *rg, int rld, int F, double *gi,
                          double *Xs,
                          double (*cv)[TB], double *dis, double (*ys)[kMaxF]) {
  const int tid = threadIdx.x;
  const int bi = tid >> 4, bs = tid & 15;
  bool bad = false;
  double v[4][4];
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const double2 lo = *reinterpret_cast<const double2 *>(g + int64_t(4 * bi + r) * ld + 4 * bs);
    const double2 hi = *reinterpret_cast<const double2 *>(g + int64_t(4 * bi + r) * ld + 4 * bs + 2);
    v[r][0] = lo.x;
    v[r][1] = lo.y;
    v[r][2] = hi.x;
    v[r][3] = hi.y;
  }
  for (int e = tid; e < TB * kMaxF; e += 256) {
    const int r = e / kMaxF, f = e % kMaxF;
    ys[r][f] = f < F ? rg[int64_t(r) * rld + f] : 0.0;
  }
  for (int p = 0; p < TB; ++p) {
    double *c = cv[p & 1];
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
    if (bs == pb) {  // column p below the pivot: A[i][p], i > p
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
    __syncthreads();
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
        const double m = c[i] * inv;
#pragma unroll
        for (int b = 0; b < 4; ++b) {
          const int sc = 4 * bs + b;
          if (sc == p) v[r][b] = -m;
          else if (sc <= i) v[r][b] = __fma_rn(-m, cs[b], v[r][b]);
        }
      }
    }
  }
  // X[i][s] = L^{-1}[i][s] / sqrt(d_i); d_i is the final diagonal slot.
  if (bi == bs) {
#pragma unroll
    for (int r = 0; r < 4; ++r) dis[4 * bi + r] = 1.0 / sqrt(v[r][r]);
  }
  __syncthreads();
#pragma unroll
  for (int r = 0; r < 4; ++r) {
    const int i = 4 * bi + r;
    const double di = dis[i];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int sc = 4 * bs + b;
      Xs[i * LDS + sc] = sc < i ? v[r][b] * di : (sc == i ? di : 0.0);
    }
  }
  __syncthreads();
  // y_j = X r_j (first F columns of the residual tile).
  double yv[2];
  int ny = 0;
  for (int e = tid; e < TB * F; e += 256) {
    const int r = e / F, f = e % F;
    double s = 0.0;
    for (int k = 0; k <= r; ++k) s = __fma_rn(Xs[r * LDS + k], ys[k][f], s);
    yv[ny++] = s;
  }
  ny = 0;
  for (int e = tid; e < TB * F; e += 256) rg[int64_t(e / F) * rld + e % F] = yv[ny++];
  for (int idx = tid; idx < TB * TB / 2; idx += 256) {
    const int r = idx >> 5, c2 = idx & 31;
    *reinterpret_cast<double2 *>(gi + r * TB + 2 * c2) =
        *reinterpret_cast<const double2 *>(Xs + r * LDS + 2 * c2);
  }
  return bad;
}

// The diagonal tile of step 0 of every slot.
__global__ void __launch_bounds__(256, 4) k_diag_chol(BigArgs a, const BigSlot *__restrict__ slots,
                                                      int j) {
  extern __shared__ double sm[];
  __shared__ double cv[2][TB];
  __shared__ double dis[TB];
  __shared__ double ys[TB][kMaxF];
  const BigSlot sl = slots[blockIdx.x];
  const int ld = sl.ld;
  const double *g = a.W + sl.base + int64_t(j) * TB * ld + int64_t(j) * TB;
  double *rg = a.W + sl.base + int64_t(j) * TB * ld + int64_t(sl.T) * TB;
  const bool bad =
      diag_tile(g, ld, rg, ld, a.F, a.inv + sl.inv + int64_t(j) * TB * TB, sm, cv, dis, ys);
  if (threadIdx.x == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// Step j of the factorisation, one launch over all slots with T > j + 1.
// CTA l of a slot owns row tiles i0 = j + 1 + 2l and i0 + 1 of tile column j:
//  1. C = A[i, j] - sum_{p<j} L[i, p] L[j, p]^T: eight warps hold 32 x 32
//     accumulators (starting at -A) for the whole K loop, the L panels stream
//     through a cp.async pipeline;
//  2. L[i, j] = C X_j^T, the triangular solve with the inverse factor of the
//     diagonal tile (made one step earlier), stored; then the forward
//     substitution r_i -= L[i, j] y_j from the accumulator registers;
//  3. CTA 0 (i0 = j + 1) forms the next diagonal tile
//     D = A[j+1, j+1] - sum_{p<=j} L[j+1, p] L[j+1, p]^T and factors it:
//     X_{j+1} and y_{j+1} = X_{j+1} r_{j+1} for step j + 1.
__global__ void __launch_bounds__(kColThreads, 2)
    k_col_step(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre, int cnt,
               int j) {
  extern __shared__ double sm[];
  // The first cnt CTAs are the slots' CTA 0 (the longest: they also form the
  // next diagonal tile), so they start in the first wave; the other CTAs
  // (l >= 1) follow, addressed through the prefix counts.
  int q, l;
  if (int(blockIdx.x) < cnt) {
    q = blockIdx.x;
    l = 0;
  } else {
    const int b = blockIdx.x - cnt;
    q = find_slot(pre, cnt, b);
    l = 1 + b - pre[q];
  }
  const BigSlot sl = slots[q];
  const int i0 = j + 1 + 2 * l;
  const bool two = i0 + 1 < sl.T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int g = lane >> 2, t = lane & 3;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int ld = sl.ld, F = a.F;
  double *W = a.W + sl.base;
  double *rcol = W + int64_t(sl.T) * TB;
  const double *gA = W + int64_t(i0) * TB * ld;
  const double *gB = W + int64_t(j) * TB * ld;
  const int arows = two ? kColRows : TB;
  const int nch = j * (TB / kKC);
  auto load = [&](int c, int stage) {
    double *sA = sm + stage * kColStage;
    double *sB = sA + kColRows * kKLD;
    const int col = c * kKC;
    for (int idx = tid; idx < (kColRows + TB) * (kKC / 2); idx += kColThreads) {
      const int r = idx / (kKC / 2), c2 = idx % (kKC / 2);
      if (r < kColRows) {
        if (r < arows) cp_async16(sA + r * kKLD + 2 * c2, gA + int64_t(r) * ld + col + 2 * c2);
      } else {
        const int rb = r - kColRows;
        cp_async16(sB + rb * kKLD + 2 * c2, gB + int64_t(rb) * ld + col + 2 * c2);
      }
    }
  };
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nch) load(s, s);
    cp_async_commit();
  }
  const bool active = two || wr < TB;
  double *C = W + int64_t(i0) * TB * ld + int64_t(j) * TB;
  double acc[4][4][2];
  if (active) {
    acc_load(acc, C, ld, wr, wc, lane);
    acc_neg(acc);
  }
  for (int c = 0; c < nch; ++c) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    if (c + kStages - 1 < nch) load(c + kStages - 1, (c + kStages - 1) % kStages);
    cp_async_commit();
    if (active) {
      const double *sA = sm + (c % kStages) * kColStage;
      mma_chunk_nt(sA, sA + kColRows * kKLD, acc, wr, wc, lane);
    }
  }
  cp_async_wait<0>();
  __syncthreads();

  // 2. L[i, j] = C X_j^T through shared memory.
  double *sC = sm;                   // kColRows x LDS
  double *sX = sm + kColRows * LDS;  // TB x LDS
  {
    const double *xg = a.inv + sl.inv + int64_t(j) * TB * TB;
    for (int idx = tid; idx < TB * TB / 2; idx += kColThreads) {
      const int r = idx >> 5, c2 = idx & 31;
      cp_async16(sX + r * LDS + 2 * c2, xg + r * TB + 2 * c2);
    }
    cp_async_commit();
  }
  if (active) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<double2 *>(sC + (wr + 8 * i + g) * LDS + wc + 8 * jj + 2 * t) =
            make_double2(-acc[i][jj][0], -acc[i][jj][1]);
  }
  cp_async_wait<0>();
  __syncthreads();
  acc_zero(acc);
  if (active) {
    mma64<false, true>(sC, sX, acc, 1.0, wr, wc, lane);
    acc_store(acc, C, ld, wr, wc, lane);
  }
  __syncthreads();  // sC and sX are free
  double *ysh = sm;               // TB x kMaxF
  double *red = sm + TB * kMaxF;  // 2 x kColRows x kMaxF
  {
    const double *yg = rcol + int64_t(j) * TB * ld;
    for (int e = tid; e < TB * kMaxF; e += kColThreads) {
      const int r = e / kMaxF, f = e % kMaxF;
      ysh[e] = f < F ? yg[int64_t(r) * ld + f] : 0.0;
    }
  }
  __syncthreads();
  for (int f = 0; f < F; ++f) {
    double pr[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      double s = 0.0;
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
#pragma unroll
        for (int h = 0; h < 2; ++h)
          s = __fma_rn(acc[i][jj][h], ysh[(wc + 8 * jj + 2 * t + h) * kMaxF + f], s);
      s += __shfl_xor_sync(0xffffffffu, s, 1);
      s += __shfl_xor_sync(0xffffffffu, s, 2);
      pr[i] = s;
    }
    if (t == 0 && active) {
#pragma unroll
      for (int i = 0; i < 4; ++i) red[((wc >> 5) * kColRows + wr + 8 * i + g) * kMaxF + f] = pr[i];
    }
  }
  __syncthreads();
  {
    double *rg = rcol + int64_t(i0) * TB * ld;
    for (int e = tid; e < arows * F; e += kColThreads) {
      const int r = e / F, f = e % F;
      rg[int64_t(r) * ld + f] -= red[r * kMaxF + f] + red[(kColRows + r) * kMaxF + f];
    }
  }
  if (l != 0) return;

  // 3. The diagonal tile of step j + 1 (this CTA's first row tile).
  __syncthreads();
  constexpr int kDStage = TB * kKLD;
  double *sL = sm + 2 * kDStage;  // L[j+1, j], TB x LDS
  if (wr < TB) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<double2 *>(sL + (wr + 8 * i + g) * LDS + wc + 8 * jj + 2 * t) =
            make_double2(acc[i][jj][0], acc[i][jj][1]);
  }
  auto loadd = [&](int c, int stage) {
    double *sD = sm + stage * kDStage;
    const int col = c * kKC;
    for (int idx = tid; idx < TB * (kKC / 2); idx += kColThreads) {
      const int r = idx / (kKC / 2), c2 = idx % (kKC / 2);
      cp_async16(sD + r * kKLD + 2 * c2, gA + int64_t(r) * ld + col + 2 * c2);
    }
  };
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nch) loadd(s, s);
    cp_async_commit();
  }
  const bool dact = wr < TB;
  double *Dg = W + int64_t(j + 1) * TB * ld + int64_t(j + 1) * TB;
  if (dact) {
    acc_load(acc, Dg, ld, wr, wc, lane);
    acc_neg(acc);
  }
  for (int c = 0; c < nch; ++c) {
    cp_async_wait<kStages - 2>();
    __syncthreads();
    if (c + kStages - 1 < nch) loadd(c + kStages - 1, (c + kStages - 1) % kStages);
    cp_async_commit();
    if (dact) {
      const double *sD = sm + (c % kStages) * kDStage;
      mma_chunk_nt(sD, sD, acc, wr, wc, lane);
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  if (dact) mma64<false, true>(sL, sL, acc, 1.0, wr, wc, lane);
  double *Ds = sm;  // TB x LDS, over the finished stages
  if (dact) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<double2 *>(Ds + (wr + 8 * i + g) * LDS + wc + 8 * jj + 2 * t) =
            make_double2(-acc[i][jj][0], -acc[i][jj][1]);
  }
  __syncthreads();
  // Scratch of the factorisation over the consumed L[j+1, j] (sL).
  double *Xs = sm + TB * LDS;
  double(*ysd)[kMaxF] = reinterpret_cast<double(*)[kMaxF]>(Xs + TB * LDS);
  double(*cv)[TB] = reinterpret_cast<double(*)[TB]>(Xs + TB * LDS + TB * kMaxF);
  double *dis = Xs + TB * LDS + TB * kMaxF + 2 * TB;
  const bool bad = diag_tile(Ds, LDS, rcol + int64_t(j + 1) * TB * ld, ld, F,
                             a.inv + sl.inv + int64_t(j + 1) * TB * TB, Xs, cv, dis, ysd);
  if (tid == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// Backward sweep L^T z = y of one slot (CTA per slot), tile row by tile row
// from the last: z_s = X_s^T (y_s - sum_{t>s} L[t, s]^T z_t), with the tile
// inverses X_s of the factorisation.  Warp w takes the tiles t = s + 1 + w,
// s + 9 + w, ... of column s and streams them from global memory (lane: two
// columns, every row coalesced); the warps' partial sums meet in shared
// memory.  z goes to zc (per slot) and, in the forward, to alpha_c per
// (patch, source).
__global__ void __launch_bounds__(256, 3) k_chol_back(BigArgs a, const BigSlot *__restrict__ slots) {
  __shared__ double part[8][TB][kMaxF];
  __shared__ double accs[TB][kMaxF];
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ld = sl.ld;
  const double *W = a.W + sl.base;
  const double *rcol = W + int64_t(sl.T) * TB;
  double *zc = a.zc + sl.zoff;
  const int rr = tid & 63, quarter = tid >> 6;
  for (int s = sl.T - 1; s >= 0; --s) {
    double acc0[kMaxF], acc1[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) acc0[f] = acc1[f] = 0.0;
    for (int t = s + 1 + warp; t < sl.T; t += 8) {
      const double *tile = W + int64_t(t) * TB * ld + int64_t(s) * TB;
      const double *zt = zc + int64_t(t) * TB * F;
#pragma unroll 8
      for (int c = 0; c < TB; ++c) {
        const double l0 = tile[int64_t(c) * ld + lane], l1 = tile[int64_t(c) * ld + lane + 32];
#pragma unroll
        for (int f = 0; f < kMaxF; ++f)
          if (f < F) {
            const double z = zt[c * F + f];
            acc0[f] = __fma_rn(l0, z, acc0[f]);
            acc1[f] = __fma_rn(l1, z, acc1[f]);
          }
      }
    }
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) {
      part[warp][lane][f] = acc0[f];
      part[warp][lane + 32][f] = acc1[f];
    }
    __syncthreads();
    for (int e = tid; e < TB * F; e += 256) {
      const int r = e / F, f = e % F;
      double sum = 0.0;
#pragma unroll
      for (int w = 0; w < 8; ++w) sum += part[w][r][f];
      accs[r][f] = rcol[int64_t(s * TB + r) * ld + f] - sum;
    }
    __syncthreads();
    // z_s[rr][f] = sum_{c >= rr} X_s[c][rr] acc_s[c][f]; quarters of c, then summed.
    const double *xs = a.inv + sl.inv + int64_t(s) * TB * TB;
    double zp[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) zp[f] = 0.0;
#pragma unroll 4
    for (int c = quarter; c < TB; c += 4) {
      if (c < rr) continue;
      const double x = xs[c * TB + rr];
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) zp[f] = __fma_rn(x, accs[c][f], zp[f]);
    }
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) part[quarter][rr][f] = zp[f];
    __syncthreads();
    for (int e = tid; e < TB * F; e += 256) {
      const int r = e / F, f = e % F;
      const double z = part[0][r][f] + part[1][r][f] + part[2][r][f] + part[3][r][f];
      const int j = s * TB + r;
      zc[int64_t(j) * F + f] = z;
      if (a.alpha_c != nullptr && j < sl.n) a.alpha_c[(a.soff[sl.k] + j) * F + f] = z;
    }
    __syncthreads();
  }
}

// local = E alpha + V beta for the targets of one slot (warp per target).
__global__ void __launch_bounds__(256) k_chol_eval(BigArgs a, const BigSlot *__restrict__ slots) {
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int64_t s0 = a.soff[sl.k], t0 = a.toff[sl.k];
  const double *beta = a.beta + sl.q * 4 * kMaxF;
  const int *act = a.act + sl.q * 3;
  const double *alpha = a.alpha_c + s0 * F;
  int bad = 0;
  for (int i = warp; i < sl.m; i += 8) {
    const double4 y = a.tgt[a.tidx[t0 + i]];
    double s[kMaxF];
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) s[f] = 0.0;
    for (int jj = lane; jj < sl.n; jj += 32) {
      const double4 x = a.src[a.sidx[s0 + jj]];
      const double ph =
          wendland<double>(a.basis, __dsqrt_rn(sqdist3(y.x, y.y, y.z, x.x, x.y, x.z)), a.rinv);
#pragma unroll
      for (int f = 0; f < kMaxF; ++f)
        if (f < F) s[f] = __fma_rn(ph, alpha[int64_t(jj) * F + f], s[f]);
    }
#pragma unroll
    for (int f = 0; f < kMaxF; ++f) s[f] = warp_sum(s[f]);
    if (lane == 0) {
      const double yc[3] = {y.x, y.y, y.z};
      for (int f = 0; f < F; ++f) {
        double v = beta[4 * f];
        for (int d = 0; d < 3; ++d)
          if (act[d] >= 0) v = __fma_rn(yc[act[d]], beta[4 * f + 1 + d], v);
        const double out = s[f] + v;
        if (!isfinite(out)) bad = 1;
        a.local[(t0 + i) * F + f] = out;
      }
    }
  }
  if (bad) atomicOr(&a.status[sl.k], 2);
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------

CholPlan chol_prefix(const std::vector<BigSlot> &slots) {
  // Step j serves the slots with T > j + 1 (a prefix: slots are sorted by
  // decreasing T), ceil((T - j - 1) / 2) CTAs each: CTA 0 of every slot first,
  // then the prefix counts of the others.
  CholPlan cp;
  const int ns = int(slots.size());
  const int steps = ns ? std::max(0, slots.front().T - 1) : 0;
  cp.ns = ns;
  cp.cnt.resize(steps);
  cp.off.resize(steps + 1);
  for (int j = 0; j < steps; ++j) {
    int c = 0;
    while (c < ns && slots[c].T > j + 1) ++c;
    cp.cnt[j] = c;
    cp.off[j] = int(cp.pre.size());
    int64_t acc = 0;
    cp.pre.push_back(0);
    for (int q = 0; q < c; ++q) {
      acc += (slots[q].T - j) / 2 - 1;  // CTAs l >= 1
      cp.pre.push_back(int(acc));
    }
    if (acc > 0x7fffffffll) throw Error{PACMAN_B200_ERR_LIMIT, "too many tiles in one launch"};
  }
  cp.off[steps] = int(cp.pre.size());
  return cp;
}

void chol_set_smem_attributes() {
  static bool done = false;
  if (done) return;
  PB_CUDA(cudaFuncSetAttribute(k_col_step, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kColSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_diag_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kDiagSmem)));
  done = true;
}

void chol_launch_steps(const BigArgs &a, const BigSlot *ds, const std::vector<BigSlot> &hs,
                       const CholPlan &cp, const int *dpre, cudaStream_t st, SolveReport &rep,
                       cudaEvent_t tail_event) {
  if (cp.ns == 0) return;
  k_diag_chol<<<cp.ns, 256, kDiagSmem, st>>>(a, ds, 0);
  note_launch();
  const int steps = int(cp.cnt.size());
  std::vector<cudaEvent_t> ev;
  if (rep.time_kernels) {
    ev.resize(2 * size_t(steps));
    for (auto &e : ev) PB_CUDA(cudaEventCreate(&e));
  }
  int sms = 0;
  PB_CUDA(cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0));
  bool tail = tail_event == nullptr;
  for (int j = 0; j < steps; ++j) {
    const int c = cp.cnt[j];
    const int n = c + cp.pre[cp.off[j] + c];
    if (!tail && n < 2 * sms) {  // from here on the steps leave SMs idle
      PB_CUDA(cudaEventRecord(tail_event, st));
      tail = true;
    }
    if (rep.time_kernels) PB_CUDA(cudaEventRecord(ev[2 * j], st));
    k_col_step<<<n, kColThreads, kColSmem, st>>>(a, ds, dpre + cp.off[j], c, j);
    note_launch();
    if (rep.time_kernels) {
      PB_CUDA(cudaEventRecord(ev[2 * j + 1], st));
      // Tile products: (T - j - 1) row tiles x (j + 1) (update + solve), and
      // j + 1 for the next diagonal tile.
      for (int q = 0; q < c; ++q)
        rep.update_flops += 2.0 * TB * TB * TB * double(hs[q].T - j) * double(j + 1);
      ++rep.update_launches;
    }
  }
  if (rep.time_kernels) {
    PB_CUDA(cudaStreamSynchronize(st));
    for (int j = 0; j < steps; ++j) {
      float ms = 0.f;
      PB_CUDA(cudaEventElapsedTime(&ms, ev[2 * j], ev[2 * j + 1]));
      rep.ms_update += ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
  }
  if (!tail) PB_CUDA(cudaEventRecord(tail_event, st));
}

void chol_launch_finish(const BigArgs &a, const BigSlot *ds, int ns, bool adjoint,
                        cudaStream_t st) {
  k_chol_back<<<ns, 256, 0, st>>>(a, ds);
  note_launch();
  if (!adjoint) {
    k_chol_eval<<<ns, 256, 0, st>>>(a, ds);
    note_launch();
  }
}

}  // namespace pacman_b200
