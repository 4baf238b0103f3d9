// Left-looking blocked Cholesky for the large patches of the B200 RBF-PUM
// transfer (precision "mixed" and the adjoint).
//
// The reference factors each patch matrix with an unpivoted LU in one GPU
// thread (src/rbf_pum/solver/solver.hpp:422-490, KokkosBatched
// SerialLU<Unblocked>).  A is symmetric positive definite, so here it is
// factored as L L^T in 64 x 64 tiles, all large patches in lockstep, one tile
// column j per step:
//   k_col_update  C[i, j] -= sum_{p<j} L[i, p] L[j, p]^T for every i >= j: the
//                 accumulator stays in registers for the whole K loop, the
//                 L panels stream through a cp.async pipeline;
//   k_diag_chol   X = L[j, j]^{-1} of C[j, j] = L[j, j] L[j, j]^T, y_j = X r_j;
//   k_col_trsm    L[i, j] = C[i, j] L[j, j]^{-T} for i > j, and the forward
//                 substitution update r_i -= L[i, j] y_j.
// Afterwards k_chol_back solves L^T alpha = y (tile inverses kept per step)
// and k_chol_eval evaluates local = E alpha + V beta (solver.hpp:270-273).
// The tile products run on the FP64 tensor cores (mma.sync m8n8k4 f64).
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
constexpr int kTrsmStrip = 4;           // row tiles per triangular-solve CTA
constexpr size_t kTrsmSmem = (size_t(3) * TB * LDS + TB * kMaxF) * sizeof(double);
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

// Column update of step j >= 1.  One CTA owns row tiles i0, i0 + 1 (i0 = j +
// 2l) of tile column j; eight warps each hold a 32 x 32 accumulator, which
// starts at -C and accumulates the products (no negation in the K loop).
__global__ void __launch_bounds__(kColThreads, 2)
    k_col_update(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre,
                 int cnt, int j) {
  extern __shared__ double sm[];
  const int q = find_slot(pre, cnt, blockIdx.x);
  const BigSlot sl = slots[q];
  const int i0 = j + 2 * (blockIdx.x - pre[q]);
  const bool two = i0 + 1 < sl.T;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int ld = sl.ld;
  const double *gA = a.W + sl.base + int64_t(i0) * TB * ld;
  const double *gB = a.W + sl.base + int64_t(j) * TB * ld;
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
  double *C = a.W + sl.base + int64_t(i0) * TB * ld + int64_t(j) * TB;
  double acc[4][4][2];
  if (active) {
    acc_load(acc, C, ld, wr, wc, lane);
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = -acc[i][jj][0], acc[i][jj][1] = -acc[i][jj][1];
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
  if (active) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj) acc[i][jj][0] = -acc[i][jj][0], acc[i][jj][1] = -acc[i][jj][1];
    acc_store(acc, C, ld, wr, wc, lane);
  }
}

// Inverse Cholesky factor of diagonal tile (j, j) of every active slot and
// y_j = X r_j.  The tile is eliminated as L D L^T with the identity carried
// along (Gauss-Jordan on [A | I]): at pivot p every row i > p gets
// R_i -= (a_ip / a_pp) R_p, which leaves U = D L^T on the left and L^{-1} on
// the right.  Each thread owns a 4 x 4 block of registers; slot (i, s) holds
// A[i][s] until pivot s and L^{-1}[i][s] afterwards.  Per pivot the owners
// publish one vector (row p of L^{-1} left of the pivot, the pivot, column p
// of A below it) and all threads update their slots: one barrier per pivot.
// Only X = L_c^{-1} = D^{-1/2} L^{-1} is kept (the trsm, the forward and the
// backward substitution use nothing else).  Non-positive pivots set status 4.
__global__ void __launch_bounds__(256, 4) k_diag_chol(BigArgs a, const BigSlot *__restrict__ slots,
                                                      int j) {
  extern __shared__ double sm[];
  double *Xs = sm;  // TB x LDS, the inverse factor at the end
  __shared__ double cv[2][TB];
  __shared__ double ys[TB][kMaxF];
  const BigSlot sl = slots[blockIdx.x];
  const int tid = threadIdx.x;
  const int bi = tid >> 4, bs = tid & 15;
  bool bad = false;
  const int ld = sl.ld, F = a.F;
  const double *g = a.W + sl.base + int64_t(j) * TB * ld + int64_t(j) * TB;
  double *rg = a.W + sl.base + int64_t(j) * TB * ld + int64_t(sl.T) * TB;
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
    ys[r][f] = f < F ? rg[int64_t(r) * ld + f] : 0.0;
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
  __shared__ double dis[TB];
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
  for (int e = tid; e < TB * F; e += 256) rg[int64_t(e / F) * ld + e % F] = yv[ny++];
  double *gi = a.inv + sl.inv + int64_t(j) * TB * TB;
  for (int idx = tid; idx < TB * TB / 2; idx += 256) {
    const int r = idx >> 5, c2 = idx & 31;
    *reinterpret_cast<double2 *>(gi + r * TB + 2 * c2) =
        *reinterpret_cast<const double2 *>(Xs + r * LDS + 2 * c2);
  }
  if (tid == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// Triangular solve of step j for up to kTrsmStrip row tiles i > j of one
// slot: L[i, j] = C[i, j] X^T (X = L[j, j]^{-1}), then r_i -= L[i, j] y_j.
__global__ void __launch_bounds__(128, 2)
    k_col_trsm(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ pre, int cnt,
               int j) {
  extern __shared__ double sm[];
  double *sI = sm;
  double *sX[2] = {sm + TB * LDS, sm + 2 * TB * LDS};
  double *sY = sm + 3 * TB * LDS;  // TB x kMaxF
  const int q = find_slot(pre, cnt, blockIdx.x);
  const BigSlot sl = slots[q];
  const int i0 = j + 1 + kTrsmStrip * (blockIdx.x - pre[q]);
  const int count = min(kTrsmStrip, sl.T - i0);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  const int ld = sl.ld, F = a.F;
  double *base = a.W + sl.base;
  const double *xinv = a.inv + sl.inv + int64_t(j) * TB * TB;
  for (int idx = tid; idx < TB * TB / 2; idx += 128) {
    const int r = idx >> 5, c2 = idx & 31;
    cp_async16(sI + r * LDS + 2 * c2, xinv + r * TB + 2 * c2);
  }
  async_tile(sX[0], base + int64_t(i0) * TB * ld + int64_t(j) * TB, ld, tid, 128);
  cp_async_commit();
  const double *yg = base + int64_t(j) * TB * ld + int64_t(sl.T) * TB;
  for (int e = tid; e < TB * kMaxF; e += 128) {
    const int r = e / kMaxF, f = e % kMaxF;
    sY[e] = f < F ? yg[int64_t(r) * ld + f] : 0.0;
  }
  for (int u = 0; u < count; ++u) {
    const int i = i0 + u;
    if (u + 1 < count) {
      async_tile(sX[(u + 1) & 1], base + int64_t(i + 1) * TB * ld + int64_t(j) * TB, ld, tid, 128);
      cp_async_commit();
      cp_async_wait<1>();
    } else {
      cp_async_wait<0>();
    }
    __syncthreads();
    double *sC = sX[u & 1];
    double acc[4][4][2];
    acc_zero(acc);
    mma64<false, true>(sC, sI, acc, 1.0, wr, wc, lane);
    acc_store(acc, base + int64_t(i) * TB * ld + int64_t(j) * TB, ld, wr, wc, lane);
    __syncthreads();
    // The L tile into shared memory for the residual update.
#pragma unroll
    for (int ii = 0; ii < 4; ++ii)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<double2 *>(sC + (wr + 8 * ii + g) * LDS + wc + 8 * jj + 2 * t) =
            make_double2(acc[ii][jj][0], acc[ii][jj][1]);
    __syncthreads();
    // out (64 x 8) = L y_j: warp w owns rows 16w .. 16w + 15.
    double o[2][2] = {{0.0, 0.0}, {0.0, 0.0}};
#pragma unroll 4
    for (int k0 = 0; k0 < TB; k0 += 4) {
      const double bf = sY[(k0 + t) * kMaxF + g];
#pragma unroll
      for (int mi = 0; mi < 2; ++mi)
        dmma(o[mi][0], o[mi][1], sC[(16 * warp + 8 * mi + g) * LDS + k0 + t], bf);
    }
    double *rg = base + int64_t(i) * TB * ld + int64_t(sl.T) * TB;
#pragma unroll
    for (int mi = 0; mi < 2; ++mi)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const int r = 16 * warp + 8 * mi + g, f = 2 * t + h;
        if (f < F) rg[int64_t(r) * ld + f] -= o[mi][h];
      }
    __syncthreads();
  }
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
  CholPlan cp;
  const int ns = int(slots.size());
  const int steps = ns ? slots.front().T : 0;
  cp.cnt.resize(steps);
  cp.off.resize(steps + 1);
  for (int j = 0; j < steps; ++j) {
    int c = 0;
    while (c < ns && slots[c].T > j) ++c;
    cp.cnt[j] = c;
    cp.off[j] = int(cp.pre.size());
    int64_t acc = 0;
    cp.pre.push_back(0);
    for (int q = 0; q < c; ++q) {
      acc += j > 0 ? (slots[q].T - j + 1) / 2 : 0;
      cp.pre.push_back(int(acc));
    }
    acc = 0;
    cp.pre.push_back(0);
    for (int q = 0; q < c; ++q) {
      acc += (slots[q].T - j - 1 + kTrsmStrip - 1) / kTrsmStrip;
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
  PB_CUDA(cudaFuncSetAttribute(k_col_update, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kColSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_diag_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kDiagSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_col_trsm, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kTrsmSmem)));
  done = true;
}

void chol_launch_steps(const BigArgs &a, const BigSlot *ds, const std::vector<BigSlot> &hs,
                       const CholPlan &cp, const int *dpre, cudaStream_t st, SolveReport &rep) {
  const int steps = int(cp.cnt.size());
  std::vector<cudaEvent_t> ev;
  if (rep.time_kernels) {
    ev.resize(2 * size_t(steps));
    for (auto &e : ev) PB_CUDA(cudaEventCreate(&e));
  }
  for (int j = 0; j < steps; ++j) {
    const int c = cp.cnt[j];
    const int *pu = dpre + cp.off[j];
    const int *pt = pu + c + 1;
    const int nu = cp.pre[cp.off[j] + c];
    const int nt = cp.pre[cp.off[j] + c + 1 + c];
    if (nu) {
      if (rep.time_kernels) PB_CUDA(cudaEventRecord(ev[2 * j], st));
      k_col_update<<<nu, kColThreads, kColSmem, st>>>(a, ds, pu, c, j);
      note_launch();
      if (rep.time_kernels) {
        PB_CUDA(cudaEventRecord(ev[2 * j + 1], st));
        for (int q = 0; q < c; ++q)
          rep.update_flops += 2.0 * TB * TB * TB * double(hs[q].T - j) * double(j);
        ++rep.update_launches;
      }
    }
    k_diag_chol<<<c, 256, kDiagSmem, st>>>(a, ds, j);
    note_launch();
    if (nt) {
      k_col_trsm<<<nt, 128, kTrsmSmem, st>>>(a, ds, pt, c, j);
      note_launch();
    }
  }
  if (rep.time_kernels) {
    PB_CUDA(cudaStreamSynchronize(st));
    for (int j = 0; j < steps; ++j) {
      if (cp.pre[cp.off[j] + cp.cnt[j]] == 0) continue;
      float ms = 0.f;
      PB_CUDA(cudaEventElapsedTime(&ms, ev[2 * j], ev[2 * j + 1]));
      rep.ms_update += ms;
    }
    for (auto &e : ev) cudaEventDestroy(e);
  }
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
