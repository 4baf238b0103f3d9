// Left-looking blocked Cholesky for the large patches of the B200 RBF-PUM
// transfer (precision "mixed" and the adjoint).
//
// The reference factors each patch matrix with an unpivoted LU in one GPU
// thread (src/rbf_pum/solver/solver.hpp:422-490, KokkosBatched
// SerialLU<Unblocked>).  A is symmetric positive definite, so here it is
// factored as L L^T in 64 x 64 tiles, all large patches in lockstep, one tile
// column j per step:
//   C[i, j] = A[i, j] - sum_{p<j} L[i, p] L[j, p]^T for every i > j, then
//   L[i, j] U_j = C solved against the diagonal tile's factor (U_j = L_jj^T,
//   made one step earlier) and the forward substitution r_i -= L[i, j] y_j.
// The column update runs on the int8 tensor cores as split-integer products
// (k_col_step_ws, with k_diag_next factoring the next diagonal tile after
// each step) or, for the columns before PACMAN_B200_INT8_FROM and without
// int8 slices, on the FP64 tensor cores (k_col_step, whose CTA of row tile
// j + 1 also forms and factors the next diagonal tile).  k_diag_chol does
// the diagonal tile of step 0.  Afterwards k_chol_back solves L^T alpha = y
// (with the kept tile inverses X_s = L_ss^-1) and k_chol_eval evaluates
// local = E alpha + V beta (solver.hpp:270-273).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
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
constexpr size_t kDiagSmem = (size_t(2) * TB * LDS + 6 * TB) * sizeof(double);

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

// Rows [ti TB, ti TB + nrows) x columns [tj TB, tj TB + TB) of a slot's
// Wendland matrix A (TeamFillA, team_ops.hpp:35-52; identity past n) into sT
// (row stride LDS), by the threads t, t + nt, ...: the step kernels evaluate
// their tiles instead of reading an assembled copy.  The row and column points
// are staged in pts (3 (nrows + TB) doubles) first; sync() must be a barrier
// over the nt threads.
template <class Sync>
__device__ __forceinline__ void gen_tile(const BigArgs &a, const BigSlot &sl, int ti, int tj,
                                         int nrows, double *sT, double *pts, int t, int nt,
                                         Sync sync, bool load_cols = true) {
  const int64_t s0 = a.soff[sl.k];
  double *rx = pts, *ry = rx + nrows, *rz = ry + nrows;
  double *cx = rz + nrows, *cy = cx + TB, *cz = cy + TB;
  // With load_cols false the column points are still in pts from a previous
  // tile of the same slot and column tile.
  for (int e = t; e < (load_cols ? nrows + TB : nrows); e += nt) {
    const int gi = e < nrows ? ti * TB + e : tj * TB + (e - nrows);
    double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
    if (gi < sl.n) p = a.src[a.sidx[s0 + gi]];
    if (e < nrows) {
      rx[e] = p.x;
      ry[e] = p.y;
      rz[e] = p.z;
    } else {
      cx[e - nrows] = p.x;
      cy[e - nrows] = p.y;
      cz[e - nrows] = p.z;
    }
  }
  sync();
  for (int e = t; e < nrows * TB; e += nt) {
    const int r = e >> 6, c = e & 63;
    const int gi = ti * TB + r, gj = tj * TB + c;
    double v;
    if (gi < sl.n && gj < sl.n)
      v = wendland<double>(a.basis, __dsqrt_rn(sqdist3(rx[r], ry[r], rz[r], cx[c], cy[c], cz[c])),
                           a.rinv);
    else
      v = (gi == gj) ? 1.0 : 0.0;
    sT[r * LDS + c] = v;
  }
}

__device__ __forceinline__ void sync_all() { __syncthreads(); }

// Cholesky of the 16 x 16 block D[kb.., kb..] (lower part, row stride ld,
// overwritten by L) by one warp in registers: lane i + 16 h holds columns
// 8 h .. 8 h + 7 of row kb + i; column c's entries reach the other lanes by
// shuffles.  A column-by-column right-looking Cholesky of the block: 1 / L_cc
// = rsqrt(d_cc) (one operation on the chain of pivots instead of a square
// root and a reciprocal), L_cc = d_cc / L_cc, L_ic = d_ic (1 / L_cc), d_ij -=
// L_ic L_jc; dis[kb + c] = 1 / L_cc.  Written without branches (selects; lane
// c keeps 1 / L_cc and stores it after the loop) so that the sixteen unrolled
// steps form one block the compiler can schedule across: FP64 operations
// and shuffles each take ~25 cycles to complete on this GPU, and a step is a
// chain of five of them.  Returns true on a pivot that is not > 0.
__device__ __noinline__ bool warp_chol16(double *D, int ld, int kb, double *dis, int lane) {
  const int i = lane & 15, h = lane >> 4;
  double a[8];
#pragma unroll
  for (int t = 0; t < 8; ++t) a[t] = 8 * h + t <= i ? D[(kb + i) * ld + kb + 8 * h + t] : 0.0;
  double myrs = 0.0;
  bool ok = true;
#pragma unroll
  for (int c = 0; c < 16; ++c) {
    const int hc = c >> 3, tc = c & 7;
    const double piv = __shfl_sync(0xffffffffu, a[tc], c + 16 * hc);
    ok = ok && piv > 0.0;
    const double rs = rsqrt(piv);
    const double sc = a[tc] * rs;
    const bool mine = h == hc;
    a[tc] = mine ? (i == c ? piv * rs : (i > c ? sc : a[tc])) : a[tc];
    myrs = lane == c ? rs : myrs;
    const double oth = __shfl_xor_sync(0xffffffffu, a[tc], 16);
    const double lic = mine ? a[tc] : oth;  // L[i][c]
#pragma unroll
    for (int jj = c + 1; jj < 16; ++jj) {
      const double ljc = __shfl_sync(0xffffffffu, a[tc], jj + 16 * hc);  // L[jj][c]
      const bool upd = h == (jj >> 3) && i >= jj;
      const double nv = __fma_rn(-lic, ljc, a[jj & 7]);
      a[jj & 7] = upd ? nv : a[jj & 7];
    }
  }
  if (lane < 16) dis[kb + lane] = myrs;
#pragma unroll
  for (int t = 0; t < 8; ++t)
    if (8 * h + t <= i) D[(kb + i) * ld + kb + 8 * h + t] = a[t];
  __syncwarp();
  return !ok;
}

// T = L_bb^-1 of the 16 x 16 lower-triangular block at D[kb..][kb..] (row
// stride ld) by one warp in registers, lane j (and j + 16) computing column j
// of T down the column (T_jj = 1 / L_jj from dis, T_ij = -(sum_{j<=k<i} L_ik
// T_kj) / L_ii), unrolled and without branches; stored transposed:
// ui[j kUiLd + i] = T_ij, i.e. ui holds (L_bb^T)^-1 = U_bb^-1.
__device__ __noinline__ void warp_trinv16(const double *D, int ld, int kb, const double *dis,
                                          double *ui, int lane) {
  const int j = lane & 15;
  double t[16];
#pragma unroll
  for (int i = 0; i < 16; ++i) {
    double s = 0.0;
#pragma unroll
    for (int k = 0; k < i; ++k) {
      const double v = __fma_rn(D[(kb + i) * ld + kb + k], t[k], s);
      s = k >= j ? v : s;
    }
    const double di = dis[kb + i];
    t[i] = i < j ? 0.0 : (i == j ? di : -s * di);
  }
  if (lane < 16) {
#pragma unroll
    for (int i = 0; i < 16; ++i) ui[j * kUiLd + i] = t[i];
  }
  __syncwarp();
}

// The diagonal tile of a step, 256 threads (8 warps): the Cholesky factor
// L_c of the 64 x 64 tile D (lower part, in shared memory at g with row stride
// ld, overwritten), X = L_c^{-1} (to gi, row stride TB), y = X r for the first
// F columns of the residual tile (rg, row stride rld, overwritten) and, with
// gu, U = L_c^T (row stride uld; zeros below its diagonal) for the triangular
// solves of the tiles below.  Blocked right-looking Cholesky in 16 x 16
// blocks: warp 0 factors the diagonal block (16 column steps synchronised
// within the warp), the eight warps solve the panel below it by substitution
// and update the trailing blocks on the FP64 tensor cores, three barriers per
// block.  X comes from the row solves X^T U = I (warp_rows_trsm8, or with
// kTensorSolve warp_rows_trsm8_tc).  Us (TB x LDS) is shared scratch for U,
// dis (TB) for 1 / diag(L_c), ys (TB x kMaxF) for r.  Returns true on a
// non-positive pivot (status 4 for the caller).
template <class Sync, bool kTensorSolve = false>
__device__ bool diag_tile_t(const double *g_in, int ld, double *rg, int rld, int F, double *gi,
                            double *Us, double (*cv)[TB], double *dis, double (*ys)[kMaxF],
                            int tid, Sync sync, double *gu = nullptr, int uld = 0,
                            double *ui = nullptr, bool ys_loaded = false) {
  (void)cv;
  double *D = const_cast<double *>(g_in);
  const int lane = tid & 31, warp = tid >> 5;
  const int gq = lane >> 2, tq = lane & 3;
  const int col16 = lane & 15, half = lane & 16, rsel = lane >> 4;
  bool bad = false;
  if (!ys_loaded)
    for (int e = tid; e < TB * kMaxF; e += 256) {
      const int r = e / kMaxF, f = e % kMaxF;
      ys[r][f] = f < F ? __ldcg(rg + int64_t(r) * rld + f) : 0.0;
    }
  const bool blockinv = !kTensorSolve && ui != nullptr;
  // (a) the first diagonal block, warp 0 (warp_chol16).
  if (warp == 0) bad |= warp_chol16(D, ld, 0, dis, lane);
  sync();
  for (int kb = 0; kb + 16 < TB; kb += 16) {
    // (b) the panel below: rows kb + 16 .. 63 solve x L_kk^T = d.
    const int r0 = kb + 16 + 8 * warp;
    if (r0 < TB) {
      double acc[4];
#pragma unroll
      for (int q = 0; q < 4; ++q) acc[q] = D[(r0 + rsel + 2 * q) * ld + kb + col16];
#pragma unroll 4
      for (int c = 0; c < 16; ++c) {
        const double d = dis[kb + c];
        const double l = D[(kb + col16) * ld + kb + c];  // L_kk[col16][c], used for col16 > c
        const bool own = col16 == c, below = col16 > c;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const double x = __shfl_sync(0xffffffffu, acc[q], half | c) * d;
          acc[q] = own ? x : (below ? __fma_rn(-x, l, acc[q]) : acc[q]);
        }
      }
#pragma unroll
      for (int q = 0; q < 4; ++q) D[(r0 + rsel + 2 * q) * ld + kb + col16] = acc[q];
    }
    sync();
    // (c) trailing blocks: D[i, j] -= P_i P_j^T (P: the panel columns), 8 x 8
    // output tiles (ti, tj) with kb + 16 <= 8 tj <= 8 ti.  Warp 0 updates
    // the next diagonal block's three tiles first and factors that block
    // (look-ahead) while warps 1..7 update the rest: the chain of diagonal
    // blocks does not wait for the whole trailing update.
    const int base = (kb + 16) / 8, nt = 8 - base;
    auto tile = [&](int ti, int tj) {
      double c0 = D[(8 * ti + gq) * ld + 8 * tj + 2 * tq];
      double c1 = D[(8 * ti + gq) * ld + 8 * tj + 2 * tq + 1];
#pragma unroll
      for (int k0 = 0; k0 < 16; k0 += 4) {
        const double av = -D[(8 * ti + gq) * ld + kb + k0 + tq];
        const double bv = D[(8 * tj + gq) * ld + kb + k0 + tq];
        dmma(c0, c1, av, bv);
      }
      D[(8 * ti + gq) * ld + 8 * tj + 2 * tq] = c0;
      D[(8 * ti + gq) * ld + 8 * tj + 2 * tq + 1] = c1;
    };
    if (warp == 0) {
      tile(base, base);
      tile(base + 1, base);
      tile(base + 1, base + 1);
      __syncwarp();
      bad |= warp_chol16(D, ld, kb + 16, dis, lane);
    } else {
      for (int u = warp - 1; u < nt * nt; u += 7) {
        const int ti = base + u / nt, tj = base + u % nt;
        if (tj > ti || (ti < base + 2 && tj < base + 2)) continue;
        tile(ti, tj);
      }
    }
    sync();
  }
  // U = L_c^T with zeros below its diagonal; 1 / diag for the row solves.
  for (int e = tid; e < TB * TB; e += 256) {
    const int p = e >> 6, i = e & 63;
    const double u = i >= p ? D[i * ld + p] : 0.0;
    Us[p * LDS + i] = u;
    if (gu) gu[int64_t(p) * uld + i] = u;
  }
  // With ui: the inverses of U's four 16 x 16 diagonal blocks, one warp each,
  // for the block-inverse row solves of X below.
  if (blockinv && warp < 4) warp_trinv16(D, ld, 16 * warp, dis, ui + 16 * warp * kUiLd, lane);
  sync();
  // X^T from X^T U = I: rows of the identity solved in place of D.
  for (int e = tid; e < TB * TB; e += 256) D[(e >> 6) * ld + (e & 63)] = (e >> 6) == (e & 63);
  sync();
  if (kTensorSolve) warp_rows_trsm8_tc(D + 8 * warp * ld, Us, dis, lane);
  else if (blockinv) warp_rows_trsm8_bi(D + 8 * warp * ld, Us, ui, lane, nullptr, 0.0);
  else warp_rows_trsm8(D + 8 * warp * ld, Us, dis, lane);
  sync();
  // X (row-major, gi) and y = X r.
  for (int e = tid; e < TB * TB; e += 256) {
    const int r = e >> 6, c = e & 63;
    gi[r * TB + c] = D[c * ld + r];
  }
  for (int e = tid; e < TB * F; e += 256) {
    const int r = e / F, f = e % F;
    double s = 0.0;
    for (int k = 0; k <= r; ++k) s = __fma_rn(D[k * ld + r], ys[k][f], s);
    rg[int64_t(r) * rld + f] = s;
  }
  // Every thread learns about a breakdown (warp 0 saw the pivots).
  __shared__ int bad_any;
  if (tid == 0) bad_any = 0;
  sync();
  if (bad) bad_any = 1;
  sync();
  return bad_any != 0;
}

__device__ __forceinline__ bool diag_tile(const double *g, int ld, double *rg, int rld, int F,
                                          double *gi, double *Xs, double (*cv)[TB], double *dis,
                                          double (*ys)[kMaxF], double *gu = nullptr,
                                          int uld = 0) {
  auto sync = [] { __syncthreads(); };
  return diag_tile_t<decltype(sync), true>(g, ld, rg, rld, F, gi, Xs, cv, dis, ys,
                                            int(threadIdx.x), sync, gu, uld);
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
  double *gt = sm + TB * LDS;  // the evaluated tile A[j, j]
  double *pts = sm + 2 * TB * LDS;
  gen_tile(a, sl, j, j, TB, gt, pts, threadIdx.x, blockDim.x, sync_all);
  __syncthreads();
  double *rg = a.W + sl.base + int64_t(j) * TB * ld + int64_t(sl.T) * TB;
  const bool bad =
      diag_tile(gt, LDS, rg, ld, a.F, a.inv + sl.inv + int64_t(j) * TB * TB, sm, cv, dis, ys,
                a.W + sl.base + int64_t(j) * TB * ld + int64_t(j) * TB, ld);
  if (threadIdx.x == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// The next diagonal tile after an int8 step j, one CTA per slot with
// T > j + 1 (the first cnt slots): D = D' - L[j+1, j] L[j+1, j]^T, with D'
// (the tile minus the products of columns p < j) written by the step's
// diagonal item to dpart and L[j+1, j] by its row item j + 1; then
// diag_tile_t with block-inverse row solves (X_{j+1}, U_{j+1}, y_{j+1}).  A
// separate launch rather than a hand-over inside the step: the factorisation
// of a 64 x 64 tile is a chain of 64 pivots that keeps one warp busy for tens
// of microseconds, and here two CTAs per SM overlap their chains while the
// step kernel's CTAs go on with their items.
constexpr size_t kDiagNextSmem =
    (size_t(2) * TB * LDS + size_t(4) * 16 * kUiLd + 3 * TB + TB * kMaxF) * sizeof(double);
__global__ void __launch_bounds__(256, 2) k_diag_next(BigArgs a, const BigSlot *__restrict__ slots,
                                                      int j) {
  extern __shared__ __align__(16) double smn[];
  double *D = smn;                  // D' and then D (TB x LDS)
  double *Ls = D + TB * LDS;        // L[j+1, j], then U scratch
  double *ui = Ls + TB * LDS;       // U's 16 x 16 diagonal block inverses
  double(*cv)[TB] = reinterpret_cast<double(*)[TB]>(ui + 4 * 16 * kUiLd);
  double *dis = ui + 4 * 16 * kUiLd + 2 * TB;
  double(*ys)[kMaxF] = reinterpret_cast<double(*)[kMaxF]>(dis + TB);
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  // The next step's launch may start now (its epilogue waits for this grid).
  asm volatile("griddepcontrol.launch_dependents;\n" ::: "memory");
  const BigSlot sl = slots[blockIdx.x];
  const int ld = sl.ld;
  double *W = a.W + sl.base;
  const double *dp = a.dpart + int64_t(sl.q) * TB * TB;
  const double *lg = W + int64_t(j + 1) * TB * ld + int64_t(j) * TB;
  for (int idx = tid; idx < TB * TB / 2; idx += 256) {
    const int r = idx >> 5, c2 = idx & 31;
    cp_async16(D + r * LDS + 2 * c2, dp + r * TB + 2 * c2);
    cp_async16(Ls + r * LDS + 2 * c2, lg + int64_t(r) * ld + 2 * c2);
  }
  // r_{j+1} (the first F columns of the residual tile), for y = X r.
  double *rg = W + int64_t(j + 1) * TB * ld + int64_t(sl.T) * TB;
  for (int e = tid; e < TB * a.F; e += 256)
    cp_async8(&ys[e / a.F][e % a.F], rg + int64_t(e / a.F) * ld + e % a.F);
  cp_async_commit();
  cp_async_wait<0>();
  __syncthreads();
  {
    const int wr = (warp >> 1) * 32, wc = (warp & 1) * 32;
    double acc[4][4][2];
    if (warp < 4) {
      acc_load(acc, D, LDS, wr, wc, lane);
      mma64<false, true>(Ls, Ls, acc, -1.0, wr, wc, lane);
    }
    __syncthreads();
    if (warp < 4) acc_store(acc, D, LDS, wr, wc, lane);
  }
  __syncthreads();
  auto sync = [] { __syncthreads(); };
  const bool bad = diag_tile_t(D, LDS, rg, ld, a.F, a.inv + sl.inv + int64_t(j + 1) * TB * TB, Ls,
                               cv, dis, ys, tid, sync,
                               W + int64_t(j + 1) * TB * ld + int64_t(j + 1) * TB, ld, ui, true);
  if (tid == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// Phase 2 of a factorisation step (256 threads, warp w: rows 16 w .. + 15,
// in two passes of 8).  sC holds C (row tiles i0, and i0 + 1 when arows =
// 2 TB; kColRows x LDS).  L[i, j] solves L[i, j] U_j = C with U_j = L_jj^T
// (the factor of the diagonal tile, loaded into sU), by blocked row solves
// (warp_rows_trsm8_tc); it is stored in the workspace and written back over C
// in sC (in place); then the forward substitution r_i -=
// L[i, j] y_j.  vec holds TB + TB kMaxF doubles (1 / diag(U_j), y_j).  Ends
// with a barrier.
__device__ void step_trsm(const BigArgs &a, const BigSlot &sl, int j, int i0, int arows,
                          double *sC, double *sU, double *vec) {
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int ld = sl.ld, F = a.F;
  double *W = a.W + sl.base;
  double *rcol = W + int64_t(sl.T) * TB;
  double *dinv = vec, *ysh = vec + TB;
  load_factor_async(sU, W + int64_t(j) * TB * ld + int64_t(j) * TB, ld, tid, kColThreads);
  cp_async_commit();
  {
    const double *yg = rcol + int64_t(j) * TB * ld;
    for (int e = tid; e < TB * kMaxF; e += kColThreads) {
      const int r = e / kMaxF, f = e % kMaxF;
      ysh[e] = f < F ? __ldcg(yg + int64_t(r) * ld + f) : 0.0;
    }
  }
  cp_async_wait<0>();
  __syncthreads();
  if (tid < TB) dinv[tid] = 1.0 / sU[tid * LDS + tid];
  __syncthreads();
  double *C = W + int64_t(i0) * TB * ld + int64_t(j) * TB;
  double *rg = rcol + int64_t(i0) * TB * ld;
  for (int pass = 0; pass < 2; ++pass) {
    const int r0 = 16 * warp + 8 * pass;
    if (r0 >= arows) break;
    warp_rows_trsm8_tc(sC + r0 * LDS, sU, dinv, lane);
    double lo[8], hi[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) {
      lo[q] = sC[(r0 + q) * LDS + lane];
      hi[q] = sC[(r0 + q) * LDS + 32 + lane];
      C[int64_t(r0 + q) * ld + lane] = lo[q];
      C[int64_t(r0 + q) * ld + 32 + lane] = hi[q];
    }
    for (int f = 0; f < F; ++f) {
      const double yl = ysh[lane * kMaxF + f], yh = ysh[(lane + 32) * kMaxF + f];
#pragma unroll
      for (int q = 0; q < 8; ++q) {
        double sum = __fma_rn(lo[q], yl, hi[q] * yh);
        for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
        if (lane == 0) rg[int64_t(r0 + q) * ld + f] -= sum;
      }
    }
  }
  __syncthreads();
}

// ---------------------------------------------------------------------------
// Column updates on the int8 tensor cores (precision "mixed")
// ---------------------------------------------------------------------------
//
// Every finished off-diagonal tile L[i, p] is also kept as kOzS int8 digit
// slices of x = L / sigma (sigma >= sqrt(max_r A_rr) bounds every entry of L,
// since the rows of L have norm sqrt(A_rr)): x = sum_s d_s 128^-s, d_1 in
// [-127, 127], d_s in [-64, 64] after.  The update
//   sum_p L[i, p] L[j, p]^T = sigma^2 sum_{a,b} 128^-(a+b) D_a[i] D_b[j]^T
// keeps the slice pairs with a + b <= kOzS + 2 (levels 2..9) and sums each
// level exactly in int32 on the tcgen05 tensor cores (kind::i8); the levels
// are combined in int64 and FP64 at the end.  A digit product is at most
// 2^12 in magnitude, so a dropped term (level >= 10) is below 2^-58 sigma^2:
// the truncation of a K-long sum stays near the FP64 rounding of the same
// sum.  Dropping level 9 as well (2^-51 per term) is not enough: on patches
// with cond(A) ~ 1e13 it multiplies the error of the local values by ~15.
// This is the split-integer emulation of an FP64 product (Ozaki, Ogita, Oishi
// and Rump 2012; Uchino, Ozaki and Imamura 2024 for integer tensor cores).
//
// Slice tile layout (28 KB): [16-byte K chunk (4)][slice (kOzS)][8-row group
// (8)][8 rows x 16 bytes], i.e. the K-major core-matrix layout of the tensor
// core, copied to shared memory with bulk async copies.
constexpr int kOzS = 7;
constexpr int kOzTileBytes = 4 * kOzS * 8 * 128;      // 28672
constexpr int kOzTmemCols = 512;                      // 8 column groups of 64 (levels 2..9)
constexpr int kOzWaitLimit = 1 << 22;                 // bounded mbarrier polls
// Polls of the waits that drain a pipeline after it gave up: they wait for
// copies and tensor-core operations already issued, which complete by
// themselves, so they get a longer limit than the pipeline waits
// (BigArgs::wait_limit) and are never shortened.
constexpr int kOzDrainLimit = 1 << 24;


__device__ __forceinline__ uint32_t saddr(const void *p) {
  return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(uint64_t *b, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(saddr(b)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *b, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(b)),
               "r"(bytes)
               : "memory");
}
__device__ __forceinline__ void mbar_arrive_cnt(uint64_t *b, uint32_t cnt) {
  asm volatile("mbarrier.arrive.release.cta.shared::cta.b64 _, [%0], %1;\n" ::"r"(saddr(b)),
               "r"(cnt)
               : "memory");
}
__device__ __forceinline__ bool mbar_try(uint64_t *b, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n.reg .pred p;\nmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(done)
      : "r"(saddr(b)), "r"(parity)
      : "memory");
  return done != 0;
}
// Bounded wait for the phase with the given parity; false on time-out.
__device__ __forceinline__ bool mbar_wait(uint64_t *b, uint32_t parity, int limit = kOzWaitLimit) {
  bool done = false;
  for (int it = 0; it < limit && !done; ++it) done = mbar_try(b, parity);
  return done;
}
// Pipeline wait of the int8 K loop: bounded by `limit` polls, and given up
// at once when the other side of the pipeline has aborted.
__device__ __forceinline__ bool mbar_wait_pipe(uint64_t *b, uint32_t parity, int limit,
                                               volatile int *abort_flag) {
  for (int it = 0; it < limit; ++it) {
    if (mbar_try(b, parity)) return true;
    if (*abort_flag) return false;
  }
  return false;
}
__device__ __forceinline__ void bulk_g2s(void *dst, const void *src, uint32_t bytes, uint64_t *b) {
  asm volatile(
      "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(
          saddr(dst)),
      "l"(src), "r"(bytes), "r"(saddr(b))
      : "memory");
}
// Shared-memory matrix descriptor, K-major core matrices without swizzle
// (layout type 0, descriptor version 1): lbo = byte step between 16-byte K
// chunks, sbo = byte step between 8-row groups.
__device__ __forceinline__ uint64_t umma_desc(uint32_t addr, uint32_t lbo, uint32_t sbo) {
  return uint64_t((addr >> 4) & 0x3FFF) | (uint64_t((lbo >> 4) & 0x3FFF) << 16) |
         (uint64_t((sbo >> 4) & 0x3FFF) << 32) | (uint64_t(1) << 46);
}
// Instruction descriptor: D s32, A and B signed int8, both K-major, M = 128.
__device__ __forceinline__ uint32_t umma_idesc_i8(int n) {
  return (2u << 4) | (1u << 7) | (1u << 10) | (uint32_t(n >> 3) << 17) | (uint32_t(128 >> 4) << 24);
}
__device__ __forceinline__ void umma_i8(uint32_t dtmem, uint64_t ad, uint64_t bd, uint32_t idesc,
                                        uint32_t accumulate) {
  asm volatile(
      "{\n.reg .pred p;\nsetp.ne.b32 p, %4, 0;\n"
      "tcgen05.mma.cta_group::1.kind::i8 [%0], %1, %2, %3, p;\n}\n" ::"r"(dtmem),
      "l"(ad), "l"(bd), "r"(idesc), "r"(accumulate)
      : "memory");
}
__device__ __forceinline__ void umma_commit(uint64_t *b) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(
                   saddr(b))
               : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
  asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
  asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory");
}

// The int8 digits of rows [0, nrows) of L tiles held in shared memory (row
// stride LDS; rows 64.. belong to the second tile) straight into their slice
// tiles in global memory (dst0: the tile of rows 0..63, dst1: rows 64..127).
// A thread unit is (row, 16-column K chunk): it builds the 16 bytes of each of
// the kOzS slices and stores each as one 16-byte word, consecutive units of a
// warp writing consecutive words.  Digits: y = round(x 128^kOzS) as an
// integer (x = L mul / 128 in [-1, 1]); balanced base-128 digits from the top,
// d = round(y / 128^(kOzS-1-s)), y -= d 128^(kOzS-1-s).
__device__ void slice_tile_smem(const double *sL, int nrows, double mul, uint8_t *dst0,
                                uint8_t *dst1, int tid, int nt) {
  for (int u = tid; u < nrows * 4; u += nt) {
    const int r = (u & 63) + 64 * (u >> 8), c16 = (u >> 6) & 3;
    uint32_t w[kOzS][4];
#pragma unroll
    for (int sl = 0; sl < kOzS; ++sl)
#pragma unroll
      for (int q = 0; q < 4; ++q) w[sl][q] = 0u;
#pragma unroll
    for (int cc = 0; cc < 16; ++cc) {
      const double xs = fmin(fmax(sL[r * LDS + 16 * c16 + cc] * mul, -127.49), 127.49);
      long long y = __double2ll_rn(xs * 0x1p42);  // x * 128 * 128^(kOzS-1)
#pragma unroll
      for (int sl = 0; sl < kOzS; ++sl) {
        const int sh = 7 * (kOzS - 1 - sl);
        const long long d = sh ? ((y + (1ll << (sh - 1))) >> sh) : y;
        y -= d << sh;
        w[sl][cc >> 2] |= uint32_t(uint8_t(int8_t(d))) << (8 * (cc & 3));
      }
    }
    uint8_t *dst = (r < 64 ? dst0 : dst1) + c16 * kOzS * 1024 + (r & 63) * 16;
#pragma unroll
    for (int sl = 0; sl < kOzS; ++sl)
      *reinterpret_cast<uint4 *>(dst + sl * 1024) = make_uint4(w[sl][0], w[sl][1], w[sl][2], w[sl][3]);
  }
}

// Step j of the factorisation, one launch over all slots with T > j + 1.
// CTA l of a slot owns row tiles i0 = j + 1 + 2l and i0 + 1 of tile column j:
//  1. C = A[i, j] - sum_{p<j} L[i, p] L[j, p]^T: eight warps hold 32 x 32
//     accumulators (starting at -A) for the whole K loop, the L panels stream
//     through a cp.async pipeline;
//  2. L[i, j] U_j = C, the triangular solve against the diagonal tile's
//     factor (made one step earlier), stored; then the forward
//     substitution r_i -= L[i, j] y_j;
//  3. CTA 0 (i0 = j + 1) forms the next diagonal tile
//     D = A[j+1, j+1] - sum_{p<=j} L[j+1, p] L[j+1, p]^T and factors it:
//     X_{j+1} and y_{j+1} = X_{j+1} r_{j+1} for step j + 1.
template <bool SLICE>
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
  const bool active = two || wr < TB;
  double acc[4][4][2];
  gen_tile(a, sl, i0, j, arows, sm, sm + kColRows * LDS, tid, kColThreads, sync_all);  // A[i, j]
  __syncthreads();
  if (active) {
    acc_load(acc, sm, LDS, wr, wc, lane);
    acc_neg(acc);
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nch) load(s, s);
    cp_async_commit();
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

  // 2. L[i, j] U_j = C through shared memory, then the forward substitution.
  if (active) {
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int jj = 0; jj < 4; ++jj)
        *reinterpret_cast<double2 *>(sm + (wr + 8 * i + g) * LDS + wc + 8 * jj + 2 * t) =
            make_double2(-acc[i][jj][0], -acc[i][jj][1]);
  }
  __syncthreads();
  step_trsm(a, sl, j, i0, arows, sm, sm + kColRows * LDS, sm + (kColRows + TB) * LDS);
  if (SLICE) {  // int8 slices of the new L tiles for the int8 steps that follow
    uint8_t *srow = a.slices + sl.sli;
    slice_tile_smem(sm, arows, a.oz_mul, srow + (int64_t(i0) * (i0 - 1) / 2 + j) * kOzTileBytes,
                    srow + (int64_t(i0 + 1) * i0 / 2 + j) * kOzTileBytes, tid, kColThreads);
  }
  if (l != 0) return;

  // 3. The diagonal tile of step j + 1 (this CTA's first row tile).
  __syncthreads();
  constexpr int kDStage = TB * kKLD;
  double *sL = sm + 2 * kDStage;  // L[j+1, j], TB x LDS (rows 0..63 of sC are below it)
  static_assert(2 * kDStage >= TB * LDS, "L[j+1, j] overlaps its copy source");
  for (int e = tid; e < TB * TB; e += kColThreads) sL[(e >> 6) * LDS + (e & 63)] = sm[(e >> 6) * LDS + (e & 63)];
  __syncthreads();
  auto loadd = [&](int c, int stage) {
    double *sD = sm + stage * kDStage;
    const int col = c * kKC;
    for (int idx = tid; idx < TB * (kKC / 2); idx += kColThreads) {
      const int r = idx / (kKC / 2), c2 = idx % (kKC / 2);
      cp_async16(sD + r * kKLD + 2 * c2, gA + int64_t(r) * ld + col + 2 * c2);
    }
  };
  const bool dact = wr < TB;
  double *Dgen = sm + 2 * kDStage + TB * LDS;  // A[j+1, j+1], after sL
  gen_tile(a, sl, j + 1, j + 1, TB, Dgen, sm, tid, kColThreads, sync_all);
  __syncthreads();
  if (dact) {
    acc_load(acc, Dgen, LDS, wr, wc, lane);
    acc_neg(acc);
  }
  __syncthreads();
#pragma unroll
  for (int s = 0; s < kStages - 1; ++s) {
    if (s < nch) loadd(s, s);
    cp_async_commit();
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
                             a.inv + sl.inv + int64_t(j + 1) * TB * TB, Xs, cv, dis, ysd,
                             W + int64_t(j + 1) * TB * ld + int64_t(j + 1) * TB, ld);
  if (tid == 0 && bad) atomicOr(&a.status[sl.k], 4);
}

// ---------------------------------------------------------------------------
// Warp-specialised int8 step (k_col_step_ws)
// ---------------------------------------------------------------------------
//
// Step j of the factorisation with the column update on the int8 tensor
// cores, organised so that the int8 K loop of one item overlaps the FP64
// epilogue of the previous one on the same SM.  An item is one 64-row tile:
// row tile i of column j (C = A[i, j] - sum_{p<j} L[i, p] L[j, p]^T, then
// L[i, j] U_j = C solved against the diagonal tile's factor, the forward
// substitution and the int8 slices of L[i, j]), or the diagonal item of a
// slot (D' of tile j + 1, left in dpart for k_diag_next).  Each CTA takes a
// contiguous range of the step's items; nothing waits on another CTA.
//   warp 0 (one thread): bulk copies of the slice half-tiles (K = 32) of the
//     item's row tile and of the column tile row through a kWsStages ring;
//   warp 1 (one thread): the tcgen05 MMAs into one TMEM accumulator;
//   warps 2..9: per item the Wendland tile (during the K loop), the TMEM
//     drain (after which the MMA thread starts the next item), the level
//     combination and the FP64 epilogue.
// The MMA operand A holds two consecutive slices of the ONE row tile (rows
// 0..63 slice a, 64..127 slice a + 1), B the slices of the column tile
// stacked along N.  With the accumulator of pair (a, a+1) starting at TMEM
// column group a - 1, column group g (64 columns) holds level g + 2 in lanes
// 0..63 and level g + 3 in lanes 64..127 whatever the pair, so four pairs
// (1,2), (3,4), (5,6), (7,0) against the column slices 1..9-a and six MMAs
// per K = 32 cover every slice pair with a + b <= 9: levels 2..9 are lanes
// 0..63 of groups 0..7 and lanes 64..127 of groups 0..6 (lanes 64..127 of
// group 7 hold a partial level 10, not read).  In shared memory a K = 32 half
// of the row tile is staged as [K chunk (2)][slice (8)][8-row group (8)][128
// B] with the eighth slice of each chunk kept zero, so that the pair (7, 0)
// adds nothing to lanes 64..127; the column tile's half is the stored layout
// itself ([K chunk (2)][slice (7)]...), one contiguous 14 KB copy.
constexpr int kWsStages = 3;
constexpr int kWsChunk = kOzS * 1024;                    // 7168: one 16-byte K chunk, 7 slices
constexpr int kWsHalf = 2 * kWsChunk;                    // 14336: one K = 32 half of a slice tile
constexpr int kWsChunkA = (kOzS + 1) * 1024;             // staged row-tile chunk with a zero slice
constexpr int kWsHalfA = 2 * kWsChunkA;                  // 16384
constexpr int kWsStage = kWsHalfA + kWsHalf;             // row half + column half
constexpr int kWsThreads = 320;                          // 2 issue warps + 8 epilogue warps
constexpr int kWsCOff = kWsStages * kWsStage;            // C / D (TB x LDS doubles)
constexpr int kWsXOff = kWsCOff + TB * LDS * 8;          // U_j, the diagonal tile's factor
constexpr int kWsLOff = kWsXOff + TB * LDS * 8;          // upper TMEM lanes' level sums
constexpr int kWsPtsOff = kWsLOff + TB * LDS * 8;        // row points (2 x TB), column points
constexpr int kWsRedOff = kWsPtsOff + 2 * TB * 32 + 3 * TB * 8;  // y_j, r_i, diag_tile vectors
constexpr int kWsUiOff = kWsRedOff + 3 * TB * kMaxF * 8;  // U_j's diagonal block inverses
constexpr int kWsBarOff = kWsUiOff + 4 * 16 * kUiLd * 8;
constexpr size_t kWsSmem = size_t(kWsBarOff) + 256;
static_assert(kWsSmem <= 232448, "shared memory of k_col_step_ws");
static_assert(kWsStage % 1024 == 0, "stages start on 1 KB boundaries");
static_assert(kOzTileBytes <= TB * LDS * 8, "slice staging does not fit the C buffer");
static_assert((TB * kMaxF + 2 * TB + TB) * 8 <= 3 * TB * kMaxF * 8, "diag_tile vectors");
static_assert(2 * TB * kMaxF + 3 * TB <= 3 * TB * kMaxF, "residual rows after the diag_tile vectors");

struct WsBars {
  uint64_t full[kWsStages], empty[kWsStages], acc_full, acc_empty, done;
  int abort_flag, ep_stop;
  uint32_t tmem;
};
static_assert(sizeof(WsBars) <= 256, "barrier area");

// The item `it` of step j: slot q (prefix counts ipre over the cnt active
// slots), and r = it - ipre[q]: r == 0 the diagonal item, else row tile j + r.
struct WsItem {
  int q, r;
};
__device__ __forceinline__ WsItem ws_item(const int *ipre, int cnt, int it) {
  const int q = find_slot(ipre, cnt, it);
  return {q, it - ipre[q]};
}
// The items of a CTA's range in order: one binary search for the first,
// then the slot advances when the item passes the next slot's first item
// (the slot record is reloaded only then).
struct WsCursor {
  int q = -1, first = 0, next = 0;
  BigSlot sl;
  int64_t s0 = 0;  // first membership entry of the slot's patch (with soff)
  __device__ __forceinline__ WsItem at(const int *ipre, const BigSlot *slots, const int64_t *soff,
                                       int cnt, int it) {
    if (q < 0 || it >= next) {
      if (q < 0) q = find_slot(ipre, cnt, it);
      else
        do ++q;
        while (it >= ipre[q + 1]);
      first = ipre[q];
      next = ipre[q + 1];
      sl = slots[q];
      if (soff) s0 = soff[sl.k];
    }
    return {q, it - first};
  }
};

// Six MMAs of one K = 32 half: pairs (1,2), (3,4), (5,6), (7,0) of the row
// tile's slices against the column tile's slices 1..9-a stacked along N.  On
// the first half of an item the first MMA to reach a column overwrites it:
// pair (1, 2) groups 0..3, pair (5, 6) groups 4..7, issued first.
__device__ __forceinline__ void ws_mma_half(uint32_t tmem, uint32_t sA, uint32_t sB, bool first) {
  const uint64_t b0 = umma_desc(sB, kWsChunk, 128), b4 = umma_desc(sB + 4 * 1024, kWsChunk, 128);
  const uint32_t acc = first ? 0u : 1u;
  const uint64_t a12 = umma_desc(sA, kWsChunkA, 128);
  const uint64_t a34 = umma_desc(sA + 2 * 1024, kWsChunkA, 128);
  const uint64_t a56 = umma_desc(sA + 4 * 1024, kWsChunkA, 128);
  const uint64_t a70 = umma_desc(sA + 6 * 1024, kWsChunkA, 128);
  umma_i8(tmem, a12, b0, umma_idesc_i8(256), acc);          // (1,2) x 1..4: groups 0..3
  umma_i8(tmem + 256, a56, b0, umma_idesc_i8(256), acc);    // (5,6) x 1..4: groups 4..7
  umma_i8(tmem + 256, a12, b4, umma_idesc_i8(192), 1u);     // (1,2) x 5..7: groups 4..6
  umma_i8(tmem + 128, a34, b0, umma_idesc_i8(256), 1u);     // (3,4) x 1..4: groups 2..5
  umma_i8(tmem + 384, a34, b4, umma_idesc_i8(128), 1u);     // (3,4) x 5..6: groups 6..7
  umma_i8(tmem + 384, a70, b0, umma_idesc_i8(128), 1u);     // (7,0) x 1..2: groups 6..7
}

// Epilogue warp e (warp 2 + e) reads TMEM lanes 32 qd .. + 31 (qd = warp % 4)
// and columns 32 h .. + 31 (h = e / 4) of the column groups: the level sums of
// its half of row r (lanes 0..63: levels 2..9 in groups 0..7, rows r = lane;
// lanes 64..127: levels 3..9 in groups 0..6, rows r = lane - 64).  The levels
// are merged in int64 first: |level| < 2^31, so the top three shifted by 7
// bits each stay below 2^53 and convert exactly, and the lower four or five
// (below 2^60 in units of 128^-9) round to within 2^-57; then two FP64
// terms (in units of sigma^2).  Lanes 0..63
// subtract sig2 x their sum from sC (which holds A); lanes 64..127 store
// theirs in sUp, which the caller subtracts after a barrier.
__device__ __forceinline__ void ws_drain(uint32_t tmem, int qd, int h, double *sC, double *sUp,
                                         double sig2, int lane) {
  constexpr int kG = kOzS + 1;  // column groups 0..7
  const uint32_t lane_base = uint32_t(32 * qd) << 16;
  const bool up = qd >= 2;
  const int ng = up ? kG - 1 : kG;  // upper lanes: group 7 holds a partial level 10
  // Four columns per step: the levels are merged into (hi, lo), the loads of
  // step cb + 1 are issued, and the conversions and stores of step cb run
  // while they are in flight.
  uint32_t z[kG][4];
  auto issue = [&](int cb) {
#pragma unroll
    for (int g = 0; g < kG; ++g) {
      if (g >= ng) break;
      const uint32_t addr = tmem + lane_base + uint32_t(64 * g + 32 * h + 4 * cb);
      asm volatile("tcgen05.ld.sync.aligned.32x32b.x4.b32 {%0,%1,%2,%3}, [%4];\n"
                   : "=r"(z[g][0]), "=r"(z[g][1]), "=r"(z[g][2]), "=r"(z[g][3])
                   : "r"(addr));
    }
  };
  issue(0);
#pragma unroll
  for (int cb = 0; cb < 8; ++cb) {
    asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory");
    long long hi[4], lo[4];
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      const long long z0 = int32_t(z[0][c]), z1 = int32_t(z[1][c]), z2 = int32_t(z[2][c]);
      const long long z3 = int32_t(z[3][c]), z4 = int32_t(z[4][c]), z5 = int32_t(z[5][c]);
      const long long z6 = int32_t(z[6][c]);
      hi[c] = (z0 * 128 + z1) * 128 + z2;
      lo[c] = up ? ((z3 * 128 + z4) * 128 + z5) * 128 + z6
                 : (((z3 * 128 + z4) * 128 + z5) * 128 + z6) * 128 + int32_t(z[7][c]);
    }
    if (cb < 7) issue(cb + 1);
#pragma unroll
    for (int c = 0; c < 4; ++c) {
      // Lower lanes: levels 2..4 and 5..9; upper lanes: 3..5 and 6..9.
      const double val = __fma_rn(double(hi[c]), up ? 0x1p-35 : 0x1p-28, double(lo[c]) * 0x1p-63);
      const int col = 32 * h + 4 * cb + c;
      if (!up) {
        double *cr = sC + (32 * qd + lane) * LDS + col;
        *cr = __fma_rn(-sig2, val, *cr);
      } else {
        sUp[(32 * (qd - 2) + lane) * LDS + col] = val;
      }
    }
  }
}

__device__ __forceinline__ void ws_sync() { asm volatile("bar.sync 1, 256;\n" ::: "memory"); }

// Row points of a tile: thread e < TB loads the membership index of row e
// early (ws_point_index) and copies the point into prow[e] later
// (ws_point_copy, cp.async; zeros past n), so that the next item's points
// arrive while the current item's epilogue runs.
__device__ __forceinline__ int ws_point_index(const BigArgs &a, const BigSlot &sl, int64_t s0,
                                              int ti, int e) {
  const int gi = ti * TB + e;
  return gi < sl.n ? a.sidx[s0 + gi] : -1;
}
__device__ __forceinline__ void ws_point_copy(const BigArgs &a, double4 *prow, int e, int idx) {
  if (idx >= 0) {
    const double *g = reinterpret_cast<const double *>(a.src + idx);
    double *d = reinterpret_cast<double *>(prow + e);
    cp_async16(d, g);
    cp_async16(d + 2, g + 2);
  } else {
    prow[e] = make_double4(0.0, 0.0, 0.0, 0.0);
  }
}
// The evaluation loop of ws_gen_tile for one basis, without branches: thread
// t takes column c = t % 64 of rows t / 64 + 4 m, m = 0..15, and the identity
// padding past n is selected, so that the unrolled evaluations form one block
// whose FP64 chains (23-cycle FMA latency on this GPU) overlap.
template <int B>
__device__ __forceinline__ void ws_gen_rows(const BigArgs &a, const BigSlot &sl, int ti, int tj,
                                            double *sT, const double4 *prow, const double *cpts,
                                            int t) {
  const double *cx = cpts, *cy = cx + TB, *cz = cy + TB;
  const int c = t & 63, gj = tj * TB + c;
  const double px = cx[c], py = cy[c], pz = cz[c];
#pragma unroll 8
  for (int m = 0; m < TB * TB / 256; ++m) {
    const int r = (t >> 6) + 4 * m;
    const int gi = ti * TB + r;
    const double4 pr = prow[r];
    const double w =
        wendland<double>(B, __dsqrt_rn(sqdist3(pr.x, pr.y, pr.z, px, py, pz)), a.rinv);
    const double pad = (gi == gj) ? 1.0 : 0.0;
    sT[r * LDS + c] = (gi < sl.n && gj < sl.n) ? w : pad;
  }
}

// A[ti, tj] of the slot (gen_tile) into sT, by the 256 epilogue threads, from
// the row points in prow (staged and waited for by the caller) and the
// column points in cpts (3 x TB, reloaded when load_cols).
__device__ __forceinline__ void ws_gen_tile(const BigArgs &a, const BigSlot &sl, int64_t s0,
                                            int ti, int tj, double *sT, const double4 *prow,
                                            double *cpts, int t, bool load_cols) {
  double *cx = cpts, *cy = cx + TB, *cz = cy + TB;
  if (load_cols)
    for (int e = t; e < TB; e += 256) {
      const int gj = tj * TB + e;
      double4 p = make_double4(0.0, 0.0, 0.0, 0.0);
      if (gj < sl.n) p = a.src[a.sidx[s0 + gj]];
      cx[e] = p.x;
      cy[e] = p.y;
      cz[e] = p.z;
    }
  ws_sync();
  switch (a.basis) {
  case kWendlandC0: ws_gen_rows<kWendlandC0>(a, sl, ti, tj, sT, prow, cpts, t); break;
  case kWendlandC2: ws_gen_rows<kWendlandC2>(a, sl, ti, tj, sT, prow, cpts, t); break;
  case kWendlandC4: ws_gen_rows<kWendlandC4>(a, sl, ti, tj, sT, prow, cpts, t); break;
  case kWendlandC6: ws_gen_rows<kWendlandC6>(a, sl, ti, tj, sT, prow, cpts, t); break;
  default: ws_gen_rows<kWendlandC8>(a, sl, ti, tj, sT, prow, cpts, t); break;
  }
}

__global__ void __launch_bounds__(kWsThreads, 1)
    k_col_step_ws(BigArgs a, const BigSlot *__restrict__ slots, const int *__restrict__ ipre,
                  int cnt, int j) {
  extern __shared__ __align__(1024) uint8_t smb[];
  WsBars *bar = reinterpret_cast<WsBars *>(smb + kWsBarOff);
  volatile int *abort_flag = &bar->abort_flag;
  const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  const int nitems = ipre[cnt];
  const int it0 = int(int64_t(blockIdx.x) * nitems / gridDim.x);
  const int it1 = int(int64_t(blockIdx.x + 1) * nitems / gridDim.x);
  const int nh = 2 * j;  // K = 32 halves per item
  auto slice_row = [&](const BigSlot &sl, int i) {
    return a.slices + sl.sli + (int64_t(i) * (i - 1) / 2) * kOzTileBytes;
  };
  if (tid == 0) {
    for (int i = 0; i < kWsStages; ++i) {
      mbar_init(&bar->full[i], 1);
      mbar_init(&bar->empty[i], 1);
    }
    mbar_init(&bar->acc_full, 1);
    mbar_init(&bar->acc_empty, 8);
    mbar_init(&bar->done, 1);
    bar->abort_flag = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(
                     saddr(&bar->tmem)),
                 "r"(kOzTmemCols)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  // The zero eighth slice of each staged row-tile chunk, made visible to the
  // tensor core (async proxy); the copies never write it.
  for (int u = tid; u < kWsStages * 2 * 64; u += kWsThreads) {
    const int st = u >> 7, ch = (u >> 6) & 1, w16 = u & 63;
    *reinterpret_cast<uint4 *>(smb + st * kWsStage + ch * kWsChunkA + kWsChunk + 16 * w16) =
        make_uint4(0u, 0u, 0u, 0u);
  }
  asm volatile("fence.proxy.async.shared::cta;\n" ::: "memory");
  tc_fence_before();
  __syncthreads();
  tc_fence_after();
  const uint32_t tmem = bar->tmem;

  if (warp == 0) {
    if (lane == 0) {
      // Producer.
      int hc = 0;
      WsCursor cur;
      for (int it = it0; it < it1 && !*abort_flag; ++it) {
        const WsItem w = cur.at(ipre, slots, nullptr, cnt, it);
        const BigSlot &sl = cur.sl;
        const uint8_t *ra = slice_row(sl, w.r == 0 ? j + 1 : j + w.r);
        const uint8_t *rb = slice_row(sl, w.r == 0 ? j + 1 : j);
        for (int hh = 0; hh < nh; ++hh, ++hc) {
          const int st = hc % kWsStages, u = hc / kWsStages;
          if (hc >= kWsStages &&
              !mbar_wait_pipe(&bar->empty[st], uint32_t((u - 1) & 1), a.wait_limit, abort_flag)) {
            *abort_flag = 1;
            break;
          }
          uint8_t *sA = smb + st * kWsStage;
          const int64_t off = int64_t(hh >> 1) * kOzTileBytes + (hh & 1) * kWsHalf;
          mbar_expect_tx(&bar->full[st], uint32_t(2 * kWsHalf));
          bulk_g2s(sA, ra + off, kWsChunk, &bar->full[st]);
          bulk_g2s(sA + kWsChunkA, ra + off + kWsChunk, kWsChunk, &bar->full[st]);
          bulk_g2s(sA + kWsHalfA, rb + off, kWsHalf, &bar->full[st]);
        }
      }
      // Drain: only the latest use of each stage can still be in flight.
      const int issued = hc;
      for (int st = 0; st < kWsStages && st < issued; ++st) {
        const int last = st + kWsStages * ((issued - 1 - st) / kWsStages);
        if (!mbar_wait(&bar->full[st], uint32_t((last / kWsStages) & 1), kOzDrainLimit))
          *abort_flag = 1;
      }
    }
  } else if (warp == 1) {
    if (lane == 0) {
      // MMA issue.
      int hc = 0, k = 0;
      bool ok = true;
      for (int it = it0; it < it1 && ok; ++it, ++k) {
        // The accumulator is free once the epilogue drained the previous item.
        if (k > 0 && !mbar_wait_pipe(&bar->acc_empty, uint32_t((k - 1) & 1), a.wait_limit,
                                     abort_flag)) {
          ok = false;
          break;
        }
        tc_fence_after();
        for (int hh = 0; hh < nh; ++hh, ++hc) {
          const int st = hc % kWsStages, u = hc / kWsStages;
          if (!mbar_wait_pipe(&bar->full[st], uint32_t(u & 1), a.wait_limit, abort_flag)) {
            ok = false;
            break;
          }
          tc_fence_after();
          const uint32_t sA = saddr(smb + st * kWsStage);
          ws_mma_half(tmem, sA, sA + kWsHalfA, hh == 0);
          umma_commit(&bar->empty[st]);
        }
        if (!ok) break;
        umma_commit(&bar->acc_full);
      }
      if (!ok) *abort_flag = 1;
      umma_commit(&bar->done);  // arrives once every MMA issued above has completed
    }
  } else {
    // Epilogue: 8 warps, etid 0..255.
    const int etid = tid - 64, ew = warp - 2;
    const int qd = warp & 3, h = ew >> 2;
    double *sC = reinterpret_cast<double *>(smb + kWsCOff);
    double *sX = reinterpret_cast<double *>(smb + kWsXOff);
    double *sL = reinterpret_cast<double *>(smb + kWsLOff);
    double4 *prows = reinterpret_cast<double4 *>(smb + kWsPtsOff);              // 2 x TB
    double *cpts = reinterpret_cast<double *>(smb + kWsPtsOff + 2 * TB * 32);  // 3 x TB
    double *ysh = reinterpret_cast<double *>(smb + kWsRedOff);  // TB x kMaxF
    double *rsh = ysh + TB * kMaxF + 3 * TB;                     // r_i, TB x kMaxF
    double *sUi = reinterpret_cast<double *>(smb + kWsUiOff);   // [b][k][c] = U_bb^-1[k][c]
                                                                 // (row stride kUiLd)
    volatile int *ep_stop = &bar->ep_stop;  // written by epilogue threads only
    if (etid == 0) *ep_stop = 0;
    // The step may be launched while the previous launch (k_diag_next of
    // step j - 1, which writes U_j, X_j and y_j and reads dpart) still runs:
    // the copy and MMA warps need only the slices of earlier steps, which
    // the launch before that wrote, but the epilogue waits for it here.
    asm volatile("griddepcontrol.wait;\n" ::: "memory");
    ws_sync();
    int xq = -1;  // slot whose U_j (factor of the diagonal tile, transposed) is in sX
    int pq = -1, ptj = -1;  // slot and column tile whose points are in cpts
    int k = 0;
    WsCursor cur, nxt;  // the item, and the next one (its row points are prefetched)
    int nidx = -1;      // membership index of this thread's row point of the next item
    if (it0 < it1) {
      const WsItem w0 = nxt.at(ipre, slots, a.soff, cnt, it0);
      if (etid < TB)
        ws_point_copy(a, prows, etid,
                      ws_point_index(a, nxt.sl, nxt.s0, w0.r == 0 ? j + 1 : j + w0.r, etid));
    }
    cp_async_commit();
    for (int it = it0; it < it1; ++it, ++k) {
      const WsItem w = cur.at(ipre, slots, a.soff, cnt, it);
      const BigSlot sl = cur.sl;
      const int ld = sl.ld, F = a.F;
      double *W = a.W + sl.base;
      double *rcol = W + int64_t(sl.T) * TB;
      const bool diag = w.r == 0;
      const int i = diag ? j + 1 : j + w.r;
      if (!diag) {
        // U_j (and its block inverses) and y_j once per slot, the
        // residual rows r_i of every item: copied while the tile is made.
        if (xq != w.q) {
          load_factor_async(sX, W + int64_t(j) * TB * ld + int64_t(j) * TB, ld, etid, 256);
          // U_bb^-1 = (X_j's diagonal block b)^T, X_j = L_jj^-1 row-major.
          const double *xg = a.inv + sl.inv + int64_t(j) * TB * TB;
          for (int e = etid; e < 4 * 256; e += 256) {
            const int b = e >> 8, k = (e >> 4) & 15, c = e & 15;
            cp_async8(sUi + (16 * b + k) * kUiLd + c, xg + (16 * b + c) * TB + 16 * b + k);
          }
          const double *yg = rcol + int64_t(j) * TB * ld;
          for (int e = etid; e < TB * F; e += 256)
            cp_async8(ysh + (e / F) * kMaxF + e % F, yg + int64_t(e / F) * ld + e % F);
          xq = w.q;
        }
        const double *rg = rcol + int64_t(i) * TB * ld;
        for (int e = etid; e < TB * F; e += 256)
          cp_async8(rsh + (e / F) * kMaxF + e % F, rg + int64_t(e / F) * ld + e % F);
      }
      cp_async_commit();
      // A[i, j] (or A[j+1, j+1]) while the MMAs of this item run, once the
      // row points (the group before the one just committed) have landed;
      // the column points stay in cpts while the slot and column tile do.
      cp_async_wait<1>();
      const int tj = diag ? j + 1 : j;
      ws_gen_tile(a, sl, cur.s0, i, tj, sC, prows + (k & 1) * TB, cpts, etid,
                  pq != w.q || ptj != tj);
      pq = w.q;
      ptj = tj;
      ws_sync();
      // Drain the accumulator, then hand it back to the MMA thread.
      // Every epilogue thread waits; the decision to stop is made uniform
      // through ep_stop (the global abort flag may change at any time).
      if (!mbar_wait_pipe(&bar->acc_full, uint32_t(k & 1), a.wait_limit, abort_flag)) *ep_stop = 1;
      ws_sync();
      if (*ep_stop) {
        *abort_flag = 1;
        break;
      }
      tc_fence_after();
      // C = A - sigma^2 (lower-lane levels + upper-lane levels): sC gets A
      // minus the lower lanes' sums, sL the upper lanes' sums.  At j = 0
      // there are no products (no MMAs were issued) and C = A.
      if (j > 0) ws_drain(tmem, qd, h, sC, sL, a.oz_sig2, lane);
      tc_fence_before();
      __syncwarp();
      if (lane == 0) mbar_arrive_cnt(&bar->acc_empty, 1);
      ws_sync();
      // The next item's membership indices, loaded while this one finishes.
      if (it + 1 < it1 && etid < TB) {
        const WsItem wn = nxt.at(ipre, slots, a.soff, cnt, it + 1);
        nidx = ws_point_index(a, nxt.sl, nxt.s0, wn.r == 0 ? j + 1 : j + wn.r, etid);
      }
      // C = sC - sigma^2 sL is formed where it is read: by the diagonal
      // item's copy, or by the triangular solve's loads.  The copies of the
      // next item's row points go out as one commit group per item.
      auto next_points = [&]() {
        if (it + 1 < it1) {
          if (etid < TB) ws_point_copy(a, prows + ((k + 1) & 1) * TB, etid, nidx);
          cp_async_commit();
        }
      };
      if (diag) {
        // D' to dpart, where the next launch (k_diag_next) factors D.
        double *dst = a.dpart + int64_t(sl.q) * TB * TB;
        for (int e = etid; e < TB * TB; e += 256) {
          const int o = (e >> 6) * LDS + (e & 63);
          dst[e] = j > 0 ? __fma_rn(-a.oz_sig2, sL[o], sC[o]) : sC[o];
        }
        next_points();
      } else {
        // L[i, j] U_j = C by blocked row solves (warp ew: rows 8 ew .. + 7),
        // stored; forward substitution; int8 slices.
        cp_async_wait<0>();
        ws_sync();
        const int r0 = 8 * ew;
        warp_rows_trsm8_bi(sC + r0 * LDS, sX, sUi, lane, j > 0 ? sL + r0 * LDS : nullptr,
                           a.oz_sig2);
        next_points();
        double lo[8], hi[8];
#pragma unroll
        for (int q = 0; q < 8; ++q) {
          lo[q] = sC[(r0 + q) * LDS + lane];
          hi[q] = sC[(r0 + q) * LDS + 32 + lane];
        }
        {
          double *Lg = W + int64_t(i) * TB * ld + int64_t(j) * TB;
          double *rg = rcol + int64_t(i) * TB * ld;
#pragma unroll
          for (int q = 0; q < 8; ++q) {
            Lg[int64_t(r0 + q) * ld + lane] = lo[q];
            Lg[int64_t(r0 + q) * ld + 32 + lane] = hi[q];
          }
          for (int f = 0; f < F; ++f) {
            const double yl = ysh[lane * kMaxF + f], yh = ysh[(lane + 32) * kMaxF + f];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
              double sum = __fma_rn(lo[q], yl, hi[q] * yh);
              for (int o = 16; o > 0; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
              if (lane == 0) rg[int64_t(r0 + q) * ld + f] = rsh[(r0 + q) * kMaxF + f] - sum;
            }
          }
        }
        ws_sync();
        {
          uint8_t *dst = slice_row(sl, i) + int64_t(j) * kOzTileBytes;
          slice_tile_smem(sC, TB, a.oz_mul, dst, dst, etid, 256);
        }
      }
      ws_sync();
    }
    cp_async_wait<0>();
  }
  __syncthreads();
  if (!mbar_wait(&bar->done, 0u, kOzDrainLimit)) *abort_flag = 1;
  tc_fence_after();
  __syncthreads();
  // After a time-out, the patches of every item of this CTA's range are
  // marked for the FP64 LU.
  if (*abort_flag)
    for (int it = it0 + tid; it < it1; it += kWsThreads)
      atomicOr(&a.status[slots[ws_item(ipre, cnt, it).q].k], 8);
  tc_fence_before();
  __syncthreads();
  if (warp == 0)
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(tmem),
                 "r"(kOzTmemCols)
                 : "memory");
}

// Backward sweep L^T z = y of one slot (CTA per slot), tile row by tile row
// from the last: z_s = X_s^T (y_s - sum_{t>s} L[t, s]^T z_t), with the tile
// inverses X_s of the factorisation.  The sweep is a chain of T dependent
// levels, so the time of a large slot is set by how fast its tiles reach the
// SM: warp 8 streams them with 16-byte cp.async (one 512-byte row per
// instruction, completion counted on an mbarrier), in sweep order and
// independent of z, through a ring of kBkStages 32 KB stages (the tiles
// L[t, s], t > s, then X_s), up to kBkStages tiles ahead of the arithmetic.
// (Bulk copies of the 512-byte rows were slower: the per-request cost of the
// bulk-copy engine capped one SM near 20 GB/s.)  Warps 0..7 take the L tiles of a
// level in turn (lane: two columns r of the tile, all rows c), then meet to
// finish z_s.  z goes to zc (per slot) and, in the forward, to alpha_c per
// (patch, source).  Every wait is bounded; a time-out marks the patch
// (status 8), the CTA keeps its barrier sequence, stops issuing copies and
// waits for the copies it issued before it returns.
constexpr int kBkTile = TB * TB * 8;  // bytes of one stage
// Ring depth: 3 stages for one or two fields, two CTAs per SM (the many short
// slots are latency-bound, and a second CTA hides it); 5 stages, one CTA per
// SM, for more fields (registers).
constexpr int bk_stages(int F) { return F <= 2 ? 3 : 5; }

size_t chol_back_smem(int F, int S = 0) {
  // stages, part, accs, full/empty barriers, abort flag and issue counter
  if (S == 0) S = bk_stages(F);
  return size_t(S) * kBkTile + size_t(8 * TB * F + TB * F) * 8 + 2 * S * 8 + 16;
}
// The deep ring of the one-field backward sweep (one CTA per SM, twice the
// tiles in flight): a slot's sweep streams its T (T - 1) / 2 tiles through
// one SM, so the largest slots' sweeps are set by the bytes one SM keeps in
// flight (PACMAN_B200_BACK_STAGES = 6 selects it).
constexpr int kBkDeep = 6;


// Bounded wait for a phase that gives up early once the CTA has aborted.
__device__ __forceinline__ bool mbar_wait_abort(uint64_t *b, uint32_t parity,
                                                volatile int *abort_flag) {
  return mbar_wait_pipe(b, parity, kOzWaitLimit, abort_flag);
}

// One 64 x 64 FP64 tile (rows ld doubles apart) into a pipeline stage by the
// 32 lanes of a warp, 16-byte cp.async each (row r: the lane's 16 bytes, so
// every instruction moves one 512-byte row); the stage's full barrier
// (initialised to 32 arrivals) counts this lane once its copies have landed.
__device__ __forceinline__ void warp_tile_g2s(double *dst, const double *src, int64_t ld,
                                              int lane, uint64_t *full) {
#pragma unroll 8
  for (int r = 0; r < TB; ++r) cp_async16(dst + r * TB + 2 * lane, src + r * ld + 2 * lane);
  asm volatile("cp.async.mbarrier.arrive.noinc.shared::cta.b64 [%0];\n" ::"r"(saddr(full))
               : "memory");
}

// Bounded wait until item x is issued, then for its data.
template <int kBkStages>
__device__ __forceinline__ bool bk_wait_item(volatile int *issued, volatile int *abort_flag,
                                             uint64_t *full, int x) {
  bool ok = false;
  for (int it = 0; it < kOzWaitLimit && !ok; ++it) {
    ok = *issued > x;
    if (*abort_flag) return false;
  }
  return ok && mbar_wait_abort(&full[x % kBkStages], uint32_t((x / kBkStages) & 1), abort_flag);
}

template <int KF, int kBkStages>  // fields held in registers (F <= KF), ring depth
__global__ void __launch_bounds__(288, kBkStages == 3 ? 2 : 1)
    k_chol_back(BigArgs a, const BigSlot *__restrict__ slots) {
  extern __shared__ __align__(128) uint8_t smem[];
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double *stage0 = reinterpret_cast<double *>(smem);
  double *part = reinterpret_cast<double *>(smem + size_t(kBkStages) * kBkTile);  // [8][TB][F]
  double *accs = part + 8 * TB * F;                                                // [TB][F]
  uint64_t *full = reinterpret_cast<uint64_t *>(accs + TB * F);
  uint64_t *empty = full + kBkStages;
  volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + kBkStages);
  // Items the producer has issued.  A consumer waits on the full barrier of
  // item x only once x is issued: x - kBkStages, the previous item of that
  // stage, has then landed and been released, so the barrier is in the
  // phase of x and the parity wait cannot match an older phase.
  volatile int *issued = abort_flag + 1;
  const int ld = sl.ld, T = sl.T;
  const double *W = a.W + sl.base;
  const double *rcol = W + int64_t(T) * TB;
  const double *X0 = a.inv + sl.inv;
  double *zc = a.zc + sl.zoff;
  if (tid == 0) {
    for (int i = 0; i < kBkStages; ++i) {
      mbar_init(&full[i], 32);  // one arrival per producer lane
      mbar_init(&empty[i], 8);
    }
    *abort_flag = 0;
    *issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (warp == 8) {
    // Producer: item g of the stream goes to stage g % kBkStages.
    int g = 0;
    bool ok = true;
    for (int s = T - 1; s >= 0 && ok; --s) {
      for (int t = s + 1; t <= T && ok; ++t, ++g) {  // t == T: X_s
        const int st = g % kBkStages, u = g / kBkStages;
        if (g >= kBkStages) {
          if (lane == 0) ok = mbar_wait_abort(&empty[st], uint32_t((u - 1) & 1), abort_flag);
          ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
          if (!ok) break;
        }
        double *dst = reinterpret_cast<double *>(smem + size_t(st) * kBkTile);
        if (t < T)
          warp_tile_g2s(dst, W + int64_t(t) * TB * ld + int64_t(s) * TB, ld, lane, &full[st]);
        else
          warp_tile_g2s(dst, X0 + int64_t(s) * TB * TB, TB, lane, &full[st]);
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          *issued = g + 1;
        }
      }
    }
    if (!ok && lane == 0) {
      *abort_flag = 1;
      atomicOr(&a.status[sl.k], 8);
    }
    // Wait (bounded) for every issued copy: the latest item of each stage.
    if (lane == 0)
      for (int st = 0; st < kBkStages && st < g; ++st) {
        const int last = st + kBkStages * ((g - 1 - st) / kBkStages);
        mbar_wait(&full[st], uint32_t((last / kBkStages) & 1));
      }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  } else {
    int g = 0;
    const int rr = tid & 63, quarter = tid >> 6;
    for (int s = T - 1; s >= 0; --s) {
      const int nt = T - 1 - s;
      double acc0[KF], acc1[KF];
#pragma unroll
      for (int f = 0; f < KF; ++f) acc0[f] = acc1[f] = 0.0;
      // z_t of the warp's next tile, one coalesced load per lane and field
      // (rows lane and lane + 32), issued before the wait for the tile; the
      // rows c are then broadcast from the lanes by shuffles.
      double zn0[KF], zn1[KF];
      if (warp < nt) {
        const double *zt = zc + int64_t(s + 1 + warp) * TB * F;
#pragma unroll
        for (int f = 0; f < KF; ++f) {
          zn0[f] = f < F ? zt[lane * F + f] : 0.0;
          zn1[f] = f < F ? zt[(lane + 32) * F + f] : 0.0;
        }
      }
      for (int k = warp; k < nt; k += 8) {
        const int gi = g + k, st = gi % kBkStages;
        double z0[KF], z1[KF];
#pragma unroll
        for (int f = 0; f < KF; ++f) {
          z0[f] = zn0[f];
          z1[f] = zn1[f];
        }
        if (k + 8 < nt) {
          const double *zt = zc + int64_t(s + 1 + k + 8) * TB * F;
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) {
              zn0[f] = zt[lane * F + f];
              zn1[f] = zt[(lane + 32) * F + f];
            }
        }
        bool ok = !*abort_flag;
        if (ok) ok = bk_wait_item<kBkStages>(issued, abort_flag, full, gi);
        if (!ok) {
          *abort_flag = 1;
          continue;
        }
        const double *tile = stage0 + size_t(st) * TB * TB;
#pragma unroll 8
        for (int c = 0; c < TB; ++c) {
          const double l0 = tile[c * TB + lane], l1 = tile[c * TB + lane + 32];
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) {
              const double z = __shfl_sync(0xffffffffu, c < 32 ? z0[f] : z1[f], c & 31);
              acc0[f] = __fma_rn(l0, z, acc0[f]);
              acc1[f] = __fma_rn(l1, z, acc1[f]);
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_cnt(&empty[st], 8);
      }
      g += nt;
#pragma unroll
      for (int f = 0; f < KF; ++f)
        if (f < F) {
          part[(warp * TB + lane) * F + f] = acc0[f];
          part[(warp * TB + lane + 32) * F + f] = acc1[f];
        }
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      for (int e = tid; e < TB * F; e += 256) {
        const int r = e / F, f = e % F;
        double sum = 0.0;
#pragma unroll
        for (int w = 0; w < 8; ++w) sum += part[(w * TB + r) * F + f];
        accs[r * F + f] = rcol[int64_t(s * TB + r) * ld + f] - sum;
      }
      // X_s: every consumer warp reads it, each releases one of 8 arrivals.
      const int st = g % kBkStages;
      bool okx = !*abort_flag;
      if (okx) okx = bk_wait_item<kBkStages>(issued, abort_flag, full, g);
      if (!okx) *abort_flag = 1;
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      // z_s[rr][f] = sum_{c >= rr} X_s[c][rr] acc_s[c][f]; quarters of c, then summed.
      const double *xs = stage0 + size_t(st) * TB * TB;
      double zp[KF];
#pragma unroll
      for (int f = 0; f < KF; ++f) zp[f] = 0.0;
      if (okx) {
#pragma unroll 4
        for (int c = quarter; c < TB; c += 4) {
          if (c < rr) continue;
          const double x = xs[c * TB + rr];
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) zp[f] = __fma_rn(x, accs[c * F + f], zp[f]);
        }
      }
      __syncwarp();
      if (lane == 0 && okx) mbar_arrive_cnt(&empty[st], 1);
      g += 1;
#pragma unroll
      for (int f = 0; f < KF; ++f)
        if (f < F) part[(quarter * TB + rr) * F + f] = zp[f];
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      for (int e = tid; e < TB * F; e += 256) {
        const int r = e / F, f = e % F;
        const double z = part[(0 * TB + r) * F + f] + part[(1 * TB + r) * F + f] +
                         part[(2 * TB + r) * F + f] + part[(3 * TB + r) * F + f];
        const int j = s * TB + r;
        zc[int64_t(j) * F + f] = z;
        if (a.alpha_c != nullptr && j < sl.n) a.alpha_c[(a.soff[sl.k] + j) * F + f] = z;
      }
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
    }
    if (tid == 0 && *abort_flag) atomicOr(&a.status[sl.k], 8);
  }
  __syncthreads();
}

// Forward sweep L y = r of one slot from kept factors (CTA per slot), for
// an execute that reuses the factorisation: y_s = X_s (r_s - sum_{t<s}
// L[s, t] y_t), tile row by tile row from the first, with the tile inverses
// X_s of the factorisation.  r is the residual column (first F columns of
// column tile T) and is overwritten with y, as the factorising steps leave
// it.  Warp 8 streams the tiles L[s, t], t < s, then X_s, through the same
// cp.async ring as k_chol_back; every consumer warp reads
// every tile: warp w owns rows 8w .. 8w + 7 and its lanes the columns c and
// c + 32, so the partial sums stay in registers until the level ends.
template <int KF, int kBkStages>  // fields held in registers (F <= KF), ring depth
__global__ void __launch_bounds__(288, kBkStages == 3 ? 2 : 1)
    k_chol_fwd(BigArgs a, const BigSlot *__restrict__ slots) {
  extern __shared__ __align__(128) uint8_t smem[];
  const BigSlot sl = slots[blockIdx.x];
  const int F = a.F, tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
  double *stage0 = reinterpret_cast<double *>(smem);
  double *accs = reinterpret_cast<double *>(smem + size_t(kBkStages) * kBkTile);  // [TB][F]
  uint64_t *full = reinterpret_cast<uint64_t *>(accs + 9 * TB * F);
  uint64_t *empty = full + kBkStages;
  volatile int *abort_flag = reinterpret_cast<volatile int *>(empty + kBkStages);
  volatile int *issued = abort_flag + 1;  // as in k_chol_back
  const int ld = sl.ld, T = sl.T;
  const double *W = a.W + sl.base;
  double *rcol = a.W + sl.base + int64_t(T) * TB;
  const double *X0 = a.inv + sl.inv;
  if (tid == 0) {
    for (int i = 0; i < kBkStages; ++i) {
      mbar_init(&full[i], 32);  // one arrival per producer lane
      mbar_init(&empty[i], 8);
    }
    *abort_flag = 0;
    *issued = 0;
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  __syncthreads();
  if (warp == 8) {
    int g = 0;
    bool ok = true;
    for (int s = 0; s < T && ok; ++s) {
      for (int t = 0; t <= s && ok; ++t, ++g) {  // t == s: X_s
        const int st = g % kBkStages, u = g / kBkStages;
        if (g >= kBkStages) {
          if (lane == 0) ok = mbar_wait_abort(&empty[st], uint32_t((u - 1) & 1), abort_flag);
          ok = __shfl_sync(0xffffffffu, ok ? 1 : 0, 0) != 0;
          if (!ok) break;
        }
        double *dst = reinterpret_cast<double *>(smem + size_t(st) * kBkTile);
        if (t < s)
          warp_tile_g2s(dst, W + int64_t(s) * TB * ld + int64_t(t) * TB, ld, lane, &full[st]);
        else
          warp_tile_g2s(dst, X0 + int64_t(s) * TB * TB, TB, lane, &full[st]);
        __syncwarp();
        if (lane == 0) {
          __threadfence_block();
          *issued = g + 1;
        }
      }
    }
    if (!ok && lane == 0) {
      *abort_flag = 1;
      atomicOr(&a.status[sl.k], 8);
    }
    if (lane == 0)
      for (int st = 0; st < kBkStages && st < g; ++st) {
        const int last = st + kBkStages * ((g - 1 - st) / kBkStages);
        mbar_wait(&full[st], uint32_t((last / kBkStages) & 1));
      }
    asm volatile("cp.async.wait_all;\n" ::: "memory");
  } else {
    int g = 0;
    const int r0 = 8 * warp;
    for (int s = 0; s < T; ++s) {
      double part[8][KF];
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int f = 0; f < KF; ++f) part[r][f] = 0.0;
      // y_t of the lane's columns, loaded one tile ahead of its use.
      double yn0[KF], yn1[KF];
#pragma unroll
      for (int f = 0; f < KF; ++f) {
        yn0[f] = (s > 0 && f < F) ? rcol[int64_t(lane) * ld + f] : 0.0;
        yn1[f] = (s > 0 && f < F) ? rcol[int64_t(lane + 32) * ld + f] : 0.0;
      }
      for (int t = 0; t < s; ++t, ++g) {
        double y0[KF], y1[KF];
#pragma unroll
        for (int f = 0; f < KF; ++f) {
          y0[f] = yn0[f];
          y1[f] = yn1[f];
        }
        if (t + 1 < s) {
          const double *yt = rcol + int64_t(t + 1) * TB * ld;
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) {
              yn0[f] = yt[int64_t(lane) * ld + f];
              yn1[f] = yt[int64_t(lane + 32) * ld + f];
            }
        }
        bool ok = !*abort_flag;
        if (ok) ok = bk_wait_item<kBkStages>(issued, abort_flag, full, g);
        if (!ok) {
          *abort_flag = 1;
          continue;
        }
        const double *tile = stage0 + size_t(g % kBkStages) * TB * TB;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const double l0 = tile[(r0 + r) * TB + lane], l1 = tile[(r0 + r) * TB + lane + 32];
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) part[r][f] = __fma_rn(l1, y1[f], __fma_rn(l0, y0[f], part[r][f]));
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_cnt(&empty[g % kBkStages], 1);
      }
      // acc_s = r_s - sum over the level, rows of this warp.
#pragma unroll
      for (int r = 0; r < 8; ++r)
#pragma unroll
        for (int f = 0; f < KF; ++f)
          if (f < F) {
            double v = part[r][f];
            for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
            if (lane == 0) accs[(r0 + r) * F + f] = rcol[int64_t(s * TB + r0 + r) * ld + f] - v;
          }
      bool okx = !*abort_flag;
      if (okx) okx = bk_wait_item<kBkStages>(issued, abort_flag, full, g);
      if (!okx) *abort_flag = 1;
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
      // y_s[rr] = sum_{c <= rr} X_s[rr][c] acc_s[c], rows rr of this warp.
      if (okx) {
        const double *xs = stage0 + size_t(g % kBkStages) * TB * TB;
#pragma unroll
        for (int r = 0; r < 8; ++r) {
          const int rr = r0 + r;
          const double x0 = lane <= rr ? xs[rr * TB + lane] : 0.0;
          const double x1 = lane + 32 <= rr ? xs[rr * TB + lane + 32] : 0.0;
#pragma unroll
          for (int f = 0; f < KF; ++f)
            if (f < F) {
              double v = __fma_rn(x1, accs[(lane + 32) * F + f], x0 * accs[lane * F + f]);
              for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
              if (lane == 0) rcol[int64_t(s * TB + rr) * ld + f] = v;
            }
        }
        __syncwarp();
        if (lane == 0) mbar_arrive_cnt(&empty[g % kBkStages], 1);
      }
      g += 1;
      asm volatile("bar.sync 1, 256;\n" ::: "memory");
    }
    if (tid == 0 && *abort_flag) atomicOr(&a.status[sl.k], 8);
  }
  __syncthreads();
}

size_t chol_fwd_smem(int F) {
  // stages, accs (with room), full/empty barriers, abort flag and issue counter
  const int S = bk_stages(F);
  return size_t(S) * kBkTile + size_t(9 * TB * F) * 8 + 2 * S * 8 + 16;
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
  // Items of the warp-specialised int8 step: T - j per slot (its diagonal
  // item, then its row tiles j + 1 .. T - 1).
  cp.ioff.resize(steps);
  for (int j = 0; j < steps; ++j) {
    const int c = cp.cnt[j];
    cp.ioff[j] = int(cp.pre.size());
    int64_t acc = 0;
    cp.pre.push_back(0);
    for (int q = 0; q < c; ++q) {
      acc += slots[q].T - j;
      cp.pre.push_back(int(acc));
    }
    if (acc > 0x7fffffffll) throw Error{PACMAN_B200_ERR_LIMIT, "too many tiles in one launch"};
  }
  return cp;
}

void chol_set_smem_attributes() {
  static bool done = false;
  if (done) return;
  PB_CUDA(cudaFuncSetAttribute(k_col_step<false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kColSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_col_step<true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kColSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_col_step_ws, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kWsSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_diag_chol, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kDiagSmem)));
  PB_CUDA(cudaFuncSetAttribute(k_diag_next, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(kDiagNextSmem)));
  {
#define PB_SWEEP_ATTR(K, F)                                                                   \
  PB_CUDA(cudaFuncSetAttribute(K<F, bk_stages(F)>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                               int(std::max(chol_back_smem(F), chol_fwd_smem(F)))))
    PB_SWEEP_ATTR(k_chol_back, 1);
    PB_CUDA(cudaFuncSetAttribute(k_chol_back<1, kBkDeep>,
                                 cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(chol_back_smem(1, kBkDeep))));
    PB_SWEEP_ATTR(k_chol_back, 2);
    PB_SWEEP_ATTR(k_chol_back, 4);
    PB_SWEEP_ATTR(k_chol_back, kMaxF);
    PB_SWEEP_ATTR(k_chol_fwd, 1);
    PB_SWEEP_ATTR(k_chol_fwd, 2);
    PB_SWEEP_ATTR(k_chol_fwd, 4);
    PB_SWEEP_ATTR(k_chol_fwd, kMaxF);
#undef PB_SWEEP_ATTR
  }
  done = true;
}

void chol_launch_steps(const BigArgs &a, const BigSlot *ds, const std::vector<BigSlot> &hs,
                       const CholPlan &cp, const int *dpre, cudaStream_t st, SolveReport &rep,
                       cudaEvent_t tail_event) {
  if (cp.ns == 0) return;
  k_diag_chol<<<cp.ns, 256, kDiagSmem, st>>>(a, ds, 0);
  note_launch();
  const int steps = int(cp.cnt.size());
  const Tuning &tu = tuning_for_current_device();
  const int sms = tu.sms;
  // First step on the int8 tensor cores: tuned, PACMAN_B200_INT8_FROM overrides.
  const int oz_from = std::max(0, tuned_int("PACMAN_B200_INT8_FROM", tu.int8_from));
  bool tail = tail_event == nullptr;
  for (int j = 0; j < steps; ++j) {
    const int c = cp.cnt[j];
    const int n = c + cp.pre[cp.off[j] + c];
    if (!tail && n < 2 * sms) {  // from here on the steps leave SMs idle
      PB_CUDA(cudaEventRecord(tail_event, st));
      tail = true;
    }
    SolveReport::TimedLaunch tl{};
    if (rep.time_kernels) {
      PB_CUDA(cudaEventCreate(&tl.e0));
      PB_CUDA(cudaEventCreate(&tl.e1));
      PB_CUDA(cudaEventRecord(tl.e0, st));
    }
    // With int8 slices: the FP64 kernel (two CTAs per SM) for the short K
    // loops of the first steps, writing the slices; the int8 kernel after.
    const bool i8 = a.slices != nullptr && j >= oz_from;
    if (a.slices == nullptr)
      k_col_step<false><<<n, kColThreads, kColSmem, st>>>(a, ds, dpre + cp.off[j], c, j);
    else if (!i8)
      k_col_step<true><<<n, kColThreads, kColSmem, st>>>(a, ds, dpre + cp.off[j], c, j);
    else {
      const int items = cp.pre[cp.ioff[j] + c];
      // Programmatic dependent launch: the step's copies and MMAs overlap
      // the tail of the previous k_diag_next (see griddepcontrol.wait in the
      // kernel); without kernel timing, where events separate the launches.
      cudaLaunchConfig_t cfg = {};
      cfg.gridDim = dim3(std::min(items, sms));
      cfg.blockDim = dim3(kWsThreads);
      cfg.dynamicSmemBytes = kWsSmem;
      cfg.stream = st;
      cudaLaunchAttribute attr[1];
      attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
      attr[0].val.programmaticStreamSerializationAllowed = rep.time_kernels ? 0 : 1;
      cfg.attrs = attr;
      cfg.numAttrs = 1;
      PB_CUDA(cudaLaunchKernelEx(&cfg, k_col_step_ws, a, ds, static_cast<const int *>(dpre + cp.ioff[j]), c, j));
      note_launch();
      k_diag_next<<<c, 256, kDiagNextSmem, st>>>(a, ds, j);
    }
    note_launch();
    if (rep.time_kernels) {
      PB_CUDA(cudaEventRecord(tl.e1, st));
      // Tile products: (T - j - 1) row tiles x (j + 1) (update + solve), and
      // j + 1 for the next diagonal tile.
      tl.kind = i8 ? 1 : 0;
      for (int q = 0; q < c; ++q) {
        tl.flops += 2.0 * TB * TB * TB * double(hs[q].T - j) * double(j + 1);
        if (i8) tl.mma_products += double(hs[q].T - j) * double(j);
      }
      rep.timed.push_back(tl);
    }
  }
  if (!tail) PB_CUDA(cudaEventRecord(tail_event, st));
}

void finish_kernel_timing(SolveReport &rep, cudaEvent_t ref) {
  if (rep.timed.empty()) return;
  // Intervals [start, end) in ms after ref, per kind and for both kinds; the
  // span is the length of their union (launches of different slot groups
  // overlap in time on their own streams).
  std::vector<std::pair<double, double>> iv[3];
  for (const auto &t : rep.timed) {
    float a0 = 0.f, a1 = 0.f;
    PB_CUDA(cudaEventElapsedTime(&a0, ref, t.e0));
    PB_CUDA(cudaEventElapsedTime(&a1, ref, t.e1));
    iv[t.kind].push_back({a0, a1});
    iv[2].push_back({a0, a1});
    rep.flops_kind[t.kind] += t.flops;
    rep.mma_products_i8 += t.mma_products;
    rep.launches_kind[t.kind] += 1;
    rep.update_flops += t.flops;
    rep.update_launches += 1;
    cudaEventDestroy(t.e0);
    cudaEventDestroy(t.e1);
  }
  rep.timed.clear();
  double span[3] = {0.0, 0.0, 0.0};
  for (int k = 0; k < 3; ++k) {
    std::sort(iv[k].begin(), iv[k].end());
    double cs = 0.0, ce = -1.0;
    bool open = false;
    for (const auto &x : iv[k]) {
      if (!open || x.first > ce) {
        if (open) span[k] += ce - cs;
        cs = x.first;
        ce = x.second;
        open = true;
      } else if (x.second > ce) {
        ce = x.second;
      }
    }
    if (open) span[k] += ce - cs;
  }
  rep.ms_kind[0] += span[0];
  rep.ms_kind[1] += span[1];
  rep.ms_update += span[2];
}

void chol_launch_finish(const BigArgs &a, const BigSlot *ds, int ns, bool adjoint,
                        cudaStream_t st) {
  const size_t smem = chol_back_smem(a.F);
  const bool deep = tuned_int("PACMAN_B200_BACK_STAGES", tuning_for_current_device().back_stages) ==
                    kBkDeep;
  if (a.F == 1 && deep)
    k_chol_back<1, kBkDeep><<<ns, 288, chol_back_smem(1, kBkDeep), st>>>(a, ds);
  else if (a.F == 1) k_chol_back<1, bk_stages(1)><<<ns, 288, smem, st>>>(a, ds);
  else if (a.F <= 2) k_chol_back<2, bk_stages(2)><<<ns, 288, smem, st>>>(a, ds);
  else if (a.F <= 4) k_chol_back<4, bk_stages(4)><<<ns, 288, smem, st>>>(a, ds);
  else k_chol_back<kMaxF, bk_stages(kMaxF)><<<ns, 288, smem, st>>>(a, ds);
  note_launch();
  if (!adjoint) {
    k_chol_eval<<<ns, 256, 0, st>>>(a, ds);
    note_launch();
  }
}

void chol_launch_forward(const BigArgs &a, const BigSlot *ds, int ns, cudaStream_t st) {
  const size_t smem = chol_fwd_smem(a.F);
  if (a.F == 1) k_chol_fwd<1, bk_stages(1)><<<ns, 288, smem, st>>>(a, ds);
  else if (a.F <= 2) k_chol_fwd<2, bk_stages(2)><<<ns, 288, smem, st>>>(a, ds);
  else if (a.F <= 4) k_chol_fwd<4, bk_stages(4)><<<ns, 288, smem, st>>>(a, ds);
  else k_chol_fwd<kMaxF, bk_stages(kMaxF)><<<ns, 288, smem, st>>>(a, ds);
  note_launch();
}

size_t oz_slot_bytes(int T) { return size_t(T) * size_t(T - 1) / 2 * size_t(kOzTileBytes); }

}  // namespace pacman_b200
