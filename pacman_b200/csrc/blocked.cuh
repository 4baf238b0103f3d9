// Shared pieces of the blocked engine for large patches (blocked.cu: LU and
// the shared assembly/polynomial kernels; cholesky.cu: the left-looking
// Cholesky factorisation): tile geometry, slot records, launch arguments and
// the FP64 tensor-core tile product.
#pragma once

#include <cstdint>
#include <vector>

#include "plan.hpp"
#include "poly.cuh"

namespace pacman_b200 {

constexpr int TB = 64;   // tile size
constexpr int LDS = 68;  // shared-memory row stride (doubles): conflict-free fragments
constexpr int kUiLd = 20;  // row stride (doubles) of the 16 x 16 block inverses in shared memory

struct BigSlot {
  int64_t base;  // offset (doubles) of the augmented matrix in the workspace
  int ld;        // row stride (doubles) = (T + 1) * TB
  int T;         // pivot tiles
  int TE;        // evaluation-row tiles
  int k;         // patch id
  int n, m;
  int64_t inv;   // offset (doubles) of the slot's inverse tiles
  int q;         // index of the slot in its wave (per-slot arrays beta, act, red)
  int64_t zoff;  // offset (doubles) of the slot's backward-sweep solution in zc
  int64_t sli;   // offset (bytes) of the slot's int8 slice tiles in slices
};

// Work of one launch is addressed by blockIdx.x through prefix counts over
// the active slots (slots are sorted by decreasing T, so the slots still
// active at step s are 0..cnt-1): pre[q] <= blockIdx.x < pre[q + 1].
__device__ __forceinline__ int find_slot(const int *__restrict__ pre, int cnt, int b) {
  int lo = 0, hi = cnt;
  while (hi - lo > 1) {
    const int mid = (lo + hi) >> 1;
    if (pre[mid] <= b) lo = mid;
    else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// FP64 tensor-core tile product
// ---------------------------------------------------------------------------

__device__ __forceinline__ void dmma(double &d0, double &d1, double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d0), "+d"(d1)
               : "d"(a), "d"(b));
}

// acc += sign * op(A) op(B) on the 32 x 32 block (wr, wc) of a 64 x 64 tile.
// Fragment layout of m8n8k4.f64: A (row) a0 = A[g][t], B (col) b0 = B[t][g],
// C c_h = C[g][2t + h], with g = lane / 4, t = lane % 4.
template <bool AT, bool BT>
__device__ __forceinline__ void mma64(const double *__restrict__ sA, const double *__restrict__ sB,
                                      double (&acc)[4][4][2], double sign, int wr, int wc,
                                      int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll 2
  for (int k0 = 0; k0 < TB; k0 += 4) {
    const int kk = k0 + t;
    double a[4], b[4];
#pragma unroll
    for (int i = 0; i < 4; ++i) {
      const int r = wr + 8 * i + g;
      a[i] = sign * (AT ? sA[kk * LDS + r] : sA[r * LDS + kk]);
    }
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int c = wc + 8 * j + g;
      b[j] = BT ? sB[c * LDS + kk] : sB[kk * LDS + c];
    }
#pragma unroll
    for (int i = 0; i < 4; ++i)
#pragma unroll
      for (int j = 0; j < 4; ++j) dmma(acc[i][j][0], acc[i][j][1], a[i], b[j]);
  }
}

__device__ __forceinline__ void load_tile(double *s, const double *g, int ld, int tid, int nt) {
  for (int idx = tid; idx < TB * TB / 2; idx += nt) {
    const int r = idx >> 5, c2 = idx & 31;
    const double2 v = *reinterpret_cast<const double2 *>(g + int64_t(r) * ld + 2 * c2);
    *reinterpret_cast<double2 *>(s + r * LDS + 2 * c2) = v;
  }
}

__device__ __forceinline__ void acc_load(double (&acc)[4][4][2], const double *C, int ld, int wr,
                                         int wc, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const double2 v = *reinterpret_cast<const double2 *>(
          C + int64_t(wr + 8 * i + g) * ld + wc + 8 * j + 2 * t);
      acc[i][j][0] = v.x;
      acc[i][j][1] = v.y;
    }
}

__device__ __forceinline__ void acc_store(const double (&acc)[4][4][2], double *C, int ld, int wr,
                                          int wc, int lane) {
  const int g = lane >> 2, t = lane & 3;
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j)
      *reinterpret_cast<double2 *>(C + int64_t(wr + 8 * i + g) * ld + wc + 8 * j + 2 * t) =
          make_double2(acc[i][j][0], acc[i][j][1]);
}

__device__ __forceinline__ void acc_zero(double (&acc)[4][4][2]) {
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
}

// Row solves x U = c for R rows of a 64-column tile by one warp: U upper
// triangular (row-major, row stride LDS, exact zeros below the diagonal) in
// shared memory and dinv[c] = 1 / U[c][c] (1 for a unit diagonal); on entry
// lo[q] / hi[q] hold columns lane and lane + 32 of row q of c, on return
// those of x.  Right-looking substitution: once x_c is known (broadcast from
// the lane holding column c), every column subtracts x_c U[c][c'] (a no-op
// left of c, where U is zero) and the lane of column c keeps x_c.  This is a
// backward-stable triangular solve (unlike a product with an explicitly
// inverted triangle, whose error grows with the condition number of the
// triangle).
template <int R>
__device__ __forceinline__ void warp_row_solve(double (&lo)[R], double (&hi)[R],
                                               const double *sU, const double *dinv, int lane) {
#pragma unroll 1
  for (int c = 0; c < 32; ++c) {
    const double d = dinv[c];
    const double ul = sU[c * LDS + lane], uh = sU[c * LDS + 32 + lane];
    const bool own = lane == c;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const double x = __shfl_sync(0xffffffffu, lo[q], c) * d;
      lo[q] = own ? x : __fma_rn(-x, ul, lo[q]);
      hi[q] = __fma_rn(-x, uh, hi[q]);
    }
  }
#pragma unroll 1
  for (int c = 32; c < 64; ++c) {
    const double d = dinv[c];
    const double uh = sU[c * LDS + 32 + lane];
    const bool own = lane + 32 == c;
#pragma unroll
    for (int q = 0; q < R; ++q) {
      const double x = __shfl_sync(0xffffffffu, hi[q], c - 32) * d;
      hi[q] = own ? x : __fma_rn(-x, uh, hi[q]);
    }
  }
}

// In-place row solve X U = C for 8 rows (row stride LDS, 64 columns) by one
// warp, blocked by 16 columns, all in registers: lane l holds column
// 16 b + l % 16 of rows l / 16 + 2 q (q = 0..3) for the four column blocks
// b.  Block b is solved by right-looking substitution against U's 16 x 16
// diagonal block, then the blocks right of it are updated with the block's
// result (broadcast by shuffles) times U's off-diagonal block, by FMAs on the
// FP64 pipe: on B200 the FP64 tensor instructions are no faster than FMAs and
// would compete with the int8 tensor-core MMAs of the same SM.  U: upper
// triangular with exact zeros below the diagonal; dinv[c] = 1 / U[c][c].
// Only the warp's own rows are touched, so no block barrier is needed; this
// is a blocked triangular solve (diagonal blocks by substitution, off-
// diagonal blocks by products), backward stable.
__device__ __forceinline__ void warp_rows_trsm8(double *rows, const double *sU,
                                                const double *dinv, int lane) {
  const int col16 = lane & 15, half = lane & 16, rsel = lane >> 4;
  double v[4][4];
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int q = 0; q < 4; ++q) v[b][q] = rows[(rsel + 2 * q) * LDS + 16 * b + col16];
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int cb = 16 * b;
#pragma unroll 4
    for (int c = 0; c < 16; ++c) {
      const double d = dinv[cb + c];
      const double u = sU[(cb + c) * LDS + cb + col16];
      const bool own = col16 == c;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double x = __shfl_sync(0xffffffffu, v[b][q], half | c) * d;
        v[b][q] = own ? x : __fma_rn(-x, u, v[b][q]);
      }
    }
    if (b < 3) {
#pragma unroll 4
      for (int k = 0; k < 16; ++k) {
        double x[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) x[q] = __shfl_sync(0xffffffffu, v[b][q], half | k);
        const double *ur = sU + (cb + k) * LDS + col16;
#pragma unroll
        for (int bb = b + 1; bb < 4; ++bb) {
          const double u = ur[16 * bb];
#pragma unroll
          for (int q = 0; q < 4; ++q) v[bb][q] = __fma_rn(-x[q], u, v[bb][q]);
        }
      }
    }
  }
#pragma unroll
  for (int b = 0; b < 4; ++b)
#pragma unroll
    for (int q = 0; q < 4; ++q) rows[(rsel + 2 * q) * LDS + 16 * b + col16] = v[b][q];
  __syncwarp();
}

// warp_rows_trsm8 with each 16-column block solved by a product with the
// inverse of U's 16 x 16 diagonal block instead of by substitution, all
// products on the FP64 tensor cores (mma.sync m8n8k4: the warp's 8 rows are
// the instruction's M): X_b = R_b Ui_b, then R_c -= X_b U_bc for the blocks
// c right of b.  Ui_b = U_bb^-1 is stored as sUi[(16 b + k) kUiLd + c] =
// U_bb^-1[k][c] (the diagonal blocks of X_j = L_jj^-1 read as X_j[16 b +
// c][16 b + k]); the padded row stride kUiLd spreads the fragment loads of
// four rows over the shared-memory banks.
// The blocks of U_jj are at most as ill-conditioned as U_jj (cond(U_bb) <=
// cond(U_jj)), and the blocked solve stays backward stable blockwise.  No
// shuffles (a 64-bit shuffle costs two of the SM's one-per-clock shuffle
// slots): operands come from shared memory.  With up, the right-hand side is C =
// rows - sig2 up (one rounding), formed first.
__device__ __forceinline__ void warp_rows_trsm8_bi(double *rows, const double *sU,
                                                   const double *sUi, int lane,
                                                   const double *up, double sig2) {
  const int g = lane >> 2, t = lane & 3;
  // The warp's 8 x 64 right-hand side stays in registers in the tensor
  // cores' accumulator layout (lane: row g, columns 8 nt + 2 t, + 1); only
  // the 8 x 16 block being solved goes through shared memory, once to be
  // read as the products' A operand and once as the result.
  double c[8][2];
#pragma unroll
  for (int nt = 0; nt < 8; ++nt)
#pragma unroll
    for (int e = 0; e < 2; ++e) {
      const int o = g * LDS + 8 * nt + 2 * t + e;
      c[nt][e] = up ? __fma_rn(-sig2, up[o], rows[o]) : rows[o];
    }
#pragma unroll
  for (int b = 0; b < 4; ++b) {
    const int cb = 16 * b;
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      rows[g * LDS + cb + 8 * h + 2 * t] = c[2 * b + h][0];
      rows[g * LDS + cb + 8 * h + 2 * t + 1] = c[2 * b + h][1];
    }
    __syncwarp();
    double af[4];
#pragma unroll
    for (int k4 = 0; k4 < 4; ++k4) af[k4] = rows[g * LDS + cb + 4 * k4 + t];
    // X_b = R_b Ui_b, two 8-column halves.
    double x[2][2];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      double c0 = 0.0, c1 = 0.0;
#pragma unroll
      for (int k4 = 0; k4 < 4; ++k4)
        dmma(c0, c1, af[k4], sUi[(cb + 4 * k4 + t) * kUiLd + 8 * h + g]);
      x[h][0] = c0;
      x[h][1] = c1;
    }
    __syncwarp();
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      rows[g * LDS + cb + 8 * h + 2 * t] = x[h][0];
      rows[g * LDS + cb + 8 * h + 2 * t + 1] = x[h][1];
    }
    if (b < 3) {
      __syncwarp();
#pragma unroll
      for (int k4 = 0; k4 < 4; ++k4) af[k4] = -rows[g * LDS + cb + 4 * k4 + t];
      // Columns to the right: R[:, n] -= X_b U[b, n], 8-column tiles.
#pragma unroll
      for (int nt = 2 * b + 2; nt < 8; ++nt)
#pragma unroll
        for (int k4 = 0; k4 < 4; ++k4)
          dmma(c[nt][0], c[nt][1], af[k4], sU[(cb + 4 * k4 + t) * LDS + 8 * nt + g]);
    }
  }
  __syncwarp();
}

// warp_rows_trsm8 with the off-diagonal block products on the FP64 tensor
// cores (mma.sync m8n8k4) through shared memory, for the FP64 step kernel,
// which runs no int8 MMAs and has fewer registers to spare.
__device__ __forceinline__ void warp_rows_trsm8_tc(double *rows, const double *sU,
                                                   const double *dinv, int lane) {
  const int g = lane >> 2, t = lane & 3;
  const int col16 = lane & 15, half = lane & 16, rsel = lane >> 4;
#pragma unroll 1
  for (int b = 0; b < 4; ++b) {
    const int cb = 16 * b;
    double acc[4];
#pragma unroll
    for (int q = 0; q < 4; ++q) acc[q] = rows[(rsel + 2 * q) * LDS + cb + col16];
#pragma unroll 4
    for (int c = 0; c < 16; ++c) {
      const double d = dinv[cb + c];
      const double u = sU[(cb + c) * LDS + cb + col16];
      const bool own = col16 == c;
#pragma unroll
      for (int q = 0; q < 4; ++q) {
        const double x = __shfl_sync(0xffffffffu, acc[q], half | c) * d;
        acc[q] = own ? x : __fma_rn(-x, u, acc[q]);
      }
    }
#pragma unroll
    for (int q = 0; q < 4; ++q) rows[(rsel + 2 * q) * LDS + cb + col16] = acc[q];
    __syncwarp();
    // Columns to the right: C[:, n] -= X_b U[b, n], 8-column tiles.
    for (int nt = 2 * b + 2; nt < 8; ++nt) {
      double c0 = rows[g * LDS + 8 * nt + 2 * t], c1 = rows[g * LDS + 8 * nt + 2 * t + 1];
#pragma unroll
      for (int k0 = 0; k0 < 16; k0 += 4) {
        const double av = -rows[g * LDS + cb + k0 + t];
        const double bv = sU[(cb + k0 + t) * LDS + 8 * nt + g];
        dmma(c0, c1, av, bv);
      }
      rows[g * LDS + 8 * nt + 2 * t] = c0;
      rows[g * LDS + 8 * nt + 2 * t + 1] = c1;
    }
    __syncwarp();
  }
}

// Asynchronous 16-byte global -> shared copies (cp.async, sm_80+).
__device__ __forceinline__ void cp_async16(void *smem, const void *gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async8(void *smem, const void *gmem) {
  const unsigned sa = static_cast<unsigned>(__cvta_generic_to_shared(smem));
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(sa), "l"(gmem));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}
__device__ __forceinline__ void async_tile(double *s, const double *g, int ld, int tid, int nt) {
  for (int idx = tid; idx < TB * TB / 2; idx += nt) {
    const int r = idx >> 5, c2 = idx & 31;
    cp_async16(s + r * LDS + 2 * c2, g + int64_t(r) * ld + 2 * c2);
  }
}

// Loads the diagonal tile's factor U = L_jj^T (row-major in the workspace's
// diagonal tile position, written by diag_tile) into sU with cp.async; the
// caller commits, waits, and then fills dinv[c] = 1 / U[c][c].
__device__ __forceinline__ void load_factor_async(double *sU, const double *gu, int ld, int tid,
                                                  int nt) {
  for (int idx = tid; idx < TB * TB / 2; idx += nt) {
    const int r = idx >> 5, c2 = idx & 31;
    cp_async16(sU + r * LDS + 2 * c2, gu + int64_t(r) * ld + 2 * c2);
  }
}

struct BigArgs {
  const double4 *src;
  const double4 *tgt;
  const double *vals;
  const int64_t *soff;
  const int *sidx;
  const int64_t *toff;
  const int *tidx;
  const double4 *centers;
  double *W;            // workspace
  double *inv;          // inverse tiles (TB x TB): LU 2 per slot, Cholesky T per slot
  double *beta;         // per slot: 4 * kMaxF
  int *act;             // per slot: 3
  int *status;          // per patch
  double *local;
  double rinv;
  int F;
  int dim;
  int basis;
  int mode;            // kBigForward, kBigForwardSave or kBigAdjoint
  double *alpha_out;   // forward + save: RBF coefficients per (patch, source)
  double *beta_out;    // forward + save: K x 4*kMaxF
  int *act_out;        // forward + save: K x 3
  const double *h;     // adjoint: weighted upstream gradient per (patch, target)
  double *g_out;       // adjoint: result per (patch, source)
  double *red_out;     // adjoint: per slot reduced moments (kRedVals)
  double *alpha_c;     // Cholesky forward: RBF coefficients per (patch, source)
  double *zc;          // Cholesky: backward-sweep solution per slot (T*TB x F)
  uint8_t *slices;     // mixed forward: int8 slices of the L tiles, or null (FP64 updates)
  double oz_mul;       // 128 / sigma (sigma bounds |L|)
  double oz_sig2;      // sigma^2
  int wait_limit;      // polls of a tensor-core pipeline wait before it gives up
  double *dpart;       // mixed forward: per slot, D' of the next diagonal tile (TB x TB)
};

// Polls of a tensor-core pipeline wait (mbarrier) before the step gives up
// and marks its patch for the FP64 LU: 2^22, or PACMAN_B200_WAIT_LIMIT (a
// test shortens it to exercise that path).
int pipeline_wait_limit();

// Left-looking Cholesky steps, backward sweep and local evaluation of one
// wave of slots (cholesky.cu).  `pre` holds, per step, the prefix counts of
// the column-update and triangular-solve launches (see chol_prefix).
struct CholPlan {
  int ns = 0;                // slots
  std::vector<int> cnt;      // active slots per step
  std::vector<int> off;      // per step: offset of its prefix arrays in pre
  std::vector<int> pre;      // per step: prefix of the CTA counts (cnt+1)
  std::vector<int> ioff;     // per step: offset in pre of the item prefix counts (cnt+1)
};
CholPlan chol_prefix(const std::vector<BigSlot> &slots);
void chol_set_smem_attributes();
// Bytes of int8 slice tiles of a slot with T tile rows (strictly lower tiles).
size_t oz_slot_bytes(int T);
// tail_event (or null) is recorded on st at the first step that leaves SMs
// idle (fewer than two CTAs per SM), else after the last step.
void chol_launch_steps(const BigArgs &a, const BigSlot *ds, const std::vector<BigSlot> &hs,
                       const CholPlan &cp, const int *dpre, cudaStream_t st, SolveReport &rep,
                       cudaEvent_t tail_event);
// Factorisations kept in a plan by an execute with PACMAN_B200_KEEP_FACTORS
// (precision "mixed"): later executes with the same basis run only the
// polynomial block, the triangular solves and the evaluation.
struct CholWaveCache {             // one wave of the large-patch engine
  DevMem W;                        // L tiles; residual column tile (F <= 8 columns)
  DevMem small;                    // tile inverses, beta, act, slot tables
  double *inv = nullptr, *beta = nullptr, *red = nullptr;
  int *act = nullptr;
  int ns = 0;
  int64_t sum_T = 0;               // zc holds sum_T * TB * kMaxF doubles (slot offsets)
  BigSlot *ds = nullptr;           // device slot table (in small), largest first
};
struct SmallRange {                // one launch of the register kernel
  size_t first = 0;                // offset into the cached patch list
  int count = 0, nmax = 0;
  size_t fac_off = 0;              // offset (doubles) of its factors
};
struct FactorCache {
  int basis = -1;
  std::vector<CholWaveCache> waves;
  DevMem small_list;               // patch ids of the small launches
  DevMem small_fac;                // their L^{-1} blocks and pivots
  std::vector<SmallRange> ranges;
  std::vector<int> redo_small, redo_big;  // re-solved by the FP64 LU every execute
  int64_t patches = 0;
};
// Bytes of the kept factors of one register-kernel patch of size class N.
inline size_t small_fac_doubles(int N) { return size_t(N) * N + N; }

// Forward sweep L y = r from kept factors (an execute that reuses them).
void chol_launch_forward(const BigArgs &a, const BigSlot *ds, int ns, cudaStream_t st);
void chol_launch_finish(const BigArgs &a, const BigSlot *ds, int ns, bool adjoint,
                        cudaStream_t st);

}  // namespace pacman_b200
