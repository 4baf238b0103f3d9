// Per-patch solve arguments shared by the shared-memory kernels (solve.cu)
// and the register-resident small-patch kernels (small.cu).
#pragma once

#include "plan.hpp"
#include "poly.cuh"

namespace pacman_b200 {

enum SolveMode {
  kLU = 0,   // forward, unpivoted LU (the reference algorithm)
  kChol = 1, // forward, Cholesky
  kAdj = 2,  // transpose (adjoint) solve with Cholesky: g = z - Q'G'^{-1}(Q'^T z - V'^T h)
};

enum PatchStatus : int {
  kStatusDropped = 1,     // the polynomial block lost at least one axis
  kStatusNonFinite = 2,   // a non-finite local value
  kStatusBreakdown = 4,   // non-positive Cholesky pivot
  kStatusTimeout = 8,     // a bounded tensor-core pipeline wait gave up
  kStatusResolved = 16,   // re-solved by the FP64 LU after one of the above (host side)
};

struct PatchArgs {
  const double4 *src;
  const double4 *tgt;
  const double *vals;
  const int64_t *soff;
  const int *sidx;
  const int64_t *toff;
  const int *tidx;
  const double4 *centers;
  double *local;
  int *status;
  double *gA;             // global workspace (patches whose A does not fit in smem)
  const int64_t *gAoff;   // per list entry offset into gA, or nullptr
  double rinv;            // 1 / support radius
  int F;
  int dim;
  int basis;
  double *alpha_out;      // forward: RBF coefficients per (patch, source), or null
  double *beta_out;       // forward: polynomial coefficients, K x 4*kMaxF, or null
  int *act_out;           // forward: active axes, K x 3, or null
  const double *h;        // adjoint: weighted upstream gradient per (patch, target)
  double *g_out;          // adjoint: result per (patch, source)
  // Register kernel (small.cu): 0 factor, 1 factor and store the eliminated
  // blocks at fac (N * N doubles per list entry), 2 load them instead of
  // assembling and factoring.
  double *fac;
  int fac_mode;
};

// Register-resident Cholesky of the patches with n <= 64 (small.cu); the
// list must hold patches of one size class (n <= 32 or 32 < n <= 64).
void launch_small_chol(const PatchArgs &a, const int *plist, int np, int nmax, cudaStream_t st);

}  // namespace pacman_b200
