// Polynomial block of a patch (src/rbf_pum/solver/utils/serial_ops.hpp:28-139,
// serial_solve.hpp:46-67, :100-110), shared by the per-patch kernels.
//
// The reference builds Q = [1, x_active] (uncentred), tests its condition
// number sigma_max / max(sigma_min, 1e-14) against 1e5 with an SVD, drops the
// active axis of smallest coordinate range while the test fails, and fits the
// values by Householder least squares.  Here the whole block comes from one
// reduction pass over the patch: the Gram matrix G of the centred monomials
// [1, x - c] (c = the patch centre, one of its points) is well conditioned;
// its Cholesky factor R gives the least-squares fit, and R times the change
// of basis back to [1, x] has exactly the singular values of the uncentred Q.
#pragma once

#include "common.cuh"

namespace pacman_b200 {

constexpr int kMaxF = 8;
constexpr int kRedVals = 10 + 4 * kMaxF + 6;

__device__ __forceinline__ double warp_sum(double v) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}

// Singular values (descending) of a pv x pv upper-triangular-ish matrix by
// one-sided Jacobi.
__device__ inline void small_svd(double M[4][4], int pv, double *sig) {
  for (int sweep = 0; sweep < 60; ++sweep) {
    bool rot = false;
    for (int i = 0; i < pv; ++i)
      for (int j = i + 1; j < pv; ++j) {
        double al = 0, be = 0, ga = 0;
        for (int r = 0; r < pv; ++r) {
          al += M[r][i] * M[r][i];
          be += M[r][j] * M[r][j];
          ga += M[r][i] * M[r][j];
        }
        if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
        rot = true;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int r = 0; r < pv; ++r) {
          const double x = M[r][i], y = M[r][j];
          M[r][i] = cs * x - sn * y;
          M[r][j] = sn * x + cs * y;
        }
      }
    if (!rot) break;
  }
  for (int j = 0; j < pv; ++j) {
    double s = 0;
    for (int r = 0; r < pv; ++r) s += M[r][j] * M[r][j];
    sig[j] = sqrt(s);
  }
  for (int i = 1; i < pv; ++i) {
    const double x = sig[i];
    int j = i - 1;
    while (j >= 0 && sig[j] < x) {
      sig[j + 1] = sig[j];
      --j;
    }
    sig[j + 1] = x;
  }
}

// Cholesky of the pv x pv SPD matrix G (upper factor R, G = R^T R).
__device__ inline bool small_chol(const double G[4][4], int pv, double R[4][4]) {
  for (int i = 0; i < 4; ++i)
    for (int j = 0; j < 4; ++j) R[i][j] = 0.0;
  for (int j = 0; j < pv; ++j) {
    double d = G[j][j];
    for (int k = 0; k < j; ++k) d -= R[k][j] * R[k][j];
    if (!(d > 0.0)) return false;
    d = sqrt(d);
    R[j][j] = d;
    for (int i = j + 1; i < pv; ++i) {
      double s = G[j][i];
      for (int k = 0; k < j; ++k) s -= R[k][j] * R[k][i];
      R[j][i] = s / d;
    }
  }
  return true;
}

// Gram matrix of the centred monomials from the reduced moments.
// red: [0]=n, [1..3]=sum dx, [4..9]=sum dx_a dx_b (aa,ab,ac,bb,bc,cc).
__device__ inline void gram_from_moments(const double *red, double G[4][4]) {
  G[0][0] = red[0];
  G[0][1] = G[1][0] = red[1];
  G[0][2] = G[2][0] = red[2];
  G[0][3] = G[3][0] = red[3];
  G[1][1] = red[4];
  G[1][2] = G[2][1] = red[5];
  G[1][3] = G[3][1] = red[6];
  G[2][2] = red[7];
  G[2][3] = G[3][2] = red[8];
  G[3][3] = red[9];
}

// Active polynomial terms of a patch (SerialFillQ's condition loop,
// serial_ops.hpp:108-139): S[0..pv) are monomial ids (0 = constant, a + 1 =
// axis a), R is the Cholesky factor of the centred Gram matrix restricted to
// S.  mn / mx are the coordinate ranges used to pick the axis to drop.
// Returns 1 if an axis was dropped.
__device__ inline int poly_axes(const double *red, int dim, const double *shift,
                                const double *mn, const double *mx, int S[4], int &pv_out,
                                double R[4][4]) {
  double G[4][4];
  gram_from_moments(red, G);
  bool active[3] = {dim > 0, dim > 1, dim > 2};
  int pv = dim + 1;
  int dropped = 0;
  const double n = red[0];
  bool have_R = false;
  for (;;) {
    int c = 0;
    S[c++] = 0;
    for (int a = 0; a < dim; ++a)
      if (active[a]) S[c++] = a + 1;
    if (pv <= 1) {
      have_R = false;
      break;
    }
    double Gs[4][4];
    for (int i = 0; i < pv; ++i)
      for (int j = 0; j < pv; ++j) Gs[i][j] = G[S[i]][S[j]];
    double cond = INFINITY;
    if (n >= double(pv) && small_chol(Gs, pv, R)) {
      double M[4][4];
      for (int i = 0; i < 4; ++i)
        for (int j = 0; j < 4; ++j) M[i][j] = 0.0;
      for (int i = 0; i < pv; ++i) {
        M[i][0] = R[i][0];
        for (int j = 1; j < pv; ++j) M[i][j] = R[i][j] + R[i][0] * shift[S[j] - 1];
      }
      double sig[4];
      small_svd(M, pv, sig);
      cond = sig[0] / fmax(sig[pv - 1], kEps);
      have_R = true;
    } else {
      have_R = false;
    }
    if (!(cond > kCondMax)) break;
    // SerialDeactivateOneAxis (serial_ops.hpp:28-57).
    double best = 1.7976931348623157e308;
    int bi = 0;
    for (int a = 0; a < dim; ++a) {
      const double rg = active[a] ? fabs(mx[a] - mn[a]) : 1.7976931348623157e308;
      if (rg < best) {
        best = rg;
        bi = a;
      }
    }
    active[bi] = false;
    --pv;
    dropped = 1;
  }
  if (!have_R) {
    double Gs[4][4];
    for (int i = 0; i < pv; ++i)
      for (int j = 0; j < pv; ++j) Gs[i][j] = G[S[i]][S[j]];
    small_chol(Gs, pv, R);
  }
  pv_out = pv;
  return dropped;
}

// Solves (R^T R) x = rhs for the pv active terms.
__device__ inline void gram_solve(const double R[4][4], int pv, const double *rhs, double *x) {
  double z[4];
  for (int i = 0; i < pv; ++i) {
    double s = rhs[i];
    for (int k = 0; k < i; ++k) s -= R[k][i] * z[k];
    z[i] = s / R[i][i];
  }
  for (int i = pv - 1; i >= 0; --i) {
    double s = z[i];
    for (int k = i + 1; k < pv; ++k) s -= R[i][k] * x[k];
    x[i] = s / R[i][i];
  }
}

// Polynomial block of one patch from the reduced moments (one thread).
// red: moments as above, [10 + 4f + c] = sum q_c b_f, [10+4F .. +6] = min
// x,y,z, max x,y,z.  Writes beta[4 x F] (uncentred basis, zero for dropped
// axes), act[0..2] (active axis ids, -1 terminated) and returns the dropped
// flag.
__device__ inline int poly_block(const double *red, int F, int dim, const double *shift,
                                 double *beta, int *act) {
  const double *mn = red + 10 + 4 * F;
  const double *mx = mn + 3;
  int S[4], pv;
  double R[4][4];
  const int dropped = poly_axes(red, dim, shift, mn, mx, S, pv, R);
  int na = 0;
  for (int i = 1; i < pv; ++i) act[na++] = S[i] - 1;
  for (int a = na; a < 3; ++a) act[a] = -1;
  for (int f = 0; f < F; ++f) {
    const double *h = red + 10 + 4 * f;
    double hs[4], bp[4];
    for (int i = 0; i < pv; ++i) hs[i] = h[S[i]];
    gram_solve(R, pv, hs, bp);
    double b0 = bp[0];
    for (int i = 1; i < pv; ++i) b0 -= shift[S[i] - 1] * bp[i];
    beta[4 * f + 0] = b0;
    for (int i = 1; i < pv; ++i) beta[4 * f + i] = bp[i];
    for (int i = pv; i < 4; ++i) beta[4 * f + i] = 0.0;
  }
  return dropped;
}
}  // namespace pacman_b200
