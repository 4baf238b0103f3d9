// Moving least squares transfer of the B200 engine (PACMAN::MLS_interpolate,
// src/mls_interface.cpp; src/mls/interpolator.hpp:49-77).  The reference
// hands the whole computation to ArborX 2.1's
// Interpolation::MovingLeastSquares with its defaults: for each target the K
// nearest sources (K = size of the quadratic basis: 3, 6, 10 in 1D, 2D, 3D),
// radius 1.1 x the farthest neighbour's distance, Wendland C0 weights
// (1 - d / radius)^2, the moment matrix A = sum_j w_j p_j p_j^T of the
// monomials of degree <= 2 of (source - target), and the value
// e_0^T A^+ (sum_j w_j f_j p_j) with A^+ the pseudo-inverse of the symmetric A.
// Here the monomials are those of (source - target) / radius: the same value
// wherever A is invertible, without the radius^4 spread of A's eigenvalues.
//
// One thread per target:
//  * K-nearest search on the uniform source grid (about one source per cell),
//    scanning shells of cells nearest first and stopping once the K-th best
//    squared distance is below ((R - 1) h)^2 (nothing unscanned can be closer;
//    one cell of slack for rounding).  The K best are kept sorted by
//    (squared distance, source index) in registers, so ties go to the lowest
//    index and the neighbour set and order are exactly the CPU oracle's.
//  * A (packed upper triangle, K(K+1)/2 doubles) and b in registers; a cyclic
//    Jacobi eigen-decomposition A = V L V^T (Rutishauser's rotation formulas)
//    whose rotations are applied to u = V^T e_0 and v = V^T b, so neither V nor
//    A^+ is formed; value = sum over |l_k| > 1e-13 max|l| of u_k v_k / l_k.
// This file is compiled without floating-point contraction (-fmad=false):
// each product and sum is rounded on its own, in the same order as the
// oracle's restatement, so the values agree bit for bit.
#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>

#include "plan.hpp"

namespace pacman_b200 {

namespace {

constexpr int kMlsSweeps = 64;

template <int DIM>
struct Mls {
  static constexpr int K = DIM == 1 ? 3 : (DIM == 2 ? 6 : 10);
  static constexpr int NP = K * (K + 1) / 2;
};

// Packed upper-triangle position of (i, j) in an M x M symmetric matrix.
__host__ __device__ constexpr int sym_at(int i, int j, int M) {
  return i <= j ? i * M - i * (i - 1) / 2 + (j - i) : j * M - j * (j - 1) / 2 + (i - j);
}

template <int DIM>
__device__ __forceinline__ void mls_basis(const double *x, double *p) {
  p[0] = 1.0;
  if (DIM == 1) {
    p[1] = x[0];
    p[2] = x[0] * x[0];
  } else if (DIM == 2) {
    p[1] = x[0];
    p[2] = x[1];
    p[3] = x[0] * x[0];
    p[4] = x[0] * x[1];
    p[5] = x[1] * x[1];
  } else {
    p[1] = x[0];
    p[2] = x[1];
    p[3] = x[2];
    p[4] = x[0] * x[0];
    p[5] = x[0] * x[1];
    p[6] = x[0] * x[2];
    p[7] = x[1] * x[1];
    p[8] = x[1] * x[2];
    p[9] = x[2] * x[2];
  }
}

// The rotation annihilating A(P, Q), applied to A, u and v.
template <int M, int P, int Q>
__device__ __forceinline__ void mls_rotate(double *a, double *u, double *v) {
  constexpr int pq = sym_at(P, Q, M), pp = sym_at(P, P, M), qq = sym_at(Q, Q, M);
  const double apq = a[pq];
  if (apq == 0.0) return;
  const double app = a[pp], aqq = a[qq];
  const double g = 100.0 * fabs(apq);
  if (fabs(app) + g == fabs(app) && fabs(aqq) + g == fabs(aqq)) {
    a[pq] = 0.0;  // below the rounding of both diagonal entries
    return;
  }
  const double h = aqq - app;
  double t;
  if (fabs(h) + g == fabs(h)) {
    t = apq / h;
  } else {
    const double theta = 0.5 * h / apq;
    t = 1.0 / (fabs(theta) + sqrt(1.0 + theta * theta));
    if (theta < 0.0) t = -t;
  }
  const double c = 1.0 / sqrt(1.0 + t * t);
  const double s = t * c;
  const double tau = s / (1.0 + c);
  a[pp] = app - t * apq;
  a[qq] = aqq + t * apq;
  a[pq] = 0.0;
#pragma unroll
  for (int r = 0; r < M; ++r) {
    if (r == P || r == Q) continue;
    const int rp = sym_at(r, P, M), rq = sym_at(r, Q, M);
    const double arp = a[rp], arq = a[rq];
    a[rp] = arp - s * (arq + tau * arp);
    a[rq] = arq + s * (arp - tau * arq);
  }
  const double up = u[P], uq = u[Q];
  u[P] = up - s * (uq + tau * up);
  u[Q] = uq + s * (up - tau * uq);
  const double vp = v[P], vq = v[Q];
  v[P] = vp - s * (vq + tau * vp);
  v[Q] = vq + s * (vp - tau * vq);
}

// One cyclic sweep over the pairs (P, Q), P < Q, row by row.
template <int M, int P, int Q>
__device__ __forceinline__ void mls_sweep(double *a, double *u, double *v) {
  if constexpr (P < M - 1) {
    mls_rotate<M, P, Q>(a, u, v);
    if constexpr (Q + 1 < M)
      mls_sweep<M, P, Q + 1>(a, u, v);
    else if constexpr (P + 2 < M)
      mls_sweep<M, P + 1, P + 2>(a, u, v);
  }
}

template <int DIM>
__global__ void __launch_bounds__(128) k_mls(int64_t M, const double4 *__restrict__ tgt,
                                             GridView g, double h,
                                             const double4 *__restrict__ src,
                                             const double *__restrict__ vals, int64_t n,
                                             double *__restrict__ out) {
  constexpr int K = Mls<DIM>::K;
  constexpr int NP = Mls<DIM>::NP;
  const int kk = n < K ? int(n) : K;
  const int rmax = max(g.nc[0], max(g.nc[1], g.nc[2]));
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < M;
       t += int64_t(gridDim.x) * blockDim.x) {
    const double4 y = tgt[t];
    const int cx = cell_coord(y.x, g.lo[0], g.inv_h, g.nc[0]);
    const int cy = cell_coord(y.y, g.lo[1], g.inv_h, g.nc[1]);
    const int cz = cell_coord(y.z, g.lo[2], g.inv_h, g.nc[2]);
    double bd[K];
    int bi[K];
#pragma unroll
    for (int k = 0; k < K; ++k) {
      bd[k] = DBL_MAX;
      bi[k] = INT_MAX;
    }
    auto scan = [&](int s, int e) {
      for (int i = s; i < e; ++i) {
        const int id = g.items[i];
        const double4 x = src[id];
        const double d2 = sqdist3(y.x, y.y, y.z, x.x, x.y, x.z);
        if (!(d2 < bd[K - 1] || (d2 == bd[K - 1] && id < bi[K - 1]))) continue;
        bd[K - 1] = d2;
        bi[K - 1] = id;
#pragma unroll
        for (int k = K - 1; k > 0; --k) {
          if (bd[k] < bd[k - 1] || (bd[k] == bd[k - 1] && bi[k] < bi[k - 1])) {
            const double td = bd[k];
            bd[k] = bd[k - 1];
            bd[k - 1] = td;
            const int ti = bi[k];
            bi[k] = bi[k - 1];
            bi[k - 1] = ti;
          }
        }
      }
    };
    for (int R = 0; R <= rmax; ++R) {
      const int x0 = max(cx - R, 0), x1 = min(cx + R, g.nc[0] - 1);
      const int y0 = max(cy - R, 0), y1 = min(cy + R, g.nc[1] - 1);
      for (int a = x0; a <= x1; ++a)
        for (int b = y0; b <= y1; ++b) {
          const int base = (a * g.nc[1] + b) * g.nc[2];
          const bool face = a == cx - R || a == cx + R || b == cy - R || b == cy + R;
          if (face) {
            const int z0 = max(cz - R, 0), z1 = min(cz + R, g.nc[2] - 1);
            scan(g.start[base + z0], g.start[base + z1 + 1]);
          } else {
            if (cz - R >= 0) scan(g.start[base + cz - R], g.start[base + cz - R + 1]);
            if (cz + R < g.nc[2]) scan(g.start[base + cz + R], g.start[base + cz + R + 1]);
          }
        }
      if (bi[K - 1] != INT_MAX && R >= 1) {
        const double lim = double(R - 1) * h;
        if (bd[K - 1] < lim * lim) break;
      }
    }
    // Weights, moment matrix and right-hand side.  With finite coordinates
    // the first kk entries are filled; the id test keeps a NaN coordinate
    // (never a neighbour) from indexing past the sources.
    bool use[K];
    double dist[K];
    double rad = 10.0 * DBL_EPSILON;
#pragma unroll
    for (int j = 0; j < K; ++j) {
      use[j] = j < kk && bi[j] != INT_MAX;
      dist[j] = use[j] ? sqrt(bd[j]) : 0.0;
      if (use[j]) rad = fmax(rad, dist[j]);
    }
    const double radius = 1.1 * rad;
    const double yc[3] = {y.x, y.y, y.z};
    double a[NP], b[K], u[K];
#pragma unroll
    for (int i = 0; i < NP; ++i) a[i] = 0.0;
#pragma unroll
    for (int i = 0; i < K; ++i) {
      b[i] = 0.0;
      u[i] = i == 0 ? 1.0 : 0.0;
    }
#pragma unroll
    for (int j = 0; j < K; ++j) {
      if (use[j]) {
        const double4 s4 = src[bi[j]];
        const double sc[3] = {s4.x, s4.y, s4.z};
        double x[3], p[K];
#pragma unroll
        for (int d = 0; d < 3; ++d) x[d] = d < DIM ? (sc[d] - yc[d]) / radius : 0.0;
        mls_basis<DIM>(x, p);
        const double rho = dist[j] / radius;
        const double w = (1.0 - rho) * (1.0 - rho);
        const double wf = w * vals[bi[j]];
#pragma unroll
        for (int r = 0; r < K; ++r) {
          const double wr = w * p[r];
#pragma unroll
          for (int c = r; c < K; ++c) a[sym_at(r, c, K)] = a[sym_at(r, c, K)] + wr * p[c];
          b[r] = b[r] + wf * p[r];
        }
      }
    }
    // e_0^T A^+ b by cyclic Jacobi, at most kMlsSweeps sweeps.
    for (int sw = 0; sw < kMlsSweeps; ++sw) {
      bool off = false;
#pragma unroll
      for (int p = 0; p < K; ++p)
#pragma unroll
        for (int q = p + 1; q < K; ++q) off |= a[sym_at(p, q, K)] != 0.0;
      if (!off) break;
      mls_sweep<K, 0, 1>(a, u, b);
    }
    double lmax = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) lmax = fmax(lmax, fabs(a[sym_at(k, k, K)]));
    const double cut = 1e-13 * lmax;
    double val = 0.0;
#pragma unroll
    for (int k = 0; k < K; ++k) {
      const double l = a[sym_at(k, k, K)];
      if (fabs(l) > cut) val = val + (u[k] * b[k]) / l;
    }
    out[t] = kk > 0 ? val : 0.0;
  }
}

}  // namespace

void mls_interpolate(int dim, const double *src_dev, int64_t n, const double *vals_dev,
                     const double *tgt_dev, int64_t m, double *out_dev, cudaStream_t st) {
  if (m == 0) return;
  if (n == 0) {  // no source: the zero fill of SetupTransferClass (transfer.hxx:100-110)
    PB_CUDA(cudaMemsetAsync(out_dev, 0, sizeof(double) * size_t(m), st));
    return;
  }
  DevMem src4, tgt4;
  double lo[3], hi[3], tlo[3], thi[3];
  pack_points(src_dev, dim, n, src4, lo, hi, st);
  pack_points(tgt_dev, dim, m, tgt4, tlo, thi, st);
  // About one source per cell: the largest extent over n^(1/dim) cells.
  double ext = 0.0;
  for (int d = 0; d < dim; ++d) ext = std::max(ext, hi[d] - lo[d]);
  const double per_axis = std::ceil(std::pow(double(n), 1.0 / dim));
  const double cell = ext > 0.0 ? ext / per_axis : 1.0;
  DevGrid grid;
  build_point_grid(grid, src4.as<double4>(), n, dim, lo, hi, cell, st);
  const double h = 1.0 / grid.view.inv_h;
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>((m + 127) / 128, 148 * 16)));
  if (dim == 1)
    k_mls<1><<<blocks, 128, 0, st>>>(m, tgt4.as<double4>(), grid.view, h, src4.as<double4>(),
                                     vals_dev, n, out_dev);
  else if (dim == 2)
    k_mls<2><<<blocks, 128, 0, st>>>(m, tgt4.as<double4>(), grid.view, h, src4.as<double4>(),
                                     vals_dev, n, out_dev);
  else
    k_mls<3><<<blocks, 128, 0, st>>>(m, tgt4.as<double4>(), grid.view, h, src4.as<double4>(),
                                     vals_dev, n, out_dev);
  note_launch();
  PB_CUDA(cudaGetLastError());
  PB_CUDA(host_sync(st));
}

}  // namespace pacman_b200
