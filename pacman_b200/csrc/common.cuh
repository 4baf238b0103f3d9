// Shared device helpers for the B200 RBF-PUM transfer.
//
// Arithmetic here is specified bit-for-bit: the geometry predicates (patch
// radius, centre cover, membership lists) must reproduce the CPU restatement
// exactly, so every expression is written with explicit IEEE intrinsics and
// never relies on compiler contraction.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

namespace pacman_b200 {

constexpr double kEps = 1.0e-14;      // fp_consts::epsilon(), src/common/types.hpp:98
constexpr double kCondMax = 1.0e5;    // serial_ops.hpp:130
constexpr int kWendlandC0 = 0x10;     // src/interface.hpp:25-31
constexpr int kWendlandC2 = 0x11;
constexpr int kWendlandC4 = 0x12;
constexpr int kWendlandC6 = 0x13;
constexpr int kWendlandC8 = 0x14;

// Squared distance of src/rbf_pum/utils/operators.hpp:125-137 with the
// reference build's contraction: acc = fma(t, t, acc) per axis, t = b - a.
// Coordinates are zero-padded to 3 axes; fma(0, 0, acc) == acc, so the 3-axis
// form equals the dim-axis form for dim < 3.
__device__ __forceinline__ double sqdist3(double ax, double ay, double az,
                                          double bx, double by, double bz) {
  const double tx = __dsub_rn(bx, ax);
  const double ty = __dsub_rn(by, ay);
  const double tz = __dsub_rn(bz, az);
  double acc = __dmul_rn(tx, tx);
  acc = __fma_rn(ty, ty, acc);
  acc = __fma_rn(tz, tz, acc);
  return acc;
}

__device__ __forceinline__ double sqdist(const double4 &a, const double4 &b) {
  return sqdist3(a.x, a.y, a.z, b.x, b.y, b.z);
}

// Wendland C0..C8 (src/rbf_pum/solver/rbf_functions.hpp:22-150), branch-free
// with the reference's support mask.  Powers are multiplication chains.
template <typename T>
__device__ __forceinline__ T wendland(int basis, T r, T rinv) {
  const T p = r * rinv;
  const T mask = (r >= T(0) && p < T(1) && p >= T(0)) ? T(1) : T(0);
  const T q = T(1) - p;
  const T q2 = q * q;
  T v;
  switch (basis) {
  case kWendlandC0:
    v = q2;
    break;
  case kWendlandC2: {
    const T q4 = q2 * q2;
    v = q4 * fma(T(4), p, T(1));
    break;
  }
  case kWendlandC4: {
    const T q6 = q2 * q2 * q2;
    v = q6 * fma(T(35), p * p, fma(T(18), p, T(3)));
    break;
  }
  case kWendlandC6: {
    const T q4 = q2 * q2;
    const T p2 = p * p;
    v = (q4 * q4) * (fma(T(32), p2 * p, T(25) * p2) + fma(T(8), p, T(1)));
    break;
  }
  default: {  // C8
    const T q4 = q2 * q2;
    const T p2 = p * p;
    T t = fma(T(1287), p2 * p2, T(1350) * p2 * p);
    t = fma(T(630), p2, t);
    v = (q4 * q4 * q2) * (t + fma(T(150), p, T(15)));
    break;
  }
  }
  return mask * v;
}

// d phi / d p of the Wendland bases (p = r / rho), zero outside the support.
// C0: -2(1-p); C2: -20p(1-p)^3; C4: -56p(1-p)^5(5p+1);
// C6: -22p(1-p)^7(16p^2+7p+1); C8: -78p(1-p)^9(231p^3+159p^2+45p+5).
__device__ __forceinline__ double wendland_dp(int basis, double p) {
  if (!(p >= 0.0 && p < 1.0)) return 0.0;
  const double q = 1.0 - p;
  const double q2 = q * q;
  switch (basis) {
  case kWendlandC0:
    return -2.0 * q;
  case kWendlandC2:
    return -20.0 * p * q2 * q;
  case kWendlandC4:
    return -56.0 * p * (q2 * q2 * q) * fma(5.0, p, 1.0);
  case kWendlandC6:
    return -22.0 * p * (q2 * q2 * q2 * q) * fma(fma(16.0, p, 7.0), p, 1.0);
  default:
    return -78.0 * p * (q2 * q2 * q2 * q2 * q) * fma(fma(fma(231.0, p, 159.0), p, 45.0), p, 5.0);
  }
}

// Monotone uint64 image of a double (total order on non-NaN values), used for
// exact, order-independent atomic min/max reductions.
__device__ __forceinline__ unsigned long long dbl_to_ordered(double x) {
  unsigned long long b = __double_as_longlong(x);
  return (b & 0x8000000000000000ull) ? ~b : (b | 0x8000000000000000ull);
}
__device__ __forceinline__ double ordered_to_dbl(unsigned long long b) {
  b = (b & 0x8000000000000000ull) ? (b & 0x7fffffffffffffffull) : ~b;
  return __longlong_as_double(b);
}

// Uniform cell grid over the source bounding box grown by one cell; cell size
// h >= patch radius, so every point within the radius of a query inside the
// source box lies in the 3x3x3 cells around the query's cell.
struct GridView {
  double lo[3];
  double inv_h;
  int nc[3];
  int ncells;
  const int *start;  // ncells + 1
  const int *items;  // point ids grouped by cell, ascending within a cell
};

__device__ __forceinline__ int cell_coord(double x, double lo, double inv_h, int nc) {
  const double f = floor(__dmul_rn(__dsub_rn(x, lo), inv_h));
  int c = (f < 0.0) ? 0 : (f > double(nc - 1) ? nc - 1 : int(f));
  return c;
}

// Calls fn(point_id) for every point in the 3^3 cells around q.
template <typename Fn>
__device__ __forceinline__ void for_neighbors(const GridView &g, double qx, double qy,
                                              double qz, Fn &&fn) {
  const int cx = cell_coord(qx, g.lo[0], g.inv_h, g.nc[0]);
  const int cy = cell_coord(qy, g.lo[1], g.inv_h, g.nc[1]);
  const int cz = cell_coord(qz, g.lo[2], g.inv_h, g.nc[2]);
  const int x0 = max(cx - 1, 0), x1 = min(cx + 1, g.nc[0] - 1);
  const int y0 = max(cy - 1, 0), y1 = min(cy + 1, g.nc[1] - 1);
  const int z0 = max(cz - 1, 0), z1 = min(cz + 1, g.nc[2] - 1);
  for (int a = x0; a <= x1; ++a)
    for (int b = y0; b <= y1; ++b) {
      const int base = (a * g.nc[1] + b) * g.nc[2];
      const int s = g.start[base + z0];
      const int e = g.start[base + z1 + 1];
      for (int i = s; i < e; ++i) fn(g.items[i]);
    }
}

}  // namespace pacman_b200
