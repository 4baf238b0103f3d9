// Finite-element transfer NEAREST_NEAREST of the B200 engine
// (src/finite_elements/FTNearest.hpp:27-56): every target takes the value of
// its nearest source.  The reference queries nearest(1) on an ArborX BVH of
// the sources (callback src/finite_elements/utils/ArborXCallbacks.hpp:172-182);
// here the sources sit in a uniform cell grid (about one source per cell) and
// each target scans shells of cells around its own cell, nearest first, until
// no unscanned cell can hold a closer source.  Ties go to the lowest source
// index (ArborX's tie order is not reproducible; this convention makes the
// result deterministic).  Squared distances are formed as everywhere else in
// this engine (sqdist3), so the chosen source is exactly the CPU oracle's.
#include <algorithm>
#include <cmath>

#include "plan.hpp"

namespace pacman_b200 {

namespace {

// One thread per target.  After shell R (cells at Chebyshev cell distance R
// from the target's cell) every unscanned source lies at least R cell widths
// away, one cell less with a source that rounding put into the neighbouring
// cell: the scan stops once the best squared distance is below ((R - 1) h)^2.
// The shells are bounded by the grid, so the loop ends.
__global__ void k_fe_nearest(int64_t M, const double4 *__restrict__ tgt, GridView g, double h,
                             const double4 *__restrict__ src, const double *__restrict__ vals,
                             double *__restrict__ out) {
  const int rmax = max(g.nc[0], max(g.nc[1], g.nc[2]));
  for (int64_t t = blockIdx.x * int64_t(blockDim.x) + threadIdx.x; t < M;
       t += int64_t(gridDim.x) * blockDim.x) {
    const double4 y = tgt[t];
    const int cx = cell_coord(y.x, g.lo[0], g.inv_h, g.nc[0]);
    const int cy = cell_coord(y.y, g.lo[1], g.inv_h, g.nc[1]);
    const int cz = cell_coord(y.z, g.lo[2], g.inv_h, g.nc[2]);
    double best = 0.0;
    int bi = -1;
    auto scan = [&](int s, int e) {
      for (int i = s; i < e; ++i) {
        const int id = g.items[i];
        const double4 x = src[id];
        const double d2 = sqdist3(y.x, y.y, y.z, x.x, x.y, x.z);
        if (bi < 0 || d2 < best || (d2 == best && id < bi)) {
          best = d2;
          bi = id;
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
          if (face) {  // the whole z run of this column is on the shell
            const int z0 = max(cz - R, 0), z1 = min(cz + R, g.nc[2] - 1);
            scan(g.start[base + z0], g.start[base + z1 + 1]);
          } else {  // only its two ends
            if (cz - R >= 0) scan(g.start[base + cz - R], g.start[base + cz - R + 1]);
            if (cz + R < g.nc[2]) scan(g.start[base + cz + R], g.start[base + cz + R + 1]);
          }
        }
      if (bi >= 0 && R >= 1) {
        const double lim = double(R - 1) * h;
        if (best < lim * lim) break;
      }
    }
    out[t] = bi >= 0 ? vals[bi] : 0.0;
  }
}

}  // namespace

void fe_nearest(int dim, const double *src_dev, int64_t n, const double *vals_dev,
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
  const int blocks = int(std::max<int64_t>(1, std::min<int64_t>((m + 127) / 128, 148 * 32)));
  k_fe_nearest<<<blocks, 128, 0, st>>>(m, tgt4.as<double4>(), grid.view, h,
                                       src4.as<double4>(), vals_dev, out_dev);
  note_launch();
  PB_CUDA(cudaGetLastError());
  PB_CUDA(host_sync(st));
}

}  // namespace pacman_b200
