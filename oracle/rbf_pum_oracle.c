/*
 * CPU oracle for the RBF-PUM transfer -- TEST INFRASTRUCTURE ONLY.
 *
 * Plain C11 / FP64 restatement of PACMAN's RBF-PUM algorithm.  Each function
 * cites the reference file:line it restates (paths relative to the
 * messahelramzi/pacman source tree).  Only tests/, __graft_entry__.smoke() and
 * bench.py's CPU-baseline leg may use it; the product never links it.
 *
 * Arithmetic conventions (shared bit-for-bit with the CUDA kernels):
 *  - squared distance: acc = 0; for each axis d: t = b[d]-a[d]; acc = fma(t,t,acc)
 *    (src/rbf_pum/utils/operators.hpp:125-137, contracted as the reference's
 *    x86-64-v3 / nvcc builds contract it);
 *  - sphere membership (ArborX 2.1 intersects(Sphere, Point), un-vendored):
 *    sqrt(squared distance) <= radius;
 *  - nearest-point ties break toward the lowest point index;
 *  - candidate centre coordinate: fma(spacing_a, (double)coord_a, lower_a)
 *    (src/rbf_pum/clustering/clustering.hpp:199-202);
 *  - per-patch index lists are sorted ascending (ArborX returns them in
 *    traversal order, which is not reproducible; the set is the same).
 *
 * Deviations from the reference, all confined to degenerate patches whose
 * polynomial block loses an axis (clustering/serial_ops.hpp:108-139):
 *  the reference re-runs its SVD on a matrix whose dropped columns still hold
 *  the previous SVD's workspace, re-views the buffer with a new column count
 *  (a reshuffle under LayoutRight), and when every axis is dropped solves the
 *  least-squares problem on that workspace.  Those values depend on
 *  un-vendored KokkosKernels internals; this oracle uses the intended
 *  semantics instead: Q = [1, x_active], condition = sigma_max / max(sigma_min,
 *  1e-14) of exactly that matrix, least squares on exactly that matrix.
 */
#include "rbf_pum_oracle.h"

#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_EPS 1.0e-14 /* fp_consts::epsilon(), src/common/types.hpp:98 */
#define ORC_COND_MAX 1.0e5 /* serial_ops.hpp:130 */

static char g_err[256];
static void set_err(const char *m) {
  strncpy(g_err, m, sizeof(g_err) - 1);
  g_err[sizeof(g_err) - 1] = 0;
}
const char *orc_last_error(void) { return g_err; }

int orc_set_threads(int nthreads) {
#ifdef _OPENMP
  if (nthreads > 0) omp_set_num_threads(nthreads);
  return omp_get_max_threads();
#else
  (void)nthreads;
  return 1;
#endif
}

/* ------------------------------------------------------------------------ */
/* Geometry helpers                                                         */
/* ------------------------------------------------------------------------ */

/* operators.hpp:125-137 (SquaredDifference) / :150-158 (NoCheck). */
static inline double sqdist(const double *a, const double *b, int dim) {
  double acc = 0.0;
  for (int d = 0; d < dim; ++d) {
    const double t = b[d] - a[d];
    acc = fma(t, t, acc);
  }
  return acc;
}

typedef struct {
  int dim;
  double lo[3];
  double inv_h;
  int64_t nc[3];
  int64_t ncells;
  int64_t *start; /* ncells + 1 */
  int32_t *items; /* point ids, by cell, ascending id within a cell */
  int64_t nitems;
} grid_t;

/* Uniform grid of cell size h >= radius over the source bounding box grown
 * by h on every side.  A point whose distance to a query inside the source
 * box is <= radius lies in one of the 3^dim cells around the query's cell. */
static int grid_build(grid_t *g, int dim, const double *pts, int64_t npts,
                      const double *bb_lo, const double *bb_hi, double radius,
                      int64_t cap_cells) {
  memset(g, 0, sizeof(*g));
  g->dim = dim;
  double h = radius * (1.0 + 0x1p-20);
  for (int it = 0; it < 64; ++it) {
    int64_t tot = 1;
    int ok = 1;
    for (int d = 0; d < dim; ++d) {
      const double ext = (bb_hi[d] - bb_lo[d]) + 2.0 * h;
      const double c = floor(ext / h) + 1.0;
      if (c > 1.0e9) { ok = 0; break; }
      g->nc[d] = (int64_t)c;
      if (tot > cap_cells / g->nc[d] + 1) { ok = 0; break; }
      tot *= g->nc[d];
    }
    if (ok && tot <= cap_cells) { g->ncells = tot; break; }
    h *= 1.5;
  }
  if (g->ncells == 0) { set_err("grid: could not size the cell grid"); return -3; }
  for (int d = 0; d < dim; ++d) g->lo[d] = bb_lo[d] - h;
  g->inv_h = 1.0 / h;
  for (int d = dim; d < 3; ++d) { g->nc[d] = 1; g->lo[d] = 0.0; }

  int64_t *cell_of = (int64_t *)malloc(sizeof(int64_t) * (size_t)(npts > 0 ? npts : 1));
  g->start = (int64_t *)calloc((size_t)g->ncells + 1, sizeof(int64_t));
  if (!cell_of || !g->start) { free(cell_of); set_err("grid: out of memory"); return -4; }
  int64_t kept = 0;
  for (int64_t i = 0; i < npts; ++i) {
    const double *p = pts + 3 * i;
    int64_t cid = 0;
    int inside = 1;
    for (int d = 0; d < dim; ++d) {
      const double hi = bb_hi[d] + h;
      if (!(p[d] >= g->lo[d] && p[d] <= hi)) { inside = 0; break; }
      int64_t c = (int64_t)floor((p[d] - g->lo[d]) * g->inv_h);
      if (c < 0) c = 0;
      if (c >= g->nc[d]) c = g->nc[d] - 1;
      cid = cid * g->nc[d] + c;
    }
    cell_of[i] = inside ? cid : -1;
    if (inside) { g->start[cid + 1]++; kept++; }
  }
  for (int64_t c = 0; c < g->ncells; ++c) g->start[c + 1] += g->start[c];
  g->items = (int32_t *)malloc(sizeof(int32_t) * (size_t)(kept > 0 ? kept : 1));
  int64_t *cur = (int64_t *)malloc(sizeof(int64_t) * (size_t)g->ncells);
  if (!g->items || !cur) { free(cell_of); free(cur); set_err("grid: out of memory"); return -4; }
  memcpy(cur, g->start, sizeof(int64_t) * (size_t)g->ncells);
  for (int64_t i = 0; i < npts; ++i)
    if (cell_of[i] >= 0) g->items[cur[cell_of[i]]++] = (int32_t)i;
  g->nitems = kept;
  free(cur);
  free(cell_of);
  return 0;
}

static void grid_free(grid_t *g) {
  free(g->start);
  free(g->items);
  memset(g, 0, sizeof(*g));
}

/* Cell range [lo_c, hi_c] per axis around query q. */
static void grid_range(const grid_t *g, const double *q, int64_t *lo_c, int64_t *hi_c) {
  for (int d = 0; d < 3; ++d) {
    if (d >= g->dim) { lo_c[d] = 0; hi_c[d] = 0; continue; }
    int64_t c = (int64_t)floor((q[d] - g->lo[d]) * g->inv_h);
    int64_t a = c - 1, b = c + 1;
    if (a < 0) a = 0;
    if (b > g->nc[d] - 1) b = g->nc[d] - 1;
    lo_c[d] = a;
    hi_c[d] = b;
  }
}

/* Nearest point to q (lowest index on ties) among those with squared distance
 * <= r2.  Returns -1 when none (the reference then tags the centre). */
static int64_t nearest_within(const grid_t *g, const double *pts, int64_t npts,
                              const double *q, double r2, int brute, double *d2_out) {
  double best = INFINITY;
  int64_t bi = -1;
  if (brute) {
    for (int64_t i = 0; i < npts; ++i) {
      const double d2 = sqdist(q, pts + 3 * i, g->dim);
      if (d2 < best || (d2 == best && i < bi)) { best = d2; bi = i; }
    }
  } else {
    int64_t lc[3], hc[3];
    grid_range(g, q, lc, hc);
    for (int64_t c0 = lc[0]; c0 <= hc[0]; ++c0)
      for (int64_t c1 = lc[1]; c1 <= hc[1]; ++c1)
        for (int64_t c2 = lc[2]; c2 <= hc[2]; ++c2) {
          const int64_t cid = (c0 * g->nc[1] + c1) * g->nc[2] + c2;
          for (int64_t s = g->start[cid]; s < g->start[cid + 1]; ++s) {
            const int64_t i = g->items[s];
            const double d2 = sqdist(q, pts + 3 * i, g->dim);
            if (d2 < best || (d2 == best && i < bi)) { best = d2; bi = i; }
          }
        }
  }
  if (d2_out) *d2_out = best;
  if (bi < 0 || !(best <= r2)) return -1;
  return bi;
}

static int cmp_i32(const void *a, const void *b) {
  const int32_t x = *(const int32_t *)a, y = *(const int32_t *)b;
  return (x > y) - (x < y);
}

/* All points with sqrt(d2) <= radius, ascending index; returns the count and
 * writes up to cap ids into out (out may be NULL to count only). */
static int64_t members(const grid_t *g, const double *pts, int64_t npts,
                       const double *q, double radius, int brute, int32_t *out) {
  int64_t cnt = 0;
  if (brute) {
    for (int64_t i = 0; i < npts; ++i)
      if (sqrt(sqdist(q, pts + 3 * i, g->dim)) <= radius) {
        if (out) out[cnt] = (int32_t)i;
        cnt++;
      }
    return cnt;
  }
  int64_t lc[3], hc[3];
  grid_range(g, q, lc, hc);
  for (int64_t c0 = lc[0]; c0 <= hc[0]; ++c0)
    for (int64_t c1 = lc[1]; c1 <= hc[1]; ++c1)
      for (int64_t c2 = lc[2]; c2 <= hc[2]; ++c2) {
        const int64_t cid = (c0 * g->nc[1] + c1) * g->nc[2] + c2;
        for (int64_t s = g->start[cid]; s < g->start[cid + 1]; ++s) {
          const int64_t i = g->items[s];
          if (sqrt(sqdist(q, pts + 3 * i, g->dim)) <= radius) {
            if (out) out[cnt] = (int32_t)i;
            cnt++;
          }
        }
      }
  if (out && cnt > 1) qsort(out, (size_t)cnt, sizeof(int32_t), cmp_i32);
  return cnt;
}

/* ------------------------------------------------------------------------ */
/* Plan                                                                     */
/* ------------------------------------------------------------------------ */

struct orc_plan {
  int dim;
  int64_t n, m;
  double *src; /* n x 3, padded with zeros */
  double *tgt; /* m x 3 */
  double lo[3], hi[3];
  double radius;
  int64_t ncand;
  int64_t K;
  double *centers; /* K x 3 */
  int64_t *soff, *toff;
  int32_t *sidx, *tidx;
  grid_t cgrid; /* grid of centres (weights) */
  int brute;
};

void orc_free(orc_plan *p) {
  if (!p) return;
  free(p->src);
  free(p->tgt);
  free(p->centers);
  free(p->soff);
  free(p->toff);
  free(p->sidx);
  free(p->tidx);
  grid_free(&p->cgrid);
  free(p);
}

double orc_radius(const orc_plan *p) { return p->radius; }
int64_t orc_num_patches(const orc_plan *p) { return p->K; }
int64_t orc_num_candidates(const orc_plan *p) { return p->ncand; }
int64_t orc_src_nnz(const orc_plan *p) { return p->soff ? p->soff[p->K] : 0; }
int64_t orc_tgt_nnz(const orc_plan *p) { return p->toff ? p->toff[p->K] : 0; }
void orc_centers(const orc_plan *p, double *out) {
  for (int64_t k = 0; k < p->K; ++k)
    for (int d = 0; d < p->dim; ++d) out[k * p->dim + d] = p->centers[3 * k + d];
}
void orc_src_csr(const orc_plan *p, int64_t *off, int32_t *idx) {
  memcpy(off, p->soff, sizeof(int64_t) * (size_t)(p->K + 1));
  memcpy(idx, p->sidx, sizeof(int32_t) * (size_t)p->soff[p->K]);
}
void orc_tgt_csr(const orc_plan *p, int64_t *off, int32_t *idx) {
  memcpy(off, p->toff, sizeof(int64_t) * (size_t)(p->K + 1));
  memcpy(idx, p->tidx, sizeof(int32_t) * (size_t)p->toff[p->K]);
}

static int cmp_dbl(const void *a, const void *b) {
  const double x = *(const double *)a, y = *(const double *)b;
  return (x > y) - (x < y);
}

/* k-th smallest (1-based k) of v[0..n) by quickselect (values only). */
static double kth_smallest(double *v, int64_t n, int64_t k) {
  int64_t lo = 0, hi = n - 1, want = k - 1;
  while (lo < hi) {
    const double piv = v[lo + (hi - lo) / 2];
    int64_t i = lo, j = hi;
    while (i <= j) {
      while (v[i] < piv) i++;
      while (v[j] > piv) j--;
      if (i <= j) { double t = v[i]; v[i] = v[j]; v[j] = t; i++; j--; }
    }
    if (want <= j) hi = j;
    else if (want >= i) lo = i;
    else return v[want];
  }
  return v[want];
}

/* FindRadius: src/rbf_pum/clustering/clusters_radius.hpp:22-125. */
static int find_radius(orc_plan *p, int k_nodes) {
  const int dim = p->dim;
  double center[3] = {0, 0, 0}, samples[7][3];
  for (int a = 0; a < dim; ++a) center[a] = (p->lo[a] + p->hi[a]) / 2.;
  const int ns = 2 * dim + 1;
  for (int s = 0; s < ns; ++s)
    for (int a = 0; a < 3; ++a) samples[s][a] = center[a];
  for (int a = 0; a < dim; ++a) {
    const double len = fabs(p->hi[a] - p->lo[a]);
    double s_a = center[a];
    s_a -= len * 0.25;
    samples[a + 1][a] = s_a;
    s_a += len * 0.5;
    samples[dim + a + 1][a] = s_a;
  }
  /* Projection onto the nearest source (callbacks.hpp:38-49, :139-149). */
  double proj[7][3];
  for (int s = 0; s < ns; ++s) {
    double best = INFINITY;
    int64_t bi = 0;
    for (int64_t i = 0; i < p->n; ++i) {
      const double d2 = sqdist(samples[s], p->src + 3 * i, dim);
      if (d2 < best) { best = d2; bi = i; }
    }
    for (int a = 0; a < 3; ++a) proj[s][a] = p->src[3 * bi + a];
  }
  /* k nearest squared distances, their max (callbacks.hpp:21-34). */
  const int64_t k = (k_nodes < p->n) ? k_nodes : p->n;
  double *d2 = (double *)malloc(sizeof(double) * (size_t)p->n);
  if (!d2) { set_err("radius: out of memory"); return -4; }
  double maxr[7];
  for (int s = 0; s < ns; ++s) {
    for (int64_t i = 0; i < p->n; ++i) d2[i] = sqdist(proj[s], p->src + 3 * i, dim);
    maxr[s] = kth_smallest(d2, p->n, k);
  }
  free(d2);
  qsort(maxr, (size_t)ns, sizeof(double), cmp_dbl);
  p->radius = sqrt(maxr[dim]);
  if (!(p->radius > 0.0) || !isfinite(p->radius)) {
    set_err("degenerate patch radius (zero or non-finite)");
    return -5;
  }
  return 0;
}

/* Neighbour offsets: clustering.hpp:34-116 (3D table :96-102). */
static int neighbor_offsets(int dim, const int64_t *shape, int64_t *off) {
  if (dim == 1) { off[0] = -1; off[1] = 1; return 2; }
  if (dim == 2) {
    static const int o2[8][2] = {{-1, -1}, {-1, 0}, {-1, 1}, {0, -1},
                                 {0, 1},   {1, -1}, {1, 0},  {1, 1}};
    for (int i = 0; i < 8; ++i) off[i] = o2[i][1] + o2[i][0] * shape[1];
    return 8;
  }
  static const int o3[26][3] = {
      {-1, -1, -1}, {-1, -1, 0}, {-1, -1, 1}, {-1, 0, 0},  {-1, 0, 1},
      {-1, 0, -1},  {-1, 1, 0},  {-1, 1, 1},  {-1, 1, -1}, {0, -1, -1},
      {0, -1, 0},   {0, -1, 1},  {0, 0, 1},   {0, 0, -1},  {0, 1, 0},
      {0, 1, 1},    {0, 1, -1},  {1, -1, -1}, {1, -1, 0},  {1, -1, 1},
      {1, 0, 0},    {1, 0, 1},   {1, 0, -1},  {1, 1, 0},   {1, 1, 1},
      {1, 1, -1}};
  for (int i = 0; i < 26; ++i)
    off[i] = o3[i][2] + o3[i][1] * shape[2] + o3[i][0] * shape[2] * shape[1];
  return 26;
}

/* CreateClusters: src/rbf_pum/clustering/clustering.hpp:127-271. */
static int create_clusters(orc_plan *p, double overlap, const grid_t *sg,
                           const grid_t *tg) {
  const int dim = p->dim;
  const double r = p->radius;
  const double r2 = r * r;
  const double spacing = sqrt(4.0 / dim) * r * (1.0 - overlap);
  int64_t shape[3] = {1, 1, 1};
  double dist[3] = {0, 0, 0};
  double min_d = DBL_MAX;
  int64_t nb = 1;
  for (int a = 0; a < dim; ++a) {
    double edge = p->hi[a] - p->lo[a];
    edge = (edge < 0) ? -edge : edge;
    const double q = fmax(1.0, edge / spacing);
    if (!(q < 2.0e9)) { set_err("candidate grid too large"); return -6; }
    shape[a] = (int64_t)ceil(q);
    dist[a] = edge / (double)shape[a];
    if (dist[a] < min_d) min_d = dist[a];
    shape[a] += 1;
    nb *= shape[a];
    if (nb > INT32_MAX) { set_err("candidate grid exceeds int32"); return -6; }
  }
  p->ncand = nb;
  double *c = (double *)calloc((size_t)nb * 3, sizeof(double));
  unsigned char *alive = (unsigned char *)malloc((size_t)nb);
  if (!c || !alive) { free(c); free(alive); set_err("clusters: out of memory"); return -4; }

  /* Steps 5-8: candidate fill (row-major storage, last axis fastest),
   * source/target emptiness tags, snap to the nearest source. */
#pragma omp parallel for schedule(static)
  for (int64_t s = 0; s < nb; ++s) {
    int64_t coords[3] = {0, 0, 0}, t = s;
    for (int a = dim - 1; a >= 0; --a) { coords[a] = t % shape[a]; t /= shape[a]; }
    double q[3] = {0, 0, 0};
    for (int a = 0; a < dim; ++a) q[a] = fma(dist[a], (double)coords[a], p->lo[a]);
    const int64_t ns = nearest_within(sg, p->src, p->n, q, r2, p->brute, NULL);
    int ok = (ns >= 0);
    if (ok && p->m > 0) ok = nearest_within(tg, p->tgt, p->m, q, r2, p->brute, NULL) >= 0;
    alive[s] = (unsigned char)ok;
    if (ok)
      for (int a = 0; a < 3; ++a) c[3 * s + a] = p->src[3 * ns + a];
    else
      for (int a = 0; a < 3; ++a) c[3 * s + a] = q[a];
  }

  /* Step 9: order-dependent proximity pruning (clustering.hpp:228-254). */
  double thr = 0.4 * min_d;
  thr *= thr;
  int64_t off[26];
  const int noff = neighbor_offsets(dim, shape, off);
  for (int64_t i = 0; i < nb; ++i) {
    if (!alive[i]) continue;
    for (int o = 0; o < noff; ++o) {
      const int64_t j = i + off[o];
      if (j >= 0 && j < nb && alive[j] && sqdist(c + 3 * i, c + 3 * j, dim) < thr) {
        alive[i] = 0;
        break;
      }
    }
  }

  /* Step 10: re-tag centres without targets; step 11: stable compaction. */
  if (p->m > 0) {
#pragma omp parallel for schedule(static)
    for (int64_t s = 0; s < nb; ++s)
      if (alive[s] && nearest_within(tg, p->tgt, p->m, c + 3 * s, r2, p->brute, NULL) < 0)
        alive[s] = 0;
  }
  int64_t K = 0;
  for (int64_t s = 0; s < nb; ++s) K += alive[s];
  p->K = K;
  p->centers = (double *)malloc(sizeof(double) * 3 * (size_t)(K > 0 ? K : 1));
  if (!p->centers) { free(c); free(alive); set_err("clusters: out of memory"); return -4; }
  int64_t w = 0;
  for (int64_t s = 0; s < nb; ++s)
    if (alive[s]) { memcpy(p->centers + 3 * w, c + 3 * s, 3 * sizeof(double)); w++; }
  free(c);
  free(alive);
  return 0;
}

/* Patch membership lists (solver.hpp:45-66, callbacks.hpp:100-114). */
static int build_csr(orc_plan *p, const grid_t *g, const double *pts, int64_t npts,
                     double radius, int64_t **off_out, int32_t **idx_out) {
  const int64_t K = p->K;
  int64_t *off = (int64_t *)calloc((size_t)K + 1, sizeof(int64_t));
  if (!off) { set_err("csr: out of memory"); return -4; }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t k = 0; k < K; ++k)
    off[k + 1] = members(g, pts, npts, p->centers + 3 * k, radius, p->brute, NULL);
  for (int64_t k = 0; k < K; ++k) off[k + 1] += off[k];
  int32_t *idx = (int32_t *)malloc(sizeof(int32_t) * (size_t)(off[K] > 0 ? off[K] : 1));
  if (!idx) { free(off); set_err("csr: out of memory"); return -4; }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t k = 0; k < K; ++k)
    members(g, pts, npts, p->centers + 3 * k, radius, p->brute, idx + off[k]);
  *off_out = off;
  *idx_out = idx;
  return 0;
}

int orc_build(int dim, const double *src, int64_t n, const double *tgt, int64_t m,
              int nodes_per_cluster, double overlap, int brute, orc_plan **out) {
  *out = NULL;
  if (dim < 1 || dim > 3) { set_err("dimension must be 1, 2 or 3"); return -1; }
  if (n <= 0) { set_err("no source points"); return -2; }
  if (nodes_per_cluster <= 0) { set_err("nodes_per_cluster must be > 0"); return -1; }
  if (!(overlap > 0.0 && overlap < 1.0)) { set_err("overlap must be in (0,1)"); return -1; }
  orc_plan *p = (orc_plan *)calloc(1, sizeof(orc_plan));
  p->dim = dim;
  p->n = n;
  p->m = m;
  p->brute = brute;
  p->src = (double *)calloc((size_t)n * 3, sizeof(double));
  p->tgt = (double *)calloc((size_t)(m > 0 ? m : 1) * 3, sizeof(double));
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) p->src[3 * i + d] = src[i * dim + d];
  for (int64_t i = 0; i < m; ++i)
    for (int d = 0; d < dim; ++d) p->tgt[3 * i + d] = tgt[i * dim + d];
  /* Source bounding box (the ArborX BVH bounds, interpolator.hpp:81-84). */
  for (int d = 0; d < 3; ++d) { p->lo[d] = 0; p->hi[d] = 0; }
  for (int d = 0; d < dim; ++d) { p->lo[d] = INFINITY; p->hi[d] = -INFINITY; }
  for (int64_t i = 0; i < n; ++i)
    for (int d = 0; d < dim; ++d) {
      const double v = p->src[3 * i + d];
      if (v < p->lo[d]) p->lo[d] = v;
      if (v > p->hi[d]) p->hi[d] = v;
    }
  int rc = find_radius(p, nodes_per_cluster);
  if (rc) { orc_free(p); return rc; }

  grid_t sg, tg;
  const int64_t cap_s = (n * 4 > (1 << 16) ? n * 4 : (1 << 16));
  const int64_t cap_t = (m * 4 > (1 << 16) ? m * 4 : (1 << 16));
  if ((rc = grid_build(&sg, dim, p->src, n, p->lo, p->hi, p->radius, cap_s))) { orc_free(p); return rc; }
  if ((rc = grid_build(&tg, dim, p->tgt, m, p->lo, p->hi, p->radius, cap_t))) { grid_free(&sg); orc_free(p); return rc; }
  rc = create_clusters(p, overlap, &sg, &tg);
  if (!rc) rc = build_csr(p, &sg, p->src, n, p->radius, &p->soff, &p->sidx);
  if (!rc) rc = build_csr(p, &tg, p->tgt, m, p->radius - ORC_EPS, &p->toff, &p->tidx);
  grid_free(&sg);
  grid_free(&tg);
  if (!rc) {
    const int64_t cap_c = (p->K * 4 > (1 << 16) ? p->K * 4 : (1 << 16));
    rc = grid_build(&p->cgrid, dim, p->centers, p->K, p->lo, p->hi, p->radius, cap_c);
  }
  if (rc) { orc_free(p); return rc; }
  *out = p;
  return 0;
}

/* ------------------------------------------------------------------------ */
/* Bases                                                                    */
/* ------------------------------------------------------------------------ */

/* Wendland C0..C8, src/rbf_pum/solver/rbf_functions.hpp:22-150 (the
 * reference's pow() calls and its fma, with a*b+c contracted). */
static inline double wendland(int basis, double r, double rinv) {
  const double p = r * rinv;
  const double mask = (double)(r >= 0.0 && p < 1.0 && p >= 0.0);
  const double q = 1.0 - p;
  switch (basis) {
  case ORC_WENDLAND_C0:
    return mask * (q * q);
  case ORC_WENDLAND_C2:
    return mask * (pow(q, 4) * fma(4.0, p, 1.0));
  case ORC_WENDLAND_C4:
    return mask * (pow(q, 6) * fma(35.0, pow(p, 2), fma(18.0, p, 3.0)));
  case ORC_WENDLAND_C6:
    return mask * (pow(q, 8) *
                   (fma(32.0, pow(p, 3), 25.0 * pow(p, 2)) + fma(8.0, p, 1.0)));
  case ORC_WENDLAND_C8: {
    double t = fma(1287.0, pow(p, 4), 1350.0 * pow(p, 3));
    t = fma(630.0, pow(p, 2), t);
    return mask * (pow(q, 10) * (t + fma(150.0, p, 15.0)));
  }
  default:
    return NAN;
  }
}

double orc_wendland(int basis, double r, double rho) { return wendland(basis, r, 1.0 / rho); }

/* ------------------------------------------------------------------------ */
/* Per-patch dense algebra                                                  */
/* ------------------------------------------------------------------------ */

/* Singular values of the n x pv matrix Q (column-major, ld n): Householder QR
 * then one-sided Jacobi on R.  Values are returned in decreasing order; when
 * n < pv the missing ones are 0.  Stands in for KokkosBatched::SerialSVD
 * (serial_solve.hpp:100-110), which is not vendored. */
static void singular_values(const double *Q, int64_t n, int pv, double *sig) {
  double R[4 * 4] = {0};
  double W[4 * 64];
  int rows = (int)(n < pv ? n : pv);
  /* Work on a copy; n may be large, so do the QR column by column. */
  double *A = (double *)malloc(sizeof(double) * (size_t)n * (size_t)pv);
  memcpy(A, Q, sizeof(double) * (size_t)n * (size_t)pv);
  (void)W;
  for (int j = 0; j < pv && j < n; ++j) {
    double *a = A + (size_t)j * n;
    double xn = 0.0;
    for (int64_t i = j + 1; i < n; ++i) xn = fma(a[i], a[i], xn);
    xn = sqrt(xn);
    const double alpha = a[j];
    if (xn == 0.0) continue;
    const double beta = -copysign(hypot(alpha, xn), alpha);
    const double tau = (beta - alpha) / beta;
    const double sc = 1.0 / (alpha - beta);
    for (int64_t i = j + 1; i < n; ++i) a[i] *= sc;
    a[j] = beta;
    for (int c2 = j + 1; c2 < pv; ++c2) {
      double *b = A + (size_t)c2 * n;
      double w = b[j];
      for (int64_t i = j + 1; i < n; ++i) w = fma(a[i], b[i], w);
      w *= tau;
      b[j] -= w;
      for (int64_t i = j + 1; i < n; ++i) b[i] = fma(-w, a[i], b[i]);
    }
  }
  for (int c2 = 0; c2 < pv; ++c2)
    for (int r2 = 0; r2 <= c2 && r2 < rows; ++r2) R[r2 * 4 + c2] = A[(size_t)c2 * n + r2];
  free(A);
  /* One-sided Jacobi on the columns of R (rows x pv). */
  for (int sweep = 0; sweep < 80; ++sweep) {
    int rotated = 0;
    for (int i = 0; i < pv; ++i)
      for (int j = i + 1; j < pv; ++j) {
        double al = 0, be = 0, ga = 0;
        for (int r2 = 0; r2 < rows; ++r2) {
          al += R[r2 * 4 + i] * R[r2 * 4 + i];
          be += R[r2 * 4 + j] * R[r2 * 4 + j];
          ga += R[r2 * 4 + i] * R[r2 * 4 + j];
        }
        if (ga == 0.0 || fabs(ga) <= 1e-15 * sqrt(al * be)) continue;
        rotated = 1;
        const double zeta = (be - al) / (2.0 * ga);
        const double t = copysign(1.0, zeta) / (fabs(zeta) + sqrt(1.0 + zeta * zeta));
        const double cs = 1.0 / sqrt(1.0 + t * t), sn = cs * t;
        for (int r2 = 0; r2 < rows; ++r2) {
          const double x = R[r2 * 4 + i], y = R[r2 * 4 + j];
          R[r2 * 4 + i] = cs * x - sn * y;
          R[r2 * 4 + j] = sn * x + cs * y;
        }
      }
    if (!rotated) break;
  }
  for (int j = 0; j < pv; ++j) {
    double s = 0;
    for (int r2 = 0; r2 < rows; ++r2) s += R[r2 * 4 + j] * R[r2 * 4 + j];
    sig[j] = sqrt(s);
  }
  /* n < pv: only n of them exist; the rest are zero. */
  qsort(sig, (size_t)pv, sizeof(double), cmp_dbl);
  for (int i = 0; i < pv / 2; ++i) { double t = sig[i]; sig[i] = sig[pv - 1 - i]; sig[pv - 1 - i] = t; }
  if (n < pv)
    for (int j = (int)n; j < pv; ++j) sig[j] = 0.0;
}

typedef struct {
  double *A;   /* n x n row-major */
  double *Q;   /* n x 4 column-major */
  double *B;   /* n x F column-major (right-hand sides / residuals) */
  double *X;   /* n x 4 */
  int64_t cap;
  int capF;
} work_t;

static int work_reserve(work_t *w, int64_t n, int F) {
  if (n <= w->cap && F <= w->capF) return 0;
  free(w->A); free(w->Q); free(w->B); free(w->X);
  w->cap = n > w->cap ? n : w->cap;
  w->capF = F > w->capF ? F : w->capF;
  w->A = (double *)malloc(sizeof(double) * (size_t)w->cap * (size_t)w->cap);
  w->Q = (double *)malloc(sizeof(double) * (size_t)w->cap * 4);
  w->B = (double *)malloc(sizeof(double) * (size_t)w->cap * (size_t)w->capF);
  w->X = (double *)malloc(sizeof(double) * (size_t)w->cap * 4);
  return (w->A && w->Q && w->B && w->X) ? 0 : -4;
}

static void fill_poly(double *P, int64_t rows, const double *pts, const int32_t *ids,
                      const int *act, int nact) {
  for (int64_t i = 0; i < rows; ++i) {
    P[i] = 1.0;
    for (int c = 0; c < nact; ++c) P[(size_t)(c + 1) * rows + i] = pts[3 * (int64_t)ids[i] + act[c]];
  }
}

/* One patch: solver.hpp:217-286 for F fields; writes local[m x F]. */
/* SerialFillQ with the SVD condition loop (serial_ops.hpp:108-139): while
 * sigma_max / max(sigma_min, eps) of Q = [1, x_active] exceeds 1e5, drop the
 * active axis with the smallest coordinate range (SerialDeactivateOneAxis,
 * serial_ops.hpp:28-57).  Q is n x 4 scratch; active[] and *pv are updated.
 * Returns 1 if an axis was dropped. */
static int poly_axes(const orc_plan *p, int64_t k, double *Q, int active[3], int *pv_io) {
  const int dim = p->dim;
  const int64_t n = p->soff[k + 1] - p->soff[k];
  const int32_t *si = p->sidx + p->soff[k];
  int pv = *pv_io, dropped = 0;
  int act[3], nact;
  for (;;) {
    nact = 0;
    for (int a = 0; a < dim; ++a) if (active[a]) act[nact++] = a;
    if (pv <= 1) break;
    fill_poly(Q, n, p->src, si, act, nact);
    double sig[4];
    singular_values(Q, n, pv, sig);
    const double cond = sig[0] / fmax(sig[pv - 1], ORC_EPS);
    if (!(cond > ORC_COND_MAX)) break;
    double range[3];
    for (int a = 0; a < dim; ++a) {
      if (!active[a]) { range[a] = DBL_MAX; continue; }
      double mn = p->src[3 * (int64_t)si[0] + a], mx = mn;
      for (int64_t i = 1; i < n; ++i) {
        const double v = p->src[3 * (int64_t)si[i] + a];
        if (v < mn) mn = v;
        if (mx < v) mx = v;
      }
      range[a] = fabs(mx - mn);
    }
    double mn = DBL_MAX;
    int mi = 0;
    for (int a = 0; a < dim; ++a) if (range[a] < mn) { mn = range[a]; mi = a; }
    active[mi] = 0;
    --pv;
    dropped = 1;
  }
  *pv_io = pv;
  return dropped;
}

int orc_poly_dropped(const orc_plan *p, int32_t *out) {
  int err = 0;
#pragma omp parallel
  {
    double *Q = NULL;
    int64_t cap = 0;
#pragma omp for schedule(dynamic, 64)
    for (int64_t k = 0; k < p->K; ++k) {
      const int64_t n = p->soff[k + 1] - p->soff[k];
      if (n > cap) {
        free(Q);
        cap = n;
        Q = (double *)malloc(sizeof(double) * (size_t)(4 * cap));
        if (!Q) { err = 1; cap = 0; }
      }
      int active[3] = {1, 1, 1};
      int pv = p->dim + 1;
      out[k] = Q ? poly_axes(p, k, Q, active, &pv) : -1;
    }
    free(Q);
  }
  if (err) { set_err("poly_dropped: out of memory"); return -4; }
  return 0;
}

static int solve_patch(const orc_plan *p, int64_t k, int basis, double rinv,
                       const double *vals, int F, int64_t ld, double *local,
                       work_t *w, int *dropped) {
  const int dim = p->dim;
  const int64_t n = p->soff[k + 1] - p->soff[k];
  const int64_t m = p->toff[k + 1] - p->toff[k];
  const int32_t *si = p->sidx + p->soff[k];
  const int32_t *ti = p->tidx + p->toff[k];
  if (work_reserve(w, n, F)) return -4;
  double *A = w->A, *Q = w->Q, *B = w->B;

  /* TeamFillA / TeamFillB (team_ops.hpp:35-52, :113-121). */
  for (int64_t i = 0; i < n; ++i) {
    const double *xi = p->src + 3 * (int64_t)si[i];
    for (int64_t j = i; j < n; ++j) {
      const double v = wendland(basis, sqrt(sqdist(xi, p->src + 3 * (int64_t)si[j], dim)), rinv);
      A[i * n + j] = v;
      A[j * n + i] = v;
    }
    for (int f = 0; f < F; ++f) B[(size_t)f * n + i] = vals[(int64_t)si[i] * ld + f];
  }

  int active[3] = {1, 1, 1};
  int pv = dim + 1;
  if (poly_axes(p, k, Q, active, &pv)) *dropped = 1;
  int act[3], nact = 0;
  for (int a = 0; a < dim; ++a) if (active[a]) act[nact++] = a;

  /* SerialSolveQR (serial_solve.hpp:46-67): Householder QR of Q, Q^T b,
   * back substitution with R; beta is pv x F. */
  fill_poly(Q, n, p->src, si, act, nact);
  double *X = w->X; /* copy of Q to factor */
  memcpy(X, Q, sizeof(double) * (size_t)n * (size_t)pv);
  double beta[4 * 8];
  double *Rhs = (double *)malloc(sizeof(double) * (size_t)n * (size_t)F);
  memcpy(Rhs, B, sizeof(double) * (size_t)n * (size_t)F);
  for (int j = 0; j < pv; ++j) {
    double *a = X + (size_t)j * n;
    double xn = 0.0;
    for (int64_t i = j + 1; i < n; ++i) xn = fma(a[i], a[i], xn);
    xn = sqrt(xn);
    const double alpha = a[j];
    if (xn == 0.0) continue;
    const double bta = -copysign(hypot(alpha, xn), alpha);
    const double tau = (bta - alpha) / bta;
    const double sc = 1.0 / (alpha - bta);
    for (int64_t i = j + 1; i < n; ++i) a[i] *= sc;
    a[j] = bta;
    for (int c2 = j + 1; c2 < pv + F; ++c2) {
      double *b = (c2 < pv) ? X + (size_t)c2 * n : Rhs + (size_t)(c2 - pv) * n;
      double s = b[j];
      for (int64_t i = j + 1; i < n; ++i) s = fma(a[i], b[i], s);
      s *= tau;
      b[j] -= s;
      for (int64_t i = j + 1; i < n; ++i) b[i] = fma(-s, a[i], b[i]);
    }
  }
  for (int f = 0; f < F; ++f) {
    const double *y = Rhs + (size_t)f * n;
    double *bt = beta + f * 4;
    for (int j = pv - 1; j >= 0; --j) {
      double s = y[j];
      for (int c2 = j + 1; c2 < pv; ++c2) s = fma(-X[(size_t)c2 * n + j], bt[c2], s);
      bt[j] = s / X[(size_t)j * n + j];
    }
  }
  free(Rhs);

  /* Residual b - Q beta (serial_ops.hpp:149-185). */
  for (int f = 0; f < F; ++f) {
    double *b = B + (size_t)f * n;
    const double *bt = beta + f * 4;
    for (int64_t i = 0; i < n; ++i) {
      double s = 0.0;
      for (int c = 0; c < pv; ++c) s = fma(Q[(size_t)c * n + i], bt[c], s);
      b[i] -= s;
    }
  }

  /* SerialLU (unblocked, no pivoting) + SerialSolveLU (serial_solve.hpp:76-84). */
  for (int64_t piv = 0; piv < n; ++piv) {
    const double a11 = A[piv * n + piv];
    for (int64_t i = piv + 1; i < n; ++i) A[i * n + piv] /= a11;
    for (int64_t i = piv + 1; i < n; ++i) {
      const double l = A[i * n + piv];
      double *ri = A + i * n;
      const double *rp = A + piv * n;
      for (int64_t j = piv + 1; j < n; ++j) ri[j] = fma(-l, rp[j], ri[j]);
    }
  }
  for (int f = 0; f < F; ++f) {
    double *b = B + (size_t)f * n;
    for (int64_t piv = 0; piv < n; ++piv) {
      const double bp = b[piv];
      for (int64_t i = piv + 1; i < n; ++i) b[i] = fma(-A[i * n + piv], bp, b[i]);
    }
    for (int64_t piv = n - 1; piv >= 0; --piv) {
      b[piv] /= A[piv * n + piv];
      const double bp = b[piv];
      for (int64_t i = 0; i < piv; ++i) b[i] = fma(-A[i * n + piv], bp, b[i]);
    }
  }

  /* local = E alpha + V beta (solver.hpp:270-273), E formed row by row. */
  for (int64_t i = 0; i < m; ++i) {
    const double *yi = p->tgt + 3 * (int64_t)ti[i];
    for (int f = 0; f < F; ++f) {
      const double *al = B + (size_t)f * n;
      double s = 0.0;
      for (int64_t j = 0; j < n; ++j) {
        const double e = wendland(basis, sqrt(sqdist(yi, p->src + 3 * (int64_t)si[j], dim)), rinv);
        s = fma(e, al[j], s);
      }
      const double *bt = beta + f * 4;
      double v = bt[0];
      for (int c = 0; c < nact; ++c) v = fma(yi[act[c]], bt[c + 1], v);
      local[i * F + f] = s + v;
    }
  }
  return 0;
}

/* Shepard weights of one target (solver.hpp:137-168): ascending centre ids
 * within the patch radius, their un-normalised C2 weights and the sum. */
static int64_t target_weights(const orc_plan *p, const double *y, int64_t *ids,
                              double *ws, int64_t cap, double *sum) {
  const double r = p->radius;
  const double rinv = 1.0 / r;
  int64_t cnt = 0;
  if (p->brute) {
    for (int64_t k = 0; k < p->K; ++k) {
      const double d = sqrt(sqdist(y, p->centers + 3 * k, p->dim));
      if (d <= r) {
        if (cnt < cap) { ids[cnt] = k; ws[cnt] = wendland(ORC_WENDLAND_C2, d, rinv); }
        cnt++;
      }
    }
  } else {
    const grid_t *g = &p->cgrid;
    int64_t lc[3], hc[3];
    /* Targets outside the grid domain (source box grown by one cell) are
     * farther than r from every centre. */
    for (int d = 0; d < p->dim; ++d) {
      const double c = floor((y[d] - g->lo[d]) * g->inv_h);
      if (!(c >= 0.0 && c < (double)g->nc[d])) { *sum = 0.0; return 0; }
    }
    grid_range(g, y, lc, hc);
    for (int64_t c0 = lc[0]; c0 <= hc[0]; ++c0)
      for (int64_t c1 = lc[1]; c1 <= hc[1]; ++c1)
        for (int64_t c2 = lc[2]; c2 <= hc[2]; ++c2) {
          const int64_t cid = (c0 * g->nc[1] + c1) * g->nc[2] + c2;
          for (int64_t s = g->start[cid]; s < g->start[cid + 1]; ++s) {
            const int64_t k = g->items[s];
            const double d = sqrt(sqdist(y, p->centers + 3 * k, p->dim));
            if (d <= r) {
              if (cnt < cap) { ids[cnt] = k; ws[cnt] = wendland(ORC_WENDLAND_C2, d, rinv); }
              cnt++;
            }
          }
        }
    /* Sort by centre id (insertion sort; lists are short). */
    const int64_t c = cnt < cap ? cnt : cap;
    for (int64_t i = 1; i < c; ++i) {
      int64_t kk = ids[i];
      double ww = ws[i];
      int64_t j = i - 1;
      while (j >= 0 && ids[j] > kk) { ids[j + 1] = ids[j]; ws[j + 1] = ws[j]; j--; }
      ids[j + 1] = kk;
      ws[j + 1] = ww;
    }
  }
  double s = 0.0;
  const int64_t c = cnt < cap ? cnt : cap;
  for (int64_t i = 0; i < c; ++i) s += ws[i];
  *sum = s;
  return cnt;
}

#define ORC_WCAP 4096

void orc_weight_sums(const orc_plan *p, double *sums) {
#pragma omp parallel
  {
    int64_t *ids = (int64_t *)malloc(sizeof(int64_t) * ORC_WCAP);
    double *ws = (double *)malloc(sizeof(double) * ORC_WCAP);
#pragma omp for schedule(static)
    for (int64_t t = 0; t < p->m; ++t) target_weights(p, p->tgt + 3 * t, ids, ws, ORC_WCAP, &sums[t]);
    free(ids);
    free(ws);
  }
}

static int64_t lower_bound_i32(const int32_t *a, int64_t n, int32_t v) {
  int64_t lo = 0, hi = n;
  while (lo < hi) {
    const int64_t mid = lo + (hi - lo) / 2;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo;
}

int orc_solve(const orc_plan *p, int basis, double support_radius, const double *vals,
              int F, int64_t ld, double *out, double *local_out,
              const int64_t *plist, int64_t nplist, int64_t *stats, int32_t *dropped_out) {
  if (basis < ORC_WENDLAND_C0 || basis > ORC_WENDLAND_C8) { set_err("unknown basis"); return -1; }
  if (F < 1 || F > 8) { set_err("nfields must be in [1, 8]"); return -1; }
  if (!(support_radius > 0.0)) { set_err("support radius must be > 0"); return -1; }
  const double rinv = 1.0 / support_radius;
  const int64_t nnz_t = orc_tgt_nnz(p);
  double *local = local_out ? local_out
                            : (double *)malloc(sizeof(double) * (size_t)(nnz_t > 0 ? nnz_t : 1) * (size_t)F);
  unsigned char *done = (unsigned char *)calloc((size_t)(p->K > 0 ? p->K : 1), 1);
  const int64_t np = plist ? nplist : p->K;
  int err = 0, ndrop = 0;
  int64_t s3 = 0, nmax = 0, sn = 0, sm = 0;
#pragma omp parallel reduction(+ : ndrop, s3, sn, sm) reduction(max : nmax)
  {
    work_t w = {0};
#pragma omp for schedule(dynamic, 1)
    for (int64_t q = 0; q < np; ++q) {
      const int64_t k = plist ? plist[q] : q;
      int dropped = 0;
      if (solve_patch(p, k, basis, rinv, vals, F, ld, local + p->toff[k] * F, &w, &dropped)) err = 1;
      done[k] = 1;
      ndrop += dropped;
      if (dropped_out) dropped_out[k] = dropped;
      const int64_t n = p->soff[k + 1] - p->soff[k];
      s3 += n * n * n;
      sn += n;
      sm += p->toff[k + 1] - p->toff[k];
      if (n > nmax) nmax = n;
    }
    free(w.A); free(w.Q); free(w.B); free(w.X);
  }
  if (err) { if (!local_out) free(local); free(done); set_err("solve: out of memory"); return -4; }

  /* Partition of unity (solver.hpp:275-285), ascending patch order per target. */
#pragma omp parallel
  {
    int64_t *ids = (int64_t *)malloc(sizeof(int64_t) * ORC_WCAP);
    double *ws = (double *)malloc(sizeof(double) * ORC_WCAP);
#pragma omp for schedule(static)
    for (int64_t t = 0; t < p->m; ++t) {
      double sum;
      const double *y = p->tgt + 3 * t;
      const int64_t c = target_weights(p, y, ids, ws, ORC_WCAP, &sum);
      double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
      for (int64_t i = 0; i < c && i < ORC_WCAP; ++i) {
        const int64_t k = ids[i];
        if (!done[k]) continue;
        const int32_t *tl = p->tidx + p->toff[k];
        const int64_t mk = p->toff[k + 1] - p->toff[k];
        const int64_t pos = lower_bound_i32(tl, mk, (int32_t)t);
        if (pos >= mk || tl[pos] != (int32_t)t) continue;
        const double wn = ws[i] / sum;
        for (int f = 0; f < F; ++f) acc[f] += wn * local[(p->toff[k] + pos) * F + f];
      }
      for (int f = 0; f < F; ++f) out[t * F + f] = acc[f];
    }
    free(ids);
    free(ws);
  }
  if (stats) {
    stats[0] = ndrop; stats[1] = s3; stats[2] = nmax; stats[3] = sn; stats[4] = sm;
    stats[5] = stats[6] = stats[7] = 0;
  }
  if (!local_out) free(local);
  free(done);
  return 0;
}

/* ------------------------------------------------------------------------
 * Finite-element transfer NEAREST_NEAREST (src/finite_elements/FTNearest.hpp:27-56):
 * every target takes the value of its nearest source (ArborX nearest(1) on a
 * BVH of the sources, src/finite_elements/utils/ArborXCallbacks.hpp:172-182).
 * Brute force here, squared distances as the kernels form them (t = b - a,
 * acc = t_x^2, then fma per further axis), ties toward the lowest source index
 * (ArborX's tie order is not reproducible; this is the documented convention).
 * Targets with no source keep 0 (SetupTransferClass zero-fills,
 * common/transfer.hxx:100-110); the status stays OUTSIDE (0), which FTNearest
 * never changes.
 * ---------------------------------------------------------------------- */
int orc_fe_nearest(int dim, const double *src, int64_t n, const double *vals,
                   const double *tgt, int64_t m, double *out, int32_t *nearest) {
  if (dim < 1 || dim > 3) {
    set_err("dimension must be 1, 2 or 3");
    return -2;
  }
#pragma omp parallel for schedule(dynamic, 256)
  for (int64_t t = 0; t < m; ++t) {
    double y[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < dim; ++d) y[d] = tgt[t * dim + d];
    double best = 0.0;
    int64_t bi = -1;
    for (int64_t i = 0; i < n; ++i) {
      double x[3] = {0.0, 0.0, 0.0};
      for (int d = 0; d < dim; ++d) x[d] = src[i * dim + d];
      const double tx = x[0] - y[0], ty = x[1] - y[1], tz = x[2] - y[2];
      double acc = tx * tx;
      acc = fma(ty, ty, acc);
      acc = fma(tz, tz, acc);
      if (bi < 0 || acc < best) {
        best = acc;
        bi = i;
      }
    }
    out[t] = bi >= 0 ? vals[bi] : 0.0;
    if (nearest) nearest[t] = (int32_t)bi;
  }
  return 0;
}

/* ------------------------------------------------------------------------
 * Moving least squares (src/mls/interpolator.hpp:49-77, src/mls_interface.cpp):
 * the reference constructs ArborX 2.1's Interpolation::MovingLeastSquares
 * (un-vendored dependency) with its defaults and interpolates one scalar
 * field.  Restated from that published algorithm:
 *  - neighbours: the K nearest sources of each target, K = the size of the
 *    quadratic polynomial basis (3, 6, 10 in 1D, 2D, 3D); fewer when there
 *    are fewer sources.  Order and ties: ascending (squared distance, source
 *    index), squared distances formed as sqdist() above;
 *  - radius: 1.1 x the largest neighbour distance (at least 10 x DBL_EPSILON),
 *    so that the farthest neighbour keeps a non-zero weight;
 *  - weights: Wendland C0 of rho = distance / radius, (1 - rho)^2;
 *  - basis: the monomials of degree <= 2 of x = (source - target) / radius
 *    (1D: 1, x, x^2; 2D: 1, x, y, x^2, xy, y^2; 3D: 1, x, y, z, x^2, xy, xz,
 *    y^2, yz, z^2), so that the value at the target is the constant
 *    coefficient.  ArborX uses source - target unscaled; the division by the
 *    radius changes no value where A is invertible (exact arithmetic) and
 *    takes the radius^4 spread out of A's eigenvalues, so the eigenvalue
 *    cut-off below is relative to a well-scaled matrix;
 *  - moment matrix A = sum_j w_j p_j p_j^T and b = sum_j w_j f_j p_j; the
 *    value is e_0^T A^+ b with A^+ the Moore-Penrose pseudo-inverse of the
 *    symmetric A.
 * A^+ comes from a cyclic Jacobi eigen-decomposition A = V L V^T (Rutishauser's
 * rotation formulas) whose rotations are applied to u = V^T e_0 and
 * v = V^T b; eigenvalues |l_k| <= 1e-13 max |l| count as zero, and the value
 * is sum_k u_k v_k / l_k over the others.  ArborX's eigenvalue cut-off and
 * tie order are not reproducible here (parity with ArborX is unpinned; the
 * reference's own MLS tests are the pins).  In exact arithmetic the value
 * equals ArborX's whenever A is invertible, and whenever A's null space is
 * orthogonal to e_0 (sources on a line or plane through the target); with
 * fewer sources than basis functions, or a degenerate neighbour set that
 * misses the target, the two pseudo-inverse fits differ by the basis scaling.  Targets keep 0 without sources
 * (SetupTransferClass zero-fills, common/transfer.hxx:100-110).
 * No fused multiply-add outside sqdist(): every product and sum below is
 * rounded on its own, and the CUDA kernel is compiled the same way.
 * ---------------------------------------------------------------------- */
#define MLS_KMAX 10
#define MLS_SWEEPS 64

int orc_mls_basis_size(int dim) { return dim == 1 ? 3 : (dim == 2 ? 6 : 10); }

static void mls_basis(int dim, const double *x, double *p) {
  p[0] = 1.0;
  if (dim == 1) {
    p[1] = x[0];
    p[2] = x[0] * x[0];
  } else if (dim == 2) {
    p[1] = x[0]; p[2] = x[1];
    p[3] = x[0] * x[0]; p[4] = x[0] * x[1]; p[5] = x[1] * x[1];
  } else {
    p[1] = x[0]; p[2] = x[1]; p[3] = x[2];
    p[4] = x[0] * x[0]; p[5] = x[0] * x[1]; p[6] = x[0] * x[2];
    p[7] = x[1] * x[1]; p[8] = x[1] * x[2]; p[9] = x[2] * x[2];
  }
}

/* One Jacobi rotation annihilating a[p][q] (p < q) of the symmetric M x M
 * matrix a (both triangles kept), applied to the vectors u and v as well. */
static void mls_rotate(int M, double a[MLS_KMAX][MLS_KMAX], double *u, double *v, int p, int q) {
  const double apq = a[p][q];
  if (apq == 0.0) return;
  const double app = a[p][p], aqq = a[q][q];
  const double g = 100.0 * fabs(apq);
  if (fabs(app) + g == fabs(app) && fabs(aqq) + g == fabs(aqq)) {
    a[p][q] = a[q][p] = 0.0;  /* below the rounding of both diagonal entries */
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
  a[p][p] = app - t * apq;
  a[q][q] = aqq + t * apq;
  a[p][q] = a[q][p] = 0.0;
  for (int r = 0; r < M; ++r) {
    if (r == p || r == q) continue;
    const double arp = a[r][p], arq = a[r][q];
    const double np_ = arp - s * (arq + tau * arp);
    const double nq_ = arq + s * (arp - tau * arq);
    a[r][p] = a[p][r] = np_;
    a[r][q] = a[q][r] = nq_;
  }
  const double up = u[p], uq = u[q];
  u[p] = up - s * (uq + tau * up);
  u[q] = uq + s * (up - tau * uq);
  const double vp = v[p], vq = v[q];
  v[p] = vp - s * (vq + tau * vp);
  v[q] = vq + s * (vp - tau * vq);
}

/* e_0^T A^+ b for the symmetric M x M moment matrix a (destroyed). */
static double mls_pinv_value(int M, double a[MLS_KMAX][MLS_KMAX], const double *b, int *sweeps) {
  double u[MLS_KMAX], v[MLS_KMAX];
  for (int i = 0; i < M; ++i) {
    u[i] = i == 0 ? 1.0 : 0.0;
    v[i] = b[i];
  }
  int sw = 0;
  for (; sw < MLS_SWEEPS; ++sw) {
    int off = 0;
    for (int p = 0; p < M; ++p)
      for (int q = p + 1; q < M; ++q) off |= a[p][q] != 0.0;
    if (!off) break;
    for (int p = 0; p < M; ++p)
      for (int q = p + 1; q < M; ++q) mls_rotate(M, a, u, v, p, q);
  }
  if (sweeps) *sweeps = sw;
  double lmax = 0.0;
  for (int k = 0; k < M; ++k) lmax = fmax(lmax, fabs(a[k][k]));
  const double cut = 1e-13 * lmax;
  double val = 0.0;
  for (int k = 0; k < M; ++k)
    if (fabs(a[k][k]) > cut) val = val + (u[k] * v[k]) / a[k][k];
  return val;
}

static inline double mls_sqdist(int dim, const double *src, int64_t i, const double *y) {
  double x[3] = {0.0, 0.0, 0.0};
  for (int d = 0; d < dim; ++d) x[d] = src[i * dim + d];
  const double tx = x[0] - y[0], ty = x[1] - y[1], tz = x[2] - y[2];
  double acc = tx * tx;
  acc = fma(ty, ty, acc);
  acc = fma(tz, tz, acc);
  return acc;
}

/* Keeps the kk smallest (squared distance, index) pairs, sorted. */
static inline void mls_keep(double acc, int64_t i, int kk, double *bd, int64_t *bi, int *cnt) {
  if (*cnt == kk && !(acc < bd[kk - 1] || (acc == bd[kk - 1] && i < bi[kk - 1]))) return;
  int pos = *cnt < kk ? (*cnt)++ : kk - 1;
  while (pos > 0 && (acc < bd[pos - 1] || (acc == bd[pos - 1] && i < bi[pos - 1]))) {
    bd[pos] = bd[pos - 1];
    bi[pos] = bi[pos - 1];
    --pos;
  }
  bd[pos] = acc;
  bi[pos] = i;
}

/* Source cell grid of the neighbour search: about two sources per cell over
 * the sources' bounding box. */
typedef struct {
  int dim;
  double lo[3], inv_h, h;
  int64_t nc[3];
  int64_t *start;
  int64_t *items;
} mls_grid_t;

static int64_t mls_cell(const mls_grid_t *g, int d, double x) {
  const double f = floor((x - g->lo[d]) * g->inv_h);
  if (!(f >= 0.0)) return 0;
  if (f > (double)(g->nc[d] - 1)) return g->nc[d] - 1;
  return (int64_t)f;
}

static int mls_grid_build(mls_grid_t *g, int dim, const double *src, int64_t n) {
  memset(g, 0, sizeof(*g));
  g->dim = dim;
  double lo[3] = {0.0, 0.0, 0.0}, hi[3] = {0.0, 0.0, 0.0}, ext = 0.0;
  for (int d = 0; d < dim; ++d) {
    lo[d] = INFINITY;
    hi[d] = -INFINITY;
    for (int64_t i = 0; i < n; ++i) {
      lo[d] = fmin(lo[d], src[i * dim + d]);
      hi[d] = fmax(hi[d], src[i * dim + d]);
    }
    ext = fmax(ext, hi[d] - lo[d]);
  }
  const double per_axis = ceil(pow(fmax((double)n / 2.0, 1.0), 1.0 / dim));
  g->h = ext > 0.0 ? ext / per_axis : 1.0;
  g->inv_h = 1.0 / g->h;
  int64_t cells = 1;
  for (int d = 0; d < 3; ++d) {
    g->lo[d] = lo[d];
    g->nc[d] = d < dim ? (int64_t)floor((hi[d] - lo[d]) * g->inv_h) + 1 : 1;
    if (g->nc[d] < 1 || g->nc[d] > (1 << 21)) {
      set_err("mls: could not size the neighbour grid");
      return -3;
    }
    cells *= g->nc[d];
  }
  g->start = (int64_t *)calloc((size_t)cells + 1, sizeof(int64_t));
  g->items = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t *cell = (int64_t *)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  if (!g->start || !g->items || !cell) {
    free(cell);
    set_err("mls: out of memory");
    return -4;
  }
  for (int64_t i = 0; i < n; ++i) {
    int64_t c = 0;
    for (int d = 0; d < 3; ++d)
      c = c * g->nc[d] + (d < dim ? mls_cell(g, d, src[i * dim + d]) : 0);
    cell[i] = c;
    g->start[c + 1]++;
  }
  for (int64_t c = 0; c < cells; ++c) g->start[c + 1] += g->start[c];
  for (int64_t i = 0; i < n; ++i) g->items[g->start[cell[i]]++] = i;
  for (int64_t c = cells; c > 0; --c) g->start[c] = g->start[c - 1];
  g->start[0] = 0;
  free(cell);
  return 0;
}

/* The kk nearest sources of y: shells of cells at Chebyshev cell distance
 * R = 0, 1, ... around y's (clamped) cell.  After shell R every unscanned
 * source lies at least R cell widths away (one less for rounding at cell
 * borders), so the scan stops once the kk-th best squared distance is below
 * ((R - 1) h)^2. */
static void mls_knn_grid(const mls_grid_t *g, const double *src, const double *y, int kk,
                         double *bd, int64_t *bi) {
  int cnt = 0;
  int64_t c[3], rmax = 0;
  for (int d = 0; d < 3; ++d) {
    c[d] = d < g->dim ? mls_cell(g, d, y[d]) : 0;
    if (g->nc[d] > rmax) rmax = g->nc[d];
  }
  for (int64_t R = 0; R <= rmax; ++R) {
    for (int64_t a = c[0] - R; a <= c[0] + R; ++a) {
      if (a < 0 || a >= g->nc[0]) continue;
      for (int64_t b = c[1] - R; b <= c[1] + R; ++b) {
        if (b < 0 || b >= g->nc[1]) continue;
        for (int64_t e = c[2] - R; e <= c[2] + R; ++e) {
          if (e < 0 || e >= g->nc[2]) continue;
          const int64_t da = llabs(a - c[0]), db = llabs(b - c[1]), de = llabs(e - c[2]);
          if (da != R && db != R && de != R) continue;  /* inside: scanned before */
          const int64_t cid = (a * g->nc[1] + b) * g->nc[2] + e;
          for (int64_t s = g->start[cid]; s < g->start[cid + 1]; ++s) {
            const int64_t i = g->items[s];
            mls_keep(mls_sqdist(g->dim, src, i, y), i, kk, bd, bi, &cnt);
          }
        }
      }
    }
    if (cnt == kk && R >= 1) {
      const double lim = (double)(R - 1) * g->h;
      if (bd[kk - 1] < lim * lim) break;
    }
  }
}

int orc_mls_interpolate(int dim, const double *src, int64_t n, const double *vals,
                        const double *tgt, int64_t m, double *out, int32_t *sweeps_out,
                        int knn_mode) {
  if (dim < 1 || dim > 3) {
    set_err("dimension must be 1, 2 or 3");
    return -2;
  }
  const int K = orc_mls_basis_size(dim);
  const int kk = n < K ? (int)n : K;
  /* knn_mode: 1 brute force, 2 cell grid, 0 the grid from 4,096 sources on. */
  const int use_grid = knn_mode == 2 || (knn_mode == 0 && n >= 4096);
  mls_grid_t grid;
  memset(&grid, 0, sizeof(grid));
  if (use_grid && n > 0) {
    const int rc = mls_grid_build(&grid, dim, src, n);
    if (rc) {
      free(grid.start);
      free(grid.items);
      return rc;
    }
  }
#pragma omp parallel for schedule(dynamic, 64)
  for (int64_t t = 0; t < m; ++t) {
    double y[3] = {0.0, 0.0, 0.0};
    for (int d = 0; d < dim; ++d) y[d] = tgt[t * dim + d];
    double bd[MLS_KMAX];
    int64_t bi[MLS_KMAX];
    if (use_grid && n > 0) {
      mls_knn_grid(&grid, src, y, kk, bd, bi);
    } else {
      int cnt = 0;
      for (int64_t i = 0; i < n; ++i) mls_keep(mls_sqdist(dim, src, i, y), i, kk, bd, bi, &cnt);
    }
    if (kk == 0) {
      out[t] = 0.0;
      if (sweeps_out) sweeps_out[t] = 0;
      continue;
    }
    double dist[MLS_KMAX];
    double rmax = 10.0 * DBL_EPSILON;
    for (int j = 0; j < kk; ++j) {
      dist[j] = sqrt(bd[j]);
      rmax = fmax(rmax, dist[j]);
    }
    const double radius = 1.1 * rmax;
    double a[MLS_KMAX][MLS_KMAX], b[MLS_KMAX];
    for (int i = 0; i < K; ++i) {
      b[i] = 0.0;
      for (int k = 0; k < K; ++k) a[i][k] = 0.0;
    }
    for (int j = 0; j < kk; ++j) {
      double x[3] = {0.0, 0.0, 0.0}, p[MLS_KMAX];
      for (int d = 0; d < dim; ++d) x[d] = (src[bi[j] * dim + d] - y[d]) / radius;
      mls_basis(dim, x, p);
      const double rho = dist[j] / radius;
      const double w = (1.0 - rho) * (1.0 - rho);
      const double wf = w * vals[bi[j]];
      for (int r = 0; r < K; ++r) {
        const double wr = w * p[r];
        for (int c = r; c < K; ++c) a[r][c] = a[r][c] + wr * p[c];
        b[r] = b[r] + wf * p[r];
      }
    }
    for (int r = 0; r < K; ++r)
      for (int c = 0; c < r; ++c) a[r][c] = a[c][r];
    int sw = 0;
    out[t] = mls_pinv_value(K, a, b, &sw);
    if (sweeps_out) sweeps_out[t] = sw;
  }
  free(grid.start);
  free(grid.items);
  return 0;
}
