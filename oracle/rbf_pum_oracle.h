/*
 * CPU oracle for the RBF-PUM transfer -- TEST INFRASTRUCTURE ONLY.
 *
 * A plain C11 / FP64 restatement of PACMAN's RBF-PUM algorithm
 * (messahelramzi/pacman, src/rbf_pum/).  It exists to check the CUDA path and
 * to time a CPU baseline.  Only tests/, __graft_entry__.smoke() and bench.py's
 * CPU-baseline leg may load it; the product library never links or calls it.
 *
 * Parity pin: the reference itself cannot be built here (it needs Kokkos 5,
 * KokkosKernels 5 and ArborX 2.1, none of which is installed), so this
 * restatement is pinned against the reference's own known-answer tests:
 * tests/test_cpp_rbf_interface.cpp:165-198 (20^3 grid, same->same,
 * rel-L2 < 1e-8 for all five Wendland bases) and tests/test_rbf-pum.py:58-74
 * (Franke 3D on the 0.03/0.003 slab meshes, rel-L2 < 1.5e-2).
 */
#ifndef PACMAN_RBF_PUM_ORACLE_H
#define PACMAN_RBF_PUM_ORACLE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Basis selector bytes, identical to src/interface.hpp:25-31. */
#define ORC_WENDLAND_C0 0x10
#define ORC_WENDLAND_C2 0x11
#define ORC_WENDLAND_C4 0x12
#define ORC_WENDLAND_C6 0x13
#define ORC_WENDLAND_C8 0x14

typedef struct orc_plan orc_plan;

/* Geometry phase: FindRadius, CreateClusters and the per-patch membership
 * lists (src/rbf_pum/interpolator.hpp:58-94 up to solver.hpp:66).
 * brute_force != 0 replaces the uniform-grid search with O(n*m) scans (used by
 * the tests to check the grid search itself).  Returns 0 or a negative code. */
int orc_build(int dim, const double *src, int64_t n, const double *tgt,
              int64_t m, int nodes_per_cluster, double relative_overlap,
              int brute_force, orc_plan **plan_out);
void orc_free(orc_plan *plan);

double orc_radius(const orc_plan *plan);
int64_t orc_num_patches(const orc_plan *plan);
int64_t orc_num_candidates(const orc_plan *plan);
void orc_centers(const orc_plan *plan, double *out /* K x dim */);
int64_t orc_src_nnz(const orc_plan *plan);
int64_t orc_tgt_nnz(const orc_plan *plan);
void orc_src_csr(const orc_plan *plan, int64_t *offsets /* K+1 */,
                 int32_t *indices /* nnz */);
void orc_tgt_csr(const orc_plan *plan, int64_t *offsets, int32_t *indices);

/* Solve phase (src/rbf_pum/solver/solver.hpp:137-286) for nfields fields.
 * vals is n x nfields with leading dimension ld_vals (row-major).
 * out (m x nfields, row-major) receives the partition-of-unity result.
 * local (optional, tgt_nnz x nfields) receives each patch's local values.
 * patch_list (optional) restricts the solve to the listed patches (used to
 * time a bounded sample); out then only holds their contributions.
 * stats (optional, 8 entries): [0] patches whose polynomial basis lost an
 * axis, [1] sum n^3, [2] max n, [3] sum n, [4] sum m, [5..7] reserved.
 * dropped (optional, K entries): 1 for each solved patch whose polynomial
 * basis lost an axis, 0 for the other solved patches (others untouched). */
int orc_solve(const orc_plan *plan, int basis, double support_radius,
              const double *vals, int nfields, int64_t ld_vals, double *out,
              double *local, const int64_t *patch_list, int64_t n_patch_list,
              int64_t *stats, int32_t *dropped);

/* Per patch, 1 if the polynomial block of its solve drops an axis
 * (serial_ops.hpp:108-139; the decision depends on the sources only), else
 * 0: K entries. */
int orc_poly_dropped(const orc_plan *plan, int32_t *out);

/* Partition-of-unity weights of every target (solver.hpp:137-168):
 * per target t, the sum S_t of the un-normalised Wendland C2 weights of all
 * centres within the patch radius (ascending centre order). */
void orc_weight_sums(const orc_plan *plan, double *sums /* m */);

/* Wendland basis value phi(r) with support radius rho (rbf_functions.hpp). */
double orc_wendland(int basis, double r, double rho);

int orc_set_threads(int nthreads);
const char *orc_last_error(void);

/* Finite-element NEAREST_NEAREST transfer: out[t] = vals[nearest source]
 * (lowest index on ties), 0 without sources; nearest (may be NULL) receives
 * the source index or -1. */
int orc_fe_nearest(int dim, const double *src, int64_t n, const double *vals,
                   const double *tgt, int64_t m, double *out, int32_t *nearest);

/* Moving least squares (ArborX MovingLeastSquares defaults: quadratic basis,
 * Wendland C0 weights, K = basis-size nearest sources): out[t] = value at
 * target t, 0 without sources; sweeps (may be NULL) receives the Jacobi sweep
 * count per target.  knn_mode: 1 brute-force neighbours, 2 a cell grid, 0 the
 * grid from 4,096 sources on (same neighbours either way). */
int orc_mls_basis_size(int dim);
int orc_mls_interpolate(int dim, const double *src, int64_t n, const double *vals,
                        const double *tgt, int64_t m, double *out, int32_t *sweeps,
                        int knn_mode);

#ifdef __cplusplus
}
#endif
#endif
