/*
 * The plain-C entry points that PACMAN's Fortran module binds through
 * ISO_C_BINDING (src/pacman_fortran.f90), exported by libpacman_b200.so with
 * the reference's names, argument types and return convention
 * (src/fortran_interface.h:69-151, implemented in
 * src/fortran_interface.cpp:22-121): no C++ exception crosses this boundary;
 * a std::exception becomes -1 and anything else -2, with the message written
 * to stderr prefixed by the function's name.
 *
 * The Fortran module itself is unchanged: it links against this library in
 * place of the reference's shim.
 */
#ifndef PACMAN_FORTRAN_SHIM_H
#define PACMAN_FORTRAN_SHIM_H

#ifdef __cplusplus
extern "C" {
#endif

#if defined(__GNUC__)
#define PACMAN_SHIM_API __attribute__((visibility("default")))
#else
#define PACMAN_SHIM_API
#endif

/* src/fortran_interface.h:69 and :75.  The B200 engine needs no runtime
 * initialisation (the reference starts and stops Kokkos here); both are
 * no-ops kept so the module's calls still resolve. */
PACMAN_SHIM_API void pacman_kokkos_initialize_c(void);
PACMAN_SHIM_API void pacman_kokkos_finalize_c(void);

/* src/fortran_interface.h:83: the preferred execution-space selector.  Always
 * CUDA (0x03): every selector runs on the B200 engine. */
PACMAN_SHIM_API int pacman_best_execspace_c(void);

/* src/fortran_interface.h:110-114: PACMAN::rbf_interpolate with plain C
 * types; targetValues is caller-allocated, nTargetPoints entries.
 * 0 on success, -1 on a std::exception (null pointer with a positive count,
 * dimension outside 1..3, unknown selector, engine error), -2 otherwise. */
PACMAN_SHIM_API int pacman_rbf_interpolate_c(int spaceDimension, int execSpace, int rbfFunction,
                                             const double *sourcePoints, int nSourcePoints,
                                             const double *sourceValues,
                                             const double *targetPoints, int nTargetPoints,
                                             double *targetValues);

/* src/fortran_interface.h:148-151: PACMAN::fe_interpolate with plain C types,
 * Fortran (1-based) connectivity.  The B200 engine serves the point-based
 * method NEAREST_NEAREST (0xF0), which reads no connectivity; other methods
 * return -1.  targetValues and targetStatus are caller-allocated. */
PACMAN_SHIM_API int pacman_fe_interpolate_c(int spaceDimension, int execSpace, int method,
                                            const double *sourcePoints, int nSourcePoints,
                                            const double *sourceValues, const int *connVal,
                                            int connValSize, const int *connOff, int connOffSize,
                                            const int *cellTypes, const double *targetPoints,
                                            int nTargetPoints, double *targetValues,
                                            int *targetStatus);

/* src/fortran_interface.h:175-179: PACMAN::MLS_interpolate with plain C
 * types; targetValues is caller-allocated, nTargetPoints entries.
 * 0 on success, -1 on a std::exception, -2 otherwise. */
PACMAN_SHIM_API int pacman_mls_interpolate_c(int spaceDimension, int execSpace,
                                             const double *sourcePoints, int nSourcePoints,
                                             const double *sourceValues,
                                             const double *targetPoints, int nTargetPoints,
                                             double *targetValues);

#ifdef __cplusplus
}
#endif
#endif /* PACMAN_FORTRAN_SHIM_H */
