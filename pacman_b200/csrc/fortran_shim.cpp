// The C functions the reference's Fortran module binds
// (include/pacman_fortran_shim.h), over the C++ drop-in of this library.
//
// The reference implements them in src/fortran_interface.cpp:22-121 over
// PACMAN::rbf_interpolate / PACMAN::fe_interpolate: each call converts the
// plain C arguments to the C++ API's types, copies the owned result vector
// into the caller's buffer, and turns exceptions into return codes (-1 for a
// std::exception, -2 for anything else) with the message on stderr.  Here
// the same conversions and codes wrap this library's PACMAN:: functions.
#include "../../include/pacman_fortran_shim.h"

#include <cstddef>
#include <exception>
#include <stdexcept>
#include <iostream>

#include "../../include/pacman_rbf.hpp"

extern "C" {

void pacman_kokkos_initialize_c(void) {}

void pacman_kokkos_finalize_c(void) {}

int pacman_best_execspace_c(void) { return static_cast<int>(PACMAN::ExecSpaces::CUDA); }

int pacman_rbf_interpolate_c(int spaceDimension, int execSpace, int rbfFunction,
                             const double *sourcePoints, int nSourcePoints,
                             const double *sourceValues, const double *targetPoints,
                             int nTargetPoints, double *targetValues) {
  try {
    if (targetValues == nullptr && nTargetPoints > 0)
      throw std::invalid_argument("targetValues is null but nTargetPoints > 0");
    // The C++ API takes non-const pointers and does not write through them.
    PACMAN::RbfInterpolateResult r = PACMAN::rbf_interpolate(
        static_cast<PACMAN::int_t>(spaceDimension), static_cast<unsigned char>(execSpace),
        static_cast<unsigned char>(rbfFunction),
        const_cast<PACMAN::coordinates_t *>(sourcePoints),
        static_cast<PACMAN::int_t>(nSourcePoints), const_cast<PACMAN::fp_t *>(sourceValues),
        const_cast<PACMAN::coordinates_t *>(targetPoints),
        static_cast<PACMAN::int_t>(nTargetPoints));
    for (int i = 0; i < nTargetPoints; ++i) targetValues[i] = r.targetValues[std::size_t(i)];
    return 0;
  } catch (const std::exception &e) {
    std::cerr << "pacman_rbf_interpolate_c: " << e.what() << "\n";
    return -1;
  } catch (...) {
    std::cerr << "pacman_rbf_interpolate_c: unknown exception\n";
    return -2;
  }
}

int pacman_fe_interpolate_c(int spaceDimension, int execSpace, int method,
                            const double *sourcePoints, int nSourcePoints,
                            const double *sourceValues, const int *connVal, int connValSize,
                            const int *connOff, int connOffSize, const int *cellTypes,
                            const double *targetPoints, int nTargetPoints, double *targetValues,
                            int *targetStatus) {
  try {
    if ((targetValues == nullptr || targetStatus == nullptr) && nTargetPoints > 0)
      throw std::invalid_argument("targetValues or targetStatus is null but nTargetPoints > 0");
    // Fortran indexing (the reference passes true): connectivity is 1-based.
    PACMAN::FeInterpolateResult r = PACMAN::fe_interpolate(
        static_cast<PACMAN::int_t>(spaceDimension), static_cast<unsigned char>(execSpace),
        static_cast<PACMAN::method_t>(method), const_cast<PACMAN::coordinates_t *>(sourcePoints),
        static_cast<PACMAN::int_t>(nSourcePoints), const_cast<PACMAN::fp_t *>(sourceValues),
        const_cast<PACMAN::int_t *>(connVal), static_cast<PACMAN::int_t>(connValSize),
        const_cast<PACMAN::offset_t *>(connOff), static_cast<PACMAN::int_t>(connOffSize),
        const_cast<PACMAN::cell_t *>(cellTypes), const_cast<PACMAN::coordinates_t *>(targetPoints),
        static_cast<PACMAN::int_t>(nTargetPoints), true);
    for (int i = 0; i < nTargetPoints; ++i) {
      targetValues[i] = r.targetValues[std::size_t(i)];
      targetStatus[i] = r.targetStatus[std::size_t(i)];
    }
    return 0;
  } catch (const std::exception &e) {
    std::cerr << "pacman_fe_interpolate_c: " << e.what() << "\n";
    return -1;
  } catch (...) {
    std::cerr << "pacman_fe_interpolate_c: unknown exception\n";
    return -2;
  }
}

int pacman_mls_interpolate_c(int spaceDimension, int execSpace, const double *sourcePoints,
                             int nSourcePoints, const double *sourceValues,
                             const double *targetPoints, int nTargetPoints,
                             double *targetValues) {
  try {
    if (targetValues == nullptr && nTargetPoints > 0)
      throw std::invalid_argument("targetValues is null but nTargetPoints > 0");
    PACMAN::MLSInterpolateResult r = PACMAN::MLS_interpolate(
        static_cast<PACMAN::int_t>(spaceDimension), static_cast<unsigned char>(execSpace),
        const_cast<PACMAN::coordinates_t *>(sourcePoints),
        static_cast<PACMAN::int_t>(nSourcePoints), const_cast<PACMAN::fp_t *>(sourceValues),
        const_cast<PACMAN::coordinates_t *>(targetPoints),
        static_cast<PACMAN::int_t>(nTargetPoints));
    for (int i = 0; i < nTargetPoints; ++i) targetValues[i] = r.targetValues[std::size_t(i)];
    return 0;
  } catch (const std::exception &e) {
    std::cerr << "pacman_mls_interpolate_c: " << e.what() << "\n";
    return -1;
  } catch (...) {
    std::cerr << "pacman_mls_interpolate_c: unknown exception\n";
    return -2;
  }
}

}  // extern "C"
