// PACMAN::rbf_interpolate on the B200 engine (include/pacman_rbf.hpp).
//
// Mirrors src/rbf_interface.cpp:101-130 of the reference: the same null
// checks and exception types, then the transfer with the reference's
// default parameters (50 nodes per cluster, 0.15 overlap, 0.1 support) in the
// reference's FP64 algorithm, returned as an owned std::vector.
#include "../../include/pacman_rbf.hpp"

#include <stdexcept>
#include <string>

#include "../../include/pacman_b200.h"

namespace PACMAN {

RbfInterpolateResult rbf_interpolate(int_t spaceDimension, unsigned char execSpace,
                                     unsigned char rbfFunction, coordinates_t *sourcePoints,
                                     int_t nSourcePoints, fp_t *sourceValues,
                                     coordinates_t *targetPoints, int_t nTargetPoints) {
  if (sourcePoints == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourcePoints is null but nSourcePoints > 0");
  if (targetPoints == nullptr && nTargetPoints > 0)
    throw std::invalid_argument("targetPoints is null but nTargetPoints > 0");
  if (sourceValues == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourceValues is null but nSourcePoints > 0");
  if (spaceDimension < 1 || spaceDimension > 3)
    throw std::runtime_error("The dimension of the points can only be: 1, 2 or 3.\n");
  if (execSpace > ExecSpaces::SYCL)
    throw std::invalid_argument("execspace: Serial, OpenMP, Threads, Cuda, HIP, SYCL");
  if (rbfFunction < RbfFunctions::WENDLANDC0 || rbfFunction > RbfFunctions::WENDLANDC8)
    throw std::invalid_argument("Unsupported RBF function selector: " +
                                std::to_string(rbfFunction));
  RbfInterpolateResult result;
  result.targetValues.assign(nTargetPoints > 0 ? size_t(nTargetPoints) : 0, 0.0);
  if (nTargetPoints <= 0) return result;
  pacman_b200_options opts;
  pacman_b200_options_init(&opts);
  const int rc = pacman_b200_rbf_interpolate(
      spaceDimension, rbfFunction, sourcePoints, nSourcePoints > 0 ? nSourcePoints : 0,
      sourceValues, 1, targetPoints, nTargetPoints, result.targetValues.data(), &opts, nullptr);
  if (rc == PACMAN_B200_ERR_INVALID) throw std::invalid_argument(pacman_b200_last_error());
  if (rc != 0) throw std::runtime_error(pacman_b200_last_error());
  return result;
}

// PACMAN::fe_interpolate (src/interface.cpp:89-121) for NEAREST_NEAREST.
FeInterpolateResult fe_interpolate(int_t spaceDimension, unsigned char execSpace,
                                   method_t method, coordinates_t *sourcePoints,
                                   int_t nSourcePoints, fp_t *sourceValues, int_t *connVal,
                                   int_t connValSize, offset_t *connOff, int_t connOffSize,
                                   cell_t *cellTypes, coordinates_t *targetPoints,
                                   int_t nTargetPoints, bool fortranIndexing) {
  (void)connVal;
  (void)connValSize;
  (void)connOff;
  (void)connOffSize;
  (void)cellTypes;
  (void)fortranIndexing;
  if (sourcePoints == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourcePoints is null but nSourcePoints > 0");
  if (targetPoints == nullptr && nTargetPoints > 0)
    throw std::invalid_argument("targetPoints is null but nTargetPoints > 0");
  if (sourceValues == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourceValues is null but nSourcePoints > 0");
  if (spaceDimension < 1 || spaceDimension > 3)
    throw std::runtime_error("The dimension of the points can only be: 1, 2 or 3.\n");
  if (execSpace > ExecSpaces::SYCL)
    throw std::invalid_argument("execspace: Serial, OpenMP, Threads, Cuda, HIP, SYCL");
  FeInterpolateResult result;
  const size_t m = nTargetPoints > 0 ? size_t(nTargetPoints) : 0;
  result.targetValues.assign(m, 0.0);
  result.targetStatus.assign(m, 0);
  const int rc = pacman_b200_fe_interpolate(
      spaceDimension, method, sourcePoints, nSourcePoints > 0 ? nSourcePoints : 0, sourceValues,
      targetPoints, int64_t(m), result.targetValues.data(), result.targetStatus.data(), nullptr);
  if (rc == PACMAN_B200_ERR_INVALID) throw std::invalid_argument(pacman_b200_last_error());
  if (rc != 0) throw std::runtime_error(pacman_b200_last_error());
  return result;
}

// PACMAN::MLS_interpolate (src/mls_interface.cpp): the reference's null and
// dimension checks, then the moving least squares transfer.
MLSInterpolateResult MLS_interpolate(int_t spaceDimension, unsigned char execSpace,
                                     coordinates_t *sourcePoints, int_t nSourcePoints,
                                     fp_t *sourceValues, coordinates_t *targetPoints,
                                     int_t nTargetPoints) {
  if (sourcePoints == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourcePoints is null but nSourcePoints > 0");
  if (targetPoints == nullptr && nTargetPoints > 0)
    throw std::invalid_argument("targetPoints is null but nTargetPoints > 0");
  if (sourceValues == nullptr && nSourcePoints > 0)
    throw std::invalid_argument("sourceValues is null but nSourcePoints > 0");
  if (spaceDimension < 1 || spaceDimension > 3)
    throw std::runtime_error("The dimension of the points can only be: 1, 2 or 3.\n");
  if (execSpace > ExecSpaces::SYCL)
    throw std::invalid_argument("execspace: Serial, OpenMP, Threads, Cuda, HIP, SYCL");
  MLSInterpolateResult result;
  const size_t m = nTargetPoints > 0 ? size_t(nTargetPoints) : 0;
  result.targetValues.assign(m, 0.0);
  if (m == 0) return result;
  const int rc = pacman_b200_mls_interpolate(
      spaceDimension, sourcePoints, nSourcePoints > 0 ? nSourcePoints : 0, sourceValues,
      targetPoints, int64_t(m), result.targetValues.data(), nullptr);
  if (rc == PACMAN_B200_ERR_INVALID) throw std::invalid_argument(pacman_b200_last_error());
  if (rc != 0) throw std::runtime_error(pacman_b200_last_error());
  return result;
}

}  // namespace PACMAN
