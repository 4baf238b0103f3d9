// C++ drop-in for PACMAN's RBF-PUM entry point, running on the B200 engine.
//
// Same names, types and error behaviour as the reference's
// src/interface.hpp:106-136 (PACMAN::rbf_interpolate) and
// src/common/types.hpp:15-21 (scalar typedefs).  Link against
// libpacman_b200.so; no Kokkos initialisation is required.
#pragma once

#include <cstdint>
#include <vector>

namespace PACMAN {

typedef double fp_t;           // src/common/types.hpp:15
typedef double coordinates_t;  // src/common/types.hpp:16
typedef int32_t int_t;         // src/common/types.hpp:18

// Execution-space selector bytes (src/common/execspaces.hpp:17-24).  Every
// selector runs on the B200 engine; there is no CPU fallback.
struct ExecSpaces {
  static constexpr unsigned char SERIAL = 0x00;
  static constexpr unsigned char OPENMP = 0x01;
  static constexpr unsigned char THREADS = 0x02;
  static constexpr unsigned char CUDA = 0x03;
  static constexpr unsigned char HIP = 0x04;
  static constexpr unsigned char SYCL = 0x05;
};

// Basis selector bytes (src/interface.hpp:25-31).
struct RbfFunctions {
  static constexpr unsigned char WENDLANDC0 = 0x10;
  static constexpr unsigned char WENDLANDC2 = 0x11;
  static constexpr unsigned char WENDLANDC4 = 0x12;
  static constexpr unsigned char WENDLANDC6 = 0x13;
  static constexpr unsigned char WENDLANDC8 = 0x14;
};

// src/interface.hpp:107-110.
struct RbfInterpolateResult {
  std::vector<fp_t> targetValues;  ///< Interpolated value per target point.
};

/// RBF-PUM interpolation of one field (src/interface.hpp:132-136).
/// Points are row-major [n x spaceDimension].  Inputs are not modified.
/// @throws std::invalid_argument on null pointers with non-zero counts, an
///         unknown basis or an unknown execution-space selector.
/// @throws std::runtime_error if spaceDimension is not 1, 2 or 3, or on a
///         device error.
__attribute__((visibility("default"))) RbfInterpolateResult rbf_interpolate(int_t spaceDimension, unsigned char execSpace,
                                     unsigned char rbfFunction, coordinates_t *sourcePoints,
                                     int_t nSourcePoints, fp_t *sourceValues,
                                     coordinates_t *targetPoints, int_t nTargetPoints);

typedef int32_t offset_t;  // src/common/types.hpp:21
typedef int32_t method_t;  // src/common/types.hpp:24
typedef int32_t cell_t;    // src/common/types.hpp:25

// Finite-element method selectors (src/common/types.hpp:29-37).  The B200
// engine runs NEAREST_NEAREST; the others throw std::invalid_argument.
enum class TransferMethods : method_t {
  NEAREST_NEAREST = 0xF0,
  INTERP_CLAMP = 0xF1,
  INTERP_NEAREST = 0xF2,
  INTERP_ZEROFILL = 0xF3,
  INTERP_EXTRAP = 0xF4,
  RBF_PUM = 0xF5,
  MLS = 0xF6,
};

// src/interface.hpp:33-40.
struct FeInterpolateResult {
  std::vector<fp_t> targetValues;   ///< Value per target point.
  std::vector<int_t> targetStatus;  ///< TransferStatus per target (0 = OUTSIDE).
};

/// Finite-element interpolation (src/interface.hpp:76-80) for
/// NEAREST_NEAREST: every target takes its nearest source's value (lowest
/// index on ties); the point-based method ignores connectivity and cell types,
/// and the status stays OUTSIDE as in the reference.
/// @throws std::invalid_argument on null pointers with non-zero counts or a
///         method other than NEAREST_NEAREST.
/// @throws std::runtime_error if spaceDimension is not 1, 2 or 3, or on a
///         device error.
__attribute__((visibility("default"))) FeInterpolateResult fe_interpolate(
    int_t spaceDimension, unsigned char execSpace, method_t method, coordinates_t *sourcePoints,
    int_t nSourcePoints, fp_t *sourceValues, int_t *connVal, int_t connValSize,
    offset_t *connOff, int_t connOffSize, cell_t *cellTypes, coordinates_t *targetPoints,
    int_t nTargetPoints, bool fortranIndexing = false);

// src/interface.hpp:143-146.
struct MLSInterpolateResult {
  std::vector<fp_t> targetValues;  ///< Interpolated scalar value per target point.
};

/// Moving least squares interpolation (src/interface.hpp:166-170): the
/// K = 3, 6, 10 (1D, 2D, 3D) nearest sources of each target, Wendland C0
/// weights, a weighted quadratic least-squares fit evaluated at the target
/// (ArborX's MovingLeastSquares defaults, which the reference calls).
/// @throws std::invalid_argument on null pointers with non-zero counts.
/// @throws std::runtime_error if spaceDimension is not 1, 2 or 3, or on a
///         device error.
__attribute__((visibility("default"))) MLSInterpolateResult MLS_interpolate(
    int_t spaceDimension, unsigned char execSpace, coordinates_t *sourcePoints,
    int_t nSourcePoints, fp_t *sourceValues, coordinates_t *targetPoints,
    int_t nTargetPoints);

}  // namespace PACMAN
