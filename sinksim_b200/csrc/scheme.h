// Scheme v1 constants of the time step (engine/include/sinksim/kernel/scheme.hpp:11-28 of the reference) and the
// JavaScript Math.max / Math.min tie rule (kernel/math.hpp:29-30), for host and device code.
#pragma once

#if defined(__CUDACC__)
#define SSB_HD __host__ __device__ __forceinline__
#else
#define SSB_HD inline
#endif

namespace ssb {

constexpr double kEmptyVolume = 1e-6;
constexpr double kFullFraction = 1.0 - 1e-7;
constexpr double kLimiterShare = 0.5;
constexpr double kOrificeHeadFloor = 0.01;
constexpr double kWeirCoefficient = 2.0 / 3.0;
constexpr double kWeirExponent = 1.5;
constexpr double kVillemonteExponent = 0.385;
constexpr int kNewtonFast = 6;
constexpr double kSlopeMin = 1e-9;
constexpr double kCentroidMinVolume = 1e-9;
constexpr double kNoHead = -1e9;
constexpr double kNoHeadTest = -1e8;
constexpr double kPitchClamp = 1.35;
constexpr double kRollClamp = 1.4;
constexpr double kPi = 3.141592653589793;

// JavaScript Math.max / Math.min: the first argument wins ties.
SSB_HD double jmax(double a, double b) { return (b > a) ? b : a; }
SSB_HD double jmin(double a, double b) { return (b < a) ? b : a; }

}  // namespace ssb
