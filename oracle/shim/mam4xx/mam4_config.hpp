// Host configuration header for compiling the mam4xx reference headers in
// the oracle build (stands in for the CMake-generated mam4_config.hpp):
// double precision, 72 levels, 40 constituents.
// TEST INFRASTRUCTURE ONLY.
#pragma once
namespace mam4 {
using Real = double;
#define MAM4XX_DOUBLE_PRECISION 1
constexpr int nlev = 72;
constexpr int pcnst = 40;
} // namespace mam4
