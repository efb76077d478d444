// Test-infrastructure stand-in: math_utils.h includes this Boost.Math header for erf_inv
// (math_utils.cpp:15), which the genotype-likelihood path never calls; calling it aborts.
#pragma once

#include <cstdio>
#include <cstdlib>

namespace boost {
namespace math {

template <class T>
T erf_inv(T)
{
    std::fprintf(stderr, "oracle/_ref: boost::math::erf_inv reached; it is not on the genotyping path\n");
    std::abort();
}

}  // namespace math
}  // namespace boost
