// Test-infrastructure stand-in for Boost.Math's binomial coefficient (Boost 1.83, the version the
// reference bundles: src/CMakeLists.txt:6; Boost itself is not installed here).  The reference's
// genotype code calls boost::math::binomial_coefficient<double>(n, k) only to count diploid
// genotypes (genotype_num_likelihoods_cache.hpp:40,49), with n below 60.  Boost evaluates small
// arguments from its factorial table and returns ceil(result - 0.5), the nearest integer; for these
// arguments that is the exact coefficient, which this restatement computes by the multiplicative
// formula in exact integer arithmetic.
#pragma once

#include <cstdint>

namespace boost {
namespace math {

template <class T>
T binomial_coefficient(unsigned n, unsigned k)
{
    if (k > n) return T(0);
    if (k > n - k) k = n - k;
    unsigned __int128 c = 1;
    for (unsigned i = 1; i <= k; ++i) c = c * (n - k + i) / i;  // exact at every step: C(n-k+i, i)
    return static_cast<T>(c);
}

}  // namespace math
}  // namespace boost
