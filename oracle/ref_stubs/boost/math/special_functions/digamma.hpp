// Test-infrastructure stand-in: math_utils.h includes this Boost.Math header, but its only use of
// boost::math::digamma (the DigammaCache, math_utils.h:182-206) is compiled out with #if 0.
#pragma once
