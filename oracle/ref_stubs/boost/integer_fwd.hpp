// Empty stand-in: the reference's AVX-512 traits header includes this Boost header but uses
// nothing from it, and Boost is not installed in this image.
#pragma once
