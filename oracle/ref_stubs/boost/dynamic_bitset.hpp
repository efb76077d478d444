// Minimal stand-in for boost::dynamic_bitset: the reference's genotype forward declarations
// name the type, and the PairHMM scheduler never uses it.
#pragma once
#include <cstddef>
#include <memory>
namespace boost {
template <typename Block = unsigned long, typename Alloc = std::allocator<Block>>
class dynamic_bitset {
public:
    dynamic_bitset() = default;
    ~dynamic_bitset() = default;
};
}  // namespace boost
