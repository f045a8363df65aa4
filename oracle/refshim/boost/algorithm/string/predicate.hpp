// Stand-in for the one Boost function the reference uses (FXY.hpp:202,210):
// boost::starts_with(std::string, const char*).  Lets the reference compile
// here without Boost, as a checker under oracle/_ref; never part of the product.
#pragma once
#include <cstring>
#include <string>

namespace boost {
inline bool starts_with(const std::string& s, const char* prefix) {
    const size_t n = std::strlen(prefix);
    return s.size() >= n && s.compare(0, n, prefix) == 0;
}
}  // namespace boost
