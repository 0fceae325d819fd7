// Stand-in for boost::hash, used by the reference only to key an
// unordered_map on (x, y) point pairs (test infrastructure only).
#ifndef ORACLE_SHIM_BOOST_HASH_HPP_
#define ORACLE_SHIM_BOOST_HASH_HPP_
#include <cstddef>
#include <functional>
#include <utility>
namespace boost {
template <class T>
struct hash {
  std::size_t operator()(const T& v) const { return std::hash<T>()(v); }
};
template <class A, class B>
struct hash<std::pair<A, B>> {
  std::size_t operator()(const std::pair<A, B>& p) const {
    std::size_t h = std::hash<A>()(p.first);
    std::size_t g = std::hash<B>()(p.second);
    return h ^ (g + 0x9e3779b97f4a7c15ULL + (h << 6) + (h >> 2));
  }
};
}  // namespace boost
#endif
