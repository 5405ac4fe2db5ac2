// Stand-in for boost::sort::block_indirect_sort in the oracle harness.  The reference only sorts
// float score rows with it; any correct sort yields the same sequence of values.
#pragma once
#include <algorithm>
namespace boost { namespace sort {
template <typename It, typename Cmp>
inline void block_indirect_sort(It first, It last, Cmp cmp, unsigned = 0) { std::sort(first, last, cmp); }
}}  // namespace boost::sort
