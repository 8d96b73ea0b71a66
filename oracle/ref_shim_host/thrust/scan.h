// Stand-in for thrust::inclusive_scan, sequential on the host (see execution_policy.h).
#pragma once
#include "execution_policy.h"
namespace thrust {
template <class Policy, class It>
It inclusive_scan(Policy, It first, It last, It out) {
  if (first == last) return out;
  auto acc = *first;
  *out++ = acc;
  for (++first; first != last; ++first) {
    acc = acc + *first;
    *out++ = acc;
  }
  return out;
}
}  // namespace thrust
