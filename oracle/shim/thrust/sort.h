/*
 * Host stand-in for thrust::sort_by_key (test infrastructure only). The
 * reference calls it on host pointers (HCGrid/gridding.cu:166); a stable sort
 * of the keys carrying the values gives thrust's documented result.
 */
#ifndef HCG_SHIM_THRUST_SORT_H
#define HCG_SHIM_THRUST_SORT_H
#include <algorithm>
#include <vector>
#include <utility>
namespace thrust {
template <class K, class V>
void sort_by_key(K *kb, K *ke, V *vals) {
    size_t n = (size_t)(ke - kb);
    std::vector<std::pair<K, V>> tmp(n);
    for (size_t i = 0; i < n; ++i) tmp[i] = std::make_pair(kb[i], vals[i]);
    std::stable_sort(tmp.begin(), tmp.end(),
                     [](const std::pair<K, V> &a, const std::pair<K, V> &b) { return a.first < b.first; });
    for (size_t i = 0; i < n; ++i) { kb[i] = tmp[i].first; vals[i] = tmp[i].second; }
}
}  // namespace thrust
#endif
