/*
 * sc_algorithm.h -- drop-in for the reference header (include/sc_algorithm.h):
 * the two selection helpers its callers use on search results.
 */
#ifndef SCG_DROPIN_SC_ALGORITHM_H_
#define SCG_DROPIN_SC_ALGORITHM_H_

#include <algorithm>
#include <cstddef>
#include <utility>
#include <vector>

namespace SC {

namespace detail {
inline void apply_pairs(float *st, int *id, const std::vector<std::pair<float, int>> &v) {
    for (size_t i = 0; i < v.size(); i++) {
        st[i] = v[i].first;
        id[i] = v[i].second;
    }
}
}  // namespace detail

/* sort_id (sc_algorithm.h:24-46): sorts [st, ed) ascending, carrying ids.
 * Equal values keep their original relative order. */
inline void sort_id(float *st, float *ed, int *id) {
    std::vector<std::pair<float, int>> v;
    for (float *p = st; p != ed; p++) v.emplace_back(*p, id[p - st]);
    std::stable_sort(v.begin(), v.end(), [](const std::pair<float, int> &a, const std::pair<float, int> &b) {
        return a.first < b.first;
    });
    detail::apply_pairs(st, id, v);
}

/* nth_element_id (sc_algorithm.h:53-75): partitions [st, ed) so that element
 * r is in sorted position with no larger value before it, carrying ids. */
inline void nth_element_id(float *st, float *ed, int *id, int r) {
    std::vector<std::pair<float, int>> v;
    for (float *p = st; p != ed; p++) v.emplace_back(*p, id[p - st]);
    if (r >= 0 && (size_t)r < v.size())
        std::nth_element(v.begin(), v.begin() + r, v.end(),
                         [](const std::pair<float, int> &a, const std::pair<float, int> &b) { return a.first < b.first; });
    detail::apply_pairs(st, id, v);
}
}  // namespace SC

#endif
