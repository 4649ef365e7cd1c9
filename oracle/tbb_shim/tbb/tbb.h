/* Stand-in for the one Intel TBB facility the reference solver uses,
 * tbb::parallel_for(first, last, step, body), mapped onto OpenMP.
 * TBB carries no arithmetic of its own here: every iteration body the
 * reference passes writes disjoint elements, so the schedule cannot change
 * any result.  Used only to compile the reference into oracle/_ref. */
#ifndef VFLIP_TBB_SHIM_H
#define VFLIP_TBB_SHIM_H
#include <unordered_map>
#include <tr1/unordered_map>

namespace tbb {
template <class Index, class Body>
void parallel_for(Index first, Index last, Index step, const Body& body) {
#pragma omp parallel for schedule(static)
  for (long long i = (long long)first; i < (long long)last; i += (long long)step)
    body((Index)i);
}
}  // namespace tbb
#endif
