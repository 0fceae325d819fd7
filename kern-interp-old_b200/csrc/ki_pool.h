// A small persistent host thread pool for the per-box bookkeeping of a
// level (near lists, ID row lists, update-block maps).  Work is split into
// chunks of `grain` indices claimed through an atomic counter; the calling
// thread works too, and the call returns when every chunk is done.  Jobs
// below `serial_below` indices run on the caller alone (thread hand-off
// costs more than small levels take), and so does a parallel_for issued
// from inside another one.
#ifndef KI_POOL_H_
#define KI_POOL_H_

#include <functional>

namespace kib {

// fn(begin, end) over [0, n) in chunks of `grain`.
void parallel_for(int n, int grain, const std::function<void(int, int)>& fn,
                  int serial_below = 64);
int pool_threads();

}  // namespace kib

#endif  // KI_POOL_H_
