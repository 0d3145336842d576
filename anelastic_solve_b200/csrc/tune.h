// tune.h -- the library's autotuner registry.
//
// Kernels with several launch shapes (rows per thread, lines per warp,
// occupancy) are timed once per device and problem shape with CUDA events
// on the caller's data layout, and the fastest variant is kept for the
// process: contexts of the same shape (serving buckets) reuse the choice.
// ANEL_TUNE=0 in the environment turns timing off (every kernel keeps its
// default variant); ANEL_TUNE_CACHE=<file> keeps the choices in a file
// that later processes read instead of timing again.
#pragma once

#include <string>
#include <vector>

namespace anel {

bool tune_enabled();
// the cached choice for `key` (kernel name and shape, device included), or -1
int tune_lookup(const std::string& key);
void tune_store(const std::string& key, int chosen, const std::vector<double>& ms);
// "key: variant v (t0 t1 ... ms per launch)" lines of every tuned entry
std::string tune_report();

}  // namespace anel
