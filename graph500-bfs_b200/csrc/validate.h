// Graph500 result validation on the device.
#pragma once

#include "bfs_internal.h"

namespace b200bfs {

// BfsValidation::validate (mpi/validate.hpp:607-976) of the last search
// against the graph's resident input edges.
void validate_device(DeviceArena& arena, cudaStream_t s, int sms, const Graph& g,
                     const BfsState& st, int64_t root, int64_t* errors, int64_t* edge_visit_count);

}  // namespace b200bfs
