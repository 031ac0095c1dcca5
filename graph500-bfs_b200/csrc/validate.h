// Graph500 result validation on the device.
#pragma once

#include "bfs_internal.h"

namespace b200bfs {

// BfsValidation::validate (mpi/validate.hpp:607-976) of a pred array
// (pred_size entries, in device or host memory: `pred` is read with
// cudaMemcpyDefault into a scratch copy, never modified) against the graph's
// resident input edges.  corebfs selects the reference's CoreBFS mode: tree
// entries carry level 0xFFFF and the depth map is rebuilt from parents.
void validate_device(DeviceArena& arena, cudaStream_t s, int sms, const Graph& g,
                     const int64_t* pred, bool corebfs, int64_t root, int64_t* errors,
                     int64_t* edge_visit_count);

}  // namespace b200bfs
