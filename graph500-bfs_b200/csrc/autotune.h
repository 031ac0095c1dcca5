// Alpha/beta auto-tuning (main.cc -A).
#pragma once

#include <functional>
#include <vector>
#include "engine.h"

namespace b200bfs {

// Runs one search from root with (alpha, beta), fills auto_tuning_data[9]
// and returns its time in seconds.
using SearchFn = std::function<double(int64_t root, double alpha, double beta, int64_t* at)>;

// auto_tuning (mpi/main.cc:361-391): tunes *alpha then *beta in place and
// returns the harmonic-mean TEPS of the final measurement.  tries counts the
// extra searches the tuning ran.
double auto_tune(const SearchFn& search, const std::vector<int64_t>& roots,
                 const std::vector<double>& nedge, int edgefactor, double* alpha, double* beta,
                 int* tries);

}  // namespace b200bfs
