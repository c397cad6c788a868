// Kernel-shape tuning table of the Debye backend: bucket keys, and the text
// file the autotuner's results are kept in.
#pragma once

#include <cstdint>
#include <map>
#include <string>
#include <tuple>

#include "pd_plan.h"

namespace pd {

// Bucket of a request: (precision, accumulation mode, more than one frame,
// floor(log2 n_atoms), floor(log2 nq)).
using TuneKey = std::tuple<int, int, int, int, int>;

struct TuneEntry {
    Tuning t;
    double ms = 0.0;  // measured time of one execution of the tuned request (0: set by hand)
};
using TuneTable = std::map<TuneKey, TuneEntry>;

TuneKey tune_key(int64_t n_atoms, int64_t nq, int precision, int mode, int64_t n_frames);

// The accumulation mode a request runs in: class mode unless its hydration
// weights give more than PD_MAX_CLASSES (species, weight) keys.
int request_mode(const pd_request *req, const uint32_t *species, const double *weights);

// Whether a shape can run a bucket (instantiated kernel, j chunk a positive
// multiple of 32).
bool valid_tuning(int precision, int mode, const Tuning &t);

// Text form, one bucket per line (blank lines and '#' comments ignored):
//   <fp32|fp64> <class|weighted> <single|frames> <log2 atoms> <log2 nq>
//   <q_block> <j_chunk> <pairs_per_thread> <ms>
// load_tuning adds the file's entries to `tab` (later lines win); a missing
// file is PD_ENOTFOUND, a malformed line PD_EINVAL naming it.
int load_tuning(const std::string &path, TuneTable &tab, std::string &msg);
int save_tuning(const std::string &path, const TuneTable &tab, std::string &msg);

}  // namespace pd
