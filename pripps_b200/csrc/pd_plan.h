// Host planner: turns a pd_request into the device layout and tile list.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

#include "pd_common.h"
#include "pripps_debye.h"

namespace pd {

// At most this many (species, hydration weight) classes use the one-
// accumulator class mode; more distinct weights switch to the weighted mode.
constexpr int PD_MAX_CLASSES = 48;
// Lattice sets per request, and the largest squared grid diagonal (bins of
// its pair-count histogram).
constexpr uint32_t PD_MAX_LATTICES = 8;
constexpr int64_t PD_MAX_LATTICE_BINS = int64_t{1} << 24;
// Pair-count tiles: 128 i points × up to 8192 j points.
constexpr int PD_LAT_IBLOCK = 128;
constexpr int PD_LAT_JCHUNK = 8192;

struct Tuning {
    int K = 64;     // q-block length
    int TJ = 2048;  // j atoms per tile
    int NP = 2;     // pairs per thread per pass (FP32 form; 1 for FP64)
};

struct Plan {
    // request shape
    int64_t n_atoms = 0;
    int32_t nq = 0;
    int32_t n_frames = 1;
    int32_t n_species = 0;
    int precision = 0;
    bool has_exc = false, has_hyd = false;
    int mode = PD_MODE_CLASS;
    int nv = 1;  // values per slot entry: 1 (class) or 4 (weighted)
    bool test_expire = false;  // PD_FLAG_TEST_EXPIRED_WAIT
    Tuning tun;
    double qmin = 0, qmax = 0, dq = 0;
    std::vector<double> qv;

    // classes and layout
    int n_cls = 0, n_pairs = 0;
    std::vector<PdClassDev> cls;
    std::vector<PdPairDev> pairs;
    std::vector<int32_t> cls_start;  // padded start of each class region
    int32_t n_pad = 0;
    std::vector<int32_t> perm;    // [n_pad] source atom or -1
    std::vector<int32_t> gvalid;  // [n_pad/32]
    std::vector<int32_t> gclass;  // [n_pad/32] class or -1

    // tiles (execution order) and the deterministic reduction lists
    std::vector<PdJob> jobs;        // all frames
    int64_t jobs_per_frame = 0;
    int64_t slots_per_frame = 0;
    int nqb = 0;
    std::vector<int64_t> lptr;  // [n_pairs * nqb + 1]
    std::vector<int64_t> lidx;  // slot indices within a frame
    uint64_t pairs_covered = 0; // per frame, unordered pairs over all tiles

    // lattice sets (class mode, one frame): their self pairs are counted per
    // integer squared offset instead of running through the pair tiles
    std::vector<PdLatDev> lat;
    std::vector<PdLatTile> lat_tiles;
    int64_t lat_bins = 0;
};

// Validate a request; fills msg and returns a PD_E* code on failure.
int validate_request(const pd_request *req, bool device_pointers, std::string &msg);

// Default shape when no tuned entry exists.
Tuning default_tuning(int64_t n_atoms, int64_t nq, int precision, int64_t n_frames = 1);
// The instantiated kernel shape a requested one runs as in a mode (the q
// block and pairs per thread adjusted where that shape has no kernel).
Tuning fit_tuning(int precision, int mode, Tuning t);

// A rank's share of a plan for a tile-sharded solve: every world-th tile of
// the cost-ordered job list, with only the slots those tiles write (numbered
// in their original order) and the reduction lists cut to them.
int shard_plan(const Plan &full, uint32_t rank, uint32_t world, Plan &out);

// Build the plan from host-side species and weights (hyd may be NULL).
// count_pairs fills Plan::pairs_covered (an O(N · tiles per block) host loop
// that only pd_plan_inspect needs).
int build_plan(const pd_request *req, const uint32_t *species_host, const double *weights_host,
               const Tuning &tun, Plan &plan, std::string &msg, bool count_pairs = false);

}  // namespace pd
