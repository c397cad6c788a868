// Internal types shared by the host planner (pd_plan.cpp) and the device
// kernels (pd_kernels.cu) of libpripps_debye.
//
// Data layout in HBM, per request:
//   * atoms are re-ordered into "classes" (species, or species × hydration
//     weight when few distinct weights exist) and each class is padded to a
//     multiple of PD_GRANULE = 32 atoms, so that every warp-row of 32 i-atoms
//     belongs to one class; padded atoms are inert (gvalid masks them);
//   * coordinates are stored as float4 {x, y, z, w} (FP32 form) or double4
//     (FP64 form), centred on the frame centroid; w carries the per-atom
//     hydration weight in the weighted mode and is unused otherwise;
//   * a tile ("job") is (frame, i-block of PD_IBLOCK atoms, contiguous j range
//     of real atoms of ONE class, q-block of K grid points); it covers the
//     pairs (i, j) with j > i;
//   * the PD_WARPS warps of a tile keep their warp-reduced FP64 partial sums
//     for the K q-points in shared memory; at the end of the tile the warps of
//     one atom class are added in warp order and written to one FP64 slot per
//     distinct class of the i-block (usually one); a second kernel adds the
//     slots of every (class pair, q) in a fixed order, so the result does not
//     depend on which SM ran which tile.
#pragma once

#include <cstdint>

#ifndef __CUDACC__
struct float4 { float x, y, z, w; };
struct double4 { double x, y, z, w; };
#else
#include <cuda_runtime.h>
#endif

constexpr int PD_GRANULE = 32;                    // atoms per warp-row
constexpr int PD_WARPS = 4;                       // warps per tile CTA
constexpr int PD_THREADS = PD_GRANULE * PD_WARPS; // 128 threads
constexpr int PD_IBLOCK = PD_THREADS;             // i-atoms per tile

// Mode of the pair accumulation.
//   PD_MODE_CLASS:    one accumulator, Σ sin(q r)/r per class pair; every
//                     per-atom factor is a per-class constant.
//   PD_MODE_WEIGHTED: two accumulators, Σ sin(q r)/r and Σ w_j sin(q r)/r, for
//                     hydration weights that vary within a species.
enum PdMode : int32_t { PD_MODE_CLASS = 0, PD_MODE_WEIGHTED = 1 };

struct PdJob {
    int32_t req;    // request index within the launch
    int32_t frame;  // frame of the request
    int32_t i0;     // first padded i index (multiple of PD_IBLOCK)
    int32_t j0, j1; // padded j range [j0, j1): real atoms of one class
    int32_t qb;     // q-block index
    // bits 0..47: first output slot of this tile; bits 48..55: the slot of
    // each warp relative to it, 2 bits per warp (warp w at bits 48 + 2w).
    // Warps of one class share a slot; slot numbers follow the first warp
    // of each class, so warp 0 always has relative slot 0.
    int64_t slot;
};
static_assert(sizeof(PdJob) == 32, "PdJob layout");
constexpr int PD_SLOT_MAP_SHIFT = 48;
constexpr int64_t PD_SLOT_MASK = (int64_t{1} << PD_SLOT_MAP_SHIFT) - 1;

// Bits of the per-request device status word (PdReqDev::status).
constexpr int32_t PD_DEV_WAIT_EXPIRED = 1;  // a bounded wait for a bulk copy gave up

// PdReqDev::flags
constexpr int32_t PD_REQF_TEST_EXPIRE = 1;  // test hook: the launch's first tile skips its copy

// Per-request descriptor read by the pair kernels.
struct PdReqDev {
    const float4 *atoms32;    // [n_frames][n_pad] (FP32 form)
    const double4 *atoms64;   // [n_frames][n_pad] (FP64 form)
    const int32_t *gvalid;    // [n_pad / 32] valid atoms per granule
    const double *qv;         // [nq] grid (FP64 form reads it directly)
    double *slots;            // [n_slots][nv][K]
    const double *radius;     // [n_frames] largest atom distance from the centroid
    int32_t *status;          // PD_DEV_* bits, OR-ed in by the pair kernel
    double qmin, dq;          // grid origin and step
    int32_t n_pad;
    int32_t nq;
    int32_t K;
    int32_t mode;
    int32_t flags;            // PD_REQF_* bits
    int32_t pad_;
};

// Per-class constants for the combine kernel.
struct PdClassDev {
    int32_t species;
    int32_t pad;
    double n;   // atoms in the class
    double w;   // hydration weight (class mode)
    double w1;  // Σ w_i over the class (weighted mode)
    double w2;  // Σ w_i² over the class (weighted mode)
};

// Per-class-pair constants: classes (a <= b) and the q = 0 pair sums
// (sinc = 1 for every pair): count, Σ w_i, Σ w_j, Σ w_i w_j.
struct PdPairDev {
    int32_t a, b;
    double q0[4];
};

// A lattice set of one class: its points are origin + spacing·(i, j, k); the
// class's self pair sums come from the exact pair count per integer squared
// offset n = |Δ(i, j, k)|², hist[hist_off + n], n < n_bins.
struct PdLatDev {
    double origin[3];
    double spacing;
    int32_t ext[3];
    int32_t cls;       // class index
    int32_t start;     // padded index of the class's first point
    int32_t n;         // points of the class
    int32_t pair;      // class-pair index (cls, cls)
    int32_t n_bins;    // max n + 1
    int64_t hist_off;  // first bin in the histogram array
};

// One CTA of the pair-count kernel: lattice `lat`, i points [i0, i0 + 128)
// of the class (relative to its start), j points [j0, j1), pairs with j > i.
struct PdLatTile {
    int32_t lat, i0, j0, j1;
};
static_assert(sizeof(PdLatTile) == 16, "PdLatTile layout");
