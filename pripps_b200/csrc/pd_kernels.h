// Host-callable launchers of the device kernels (pd_kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "pd_common.h"

namespace pd {

bool valid_q_block(int precision, int K);
bool valid_shape(int precision, int mode, int K, int NP);
int pairs_blocks_per_sm(int precision, int K, int NP, int mode);
// Set the launch attributes of every FP32 pair-kernel shape on the current
// device (their shared-memory opt-in), so that no later launch — one inside a
// stream capture included — has to.
cudaError_t prepare_pair_kernels();

// n_jobs points to the tile count in device memory (read once per CTA).
cudaError_t launch_pairs(int precision, int K, int NP, int mode, const PdJob *jobs,
                         const int *n_jobs, const PdReqDev *reqs, int *counter, int grid,
                         cudaStream_t st);
cudaError_t launch_centroid(const double *xyz, int64_t n_atoms, int n_frames, double *centroid,
                            double *radius, cudaStream_t st);
cudaError_t launch_pack(const double *xyz, const double *weights, const int32_t *perm,
                        const double *centroid, int64_t n_atoms, int32_t n_pad, int32_t n_frames,
                        float4 *out32, double4 *out64, cudaStream_t st);
cudaError_t launch_reduce(const double *slots, const int64_t *lptr, const int64_t *lidx,
                          const PdPairDev *pairs, const double *qv, int32_t n_pairs, int32_t nq,
                          int32_t K, int32_t nv, int32_t n_frames, int64_t slots_per_frame,
                          const double *radius, double qmin, double dq, int residual_form,
                          int add_exact, double *pairsum, cudaStream_t st);
cudaError_t launch_combine(const double *pairsum, const PdClassDev *cls, const PdPairDev *pairs,
                           int32_t n_cls, int32_t n_pairs, int32_t nq, int32_t nv,
                           int32_t n_frames, const double *ffA, const double *ffC,
                           const double *ffW, int add_diag, double *terms, cudaStream_t st);
// Lattice sets: integer coordinates of their points and the exact pair count
// per squared offset (after pack), then their self pair sums (after the slot
// reduction, overwriting those class pairs' entries of pairsum).
cudaError_t launch_lattice(const double *xyz, const int32_t *perm, const PdLatDev *lat_dev,
                           const PdLatDev *lat_host, int n_lat, const PdLatTile *tiles,
                           int64_t n_tiles, int4 *idx, unsigned long long *hist, int64_t n_bins,
                           int *err, cudaStream_t st);
cudaError_t launch_lattice_sums(const unsigned long long *hist, const PdLatDev *lat, int n_lat,
                                const double *qv, int32_t nq, int add_exact, const int *err,
                                double *pairsum, cudaStream_t st);
cudaError_t launch_frame_mean(const double *terms, const double *fw, int32_t n_frames, int32_t nq,
                              double *out, cudaStream_t st, bool normalize = true);
// Direct transform: (Re A, Im A, |A|², Σ_m |F_m|²) per q-vector for points
// in molecules of mol_size (n_points a multiple of it). part holds
// direct_chunks(n_points, mol_size, n_vec) × n_vec × 5 doubles; the launch
// has direct_blocks(…) blocks (at most 2^31 - 1).
cudaError_t launch_direct(const double *xyz, const uint32_t *kind, const double *weight,
                          const double *ff, int32_t n_kinds, const double *qvec, int64_t n_vec,
                          int64_t n_points, int64_t mol_size, double *part, int64_t part_chunks,
                          double *out, cudaStream_t st);
int64_t direct_chunks(int64_t n_points, int64_t mol_size, int64_t n_vec);
// Direct transform at lattice vectors q = 2π·hkl/box from per-point phase
// tables (indices |h|, |k|, |l| <= nmax, with direct_table_points(nmax) >= 1);
// same part and out layouts as launch_direct.
int direct_table_points(int32_t nmax);
cudaError_t launch_direct_table(const double *xyz, const uint32_t *kind, const double *weight,
                                const double *ff, const int32_t *hkl, int32_t nmax,
                                const double box[3], int64_t n_vec, int64_t n_points,
                                int64_t mol_size, double *part, int64_t part_chunks, double *out,
                                cudaStream_t st);
int64_t direct_blocks(int64_t n_points, int64_t mol_size, int64_t n_vec);
// Form-factor tables [n_ff][nq] on the uniform grid; *bad = index + 1 of a
// form factor whose range misses a grid point (0 if none).
cudaError_t launch_ff_eval(const int32_t *desc, const double *range, const double *params,
                           int32_t n_ff, double qmin, double qmax, int64_t nq, int *bad,
                           double *out, cudaStream_t st);
cudaError_t launch_stream_accumulate(const double *batch, double scale, int32_t n, double *acc,
                                     cudaStream_t st);
cudaError_t launch_ffma_probe(float *out, int iters, int grid, int block, bool packed,
                              cudaStream_t st);

}  // namespace pd
