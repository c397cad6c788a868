// Device kernels of the Debye backend (sm_100a).
//
// K1 (pd_pairs_fp32): for each tile (i-block × j-range × q-block) every thread
// owns one i atom and walks the j atoms of the range two at a time. For a pair
// at distance r it needs sin(q_k r) for the K consecutive grid points
// q_k = q_s + k·Δq of the block. With x = Δq·r reduced as x = mπ + x'
// (|x'| <= π/2) the sequence is s_k = σ^k·u_k, σ = (-1)^m, where
// u_k = sin(θ + k x'), θ = q_s r. u_k follows the three-term recurrence
// u_{k+1} = 2cos(x')·u_k − u_{k−1}, evaluated in Reinsch's difference form
//   d_{k+1} = d_k − α·u_k,  u_{k+1} = u_k + d_{k+1},  α = 4 sin²(x'/2),
// which stays accurate for small x' (Reinsch's modification of the Goertzel
// recurrence; errors grow linearly in k). It is reseeded every K steps from an
// accurate sincosf(θ). One step plus the accumulation acc_k += σ^k u_k / r is
// FFMA + FADD + FFMA, all on the FP32 pipes. acc_k sums sin(q_k r)/r over the
// thread's pairs; dividing by q_k in FP64 afterwards gives Σ sinc(q_k r).
// Per-tile sums stay in FP32 registers; they are warp-reduced and written as
// FP64 slots, and every later sum is FP64.
//
// K2 (pd_pairs_fp64): the same tiling with sin(q_k r) from the FP64 sin() for
// every pair and q, and FP64 accumulation throughout.
#include <cuda_runtime.h>

#include <cstdint>
#include <cstdio>

#include "pd_common.h"
#include "pd_kernels.h"

namespace pd {

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sin and cos on |h| <= π/4 as polynomials in h² whose FP32 coefficients were
// fitted (least squares on Chebyshev nodes, each coefficient rounded to FP32
// before the next ones were refitted): |error| < 4e-11 for sin and < 1e-11
// for cos on the interval, in exact arithmetic, far under the FP32 rounding
// of the result. Taylor coefficients rounded to FP32 leave a one-signed
// error of ~1e-9, which a sum over 10^8 pairs turns into a bias.
__device__ __forceinline__ float sin_small(float h) {
    const float h2 = h * h;
    float p = -2.597475088e-7f;
    p = fmaf(p, h2, 3.148236829e-6f);
    p = fmaf(p, h2, -1.986468124e-4f);
    p = fmaf(p, h2, 8.333391510e-3f);
    p = fmaf(p, h2, -1.666666716e-1f);
    return fmaf(h * h2, p, h);
}
__device__ __forceinline__ float cos_small(float h) {
    const float h2 = h * h;
    float p = -2.870663707e-7f;
    p = fmaf(p, h2, 2.482019954e-5f);
    p = fmaf(p, h2, -1.388897537e-3f);
    p = fmaf(p, h2, 4.166666791e-2f);
    p = fmaf(p, h2, -0.5f);
    return fmaf(h2, p, 1.0f);
}

// Three-part π/2 for the reduction: C1 has 8 significant bits, so n·C1 and
// th − n·C1 are exact for n < 2^15; C2 = fl32(π/2 − C1); C3 = fl32(π/2 − C1 − C2).
constexpr float kPio2C1 = 1.5703125f;
constexpr float kPio2C2 = 4.838267923333e-4f;
constexpr float kPio2C3 = 2.563282919255e-12f;

// sin and cos of an angle given as an unevaluated sum th_hi + th_lo
// (|th_hi| <~ 1e4, |th_lo| a few ulp of th_hi), without a branch:
// th = n·π/2 + t, t = (th_hi − n·C1) + (th_lo − n·C2 − n·C3), then the
// polynomials on |t| <= π/4 and the quadrant of n.
//
// Why the low part: th_hi lies on the FP32 grid of its binade, and th_hi − n·C1
// is exact, so rounding (th_hi − n·π/2) to FP32 in one step gives the same
// rounding error to every pair of that quadrant and binade — a bias of
// ~2e-9 per sin that survives a sum over 10^7..10^10 pairs. th_lo carries
// the pair's own rounding residue of q·r, so the final rounding of t falls
// at a random place between grid points and averages out.
__device__ __forceinline__ void sincos_reduced(float th_hi, float th_lo, float &s, float &c) {
    const float n = rintf(th_hi * 0.636619772f);
    const float t1 = fmaf(-n, kPio2C1, th_hi);  // exact
    float u = fmaf(-n, kPio2C2, th_lo);
    u = fmaf(-n, kPio2C3, u);
    const float t = t1 + u;
    const float st = sin_small(t), ct = cos_small(t);
    const int qd = static_cast<int>(n);
    const bool swap = (qd & 1) != 0;
    float ss = swap ? ct : st;
    float cc = swap ? st : ct;
    s = (qd & 2) ? -ss : ss;
    c = ((qd + 1) & 2) ? -cc : cc;
}

// Seed of one pair for a q-block. The K values s_k = sin(θ + k x), θ = q_s r,
// x = Δq r, are produced as two interleaved sequences, even k and odd k, each
// a sinusoid in j = k/2 with step y = 2x: s_{2j} = sin(θ + j y) and
// s_{2j+1} = sin(θ + x + j y). With y = mπ + y' (|y'| <= π/2) and σ = (-1)^m,
// both are σ^j·v_j where v follows the Reinsch recurrence with
// α = 4 sin²(y'/2). Two independent chains per pair halve the dependency
// stall of the FFMA → FADD step without adding instructions.
struct PairSeed {
    float ve, de, vo, dd, na, we, wo;
};

// Three-part π for the step reduction (C1 = 3.140625 has 8 significant bits).
constexpr float kPiC1 = 3.140625f;
constexpr float kPiC2 = 9.676535846666e-4f;
constexpr float kPiC3 = 5.126565838511e-12f;

__device__ __forceinline__ PairSeed pair_seed(float4 pi, float4 pj, bool valid, float qs_hi,
                                              float qs_lo, float dq2_hi, float dq2_lo) {
    const float dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
    float r2 = fmaf(dx, dx, fmaf(dy, dy, dz * dz));
    // Coincident points: sinc(0) = 1, i.e. sin(q r)/r -> q; r = 1e-6 Å gives
    // that limit to 1e-13 relative.
    r2 = fmaxf(r2, 1e-12f);
    float inv_r = rsqrtf(r2);
    // r = r_hi + r_lo to ~2^-44 relative: one Newton step on sqrt, its
    // correction kept apart.
    const float r_hi = r2 * inv_r;
    const float hinv = 0.5f * inv_r;
    const float r_lo = hinv * fmaf(-r_hi, r_hi, r2);
    // One Newton step on 1/r as well: the weight multiplies every term of the
    // pair, so its error must be unbiased, not just small.
    inv_r = fmaf(hinv, fmaf(-r2 * inv_r, inv_r, 1.0f), inv_r);
    // θ = q_s·r and y = 2Δq·r as hi + lo pairs (exact product residue plus the
    // cross terms of the two double-float factors).
    const float th_hi = qs_hi * r_hi;
    const float th_lo = fmaf(qs_hi, r_hi, -th_hi) + fmaf(qs_hi, r_lo, qs_lo * r_hi);
    const float y_hi = dq2_hi * r_hi;
    const float y_lo = fmaf(dq2_hi, r_hi, -y_hi) + fmaf(dq2_hi, r_lo, dq2_lo * r_hi);
    // y = mπ + y', |y'| <= π/2, reduced like θ.
    const float m = rintf(y_hi * 0.318309886f);
    float yl = fmaf(-m, kPiC2, y_lo);
    yl = fmaf(-m, kPiC3, yl);
    const float yr = fmaf(-m, kPiC1, y_hi) + yl;
    const int mi = static_cast<int>(m);
    const float h = 0.5f * yr;  // x = m·π/2 + h
    const float sh = sin_small(h), ch = cos_small(h);
    // sin x, cos x from the quadrant of m
    const bool swap = (mi & 1) != 0;
    float sx = swap ? ch : sh;
    float cx = swap ? sh : ch;
    sx = (mi & 2) ? -sx : sx;
    cx = ((mi + 1) & 2) ? -cx : cx;
    float s0, c0;
    sincos_reduced(th_hi, th_lo, s0, c0);
    const float s1 = fmaf(s0, cx, c0 * sx);   // sin(θ + x)
    const float c1 = fmaf(c0, cx, -s0 * sx);  // cos(θ + x)
    const float sh2 = 2.0f * sh;
    PairSeed ps;
    ps.ve = s0;                                // v_0 even = sin θ
    ps.de = sh2 * fmaf(c0, ch, s0 * sh);       // sin θ − sin(θ − y') = 2 sin h cos(θ − h)
    ps.vo = s1;                                // v_0 odd = sin(θ + x)
    ps.dd = sh2 * fmaf(c1, ch, s1 * sh);
    ps.na = -sh2 * sh2;                        // −α = −4 sin² h
    const float w = valid ? inv_r : 0.0f;
    ps.we = w;
    ps.wo = (mi & 1) ? -w : w;
    return ps;
}

// Small-q residual form: where q·(2·radius) < 2 every pair has q·r < 2 and
// the terms sin(q r)/r lie within a factor 0.45..1 of q, so a sequential FP32
// sum of them rounds with a systematic bias. There the kernel accumulates
// sin(q r)/r − q and the reduction adds (pair count)·q back in FP64. Both
// kernels evaluate this predicate on the same FP64 values.
__host__ __device__ __forceinline__ bool residual_q(double q, double radius) {
    return q * (2.0 * radius) < 2.0;
}

// ---------------------------------------------------------------- K1 (FP32)
// NP pairs per thread per pass, two chains each: 2·NP independent recurrences.
template <int K, int MODE, int NP, bool RESID>
__device__ __forceinline__ void pairs_range(const float4 *__restrict__ at, float4 pi, int i,
                                            bool ivalid, int j0, int j1, float qs_hi,
                                            float qs_lo, float dq_hi, float dq_lo,
                                            const float *__restrict__ s_qres,
                                            float (&acc)[(MODE == PD_MODE_WEIGHTED) ? 2 : 1][K]) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    static_assert(K % 4 == 0, "K must be a multiple of 4");
    for (int j = j0; j < j1; j += NP) {
        PairSeed S[NP];
        float wj[NP];
        float vsum = 0.0f, vwsum = 0.0f;
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int jj = j + p;
            const bool inr = jj < j1;
            const float4 pj = __ldg(at + (inr ? jj : j));
            const bool valid = ivalid && inr && (jj > i);
            S[p] = pair_seed(pi, pj, valid, qs_hi, qs_lo, dq_hi, dq_lo);
            wj[p] = pj.w;
            if (RESID) {
                vsum += valid ? 1.0f : 0.0f;
                if (MODE == PD_MODE_WEIGHTED) vwsum += valid ? pj.w : 0.0f;
            }
        }
        float we_w[NP], wo_w[NP];
        if (MODE == PD_MODE_WEIGHTED) {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                we_w[p] = S[p].we * wj[p];
                wo_w[p] = S[p].wo * wj[p];
            }
        }
        // The q table is the same in every pass; an opaque zero offset keeps
        // the compiler from hoisting all K loads into registers.
        int qoff = 0;
        if (RESID) asm volatile("mov.b32 %0, %0;" : "+r"(qoff));
#pragma unroll
        for (int k = 0; k < K; k += 4) {
#pragma unroll
            for (int h = 0; h < 4; ++h) {
                const int kk = k + h;
                const bool odd_chain = (h & 1) != 0;  // k = 4t+1, 4t+3
                const bool odd_j = (h & 2) != 0;      // j = 2t+1: weight σ·w
                if (RESID) {
                    const float qk = s_qres[kk + qoff];
                    acc[0][kk] = fmaf(-vsum, qk, acc[0][kk]);
                    if (MODE == PD_MODE_WEIGHTED)
                        acc[NACC - 1][kk] = fmaf(-vwsum, qk, acc[NACC - 1][kk]);
                }
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float w = odd_j ? S[p].wo : S[p].we;
                    float &v = odd_chain ? S[p].vo : S[p].ve;
                    float &d = odd_chain ? S[p].dd : S[p].de;
                    acc[0][kk] = fmaf(w, v, acc[0][kk]);
                    if (MODE == PD_MODE_WEIGHTED)
                        acc[NACC - 1][kk] = fmaf(odd_j ? wo_w[p] : we_w[p], v, acc[NACC - 1][kk]);
                    d = fmaf(S[p].na, v, d);
                    v += d;
                }
            }
        }
    }
}

// Resident CTAs per SM each FP32 shape is compiled for (register budget
// 65536 / (128 · blocks) per thread).
constexpr int fp32_min_blocks(int K, int MODE, int NP) {
    return MODE == PD_MODE_CLASS ? (K <= 64 ? 4 : (NP == 2 ? 3 : 2)) : (K <= 32 ? 4 : 2);
}

template <int K, int MODE, int NP>
__global__ void __launch_bounds__(PD_THREADS, fp32_min_blocks(K, MODE, NP))
    pd_pairs_fp32(const PdJob *__restrict__ jobs,
                                                            const int *__restrict__ n_jobs_ptr,
                                                            const PdReqDev *__restrict__ reqs,
                                                            int *__restrict__ counter) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    __shared__ int s_job;
    __shared__ float s_qres[K];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int n_jobs = *n_jobs_ptr;
    for (;;) {
        if (threadIdx.x == 0) s_job = atomicAdd(counter, 1);
        __syncthreads();
        const int jid = s_job;
        if (jid >= n_jobs) break;
        const PdJob jb = jobs[jid];
        const PdReqDev rq = reqs[jb.req];
        const int kq0 = jb.qb * K;
        const double radius = rq.radius[jb.frame];
        const bool resid = kq0 < rq.nq && residual_q(rq.qv[kq0], radius);
        if (resid && threadIdx.x < K) {
            const int kq = kq0 + threadIdx.x;
            const bool on = kq < rq.nq && residual_q(rq.qv[kq], radius);
            s_qres[threadIdx.x] = on ? static_cast<float>(rq.qv[kq]) : 0.0f;
        }
        __syncthreads();  // s_qres ready; every thread has read s_job
        const float4 *__restrict__ at = rq.atoms32 + static_cast<size_t>(jb.frame) * rq.n_pad;
        const int i = jb.i0 + threadIdx.x;
        const float4 pi = at[i];
        const bool ivalid = lane < rq.gvalid[(jb.i0 >> 5) + warp];
        const double qs = rq.qmin + static_cast<double>(kq0) * rq.dq;
        const float qs_hi = static_cast<float>(qs);
        const float qs_lo = static_cast<float>(qs - static_cast<double>(qs_hi));
        const double dq2 = 2.0 * rq.dq;  // step of the even/odd chains
        const float dq_hi = static_cast<float>(dq2);
        const float dq_lo = static_cast<float>(dq2 - static_cast<double>(dq_hi));

        float acc[NACC][K];
#pragma unroll
        for (int a = 0; a < NACC; ++a)
#pragma unroll
            for (int k = 0; k < K; ++k) acc[a][k] = 0.0f;

        if (resid)
            pairs_range<K, MODE, NP, true>(at, pi, i, ivalid, jb.j0, jb.j1, qs_hi, qs_lo, dq_hi,
                                           dq_lo, s_qres, acc);
        else
            pairs_range<K, MODE, NP, false>(at, pi, i, ivalid, jb.j0, jb.j1, qs_hi, qs_lo, dq_hi,
                                            dq_lo, s_qres, acc);

        // Warp-reduce and write this warp's slot: [nv][K] FP64 values.
        double *slot = rq.slots + (jb.slot + warp) * static_cast<int64_t>(K) *
                                      (MODE == PD_MODE_WEIGHTED ? 4 : 1);
        if (MODE == PD_MODE_CLASS) {
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float v = warp_sum(acc[0][k]);
                if (lane == (k & 31)) slot[k] = static_cast<double>(v);
            }
        } else {
            const float wi = ivalid ? pi.w : 0.0f;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const float t0 = warp_sum(acc[0][k]);
                const float ti = warp_sum(wi * acc[0][k]);
                const float tj = warp_sum(acc[NACC - 1][k]);
                const float tij = warp_sum(wi * acc[NACC - 1][k]);
                if (lane == (k & 31)) {
                    slot[k] = t0;
                    slot[K + k] = ti;
                    slot[2 * K + k] = tj;
                    slot[3 * K + k] = tij;
                }
            }
        }
        __syncthreads();  // s_qres and s_job are rewritten by the next tile
    }
}

// ---------------------------------------------------------------- K2 (FP64)
template <int K, int MODE>
__global__ void __launch_bounds__(PD_THREADS) pd_pairs_fp64(const PdJob *__restrict__ jobs,
                                                            const int *__restrict__ n_jobs_ptr,
                                                            const PdReqDev *__restrict__ reqs,
                                                            int *__restrict__ counter) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    __shared__ int s_job;
    __shared__ double s_q[K];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int n_jobs = *n_jobs_ptr;
    for (;;) {
        if (threadIdx.x == 0) s_job = atomicAdd(counter, 1);
        __syncthreads();
        const int jid = s_job;
        if (jid >= n_jobs) break;
        const PdJob jb = jobs[jid];
        const PdReqDev rq = reqs[jb.req];
        if (threadIdx.x < K) {
            const int kq = jb.qb * K + threadIdx.x;
            s_q[threadIdx.x] = kq < rq.nq ? rq.qv[kq] : 0.0;
        }
        __syncthreads();
        const double4 *__restrict__ at = rq.atoms64 + static_cast<size_t>(jb.frame) * rq.n_pad;
        const int i = jb.i0 + threadIdx.x;
        const double4 pi = at[i];
        const bool ivalid = lane < rq.gvalid[(jb.i0 >> 5) + warp];

        double acc[NACC][K];
#pragma unroll
        for (int a = 0; a < NACC; ++a)
#pragma unroll
            for (int k = 0; k < K; ++k) acc[a][k] = 0.0;

        for (int j = jb.j0; j < jb.j1; ++j) {
            const double4 pj = at[j];
            const double dx = pi.x - pj.x, dy = pi.y - pj.y, dz = pi.z - pj.z;
            double r2 = dx * dx + dy * dy + dz * dz;
            r2 = fmax(r2, 1e-24);
            const double r = sqrt(r2);
            const double w0 = (ivalid && j > i) ? 1.0 / r : 0.0;
            const double w1 = w0 * pj.w;
#pragma unroll
            for (int k = 0; k < K; ++k) {
                const double s = sin(s_q[k] * r);
                acc[0][k] = fma(w0, s, acc[0][k]);
                if (MODE == PD_MODE_WEIGHTED) acc[NACC - 1][k] = fma(w1, s, acc[NACC - 1][k]);
            }
        }

        double *slot = rq.slots + (jb.slot + warp) * static_cast<int64_t>(K) *
                                      (MODE == PD_MODE_WEIGHTED ? 4 : 1);
        const double wi = ivalid ? pi.w : 0.0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double t0 = warp_sum(acc[0][k]);
            if (MODE == PD_MODE_CLASS) {
                if (lane == (k & 31)) slot[k] = t0;
            } else {
                const double ti = warp_sum(wi * acc[0][k]);
                const double tj = warp_sum(acc[NACC - 1][k]);
                const double tij = warp_sum(wi * acc[NACC - 1][k]);
                if (lane == (k & 31)) {
                    slot[k] = t0;
                    slot[K + k] = ti;
                    slot[2 * K + k] = tj;
                    slot[3 * K + k] = tij;
                }
            }
        }
        __syncthreads();  // s_q is rewritten by the next tile
    }
}

// ------------------------------------------------------- pack and centroid
// Per-frame centroid of the input positions (FP64, fixed-order tree) and the
// largest distance of an atom from it.
__global__ void pd_centroid(const double *__restrict__ xyz, int64_t n_atoms,
                            double *__restrict__ centroid, double *__restrict__ radius) {
    __shared__ double red[3][256];
    const int f = blockIdx.x;
    const double *p = xyz + static_cast<size_t>(f) * n_atoms * 3;
    double sx = 0, sy = 0, sz = 0;
    for (int64_t i = threadIdx.x; i < n_atoms; i += blockDim.x) {
        sx += p[3 * i];
        sy += p[3 * i + 1];
        sz += p[3 * i + 2];
    }
    red[0][threadIdx.x] = sx;
    red[1][threadIdx.x] = sy;
    red[2][threadIdx.x] = sz;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) {
            red[0][threadIdx.x] += red[0][threadIdx.x + s];
            red[1][threadIdx.x] += red[1][threadIdx.x + s];
            red[2][threadIdx.x] += red[2][threadIdx.x + s];
        }
        __syncthreads();
    }
    const double cx = red[0][0] / static_cast<double>(n_atoms);
    const double cy = red[1][0] / static_cast<double>(n_atoms);
    const double cz = red[2][0] / static_cast<double>(n_atoms);
    __syncthreads();
    if (threadIdx.x == 0) {
        centroid[3 * f] = cx;
        centroid[3 * f + 1] = cy;
        centroid[3 * f + 2] = cz;
    }
    double rm = 0.0;
    for (int64_t i = threadIdx.x; i < n_atoms; i += blockDim.x) {
        const double dx = p[3 * i] - cx, dy = p[3 * i + 1] - cy, dz = p[3 * i + 2] - cz;
        rm = fmax(rm, dx * dx + dy * dy + dz * dz);
    }
    red[0][threadIdx.x] = rm;
    __syncthreads();
    for (int s = blockDim.x / 2; s > 0; s >>= 1) {
        if (threadIdx.x < s) red[0][threadIdx.x] = fmax(red[0][threadIdx.x], red[0][threadIdx.x + s]);
        __syncthreads();
    }
    if (threadIdx.x == 0) radius[f] = sqrt(red[0][0]);
}

// Gather positions into the class-sorted, padded layout, centred per frame.
__global__ void pd_pack(const double *__restrict__ xyz, const double *__restrict__ weights,
                        const int32_t *__restrict__ perm, const double *__restrict__ centroid,
                        int64_t n_atoms, int32_t n_pad, int32_t n_frames,
                        float4 *__restrict__ out32, double4 *__restrict__ out64) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= static_cast<int64_t>(n_pad) * n_frames) return;
    const int f = static_cast<int>(t / n_pad);
    const int p = static_cast<int>(t % n_pad);
    const int src = perm[p];
    double x = 0, y = 0, z = 0, w = 0;
    if (src >= 0) {
        const double *s = xyz + (static_cast<size_t>(f) * n_atoms + src) * 3;
        x = s[0] - centroid[3 * f];
        y = s[1] - centroid[3 * f + 1];
        z = s[2] - centroid[3 * f + 2];
        w = weights ? weights[src] : 0.0;
    }
    if (out32) out32[t] = make_float4(static_cast<float>(x), static_cast<float>(y),
                                      static_cast<float>(z), static_cast<float>(w));
    if (out64) out64[t] = make_double4(x, y, z, w);
}

// ------------------------------------------------------------ reductions
// Sum the slots of every (frame, class pair, q) in list order, then turn the
// Σ sin(q r)/r partials into Σ sinc(q r) by dividing by q; q = 0 takes the
// exact pair sums. pairsum is [frame][nv][n_pairs][nq].
__global__ void pd_reduce_pairs(const double *__restrict__ slots, const int64_t *__restrict__ lptr,
                                const int64_t *__restrict__ lidx, const PdPairDev *__restrict__ pairs,
                                const double *__restrict__ qv, int32_t n_pairs, int32_t nq,
                                int32_t K, int32_t nv, int32_t n_frames, int64_t slots_per_frame,
                                const double *__restrict__ radius, double qmin, double dq,
                                int32_t residual_form, int32_t add_exact,
                                double *__restrict__ pairsum) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    const int64_t per_frame = static_cast<int64_t>(n_pairs) * nq;
    if (t >= per_frame * n_frames) return;
    const int f = static_cast<int>(t / per_frame);
    const int rem = static_cast<int>(t % per_frame);
    const int p = rem / nq;
    const int q = rem % nq;
    const int nqb = (nq + K - 1) / K;
    const int qb = q / K, kk = q % K;
    const double qval = qv[q];
    double s[4] = {0, 0, 0, 0};
    if (qval > 0.0) {
        const int64_t e0 = lptr[p * nqb + qb], e1 = lptr[p * nqb + qb + 1];
        const int64_t fbase = static_cast<int64_t>(f) * slots_per_frame;
        for (int64_t e = e0; e < e1; ++e) {
            const double *sl = slots + (fbase + lidx[e]) * static_cast<int64_t>(nv) * K;
            for (int v = 0; v < nv; ++v) s[v] += sl[v * K + kk];
        }
        for (int v = 0; v < nv; ++v) s[v] /= qval;
        if (add_exact && residual_form && residual_q(qval, radius[f]))
            for (int v = 0; v < nv; ++v) s[v] += pairs[p].q0[v];
    } else if (add_exact) {
        for (int v = 0; v < 4; ++v) s[v] = pairs[p].q0[v];
    }
    const int64_t ob = static_cast<int64_t>(f) * nv * per_frame;
    for (int v = 0; v < nv; ++v) pairsum[ob + static_cast<int64_t>(v) * per_frame + rem] = s[v];
}

// Six profiles per (frame, q) from the class-pair sums, in FP64.
__global__ void pd_combine_terms(const double *__restrict__ pairsum,
                                 const PdClassDev *__restrict__ cls,
                                 const PdPairDev *__restrict__ pairs, int32_t n_cls,
                                 int32_t n_pairs, int32_t nq, int32_t nv, int32_t n_frames,
                                 const double *__restrict__ ffA, const double *__restrict__ ffC,
                                 const double *__restrict__ ffW, int32_t add_diag,
                                 double *__restrict__ terms) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= static_cast<int64_t>(nq) * n_frames) return;
    const int f = static_cast<int>(t / nq);
    const int q = static_cast<int>(t % nq);
    const double fw = ffW ? ffW[q] : 0.0;
    const bool weighted = (nv == 4);
    double AA = 0, CC = 0, BB = 0, AC = 0, AB = 0, CB = 0;
    for (int c = 0; c < (add_diag ? n_cls : 0); ++c) {  // i = j terms
        const double fa = ffA[static_cast<int64_t>(cls[c].species) * nq + q];
        const double ca = ffC ? ffC[static_cast<int64_t>(cls[c].species) * nq + q] : 0.0;
        const double n = cls[c].n;
        AA += n * fa * fa;
        CC += n * ca * ca;
        AC += n * fa * ca;
        if (weighted) {
            BB += fw * fw * cls[c].w2;
            AB += fa * fw * cls[c].w1;
            CB += ca * fw * cls[c].w1;
        } else {
            const double b = cls[c].w * fw;
            BB += n * b * b;
            AB += n * fa * b;
            CB += n * ca * b;
        }
    }
    const int64_t per_frame = static_cast<int64_t>(n_pairs) * nq;
    const double *ps = pairsum + static_cast<int64_t>(f) * nv * per_frame;
    for (int p = 0; p < n_pairs; ++p) {  // i < j terms
        const int a = pairs[p].a, b = pairs[p].b;
        const double fa = ffA[static_cast<int64_t>(cls[a].species) * nq + q];
        const double fb = ffA[static_cast<int64_t>(cls[b].species) * nq + q];
        const double ca = ffC ? ffC[static_cast<int64_t>(cls[a].species) * nq + q] : 0.0;
        const double cb = ffC ? ffC[static_cast<int64_t>(cls[b].species) * nq + q] : 0.0;
        const double s0 = ps[static_cast<int64_t>(p) * nq + q];
        AA += 2.0 * fa * fb * s0;
        CC += 2.0 * ca * cb * s0;
        AC += (fa * cb + ca * fb) * s0;
        if (weighted) {
            const double si = ps[per_frame + static_cast<int64_t>(p) * nq + q];
            const double sj = ps[2 * per_frame + static_cast<int64_t>(p) * nq + q];
            const double sij = ps[3 * per_frame + static_cast<int64_t>(p) * nq + q];
            BB += 2.0 * fw * fw * sij;
            AB += fw * (fa * sj + fb * si);
            CB += fw * (ca * sj + cb * si);
        } else {
            const double ba = cls[a].w * fw, bb = cls[b].w * fw;
            BB += 2.0 * ba * bb * s0;
            AB += (fa * bb + ba * fb) * s0;
            CB += (ca * bb + ba * cb) * s0;
        }
    }
    double *o = terms + static_cast<int64_t>(f) * 6 * nq;
    o[q] = AA;
    o[nq + q] = CC;
    o[2 * nq + q] = BB;
    o[3 * nq + q] = AC;
    o[4 * nq + q] = AB;
    o[5 * nq + q] = CB;
}

// Frame-weighted mean of the six profiles, frames added in order.
__global__ void pd_frame_mean(const double *__restrict__ terms, const double *__restrict__ fw,
                              int32_t n_frames, int32_t nq, double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * nq) return;
    double s = 0.0, wsum = 0.0;
    for (int f = 0; f < n_frames; ++f) {
        const double w = fw ? fw[f] : 1.0;
        s += w * terms[static_cast<int64_t>(f) * 6 * nq + t];
        wsum += w;
    }
    out[t] = s / wsum;
}

// ------------------------------------------------------------ FP32 probe
// Register-only FFMA throughput: 8 independent chains per thread.
__global__ void pd_ffma_probe(float *out, int iters, float a, float b) {
    float v[8];
#pragma unroll
    for (int c = 0; c < 8; ++c) v[c] = threadIdx.x * 1e-3f + c;
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 8; ++c) v[c] = fmaf(v[c], a, b);
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) s += v[c];
    if (s == 12345.678f) out[0] = s;
}

// Same with packed FP32x2 FMAs (fma.rn.f32x2, sm_100a).
__global__ void pd_ffma2_probe(float *out, int iters, float a, float b) {
    unsigned long long v[8];
    float2 init;
    unsigned long long av, bv;
    {
        float2 t = make_float2(a, a);
        av = *reinterpret_cast<unsigned long long *>(&t);
        t = make_float2(b, b);
        bv = *reinterpret_cast<unsigned long long *>(&t);
    }
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        init = make_float2(threadIdx.x * 1e-3f + c, c * 0.5f);
        v[c] = *reinterpret_cast<unsigned long long *>(&init);
    }
    for (int it = 0; it < iters; ++it) {
#pragma unroll
        for (int u = 0; u < 16; ++u)
#pragma unroll
            for (int c = 0; c < 8; ++c)
                asm volatile("fma.rn.f32x2 %0, %0, %1, %2;" : "+l"(v[c]) : "l"(av), "l"(bv));
    }
    float s = 0;
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        float2 t = *reinterpret_cast<float2 *>(&v[c]);
        s += t.x + t.y;
    }
    if (s == 12345.678f) out[0] = s;
}

// ------------------------------------------------------------ launchers
template <int K, int MODE, int NP>
static cudaError_t launch_fp32_t(const PdJob *jobs, const int *n_jobs, const PdReqDev *reqs,
                                 int *counter, int grid, cudaStream_t st) {
    pd_pairs_fp32<K, MODE, NP><<<grid, PD_THREADS, 0, st>>>(jobs, n_jobs, reqs, counter);
    return cudaGetLastError();
}
template <int K, int MODE>
static cudaError_t launch_fp64_t(const PdJob *jobs, const int *n_jobs, const PdReqDev *reqs,
                                 int *counter, int grid, cudaStream_t st) {
    pd_pairs_fp64<K, MODE><<<grid, PD_THREADS, 0, st>>>(jobs, n_jobs, reqs, counter);
    return cudaGetLastError();
}
template <int K, int MODE, int NP>
static int occupancy_fp32() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pd_pairs_fp32<K, MODE, NP>, PD_THREADS, 0);
    return n;
}
template <int K, int MODE>
static int occupancy_fp64() {
    int n = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pd_pairs_fp64<K, MODE>, PD_THREADS, 0);
    return n;
}

// (K, NP) shapes instantiated for the FP32 form; the weighted mode (two
// accumulators per q) only up to K = 64 to stay within 255 registers.
bool valid_shape(int precision, int mode, int K, int NP) {
    if (precision == 1) return (K == 16 || K == 32) && NP == 1;
    if (mode == PD_MODE_WEIGHTED) return (K == 32 && NP == 2) || (K == 64 && NP == 2);
    return (K == 32 && NP == 4) || (K == 64 && (NP == 2 || NP == 4)) || (K == 96 && NP == 2) ||
           (K == 128 && (NP == 2 || NP == 4));
}

bool valid_q_block(int precision, int K) {
    if (precision == 1) return K == 16 || K == 32;
    return K == 32 || K == 64 || K == 96 || K == 128;
}

#define PD_F32(K, M, NP)                                                                 \
    if (K_ == K && mode == M && NP_ == NP)                                               \
        return launch_fp32_t<K, M, NP>(jobs, n_jobs, reqs, counter, grid, st);
#define PD_F64(K, M) \
    if (K_ == K && mode == M) return launch_fp64_t<K, M>(jobs, n_jobs, reqs, counter, grid, st);

cudaError_t launch_pairs(int precision, int K_, int NP_, int mode, const PdJob *jobs,
                         const int *n_jobs, const PdReqDev *reqs, int *counter, int grid,
                         cudaStream_t st) {
    if (precision == 1) {
        PD_F64(16, 0) PD_F64(16, 1) PD_F64(32, 0) PD_F64(32, 1)
        return cudaErrorInvalidValue;
    }
    PD_F32(32, 0, 4) PD_F32(64, 0, 2) PD_F32(64, 0, 4) PD_F32(96, 0, 2) PD_F32(128, 0, 2)
    PD_F32(128, 0, 4) PD_F32(32, 1, 2) PD_F32(64, 1, 2)
    return cudaErrorInvalidValue;
}

#define PD_O32(K, M, NP) \
    if (K_ == K && mode == M && NP_ == NP) return occupancy_fp32<K, M, NP>();
#define PD_O64(K, M) \
    if (K_ == K && mode == M) return occupancy_fp64<K, M>();

int pairs_blocks_per_sm(int precision, int K_, int NP_, int mode) {
    if (precision == 1) {
        PD_O64(16, 0) PD_O64(16, 1) PD_O64(32, 0) PD_O64(32, 1)
        return 0;
    }
    PD_O32(32, 0, 4) PD_O32(64, 0, 2) PD_O32(64, 0, 4) PD_O32(96, 0, 2) PD_O32(128, 0, 2)
    PD_O32(128, 0, 4) PD_O32(32, 1, 2) PD_O32(64, 1, 2)
    return 0;
}

cudaError_t launch_centroid(const double *xyz, int64_t n_atoms, int n_frames, double *centroid,
                            double *radius, cudaStream_t st) {
    pd_centroid<<<n_frames, 256, 0, st>>>(xyz, n_atoms, centroid, radius);
    return cudaGetLastError();
}

cudaError_t launch_pack(const double *xyz, const double *weights, const int32_t *perm,
                        const double *centroid, int64_t n_atoms, int32_t n_pad, int32_t n_frames,
                        float4 *out32, double4 *out64, cudaStream_t st) {
    const int64_t total = static_cast<int64_t>(n_pad) * n_frames;
    const int grid = static_cast<int>((total + 255) / 256);
    pd_pack<<<grid, 256, 0, st>>>(xyz, weights, perm, centroid, n_atoms, n_pad, n_frames, out32,
                                  out64);
    return cudaGetLastError();
}

cudaError_t launch_reduce(const double *slots, const int64_t *lptr, const int64_t *lidx,
                          const PdPairDev *pairs, const double *qv, int32_t n_pairs, int32_t nq,
                          int32_t K, int32_t nv, int32_t n_frames, int64_t slots_per_frame,
                          const double *radius, double qmin, double dq, int residual_form,
                          int add_exact, double *pairsum, cudaStream_t st) {
    const int64_t total = static_cast<int64_t>(n_pairs) * nq * n_frames;
    const int grid = static_cast<int>((total + 127) / 128);
    pd_reduce_pairs<<<grid, 128, 0, st>>>(slots, lptr, lidx, pairs, qv, n_pairs, nq, K, nv,
                                          n_frames, slots_per_frame, radius, qmin, dq,
                                          residual_form, add_exact, pairsum);
    return cudaGetLastError();
}

cudaError_t launch_combine(const double *pairsum, const PdClassDev *cls, const PdPairDev *pairs,
                           int32_t n_cls, int32_t n_pairs, int32_t nq, int32_t nv,
                           int32_t n_frames, const double *ffA, const double *ffC,
                           const double *ffW, int add_diag, double *terms, cudaStream_t st) {
    const int64_t total = static_cast<int64_t>(nq) * n_frames;
    const int grid = static_cast<int>((total + 127) / 128);
    pd_combine_terms<<<grid, 128, 0, st>>>(pairsum, cls, pairs, n_cls, n_pairs, nq, nv, n_frames,
                                           ffA, ffC, ffW, add_diag, terms);
    return cudaGetLastError();
}

cudaError_t launch_frame_mean(const double *terms, const double *fw, int32_t n_frames, int32_t nq,
                              double *out, cudaStream_t st) {
    const int grid = (6 * nq + 127) / 128;
    pd_frame_mean<<<grid, 128, 0, st>>>(terms, fw, n_frames, nq, out);
    return cudaGetLastError();
}

cudaError_t launch_ffma_probe(float *out, int iters, int grid, int block, bool packed,
                              cudaStream_t st) {
    if (packed)
        pd_ffma2_probe<<<grid, block, 0, st>>>(out, iters, 0.999999f, 1e-7f);
    else
        pd_ffma_probe<<<grid, block, 0, st>>>(out, iters, 0.999999f, 1e-7f);
    return cudaGetLastError();
}

}  // namespace pd
