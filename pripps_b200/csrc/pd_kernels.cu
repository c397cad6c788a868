// Device kernels of the Debye backend (sm_100a).
//
// K1 (pd_pairs_fp32): for each tile (i-block × j-range × q-block) every thread
// owns one i atom and walks the j atoms of the range NP at a time. For a pair
// at distance r it needs sin(q_k r) for the K consecutive grid points
// q_k = q_s + k·Δq of the block. With x = Δq·r reduced as x = mπ + x'
// (|x'| <= π/2) the sequence is s_k = σ^k·u_k, σ = (-1)^m, where
// u_k = sin(θ + k x'), θ = q_s r. u_k follows the three-term recurrence
// u_{k+1} = 2cos(x')·u_k − u_{k−1}, evaluated in Reinsch's difference form
//   d_{k+1} = d_k − α·u_k,  u_{k+1} = u_k + d_{k+1},  α = 4 sin²(x'/2),
// which stays accurate for small x' (Reinsch's modification of the Goertzel
// recurrence; errors grow linearly in k). It is reseeded every K steps from
// sin θ and cos θ evaluated in FP32 with a double-float phase and our own
// fitted polynomials (see sincos_poly). One step plus the accumulation
// acc_k += σ^k u_k / r is FFMA + FADD + FADD, all on the FP32 pipes (the
// weight 1/r scales the pair's initial u and d, and the pairs' terms are
// summed before they reach acc_k; with the general step, σ alternating, the
// accumulation is an FFMA with ±1/r). acc_k sums sin(q_k r)/r over the
// thread's pairs; dividing by q_k in FP64 afterwards gives Σ sinc(q_k r).
// With a hydration weight per atom (weighted mode) a second accumulator sums
// the terms times w_j (one more FFMA). Both modes run the even and odd grid
// points of a pair as the two halves of packed FP32x2 instructions.
// Per-sub-chunk sums stay in FP32 registers; they are warp-reduced into FP64
// partial sums in shared memory, merged per atom class at the end of the
// tile into FP64 slots, and every later sum is FP64.
//
// K2 (pd_pairs_fp64): the same tiling with sin(q_k r) from the FP64 sin() for
// every pair and q, and FP64 accumulation throughout.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstdint>
#include <cstdio>

#include "pd_common.h"
#include "pd_kernels.h"
#include "pripps_debye.h"

namespace pd {

__device__ __forceinline__ float warp_sum(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}
// Reduce-scatter of 2·NT values per lane (NT packed pairs, NT a multiple of
// 32) over a warp: at each of five levels a lane keeps one half of its
// pairs, sends the other half to its partner lane^o and adds what the
// partner sends for the half it keeps. Afterwards lane l holds the warp sums
// of the values [l·2NT/32, (l+1)·2NT/32) in v[0 .. NT/32). About 2·NT
// shuffles and NT packed additions instead of the 10·NT shuffles and
// additions of one butterfly per value; the order of the additions is fixed,
// so the sums are deterministic.
#ifndef PD_FLUSH_RS
#define PD_FLUSH_RS 1
#endif
template <int NT>
__device__ __forceinline__ void warp_reduce_scatter(float2 (&v)[NT], int lane) {
    static_assert(NT % 32 == 0, "2·NT values must split evenly over 32 lanes in pairs");
#pragma unroll
    for (int lev = 0; lev < 5; ++lev) {
        const int o = 16 >> lev;
        const int h = (NT >> lev) / 2;  // packed pairs kept
        const bool up = (lane & o) != 0;
#pragma unroll
        for (int k = 0; k < h; ++k) {
            const float2 lo = v[k], hi = v[k + h];
            const float2 keep = up ? hi : lo;
            const float2 send = up ? lo : hi;
            const float2 got = make_float2(__shfl_xor_sync(0xffffffffu, send.x, o),
                                           __shfl_xor_sync(0xffffffffu, send.y, o));
            v[k] = __fadd2_rn(keep, got);
        }
    }
}

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
    return v;
}

// sin and cos on |t| <= π/4 (+ a few ulp) as polynomials in t² whose FP32
// coefficients we fitted (least squares on Chebyshev nodes, each coefficient
// rounded to FP32 before the next ones were refitted): |error| < 8e-11 for sin
// and < 1.1e-10 for cos in exact arithmetic, under the FP32 rounding of the
// result and oscillating in sign. Taylor coefficients rounded to FP32 would
// leave a one-signed error of ~1e-9, which a sum over 10^8 pairs turns into a
// bias.
__device__ __forceinline__ void sincos_poly(float t, float &s, float &c) {
    const float t2 = t * t;
    float ps = 2.789128530e-6f;
    ps = fmaf(ps, t2, -1.984876289e-4f);
    ps = fmaf(ps, t2, 8.333369158e-3f);
    ps = fmaf(ps, t2, -1.666666716e-1f);
    s = fmaf(t * t2, ps, t);
    float pc = 2.443297126e-5f;
    pc = fmaf(pc, t2, -1.388731296e-3f);
    pc = fmaf(pc, t2, 4.166664556e-2f);
    pc = fmaf(pc, t2, -0.5f);
    c = fmaf(t2, pc, 1.0f);
}

// Two-part π/2 for the reduction: C1 has 8 significant bits, so n·C1 and
// a_hi − n·C1 are exact for n < 2^15; C2 = fl32(π/2 − C1). The part of π/2
// below C2 (2.6e-12) scales every phase by the same 1 + 1.6e-12: a q-axis
// stretch far below anything the FP64 oracle comparison can see.
constexpr float kPio2C1 = 1.5703125f;
constexpr float kPio2C2 = 4.838267923333e-4f;
constexpr float kRoundMagic = 12582912.0f;  // 1.5·2^23: fma(a, 2/π, magic) rounds to an integer

// Reduction of an angle a = a_hi + a_lo (unevaluated sum, |a| <~ 1e4):
// a = n·π/2 + t with |t| <= π/4 + ε; returns t and the quadrant n mod 4.
//
// Why the low part: a_hi lies on the FP32 grid of its binade and a_hi − n·C1
// is exact, so rounding a_hi − n·π/2 to FP32 in one step would give the same
// rounding error to every pair of a quadrant and binade — a bias of ~2e-9 per
// sin that survives a sum over 10^7..10^10 pairs. a_lo carries the pair's own
// rounding residue of q·r, so the final rounding of t falls at a pair-
// specific place between grid points and averages out.
__device__ __forceinline__ float reduce_pio2(float a_hi, float a_lo, int &quadrant) {
    const float nm = fmaf(a_hi, 0.636619772f, kRoundMagic);
    const float n = nm - kRoundMagic;  // exact
    quadrant = __float_as_int(nm) & 3;  // the low mantissa bits hold n
    const float t1 = fmaf(-n, kPio2C1, a_hi);
    return t1 + fmaf(-n, kPio2C2, a_lo);
}

// sin and cos of n·π/2 + t from the polynomial values at t.
__device__ __forceinline__ void apply_quadrant(int q, float st, float ct, float &s, float &c) {
    const bool swap = (q & 1) != 0;
    const float a = swap ? ct : st;
    const float b = swap ? st : ct;
    s = (q & 2) ? -a : a;
    c = ((q + 1) & 2) ? -b : b;
}

// Seed of one pair for a q-block. The K values s_k = sin(θ + k x), θ = q_s r,
// x = Δq r, are produced as two interleaved sequences, even k and odd k, each
// a sinusoid in j = k/2 with step y = 2x: s_{2j} = sin(θ + j y) and
// s_{2j+1} = sin(θ + x + j y). With x = m·π/2 + h (|h| <= π/4), y = mπ + 2h
// and both sequences are σ^j·v_j, σ = (−1)^m, where v follows the Reinsch
// recurrence with step 2h: d_{j+1} = d_j − α v_j, v_{j+1} = v_j + d_{j+1},
// α = 4 sin²h. Two independent chains per pair halve the dependency stall of
// the FFMA → FADD step without adding instructions.
//
// GENERAL_STEP = false is the path every pair of a tile takes when
// Δq·(largest distance) <= π/4: then m = 0, h = x, σ = 1 and the step needs
// no reduction.
struct PairSeed {
    float ve, de, vo, dd, na, we, wo;
};

template <bool GENERAL_STEP>
__device__ __forceinline__ PairSeed pair_seed(float4 pi, float4 pj, bool valid, float qs_hi,
                                              float qs_lo, float dq_hi, float dq_lo) {
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
    // One Newton step on 1/r as well (1 − r2·inv² = 1 − r_hi·inv): the weight
    // multiplies every term of the pair, so its error must be unbiased, not
    // just small.
    inv_r = fmaf(hinv, fmaf(-r_hi, inv_r, 1.0f), inv_r);
    // θ = q_s·r as hi + lo (exact product residue plus the cross terms of the
    // two double-float factors).
    const float th_hi = qs_hi * r_hi;
    const float th_lo = fmaf(qs_lo, r_hi, fmaf(qs_hi, r_lo, fmaf(qs_hi, r_hi, -th_hi)));
    int qt;
    const float t = reduce_pio2(th_hi, th_lo, qt);
    float st, ct, s0, c0;
    sincos_poly(t, st, ct);
    apply_quadrant(qt, st, ct, s0, c0);
    const float w = valid ? inv_r : 0.0f;
    PairSeed ps;
    ps.ve = s0;  // v_0 even = sin θ
    if (!GENERAL_STEP) {
        // r_lo matters here: rsqrtf's error need not average to zero, and a
        // step biased by δ moves the phase of the k-th point by k·δ.
        const float x = fmaf(dq_hi, r_hi, fmaf(dq_hi, r_lo, dq_lo * r_hi));
        float sx, cx;
        sincos_poly(x, sx, cx);
        const float sx2 = 2.0f * sx;
        ps.de = sx2 * fmaf(c0, cx, s0 * sx);  // sin θ − sin(θ − 2x) = 2 sin x cos(θ − x)
        ps.vo = fmaf(s0, cx, c0 * sx);        // sin(θ + x)
        ps.dd = sx2 * c0;                     // sin(θ + x) − sin(θ − x) = 2 sin x cos θ
        ps.na = -sx2 * sx2;                   // −α = −4 sin² x
        ps.we = w;
        ps.wo = w;
    } else {
        const float x_hi = dq_hi * r_hi;
        const float x_lo = fmaf(dq_lo, r_hi, fmaf(dq_hi, r_lo, fmaf(dq_hi, r_hi, -x_hi)));
        int qm;
        const float h = reduce_pio2(x_hi, x_lo, qm);
        float sh, ch, sx, cx;
        sincos_poly(h, sh, ch);
        apply_quadrant(qm, sh, ch, sx, cx);
        const float s1 = fmaf(s0, cx, c0 * sx);   // sin(θ + x)
        const float c1 = fmaf(c0, cx, -s0 * sx);  // cos(θ + x)
        const float sh2 = 2.0f * sh;
        ps.de = sh2 * fmaf(c0, ch, s0 * sh);      // sin θ − sin(θ − 2h) = 2 sin h cos(θ − h)
        ps.vo = s1;
        ps.dd = sh2 * fmaf(c1, ch, s1 * sh);      // sin(θ + x) − sin(θ + x − 2h)
        ps.na = -sh2 * sh2;                       // −α = −4 sin² h
        ps.we = w;
        ps.wo = (qm & 1) ? -w : w;                // σ = (−1)^m
    }
    return ps;
}

// The seeds of two pairs at once on packed FP32x2 instructions: every
// operation of pair_seed, in the same order and with the same roundings (a
// negation is a multiplication by -1, exact), with pair 0 in the low and
// pair 1 in the high half. Half the issue slots of two scalar seeds, and the
// packed operations occupy both FP32 sub-pipes together instead of leaving
// one of them idle beside a scalar operation.
#ifndef PD_SEED_X2
#define PD_SEED_X2 1
#endif
__device__ __forceinline__ float2 f2(float a) { return make_float2(a, a); }
__device__ __forceinline__ void sincos_poly_x2(float2 t, float2 &s, float2 &c) {
    const float2 t2 = __fmul2_rn(t, t);
    float2 ps = f2(2.789128530e-6f);
    ps = __ffma2_rn(ps, t2, f2(-1.984876289e-4f));
    ps = __ffma2_rn(ps, t2, f2(8.333369158e-3f));
    ps = __ffma2_rn(ps, t2, f2(-1.666666716e-1f));
    s = __ffma2_rn(__fmul2_rn(t, t2), ps, t);
    float2 pc = f2(2.443297126e-5f);
    pc = __ffma2_rn(pc, t2, f2(-1.388731296e-3f));
    pc = __ffma2_rn(pc, t2, f2(4.166664556e-2f));
    pc = __ffma2_rn(pc, t2, f2(-0.5f));
    c = __ffma2_rn(t2, pc, f2(1.0f));
}
// reduce_pio2 on both halves; the quadrants come back as integers.
__device__ __forceinline__ float2 reduce_pio2_x2(float2 a_hi, float2 a_lo, int &q0, int &q1) {
    const float2 nm = __ffma2_rn(a_hi, f2(0.636619772f), f2(kRoundMagic));
    const float2 n = __fadd2_rn(nm, f2(-kRoundMagic));  // exact
    q0 = __float_as_int(nm.x) & 3;
    q1 = __float_as_int(nm.y) & 3;
    const float2 t1 = __ffma2_rn(n, f2(-kPio2C1), a_hi);
    return __fadd2_rn(t1, __ffma2_rn(n, f2(-kPio2C2), a_lo));
}

template <bool GENERAL_STEP>
__device__ __forceinline__ void pair_seed_x2(float4 pi, float4 pj0, float4 pj1, bool valid0,
                                             bool valid1, float qs_hi, float qs_lo, float dq_hi,
                                             float dq_lo, PairSeed &S0, PairSeed &S1) {
    const float2 M1 = f2(-1.0f);
    const float2 dx = __ffma2_rn(make_float2(pj0.x, pj1.x), M1, f2(pi.x));
    const float2 dy = __ffma2_rn(make_float2(pj0.y, pj1.y), M1, f2(pi.y));
    const float2 dz = __ffma2_rn(make_float2(pj0.z, pj1.z), M1, f2(pi.z));
    float2 r2 = __ffma2_rn(dx, dx, __ffma2_rn(dy, dy, __fmul2_rn(dz, dz)));
    r2 = make_float2(fmaxf(r2.x, 1e-12f), fmaxf(r2.y, 1e-12f));
    float2 inv_r = make_float2(rsqrtf(r2.x), rsqrtf(r2.y));
    const float2 r_hi = __fmul2_rn(r2, inv_r);
    const float2 nr_hi = __fmul2_rn(r_hi, M1);
    const float2 hinv = __fmul2_rn(f2(0.5f), inv_r);
    const float2 r_lo = __fmul2_rn(hinv, __ffma2_rn(nr_hi, r_hi, r2));
    inv_r = __ffma2_rn(hinv, __ffma2_rn(nr_hi, inv_r, f2(1.0f)), inv_r);
    const float2 th_hi = __fmul2_rn(f2(qs_hi), r_hi);
    const float2 th_lo =
        __ffma2_rn(f2(qs_lo), r_hi,
                   __ffma2_rn(f2(qs_hi), r_lo,
                              __ffma2_rn(f2(qs_hi), r_hi, __fmul2_rn(th_hi, M1))));
    int qt0, qt1;
    const float2 t = reduce_pio2_x2(th_hi, th_lo, qt0, qt1);
    float2 st, ct;
    sincos_poly_x2(t, st, ct);
    float s0a, c0a, s0b, c0b;
    apply_quadrant(qt0, st.x, ct.x, s0a, c0a);
    apply_quadrant(qt1, st.y, ct.y, s0b, c0b);
    const float2 s0 = make_float2(s0a, s0b), c0 = make_float2(c0a, c0b);
    const float w0 = valid0 ? inv_r.x : 0.0f, w1 = valid1 ? inv_r.y : 0.0f;
    S0.ve = s0a;
    S1.ve = s0b;
    if (!GENERAL_STEP) {
        const float2 x = __ffma2_rn(f2(dq_hi), r_hi,
                                    __ffma2_rn(f2(dq_hi), r_lo, __fmul2_rn(f2(dq_lo), r_hi)));
        float2 sx, cx;
        sincos_poly_x2(x, sx, cx);
        const float2 sx2 = __fmul2_rn(f2(2.0f), sx);
        const float2 de = __fmul2_rn(sx2, __ffma2_rn(c0, cx, __fmul2_rn(s0, sx)));
        const float2 vo = __ffma2_rn(s0, cx, __fmul2_rn(c0, sx));
        const float2 dd = __fmul2_rn(sx2, c0);
        const float2 na = __fmul2_rn(__fmul2_rn(sx2, M1), sx2);
        S0.de = de.x; S1.de = de.y;
        S0.vo = vo.x; S1.vo = vo.y;
        S0.dd = dd.x; S1.dd = dd.y;
        S0.na = na.x; S1.na = na.y;
        S0.we = S0.wo = w0;
        S1.we = S1.wo = w1;
    } else {
        const float2 x_hi = __fmul2_rn(f2(dq_hi), r_hi);
        const float2 x_lo =
            __ffma2_rn(f2(dq_lo), r_hi,
                       __ffma2_rn(f2(dq_hi), r_lo,
                                  __ffma2_rn(f2(dq_hi), r_hi, __fmul2_rn(x_hi, M1))));
        int qm0, qm1;
        const float2 h = reduce_pio2_x2(x_hi, x_lo, qm0, qm1);
        float2 sh, ch;
        sincos_poly_x2(h, sh, ch);
        float sxa, cxa, sxb, cxb;
        apply_quadrant(qm0, sh.x, ch.x, sxa, cxa);
        apply_quadrant(qm1, sh.y, ch.y, sxb, cxb);
        const float2 sx = make_float2(sxa, sxb), cx = make_float2(cxa, cxb);
        const float2 s1 = __ffma2_rn(s0, cx, __fmul2_rn(c0, sx));
        const float2 c1 = __ffma2_rn(c0, cx, __fmul2_rn(__fmul2_rn(s0, M1), sx));
        const float2 sh2 = __fmul2_rn(f2(2.0f), sh);
        const float2 de = __fmul2_rn(sh2, __ffma2_rn(c0, ch, __fmul2_rn(s0, sh)));
        const float2 dd = __fmul2_rn(sh2, __ffma2_rn(c1, ch, __fmul2_rn(s1, sh)));
        const float2 na = __fmul2_rn(__fmul2_rn(sh2, M1), sh2);
        S0.de = de.x; S1.de = de.y;
        S0.vo = s1.x; S1.vo = s1.y;
        S0.dd = dd.x; S1.dd = dd.y;
        S0.na = na.x; S1.na = na.y;
        S0.we = w0;
        S1.we = w1;
        S0.wo = (qm0 & 1) ? -w0 : w0;
        S1.wo = (qm1 & 1) ? -w1 : w1;
    }
}

// Small-q residual form: where q·(2·radius) < 2 every pair has q·r < 2 and
// the terms sin(q r)/r lie within a factor 0.45..1 of q, so a sequential FP32
// sum of them rounds with a systematic bias. There the kernel accumulates
// sin(q r)/r − q and the reduction adds (pair count)·q back in FP64. Both
// kernels evaluate this predicate on the same FP64 values.
__host__ __device__ __forceinline__ bool residual_q(double q, double radius) {
    return q * (2.0 * radius) < 2.0;
}

// ------------------------------------------------- shared-memory staging (TMA)
// One-dimensional bulk copies (cp.async.bulk, no multicast) of j-atom chunks
// into shared memory, completed on an mbarrier. Every wait is bounded: a
// copy that does not land within its poll limit makes the wait return false;
// the pair kernel then stops issuing copies, waits (bounded) for the ones in
// flight, poisons its results with NaN and sets a status bit the host reads,
// instead of hanging the GPU.
__device__ __forceinline__ uint32_t smem_addr(const void *p) {
    return static_cast<uint32_t>(__cvta_generic_to_shared(p));
}
__device__ __forceinline__ void mbar_init(unsigned long long *bar, uint32_t count) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_addr(bar)), "r"(count)
                 : "memory");
}
__device__ __forceinline__ void mbar_init_fence() {
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
}
// Thread 0 only: `bytes` (a multiple of 16, <= 2^20) from global `src`
// (16-byte aligned) to shared `dst` (16-byte aligned), completing on `bar`.
__device__ __forceinline__ void bulk_copy_to_shared(void *dst, const void *src, uint32_t bytes,
                                                    unsigned long long *bar) {
    // order earlier generic-proxy reads of dst before the async-proxy write
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_addr(bar)),
                 "r"(bytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::
            "r"(smem_addr(dst)),
        "l"(src), "r"(bytes), "r"(smem_addr(bar))
        : "memory");
}
__device__ __forceinline__ bool mbar_wait(unsigned long long *bar, uint32_t phase, int polls) {
    for (int it = 0; it < polls; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
            " selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(smem_addr(bar)), "r"(phase)
            : "memory");
        if (done) return true;
    }
    return false;
}

// ---------------------------------------------------------------- K1 (FP32)
// Seeds of NP consecutive j atoms (clamped reads past the range are masked).
template <int MODE, int NP, bool RESID, bool GENERAL_STEP>
struct SeedGroup {
    PairSeed S[NP];
    float wj[NP];
    float vsum, vwsum;

    // `at` holds the atoms [jbase, j1) (a chunk staged in shared memory).
    __device__ __forceinline__ void make(const float4 *__restrict__ at, int jbase, float4 pi,
                                         int i, bool ivalid, int j, int j1, float qs_hi,
                                         float qs_lo, float dq_hi, float dq_lo) {
        vsum = 0.0f;
        vwsum = 0.0f;
        if constexpr (PD_SEED_X2 && NP % 2 == 0) {
#pragma unroll
            for (int p = 0; p < NP; p += 2) {
                const int ja = j + p, jb = j + p + 1;
                const bool ina = ja < j1, inb = jb < j1;
                const float4 pja = at[(ina ? ja : j1 - 1) - jbase];
                const float4 pjb = at[(inb ? jb : j1 - 1) - jbase];
                const bool va = ivalid && ina && (ja > i), vb = ivalid && inb && (jb > i);
                pair_seed_x2<GENERAL_STEP>(pi, pja, pjb, va, vb, qs_hi, qs_lo, dq_hi, dq_lo,
                                           S[p], S[p + 1]);
                if (MODE == PD_MODE_WEIGHTED) {
                    wj[p] = pja.w;
                    wj[p + 1] = pjb.w;
                }
                if (RESID) {
                    vsum += (va ? 1.0f : 0.0f) + (vb ? 1.0f : 0.0f);
                    if (MODE == PD_MODE_WEIGHTED) {
                        vwsum += va ? pja.w : 0.0f;
                        vwsum += vb ? pjb.w : 0.0f;
                    }
                }
            }
            return;
        }
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const int jj = j + p;
            const bool inr = jj < j1;
            const float4 pj = at[(inr ? jj : j1 - 1) - jbase];
            const bool valid = ivalid && inr && (jj > i);
            S[p] = pair_seed<GENERAL_STEP>(pi, pj, valid, qs_hi, qs_lo, dq_hi, dq_lo);
            if (MODE == PD_MODE_WEIGHTED) wj[p] = pj.w;
            if (RESID) {
                vsum += valid ? 1.0f : 0.0f;
                if (MODE == PD_MODE_WEIGHTED) vwsum += valid ? pj.w : 0.0f;
            }
        }
    }
};

// NP pairs per thread per pass, two chains each: 2·NP independent
// recurrences. The seeds of the next pass are computed in the same straight-
// line block as the K steps of the current one, so their long dependency
// chains (sqrt, reductions, polynomials) overlap the recurrence instead of
// stalling the warp between passes.
template <int K, int MODE, int NP, bool RESID, bool GENERAL_STEP>
__device__ __forceinline__ void pairs_range(const float4 *__restrict__ at, int jbase, float4 pi,
                                            int i, bool ivalid, int j0, int j1, float qs_hi,
                                            float qs_lo, float dq_hi, float dq_lo,
                                            const float *__restrict__ s_qres,
                                            float (&acc)[(MODE == PD_MODE_WEIGHTED) ? 2 : 1][K]) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    static_assert(K % 4 == 0, "K must be a multiple of 4");
    if (j0 >= j1) return;
    SeedGroup<MODE, NP, RESID, GENERAL_STEP> cur;
    cur.make(at, jbase, pi, i, ivalid, j0, j1, qs_hi, qs_lo, dq_hi, dq_lo);
    for (int j = j0; j < j1; j += NP) {
        SeedGroup<MODE, NP, RESID, GENERAL_STEP> nxt;  // unused after the last pass
        nxt.make(at, jbase, pi, i, ivalid, j + NP, j1, qs_hi, qs_lo, dq_hi, dq_lo);
        float we_w[NP], wo_w[NP];
        if (MODE == PD_MODE_WEIGHTED) {
#pragma unroll
            for (int p = 0; p < NP; ++p) {
                we_w[p] = cur.S[p].we * cur.wj[p];
                wo_w[p] = cur.S[p].wo * cur.wj[p];
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
                    acc[0][kk] = fmaf(-cur.vsum, qk, acc[0][kk]);
                    if (MODE == PD_MODE_WEIGHTED)
                        acc[NACC - 1][kk] = fmaf(-cur.vwsum, qk, acc[NACC - 1][kk]);
                }
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    const float w = odd_j ? cur.S[p].wo : cur.S[p].we;
                    float &v = odd_chain ? cur.S[p].vo : cur.S[p].ve;
                    float &d = odd_chain ? cur.S[p].dd : cur.S[p].de;
                    acc[0][kk] = fmaf(w, v, acc[0][kk]);
                    if (MODE == PD_MODE_WEIGHTED)
                        acc[NACC - 1][kk] = fmaf(odd_j ? wo_w[p] : we_w[p], v, acc[NACC - 1][kk]);
                    d = fmaf(cur.S[p].na, v, d);
                    v += d;
                }
            }
        }
        cur = nxt;
    }
}

// Class mode on packed FP32x2 instructions (fma.rn.f32x2 / add.rn.f32x2,
// sm_100): the even and odd chain of a pair sit in the two halves of one
// register pair, V = (v_even, v_odd), D = (d_even, d_odd), and so do the
// accumulators of grid points 2t and 2t+1: one step t advances both chains
// and both accumulators with FFMA2 + FADD2 + FFMA2. The FP32 pipe does the
// same lane work as with scalar instructions, but a warp needs half the issue
// slots for it, which leaves the issue port to the seeds and lets the FMA
// pipe, not instruction issue, bound the kernel. Each half rounds exactly as
// the scalar fmaf/add would.
//
// A block runs only its first `nchunk` chunks of 16 grid points: the last
// q-block of a grid whose length is not a multiple of K skips the steps past
// the grid end instead of computing and discarding them. (One uniform branch
// per chunk in a single code path measured faster on B200 than a separate
// copy of the loop for tail blocks, which raised register spills.)
#ifndef PD_SCALED_V
#define PD_SCALED_V 1
#endif
// Where the seeds of a pass are computed. Computing each pass's seeds
// before its steps holds no next-pass seeds through the steps: fewer
// registers, so more resident CTAs or fewer spills, and the extra warps per
// scheduler hide the seeds' dependency chains. Measured on B200 (pair-kernel
// time): K = 128 with four pairs per thread fits 168 registers and three CTAs
// per SM instead of 255 and two, 546.7 ms against 556.0 ms on the
// 100,000-atom solve (558.5 ms with the seeds at the top but two CTAs); K = 64
// with four pairs loses its spills at four CTAs, 0.216 against 0.232 ms on
// 3,000 atoms at nq 300; the weighted mode's K = 64 fits three CTAs instead of
// two, 814 against 842 ms on the 100,000-atom solve with per-atom weights.
// The other shapes compute the next pass's seeds while the current pass
// steps (K = 128 with two pairs: 3.117 against 3.121 ms on 10,000 atoms).
#ifndef PD_SEED_TOP
#define PD_SEED_TOP 1
#endif
template <int K, int NP>
constexpr bool seeds_at_top() {
    return PD_SEED_TOP && (K == 64 || (K == 128 && NP == 4));
}
template <int K, int NP>
constexpr bool seeds_at_top_w() {
    return PD_SEED_TOP && K == 64;
}
// Instruction order within a step: 0 = d-steps, accumulations, v-steps;
// 1 = d-steps, then per pair its accumulation and v-step; 2 (with
// PD_SCALED_V, two or four pairs) = the pairs' scaled terms summed, then
// added to the accumulator (measured 1.5 % faster than 0 on the 100,000-atom
// solve: the accumulator's dependency chain is one add per step instead of
// one per pair).
#ifndef PD_STEP_ORDER
#define PD_STEP_ORDER 2
#endif
// Steps between two checks for the end of the grid (a chunk of 2·PD_CHUNK_T
// grid points).
#ifndef PD_CHUNK_T
#define PD_CHUNK_T 8
#endif
template <int K, int NP, bool RESID, bool GENERAL_STEP>
__device__ __forceinline__ void pairs_range_x2(const float4 *__restrict__ at, int jbase, float4 pi,
                                               int i, bool ivalid, int j0, int j1, float qs_hi,
                                               float qs_lo, float dq_hi, float dq_lo,
                                               const float2 *__restrict__ s_qres2,
                                               float2 (&acc)[K / 2], int nchunk,
                                               int rchunk = K / 16) {
    static_assert(K % 16 == 0, "K must be a multiple of 16");
    if (j0 >= j1) return;
    SeedGroup<PD_MODE_CLASS, NP, RESID, GENERAL_STEP> cur;
    constexpr bool TOP = seeds_at_top<K, NP>();
    if (!TOP) cur.make(at, jbase, pi, i, ivalid, j0, j1, qs_hi, qs_lo, dq_hi, dq_lo);
    for (int j = j0; j < j1; j += NP) {
        if (TOP) cur.make(at, jbase, pi, i, ivalid, j, j1, qs_hi, qs_lo, dq_hi, dq_lo);
        // SCALED: without the general step every term of a pair has the
        // weight w = 1/r, which the linear recurrence can carry in v and d
        // themselves; the accumulation is then a plain add.
        constexpr bool SCALED = PD_SCALED_V && !GENERAL_STEP;
        float2 V[NP], D[NP], NA[NP], WE[NP], WO[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            if (SCALED) {
                const float w = cur.S[p].we;
                V[p] = make_float2(w * cur.S[p].ve, w * cur.S[p].vo);
                D[p] = make_float2(w * cur.S[p].de, w * cur.S[p].dd);
            } else {
                V[p] = make_float2(cur.S[p].ve, cur.S[p].vo);
                D[p] = make_float2(cur.S[p].de, cur.S[p].dd);
                WE[p] = make_float2(cur.S[p].we, cur.S[p].we);
                WO[p] = GENERAL_STEP ? make_float2(cur.S[p].wo, cur.S[p].wo) : WE[p];
            }
            NA[p] = make_float2(cur.S[p].na, cur.S[p].na);
        }
        const float2 mvs = make_float2(-cur.vsum, -cur.vsum);
        // the next pass's seeds (unused after the last pass), computed in
        // place while the steps below run on this pass's copies
        if (!TOP) cur.make(at, jbase, pi, i, ivalid, j + NP, j1, qs_hi, qs_lo, dq_hi, dq_lo);
        int qoff = 0;  // opaque zero: keeps the K/2 q loads in the loop
        if (RESID) asm volatile("mov.b32 %0, %0;" : "+r"(qoff));
#pragma unroll
        for (int t = 0; t < K / 2; ++t) {
            if ((t % PD_CHUNK_T) == 0 && t / PD_CHUNK_T >= nchunk) break;
            // the residual points are a prefix of the block: only its first
            // rchunk 16-point chunks subtract q
            if (RESID && (t / 8) < rchunk) acc[t] = __ffma2_rn(mvs, s_qres2[t + qoff], acc[t]);
            // d-steps of all pairs, then the accumulations, then the
            // v-steps: every instruction's operands are a group old
            // (measured 0.5 % faster than the per-pair order).
#pragma unroll
            for (int p = 0; p < NP; ++p) D[p] = __ffma2_rn(NA[p], V[p], D[p]);
            if constexpr (SCALED && PD_STEP_ORDER == 2 && (NP == 2 || NP == 4)) {
                // the pairs' scaled terms added among themselves first, then
                // to the accumulator: one dependent add per step on acc[t]
                float2 sum = __fadd2_rn(V[0], V[1]);
                if constexpr (NP == 4) sum = __fadd2_rn(sum, __fadd2_rn(V[2], V[3]));
#pragma unroll
                for (int p = 0; p < NP; ++p) V[p] = __fadd2_rn(V[p], D[p]);
                acc[t] = __fadd2_rn(acc[t], sum);
            } else if constexpr (PD_STEP_ORDER == 0 || PD_STEP_ORDER == 2) {
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    if constexpr (SCALED)
                        acc[t] = __fadd2_rn(V[p], acc[t]);
                    else
                        acc[t] = __ffma2_rn((t & 1) ? WO[p] : WE[p], V[p], acc[t]);
                }
#pragma unroll
                for (int p = 0; p < NP; ++p) V[p] = __fadd2_rn(V[p], D[p]);
            } else {
                // each pair's accumulation, then its v-step
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    if constexpr (SCALED)
                        acc[t] = __fadd2_rn(V[p], acc[t]);
                    else
                        acc[t] = __ffma2_rn((t & 1) ? WO[p] : WE[p], V[p], acc[t]);
                    V[p] = __fadd2_rn(V[p], D[p]);
                }
            }
        }
    }
}

// Weighted mode on packed FP32x2 instructions: the same chains as
// pairs_range_x2 with two accumulators per grid point, Σ w d/r-terms (acc0)
// and Σ w_j·terms (acc1). Without the general step the weight 1/r rides in
// v and d (SCALED), acc0 takes the pairs' terms summed among themselves and
// acc1 one FFMA2 per pair with w_j: four FP32 lane slots per pair·q (d-step,
// v-step, the two accumulations), on half the issue slots of the scalar
// form.
#ifndef PD_WEIGHTED_X2
#define PD_WEIGHTED_X2 1
#endif
template <int K, int NP, bool RESID, bool GENERAL_STEP>
__device__ __forceinline__ void pairs_range_x2w(const float4 *__restrict__ at, int jbase,
                                                float4 pi, int i, bool ivalid, int j0, int j1,
                                                float qs_hi, float qs_lo, float dq_hi,
                                                float dq_lo, const float2 *__restrict__ s_qres2,
                                                float2 (&acc0)[K / 2], float2 (&acc1)[K / 2],
                                                int nchunk, int rchunk = K / 16) {
    static_assert(K % 16 == 0, "K must be a multiple of 16");
    if (j0 >= j1) return;
    constexpr bool SCALED = PD_SCALED_V && !GENERAL_STEP;
    SeedGroup<PD_MODE_WEIGHTED, NP, RESID, GENERAL_STEP> cur;
    constexpr bool TOP = seeds_at_top_w<K, NP>();
    if (!TOP) cur.make(at, jbase, pi, i, ivalid, j0, j1, qs_hi, qs_lo, dq_hi, dq_lo);
    for (int j = j0; j < j1; j += NP) {
        if (TOP) cur.make(at, jbase, pi, i, ivalid, j, j1, qs_hi, qs_lo, dq_hi, dq_lo);
        float2 V[NP], D[NP], NA[NP], WJ[NP], WE[NP], WO[NP], WJE[NP], WJO[NP];
#pragma unroll
        for (int p = 0; p < NP; ++p) {
            const float w = cur.S[p].we;
            if (SCALED) {
                V[p] = make_float2(w * cur.S[p].ve, w * cur.S[p].vo);
                D[p] = make_float2(w * cur.S[p].de, w * cur.S[p].dd);
                WJ[p] = make_float2(cur.wj[p], cur.wj[p]);
            } else {
                V[p] = make_float2(cur.S[p].ve, cur.S[p].vo);
                D[p] = make_float2(cur.S[p].de, cur.S[p].dd);
                const float wo = cur.S[p].wo;
                WE[p] = make_float2(w, w);
                WO[p] = make_float2(wo, wo);
                WJE[p] = make_float2(w * cur.wj[p], w * cur.wj[p]);
                WJO[p] = make_float2(wo * cur.wj[p], wo * cur.wj[p]);
            }
            NA[p] = make_float2(cur.S[p].na, cur.S[p].na);
        }
        const float2 mvs = make_float2(-cur.vsum, -cur.vsum);
        const float2 mvws = make_float2(-cur.vwsum, -cur.vwsum);
        if (!TOP) cur.make(at, jbase, pi, i, ivalid, j + NP, j1, qs_hi, qs_lo, dq_hi, dq_lo);
        int qoff = 0;  // opaque zero: keeps the K/2 q loads in the loop
        if (RESID) asm volatile("mov.b32 %0, %0;" : "+r"(qoff));
#pragma unroll
        for (int t = 0; t < K / 2; ++t) {
            if ((t % PD_CHUNK_T) == 0 && t / PD_CHUNK_T >= nchunk) break;
            if (RESID && (t / 8) < rchunk) {
                const float2 q2 = s_qres2[t + qoff];
                acc0[t] = __ffma2_rn(mvs, q2, acc0[t]);
                acc1[t] = __ffma2_rn(mvws, q2, acc1[t]);
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) D[p] = __ffma2_rn(NA[p], V[p], D[p]);
            if constexpr (SCALED) {
                float2 sum = V[0];
#pragma unroll
                for (int p = 1; p < NP; ++p) sum = __fadd2_rn(sum, V[p]);
                float2 a1 = acc1[t];
#pragma unroll
                for (int p = 0; p < NP; ++p) a1 = __ffma2_rn(WJ[p], V[p], a1);
                acc1[t] = a1;
                acc0[t] = __fadd2_rn(acc0[t], sum);
            } else {
#pragma unroll
                for (int p = 0; p < NP; ++p) {
                    acc0[t] = __ffma2_rn((t & 1) ? WO[p] : WE[p], V[p], acc0[t]);
                    acc1[t] = __ffma2_rn((t & 1) ? WJO[p] : WJE[p], V[p], acc1[t]);
                }
            }
#pragma unroll
            for (int p = 0; p < NP; ++p) V[p] = __fadd2_rn(V[p], D[p]);
        }
    }
}

// Pairs a thread adds in FP32 before the warp's partial sums go into its
// FP64 slot. A j range of a tile is walked in sub-chunks of this length with
// fresh FP32 accumulators: FP32 running sums over thousands of terms lose
// ε·|running sum| per addition (and over same-sign terms that loss has a
// sign), which on sums of 10^9 pairs that cancel to 10^-5 of their scale
// shows up in the result; short FP32 runs keep it far below the profile.
#ifndef PD_JFLUSH
#define PD_JFLUSH 512
#endif
// j atoms per bulk copy into shared memory (two buffers of PD_JSTAGE float4,
// 64 KB of dynamic shared memory per CTA); a multiple of PD_JFLUSH. One CTA
// barrier per stage releases the buffer for the next copy.
#ifndef PD_JSTAGE_ATOMS
#define PD_JSTAGE_ATOMS 2048
#endif
constexpr int PD_JSTAGE = PD_JSTAGE_ATOMS;
static_assert(PD_JSTAGE % PD_JFLUSH == 0, "stage must hold whole sub-chunks");
constexpr size_t PD_FP32_DYN_SMEM = 2 * PD_JSTAGE * sizeof(float4);

// Resident CTAs per SM each FP32 shape is compiled for (register budget
// 65536 / (128 · blocks) per thread).
constexpr int fp32_min_blocks(int K, int MODE, int NP) {
    return MODE == PD_MODE_CLASS
               ? (K <= 64 ? 4 : (K <= 128 && (NP <= 2 || (PD_SEED_TOP && K == 128 && NP == 4)) ? 3 : 2))
               : (K <= 32 ? 4 : (PD_SEED_TOP && K == 64 ? 3 : 2));
}

// Polls of a bulk-copy wait before it gives up: the normal limit, and the
// short one of the test hook (PD_REQF_TEST_EXPIRE), whose copy is never
// issued.
constexpr int PD_WAIT_POLLS = 1 << 22;
constexpr int PD_TEST_WAIT_POLLS = 1 << 10;

// Weighted-mode flush of one accumulator array: the warp sums of acc and of
// w_i·acc, reduce-scattered (lane l ends with grid points
// [l·K/32, (l+1)·K/32)) and added to part[k] and part[K + k].
template <int K>
__device__ __forceinline__ void flush_weighted_rs(float2 (&acc)[K / 2], float wi,
                                                  double *__restrict__ part, int lane,
                                                  bool first) {
    const float2 wi2 = make_float2(wi, wi);
    float2 tw[K / 2];
#pragma unroll
    for (int t = 0; t < K / 2; ++t) tw[t] = __fmul2_rn(wi2, acc[t]);
    warp_reduce_scatter<K / 2>(acc, lane);
    warp_reduce_scatter<K / 2>(tw, lane);
#pragma unroll
    for (int m = 0; m < K / 32; ++m) {
        const int k = lane * (K / 32) + m;
        const float s = (m & 1) ? acc[m >> 1].y : acc[m >> 1].x;
        const float sw = (m & 1) ? tw[m >> 1].y : tw[m >> 1].x;
        part[k] = (first ? 0.0 : part[k]) + static_cast<double>(s);
        part[K + k] = (first ? 0.0 : part[K + k]) + static_cast<double>(sw);
    }
}

// End of a tile: the warps' FP64 partial sums (part[w·nvk + e], e < nvk) of
// one class are added in warp order and written to that class's slot; a CTA
// whose copy wait expired writes NaN instead, and an empty tile zeros.
__device__ __forceinline__ void merge_tile_slots(const double *__restrict__ part, int nvk,
                                                 int64_t slot_word, double *__restrict__ slots,
                                                 bool dead, bool empty) {
    const int64_t slot0 = slot_word & PD_SLOT_MASK;
    const int smap = static_cast<int>(slot_word >> PD_SLOT_MAP_SHIFT) & 0xff;
    const double nan = __longlong_as_double(0x7ff8000000000000ll);
    for (int e = threadIdx.x; e < nvk; e += blockDim.x) {
        double a[PD_WARPS];
        int used = 0;
#pragma unroll
        for (int w = 0; w < PD_WARPS; ++w) {
            const int s = (smap >> (2 * w)) & 3;
            const double v = part[w * nvk + e];
            a[s] = (used & (1 << s)) ? a[s] + v : v;
            used |= 1 << s;
        }
#pragma unroll
        for (int s = 0; s < PD_WARPS; ++s)
            if (used & (1 << s))
                slots[(slot0 + s) * nvk + e] = dead ? nan : (empty ? 0.0 : a[s]);
    }
}

template <int K, int MODE, int NP>
__global__ void __launch_bounds__(PD_THREADS, fp32_min_blocks(K, MODE, NP))
    pd_pairs_fp32(const PdJob *__restrict__ jobs, const int *__restrict__ n_jobs_ptr,
                  const PdReqDev *__restrict__ reqs, int *__restrict__ counter) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    constexpr int NV = (MODE == PD_MODE_WEIGHTED) ? 4 : 1;  // FP64 values per q in a slot
    constexpr bool PACKED = (MODE == PD_MODE_CLASS);
    constexpr bool PACKED_W =
        (MODE == PD_MODE_WEIGHTED) && PD_WEIGHTED_X2 && (K / 2) % 32 == 0 && NP % 2 == 0;
    __shared__ int s_job;
    __shared__ __align__(16) float s_qres[K];
    // per-warp FP64 partial sums of the current tile, [warp][NV][K]
    __shared__ double s_part[PD_WARPS * NV * K];
    // j atoms of the current and the next stage, staged by bulk copies
    // (PD_FP32_DYN_SMEM bytes of dynamic shared memory)
    extern __shared__ __align__(128) float4 pd_dyn_atoms[];
    float4 *s_atoms[2] = {pd_dyn_atoms, pd_dyn_atoms + PD_JSTAGE};
    __shared__ __align__(8) unsigned long long s_bar[2];
    // Once a copy wait of this CTA expires the CTA is "dead" for the rest of
    // the launch: it issues no more copies, computes nothing, writes NaN to
    // the slots of every tile it still takes and flags each tile's request
    // in its status word. This state lives in shared memory, not registers,
    // so that it adds nothing to the register pressure of the steps.
    __shared__ int s_dead, s_polls, s_skip;
    __shared__ uint32_t s_inflight, s_par;  // thread 0: copies in flight, their parities
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int n_jobs = *n_jobs_ptr;
    if (threadIdx.x == 0) {
        mbar_init(&s_bar[0], 1);
        mbar_init(&s_bar[1], 1);
        mbar_init_fence();
        s_dead = 0;
    }
    __syncthreads();
    uint32_t phase = 0;  // bit b: parity of buffer b's next completion
    double *part = s_part + warp * NV * K;
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
        int nres = 0;  // leading grid points of the block in the residual form
        if (resid) {
            for (int base = 0; base < K; base += PD_THREADS) {
                const int t = base + threadIdx.x;
                bool on = false;
                if (t < K) {
                    const int kq = kq0 + t;
                    on = kq < rq.nq && residual_q(rq.qv[kq], radius);
                    s_qres[t] = on ? static_cast<float>(rq.qv[kq]) : 0.0f;
                }
                nres += __syncthreads_count(on);
            }
        }
        const int rchunk = (nres + 15) >> 4;
        if (threadIdx.x == 0) {
            // test hook: the CTA that takes the launch's first tile waits for
            // a copy that is never issued, briefly, so that its wait expires
            // with no copy in flight
            s_skip = (rq.flags & PD_REQF_TEST_EXPIRE) != 0 && jid == 0;
            s_polls = s_skip ? PD_TEST_WAIT_POLLS : PD_WAIT_POLLS;
            s_inflight = 0;
            s_par = 0;
        }
        __syncthreads();  // s_qres and the tile state ready; every thread has read s_job
        const float4 *__restrict__ at = rq.atoms32 + static_cast<size_t>(jb.frame) * rq.n_pad;
        const int i = jb.i0 + threadIdx.x;
        const float4 pi = at[i];
        const bool ivalid = lane < rq.gvalid[(jb.i0 >> 5) + warp];
        const double qs = rq.qmin + static_cast<double>(kq0) * rq.dq;
        const float qs_hi = static_cast<float>(qs);
        const float qs_lo = static_cast<float>(qs - static_cast<double>(qs_hi));
        const float dq_hi = static_cast<float>(rq.dq);
        const float dq_lo = static_cast<float>(rq.dq - static_cast<double>(dq_hi));
        // Every pair distance is at most 2·radius (positions are centred):
        // below π/4 for the step angle Δq·r the seeds skip its reduction.
        const bool general_step = rq.dq * (2.0 * radius) > 0.78;
        const int nstage = s_dead ? 0 : (jb.j1 - jb.j0 + PD_JSTAGE - 1) / PD_JSTAGE;
        if (threadIdx.x == 0 && nstage > 0 && !s_skip) {
            bulk_copy_to_shared(s_atoms[0], at + jb.j0,
                                static_cast<uint32_t>(min(jb.j1 - jb.j0, PD_JSTAGE)) * 16,
                                &s_bar[0]);
            s_inflight = 1u;
            s_par = phase & 1u;
        }
        for (int stg = 0; stg < nstage; ++stg) {
            const int jss = jb.j0 + stg * PD_JSTAGE;
            const int jse = min(jb.j1, jss + PD_JSTAGE);
            if (threadIdx.x == 0 && stg + 1 < nstage) {  // its buffer was released at stg - 1
                const int nb = (stg + 1) & 1;
                bulk_copy_to_shared(s_atoms[nb], at + jse,
                                    static_cast<uint32_t>(min(jb.j1 - jse, PD_JSTAGE)) * 16,
                                    &s_bar[nb]);
                s_inflight |= 1u << nb;
                s_par = (s_par & ~(1u << nb)) | (phase & (1u << nb));
            }
            const int b = stg & 1;
            const bool landed = mbar_wait(&s_bar[b], (phase >> b) & 1u, s_polls);
            phase ^= 1u << b;
            if (threadIdx.x == 0 && landed) s_inflight &= ~(1u << b);
            // A chunk that did not land is computed anyway (its shared memory
            // holds stale atoms, harmless to read) and the tile is poisoned
            // below: no branch around the steps.
            const float4 *chunk = s_atoms[b];
            {
                for (int js = jss; js < jse; js += PD_JFLUSH) {
                    const int je = min(jse, js + PD_JFLUSH);
                    const bool first = js == jb.j0;
                    if constexpr (PACKED) {
                        const float2 *q2 = reinterpret_cast<const float2 *>(s_qres);
                        // 16-point chunks of this block that lie on the grid.
                        // The small-q residual blocks (the first of a grid)
                        // run whole: a tail check there costs the register
                        // spills it saves in steps.
                        const int nchunk =
                            (min(K, rq.nq - kq0) + 2 * PD_CHUNK_T - 1) / (2 * PD_CHUNK_T);
                        float2 acc[K / 2];
#pragma unroll
                        for (int t = 0; t < K / 2; ++t) acc[t] = make_float2(0.0f, 0.0f);
                        if (resid) {
                            if (general_step)
                                pairs_range_x2<K, NP, true, true>(chunk, jss, pi, i, ivalid, js, je,
                                                                  qs_hi, qs_lo, dq_hi, dq_lo, q2,
                                                                  acc, K / (2 * PD_CHUNK_T), rchunk);
                            else
                                pairs_range_x2<K, NP, true, false>(chunk, jss, pi, i, ivalid, js,
                                                                   je, qs_hi, qs_lo, dq_hi, dq_lo,
                                                                   q2, acc, K / (2 * PD_CHUNK_T),
                                                                   rchunk);
                        } else {
                            if (general_step)
                                pairs_range_x2<K, NP, false, true>(chunk, jss, pi, i, ivalid, js,
                                                                   je, qs_hi, qs_lo, dq_hi, dq_lo,
                                                                   q2, acc, nchunk);
                            else
                                pairs_range_x2<K, NP, false, false>(chunk, jss, pi, i, ivalid, js,
                                                                    je, qs_hi, qs_lo, dq_hi, dq_lo,
                                                                    q2, acc, nchunk);
                        }
                        // Warp-reduce and add into this warp's partial sums,
                        // in sub-chunk order (one warp owns them).
                        if constexpr (PD_FLUSH_RS && (K / 2) % 32 == 0) {
                        // reduce-scatter: lane l ends with the warp sums of
                        // grid points [l·K/32, (l+1)·K/32)
                        warp_reduce_scatter<K / 2>(acc, lane);
#pragma unroll
                        for (int m = 0; m < K / 32; ++m) {
                            double &d = part[lane * (K / 32) + m];
                            const float sum = (m & 1) ? acc[m >> 1].y : acc[m >> 1].x;
                            d = (first ? 0.0 : d) + static_cast<double>(sum);
                        }
                        } else {
#pragma unroll
                        for (int t = 0; t < K / 2; ++t) {
                            const float v0 = warp_sum(acc[t].x);
                            const float v1 = warp_sum(acc[t].y);
                            if (lane == ((2 * t) & 31))
                                part[2 * t] = (first ? 0.0 : part[2 * t]) + static_cast<double>(v0);
                            if (lane == ((2 * t + 1) & 31))
                                part[2 * t + 1] =
                                    (first ? 0.0 : part[2 * t + 1]) + static_cast<double>(v1);
                        }
                        }
                    } else if constexpr (PACKED_W) {
                        const float2 *q2 = reinterpret_cast<const float2 *>(s_qres);
                        const int nchunk =
                            (min(K, rq.nq - kq0) + 2 * PD_CHUNK_T - 1) / (2 * PD_CHUNK_T);
                        float2 acc0[K / 2], acc1[K / 2];
#pragma unroll
                        for (int t = 0; t < K / 2; ++t) {
                            acc0[t] = make_float2(0.0f, 0.0f);
                            acc1[t] = make_float2(0.0f, 0.0f);
                        }
                        if (resid) {
                            if (general_step)
                                pairs_range_x2w<K, NP, true, true>(
                                    chunk, jss, pi, i, ivalid, js, je, qs_hi, qs_lo, dq_hi, dq_lo,
                                    q2, acc0, acc1, K / (2 * PD_CHUNK_T), rchunk);
                            else
                                pairs_range_x2w<K, NP, true, false>(
                                    chunk, jss, pi, i, ivalid, js, je, qs_hi, qs_lo, dq_hi, dq_lo,
                                    q2, acc0, acc1, K / (2 * PD_CHUNK_T), rchunk);
                        } else {
                            if (general_step)
                                pairs_range_x2w<K, NP, false, true>(chunk, jss, pi, i, ivalid, js,
                                                                    je, qs_hi, qs_lo, dq_hi, dq_lo,
                                                                    q2, acc0, acc1, nchunk);
                            else
                                pairs_range_x2w<K, NP, false, false>(
                                    chunk, jss, pi, i, ivalid, js, je, qs_hi, qs_lo, dq_hi, dq_lo,
                                    q2, acc0, acc1, nchunk);
                        }
                        // the four warp sums of each grid point: Σ acc0,
                        // Σ w_i·acc0, Σ acc1, Σ w_i·acc1
                        const float wi = ivalid ? pi.w : 0.0f;
                        flush_weighted_rs<K>(acc0, wi, part, lane, first);
                        flush_weighted_rs<K>(acc1, wi, part + 2 * K, lane, first);
                    } else {
                        const float wi = ivalid ? pi.w : 0.0f;
                        float acc[NACC][K];
#pragma unroll
                        for (int a = 0; a < NACC; ++a)
#pragma unroll
                            for (int k = 0; k < K; ++k) acc[a][k] = 0.0f;
                        if (resid) {
                            if (general_step)
                                pairs_range<K, MODE, NP, true, true>(chunk, jss, pi, i, ivalid, js,
                                                                     je, qs_hi, qs_lo, dq_hi,
                                                                     dq_lo, s_qres, acc);
                            else
                                pairs_range<K, MODE, NP, true, false>(chunk, jss, pi, i, ivalid, js,
                                                                      je, qs_hi, qs_lo, dq_hi,
                                                                      dq_lo, s_qres, acc);
                        } else {
                            if (general_step)
                                pairs_range<K, MODE, NP, false, true>(chunk, jss, pi, i, ivalid, js,
                                                                      je, qs_hi, qs_lo, dq_hi,
                                                                      dq_lo, s_qres, acc);
                            else
                                pairs_range<K, MODE, NP, false, false>(chunk, jss, pi, i, ivalid,
                                                                       js, je, qs_hi, qs_lo, dq_hi,
                                                                       dq_lo, s_qres, acc);
                        }
                        // Warp-reduce into this warp's [4][K] partial sums.
#pragma unroll
                        for (int k = 0; k < K; ++k) {
                            const float t0 = warp_sum(acc[0][k]);
                            const float ti = warp_sum(wi * acc[0][k]);
                            const float tj = warp_sum(acc[NACC - 1][k]);
                            const float tij = warp_sum(wi * acc[NACC - 1][k]);
                            if (lane == (k & 31)) {
                                part[k] = (first ? 0.0 : part[k]) + static_cast<double>(t0);
                                part[K + k] = (first ? 0.0 : part[K + k]) + static_cast<double>(ti);
                                part[2 * K + k] =
                                    (first ? 0.0 : part[2 * K + k]) + static_cast<double>(tj);
                                part[3 * K + k] =
                                    (first ? 0.0 : part[3 * K + k]) + static_cast<double>(tij);
                            }
                        }
                    }
                }
            }
            // every read of buffer b done before it is refilled; an expired
            // wait in any thread makes the whole CTA dead
            if (__syncthreads_or(!landed)) {
                if (threadIdx.x == 0) s_dead = 1;
                break;
            }
        }
        __syncthreads();  // every warp's partial sums are complete; s_dead final
        {
            // The job and request fields of the epilogue are loaded again here
            // (an opaque index keeps the compiler from holding them in
            // registers through the steps).
            int jid2 = s_job;
            asm volatile("" : "+r"(jid2));
            const int64_t slot_word = jobs[jid2].slot;
            const PdReqDev *rq2 = reqs + jobs[jid2].req;
            const bool dead = s_dead != 0;
            if (dead && threadIdx.x == 0) {
                // no copy of this CTA may land in shared memory after it
                // moves on: wait (bounded) for the ones still in flight
                for (int b = 0; b < 2; ++b)
                    if (s_inflight & (1u << b))
                        mbar_wait(&s_bar[b], (s_par >> b) & 1u, PD_WAIT_POLLS);
                atomicOr(rq2->status, PD_DEV_WAIT_EXPIRED);
            }
            merge_tile_slots(s_part, NV * K, slot_word, rq2->slots, dead,
                             jobs[jid2].j1 <= jobs[jid2].j0 && !dead);
        }
        __syncthreads();  // s_qres, s_part, s_job and the tile state are rewritten next
    }
}

// ---------------------------------------------------------------- K2 (FP64)
template <int K, int MODE>
__global__ void __launch_bounds__(PD_THREADS) pd_pairs_fp64(const PdJob *__restrict__ jobs,
                                                            const int *__restrict__ n_jobs_ptr,
                                                            const PdReqDev *__restrict__ reqs,
                                                            int *__restrict__ counter) {
    constexpr int NACC = (MODE == PD_MODE_WEIGHTED) ? 2 : 1;
    constexpr int NV = (MODE == PD_MODE_WEIGHTED) ? 4 : 1;
    __shared__ int s_job;
    __shared__ double s_q[K];
    __shared__ double s_part[PD_WARPS * NV * K];
    const int lane = threadIdx.x & 31;
    const int warp = threadIdx.x >> 5;
    const int n_jobs = *n_jobs_ptr;
    double *part = s_part + warp * NV * K;
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

        const double wi = ivalid ? pi.w : 0.0;
#pragma unroll
        for (int k = 0; k < K; ++k) {
            const double t0 = warp_sum(acc[0][k]);
            if (MODE == PD_MODE_CLASS) {
                if (lane == (k & 31)) part[k] = t0;
            } else {
                const double ti = warp_sum(wi * acc[0][k]);
                const double tj = warp_sum(acc[NACC - 1][k]);
                const double tij = warp_sum(wi * acc[NACC - 1][k]);
                if (lane == (k & 31)) {
                    part[k] = t0;
                    part[K + k] = ti;
                    part[2 * K + k] = tj;
                    part[3 * K + k] = tij;
                }
            }
        }
        __syncthreads();  // every warp's partial sums are complete
        merge_tile_slots(s_part, NV * K, jb.slot, rq.slots, false, false);
        __syncthreads();  // s_q, s_part and s_job are rewritten by the next tile
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
template <int NV>
__global__ void pd_reduce_pairs(const double *__restrict__ slots, const int64_t *__restrict__ lptr,
                                const int64_t *__restrict__ lidx, const PdPairDev *__restrict__ pairs,
                                const double *__restrict__ qv, int32_t n_pairs, int32_t nq,
                                int32_t K, int32_t /*nv: the template's NV*/, int32_t n_frames,
                                int64_t slots_per_frame, const double *__restrict__ radius,
                                double qmin, double dq, int32_t residual_form, int32_t add_exact,
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
    constexpr int nv = NV;  // values per slot entry: 1 (class) or 4 (weighted)
    double s[4] = {0, 0, 0, 0};
    if (qval > 0.0) {
        const int64_t e0 = lptr[p * nqb + qb], e1 = lptr[p * nqb + qb + 1];
        const int64_t fbase = static_cast<int64_t>(f) * slots_per_frame;
        const int64_t stride = static_cast<int64_t>(nv) * K;
        // eight slots in flight per thread, added in list order (the same
        // order, and so the same rounding, as one slot at a time)
        int64_t e = e0;
        for (; e + 8 <= e1; e += 8) {
            double x[8][4];
#pragma unroll
            for (int u = 0; u < 8; ++u) {
                const double *sl = slots + (fbase + lidx[e + u]) * stride + kk;
                for (int v = 0; v < nv; ++v) x[u][v] = sl[v * K];
            }
#pragma unroll
            for (int u = 0; u < 8; ++u)
                for (int v = 0; v < nv; ++v) s[v] += x[u][v];
        }
        for (; e < e1; ++e) {
            const double *sl = slots + (fbase + lidx[e]) * stride + kk;
            for (int v = 0; v < nv; ++v) s[v] += sl[v * K];
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

// ------------------------------------------------------------ lattice sets
// Integer lattice coordinates of every point of every lattice set, from the
// FP64 input positions (frame 0): i = rint((x - origin)/spacing) per axis. A
// point farther than 1e-6·spacing from its lattice node, or outside the
// extents, sets *err (the profiles of the request then become NaN).
__global__ void pd_lattice_index(const double *__restrict__ xyz, const int32_t *__restrict__ perm,
                                 const PdLatDev *__restrict__ lat, int4 *__restrict__ idx,
                                 int *__restrict__ err) {
    const PdLatDev d = lat[blockIdx.y];
    for (int r = blockIdx.x * blockDim.x + threadIdx.x; r < d.n; r += gridDim.x * blockDim.x) {
        const int p = d.start + r;
        const int64_t src = perm[p];
        int c[3] = {0, 0, 0};  // an invalid point counts at the origin node (in range)
        bool ok = src >= 0;
        for (int a = 0; a < 3 && ok; ++a) {
            const double x = xyz[3 * src + a];
            const double u = (x - d.origin[a]) / d.spacing;
            const double ur = rint(u);
            ok = fabs(x - (d.origin[a] + ur * d.spacing)) <= 1e-6 * d.spacing && ur >= 0.0 &&
                 ur < static_cast<double>(d.ext[a]);
            c[a] = ok ? static_cast<int>(ur) : 0;
        }
        if (!ok) atomicOr(err, 1);
        idx[p] = make_int4(c[0], c[1], c[2], 0);
    }
}

// Exact pair counts per integer squared offset n = |Δ(i, j, k)|² of a
// lattice set: one CTA per tile (128 i points, a range of j points, j > i),
// counted in a shared-memory histogram (32-bit: a tile holds at most
// 128 × 8192 pairs) and added to the FP64-free 64-bit global histogram at the
// end. Integer sums: the counts do not depend on the order the CTAs run in.
// With more bins than fit in shared memory (`shared_bins` = 0) the CTA adds
// straight to the global histogram.
__global__ void __launch_bounds__(128) pd_lattice_hist(const PdLatTile *__restrict__ tiles,
                                                       const PdLatDev *__restrict__ lat,
                                                       const int4 *__restrict__ idx,
                                                       unsigned long long *__restrict__ hist,
                                                       int shared_bins) {
    extern __shared__ unsigned int s_hist[];
    const PdLatTile t = tiles[blockIdx.x];
    const PdLatDev d = lat[t.lat];
    const bool use_shared = shared_bins > 0;
    if (use_shared)
        for (int b = threadIdx.x; b < d.n_bins; b += blockDim.x) s_hist[b] = 0u;
    __syncthreads();
    const int i = t.i0 + threadIdx.x;
    if (i < d.n) {
        const int4 a = idx[d.start + i];
        for (int j = max(t.j0, i + 1); j < t.j1; ++j) {
            const int4 b = idx[d.start + j];
            const int dx = a.x - b.x, dy = a.y - b.y, dz = a.z - b.z;
            const int n = dx * dx + dy * dy + dz * dz;  // < n_bins: both points in the extents
            if (use_shared)
                atomicAdd(&s_hist[n], 1u);
            else
                atomicAdd(&hist[d.hist_off + n], 1ull);
        }
    }
    __syncthreads();
    if (use_shared)
        for (int b = threadIdx.x; b < d.n_bins; b += blockDim.x) {
            const unsigned int v = s_hist[b];
            if (v) atomicAdd(&hist[d.hist_off + b], static_cast<unsigned long long>(v));
        }
}

// Self pair sums of the lattice sets from their pair counts:
// Σ_{i<j} sinc(q r_ij) = Σ_n count(n)·sinc(q·spacing·√n), FP64, one CTA per
// (q, lattice); each thread adds the bins n ≡ thread (mod 256) in ascending
// order and a fixed tree adds the threads, so the sum is deterministic. The
// value overwrites the class pair's entry of `pairsum` (the pair tiles skip
// those pairs). Only the rank that adds the exact terms writes a sum; the
// others write 0. *err set: NaN.
__global__ void __launch_bounds__(256) pd_lattice_sums(const unsigned long long *__restrict__ hist,
                                                       const PdLatDev *__restrict__ lat,
                                                       const double *__restrict__ qv, int32_t nq,
                                                       int32_t add_exact,
                                                       const int *__restrict__ err,
                                                       double *__restrict__ pairsum) {
    __shared__ double s_part[256];
    const int q = blockIdx.x;
    const PdLatDev d = lat[blockIdx.y];
    const double qval = qv[q];
    double acc = 0.0;
    for (int n = 1 + threadIdx.x; n < d.n_bins; n += 256) {
        const unsigned long long c = hist[d.hist_off + n];
        if (c == 0ull) continue;
        const double x = qval * d.spacing * sqrt(static_cast<double>(n));
        // sinc as the reference defines it (src/debye.rs:17-24)
        const double sc = fabs(x) < 1e-8 ? 1.0 : sin(x) / x;
        acc += static_cast<double>(c) * sc;
    }
    s_part[threadIdx.x] = acc;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (threadIdx.x < w) s_part[threadIdx.x] += s_part[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        double v = add_exact ? s_part[0] : 0.0;
        if (*err) v = __longlong_as_double(0x7ff8000000000000ll);  // NaN
        pairsum[static_cast<int64_t>(d.pair) * nq + q] = v;
    }
}

// Frame-weighted mean of the six profiles, frames added in order.
__global__ void pd_frame_mean(const double *__restrict__ terms, const double *__restrict__ fw,
                              int32_t n_frames, int32_t nq, int32_t normalize,
                              double *__restrict__ out) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= 6 * nq) return;
    double s = 0.0, wsum = 0.0;
    for (int f = 0; f < n_frames; ++f) {
        const double w = fw ? fw[f] : 1.0;
        s += w * terms[static_cast<int64_t>(f) * 6 * nq + t];
        wsum += w;
    }
    out[t] = normalize ? s / wsum : s;
}

// Streamed trajectories: acc += batch, where batch is one batch's
// unnormalised Σ_f w_f·T_f (or, for a one-frame batch, T times its weight).
// Batches are added in submission order.
__global__ void pd_stream_accumulate(const double *__restrict__ batch, double scale, int32_t n,
                                     double *__restrict__ acc) {
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t < n) acc[t] += scale * batch[t];
}

// ------------------------------------------------------------ Direct transform
// Amplitudes of a periodic box at explicit q-vectors (the reference's
// DirectTransform, src/explicit.rs:138-147 and :208-230), FP64 throughout:
// F(q) = Σ_j f_j(q)·e^{i q·r_j} with q·r evaluated as q_x·x + q_y·y + q_z·z and
// one sincos per (vector, point). The points are split into chunks that never
// straddle a molecule: groups of whole molecules (molecules of at most
// a chunk length of points), for which the chunk also forms Σ_m |F_m|², or
// slices of that many points of one molecule (the last one shorter), whose
// partial amplitudes the reduction joins per molecule. The chunk length is
// 1,024, 512 or 256 points: the longest that still gives PD_DIRECT_BLOCKS
// blocks, so that the last wave of blocks is a small part of the launch.
//
// A block of 128 threads owns 2 × 128 q-vectors (two independent sincos
// chains per thread) and walks its chunk in stages of PD_DIRECT_STAGE points
// copied to shared memory (coordinates, weight, kind), which every thread then
// reads as broadcasts; the form factors of up to PD_DIRECT_SMEM_KINDS kinds for
// the block's vectors sit in shared memory as well, so the inner loop reads no
// global memory.
constexpr int PD_DIRECT_CHUNK_MAX = 1024, PD_DIRECT_CHUNK_MIN = 256;
constexpr int64_t PD_DIRECT_BLOCKS = 4096;  // about 6 waves of 148 SMs x 5 blocks
constexpr int PD_DIRECT_THREADS = 128;
constexpr int PD_DIRECT_V = 2;  // q-vectors per thread
constexpr int PD_DIRECT_STAGE = 256;
constexpr int PD_DIRECT_SMEM_KINDS = 16;

__global__ void __launch_bounds__(PD_DIRECT_THREADS)
    pd_direct_chunks(const double *__restrict__ xyz, const uint32_t *__restrict__ kind,
                     const double *__restrict__ weight, const double *__restrict__ ff,
                     const double *__restrict__ qvec, int64_t n_vec, int64_t n_vblocks,
                     int64_t mol_size, int64_t chunk_points, int64_t slices_per_mol,
                     int64_t n_points, int32_t n_kinds, double *__restrict__ part) {
    constexpr int V = PD_DIRECT_V, T = PD_DIRECT_THREADS;
    __shared__ double s_x[PD_DIRECT_STAGE], s_y[PD_DIRECT_STAGE], s_z[PD_DIRECT_STAGE],
        s_w[PD_DIRECT_STAGE];
    __shared__ uint32_t s_k[PD_DIRECT_STAGE];
    __shared__ double s_f[PD_DIRECT_SMEM_KINDS][V * T];
    const int tid = threadIdx.x;
    // consecutive blocks: the vector blocks of one chunk (its points stay in L2)
    const int64_t c = blockIdx.x / n_vblocks, vb = blockIdx.x % n_vblocks;
    int64_t v[V];
    bool ok[V];
    double qx[V], qy[V], qz[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        v[j] = vb * (V * T) + j * T + tid;
        ok[j] = v[j] < n_vec;
        qx[j] = ok[j] ? qvec[3 * v[j]] : 0.0;
        qy[j] = ok[j] ? qvec[3 * v[j] + 1] : 0.0;
        qz[j] = ok[j] ? qvec[3 * v[j] + 2] : 0.0;
    }
    const bool smem_ff = n_kinds <= PD_DIRECT_SMEM_KINDS;
    if (smem_ff)
        for (int k = 0; k < n_kinds; ++k)
#pragma unroll
            for (int j = 0; j < V; ++j)
                s_f[k][j * T + tid] = ok[j] ? ff[static_cast<int64_t>(k) * n_vec + v[j]] : 0.0;
    int64_t p0, p1;
    if (slices_per_mol == 1) {  // whole molecules
        p0 = c * chunk_points;
        p1 = min(n_points, p0 + chunk_points);
    } else {                    // slice s of molecule m
        const int64_t m = c / slices_per_mol, sl = c % slices_per_mol;
        p0 = m * mol_size + sl * chunk_points;
        p1 = min((m + 1) * mol_size, p0 + chunk_points);
    }
    const bool whole = slices_per_mol == 1;
    int64_t mol_end = (p0 / mol_size + 1) * mol_size;  // first molecule end after p0
    double ar[V], ai[V], self[V], fr[V], fi[V];
#pragma unroll
    for (int j = 0; j < V; ++j) ar[j] = ai[j] = self[j] = fr[j] = fi[j] = 0.0;
    for (int64_t s0 = p0; s0 < p1; s0 += PD_DIRECT_STAGE) {
        const int ns = static_cast<int>(min(static_cast<int64_t>(PD_DIRECT_STAGE), p1 - s0));
        __syncthreads();  // the previous stage is read (and s_f written)
        for (int t = tid; t < ns; t += T) {
            const int64_t p = s0 + t;
            s_x[t] = xyz[3 * p];
            s_y[t] = xyz[3 * p + 1];
            s_z[t] = xyz[3 * p + 2];
            s_w[t] = weight ? weight[p] : 1.0;
            s_k[t] = kind[p];
        }
        __syncthreads();
        for (int t = 0; t < ns; ++t) {
            const double x = s_x[t], y = s_y[t], z = s_z[t], w = s_w[t];
            const uint32_t k = s_k[t];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                double f = smem_ff ? s_f[k][j * T + tid]
                                   : (ok[j] ? ff[static_cast<int64_t>(k) * n_vec + v[j]] : 0.0);
                if (weight) f = w * f;  // DummySet::Weighted: w·F
                const double qr = qx[j] * x + qy[j] * y + qz[j] * z;
                double sn, cs;
                sincos(qr, &sn, &cs);
                fr[j] += f * cs;
                fi[j] += f * sn;
            }
            if (whole && s0 + t + 1 == mol_end) {  // a molecule ends inside this chunk
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    ar[j] += fr[j];
                    ai[j] += fi[j];
                    self[j] += fr[j] * fr[j] + fi[j] * fi[j];
                    fr[j] = 0.0;
                    fi[j] = 0.0;
                }
                mol_end += mol_size;
            }
        }
    }
    // whole molecules: (A, Σ|F_m|²); a slice of a molecule: its open partial F
#pragma unroll
    for (int j = 0; j < V; ++j) {
        if (!ok[j]) continue;
        double *o = part + (c * n_vec + v[j]) * 5;
        o[0] = ar[j];
        o[1] = ai[j];
        o[2] = self[j];
        o[3] = fr[j];
        o[4] = fi[j];
    }
}

// Direct transform at reciprocal-lattice vectors q = 2π·(h, k, l)/L: the phase
// of a term is e^{i2πh·x/Lx}·e^{i2πk·y/Ly}·e^{i2πl·z/Lz}. Per stage of points
// the block builds, in shared memory, each point's powers e^{i2πn·x_a/L_a} for
// n = 0..nmax on every axis (segments of a row start from a sincos and step by
// products with e^{i2π·x_a/L_a}; negative n by conjugation: the reference's
// PhaseTable, src/explicit.rs:85-135). A term then costs three table reads and two
// complex products instead of a sincos. Same chunks, partial layout and
// reduction as pd_direct_chunks; 256 threads own 3 × 256 vectors.
constexpr int PD_DTAB_THREADS = 256;
constexpr int PD_DTAB_V = 3;
constexpr int PD_DTAB_MAX_POINTS = 64;
constexpr int PD_DTAB_TABLE_BYTES = 96 * 1024;

__device__ __forceinline__ double2 cmul(double2 a, double2 b) {
    return make_double2(fma(a.x, b.x, -a.y * b.y), fma(a.x, b.y, a.y * b.x));
}
// a, or its conjugate when neg is the sign bit of the high word
__device__ __forceinline__ double2 conj_if(double2 a, int neg) {
    return make_double2(a.x, __hiloint2double(__double2hiint(a.y) ^ neg, __double2loint(a.y)));
}

__global__ void __launch_bounds__(PD_DTAB_THREADS, 2)
    pd_direct_table(const double *__restrict__ xyz, const uint32_t *__restrict__ kind,
                    const double *__restrict__ weight, const double *__restrict__ ff,
                    const int32_t *__restrict__ hkl, double lx, double ly, double lz,
                    int32_t stride, int32_t npts, int64_t n_vec, int64_t n_vblocks,
                    int64_t mol_size, int64_t chunk_points, int64_t slices_per_mol,
                    int64_t n_points, double *__restrict__ part) {
    constexpr int V = PD_DTAB_V, T = PD_DTAB_THREADS;
    extern __shared__ __align__(16) double2 pd_dtab[];  // [npts][3][stride]
    __shared__ double s_w[PD_DTAB_MAX_POINTS];
    __shared__ uint32_t s_k[PD_DTAB_MAX_POINTS];
    const int tid = threadIdx.x;
    const int64_t c = blockIdx.x / n_vblocks, vb = blockIdx.x % n_vblocks;
    int64_t v[V];
    bool ok[V];
    int ox[V], oy[V], oz[V], sx[V], sy[V], sz[V];
#pragma unroll
    for (int j = 0; j < V; ++j) {
        v[j] = vb * (V * T) + j * T + tid;
        ok[j] = v[j] < n_vec;
        const int h = ok[j] ? hkl[3 * v[j]] : 0, k = ok[j] ? hkl[3 * v[j] + 1] : 0,
                  l = ok[j] ? hkl[3 * v[j] + 2] : 0;
        ox[j] = abs(h);
        oy[j] = stride + abs(k);
        oz[j] = 2 * stride + abs(l);
        sx[j] = h < 0 ? static_cast<int>(0x80000000u) : 0;
        sy[j] = k < 0 ? static_cast<int>(0x80000000u) : 0;
        sz[j] = l < 0 ? static_cast<int>(0x80000000u) : 0;
    }
    int64_t p0, p1;
    if (slices_per_mol == 1) {
        p0 = c * chunk_points;
        p1 = min(n_points, p0 + chunk_points);
    } else {
        const int64_t m = c / slices_per_mol, sl = c % slices_per_mol;
        p0 = m * mol_size + sl * chunk_points;
        p1 = min((m + 1) * mol_size, p0 + chunk_points);
    }
    const bool whole = slices_per_mol == 1;
    int64_t mol_end = (p0 / mol_size + 1) * mol_size;
    double ar[V], ai[V], self[V], fr[V], fi[V];
#pragma unroll
    for (int j = 0; j < V; ++j) ar[j] = ai[j] = self[j] = fr[j] = fi[j] = 0.0;
    for (int64_t s0 = p0; s0 < p1; s0 += npts) {
        const int ns = static_cast<int>(min(static_cast<int64_t>(npts), p1 - s0));
        __syncthreads();  // the previous stage's table is read
        // the rows e^{i2πn·x_a/L_a}, n = 0..stride-1, one per (point, axis),
        // each cut into up to 16-entry segments so that every thread takes
        // part: a segment starts from its own sincos and steps by products
        const int rows = 3 * ns;
        const int nseg = max(1, min((stride + 15) / 16, T / rows));
        const int seglen = (stride + nseg - 1) / nseg;
        for (int t = tid; t < rows * nseg; t += T) {
            const int rw = t / nseg, sg = t - rw * nseg;
            const int pt = rw / 3, a = rw - 3 * pt;
            const int n0 = sg * seglen, n1 = min(stride, n0 + seglen);
            const double x = xyz[3 * (s0 + pt) + a];
            const double L = a == 0 ? lx : (a == 1 ? ly : lz);
            const double th = 2.0 * 3.141592653589793 * x / L;
            double sn, cs;
            sincos(th, &sn, &cs);
            const double2 step = make_double2(cs, sn);
            double2 e = make_double2(1.0, 0.0);
            if (n0 > 0) {
                sincos(static_cast<double>(n0) * th, &sn, &cs);
                e = make_double2(cs, sn);
            }
            double2 *row = pd_dtab + rw * stride;
            for (int n = n0; n < n1; ++n) {
                row[n] = e;
                e = cmul(e, step);
            }
        }
        for (int t = tid; t < ns; t += T) {
            s_w[t] = weight ? weight[s0 + t] : 1.0;
            s_k[t] = kind[s0 + t];
        }
        __syncthreads();
        for (int pt = 0; pt < ns; ++pt) {
            const double2 *row = pd_dtab + 3 * pt * stride;
            const double w = s_w[pt];
            const uint32_t k = s_k[pt];
#pragma unroll
            for (int j = 0; j < V; ++j) {
                double f = ok[j] ? ff[static_cast<int64_t>(k) * n_vec + v[j]] : 0.0;
                if (weight) f = w * f;  // DummySet::Weighted: w·F
                const double2 ph = cmul(cmul(conj_if(row[ox[j]], sx[j]), conj_if(row[oy[j]], sy[j])),
                                        conj_if(row[oz[j]], sz[j]));
                fr[j] += f * ph.x;
                fi[j] += f * ph.y;
            }
            if (whole && s0 + pt + 1 == mol_end) {
#pragma unroll
                for (int j = 0; j < V; ++j) {
                    ar[j] += fr[j];
                    ai[j] += fi[j];
                    self[j] += fr[j] * fr[j] + fi[j] * fi[j];
                    fr[j] = 0.0;
                    fi[j] = 0.0;
                }
                mol_end += mol_size;
            }
        }
    }
#pragma unroll
    for (int j = 0; j < V; ++j) {
        if (!ok[j]) continue;
        double *o = part + (c * n_vec + v[j]) * 5;
        o[0] = ar[j];
        o[1] = ai[j];
        o[2] = self[j];
        o[3] = fr[j];
        o[4] = fi[j];
    }
}

// Per q-vector: A = Σ chunks, Σ_m |F_m|² with the slices of a molecule joined
// first. out[v] = (Re A, Im A, |A|², Σ_m |F_m|²). A block takes 32 vectors (a
// lane each); its 32 warps sum 32 fixed runs of whole molecules' chunks, each in
// chunk order, and the run totals are added in run order: the same sums, in
// the same order, on every call.
constexpr int PD_DIRECT_RED_WARPS = 32;

__global__ void __launch_bounds__(32 * PD_DIRECT_RED_WARPS)
    pd_direct_reduce(const double *__restrict__ part, int64_t n_vec, int64_t n_chunks,
                     int64_t slices_per_mol, double *__restrict__ out) {
    __shared__ double s_run[PD_DIRECT_RED_WARPS][3][32];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    const int64_t v = static_cast<int64_t>(blockIdx.x) * 32 + lane;
    const bool ok = v < n_vec;
    // runs of whole molecules: chunks [u0·spm, u1·spm)
    const int64_t units = n_chunks / slices_per_mol;
    const int64_t u0 = units * w / PD_DIRECT_RED_WARPS, u1 = units * (w + 1) / PD_DIRECT_RED_WARPS;
    double ar = 0.0, ai = 0.0, self = 0.0, fr = 0.0, fi = 0.0;
    if (ok) {
        for (int64_t c = u0 * slices_per_mol; c < u1 * slices_per_mol; ++c) {
            const double *o = part + (c * n_vec + v) * 5;
            ar += o[0];
            ai += o[1];
            self += o[2];
            if (slices_per_mol > 1) {
                fr += o[3];
                fi += o[4];
                if ((c + 1) % slices_per_mol == 0) {
                    ar += fr;
                    ai += fi;
                    self += fr * fr + fi * fi;
                    fr = 0.0;
                    fi = 0.0;
                }
            }
        }
    }
    s_run[w][0][lane] = ar;
    s_run[w][1][lane] = ai;
    s_run[w][2][lane] = self;
    __syncthreads();
    if (w == 0 && ok) {
        double a = 0.0, b = 0.0, sf = 0.0;
        for (int r = 0; r < PD_DIRECT_RED_WARPS; ++r) {
            a += s_run[r][0][lane];
            b += s_run[r][1][lane];
            sf += s_run[r][2][lane];
        }
        out[4 * v] = a;
        out[4 * v + 1] = b;
        out[4 * v + 2] = a * a + b * b;
        out[4 * v + 3] = sf;
    }
}

// ------------------------------------------------------------ form factors
// One thread per (form factor, grid point): the reference's FormFactor::eval
// (src/formfactor.rs:188-201) in FP64 on q_k = qmin + (qmax - qmin)·k/denom.
// Descriptor d: type, n, offset of its parameters in `params`; range [lo, hi].
// A point outside the range records the form factor's index + 1 in *bad.
__global__ void pd_ff_eval(const int32_t *__restrict__ desc, const double *__restrict__ range,
                           const double *__restrict__ params, int32_t n_ff, double qmin,
                           double qmax, int64_t nq, int *__restrict__ bad,
                           double *__restrict__ out) {
    const int64_t t = blockIdx.x * static_cast<int64_t>(blockDim.x) + threadIdx.x;
    if (t >= n_ff * nq) return;
    const int f = static_cast<int>(t / nq);
    const int64_t k = t % nq;
    const double denom = static_cast<double>(nq > 1 ? nq - 1 : 1);
    const double q = qmin + (qmax - qmin) * static_cast<double>(k) / denom;
    const int type = desc[3 * f], n = desc[3 * f + 1];
    const double *p = params + desc[3 * f + 2];
    double v = 0.0;
    if (!(range[2 * f] <= q && q <= range[2 * f + 1])) {
        atomicMax(bad, f + 1);
    } else if (type == PD_FF_CONSTANT) {
        v = p[0];
    } else if (type == PD_FF_GAUSSIAN) {
        const double PI = 3.14159265358979323846;
        const double s2 = q * q / (16.0 * PI * PI);
        double sum = 0.0;
        for (int i = 0; i < n; ++i) sum += p[1 + 2 * i] * exp(-p[2 + 2 * i] * s2);
        v = sum + p[0];
    } else if (type == PD_FF_SINGLE_GAUSSIAN) {
        v = p[0] * exp(-p[1] * q * q);
    } else if (type == PD_FF_POLYNOMIAL) {
        double sum = 0.0;
        for (int i = 0; i < n; ++i) {
            double pw = 1.0;
            for (int e = 0; e < i; ++e) pw *= q;  // q^i by repeated products (Rust powi)
            sum += p[i] * pw;
        }
        v = sum;
    } else if (type == PD_FF_TABLE) {
        const double *xs = p, *ys = p + n;
        int low = 0, high = n - 1;
        bool hit = false;
        while (low < high) {
            const int mid = (low + high) / 2;
            if (q < xs[mid]) {
                high = mid;
            } else if (q > xs[mid]) {
                low = mid + 1;
            } else {
                v = ys[mid];
                hit = true;
                break;
            }
        }
        if (!hit) {
            if (low == 0) {  // q == xs[0] is a hit; below xs[0] is out of range
                v = ys[0];
            } else {
                const double x0 = xs[low - 1], y0 = ys[low - 1], x1 = xs[low], y1 = ys[low];
                v = y0 + (q - x0) * (y1 - y0) / (x1 - x0);
            }
        }
    }
    out[t] = v;
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
static cudaError_t fp32_smem_attr() {
    // Above 48 KB of dynamic shared memory needs the opt-in attribute, set
    // once per device (the occupancy query sets it before any stream capture).
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev < 64 ? (uint64_t{1} << dev) : 0;
    if (bit && (done.load() & bit)) return cudaSuccess;
    const cudaError_t e = cudaFuncSetAttribute(pd_pairs_fp32<K, MODE, NP>,
                                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                                               static_cast<int>(PD_FP32_DYN_SMEM));
    if (e == cudaSuccess && bit) done.fetch_or(bit);
    return e;
}
template <int K, int MODE, int NP>
static cudaError_t launch_fp32_t(const PdJob *jobs, const int *n_jobs, const PdReqDev *reqs,
                                 int *counter, int grid, cudaStream_t st) {
    cudaError_t e = fp32_smem_attr<K, MODE, NP>();
    if (e != cudaSuccess) return e;
    pd_pairs_fp32<K, MODE, NP><<<grid, PD_THREADS, PD_FP32_DYN_SMEM, st>>>(jobs, n_jobs, reqs,
                                                                           counter);
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
    if (fp32_smem_attr<K, MODE, NP>() != cudaSuccess) return 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, pd_pairs_fp32<K, MODE, NP>, PD_THREADS,
                                                  PD_FP32_DYN_SMEM);
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
    if (mode == PD_MODE_WEIGHTED) return (K == 32 && NP == 2) || (K == 64 && (NP == 2 || NP == 4));
    return (K == 32 && NP == 4) || (K == 64 && NP >= 1 && NP != 3) || (K == 96 && NP == 2) ||
           (K == 128 && NP >= 1 && NP != 3) || ((K == 160 || K == 192) && NP == 1);
}

bool valid_q_block(int precision, int K) {
    if (precision == 1) return K == 16 || K == 32;
    return K == 32 || K == 64 || K == 96 || K == 128 || K == 160 || K == 192;
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
    PD_F32(32, 0, 4) PD_F32(64, 0, 1) PD_F32(64, 0, 2) PD_F32(64, 0, 4) PD_F32(96, 0, 2)
    PD_F32(128, 0, 1) PD_F32(128, 0, 2) PD_F32(128, 0, 4) PD_F32(160, 0, 1) PD_F32(192, 0, 1)
    PD_F32(32, 1, 2) PD_F32(64, 1, 2) PD_F32(64, 1, 4)
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
    PD_O32(32, 0, 4) PD_O32(64, 0, 1) PD_O32(64, 0, 2) PD_O32(64, 0, 4) PD_O32(96, 0, 2)
    PD_O32(128, 0, 1) PD_O32(128, 0, 2) PD_O32(128, 0, 4) PD_O32(160, 0, 1) PD_O32(192, 0, 1)
    PD_O32(32, 1, 2) PD_O32(64, 1, 2) PD_O32(64, 1, 4)
    return 0;
}

cudaError_t prepare_pair_kernels() {
    const int shapes[][3] = {{32, 0, 4},  {64, 0, 1},  {64, 0, 2},  {64, 0, 4},
                             {96, 0, 2},  {128, 0, 1}, {128, 0, 2}, {128, 0, 4},
                             {160, 0, 1}, {192, 0, 1}, {32, 1, 2},  {64, 1, 2},
                             {64, 1, 4}};
    for (const auto &sh : shapes)
        if (pairs_blocks_per_sm(0, sh[0], sh[2], sh[1]) <= 0) return cudaErrorInvalidValue;
    return cudaSuccess;
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
    if (nv == 4)
        pd_reduce_pairs<4><<<grid, 128, 0, st>>>(slots, lptr, lidx, pairs, qv, n_pairs, nq, K,
                                                 nv, n_frames, slots_per_frame, radius, qmin, dq,
                                                 residual_form, add_exact, pairsum);
    else
        pd_reduce_pairs<1><<<grid, 128, 0, st>>>(slots, lptr, lidx, pairs, qv, n_pairs, nq, K,
                                                 nv, n_frames, slots_per_frame, radius, qmin, dq,
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

cudaError_t launch_lattice(const double *xyz, const int32_t *perm, const PdLatDev *lat_dev,
                           const PdLatDev *lat_host, int n_lat, const PdLatTile *tiles,
                           int64_t n_tiles, int4 *idx, unsigned long long *hist, int64_t n_bins,
                           int *err, cudaStream_t st) {
    if (n_lat == 0) return cudaSuccess;
    cudaError_t e = cudaMemsetAsync(hist, 0, static_cast<size_t>(n_bins) * 8, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), st);
    if (e != cudaSuccess) return e;
    int max_n = 1, max_bins = 1;
    for (int l = 0; l < n_lat; ++l) {
        max_n = max(max_n, lat_host[l].n);
        max_bins = max(max_bins, lat_host[l].n_bins);
    }
    const dim3 g1(static_cast<unsigned>(min((max_n + 255) / 256, 4096)), n_lat);
    pd_lattice_index<<<g1, 256, 0, st>>>(xyz, perm, lat_dev, idx, err);
    if ((e = cudaGetLastError()) != cudaSuccess || n_tiles == 0) return e;
    // shared-memory histogram when the bins fit (opt-in limit of the device)
    int dev = 0, smem_optin = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&smem_optin, cudaDevAttrMaxSharedMemoryPerBlockOptin, dev);
    const size_t need = static_cast<size_t>(max_bins) * 4;
    int shared_bins = need <= static_cast<size_t>(smem_optin) ? max_bins : 0;
    size_t smem = shared_bins ? need : 0;
    if (smem > 48 * 1024) {
        e = cudaFuncSetAttribute(pd_lattice_hist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 static_cast<int>(smem));
        if (e != cudaSuccess) {
            (void)cudaGetLastError();
            shared_bins = 0;
            smem = 0;
        }
    }
    pd_lattice_hist<<<static_cast<unsigned>(n_tiles), 128, smem, st>>>(tiles, lat_dev, idx, hist,
                                                                        shared_bins);
    return cudaGetLastError();
}

cudaError_t launch_lattice_sums(const unsigned long long *hist, const PdLatDev *lat, int n_lat,
                                const double *qv, int32_t nq, int add_exact, const int *err,
                                double *pairsum, cudaStream_t st) {
    if (n_lat == 0) return cudaSuccess;
    pd_lattice_sums<<<dim3(nq, n_lat), 256, 0, st>>>(hist, lat, qv, nq, add_exact, err, pairsum);
    return cudaGetLastError();
}

cudaError_t launch_frame_mean(const double *terms, const double *fw, int32_t n_frames, int32_t nq,
                              double *out, cudaStream_t st, bool normalize) {
    const int grid = (6 * nq + 127) / 128;
    pd_frame_mean<<<grid, 128, 0, st>>>(terms, fw, n_frames, nq, normalize ? 1 : 0, out);
    return cudaGetLastError();
}

cudaError_t launch_stream_accumulate(const double *batch, double scale, int32_t n, double *acc,
                                     cudaStream_t st) {
    pd_stream_accumulate<<<(n + 127) / 128, 128, 0, st>>>(batch, scale, n, acc);
    return cudaGetLastError();
}

// Chunking of n_points points in molecules of mol_size for n_vec vectors:
// (points per chunk, slices per molecule, number of chunks).
static void direct_layout(int64_t n_points, int64_t mol_size, int64_t n_vec, int64_t *chunk,
                          int64_t *spm, int64_t *n_chunks) {
    const int64_t vblocks = (n_vec + PD_DIRECT_V * PD_DIRECT_THREADS - 1) /
                            (PD_DIRECT_V * PD_DIRECT_THREADS);
    for (int64_t len = PD_DIRECT_CHUNK_MAX;; len /= 2) {
        if (mol_size <= len) {
            *chunk = (len / mol_size) * mol_size;
            *spm = 1;
            *n_chunks = (n_points + *chunk - 1) / *chunk;
        } else {
            *chunk = len;
            *spm = (mol_size + len - 1) / len;
            *n_chunks = (n_points / mol_size) * *spm;
        }
        if (len <= PD_DIRECT_CHUNK_MIN || *n_chunks * vblocks >= PD_DIRECT_BLOCKS) return;
    }
}

int64_t direct_chunks(int64_t n_points, int64_t mol_size, int64_t n_vec) {
    int64_t chunk, spm, n;
    direct_layout(n_points, mol_size, n_vec, &chunk, &spm, &n);
    return n;
}

int64_t direct_blocks(int64_t n_points, int64_t mol_size, int64_t n_vec) {
    const int64_t vblocks = (n_vec + PD_DIRECT_V * PD_DIRECT_THREADS - 1) /
                            (PD_DIRECT_V * PD_DIRECT_THREADS);
    return direct_chunks(n_points, mol_size, n_vec) * vblocks;
}

cudaError_t launch_direct(const double *xyz, const uint32_t *kind, const double *weight,
                          const double *ff, int32_t n_kinds, const double *qvec, int64_t n_vec,
                          int64_t n_points, int64_t mol_size, double *part, int64_t part_chunks,
                          double *out, cudaStream_t st) {
    int64_t chunk, spm, n_chunks;
    direct_layout(n_points, mol_size, n_vec, &chunk, &spm, &n_chunks);
    constexpr int64_t per_block = PD_DIRECT_V * PD_DIRECT_THREADS;
    const int64_t vblocks = (n_vec + per_block - 1) / per_block;
    if (n_chunks > part_chunks || n_vec < 1 || n_chunks * vblocks > 0x7fffffffLL)
        return cudaErrorInvalidValue;
    pd_direct_chunks<<<static_cast<unsigned>(n_chunks * vblocks), PD_DIRECT_THREADS, 0, st>>>(
        xyz, kind, weight, ff, qvec, n_vec, vblocks, mol_size, chunk, spm, n_points, n_kinds,
        part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pd_direct_reduce<<<static_cast<unsigned>((n_vec + 31) / 32), 32 * PD_DIRECT_RED_WARPS, 0, st>>>(
        part, n_vec, n_chunks, spm, out);
    return cudaGetLastError();
}

// Stage length of the table kernel for indices up to nmax (0 when a single
// point's table does not fit).
int direct_table_points(int32_t nmax) {
    const int64_t per_point = 3LL * (nmax + 1) * static_cast<int64_t>(sizeof(double2));
    return static_cast<int>(std::min<int64_t>(PD_DTAB_MAX_POINTS, PD_DTAB_TABLE_BYTES / per_point));
}

cudaError_t launch_direct_table(const double *xyz, const uint32_t *kind, const double *weight,
                                const double *ff, const int32_t *hkl, int32_t nmax,
                                const double box[3], int64_t n_vec, int64_t n_points,
                                int64_t mol_size, double *part, int64_t part_chunks, double *out,
                                cudaStream_t st) {
    const int npts = direct_table_points(nmax);
    if (npts < 1 || n_vec < 1) return cudaErrorInvalidValue;
    const int stride = nmax + 1;
    const size_t smem = static_cast<size_t>(npts) * 3 * stride * sizeof(double2);
    // above 48 KB of dynamic shared memory needs the opt-in, set once per device
    static std::atomic<uint64_t> done{0};
    int dev = 0;
    cudaGetDevice(&dev);
    const uint64_t bit = dev < 64 ? (uint64_t{1} << dev) : 0;
    if (!bit || !(done.load() & bit)) {
        const cudaError_t e = cudaFuncSetAttribute(
            pd_direct_table, cudaFuncAttributeMaxDynamicSharedMemorySize, PD_DTAB_TABLE_BYTES);
        if (e != cudaSuccess) return e;
        if (bit) done.fetch_or(bit);
    }
    int64_t chunk, spm, n_chunks;
    direct_layout(n_points, mol_size, n_vec, &chunk, &spm, &n_chunks);
    constexpr int64_t per_block = PD_DTAB_V * PD_DTAB_THREADS;
    const int64_t vblocks = (n_vec + per_block - 1) / per_block;
    if (n_chunks > part_chunks || n_chunks * vblocks > 0x7fffffffLL) return cudaErrorInvalidValue;
    pd_direct_table<<<static_cast<unsigned>(n_chunks * vblocks), PD_DTAB_THREADS, smem, st>>>(
        xyz, kind, weight, ff, hkl, box[0], box[1], box[2], stride, npts, n_vec, vblocks,
        mol_size, chunk, spm, n_points, part);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    pd_direct_reduce<<<static_cast<unsigned>((n_vec + 31) / 32), 32 * PD_DIRECT_RED_WARPS, 0, st>>>(
        part, n_vec, n_chunks, spm, out);
    return cudaGetLastError();
}

cudaError_t launch_ff_eval(const int32_t *desc, const double *range, const double *params,
                           int32_t n_ff, double qmin, double qmax, int64_t nq, int *bad,
                           double *out, cudaStream_t st) {
    const int64_t total = static_cast<int64_t>(n_ff) * nq;
    pd_ff_eval<<<static_cast<unsigned>((total + 127) / 128), 128, 0, st>>>(
        desc, range, params, n_ff, qmin, qmax, nq, bad, out);
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
