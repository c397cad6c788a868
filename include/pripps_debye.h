/*
 * pripps_debye.h — C ABI of the B200 Debye backend (libpripps_debye.so).
 *
 * One backend only: every entry point runs the sum on an NVIDIA B200
 * (sm_100a). There is no CPU fallback; without a usable device the calls
 * return PD_ENODEV.
 *
 * The library computes, for one structure (or a batch of trajectory frames),
 * the six partial Debye profiles that the reference caches per q
 * (DebyeTerms, src/debye.rs:176-184), in this row order:
 *
 *   row 0  atoms               Σ_i A_i² + 2 Σ_{i<j} A_i A_j sinc(q r_ij)
 *   row 1  excluded            same with C_i (excluded-volume dummies)
 *   row 2  hydration           same with B_i (hydration dummies)
 *   row 3  atom_excluded       Σ_a Σ_b A_a C_b sinc(q r_ab)   (i = j included)
 *   row 4  atom_hydration      Σ_a Σ_b A_a B_b sinc(q r_ab)
 *   row 5  excluded_hydration  Σ_a Σ_b C_a B_b sinc(q r_ab)
 *
 * on the reference's uniform grid q_k = qmin + (qmax-qmin)·k/max(nq-1, 1)
 * (src/q_sampler.rs:24-29), with A_i = F_{s_i}(q), C_i = C_{s_i}(q) and
 * B_i = w_i·F_H2O(q): the atom, excluded-volume and hydration scatterers all
 * sit at the atom positions, as the reference's Fraser/FoXS excluded volume
 * (src/solvent/fraser.rs:64-100), per-kind excluded solvent
 * (src/solvent/per_kind_excluded.rs:16-39) and SASA hydration
 * (src/solvent/sasa.rs:34-71) place them.
 *
 * Conventions: every int-returning call returns PD_OK (0) or a negative
 * PD_E* code, and pd_last_error() describes the most recent failure of the
 * calling thread on that context. Output buffers are caller-owned. Request
 * inputs are copied at submission: the caller may free them once
 * pd_submit()/pd_solve() returns. A context is internally synchronised; any
 * host thread may use it.
 */
#ifndef PRIPPS_DEBYE_H
#define PRIPPS_DEBYE_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PD_ABI_VERSION 2

/* ---- status codes ---- */
#define PD_OK 0
#define PD_EINVAL (-1)    /* malformed request: nq = 0, N = 0, NaN input, bad ids */
#define PD_ENOMEM (-2)    /* a host or device allocation failed */
#define PD_EBUDGET (-3)   /* the request can never fit the context's memory budget */
#define PD_ETIMEOUT (-4)  /* pd_wait timed out, or a bounded device wait expired */
#define PD_EDEVICE (-5)   /* a CUDA call failed (message in pd_last_error) */
#define PD_ENOTFOUND (-6) /* unknown ticket */
#define PD_ECANCELED (-7) /* the request was cancelled before it finished */
#define PD_ENODEV (-8)    /* no sm_100 device at the requested ordinal */

/* ---- request flags ----
 * PD_FLAG_TEST_EXPIRED_WAIT is a test hook for the failure path of the FP32
 * pair kernel: the CTA that takes the first tile of a launch (when that tile
 * belongs to a flagged request) waits for a bulk copy of atoms that is never
 * issued, with a short poll limit, so that the bounded wait expires with no
 * copy in flight. That CTA then stops, writes NaN to the
 * slots of every tile it still takes and sets the request's device status;
 * blocking calls (pd_solve, pd_plan_execute_host, pd_wait, pd_stream_finish)
 * return PD_ETIMEOUT, calls that leave the result on the device show NaN
 * rows, and the context stays usable. It has no effect on PD_FP64 requests,
 * whose kernel stages nothing. */
#define PD_FLAG_TEST_EXPIRED_WAIT 0x80000000u

/* ---- precision forms ---- */
#define PD_FP32_FP64RED 0 /* FP32 recurrence sinc, FP32 per-tile sums, FP64 reduction */
#define PD_FP64 1         /* plain FP64 sinc and accumulation throughout */

/* ---- output layout ---- */
#define PD_NUM_TERMS 6 /* rows of the [6][nq] output, see above */

typedef struct pd_ctx pd_ctx;

/*
 * A lattice set (ABI version 2). Every point of species `species` sits at
 * origin + spacing·(i, j, k) with integers 0 <= i < extent[0],
 * 0 <= j < extent[1], 0 <= k < extent[2], as the reference's grid solvent
 * models place their dummies (ExcludedVolume::Grid,
 * src/solvent/grid_excluded.rs:34-73; Hydration::Grid, src/solvent/grid.rs:
 * 40-95). The self pair sum of such a set depends only on the integer squared
 * offsets n = |(i,j,k) - (i',j',k')|², so the library counts the pairs of
 * every n exactly (integer work on the device) and evaluates
 * Σ_n count(n)·sinc(q·spacing·√n) in FP64 instead of summing a sinc per pair:
 * on a lattice whole classes of pairs share one distance, and a per-pair FP32
 * evaluation would repeat the same rounding for all of them. Pairs between
 * the set and other points are summed per pair as usual.
 * Requirements: the species' points share one hydration weight (or there are
 * no hydration weights), the request has one frame and fewer than 49
 * (species, weight) classes. A point of the species that lies off the lattice
 * by more than 1e-6·spacing or outside the extents makes the result NaN
 * (pd_solve and pd_wait then return PD_EINVAL).
 */
typedef struct pd_lattice {
    uint32_t species;    /* species id whose points form the lattice set */
    uint32_t reserved;   /* must be 0 */
    double origin[3];    /* Å */
    double spacing;      /* Å, > 0 */
    uint32_t extent[3];  /* grid steps per axis, each >= 1 */
    uint32_t reserved2;  /* must be 0 */
} pd_lattice;

/*
 * One Debye solve. Replaces the inputs the reference's build_model gathers
 * per q (src/debye.rs:83-101): the structure (Structure{pos, ids},
 * src/structure.rs:27-31), the per-species form factors evaluated on the q
 * grid (formfactor_by_index, src/formfactor.rs:528-544), the excluded-volume
 * dummy form factors (ExcludedVolume::unit_scale_dummies,
 * src/solvent/mod.rs:385-403) and the hydration weights plus shared water
 * form factor (DummySet::Weighted, src/solvent/mod.rs:365-371).
 */
typedef struct pd_request {
    uint64_t n_atoms;           /* N >= 1 */
    const double *xyz;          /* [n_frames][N][3] positions in Å (AoS) */
    const uint32_t *species;    /* [N] species ids, each < n_species */
    uint32_t n_species;         /* S >= 1 */
    uint32_t precision;         /* PD_FP32_FP64RED or PD_FP64 */
    const double *ff_atoms;     /* [S][nq] F_s(q_k); required */
    const double *ff_excluded;  /* [S][nq] C_s(q_k), or NULL: no excluded volume */
    const double *hyd_weights;  /* [N] w_i, or NULL: no hydration */
    const double *ff_water;     /* [nq] F_H2O(q_k); required iff hyd_weights */
    double qmin, qmax;          /* grid ends (inclusive), qmin >= 0 */
    uint64_t nq;                /* >= 1 */
    uint64_t n_frames;          /* 0 or 1: one structure; > 1: trajectory batch */
    const double *frame_weights;/* [n_frames] weights of the mean, or NULL: uniform */
    uint32_t flags;             /* 0, or PD_FLAG_TEST_EXPIRED_WAIT (tests only) */
    uint32_t n_lattices;        /* 0..8 lattice sets (ABI version 1: must be 0) */
    const pd_lattice *lattices; /* [n_lattices], read only when n_lattices > 0 */
} pd_request;

/* Create a context on CUDA device `device`. `mem_budget_bytes` caps the
 * device memory the context holds for admitted requests (0 = 90 % of the
 * device's free memory). No reference counterpart: the reference holds no
 * device state (its Debye path is rayon on the host, src/debye.rs:90-92). */
int pd_ctx_create(int device, uint64_t mem_budget_bytes, pd_ctx **out);

/* Release every resource of the context; outstanding tickets are cancelled. */
void pd_ctx_destroy(pd_ctx *ctx);

/* Blocking solve with host buffers: out_terms is [6][nq] (n_frames <= 1) or
 * the frame-weighted mean Σ_f w_f·T_f / Σ_f w_f of the six profiles.
 * Replaces the per-q body of build_model (src/debye.rs:90-130) and, for the
 * vacuum path, QSampler::run_parallel over intensity_at_q
 * (src/debye.rs:58-60, :200-211) — rows 1..5 are zero then — and the frame
 * loop of trajectory_average (src/trajectory.rs:198-248; the weighted mean of
 * the terms combines to the weighted mean of the totals because combine is
 * linear in the terms). */
int pd_solve(pd_ctx *ctx, const pd_request *req, double *out_terms);

/* Plans: the host-side preparation of a request (atom classes, padded
 * layout, tile list, reduction lists, uploaded form-factor tables) split from
 * its execution, for callers that solve the same topology many times with new
 * coordinates — trajectory frames (src/trajectory.rs:198-223) or a caller
 * whose coordinates already live in device memory. pd_plan_create reads every
 * pointer of `req` as HOST memory except `xyz`, which may be NULL (coordinates
 * are supplied per execution). No reference counterpart beyond build_model
 * (src/debye.rs:78-136), which re-derives all of this on every call. */
typedef struct pd_plan pd_plan;
int pd_plan_create(pd_ctx *ctx, const pd_request *req, pd_plan **out);

/* Enqueue one solve of `plan` on `stream` (a cudaStream_t; NULL = legacy
 * default stream). xyz_dev is DEVICE memory [n_frames][N][3] and
 * out_terms_dev DEVICE memory for the [6][nq] result; both must stay valid
 * until the stream passes this call. Executions of one plan on several
 * streams at once race on the plan's scratch and must be serialised. */
int pd_plan_execute(pd_ctx *ctx, pd_plan *plan, const double *xyz_dev, double *out_terms_dev,
                    void *stream);

/* Blocking execution with HOST coordinates and a HOST [6][nq] result. */
int pd_plan_execute_host(pd_ctx *ctx, pd_plan *plan, const double *xyz_host, double *out_terms);

/* q-block length, atom-chunk length, pairs per thread, tiles per execution,
 * device bytes held and bytes uploaded from the host when the plan is
 * created. */
int pd_plan_info(const pd_plan *plan, uint32_t *q_block, uint32_t *j_chunk,
                 uint32_t *pairs_per_thread, uint64_t *n_tiles, uint64_t *device_bytes,
                 uint64_t *upload_bytes);

/* Multi-GPU: restrict a plan to rank's share of the tiles (every world-th
 * tile in cost order). Each execution then yields partial profiles whose sum
 * over the ranks is the full [6][nq] result — rank 0 also carries the i = j
 * terms and the exact q = 0 sums — so the caller adds them across devices
 * (one all-reduce of 6·nq doubles). world = 1 restores the whole plan. No
 * reference counterpart (the reference is single-process). */
int pd_plan_set_shard(pd_ctx *ctx, pd_plan *plan, uint32_t rank, uint32_t world);

/* Host-only view of a request's tiles in rank's share: five int32 per tile
 * (first i of the 128-atom block, j range [j0, j1), q-block, frame) in padded
 * atom indices, and the padded-index -> atom permutation (-1 = padding). */
int pd_plan_tiles(pd_ctx *ctx, const pd_request *req, uint32_t rank, uint32_t world,
                  int32_t *tiles, uint64_t cap, uint64_t *n_tiles, int32_t *perm,
                  uint64_t perm_cap, uint64_t *n_padded);

/* Kernel timing: with profiling enabled every pd_plan_execute brackets its
 * pair kernel with CUDA events on the execution stream; pd_plan_pair_kernel_ms
 * waits for them and reports the summed duration and the number of timed
 * launches since profiling was (re)enabled. */
int pd_plan_set_profiling(pd_ctx *ctx, pd_plan *plan, int enable);
int pd_plan_pair_kernel_ms(pd_ctx *ctx, pd_plan *plan, double *total_ms, uint64_t *n_launches);
void pd_plan_destroy(pd_ctx *ctx, pd_plan *plan);

/* Streamed trajectory averages: the frame loop of trajectory_average
 * (src/trajectory.rs:198-248) for trajectories too long to hold in one
 * request, fed frame by frame from any reader (the reference reads XTC files
 * through its XtcIterator, src/trajectory.rs:36-118). pd_stream_open takes
 * the topology of `req` (species, tables, q grid, precision; req->xyz,
 * n_frames and frame_weights are ignored; no lattice sets) and the number of
 * frames solved per batch. pd_stream_push copies n_frames frames
 * ([n_frames][N][3] HOST memory, Å) and their weights (NULL = 1) into pinned
 * batches; each full batch is uploaded on its own stream while the previous
 * one is solved, and push blocks only while both batch buffers are in use.
 * pd_stream_finish solves the last partial batch, writes the weighted mean
 * Σ_f w_f·T_f / Σ_f w_f of the six profiles to out_terms ([6][nq] HOST; may
 * be NULL) and releases the stream; a weight sum that is zero or not normal
 * is PD_EINVAL, as in the reference (src/trajectory.rs:234-238). */
typedef struct pd_stream pd_stream;
int pd_stream_open(pd_ctx *ctx, const pd_request *req, uint32_t frames_per_batch,
                   pd_stream **out);
int pd_stream_push(pd_ctx *ctx, pd_stream *s, const double *xyz, const double *weights,
                   uint64_t n_frames);
int pd_stream_finish(pd_ctx *ctx, pd_stream *s, double *out_terms);

/* Direct transform of a periodic box (the reference's DirectTransform,
 * src/explicit.rs:138-147 and :208-230, and the amplitude part of its
 * DirectModel, :296-325): for each explicit q-vector q_v (Å⁻¹; the
 * reference's 2π·n/L for integer n), the amplitude
 * A(q_v) = Σ_j w_j·f_{kind_j}(|q_v|)·e^{i q_v·r_j} over n_points points, and the
 * self term Σ_m |F_m(q_v)|² over n_molecules equal contiguous molecules
 * (0 or 1: the whole box; n_points must be a multiple). ff is
 * [n_kinds][n_vectors]: each kind's form factor at each vector's |q|, as the
 * host evaluates it (eval_atom_form_factors, src/explicit.rs:360-370). FP64
 * throughout, one sincos per (vector, point). out is [n_vectors][4]:
 * Re A, Im A, |A|², Σ_m |F_m|². Blocking; HOST buffers. */
typedef struct pd_direct_request {
    uint64_t n_points;         /* >= 1 */
    const double *xyz;         /* [n_points][3] Å */
    const uint32_t *kind;      /* [n_points], each < n_kinds */
    uint32_t n_kinds;          /* >= 1 */
    uint32_t reserved;         /* must be 0 */
    const double *ff;          /* [n_kinds][n_vectors] */
    uint64_t n_vectors;        /* >= 1 */
    const double *qvec;        /* [n_vectors][3] Å⁻¹ */
    uint64_t n_molecules;      /* 0 or 1 = whole box, else divides n_points */
    const double *weight;      /* [n_points] factor on each point's form factor, or NULL
                                  (DummySet::Weighted, src/solvent/mod.rs:365-371) */
} pd_direct_request;
int pd_direct(pd_ctx *ctx, const pd_direct_request *req, double *out);
/* The same rows at reciprocal-lattice vectors q = 2π·(h, k, l)/box, given as
 * integer indices hkl [n_vectors][3] (req->qvec is not read; ff columns follow
 * the hkl rows). Each term's phase comes from per-point tables of
 * e^{i2πn·x_a/L_a}, n = 0..max|index| (negative n by conjugation), built on
 * the device — the reference's PhaseTable (src/explicit.rs:85-135) — instead
 * of a sincos; indices beyond 512 take the sincos kernel at q = 2π·hkl/box.
 * Within 1e-12 of pd_direct at the same vectors. box sides finite and > 0. */
int pd_direct_lattice(pd_ctx *ctx, const pd_direct_request *req, const int32_t *hkl,
                      const double box[3], double *out);

/* Form factors evaluated on the device: the reference's FormFactor kinds
 * (src/formfactor.rs:130-201; United is a 101-point Table after loading,
 * :642-698) on the uniform grid q_k = qmin + (qmax-qmin)·k/max(nq-1, 1),
 * FP64:
 *   PD_FF_CONSTANT        c                          params = [c]
 *   PD_FF_GAUSSIAN        Σ a_i·exp(-b_i·s²) + c, s² = q²/(16π²)
 *                                                    params = [c, a_0, b_0, …], n = pairs
 *   PD_FF_SINGLE_GAUSSIAN a·exp(-b·q²)               params = [a, b]
 *   PD_FF_POLYNOMIAL      Σ c_i·q^i                  params = [c_0 … c_{n-1}]
 *   PD_FF_TABLE           linear interpolation, exact hit returns the value
 *                                                    params = [x_0 … x_{n-1}, y_0 … y_{n-1}]
 * A grid point outside [qlo, qhi] of a form factor is the reference's
 * QOutOfRange (src/formfactor.rs:191-193): PD_EINVAL, naming it. out is
 * [n_ff][nq] HOST memory. Blocking. */
#define PD_FF_CONSTANT 0
#define PD_FF_GAUSSIAN 1
#define PD_FF_SINGLE_GAUSSIAN 2
#define PD_FF_POLYNOMIAL 3
#define PD_FF_TABLE 4
typedef struct pd_formfactor {
    uint32_t type;          /* PD_FF_* */
    uint32_t n;             /* Gaussian pairs, polynomial coefficients or table points */
    double qlo, qhi;        /* valid q range, inclusive */
    const double *params;   /* as listed above */
} pd_formfactor;
int pd_formfactor_tables(pd_ctx *ctx, const pd_formfactor *ff, uint32_t n_ff, double qmin,
                         double qmax, uint64_t nq, double *out);

/* Continuous-batching request loop. pd_submit copies the request, queues it
 * for admission (admitted when device memory within the budget frees up) and
 * returns a ticket at once; its tiles then run interleaved with those of the
 * other admitted requests. pd_wait blocks up to timeout_ms (< 0: forever) and
 * copies the [6][nq] result out; pd_poll returns 1 when the ticket finished,
 * 0 while it is pending, or a negative code. The result of a ticket is
 * independent of what else ran beside it (deterministic per-request
 * reduction). pd_wait hands the result out once: it then frees it, and a
 * second pd_wait with a non-NULL out_terms returns PD_EINVAL. */
int pd_submit(pd_ctx *ctx, const pd_request *req, uint64_t *ticket);
int pd_wait(pd_ctx *ctx, uint64_t ticket, int timeout_ms, double *out_terms);
int pd_poll(pd_ctx *ctx, uint64_t ticket);
int pd_cancel(pd_ctx *ctx, uint64_t ticket);

/* Serving replicas across GPUs: one request loop (context) per device in
 * `devices` (the same ordinal may repeat: several loops share that GPU), and
 * a router that sends each whole request to the replica with the least work
 * still pending (pair·q × frames, FP64 counted 24×, the weighted mode 1.5×;
 * ties go to the lowest index). Whole requests never split across replicas,
 * so each result is the one its replica's loop gives alone. Tickets carry the
 * replica in their top 8 bits. pd_router_wait / _poll / _cancel behave as
 * pd_wait / pd_poll / pd_cancel on the replica; pd_router_replica names the
 * replica and its context ticket (for pd_ticket_times); pd_route_choose is
 * the routing policy itself (host-only): the index of the smallest pending
 * work. Errors of router calls are described by pd_router_last_error().
 * No reference counterpart (the reference is one process on one host). */
typedef struct pd_router pd_router;
int pd_router_create(const int *devices, uint32_t n_devices, uint64_t mem_budget_bytes,
                     pd_router **out);
void pd_router_destroy(pd_router *router);
int pd_router_submit(pd_router *router, const pd_request *req, uint64_t *ticket);
int pd_router_wait(pd_router *router, uint64_t ticket, int timeout_ms, double *out_terms);
int pd_router_poll(pd_router *router, uint64_t ticket);
int pd_router_cancel(pd_router *router, uint64_t ticket);
int pd_router_replica(pd_router *router, uint64_t ticket, uint32_t *replica, pd_ctx **ctx,
                      uint64_t *ctx_ticket);
int pd_route_choose(const double *pending_work, uint32_t n, uint32_t *choice);
const char *pd_router_last_error(void);

/* Timestamps of a finished ticket in seconds on the context's monotonic
 * clock: submission, admission to the device, completion. */
int pd_ticket_times(pd_ctx *ctx, uint64_t ticket, double *t_submit, double *t_admit,
                    double *t_done);

/* The recombination of the six terms into I(q) (DebyeTerms::combine,
 * src/debye.rs:187-194); total is [nq]. Host-only. */
int pd_combine(const double *terms, uint64_t nq, double volume_scale,
               double contrast_density, double *total);

/* Message describing the last failure on this context from the calling
 * thread ("" if none); NULL ctx gives the last context-free failure. */
const char *pd_last_error(pd_ctx *ctx);

/* Kernel shapes. Every solve, plan, stream and request of the loop picks
 * its shape — the q-block length K of the recurrence (FP32: 32, 64, 96, 128,
 * 160, 192; FP64: 16, 32), the atom-chunk length of a tile (multiple of 32)
 * and the pairs each thread advances together (FP32: 1, 2 or 4) — from the
 * context's tuning table by the request's bucket: (precision, accumulation
 * mode (class or weighted), one frame or several, floor(log2 n_atoms),
 * floor(log2 nq)); a bucket without an entry takes a default shape. No
 * reference counterpart (the reference has one CPU loop shape).
 *
 * pd_ctx_create loads the table from the file named by the environment
 * variable PRIPPS_DEBYE_TUNING (where the autotuner then also saves its
 * results), else from data/tuning_b200.txt beside the library when present.
 * The file is text, one bucket per line:
 *   <fp32|fp64> <class|weighted> <single|frames> <log2 atoms> <log2 nq>
 *   <q_block> <j_chunk> <pairs_per_thread> <ms>
 *
 * pd_autotune_request times every candidate shape on the caller's own
 * request (its structure, solvent model and grid; no lattice sets), each
 * timed execution after an L2 flush, stores the fastest for the request's
 * bucket (of the shapes within 0.3 % of the fastest time, the one that holds
 * the least device memory) and returns it with its time; pd_autotune does the same on a
 * synthetic solvent globule of n_atoms atoms (class mode, one frame). Both
 * run on the context's stream: do not overlap them with other work on the
 * context. pd_get_tuning / pd_set_tuning read and write the class-mode,
 * one-frame bucket of (n_atoms, nq, precision); pd_tuning_lookup reports the
 * shape a request would get and whether it came from the table (host-only).
 * Calls without a context (pd_solve_noalloc, and the host-only queries with
 * ctx = NULL) use the table a new context would load, read once per
 * process. pd_tuning_load adds a file's entries to the
 * context's table, pd_tuning_save writes the table; pd_tuning_check parses a
 * tuning file without a context (host-only) and counts its entries. */
int pd_get_tuning(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision,
                  uint32_t *q_block, uint32_t *j_chunk, uint32_t *pairs_per_thread);
int pd_set_tuning(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision,
                  uint32_t q_block, uint32_t j_chunk, uint32_t pairs_per_thread);
int pd_autotune(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision);
int pd_autotune_request(pd_ctx *ctx, const pd_request *req, uint32_t *q_block,
                        uint32_t *j_chunk, uint32_t *pairs_per_thread, double *ms);
int pd_tuning_lookup(pd_ctx *ctx, const pd_request *req, uint32_t *q_block, uint32_t *j_chunk,
                     uint32_t *pairs_per_thread, int *from_table);
int pd_tuning_load(pd_ctx *ctx, const char *path);
int pd_tuning_save(pd_ctx *ctx, const char *path);
int pd_tuning_check(const char *path, uint64_t *n_entries);

/* Host-only planning report for a request (no device work): number of atom
 * classes (species × hydration weight), padded atom count, tiles launched and
 * the unordered pairs those tiles cover in total, which must equal
 * N(N-1)/2. ctx may be NULL (default tuning). */
int pd_plan_inspect(pd_ctx *ctx, const pd_request *req, uint64_t *n_classes,
                    uint64_t *n_padded, uint64_t *n_tiles, uint64_t *pairs_covered);

/* Host-only: device bytes one solve of `req` holds with the tuning the
 * context would pick (ctx may be NULL: default tuning). host_coordinates != 0
 * counts the device copy of the coordinates that pd_solve and pd_submit make;
 * 0 is the layout of a plan execution or of pd_solve_noalloc, whose
 * coordinates are the caller's device memory. No reference counterpart. */
int pd_request_device_bytes(pd_ctx *ctx, const pd_request *req, int host_coordinates,
                            uint64_t *device_bytes);

/* Measured FP32 issue peak of the device: FFMA throughput of a register-only
 * microbenchmark, in TFLOP/s at the clock the device runs during the call. */
int pd_measure_fp32_peak(pd_ctx *ctx, double *tflops_ffma, double *tflops_ffma2);

/* Number of kernel launches the context has issued since creation. */
uint64_t pd_launch_count(pd_ctx *ctx);

/* ---- allocation-free solve ----
 * No counterpart in the reference (it has no device memory to manage).
 *
 * Some callers cannot allocate device memory when they call in: a process
 * whose framework owns all device memory through its own allocator or
 * reserved pool (a cudaMalloc there fails or fragments the pool), a latency-
 * critical serving loop where cudaMalloc/cudaFree would synchronise the
 * device and stall every other stream, or a plug-in loaded into a host whose
 * memory policy it does not control. For them pd_solve_noalloc runs one
 * solve using only a fixed scratch array compiled into the library, of
 * PD_NOALLOC_SCRATCH_BYTES bytes. It calls no cudaMalloc, cudaFree, pool or
 * pinned-host allocation (the host planner itself uses ordinary heap memory).
 *
 * Inputs and outputs stay the caller's: `req` is read as HOST memory except
 * req->xyz, which is ignored; the coordinates are xyz_dev, DEVICE memory
 * [n_frames][N][3]; the [6][nq] result (or the frame-weighted mean) is
 * written to out_terms_dev, DEVICE memory. The work is enqueued on `stream`
 * (a cudaStream_t of the current device; NULL = legacy default stream) and
 * the call returns without waiting for it. It uploads the request's tables
 * and tile list from host memory that lives only during the call, so it
 * cannot be captured into a CUDA graph: on a stream that is capturing it
 * returns PD_EINVAL before any device work. Because it does not wait, a
 * device-side failure cannot be returned: a bounded wait inside the pair
 * kernel that expired leaves NaN in the affected rows of out_terms_dev, so
 * check the result for NaN after synchronising the stream.
 *
 * Limits and sharing:
 *  - A request whose device layout (tables, tile list, packed atoms, tile
 *    partial sums) needs more than PD_NOALLOC_SCRATCH_BYTES fails with
 *    PD_EBUDGET and a message naming both sizes, before any device work.
 *    pd_request_device_bytes(ctx, req, 0, &bytes) gives a request's need
 *    beforehand; the need depends on the atom classes and on the j chunk
 *    the tuning table picks for the request's bucket as well as on N and
 *    nq. As a guide, at nq = 1,000 an FP32 solve with solvent and one
 *    hydration weight per element fits up to roughly 130,000 atoms (the
 *    100,000-atom ellipsoid needs 49 MB) and 200,000 atoms are refused;
 *    with a hydration weight per atom (four partial sums per grid point)
 *    up to about 20,000 atoms fit, and larger requests may not.
 *  - The array occupies PD_NOALLOC_SCRATCH_BYTES of memory on every GPU that
 *    loads the library's device code, until the process exits.
 *  - Every call shares the array, which keeps the previous call's contents;
 *    the call overwrites or zeroes everything it reads. Calls whose device
 *    work overlaps (two streams, or two host threads with different streams)
 *    race on the array: serialise them on one stream.
 *  - The first call on each device (the current one) looks up the array's
 *    device address and the SM count; make that first call before any stream
 *    capture on that device.
 */
#define PD_NOALLOC_SCRATCH_BYTES (64ull << 20)
int pd_solve_noalloc(const pd_request *req, const double *xyz_dev, double *out_terms_dev,
                     void *stream);

#ifdef __cplusplus
}
#endif
#endif /* PRIPPS_DEBYE_H */
