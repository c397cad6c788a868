// C ABI of the Debye backend: context, device arena, plan upload and
// execution, blocking solve, the continuous-batching request loop, the
// autotuner and the FP32 peak probe. Declarations and contracts are in
// include/pripps_debye.h.
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <random>
#include <string>
#include <thread>
#include <tuple>
#include <unordered_map>
#include <vector>

#include "pd_common.h"
#include "pd_kernels.h"
#include "pd_plan.h"
#include "pd_tuning.h"
#include "pripps_debye.h"

#include <dlfcn.h>
#include <nvtx3/nvToolsExt.h>

using pd::Plan;
using pd::Tuning;

namespace {

std::mutex g_err_mu;
std::string g_err;  // context-free failures (pd_ctx_create)

double now_s() {
    using clk = std::chrono::steady_clock;
    static const clk::time_point t0 = clk::now();
    return std::chrono::duration<double>(clk::now() - t0).count();
}

inline uint64_t align_up(uint64_t v, uint64_t a) { return (v + a - 1) / a * a; }

// NVTX range over a host phase (planning, upload, the launches of each
// kernel stage, the request loop's admission, steps and finishes), so that a
// profiler timeline lines the host work up with the kernels it launched.
// Without a profiler attached a range costs a few nanoseconds.
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

// Offsets of every array of one request inside its single device chunk. The
// first `upload_bytes` bytes mirror a host staging image uploaded with one
// copy; the rest is device-only scratch.
struct Layout {
    uint64_t qv, ffA, ffC, ffW, hw, fw, cls, pairs, perm, gvalid, jobs, lptr, lidx, req, njobs,
        xyz, lat, lat_tiles;
    uint64_t upload_bytes;
    uint64_t hres;         // host-only: pinned landing area of the [6][nq] result
    uint64_t stage_bytes;  // pinned image size (upload + result area)
    uint64_t centroid, radius, atoms, slots, pairsum, terms, out, counter;
    uint64_t status;  // int32 device status of the pair kernel, right after out
    uint64_t lat_idx, hist, lat_err;  // lattice sets: coordinates, pair counts, error flag
    uint64_t total;
};

Layout make_layout(const Plan &P, bool host_xyz) {
    Layout L{};
    uint64_t o = 0;
    auto take = [&](uint64_t bytes) {
        const uint64_t at = o;
        o = align_up(o + std::max<uint64_t>(bytes, 1), 256);
        return at;
    };
    const uint64_t nq = P.nq, S = P.n_species;
    L.qv = take(nq * 8);
    L.ffA = take(S * nq * 8);
    L.ffC = take(P.has_exc ? S * nq * 8 : 0);
    L.ffW = take(P.has_hyd ? nq * 8 : 0);
    L.hw = take(P.has_hyd ? static_cast<uint64_t>(P.n_atoms) * 8 : 0);
    L.fw = take(static_cast<uint64_t>(P.n_frames) * 8);
    L.cls = take(P.cls.size() * sizeof(PdClassDev));
    L.pairs = take(P.pairs.size() * sizeof(PdPairDev));
    L.perm = take(P.perm.size() * 4);
    L.gvalid = take(P.gvalid.size() * 4);
    L.jobs = take(P.jobs.size() * sizeof(PdJob));
    L.lptr = take(P.lptr.size() * 8);
    L.lidx = take(P.lidx.size() * 8);
    L.req = take(sizeof(PdReqDev));
    L.njobs = take(sizeof(int));
    L.xyz = take(host_xyz ? static_cast<uint64_t>(P.n_atoms) * 3 * P.n_frames * 8 : 0);
    L.lat = take(P.lat.size() * sizeof(PdLatDev));
    L.lat_tiles = take(P.lat_tiles.size() * sizeof(PdLatTile));
    L.upload_bytes = o;
    L.hres = o;
    L.stage_bytes = align_up(o + 6 * nq * 8 + 8, 256);  // result and status land here
    L.centroid = take(static_cast<uint64_t>(P.n_frames) * 3 * 8);
    L.radius = take(static_cast<uint64_t>(P.n_frames) * 8);
    L.atoms = take(static_cast<uint64_t>(P.n_pad) * P.n_frames *
                   (P.precision == PD_FP64 ? sizeof(double4) : sizeof(float4)));
    L.slots = take(static_cast<uint64_t>(P.slots_per_frame) * P.n_frames * P.nv * P.tun.K * 8);
    L.pairsum = take(static_cast<uint64_t>(P.n_frames) * P.nv * P.n_pairs * nq * 8);
    L.terms = take(static_cast<uint64_t>(P.n_frames) * 6 * nq * 8);
    L.out = take(6 * nq * 8 + 8);
    L.status = L.out + 6 * nq * 8;
    L.counter = take(sizeof(int) * 4);
    L.lat_idx = take(P.lat.empty() ? 0 : static_cast<uint64_t>(P.n_pad) * sizeof(int4));
    L.hist = take(static_cast<uint64_t>(P.lat_bins) * 8);
    L.lat_err = take(sizeof(int));
    L.total = o;
    return L;
}

}  // namespace

// ---------------------------------------------------------------- context
struct PdTicket;

namespace {

// Pinned host blocks in power-of-two size classes, reused across requests:
// admitting and retiring a request then calls neither cudaHostAlloc nor
// cudaFreeHost (which waits for the whole device). Blocks go back to the pool
// only once no copy of theirs can be in flight.
struct PinnedPool {
    std::mutex mu;
    std::map<uint64_t, std::vector<char *>> free_blocks;
    std::vector<char *> all;

    static uint64_t size_class(uint64_t bytes) {
        uint64_t c = uint64_t{64} << 10;
        while (c < bytes) c <<= 1;
        return c;
    }
    cudaError_t get(uint64_t bytes, char **out, uint64_t *cls) {
        const uint64_t c = size_class(bytes);
        {
            std::lock_guard<std::mutex> g(mu);
            auto it = free_blocks.find(c);
            if (it != free_blocks.end() && !it->second.empty()) {
                *out = it->second.back();
                it->second.pop_back();
                *cls = c;
                return cudaSuccess;
            }
        }
        char *p = nullptr;
        const cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&p), c, cudaHostAllocDefault);
        if (e != cudaSuccess) return e;
        std::lock_guard<std::mutex> g(mu);
        all.push_back(p);
        *out = p;
        *cls = c;
        return cudaSuccess;
    }
    void put(char *p, uint64_t cls) {
        std::lock_guard<std::mutex> g(mu);
        free_blocks[cls].push_back(p);
    }
    void release() {
        std::lock_guard<std::mutex> g(mu);
        for (char *p : all) cudaFreeHost(p);
        all.clear();
        free_blocks.clear();
    }
};

}  // namespace

struct pd_ctx {
    int device = 0;
    int sm_count = 0;
    uint64_t budget = 0;
    std::atomic<uint64_t> in_use{0};
    std::atomic<uint64_t> launches{0};
    cudaStream_t stream = nullptr;  // blocking solves and the request loop
    cudaMemPool_t pool = nullptr;
    PinnedPool pinned;              // staging images of planned requests

    std::mutex mu;  // tuning table, per-thread errors
    pd::TuneTable tuning;     // kernel shape per request bucket
    std::string tuning_path;  // file the autotuner's results are saved to ("" = none)
    std::unordered_map<std::thread::id, std::string> errors;
    std::mutex solve_mu;  // serialises blocking solves on `stream`

    // request loop
    std::mutex qmu;
    std::condition_variable qcv;
    std::condition_variable done_cv;
    std::deque<uint64_t> pending;                       // admission order
    std::deque<std::shared_ptr<PdTicket>> to_plan;      // awaiting host planning
    std::condition_variable plan_cv;
    std::map<uint64_t, std::shared_ptr<PdTicket>> tickets;
    uint64_t next_ticket = 1;
    bool stop = false;
    std::thread worker;
    std::vector<std::thread> planners;  // host planning, PD_PLANNERS threads
    bool worker_started = false;

    void set_error(const std::string &m) {
        std::lock_guard<std::mutex> g(mu);
        errors[std::this_thread::get_id()] = m;
    }
};

namespace {

int cuda_fail(pd_ctx *ctx, cudaError_t e, const char *what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    if (ctx) ctx->set_error(m);
    return PD_EDEVICE;
}

#define PD_CUDA(ctx, call)                                  \
    do {                                                    \
        cudaError_t e__ = (call);                           \
        if (e__ != cudaSuccess) return cuda_fail(ctx, e__, #call); \
    } while (0)

// One planned request resident on the device.
struct DevPlan {
    Plan P;
    Layout L{};
    char *base = nullptr;   // device chunk
    char *stage = nullptr;  // pinned host image of the uploaded part
    uint64_t stage_cls = 0; // its size class in the context's pinned pool
    uint64_t charged = 0;
    bool host_xyz = false;
    const double *xyz_dev = nullptr;  // coordinates used by pack
    // Tile share of a multi-GPU solve: the tiles in the device job list are
    // this rank's; rank 0 adds the i = j terms and the exact q = 0 sums.
    uint32_t rank = 0, world = 1;
    // Finish with the unnormalised frame sum Σ_f w_f·T_f instead of the mean
    // (streamed trajectories add batches before dividing once).
    bool frame_sum = false;
    template <class T>
    T *dptr(uint64_t off) const {
        return reinterpret_cast<T *>(base + off);
    }
    template <class T>
    T *hptr(uint64_t off) const {
        return reinterpret_cast<T *>(stage + off);
    }
};

// The tuning table a context starts from: the file named by
// PRIPPS_DEBYE_TUNING, else data/tuning_b200.txt beside this library.
int load_default_tuning(pd::TuneTable &tab, bool *from_env, std::string &msg) {
    std::string path;
    const char *env = std::getenv("PRIPPS_DEBYE_TUNING");
    *from_env = env && *env;
    if (*from_env) {
        path = env;
    } else {
        Dl_info info{};
        if (dladdr(reinterpret_cast<void *>(&load_default_tuning), &info) && info.dli_fname) {
            const std::string so = info.dli_fname;
            const size_t slash = so.rfind('/');
            path = (slash == std::string::npos ? std::string(".") : so.substr(0, slash)) +
                   "/data/tuning_b200.txt";
        }
    }
    if (path.empty()) return PD_ENOTFOUND;
    return pd::load_tuning(path, tab, msg);
}

// Calls without a context (pd_solve_noalloc, host-only queries with NULL)
// use the table a new context would load, read once per process.
const pd::TuneTable &process_tuning() {
    static pd::TuneTable tab;
    static std::once_flag once;
    std::call_once(once, [] {
        std::string msg;
        bool from_env = false;
        pd::TuneTable t;
        if (load_default_tuning(t, &from_env, msg) == PD_OK) tab = std::move(t);
    });
    return tab;
}

// Kernel shape for a request bucket: the tuning table entry (the
// autotuner's measurement, loaded from a tuning file or set by hand) of the
// context, or of the process without one; else the default shape.
Tuning tuning_for(pd_ctx *ctx, int64_t n, int64_t nq, int precision, int64_t n_frames, int mode,
                  bool *from_table = nullptr) {
    if (from_table) *from_table = false;
    const pd::TuneKey key = pd::tune_key(n, nq, precision, mode, n_frames);
    if (ctx) {
        std::lock_guard<std::mutex> g(ctx->mu);
        auto it = ctx->tuning.find(key);
        if (it != ctx->tuning.end()) {
            if (from_table) *from_table = true;
            return it->second.t;
        }
    } else {
        const pd::TuneTable &tab = process_tuning();
        auto it = tab.find(key);
        if (it != tab.end()) {
            if (from_table) *from_table = true;
            return it->second.t;
        }
    }
    return pd::fit_tuning(precision, mode, pd::default_tuning(n, nq, precision, n_frames));
}

Tuning tuning_for_request(pd_ctx *ctx, const pd_request *req, const uint32_t *species,
                          const double *weights, bool *from_table = nullptr) {
    return tuning_for(ctx, static_cast<int64_t>(req->n_atoms), static_cast<int64_t>(req->nq),
                      static_cast<int>(req->precision),
                      static_cast<int64_t>(req->n_frames ? req->n_frames : 1),
                      pd::request_mode(req, species, weights), from_table);
}

void free_devplan(pd_ctx *ctx, DevPlan &dp, cudaStream_t st) {
    if (dp.base) cudaFreeAsync(dp.base, st);
    if (dp.stage) ctx->pinned.put(dp.stage, dp.stage_cls);
    dp.base = nullptr;
    dp.stage = nullptr;
    if (dp.charged) ctx->in_use.fetch_sub(dp.charged);
    dp.charged = 0;
}

// A request with lattice sets whose result came back NaN had a point off its
// lattice (the device flags it that way; see pd_lattice in pripps_debye.h).
bool lattice_failed(const Plan &P, const double *terms) {
    if (P.lat.empty()) return false;
    for (size_t i = 0; i < static_cast<size_t>(6) * P.nq; ++i)
        if (std::isnan(terms[i])) return true;
    return false;
}
constexpr const char *kLatticeMsg =
    "a point of a lattice species lies off its lattice (by more than 1e-6 spacing) or outside "
    "its extents";
constexpr const char *kExpiredMsg =
    "a bounded wait in the pair kernel expired (a bulk copy of atoms into shared memory did not "
    "complete); the result is invalid";

// The outcome of a finished solve from the pair kernel's status word and the
// host result: an expired wait, then a point off its lattice.
int result_status(pd_ctx *ctx, const Plan &P, int32_t status, const double *terms) {
    if (status & PD_DEV_WAIT_EXPIRED) {
        if (ctx) ctx->set_error(kExpiredMsg);
        return PD_ETIMEOUT;
    }
    if (terms && lattice_failed(P, terms)) {
        if (ctx) ctx->set_error(kLatticeMsg);
        return PD_EINVAL;
    }
    return PD_OK;
}

// Fill the pinned staging image (tables, layout, tiles, lists, descriptor).
// Sizes of the request-derived regions of the staging image (tables,
// weights, coordinates), which a re-staged plan copies unchanged.
struct InputRegions {
    uint64_t off[7];
    uint64_t bytes[7];
};
InputRegions input_regions(const DevPlan &dp) {
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    const uint64_t tab = static_cast<uint64_t>(P.n_species) * P.nq * 8;
    return InputRegions{
        {L.qv, L.ffA, L.ffC, L.ffW, L.hw, L.fw, L.xyz},
        {static_cast<uint64_t>(P.nq) * 8, tab, P.has_exc ? tab : 0,
         P.has_hyd ? static_cast<uint64_t>(P.nq) * 8 : 0,
         P.has_hyd ? static_cast<uint64_t>(P.n_atoms) * 8 : 0,
         static_cast<uint64_t>(P.n_frames) * 8,
         dp.host_xyz ? static_cast<uint64_t>(P.n_atoms) * 3 * P.n_frames * 8 : 0}};
}

// The plan-derived part of the staging image: classes, layout, tiles,
// reduction lists, lattice descriptors and the request descriptor.
void stage_structure(DevPlan &dp);

int stage_plan(pd_ctx *ctx, DevPlan &dp, const pd_request *req) {
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    std::memcpy(dp.hptr<double>(L.qv), P.qv.data(), P.qv.size() * 8);
    const size_t tab = static_cast<size_t>(P.n_species) * P.nq;
    std::memcpy(dp.hptr<double>(L.ffA), req->ff_atoms, tab * 8);
    if (P.has_exc) std::memcpy(dp.hptr<double>(L.ffC), req->ff_excluded, tab * 8);
    if (P.has_hyd) {
        std::memcpy(dp.hptr<double>(L.ffW), req->ff_water, static_cast<size_t>(P.nq) * 8);
        std::memcpy(dp.hptr<double>(L.hw), req->hyd_weights, static_cast<size_t>(P.n_atoms) * 8);
    }
    double *fw = dp.hptr<double>(L.fw);
    for (int f = 0; f < P.n_frames; ++f) fw[f] = req->frame_weights ? req->frame_weights[f] : 1.0;
    if (dp.host_xyz)
        std::memcpy(dp.hptr<double>(L.xyz), req->xyz,
                    static_cast<size_t>(P.n_atoms) * 3 * P.n_frames * 8);
    stage_structure(dp);
    (void)ctx;
    return PD_OK;
}

void stage_structure(DevPlan &dp) {
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    std::memcpy(dp.hptr<char>(L.cls), P.cls.data(), P.cls.size() * sizeof(PdClassDev));
    std::memcpy(dp.hptr<char>(L.pairs), P.pairs.data(), P.pairs.size() * sizeof(PdPairDev));
    std::memcpy(dp.hptr<char>(L.perm), P.perm.data(), P.perm.size() * 4);
    std::memcpy(dp.hptr<char>(L.gvalid), P.gvalid.data(), P.gvalid.size() * 4);
    std::memcpy(dp.hptr<char>(L.jobs), P.jobs.data(), P.jobs.size() * sizeof(PdJob));
    std::memcpy(dp.hptr<char>(L.lptr), P.lptr.data(), P.lptr.size() * 8);
    std::memcpy(dp.hptr<char>(L.lidx), P.lidx.data(), P.lidx.size() * 8);
    if (!P.lat.empty()) {
        std::memcpy(dp.hptr<char>(L.lat), P.lat.data(), P.lat.size() * sizeof(PdLatDev));
        std::memcpy(dp.hptr<char>(L.lat_tiles), P.lat_tiles.data(),
                    P.lat_tiles.size() * sizeof(PdLatTile));
    }
    PdReqDev rd{};
    if (P.precision == PD_FP64)
        rd.atoms64 = dp.dptr<double4>(L.atoms);
    else
        rd.atoms32 = dp.dptr<float4>(L.atoms);
    rd.gvalid = dp.dptr<int32_t>(L.gvalid);
    rd.qv = dp.dptr<double>(L.qv);
    rd.slots = dp.dptr<double>(L.slots);
    rd.radius = dp.dptr<double>(L.radius);
    rd.status = dp.dptr<int32_t>(L.status);
    rd.flags = P.test_expire ? PD_REQF_TEST_EXPIRE : 0;
    rd.qmin = P.qmin;
    rd.dq = P.dq;
    rd.n_pad = P.n_pad;
    rd.nq = P.nq;
    rd.K = P.tun.K;
    rd.mode = P.mode;
    std::memcpy(dp.hptr<char>(L.req), &rd, sizeof(rd));
    const int nj = static_cast<int>(P.jobs.size());
    std::memcpy(dp.hptr<char>(L.njobs), &nj, sizeof(int));
}

constexpr int kBudgetWait = -100;  // internal: does not fit the budget right now

// Host planning only: tiles, lists and the device layout.
int plan_host(pd_ctx *ctx, const pd_request *req, const uint32_t *species, const double *weights,
              bool host_xyz, DevPlan &dp, const Tuning *force = nullptr) {
    NvtxRange nvtx("pd plan (host)");
    std::string msg;
    const Tuning tun = force ? *force : tuning_for_request(ctx, req, species, weights);
    int rc = pd::build_plan(req, species, weights, tun, dp.P, msg);
    if (rc != PD_OK) {
        ctx->set_error(msg);
        return rc;
    }
    dp.host_xyz = host_xyz;
    dp.L = make_layout(dp.P, host_xyz);
    if (dp.L.total > ctx->budget) {
        ctx->set_error("request needs " + std::to_string(dp.L.total) +
                       " device bytes, the budget is " + std::to_string(ctx->budget));
        return PD_EBUDGET;
    }
    return PD_OK;
}

// Charge the budget, allocate the device chunk and the pinned image, stage and
// upload. With `wait` a full budget returns kBudgetWait (retry after frees);
// without it a full budget is PD_EBUDGET.
int plan_device(pd_ctx *ctx, const pd_request *req, DevPlan &dp, cudaStream_t st, bool wait) {
    NvtxRange nvtx("pd upload");
    const uint64_t need = dp.L.total;
    uint64_t cur = ctx->in_use.load();
    for (;;) {
        if (cur + need > ctx->budget) {
            if (wait) return kBudgetWait;
            ctx->set_error("device memory budget exhausted");
            return PD_EBUDGET;
        }
        if (ctx->in_use.compare_exchange_weak(cur, cur + need)) break;
    }
    dp.charged = need;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&dp.base), need, ctx->pool, st);
    if (e != cudaSuccess) {
        free_devplan(ctx, dp, st);
        ctx->set_error(std::string("device allocation failed: ") + cudaGetErrorString(e));
        return PD_ENOMEM;
    }
    e = ctx->pinned.get(dp.L.stage_bytes, &dp.stage, &dp.stage_cls);
    if (e != cudaSuccess) {
        free_devplan(ctx, dp, st);
        ctx->set_error(std::string("pinned allocation failed: ") + cudaGetErrorString(e));
        return PD_ENOMEM;
    }
    stage_plan(ctx, dp, req);
    e = cudaMemcpyAsync(dp.base, dp.stage, dp.L.upload_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(dp.base + dp.L.status, 0, 8, st);
    if (e != cudaSuccess) {
        free_devplan(ctx, dp, st);
        return cuda_fail(ctx, e, "plan upload");
    }
    if (dp.host_xyz) dp.xyz_dev = dp.dptr<double>(dp.L.xyz);
    return PD_OK;
}

int create_devplan(pd_ctx *ctx, const pd_request *req, const uint32_t *species,
                   const double *weights, bool host_xyz, DevPlan &dp, cudaStream_t st,
                   const Tuning *force = nullptr) {
    int rc = plan_host(ctx, req, species, weights, host_xyz, dp, force);
    if (rc) return rc;
    return plan_device(ctx, req, dp, st, false);
}

// Everything after the pair kernel: slot reduction, six-profile combine and
// the frame mean; leaves the [6][nq] result at L.out (or out_dev).
int finish_devplan(pd_ctx *ctx, DevPlan &dp, double *out_dev, cudaStream_t st) {
    NvtxRange nvtx("pd reduce + combine");
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    PD_CUDA(ctx, pd::launch_reduce(dp.dptr<double>(L.slots), dp.dptr<int64_t>(L.lptr),
                                   dp.dptr<int64_t>(L.lidx), dp.dptr<PdPairDev>(L.pairs),
                                   dp.dptr<double>(L.qv), P.n_pairs, P.nq, P.tun.K, P.nv,
                                   P.n_frames, P.slots_per_frame, dp.dptr<double>(L.radius),
                                   P.qmin, P.dq, P.precision == PD_FP32_FP64RED ? 1 : 0,
                                   dp.rank == 0 ? 1 : 0, dp.dptr<double>(L.pairsum), st));
    if (!P.lat.empty()) {
        PD_CUDA(ctx, pd::launch_lattice_sums(
                         reinterpret_cast<const unsigned long long *>(dp.dptr<char>(L.hist)),
                         dp.dptr<PdLatDev>(L.lat), static_cast<int>(P.lat.size()),
                         dp.dptr<double>(L.qv), P.nq, dp.rank == 0 ? 1 : 0,
                         dp.dptr<int>(L.lat_err), dp.dptr<double>(L.pairsum), st));
        ctx->launches += 1;
    }
    PD_CUDA(ctx, pd::launch_combine(dp.dptr<double>(L.pairsum), dp.dptr<PdClassDev>(L.cls),
                                    dp.dptr<PdPairDev>(L.pairs), P.n_cls, P.n_pairs, P.nq, P.nv,
                                    P.n_frames, dp.dptr<double>(L.ffA),
                                    P.has_exc ? dp.dptr<double>(L.ffC) : nullptr,
                                    P.has_hyd ? dp.dptr<double>(L.ffW) : nullptr,
                                    dp.rank == 0 ? 1 : 0, dp.dptr<double>(L.terms), st));
    ctx->launches += 2;
    double *dst = out_dev ? out_dev : dp.dptr<double>(L.out);
    if (P.n_frames > 1) {
        PD_CUDA(ctx, pd::launch_frame_mean(dp.dptr<double>(L.terms), dp.dptr<double>(L.fw),
                                           P.n_frames, P.nq, dst, st, !dp.frame_sum));
        ctx->launches += 1;
    } else {
        PD_CUDA(ctx, cudaMemcpyAsync(dst, dp.dptr<double>(L.terms),
                                     static_cast<size_t>(6) * P.nq * 8,
                                     cudaMemcpyDeviceToDevice, st));
    }
    return PD_OK;
}

// centroid + pack of the coordinates into the padded class layout.
int pack_devplan(pd_ctx *ctx, DevPlan &dp, cudaStream_t st) {
    NvtxRange nvtx("pd pack");
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    PD_CUDA(ctx, pd::launch_centroid(dp.xyz_dev, P.n_atoms, P.n_frames, dp.dptr<double>(L.centroid),
                                     dp.dptr<double>(L.radius), st));
    PD_CUDA(ctx, pd::launch_pack(dp.xyz_dev, P.has_hyd ? dp.dptr<double>(L.hw) : nullptr,
                                 dp.dptr<int32_t>(L.perm), dp.dptr<double>(L.centroid), P.n_atoms,
                                 P.n_pad, P.n_frames,
                                 P.precision == PD_FP64 ? nullptr : dp.dptr<float4>(L.atoms),
                                 P.precision == PD_FP64 ? dp.dptr<double4>(L.atoms) : nullptr, st));
    ctx->launches += 2;
    if (!P.lat.empty()) {
        PD_CUDA(ctx, pd::launch_lattice(dp.xyz_dev, dp.dptr<int32_t>(L.perm),
                                        dp.dptr<PdLatDev>(L.lat), P.lat.data(),
                                        static_cast<int>(P.lat.size()),
                                        dp.dptr<PdLatTile>(L.lat_tiles),
                                        static_cast<int64_t>(P.lat_tiles.size()),
                                        dp.dptr<int4>(L.lat_idx),
                                        reinterpret_cast<unsigned long long *>(dp.dptr<char>(L.hist)),
                                        P.lat_bins, dp.dptr<int>(L.lat_err), st));
        ctx->launches += P.lat_tiles.empty() ? 1 : 2;
    }
    return PD_OK;
}

int persistent_grid(pd_ctx *ctx, const Plan &P, int64_t n_jobs) {
    const int per_sm =
        std::max(1, pd::pairs_blocks_per_sm(P.precision, P.tun.K, P.tun.NP, P.mode));
    const int64_t g = std::min<int64_t>(n_jobs, static_cast<int64_t>(ctx->sm_count) * per_sm);
    return static_cast<int>(std::max<int64_t>(g, 1));
}

// The whole device pipeline of one plan on stream st; ev (optional) brackets
// the pair kernel.
int run_devplan(pd_ctx *ctx, DevPlan &dp, double *out_dev, cudaStream_t st,
                std::pair<cudaEvent_t, cudaEvent_t> *ev = nullptr) {
    const Plan &P = dp.P;
    const Layout &L = dp.L;
    int rc = pack_devplan(ctx, dp, st);
    if (rc) return rc;
    // a streamed trajectory keeps the status of all its batches
    if (!dp.frame_sum) PD_CUDA(ctx, cudaMemsetAsync(dp.base + L.status, 0, 8, st));
    if (ev) cudaEventRecord(ev->first, st);
    if (dp.world > 1)  // a frame's slot may be written by another rank's tile only
        PD_CUDA(ctx, cudaMemsetAsync(dp.dptr<double>(L.slots), 0,
                                     static_cast<size_t>(P.slots_per_frame) * P.n_frames * P.nv *
                                         P.tun.K * 8,
                                     st));
    if (!P.jobs.empty()) {
        NvtxRange nvtx("pd pair kernel");
        PD_CUDA(ctx, cudaMemsetAsync(dp.dptr<int>(L.counter), 0, sizeof(int), st));
        PD_CUDA(ctx, pd::launch_pairs(P.precision, P.tun.K, P.tun.NP, P.mode, dp.dptr<PdJob>(L.jobs),
                                      dp.dptr<int>(L.njobs), dp.dptr<PdReqDev>(L.req),
                                      dp.dptr<int>(L.counter),
                                      persistent_grid(ctx, P, static_cast<int64_t>(P.jobs.size())),
                                      st));
        ctx->launches += 1;
    }
    if (ev) cudaEventRecord(ev->second, st);
    return finish_devplan(ctx, dp, out_dev, st);
}

}  // namespace

// ---------------------------------------------------------------- plan API
struct pd_plan {
    DevPlan dp;
    std::unique_ptr<Plan> full;  // the whole plan, kept once a shard replaces it
    bool profiling = false;
    std::vector<std::pair<cudaEvent_t, cudaEvent_t>> pair_events;  // one per execution
};

// ---------------------------------------------------------------- request loop
struct PdTicket {
    uint64_t id = 0;
    pd_request req{};                 // pointers below own the copies
    std::vector<double> xyz, ffA, ffC, hw, ffW, fw;
    std::vector<uint32_t> species;
    std::vector<pd_lattice> lats;
    DevPlan dp;
    int status = 1;                   // 1 pending/running, 0 done, < 0 error
    int plan_state = 0;               // host planning: 0 not yet, 1 done, < 0 failed (code)
    std::string plan_err;
    bool admitted = false;
    bool canceled = false;
    bool taken = false;               // result copied out by pd_wait
    size_t next_job = 0;              // first tile not yet issued
    bool express_wait = false;        // small: waits for a free express lane
    bool finish_issued = false;       // reduction (or, if cancelled, the drain) enqueued
    bool drained_only = false;        // cancelled after admission: no reduction was run
    uint32_t used_streams = 0;        // lane streams that ran some of its tiles
    cudaEvent_t done_ev = nullptr;
    std::vector<double> result;
    std::string err;
    double t_submit = 0, t_admit = 0, t_done = 0;
};

namespace {

// One lane of a step buffer: the tiles of one kernel variant, their request
// descriptors and the counter of the persistent kernel, uploaded from pinned
// memory and run by a captured graph (upload, counter reset, pair kernel) on
// the lane's own stream.
struct Lane {
    PdJob *h_jobs = nullptr, *d_jobs = nullptr;
    PdReqDev *h_reqs = nullptr, *d_reqs = nullptr;
    int *h_n = nullptr, *d_n = nullptr;
    int *d_counter = nullptr;
    cudaStream_t st = nullptr;
    cudaEvent_t ev = nullptr;  // recorded after the lane's last launch
    bool busy = false;         // ev pending: h_* may still be read by the upload
    std::map<std::tuple<int, int, int, int>, cudaGraphExec_t> graphs;  // (precision, K, NP, mode)
};

#ifndef PD_STEP_COST
#define PD_STEP_COST 4.0e10
#endif
constexpr int STEP_BUFS = 2;       // steps in flight
constexpr int STEP_LANES = 4;      // kernel variants per step
constexpr size_t STEP_MAX_JOBS = 1 << 14;
constexpr size_t STEP_MAX_REQS = 1024;
constexpr double STEP_COST = PD_STEP_COST;  // ≈ 5 ms of FP32 class-mode work per step
constexpr double RR_QUANTUM = 1.0e9;   // work a request adds per round-robin turn
// Requests of at most this much work (≈1.4 ms alone) skip the steps: at
// admission their tiles go to an express lane whose stream has the highest
// priority, so its CTAs take the first SM slots that the running step frees.
// (1e11 measured worse: 400 requests at once 5.87e12 against 6.81e12
// pair·q/s, p99 of the 10,000-request stream at 60/s 396 against 312 ms.)
#ifndef PD_EXPRESS_COST
#define PD_EXPRESS_COST 1.0e10
#endif
constexpr double EXPRESS_COST = PD_EXPRESS_COST;
// A small request waits for a free express lane at most this long (s) before
// it joins the steps. When many arrive at once (a burst admitted in one pass)
// the four lanes serve them in admission order, a launch of each lane taking
// every waiting request of its variant that fits, instead of sending the
// overflow into the round-robin steps beside the large requests.
#ifndef PD_EXPRESS_MAX_WAIT
#define PD_EXPRESS_MAX_WAIT 0.25
#endif
constexpr double EXPRESS_MAX_WAIT = PD_EXPRESS_MAX_WAIT;
constexpr int EXPRESS = STEP_BUFS;  // row of the express lanes
static_assert((STEP_BUFS + 1) * STEP_LANES <= 32, "lane bits of PdTicket::used_streams");

// Relative cost of one pair·q of a tile (FP32 class mode = 1).
double tile_cost(const Plan &P, const PdJob &jb) {
    double c = static_cast<double>(PD_IBLOCK) * (jb.j1 - jb.j0) * P.tun.K;
    if (P.precision == PD_FP64) c *= 24.0;
    if (P.mode == PD_MODE_WEIGHTED) c *= 1.5;
    return c;
}

int lane_graph(pd_ctx *ctx, Lane &ln, int precision, int K, int NP, int mode,
               cudaGraphExec_t *out) {
    auto key = std::make_tuple(precision, K, NP, mode);
    auto it = ln.graphs.find(key);
    if (it != ln.graphs.end()) {
        *out = it->second;
        return PD_OK;
    }
    Plan dummy;
    dummy.precision = precision;
    dummy.tun.K = K;
    dummy.tun.NP = NP;
    dummy.mode = mode;
    const int grid = persistent_grid(ctx, dummy, 1 << 30);
    cudaGraph_t g = nullptr;
    PD_CUDA(ctx, cudaStreamBeginCapture(ln.st, cudaStreamCaptureModeThreadLocal));
    cudaMemcpyAsync(ln.d_n, ln.h_n, sizeof(int), cudaMemcpyHostToDevice, ln.st);
    cudaMemcpyAsync(ln.d_reqs, ln.h_reqs, STEP_MAX_REQS * sizeof(PdReqDev), cudaMemcpyHostToDevice,
                    ln.st);
    cudaMemcpyAsync(ln.d_jobs, ln.h_jobs, STEP_MAX_JOBS * sizeof(PdJob), cudaMemcpyHostToDevice,
                    ln.st);
    cudaMemsetAsync(ln.d_counter, 0, sizeof(int), ln.st);
    pd::launch_pairs(precision, K, NP, mode, ln.d_jobs, ln.d_n, ln.d_reqs, ln.d_counter, grid,
                     ln.st);
    PD_CUDA(ctx, cudaStreamEndCapture(ln.st, &g));
    cudaGraphExec_t ge = nullptr;
    cudaError_t e = cudaGraphInstantiate(&ge, g, 0);
    cudaGraphDestroy(g);
    if (e != cudaSuccess) return cuda_fail(ctx, e, "cudaGraphInstantiate");
    ln.graphs[key] = ge;
    *out = ge;
    return PD_OK;
}

// Host planning of submitted requests, taken in submission order, off the
// loop thread: the loop keeps issuing steps while a large request is planned.
// Several planner threads plan consecutive requests at once (admission still
// takes them in submission order), so a burst of submissions is planned at a
// multiple of one core's rate: 400 requests of the serving stream take about
// 0.3 s of planning on one core.
#ifndef PD_PLANNERS
#define PD_PLANNERS 4
#endif
void planner_main(pd_ctx *ctx) {
    for (;;) {
        std::shared_ptr<PdTicket> t;
        {
            std::unique_lock<std::mutex> lk(ctx->qmu);
            ctx->plan_cv.wait(lk, [&] { return ctx->stop || !ctx->to_plan.empty(); });
            if (ctx->stop) return;
            t = ctx->to_plan.front();
            ctx->to_plan.pop_front();
        }
        int rc = PD_OK;
        std::string m;
        if (!t->canceled) {
            rc = plan_host(ctx, &t->req, t->req.species, t->req.hyd_weights, true, t->dp);
            if (rc != PD_OK) {
                std::lock_guard<std::mutex> g(ctx->mu);
                m = ctx->errors[std::this_thread::get_id()];
            }
        }
        {
            std::lock_guard<std::mutex> lk(ctx->qmu);
            t->plan_err = m;
            t->plan_state = rc == PD_OK ? 1 : rc;
        }
        ctx->qcv.notify_all();
    }
}

// The device request loop. Streams: `sa` admits (device chunk from the pool,
// upload, pack), each lane of each step buffer runs its tiles, `sf` finishes
// (slot reduction, combine, result download). Lanes wait for the admission
// event; a request's finish waits for the lanes that ran its tiles. Steps on
// different buffers overlap on the GPU, so the tail of one persistent kernel
// is filled by the next.
void worker_main(pd_ctx *ctx) {
    cudaSetDevice(ctx->device);
    cudaStream_t sa = nullptr, sf = nullptr;
    cudaEvent_t ev_admit = nullptr;
    bool init_ok = cudaStreamCreateWithFlags(&sa, cudaStreamNonBlocking) == cudaSuccess &&
                   cudaStreamCreateWithFlags(&sf, cudaStreamNonBlocking) == cudaSuccess &&
                   cudaEventCreateWithFlags(&ev_admit, cudaEventDisableTiming) == cudaSuccess;
    Lane lanes[STEP_BUFS + 1][STEP_LANES];  // step buffers, then the express row
    int prio_least = 0, prio_greatest = 0;
    cudaDeviceGetStreamPriorityRange(&prio_least, &prio_greatest);
    for (int b = 0; b <= STEP_BUFS; ++b)
        for (auto &ln : lanes[b]) {
            if (!init_ok) break;
            init_ok &= cudaHostAlloc(reinterpret_cast<void **>(&ln.h_jobs), STEP_MAX_JOBS * sizeof(PdJob), 0) == cudaSuccess;
            init_ok &= cudaHostAlloc(reinterpret_cast<void **>(&ln.h_reqs), STEP_MAX_REQS * sizeof(PdReqDev), 0) == cudaSuccess;
            init_ok &= cudaHostAlloc(reinterpret_cast<void **>(&ln.h_n), sizeof(int), 0) == cudaSuccess;
            init_ok &= cudaMalloc(reinterpret_cast<void **>(&ln.d_jobs), STEP_MAX_JOBS * sizeof(PdJob)) == cudaSuccess;
            init_ok &= cudaMalloc(reinterpret_cast<void **>(&ln.d_reqs), STEP_MAX_REQS * sizeof(PdReqDev)) == cudaSuccess;
            init_ok &= cudaMalloc(reinterpret_cast<void **>(&ln.d_n), sizeof(int)) == cudaSuccess;
            init_ok &= cudaMalloc(reinterpret_cast<void **>(&ln.d_counter), sizeof(int)) == cudaSuccess;
            init_ok &= cudaStreamCreateWithPriority(&ln.st, cudaStreamNonBlocking,
                                                    b == EXPRESS ? prio_greatest : prio_least) ==
                       cudaSuccess;
            init_ok &= cudaEventCreateWithFlags(&ln.ev, cudaEventDisableTiming) == cudaSuccess;
        }
    auto lane_of_bit = [&](int bit) -> Lane & { return lanes[bit / STEP_LANES][bit % STEP_LANES]; };
    auto sync_all = [&] {
        if (sa) cudaStreamSynchronize(sa);
        if (sf) cudaStreamSynchronize(sf);
        for (auto &buf : lanes)
            for (auto &ln : buf)
                if (ln.st) cudaStreamSynchronize(ln.st);
    };
    auto fail = [&](const std::shared_ptr<PdTicket> &t, int code, const std::string &m) {
        sync_all();  // nothing of the request may still be in flight when its memory returns
        std::lock_guard<std::mutex> lk(ctx->qmu);
        t->status = code;
        t->err = m;
        t->t_done = now_s();
        if (t->dp.base || t->dp.stage) free_devplan(ctx, t->dp, sa);
        ctx->done_cv.notify_all();
    };

    std::vector<std::shared_ptr<PdTicket>> active;  // admitted, in admission order
    bool admit_recorded = false;
    int cur = 0;
    size_t rr = 0;
    for (;;) {
        std::vector<std::shared_ptr<PdTicket>> head;  // planned front of the queue
        {
            std::unique_lock<std::mutex> lk(ctx->qmu);
            bool waiting_device = false;
            for (auto &t : active) waiting_device |= t->finish_issued;
            if (active.empty() && !ctx->stop) {
                bool ready = false;
                for (uint64_t id : ctx->pending) ready |= ctx->tickets[id]->plan_state != 0;
                if (!ready) ctx->qcv.wait_for(lk, std::chrono::milliseconds(50));
            }
            if (ctx->stop) break;
            // drop cancelled pending tickets
            for (auto it = ctx->pending.begin(); it != ctx->pending.end();) {
                auto t = ctx->tickets[*it];
                if (t->canceled) {
                    t->status = PD_ECANCELED;
                    t->t_done = now_s();
                    it = ctx->pending.erase(it);
                    ctx->done_cv.notify_all();
                } else {
                    ++it;
                }
            }
            for (uint64_t id : ctx->pending) {
                auto t = ctx->tickets[id];
                if (t->plan_state == 0) break;  // FIFO: wait for its planning
                head.push_back(t);
            }
            (void)waiting_device;
        }
        if (!init_ok) {
            std::lock_guard<std::mutex> lk(ctx->qmu);
            for (auto &t : head) {
                t->status = PD_ENOMEM;
                t->err = "request loop could not allocate its streams and step buffers";
                t->t_done = now_s();
                ctx->pending.erase(std::find(ctx->pending.begin(), ctx->pending.end(), t->id));
            }
            ctx->done_cv.notify_all();
            if (head.empty()) std::this_thread::sleep_for(std::chrono::milliseconds(1));
            continue;
        }
        nvtxRangePushA("pd admit");
        // ---- admission in FIFO order while the budget allows
        bool admitted_now = false;
        for (auto &t : head) {
            int rc = t->plan_state < 0 ? t->plan_state : PD_OK;
            if (rc == PD_OK) rc = plan_device(ctx, &t->req, t->dp, sa, /*wait=*/true);
            if (rc == kBudgetWait) break;  // keep FIFO order; retry after frees
            {
                std::lock_guard<std::mutex> lk(ctx->qmu);
                ctx->pending.pop_front();
            }
            if (rc != PD_OK) {
                std::string m = t->plan_err;
                if (m.empty()) {
                    std::lock_guard<std::mutex> g(ctx->mu);
                    m = ctx->errors[std::this_thread::get_id()];
                }
                fail(t, rc, m);
                continue;
            }
            if (pack_devplan(ctx, t->dp, sa) != PD_OK) {
                fail(t, PD_EDEVICE, "pack failed");
                continue;
            }
            {
                // small enough for an express lane?
                const Plan &P = t->dp.P;
                double cost = 0;
                for (const PdJob &jb : P.jobs) {
                    cost += tile_cost(P, jb);
                    if (cost > EXPRESS_COST) break;
                }
                t->express_wait =
                    !P.jobs.empty() && cost <= EXPRESS_COST && P.jobs.size() <= STEP_MAX_JOBS;
            }
            // the device and the pinned image hold the inputs now
            t->xyz = {};
            t->ffA = {};
            t->ffC = {};
            t->hw = {};
            t->ffW = {};
            t->fw = {};
            t->species = {};
            t->admitted = true;
            t->t_admit = now_s();
            active.push_back(t);
            admitted_now = true;
        }
        if (admitted_now) {
            cudaEventRecord(ev_admit, sa);
            admit_recorded = true;
        }

        nvtxRangePop();
        nvtxRangePushA("pd express + step");
        // ---- express: small requests, in admission order, get all their
        // tiles on a free express lane of their kernel variant; one that
        // finds none waits for the next pass, up to EXPRESS_MAX_WAIT, then
        // takes the steps
        {
            Lane *ex = lanes[EXPRESS];
            std::tuple<int, int, int, int> ex_key[STEP_LANES];
            std::vector<std::shared_ptr<PdTicket>> ex_members[STEP_LANES];
            size_t ex_nj[STEP_LANES] = {0, 0, 0, 0};
            bool ex_used[STEP_LANES] = {false, false, false, false};
            const double now = now_s();
            for (auto &t : active) {
                if (!t->express_wait) continue;
                const Plan &P = t->dp.P;
                if (t->canceled || t->next_job != 0) {
                    t->express_wait = false;
                    continue;
                }
                const auto key = std::make_tuple(P.precision, P.tun.K, P.tun.NP, P.mode);
                int l = -1;
                for (int c = 0; c < STEP_LANES && l < 0; ++c)
                    if (ex_used[c] && ex_key[c] == key && ex_nj[c] + P.jobs.size() <= STEP_MAX_JOBS &&
                        ex_members[c].size() < STEP_MAX_REQS)
                        l = c;
                for (int c = 0; c < STEP_LANES && l < 0; ++c) {
                    if (ex_used[c]) continue;
                    if (ex[c].busy) {
                        if (cudaEventQuery(ex[c].ev) != cudaSuccess) continue;
                        ex[c].busy = false;  // its previous launch (and upload) is done
                    }
                    if (P.jobs.size() > STEP_MAX_JOBS) break;
                    ex_used[c] = true;
                    ex_key[c] = key;
                    l = c;
                }
                if (l < 0) {
                    if (now - t->t_admit > EXPRESS_MAX_WAIT) t->express_wait = false;
                    continue;
                }
                t->express_wait = false;
                const int slot = static_cast<int>(ex_members[l].size());
                ex_members[l].push_back(t);
                for (; t->next_job < P.jobs.size(); ++t->next_job) {
                    PdJob jb = P.jobs[t->next_job];
                    jb.req = slot;
                    ex[l].h_jobs[ex_nj[l]++] = jb;
                }
            }
            for (int l = 0; l < STEP_LANES; ++l) {
                if (!ex_used[l]) continue;
                Lane &ln = ex[l];
                for (size_t m = 0; m < ex_members[l].size(); ++m)
                    std::memcpy(&ln.h_reqs[m],
                                ex_members[l][m]->dp.hptr<char>(ex_members[l][m]->dp.L.req),
                                sizeof(PdReqDev));
                *ln.h_n = static_cast<int>(ex_nj[l]);
                cudaGraphExec_t ge = nullptr;
                int rc = lane_graph(ctx, ln, std::get<0>(ex_key[l]), std::get<1>(ex_key[l]),
                                    std::get<2>(ex_key[l]), std::get<3>(ex_key[l]), &ge);
                if (rc == PD_OK && cudaStreamWaitEvent(ln.st, ev_admit, 0) != cudaSuccess)
                    rc = PD_EDEVICE;
                if (rc == PD_OK && cudaGraphLaunch(ge, ln.st) == cudaSuccess &&
                    cudaEventRecord(ln.ev, ln.st) == cudaSuccess) {
                    ctx->launches += 1;
                    ln.busy = true;
                    const uint32_t bit = 1u << (EXPRESS * STEP_LANES + l);
                    for (auto &t : ex_members[l]) t->used_streams |= bit;
                } else {
                    for (auto &t : ex_members[l]) fail(t, PD_EDEVICE, "express launch failed");
                }
            }
        }

        // ---- one step: round-robin turns of RR_QUANTUM over the issuable
        // requests (rotating start), each request's tiles into the lane of
        // its kernel variant; up to STEP_LANES variants per step.
        std::vector<std::shared_ptr<PdTicket>> cand;
        for (auto &t : active)
            if (!t->canceled && !t->express_wait && t->next_job < t->dp.P.jobs.size())
                cand.push_back(t);
        Lane *step = lanes[cur];
        std::tuple<int, int, int, int> lane_key[STEP_LANES];
        std::vector<std::shared_ptr<PdTicket>> members[STEP_LANES];
        size_t nj[STEP_LANES] = {0, 0, 0, 0};
        int n_lanes = 0;
        if (!cand.empty()) {
            std::vector<int> lane_of(cand.size(), -1), slot_of(cand.size(), -1);
            double work = 0;
            bool progress = true;
            const size_t start = rr % cand.size();
            while (progress && work < STEP_COST) {
                progress = false;
                for (size_t c = 0; c < cand.size() && work < STEP_COST; ++c) {
                    const size_t ci = (start + c) % cand.size();
                    auto &t = cand[ci];
                    const Plan &P = t->dp.P;
                    if (t->next_job >= P.jobs.size()) continue;
                    if (lane_of[ci] < 0) {
                        const auto key = std::make_tuple(P.precision, P.tun.K, P.tun.NP, P.mode);
                        int l = 0;
                        while (l < n_lanes && lane_key[l] != key) ++l;
                        if (l == n_lanes) {
                            if (n_lanes == STEP_LANES) continue;  // next step
                            Lane &ln = step[l];
                            // a lane still running its previous step is not
                            // waited for (the loop polls again): its request
                            // and any new variant take a later step
                            if (ln.busy) {
                                if (cudaEventQuery(ln.ev) != cudaSuccess) continue;
                                ln.busy = false;
                            }
                            lane_key[n_lanes++] = key;
                        }
                        if (members[l].size() >= STEP_MAX_REQS) continue;
                        lane_of[ci] = l;
                        slot_of[ci] = static_cast<int>(members[l].size());
                        members[l].push_back(t);
                    }
                    const int l = lane_of[ci];
                    Lane &ln = step[l];
                    double turn = 0;
                    while (t->next_job < P.jobs.size() && nj[l] < STEP_MAX_JOBS &&
                           turn < RR_QUANTUM) {
                        PdJob jb = P.jobs[t->next_job++];
                        turn += tile_cost(P, jb);
                        jb.req = slot_of[ci];
                        ln.h_jobs[nj[l]++] = jb;
                        progress = true;
                    }
                    work += turn;
                }
            }
            rr = start + 1;
        }
        bool launch_failed = false;
        for (int l = 0; l < n_lanes; ++l) {
            Lane &ln = step[l];
            for (size_t m = 0; m < members[l].size(); ++m)
                std::memcpy(&ln.h_reqs[m], members[l][m]->dp.hptr<char>(members[l][m]->dp.L.req),
                            sizeof(PdReqDev));
            *ln.h_n = static_cast<int>(nj[l]);
            cudaGraphExec_t ge = nullptr;
            int rc = lane_graph(ctx, ln, std::get<0>(lane_key[l]), std::get<1>(lane_key[l]),
                                std::get<2>(lane_key[l]), std::get<3>(lane_key[l]), &ge);
            if (rc == PD_OK && admit_recorded) {
                if (cudaStreamWaitEvent(ln.st, ev_admit, 0) != cudaSuccess) rc = PD_EDEVICE;
            }
            if (rc == PD_OK && cudaGraphLaunch(ge, ln.st) == cudaSuccess &&
                cudaEventRecord(ln.ev, ln.st) == cudaSuccess) {
                ctx->launches += 1;
                ln.busy = true;
                const uint32_t bit = 1u << (cur * STEP_LANES + l);
                for (auto &t : members[l]) t->used_streams |= bit;
            } else {
                launch_failed = true;
                for (auto &t : members[l]) fail(t, PD_EDEVICE, "step launch failed");
            }
        }
        if (n_lanes) cur = (cur + 1) % STEP_BUFS;
        (void)launch_failed;

        nvtxRangePop();
        nvtxRangePushA("pd finish + retire");
        // ---- finish requests whose tiles are all issued (or drain cancelled ones)
        for (auto &t : active) {
            if (t->status != 1 || t->finish_issued) continue;
            const bool all_issued = t->next_job >= t->dp.P.jobs.size();
            if (!all_issued && !t->canceled) continue;
            if (admit_recorded) cudaStreamWaitEvent(sf, ev_admit, 0);
            for (int bit = 0; bit < (STEP_BUFS + 1) * STEP_LANES; ++bit)
                if (t->used_streams & (1u << bit)) cudaStreamWaitEvent(sf, lane_of_bit(bit).ev, 0);
            if (t->canceled) {
                t->drained_only = true;
            } else {
                if (finish_devplan(ctx, t->dp, nullptr, sf) != PD_OK) {
                    fail(t, PD_EDEVICE, "reduction launch failed");
                    continue;
                }
                // the result and the pair kernel's status word behind it
                cudaMemcpyAsync(t->dp.hptr<double>(t->dp.L.hres), t->dp.dptr<double>(t->dp.L.out),
                                static_cast<size_t>(6) * t->dp.P.nq * 8 + 8,
                                cudaMemcpyDeviceToHost, sf);
            }
            if (cudaEventCreateWithFlags(&t->done_ev, cudaEventDisableTiming) != cudaSuccess ||
                cudaEventRecord(t->done_ev, sf) != cudaSuccess) {
                fail(t, PD_EDEVICE, "event record failed");
                continue;
            }
            t->finish_issued = true;
        }

        // ---- retire finished and cancelled requests
        for (auto it = active.begin(); it != active.end();) {
            auto &t = *it;
            bool remove = false;
            if (t->status < 0) {
                remove = true;
            } else if (t->finish_issued) {
                const cudaError_t q = cudaEventQuery(t->done_ev);
                if (q == cudaSuccess) {
                    cudaEventDestroy(t->done_ev);
                    t->done_ev = nullptr;
                    int rs = PD_OK;
                    if (!t->drained_only) {
                        const double *res = t->dp.hptr<double>(t->dp.L.hres);
                        const size_t n6 = static_cast<size_t>(6) * t->dp.P.nq;
                        t->result.assign(res, res + n6);
                        int32_t dev_status = 0;
                        std::memcpy(&dev_status, res + n6, sizeof(int32_t));
                        rs = result_status(nullptr, t->dp.P, dev_status, res);
                    }
                    free_devplan(ctx, t->dp, sa);
                    std::lock_guard<std::mutex> lk(ctx->qmu);
                    t->status = t->drained_only ? PD_ECANCELED : rs;
                    if (rs == PD_ETIMEOUT) t->err = kExpiredMsg;
                    if (rs == PD_EINVAL) t->err = kLatticeMsg;
                    t->t_done = now_s();
                    ctx->done_cv.notify_all();
                    remove = true;
                } else if (q != cudaErrorNotReady) {
                    fail(t, PD_EDEVICE, std::string("device error: ") + cudaGetErrorString(q));
                    remove = true;
                }
            }
            it = remove ? active.erase(it) : it + 1;
        }

        nvtxRangePop();
        // ---- nothing to issue: wait briefly for a submission or the GPU
        bool issuable = false;
        for (auto &t : active)
            if (!t->canceled && t->next_job < t->dp.P.jobs.size()) issuable = true;
        if (!issuable && !active.empty()) {
            std::unique_lock<std::mutex> lk(ctx->qmu);
            bool ready = false;
            for (uint64_t id : ctx->pending) ready |= ctx->tickets[id]->plan_state != 0;
            if (!ready && !ctx->stop) ctx->qcv.wait_for(lk, std::chrono::microseconds(200));
        } else if (issuable && n_lanes == 0) {
            // no lane of the step buffer was free: poll again in 100 µs, or at
            // once when a request is submitted or planned
            std::unique_lock<std::mutex> lk(ctx->qmu);
            if (!ctx->stop) ctx->qcv.wait_for(lk, std::chrono::microseconds(100));
        }
    }
    sync_all();
    for (auto &t : active) {
        if (t->done_ev) cudaEventDestroy(t->done_ev);
        free_devplan(ctx, t->dp, sa);
    }
    if (sa) cudaStreamSynchronize(sa);
    for (auto &buf : lanes)
        for (auto &ln : buf) {
            for (auto &kv : ln.graphs) cudaGraphExecDestroy(kv.second);
            if (ln.h_jobs) cudaFreeHost(ln.h_jobs);
            if (ln.h_reqs) cudaFreeHost(ln.h_reqs);
            if (ln.h_n) cudaFreeHost(ln.h_n);
            if (ln.d_jobs) cudaFree(ln.d_jobs);
            if (ln.d_reqs) cudaFree(ln.d_reqs);
            if (ln.d_n) cudaFree(ln.d_n);
            if (ln.d_counter) cudaFree(ln.d_counter);
            if (ln.ev) cudaEventDestroy(ln.ev);
            if (ln.st) cudaStreamDestroy(ln.st);
        }
    if (ev_admit) cudaEventDestroy(ev_admit);
    if (sa) cudaStreamDestroy(sa);
    if (sf) cudaStreamDestroy(sf);
}

}  // namespace

// ====================================================================== ABI
extern "C" {

int pd_ctx_create(int device, uint64_t mem_budget_bytes, pd_ctx **out) {
    if (!out) return PD_EINVAL;
    *out = nullptr;
    int count = 0;
    cudaError_t e = cudaGetDeviceCount(&count);
    if (e != cudaSuccess || device < 0 || device >= count) {
        std::lock_guard<std::mutex> g(g_err_mu);
        g_err = std::string("no CUDA device ") + std::to_string(device) +
                (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : std::string());
        return PD_ENODEV;
    }
    cudaDeviceProp prop{};
    cudaGetDeviceProperties(&prop, device);
    if (prop.major < 10) {
        std::lock_guard<std::mutex> g(g_err_mu);
        g_err = "device " + std::to_string(device) + " is sm_" + std::to_string(prop.major) +
                std::to_string(prop.minor) + "; this library is built for sm_100a";
        return PD_ENODEV;
    }
    auto *ctx = new pd_ctx();
    ctx->device = device;
    ctx->sm_count = prop.multiProcessorCount;
    cudaSetDevice(device);
    size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    ctx->budget = mem_budget_bytes ? mem_budget_bytes : static_cast<uint64_t>(free_b * 0.9);
    e = pd::prepare_pair_kernels();
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&ctx->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) {
        cudaMemPoolProps pp{};
        pp.allocType = cudaMemAllocationTypePinned;
        pp.handleTypes = cudaMemHandleTypeNone;
        pp.location.type = cudaMemLocationTypeDevice;
        pp.location.id = device;
        e = cudaMemPoolCreate(&ctx->pool, &pp);
        if (e == cudaSuccess) {
            uint64_t thr = UINT64_MAX;
            cudaMemPoolSetAttribute(ctx->pool, cudaMemPoolAttrReleaseThreshold, &thr);
        }
    }
    if (e != cudaSuccess) {
        std::lock_guard<std::mutex> g(g_err_mu);
        g_err = std::string("context setup failed: ") + cudaGetErrorString(e);
        if (ctx->stream) cudaStreamDestroy(ctx->stream);
        delete ctx;
        return PD_EDEVICE;
    }
    // Tuning table: the file named by PRIPPS_DEBYE_TUNING (the autotuner
    // also saves its results there), else the table shipped beside the
    // library. A missing file leaves the defaults; a malformed one fails the
    // context.
    {
        std::string msg;
        bool from_env = false;
        const int trc = load_default_tuning(ctx->tuning, &from_env, msg);
        if (from_env) ctx->tuning_path = std::getenv("PRIPPS_DEBYE_TUNING");
        if (trc != PD_OK && trc != PD_ENOTFOUND) {
            std::lock_guard<std::mutex> g(g_err_mu);
            g_err = msg;
            cudaStreamDestroy(ctx->stream);
            if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
            delete ctx;
            return trc;
        }
    }
    *out = ctx;
    return PD_OK;
}

void pd_ctx_destroy(pd_ctx *ctx) {
    if (!ctx) return;
    {
        std::lock_guard<std::mutex> lk(ctx->qmu);
        ctx->stop = true;
        for (auto &kv : ctx->tickets)
            if (kv.second->status == 1) kv.second->canceled = true;
    }
    ctx->qcv.notify_all();
    ctx->plan_cv.notify_all();
    if (ctx->worker_started) {
        ctx->worker.join();
        for (auto &th : ctx->planners) th.join();
    }
    {
        std::lock_guard<std::mutex> lk(ctx->qmu);
        for (auto &kv : ctx->tickets)
            if (kv.second->status == 1) kv.second->status = PD_ECANCELED;
        ctx->done_cv.notify_all();
    }
    cudaSetDevice(ctx->device);
    cudaStreamSynchronize(ctx->stream);
    cudaStreamDestroy(ctx->stream);
    ctx->pinned.release();
    if (ctx->pool) cudaMemPoolDestroy(ctx->pool);
    delete ctx;
}

const char *pd_last_error(pd_ctx *ctx) {
    static thread_local std::string copy;
    if (!ctx) {
        std::lock_guard<std::mutex> g(g_err_mu);
        copy = g_err;
        return copy.c_str();
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    auto it = ctx->errors.find(std::this_thread::get_id());
    copy = it == ctx->errors.end() ? std::string() : it->second;
    return copy.c_str();
}

int pd_solve(pd_ctx *ctx, const pd_request *req, double *out_terms) {
    if (!ctx || !out_terms) return PD_EINVAL;
    NvtxRange nvtx("pd_solve");
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    DevPlan dp;
    rc = create_devplan(ctx, req, req->species, req->hyd_weights, true, dp, ctx->stream);
    if (rc) return rc;
    rc = run_devplan(ctx, dp, nullptr, ctx->stream);
    if (rc == PD_OK) {
        int32_t dev_status = 0;
        cudaError_t e = cudaMemcpyAsync(out_terms, dp.dptr<double>(dp.L.out),
                                        static_cast<size_t>(6) * dp.P.nq * 8,
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&dev_status, dp.base + dp.L.status, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "pd_solve");
        if (rc == PD_OK) rc = result_status(ctx, dp.P, dev_status, out_terms);
    }
    free_devplan(ctx, dp, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return rc;
}

namespace {
int plan_create_impl(pd_ctx *ctx, const pd_request *req, pd_plan **out, const Tuning *force);
}

int pd_plan_create(pd_ctx *ctx, const pd_request *req, pd_plan **out) {
    return plan_create_impl(ctx, req, out, nullptr);
}

namespace {
int plan_create_impl(pd_ctx *ctx, const pd_request *req, pd_plan **out, const Tuning *force) {
    if (!ctx || !out || !req) return PD_EINVAL;
    *out = nullptr;
    // Coordinates arrive at execute time; validate the rest on the host.
    pd_request r = *req;
    static const double zero3[3] = {0, 0, 0};
    std::vector<double> dummy;
    const uint64_t nf = r.n_frames ? r.n_frames : 1;
    if (!r.xyz) {
        dummy.assign(static_cast<size_t>(r.n_atoms) * 3 * nf, 0.0);
        r.xyz = dummy.data();
    }
    (void)zero3;
    std::string msg;
    int rc = pd::validate_request(&r, false, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    auto *p = new pd_plan();
    rc = create_devplan(ctx, &r, r.species, r.hyd_weights, false, p->dp, ctx->stream, force);
    if (rc == PD_OK) {
        cudaError_t e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "pd_plan_create");
    }
    if (rc) {
        free_devplan(ctx, p->dp, ctx->stream);
        delete p;
        return rc;
    }
    *out = p;
    return PD_OK;
}
}  // namespace

int pd_plan_execute(pd_ctx *ctx, pd_plan *plan, const double *xyz_dev, double *out_terms_dev,
                    void *stream) {
    if (!ctx || !plan || !xyz_dev || !out_terms_dev) return PD_EINVAL;
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    cudaSetDevice(ctx->device);
    plan->dp.xyz_dev = xyz_dev;
    if (!plan->profiling) return run_devplan(ctx, plan->dp, out_terms_dev, st);
    std::pair<cudaEvent_t, cudaEvent_t> ev{nullptr, nullptr};
    PD_CUDA(ctx, cudaEventCreate(&ev.first));
    PD_CUDA(ctx, cudaEventCreate(&ev.second));
    plan->pair_events.push_back(ev);
    return run_devplan(ctx, plan->dp, out_terms_dev, st, &plan->pair_events.back());
}

int pd_plan_set_profiling(pd_ctx *ctx, pd_plan *plan, int enable) {
    if (!ctx || !plan) return PD_EINVAL;
    cudaSetDevice(ctx->device);
    for (auto &e : plan->pair_events) {
        cudaEventSynchronize(e.second);
        cudaEventDestroy(e.first);
        cudaEventDestroy(e.second);
    }
    plan->pair_events.clear();
    plan->profiling = enable != 0;
    return PD_OK;
}

int pd_plan_pair_kernel_ms(pd_ctx *ctx, pd_plan *plan, double *total_ms, uint64_t *n_launches) {
    if (!ctx || !plan) return PD_EINVAL;
    cudaSetDevice(ctx->device);
    double tot = 0.0;
    for (auto &e : plan->pair_events) {
        cudaError_t err = cudaEventSynchronize(e.second);
        if (err != cudaSuccess) return cuda_fail(ctx, err, "pd_plan_pair_kernel_ms");
        float ms = 0.0f;
        cudaEventElapsedTime(&ms, e.first, e.second);
        tot += ms;
    }
    if (total_ms) *total_ms = tot;
    if (n_launches) *n_launches = plan->pair_events.size();
    return PD_OK;
}

int pd_plan_execute_host(pd_ctx *ctx, pd_plan *plan, const double *xyz_host, double *out_terms) {
    if (!ctx || !plan || !xyz_host || !out_terms) return PD_EINVAL;
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    const Plan &P = plan->dp.P;
    const size_t nx = static_cast<size_t>(P.n_atoms) * 3 * P.n_frames;
    for (size_t i = 0; i < nx; ++i)
        if (!std::isfinite(xyz_host[i])) {
            ctx->set_error("non-finite coordinate at index " + std::to_string(i));
            return PD_EINVAL;
        }
    double *xyz_dev = nullptr;
    PD_CUDA(ctx, cudaMallocFromPoolAsync(reinterpret_cast<void **>(&xyz_dev), nx * 8, ctx->pool, ctx->stream));
    cudaMemcpyAsync(xyz_dev, xyz_host, nx * 8, cudaMemcpyHostToDevice, ctx->stream);
    plan->dp.xyz_dev = xyz_dev;
    int rc = run_devplan(ctx, plan->dp, nullptr, ctx->stream);
    if (rc == PD_OK) {
        int32_t dev_status = 0;
        cudaError_t e = cudaMemcpyAsync(out_terms, plan->dp.dptr<double>(plan->dp.L.out),
                                        static_cast<size_t>(6) * P.nq * 8,
                                        cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(&dev_status, plan->dp.base + plan->dp.L.status, sizeof(int32_t),
                                cudaMemcpyDeviceToHost, ctx->stream);
        if (e == cudaSuccess) e = cudaStreamSynchronize(ctx->stream);
        if (e != cudaSuccess) rc = cuda_fail(ctx, e, "pd_plan_execute_host");
        if (rc == PD_OK) rc = result_status(ctx, P, dev_status, out_terms);
    }
    cudaFreeAsync(xyz_dev, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    return rc;
}

void pd_plan_destroy(pd_ctx *ctx, pd_plan *plan) {
    if (!ctx || !plan) return;
    pd_plan_set_profiling(ctx, plan, 0);
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    // Executions may be in flight on caller streams.
    cudaDeviceSynchronize();
    free_devplan(ctx, plan->dp, ctx->stream);
    cudaStreamSynchronize(ctx->stream);
    delete plan;
}

int pd_plan_info(const pd_plan *plan, uint32_t *q_block, uint32_t *j_chunk, uint32_t *pairs_per_thread,
                 uint64_t *n_tiles, uint64_t *device_bytes, uint64_t *upload_bytes) {
    if (!plan) return PD_EINVAL;
    if (pairs_per_thread) *pairs_per_thread = static_cast<uint32_t>(plan->dp.P.tun.NP);
    if (upload_bytes) *upload_bytes = plan->dp.L.upload_bytes;
    if (q_block) *q_block = static_cast<uint32_t>(plan->dp.P.tun.K);
    if (j_chunk) *j_chunk = static_cast<uint32_t>(plan->dp.P.tun.TJ);
    if (n_tiles) *n_tiles = plan->dp.P.jobs.size();
    if (device_bytes) *device_bytes = plan->dp.L.total;
    return PD_OK;
}

int pd_plan_set_shard(pd_ctx *ctx, pd_plan *plan, uint32_t rank, uint32_t world) {
    if (!ctx || !plan || world == 0 || rank >= world) return PD_EINVAL;
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    DevPlan &dp = plan->dp;
    if (!plan->full) plan->full = std::make_unique<Plan>(dp.P);
    // A new device chunk holding only this rank's tiles, slots and lists;
    // the request's tables are copied from the current staging image.
    DevPlan nd;
    pd::shard_plan(*plan->full, rank, world, nd.P);
    nd.host_xyz = dp.host_xyz;
    nd.frame_sum = dp.frame_sum;
    nd.rank = rank;
    nd.world = world;
    nd.L = make_layout(nd.P, nd.host_xyz);
    cudaStream_t st = ctx->stream;
    // wait for executions of the old chunk first (they may be on caller streams)
    PD_CUDA(ctx, cudaDeviceSynchronize());
    const uint64_t need = nd.L.total;
    const uint64_t have = dp.charged;
    if (ctx->in_use.load() - have + need > ctx->budget) {
        ctx->set_error("sharded plan does not fit the memory budget");
        return PD_EBUDGET;
    }
    ctx->in_use.fetch_add(need);
    nd.charged = need;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&nd.base), need, ctx->pool, st);
    if (e == cudaSuccess) e = ctx->pinned.get(nd.L.stage_bytes, &nd.stage, &nd.stage_cls);
    if (e != cudaSuccess) {
        free_devplan(ctx, nd, st);
        return cuda_fail(ctx, e, "pd_plan_set_shard");
    }
    const InputRegions from = input_regions(dp), to = input_regions(nd);
    for (int r = 0; r < 7; ++r)
        if (from.bytes[r]) std::memcpy(nd.stage + to.off[r], dp.stage + from.off[r], from.bytes[r]);
    stage_structure(nd);
    e = cudaMemcpyAsync(nd.base, nd.stage, nd.L.upload_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(nd.base + nd.L.status, 0, 8, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e != cudaSuccess) {
        free_devplan(ctx, nd, st);
        return cuda_fail(ctx, e, "pd_plan_set_shard");
    }
    free_devplan(ctx, dp, st);
    cudaStreamSynchronize(st);
    dp = std::move(nd);
    nd.base = nullptr;
    nd.stage = nullptr;
    nd.charged = 0;
    return PD_OK;
}

int pd_plan_tiles(pd_ctx *ctx, const pd_request *req, uint32_t rank, uint32_t world,
                  int32_t *tiles, uint64_t cap, uint64_t *n_tiles, int32_t *perm,
                  uint64_t perm_cap, uint64_t *n_padded) {
    if (!req || world == 0 || rank >= world) return PD_EINVAL;
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    Tuning tun = tuning_for_request(ctx, req, req->species, req->hyd_weights);
    Plan P;
    rc = pd::build_plan(req, req->species, req->hyd_weights, tun, P, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    uint64_t n = 0;
    for (size_t t = rank; t < P.jobs.size(); t += world, ++n) {
        if (tiles && n < cap) {
            int32_t *o = tiles + 5 * n;
            o[0] = P.jobs[t].i0;
            o[1] = P.jobs[t].j0;
            o[2] = P.jobs[t].j1;
            o[3] = P.jobs[t].qb;
            o[4] = P.jobs[t].frame;
        }
    }
    if (n_tiles) *n_tiles = n;
    if (perm && perm_cap >= P.perm.size())
        std::memcpy(perm, P.perm.data(), P.perm.size() * sizeof(int32_t));
    if (n_padded) *n_padded = static_cast<uint64_t>(P.n_pad);
    if (tiles && n > cap) return PD_ENOMEM;
    return PD_OK;
}

int pd_submit(pd_ctx *ctx, const pd_request *req, uint64_t *ticket) {
    if (!ctx || !ticket) return PD_EINVAL;
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    auto t = std::make_shared<PdTicket>();
    const uint64_t n = req->n_atoms, nq = req->nq, S = req->n_species;
    const uint64_t nf = req->n_frames ? req->n_frames : 1;
    t->xyz.assign(req->xyz, req->xyz + n * 3 * nf);
    t->species.assign(req->species, req->species + n);
    t->ffA.assign(req->ff_atoms, req->ff_atoms + S * nq);
    if (req->ff_excluded) t->ffC.assign(req->ff_excluded, req->ff_excluded + S * nq);
    if (req->hyd_weights) {
        t->hw.assign(req->hyd_weights, req->hyd_weights + n);
        t->ffW.assign(req->ff_water, req->ff_water + nq);
    }
    if (req->frame_weights) t->fw.assign(req->frame_weights, req->frame_weights + nf);
    if (req->n_lattices) t->lats.assign(req->lattices, req->lattices + req->n_lattices);
    t->req = *req;
    t->req.lattices = t->lats.empty() ? nullptr : t->lats.data();
    t->req.xyz = t->xyz.data();
    t->req.species = t->species.data();
    t->req.ff_atoms = t->ffA.data();
    t->req.ff_excluded = req->ff_excluded ? t->ffC.data() : nullptr;
    t->req.hyd_weights = req->hyd_weights ? t->hw.data() : nullptr;
    t->req.ff_water = req->hyd_weights ? t->ffW.data() : nullptr;
    t->req.frame_weights = req->frame_weights ? t->fw.data() : nullptr;
    t->t_submit = now_s();
    {
        std::lock_guard<std::mutex> lk(ctx->qmu);
        if (!ctx->worker_started) {
            ctx->worker = std::thread(worker_main, ctx);
            const unsigned hw = std::max(1u, std::thread::hardware_concurrency());
            const int n_planners = std::max(1, std::min<int>(PD_PLANNERS, static_cast<int>(hw / 2)));
            for (int k = 0; k < n_planners; ++k)
                ctx->planners.emplace_back(planner_main, ctx);
            ctx->worker_started = true;
        }
        t->id = ctx->next_ticket++;
        ctx->tickets[t->id] = t;
        ctx->pending.push_back(t->id);
        ctx->to_plan.push_back(t);
        *ticket = t->id;
    }
    ctx->plan_cv.notify_all();
    ctx->qcv.notify_all();
    return PD_OK;
}

int pd_poll(pd_ctx *ctx, uint64_t ticket) {
    if (!ctx) return PD_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->qmu);
    auto it = ctx->tickets.find(ticket);
    if (it == ctx->tickets.end()) return PD_ENOTFOUND;
    const int s = it->second->status;
    return s == 0 ? 1 : (s == 1 ? 0 : s);
}

int pd_wait(pd_ctx *ctx, uint64_t ticket, int timeout_ms, double *out_terms) {
    if (!ctx) return PD_EINVAL;
    std::unique_lock<std::mutex> lk(ctx->qmu);
    auto it = ctx->tickets.find(ticket);
    if (it == ctx->tickets.end()) {
        ctx->set_error("unknown ticket " + std::to_string(ticket));
        return PD_ENOTFOUND;
    }
    auto t = it->second;
    auto pred = [&] { return t->status != 1; };
    if (timeout_ms < 0)
        ctx->done_cv.wait(lk, pred);
    else if (!ctx->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), pred)) {
        ctx->set_error("ticket " + std::to_string(ticket) + " still running");
        return PD_ETIMEOUT;
    }
    if (t->status < 0) {
        ctx->set_error(t->err.empty() ? "request failed" : t->err);
        return t->status;
    }
    if (out_terms) {
        if (t->taken) {
            ctx->set_error("the result of ticket " + std::to_string(ticket) + " was already taken");
            return PD_EINVAL;
        }
        std::memcpy(out_terms, t->result.data(), t->result.size() * 8);
        t->result = {};
        t->result.shrink_to_fit();
        t->taken = true;
    }
    return PD_OK;
}

int pd_cancel(pd_ctx *ctx, uint64_t ticket) {
    if (!ctx) return PD_EINVAL;
    {
        std::lock_guard<std::mutex> lk(ctx->qmu);
        auto it = ctx->tickets.find(ticket);
        if (it == ctx->tickets.end()) return PD_ENOTFOUND;
        if (it->second->status == 1) it->second->canceled = true;
    }
    ctx->qcv.notify_all();
    return PD_OK;
}

int pd_ticket_times(pd_ctx *ctx, uint64_t ticket, double *t_submit, double *t_admit,
                    double *t_done) {
    if (!ctx) return PD_EINVAL;
    std::lock_guard<std::mutex> lk(ctx->qmu);
    auto it = ctx->tickets.find(ticket);
    if (it == ctx->tickets.end()) return PD_ENOTFOUND;
    if (t_submit) *t_submit = it->second->t_submit;
    if (t_admit) *t_admit = it->second->t_admit;
    if (t_done) *t_done = it->second->t_done;
    return PD_OK;
}

int pd_combine(const double *terms, uint64_t nq, double vs, double c, double *total) {
    if (!terms || !total) return PD_EINVAL;
    for (uint64_t k = 0; k < nq; ++k) {
        // DebyeTerms::combine (src/debye.rs:187-194), same operation order.
        total[k] = terms[k] + vs * vs * terms[nq + k] + c * c * terms[2 * nq + k] -
                   2.0 * vs * terms[3 * nq + k] + 2.0 * c * terms[4 * nq + k] -
                   2.0 * vs * c * terms[5 * nq + k];
    }
    return PD_OK;
}

int pd_get_tuning(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision,
                  uint32_t *q_block, uint32_t *j_chunk, uint32_t *pairs_per_thread) {
    Tuning t = tuning_for(ctx, static_cast<int64_t>(n_atoms), static_cast<int64_t>(nq),
                          static_cast<int>(precision), 1, PD_MODE_CLASS);
    if (q_block) *q_block = static_cast<uint32_t>(t.K);
    if (j_chunk) *j_chunk = static_cast<uint32_t>(t.TJ);
    if (pairs_per_thread) *pairs_per_thread = static_cast<uint32_t>(t.NP);
    return PD_OK;
}

int pd_set_tuning(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision, uint32_t q_block,
                  uint32_t j_chunk, uint32_t pairs_per_thread) {
    if (!ctx) return PD_EINVAL;
    Tuning t;
    t.K = static_cast<int>(q_block);
    t.TJ = static_cast<int>(j_chunk);
    t.NP = precision == PD_FP64 ? 1 : static_cast<int>(pairs_per_thread);
    if (precision > PD_FP64 || !pd::valid_tuning(static_cast<int>(precision), PD_MODE_CLASS, t)) {
        ctx->set_error("invalid tuning");
        return PD_EINVAL;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->tuning[pd::tune_key(static_cast<int64_t>(n_atoms), static_cast<int64_t>(nq),
                             static_cast<int>(precision), PD_MODE_CLASS, 1)] = pd::TuneEntry{t, 0.0};
    return PD_OK;
}

namespace {

// Candidate shapes of a bucket: the instantiated (q block, pairs per thread)
// shapes of its precision and mode, each with j chunks of about N/32 .. N/4
// atoms (powers of two, 256 .. 16,384), and the default shape.
std::vector<Tuning> tune_candidates(const pd_request *req, int mode) {
    const int precision = static_cast<int>(req->precision);
    const int64_t n = static_cast<int64_t>(req->n_atoms), nq = static_cast<int64_t>(req->nq);
    std::vector<std::pair<int, int>> shapes;
    if (precision == PD_FP64)
        shapes = {{16, 1}, {32, 1}};
    else if (mode == PD_MODE_WEIGHTED)
        shapes = {{32, 2}, {64, 2}, {64, 4}};
    else if (nq <= 32)
        shapes = {{32, 4}};
    else
        shapes = {{64, 2}, {64, 4}, {96, 2}, {128, 1}, {128, 2}, {128, 4}};
    std::vector<int> tjs;
    for (int d : {32, 16, 8, 4, 2}) {
        int tj = 256;
        while (tj < n / d && tj < 65536) tj <<= 1;
        if (std::find(tjs.begin(), tjs.end(), tj) == tjs.end()) tjs.push_back(tj);
    }
    std::vector<Tuning> out;
    // every candidate as the planner would run it, so the table records the
    // shape that was timed
    const Tuning def = pd::fit_tuning(
        precision, mode, pd::default_tuning(n, nq, precision, static_cast<int64_t>(req->n_frames)));
    out.push_back(def);
    for (auto sh : shapes)
        for (int tj : tjs) {
            Tuning t;
            t.K = sh.first;
            t.NP = sh.second;
            t.TJ = tj;
            if (!pd::valid_tuning(precision, mode, t)) continue;
            bool dup = false;
            for (const Tuning &o : out) dup |= o.K == t.K && o.NP == t.NP && o.TJ == t.TJ;
            if (!dup) out.push_back(t);
        }
    return out;
}

// Times every candidate shape on the caller's request and keeps the fastest
// for the request's bucket. Each timed execution starts with L2 flushed (a
// 256 MiB write), as a stream of independent requests would meet it.
int autotune_request(pd_ctx *ctx, const pd_request *req, Tuning *best_out, double *best_ms) {
    NvtxRange nvtx("pd autotune");
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    if (req->n_lattices) {
        ctx->set_error("pd_autotune_request: tune the request without its lattice sets");
        return PD_EINVAL;
    }
    const int mode = pd::request_mode(req, req->species, req->hyd_weights);
    const std::vector<Tuning> cands = tune_candidates(req, mode);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const uint64_t nf = req->n_frames ? req->n_frames : 1;
    const size_t nxyz = static_cast<size_t>(req->n_atoms) * 3 * nf;
    const size_t flush_bytes = size_t{256} << 20;
    double *xyz_dev = nullptr, *out_dev = nullptr;
    char *flush = nullptr;
    cudaEvent_t e0 = nullptr, e1 = nullptr;
    cudaError_t e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&xyz_dev), nxyz * 8, ctx->pool, st);
    if (e == cudaSuccess)
        e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&out_dev), 6 * req->nq * 8, ctx->pool, st);
    if (e == cudaSuccess)
        e = cudaMallocFromPoolAsync(reinterpret_cast<void **>(&flush), flush_bytes, ctx->pool, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(xyz_dev, req->xyz, nxyz * 8, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaEventCreate(&e0);
    if (e == cudaSuccess) e = cudaEventCreate(&e1);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    // measured time and device bytes of every candidate that ran
    std::vector<std::pair<double, uint64_t>> measured(cands.size(), {1e300, 0});
    for (size_t c = 0; c < cands.size() && e == cudaSuccess; ++c) {
        pd_plan *plan = nullptr;
        if (plan_create_impl(ctx, req, &plan, &cands[c]) != PD_OK) continue;
        const uint64_t bytes = plan->dp.L.total;
        // warm-up, then timed executions (one when a run takes over 0.25 s)
        bool ok = pd_plan_execute(ctx, plan, xyz_dev, out_dev, st) == PD_OK;
        double total = 0.0;
        int reps = 0;
        for (int rep = 0; rep < 3 && ok; ++rep) {
            ok = cudaMemsetAsync(flush, rep + 1, flush_bytes, st) == cudaSuccess &&
                 cudaEventRecord(e0, st) == cudaSuccess &&
                 pd_plan_execute(ctx, plan, xyz_dev, out_dev, st) == PD_OK &&
                 cudaEventRecord(e1, st) == cudaSuccess && cudaEventSynchronize(e1) == cudaSuccess;
            float ms = 0.0f;
            if (ok) ok = cudaEventElapsedTime(&ms, e0, e1) == cudaSuccess;
            if (!ok) break;
            total += ms;
            ++reps;
            if (ms > 250.0f && reps >= 1) break;
        }
        pd_plan_destroy(ctx, plan);
        if (ok && reps > 0) measured[c] = {total / reps, bytes};
    }
    // The fastest shape; among shapes within TUNE_TIE of its time the one
    // that holds the least device memory (a longer j chunk means fewer tiles
    // and FP64 tile slots at the same speed).
    constexpr double TUNE_TIE = 0.003;
    double best = 1e300;
    for (const auto &m : measured) best = std::min(best, m.first);
    Tuning best_t = cands.front();
    double pick_ms = 1e300;
    uint64_t pick_bytes = ~uint64_t{0};
    for (size_t c = 0; c < cands.size() && best < 1e300; ++c) {
        const auto &m = measured[c];
        if (m.first > best * (1.0 + TUNE_TIE)) continue;
        if (m.second < pick_bytes || (m.second == pick_bytes && m.first < pick_ms)) {
            best_t = cands[c];
            pick_ms = m.first;
            pick_bytes = m.second;
        }
    }
    if (best < 1e300) best = pick_ms;
    if (xyz_dev) cudaFreeAsync(xyz_dev, st);
    if (out_dev) cudaFreeAsync(out_dev, st);
    if (flush) cudaFreeAsync(flush, st);
    if (e0) cudaEventDestroy(e0);
    if (e1) cudaEventDestroy(e1);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pd_autotune_request");
    if (best >= 1e300) {
        ctx->set_error("pd_autotune_request: no candidate shape ran");
        return PD_EDEVICE;
    }
    std::string path;
    pd::TuneTable snapshot;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        ctx->tuning[pd::tune_key(static_cast<int64_t>(req->n_atoms), static_cast<int64_t>(req->nq),
                                 static_cast<int>(req->precision), mode,
                                 static_cast<int64_t>(nf))] = pd::TuneEntry{best_t, best};
        path = ctx->tuning_path;
        if (!path.empty()) snapshot = ctx->tuning;
    }
    if (!path.empty() && pd::save_tuning(path, snapshot, msg) != PD_OK) {
        ctx->set_error(msg);
        return PD_EINVAL;
    }
    if (best_out) *best_out = best_t;
    if (best_ms) *best_ms = best;
    return PD_OK;
}

}  // namespace

int pd_autotune_request(pd_ctx *ctx, const pd_request *req, uint32_t *q_block, uint32_t *j_chunk,
                        uint32_t *pairs_per_thread, double *ms) {
    if (!ctx || !req) return PD_EINVAL;
    Tuning t;
    double best = 0.0;
    const int rc = autotune_request(ctx, req, &t, &best);
    if (rc) return rc;
    if (q_block) *q_block = static_cast<uint32_t>(t.K);
    if (j_chunk) *j_chunk = static_cast<uint32_t>(t.TJ);
    if (pairs_per_thread) *pairs_per_thread = static_cast<uint32_t>(t.NP);
    if (ms) *ms = best;
    return PD_OK;
}

int pd_autotune(pd_ctx *ctx, uint64_t n_atoms, uint64_t nq, uint32_t precision) {
    if (!ctx || n_atoms < 2 || nq < 1 || precision > PD_FP64) return PD_EINVAL;
    // Synthetic solvent globule of the bucket's size: uniform in a sphere at
    // the density of a protein (about 12 Å³ per atom), four species, the
    // outer shell hydrated with one weight per species (class mode, as the
    // FoXS-style surface hydration of real requests runs).
    std::mt19937_64 rng(12345);
    std::uniform_real_distribution<double> U(-1.0, 1.0);
    const double R = std::cbrt(12.0 * static_cast<double>(n_atoms) * 3.0 / (4.0 * M_PI));
    std::vector<double> xyz(n_atoms * 3), hw(n_atoms);
    std::vector<uint32_t> sp(n_atoms);
    for (uint64_t i = 0; i < n_atoms; ++i) {
        double x, y, z;
        do {
            x = U(rng);
            y = U(rng);
            z = U(rng);
        } while (x * x + y * y + z * z > 1.0);
        xyz[3 * i] = R * x;
        xyz[3 * i + 1] = R * y;
        xyz[3 * i + 2] = R * z;
        sp[i] = static_cast<uint32_t>(i % 4);
        const double rr = R * std::sqrt(x * x + y * y + z * z);
        hw[i] = (rr > R - 3.0 && U(rng) < -0.3) ? 1.5 + 0.25 * sp[i] : 0.0;
    }
    std::vector<double> ffA(4 * nq), ffC(4 * nq), ffW(nq);
    for (uint64_t k = 0; k < nq; ++k) {
        const double q = 0.5 * static_cast<double>(k) / static_cast<double>(nq > 1 ? nq - 1 : 1);
        for (int s = 0; s < 4; ++s) {
            ffA[s * nq + k] = (6.0 + s) * std::exp(-0.1 * q * q);
            ffC[s * nq + k] = (2.0 + 0.5 * s) * std::exp(-0.4 * q * q);
        }
        ffW[k] = 10.0 * std::exp(-0.2 * q * q);
    }
    pd_request rq{};
    rq.n_atoms = n_atoms;
    rq.xyz = xyz.data();
    rq.species = sp.data();
    rq.n_species = 4;
    rq.precision = precision;
    rq.ff_atoms = ffA.data();
    rq.ff_excluded = ffC.data();
    rq.hyd_weights = hw.data();
    rq.ff_water = ffW.data();
    rq.qmin = 0.0;
    rq.qmax = 0.5;
    rq.nq = nq;
    return autotune_request(ctx, &rq, nullptr, nullptr);
}

int pd_tuning_load(pd_ctx *ctx, const char *path) {
    if (!ctx || !path) return PD_EINVAL;
    pd::TuneTable tab;
    std::string msg;
    const int rc = pd::load_tuning(path, tab, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    for (auto &kv : tab) ctx->tuning[kv.first] = kv.second;
    return PD_OK;
}

int pd_tuning_save(pd_ctx *ctx, const char *path) {
    if (!ctx || !path) return PD_EINVAL;
    pd::TuneTable snapshot;
    {
        std::lock_guard<std::mutex> g(ctx->mu);
        snapshot = ctx->tuning;
    }
    std::string msg;
    const int rc = pd::save_tuning(path, snapshot, msg);
    if (rc) ctx->set_error(msg);
    return rc;
}

int pd_tuning_lookup(pd_ctx *ctx, const pd_request *req, uint32_t *q_block, uint32_t *j_chunk,
                     uint32_t *pairs_per_thread, int *from_table) {
    if (!req) return PD_EINVAL;
    std::string msg;
    const int rc = pd::validate_request(req, false, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    bool tab = false;
    const Tuning t = tuning_for_request(ctx, req, req->species, req->hyd_weights, &tab);
    if (q_block) *q_block = static_cast<uint32_t>(t.K);
    if (j_chunk) *j_chunk = static_cast<uint32_t>(t.TJ);
    if (pairs_per_thread) *pairs_per_thread = static_cast<uint32_t>(t.NP);
    if (from_table) *from_table = tab ? 1 : 0;
    return PD_OK;
}

int pd_tuning_check(const char *path, uint64_t *n_entries) {
    if (!path) return PD_EINVAL;
    pd::TuneTable tab;
    std::string msg;
    const int rc = pd::load_tuning(path, tab, msg);
    if (rc) {
        std::lock_guard<std::mutex> g(g_err_mu);
        g_err = msg;
        return rc;
    }
    if (n_entries) *n_entries = tab.size();
    return PD_OK;
}

int pd_plan_inspect(pd_ctx *ctx, const pd_request *req, uint64_t *n_classes, uint64_t *n_padded,
                    uint64_t *n_tiles, uint64_t *pairs_covered) {
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    Tuning tun = tuning_for_request(ctx, req, req->species, req->hyd_weights);
    Plan P;
    rc = pd::build_plan(req, req->species, req->hyd_weights, tun, P, msg, /*count_pairs=*/true);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    if (n_classes) *n_classes = static_cast<uint64_t>(P.n_cls);
    if (n_padded) *n_padded = static_cast<uint64_t>(P.n_pad);
    if (n_tiles) *n_tiles = P.jobs.size();
    if (pairs_covered) *pairs_covered = P.pairs_covered;
    return PD_OK;
}

int pd_request_device_bytes(pd_ctx *ctx, const pd_request *req, int host_coordinates,
                            uint64_t *device_bytes) {
    if (!req || !device_bytes) return PD_EINVAL;
    std::string msg;
    int rc = pd::validate_request(req, false, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    Tuning tun = tuning_for_request(ctx, req, req->species, req->hyd_weights);
    Plan P;
    rc = pd::build_plan(req, req->species, req->hyd_weights, tun, P, msg);
    if (rc) {
        if (ctx) ctx->set_error(msg);
        return rc;
    }
    *device_bytes = make_layout(P, host_coordinates != 0).total;
    return PD_OK;
}

int pd_measure_fp32_peak(pd_ctx *ctx, double *tflops_ffma, double *tflops_ffma2) {
    if (!ctx) return PD_EINVAL;
    cudaSetDevice(ctx->device);
    float *d = nullptr;
    PD_CUDA(ctx, cudaMalloc(reinterpret_cast<void **>(&d), 4));
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    const int block = 256, grid = ctx->sm_count * 8, iters = 4096;
    const double flops = 2.0 * 16 * 8 * static_cast<double>(iters) * block * grid;
    for (int packed = 0; packed < 2; ++packed) {
        pd::launch_ffma_probe(d, iters / 8, grid, block, packed != 0, ctx->stream);  // warm-up
        cudaEventRecord(e0, ctx->stream);
        pd::launch_ffma_probe(d, iters, grid, block, packed != 0, ctx->stream);
        cudaEventRecord(e1, ctx->stream);
        cudaError_t e = cudaEventSynchronize(e1);
        if (e != cudaSuccess) return cuda_fail(ctx, e, "fp32 probe");
        float ms = 0;
        cudaEventElapsedTime(&ms, e0, e1);
        const double tf = flops * (packed ? 2.0 : 1.0) / (ms * 1e-3) / 1e12;
        if (packed == 0 && tflops_ffma) *tflops_ffma = tf;
        if (packed == 1 && tflops_ffma2) *tflops_ffma2 = tf;
        ctx->launches += 2;
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    cudaFree(d);
    return PD_OK;
}

uint64_t pd_launch_count(pd_ctx *ctx) { return ctx ? ctx->launches.load() : 0; }

}  // extern "C"

// ---------------------------------------------------------------- direct transform
namespace {

// Checks shared by pd_direct and pd_direct_lattice (the q-vectors apart).
std::string direct_validate(const pd_direct_request *req) {
    const uint64_t n = req->n_points, nv = req->n_vectors;
    const uint64_t nm = req->n_molecules ? req->n_molecules : 1;
    if (n == 0 || nv == 0 || req->n_kinds == 0 || !req->xyz || !req->kind || !req->ff ||
        req->reserved)
        return "pd_direct: n_points, n_vectors, n_kinds >= 1 and xyz, kind, ff required";
    if (n > (1ull << 30) || nv > (1ull << 26) || req->n_kinds > (1u << 24))
        return "pd_direct: n_points <= 2^30, n_vectors <= 2^26 and n_kinds <= 2^24";
    if (n % nm)
        return "box point count (" + std::to_string(n) + ") is not a multiple of the molecule "
               "count (" + std::to_string(nm) + ")";
    for (uint64_t i = 0; i < n; ++i)
        if (req->kind[i] >= req->n_kinds)
            return "kind " + std::to_string(req->kind[i]) + " at point " + std::to_string(i) +
                   " is >= n_kinds";
    for (uint64_t i = 0; i < 3 * n; ++i)
        if (!std::isfinite(req->xyz[i])) return "non-finite coordinate";
    for (uint64_t i = 0; i < nv * req->n_kinds; ++i)
        if (!std::isfinite(req->ff[i])) return "non-finite form factor";
    for (uint64_t i = 0; req->weight && i < n; ++i)
        if (!std::isfinite(req->weight[i])) return "non-finite point weight";
    return std::string();
}

// One blocking Direct solve: either explicit q-vectors (qvec, the sincos
// kernel) or lattice indices (hkl with |index| <= nmax and box, the phase-table
// kernel). ff is [n_kinds][n_vectors] in the order of the vectors given.
int direct_run(pd_ctx *ctx, const pd_direct_request *req, const double *ff, const double *qvec,
               const int32_t *hkl, int32_t nmax, const double *box, double *out) {
    const uint64_t n = req->n_points, nv = req->n_vectors;
    const uint64_t nm = req->n_molecules ? req->n_molecules : 1;
    const int64_t mol = static_cast<int64_t>(n / nm);
    const int64_t chunks = pd::direct_chunks(static_cast<int64_t>(n), mol, static_cast<int64_t>(nv));
    if (pd::direct_blocks(static_cast<int64_t>(n), mol, static_cast<int64_t>(nv)) > 0x7fffffffLL ||
        static_cast<double>(chunks) * static_cast<double>(nv) * 40.0 > 8.0 * (1ull << 30)) {
        ctx->set_error("pd_direct: points x vectors too large for one call (per-chunk partial "
                       "amplitudes above 8 GiB); split the q-vectors into batches");
        return PD_EINVAL;
    }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t b_xyz = n * 24, b_kind = n * 4, b_ff = nv * req->n_kinds * 8,
                 b_q = hkl ? nv * 12 : nv * 24, b_part = static_cast<size_t>(chunks) * nv * 40,
                 b_out = nv * 32, b_w = req->weight ? n * 8 : 0;
    const size_t total = align_up(b_xyz, 256) + align_up(b_kind, 256) + align_up(b_ff, 256) +
                         align_up(b_q, 256) + align_up(b_part, 256) + align_up(b_w, 256) + b_out;
    char *base = nullptr;
    PD_CUDA(ctx, cudaMallocFromPoolAsync(reinterpret_cast<void **>(&base), total, ctx->pool, st));
    char *cur = base;
    auto take = [&](size_t bytes) {
        char *r = cur;
        cur += align_up(bytes, 256);
        return r;
    };
    double *d_xyz = reinterpret_cast<double *>(take(b_xyz));
    uint32_t *d_kind = reinterpret_cast<uint32_t *>(take(b_kind));
    double *d_ff = reinterpret_cast<double *>(take(b_ff));
    char *d_q = take(b_q);
    double *d_part = reinterpret_cast<double *>(take(b_part));
    double *d_w = req->weight ? reinterpret_cast<double *>(take(b_w)) : nullptr;
    double *d_out = reinterpret_cast<double *>(take(b_out));
    cudaError_t e = cudaMemcpyAsync(d_xyz, req->xyz, b_xyz, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_kind, req->kind, b_kind, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_ff, ff, b_ff, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(d_q, hkl ? static_cast<const void *>(hkl) : qvec, b_q,
                            cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess && d_w)
        e = cudaMemcpyAsync(d_w, req->weight, b_w, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        if (hkl)
            e = pd::launch_direct_table(d_xyz, d_kind, d_w, d_ff, reinterpret_cast<int32_t *>(d_q),
                                        nmax, box, static_cast<int64_t>(nv),
                                        static_cast<int64_t>(n), mol, d_part, chunks, d_out, st);
        else
            e = pd::launch_direct(d_xyz, d_kind, d_w, d_ff, static_cast<int32_t>(req->n_kinds),
                                  reinterpret_cast<double *>(d_q), static_cast<int64_t>(nv),
                                  static_cast<int64_t>(n), mol, d_part, chunks, d_out, st);
    }
    if (e == cudaSuccess) {
        ctx->launches += 2;
        e = cudaMemcpyAsync(out, d_out, b_out, cudaMemcpyDeviceToHost, st);
    }
    cudaFreeAsync(base, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pd_direct");
    return PD_OK;
}

// Lattice indices up to this bound use the phase tables; beyond it a table
// row costs more than the sincos it saves, and the vectors go to the sincos
// kernel as q = 2π·hkl/L.
constexpr int64_t kDirectTableMaxIndex = 512;

}  // namespace

extern "C" int pd_direct(pd_ctx *ctx, const pd_direct_request *req, double *out) {
    if (!ctx || !req || !out) return PD_EINVAL;
    std::string msg = req->qvec ? direct_validate(req) : "pd_direct: qvec required";
    for (uint64_t i = 0; msg.empty() && i < 3 * req->n_vectors; ++i)
        if (!std::isfinite(req->qvec[i])) msg = "non-finite q-vector";
    if (!msg.empty()) {
        ctx->set_error(msg);
        return PD_EINVAL;
    }
    return direct_run(ctx, req, req->ff, req->qvec, nullptr, 0, nullptr, out);
}

extern "C" int pd_direct_lattice(pd_ctx *ctx, const pd_direct_request *req, const int32_t *hkl,
                                 const double box[3], double *out) {
    if (!ctx || !req || !out) return PD_EINVAL;
    std::string msg = (hkl && box) ? direct_validate(req) : "pd_direct_lattice: hkl and box required";
    for (int a = 0; msg.empty() && a < 3; ++a)
        if (!std::isfinite(box[a]) || !(box[a] > 0.0)) msg = "box sides must be finite and > 0";
    if (!msg.empty()) {
        ctx->set_error(msg);
        return PD_EINVAL;
    }
    const uint64_t nv = req->n_vectors, nk = req->n_kinds;
    int64_t nmax = 0;
    for (uint64_t i = 0; i < 3 * nv; ++i)
        nmax = std::max<int64_t>(nmax, std::llabs(static_cast<long long>(hkl[i])));
    if (nmax > kDirectTableMaxIndex || pd::direct_table_points(static_cast<int32_t>(nmax)) < 1) {
        std::vector<double> q(3 * nv);
        for (uint64_t i = 0; i < nv; ++i)
            for (int a = 0; a < 3; ++a)
                q[3 * i + a] = (2.0 * M_PI * static_cast<double>(hkl[3 * i + a])) / box[a];
        return direct_run(ctx, req, req->ff, q.data(), nullptr, 0, nullptr, out);
    }
    // vectors in (h, k, l) order, so that a warp's table reads share rows
    std::vector<uint32_t> perm(nv);
    for (uint64_t i = 0; i < nv; ++i) perm[i] = static_cast<uint32_t>(i);
    std::stable_sort(perm.begin(), perm.end(), [&](uint32_t x, uint32_t y) {
        return std::lexicographical_compare(hkl + 3 * x, hkl + 3 * x + 3, hkl + 3 * y, hkl + 3 * y + 3);
    });
    std::vector<int32_t> hs(3 * nv);
    std::vector<double> fs(nk * nv), os(4 * nv);
    for (uint64_t i = 0; i < nv; ++i) {
        for (int a = 0; a < 3; ++a) hs[3 * i + a] = hkl[3 * perm[i] + a];
        for (uint64_t k = 0; k < nk; ++k) fs[k * nv + i] = req->ff[k * nv + perm[i]];
    }
    const int rc = direct_run(ctx, req, fs.data(), nullptr, hs.data(), static_cast<int32_t>(nmax),
                              box, os.data());
    if (rc != PD_OK) return rc;
    for (uint64_t i = 0; i < nv; ++i)
        for (int c = 0; c < 4; ++c) out[4 * perm[i] + c] = os[4 * i + c];
    return PD_OK;
}

// ---------------------------------------------------------------- form factors
extern "C" int pd_formfactor_tables(pd_ctx *ctx, const pd_formfactor *ff, uint32_t n_ff,
                                    double qmin, double qmax, uint64_t nq, double *out) {
    if (!ctx || !ff || !out || n_ff == 0 || nq == 0 || nq > (1ull << 24)) return PD_EINVAL;
    if (!std::isfinite(qmin) || !std::isfinite(qmax) || qmin < 0.0 || qmax < qmin) {
        ctx->set_error("q range must satisfy 0 <= qmin <= qmax (finite)");
        return PD_EINVAL;
    }
    std::vector<int32_t> desc(3 * n_ff);
    std::vector<double> range(2 * n_ff), params;
    for (uint32_t f = 0; f < n_ff; ++f) {
        const pd_formfactor &d = ff[f];
        size_t np = 0;
        bool ok = d.params != nullptr && !(d.qlo > d.qhi) && !std::isnan(d.qlo) &&
                  !std::isnan(d.qhi);
        switch (d.type) {
            case PD_FF_CONSTANT: np = 1; break;
            case PD_FF_GAUSSIAN: np = 1 + 2 * static_cast<size_t>(d.n); break;
            case PD_FF_SINGLE_GAUSSIAN: np = 2; break;
            case PD_FF_POLYNOMIAL: np = d.n; ok = ok && d.n >= 1; break;
            case PD_FF_TABLE: np = 2 * static_cast<size_t>(d.n); ok = ok && d.n >= 2; break;
            default: ok = false;
        }
        if (ok && d.n > 4096) ok = false;
        for (size_t i = 0; ok && i < np; ++i) ok = std::isfinite(d.params[i]);
        if (ok && d.type == PD_FF_TABLE)
            for (uint32_t i = 1; ok && i < d.n; ++i) ok = d.params[i] > d.params[i - 1];
        if (!ok) {
            ctx->set_error("form factor " + std::to_string(f) +
                           ": unknown type, bad parameters or range (tables need >= 2 "
                           "increasing points)");
            return PD_EINVAL;
        }
        desc[3 * f] = static_cast<int32_t>(d.type);
        desc[3 * f + 1] = static_cast<int32_t>(d.n);
        desc[3 * f + 2] = static_cast<int32_t>(params.size());
        range[2 * f] = d.qlo;
        range[2 * f + 1] = d.qhi;
        params.insert(params.end(), d.params, d.params + np);
    }
    if (params.size() > (1u << 26)) return PD_EINVAL;
    params.push_back(0.0);
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    cudaStream_t st = ctx->stream;
    const size_t b_desc = desc.size() * 4, b_range = range.size() * 8,
                 b_par = params.size() * 8, b_out = static_cast<size_t>(n_ff) * nq * 8;
    const size_t total = align_up(b_desc, 256) + align_up(b_range, 256) + align_up(b_par, 256) +
                         align_up(4, 256) + b_out;
    char *base = nullptr;
    PD_CUDA(ctx, cudaMallocFromPoolAsync(reinterpret_cast<void **>(&base), total, ctx->pool, st));
    char *cur = base;
    auto take = [&](size_t bytes) {
        char *r = cur;
        cur += align_up(bytes, 256);
        return r;
    };
    int32_t *d_desc = reinterpret_cast<int32_t *>(take(b_desc));
    double *d_range = reinterpret_cast<double *>(take(b_range));
    double *d_par = reinterpret_cast<double *>(take(b_par));
    int *d_bad = reinterpret_cast<int *>(take(4));
    double *d_out = reinterpret_cast<double *>(take(b_out));
    int bad = 0;
    cudaError_t e = cudaMemcpyAsync(d_desc, desc.data(), b_desc, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_range, range.data(), b_range, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_par, params.data(), b_par, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_bad, 0, 4, st);
    if (e == cudaSuccess)
        e = pd::launch_ff_eval(d_desc, d_range, d_par, static_cast<int32_t>(n_ff), qmin, qmax,
                               static_cast<int64_t>(nq), d_bad, d_out, st);
    if (e == cudaSuccess) {
        ctx->launches += 1;
        e = cudaMemcpyAsync(out, d_out, b_out, cudaMemcpyDeviceToHost, st);
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(&bad, d_bad, 4, cudaMemcpyDeviceToHost, st);
    cudaFreeAsync(base, st);
    const cudaError_t e2 = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = e2;
    if (e != cudaSuccess) return cuda_fail(ctx, e, "pd_formfactor_tables");
    if (bad) {
        const pd_formfactor &d = ff[bad - 1];
        ctx->set_error("q outside the range [" + std::to_string(d.qlo) + ", " +
                       std::to_string(d.qhi) + "] of form factor " + std::to_string(bad - 1) +
                       " (QOutOfRange)");
        return PD_EINVAL;
    }
    return PD_OK;
}

// ---------------------------------------------------------------- streamed trajectories
// A trajectory average fed frame by frame: frames are assembled in pinned
// batches of B frames, each batch is uploaded on its own stream while the
// previous batch is solved, and every batch adds its unnormalised
// Σ_f w_f·T_f to an FP64 accumulator (batches in submission order); finish
// divides once by Σ w_f, as the reference's frame loop does
// (src/trajectory.rs:198-248).
struct pd_stream {
    DevPlan dp;
    uint32_t B = 0;
    uint64_t frame_doubles = 0;       // 3·N
    cudaStream_t cs = nullptr, us = nullptr;  // compute, upload
    double *d_xyz[2] = {nullptr, nullptr};
    double *h_xyz[2] = {nullptr, nullptr};
    double *h_w[2] = {nullptr, nullptr};
    cudaEvent_t uploaded[2] = {nullptr, nullptr}, computed[2] = {nullptr, nullptr};
    bool pending[2] = {false, false};
    int cur = 0;
    uint32_t fill = 0;
    double *d_acc = nullptr, *d_batch = nullptr;
    double wsum = 0.0;
    uint64_t frames = 0;
    bool failed = false;
};

namespace {

void stream_free(pd_ctx *ctx, pd_stream *s) {
    if (s->cs) cudaStreamSynchronize(s->cs);
    if (s->us) cudaStreamSynchronize(s->us);
    for (int b = 0; b < 2; ++b) {
        if (s->d_xyz[b]) cudaFree(s->d_xyz[b]);
        if (s->h_xyz[b]) cudaFreeHost(s->h_xyz[b]);
        if (s->h_w[b]) cudaFreeHost(s->h_w[b]);
        if (s->uploaded[b]) cudaEventDestroy(s->uploaded[b]);
        if (s->computed[b]) cudaEventDestroy(s->computed[b]);
    }
    if (s->d_acc) cudaFree(s->d_acc);
    if (s->d_batch) cudaFree(s->d_batch);
    free_devplan(ctx, s->dp, s->cs ? s->cs : ctx->stream);
    if (s->cs) cudaStreamSynchronize(s->cs);
    if (s->cs) cudaStreamDestroy(s->cs);
    if (s->us) cudaStreamDestroy(s->us);
    delete s;
}

// Upload and solve the frames assembled in host buffer s->cur.
int stream_submit(pd_ctx *ctx, pd_stream *s) {
    const int b = s->cur;
    const uint32_t n = s->fill;
    if (n == 0) return PD_OK;
    const size_t fb = s->frame_doubles * 8;
    // pad a partial batch with copies of its first frame at weight 0
    double wb = 0.0;
    for (uint32_t f = 0; f < n; ++f) wb += s->h_w[b][f];
    for (uint32_t f = n; f < s->B; ++f) {
        std::memcpy(s->h_xyz[b] + f * s->frame_doubles, s->h_xyz[b], fb);
        s->h_w[b][f] = 0.0;
    }
    // device buffer b was last read by the batch that recorded computed[b]
    if (s->pending[b]) PD_CUDA(ctx, cudaStreamWaitEvent(s->us, s->computed[b], 0));
    PD_CUDA(ctx, cudaMemcpyAsync(s->d_xyz[b], s->h_xyz[b], fb * s->B, cudaMemcpyHostToDevice,
                                 s->us));
    PD_CUDA(ctx, cudaEventRecord(s->uploaded[b], s->us));
    PD_CUDA(ctx, cudaStreamWaitEvent(s->cs, s->uploaded[b], 0));
    const Layout &L = s->dp.L;
    PD_CUDA(ctx, cudaMemcpyAsync(s->dp.dptr<double>(L.fw), s->h_w[b], 8ull * s->B,
                                 cudaMemcpyHostToDevice, s->cs));
    s->dp.xyz_dev = s->d_xyz[b];
    int rc = run_devplan(ctx, s->dp, s->d_batch, s->cs);
    if (rc) return rc;
    // one-frame plans finish with the frame's terms: weight them here
    const double scale = s->B == 1 ? s->h_w[b][0] : 1.0;
    PD_CUDA(ctx, pd::launch_stream_accumulate(s->d_batch, scale, 6 * s->dp.P.nq, s->d_acc, s->cs));
    ctx->launches += 1;
    PD_CUDA(ctx, cudaEventRecord(s->computed[b], s->cs));
    s->pending[b] = true;
    s->wsum += wb;
    s->frames += n;
    s->cur ^= 1;
    s->fill = 0;
    return PD_OK;
}

}  // namespace

extern "C" int pd_stream_open(pd_ctx *ctx, const pd_request *req, uint32_t frames_per_batch,
                              pd_stream **out) {
    if (!ctx || !req || !out || frames_per_batch == 0 || frames_per_batch > 4096) return PD_EINVAL;
    *out = nullptr;
    pd_request r = *req;
    std::vector<double> dummy;
    if (r.n_atoms == 0) {
        ctx->set_error("n_atoms must be >= 1");
        return PD_EINVAL;
    }
    if (r.n_lattices) {
        ctx->set_error("streamed trajectories take atoms only (lattice sets need one frame)");
        return PD_EINVAL;
    }
    r.n_frames = frames_per_batch;
    r.frame_weights = nullptr;
    dummy.assign(static_cast<size_t>(r.n_atoms) * 3 * frames_per_batch, 0.0);
    r.xyz = dummy.data();
    std::string msg;
    int rc = pd::validate_request(&r, false, msg);
    if (rc) {
        ctx->set_error(msg);
        return rc;
    }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    auto *s = new pd_stream();
    s->B = frames_per_batch;
    s->frame_doubles = static_cast<uint64_t>(r.n_atoms) * 3;
    s->dp.frame_sum = true;
    cudaError_t e = cudaStreamCreateWithFlags(&s->cs, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->us, cudaStreamNonBlocking);
    if (e != cudaSuccess) {
        stream_free(ctx, s);
        return cuda_fail(ctx, e, "pd_stream_open: streams");
    }
    rc = create_devplan(ctx, &r, r.species, r.hyd_weights, false, s->dp, s->cs);
    if (rc) {
        stream_free(ctx, s);
        return rc;
    }
    const size_t fb = s->frame_doubles * 8 * s->B;
    const size_t nq6 = 6ull * r.nq * 8;
    for (int b = 0; b < 2 && e == cudaSuccess; ++b) {
        e = cudaMalloc(reinterpret_cast<void **>(&s->d_xyz[b]), fb);
        if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&s->h_xyz[b]), fb, 0);
        if (e == cudaSuccess) e = cudaHostAlloc(reinterpret_cast<void **>(&s->h_w[b]), 8ull * s->B, 0);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->uploaded[b], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s->computed[b], cudaEventDisableTiming);
    }
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&s->d_acc), nq6);
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&s->d_batch), nq6);
    if (e == cudaSuccess) e = cudaMemsetAsync(s->d_acc, 0, nq6, s->cs);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->cs);
    if (e != cudaSuccess) {
        stream_free(ctx, s);
        return cuda_fail(ctx, e, "pd_stream_open: buffers");
    }
    *out = s;
    return PD_OK;
}

extern "C" int pd_stream_push(pd_ctx *ctx, pd_stream *s, const double *xyz,
                              const double *weights, uint64_t n_frames) {
    if (!ctx || !s || (!xyz && n_frames)) return PD_EINVAL;
    if (s->failed) {
        ctx->set_error("the stream failed earlier");
        return PD_EDEVICE;
    }
    for (uint64_t i = 0; i < n_frames * s->frame_doubles; ++i)
        if (!std::isfinite(xyz[i])) {
            ctx->set_error("non-finite coordinate at index " + std::to_string(i));
            return PD_EINVAL;
        }
    for (uint64_t f = 0; weights && f < n_frames; ++f)
        if (!std::isfinite(weights[f])) {
            ctx->set_error("non-finite frame weight");
            return PD_EINVAL;
        }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    for (uint64_t f = 0; f < n_frames; ++f) {
        const int b = s->cur;
        if (s->fill == 0 && s->pending[b]) {  // host buffer b is read until its batch is done
            cudaError_t e = cudaEventSynchronize(s->computed[b]);
            if (e != cudaSuccess) {
                s->failed = true;
                return cuda_fail(ctx, e, "pd_stream_push");
            }
        }
        std::memcpy(s->h_xyz[b] + s->fill * s->frame_doubles, xyz + f * s->frame_doubles,
                    s->frame_doubles * 8);
        s->h_w[b][s->fill] = weights ? weights[f] : 1.0;
        if (++s->fill == s->B) {
            int rc = stream_submit(ctx, s);
            if (rc) {
                s->failed = true;
                return rc;
            }
        }
    }
    return PD_OK;
}

extern "C" int pd_stream_finish(pd_ctx *ctx, pd_stream *s, double *out_terms) {
    if (!ctx || !s) return PD_EINVAL;
    int rc = PD_OK;
    {
        std::lock_guard<std::mutex> g(ctx->solve_mu);
        cudaSetDevice(ctx->device);
        if (!s->failed) rc = stream_submit(ctx, s);
        const size_t n6 = 6ull * s->dp.P.nq;
        std::vector<double> acc(n6);
        if (rc == PD_OK && !s->failed) {
            int32_t dev_status = 0;  // of every batch: a stream's plan keeps it
            cudaError_t e = cudaMemcpyAsync(acc.data(), s->d_acc, n6 * 8, cudaMemcpyDeviceToHost, s->cs);
            if (e == cudaSuccess)
                e = cudaMemcpyAsync(&dev_status, s->dp.base + s->dp.L.status, sizeof(int32_t),
                                    cudaMemcpyDeviceToHost, s->cs);
            if (e == cudaSuccess) e = cudaStreamSynchronize(s->cs);
            if (e != cudaSuccess) rc = cuda_fail(ctx, e, "pd_stream_finish");
            if (rc == PD_OK) rc = result_status(ctx, s->dp.P, dev_status, nullptr);
        } else if (rc == PD_OK) {
            ctx->set_error("the stream failed earlier");
            rc = PD_EDEVICE;
        }
        if (rc == PD_OK && s->frames == 0) {
            ctx->set_error("no frames were pushed");
            rc = PD_EINVAL;
        }
        // trajectory_average rejects a weight sum that is zero or not normal
        // (src/trajectory.rs:234-238)
        if (rc == PD_OK && !std::isnormal(std::fabs(s->wsum))) {
            ctx->set_error("weights of the " + std::to_string(s->frames) +
                           " averaged frames sum to " + std::to_string(s->wsum) +
                           "; cannot normalize");
            rc = PD_EINVAL;
        }
        if (rc == PD_OK && out_terms)
            for (size_t t = 0; t < n6; ++t) out_terms[t] = acc[t] / s->wsum;
    }
    std::lock_guard<std::mutex> g(ctx->solve_mu);
    cudaSetDevice(ctx->device);
    stream_free(ctx, s);
    return rc;
}


// ------------------------------------------------ allocation-free solve
// pd_solve_noalloc runs the same pipeline as a plan execution, but every
// device array of the request (tables, tile list, packed atoms, per-warp
// slots, partial sums) lives in one fixed array compiled into the library
// instead of memory from cudaMalloc or a pool. It serves callers that cannot
// allocate device memory at call time.
namespace {

// The scratch array. Host code may not use this name as a device address: on
// the host it names a stand-in object, so the kernels get the address that
// cudaGetSymbolAddress returns for the current device.
static __device__ __align__(256) unsigned char g_noalloc_scratch[PD_NOALLOC_SCRATCH_BYTES];

struct NoallocDevice {
    char *scratch = nullptr;      // device address of g_noalloc_scratch
    std::unique_ptr<pd_ctx> ctx;  // launch bookkeeping only: no stream, no pool
    std::mutex mu;                // one call at a time on this device
};
std::mutex g_noalloc_mu;  // guards the map only
std::map<int, std::unique_ptr<NoallocDevice>> g_noalloc;  // per device ordinal, set up on first use

int noalloc_fail(int rc, const std::string &m) {
    std::lock_guard<std::mutex> g(g_err_mu);
    g_err = m;
    return rc;
}

// The host-side checks of validate_request for a request whose coordinates
// are device memory: ids and tables are read here, the coordinates are not.
int noalloc_validate(const pd_request *req, std::string &msg) {
    int rc = pd::validate_request(req, true, msg);
    if (rc) return rc;
    for (uint64_t i = 0; i < req->n_atoms; ++i)
        if (req->species[i] >= req->n_species) {
            msg = "species id at atom " + std::to_string(i) + " is >= n_species";
            return PD_EINVAL;
        }
    const uint64_t nt = static_cast<uint64_t>(req->n_species) * req->nq;
    for (uint64_t i = 0; i < nt; ++i)
        if (!std::isfinite(req->ff_atoms[i]) ||
            (req->ff_excluded && !std::isfinite(req->ff_excluded[i]))) {
            msg = "non-finite form-factor table entry";
            return PD_EINVAL;
        }
    if (req->hyd_weights) {
        for (uint64_t i = 0; i < req->n_atoms; ++i)
            if (!std::isfinite(req->hyd_weights[i])) {
                msg = "non-finite hydration weight";
                return PD_EINVAL;
            }
        for (uint64_t i = 0; i < req->nq; ++i)
            if (!std::isfinite(req->ff_water[i])) {
                msg = "non-finite water form factor";
                return PD_EINVAL;
            }
    }
    if (req->frame_weights) {
        const uint64_t nf = req->n_frames ? req->n_frames : 1;
        double s = 0.0;
        for (uint64_t f = 0; f < nf; ++f) {
            if (!std::isfinite(req->frame_weights[f])) {
                msg = "non-finite frame weight";
                return PD_EINVAL;
            }
            s += req->frame_weights[f];
        }
        if (!std::isnormal(std::fabs(s))) {
            msg = "frame weights sum to zero or a non-normal value; cannot normalize";
            return PD_EINVAL;
        }
    }
    return PD_OK;
}

// Once per device, with that device current: the scratch address and the SM
// count. Returns the device's entry or nullptr (g_err set).
NoallocDevice *noalloc_device(int dev, int *rc) {
    std::lock_guard<std::mutex> g(g_noalloc_mu);
    auto it = g_noalloc.find(dev);
    if (it != g_noalloc.end()) return it->second.get();
    int major = 0, sms = 0;
    cudaError_t e = cudaDeviceGetAttribute(&major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess || major < 10) {
        *rc = noalloc_fail(PD_ENODEV, "pd_solve_noalloc: device " + std::to_string(dev) +
                                          " is not an sm_100 device" +
                                          (e != cudaSuccess ? std::string(": ") +
                                                                  cudaGetErrorString(e)
                                                            : std::string()));
        return nullptr;
    }
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess || !p) {
        *rc = noalloc_fail(PD_EDEVICE, std::string("pd_solve_noalloc: scratch address: ") +
                                           cudaGetErrorString(e));
        return nullptr;
    }
    auto nd = std::make_unique<NoallocDevice>();
    nd->scratch = static_cast<char *>(p);
    nd->ctx = std::make_unique<pd_ctx>();
    nd->ctx->device = dev;
    nd->ctx->sm_count = sms;
    e = pd::prepare_pair_kernels();  // launch attributes, before any capture
    if (e != cudaSuccess) {
        *rc = noalloc_fail(PD_EDEVICE, std::string("pd_solve_noalloc: kernel set-up failed: ") +
                                           cudaGetErrorString(e));
        return nullptr;
    }
    return g_noalloc.emplace(dev, std::move(nd)).first->second.get();
}

}  // namespace

extern "C" int pd_solve_noalloc(const pd_request *req, const double *xyz_dev,
                                double *out_terms_dev, void *stream) {
    if (!req || !xyz_dev || !out_terms_dev)
        return noalloc_fail(PD_EINVAL, "pd_solve_noalloc: req, xyz_dev and out_terms_dev are required");
    pd_request r = *req;
    r.xyz = xyz_dev;  // only checked for NULL; never read on the host
    std::string msg;
    int rc = noalloc_validate(&r, msg);
    if (rc) return noalloc_fail(rc, "pd_solve_noalloc: " + msg);
    DevPlan dp;
    Tuning tun = tuning_for_request(nullptr, &r, r.species, r.hyd_weights);
    rc = pd::build_plan(&r, r.species, r.hyd_weights, tun, dp.P, msg);
    if (rc) return noalloc_fail(rc, "pd_solve_noalloc: " + msg);
    dp.L = make_layout(dp.P, false);
    if (dp.L.total > PD_NOALLOC_SCRATCH_BYTES)
        return noalloc_fail(PD_EBUDGET,
                            "pd_solve_noalloc: the request needs " + std::to_string(dp.L.total) +
                                " bytes of device scratch; the fixed scratch holds " +
                                std::to_string(static_cast<uint64_t>(PD_NOALLOC_SCRATCH_BYTES)) +
                                " (use pd_solve or a plan for larger requests)");
    // The plan is uploaded from a host image that lives only for this call,
    // which a captured graph would replay after it is gone: the first CUDA
    // call of the entry point refuses a capturing stream.
    cudaStream_t st = static_cast<cudaStream_t>(stream);
    {
        cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
        const cudaError_t ce = cudaStreamIsCapturing(st, &cs);
        if (ce == cudaErrorNoDevice || ce == cudaErrorInsufficientDriver)
            return noalloc_fail(PD_ENODEV, std::string("pd_solve_noalloc: no CUDA device: ") +
                                               cudaGetErrorString(ce));
        if (ce != cudaSuccess || cs != cudaStreamCaptureStatusNone)
            return noalloc_fail(PD_EINVAL,
                                std::string("pd_solve_noalloc: the stream is being captured "
                                            "into a CUDA graph (capture query: ") +
                                    cudaGetErrorString(ce) +
                                    "); this call uploads from call-local host memory and "
                                    "cannot be captured");
    }
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess)
        return noalloc_fail(PD_ENODEV, std::string("pd_solve_noalloc: no current CUDA device: ") +
                                           cudaGetErrorString(e));
    NoallocDevice *nd = noalloc_device(dev, &rc);
    if (!nd) return rc;
    // One call at a time per device on the host; the device work of calls on
    // different streams may still overlap, and then they race on the scratch.
    std::lock_guard<std::mutex> g(nd->mu);
    pd_ctx *ctx = nd->ctx.get();
    // Host image of the uploaded part in ordinary heap memory: a copy from
    // pageable memory returns once the driver has taken the bytes, so the
    // image may go out of scope when this call returns.
    std::vector<char> image(dp.L.upload_bytes);
    dp.base = nd->scratch;
    dp.stage = image.data();
    stage_plan(ctx, dp, &r);
    dp.stage = nullptr;
    e = cudaMemcpyAsync(dp.base, image.data(), dp.L.upload_bytes, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) {
        dp.xyz_dev = xyz_dev;
        rc = run_devplan(ctx, dp, out_terms_dev, st);  // also zeroes the counter and status
    } else {
        rc = cuda_fail(ctx, e, "pd_solve_noalloc: upload");
    }
    dp.base = nullptr;  // the scratch is never freed
    if (rc) {
        std::string m;
        {
            std::lock_guard<std::mutex> g2(ctx->mu);
            auto it = ctx->errors.find(std::this_thread::get_id());
            if (it != ctx->errors.end()) m = it->second;
        }
        return noalloc_fail(rc, "pd_solve_noalloc: " + m);
    }
    return PD_OK;
}
