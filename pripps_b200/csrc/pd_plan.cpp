// Host planner of the Debye backend: classes, padded layout, tiles and the
// fixed-order reduction lists (see pd_common.h for the layout).
#include "pd_plan.h"

#include <algorithm>
#include <cmath>
#include <numeric>
#include <utility>

#include "pd_kernels.h"

namespace pd {

int validate_request(const pd_request *req, bool device_pointers, std::string &msg) {
    if (!req) {
        msg = "request is NULL";
        return PD_EINVAL;
    }
    if (req->n_atoms == 0) {
        msg = "n_atoms must be >= 1";
        return PD_EINVAL;
    }
    if (req->n_atoms > (1ull << 30)) {
        msg = "n_atoms exceeds 2^30";
        return PD_EINVAL;
    }
    if (req->nq == 0 || req->nq > (1ull << 24)) {
        msg = "nq must be in [1, 2^24]";
        return PD_EINVAL;
    }
    if (req->n_species == 0) {
        msg = "n_species must be >= 1";
        return PD_EINVAL;
    }
    if (req->precision != PD_FP32_FP64RED && req->precision != PD_FP64) {
        msg = "precision must be PD_FP32_FP64RED or PD_FP64";
        return PD_EINVAL;
    }
    if (!req->xyz || !req->species || !req->ff_atoms) {
        msg = "xyz, species and ff_atoms are required";
        return PD_EINVAL;
    }
    if (req->hyd_weights && !req->ff_water) {
        msg = "ff_water is required when hyd_weights is given";
        return PD_EINVAL;
    }
    if ((req->flags & ~PD_FLAG_TEST_EXPIRED_WAIT) != 0) {
        msg = "flags must be 0 (or PD_FLAG_TEST_EXPIRED_WAIT)";
        return PD_EINVAL;
    }
    if (req->n_lattices > PD_MAX_LATTICES || (req->n_lattices && !req->lattices)) {
        msg = "n_lattices must be <= " + std::to_string(PD_MAX_LATTICES) +
              " with a lattices array";
        return PD_EINVAL;
    }
    for (uint32_t l = 0; l < req->n_lattices; ++l) {
        const pd_lattice &L = req->lattices[l];
        if (L.species >= req->n_species || L.reserved || L.reserved2 ||
            !(std::isfinite(L.spacing) && L.spacing > 0.0) || !std::isfinite(L.origin[0]) ||
            !std::isfinite(L.origin[1]) || !std::isfinite(L.origin[2]) || L.extent[0] < 1 ||
            L.extent[1] < 1 || L.extent[2] < 1 || L.extent[0] > (1u << 16) ||
            L.extent[1] > (1u << 16) || L.extent[2] > (1u << 16)) {
            msg = "lattice " + std::to_string(l) +
                  ": species < n_species, spacing > 0, finite origin, extents in [1, 65536] "
                  "and zero reserved fields required";
            return PD_EINVAL;
        }
        const double e0 = L.extent[0] - 1.0, e1 = L.extent[1] - 1.0, e2 = L.extent[2] - 1.0;
        if (e0 * e0 + e1 * e1 + e2 * e2 >= static_cast<double>(PD_MAX_LATTICE_BINS)) {
            msg = "lattice " + std::to_string(l) + " is too large: its squared diagonal exceeds " +
                  std::to_string(PD_MAX_LATTICE_BINS) + " grid steps²";
            return PD_EINVAL;
        }
        for (uint32_t m = 0; m < l; ++m)
            if (req->lattices[m].species == L.species) {
                msg = "two lattices name species " + std::to_string(L.species);
                return PD_EINVAL;
            }
    }
    if (req->n_lattices && req->n_frames > 1) {
        msg = "lattice sets need a single frame";
        return PD_EINVAL;
    }
    if (!std::isfinite(req->qmin) || !std::isfinite(req->qmax) || req->qmin < 0.0 ||
        req->qmax < req->qmin) {
        msg = "q range must satisfy 0 <= qmin <= qmax (finite)";
        return PD_EINVAL;
    }
    const uint64_t nf = req->n_frames ? req->n_frames : 1;
    if (nf > (1u << 20)) {
        msg = "n_frames exceeds 2^20";
        return PD_EINVAL;
    }
    if (device_pointers) return PD_OK;
    // Host buffers: check the values the planner and the kernels rely on.
    const uint64_t n = req->n_atoms;
    for (uint64_t i = 0; i < n; ++i) {
        if (req->species[i] >= req->n_species) {
            msg = "species id " + std::to_string(req->species[i]) + " at atom " +
                  std::to_string(i) + " is >= n_species";
            return PD_EINVAL;
        }
    }
    for (uint64_t i = 0; i < n * 3 * nf; ++i) {
        if (!std::isfinite(req->xyz[i])) {
            msg = "non-finite coordinate at index " + std::to_string(i);
            return PD_EINVAL;
        }
    }
    const uint64_t nt = static_cast<uint64_t>(req->n_species) * req->nq;
    for (uint64_t i = 0; i < nt; ++i) {
        if (!std::isfinite(req->ff_atoms[i]) ||
            (req->ff_excluded && !std::isfinite(req->ff_excluded[i]))) {
            msg = "non-finite form-factor table entry";
            return PD_EINVAL;
        }
    }
    if (req->hyd_weights) {
        for (uint64_t i = 0; i < n; ++i)
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
        double s = 0.0;
        for (uint64_t f = 0; f < nf; ++f) {
            if (!std::isfinite(req->frame_weights[f])) {
                msg = "non-finite frame weight";
                return PD_EINVAL;
            }
            s += req->frame_weights[f];
        }
        // trajectory_average rejects a sum that is zero or not normal
        // (src/trajectory.rs:234-238).
        if (!std::isnormal(std::fabs(s))) {
            msg = "frame weights sum to zero or a non-normal value; cannot normalize";
            return PD_EINVAL;
        }
    }
    return PD_OK;
}

static int next_pow2(int64_t v) {
    int p = 1;
    while (p < v && p < (1 << 30)) p <<= 1;
    return p;
}

Tuning fit_tuning(int precision, int mode, Tuning t) {
    // Two accumulators per q (weighted mode) allow q blocks up to 64 (there
    // four pairs per thread measured fastest: 814 ms on the 100,000-atom solve
    // with per-atom hydration weights against 835 ms with two); FP64 runs one
    // pair per pass.
    if (precision == PD_FP64) {
        t.NP = 1;
    } else if (!valid_shape(precision, mode, t.K, t.NP)) {
        if (mode == PD_MODE_WEIGHTED) {
            t.K = t.K > 32 ? 64 : 32;
            t.NP = t.K == 64 ? 4 : 2;
        } else {
            t.NP = t.K == 32 ? 4 : 2;
        }
    }
    return t;
}

Tuning default_tuning(int64_t n_atoms, int64_t nq, int precision, int64_t n_frames) {
    Tuning t;
    if (precision == PD_FP64) {
        t.K = 32;
        t.NP = 1;
        t.TJ = std::clamp(next_pow2(n_atoms / 16), 256, 4096);
        return t;
    }
    // Measured on B200 (class mode): K = 128 with 4 pairs per thread (three
    // CTAs per SM, seeds computed at the top of each pass) is the fastest
    // shape from ~4k atoms up — 546.7 ms on the 100,000-atom solve against
    // 561.5 ms with 2 pairs — and K = 64 with 4 pairs below; a j chunk of about N/8 atoms balances
    // tile count against per-tile overhead. The last q-block of a grid runs
    // only the 16-point chunks that lie on it, so a long block wastes at most
    // 15 grid points per request. (These are the shapes of buckets the tuning
    // table does not name.)
    if (n_atoms < 4000) {
        t.K = 64;
        t.NP = 4;
    } else {
        t.K = 128;
        t.NP = 4;
    }
    if (nq <= 32) {
        t.K = 32;
        t.NP = 4;
    }
    // j chunk: about N/8 atoms, halved while a solve would have fewer than
    // ~6 tiles per resident CTA of a B200 (148 SMs × 3): the longest-first
    // tile order then ends with short tiles on every SM. Measured step times
    // (pair kernel + slot reduction): 10,000 atoms, nq 500: 3.82 / 3.51 /
    // 3.54 / 3.74 ms at 2,048 / 1,024 / 512 / 256; 20,000 atoms, nq 512:
    // 13.24 / 12.78 / 12.89 ms at 4,096 / 2,048 / 1,024; 100,000 atoms, nq
    // 1,000: 589.5 / 592.5 ms at 16,384 / 4,096.
    t.TJ = std::clamp(next_pow2(n_atoms / 8), 256, 16384);
    const double iblocks = static_cast<double>((n_atoms + 127) / 128);
    const double nqb = static_cast<double>((nq + t.K - 1) / t.K);
    const double frames = static_cast<double>(std::max<int64_t>(n_frames, 1));
    while (t.TJ > 256 &&
           iblocks * std::ceil(static_cast<double>(n_atoms) / t.TJ) * 0.5 * nqb * frames <
               6.0 * 148 * 3)
        t.TJ /= 2;
    return t;
}

// The distinct (species, weight) keys of the atoms in ascending order and
// each atom's index among them; false as soon as there are more than
// max_keys. Weights are finite (validated), so equality is the map order's
// equivalence. A linear search from the previous atom's key: atoms of one
// residue or surface patch repeat keys, and there are at most max_keys.
static bool weight_class_keys(int64_t n, const uint32_t *species, const double *w,
                              int max_keys, std::vector<std::pair<uint32_t, double>> &keys,
                              std::vector<int32_t> &atom_key) {
    std::vector<std::pair<uint32_t, double>> seen;  // first-seen order
    size_t last = 0;
    for (int64_t i = 0; i < n; ++i) {
        const std::pair<uint32_t, double> k(species[i], w[i]);
        if (seen.empty() || !(seen[last] == k)) {
            last = std::find(seen.begin(), seen.end(), k) - seen.begin();
            if (last == seen.size()) {
                if (static_cast<int>(seen.size()) == max_keys) return false;
                seen.push_back(k);
            }
        }
        atom_key[i] = static_cast<int32_t>(last);
    }
    std::vector<int32_t> order(seen.size()), rank(seen.size());
    std::iota(order.begin(), order.end(), 0);
    std::sort(order.begin(), order.end(), [&](int32_t a, int32_t b) { return seen[a] < seen[b]; });
    keys.resize(seen.size());
    for (size_t r = 0; r < order.size(); ++r) {
        rank[order[r]] = static_cast<int32_t>(r);
        keys[r] = seen[order[r]];
    }
    for (int64_t i = 0; i < n; ++i) atom_key[i] = rank[atom_key[i]];
    return true;
}

// One key per species present (weight 0), in ascending species order.
static void species_class_keys(int64_t n, const uint32_t *species, int32_t n_species,
                               std::vector<std::pair<uint32_t, double>> &keys,
                               std::vector<int32_t> &atom_key) {
    std::vector<int32_t> rank(n_species, -1);
    for (int64_t i = 0; i < n; ++i) rank[species[i]] = 0;
    keys.clear();
    for (int32_t sp = 0; sp < n_species; ++sp)
        if (rank[sp] >= 0) {
            rank[sp] = static_cast<int32_t>(keys.size());
            keys.emplace_back(static_cast<uint32_t>(sp), 0.0);
        }
    for (int64_t i = 0; i < n; ++i) atom_key[i] = rank[species[i]];
}

int build_plan(const pd_request *req, const uint32_t *species, const double *w,
               const Tuning &tun, Plan &P, std::string &msg, bool count_pairs) {
    P = Plan();
    P.n_atoms = static_cast<int64_t>(req->n_atoms);
    P.nq = static_cast<int32_t>(req->nq);
    P.n_frames = static_cast<int32_t>(req->n_frames ? req->n_frames : 1);
    P.n_species = static_cast<int32_t>(req->n_species);
    P.precision = static_cast<int>(req->precision);
    P.has_exc = req->ff_excluded != nullptr;
    P.has_hyd = req->hyd_weights != nullptr;
    P.test_expire = (req->flags & PD_FLAG_TEST_EXPIRED_WAIT) != 0;
    P.tun = tun;
    if (!valid_q_block(P.precision, tun.K) || tun.TJ < 32 || tun.TJ % 32 != 0 ||
        tun.NP < 1 || tun.NP > 4) {
        msg = "invalid tuning (q block " + std::to_string(tun.K) + ", j chunk " +
              std::to_string(tun.TJ) + ")";
        return PD_EINVAL;
    }
    P.qmin = req->qmin;
    P.qmax = req->qmax;
    // Grid exactly as linear_q_values (src/q_sampler.rs:24-29).
    const double denom = static_cast<double>(P.nq > 1 ? P.nq - 1 : 1);
    P.qv.resize(P.nq);
    for (int k = 0; k < P.nq; ++k)
        P.qv[k] = P.qmin + (P.qmax - P.qmin) * static_cast<double>(k) / denom;
    P.dq = (P.qmax - P.qmin) / denom;

    const int64_t n = P.n_atoms;
    // ---- classes: species, or (species, weight) while few distinct weights;
    // numbered in ascending (species, weight) order
    std::vector<std::pair<uint32_t, double>> keys;
    std::vector<int32_t> atom_cls(n);
    const bool by_weight =
        P.has_hyd && weight_class_keys(n, species, w, PD_MAX_CLASSES, keys, atom_cls);
    if (!by_weight) species_class_keys(n, species, P.n_species, keys, atom_cls);
    P.mode = (P.has_hyd && !by_weight) ? PD_MODE_WEIGHTED : PD_MODE_CLASS;
    P.nv = P.mode == PD_MODE_WEIGHTED ? 4 : 1;
    P.tun = fit_tuning(P.precision, P.mode, P.tun);
    const int c = static_cast<int>(keys.size());
    P.n_cls = c;
    P.cls.assign(c, PdClassDev{});
    for (int ci = 0; ci < c; ++ci) {
        P.cls[ci].species = static_cast<int32_t>(keys[ci].first);
        P.cls[ci].w = keys[ci].second;
    }
    // ---- lattice sets: one class each, class mode only
    std::vector<int> lat_of_cls(c, -1);
    P.lat.clear();
    for (uint32_t l = 0; l < req->n_lattices; ++l) {
        const pd_lattice &L = req->lattices[l];
        int found = -1, count = 0;
        for (int k = 0; k < c; ++k)
            if (P.cls[k].species == static_cast<int32_t>(L.species)) {
                found = k;
                ++count;
            }
        if (count == 0) continue;  // no point of the species: nothing to sum
        if (count > 1 || P.mode != PD_MODE_CLASS) {
            msg = "the points of lattice species " + std::to_string(L.species) +
                  " must share one hydration weight (and the request have at most " +
                  std::to_string(PD_MAX_CLASSES) + " species × weight classes)";
            return PD_EINVAL;
        }
        PdLatDev d{};
        for (int a = 0; a < 3; ++a) {
            d.origin[a] = L.origin[a];
            d.ext[a] = static_cast<int32_t>(L.extent[a]);
        }
        d.spacing = L.spacing;
        d.cls = found;
        const int64_t e0 = L.extent[0] - 1, e1 = L.extent[1] - 1, e2 = L.extent[2] - 1;
        d.n_bins = static_cast<int32_t>(e0 * e0 + e1 * e1 + e2 * e2 + 1);
        lat_of_cls[found] = static_cast<int>(P.lat.size());
        P.lat.push_back(d);
    }
    std::vector<std::vector<int32_t>> members(c);
    for (int64_t i = 0; i < n; ++i) members[atom_cls[i]].push_back(static_cast<int32_t>(i));
    // ---- padded layout
    P.cls_start.assign(c, 0);
    int64_t cur = 0;
    for (int k = 0; k < c; ++k) {
        P.cls_start[k] = static_cast<int32_t>(cur);
        const int64_t nk = static_cast<int64_t>(members[k].size());
        cur += (nk + PD_GRANULE - 1) / PD_GRANULE * PD_GRANULE;
    }
    cur = (cur + PD_IBLOCK - 1) / PD_IBLOCK * PD_IBLOCK;
    if (cur > (int64_t{1} << 31) - PD_IBLOCK) {
        msg = "padded atom count overflows";
        return PD_EINVAL;
    }
    P.n_pad = static_cast<int32_t>(cur);
    P.perm.assign(P.n_pad, -1);
    const int ng = P.n_pad / PD_GRANULE;
    P.gvalid.assign(ng, 0);
    P.gclass.assign(ng, -1);
    for (int k = 0; k < c; ++k) {
        const int64_t nk = static_cast<int64_t>(members[k].size());
        double s1 = 0, s2 = 0;
        for (int64_t r = 0; r < nk; ++r) {
            const int32_t src = members[k][r];
            P.perm[P.cls_start[k] + r] = src;
            if (P.has_hyd) {
                s1 += w[src];
                s2 += w[src] * w[src];
            }
        }
        P.cls[k].n = static_cast<double>(nk);
        P.cls[k].w1 = s1;
        P.cls[k].w2 = s2;
        for (int64_t g = 0; g < (nk + PD_GRANULE - 1) / PD_GRANULE; ++g) {
            const int gi = P.cls_start[k] / PD_GRANULE + static_cast<int>(g);
            P.gclass[gi] = k;
            P.gvalid[gi] = static_cast<int32_t>(std::min<int64_t>(PD_GRANULE, nk - g * PD_GRANULE));
        }
    }
    // ---- class pairs (a <= b) and their exact q = 0 sums
    std::vector<int> pair_index(static_cast<size_t>(c) * c, -1);
    for (int a = 0; a < c; ++a)
        for (int b = a; b < c; ++b) {
            PdPairDev pd{};
            pd.a = a;
            pd.b = b;
            const double na = P.cls[a].n, nb = P.cls[b].n;
            if (a != b) {
                pd.q0[0] = na * nb;
                pd.q0[1] = P.cls[a].w1 * nb;
                pd.q0[2] = na * P.cls[b].w1;
                pd.q0[3] = P.cls[a].w1 * P.cls[b].w1;
            } else {
                pd.q0[0] = na * (na - 1.0) / 2.0;
                // Σ_{i<j} w_i and Σ_{i<j} w_j in padded order within the class.
                double ti = 0, tj = 0, tij = 0, pre = 0;
                const int64_t nk = static_cast<int64_t>(members[a].size());
                for (int64_t r = 0; r < nk; ++r) {
                    const double wr = P.has_hyd ? w[members[a][r]] : 0.0;
                    ti += wr * static_cast<double>(nk - 1 - r);
                    tj += wr * static_cast<double>(r);
                    tij += wr * pre;
                    pre += wr;
                }
                pd.q0[1] = ti;
                pd.q0[2] = tj;
                pd.q0[3] = tij;
            }
            pair_index[a * c + b] = static_cast<int>(P.pairs.size());
            P.pairs.push_back(pd);
        }
    P.n_pairs = static_cast<int>(P.pairs.size());
    // lattice layout: class range, self pair, histogram bins, count tiles
    {
        int64_t off = 0;
        P.lat_tiles.clear();
        for (size_t l = 0; l < P.lat.size(); ++l) {
            PdLatDev &d = P.lat[l];
            d.start = P.cls_start[d.cls];
            d.n = static_cast<int32_t>(members[d.cls].size());
            d.pair = pair_index[d.cls * c + d.cls];
            d.hist_off = off;
            off += d.n_bins;
            for (int32_t i0 = 0; i0 < d.n; i0 += PD_LAT_IBLOCK)
                for (int32_t j0 = i0; j0 < d.n; j0 += PD_LAT_JCHUNK)
                    if (std::min(d.n, j0 + PD_LAT_JCHUNK) - 1 > i0)
                        P.lat_tiles.push_back(PdLatTile{static_cast<int32_t>(l), i0, j0,
                                                        std::min(d.n, j0 + PD_LAT_JCHUNK)});
        }
        P.lat_bins = off;
    }

    // ---- tiles of one frame, in creation order
    const int K = P.tun.K, TJ = P.tun.TJ;
    P.nqb = (P.nq + K - 1) / K;
    struct Tile {
        int32_t i0, j0, j1, cls;
    };
    std::vector<Tile> tiles;
    const int nblocks = P.n_pad / PD_IBLOCK;
    for (int ib = 0; ib < nblocks; ++ib) {
        const int32_t i0 = ib * PD_IBLOCK;
        int min_cls = -1;
        for (int wv = 0; wv < PD_WARPS; ++wv) {
            const int g = ib * PD_WARPS + wv;
            if (P.gvalid[g] > 0) {
                min_cls = P.gclass[g];
                break;
            }
        }
        if (min_cls < 0) continue;
        for (int k = min_cls; k < c; ++k) {
            const int32_t cend = P.cls_start[k] + static_cast<int32_t>(members[k].size());
            const int32_t s0 = std::max(i0, P.cls_start[k]);
            if (cend - 1 <= i0) continue;  // no j > the block's first atom
            if (lat_of_cls[k] >= 0) {
                // a lattice class's self pairs come from its pair counts: drop
                // the tiles whose i atoms all belong to it
                bool all_k = true;
                for (int wv = 0; wv < PD_WARPS; ++wv) {
                    const int g = ib * PD_WARPS + wv;
                    if (P.gvalid[g] > 0 && P.gclass[g] != k) all_k = false;
                }
                if (all_k) continue;
            }
            for (int32_t j0 = s0; j0 < cend; j0 += TJ)
                tiles.push_back(Tile{i0, j0, std::min(cend, j0 + TJ), k});
        }
    }
    P.jobs_per_frame = static_cast<int64_t>(tiles.size()) * P.nqb;
    if (P.jobs_per_frame * P.n_frames > (int64_t{1} << 31) - 1) {
        msg = "too many tiles for one launch; use a larger j chunk";
        return PD_EINVAL;
    }
    // Slots: the warps of one class in an i-block share one slot (the kernel
    // adds them in warp order at the end of the tile); a padding warp (no
    // valid atom, all-zero sums) joins slot 0. Reduction lists: (pair,
    // q-block) -> slots in creation order.
    std::vector<std::vector<int64_t>> lists(static_cast<size_t>(P.n_pairs) * P.nqb);
    std::vector<PdJob> frame_jobs;
    frame_jobs.reserve(P.jobs_per_frame);
    uint64_t covered = 0;
    int64_t next_slot = 0;
    for (const Tile &t : tiles) {
        int rel[PD_WARPS];
        int cls_of_slot[PD_WARPS];
        int nslot = 0;
        int64_t map = 0;
        for (int wv = 0; wv < PD_WARPS; ++wv) {
            const int g = t.i0 / PD_GRANULE + wv;
            const int a = P.gvalid[g] > 0 ? P.gclass[g] : -1;
            int s = -1;
            for (int u = 0; u < nslot && s < 0; ++u)
                if (cls_of_slot[u] == a) s = u;
            if (s < 0 && a < 0 && nslot > 0) s = 0;  // padding joins slot 0
            if (s < 0) {
                s = nslot;
                cls_of_slot[nslot++] = a;
            }
            rel[wv] = s;
            map |= static_cast<int64_t>(s) << (PD_SLOT_MAP_SHIFT + 2 * wv);
        }
        for (int qb = 0; qb < P.nqb; ++qb) {
            PdJob jb{};
            jb.req = 0;
            jb.frame = 0;
            jb.i0 = t.i0;
            jb.j0 = t.j0;
            jb.j1 = t.j1;
            jb.qb = qb;
            jb.slot = next_slot | map;
            frame_jobs.push_back(jb);
            bool listed[PD_WARPS] = {false, false, false, false};
            for (int wv = 0; wv < PD_WARPS; ++wv) {
                const int g = t.i0 / PD_GRANULE + wv;
                const int a = P.gclass[g];
                if (a < 0 || P.gvalid[g] == 0 || a > t.cls) continue;
                if (a == t.cls && lat_of_cls[a] >= 0) continue;  // from the pair counts
                const int64_t ilo = static_cast<int64_t>(g) * PD_GRANULE;
                const int64_t ihi = ilo + P.gvalid[g];  // exclusive
                if (t.j1 - 1 <= ilo) continue;          // every j <= every i
                if (!listed[rel[wv]]) {
                    lists[static_cast<size_t>(pair_index[a * c + t.cls]) * P.nqb + qb].push_back(
                        next_slot + rel[wv]);
                    listed[rel[wv]] = true;
                }
                if (qb == 0 && count_pairs) {
                    // Σ_{i in [ilo, ihi)} max(0, j1 − max(j0, i + 1)): the i
                    // below j0 − 1 see the whole range, the others an
                    // arithmetic series j1 − 1 − i
                    const int64_t j0 = t.j0, j1 = t.j1;
                    const int64_t a_end = std::min(ihi, j0 - 1);
                    if (a_end > ilo) covered += static_cast<uint64_t>((a_end - ilo) * (j1 - j0));
                    const int64_t b0 = std::max(ilo, j0 - 1), b1 = std::min(ihi, j1 - 1);
                    if (b1 > b0)  // terms j1 − 1 − b0 down to j1 − b1
                        covered += static_cast<uint64_t>(((j1 - 1 - b0) + (j1 - b1)) * (b1 - b0) / 2);
                }
            }
            next_slot += nslot;
        }
    }
    P.slots_per_frame = next_slot;
    if (P.slots_per_frame * P.n_frames >= (int64_t{1} << (PD_SLOT_MAP_SHIFT - 1))) {
        msg = "too many tile slots for one request";
        return PD_EINVAL;
    }
    for (const PdLatDev &d : P.lat)
        covered += static_cast<uint64_t>(d.n) * static_cast<uint64_t>(d.n - 1) / 2;
    P.pairs_covered = covered;
    P.lptr.assign(static_cast<size_t>(P.n_pairs) * P.nqb + 1, 0);
    for (size_t e = 0; e < lists.size(); ++e) P.lptr[e + 1] = P.lptr[e] + lists[e].size();
    P.lidx.reserve(P.lptr.back());
    for (auto &l : lists) P.lidx.insert(P.lidx.end(), l.begin(), l.end());

    // Execution order: longest tiles first (j length), stable; replicated
    // per frame with frame-offset slots. A tile's q-block jobs are
    // consecutive in creation order and of one length, so sorting the tiles
    // gives the order a stable sort of the jobs would.
    std::vector<int64_t> order(tiles.size());
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int64_t x, int64_t y) {
        return (tiles[x].j1 - tiles[x].j0) > (tiles[y].j1 - tiles[y].j0);
    });
    P.jobs.reserve(frame_jobs.size() * P.n_frames);
    for (int64_t o : order) {
        for (int qb = 0; qb < P.nqb; ++qb) {
            for (int f = 0; f < P.n_frames; ++f) {
                PdJob jb = frame_jobs[o * P.nqb + qb];
                jb.frame = f;
                jb.slot += static_cast<int64_t>(f) * P.slots_per_frame;
                P.jobs.push_back(jb);
            }
        }
    }
    return PD_OK;
}

int shard_plan(const Plan &full, uint32_t rank, uint32_t world, Plan &out) {
    out = full;
    if (world <= 1) return PD_OK;
    if (rank >= world) return PD_EINVAL;
    const int64_t spf = full.slots_per_frame;
    std::vector<int64_t> remap(static_cast<size_t>(spf), -1);
    auto local_of = [&](const PdJob &jb) {
        return (jb.slot & PD_SLOT_MASK) - static_cast<int64_t>(jb.frame) * spf;
    };
    auto nslot_of = [](const PdJob &jb) {
        int n = 1;
        for (int w = 0; w < PD_WARPS; ++w)
            n = std::max(n, 1 + static_cast<int>((jb.slot >> (PD_SLOT_MAP_SHIFT + 2 * w)) & 3));
        return n;
    };
    out.jobs.clear();
    for (size_t t = rank; t < full.jobs.size(); t += world) {
        const PdJob &jb = full.jobs[t];
        const int64_t loc = local_of(jb);
        for (int s = 0; s < nslot_of(jb); ++s) remap[static_cast<size_t>(loc + s)] = 0;
        out.jobs.push_back(jb);
    }
    // this rank's slots, numbered in their original order (list order kept)
    int64_t k = 0;
    for (auto &r : remap)
        if (r >= 0) r = k++;
    out.slots_per_frame = k;
    for (PdJob &jb : out.jobs) {
        const int64_t loc = local_of(jb);
        jb.slot = (jb.slot & ~PD_SLOT_MASK) |
                  (static_cast<int64_t>(jb.frame) * k + remap[static_cast<size_t>(loc)]);
    }
    out.lidx.clear();
    out.lptr.assign(full.lptr.size(), 0);
    for (size_t e = 0; e + 1 < full.lptr.size(); ++e) {
        for (int64_t x = full.lptr[e]; x < full.lptr[e + 1]; ++x) {
            const int64_t r = remap[static_cast<size_t>(full.lidx[static_cast<size_t>(x)])];
            if (r >= 0) out.lidx.push_back(r);
        }
        out.lptr[e + 1] = static_cast<int64_t>(out.lidx.size());
    }
    return PD_OK;
}

}  // namespace pd
