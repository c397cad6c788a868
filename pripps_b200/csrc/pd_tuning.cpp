// Kernel-shape tuning table: bucket keys and the tuning file.
#include "pd_tuning.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <vector>
#include <sstream>
#include <utility>

#include "pd_kernels.h"

namespace pd {

static int floor_log2(int64_t v) {
    int b = 0;
    while (v > 1) {
        v >>= 1;
        ++b;
    }
    return b;
}

TuneKey tune_key(int64_t n_atoms, int64_t nq, int precision, int mode, int64_t n_frames) {
    return TuneKey(precision, mode, n_frames > 1 ? 1 : 0, floor_log2(std::max<int64_t>(n_atoms, 1)),
                   floor_log2(std::max<int64_t>(nq, 1)));
}

int request_mode(const pd_request *req, const uint32_t *species, const double *weights) {
    if (!req->hyd_weights || !weights) return PD_MODE_CLASS;
    // distinct (species, weight) keys, searched from the previous atom's
    std::vector<std::pair<uint32_t, double>> keys;
    size_t last = 0;
    for (uint64_t i = 0; i < req->n_atoms; ++i) {
        const std::pair<uint32_t, double> k(species[i], weights[i]);
        if (!keys.empty() && keys[last] == k) continue;
        last = std::find(keys.begin(), keys.end(), k) - keys.begin();
        if (last == keys.size()) {
            if (static_cast<int>(keys.size()) == PD_MAX_CLASSES) return PD_MODE_WEIGHTED;
            keys.push_back(k);
        }
    }
    return PD_MODE_CLASS;
}

bool valid_tuning(int precision, int mode, const Tuning &t) {
    if (!valid_q_block(precision, t.K) || t.TJ < 32 || t.TJ % 32 != 0) return false;
    if (precision == PD_FP64) return t.NP == 1;
    return valid_shape(precision, mode, t.K, t.NP);
}

int load_tuning(const std::string &path, TuneTable &tab, std::string &msg) {
    std::ifstream f(path);
    if (!f) {
        msg = "no tuning file at " + path;
        return PD_ENOTFOUND;
    }
    std::string line;
    int lineno = 0;
    TuneTable add;
    while (std::getline(f, line)) {
        ++lineno;
        const size_t hash = line.find('#');
        if (hash != std::string::npos) line.resize(hash);
        std::istringstream is(line);
        std::string prec, mode, frames;
        if (!(is >> prec)) continue;  // blank
        int nb = 0, qb = 0;
        Tuning t;
        double ms = 0;
        const bool ok = static_cast<bool>(is >> mode >> frames >> nb >> qb >> t.K >> t.TJ >> t.NP >> ms);
        std::string extra;
        const int p = prec == "fp32" ? PD_FP32_FP64RED : (prec == "fp64" ? PD_FP64 : -1);
        const int m = mode == "class" ? PD_MODE_CLASS : (mode == "weighted" ? PD_MODE_WEIGHTED : -1);
        const int fr = frames == "single" ? 0 : (frames == "frames" ? 1 : -1);
        if (!ok || (is >> extra) || p < 0 || m < 0 || fr < 0 || nb < 0 || nb > 40 || qb < 0 ||
            qb > 40 || !(ms >= 0.0) || !valid_tuning(p, m, t)) {
            msg = path + ":" + std::to_string(lineno) + ": malformed tuning line";
            return PD_EINVAL;
        }
        add[TuneKey(p, m, fr, nb, qb)] = TuneEntry{t, ms};
    }
    for (auto &kv : add) tab[kv.first] = kv.second;
    return PD_OK;
}

int save_tuning(const std::string &path, const TuneTable &tab, std::string &msg) {
    const std::string tmp = path + ".tmp";
    {
        std::ofstream f(tmp);
        if (!f) {
            msg = "cannot write " + tmp;
            return PD_EINVAL;
        }
        f << "# pripps_b200 kernel-shape tuning table\n"
             "# precision mode frames log2_atoms log2_nq q_block j_chunk pairs_per_thread ms\n";
        for (const auto &kv : tab) {
            const TuneKey &k = kv.first;
            const TuneEntry &e = kv.second;
            char buf[256];
            std::snprintf(buf, sizeof buf, "%s %s %s %d %d %d %d %d %.4f\n",
                          std::get<0>(k) == PD_FP64 ? "fp64" : "fp32",
                          std::get<1>(k) == PD_MODE_WEIGHTED ? "weighted" : "class",
                          std::get<2>(k) ? "frames" : "single", std::get<3>(k), std::get<4>(k),
                          e.t.K, e.t.TJ, e.t.NP, e.ms);
            f << buf;
        }
        if (!f) {
            msg = "write failed: " + tmp;
            return PD_EINVAL;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) {
        msg = "cannot replace " + path;
        return PD_EINVAL;
    }
    return PD_OK;
}

}  // namespace pd
