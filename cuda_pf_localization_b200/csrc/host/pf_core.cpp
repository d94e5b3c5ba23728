// pf_core.cpp — C++ restatement of the reference's Rust host layer over the
// drop-in C-ABI.  It issues the same pfc_* / pfgl_* calls, with the same
// arguments and in the same order, as crates/pf_core/src/{cuda.rs,
// particle_filter.rs,global_loc.rs}, so the library is exercised exactly as
// the Rust CudaBackend / CudaGlobalLoc exercise it.
#include "pf_core.h"

#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <cmath>
#include <new>
#include <optional>
#include <sstream>
#include <string>
#include <vector>

#include "markley.h"
#include "pfc_abi.h"

namespace {

thread_local std::string t_err;

void set_err(const std::string& s) { t_err = s; }

struct Vec3 {
    double x = 0, y = 0, z = 0;
};

// LandmarkMap, crates/pf_core/src/landmark_map.rs:7-80.
struct LandmarkMap {
    std::vector<std::optional<Vec3>> positions;

    void add(int id, Vec3 p) {
        if (id < 0) return;
        if ((int)positions.size() <= id) positions.resize((size_t)id + 1);
        positions[(size_t)id] = p;
    }
    bool has(int id) const {
        return id >= 0 && (size_t)id < positions.size() &&
               positions[(size_t)id].has_value();
    }
    size_t capacity() const { return positions.size(); }
    size_t len_defined() const {
        size_t n = 0;
        for (const auto& p : positions) n += p.has_value();
        return n;
    }

    // Rust's f64 grammar (str::parse::<f64>): optional sign, then digits with
    // an optional '.' and exponent, or inf / infinity / nan in any case.
    // strtod also takes hexadecimal and "nan(...)" forms, which Rust rejects.
    static bool parse_f64(const std::string& s, double& v) {
        if (s.empty()) return false;
        for (char c : s)
            if (c == 'x' || c == 'X' || c == '(' || c == ')' || isspace((unsigned char)c))
                return false;
        char* end = nullptr;
        v = strtod(s.c_str(), &end);
        return end != s.c_str() && *end == '\0';
    }

    // Rust's `f64 as i32`: truncation toward zero, saturating at the i32
    // range, NaN -> 0.
    static long long saturating_i32(double v) {
        if (std::isnan(v)) return 0;
        if (v >= 2147483647.0) return 2147483647;
        if (v <= -2147483648.0) return -2147483648LL;
        return (long long)v;
    }

    // load_from_str (landmark_map.rs:59-80): '#' starts a comment; '[', ']',
    // ':' and ',' become spaces; a non-empty line must hold exactly four
    // numbers; the id is parsed as f64 and cast.  Each line is added as it is
    // parsed, so the lines before a bad one stay in the map, as in the
    // reference.  A negative id is an error here (the reference's add()
    // panics on it).
    int load_from_str(const std::string& text, std::string& err) {
        std::istringstream in(text);
        std::string line;
        int count = 0, lineno = 0;
        while (std::getline(in, line)) {
            ++lineno;
            const size_t hash = line.find('#');
            if (hash != std::string::npos) line = line.substr(0, hash);
            for (char& c : line)
                if (c == '[' || c == ']' || c == ':' || c == ',') c = ' ';
            std::istringstream ls(line);
            std::vector<std::string> toks;
            std::string t;
            while (ls >> t) toks.push_back(t);
            if (toks.empty()) continue;
            if (toks.size() != 4) {
                err = "line " + std::to_string(lineno) +
                      ": expected 'id: [x, y, z]'";
                return -1;
            }
            double v[4];
            for (int k = 0; k < 4; ++k) {
                if (!parse_f64(toks[(size_t)k], v[k])) {
                    err = "line " + std::to_string(lineno) + ": invalid float literal";
                    return -1;
                }
            }
            const long long id = saturating_i32(v[0]);
            if (id < 0) {
                err = "line " + std::to_string(lineno) +
                      ": landmark ids must be non-negative";
                return -1;
            }
            add((int)id, Vec3{v[1], v[2], v[3]});
            ++count;
        }
        return count;
    }
};

// CudaBackend, crates/pf_core/src/cuda.rs:97-358.
struct CudaBackend {
    void* handle = nullptr;
    int n = 0;
    PfcoreConfig cfg{};
    std::vector<float> lm_cache;
    static constexpr int kObsCap = 256;  // OBS_CAP, cuda.rs:95

    bool create() {
        if (pfc_device_available() != 1) {
            set_err("no CUDA device");
            return false;
        }
        handle = pfc_create(kObsCap);
        if (!handle) {
            set_err("pfc_create failed");
            return false;
        }
        return true;
    }
    ~CudaBackend() {
        if (handle) pfc_destroy(handle);
    }

    bool init(int count, const PfcoreConfig& c) {
        n = count;
        cfg = c;
        if (pfc_init(handle, count, (unsigned)c.seed) != 0) return false;
        // update() resamples when the first estimate's ESS is below
        // ratio * N and then discards that estimate's covariances
        return pfc_set_ess_hint(handle, c.resample_ess_ratio) == 0;
    }

    void reinit(const double pose[7], const double ps[3], const double rs[3]) {
        const float psf[3] = {(float)ps[0], (float)ps[1], (float)ps[2]};
        const float rsf[3] = {(float)rs[0], (float)rs[1], (float)rs[2]};
        pfc_reinit(handle, (float)pose[0], (float)pose[1], (float)pose[2],
                   (float)pose[3], (float)pose[4], (float)pose[5],
                   (float)pose[6], psf, rsf);
    }

    void predict(const PfcoreOdom& o) {
        const float t[3] = {(float)o.trans_noise[0], (float)o.trans_noise[1],
                            (float)o.trans_noise[2]};
        const float r[3] = {(float)o.rot_noise[0], (float)o.rot_noise[1],
                            (float)o.rot_noise[2]};
        pfc_predict(handle, (float)o.translation[0], (float)o.translation[1],
                    (float)o.translation[2], (float)o.rotation[0],
                    (float)o.rotation[1], (float)o.rotation[2],
                    (float)o.rotation[3], t, r);
    }

    // sync_landmarks, cuda.rs:140-154: dense table, upload only on change.
    void sync_landmarks(const LandmarkMap& map) {
        const size_t cap = map.capacity() > 0 ? map.capacity() : 1;
        std::vector<float> flat(cap * 3, 0.0f);
        for (size_t id = 0; id < map.positions.size(); ++id)
            if (map.positions[id]) {
                flat[id * 3] = (float)map.positions[id]->x;
                flat[id * 3 + 1] = (float)map.positions[id]->y;
                flat[id * 3 + 2] = (float)map.positions[id]->z;
            }
        if (flat != lm_cache) {
            pfc_upload_landmarks(handle, flat.data(), (int)cap);
            lm_cache.swap(flat);
        }
    }

    // cuda.rs:227-256: drop observations without a map entry; none left ->
    // pfc_weight(NULL, 0) (uniform weights); else upload the table if it
    // changed and pass at most OBS_CAP observations.
    std::vector<CObservation> cobs;
    void weight(const PfcoreObservation* obs, int nobs, const LandmarkMap& map,
                bool upload_only = false) {
        cobs.clear();
        for (int k = 0; k < nobs; ++k)
            if (map.has(obs[k].landmark_id)) {
                if ((int)cobs.size() >= kObsCap) break;
                const PfcoreObservation& o = obs[k];
                CObservation c;
                c.id = o.landmark_id;
                c.mode = o.mode == 0 ? 0 : 1;
                c.dx = (float)o.vector[0];
                c.dy = (float)o.vector[1];
                c.dz = (float)o.vector[2];
                c.range = (float)o.range;
                cobs.push_back(c);
            }
        const float sr = (float)cfg.range_noise, sb = (float)cfg.bearing_noise,
                    g = (float)cfg.gate_sigma;
        if (upload_only) {
            if (!cobs.empty()) sync_landmarks(map);
            return;
        }
        if (cobs.empty()) {
            pfc_weight(handle, nullptr, 0, sr, sb, g);
            return;
        }
        sync_landmarks(map);
        pfc_weight(handle, cobs.data(), (int)cobs.size(), sr, sb, g);
    }

    void resample(double inject) { pfc_resample(handle, (float)inject); }

    // cuda.rs:264-329, in two steps: the moments (pfc_est_sums, the Markley
    // mean on the host, the ESS), then the covariances around that mean
    // (pfc_covs).  pfc_covs reads the particle state and changes nothing, so
    // a caller that only needs the ESS of an estimate it will discard may
    // stop after the first step.
    bool estimate_moments(PfcoreEstimate& e) {
        memset(&e, 0, sizeof(e));
        if (n == 0) {
            e.attitude[0] = 1.0;
            for (int k = 0; k < 9; ++k) e.pos_cov[k] = e.att_cov[k] = 1.0;
            return true;
        }
        double sums[14];
        if (pfc_est_sums(handle, sums) != 0) {
            set_err("pfc_est_sums failed");
            return false;
        }
        double q[4];
        pfb::markley_mean(&sums[3], q);
        for (int k = 0; k < 3; ++k) e.position[k] = sums[k];
        for (int k = 0; k < 4; ++k) e.attitude[k] = q[k];
        e.ess = sums[13] > 0.0 ? 1.0 / sums[13] : 0.0;
        return true;
    }

    bool estimate_covs(PfcoreEstimate& e) {
        if (n == 0) return true;
        double cv[12];
        if (pfc_covs(handle, (float)e.position[0], (float)e.position[1],
                     (float)e.position[2], (float)e.attitude[0], (float)e.attitude[1],
                     (float)e.attitude[2], (float)e.attitude[3], cv) != 0) {
            set_err("pfc_covs failed");
            return false;
        }
        auto sym3 = [&](int o, double* m) {
            for (int r = 0; r < 3; ++r)
                for (int c = r; c < 3; ++c) {
                    const double x = cv[o + 3 * r - r * (r - 1) / 2 + (c - r)];
                    m[r * 3 + c] = x;
                    m[c * 3 + r] = x;
                }
        };
        sym3(0, e.pos_cov);
        sym3(6, e.att_cov);
        e.valid = 1;
        return true;
    }

    bool estimate(PfcoreEstimate& e) { return estimate_moments(e) && estimate_covs(e); }

    // The ESS of the current estimate alone (1 / sums[13], as estimate()
    // reports it), which is all update() reads of an estimate it discards.
    bool estimate_ess(double& ess) {
        ess = 0.0;
        if (n == 0) return true;
        if (pfc_est_ess(handle, &ess) != 0) {
            set_err("pfc_est_ess failed");
            return false;
        }
        return true;
    }
};

// ParticleFilter, crates/pf_core/src/particle_filter.rs:73-133.
struct ParticleFilter {
    PfcoreConfig cfg{};
    LandmarkMap map;
    CudaBackend backend;
};

struct GlobalLoc {
    void* handle = nullptr;
    PfcoreGlParams params{};
    ~GlobalLoc() {
        if (handle) pfgl_destroy(handle);
    }
};

}  // namespace

extern "C" {

const char* pfcore_last_error(void) { return t_err.c_str(); }

void pfcore_config_default(PfcoreConfig* c) {
    if (!c) return;
    c->particle_count = 4096;
    c->trans_noise[0] = 0.05;
    c->trans_noise[1] = 0.05;
    c->trans_noise[2] = 0.02;
    c->rot_noise[0] = 0.02;
    c->rot_noise[1] = 0.02;
    c->rot_noise[2] = 0.03;
    c->range_noise = 0.05;
    c->bearing_noise = 0.02;
    c->resample_ess_ratio = 0.5;
    c->random_inject_ratio = 0.0;
    c->gate_sigma = 0.0;
    c->seed = 42;
}

void* pfcore_filter_new(const PfcoreConfig* cfg) {
    if (!cfg) return nullptr;
    ParticleFilter* pf = new (std::nothrow) ParticleFilter();
    if (!pf) return nullptr;
    pf->cfg = *cfg;
    if (!pf->backend.create() || !pf->backend.init(cfg->particle_count, *cfg)) {
        if (t_err.empty()) set_err("pfc_init failed");
        delete pf;
        return nullptr;
    }
    return pf;
}

void pfcore_filter_free(void* p) { delete static_cast<ParticleFilter*>(p); }

int pfcore_map_add(void* p, int id, double x, double y, double z) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf) return -1;
    return pfcore_landmarks_add(&pf->map, id, x, y, z);
}

int pfcore_map_clear(void* p) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf) return -1;
    pf->map.positions.clear();
    return 0;
}

int pfcore_map_load_text(void* p, const char* text) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf || !text) return -1;
    return pfcore_landmarks_load_text(&pf->map, text);
}

int pfcore_map_capacity(void* p) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    return pf ? (int)pf->map.capacity() : -1;
}

// ---- LandmarkMap as a value of its own (landmark_map.rs:7-80), host only.

void* pfcore_landmarks_new(void) { return new (std::nothrow) LandmarkMap(); }

void pfcore_landmarks_free(void* m) { delete static_cast<LandmarkMap*>(m); }

int pfcore_landmarks_add(void* mv, int id, double x, double y, double z) {
    LandmarkMap* m = static_cast<LandmarkMap*>(mv);
    if (!m) return -1;
    if (id < 0) {
        set_err("landmark ids must be non-negative");
        return -1;
    }
    try {
        m->add(id, Vec3{x, y, z});
    } catch (const std::bad_alloc&) {
        set_err("landmark id too large to allocate");
        return -1;
    }
    return 0;
}

int pfcore_landmarks_has(void* mv, int id) {
    const LandmarkMap* m = static_cast<const LandmarkMap*>(mv);
    return m && m->has(id) ? 1 : 0;
}

int pfcore_landmarks_at(void* mv, int id, double out[3]) {
    const LandmarkMap* m = static_cast<const LandmarkMap*>(mv);
    if (!m || !out || !m->has(id)) {
        set_err("landmark id not present");
        return -1;
    }
    const Vec3& p = *m->positions[(size_t)id];
    out[0] = p.x;
    out[1] = p.y;
    out[2] = p.z;
    return 0;
}

int pfcore_landmarks_capacity(void* mv) {
    const LandmarkMap* m = static_cast<const LandmarkMap*>(mv);
    return m ? (int)m->capacity() : -1;
}

int pfcore_landmarks_len_defined(void* mv) {
    const LandmarkMap* m = static_cast<const LandmarkMap*>(mv);
    return m ? (int)m->len_defined() : -1;
}

int pfcore_landmarks_load_text(void* mv, const char* text) {
    LandmarkMap* m = static_cast<LandmarkMap*>(mv);
    if (!m || !text) return -1;
    std::string err;
    int n;
    try {
        n = m->load_from_str(text, err);
    } catch (const std::bad_alloc&) {
        err = "landmark id too large to allocate";
        n = -1;
    }
    if (n < 0) set_err(err);
    return n;
}

int pfcore_filter_set_map(void* p, void* mv) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    const LandmarkMap* m = static_cast<const LandmarkMap*>(mv);
    if (!pf || !m) return -1;
    pf->map = *m;
    return 0;
}

int pfcore_filter_reinitialize(void* p, const double pose[7],
                               const double pos_std[3],
                               const double rot_std[3]) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf || !pose || !pos_std || !rot_std) return -1;
    pf->backend.reinit(pose, pos_std, rot_std);
    return 0;
}

int pfcore_filter_update(void* p, const PfcoreOdom* odom,
                         const PfcoreObservation* obs, int nobs,
                         PfcoreEstimate* out) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf || !odom || !out) return -1;
    pf->backend.predict(*odom);
    pf->backend.weight(obs, obs ? nobs : 0, pf->map);
    // update() estimates, then resamples and estimates again when the ESS is
    // low.  Of the first estimate only its ESS decides when it is discarded;
    // the library, told the rule (pfc_set_ess_hint), then reports only the
    // ESS, and the full estimate is taken of the one returned.  The returned
    // estimate is the same.
    PfcoreEstimate est;
    double ess0 = 0.0;
    if (!pf->backend.estimate_ess(ess0)) return -1;
    const double threshold =
        pf->cfg.resample_ess_ratio * (double)pf->cfg.particle_count;
    int resampled = 0;
    if (pf->cfg.resample_ess_ratio > 0.0 && ess0 < threshold) {
        pf->backend.resample(pf->cfg.random_inject_ratio);
        if (!pf->backend.estimate(est)) return -1;
        resampled = 1;
    } else if (!pf->backend.estimate(est)) {
        return -1;
    }
    est.resampled = resampled;
    *out = est;
    return 0;
}

int pfcore_filter_update_fused(void* p, const PfcoreOdom* odom,
                               const PfcoreObservation* obs, int nobs,
                               PfcoreEstimate* out) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf || !odom || !out) return -1;
    CudaBackend& be = pf->backend;
    // Same observation filtering and landmark upload as the plain path.
    be.weight(obs, obs ? nobs : 0, pf->map, /*upload_only=*/true);
    PfcOdom o;
    for (int k = 0; k < 3; ++k) {
        o.t[k] = (float)odom->translation[k];
        o.tstd[k] = (float)odom->trans_noise[k];
        o.rstd[k] = (float)odom->rot_noise[k];
    }
    for (int k = 0; k < 4; ++k) o.q[k] = (float)odom->rotation[k];
    PfcCycleParams prm{};
    prm.sigma_r = (float)pf->cfg.range_noise;
    prm.sigma_b = (float)pf->cfg.bearing_noise;
    prm.gate = (float)pf->cfg.gate_sigma;
    prm.resample_ess_ratio = pf->cfg.resample_ess_ratio;
    prm.random_inject_ratio = (float)pf->cfg.random_inject_ratio;
    double r[PFC_EST_LEN];
    if (pfc_cycle(be.handle, &o, be.cobs.data(), (int)be.cobs.size(), &prm,
                  r) != 0) {
        set_err(pfc_last_error_message());
        return -1;
    }
    memset(out, 0, sizeof(*out));
    for (int k = 0; k < 3; ++k) out->position[k] = r[PFC_EST_POS + k];
    for (int k = 0; k < 4; ++k) out->attitude[k] = r[PFC_EST_QUAT + k];
    auto sym3 = [&](int o0, double* m) {
        int e = 0;
        for (int rr = 0; rr < 3; ++rr)
            for (int c = rr; c < 3; ++c) {
                m[rr * 3 + c] = r[o0 + e];
                m[c * 3 + rr] = r[o0 + e];
                ++e;
            }
    };
    sym3(PFC_EST_POSCOV, out->pos_cov);
    sym3(PFC_EST_ATTCOV, out->att_cov);
    out->ess = r[PFC_EST_ESS];
    out->valid = 1;
    out->resampled = r[PFC_EST_RESAMPLED] != 0.0;
    return 0;
}

int pfcore_filter_snapshot(void* p, double* pos3n, double* quat4n, double* w) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    if (!pf || !pos3n || !quat4n) return -1;
    const int n = pf->backend.n;
    std::vector<float> pos((size_t)n * 3), quat((size_t)n * 4), wf((size_t)n);
    if (pfc_snapshot(pf->backend.handle, pos.data(), quat.data()) != 0)
        return -1;
    for (size_t i = 0; i < pos.size(); ++i) pos3n[i] = pos[i];
    for (size_t i = 0; i < quat.size(); ++i) quat4n[i] = quat[i];
    if (w) {
        if (pfc_get_weights(pf->backend.handle, wf.data()) != 0) return -1;
        for (int i = 0; i < n; ++i) w[i] = wf[(size_t)i];
    }
    return 0;
}

void* pfcore_filter_handle(void* p) {
    ParticleFilter* pf = static_cast<ParticleFilter*>(p);
    return pf ? pf->backend.handle : nullptr;
}

void pfcore_quat_mean(const double m10[10], double q_out[4]) {
    pfb::markley_mean(m10, q_out);
}

// ------------------------------------------------------------------- GL

void pfcore_gl_params_default(PfcoreGlParams* p) {
    if (!p) return;
    p->hypotheses = 50000;
    p->rays = 360;
    p->rmax = 10.0;
    p->ang_span = 6.283185307179586;
    p->topk = 10;
    p->seed = 42;
}

void* pfcore_gl_new(int w, int h, double res, double ox, double oy,
                    const unsigned char* cells, const PfcoreGlParams* p) {
    if (!cells || !p) return nullptr;
    GlobalLoc* g = new (std::nothrow) GlobalLoc();
    if (!g) return nullptr;
    g->params = *p;
    g->handle = pfgl_create(w, h, (float)res, (float)ox, (float)oy, cells,
                            p->hypotheses);
    if (!g->handle) {
        set_err("pfgl_create failed");
        delete g;
        return nullptr;
    }
    return g;
}

void pfcore_gl_free(void* gv) { delete static_cast<GlobalLoc*>(gv); }

int pfcore_gl_free_cells(void* gv) {
    GlobalLoc* g = static_cast<GlobalLoc*>(gv);
    return g ? pfgl_free_cells(g->handle) : -1;
}

int pfcore_gl_set_seed(void* gv, unsigned long long seed) {
    GlobalLoc* g = static_cast<GlobalLoc*>(gv);
    if (!g) return -1;
    g->params.seed = seed;
    return 0;
}

// CudaGlobalLoc::localize, global_loc.rs:306-327.
int pfcore_gl_localize(void* gv, const float* scan, int nrays,
                       PfcorePoseHypothesis* out) {
    GlobalLoc* g = static_cast<GlobalLoc*>(gv);
    if (!g || !scan || !out) return -1;
    const PfcoreGlParams& p = g->params;
    if (pfgl_generate(g->handle, p.hypotheses, p.seed) != 0) {
        set_err("pfgl_generate failed");
        return -1;
    }
    if (pfgl_score(g->handle, scan, nrays, (float)p.rmax, (float)p.ang_span) !=
        0) {
        set_err("pfgl_score failed");
        return -1;
    }
    std::vector<float> o((size_t)p.topk * 3);
    const int k = pfgl_topk(g->handle, p.topk, o.data());
    if (k <= 0) {
        set_err("pfgl_topk failed");
        return -1;
    }
    for (int j = 0; j < k; ++j) {
        out[j].x = o[(size_t)j * 3];
        out[j].y = o[(size_t)j * 3 + 1];
        out[j].theta = o[(size_t)j * 3 + 2];
        out[j].caer = NAN;
    }
    return k;
}

void* pfcore_gl_handle(void* gv) {
    GlobalLoc* g = static_cast<GlobalLoc*>(gv);
    return g ? g->handle : nullptr;
}

// OccGrid::from_pgm_yaml, global_loc.rs:30-130: minimal YAML keys
// (resolution, origin, occupied_thresh default 0.65), P5 PGM, occupied when
// (255 - px)/255 > thresh, rows flipped so row 0 is the lowest y.
int pfcore_grid_from_pgm_yaml(const unsigned char* pgm, size_t pgm_len,
                              const char* yaml, int* w, int* h, double* res,
                              double* ox, double* oy, unsigned char* cells) {
    if (!pgm || !yaml || !w || !h || !res || !ox || !oy) return -1;
    auto strip = [](std::string s) {
        const size_t a = s.find_first_not_of(" \t\r");
        if (a == std::string::npos) return std::string();
        const size_t b = s.find_last_not_of(" \t\r");
        return s.substr(a, b - a + 1);
    };
    auto get_f = [&](const std::string& key, double& out) -> bool {
        std::istringstream in(yaml);
        std::string line;
        bool hit = false;
        while (std::getline(in, line)) {
            std::string t = line.substr(0, line.find('#'));
            t = strip(t);
            if (t.compare(0, key.size(), key) != 0) continue;
            std::string rest = strip(t.substr(key.size()));
            if (rest.empty() || rest[0] != ':') continue;
            rest = strip(rest.substr(1));
            char* end = nullptr;
            const double v = strtod(rest.c_str(), &end);
            if (end != rest.c_str() && *end == '\0') {
                out = v;
                hit = true;
            } else {
                hit = false;
            }
        }
        return hit;
    };
    double r = 0.0;
    if (!get_f("resolution", r)) {
        set_err("yaml: no resolution");
        return -1;
    }
    double o_x = 0.0, o_y = 0.0;
    {
        std::istringstream in(yaml);
        std::string line;
        bool found = false;
        while (std::getline(in, line)) {
            const std::string t = strip(line);
            if (t.compare(0, 6, "origin") != 0) continue;
            const size_t lb = line.find('[');
            if (lb == std::string::npos) break;
            std::string body = line.substr(lb + 1);
            while (!body.empty() && (body.back() == ']' || body.back() == '\r' ||
                                     body.back() == ' '))
                body.pop_back();
            std::vector<double> vals;
            std::istringstream bs(body);
            std::string tok;
            while (std::getline(bs, tok, ',')) {
                tok = strip(tok);
                char* end = nullptr;
                const double v = strtod(tok.c_str(), &end);
                if (end != tok.c_str() && *end == '\0') vals.push_back(v);
            }
            if (!vals.empty()) o_x = vals[0];
            if (vals.size() > 1) o_y = vals[1];
            found = true;
            break;
        }
        if (!found) {
            set_err("yaml: no origin");
            return -1;
        }
    }
    double occ_th = 0.65;
    get_f("occupied_thresh", occ_th);
    // P5 header tokens with '#' comments.
    size_t idx = 0;
    auto token = [&](std::string& out) -> bool {
        for (;;) {
            while (idx < pgm_len && isspace(pgm[idx])) ++idx;
            if (idx < pgm_len && pgm[idx] == '#') {
                while (idx < pgm_len && pgm[idx] != '\n') ++idx;
                continue;
            }
            break;
        }
        const size_t start = idx;
        while (idx < pgm_len && !isspace(pgm[idx])) ++idx;
        if (start == idx) return false;
        out.assign((const char*)pgm + start, idx - start);
        return true;
    };
    std::string magic, ws, hs, ms;
    if (!token(magic)) {
        set_err("pgm: truncated");
        return -1;
    }
    if (magic != "P5") {
        set_err("pgm: expected P5, got " + magic);
        return -1;
    }
    if (!token(ws) || !token(hs) || !token(ms)) {
        set_err("pgm: truncated");
        return -1;
    }
    const long W = strtol(ws.c_str(), nullptr, 10),
               H = strtol(hs.c_str(), nullptr, 10);
    if (W <= 0 || H <= 0) {
        set_err("pgm: bad size");
        return -1;
    }
    idx += 1;  // single whitespace after maxval
    const size_t need = (size_t)W * (size_t)H;
    if (pgm_len < idx + need) {
        set_err("pgm: short pixel data");
        return -1;
    }
    *w = (int)W;
    *h = (int)H;
    *res = r;
    *ox = o_x;
    *oy = o_y;
    if (!cells) return 0;
    for (long y = 0; y < H; ++y)
        for (long x = 0; x < W; ++x) {
            const unsigned char px = pgm[idx + (size_t)y * W + x];
            const double occ_p = (double)(255 - px) / 255.0;
            cells[(size_t)(H - 1 - y) * W + x] = occ_p > occ_th ? 1 : 0;
        }
    return 0;
}

}  // extern "C"
