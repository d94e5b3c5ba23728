// pf_oracle.cpp — CPU ORACLE.  TEST INFRASTRUCTURE ONLY.
//
// Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load
// this library; the product (libpf_kernels.so / libpf_core.so) never calls
// into it.  It restates, in plain C++ (FP64 unless stated), the reference's
// CPU algorithms for the particle-filter cycle and the global-localization
// stage, each function citing the reference file:line it follows (paths
// within the reference project), plus CPU mirrors of the deterministic
// specifications of the GPU path (fixed-point resampling, Philox noise,
// splitmix injection, composite-key bottom-k, the f32 DDA) so those can be
// checked bit for bit.
//
// Pinning: the reference ships no golden vectors; the oracle is pinned by the
// reference's own known-answer and tolerance tests (crates/pf_core/tests/
// {integration,cuda_agreement,global_loc}.rs), restated in tests/, and by
// fixtures produced by the reference library itself (tests/golden/).
//
// Parallelism mirrors the reference's rayon split: OpenMP over the par_iter
// regions (reinit, predict, log-likelihoods, CAER), everything else
// sequential (cpu.rs:182-192,199-216,234-248; global_loc.rs:388-394).
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <numeric>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

extern "C" {

// ----------------------------------------------------------------- types

struct OrcQ {
    double w, x, y, z;
};
struct OrcV {
    double x, y, z;
};

static inline OrcQ qmul(const OrcQ& a, const OrcQ& b) {
    return {a.w * b.w - a.x * b.x - a.y * b.y - a.z * b.z,
            a.w * b.x + a.x * b.w + a.y * b.z - a.z * b.y,
            a.w * b.y - a.x * b.z + a.y * b.w + a.z * b.x,
            a.w * b.z + a.x * b.y - a.y * b.x + a.z * b.w};
}
static inline OrcQ qconj(const OrcQ& q) { return {q.w, -q.x, -q.y, -q.z}; }
static inline OrcV cross(const OrcV& a, const OrcV& b) {
    return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
// nalgebra UnitQuaternion::transform_vector: t = 2 u x v; v + w t + u x t.
static inline OrcV qrot(const OrcQ& q, const OrcV& v) {
    OrcV u{q.x, q.y, q.z};
    OrcV t = cross(u, v);
    t = {2 * t.x, 2 * t.y, 2 * t.z};
    OrcV c = cross(u, t);
    return {v.x + q.w * t.x + c.x, v.y + q.w * t.y + c.y, v.z + q.w * t.z + c.z};
}

// --------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon et al., SC'11), restated independently of the
// product code; the GPU noise spec is (seed, particle, generation, block).
static void orc_philox(uint32_t c[4], uint32_t k0, uint32_t k1) {
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += 0x9E3779B9u;
            k1 += 0xBB67AE85u;
        }
        const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
        const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
        const uint32_t n0 = (uint32_t)(p1 >> 32) ^ c[1] ^ k0;
        const uint32_t n1 = (uint32_t)p1;
        const uint32_t n2 = (uint32_t)(p0 >> 32) ^ c[3] ^ k1;
        const uint32_t n3 = (uint32_t)p0;
        c[0] = n0;
        c[1] = n1;
        c[2] = n2;
        c[3] = n3;
    }
}

void orc_philox4x32_10(const uint32_t ctr[4], uint64_t key, uint32_t out[4]) {
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    orc_philox(c, (uint32_t)key, (uint32_t)(key >> 32));
    memcpy(out, c, sizeof(c));
}

static inline double u01o(uint32_t x) {
    return ((double)(x >> 9) + 0.5) * (1.0 / 8388608.0);
}

// Six standard normals of particle i in generation gen (Box–Muller in FP64).
void orc_normals6(uint64_t seed, uint64_t gen, uint32_t i, double n[6]) {
    uint32_t a[4] = {i, (uint32_t)gen, (uint32_t)(gen >> 32), 0u};
    uint32_t b[4] = {i, (uint32_t)gen, (uint32_t)(gen >> 32), 1u};
    orc_philox(a, (uint32_t)seed, (uint32_t)(seed >> 32));
    orc_philox(b, (uint32_t)seed, (uint32_t)(seed >> 32));
    const double u[6] = {u01o(a[0]), u01o(a[1]), u01o(a[2]),
                         u01o(a[3]), u01o(b[0]), u01o(b[1])};
    for (int k = 0; k < 3; ++k) {
        const double r = std::sqrt(-2.0 * std::log(u[2 * k]));
        n[2 * k] = r * std::cos(2.0 * M_PI * u[2 * k + 1]);
        n[2 * k + 1] = r * std::sin(2.0 * M_PI * u[2 * k + 1]);
    }
}

// noise_dq, crates/pf_core/src/cpu.rs:30-42.
static OrcQ noise_dq(const double rs[3], const double w3[3]) {
    const OrcV ax{rs[0] * w3[0], rs[1] * w3[1], rs[2] * w3[2]};
    const double ang = std::sqrt(ax.x * ax.x + ax.y * ax.y + ax.z * ax.z);
    if (!(ang > 1e-12)) return {1, 0, 0, 0};
    const double s = std::sin(0.5 * ang) / ang;
    return {std::cos(0.5 * ang), ax.x * s, ax.y * s, ax.z * s};
}

// ------------------------------------------------------ particle filter

// CpuBackend state, crates/pf_core/src/cpu.rs:99-112 (SoA, FP64).
struct OrcPf {
    int n;
    uint64_t seed;
    uint64_t gen;
    std::vector<OrcV> pos;
    std::vector<OrcQ> att;
    std::vector<double> w;
    double range_noise, bearing_noise, gate, ess_ratio, inject;
    uint64_t lcg;
};

void* orc_pf_new(int n, uint64_t seed, double range_noise, double bearing_noise,
                 double gate, double ess_ratio, double inject) {
    OrcPf* p = new OrcPf();
    p->n = n;
    p->seed = seed ? seed : 42;
    p->gen = 0;
    p->pos.assign((size_t)n, OrcV{0, 0, 0});
    p->att.assign((size_t)n, OrcQ{1, 0, 0, 0});
    p->w.assign((size_t)n, 1.0 / n);
    p->range_noise = range_noise;
    p->bearing_noise = bearing_noise;
    p->gate = gate;
    p->ess_ratio = ess_ratio;
    p->inject = inject;
    p->lcg = 0x243F6A8885A308D3ull;
    return p;
}

void orc_pf_free(void* h) { delete static_cast<OrcPf*>(h); }

int orc_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}

void orc_set_threads(int t) {
#ifdef _OPENMP
    if (t > 0) omp_set_num_threads(t);
#else
    (void)t;
#endif
}

// pos3n / quat4n (w first) / w, FP64 in and out.
void orc_pf_set_state(void* h, const double* pos3n, const double* quat4n,
                      const double* w) {
    OrcPf* p = static_cast<OrcPf*>(h);
    for (int i = 0; i < p->n; ++i) {
        p->pos[(size_t)i] = {pos3n[3 * i], pos3n[3 * i + 1], pos3n[3 * i + 2]};
        p->att[(size_t)i] = {quat4n[4 * i], quat4n[4 * i + 1], quat4n[4 * i + 2],
                             quat4n[4 * i + 3]};
        p->w[(size_t)i] = w ? w[i] : 1.0 / p->n;
    }
}

void orc_pf_get_state(void* h, double* pos3n, double* quat4n, double* w) {
    OrcPf* p = static_cast<OrcPf*>(h);
    for (int i = 0; i < p->n; ++i) {
        const OrcV& v = p->pos[(size_t)i];
        const OrcQ& q = p->att[(size_t)i];
        pos3n[3 * i] = v.x;
        pos3n[3 * i + 1] = v.y;
        pos3n[3 * i + 2] = v.z;
        quat4n[4 * i] = q.w;
        quat4n[4 * i + 1] = q.x;
        quat4n[4 * i + 2] = q.y;
        quat4n[4 * i + 3] = q.z;
        if (w) w[i] = p->w[(size_t)i];
    }
}

void orc_pf_set_gen(void* h, uint64_t gen) { static_cast<OrcPf*>(h)->gen = gen; }
void orc_pf_set_lcg(void* h, uint64_t lcg) { static_cast<OrcPf*>(h)->lcg = lcg; }

// reinit, crates/pf_core/src/cpu.rs:180-195 (noise from the Philox spec).
void orc_pf_reinit(void* h, const double pose[7], const double ps[3],
                   const double rs[3]) {
    OrcPf* p = static_cast<OrcPf*>(h);
    p->gen++;
    const OrcQ q0{pose[3], pose[4], pose[5], pose[6]};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i) {
        double nz[6];
        orc_normals6(p->seed, p->gen, (uint32_t)i, nz);
        p->pos[(size_t)i] = {pose[0] + ps[0] * nz[0], pose[1] + ps[1] * nz[1],
                             pose[2] + ps[2] * nz[2]};
        p->att[(size_t)i] = qmul(q0, noise_dq(rs, nz + 3));
    }
    std::fill(p->w.begin(), p->w.end(), 1.0 / p->n);
}

// predict, crates/pf_core/src/cpu.rs:197-218.
void orc_pf_predict(void* h, const double t[3], const double qodo[4],
                    const double tn[3], const double rn[3]) {
    OrcPf* p = static_cast<OrcPf*>(h);
    p->gen++;
    const OrcQ qo{qodo[0], qodo[1], qodo[2], qodo[3]};
#pragma omp parallel for schedule(static)
    for (int i = 0; i < p->n; ++i) {
        double nz[6];
        orc_normals6(p->seed, p->gen, (uint32_t)i, nz);
        const OrcV body{t[0] + tn[0] * nz[0], t[1] + tn[1] * nz[1],
                        t[2] + tn[2] * nz[2]};
        const OrcQ q = p->att[(size_t)i];
        const OrcV wd = qrot(q, body);
        OrcV& v = p->pos[(size_t)i];
        v = {v.x + wd.x, v.y + wd.y, v.z + wd.z};
        p->att[(size_t)i] = qmul(qmul(q, qo), noise_dq(rn, nz + 3));
    }
}

// MeasModel, crates/pf_core/src/cpu.rs:44-97: gated Cartesian and
// range-bearing log-likelihoods.  lm: dense table of 3 doubles per id;
// obs: (id, mode, vx, vy, vz, range) rows, already filtered to known ids.
struct OrcObs {
    int id;
    int mode;
    double v[3];
    double range;
};

static double meas_ll(const OrcV& pred, const OrcObs& o, double sr_in,
                      double sb_in, double gate) {
    const double sr = std::max(sr_in, 1e-6), sb = std::max(sb_in, 1e-6);
    const double inv2rr = 1.0 / (2.0 * sr * sr), inv2bb = 1.0 / (2.0 * sb * sb);
    const double g2 = gate * gate;
    if (o.mode == 0) {
        const double ex = pred.x - o.v[0], ey = pred.y - o.v[1],
                     ez = pred.z - o.v[2];
        const double r2 = ex * ex + ey * ey + ez * ez;
        if (gate > 0.0 && r2 > g2 * 3.0 * sr * sr) return -0.5 * gate * gate * 3.0;
        return -r2 * inv2rr;
    }
    const double rn =
        std::max(std::sqrt(pred.x * pred.x + pred.y * pred.y + pred.z * pred.z), 1e-9);
    const double er = rn - o.range;
    double dot = -(pred.x * o.v[0] + pred.y * o.v[1] + pred.z * o.v[2]) / rn;
    dot = std::min(1.0, std::max(-1.0, dot));
    const double eb = std::acos(dot);
    const double rl = (gate > 0.0 && er * er > g2 * sr * sr) ? -0.5 * gate * gate
                                                             : -er * er * inv2rr;
    const double bl = (gate > 0.0 && eb * eb > g2 * sb * sb) ? -0.5 * gate * gate
                                                             : -eb * eb * inv2bb;
    return rl + bl;
}

// Log-likelihood of every particle (the par_iter of cpu.rs:234-248).
void orc_loglik(int n, const double* pos3n, const double* quat4n,
                const double* lm3, int lm_count, const OrcObs* obs, int nobs,
                double sr, double sb, double gate, double* ll) {
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const OrcV p{pos3n[3 * i], pos3n[3 * i + 1], pos3n[3 * i + 2]};
        const OrcQ qc = qconj({quat4n[4 * i], quat4n[4 * i + 1],
                               quat4n[4 * i + 2], quat4n[4 * i + 3]});
        double acc = 0.0;
        for (int k = 0; k < nobs; ++k) {
            const OrcObs& o = obs[k];
            if (o.id < 0 || o.id >= lm_count) continue;
            const OrcV d{lm3[3 * o.id] - p.x, lm3[3 * o.id + 1] - p.y,
                         lm3[3 * o.id + 2] - p.z};
            acc += meas_ll(qrot(qc, d), o, sr, sb, gate);
        }
        ll[i] = acc;
    }
}

// weight, crates/pf_core/src/cpu.rs:220-260 (obs already filtered; nobs == 0
// means uniform).  Returns 1 when the softmax was applied, 0 when uniform.
int orc_pf_weight(void* h, const double* lm3, int lm_count, const OrcObs* obs,
                  int nobs) {
    OrcPf* p = static_cast<OrcPf*>(h);
    const int n = p->n;
    if (nobs <= 0) {
        std::fill(p->w.begin(), p->w.end(), 1.0 / n);
        return 0;
    }
    std::vector<double> ll((size_t)n);
    const double sr = std::max(p->range_noise, 1e-6), sb = std::max(p->bearing_noise, 1e-6);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n; ++i) {
        const OrcV pp = p->pos[(size_t)i];
        const OrcQ qc = qconj(p->att[(size_t)i]);
        double acc = 0.0;
        for (int k = 0; k < nobs; ++k) {
            const OrcObs& o = obs[k];
            const OrcV d{lm3[3 * o.id] - pp.x, lm3[3 * o.id + 1] - pp.y,
                         lm3[3 * o.id + 2] - pp.z};
            acc += meas_ll(qrot(qc, d), o, sr, sb, p->gate);
        }
        ll[(size_t)i] = acc;
    }
    double mx = -INFINITY;
    for (double v : ll) mx = std::max(mx, v);
    double sum = 0.0;
    for (double v : ll) sum += std::exp(v - mx);
    if (!(sum > 0.0) || !std::isfinite(sum)) {
        std::fill(p->w.begin(), p->w.end(), 1.0 / n);
        return 0;
    }
    for (int i = 0; i < n; ++i) p->w[(size_t)i] = std::exp(ll[(size_t)i] - mx) / sum;
    return 1;
}

// splitmix64 step (Steele, Lea, Flood 2014), the generator of the reference's
// k_inject (src/cuda/pf_kernels.cu:323-352).
static inline uint64_t orc_sm64(uint64_t& z) {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t r = z;
    r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
    r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
    return r ^ (r >> 31);
}

// Draw j of the injection stream: particle index and f32 jitter.
void orc_inject_draw(uint64_t lcg, uint64_t gen, int j, int n, int* idx,
                     float jit[3]) {
    uint64_t z = lcg ^ (gen * 0x9E3779B97F4A7C15ull) ^
                 ((uint64_t)j + 1) * 0xBF58476D1CE4E5B9ull;
    if (z == 0) z = 0x243F6A8885A308D3ull;
    double u = (double)(orc_sm64(z) >> 11) * (1.0 / 9007199254740992.0);
    int k = (int)(u * n);
    *idx = k >= n ? n - 1 : k;
    for (int c = 0; c < 3; ++c) {
        u = (double)(orc_sm64(z) >> 11) * (1.0 / 9007199254740992.0);
        jit[c] = (float)(u - 0.5);
    }
}

// LCG advance of the reference's resample offset (pf_kernels.cu:653-657).
uint64_t orc_lcg_next(uint64_t lcg) {
    return lcg * 6364136223846793005ull + 1442695040888963407ull;
}
double orc_lcg_u01(uint64_t lcg) {
    return (double)(lcg >> 11) * (1.0 / 9007199254740992.0);
}

// Fixed-point systematic resampling spec of the GPU path: W = rn(w * 2^62),
// exact integer scan, t_i = u0 + i*step (two roundings), ancestor = first j
// with C_j >= ceil(t_i * 2^62), clamped.  Returns 1 when valid, 0 when the
// total is invalid (weights then reset to uniform, no gather).
int orc_resample_fixed(const float* w, int n, double u01, int* anc,
                       double* total_out) {
    std::vector<uint64_t> C((size_t)n);
    uint64_t run = 0;
    for (int j = 0; j < n; ++j) {
        const float wf = w[j];
        if (!(wf >= 0.0f) || !(wf <= 1.0f)) return 0;
        run += (uint64_t)std::nearbyint((double)wf * 0x1p62);
        C[(size_t)j] = run;
    }
    if (run == 0) return 0;
    const double total = (double)run * 0x1p-62;
    if (total_out) *total_out = total;
    const double step = total / (double)n;
    const double u0 = u01 * step;
    int j = 0;
    for (int i = 0; i < n; ++i) {
        volatile double prod = (double)i * step;
        const double t = u0 + prod;
        const double s = t * 0x1p62;
        uint64_t T;
        if (!(s > 0.0))
            T = 0;
        else if (s >= 0x1p64)
            T = ~0ull;
        else
            T = (uint64_t)std::ceil(s);
        while (j < n - 1 && C[(size_t)j] < T) ++j;
        anc[i] = j;
    }
    return 1;
}

// The reference CPU resample with an f64 sequential cum (cpu.rs:262-306)
// and a given offset fraction; ancestors only.
int orc_resample_f64(const double* w, int n, double u01, int* anc) {
    std::vector<double> cum((size_t)n);
    cum[0] = w[0];
    for (int i = 1; i < n; ++i) cum[(size_t)i] = cum[(size_t)i - 1] + w[i];
    const double total = cum[(size_t)n - 1];
    if (total <= 0.0 || !std::isfinite(total)) return 0;
    const double u0 = u01 * (total / (double)n);
    const double step = total / (double)n;
    int j = 0;
    for (int i = 0; i < n; ++i) {
        volatile double prod = (double)i * step;
        const double t = u0 + prod;
        while (j < n - 1 && cum[(size_t)j] < t) ++j;
        anc[i] = j;
    }
    return 1;
}

// The reference's GPU pick rule on a given cum (pf_kernels.cu:304-321):
// t = fma(i, step, u0), lower_bound, clamp.
void orc_pick_from_cum(const double* cum, int n, double u0, double total,
                       int* anc) {
    const double step = total / (double)n;
    for (int i = 0; i < n; ++i) {
        const double t = std::fma((double)i, step, u0);
        int lo = 0, hi = n - 1;
        while (lo < hi) {
            const int mid = (lo + hi) >> 1;
            if (cum[mid] < t)
                lo = mid + 1;
            else
                hi = mid;
        }
        anc[i] = lo;
    }
}

// Apply k injections to f32 positions (3n) in ascending draw order.
void orc_inject_apply(float* pos3n, int n, int k, uint64_t lcg, uint64_t gen) {
    for (int j = 0; j < k; ++j) {
        int idx;
        float jit[3];
        orc_inject_draw(lcg, gen, j, n, &idx, jit);
        pos3n[3 * idx] += jit[0];
        pos3n[3 * idx + 1] += jit[1];
        pos3n[3 * idx + 2] += jit[2];
    }
}

// resample on the FP64 backend: f64 sequential cum (cpu.rs), offset from the
// reference LCG stream, injection from the splitmix stream (f64 positions).
void orc_pf_resample(void* h) {
    OrcPf* p = static_cast<OrcPf*>(h);
    const int n = p->n;
    std::vector<double> cum((size_t)n);
    cum[0] = p->w[0];
    for (int i = 1; i < n; ++i) cum[(size_t)i] = cum[(size_t)i - 1] + p->w[(size_t)i];
    const double total = cum[(size_t)n - 1];
    if (total <= 0.0 || !std::isfinite(total)) return;
    p->lcg = orc_lcg_next(p->lcg);
    const double step = total / (double)n;
    const double u0 = orc_lcg_u01(p->lcg) * step;
    std::vector<OrcV> op((size_t)n);
    std::vector<OrcQ> oa((size_t)n);
    int j = 0;
    for (int i = 0; i < n; ++i) {
        const double t = u0 + (double)i * step;
        while (j < n - 1 && cum[(size_t)j] < t) ++j;
        op[(size_t)i] = p->pos[(size_t)j];
        oa[(size_t)i] = p->att[(size_t)j];
    }
    if (p->inject > 0.0) {
        int k = (int)((float)p->inject * (float)n);
        if (k > n) k = n;
        for (int jj = 0; jj < k; ++jj) {
            int idx;
            float jit[3];
            orc_inject_draw(p->lcg, p->gen, jj, n, &idx, jit);
            op[(size_t)idx].x += jit[0];
            op[(size_t)idx].y += jit[1];
            op[(size_t)idx].z += jit[2];
        }
    }
    p->pos.swap(op);
    p->att.swap(oa);
    std::fill(p->w.begin(), p->w.end(), 1.0 / n);
}

// Symmetric 4x4 eigenproblem by cyclic Jacobi (Golub & Van Loan 8.5);
// eigenvalues on the diagonal of a, eigenvectors in the columns of v.
static void orc_jacobi4(double a[16], double v[16]) {
    for (int i = 0; i < 16; ++i) v[i] = (i % 5 == 0) ? 1.0 : 0.0;
    for (int sweep = 0; sweep < 100; ++sweep) {
        double off = 0.0;
        for (int p = 0; p < 4; ++p)
            for (int q = p + 1; q < 4; ++q) off += a[p * 4 + q] * a[p * 4 + q];
        if (off < 1e-300) break;
        for (int p = 0; p < 3; ++p)
            for (int q = p + 1; q < 4; ++q) {
                const double apq = a[p * 4 + q];
                if (std::fabs(apq) < 1e-300) continue;
                const double th = (a[q * 4 + q] - a[p * 4 + p]) / (2.0 * apq);
                const double t = (th >= 0 ? 1.0 : -1.0) /
                                 (std::fabs(th) + std::sqrt(th * th + 1.0));
                const double c = 1.0 / std::sqrt(t * t + 1.0), s = t * c;
                for (int k = 0; k < 4; ++k) {
                    const double x = a[k * 4 + p], y = a[k * 4 + q];
                    a[k * 4 + p] = c * x - s * y;
                    a[k * 4 + q] = s * x + c * y;
                }
                for (int k = 0; k < 4; ++k) {
                    const double x = a[p * 4 + k], y = a[q * 4 + k];
                    a[p * 4 + k] = c * x - s * y;
                    a[q * 4 + k] = s * x + c * y;
                }
                for (int k = 0; k < 4; ++k) {
                    const double x = v[k * 4 + p], y = v[k * 4 + q];
                    v[k * 4 + p] = c * x - s * y;
                    v[k * 4 + q] = s * x + c * y;
                }
            }
    }
}

// quat_mean, crates/pf_core/src/types.rs:128-143: largest eigenvalue's
// eigenvector of (M^T + M)/2, normalised, w >= 0.  m = full 4x4 row-major.
void orc_quat_mean(const double m[16], double q[4]) {
    double a[16], v[16];
    for (int r = 0; r < 4; ++r)
        for (int c = 0; c < 4; ++c) a[r * 4 + c] = 0.5 * (m[r * 4 + c] + m[c * 4 + r]);
    orc_jacobi4(a, v);
    int idx = 0;
    for (int i = 1; i < 4; ++i)
        if (a[i * 4 + i] > a[idx * 4 + idx]) idx = i;
    double x[4] = {v[idx], v[4 + idx], v[8 + idx], v[12 + idx]};
    const double nr = std::sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2] + x[3] * x[3]);
    const double s = x[0] < 0.0 ? -1.0 : 1.0;
    for (int k = 0; k < 4; ++k) q[k] = s * x[k] / nr;
}

// The 14 sums of pfc_est_sums from f32 state and f32 weights, in FP64
// (layout src/cuda/pf_kernels.cu:354-357; semantics cpu.rs:308-320).
void orc_est_sums(int n, const float* pos3n, const float* quat4n,
                  const float* w, double out[14]) {
    for (int k = 0; k < 14; ++k) out[k] = 0.0;
    for (int i = 0; i < n; ++i) {
        const double wi = (double)w[i];
        out[0] += wi * (double)pos3n[3 * i];
        out[1] += wi * (double)pos3n[3 * i + 1];
        out[2] += wi * (double)pos3n[3 * i + 2];
        const double q[4] = {(double)quat4n[4 * i], (double)quat4n[4 * i + 1],
                             (double)quat4n[4 * i + 2], (double)quat4n[4 * i + 3]};
        int e = 3;
        for (int r = 0; r < 4; ++r)
            for (int c = r; c < 4; ++c) out[e++] += wi * q[r] * q[c];
        out[13] += wi * wi;
    }
}

// Canonical attitude residual (cpu.rs:346-366).
static void att_res(const OrcQ& qm, const OrcQ& q, double aav[3]) {
    OrcQ d = qmul(qconj(qm), q);
    if (d.w < 0.0) d = {-d.w, -d.x, -d.y, -d.z};
    const double hv = std::sqrt(d.x * d.x + d.y * d.y + d.z * d.z);
    const double ang = 2.0 * std::atan2(hv, d.w);
    if (hv > 1e-12) {
        aav[0] = d.x / hv * ang;
        aav[1] = d.y / hv * ang;
        aav[2] = d.z / hv * ang;
    } else {
        aav[0] = aav[1] = aav[2] = 0.0;
    }
}

// The 12 sums of pfc_covs around given f32 means, in FP64 (layout
// pf_kernels.cu:406-410; semantics cpu.rs:322-366).
void orc_covs(int n, const float* pos3n, const float* quat4n, const float* w,
              const float mp[3], const float mq[4], double out[12]) {
    for (int k = 0; k < 12; ++k) out[k] = 0.0;
    const OrcQ qm{(double)mq[0], (double)mq[1], (double)mq[2], (double)mq[3]};
    for (int i = 0; i < n; ++i) {
        const double wi = (double)w[i];
        const double dp[3] = {(double)pos3n[3 * i] - (double)mp[0],
                              (double)pos3n[3 * i + 1] - (double)mp[1],
                              (double)pos3n[3 * i + 2] - (double)mp[2]};
        int e = 0;
        for (int r = 0; r < 3; ++r)
            for (int c = r; c < 3; ++c) out[e++] += wi * dp[r] * dp[c];
        double aav[3];
        att_res(qm, {(double)quat4n[4 * i], (double)quat4n[4 * i + 1],
                     (double)quat4n[4 * i + 2], (double)quat4n[4 * i + 3]},
                aav);
        for (int r = 0; r < 3; ++r)
            for (int c = r; c < 3; ++c) out[e++] += wi * aav[r] * aav[c];
    }
}

// estimate, crates/pf_core/src/cpu.rs:308-368.  out: pos[3], quat[4],
// pos_cov[9], att_cov[9], ess.
void orc_pf_estimate(void* h, double* out) {
    OrcPf* p = static_cast<OrcPf*>(h);
    double s2 = 0.0;
    for (double x : p->w) s2 += x * x;
    const double ess = s2 > 0.0 ? 1.0 / s2 : 0.0;
    double m[16] = {0};
    OrcV mean{0, 0, 0};
    for (int i = 0; i < p->n; ++i) {
        const double w = p->w[(size_t)i];
        const OrcV& v = p->pos[(size_t)i];
        mean = {mean.x + w * v.x, mean.y + w * v.y, mean.z + w * v.z};
        const OrcQ& q = p->att[(size_t)i];
        const double qq[4] = {q.w, q.x, q.y, q.z};
        for (int r = 0; r < 4; ++r)
            for (int c = 0; c < 4; ++c) m[r * 4 + c] += w * qq[r] * qq[c];
    }
    double qm[4];
    orc_quat_mean(m, qm);
    const OrcQ qmq{qm[0], qm[1], qm[2], qm[3]};
    double pc[9] = {0}, ac[9] = {0};
    for (int i = 0; i < p->n; ++i) {
        const double w = p->w[(size_t)i];
        const OrcV& v = p->pos[(size_t)i];
        const double dp[3] = {v.x - mean.x, v.y - mean.y, v.z - mean.z};
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) pc[r * 3 + c] += w * dp[r] * dp[c];
        double aav[3];
        att_res(qmq, p->att[(size_t)i], aav);
        for (int r = 0; r < 3; ++r)
            for (int c = 0; c < 3; ++c) ac[r * 3 + c] += w * aav[r] * aav[c];
    }
    out[0] = mean.x;
    out[1] = mean.y;
    out[2] = mean.z;
    for (int k = 0; k < 4; ++k) out[3 + k] = qm[k];
    for (int k = 0; k < 9; ++k) out[7 + k] = pc[k];
    for (int k = 0; k < 9; ++k) out[16 + k] = ac[k];
    out[25] = ess;
}

// ParticleFilter::update (particle_filter.rs:111-124) on the FP64 backend.
// Returns 1 when the cycle resampled.  est_out as orc_pf_estimate.
int orc_pf_update(void* h, const double t[3], const double qodo[4],
                  const double tn[3], const double rn[3], const double* lm3,
                  int lm_count, const OrcObs* obs, int nobs, double* est_out) {
    OrcPf* p = static_cast<OrcPf*>(h);
    orc_pf_predict(h, t, qodo, tn, rn);
    std::vector<OrcObs> valid;
    for (int k = 0; k < nobs; ++k)
        if (obs[k].id >= 0 && obs[k].id < lm_count) valid.push_back(obs[k]);
    orc_pf_weight(h, lm3, lm_count, valid.data(), (int)valid.size());
    orc_pf_estimate(h, est_out);
    if (p->ess_ratio > 0.0 && est_out[25] < p->ess_ratio * (double)p->n) {
        orc_pf_resample(h);
        orc_pf_estimate(h, est_out);
        return 1;
    }
    return 0;
}

// ---------------------------------------------------- global localization

struct OrcGrid {
    int w, h;
    double res, ox, oy;
    const unsigned char* cells;
};

// world_to_cell + cast_ray, crates/pf_core/src/global_loc.rs:136-196 (FP64,
// occupied == 1).
double orc_cast_ray(int W, int H, double res, double ox, double oy,
                    const unsigned char* cells, double px, double py,
                    double dirx, double diry, double rmax) {
    const double fx = (px - ox) / res, fy = (py - oy) / res;
    if (fx < 0.0 || fy < 0.0) return rmax;
    uint64_t cx = (uint64_t)fx, cy = (uint64_t)fy;
    if (!(cx < (uint64_t)W && cy < (uint64_t)H)) return rmax;
    const int64_t sx = dirx > 0.0 ? 1 : -1, sy = diry > 0.0 ? 1 : -1;
    const double adx = std::fabs(dirx), ady = std::fabs(diry);
    const double tdx = adx > 1e-9 ? res / adx : INFINITY;
    const double tdy = ady > 1e-9 ? res / ady : INFINITY;
    const double frx = (px - ox) / res - (double)cx;
    const double fry = (py - oy) / res - (double)cy;
    double tmx = adx > 1e-9 ? (dirx > 0.0 ? 1.0 - frx : frx) * tdx : INFINITY;
    double tmy = ady > 1e-9 ? (diry > 0.0 ? 1.0 - fry : fry) * tdy : INFINITY;
    for (int s = 0; s < 8192; ++s) {
        double dist;
        if (tmx <= tmy) {
            dist = tmx;
            tmx += tdx;
            cx = (uint64_t)((int64_t)cx + sx);
        } else {
            dist = tmy;
            tmy += tdy;
            cy = (uint64_t)((int64_t)cy + sy);
        }
        if (dist > rmax) return rmax;
        if (cx >= (uint64_t)W || cy >= (uint64_t)H) return rmax;
        if (cells[cy * (uint64_t)W + cx] == 1) return std::min(dist, rmax);
    }
    return rmax;
}

// map_scan, global_loc.rs:198-214.
void orc_map_scan(int W, int H, double res, double ox, double oy,
                  const unsigned char* cells, double x, double y, double th,
                  int nrays, double span, double rmax, double* out) {
    for (int r = 0; r < nrays; ++r) {
        const double a =
            th + (nrays > 1 ? span * (double)r / (double)(nrays - 1) : 0.0);
        out[r] = orc_cast_ray(W, H, res, ox, oy, cells, x, y, std::cos(a),
                              std::sin(a), rmax);
    }
}

// caer_of, global_loc.rs:216-221, for n hypotheses (x,y,theta rows);
// parallel over hypotheses like CpuGlobalLoc::localize.
void orc_caer(int W, int H, double res, double ox, double oy,
              const unsigned char* cells, const double* scan, int nrays,
              double span, double rmax, const double* hyp3, int n,
              double* caer) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        double acc = 0.0;
        const double x = hyp3[3 * i], y = hyp3[3 * i + 1], th = hyp3[3 * i + 2];
        for (int r = 0; r < nrays; ++r) {
            const double a =
                th + (nrays > 1 ? span * (double)r / (double)(nrays - 1) : 0.0);
            acc += std::fabs(scan[r] - orc_cast_ray(W, H, res, ox, oy, cells, x, y,
                                                    std::cos(a), std::sin(a), rmax));
        }
        caer[i] = acc;
    }
}

// disperse, global_loc.rs:356-382 (xorshift64, s % 1e6 / 1e6).
void orc_disperse(int W, int H, double res, double ox, double oy,
                  const unsigned char* cells, int n, uint64_t seed,
                  double* hyp3) {
    uint64_t s = seed | 1;
    auto next_u = [&s]() {
        s ^= s << 13;
        s ^= s >> 7;
        s ^= s << 17;
        return (double)(s % 1000000ull) / 1000000.0;
    };
    std::vector<std::pair<int, int>> fr;
    for (int i = 0; i < W * H; ++i)
        if (cells[i] == 0) fr.push_back({i % W, i / W});
    if (fr.empty()) return;
    for (int k = 0; k < n; ++k) {
        size_t idx = (size_t)(next_u() * (double)fr.size());
        if (idx > fr.size() - 1) idx = fr.size() - 1;
        const auto c = fr[idx];
        const double x = ox + ((double)c.first + next_u()) * res;
        const double y = oy + ((double)c.second + next_u()) * res;
        const double th = -M_PI + next_u() * (2.0 * M_PI);
        hyp3[3 * k] = x;
        hyp3[3 * k + 1] = y;
        hyp3[3 * k + 2] = th;
    }
}

// CpuGlobalLoc::localize, global_loc.rs:384-398: disperse, CAER, stable
// sort ascending, truncate.  out rows (x, y, theta, caer).  Returns count.
int orc_gl_localize(int W, int H, double res, double ox, double oy,
                    const unsigned char* cells, const double* scan, int nrays,
                    double span, double rmax, int nh, int topk, uint64_t seed,
                    double* out4) {
    std::vector<double> hyp((size_t)nh * 3), caer((size_t)nh);
    orc_disperse(W, H, res, ox, oy, cells, nh, seed, hyp.data());
    orc_caer(W, H, res, ox, oy, cells, scan, nrays, span, rmax, hyp.data(), nh,
             caer.data());
    std::vector<int> order((size_t)nh);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(),
                     [&](int a, int b) { return caer[(size_t)a] < caer[(size_t)b]; });
    const int k = std::min(topk, nh);
    for (int j = 0; j < k; ++j) {
        const int i = order[(size_t)j];
        out4[4 * j] = hyp[3 * (size_t)i];
        out4[4 * j + 1] = hyp[3 * (size_t)i + 1];
        out4[4 * j + 2] = hyp[3 * (size_t)i + 2];
        out4[4 * j + 3] = caer[(size_t)i];
    }
    return k;
}

// Bottom-k of f32 scores ordered by (float_as_ordered key, index): the order
// of the reference's stable radix sort (pf_kernels.cu:151-155,995-1023).
static inline int ordered_i(float f) {
    int i;
    memcpy(&i, &f, 4);
    return i >= 0 ? i : (i ^ 0x7FFFFFFF);
}
void orc_topk_from_scores(const float* caer, int n, int k, int* idx) {
    std::vector<int> order((size_t)n);
    std::iota(order.begin(), order.end(), 0);
    std::stable_sort(order.begin(), order.end(), [&](int a, int b) {
        return ordered_i(caer[a]) < ordered_i(caer[b]);
    });
    for (int j = 0; j < std::min(k, n); ++j) idx[j] = order[(size_t)j];
}

// f32 mirror of the GPU DDA (pf_kernels.cu:774-808: any nonzero byte is
// occupied, floorf start cell) for one ray with a given direction.
float orc_cast_ray_f32(int W, int H, float res, float ox, float oy,
                       const unsigned char* cells, float px, float py,
                       float dirx, float diry, float rmax) {
    const float fx = (px - ox) / res, fy = (py - oy) / res;
    int cx = (int)std::floor(fx), cy = (int)std::floor(fy);
    if (!(cx >= 0 && cy >= 0 && cx < W && cy < H)) return rmax;
    const int sx = dirx > 0 ? 1 : -1, sy = diry > 0 ? 1 : -1;
    const float adx = std::fabs(dirx), ady = std::fabs(diry);
    const float tdx = adx > 1e-9f ? res / adx : INFINITY;
    const float tdy = ady > 1e-9f ? res / ady : INFINITY;
    const float frx = (px - ox) / res - (float)cx;
    const float fry = (py - oy) / res - (float)cy;
    float tmx = adx > 1e-9f ? ((dirx > 0 ? 1.f - frx : frx) * tdx) : INFINITY;
    float tmy = ady > 1e-9f ? ((diry > 0 ? 1.f - fry : fry) * tdy) : INFINITY;
    for (int s = 0; s < 8192; ++s) {
        float dist;
        if (tmx <= tmy) {
            dist = tmx;
            tmx += tdx;
            cx += sx;
        } else {
            dist = tmy;
            tmy += tdy;
            cy += sy;
        }
        if (dist > rmax) return rmax;
        if (cx < 0 || cy < 0 || cx >= W || cy >= H) return rmax;
        if (cells[(size_t)cy * W + cx]) return dist;
    }
    return rmax;
}

// DDA cell steps of every ray of n hypotheses until the first occupied cell
// or the step that leaves the grid, as the GPU scorer's loop takes them (no
// range or step limit inside the loop); directions from cos/sin of the f32
// ray angle.  Hypotheses outside the grid cast no ray.
long long orc_dda_visits(int W, int H, float res, float ox, float oy,
                         const unsigned char* cells, const float* hyp3, int n,
                         int nrays, float span) {
    long long total = 0;
#pragma omp parallel for schedule(dynamic, 16) reduction(+ : total)
    for (int i = 0; i < n; ++i) {
        const float px = hyp3[3 * i], py = hyp3[3 * i + 1], th = hyp3[3 * i + 2];
        const float fx = (px - ox) / res, fy = (py - oy) / res;
        const int cx0 = (int)std::floor(fx), cy0 = (int)std::floor(fy);
        if (!(cx0 >= 0 && cy0 >= 0 && cx0 < W && cy0 < H)) continue;
        for (int r = 0; r < nrays; ++r) {
            const float a = th + (nrays > 1 ? span * (float)r / (float)(nrays - 1) : 0.f);
            const float dirx = std::cos(a), diry = std::sin(a);
            int cx = cx0, cy = cy0;
            const int sx = dirx > 0 ? 1 : -1, sy = diry > 0 ? 1 : -1;
            const float adx = std::fabs(dirx), ady = std::fabs(diry);
            const float tdx = adx > 1e-9f ? res / adx : INFINITY;
            const float tdy = ady > 1e-9f ? res / ady : INFINITY;
            const float frx = (px - ox) / res - (float)cx;
            const float fry = (py - oy) / res - (float)cy;
            float tmx = adx > 1e-9f ? ((dirx > 0 ? 1.f - frx : frx) * tdx) : INFINITY;
            float tmy = ady > 1e-9f ? ((diry > 0 ? 1.f - fry : fry) * tdy) : INFINITY;
            for (;;) {
                ++total;
                if (tmx <= tmy) {
                    tmx += tdx;
                    cx += sx;
                } else {
                    tmy += tdy;
                    cy += sy;
                }
                if (cx < 0 || cy < 0 || cx >= W || cy >= H) break;
                if (cells[(size_t)cy * W + cx]) break;
            }
        }
    }
    return total;
}

// f32 CAER mirror (directions from sinf/cosf of the f32 ray angle).
void orc_caer_f32(int W, int H, float res, float ox, float oy,
                  const unsigned char* cells, const float* scan, int nrays,
                  float span, float rmax, const float* hyp3, int n,
                  float* caer) {
#pragma omp parallel for schedule(dynamic, 64)
    for (int i = 0; i < n; ++i) {
        const float x = hyp3[3 * i], y = hyp3[3 * i + 1], th = hyp3[3 * i + 2];
        double acc = 0.0;
        for (int r = 0; r < nrays; ++r) {
            const float a =
                th + (nrays > 1 ? span * (float)r / (float)(nrays - 1) : 0.f);
            const float d = orc_cast_ray_f32(W, H, res, ox, oy, cells, x, y,
                                             std::cos(a), std::sin(a), rmax);
            acc += std::fabs(scan[r] - d);
        }
        caer[i] = (float)acc;
    }
}

// Uniform dispersion spec of the GPU path (Philox counter (p,0,0,2), the
// reference's cell/offset/yaw mapping, f32 with the device's fused
// multiply-adds).
void orc_gl_generate(int nfree, const int* free_xy, float ox, float oy,
                     float res, int n_pos, int n_yaw, uint64_t seed,
                     float* hyp3) {
    for (int p = 0; p < n_pos; ++p) {
        uint32_t c[4] = {(uint32_t)p, 0u, 0u, 2u};
        orc_philox(c, (uint32_t)seed, (uint32_t)(seed >> 32));
        const float ux = (float)u01o(c[0]), uy = (float)u01o(c[1]),
                    uz = (float)u01o(c[2]), uw = (float)u01o(c[3]);
        const int cell = std::min((int)(uw * (float)nfree), nfree - 1);
        const float th0 = std::fma(6.28318530f, uz, -3.14159265f);
        const float x = std::fma((float)free_xy[2 * cell] + ux, res, ox);
        const float y = std::fma((float)free_xy[2 * cell + 1] + uy, res, oy);
        for (int j = 0; j < n_yaw; ++j) {
            const int i = p * n_yaw + j;
            hyp3[3 * i] = x;
            hyp3[3 * i + 1] = y;
            hyp3[3 * i + 2] =
                n_yaw > 1 ? std::fma(6.28318530f / (float)n_yaw, (float)j, th0)
                          : th0;
        }
    }
}

}  // extern "C"
