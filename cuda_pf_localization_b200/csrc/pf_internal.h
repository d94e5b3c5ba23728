// pf_internal.h — particle-filter handle, device layouts and the launchers
// shared between the kernel translation units and the C-ABI layer.
//
// HBM layout (SoA, one plane per component, each plane padded to a multiple
// of 1024 particles so float4 loads stay aligned):
//   state[2]  ping-pong particle sets: px py pz qw qx qy qz   (7 planes)
//   ll        f32 log-likelihood of the last weighting          (1 plane)
//   w         f32 normalised weight (materialised on demand)    (1 plane)
//   anc       i32 ancestor of each particle in the last resample
//   marker    i32 run starts of a resample (-1 elsewhere)
//   prefix    u64 exclusive fixed-point weight prefix per 2048 particles
// plus the injection buckets per 2048-output tile, small per-block partial
// buffers and one CycleCtl control block.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <vector>

#include "pf_common.cuh"

namespace pfb {

constexpr int kEstN = 14;  // pfc_est_sums layout
constexpr int kPrefixBlock = 2048;  // particles per fixed-point prefix entry
constexpr int kCovN = 12;  // pfc_covs layout
// Threads per weighting block (two particles each, 256 particles per block):
// the blocks that finish the kernel's last wave carry half the work of
// 512-particle blocks.  The block partition fixes the softmax partials, so
// the single-filter, batched and sharded weighting kernels all use it.
constexpr int kWThreads = 128;

// Weight plane semantics.
enum WeightMode : int {
    WMODE_UNIFORM = 0,  // w_i = 1.0f / n (not stored)
    WMODE_LL = 1,       // w_i = (float)(exp(ll_i - M) / S), not yet stored
    WMODE_STORED = 2,   // w plane holds the weights
};

struct Planes {
    float* px;
    float* py;
    float* pz;
    float* qw;
    float* qx;
    float* qy;
    float* qz;
};

// Device control block: reduction results and cross-kernel flags.  One copy
// lives in device memory, one mirror in pinned host memory.
struct CycleCtl {
    // softmax
    float ll_max;         // M = max ll
    float ll_sumexp;      // S = sum expf(ll - M), f32 in a fixed order
    int weights_valid;    // 1 when S is finite and > 0
    int wmode;            // WeightMode of the current cloud
    // estimate pass 1
    double est[kEstN];
    double qmean[4];      // device Markley mean (FP64)
    float cov_mean_p[3];  // f32 arguments the covariance pass used
    float cov_mean_q[4];
    double covs[kCovN];
    double ess;           // 1 / sum w^2 of the estimate above
    // fused-cycle decision and outputs
    int resample_now;     // 1 when this cycle resamples
    int resampled;        // set when a resample ran in the current cycle
    double ess_pre;       // ESS before the resample
    double out[PFC_EST_LEN];
    // resample
    unsigned long long lcg;  // resample offset stream (host LCG in reference)
    double u01_override;     // >= 0: use this offset fraction instead of LCG
    uint64_t total_fx;       // fixed-point weight total T
    double total;            // T * 2^-62
    double u0, step;         // systematic offsets
    int resample_valid;      // total finite and > 0
    // diagnostics
    unsigned err;            // ERR_* bits
    int live;                // which ping-pong particle set is current
    // exact fixed-point weight total of the current weights (by-product of
    // the estimate pass) and whether any weight is outside [0,1] / NaN
    uint64_t w_total_fx;
    int w_bad;
    unsigned long long lcg_next;     // LCG word after the running resample
    // sum w^2 of the weights the weight pass (k_ess) materialised, in its
    // fixed order; the estimate queued after it reports this value
    double sq_w;
    // the estimate pass skipped sums 0..12 (a resample follows, the caller
    // said so with pfc_set_ess_hint); pfc_est_sums computes them on demand
    int est_partial;
};

// Fixed-point image of a normalised f32 weight: round-to-nearest-even of
// w * 2^62 (exact in FP64 for w in [0,1]).
__device__ __forceinline__ uint64_t weight_fx(float w) {
    return __double2ull_rn((double)w * 0x1p62);
}
__device__ __forceinline__ bool weight_bad(float w) {
    return !(w >= 0.0f) || !(w <= 1.0f);
}

// Normalised weight of a log-likelihood, in f32 as the reference computes
// it (expf(ll - max) / total, src/cuda/pf_kernels.cu:292-297), with the
// roundings spelled out so every kernel produces the same bits.
__device__ __forceinline__ float weight_from_ll(float l, float M, float S) {
    return __fdiv_rn(expf(__fsub_rn(l, M)), S);
}

// The correctly rounded f32 quotient e / S without the f32 division on the
// common path, given rS = RN(1 / S) in FP64.  The FP64 product p = e * rS
// differs from q = e / S by a relative error below 2^-52 (two FP64
// roundings).  For 24-bit e and S, a quotient in the normal f32 range is
// never a midpoint of the f32 grid (a midpoint's odd part needs 25 bits, the
// odd part of e has at most 24) and lies at least 2^-49 (relative) from every
// midpoint (|e - m S| is a nonzero multiple of ulp(m) * 2^se, S < 2^(se+24)),
// so RN_f32(p) == RN_f32(q): the double-rounding argument of S. A. Figueroa,
// "When is double rounding innocuous?" (SIGNUM Newsletter 30(3), 1995), with
// the product's two roundings counted.
// Below 2^-126 the f32 step is fixed at 2^-149 and exact midpoints occur, so
// the quotient is rounded as an integer count of 2^-149: x = e * 2^149 is an
// integer (exact in FP64) and the result is RNE(x / S) * 2^-149.  With
// q < 2^-125, x / S < 2^24 and y = x * rS is within 2^-29 of it; y decides
// unless it lies within 2^-28 of a half-integer, where the exact residual
// x - (floor(y) + 1/2) S (one FMA: both terms are multiples of 2^min(0, se-1)
// and the residual is tiny) gives the direction and ties go to even.  This
// holds for 1 <= S <= 2^100 (the normaliser is at least 1, the maximum's own
// term).  Zero numerators (underflowed exponentials, most of a sharply
// weighted cloud) return +0 first, so only warps holding a nonzero weight
// below 2^-126 run the integer rounding.  Other operands (NaN, infinities,
// S < 1) take the IEEE division.
__device__ __forceinline__ float weight_div(float e, float S, double rS) {
    const double p = (double)e * rS;
    if (p >= 0x1.0000000000004p-126) return __double2float_rn(p);
    if (e == 0.0f && S > 0.0f) return 0.0f;
    if (e >= 0.0f && S >= 1.0f && S <= 0x1p100f) {
        const double x = (double)e * 0x1p149;
        const double y = __dmul_rn(x, rS);
        const double fl = floor(y);
        const double dm = __dsub_rn(y, fl + 0.5);
        double k = dm > 0.0 ? fl + 1.0 : fl;
        if (fabs(dm) <= 0x1p-28) {
            const double r = fma(-(fl + 0.5), (double)S, x);
            const bool odd = ((long long)fl & 1) != 0;
            k = (r > 0.0 || (r == 0.0 && odd)) ? fl + 1.0 : fl;
        }
        return __double2float_rn(k * 0x1p-149);
    }
    return __fdiv_rn(e, S);
}

// weight_from_ll with rS = RN(1 / S) in FP64 computed once by the caller;
// the same bits as the three-argument form.
__device__ __forceinline__ float weight_from_ll(float l, float M, float S, double rS) {
    return weight_div(expf(__fsub_rn(l, M)), S, rS);
}

// Normalised f32 weight of particle i under the cloud's weight mode.
__device__ __forceinline__ float weight_of(int wmode, long long i, int n,
                                           const float* __restrict__ w,
                                           const float* __restrict__ ll,
                                           float M, float S) {
    if (wmode == 0) return 1.0f / (float)n;
    if (wmode == 2) return w[i];
    return weight_from_ll(ll[i], M, S);
}

// Both ping-pong particle sets, passed to kernels by value.
struct PlaneSet {
    Planes s[2];
};

// Select a set with a register select rather than an indexed parameter
// array (indexing the kernel parameter array with a run-time value makes
// the compiler copy it to local memory).
__device__ __forceinline__ Planes pick_planes(const PlaneSet& ps, int which) {
    Planes p;
    p.px = which ? ps.s[1].px : ps.s[0].px;
    p.py = which ? ps.s[1].py : ps.s[0].py;
    p.pz = which ? ps.s[1].pz : ps.s[0].pz;
    p.qw = which ? ps.s[1].qw : ps.s[0].qw;
    p.qx = which ? ps.s[1].qx : ps.s[0].qx;
    p.qy = which ? ps.s[1].qy : ps.s[0].qy;
    p.qz = which ? ps.s[1].qz : ps.s[0].qz;
    return p;
}

// Kernel kinds for launch accounting and CUDA-event timing.
enum KernelKind : int {
    KK_REINIT = 0,
    KK_PREDICT,
    KK_WEIGHT,
    KK_EST,
    KK_COVS,
    KK_SCAN,
    KK_GATHER,
    KK_INJECT,
    KK_COMMIT,
    KK_MISC,
    KK_COUNT
};

struct PfProfiler {
    bool on = false;
    static constexpr int kPool = 2048;
    cudaEvent_t ev[kPool][2] = {};
    int kind[kPool] = {};
    int used = 0;
    double ms[KK_COUNT] = {};
    long long count[KK_COUNT] = {};
};

struct CycleArgs;

struct PfHandle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    int n = 0;
    int n_pad = 0;
    int cap_obs = 64;
    uint64_t seed = 42;
    uint64_t gen = 0;
    // sharded filter (pfc_shard_init): this handle holds the whole cloud and
    // predicts and weights particles [shard_rank * shard_chunk, ...) of it
    int shard_world = 0;
    int shard_rank = 0;
    int shard_chunk = 0;
    int shard_nobs = 0;  // observations of the slice weighting in flight

    float* d_state[2] = {nullptr, nullptr};  // 7 planes each
    float* d_ll = nullptr;
    float* d_w = nullptr;
    int* d_anc = nullptr;
    uint64_t* d_wprefix = nullptr;      // fixed-point weight prefix per block
    int* d_marker = nullptr;            // run starts of a resample (-1: none)
    int* d_inj_cnt = nullptr;           // injection draws per resampling tile
    int* d_inj_bucket = nullptr;        // their draw indices (inj_cap per tile)
    int inj_cap = 0;
    double* d_part = nullptr;           // per-block partials (max over uses)
    int part_cap = 0;                   // doubles in d_part
    unsigned long long* d_part_u64 = nullptr;  // per-block integer partials
    bool prefix_valid = false;  // ctl w_total_fx and d_wprefix describe the
                                // current weights
    unsigned* d_done = nullptr;         // last-block counters
    CycleCtl* d_ctl = nullptr;
    CycleCtl* h_ctl = nullptr;          // pinned mirror

    // landmarks: device table + host shadow
    float* d_lm = nullptr;
    int lm_count = 0;
    int lm_cap = 0;

    // observations: device buffer + pinned staging ring
    CObservation* d_obs = nullptr;
    int d_obs_cap = 0;
    static constexpr int kRing = 4;
    CObservation* h_obs_ring = nullptr;  // kRing * cap_obs records
    cudaEvent_t ring_ev[kRing] = {};
    int ring_pos = 0;

    // pending (deferred) predict, fused into the next weighting
    bool pending_predict = false;
    uint64_t pending_gen = 0;
    PfcOdom pending_odom{};

    // speculative estimate bookkeeping
    // > 0: the caller resamples when the ESS of the estimate that follows a
    // weighting is below ess_hint * n (pfc_set_ess_hint)
    double ess_hint = 0.0;
    bool est_valid = false;    // h_ctl est/covs describe the current cloud
    bool est_inflight = false; // est + covs launched, not yet synced
    cudaEvent_t est_ev = nullptr;

    int weight_variant = 0;
    bool record_anc = false;
    bool anc_valid = false;
    unsigned inj_epoch = 0;    // injection list epoch (never 0 when used)
    float* d_stage = nullptr;  // AoS staging for snapshot / set_state (7n)

    // fused cycle as a CUDA graph: per-cycle values staged through a pinned
    // ring into d_cargs; the graph is re-captured when its key changes
    CycleArgs* d_cargs = nullptr;
    CycleArgs* h_cargs = nullptr;  // kRing slots
    cudaEvent_t cargs_ev[kRing] = {};
    int cargs_pos = 0;
    bool use_graph = true;
    cudaGraph_t cyc_graph = nullptr;
    cudaGraphExec_t cyc_exec = nullptr;
    long long graph_key[12] = {};
    int graph_kernels = 0;

    // accounting: kernels launched, bytes copied host<->device, host syncs
    PfcStats stats{};
    PfProfiler prof;

    Planes planes(int which) const {
        float* b = d_state[which];
        size_t p = (size_t)n_pad;
        return {b, b + p, b + 2 * p, b + 3 * p, b + 4 * p, b + 5 * p,
                b + 6 * p};
    }
};

// ------------------------------------------------------- accounting helpers
// Bracket one kernel launch: counts it and, when profiling is on, records a
// pair of CUDA events around it on the handle's stream.
void prof_begin(PfHandle* h, int kind);
void prof_drain_public(PfHandle* h);
void prof_end(PfHandle* h, int kind);

struct KernelScope {
    PfHandle* h;
    int kind;
    KernelScope(PfHandle* hh, int k) : h(hh), kind(k) { prof_begin(h, kind); }
    ~KernelScope() { prof_end(h, kind); }
};

// ---------------------------------------------------------------- launchers
// Each returns 0 or -1 (with the error recorded).  All are asynchronous on
// h->stream.

struct PredictArgs {
    int enabled;
    uint64_t gen;
    float t[3], q[4], tstd[3], rstd[3];
};

// Per-cycle values of a fused cycle replayed as a CUDA graph: the kernels of
// the captured cycle read them from device memory (the values passed as
// kernel arguments at capture time are ignored when this pointer is set).
struct CycleArgs {
    PredictArgs pa;
    const CObservation* obs;
    int nobs;
    unsigned inj_epoch;
    unsigned long long gen;
};

struct WeightArgs {
    float sigma_r, sigma_b, gate;
    int nobs;
};

int launch_reinit(PfHandle* h, const float p0[3], const float q0[4],
                  const float pstd[3], const float rstd[3]);
// Reinitialisation around k device-resident planar poses (x, y, yaw).
int launch_reinit_poses(PfHandle* h, const float* d_poses, int k, float z,
                        const float pstd[3], const float rstd[3]);
int launch_predict(PfHandle* h, const PredictArgs& pa);
// Weighting (optionally fused with a deferred predict): writes ll, block
// (max, sumexp) partials and the finalised M, S into the control block.
int launch_weight(PfHandle* h, const PredictArgs& pa, const CObservation* d_obs,
                  int nobs, float sigma_r, float sigma_b, float gate,
                  const CycleArgs* dargs = nullptr);
// A sharded filter's slice (predict + weighting, block partials kept for the
// exchange), and the softmax combine over every rank's partials after it.
int launch_weight_shard(PfHandle* h, const PredictArgs& pa, const CObservation* d_obs,
                        int nobs, float sigma_r, float sigma_b, float gate);
int launch_softmax_combine(PfHandle* h);
// Estimate pass 1 (+ device Markley mean) and the speculative covariance pass
// around (float)mean, (float)qmean.  When use_args is set the covariance pass
// uses the given f32 means instead; cycle_output also assembles the fused
// cycle's output record.  skip_ratio > 0 skips the covariance pass on the
// device when the estimate's ESS is below skip_ratio * n (a resample follows
// and discards it; pfc_covs then computes it on demand).
// sq_from_ess: the weights were just materialised by k_ess, whose sum w^2
// the estimate reports; with skip_ratio > 0 it then skips its other sums when
// the ESS is below skip_ratio * n.
int launch_est_sums(PfHandle* h, bool sq_from_ess = false, double skip_ratio = 0.0);
int launch_covs(PfHandle* h, bool use_args, const float mp[3],
                const float mq[4], bool cycle_output, double skip_ratio = 0.0);
// Systematic resampling fused with the gather, the injection and the
// estimate pass of the resulting cloud (14 FP64 sums, device Markley mean,
// then the commit of the new live set): the weight pass runs first when the
// weights changed since the last, and the injection draws are filed by output
// tile.  cond_on_ctl: resample only when ctl->resample_now, else run the
// estimate pass over the current cloud.
int launch_resample_est(PfHandle* h, float inject_ratio, bool cond_on_ctl,
                        bool use_u01, double u01, const CycleArgs* dargs = nullptr);
// Output tiles of the resampler (injection counts are kept per tile), and the
// injection buckets for k draws (allocated outside any graph capture).
int resample_tiles(int n);
// FP64 partials (doubles of d_part) the resampler uses.
int resample_part_doubles(int n);
int ensure_inject_buckets(PfHandle* h, int k);
// Weight pass before a resample: materialises the weights, their ESS, the
// fixed-point total and the per-block prefixes (kPrefixBlock particles per
// block); with decide set it also takes the fused cycle's resample decision
// (device ESS vs ratio * n).
int launch_weight_prefix(PfHandle* h, bool decide, double ess_ratio);
int launch_cycle_decide(PfHandle* h, double ess_ratio);
int launch_materialize_weights(PfHandle* h);
int launch_pick_from_cum(PfHandle* h, const double* d_cum, int n, double u0,
                         double total, int* d_anc);
// weight_div and the IEEE division side by side on n device pairs (e, S).
int launch_weight_div_check(PfHandle* h, const float* d_e, const float* d_s, int n,
                            float* d_fast, float* d_ieee);

}  // namespace pfb
