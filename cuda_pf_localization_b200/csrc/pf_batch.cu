// pf_batch.cu — many independent particle filters of uneven size advanced by
// one CUDA-graph launch per cycle.
//
// Layout.  All filters' particles live in one arena of SoA planes (two
// ping-pong sets of px py pz qw qx qy qz, plus ll, w and the resampler's
// run-start markers); filter f owns the
// slice [off_f, off_f + n_f), off_f a multiple of 1024.  Every kernel of the
// cycle covers all filters through a tile table: a tile is a particle range
// of one filter.  Per-filter reductions are finished by the last tile of that
// filter to complete (an atomic counter per filter), so a cycle is a fixed
// chain of kernels whatever the filter sizes:
//   begin -> weight (+ predict) -> weights + ESS decision -> resample
//   (look-back scan, run-start markers) -> gather (ancestors from the
//   markers, the copy, the estimate sums of the new cloud per tile) ->
//   injection (link, apply, each draw's position change) -> commit ->
//   estimate sums of the resampled filters (tile partials + injection
//   changes, Markley mean) -> estimate pass of the others -> covariances
//   (output record).
// The chain is captured once into a CUDA graph; a cycle is one graph launch
// fed by one copy of the per-filter inputs.
//
// Equality with the single-filter path.  The weighting tiles are the
// single-filter kernel's blocks (256 particles, two per thread) and the
// softmax partials and their combine are the same device routines, so the
// log-likelihoods, the normaliser, the f32 weights, the fixed-point scan, the
// ancestors, the injection and hence the particle states of filter f equal
// those of the same filter run alone through pfc_cycle.  Only the FP64
// estimate/covariance sums are partitioned differently (gather tiles for a
// filter that resampled, estimate tiles autotuned per size bucket for one
// that did not), which changes them in the last bits.
#include <math.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "markley.h"
#include "pf_device.cuh"

namespace pfb {
namespace batch {

using namespace pfb::dev;

constexpr int kThreads = kBlk;
constexpr int kWTile = 2 * kWThreads;  // particles per weighting tile (= the single filter's block)
constexpr int kScanItems = 16;
constexpr int kRTile = kBlk * kScanItems;  // particles per resampling tile
constexpr int kGTile = 2048;  // outputs per gather tile
constexpr int kBuckets = 4;
// Size buckets for the autotuned estimate tile: n < 8k, < 32k, < 128k, more.
constexpr int kBucketLimit[kBuckets - 1] = {8192, 32768, 131072};
constexpr int kEstTileChoices[] = {2048, 4096, 8192, 16384, 32768};

struct BFilter {
    long long off;
    int n;
    int lm_off, lm_count;
    int wtile0, nwtiles;
    int etile0, netiles;
    int rtile0, nrtiles;
    int gtile0, ngtiles;
    int inj_k, inj_off;
    uint64_t seed;
    float sigma_r, sigma_b, gate, inject_ratio;
    double ess_ratio;
};

struct BTile {
    int f;
    int start;  // filter-local first particle
    int count;
    int local;  // tile index within the filter
};

struct BCtl {
    float M, S;
    int wmode, wvalid;
    double est[kEstN], qmean[4], covs[kCovN];
    double ess, ess_pre;
    float cmp[3], cmq[4];
    int resample_now, resampled, resample_valid, w_bad;
    unsigned long long w_total_fx;
    unsigned long long lcg, lcg_next;
    unsigned long long gen;
    int live;
    unsigned done_w, done_e, done_c;
    unsigned err;
};

struct BGlobal {
    unsigned scan_epoch;
    unsigned inj_epoch;
    unsigned tile_counter;
    unsigned err;
    // look-back polls before a wait gives up (kSpinLimit unless the host
    // lowers it), and the filter whose first resampling tile publishes its
    // prefix under a stale epoch (-1: none), so that the waits of its later
    // tiles run out: both set only by pfc_batch_set_wait_test
    int spin_limit;
    int stall_f;
};

struct Arena {
    float* p[2][7];
    float* ll;
    float* w;
    int* marker;  // run starts of a resample (-1 elsewhere; reset by the gather)
};

// Planes of one filter in set `which`, selected with register selects (an
// indexed kernel-parameter array would be copied to local memory).
__device__ __forceinline__ Planes filter_planes(const Arena& A, int which,
                                                long long off) {
    Planes s;
    s.px = (which ? A.p[1][0] : A.p[0][0]) + off;
    s.py = (which ? A.p[1][1] : A.p[0][1]) + off;
    s.pz = (which ? A.p[1][2] : A.p[0][2]) + off;
    s.qw = (which ? A.p[1][3] : A.p[0][3]) + off;
    s.qx = (which ? A.p[1][4] : A.p[0][4]) + off;
    s.qy = (which ? A.p[1][5] : A.p[0][5]) + off;
    s.qz = (which ? A.p[1][6] : A.p[0][6]) + off;
    return s;
}

// ------------------------------------------------------------------ kernels

__global__ void k_b_init(BCtl* C, BGlobal* G, int nf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f == 0) {
        G->scan_epoch = 1u;
        G->inj_epoch = 1u;
        G->tile_counter = 0u;
        G->err = 0u;
        G->spin_limit = kSpinLimit;
        G->stall_f = -1;
    }
    if (f >= nf) return;
    BCtl c;
    memset(&c, 0, sizeof(c));
    c.lcg = 0x243F6A8885A308D3ull;  // the single-filter handle's initial word
    c.wmode = WMODE_UNIFORM;
    C[f] = c;
}

// Generation counter of every filter: the single-filter path increments it
// at each reinit and predict.
__global__ void k_b_gen_inc(BCtl* C, int nf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) C[f].gen += 1ull;
}

// Prior: pose7 + pos_std3 + rot_std3 per filter (13 floats).
__global__ void __launch_bounds__(kThreads)
    k_b_reinit(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
               BCtl* C, const float* __restrict__ prior) {
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    const float* pr = prior + 13 * t.f;
    const Planes s = filter_planes(A, C[t.f].live, fl.off);
    const unsigned long long gen = C[t.f].gen;
    for (int r = threadIdx.x; r < t.count; r += kThreads) {
        const int i = t.start + r;
        float nz[6];
        pf_normals6(fl.seed, gen, (uint32_t)i, nz);
        const float3 p = make_float3(pr[0] + pr[7] * nz[0], pr[1] + pr[8] * nz[1],
                                     pr[2] + pr[9] * nz[2]);
        const float3 axis =
            make_float3(pr[10] * nz[3], pr[11] * nz[4], pr[12] * nz[5]);
        const float ang = norm3(axis);
        const Quat q0{pr[3], pr[4], pr[5], pr[6]};
        store_pose(s, i, p, q_product(q0, q_from_axis_angle(axis, ang)));
    }
    if (threadIdx.x == 0 && t.local == 0) {
        C[t.f].wmode = WMODE_UNIFORM;
        C[t.f].resampled = 0;  // a new cloud: the estimate pass covers it
    }
}

// Predict (generation gen + 1) and gated weighting of one 256-particle tile
// (kWThreads threads, two particles each, as the single filter's weighting
// blocks); the last tile of a filter combines the softmax partials.  Six
// blocks per SM: with few observations per filter the predict is a larger
// share, and six measured 1.093 ms per 512-filter cycle against 1.134 ms at
// five (the single filter's residency at 256 observations).
__global__ void __launch_bounds__(kWThreads, 6)
    k_b_weight(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
               BCtl* C, const PfcBatchCycle* __restrict__ cyc,
               const CObservation* __restrict__ obs, const float* __restrict__ lm,
               float2* __restrict__ wpart, int use_packed) {
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    BCtl* c = C + t.f;
    const PfcBatchCycle in = cyc[t.f];
    const Planes s = filter_planes(A, c->live, fl.off);
    PredictArgs pa;
    pa.enabled = 1;
    pa.gen = c->gen;
    for (int k = 0; k < 3; ++k) {
        pa.t[k] = in.odom.t[k];
        pa.tstd[k] = in.odom.tstd[k];
        pa.rstd[k] = in.odom.rstd[k];
    }
    for (int k = 0; k < 4; ++k) pa.q[k] = in.odom.q[k];
    const int i0 = t.start + threadIdx.x, i1 = i0 + kWThreads;
    const bool v0 = threadIdx.x < t.count, v1 = threadIdx.x + kWThreads < t.count;
    float3 p0 = make_float3(0.f, 0.f, 0.f), p1 = p0;
    Quat q0 = {1.f, 0.f, 0.f, 0.f}, q1 = q0;
    if (v0) {
        load_pose(s, i0, p0, q0);
        apply_predict(pa, fl.seed, i0, p0, q0);
        store_pose(s, i0, p0, q0);
    }
    if (v1) {
        load_pose(s, i1, p1, q1);
        apply_predict(pa, fl.seed, i1, p1, q1);
        store_pose(s, i1, p1, q1);
    }
    const int nobs = in.nobs;
    if (nobs <= 0) {
        // predict only: the single-filter cycle resets the weights to uniform
        if (threadIdx.x == 0 && t.local == 0) c->wmode = WMODE_UNIFORM;
        return;
    }
    float acc0, acc1;
    weight_two(obs + in.obs_off, nobs, lm + 3 * (size_t)fl.lm_off, fl.lm_count,
               fl.sigma_r, fl.sigma_b, fl.gate, p0, q0, p1, q1, use_packed, acc0,
               acc1);
    float* ll = A.ll + fl.off;
    if (v0) ll[i0] = acc0;
    if (v1) ll[i1] = acc1;
    const float2 pb = block_softmax_partial(acc0, v0, acc1, v1);
    __shared__ bool s_last;
    if (threadIdx.x == 0) {
        wpart[fl.wtile0 + t.local] = pb;
        __threadfence();
        s_last = (atomicAdd(&c->done_w, 1u) == (unsigned)fl.nwtiles - 1u);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const float2 ms = softmax_combine(wpart + fl.wtile0, fl.nwtiles);
    if (threadIdx.x == 0) {
        c->M = ms.x;
        c->S = ms.y;
        const int ok = (ms.y > 0.0f && isfinite(ms.y)) ? 1 : 0;
        c->wvalid = ok;
        c->wmode = ok ? WMODE_LL : WMODE_UNIFORM;
        c->done_w = 0u;
    }
}

// Block partial of NV FP64 sums (fixed order) into part[NV]; returns true in
// every thread of the filter's last tile after its partials are visible.
// Block partial of NV per-thread FP64 accumulators (xor butterfly per warp,
// warps in order) into part[0..NV).
template <int NV>
__device__ __forceinline__ void block_partial(double (&acc)[NV], double* part) {
    __shared__ double s_w[NV][kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        const double v = warp_sum_d(acc[k]);
        if (lane == 0) s_w[k][warp] = v;
    }
    __syncthreads();
    if (tid < NV) {
        double v = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) v += s_w[tid][k];
        part[tid] = v;
    }
}

// block_partial, then true in every thread of the filter's last tile to
// finish (an atomic counter per filter).
template <int NV>
__device__ __forceinline__ bool tile_partial(double (&acc)[NV], double* part,
                                             unsigned* done, int ntiles) {
    __shared__ bool s_last;
    block_partial<NV>(acc, part);
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(done, 1u) == (unsigned)ntiles - 1u);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    return true;
}

// Sum of the filter's tile partials in tile order (warp k: component k).
template <int NV>
__device__ __forceinline__ void tiles_combine(const double* part, int ntiles,
                                              double* out) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int k = warp; k < NV; k += kThreads / 32) {
        double v = 0.0;
        for (int b = lane; b < ntiles; b += 32) v += __ldcg(&part[(size_t)b * NV + k]);
        v = warp_sum_d(v);
        if (lane == 0) out[k] = v;
    }
    __syncthreads();
}

// Sum w^2 (FP64), the fixed-point weight total and the bad-weight flag over
// the float4 groups [q0, q1) of one tile, the weights materialised when they
// are still log-likelihoods.  A thread takes groups q0 + tid, q0 + tid + 256,
// ... in that order; four groups are loaded before any is used so a thread
// keeps four loads in flight (the weight store cannot alias the next load).
template <int kMode>
__device__ __forceinline__ void ess_span(const float* __restrict__ ll, float* __restrict__ w,
                                         int q0, int q1, int n, float M, float S,
                                         double rS, float wuni, double& sq,
                                         unsigned long long& tfx, int& bad) {
    constexpr int kU = 4;
    const float4* __restrict__ src =
        reinterpret_cast<const float4*>(kMode == WMODE_STORED ? w : ll);
    float4* __restrict__ dst = reinterpret_cast<float4*>(w);
    for (int b = q0 + threadIdx.x; b < q1; b += kU * kThreads) {
        float4 V[kU];
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int i4 = b + u * kThreads;
            if (kMode == WMODE_UNIFORM)
                V[u] = make_float4(wuni, wuni, wuni, wuni);
            else
                V[u] = i4 < q1 ? src[i4] : make_float4(0.f, 0.f, 0.f, 0.f);
        }
#pragma unroll
        for (int u = 0; u < kU; ++u) {
            const int i4 = b + u * kThreads;
            if (i4 >= q1) break;
            float4 W = V[u];
            if (kMode == WMODE_LL) {
                W = make_float4(weight_from_ll(W.x, M, S, rS), weight_from_ll(W.y, M, S, rS),
                                weight_from_ll(W.z, M, S, rS), weight_from_ll(W.w, M, S, rS));
                dst[i4] = W;
            }
#pragma unroll
            for (int k = 0; k < 4; ++k) {
                if (4 * i4 + k >= n) break;
                const float wf = comp(W, k);
                bad |= weight_bad(wf) ? 1 : 0;
                tfx += weight_bad(wf) ? 0ull : weight_fx(wf);
                const double wd = (double)wf;
                sq = __fma_rn(wd, wd, sq);
            }
        }
    }
}

// Weight pass over one estimate tile before the resample decision: the
// weights materialised from the log-likelihoods, sum w^2 in FP64, the exact
// fixed-point weight total and the bad-weight flag; the filter's last tile
// combines them and takes ParticleFilter::update's decision
// ratio > 0 && ess < ratio * N (crates/pf_core/src/particle_filter.rs:115-117).
// Reads 4 B per particle where the estimate pass reads 32 B.
__global__ void __launch_bounds__(kThreads)
    k_b_ess(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
            BCtl* C, double* __restrict__ epart,
            unsigned long long* __restrict__ eupart, double* __restrict__ out) {
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    BCtl* c = C + t.f;
    const int wmode = c->wmode;
    const float M = c->M, S = c->S;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)fl.n;
    float* w = A.w + fl.off;
    const float* ll = A.ll + fl.off;
    double acc[1] = {0.0};
    unsigned long long tfx = 0;
    int bad = 0;
    const int q0 = t.start >> 2, q1 = (t.start + t.count + 3) >> 2;
    if (wmode == WMODE_STORED)
        ess_span<WMODE_STORED>(ll, w, q0, q1, fl.n, M, S, rS, wuni, acc[0], tfx, bad);
    else if (wmode == WMODE_UNIFORM)
        ess_span<WMODE_UNIFORM>(ll, w, q0, q1, fl.n, M, S, rS, wuni, acc[0], tfx, bad);
    else
        ess_span<WMODE_LL>(ll, w, q0, q1, fl.n, M, S, rS, wuni, acc[0], tfx, bad);
    // integer total and bad flag of the tile
    __shared__ unsigned long long s_u[kThreads / 32];
    const unsigned long long u = warp_sum_u64(tfx);
    if ((threadIdx.x & 31) == 0) s_u[threadIdx.x >> 5] = u;
    const int any_bad = __syncthreads_or(bad);
    if (threadIdx.x == 0) {
        unsigned long long tot = 0;
        for (int k = 0; k < kThreads / 32; ++k) tot += s_u[k];
        eupart[2 * (size_t)(fl.etile0 + t.local)] = tot;
        eupart[2 * (size_t)(fl.etile0 + t.local) + 1] = any_bad ? 1ull : 0ull;
    }
    if (!tile_partial<1>(acc, epart + (size_t)(fl.etile0 + t.local) * kEstN,
                         &c->done_e, fl.netiles))
        return;
    // warp 0 combines the tiles: sum w^2 in the lane-strided order, the
    // integer total and the flag (exact, any order)
    if (threadIdx.x >= 32) return;
    const int lane = threadIdx.x;
    double sq = 0.0;
    unsigned long long tot = 0, fb = 0;
    for (int b = lane; b < fl.netiles; b += 32) {
        sq += __ldcg(&epart[(size_t)(fl.etile0 + b) * kEstN]);
        tot += __ldcg(&eupart[2 * (size_t)(fl.etile0 + b)]);
        fb |= __ldcg(&eupart[2 * (size_t)(fl.etile0 + b) + 1]);
    }
    sq = warp_sum_d(sq);
    tot = warp_sum_u64(tot);
    const bool any_fb = __any_sync(0xffffffffu, fb != 0ull);
    if (lane == 0) {
        const double ess = sq > 0.0 ? 1.0 / sq : 0.0;
        c->ess = ess;
        c->ess_pre = ess;
        double* o = out + (size_t)t.f * PFC_EST_LEN;
        o[PFC_EST_ESS_PRE] = ess;
        c->resample_now = (fl.ess_ratio > 0.0 && ess < fl.ess_ratio * (double)fl.n) ? 1 : 0;
        c->resampled = 0;
        o[PFC_EST_RESAMPLED] = 0.0;
        c->w_total_fx = tot;
        c->w_bad = any_fb ? 1 : 0;
        if (wmode == WMODE_LL) c->wmode = WMODE_STORED;
        c->done_e = 0u;
    }
}

// Estimate pass over one estimate tile: 14 FP64 sums (and the weight
// materialisation when the weights are still log-likelihoods); the filter's
// last tile combines, runs the Markley mean and stores the f32 covariance
// means.  Three blocks per SM (80 registers): the pass waits on its loads,
// and the third block's warps hide more of that than the spill of a few
// values costs (1.797 against 1.812 ms per 512-filter cycle at two).
__global__ void __launch_bounds__(kThreads, 3)
    k_b_est(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
            BCtl* C, double* __restrict__ epart) {
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    BCtl* c = C + t.f;
    // a filter that resampled in the last cycle has its sums from k_b_est_src
    if (c->resampled) return;
    const Planes s = filter_planes(A, c->live, fl.off);
    const int wmode = c->wmode;
    const float M = c->M, S = c->S;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)fl.n;
    float* w = A.w + fl.off;
    const float* ll = A.ll + fl.off;
    double acc[kEstN];
#pragma unroll
    for (int k = 0; k < kEstN; ++k) acc[k] = 0.0;
    const int q0 = t.start >> 2, q1 = (t.start + t.count + 3) >> 2;
    const float4* px = reinterpret_cast<const float4*>(s.px);
    const float4* py = reinterpret_cast<const float4*>(s.py);
    const float4* pz = reinterpret_cast<const float4*>(s.pz);
    const float4* qw = reinterpret_cast<const float4*>(s.qw);
    const float4* qx = reinterpret_cast<const float4*>(s.qx);
    const float4* qy = reinterpret_cast<const float4*>(s.qy);
    const float4* qz = reinterpret_cast<const float4*>(s.qz);
    for (int i4 = q0 + threadIdx.x; i4 < q1; i4 += kThreads) {
        const float4 X = px[i4], Y = py[i4], Z = pz[i4];
        const float4 QW = qw[i4], QX = qx[i4], QY = qy[i4], QZ = qz[i4];
        float4 W;
        if (wmode == WMODE_STORED) {
            W = reinterpret_cast<const float4*>(w)[i4];
        } else if (wmode == WMODE_UNIFORM) {
            W = make_float4(wuni, wuni, wuni, wuni);
        } else {
            const float4 L = reinterpret_cast<const float4*>(ll)[i4];
            W = make_float4(weight_from_ll(L.x, M, S, rS), weight_from_ll(L.y, M, S, rS),
                            weight_from_ll(L.z, M, S, rS), weight_from_ll(L.w, M, S, rS));
            reinterpret_cast<float4*>(w)[i4] = W;
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (4 * i4 + k >= fl.n) break;
            const float wf = comp(W, k);
            est_add(acc, wf, comp(X, k), comp(Y, k), comp(Z, k), comp(QW, k),
                    comp(QX, k), comp(QY, k), comp(QZ, k));
        }
    }
    if (!tile_partial<kEstN>(acc, epart + (size_t)(fl.etile0 + t.local) * kEstN,
                             &c->done_e, fl.netiles))
        return;
    __shared__ double s_out[kEstN];
    tiles_combine<kEstN>(epart + (size_t)fl.etile0 * kEstN, fl.netiles, s_out);
    double qm[4];
    if (threadIdx.x < 32) markley_mean_warp_call(&s_out[3], qm);  // warp 0
    if (threadIdx.x == 0) {
        for (int k = 0; k < kEstN; ++k) c->est[k] = s_out[k];
        c->ess = s_out[13] > 0.0 ? 1.0 / s_out[13] : 0.0;
        for (int k = 0; k < 4; ++k) c->qmean[k] = qm[k];
        for (int k = 0; k < 3; ++k) c->cmp[k] = (float)s_out[k];
        for (int k = 0; k < 4; ++k) c->cmq[k] = (float)qm[k];
        if (wmode == WMODE_LL) c->wmode = WMODE_STORED;
        c->done_e = 0u;
    }
}

// Covariance pass and the filter's output record.  Three blocks per SM, as
// the estimate pass (1.788 against 1.799 ms per 512-filter cycle at two).
__global__ void __launch_bounds__(kThreads, 3)
    k_b_covs(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
             BCtl* C, double* __restrict__ cpart, double* __restrict__ out) {
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    BCtl* c = C + t.f;
    const Planes s = filter_planes(A, c->live, fl.off);
    const int wmode = c->wmode;
    const float M = c->M, S = c->S;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)fl.n;
    const float* w = A.w + fl.off;
    const float* ll = A.ll + fl.off;
    const double mp[3] = {(double)c->cmp[0], (double)c->cmp[1], (double)c->cmp[2]};
    const double qm[4] = {(double)c->cmq[0], (double)c->cmq[1], (double)c->cmq[2],
                          (double)c->cmq[3]};
    double acc[kCovN];
#pragma unroll
    for (int k = 0; k < kCovN; ++k) acc[k] = 0.0;
    const int q0 = t.start >> 2, q1 = (t.start + t.count + 3) >> 2;
    const float4* px = reinterpret_cast<const float4*>(s.px);
    const float4* py = reinterpret_cast<const float4*>(s.py);
    const float4* pz = reinterpret_cast<const float4*>(s.pz);
    const float4* qw = reinterpret_cast<const float4*>(s.qw);
    const float4* qx = reinterpret_cast<const float4*>(s.qx);
    const float4* qy = reinterpret_cast<const float4*>(s.qy);
    const float4* qz = reinterpret_cast<const float4*>(s.qz);
    for (int i4 = q0 + threadIdx.x; i4 < q1; i4 += kThreads) {
        const float4 X = px[i4], Y = py[i4], Z = pz[i4];
        const float4 QW = qw[i4], QX = qx[i4], QY = qy[i4], QZ = qz[i4];
        float4 W;
        if (wmode == WMODE_STORED) {
            W = reinterpret_cast<const float4*>(w)[i4];
        } else if (wmode == WMODE_UNIFORM) {
            W = make_float4(wuni, wuni, wuni, wuni);
        } else {
            const float4 L = reinterpret_cast<const float4*>(ll)[i4];
            W = make_float4(weight_from_ll(L.x, M, S, rS), weight_from_ll(L.y, M, S, rS),
                            weight_from_ll(L.z, M, S, rS), weight_from_ll(L.w, M, S, rS));
        }
#pragma unroll
        for (int k = 0; k < 4; ++k) {
            if (4 * i4 + k >= fl.n) break;
            cov_add(acc, (double)comp(W, k), comp(X, k), comp(Y, k), comp(Z, k),
                    comp(QW, k), comp(QX, k), comp(QY, k), comp(QZ, k), mp, qm);
        }
    }
    if (!tile_partial<kCovN>(acc, cpart + (size_t)(fl.etile0 + t.local) * kCovN,
                             &c->done_c, fl.netiles))
        return;
    __shared__ double s_out[kCovN];
    tiles_combine<kCovN>(cpart + (size_t)fl.etile0 * kCovN, fl.netiles, s_out);
    if (threadIdx.x == 0) {
        for (int k = 0; k < kCovN; ++k) c->covs[k] = s_out[k];
        double* o = out + (size_t)t.f * PFC_EST_LEN;
        for (int k = 0; k < 3; ++k) o[PFC_EST_POS + k] = c->est[k];
        for (int k = 0; k < 4; ++k) o[PFC_EST_QUAT + k] = c->qmean[k];
        for (int k = 0; k < 6; ++k) o[PFC_EST_POSCOV + k] = s_out[k];
        for (int k = 0; k < 6; ++k) o[PFC_EST_ATTCOV + k] = s_out[6 + k];
        // without a resample the record carries the ESS the decision used,
        // as ParticleFilter::update returns its first estimate
        o[PFC_EST_ESS] = c->resampled ? c->ess : c->ess_pre;
        o[PFC_EST_RESAMPLED] = c->resampled ? 1.0 : 0.0;
        c->done_c = 0u;
    }
}

// Resampling of one 4096-particle tile of a filter that resamples: the
// single-filter specification, with tiles taken in a global dynamic order (a
// filter's tiles are consecutive in that order, so each tile's predecessors
// are already running when it looks back).  Source j writes j at the first
// output of its run and at every gather-tile boundary inside it (runs are
// disjoint, so no two sources write the same marker); k_b_gather copies.
__global__ void __launch_bounds__(kThreads)
    k_b_resample(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
                 BCtl* C, BGlobal* G, unsigned* flags, uint64_t* vals) {
    __shared__ unsigned s_tile;
    __shared__ uint64_t s_warp[kThreads / 32];
    __shared__ uint64_t s_prefix, s_agg;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&G->tile_counter, 1u);
    __syncthreads();
    const BTile t = T[s_tile];
    const BFilter& fl = F[t.f];
    BCtl* c = C + t.f;
    if (!c->resample_now) return;
    const int n = fl.n;
    const uint64_t Tfx = c->w_total_fx;
    if (Tfx == 0 || c->w_bad) {
        if (t.local == 0 && tid == 0) c->resample_valid = 0;
        return;
    }
    const unsigned epoch = G->scan_epoch;
    const unsigned long long lcg1 =
        c->lcg * 6364136223846793005ull + 1442695040888963407ull;
    const double u01 = (double)(lcg1 >> 11) * (1.0 / 9007199254740992.0);
    const double total = (double)Tfx * 0x1p-62;
    const double step = total / (double)n;
    const double u0 = u01 * step;
    if (tid == 0 && t.local == 0) {
        c->lcg_next = lcg1;
        c->resample_valid = 1;
    }
    const int wmode = c->wmode;
    const float M = c->M, S = c->S;
    int* mk = A.marker + fl.off;
    const float* w = A.w + fl.off;
    const float* ll = A.ll + fl.off;
    unsigned* fflags = flags + fl.rtile0;
    uint64_t* fvals = vals + 2 * (size_t)fl.rtile0;
    const int tile = t.local;

    const long long j0 = (long long)tile * kRTile + tid * kScanItems;
    uint64_t v[kScanItems];
    uint64_t run = 0;
    if (wmode == WMODE_STORED && j0 + kScanItems <= n) {
        const float4* w4 = reinterpret_cast<const float4*>(w + j0);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const float4 a = w4[q];
            run += weight_fx(a.x);
            v[4 * q] = run;
            run += weight_fx(a.y);
            v[4 * q + 1] = run;
            run += weight_fx(a.z);
            v[4 * q + 2] = run;
            run += weight_fx(a.w);
            v[4 * q + 3] = run;
        }
    } else {
#pragma unroll
        for (int k = 0; k < kScanItems; ++k) {
            const long long j = j0 + k;
            if (j < n) run += weight_fx(weight_of(wmode, j, n, w, ll, M, S));
            v[k] = run;
        }
    }
    uint64_t x = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = shfl_up_u64(x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (tid == 0) {
        uint64_t acc = 0;
        for (int k = 0; k < kThreads / 32; ++k) {
            const uint64_t tt = s_warp[k];
            s_warp[k] = acc;
            acc += tt;
        }
        s_agg = acc;
        if (tile == 0) {
            fvals[1] = acc;
            __threadfence();
            // a stale epoch (host-planted wait test) is a flag no waiter accepts
            const unsigned pub = t.f == G->stall_f ? (epoch ^ 0x20000000u) : epoch;
            st_release(&fflags[0], (pub << 2) | TILE_INCL);
            s_prefix = 0;
        } else {
            fvals[2 * (size_t)tile] = acc;
            __threadfence();
            st_release(&fflags[tile], (epoch << 2) | TILE_AGG);
        }
    }
    __syncthreads();
    if (tile > 0 && warp == 0) {
        const uint64_t prefix =
            look_back(fflags, fvals, tile, epoch, &c->err, G->spin_limit);
        if (lane == 0) {
            fvals[2 * (size_t)tile + 1] = prefix + s_agg;
            __threadfence();
            st_release(&fflags[tile], (epoch << 2) | TILE_INCL);
            s_prefix = prefix;
        }
    }
    __syncthreads();
    const uint64_t c_prev = s_prefix + s_warp[warp] + (x - run);
    long long st = (j0 == 0) ? 0 : count_le(c_prev, n, u0, step);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long j = j0 + k;
        if (j >= n) break;
        const long long e =
            (j == n - 1) ? (long long)n : count_le(c_prev + v[k], n, u0, step);
        if (e > st) {
            mk[st] = (int)j;
            for (long long b = (st / kGTile + 1) * kGTile; b < e; b += kGTile) mk[b] = (int)j;
        }
        st = e;
    }
}

// Output-parallel copy of one 2048-output tile of a filter that resampled:
// the tile's markers (every tile starts with one) give each output its
// ancestor by a running maximum (ancestors increase with the output index),
// the markers read are reset for the next resample, and the seven planes are
// copied with 16-byte stores (filter offsets are multiples of 1024).  The
// copied values, already in registers, go into the 14 estimate sums of the
// new cloud: every output has the weight wd = 1/n, so a thread sums x, y, z
// and the exact FP64 products of the quaternion components, counts its
// outputs and scales by wd (wd^2 for the sum of squared weights) once; one
// partial per tile in gpart, so the cycle needs no estimate pass over the
// resampled filters.
__global__ void __launch_bounds__(kThreads)
    k_b_gather(Arena A, const BFilter* __restrict__ F, const BTile* __restrict__ T,
               const BCtl* C, double* __restrict__ gpart) {
    __shared__ int s_anc[kGTile];
    __shared__ int s_wmax[kThreads / 32];
    const BTile t = T[blockIdx.x];
    const BFilter& fl = F[t.f];
    const BCtl* c = C + t.f;
    if (!c->resample_now || !c->resample_valid) return;
    const int n = fl.n;
    int* mk = A.marker + fl.off;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int i0 = t.start + 8 * tid;
    int m[8];
#pragma unroll
    for (int h = 0; h < 2; ++h) {
        const int ib = i0 + 4 * h;
        int4 v = make_int4(-1, -1, -1, -1);
        if (ib + 4 <= n) {
            v = __ldcg(reinterpret_cast<const int4*>(mk + ib));
        } else {
            if (ib < n) v.x = __ldcg(mk + ib);
            if (ib + 1 < n) v.y = __ldcg(mk + ib + 1);
            if (ib + 2 < n) v.z = __ldcg(mk + ib + 2);
        }
        m[4 * h] = v.x;
        m[4 * h + 1] = v.y;
        m[4 * h + 2] = v.z;
        m[4 * h + 3] = v.w;
    }
#pragma unroll
    for (int q = 0; q < 8; ++q)
        if (m[q] >= 0) mk[i0 + q] = -1;
#pragma unroll
    for (int q = 1; q < 8; ++q) m[q] = max(m[q], m[q - 1]);
    int x = m[7];
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const int y = __shfl_up_sync(~0u, x, d);
        if (lane >= d) x = max(x, y);
    }
    const int excl = __shfl_up_sync(~0u, x, 1);
    if (lane == 31) s_wmax[warp] = x;
    __syncthreads();
    int before = lane > 0 ? excl : -1;
    for (int k = 0; k < warp; ++k) before = max(before, s_wmax[k]);
#pragma unroll
    for (int q = 0; q < 8; ++q) s_anc[8 * tid + q] = min(max(max(m[q], before), 0), n - 1);
    __syncthreads();
    const Planes src = filter_planes(A, c->live, fl.off);
    const Planes dst = filter_planes(A, 1 - c->live, fl.off);
    float* const sp[7] = {src.px, src.py, src.pz, src.qw, src.qx, src.qy, src.qz};
    float* const dp[7] = {dst.px, dst.py, dst.pz, dst.qw, dst.qx, dst.qy, dst.qz};
    const float wuni = 1.0f / (float)n;
    double acc[kEstN];
#pragma unroll
    for (int q = 0; q < kEstN; ++q) acc[q] = 0.0;
    // thread t copies outputs [4t, 4t + 4) and [1024 + 4t, 1024 + 4t + 4)
#pragma unroll 1
    for (int h = 0; h < 2; ++h) {
        const int l0 = h * (kGTile / 2) + 4 * tid;
        const int ib = t.start + l0;
        if (ib >= n) break;
        int a[4];
#pragma unroll
        for (int q = 0; q < 4; ++q) a[q] = s_anc[l0 + q];
        float v[7][4];
#pragma unroll
        for (int k = 0; k < 7; ++k)
#pragma unroll
            for (int q = 0; q < 4; ++q) v[k][q] = sp[k][a[q]];
        if (ib + 4 <= n) {
#pragma unroll
            for (int k = 0; k < 7; ++k)
                reinterpret_cast<float4*>(dp[k] + ib)[0] =
                    make_float4(v[k][0], v[k][1], v[k][2], v[k][3]);
        } else {
#pragma unroll
            for (int k = 0; k < 7; ++k)
#pragma unroll
                for (int q = 0; q < 4; ++q)
                    if (ib + q < n) dp[k][ib + q] = v[k][q];
        }
#pragma unroll
        for (int q = 0; q < 4; ++q)
            if (ib + q < n) {
                acc[0] += (double)v[0][q];
                acc[1] += (double)v[1][q];
                acc[2] += (double)v[2][q];
                const double qd[4] = {v[3][q], v[4][q], v[5][q], v[6][q]};
                int e = 3;
#pragma unroll
                for (int r = 0; r < 4; ++r)
#pragma unroll
                    for (int cc = r; cc < 4; ++cc) {
                        acc[e] = fma(qd[r], qd[cc], acc[e]);
                        ++e;
                    }
                acc[13] += 1.0;
            }
    }
    const double wd = (double)wuni;
#pragma unroll
    for (int q = 0; q < 13; ++q) acc[q] *= wd;
    acc[13] *= wd * wd;
    block_partial<kEstN>(acc, gpart + (size_t)(fl.gtile0 + t.local) * kEstN);
}

// Injection: global draw d belongs to filter draw_f[d] (local draw
// j = d - inj_off).  Lists per arena particle, tags (epoch << 32 | d).
__global__ void k_b_inject_link(const BFilter* __restrict__ F, const BCtl* C,
                                const BGlobal* G, const int* __restrict__ draw_f,
                                int total, uint64_t* head, int* next) {
    const int d = blockIdx.x * kThreads + threadIdx.x;
    if (d >= total) return;
    const int f = draw_f[d];
    const BCtl& c = C[f];
    if (!c.resample_now || !c.resample_valid) return;
    const BFilter& fl = F[f];
    const InjDraw dr = inj_draw(c.lcg_next, c.gen, d - fl.inj_off, fl.n);
    const unsigned epoch = G->inj_epoch;
    const uint64_t tag = ((uint64_t)epoch << 32) | (uint32_t)d;
    const uint64_t prev = atomicExch((unsigned long long*)&head[fl.off + dr.idx],
                                     (unsigned long long)tag);
    next[d] = ((uint32_t)(prev >> 32) == epoch) ? (int)(uint32_t)prev : -1;
}

// The thread of a particle's first draw applies its draws in ascending draw
// order and records each draw's exact position change (a difference of two
// f32 values) in icorr[3d..3d+2] for the filter's estimate sums.
__global__ void k_b_inject_apply(Arena A, const BFilter* __restrict__ F,
                                 const BCtl* C, const BGlobal* G,
                                 const int* __restrict__ draw_f, int total,
                                 const uint64_t* head, const int* next,
                                 double* __restrict__ icorr) {
    const int d = blockIdx.x * kThreads + threadIdx.x;
    if (d >= total) return;
    const int f = draw_f[d];
    const BCtl& c = C[f];
    if (!c.resample_now || !c.resample_valid) return;
    const BFilter& fl = F[f];
    const uint64_t lcg = c.lcg_next;
    const InjDraw dr = inj_draw(lcg, c.gen, d - fl.inj_off, fl.n);
    const unsigned epoch = G->inj_epoch;
    const uint64_t h = head[fl.off + dr.idx];
    if ((uint32_t)(h >> 32) != epoch || (int)(uint32_t)h != d) return;
    const Planes dst = filter_planes(A, 1 - c.live, fl.off);
    float px = dst.px[dr.idx], py = dst.py[dr.idx], pz = dst.pz[dr.idx];
    int last = -1;
    for (;;) {
        int best = -1;
        for (int x = d; x >= 0; x = next[x])
            if (x > last && (best < 0 || x < best)) best = x;
        if (best < 0) break;
        const InjDraw e =
            (best == d) ? dr : inj_draw(lcg, c.gen, best - fl.inj_off, fl.n);
        const float nx = px + e.jx, ny = py + e.jy, nz = pz + e.jz;
        icorr[3 * (size_t)best] = (double)nx - (double)px;
        icorr[3 * (size_t)best + 1] = (double)ny - (double)py;
        icorr[3 * (size_t)best + 2] = (double)nz - (double)pz;
        px = nx;
        py = ny;
        pz = nz;
        last = best;
    }
    dst.px[dr.idx] = px;
    dst.py[dr.idx] = py;
    dst.pz[dr.idx] = pz;
}

__global__ void k_b_commit(BCtl* C, BGlobal* G, int nf) {
    const int f = blockIdx.x * blockDim.x + threadIdx.x;
    if (f < nf) {
        BCtl& c = C[f];
        if (c.resample_now) {
            if (c.resample_valid) {
                c.live = 1 - c.live;
                c.resampled = 1;
                c.lcg = c.lcg_next;
            }
            c.wmode = WMODE_UNIFORM;
        }
        if (c.err) atomicOr(&G->err, c.err);
    }
    if (f == 0) {
        G->tile_counter = 0u;
        unsigned e = (G->scan_epoch + 1u) & 0x3FFFFFFFu;
        G->scan_epoch = e ? e : 1u;
        e = G->inj_epoch + 1u;
        G->inj_epoch = e ? e : 1u;
    }
}

// Estimate sums of a filter that resampled this cycle, without a pass over
// the new cloud: its gather tiles' sums in tile order, plus wd times the
// injection's position changes in draw order; then the Markley mean and the
// f32 means of the covariance pass, as the estimate pass's last tile leaves
// them.  One block per filter; the others take the estimate pass.
__global__ void __launch_bounds__(kThreads)
    k_b_est_src(const BFilter* __restrict__ F, BCtl* C, const double* __restrict__ gpart,
                const double* __restrict__ icorr) {
    const BFilter& fl = F[blockIdx.x];
    BCtl* c = C + blockIdx.x;
    if (!c->resampled) return;
    __shared__ double s_out[kEstN];
    tiles_combine<kEstN>(gpart + (size_t)fl.gtile0 * kEstN, fl.ngtiles, s_out);
    double qm[4];
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double d[3] = {0.0, 0.0, 0.0};
        for (int j = lane; j < fl.inj_k; j += 32)
#pragma unroll
            for (int q = 0; q < 3; ++q) d[q] += icorr[3 * (size_t)(fl.inj_off + j) + q];
        const double wd = (double)(1.0f / (float)fl.n);
#pragma unroll
        for (int q = 0; q < 3; ++q) d[q] = warp_sum_d(d[q]);
        if (lane == 0)
            for (int q = 0; q < 3; ++q) s_out[q] += wd * d[q];
        __syncwarp();
        markley_mean_warp_call(&s_out[3], qm);
    }
    if (threadIdx.x == 0) {
        for (int k = 0; k < kEstN; ++k) c->est[k] = s_out[k];
        c->ess = s_out[13] > 0.0 ? 1.0 / s_out[13] : 0.0;
        for (int k = 0; k < 4; ++k) c->qmean[k] = qm[k];
        for (int k = 0; k < 3; ++k) c->cmp[k] = (float)s_out[k];
        for (int k = 0; k < 4; ++k) c->cmq[k] = (float)qm[k];
    }
}

// Weights of one filter as f32 (materialised from the current mode).
__global__ void k_b_weights(Arena A, const BFilter* F, const BCtl* C, int f,
                            float* out) {
    const BFilter& fl = F[f];
    const BCtl& c = C[f];
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < fl.n;
         i += gridDim.x * kThreads)
        out[i] = weight_of(c.wmode, i, fl.n, A.w + fl.off, A.ll + fl.off, c.M, c.S);
}

__global__ void k_b_pack(Arena A, const BFilter* F, const BCtl* C, int f,
                         float* pos3, float* quat4) {
    const BFilter& fl = F[f];
    const Planes s = filter_planes(A, C[f].live, fl.off);
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < fl.n;
         i += gridDim.x * kThreads) {
        pos3[3 * i] = s.px[i];
        pos3[3 * i + 1] = s.py[i];
        pos3[3 * i + 2] = s.pz[i];
        quat4[4 * i] = s.qw[i];
        quat4[4 * i + 1] = s.qx[i];
        quat4[4 * i + 2] = s.qy[i];
        quat4[4 * i + 3] = s.qz[i];
    }
}

// ------------------------------------------------------------------ handle

struct BatchHandle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    int nf = 0;
    std::vector<BFilter> filters;
    std::vector<int> est_tile;  // per bucket
    int use_packed = 1;
    long long arena = 0;         // particles incl. padding
    float* d_planes = nullptr;   // 2 x 7 planes + ll + w
    Arena A{};
    BFilter* d_F = nullptr;
    BTile* d_wt = nullptr;
    int n_wt = 0;
    BTile* d_et = nullptr;
    int n_et = 0;
    BTile* d_rt = nullptr;
    int n_rt = 0;
    BCtl* d_C = nullptr;
    BGlobal* d_G = nullptr;
    BGlobal* h_G = nullptr;
    float2* d_wpart = nullptr;
    double* d_epart = nullptr;
    unsigned long long* d_eupart = nullptr;
    double* d_cpart = nullptr;
    unsigned* d_flags = nullptr;
    uint64_t* d_vals = nullptr;
    double* d_gpart = nullptr;   // estimate sums of the new cloud per gather tile
    BTile* d_gt = nullptr;
    int n_gt = 0;
    int* d_marker = nullptr;
    int* d_draw_f = nullptr;
    int total_draws = 0;
    uint64_t* d_inj_head = nullptr;
    int* d_inj_next = nullptr;
    double* d_icorr = nullptr;   // position change of every injection draw
    float* d_lm = nullptr;
    int lm_total = 0;
    PfcBatchCycle* d_cyc = nullptr;
    PfcBatchCycle* h_cyc = nullptr;  // pinned
    CObservation* d_obs = nullptr;
    CObservation* h_obs = nullptr;   // pinned
    int obs_cap = 0;
    double* d_out = nullptr;
    double* h_out = nullptr;         // pinned
    float* d_prior = nullptr;
    float* d_tmp = nullptr;
    long long tmp_cap = 0;
    bool use_graph = true;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    long long launches = 0;        // kernels launched (a graph counts its kernels)
    int kernels_per_cycle = 0;
};

BatchHandle* as_b(void* p) { return static_cast<BatchHandle*>(p); }

int bucket_of(int n) {
    for (int b = 0; b < kBuckets - 1; ++b)
        if (n < kBucketLimit[b]) return b;
    return kBuckets - 1;
}

std::vector<BTile> make_tiles(const std::vector<BFilter>& F, int which,
                              const std::vector<int>& est_tile) {
    std::vector<BTile> t;
    for (int f = 0; f < (int)F.size(); ++f) {
        const int sz = which == 0   ? kWTile
                       : which == 1 ? est_tile[bucket_of(F[f].n)]
                       : which == 2 ? kRTile
                                    : kGTile;
        const int nt = ceil_div(F[f].n, sz);
        for (int k = 0; k < nt; ++k)
            t.push_back(BTile{f, k * sz, std::min(sz, F[f].n - k * sz), k});
    }
    return t;
}

void drop_graph(BatchHandle* h) {
    if (h->exec) cudaGraphExecDestroy(h->exec);
    if (h->graph) cudaGraphDestroy(h->graph);
    h->exec = nullptr;
    h->graph = nullptr;
}

// (Re)build the estimate tile table after a tile-size change.
int rebuild_est_tiles(BatchHandle* h) {
    std::vector<BTile> et = make_tiles(h->filters, 1, h->est_tile);
    int e0 = 0;
    for (int f = 0; f < h->nf; ++f) {
        h->filters[f].etile0 = e0;
        h->filters[f].netiles = ceil_div(h->filters[f].n,
                                         h->est_tile[bucket_of(h->filters[f].n)]);
        e0 += h->filters[f].netiles;
    }
    if ((int)et.size() > h->n_et) {
        cudaFree(h->d_et);
        cudaFree(h->d_epart);
        cudaFree(h->d_eupart);
        cudaFree(h->d_cpart);
        h->d_et = nullptr;
        h->d_epart = nullptr;
        h->d_eupart = nullptr;
        h->d_cpart = nullptr;
        const size_t ne = et.size();
        PFB_CK(cudaMalloc((void**)&h->d_et, sizeof(BTile) * ne));
        PFB_CK(cudaMalloc((void**)&h->d_epart, sizeof(double) * kEstN * ne));
        PFB_CK(cudaMalloc((void**)&h->d_eupart, sizeof(unsigned long long) * 2 * ne));
        PFB_CK(cudaMalloc((void**)&h->d_cpart, sizeof(double) * kCovN * ne));
    }
    h->n_et = (int)et.size();
    PFB_CK(cudaMemcpyAsync(h->d_et, et.data(), sizeof(BTile) * et.size(),
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaMemcpyAsync(h->d_F, h->filters.data(), sizeof(BFilter) * h->nf,
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    return 0;
}

int launch_est_covs(BatchHandle* h) {
    k_b_est<<<h->n_et, kThreads, 0, h->stream>>>(h->A, h->d_F, h->d_et, h->d_C,
                                                 h->d_epart);
    k_b_covs<<<h->n_et, kThreads, 0, h->stream>>>(h->A, h->d_F, h->d_et, h->d_C,
                                                  h->d_cpart, h->d_out);
    h->launches += 2;
    PFB_KL();
    return 0;
}

// The kernel chain of one cycle on h->stream (inputs in d_cyc / d_obs).
int enqueue_cycle(BatchHandle* h) {
    cudaStream_t s = h->stream;
    k_b_gen_inc<<<ceil_div(h->nf, kThreads), kThreads, 0, s>>>(h->d_C, h->nf);
    k_b_weight<<<h->n_wt, kWThreads, 0, s>>>(h->A, h->d_F, h->d_wt, h->d_C, h->d_cyc,
                                            h->d_obs, h->d_lm, h->d_wpart,
                                            h->use_packed);
    k_b_ess<<<h->n_et, kThreads, 0, s>>>(h->A, h->d_F, h->d_et, h->d_C, h->d_epart,
                                         h->d_eupart, h->d_out);
    h->launches += 3;
    PFB_KL();
    k_b_resample<<<h->n_rt, kThreads, 0, s>>>(h->A, h->d_F, h->d_rt, h->d_C, h->d_G,
                                              h->d_flags, h->d_vals);
    k_b_gather<<<h->n_gt, kThreads, 0, s>>>(h->A, h->d_F, h->d_gt, h->d_C, h->d_gpart);
    h->launches += 2;
    if (h->total_draws > 0) {
        const int g = ceil_div(h->total_draws, kThreads);
        k_b_inject_link<<<g, kThreads, 0, s>>>(h->d_F, h->d_C, h->d_G, h->d_draw_f,
                                               h->total_draws, h->d_inj_head,
                                               h->d_inj_next);
        k_b_inject_apply<<<g, kThreads, 0, s>>>(h->A, h->d_F, h->d_C, h->d_G,
                                                h->d_draw_f, h->total_draws,
                                                h->d_inj_head, h->d_inj_next, h->d_icorr);
        h->launches += 2;
    }
    k_b_commit<<<ceil_div(h->nf, kThreads), kThreads, 0, s>>>(h->d_C, h->d_G, h->nf);
    k_b_est_src<<<h->nf, kThreads, 0, s>>>(h->d_F, h->d_C, h->d_gpart, h->d_icorr);
    h->launches += 2;
    PFB_KL();
    if (launch_est_covs(h)) return -1;
    PFB_CK(cudaMemcpyAsync(h->h_G, h->d_G, sizeof(BGlobal), cudaMemcpyDeviceToHost, s));
    return 0;
}

int run_cycle(BatchHandle* h) {
    if (!h->use_graph) return enqueue_cycle(h);
    if (!h->exec) {
        PFB_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const long long l0 = h->launches;
        const int rc = enqueue_cycle(h);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        h->kernels_per_cycle = (int)(h->launches - l0);
        h->launches = l0;
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_error("pf_b200: batch cycle capture failed: %s", cudaGetErrorString(e));
            return -1;
        }
        h->graph = g;
        PFB_CK(cudaGraphInstantiate(&h->exec, g, 0));
    }
    PFB_CK(cudaGraphLaunch(h->exec, h->stream));
    h->launches += h->kernels_per_cycle;
    return 0;
}

int finish(BatchHandle* h, double* est_out) {
    if (est_out)
        PFB_CK(cudaMemcpyAsync(h->h_out, h->d_out,
                               sizeof(double) * PFC_EST_LEN * (size_t)h->nf,
                               cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    if (h->h_G->err & ERR_SPIN_TIMEOUT) {
        set_error("pf_b200: batch look-back wait timed out");
        return -1;
    }
    if (est_out)
        memcpy(est_out, h->h_out, sizeof(double) * PFC_EST_LEN * (size_t)h->nf);
    return 0;
}

void free_batch(BatchHandle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_graph(h);
    cudaFree(h->d_planes);
    cudaFree(h->d_F);
    cudaFree(h->d_wt);
    cudaFree(h->d_et);
    cudaFree(h->d_rt);
    cudaFree(h->d_C);
    cudaFree(h->d_G);
    cudaFreeHost(h->h_G);
    cudaFree(h->d_wpart);
    cudaFree(h->d_epart);
    cudaFree(h->d_eupart);
    cudaFree(h->d_cpart);
    cudaFree(h->d_flags);
    cudaFree(h->d_vals);
    cudaFree(h->d_gpart);
    cudaFree(h->d_gt);
    cudaFree(h->d_marker);
    cudaFree(h->d_draw_f);
    cudaFree(h->d_inj_head);
    cudaFree(h->d_inj_next);
    cudaFree(h->d_icorr);
    cudaFree(h->d_lm);
    cudaFree(h->d_cyc);
    cudaFreeHost(h->h_cyc);
    cudaFree(h->d_obs);
    cudaFreeHost(h->h_obs);
    cudaFree(h->d_out);
    cudaFreeHost(h->h_out);
    cudaFree(h->d_prior);
    cudaFree(h->d_tmp);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
}

int ensure_tmp(BatchHandle* h, long long floats) {
    if (floats <= h->tmp_cap) return 0;
    cudaFree(h->d_tmp);
    h->d_tmp = nullptr;
    PFB_CK(cudaMalloc((void**)&h->d_tmp, sizeof(float) * (size_t)floats));
    h->tmp_cap = floats;
    return 0;
}

}  // namespace batch
}  // namespace pfb

using namespace pfb;
using namespace pfb::batch;

extern "C" {

void* pfc_batch_create(int n_filters, const int* n, const unsigned* seeds,
                       int obs_cap) {
    clear_error();
    if (n_filters <= 0 || !n || obs_cap < 0) {
        set_error("pf_b200: pfc_batch_create: bad arguments");
        return nullptr;
    }
    for (int f = 0; f < n_filters; ++f)
        if (n[f] <= 0) {
            set_error("pf_b200: pfc_batch_create: filter %d has n = %d", f, n[f]);
            return nullptr;
        }
    BatchHandle* h = new (std::nothrow) BatchHandle();
    if (!h) return nullptr;
    h->nf = n_filters;
    h->est_tile.assign(kBuckets, 8192);
    h->filters.resize(n_filters);
    long long off = 0;
    int w0 = 0, r0 = 0, g0 = 0;
    for (int f = 0; f < n_filters; ++f) {
        BFilter& b = h->filters[f];
        memset(&b, 0, sizeof(b));
        b.off = off;
        b.n = n[f];
        off += (n[f] + 1023) / 1024 * 1024;
        b.wtile0 = w0;
        b.nwtiles = ceil_div(n[f], kWTile);
        w0 += b.nwtiles;
        b.rtile0 = r0;
        b.nrtiles = ceil_div(n[f], kRTile);
        r0 += b.nrtiles;
        b.gtile0 = g0;
        b.ngtiles = ceil_div(n[f], kGTile);
        g0 += b.ngtiles;
        const unsigned sd = seeds ? seeds[f] : 42u;
        b.seed = sd == 0 ? 42ull : (uint64_t)sd;
        b.sigma_r = 0.05f;
        b.sigma_b = 0.02f;
        b.gate = 3.0f;
        b.ess_ratio = 0.5;
        b.inject_ratio = 0.0f;
    }
    h->arena = off;
    bool ok = false;
    do {
        if (cudaGetDevice(&h->dev) != cudaSuccess) break;
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) != cudaSuccess)
            break;
        const size_t ap = (size_t)h->arena;
        if (cudaMalloc((void**)&h->d_planes, sizeof(float) * ap * 16) != cudaSuccess)
            break;
        if (cudaMemset(h->d_planes, 0, sizeof(float) * ap * 16) != cudaSuccess) break;
        for (int b = 0; b < 2; ++b)
            for (int k = 0; k < 7; ++k) h->A.p[b][k] = h->d_planes + ap * (7 * b + k);
        h->A.ll = h->d_planes + ap * 14;
        h->A.w = h->d_planes + ap * 15;
        std::vector<BTile> wt = make_tiles(h->filters, 0, h->est_tile);
        std::vector<BTile> rt = make_tiles(h->filters, 2, h->est_tile);
        h->n_wt = (int)wt.size();
        h->n_rt = (int)rt.size();
        if (cudaMalloc((void**)&h->d_F, sizeof(BFilter) * n_filters) != cudaSuccess ||
            cudaMalloc((void**)&h->d_wt, sizeof(BTile) * wt.size()) != cudaSuccess ||
            cudaMalloc((void**)&h->d_rt, sizeof(BTile) * rt.size()) != cudaSuccess ||
            cudaMalloc((void**)&h->d_C, sizeof(BCtl) * n_filters) != cudaSuccess ||
            cudaMalloc((void**)&h->d_G, sizeof(BGlobal)) != cudaSuccess ||
            cudaMallocHost((void**)&h->h_G, sizeof(BGlobal)) != cudaSuccess ||
            cudaMalloc((void**)&h->d_wpart, sizeof(float2) * wt.size()) != cudaSuccess ||
            cudaMalloc((void**)&h->d_flags, sizeof(unsigned) * rt.size()) != cudaSuccess ||
            cudaMalloc((void**)&h->d_vals, sizeof(uint64_t) * 2 * rt.size()) != cudaSuccess)
            break;
        if (cudaMemset(h->d_flags, 0, sizeof(unsigned) * rt.size()) != cudaSuccess) break;
        if (cudaMalloc((void**)&h->d_marker, sizeof(int) * ap) != cudaSuccess ||
            cudaMemset(h->d_marker, 0xFF, sizeof(int) * ap) != cudaSuccess)
            break;
        h->A.marker = h->d_marker;
        std::vector<BTile> gt = make_tiles(h->filters, 3, h->est_tile);
        h->n_gt = (int)gt.size();
        if (cudaMalloc((void**)&h->d_gt, sizeof(BTile) * gt.size()) != cudaSuccess ||
            cudaMalloc((void**)&h->d_gpart, sizeof(double) * kEstN * gt.size()) != cudaSuccess ||
            cudaMemcpy(h->d_gt, gt.data(), sizeof(BTile) * gt.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_inj_head, sizeof(uint64_t) * ap) != cudaSuccess ||
            cudaMemset(h->d_inj_head, 0, sizeof(uint64_t) * ap) != cudaSuccess)
            break;
        h->obs_cap = std::max(1, obs_cap);
        if (cudaMalloc((void**)&h->d_cyc, sizeof(PfcBatchCycle) * n_filters) != cudaSuccess ||
            cudaMallocHost((void**)&h->h_cyc, sizeof(PfcBatchCycle) * n_filters) != cudaSuccess ||
            cudaMalloc((void**)&h->d_obs, sizeof(CObservation) * h->obs_cap) != cudaSuccess ||
            cudaMallocHost((void**)&h->h_obs, sizeof(CObservation) * h->obs_cap) != cudaSuccess ||
            cudaMalloc((void**)&h->d_out, sizeof(double) * PFC_EST_LEN * n_filters) != cudaSuccess ||
            cudaMallocHost((void**)&h->h_out, sizeof(double) * PFC_EST_LEN * n_filters) != cudaSuccess ||
            cudaMalloc((void**)&h->d_prior, sizeof(float) * 13 * n_filters) != cudaSuccess)
            break;
        if (cudaMemset(h->d_cyc, 0, sizeof(PfcBatchCycle) * n_filters) != cudaSuccess ||
            cudaMemset(h->d_out, 0, sizeof(double) * PFC_EST_LEN * n_filters) != cudaSuccess)
            break;
        // an empty landmark table until landmarks are uploaded
        if (cudaMalloc((void**)&h->d_lm, sizeof(float) * 3) != cudaSuccess) break;
        if (cudaMemcpy(h->d_wt, wt.data(), sizeof(BTile) * wt.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess ||
            cudaMemcpy(h->d_rt, rt.data(), sizeof(BTile) * rt.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            break;
        k_b_init<<<ceil_div(n_filters, kThreads), kThreads, 0, h->stream>>>(h->d_C, h->d_G,
                                                                           n_filters);
        if (cudaGetLastError() != cudaSuccess) break;
        if (rebuild_est_tiles(h)) break;
        ok = true;
    } while (0);
    if (!ok) {
        set_error("pf_b200: pfc_batch_create failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
        free_batch(h);
        return nullptr;
    }
    return h;
}

int pfc_batch_destroy(void* p) {
    free_batch(as_b(p));
    return 0;
}

void* pfc_batch_stream(void* p) {
    BatchHandle* h = as_b(p);
    return h ? (void*)h->stream : nullptr;
}

int pfc_batch_size(void* p, int f) {
    BatchHandle* h = as_b(p);
    if (!h || f < 0 || f >= h->nf) return -1;
    return h->filters[f].n;
}

int pfc_batch_set_params(void* p, const PfcCycleParams* prm) {
    BatchHandle* h = as_b(p);
    if (!h || !prm) return -1;
    // injection counts: k = floor(ratio * n) with the single-filter path's
    // f32 product; global draw offsets in filter order
    std::vector<int> draw_f;
    for (int f = 0; f < h->nf; ++f) {
        BFilter& b = h->filters[f];
        b.sigma_r = prm[f].sigma_r;
        b.sigma_b = prm[f].sigma_b;
        b.gate = prm[f].gate;
        b.ess_ratio = prm[f].resample_ess_ratio;
        b.inject_ratio = prm[f].random_inject_ratio;
        int k = (b.inject_ratio > 0.f) ? (int)(b.inject_ratio * (float)b.n) : 0;
        if (k > b.n) k = b.n;
        b.inj_k = k;
        b.inj_off = (int)draw_f.size();
        draw_f.insert(draw_f.end(), (size_t)k, f);
    }
    if ((int)draw_f.size() > h->total_draws) {
        cudaFree(h->d_draw_f);
        cudaFree(h->d_inj_next);
        cudaFree(h->d_icorr);
        h->d_draw_f = nullptr;
        h->d_inj_next = nullptr;
        h->d_icorr = nullptr;
        PFB_CK(cudaMalloc((void**)&h->d_draw_f, sizeof(int) * draw_f.size()));
        PFB_CK(cudaMalloc((void**)&h->d_inj_next, sizeof(int) * draw_f.size()));
        PFB_CK(cudaMalloc((void**)&h->d_icorr, sizeof(double) * 3 * draw_f.size()));
    }
    h->total_draws = (int)draw_f.size();
    if (!draw_f.empty())
        PFB_CK(cudaMemcpyAsync(h->d_draw_f, draw_f.data(), sizeof(int) * draw_f.size(),
                               cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaMemcpyAsync(h->d_F, h->filters.data(), sizeof(BFilter) * h->nf,
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    return 0;
}

int pfc_batch_upload_landmarks(void* p, const float* xyz, const int* counts) {
    BatchHandle* h = as_b(p);
    if (!h || !counts) return -1;
    long long tot = 0;
    for (int f = 0; f < h->nf; ++f) {
        if (counts[f] < 0) return -1;
        h->filters[f].lm_off = (int)tot;
        h->filters[f].lm_count = counts[f];
        tot += counts[f];
    }
    if (tot > 0 && !xyz) return -1;
    if (tot > h->lm_total) {
        cudaFree(h->d_lm);
        h->d_lm = nullptr;
        PFB_CK(cudaMalloc((void**)&h->d_lm, sizeof(float) * 3 * (size_t)tot));
        h->lm_total = (int)tot;
    }
    if (tot > 0)
        PFB_CK(cudaMemcpyAsync(h->d_lm, xyz, sizeof(float) * 3 * (size_t)tot,
                               cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaMemcpyAsync(h->d_F, h->filters.data(), sizeof(BFilter) * h->nf,
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    drop_graph(h);
    return 0;
}

int pfc_batch_reinit(void* p, const float* pose7, const float* pos_std3,
                     const float* rot_std3) {
    BatchHandle* h = as_b(p);
    if (!h || !pose7 || !pos_std3 || !rot_std3) return -1;
    std::vector<float> pr(13 * (size_t)h->nf);
    for (int f = 0; f < h->nf; ++f) {
        for (int k = 0; k < 7; ++k) pr[13 * f + k] = pose7[7 * f + k];
        for (int k = 0; k < 3; ++k) pr[13 * f + 7 + k] = pos_std3[3 * f + k];
        for (int k = 0; k < 3; ++k) pr[13 * f + 10 + k] = rot_std3[3 * f + k];
    }
    PFB_CK(cudaMemcpyAsync(h->d_prior, pr.data(), sizeof(float) * pr.size(),
                           cudaMemcpyHostToDevice, h->stream));
    k_b_gen_inc<<<ceil_div(h->nf, kThreads), kThreads, 0, h->stream>>>(h->d_C, h->nf);
    k_b_reinit<<<h->n_wt, kThreads, 0, h->stream>>>(h->A, h->d_F, h->d_wt, h->d_C,
                                                    h->d_prior);
    h->launches += 2;
    PFB_KL();
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_batch_cycle(void* p, const PfcOdom* odom, const CObservation* obs,
                    const int* nobs, double* est_out) {
    BatchHandle* h = as_b(p);
    if (!h || !odom || !nobs) return -1;
    int off = 0;
    for (int f = 0; f < h->nf; ++f) {
        h->h_cyc[f].odom = odom[f];
        h->h_cyc[f].obs_off = off;
        h->h_cyc[f].nobs = std::max(0, nobs[f]);
        off += std::max(0, nobs[f]);
    }
    if (off > h->obs_cap) {
        set_error("pf_b200: pfc_batch_cycle: %d observations exceed capacity %d", off,
                  h->obs_cap);
        return -1;
    }
    if (off > 0 && !obs) return -1;
    if (off > 0) memcpy(h->h_obs, obs, sizeof(CObservation) * (size_t)off);
    PFB_CK(cudaMemcpyAsync(h->d_cyc, h->h_cyc, sizeof(PfcBatchCycle) * h->nf,
                           cudaMemcpyHostToDevice, h->stream));
    if (off > 0)
        PFB_CK(cudaMemcpyAsync(h->d_obs, h->h_obs, sizeof(CObservation) * (size_t)off,
                               cudaMemcpyHostToDevice, h->stream));
    if (run_cycle(h)) return -1;
    return finish(h, est_out);
}

int pfc_batch_cycle_device(void* p, const PfcBatchCycle* d_cycle,
                           const CObservation* d_obs, int n_obs, double* est_out) {
    BatchHandle* h = as_b(p);
    if (!h || !d_cycle || n_obs < 0 || n_obs > h->obs_cap) return -1;
    PFB_CK(cudaMemcpyAsync(h->d_cyc, d_cycle, sizeof(PfcBatchCycle) * h->nf,
                           cudaMemcpyDeviceToDevice, h->stream));
    if (n_obs > 0)
        PFB_CK(cudaMemcpyAsync(h->d_obs, d_obs, sizeof(CObservation) * (size_t)n_obs,
                               cudaMemcpyDeviceToDevice, h->stream));
    if (run_cycle(h)) return -1;
    if (!est_out) return 0;
    return finish(h, est_out);
}

int pfc_batch_result(void* p, double* est_out) {
    BatchHandle* h = as_b(p);
    if (!h || !est_out) return -1;
    return finish(h, est_out);
}

int pfc_batch_use_graph(void* p, int on) {
    BatchHandle* h = as_b(p);
    if (!h) return -1;
    h->use_graph = on != 0;
    if (!h->use_graph) drop_graph(h);
    return 0;
}

int pfc_batch_set_tiles(void* p, const int* est_tile, int use_packed) {
    BatchHandle* h = as_b(p);
    if (!h || !est_tile) return -1;
    for (int b = 0; b < kBuckets; ++b) {
        const int t = est_tile[b];
        if (t < 256 || t % 1024 != 0 || t > (1 << 20)) {
            set_error("pf_b200: estimate tile %d must be a multiple of 1024", t);
            return -1;
        }
    }
    h->est_tile.assign(est_tile, est_tile + kBuckets);
    h->use_packed = use_packed ? 1 : 0;
    return rebuild_est_tiles(h);
}

int pfc_batch_get_tiles(void* p, int* est_tile, int* use_packed) {
    BatchHandle* h = as_b(p);
    if (!h || !est_tile) return -1;
    for (int b = 0; b < kBuckets; ++b) est_tile[b] = h->est_tile[b];
    if (use_packed) *use_packed = h->use_packed;
    return 0;
}

// Autotuner: per size bucket, the estimate tile that minimises the time of
// the estimate + covariance passes (CUDA events, best of `reps`), then the
// weighting variant.  Timing runs re-evaluate the current state only (the
// passes are idempotent for a fixed cloud).  Writes the choices.
int pfc_batch_autotune(void* p, int reps, int* est_tile_out, int* packed_out) {
    BatchHandle* h = as_b(p);
    if (!h) return -1;
    if (reps <= 0) reps = 3;
    cudaEvent_t e0, e1;
    PFB_CK(cudaEventCreate(&e0));
    PFB_CK(cudaEventCreate(&e1));
    int rc = 0;
    auto time_est = [&](float* best) -> int {
        *best = 1e30f;
        for (int r = 0; r < reps; ++r) {
            if (cudaEventRecord(e0, h->stream) != cudaSuccess) return -1;
            // as in a cycle: filters that resampled take only the covariances
            if (launch_est_covs(h)) return -1;
            if (cudaEventRecord(e1, h->stream) != cudaSuccess) return -1;
            if (cudaEventSynchronize(e1) != cudaSuccess) return -1;
            float ms = 0.f;
            cudaEventElapsedTime(&ms, e0, e1);
            *best = std::min(*best, ms);
        }
        return 0;
    };
    for (int b = 0; b < kBuckets && rc == 0; ++b) {
        bool any = false;
        for (const BFilter& f : h->filters) any |= bucket_of(f.n) == b;
        if (!any) continue;
        int best_t = h->est_tile[b];
        float best_ms = 1e30f;
        for (int t : kEstTileChoices) {
            h->est_tile[b] = t;
            if (rebuild_est_tiles(h)) {
                rc = -1;
                break;
            }
            float ms;
            if (time_est(&ms)) {
                rc = -1;
                break;
            }
            if (ms < best_ms) {
                best_ms = ms;
                best_t = t;
            }
        }
        h->est_tile[b] = best_t;
    }
    if (rc == 0) rc = rebuild_est_tiles(h);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    if (rc) return -1;
    if (est_tile_out)
        for (int b = 0; b < kBuckets; ++b) est_tile_out[b] = h->est_tile[b];
    if (packed_out) *packed_out = h->use_packed;
    return 0;
}

int pfc_batch_snapshot(void* p, int f, float* pos3n, float* quat4n) {
    BatchHandle* h = as_b(p);
    if (!h || f < 0 || f >= h->nf || !pos3n || !quat4n) return -1;
    const int n = h->filters[f].n;
    if (ensure_tmp(h, 7ll * n)) return -1;
    k_b_pack<<<std::min(ceil_div(n, kThreads), 1184), kThreads, 0, h->stream>>>(
        h->A, h->d_F, h->d_C, f, h->d_tmp, h->d_tmp + 3 * (size_t)n);
    PFB_KL();
    PFB_CK(cudaMemcpyAsync(pos3n, h->d_tmp, sizeof(float) * 3 * (size_t)n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaMemcpyAsync(quat4n, h->d_tmp + 3 * (size_t)n,
                           sizeof(float) * 4 * (size_t)n, cudaMemcpyDeviceToHost,
                           h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_batch_get_weights(void* p, int f, float* w) {
    BatchHandle* h = as_b(p);
    if (!h || f < 0 || f >= h->nf || !w) return -1;
    const int n = h->filters[f].n;
    if (ensure_tmp(h, n)) return -1;
    k_b_weights<<<std::min(ceil_div(n, kThreads), 1184), kThreads, 0, h->stream>>>(
        h->A, h->d_F, h->d_C, f, h->d_tmp);
    PFB_KL();
    PFB_CK(cudaMemcpyAsync(w, h->d_tmp, sizeof(float) * (size_t)n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_batch_set_wait_test(void* p, int spin_limit, int stall_filter) {
    BatchHandle* h = as_b(p);
    if (!h || spin_limit < 0 || stall_filter < -1 || stall_filter >= h->nf) {
        set_error("pf_b200: pfc_batch_set_wait_test: bad arguments");
        return -1;
    }
    const int v[2] = {spin_limit > 0 ? spin_limit : kSpinLimit, stall_filter};
    PFB_CK(cudaMemcpyAsync(&h->d_G->spin_limit, v, sizeof(v), cudaMemcpyHostToDevice,
                           h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

long long pfc_batch_launches(void* p) {
    BatchHandle* h = as_b(p);
    return h ? h->launches : -1;
}

}  // extern "C"
