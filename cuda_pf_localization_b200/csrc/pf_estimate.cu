// pf_estimate.cu — weighted mean / moment / covariance reductions in FP64 and
// the device Markley mean.
//
// Pass 1 (k_est_sums) reads pose + weight (28 + 4 B per particle) and writes
// the 14 sums of the reference's pfc_est_sums layout
// (src/cuda/pf_kernels.cu:354-404).  Every per-particle product and every
// partial is FP64 (the reference accumulates per thread in f32).  The last
// block combines the per-block partials in block order,
// runs the Markley eigen-solve and stores the f32 means that the covariance
// pass uses.
// Pass 2 (k_covs) reads pose + weight again and writes the 12 covariance sums
// of the reference's pfc_covs layout (src/cuda/pf_kernels.cu:406-471), with
// the attitude residual of (qm^-1 * q) in FP64.
//
// Both passes read four particles per iteration with 16-byte loads from each
// SoA plane (eight loads in flight per thread), which is what keeps HBM busy
// at two resident blocks per SM.
//
// Before a resample a lighter pass (k_ess) reads only the weights or
// log-likelihoods: it materialises the weights and forms sum w^2, the exact
// fixed-point weight total and the per-block prefixes the resampler starts
// from; in the fused cycle it also takes the resample decision, so the full
// estimate and covariance passes run once, over the cloud the cycle ends
// with.
#include <math.h>

#include "markley.h"
#include "pf_device.cuh"

namespace pfb {

namespace {

using namespace pfb::dev;
constexpr int kThreads = kBlk;
// Two resident blocks per SM keep enough 16-byte loads in flight; a fixed,
// small grid also keeps the last block's combine short.
constexpr int kMaxBlocks = 2 * 148;

PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

// Reduce NV per-thread FP64 accumulators over the block into part[blk*NV+k];
// the last block to finish sums the partials of all blocks (G <= kMaxBlocks)
// in block order into out[k] and returns true (in every thread of that
// block).  The last block first stages every partial in shared memory with
// one round of loads, so the combine costs one L2 round trip.
template <int NV>
__device__ bool block_reduce_last(double (&acc)[NV], double* part,
                                  unsigned* done, double* out) {
    __shared__ double s_w[NV][kThreads / 32];
    __shared__ double s_p[NV * kMaxBlocks];  // [k][block]
    __shared__ bool s_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int k = 0; k < NV; ++k) {
        double v = warp_sum_d(acc[k]);
        if (lane == 0) s_w[k][warp] = v;
    }
    __syncthreads();
    if (tid < NV) {
        double v = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) v += s_w[tid][k];
        part[(size_t)blockIdx.x * NV + tid] = v;
        __threadfence();
    }
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    const int G = gridDim.x;
    const int tot = G * NV;
    constexpr int kPer = (NV * kMaxBlocks + kThreads - 1) / kThreads;
    double v[kPer];
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        const int idx = tid + r * kThreads;
        v[r] = idx < tot ? __ldcg(&part[idx]) : 0.0;
    }
#pragma unroll
    for (int r = 0; r < kPer; ++r) {
        const int idx = tid + r * kThreads;
        if (idx < tot) s_p[(idx % NV) * kMaxBlocks + idx / NV] = v[r];
    }
    __syncthreads();
    for (int k = warp; k < NV; k += kThreads / 32) {
        double a = 0.0;
        for (int b = lane; b < G; b += 32) a += s_p[k * kMaxBlocks + b];
        a = warp_sum_d(a);
        if (lane == 0) out[k] = a;
    }
    __syncthreads();
    if (tid == 0) *done = 0u;
    return true;
}

__global__ void __launch_bounds__(kThreads, 2)
    k_est_sums(PlaneSet ps, int n, const float* __restrict__ ll,
               float* __restrict__ w, double* part, unsigned* done,
               CycleCtl* ctl, int sq_from_ess, double skip_ratio) {
    pdl_wait();
    if (sq_from_ess && skip_ratio > 0.0) {
        // the caller resamples when this estimate's ESS is below
        // skip_ratio * n and then discards it: only sum w^2 is reported
        const double sq = ctl->sq_w;
        const double ess = sq > 0.0 ? 1.0 / sq : 0.0;
        if (ess < skip_ratio * (double)n) {
            if (blockIdx.x == 0 && threadIdx.x == 0) {
                ctl->est[13] = sq;
                ctl->ess = ess;
                ctl->est_partial = 1;
                ctl->cov_mean_p[0] = __int_as_float(0x7fc00000);
            }
            return;
        }
    }
    const Planes s = pick_planes(ps, ctl->live);
    const int wmode = ctl->wmode;
    const float M = ctl->ll_max, S = ctl->ll_sumexp;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)n;
    double acc[kEstN];
#pragma unroll
    for (int k = 0; k < kEstN; ++k) acc[k] = 0.0;
    const int n4 = (n + 3) >> 2;
    const float4* px = reinterpret_cast<const float4*>(s.px);
    const float4* py = reinterpret_cast<const float4*>(s.py);
    const float4* pz = reinterpret_cast<const float4*>(s.pz);
    const float4* qw = reinterpret_cast<const float4*>(s.qw);
    const float4* qx = reinterpret_cast<const float4*>(s.qx);
    const float4* qy = reinterpret_cast<const float4*>(s.qy);
    const float4* qz = reinterpret_cast<const float4*>(s.qz);
    for (int i4 = blockIdx.x * kThreads + threadIdx.x; i4 < n4;
         i4 += gridDim.x * kThreads) {
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
        for (int c = 0; c < 4; ++c) {
            if (4 * i4 + c >= n) break;
            const float wf = comp(W, c);
            est_add(acc, wf, comp(X, c), comp(Y, c), comp(Z, c), comp(QW, c),
                    comp(QX, c), comp(QY, c), comp(QZ, c));
        }
    }
    __shared__ double s_out[kEstN];
    if (!block_reduce_last<kEstN>(acc, part, done, s_out)) return;
    double qm[4];
    if (threadIdx.x < 32) markley_mean_warp_call(&s_out[3], qm);  // warp 0
    if (threadIdx.x == 0) {
        if (sq_from_ess) s_out[13] = ctl->sq_w;
        for (int k = 0; k < kEstN; ++k) ctl->est[k] = s_out[k];
        ctl->ess = s_out[13] > 0.0 ? 1.0 / s_out[13] : 0.0;
        ctl->est_partial = 0;
        for (int k = 0; k < 4; ++k) ctl->qmean[k] = qm[k];
        for (int k = 0; k < 3; ++k) ctl->cov_mean_p[k] = (float)s_out[k];
        for (int k = 0; k < 4; ++k) ctl->cov_mean_q[k] = (float)qm[k];
        if (wmode == WMODE_LL) ctl->wmode = WMODE_STORED;
    }
}

// mode: 0 plain, 1 last pass of a fused cycle (also emits the output record).
// skip_ratio > 0: the caller resamples whenever the ESS of the estimate just
// computed is below skip_ratio * n (ParticleFilter::update's rule), and then
// discards this estimate's covariances; the pass is skipped in that case and
// the cached mean is made unusable, so pfc_covs computes them on demand.
__global__ void __launch_bounds__(kThreads, 2)
    k_covs(PlaneSet ps, int n, const float* __restrict__ ll,
           const float* __restrict__ w, double* part, unsigned* done,
           CycleCtl* ctl, int use_args, float3 mp_arg, float4 mq_arg,
           int mode, double skip_ratio) {
    pdl_wait();
    if (skip_ratio > 0.0 && ctl->ess < skip_ratio * (double)n) {
        if (blockIdx.x == 0 && threadIdx.x == 0) ctl->cov_mean_p[0] = __int_as_float(0x7fc00000);
        return;
    }
    const Planes s = pick_planes(ps, ctl->live);
    const int wmode = ctl->wmode;
    const float M = ctl->ll_max, S = ctl->ll_sumexp;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)n;
    float3 mpf;
    float4 mqf;
    if (use_args) {
        mpf = mp_arg;
        mqf = mq_arg;
    } else {
        mpf = make_float3(ctl->cov_mean_p[0], ctl->cov_mean_p[1],
                          ctl->cov_mean_p[2]);
        mqf = make_float4(ctl->cov_mean_q[0], ctl->cov_mean_q[1],
                          ctl->cov_mean_q[2], ctl->cov_mean_q[3]);
    }
    const double mp[3] = {(double)mpf.x, (double)mpf.y, (double)mpf.z};
    const double qm[4] = {(double)mqf.x, (double)mqf.y, (double)mqf.z,
                          (double)mqf.w};
    double acc[kCovN];
#pragma unroll
    for (int k = 0; k < kCovN; ++k) acc[k] = 0.0;
    const int n4 = (n + 3) >> 2;
    const float4* px = reinterpret_cast<const float4*>(s.px);
    const float4* py = reinterpret_cast<const float4*>(s.py);
    const float4* pz = reinterpret_cast<const float4*>(s.pz);
    const float4* qw = reinterpret_cast<const float4*>(s.qw);
    const float4* qx = reinterpret_cast<const float4*>(s.qx);
    const float4* qy = reinterpret_cast<const float4*>(s.qy);
    const float4* qz = reinterpret_cast<const float4*>(s.qz);
    for (int i4 = blockIdx.x * kThreads + threadIdx.x; i4 < n4;
         i4 += gridDim.x * kThreads) {
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
        for (int c = 0; c < 4; ++c) {
            if (4 * i4 + c >= n) break;
            cov_add(acc, (double)comp(W, c), comp(X, c), comp(Y, c), comp(Z, c),
                    comp(QW, c), comp(QX, c), comp(QY, c), comp(QZ, c), mp, qm);
        }
    }
    __shared__ double s_out[kCovN];
    if (!block_reduce_last<kCovN>(acc, part, done, s_out)) return;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kCovN; ++k) ctl->covs[k] = s_out[k];
        ctl->cov_mean_p[0] = mpf.x;
        ctl->cov_mean_p[1] = mpf.y;
        ctl->cov_mean_p[2] = mpf.z;
        ctl->cov_mean_q[0] = mqf.x;
        ctl->cov_mean_q[1] = mqf.y;
        ctl->cov_mean_q[2] = mqf.z;
        ctl->cov_mean_q[3] = mqf.w;
        if (mode == 1) {
            double* o = ctl->out;
            for (int k = 0; k < 3; ++k) o[PFC_EST_POS + k] = ctl->est[k];
            for (int k = 0; k < 4; ++k) o[PFC_EST_QUAT + k] = ctl->qmean[k];
            for (int k = 0; k < 6; ++k) o[PFC_EST_POSCOV + k] = s_out[k];
            for (int k = 0; k < 6; ++k) o[PFC_EST_ATTCOV + k] = s_out[6 + k];
            // without a resample the cycle reports the ESS its decision used,
            // as ParticleFilter::update returns its first estimate
            o[PFC_EST_ESS] = ctl->resampled ? ctl->ess : ctl->ess_pre;
            o[PFC_EST_RESAMPLED] = ctl->resampled ? 1.0 : 0.0;
        }
    }
}

// Weight pass before a resample: weights materialised from the
// log-likelihoods (4 B read, 4 B written per particle), sum w^2 in FP64, the
// exact fixed-point weight total, the bad-weight flag and the exclusive
// fixed-point prefix of every run of kPrefixBlock particles, which the
// resampler starts from (so it needs no inter-block look-back).  With decide
// set it also takes ParticleFilter::update's decision ratio > 0 &&
// ess < ratio * N (crates/pf_core/src/particle_filter.rs:115-117) for the
// fused cycle.  One float4 of weights per thread, kPrefixBlock particles per
// block, so the grid fills every SM; the FP64 sum is reduced in a fixed order
// (block butterfly, then block partials in block order).
__global__ void __launch_bounds__(kThreads)
    k_ess(int n, const float* __restrict__ ll, float* __restrict__ w,
          double* part, unsigned long long* partu, uint64_t* prefix,
          unsigned* done, CycleCtl* ctl, int decide, double ess_ratio) {
    pdl_wait();
    static_assert(kPrefixBlock == 8 * kThreads, "two float4 per thread");
    const int wmode = ctl->wmode;
    const float M = ctl->ll_max, S = ctl->ll_sumexp;
    const double rS = __drcp_rn((double)S);
    const float wuni = 1.0f / (float)n;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    double sq = 0.0;
    unsigned long long tfx = 0;
    int bad = 0;
#pragma unroll
    for (int hh = 0; hh < 2; ++hh) {
        const int i4 = blockIdx.x * 2 * kThreads + hh * kThreads + tid;
        if (4 * i4 >= n) break;
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
        for (int c = 0; c < 4; ++c) {
            if (4 * i4 + c >= n) break;
            const float wf = comp(W, c);
            bad |= weight_bad(wf) ? 1 : 0;
            tfx += weight_bad(wf) ? 0ull : weight_fx(wf);
            const double wd = (double)wf;
            sq = __fma_rn(wd, wd, sq);
        }
    }
    constexpr int kStage = 4096;  // block totals staged by the last block
    __shared__ double s_d[kThreads / 32];
    __shared__ unsigned long long s_u[kThreads / 32];
    __shared__ unsigned long long s_tot[kStage];
    __shared__ bool s_last;
    sq = warp_sum_d(sq);
    tfx = warp_sum_u64(tfx);
    if (lane == 0) {
        s_d[warp] = sq;
        s_u[warp] = tfx;
    }
    const int any_bad = __syncthreads_or(bad);
    if (tid == 0) {
        double a = 0.0;
        unsigned long long u = 0;
        for (int k = 0; k < kThreads / 32; ++k) {
            a += s_d[k];
            u += s_u[k];
        }
        part[blockIdx.x] = a;
        partu[2 * (size_t)blockIdx.x] = u;
        partu[2 * (size_t)blockIdx.x + 1] = any_bad ? 1ull : 0ull;
        __threadfence();
        s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Last block: sum w^2 over the block partials, and the exclusive prefix
    // of the block totals (each thread scans a contiguous range of blocks).
    // Up to kStage block totals are staged in shared memory with all loads
    // in flight at once; larger grids read them from L2 twice.
    const int G = gridDim.x;
    double a = 0.0;
    int fb = 0;
#pragma unroll 4
    for (int b = tid; b < G; b += kThreads) {
        a += __ldcg(&part[b]);
        fb |= __ldcg(&partu[2 * (size_t)b + 1]) != 0ull ? 1 : 0;
    }
    a = warp_sum_d(a);
    const bool staged = G <= kStage;
    if (staged) {
#pragma unroll 4
        for (int b = tid; b < G; b += kThreads) s_tot[b] = __ldcg(&partu[2 * (size_t)b]);
    }
    __syncthreads();
    const int per = (G + kThreads - 1) / kThreads;
    const int b0 = min(G, tid * per), b1 = min(G, b0 + per);
    unsigned long long run = 0;
    for (int b = b0; b < b1; ++b) run += staged ? s_tot[b] : __ldcg(&partu[2 * (size_t)b]);
    // block-exclusive scan of the thread ranges
    unsigned long long x = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const unsigned long long y = __shfl_up_sync(~0u, x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_u[warp] = x;
    if (lane == 0) s_d[warp] = a;
    const int any_fb = __syncthreads_or(fb);
    unsigned long long wbase = 0, T = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
        wbase += (k < warp) ? s_u[k] : 0ull;
        T += s_u[k];
    }
    unsigned long long off = wbase + x - run;
    for (int b = b0; b < b1; ++b) {
        prefix[b] = off;
        off += staged ? s_tot[b] : __ldcg(&partu[2 * (size_t)b]);
    }
    if (tid == 0) {
        double sum = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) sum += s_d[k];
        const double ess = sum > 0.0 ? 1.0 / sum : 0.0;
        if (decide) {
            ctl->ess = ess;
            ctl->ess_pre = ess;
            ctl->out[PFC_EST_ESS_PRE] = ess;
            ctl->resample_now =
                (ess_ratio > 0.0 && ess < ess_ratio * (double)n) ? 1 : 0;
            ctl->resampled = 0;
            ctl->out[PFC_EST_RESAMPLED] = 0.0;
        }
        ctl->w_total_fx = T;
        ctl->w_bad = any_fb;
        ctl->sq_w = sum;
        if (wmode == WMODE_LL) ctl->wmode = WMODE_STORED;
        *done = 0u;
    }
}

__global__ void k_materialize_w(int n, const float* __restrict__ ll,
                                float* __restrict__ w, CycleCtl* ctl) {
    const int wmode = ctl->wmode;
    const float M = ctl->ll_max, S = ctl->ll_sumexp;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
         i += gridDim.x * kThreads) {
        const float wf = weight_of(wmode, i, n, w, ll, M, S);
        if (wmode != WMODE_STORED) w[i] = wf;
    }
}

__global__ void k_set_stored(CycleCtl* ctl) { ctl->wmode = WMODE_STORED; }

// Both quotient forms of the weight normalisation on caller pairs (e, S).
__global__ void k_weight_div_check(const float* __restrict__ e, const float* __restrict__ s,
                                   int n, float* __restrict__ fast,
                                   float* __restrict__ ieee) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const float S = s[i];
    fast[i] = weight_div(e[i], S, __drcp_rn((double)S));
    ieee[i] = __fdiv_rn(e[i], S);
}

int est_grid(int n) {
    int g = ceil_div(ceil_div(n, 4), kThreads);
    return g < kMaxBlocks ? g : kMaxBlocks;
}

}  // namespace

int launch_est_sums(PfHandle* h, bool sq_from_ess, double skip_ratio) {
    KernelScope ks(h, KK_EST);
    PFB_CK(launch_pdl(k_est_sums, est_grid(h->n), kThreads, 0, h->stream, plane_set(h),
                      h->n, h->d_ll, h->d_w, h->d_part, h->d_done + 1, h->d_ctl,
                      sq_from_ess ? 1 : 0, skip_ratio));
    PFB_KL();
    return 0;
}

int launch_covs(PfHandle* h, bool use_args, const float mp[3],
                const float mq[4], bool cycle_output, double skip_ratio) {
    float3 a = use_args ? make_float3(mp[0], mp[1], mp[2])
                        : make_float3(0.f, 0.f, 0.f);
    float4 b = use_args ? make_float4(mq[0], mq[1], mq[2], mq[3])
                        : make_float4(1.f, 0.f, 0.f, 0.f);
    KernelScope ks(h, KK_COVS);
    PFB_CK(launch_pdl(k_covs, est_grid(h->n), kThreads, 0, h->stream, plane_set(h), h->n,
                      h->d_ll, h->d_w, h->d_part, h->d_done + 2, h->d_ctl,
                      use_args ? 1 : 0, a, b, cycle_output ? 1 : 0, skip_ratio));
    PFB_KL();
    return 0;
}

int launch_weight_prefix(PfHandle* h, bool decide, double ess_ratio) {
    KernelScope ks(h, KK_EST);
    PFB_CK(launch_pdl(k_ess, ceil_div(h->n, kPrefixBlock), kThreads, 0, h->stream, h->n,
                      h->d_ll, h->d_w, h->d_part, h->d_part_u64, h->d_wprefix,
                      h->d_done + 3, h->d_ctl, decide ? 1 : 0, ess_ratio));
    PFB_KL();
    h->prefix_valid = true;
    return 0;
}

int launch_cycle_decide(PfHandle* h, double ess_ratio) {
    return launch_weight_prefix(h, true, ess_ratio);
}

int launch_weight_div_check(PfHandle* h, const float* d_e, const float* d_s, int n,
                            float* d_fast, float* d_ieee) {
    k_weight_div_check<<<ceil_div(n, kThreads), kThreads, 0, h->stream>>>(d_e, d_s, n,
                                                                          d_fast, d_ieee);
    PFB_KL();
    return 0;
}

int launch_materialize_weights(PfHandle* h) {
    {
        KernelScope ks(h, KK_MISC);
        k_materialize_w<<<est_grid(h->n), kThreads, 0, h->stream>>>(
            h->n, h->d_ll, h->d_w, h->d_ctl);
    }
    PFB_KL();
    {
        KernelScope ks(h, KK_MISC);
        k_set_stored<<<1, 1, 0, h->stream>>>(h->d_ctl);
    }
    PFB_KL();
    return 0;
}

}  // namespace pfb
