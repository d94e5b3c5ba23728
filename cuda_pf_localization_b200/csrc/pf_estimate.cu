// pf_estimate.cu — weighted mean / moment / covariance reductions in FP64 and
// the device Markley mean.
//
// Pass 1 (k_est_sums) reads pose + weight (28 + 4 B per particle) and writes
// the 14 sums of the reference's pfc_est_sums layout
// (src/cuda/pf_kernels.cu:354-404).  Every per-particle product and every
// partial is FP64 (the reference accumulates per thread in f32).  The last
// block combines the per-block partials in block order, runs the Markley
// eigen-solve and stores the f32 means that the covariance pass uses.
// Pass 2 (k_covs) reads pose + weight again and writes the 12 covariance sums
// of the reference's pfc_covs layout (src/cuda/pf_kernels.cu:406-471), with
// the attitude residual of (qm^-1 * q) in FP64.
#include <math.h>

#include "markley.h"
#include "pf_internal.h"

namespace pfb {

namespace {

constexpr int kThreads = 256;
constexpr int kMaxBlocks = 1184;  // 148 SMs x 8 resident blocks

struct PlaneSet {
    Planes s[2];
};
PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    return v;
}

// Normalised f32 weight of particle i under the cloud's weight mode.
__device__ __forceinline__ float weight_of(int wmode, int i, int n,
                                           const float* __restrict__ w,
                                           const float* __restrict__ ll,
                                           double M, double S) {
    if (wmode == WMODE_UNIFORM) return 1.0f / (float)n;
    if (wmode == WMODE_STORED) return w[i];
    return (float)(exp((double)ll[i] - M) / S);
}

// Reduce NV per-thread FP64 accumulators over the block into part[blk*NV+k];
// the last block to finish sums the partials of all blocks in block order
// into out[k] and returns true (in every thread of that block).
template <int NV>
__device__ bool block_reduce_last(double (&acc)[NV], double* part,
                                  unsigned* done, double* out) {
    __shared__ double s_w[NV][kThreads / 32];
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
    }
    __threadfence();
    __syncthreads();
    if (tid == 0) s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    __syncthreads();
    if (!s_last) return false;
    __threadfence();
    const int G = gridDim.x;
    // warp w combines components w, w+8, ...; lanes stride over blocks.
    for (int k = warp; k < NV; k += kThreads / 32) {
        double v = 0.0;
        for (int b = lane; b < G; b += 32) v += __ldcg(&part[(size_t)b * NV + k]);
        v = warp_sum_d(v);
        if (lane == 0) out[k] = v;
    }
    __syncthreads();
    if (tid == 0) *done = 0u;
    return true;
}

__global__ void __launch_bounds__(kThreads)
    k_est_sums(PlaneSet ps, int n, const float* __restrict__ ll,
               float* __restrict__ w, double* part, unsigned* done,
               CycleCtl* ctl, int cond_second) {
    if (cond_second && !ctl->resample_now) return;
    const Planes s = ps.s[ctl->live];
    const int wmode = ctl->wmode;
    const double M = ctl->ll_max, S = ctl->ll_sumexp;
    double acc[kEstN];
#pragma unroll
    for (int k = 0; k < kEstN; ++k) acc[k] = 0.0;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
         i += gridDim.x * kThreads) {
        const float wf = weight_of(wmode, i, n, w, ll, M, S);
        if (wmode == WMODE_LL) w[i] = wf;
        const double wd = (double)wf;
        acc[0] += wd * (double)s.px[i];
        acc[1] += wd * (double)s.py[i];
        acc[2] += wd * (double)s.pz[i];
        const double q[4] = {(double)s.qw[i], (double)s.qx[i], (double)s.qy[i],
                             (double)s.qz[i]};
        int e = 3;
#pragma unroll
        for (int r = 0; r < 4; ++r)
#pragma unroll
            for (int c = r; c < 4; ++c) acc[e++] += wd * q[r] * q[c];
        acc[13] += wd * wd;
    }
    __shared__ double s_out[kEstN];
    if (!block_reduce_last<kEstN>(acc, part, done, s_out)) return;
    if (threadIdx.x == 0) {
        for (int k = 0; k < kEstN; ++k) ctl->est[k] = s_out[k];
        ctl->ess = s_out[13] > 0.0 ? 1.0 / s_out[13] : 0.0;
        double qm[4];
        markley_mean(&s_out[3], qm);
        for (int k = 0; k < 4; ++k) ctl->qmean[k] = qm[k];
        for (int k = 0; k < 3; ++k) ctl->cov_mean_p[k] = (float)s_out[k];
        for (int k = 0; k < 4; ++k) ctl->cov_mean_q[k] = (float)qm[k];
        if (wmode == WMODE_LL) ctl->wmode = WMODE_STORED;
    }
}

// Attitude residual of q about qm as a canonical rotation vector
// (w >= 0, angle = 2 atan2(|v|, w)), in FP64 — the form of
// src/cuda/pf_kernels.cu:435-447 and crates/pf_core/src/cpu.rs:346-366.
__device__ __forceinline__ void att_residual(const double qm[4],
                                             const double q[4], double aav[3]) {
    // dq = conj(qm) * q
    const double aw = qm[0], ax = -qm[1], ay = -qm[2], az = -qm[3];
    double dw = aw * q[0] - ax * q[1] - ay * q[2] - az * q[3];
    double dx = aw * q[1] + ax * q[0] + ay * q[3] - az * q[2];
    double dy = aw * q[2] - ax * q[3] + ay * q[0] + az * q[1];
    double dz = aw * q[3] + ax * q[2] - ay * q[1] + az * q[0];
    if (dw < 0.0) {
        dw = -dw;
        dx = -dx;
        dy = -dy;
        dz = -dz;
    }
    const double hv = sqrt(dx * dx + dy * dy + dz * dz);
    const double ang = 2.0 * atan2(hv, dw);
    if (hv > 1e-12) {
        aav[0] = dx / hv * ang;
        aav[1] = dy / hv * ang;
        aav[2] = dz / hv * ang;
    } else {
        aav[0] = aav[1] = aav[2] = 0.0;
    }
}

// mode: 0 plain, 1 first pass of a fused cycle (decide resample), 2 second
// pass of a fused cycle (skip unless resampling; emit the output record).
__global__ void __launch_bounds__(kThreads)
    k_covs(PlaneSet ps, int n, const float* __restrict__ ll,
           const float* __restrict__ w, double* part, unsigned* done,
           CycleCtl* ctl, int use_args, float3 mp_arg, float4 mq_arg,
           int mode, double ess_ratio) {
    if (mode == 2 && !ctl->resample_now) return;
    const Planes s = ps.s[ctl->live];
    const int wmode = ctl->wmode;
    const double M = ctl->ll_max, S = ctl->ll_sumexp;
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
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
         i += gridDim.x * kThreads) {
        const double wd = (double)weight_of(wmode, i, n, w, ll, M, S);
        const double dp[3] = {(double)s.px[i] - mp[0], (double)s.py[i] - mp[1],
                              (double)s.pz[i] - mp[2]};
        int e = 0;
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = r; c < 3; ++c) acc[e++] += wd * dp[r] * dp[c];
        const double q[4] = {(double)s.qw[i], (double)s.qx[i], (double)s.qy[i],
                             (double)s.qz[i]};
        double aav[3];
        att_residual(qm, q, aav);
#pragma unroll
        for (int r = 0; r < 3; ++r)
#pragma unroll
            for (int c = r; c < 3; ++c) acc[e++] += wd * aav[r] * aav[c];
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
        if (mode == 1 || mode == 2) {
            double* o = ctl->out;
            for (int k = 0; k < 3; ++k) o[PFC_EST_POS + k] = ctl->est[k];
            for (int k = 0; k < 4; ++k) o[PFC_EST_QUAT + k] = ctl->qmean[k];
            for (int k = 0; k < 6; ++k) o[PFC_EST_POSCOV + k] = s_out[k];
            for (int k = 0; k < 6; ++k) o[PFC_EST_ATTCOV + k] = s_out[6 + k];
            o[PFC_EST_ESS] = ctl->ess;
        }
        if (mode == 1) {
            // ParticleFilter::update's trigger: ratio > 0 && ess < ratio * N
            // (crates/pf_core/src/particle_filter.rs:115-117).
            ctl->ess_pre = ctl->ess;
            ctl->out[PFC_EST_ESS_PRE] = ctl->ess;
            const int go =
                (ess_ratio > 0.0 && ctl->ess < ess_ratio * (double)n) ? 1 : 0;
            ctl->resample_now = go;
            ctl->resampled = 0;
            ctl->out[PFC_EST_RESAMPLED] = 0.0;
        }
        if (mode == 2) ctl->out[PFC_EST_RESAMPLED] = ctl->resampled ? 1.0 : 0.0;
    }
}

__global__ void k_materialize_w(int n, const float* __restrict__ ll,
                                float* __restrict__ w, CycleCtl* ctl) {
    const int wmode = ctl->wmode;
    const double M = ctl->ll_max, S = ctl->ll_sumexp;
    for (int i = blockIdx.x * kThreads + threadIdx.x; i < n;
         i += gridDim.x * kThreads) {
        const float wf = weight_of(wmode, i, n, w, ll, M, S);
        if (wmode != WMODE_STORED) w[i] = wf;
    }
}

__global__ void k_set_stored(CycleCtl* ctl) { ctl->wmode = WMODE_STORED; }

int est_grid(int n) {
    int g = ceil_div(n, kThreads);
    return g < kMaxBlocks ? g : kMaxBlocks;
}

}  // namespace

int launch_est_sums(PfHandle* h, bool cycle_second) {
    KernelScope ks(h, KK_EST);
    k_est_sums<<<est_grid(h->n), kThreads, 0, h->stream>>>(
        plane_set(h), h->n, h->d_ll, h->d_w, h->d_part, h->d_done + 1,
        h->d_ctl, cycle_second ? 1 : 0);
    PFB_KL();
    return 0;
}

int launch_covs(PfHandle* h, bool use_args, const float mp[3],
                const float mq[4], bool cycle_second) {
    float3 a = use_args ? make_float3(mp[0], mp[1], mp[2])
                        : make_float3(0.f, 0.f, 0.f);
    float4 b = use_args ? make_float4(mq[0], mq[1], mq[2], mq[3])
                        : make_float4(1.f, 0.f, 0.f, 0.f);
    KernelScope ks(h, KK_COVS);
    k_covs<<<est_grid(h->n), kThreads, 0, h->stream>>>(
        plane_set(h), h->n, h->d_ll, h->d_w, h->d_part, h->d_done + 2, h->d_ctl,
        use_args ? 1 : 0, a, b, cycle_second ? 2 : 0, 0.0);
    PFB_KL();
    return 0;
}

// First covariance pass of a fused cycle: also decides the resample.
int launch_cycle_decide(PfHandle* h, double ess_ratio) {
    float3 a = make_float3(0.f, 0.f, 0.f);
    float4 b = make_float4(1.f, 0.f, 0.f, 0.f);
    KernelScope ks(h, KK_COVS);
    k_covs<<<est_grid(h->n), kThreads, 0, h->stream>>>(
        plane_set(h), h->n, h->d_ll, h->d_w, h->d_part, h->d_done + 2, h->d_ctl,
        0, a, b, 1, ess_ratio);
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

int launch_cycle_output(PfHandle* h) {
    (void)h;
    return 0;
}

}  // namespace pfb
