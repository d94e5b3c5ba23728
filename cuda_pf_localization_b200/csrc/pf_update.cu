// pf_update.cu — prior (reinit), motion update (predict) and landmark
// weighting kernels on the SoA particle planes.
//
// The weighting kernel optionally runs a deferred predict first, so one pass
// over HBM reads the old pose, writes the new pose and the log-likelihood,
// and leaves per-block softmax partials (block max, sum exp(ll - block max)
// in FP64).  The last block to finish combines the partials in block order,
// so M = max ll and S = sum exp(ll - M) are deterministic.
#include <math.h>

#include "pf_device.cuh"

namespace pfb {

namespace {

using namespace pfb::dev;
constexpr int kThreads = kBlk;


PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__global__ void __launch_bounds__(kThreads)
    k_reinit(PlaneSet ps, int n, uint64_t seed, uint64_t gen, float3 p0,
             Quat q0, float3 pstd, float3 rstd, CycleCtl* ctl) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const Planes s = pick_planes(ps, ctl->live);
    float nz[6];
    pf_normals6(seed, gen, (uint32_t)i, nz);
    float3 p = make_float3(p0.x + pstd.x * nz[0], p0.y + pstd.y * nz[1],
                           p0.z + pstd.z * nz[2]);
    float3 axis = make_float3(rstd.x * nz[3], rstd.y * nz[4], rstd.z * nz[5]);
    float ang = norm3(axis);
    Quat dq = q_from_axis_angle(axis, ang);
    store_pose(s, i, p, q_product(q0, dq));
}

// Reinitialisation around k planar poses (x, y, yaw) held in device memory:
// particle i starts from pose i mod k at height z with attitude = yaw about
// +z, then the same Gaussian perturbation as k_reinit.
__global__ void __launch_bounds__(kThreads)
    k_reinit_poses(PlaneSet ps, int n, uint64_t seed, uint64_t gen,
                   const float* __restrict__ poses, int k, float z, float3 pstd,
                   float3 rstd, CycleCtl* ctl) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const Planes s = pick_planes(ps, ctl->live);
    const int j = i % k;
    const float x0 = poses[3 * j], y0 = poses[3 * j + 1], yaw = poses[3 * j + 2];
    float sh, ch;
    sincosf(0.5f * yaw, &sh, &ch);
    const Quat q0{ch, 0.0f, 0.0f, sh};
    float nz[6];
    pf_normals6(seed, gen, (uint32_t)i, nz);
    float3 p = make_float3(x0 + pstd.x * nz[0], y0 + pstd.y * nz[1],
                           z + pstd.z * nz[2]);
    float3 axis = make_float3(rstd.x * nz[3], rstd.y * nz[4], rstd.z * nz[5]);
    float ang = norm3(axis);
    Quat dq = q_from_axis_angle(axis, ang);
    store_pose(s, i, p, q_product(q0, dq));
}

__global__ void __launch_bounds__(kThreads)
    k_predict(PlaneSet ps, int n, uint64_t seed, PredictArgs pa,
              CycleCtl* ctl) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const Planes s = pick_planes(ps, ctl->live);
    float3 p;
    Quat q;
    load_pose(s, i, p, q);
    apply_predict(pa, seed, i, p, q);
    store_pose(s, i, p, q);
}

// M and S of the softmax into the control block (weights valid when S is a
// positive finite sum).
__device__ __forceinline__ void softmax_commit(float2 ms, CycleCtl* ctl) {
    const float M = ms.x, S = ms.y;
    ctl->ll_max = M;
    ctl->ll_sumexp = S;
    const int ok = (S > 0.0f && isfinite(S)) ? 1 : 0;
    ctl->weights_valid = ok;
    ctl->wmode = ok ? WMODE_LL : WMODE_UNIFORM;
}

// Softmax partial of one block (two log-likelihoods per thread) + the
// last-block combine into M and S.
__device__ __forceinline__ void softmax_partials(float acc0, bool v0,
                                                 float acc1, bool v1,
                                                 float2* part,
                                                 unsigned* done,
                                                 CycleCtl* ctl) {
    __shared__ bool s_last;
    const float2 pb = block_softmax_partial(acc0, v0, acc1, v1);
    if (threadIdx.x == 0) {
        part[blockIdx.x] = pb;
        __threadfence();
        s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    const float2 ms = softmax_combine(part, gridDim.x);
    if (threadIdx.x == 0) {
        softmax_commit(ms, ctl);
        *done = 0u;
    }
}

// The combine of a sharded filter, once every rank's block partials are in
// part[0, G): one block, the same combine as the last block above, so M and
// S equal the unsharded filter's bit for bit.
__global__ void __launch_bounds__(kWThreads) k_softmax_combine(const float2* part, int G,
                                                              CycleCtl* ctl) {
    const float2 ms = softmax_combine(part, G);
    if (threadIdx.x == 0) softmax_commit(ms, ctl);
}

// Two particles per thread (i and i + kWThreads): every staged observation
// read from shared memory serves both.  Five 128-thread blocks per SM (84
// registers, no spills; 20 warps): measured 1.4 % faster than six (77
// registers) and faster than four, seven or eight.
// kShard: one rank's slice of a sharded filter; block b of the launch is
// block block0 + b of the whole cloud, and the block partials are left for
// the combine that follows the exchange (k_softmax_combine).
template <bool kPredict, bool kShard>
__global__ void __launch_bounds__(kWThreads, 5)
    k_weight(PlaneSet ps, int n, uint64_t seed, PredictArgs pa,
             const CObservation* __restrict__ obs, int nobs,
             const float* __restrict__ lm, int lm_count, float sigma_r,
             float sigma_b, float gate, float* __restrict__ ll,
             float2* part, unsigned* done, CycleCtl* ctl, int use_packed,
             const CycleArgs* ca, int block0) {
    pdl_wait();
    if (ca) {  // graph replay: this cycle's values
        pa = ca->pa;
        obs = ca->obs;
        nobs = ca->nobs;
    }
    const Planes s = pick_planes(ps, ctl->live);
    const int blk = kShard ? (int)blockIdx.x + block0 : (int)blockIdx.x;
    const int i0 = blk * (2 * kWThreads) + threadIdx.x;
    const int i1 = i0 + kWThreads;
    const bool v0 = i0 < n, v1 = i1 < n;
    float3 p0 = make_float3(0.f, 0.f, 0.f), p1 = p0;
    Quat q0 = {1.f, 0.f, 0.f, 0.f}, q1 = q0;
    if (v0) {
        load_pose(s, i0, p0, q0);
        if (kPredict) {
            apply_predict(pa, seed, i0, p0, q0);
            store_pose(s, i0, p0, q0);
        }
    }
    if (v1) {
        load_pose(s, i1, p1, q1);
        if (kPredict) {
            apply_predict(pa, seed, i1, p1, q1);
            store_pose(s, i1, p1, q1);
        }
    }
    float acc0, acc1;
    weight_two(obs, nobs, lm, lm_count, sigma_r, sigma_b, gate, p0, q0, p1, q1,
               use_packed, acc0, acc1);
    if (v0) ll[i0] = acc0;
    if (v1) ll[i1] = acc1;
    if (kShard) {
        const float2 pb = block_softmax_partial(acc0, v0, acc1, v1);
        if (threadIdx.x == 0) part[blk] = pb;
    } else {
        softmax_partials(acc0, v0, acc1, v1, part, done, ctl);
    }
}

}  // namespace

int launch_reinit(PfHandle* h, const float p0[3], const float q0[4],
                  const float pstd[3], const float rstd[3]) {
    const int grid = ceil_div(h->n, kThreads);
    KernelScope ks(h, KK_REINIT);
    k_reinit<<<grid, kThreads, 0, h->stream>>>(
        plane_set(h), h->n, h->seed, h->gen, make_float3(p0[0], p0[1], p0[2]),
        Quat{q0[0], q0[1], q0[2], q0[3]},
        make_float3(pstd[0], pstd[1], pstd[2]),
        make_float3(rstd[0], rstd[1], rstd[2]), h->d_ctl);
    PFB_KL();
    return 0;
}

int launch_reinit_poses(PfHandle* h, const float* d_poses, int k, float z,
                        const float pstd[3], const float rstd[3]) {
    const int grid = ceil_div(h->n, kThreads);
    KernelScope ks(h, KK_REINIT);
    k_reinit_poses<<<grid, kThreads, 0, h->stream>>>(
        plane_set(h), h->n, h->seed, h->gen, d_poses, k, z,
        make_float3(pstd[0], pstd[1], pstd[2]),
        make_float3(rstd[0], rstd[1], rstd[2]), h->d_ctl);
    PFB_KL();
    return 0;
}

int launch_predict(PfHandle* h, const PredictArgs& pa) {
    const int grid = ceil_div(h->n, kThreads);
    KernelScope ks(h, KK_PREDICT);
    k_predict<<<grid, kThreads, 0, h->stream>>>(plane_set(h), h->n, h->seed,
                                                pa, h->d_ctl);
    PFB_KL();
    return 0;
}

int launch_weight(PfHandle* h, const PredictArgs& pa, const CObservation* d_obs,
                  int nobs, float sigma_r, float sigma_b, float gate,
                  const CycleArgs* dargs) {
    const int grid = ceil_div(h->n, 2 * kWThreads);
    float2* part = reinterpret_cast<float2*>(h->d_part);
    KernelScope ks(h, KK_WEIGHT);
    if (pa.enabled) {
        PFB_CK(launch_pdl(k_weight<true, false>, grid, kWThreads, 0, h->stream, plane_set(h),
                          h->n, h->seed, pa, d_obs, nobs, h->d_lm, h->lm_count,
                          sigma_r, sigma_b, gate, h->d_ll, part, h->d_done + 0,
                          h->d_ctl, h->weight_variant == 0 ? 1 : 0, dargs, 0));
    } else {
        PFB_CK(launch_pdl(k_weight<false, false>, grid, kWThreads, 0, h->stream, plane_set(h),
                          h->n, h->seed, pa, d_obs, nobs, h->d_lm, h->lm_count,
                          sigma_r, sigma_b, gate, h->d_ll, part, h->d_done + 0,
                          h->d_ctl, h->weight_variant == 0 ? 1 : 0, dargs, 0));
    }
    PFB_KL();
    h->prefix_valid = false;
    return 0;
}

// One rank's slice of a sharded filter: particles [rank * chunk,
// min((rank + 1) * chunk, n)), predicted and weighted; their block partials
// land at their global block index of d_part (float2 per 256 particles) for
// the exchange.
int launch_weight_shard(PfHandle* h, const PredictArgs& pa, const CObservation* d_obs,
                        int nobs, float sigma_r, float sigma_b, float gate) {
    const long long first = (long long)h->shard_rank * h->shard_chunk;
    const long long last = std::min<long long>(first + h->shard_chunk, h->n);
    if (last <= first) return 0;  // a rank past the end of the cloud
    const int block0 = (int)(first / (2 * kWThreads));
    const int grid = (int)ceil_div_ll(last - first, 2 * kWThreads);
    float2* part = reinterpret_cast<float2*>(h->d_part);
    KernelScope ks(h, KK_WEIGHT);
    PFB_CK(launch_pdl(k_weight<true, true>, grid, kWThreads, 0, h->stream, plane_set(h), h->n,
                      h->seed, pa, d_obs, nobs, h->d_lm, h->lm_count, sigma_r, sigma_b, gate,
                      h->d_ll, part, h->d_done + 0, h->d_ctl,
                      h->weight_variant == 0 ? 1 : 0, (const CycleArgs*)nullptr, block0));
    PFB_KL();
    h->prefix_valid = false;
    return 0;
}

// The softmax of a sharded filter over all ceil(n / 256) block partials.
int launch_softmax_combine(PfHandle* h) {
    const int G = (int)ceil_div_ll(h->n, 2 * kWThreads);
    KernelScope ks(h, KK_WEIGHT);
    k_softmax_combine<<<1, kWThreads, 0, h->stream>>>(
        reinterpret_cast<const float2*>(h->d_part), G, h->d_ctl);
    PFB_KL();
    h->prefix_valid = false;
    return 0;
}

}  // namespace pfb
