// pf_abi.cu — the pfc_* C-ABI: handle lifecycle, host<->device plumbing and
// the scheduling that keeps the drop-in call sequence of the Rust
// CudaBackend (crates/pf_core/src/cuda.rs) to one host sync per estimate.
//
// Scheduling on the handle's private stream:
//   pfc_predict   records the odometry; the motion update runs fused into the
//                 next weighting pass (or alone, when anything else needs the
//                 cloud first).
//   pfc_weight    fused predict + weight + softmax partials, then the estimate
//                 pass, the device Markley mean and the covariance pass around
//                 that mean are queued speculatively, followed by one copy of
//                 the control block to pinned host memory.
//   pfc_est_sums  waits for that copy.
//   pfc_covs      returns the speculative covariances when the caller's f32
//                 means equal the ones the device used (the Rust caller passes
//                 exactly (float) of the returned sums and of its Markley
//                 mean); otherwise it runs the covariance pass with the
//                 caller's means.
//   pfc_resample  fixed-point scan + merge-path gather + injection, then the
//                 speculative estimate again.
#include <limits.h>
#include <math.h>
#include <stdarg.h>
#include <stdlib.h>
#include <string.h>

#include <algorithm>
#include <new>
#include <vector>

#include "pf_internal.h"

namespace pfb {

static thread_local char t_err[512] = "";

void set_error(const char* fmt, ...) {
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(t_err, sizeof(t_err), fmt, ap);
    va_end(ap);
    fprintf(stderr, "%s\n", t_err);
}

void clear_error() { t_err[0] = '\0'; }

// Drain recorded event pairs into the per-kind totals (waits for them).
static void prof_drain(PfHandle* h) {
    PfProfiler& p = h->prof;
    for (int k = 0; k < p.used; ++k) {
        float ms = 0.f;
        if (cudaEventSynchronize(p.ev[k][1]) == cudaSuccess &&
            cudaEventElapsedTime(&ms, p.ev[k][0], p.ev[k][1]) == cudaSuccess) {
            p.ms[p.kind[k]] += ms;
            p.count[p.kind[k]] += 1;
        }
    }
    p.used = 0;
}

void prof_drain_public(PfHandle* h) { prof_drain(h); }

void prof_begin(PfHandle* h, int kind) {
    h->stats.launches += 1;
    PfProfiler& p = h->prof;
    if (!p.on) return;
    if (p.used == PfProfiler::kPool) prof_drain(h);
    if (!p.ev[p.used][0]) {
        cudaEventCreate(&p.ev[p.used][0]);
        cudaEventCreate(&p.ev[p.used][1]);
    }
    p.kind[p.used] = kind;
    cudaEventRecord(p.ev[p.used][0], h->stream);
}

void prof_end(PfHandle* h, int kind) {
    (void)kind;
    PfProfiler& p = h->prof;
    if (!p.on) return;
    cudaEventRecord(p.ev[p.used][1], h->stream);
    p.used += 1;
}

namespace {

constexpr int kThreads = 256;

PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__global__ void k_ctl_reset(CycleCtl* ctl, int first) {
    unsigned long long lcg = first ? 0x243F6A8885A308D3ull : ctl->lcg;
    memset(ctl, 0, sizeof(CycleCtl));
    ctl->lcg = lcg;
    ctl->wmode = WMODE_UNIFORM;
    ctl->live = 0;
}

__global__ void k_set_wmode(CycleCtl* ctl, int mode) { ctl->wmode = mode; }

__global__ void k_pack(PlaneSet ps, int n, float* pos3, float* quat4,
                       const CycleCtl* ctl) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const Planes s = pick_planes(ps, ctl->live);
    pos3[3 * i] = s.px[i];
    pos3[3 * i + 1] = s.py[i];
    pos3[3 * i + 2] = s.pz[i];
    quat4[4 * i] = s.qw[i];
    quat4[4 * i + 1] = s.qx[i];
    quat4[4 * i + 2] = s.qy[i];
    quat4[4 * i + 3] = s.qz[i];
}

__global__ void k_unpack(PlaneSet ps, int n, const float* pos3,
                         const float* quat4, const CycleCtl* ctl) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const Planes s = pick_planes(ps, ctl->live);
    s.px[i] = pos3[3 * i];
    s.py[i] = pos3[3 * i + 1];
    s.pz[i] = pos3[3 * i + 2];
    s.qw[i] = quat4[4 * i];
    s.qx[i] = quat4[4 * i + 1];
    s.qy[i] = quat4[4 * i + 2];
    s.qz[i] = quat4[4 * i + 3];
}

PfHandle* as_pf(void* h) { return static_cast<PfHandle*>(h); }

void drop_cycle_graph(PfHandle* h) {
    if (h->cyc_exec) cudaGraphExecDestroy(h->cyc_exec);
    if (h->cyc_graph) cudaGraphDestroy(h->cyc_graph);
    h->cyc_exec = nullptr;
    h->cyc_graph = nullptr;
}

void free_particles(PfHandle* h) {
    drop_cycle_graph(h);
    cudaFree(h->d_state[0]);
    cudaFree(h->d_state[1]);
    cudaFree(h->d_ll);
    cudaFree(h->d_w);
    cudaFree(h->d_anc);
    cudaFree(h->d_wprefix);
    cudaFree(h->d_marker);
    cudaFree(h->d_inj_cnt);
    cudaFree(h->d_inj_bucket);
    cudaFree(h->d_part);
    cudaFree(h->d_part_u64);
    cudaFree(h->d_stage);
    h->d_state[0] = h->d_state[1] = nullptr;
    h->d_ll = h->d_w = nullptr;
    h->d_anc = nullptr;
    h->d_wprefix = nullptr;
    h->d_marker = nullptr;
    h->d_inj_cnt = nullptr;
    h->d_inj_bucket = nullptr;
    h->inj_cap = 0;
    h->d_part = nullptr;
    h->d_part_u64 = nullptr;
    h->d_stage = nullptr;
    h->n = 0;
}

PredictArgs pending_args(const PfHandle* h) {
    PredictArgs pa{};
    pa.enabled = h->pending_predict ? 1 : 0;
    pa.gen = h->pending_gen;
    for (int k = 0; k < 3; ++k) {
        pa.t[k] = h->pending_odom.t[k];
        pa.tstd[k] = h->pending_odom.tstd[k];
        pa.rstd[k] = h->pending_odom.rstd[k];
    }
    for (int k = 0; k < 4; ++k) pa.q[k] = h->pending_odom.q[k];
    return pa;
}

// Run a deferred predict on its own when the next operation is not a
// weighting pass.
int flush_predict(PfHandle* h) {
    if (!h->pending_predict) return 0;
    PredictArgs pa = pending_args(h);
    h->pending_predict = false;
    return launch_predict(h, pa);
}

int device_error(PfHandle* h) {
    if (h->h_ctl->err & ERR_SPIN_TIMEOUT) {
        set_error("pf_b200: a device wait timed out");
        return -1;
    }
    return 0;
}

// Queue estimate pass 1 + Markley (unless a fused resample already did) +
// speculative covariance pass + the copy of the control block.
// sq_from_ess: queued right after the weight pass (k_ess), whose sum w^2 the
// estimate reports; skip_ratio: the caller's resampling rule (ess hint).
int queue_estimate(PfHandle* h, bool sums_done = false, double skip_ratio = 0.0,
                   bool sq_from_ess = false) {
    if (!sums_done && launch_est_sums(h, sq_from_ess, skip_ratio)) return -1;
    if (launch_covs(h, false, nullptr, nullptr, false, skip_ratio)) return -1;
    PFB_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(CycleCtl),
                           cudaMemcpyDeviceToHost, h->stream));
    h->stats.d2h_bytes += sizeof(CycleCtl);
    PFB_CK(cudaEventRecord(h->est_ev, h->stream));
    h->est_inflight = true;
    h->est_valid = false;
    return 0;
}

int wait_estimate(PfHandle* h) {
    if (!h->est_inflight) return 0;
    PFB_CK(cudaEventSynchronize(h->est_ev));
    h->stats.host_syncs += 1;
    h->est_inflight = false;
    h->est_valid = true;
    return device_error(h);
}

// Copy nobs observations into the next pinned ring slot and queue the
// transfer to the device buffer.
int stage_observations(PfHandle* h, const CObservation* obs, int nobs) {
    const int slot = h->ring_pos;
    h->ring_pos = (h->ring_pos + 1) % PfHandle::kRing;
    PFB_CK(cudaEventSynchronize(h->ring_ev[slot]));
    CObservation* dst = h->h_obs_ring + (size_t)slot * h->cap_obs;
    memcpy(dst, obs, (size_t)nobs * sizeof(CObservation));
    PFB_CK(cudaMemcpyAsync(h->d_obs, dst, (size_t)nobs * sizeof(CObservation),
                           cudaMemcpyHostToDevice, h->stream));
    h->stats.h2d_bytes += (size_t)nobs * sizeof(CObservation);
    PFB_CK(cudaEventRecord(h->ring_ev[slot], h->stream));
    return 0;
}

int set_wmode(PfHandle* h, int mode) {
    KernelScope ks(h, KK_MISC);
    k_set_wmode<<<1, 1, 0, h->stream>>>(h->d_ctl, mode);
    PFB_KL();
    h->prefix_valid = false;
    return 0;
}

int ensure_stage(PfHandle* h) {
    if (h->d_stage) return 0;
    PFB_CK(cudaMalloc((void**)&h->d_stage, (size_t)7 * h->n * sizeof(float)));
    return 0;
}

bool valid_handle(PfHandle* h) { return h != nullptr && h->n > 0; }

// Everything a captured cycle depends on besides the per-cycle values.
void cycle_graph_key(const PfHandle* h, const PfcCycleParams* prm, long long k[12]) {
    auto f2l = [](float v) { long long r = 0; memcpy(&r, &v, sizeof v); return r; };
    long long e = 0;
    memcpy(&e, &prm->resample_ess_ratio, sizeof e);
    k[0] = h->n;
    k[1] = (long long)(uintptr_t)h->d_state[0];
    k[2] = (long long)(uintptr_t)h->d_lm;
    k[3] = h->lm_count;
    k[4] = f2l(prm->sigma_r);
    k[5] = f2l(prm->sigma_b);
    k[6] = f2l(prm->gate);
    k[7] = e;
    k[8] = f2l(prm->random_inject_ratio);
    k[9] = h->weight_variant;
    k[10] = h->record_anc ? 1 : 0;
    k[11] = 1;
}

int enqueue_cycle(PfHandle* h, const PredictArgs& pa, const CObservation* obs_dev,
                  int nobs, const PfcCycleParams* prm, const CycleArgs* dargs);

// A fused cycle replayed from a CUDA graph (same kernels and arguments as the
// direct launches; the per-cycle values come from d_cargs).  Used when there
// are observations and per-kernel profiling is off.
int run_cycle_graph(PfHandle* h, const PfcOdom* odom, const CObservation* obs_dev,
                    int nobs, const PfcCycleParams* prm) {
    h->gen++;
    const int slot = h->cargs_pos;
    h->cargs_pos = (h->cargs_pos + 1) % PfHandle::kRing;
    PFB_CK(cudaEventSynchronize(h->cargs_ev[slot]));
    CycleArgs& a = h->h_cargs[slot];
    memset(&a, 0, sizeof a);
    a.pa.enabled = 1;
    a.pa.gen = h->gen;
    for (int k = 0; k < 3; ++k) {
        a.pa.t[k] = odom->t[k];
        a.pa.tstd[k] = odom->tstd[k];
        a.pa.rstd[k] = odom->rstd[k];
    }
    for (int k = 0; k < 4; ++k) a.pa.q[k] = odom->q[k];
    a.obs = obs_dev;
    a.nobs = nobs;
    a.gen = h->gen;
    const int kinj = (prm->random_inject_ratio > 0.f)
                         ? std::min(h->n, (int)(prm->random_inject_ratio * (float)h->n))
                         : 0;
    // buffers the captured kernels use are allocated before the capture
    if (ensure_inject_buckets(h, kinj)) return -1;
    PFB_CK(cudaMemcpyAsync(h->d_cargs, &a, sizeof(CycleArgs), cudaMemcpyHostToDevice,
                           h->stream));
    PFB_CK(cudaEventRecord(h->cargs_ev[slot], h->stream));
    h->stats.h2d_bytes += sizeof(CycleArgs);
    long long key[12];
    cycle_graph_key(h, prm, key);
    if (h->cyc_exec && memcmp(key, h->graph_key, sizeof key) != 0) drop_cycle_graph(h);
    if (!h->cyc_exec) {
        const long long l0 = h->stats.launches;
        const size_t d0 = h->stats.d2h_bytes;
        PFB_CK(cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeThreadLocal));
        const int rc = enqueue_cycle(h, a.pa, obs_dev, nobs, prm, h->d_cargs);
        cudaGraph_t g = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &g);
        h->graph_kernels = (int)(h->stats.launches - l0);
        h->stats.launches = l0;
        h->stats.d2h_bytes = d0;
        if (rc || e != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            set_error("pf_b200: cycle graph capture failed: %s", cudaGetErrorString(e));
            return -1;
        }
        h->cyc_graph = g;
        PFB_CK(cudaGraphInstantiate(&h->cyc_exec, g, 0));
        memcpy(h->graph_key, key, sizeof key);
    }
    PFB_CK(cudaGraphLaunch(h->cyc_exec, h->stream));
    PFB_CK(cudaEventRecord(h->est_ev, h->stream));
    h->stats.launches += h->graph_kernels;
    h->stats.d2h_bytes += sizeof(CycleCtl);
    h->prefix_valid = false;
    h->anc_valid = true;
    h->est_inflight = true;
    h->est_valid = false;
    return 0;
}

// One fused cycle; obs_dev points at device-resident observations.
int run_cycle(PfHandle* h, const PfcOdom* odom, const CObservation* obs_dev,
              int nobs, const PfcCycleParams* prm) {
    if (flush_predict(h)) return -1;
    if (h->use_graph && nobs > 0 && !h->prof.on && h->d_cargs)
        return run_cycle_graph(h, odom, obs_dev, nobs, prm);
    h->gen++;
    PredictArgs pa{};
    pa.enabled = 1;
    pa.gen = h->gen;
    for (int k = 0; k < 3; ++k) {
        pa.t[k] = odom->t[k];
        pa.tstd[k] = odom->tstd[k];
        pa.rstd[k] = odom->rstd[k];
    }
    for (int k = 0; k < 4; ++k) pa.q[k] = odom->q[k];
    if (nobs <= 0) {
        if (launch_predict(h, pa)) return -1;
        if (set_wmode(h, WMODE_UNIFORM)) return -1;
    }
    if (enqueue_cycle(h, pa, obs_dev, nobs, prm, nullptr)) return -1;
    h->est_inflight = true;
    h->est_valid = false;
    return 0;
}

// The kernels of a cycle after the predict / weighting decision, then the copy
// of the control block.  With dargs (graph capture) the weighting pass runs
// and reads its per-cycle values from dargs.
int enqueue_cycle(PfHandle* h, const PredictArgs& pa, const CObservation* obs_dev,
                  int nobs, const PfcCycleParams* prm, const CycleArgs* dargs) {
    if (nobs > 0 &&
        launch_weight(h, pa, obs_dev, nobs, prm->sigma_r, prm->sigma_b, prm->gate,
                      dargs))
        return -1;
    if (launch_cycle_decide(h, prm->resample_ess_ratio)) return -1;
    // resample (when decided) fused with the estimate sums of the cycle's
    // final cloud, then its covariance pass and the output record
    if (launch_resample_est(h, prm->random_inject_ratio, true, false, 0.0, dargs))
        return -1;
    if (launch_covs(h, false, nullptr, nullptr, true)) return -1;
    PFB_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(CycleCtl),
                           cudaMemcpyDeviceToHost, h->stream));
    h->stats.d2h_bytes += sizeof(CycleCtl);
    // an event recorded inside a capture cannot be waited on afterwards: the
    // graph path records it after the launch
    if (!dargs) PFB_CK(cudaEventRecord(h->est_ev, h->stream));
    return 0;
}

int init_particles(PfHandle* h, int n, unsigned int seed, int n_pad);

int finish_cycle(PfHandle* h, double* est_out) {
    if (wait_estimate(h)) return -1;
    if (est_out) memcpy(est_out, h->h_ctl->out, sizeof(double) * PFC_EST_LEN);
    return 0;
}

}  // namespace
}  // namespace pfb

using namespace pfb;

extern "C" {

const char* pfc_last_error_message(void) { return t_err; }

int pfc_version(void) { return 100; }

int pfc_device_available(void) {
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev < 1) return 0;
    cudaDeviceProp prop{};
    if (cudaGetDeviceProperties(&prop, 0) != cudaSuccess) return 0;
    return prop.major >= 3 ? 1 : 0;
}

void* pfc_create(int cap_obs) {
    clear_error();
    PfHandle* h = new (std::nothrow) PfHandle();
    if (!h) return nullptr;
    if (cap_obs < 1 || cap_obs > 4096) cap_obs = 64;
    h->cap_obs = cap_obs;
    bool ok = false;
    do {
        if (cudaGetDevice(&h->dev) != cudaSuccess) break;
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_ctl, sizeof(CycleCtl)) != cudaSuccess) break;
        if (cudaMallocHost((void**)&h->h_ctl, sizeof(CycleCtl)) != cudaSuccess)
            break;
        memset(h->h_ctl, 0, sizeof(CycleCtl));
        if (cudaMalloc((void**)&h->d_done, 8 * sizeof(unsigned)) != cudaSuccess)
            break;
        if (cudaMemsetAsync(h->d_done, 0, 8 * sizeof(unsigned), h->stream) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_obs, (size_t)cap_obs * sizeof(CObservation)) !=
            cudaSuccess)
            break;
        h->d_obs_cap = cap_obs;
        if (cudaMallocHost((void**)&h->h_obs_ring,
                           (size_t)PfHandle::kRing * cap_obs *
                               sizeof(CObservation)) != cudaSuccess)
            break;
        bool ev_ok = true;
        for (int k = 0; k < PfHandle::kRing; ++k)
            ev_ok = ev_ok && cudaEventCreateWithFlags(&h->ring_ev[k],
                                                      cudaEventDisableTiming) ==
                                 cudaSuccess;
        if (!ev_ok) break;
        if (cudaEventCreateWithFlags(&h->est_ev, cudaEventDisableTiming) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_cargs, sizeof(CycleArgs)) != cudaSuccess ||
            cudaMallocHost((void**)&h->h_cargs,
                           PfHandle::kRing * sizeof(CycleArgs)) != cudaSuccess)
            break;
        for (int k = 0; k < PfHandle::kRing; ++k)
            ev_ok = ev_ok && cudaEventCreateWithFlags(&h->cargs_ev[k],
                                                      cudaEventDisableTiming) ==
                                 cudaSuccess;
        if (!ev_ok) break;
        k_ctl_reset<<<1, 1, 0, h->stream>>>(h->d_ctl, 1);
        if (cudaGetLastError() != cudaSuccess) break;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) break;
        ok = true;
    } while (0);
    if (!ok) {
        set_error("pf_b200: pfc_create failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
        pfc_destroy(h);
        return nullptr;
    }
    return h;
}

int pfc_destroy(void* hv) {
    PfHandle* h = as_pf(hv);
    if (!h) return 0;
    if (h->stream) cudaStreamSynchronize(h->stream);
    free_particles(h);
    cudaFree(h->d_ctl);
    cudaFreeHost(h->h_ctl);
    cudaFree(h->d_done);
    cudaFree(h->d_obs);
    cudaFreeHost(h->h_obs_ring);
    cudaFree(h->d_lm);
    cudaFree(h->d_cargs);
    cudaFreeHost(h->h_cargs);
    for (int k = 0; k < PfHandle::kRing; ++k) {
        if (h->ring_ev[k]) cudaEventDestroy(h->ring_ev[k]);
        if (h->cargs_ev[k]) cudaEventDestroy(h->cargs_ev[k]);
    }
    if (h->est_ev) cudaEventDestroy(h->est_ev);
    for (int k = 0; k < PfProfiler::kPool; ++k)
        for (int e = 0; e < 2; ++e)
            if (h->prof.ev[k][e]) cudaEventDestroy(h->prof.ev[k][e]);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

int pfc_init(void* hv, int n, unsigned int seed) {
    PfHandle* h = as_pf(hv);
    if (!h || n <= 0) return -1;
    h->shard_world = h->shard_rank = h->shard_chunk = 0;
    return init_particles(h, n, seed, (int)(ceil_div_ll(n, 1024) * 1024));
}

}  // extern "C"

namespace pfb {
namespace {

// Allocate and reset a cloud of n particles in planes of n_pad (a multiple
// of 1024, at least n).
int init_particles(PfHandle* h, int n, unsigned int seed, int n_pad) {
    PFB_CK(cudaStreamSynchronize(h->stream));
    free_particles(h);
    h->n = n;
    h->n_pad = n_pad;
    h->seed = seed ? (uint64_t)seed : 42ull;
    h->gen = 0;
    h->pending_predict = false;
    h->est_valid = h->est_inflight = false;
    h->anc_valid = false;
    h->prefix_valid = false;
    const size_t np = (size_t)h->n_pad;
    const int nprefix = ceil_div(n, kPrefixBlock);
    // doubles: the largest of the kernels' partial arrays (float2 softmax
    // partials of every 256-particle block of the planes included)
    const int part = std::max(std::max(2 * ceil_div(n, kThreads), resample_part_doubles(n)),
                              std::max(1184 * 16, n_pad / (2 * kWThreads)));
    PFB_CK(cudaMalloc((void**)&h->d_state[0], 7 * np * sizeof(float)));
    PFB_CK(cudaMalloc((void**)&h->d_state[1], 7 * np * sizeof(float)));
    PFB_CK(cudaMalloc((void**)&h->d_ll, np * sizeof(float)));
    PFB_CK(cudaMalloc((void**)&h->d_w, np * sizeof(float)));
    PFB_CK(cudaMalloc((void**)&h->d_part_u64,
                      2 * (size_t)std::max(nprefix, 1184) * sizeof(unsigned long long)));
    PFB_CK(cudaMalloc((void**)&h->d_anc, (size_t)n * sizeof(int)));
    PFB_CK(cudaMalloc((void**)&h->d_wprefix, (size_t)nprefix * sizeof(uint64_t)));
    PFB_CK(cudaMalloc((void**)&h->d_marker, np * sizeof(int)));
    PFB_CK(cudaMemsetAsync(h->d_marker, 0xFF, np * sizeof(int), h->stream));
    const int rtiles = resample_tiles(n);
    PFB_CK(cudaMalloc((void**)&h->d_inj_cnt, (size_t)rtiles * sizeof(int)));
    PFB_CK(cudaMemsetAsync(h->d_inj_cnt, 0, (size_t)rtiles * sizeof(int), h->stream));
    PFB_CK(cudaMalloc((void**)&h->d_part, (size_t)part * sizeof(double)));
    h->part_cap = part;
    PFB_CK(cudaMemsetAsync(h->d_state[0], 0, 7 * np * sizeof(float), h->stream));
    PFB_CK(cudaMemsetAsync(h->d_state[1], 0, 7 * np * sizeof(float), h->stream));
    PFB_CK(cudaMemsetAsync(h->d_ll, 0, np * sizeof(float), h->stream));
    PFB_CK(cudaMemsetAsync(h->d_done, 0, 8 * sizeof(unsigned), h->stream));
    h->inj_epoch = 0;
    k_ctl_reset<<<1, 1, 0, h->stream>>>(h->d_ctl, 0);
    PFB_KL();
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

}  // namespace
}  // namespace pfb

extern "C" {

int pfc_upload_landmarks(void* hv, const float* xyz, int count) {
    PfHandle* h = as_pf(hv);
    if (!h || !xyz || count < 0) return -1;
    // Table semantics of src/cuda/pf_kernels.cu:553-565: count 0 clears, the
    // valid-id bound only grows otherwise.
    if (count == 0) {
        h->lm_count = 0;
        return 0;
    }
    if (count > h->lm_cap) {
        PFB_CK(cudaStreamSynchronize(h->stream));
        cudaFree(h->d_lm);
        h->d_lm = nullptr;
        PFB_CK(cudaMalloc((void**)&h->d_lm, 3 * sizeof(float) * (size_t)count));
        h->lm_cap = count;
    }
    if (count > h->lm_count) h->lm_count = count;
    PFB_CK(cudaMemcpyAsync(h->d_lm, xyz, 3 * sizeof(float) * (size_t)count,
                           cudaMemcpyHostToDevice, h->stream));
    h->stats.h2d_bytes += 3 * sizeof(float) * (size_t)count;
    PFB_CK(cudaStreamSynchronize(h->stream));
    h->stats.host_syncs += 1;
    return 0;
}

int pfc_reinit(void* hv, float x, float y, float z, float qw, float qx,
               float qy, float qz, const float* pos_std, const float* rot_std) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !pos_std || !rot_std) return -1;
    h->pending_predict = false;  // the prior overwrites every pose
    h->gen++;
    const float p0[3] = {x, y, z}, q0[4] = {qw, qx, qy, qz};
    if (launch_reinit(h, p0, q0, pos_std, rot_std)) return -1;
    if (set_wmode(h, WMODE_UNIFORM)) return -1;
    h->est_valid = h->est_inflight = false;
    h->prefix_valid = false;
    return 0;
}

int pfc_reinit_poses(void* hv, const float* d_pose3k, int k, float z,
                     const float* pos_std, const float* rot_std) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !d_pose3k || k <= 0 || !pos_std || !rot_std)
        return -1;
    h->pending_predict = false;
    h->gen++;
    if (launch_reinit_poses(h, d_pose3k, k, z, pos_std, rot_std)) return -1;
    if (set_wmode(h, WMODE_UNIFORM)) return -1;
    h->est_valid = h->est_inflight = false;
    h->prefix_valid = false;
    return 0;
}

int pfc_predict(void* hv, float tx, float ty, float tz, float qw, float qx,
                float qy, float qz, const float* tstd, const float* rstd) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !tstd || !rstd) return -1;
    if (flush_predict(h)) return -1;
    h->gen++;
    h->pending_predict = true;
    h->pending_gen = h->gen;
    PfcOdom& o = h->pending_odom;
    o.t[0] = tx;
    o.t[1] = ty;
    o.t[2] = tz;
    o.q[0] = qw;
    o.q[1] = qx;
    o.q[2] = qy;
    o.q[3] = qz;
    for (int k = 0; k < 3; ++k) {
        o.tstd[k] = tstd[k];
        o.rstd[k] = rstd[k];
    }
    h->est_valid = false;
    return 0;
}

int pfc_weight(void* hv, const CObservation* obs, int nobs, float sigma_r,
               float sigma_b, float gate) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h)) return -1;
    if (nobs > h->cap_obs) nobs = h->cap_obs;
    if (nobs <= 0 || !obs) {
        if (flush_predict(h)) return -1;
        if (set_wmode(h, WMODE_UNIFORM)) return -1;
        return queue_estimate(h, false, h->ess_hint);
    }
    if (stage_observations(h, obs, nobs)) return -1;
    PredictArgs pa = pending_args(h);
    h->pending_predict = false;
    if (launch_weight(h, pa, h->d_obs, nobs, sigma_r, sigma_b, gate)) return -1;
    // materialise the weights with the resampler's prefixes now: the estimate
    // pass then reads them instead of re-deriving them from ll
    if (launch_weight_prefix(h, false, 0.0)) return -1;
    return queue_estimate(h, false, h->ess_hint, true);
}

int pfc_set_ess_hint(void* hv, double resample_ess_ratio) {
    PfHandle* h = as_pf(hv);
    if (!h || !(resample_ess_ratio == resample_ess_ratio)) return -1;
    h->ess_hint = resample_ess_ratio > 0.0 ? resample_ess_ratio : 0.0;
    return 0;
}

int pfc_resample(void* hv, float random_inject_ratio) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h)) return -1;
    if (flush_predict(h)) return -1;
    if (launch_resample_est(h, random_inject_ratio, false, false, 0.0)) return -1;
    return queue_estimate(h, true);
}

int pfc_resample_u01(void* hv, double u01, float random_inject_ratio) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !(u01 >= 0.0) || !(u01 < 1.0)) return -1;
    if (flush_predict(h)) return -1;
    if (launch_resample_est(h, random_inject_ratio, false, true, u01)) return -1;
    return queue_estimate(h, true);
}

int pfc_est_sums(void* hv, double* out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !out) return -1;
    if (h->pending_predict || (!h->est_inflight && !h->est_valid)) {
        if (flush_predict(h)) return -1;
        if (queue_estimate(h)) return -1;
    }
    if (wait_estimate(h)) return -1;
    if (h->h_ctl->est_partial) {
        // the estimate after the last weighting reported only sum w^2 (ess
        // hint); the cloud and its weights are unchanged since, so the full
        // pass reports the same sum w^2 (the weight pass's).  The covariance
        // pass follows, as with every queued estimate, so the cached
        // covariances match the cached mean.
        if (launch_est_sums(h, true, 0.0)) return -1;
        if (launch_covs(h, false, nullptr, nullptr, false)) return -1;
        PFB_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(CycleCtl),
                               cudaMemcpyDeviceToHost, h->stream));
        PFB_CK(cudaStreamSynchronize(h->stream));
        h->stats.d2h_bytes += sizeof(CycleCtl);
        h->stats.host_syncs += 1;
        if (device_error(h)) return -1;
    }
    memcpy(out, h->h_ctl->est, sizeof(double) * kEstN);
    return 0;
}

int pfc_est_ess(void* hv, double* ess) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !ess) return -1;
    if (h->pending_predict || (!h->est_inflight && !h->est_valid)) {
        if (flush_predict(h)) return -1;
        if (queue_estimate(h)) return -1;
    }
    if (wait_estimate(h)) return -1;
    *ess = h->h_ctl->ess;
    return 0;
}

int pfc_covs(void* hv, float mx, float my, float mz, float qw, float qx,
             float qy, float qz, double* out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !out) return -1;
    if (flush_predict(h)) return -1;
    if (wait_estimate(h)) return -1;
    const CycleCtl* c = h->h_ctl;
    const bool hit = h->est_valid && c->cov_mean_p[0] == mx &&
                     c->cov_mean_p[1] == my && c->cov_mean_p[2] == mz &&
                     c->cov_mean_q[0] == qw && c->cov_mean_q[1] == qx &&
                     c->cov_mean_q[2] == qy && c->cov_mean_q[3] == qz;
    if (!hit) {
        const float mp[3] = {mx, my, mz}, mq[4] = {qw, qx, qy, qz};
        if (launch_covs(h, true, mp, mq, false)) return -1;
        PFB_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(CycleCtl),
                               cudaMemcpyDeviceToHost, h->stream));
        PFB_CK(cudaStreamSynchronize(h->stream));
        h->stats.d2h_bytes += sizeof(CycleCtl);
        h->stats.host_syncs += 1;
        if (device_error(h)) return -1;
    }
    memcpy(out, h->h_ctl->covs, sizeof(double) * kCovN);
    return 0;
}

int pfc_snapshot(void* hv, float* pos, float* quat) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !pos || !quat) return -1;
    if (flush_predict(h)) return -1;
    if (ensure_stage(h)) return -1;
    float* p3 = h->d_stage;
    float* q4 = h->d_stage + 3 * (size_t)h->n;
    {
        KernelScope ks(h, KK_MISC);
        k_pack<<<ceil_div(h->n, kThreads), kThreads, 0, h->stream>>>(
            plane_set(h), h->n, p3, q4, h->d_ctl);
    }
    PFB_KL();
    h->stats.d2h_bytes += 7 * sizeof(float) * (size_t)h->n;
    h->stats.host_syncs += 1;
    PFB_CK(cudaMemcpyAsync(pos, p3, 3 * sizeof(float) * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaMemcpyAsync(quat, q4, 4 * sizeof(float) * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

// ------------------------------------------------------------- additive

int pfc_cycle(void* hv, const PfcOdom* odom, const CObservation* obs, int nobs,
              const PfcCycleParams* prm, double* est_out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !odom || !prm) return -1;
    if (nobs > h->cap_obs) nobs = h->cap_obs;
    if (!obs) nobs = 0;
    if (nobs > 0 && stage_observations(h, obs, nobs)) return -1;
    if (run_cycle(h, odom, h->d_obs, nobs, prm)) return -1;
    return finish_cycle(h, est_out);
}

int pfc_cycle_device(void* hv, const PfcOdom* odom, const void* d_obs, int nobs,
                     const PfcCycleParams* prm, double* est_out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !odom || !prm) return -1;
    if (nobs > h->cap_obs) nobs = h->cap_obs;
    if (!d_obs) nobs = 0;
    if (run_cycle(h, odom, static_cast<const CObservation*>(d_obs), nobs, prm))
        return -1;
    if (!est_out) return 0;
    return finish_cycle(h, est_out);
}

int pfc_set_graph(void* hv, int on) {
    PfHandle* h = as_pf(hv);
    if (!h) return -1;
    h->use_graph = on != 0;
    if (!h->use_graph) drop_cycle_graph(h);
    return 0;
}

int pfc_cycle_result(void* hv, double* est_out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !est_out) return -1;
    return finish_cycle(h, est_out);
}

// ---------------------------------------------------------- sharded filter

int pfc_shard_init(void* hv, int n, int world, int rank, unsigned int seed) {
    PfHandle* h = as_pf(hv);
    if (!h || n <= 0 || world < 1 || rank < 0 || rank >= world) {
        set_error("pf_b200: pfc_shard_init: bad arguments (n %d, world %d, rank %d)", n,
                  world, rank);
        return -1;
    }
    const long long chunk = ceil_div_ll(ceil_div_ll(n, world), kPrefixBlock) * kPrefixBlock;
    const long long n_pad = std::max<long long>(ceil_div_ll(n, 1024) * 1024, chunk * world);
    if (n_pad > (long long)INT_MAX / 7) {
        set_error("pf_b200: pfc_shard_init: %d particles over %d ranks too large", n, world);
        return -1;
    }
    h->shard_world = world;
    h->shard_rank = rank;
    h->shard_chunk = (int)chunk;
    h->shard_nobs = 0;
    if (init_particles(h, n, seed, (int)n_pad)) {
        h->shard_world = h->shard_rank = h->shard_chunk = 0;
        return -1;
    }
    return 0;
}

int pfc_shard_layout(void* hv, int* chunk, int* n_pad) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || h->shard_world < 1) return -1;
    if (chunk) *chunk = h->shard_chunk;
    if (n_pad) *n_pad = h->n_pad;
    return 0;
}

int pfc_shard_weight(void* hv, const PfcOdom* odom, const CObservation* obs, int nobs,
                     const PfcCycleParams* prm) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !odom || !prm) return -1;
    if (h->shard_world < 1) {
        set_error("pf_b200: pfc_shard_weight: not a shard handle (pfc_shard_init)");
        return -1;
    }
    if (nobs > h->cap_obs) nobs = h->cap_obs;
    if (!obs || nobs < 0) nobs = 0;
    if (flush_predict(h)) return -1;
    if (nobs > 0 && stage_observations(h, obs, nobs)) return -1;
    h->gen++;
    PredictArgs pa{};
    pa.enabled = 1;
    pa.gen = h->gen;
    for (int k = 0; k < 3; ++k) {
        pa.t[k] = odom->t[k];
        pa.tstd[k] = odom->tstd[k];
        pa.rstd[k] = odom->rstd[k];
    }
    for (int k = 0; k < 4; ++k) pa.q[k] = odom->q[k];
    if (launch_weight_shard(h, pa, h->d_obs, nobs, prm->sigma_r, prm->sigma_b, prm->gate))
        return -1;
    h->shard_nobs = nobs;
    h->est_valid = false;
    return 0;
}

int pfc_shard_views(void* hv, float** planes7, float** ll, float** part) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !planes7 || h->shard_world < 1) return -1;
    PFB_CK(cudaStreamSynchronize(h->stream));
    int live = 0;
    PFB_CK(cudaMemcpy(&live, &h->d_ctl->live, sizeof(int), cudaMemcpyDeviceToHost));
    const Planes s = h->planes(live ? 1 : 0);
    float* const p[7] = {s.px, s.py, s.pz, s.qw, s.qx, s.qy, s.qz};
    for (int k = 0; k < 7; ++k) planes7[k] = p[k];
    if (ll) *ll = h->d_ll;
    if (part) *part = reinterpret_cast<float*>(h->d_part);
    return 0;
}

int pfc_shard_finish(void* hv, const PfcCycleParams* prm, double* est_out) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !prm) return -1;
    if (h->shard_world < 1) {
        set_error("pf_b200: pfc_shard_finish: not a shard handle (pfc_shard_init)");
        return -1;
    }
    // the cycle without observations keeps uniform weights, as pfc_cycle's
    if (h->shard_nobs > 0 ? launch_softmax_combine(h) : set_wmode(h, WMODE_UNIFORM))
        return -1;
    const PredictArgs none{};
    if (enqueue_cycle(h, none, nullptr, 0, prm, nullptr)) return -1;
    h->est_inflight = true;
    h->est_valid = false;
    return finish_cycle(h, est_out);
}

void* pfc_stream(void* hv) {
    PfHandle* h = as_pf(hv);
    return h ? (void*)h->stream : nullptr;
}

int pfc_size(void* hv) {
    PfHandle* h = as_pf(hv);
    return h ? h->n : -1;
}

int pfc_get_weights(void* hv, float* w) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !w) return -1;
    if (launch_materialize_weights(h)) return -1;
    PFB_CK(cudaMemcpyAsync(w, h->d_w, sizeof(float) * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_get_ll(void* hv, float* ll) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !ll) return -1;
    PFB_CK(cudaMemcpyAsync(ll, h->d_ll, sizeof(float) * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_set_state(void* hv, const float* pos3n, const float* quat4n,
                  const float* w) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !pos3n || !quat4n) return -1;
    h->pending_predict = false;
    if (ensure_stage(h)) return -1;
    const size_t n = (size_t)h->n;
    float* p3 = h->d_stage;
    float* q4 = h->d_stage + 3 * n;
    PFB_CK(cudaMemcpyAsync(p3, pos3n, 3 * sizeof(float) * n,
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaMemcpyAsync(q4, quat4n, 4 * sizeof(float) * n,
                           cudaMemcpyHostToDevice, h->stream));
    KernelScope ks(h, KK_MISC);
    k_unpack<<<ceil_div(h->n, kThreads), kThreads, 0, h->stream>>>(
        plane_set(h), h->n, p3, q4, h->d_ctl);
    PFB_KL();
    if (w) {
        // The fixed-point resampler needs sum w < 4: rescale weights whose
        // sum lies outside [0.5, 2] to sum 1 (resampling is scale-invariant).
        double sum = 0.0;
        bool bad = false;
        for (size_t i = 0; i < n; ++i) {
            if (!(w[i] >= 0.0f) || !std::isfinite(w[i])) bad = true;
            sum += (double)w[i];
        }
        std::vector<float> tmp;
        const float* src = w;
        if (!bad && sum > 0.0 && (sum < 0.5 || sum > 2.0)) {
            tmp.resize(n);
            for (size_t i = 0; i < n; ++i) tmp[i] = (float)((double)w[i] / sum);
            src = tmp.data();
        }
        PFB_CK(cudaMemcpyAsync(h->d_w, src, sizeof(float) * n,
                               cudaMemcpyHostToDevice, h->stream));
        PFB_CK(cudaStreamSynchronize(h->stream));
        if (set_wmode(h, WMODE_STORED)) return -1;
    } else {
        if (set_wmode(h, WMODE_UNIFORM)) return -1;
    }
    PFB_CK(cudaStreamSynchronize(h->stream));
    h->est_valid = h->est_inflight = false;
    h->prefix_valid = false;
    return 0;
}

int pfc_record_ancestors(void* hv, int on) {
    PfHandle* h = as_pf(hv);
    if (!h) return -1;
    h->record_anc = on != 0;
    return 0;
}

int pfc_get_ancestors(void* hv, int* anc) {
    PfHandle* h = as_pf(hv);
    if (!valid_handle(h) || !anc) return -1;
    if (!h->anc_valid) {
        set_error("pf_b200: no resample has run on this particle set");
        return -1;
    }
    PFB_CK(cudaStreamSynchronize(h->stream));
    PFB_CK(cudaMemcpyAsync(anc, h->d_anc, sizeof(int) * (size_t)h->n,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_pick_from_cum(void* hv, const double* cum, int n, double u0,
                      double total, int* anc) {
    PfHandle* h = as_pf(hv);
    if (!h || !cum || !anc || n <= 0) return -1;
    double* d_cum = nullptr;
    int* d_anc = nullptr;
    int rc = -1;
    if (cudaMalloc((void**)&d_cum, sizeof(double) * (size_t)n) == cudaSuccess &&
        cudaMalloc((void**)&d_anc, sizeof(int) * (size_t)n) == cudaSuccess &&
        cudaMemcpyAsync(d_cum, cum, sizeof(double) * (size_t)n,
                        cudaMemcpyHostToDevice, h->stream) == cudaSuccess &&
        launch_pick_from_cum(h, d_cum, n, u0, total, d_anc) == 0 &&
        cudaMemcpyAsync(anc, d_anc, sizeof(int) * (size_t)n,
                        cudaMemcpyDeviceToHost, h->stream) == cudaSuccess &&
        cudaStreamSynchronize(h->stream) == cudaSuccess)
        rc = 0;
    if (rc) set_error("pf_b200: pfc_pick_from_cum failed");
    cudaFree(d_cum);
    cudaFree(d_anc);
    return rc;
}

int pfc_weight_div_check(void* hv, const float* e, const float* s, int n,
                         float* fast, float* ieee) {
    PfHandle* h = as_pf(hv);
    if (!h || !e || !s || !fast || !ieee || n <= 0) return -1;
    float* d = nullptr;
    const size_t bytes = sizeof(float) * (size_t)n;
    int rc = -1;
    if (cudaMalloc((void**)&d, 4 * bytes) == cudaSuccess &&
        cudaMemcpyAsync(d, e, bytes, cudaMemcpyHostToDevice, h->stream) == cudaSuccess &&
        cudaMemcpyAsync(d + n, s, bytes, cudaMemcpyHostToDevice, h->stream) == cudaSuccess &&
        launch_weight_div_check(h, d, d + n, n, d + 2 * (size_t)n, d + 3 * (size_t)n) == 0 &&
        cudaMemcpyAsync(fast, d + 2 * (size_t)n, bytes, cudaMemcpyDeviceToHost,
                        h->stream) == cudaSuccess &&
        cudaMemcpyAsync(ieee, d + 3 * (size_t)n, bytes, cudaMemcpyDeviceToHost,
                        h->stream) == cudaSuccess &&
        cudaStreamSynchronize(h->stream) == cudaSuccess)
        rc = 0;
    if (rc) set_error("pf_b200: pfc_weight_div_check failed");
    cudaFree(d);
    return rc;
}

int pfc_get_lcg(void* hv, unsigned long long* lcg) {
    PfHandle* h = as_pf(hv);
    if (!h || !lcg) return -1;
    PFB_CK(cudaMemcpyAsync(lcg, &h->d_ctl->lcg, sizeof(unsigned long long),
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_set_lcg(void* hv, unsigned long long lcg) {
    PfHandle* h = as_pf(hv);
    if (!h) return -1;
    PFB_CK(cudaMemcpyAsync(&h->d_ctl->lcg, &lcg, sizeof(unsigned long long),
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfc_set_weight_kernel(void* hv, int variant) {
    PfHandle* h = as_pf(hv);
    if (!h || variant < 0 || variant > 1) return -1;
    h->weight_variant = variant;
    return 0;
}

}  // extern "C"

extern "C" {

int pfc_get_stats(void* hv, PfcStats* out) {
    PfHandle* h = static_cast<PfHandle*>(hv);
    if (!h || !out) return -1;
    *out = h->stats;
    return 0;
}

int pfc_reset_stats(void* hv) {
    PfHandle* h = static_cast<PfHandle*>(hv);
    if (!h) return -1;
    h->stats = PfcStats{};
    return 0;
}

int pfc_profile(void* hv, int on) {
    PfHandle* h = static_cast<PfHandle*>(hv);
    if (!h) return -1;
    if (!on && h->prof.on) pfb::prof_drain_public(h);
    h->prof.on = on != 0;
    return 0;
}

int pfc_profile_read(void* hv, double* ms, long long* counts) {
    PfHandle* h = static_cast<PfHandle*>(hv);
    if (!h || !ms || !counts) return -1;
    pfb::prof_drain_public(h);
    for (int k = 0; k < KK_COUNT; ++k) {
        ms[k] = h->prof.ms[k];
        counts[k] = h->prof.count[k];
        h->prof.ms[k] = 0.0;
        h->prof.count[k] = 0;
    }
    return 0;
}

}  // extern "C"
