// pf_resample.cu — systematic resampling with an exact fixed-point scan.
//
// Specification (semantics of src/cuda/pf_kernels.cu:638-676 and
// crates/pf_core/src/cpu.rs:262-306, made exact and deterministic):
//   W_j   = round_nearest_even(w_j * 2^62)             (u64, w_j in [0,1])
//   C_j   = W_0 + ... + W_j                            (exact integer scan)
//   total = (double)C_{n-1} * 2^-62;  invalid (no resample, weights reset to
//           uniform) when C_{n-1} == 0 or any w_j is outside [0,1] / NaN
//   u01   = (lcg >> 11) * 2^-53 after lcg <- lcg*6364136223846793005
//           + 1442695040888963407 (the reference's host LCG, advanced only
//           for a valid total), step = total / n, u0 = u01 * step
//   t_i   = u0 + (double)i * step   (two roundings, as cpu.rs)
//   anc_i = min(first j with C_j >= ceil(t_i * 2^62), n - 1)
// Because C_j is an integer, C_j >= ceil(t * 2^62) is exactly C_j * 2^-62 >= t.
//
// Kernels: (1) single-pass scan with decoupled look-back (Merrill & Garland,
// "Single-pass parallel prefix scan with decoupled look-back", 2016) over
// 4096-particle tiles with dynamic tile ids and bounded spins; (2) merge-path
// gather (Green, McColl, Bader, "GPU merge path", 2012) over the merged
// sequence of thresholds and cumulative weights, so every thread handles the
// same number of merge steps whatever the weight distribution; (3) uniform
// re-injection with the reference's splitmix64 streams
// (src/cuda/pf_kernels.cu:323-352), applied per particle in ascending draw
// order so the f32 result is deterministic; (4) a one-thread commit that flips
// the live ping-pong buffer.
#include <math.h>

#include "pf_internal.h"

namespace pfb {

namespace {

constexpr int kScanThreads = 256;
constexpr int kScanItems = 16;
constexpr int kScanTile = kScanThreads * kScanItems;  // 4096
constexpr int kMergeItems = 16;                       // merge steps per thread
constexpr int kThreads = 256;

struct PlaneSet {
    Planes s[2];
};
PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__device__ __forceinline__ float weight_of(int wmode, int i, int n,
                                           const float* __restrict__ w,
                                           const float* __restrict__ ll,
                                           double M, double S) {
    if (wmode == WMODE_UNIFORM) return 1.0f / (float)n;
    if (wmode == WMODE_STORED) return w[i];
    return (float)(exp((double)ll[i] - M) / S);
}

__device__ __forceinline__ uint64_t shfl_up_u64(uint64_t v, int d) {
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    lo = __shfl_up_sync(~0u, lo, d);
    hi = __shfl_up_sync(~0u, hi, d);
    return ((uint64_t)hi << 32) | lo;
}

__device__ __forceinline__ unsigned ld_acquire(const unsigned* p) {
    unsigned v;
    asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(p)
                 : "memory");
    return v;
}
__device__ __forceinline__ void st_release(unsigned* p, unsigned v) {
    asm volatile("st.release.gpu.global.u32 [%0], %1;" ::"l"(p), "r"(v)
                 : "memory");
}

enum : unsigned { TILE_AGG = 1u, TILE_INCL = 2u };

__global__ void __launch_bounds__(kScanThreads)
    k_scan(int n, const float* __restrict__ w, const float* __restrict__ ll,
           uint64_t* __restrict__ cum, unsigned* flags, uint64_t* vals,
           CycleCtl* ctl, int cond, unsigned epoch, int use_u01,
           double u01_arg) {
    if (cond && !ctl->resample_now) return;
    __shared__ unsigned s_tile;
    __shared__ uint64_t s_warp[kScanThreads / 32];
    __shared__ uint64_t s_prefix;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (tid == 0) s_tile = atomicAdd(&ctl->tile_counter, 1u);
    __syncthreads();
    const int tile = (int)s_tile;
    const int ntiles = ceil_div(n, kScanTile);
    const int wmode = ctl->wmode;
    const double M = ctl->ll_max, S = ctl->ll_sumexp;

    // Load and convert this thread's 16 consecutive weights.
    const long long base = (long long)tile * kScanTile + tid * kScanItems;
    uint64_t v[kScanItems];
    bool bad = false;
    uint64_t run = 0;
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long j = base + k;
        uint64_t W = 0;
        if (j < n) {
            const float wf = weight_of(wmode, (int)j, n, w, ll, M, S);
            if (!(wf >= 0.0f) || !(wf <= 1.0f)) {
                bad = true;
            } else {
                W = __double2ull_rn((double)wf * 0x1p62);
            }
        }
        run += W;
        v[k] = run;
    }
    // Block exclusive scan of the thread totals.
    uint64_t x = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        uint64_t y = shfl_up_u64(x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    const int any_bad = __syncthreads_or(bad ? 1 : 0);
    if (tid == 0) {
        uint64_t acc = 0;
        for (int k = 0; k < kScanThreads / 32; ++k) {
            uint64_t t = s_warp[k];
            s_warp[k] = acc;
            acc += t;
        }
        // acc = tile aggregate; publish and look back.
        if (any_bad) atomicOr(&ctl->err, ERR_SCAN_OVERFLOW);
        uint64_t prefix = 0;
        if (tile == 0) {
            vals[1] = acc;
            __threadfence();
            st_release(&flags[0], (epoch << 2) | TILE_INCL);
        } else {
            vals[2 * (size_t)tile] = acc;
            __threadfence();
            st_release(&flags[tile], (epoch << 2) | TILE_AGG);
            int j = tile - 1;
            int spins = 0;
            while (j >= 0) {
                const unsigned f = ld_acquire(&flags[j]);
                if ((f >> 2) != epoch || (f & 3u) == 0u) {
                    if (++spins > kSpinLimit) {
                        atomicOr(&ctl->err, ERR_SPIN_TIMEOUT);
                        break;
                    }
                    continue;
                }
                if ((f & 3u) == TILE_INCL) {
                    prefix += __ldcg(&vals[2 * (size_t)j + 1]);
                    break;
                }
                prefix += __ldcg(&vals[2 * (size_t)j]);
                --j;
            }
            vals[2 * (size_t)tile + 1] = prefix + acc;
            __threadfence();
            st_release(&flags[tile], (epoch << 2) | TILE_INCL);
        }
        s_prefix = prefix;
        if (tile == ntiles - 1) {
            // Last tile: every predecessor has published, so the error bits
            // of all tiles are visible here.
            const uint64_t T = prefix + acc;
            const bool ok = (T != 0) && !(atomicOr(&ctl->err, 0u) &
                                          (ERR_SCAN_OVERFLOW | ERR_SPIN_TIMEOUT));
            ctl->total_fx = T;
            ctl->resample_valid = ok ? 1 : 0;
            if (ok) {
                double u01;
                if (use_u01) {
                    u01 = u01_arg;
                } else {
                    unsigned long long l = ctl->lcg;
                    l = l * 6364136223846793005ull + 1442695040888963407ull;
                    ctl->lcg = l;
                    u01 = (double)(l >> 11) * (1.0 / 9007199254740992.0);
                }
                const double total = (double)T * 0x1p-62;
                const double step = total / (double)n;
                ctl->total = total;
                ctl->step = step;
                ctl->u0 = u01 * step;
            } else {
                ctl->total = (double)T * 0x1p-62;
                ctl->wmode = WMODE_UNIFORM;
            }
        }
    }
    __syncthreads();
    const uint64_t off = s_prefix + s_warp[warp] + (x - run);
#pragma unroll
    for (int k = 0; k < kScanItems; ++k) {
        const long long j = base + k;
        if (j < n) cum[j] = off + v[k];
    }
}

// Fixed-point threshold of output i (see the specification above).
__device__ __forceinline__ uint64_t threshold_fx(int i, double u0,
                                                 double step) {
    const double t = __dadd_rn(u0, __dmul_rn((double)i, step));
    const double s = t * 0x1p62;
    if (!(s > 0.0)) return 0ull;
    if (s >= 0x1p64) return ~0ull;
    return __double2ull_ru(s);
}

__global__ void __launch_bounds__(kThreads)
    k_gather(PlaneSet ps, int n, const uint64_t* __restrict__ cum,
             int* __restrict__ anc_out, int record_anc, CycleCtl* ctl,
             int cond) {
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const double u0 = ctl->u0, step = ctl->step;
    const int live = ctl->live;
    const Planes src = ps.s[live], dst = ps.s[1 - live];
    const long long g = (long long)blockIdx.x * kThreads + threadIdx.x;
    const long long diag = g * kMergeItems;
    const long long total_len = 2LL * n;
    if (diag >= total_len) return;
    // Merge-path split of the first `diag` merged items: thresholds A_i
    // precede cumulative values B_j when A_i <= B_j.
    long long lo = diag > n ? diag - n : 0;
    long long hi = diag < n ? diag : n;
    while (lo < hi) {
        const long long mid = (lo + hi) >> 1;
        if (threshold_fx((int)mid, u0, step) <= __ldg(&cum[diag - 1 - mid]))
            lo = mid + 1;
        else
            hi = mid;
    }
    long long a = lo, b = diag - lo;
    uint64_t ta = a < n ? threshold_fx((int)a, u0, step) : 0ull;
    for (int it = 0; it < kMergeItems && a + b < total_len; ++it) {
        if (a < n && (b >= n || ta <= __ldg(&cum[b]))) {
            const int j = (int)(b < n ? b : n - 1);
            const int i = (int)a;
            dst.px[i] = src.px[j];
            dst.py[i] = src.py[j];
            dst.pz[i] = src.pz[j];
            dst.qw[i] = src.qw[j];
            dst.qx[i] = src.qx[j];
            dst.qy[i] = src.qy[j];
            dst.qz[i] = src.qz[j];
            if (record_anc) anc_out[i] = j;
            ++a;
            if (a < n) ta = threshold_fx((int)a, u0, step);
        } else {
            ++b;
        }
    }
}

// splitmix64 step (Steele, Lea, Flood, "Fast splittable pseudorandom number
// generators", OOPSLA 2014), the generator of the reference's k_inject.
__device__ __forceinline__ uint64_t splitmix_next(uint64_t& z) {
    z += 0x9E3779B97F4A7C15ull;
    uint64_t r = z;
    r = (r ^ (r >> 30)) * 0xBF58476D1CE4E5B9ull;
    r = (r ^ (r >> 27)) * 0x94D049BB133111EBull;
    return r ^ (r >> 31);
}

struct InjDraw {
    int idx;
    float jx, jy, jz;
};

// Draw j of the injection stream: stream seed lcg ^ gen*phi ^ (j+1)*c as in
// src/cuda/pf_kernels.cu:337-348.
__device__ __forceinline__ InjDraw inj_draw(uint64_t lcg, uint64_t gen, int j,
                                            int n) {
    uint64_t z = lcg ^ (gen * 0x9E3779B97F4A7C15ull) ^
                 ((uint64_t)j + 1) * 0xBF58476D1CE4E5B9ull;
    if (z == 0) z = 0x243F6A8885A308D3ull;
    InjDraw d;
    double u = (double)(splitmix_next(z) >> 11) * (1.0 / 9007199254740992.0);
    int idx = (int)(u * n);
    d.idx = idx >= n ? n - 1 : idx;
    u = (double)(splitmix_next(z) >> 11) * (1.0 / 9007199254740992.0);
    d.jx = (float)(u - 0.5);
    u = (double)(splitmix_next(z) >> 11) * (1.0 / 9007199254740992.0);
    d.jy = (float)(u - 0.5);
    u = (double)(splitmix_next(z) >> 11) * (1.0 / 9007199254740992.0);
    d.jz = (float)(u - 0.5);
    return d;
}

// Injection lists: head[idx] holds (epoch << 32 | last inserted j), next[j]
// chains the rest; entries of older epochs read as empty.
__global__ void k_inject_link(int n, int k, uint64_t gen, uint64_t* head,
                              int* next, CycleCtl* ctl, int cond,
                              unsigned epoch) {
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= k) return;
    const InjDraw d = inj_draw(ctl->lcg, gen, j, n);
    const uint64_t tag = ((uint64_t)epoch << 32) | (uint32_t)j;
    const uint64_t prev = atomicExch((unsigned long long*)&head[d.idx],
                                     (unsigned long long)tag);
    next[j] = ((uint32_t)(prev >> 32) == epoch) ? (int)(uint32_t)prev : -1;
}

__global__ void k_inject_apply(PlaneSet ps, int n, int k, uint64_t gen,
                               const uint64_t* head, const int* next,
                               CycleCtl* ctl, int cond, unsigned epoch) {
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= k) return;
    const uint64_t lcg = ctl->lcg;
    const InjDraw d = inj_draw(lcg, gen, j, n);
    const uint64_t h = head[d.idx];
    if ((uint32_t)(h >> 32) != epoch || (int)(uint32_t)h != j) return;
    // This thread inserted last for particle d.idx: apply every draw of the
    // list in ascending j (selection over the short list).
    const Planes dst = ps.s[1 - ctl->live];
    float px = dst.px[d.idx], py = dst.py[d.idx], pz = dst.pz[d.idx];
    int last = -1;
    for (;;) {
        int best = -1;
        for (int x = j; x >= 0; x = next[x])
            if (x > last && (best < 0 || x < best)) best = x;
        if (best < 0) break;
        const InjDraw e = (best == j) ? d : inj_draw(lcg, gen, best, n);
        px += e.jx;
        py += e.jy;
        pz += e.jz;
        last = best;
    }
    dst.px[d.idx] = px;
    dst.py[d.idx] = py;
    dst.pz[d.idx] = pz;
}

__global__ void k_commit(CycleCtl* ctl, int cond) {
    if (!(cond && !ctl->resample_now)) {
        if (ctl->resample_valid) {
            ctl->live = 1 - ctl->live;
            ctl->resampled = 1;
        }
        ctl->wmode = WMODE_UNIFORM;
    }
    ctl->tile_counter = 0u;
    ctl->err &= ~ERR_SCAN_OVERFLOW;
}

// The reference's pick rule (src/cuda/pf_kernels.cu:304-321) on a given cum:
// t = u0 + i*step evaluated as one fused multiply-add, lower_bound, clamp.
__global__ void k_pick_from_cum(const double* __restrict__ cum, int n,
                                double u0, double total, int* anc) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const double step = total / (double)n;
    const double t = fma((double)i, step, u0);
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

}  // namespace

int launch_resample(PfHandle* h, float inject_ratio, bool cond_on_ctl,
                    bool use_u01, double u01) {
    const int n = h->n;
    const int ntiles = ceil_div(n, kScanTile);
    // Look-back epochs are per handle and fit in 30 bits; 0 is never used.
    h->scan_epoch = (h->scan_epoch + 1u) & 0x3FFFFFFFu;
    if (h->scan_epoch == 0u) h->scan_epoch = 1u;
    const unsigned epoch = h->scan_epoch;
    const int cond = cond_on_ctl ? 1 : 0;
    {
        KernelScope ks(h, KK_SCAN);
        k_scan<<<ntiles, kScanThreads, 0, h->stream>>>(
            n, h->d_w, h->d_ll, h->d_cum, h->d_scan_flags, h->d_scan_vals,
            h->d_ctl, cond, epoch, use_u01 ? 1 : 0, u01);
    }
    PFB_KL();
    const long long merge_threads = ceil_div_ll(2LL * n, kMergeItems);
    const int mgrid = (int)ceil_div_ll(merge_threads, kThreads);
    {
        KernelScope ks(h, KK_GATHER);
        k_gather<<<mgrid, kThreads, 0, h->stream>>>(
            plane_set(h), n, h->d_cum, h->d_anc, h->record_anc ? 1 : 0,
            h->d_ctl, cond);
    }
    PFB_KL();
    // k = floor(ratio * n) with the reference's f32 product
    // (src/cuda/pf_kernels.cu:667-671).
    int k = (inject_ratio > 0.f) ? (int)(inject_ratio * (float)n) : 0;
    if (k > n) k = n;
    if (k > 0) {
        h->inj_epoch = (h->inj_epoch + 1u);
        if (h->inj_epoch == 0u) h->inj_epoch = 1u;
        const int ig = ceil_div(k, kThreads);
        {
            KernelScope ks(h, KK_INJECT);
            k_inject_link<<<ig, kThreads, 0, h->stream>>>(
                n, k, h->gen, h->d_inj_head, h->d_inj_next, h->d_ctl, cond,
                h->inj_epoch);
        }
        PFB_KL();
        {
            KernelScope ks(h, KK_INJECT);
            k_inject_apply<<<ig, kThreads, 0, h->stream>>>(
                plane_set(h), n, k, h->gen, h->d_inj_head, h->d_inj_next,
                h->d_ctl, cond, h->inj_epoch);
        }
        PFB_KL();
    }
    {
        KernelScope ks(h, KK_COMMIT);
        k_commit<<<1, 1, 0, h->stream>>>(h->d_ctl, cond);
    }
    PFB_KL();
    h->anc_valid = h->record_anc;
    return 0;
}

int launch_pick_from_cum(PfHandle* h, const double* d_cum, int n, double u0,
                         double total, int* d_anc) {
    KernelScope ks(h, KK_MISC);
    k_pick_from_cum<<<ceil_div(n, kThreads), kThreads, 0, h->stream>>>(
        d_cum, n, u0, total, d_anc);
    PFB_KL();
    return 0;
}

}  // namespace pfb
