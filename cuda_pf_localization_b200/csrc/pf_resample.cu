// pf_resample.cu — systematic resampling with an exact fixed-point scan,
// fused with the ancestor gather.
//
// Specification (semantics of src/cuda/pf_kernels.cu:638-676 and
// crates/pf_core/src/cpu.rs:262-306, made exact and deterministic):
//   W_j   = round_nearest_even(w_j * 2^62)             (u64, w_j in [0,1])
//   C_j   = W_0 + ... + W_j                            (exact integer scan)
//   T     = C_{n-1};  invalid (no resample, weights reset to uniform) when
//           T == 0 or any w_j is outside [0,1] / NaN
//   u01   = (lcg >> 11) * 2^-53 after lcg <- lcg*6364136223846793005
//           + 1442695040888963407 (the reference's host LCG, advanced only
//           for a valid total); total = T * 2^-62, step = total / n,
//           u0 = u01 * step
//   t_i   = u0 + (double)i * step   (two roundings, as cpu.rs)
//   anc_i = min(first j with C_j >= ceil(t_i * 2^62), n - 1)
// Because C_j is an integer, C_j >= ceil(t * 2^62) is exactly C_j * 2^-62 >= t.
//
// The weight pass that precedes every resample (k_ess) forms T and the
// exclusive fixed-point prefix of every block of kPrefixBlock particles, so
// thresholds and each tile's starting sum are known before the resampler
// starts; a tile then scans its own weights in shared registers (no
// inter-block look-back) and gives each particle j its C_{j-1} and C_j.  The
// outputs whose ancestor is j are exactly the run [cnt(C_{j-1}), cnt(C_j)),
// cnt(X) = #{i : T_i <= X}: a thread finds its first run start in closed form
// from the arithmetic threshold sequence (corrected against the exact T_i)
// and then steps the thresholds run by run, writing the ancestor of each
// output of the run; no cumulative array is stored.  Runs longer than kHeavy
// (one particle holding most of the weight) are appended to a list and
// filled by a second, output-parallel kernel.  A third, output-parallel
// kernel then gathers the particles (coalesced 16-byte stores), so the copy
// work does not pile up on the few tiles that hold most of the weight.
//
// Injection uses the reference's splitmix64 streams
// (src/cuda/pf_kernels.cu:323-352), applied per particle in ascending draw
// order so the f32 result is deterministic; a one-thread commit flips the
// live ping-pong buffer and advances the LCG.
#include <math.h>

#include "pf_device.cuh"

namespace pfb {

namespace {

using namespace pfb::dev;

constexpr int kScanThreads = 256;
constexpr int kScanItems = 8;
constexpr int kScanTile = kScanThreads * kScanItems;  // 2048
static_assert(kScanTile % kPrefixBlock == 0, "tiles start on prefix blocks");
constexpr int kHeavy = 32;  // longest run whose ancestors a scan thread writes
constexpr int kStep = 4;    // thresholds stepped before the closed form
constexpr int kThreads = kBlk;

PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__global__ void __launch_bounds__(kScanThreads)
    k_resample(int n, const float* __restrict__ w, const float* __restrict__ ll,
               const uint64_t* __restrict__ prefix, int* __restrict__ anc,
               HeavyRun* heavy, int heavy_cap, CycleCtl* ctl, int cond,
               int use_u01, double u01_arg) {
    pdl_wait();
    if (cond && !ctl->resample_now) return;
    const uint64_t T = ctl->w_total_fx;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    if (T == 0 || ctl->w_bad) {
        if (blockIdx.x == 0 && tid == 0) ctl->resample_valid = 0;
        return;
    }
    // Offsets: every block derives the same values from T and the LCG.
    const unsigned long long lcg0 = ctl->lcg;
    const unsigned long long lcg1 =
        use_u01 ? lcg0 : lcg0 * 6364136223846793005ull + 1442695040888963407ull;
    const double u01 =
        use_u01 ? u01_arg : (double)(lcg1 >> 11) * (1.0 / 9007199254740992.0);
    const double total = (double)T * 0x1p-62;
    const double step = total / (double)n;
    const double u0 = u01 * step;
    if (blockIdx.x == 0 && tid == 0) {
        ctl->lcg_next = lcg1;
        ctl->resample_valid = 1;
        ctl->total_fx = T;
        ctl->total = total;
        ctl->step = step;
        ctl->u0 = u0;
    }
    __shared__ uint64_t s_warp[kScanThreads / 32];
    const int tile = blockIdx.x;
    // the tile's starting sum, fetched early (it is needed after the scan)
    const uint64_t tile_base =
        tid == 0 ? __ldcg(&prefix[(size_t)tile * (kScanTile / kPrefixBlock)]) : 0ull;
    const int wmode = ctl->wmode;
    const double M = ctl->ll_max, S = ctl->ll_sumexp;

    // This thread's total over its kScanItems consecutive weights.
    const long long j0 = (long long)tile * kScanTile + tid * kScanItems;
    uint64_t run = 0;
    if (wmode == WMODE_STORED && j0 + kScanItems <= n) {
        const float4* w4 = reinterpret_cast<const float4*>(w + j0);
#pragma unroll
        for (int q = 0; q < kScanItems / 4; ++q) {
            const float4 a = w4[q];
            run += weight_fx(a.x) + weight_fx(a.y) + weight_fx(a.z) + weight_fx(a.w);
        }
    } else {
        for (int k = 0; k < kScanItems; ++k) {
            const long long j = j0 + k;
            if (j < n) run += weight_fx(weight_of(wmode, j, n, w, ll, M, S));
        }
    }
    // Block scan of the thread totals; the tile's own start comes from the
    // prefix pass.
    uint64_t x = run;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint64_t y = shfl_up_u64(x, d);
        if (lane >= d) x += y;
    }
    if (lane == 31) s_warp[warp] = x;
    __syncthreads();
    if (tid == 0) {
        uint64_t acc = tile_base;
        for (int k = 0; k < kScanThreads / 32; ++k) {
            const uint64_t t = s_warp[k];
            s_warp[k] = acc;
            acc += t;
        }
    }
    __syncthreads();

    // Ancestor runs.  C_{j0-1} = tile prefix + exclusive offset of this
    // thread.  The end of each run, cnt(C_j), is found by stepping the
    // thresholds from the end of the previous run (one threshold per output
    // plus one), switching to the closed form once a run exceeds kStep
    // outputs (the steps form a serial FP64 chain); runs longer than kHeavy
    // are filled by the output-parallel expansion.
    uint64_t C = s_warp[warp] + (x - run);
    long long s = (j0 == 0) ? 0 : count_le(C, n, u0, step);
#pragma unroll 1
    for (int k = 0; k < kScanItems; ++k) {
        const long long j = j0 + k;
        if (j >= n) break;
        C += weight_fx(weight_of(wmode, j, n, w, ll, M, S));
        long long e;
        if (j == n - 1) {
            e = n;
        } else {
            e = s;
            while (e < n && e - s < kStep && threshold_fx(e, u0, step) <= C) ++e;
            if (e - s == kStep) e = count_le(C, n, u0, step);
        }
        if (e - s > kHeavy) {
            push_run(heavy, heavy_cap, &ctl->heavy_count, &ctl->err, (int)j, s, e, 0);
        } else {
            for (long long i = s; i < e; ++i) anc[i] = (int)j;
        }
        s = e;
    }
}

// Output-parallel ancestors of the long runs: each recorded piece (at most
// kSplit outputs) is filled by one block.
__global__ void __launch_bounds__(kThreads)
    k_expand_runs(const HeavyRun* heavy, int heavy_cap, int* __restrict__ anc,
                  CycleCtl* ctl, int cond) {
    pdl_wait();
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int count = min(ctl->heavy_count, heavy_cap);
    for (int r = blockIdx.x; r < count; r += gridDim.x) {
        const HeavyRun h = heavy[r];
        for (int i = h.start + (int)threadIdx.x; i < h.end; i += kThreads) anc[i] = h.j;
    }
}

// Output-parallel gather: output i takes particle anc[i] of the live set
// (four outputs per thread, 16-byte stores on every plane; the ancestors are
// non-decreasing, so the loads walk the source planes in order).
__global__ void __launch_bounds__(kThreads)
    k_gather(PlaneSet ps, int n, const int* __restrict__ anc, CycleCtl* ctl,
             int cond) {
    pdl_wait();
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int live = ctl->live;
    const Planes src = pick_planes(ps, live), dst = pick_planes(ps, 1 - live);
    const int i4 = blockIdx.x * kThreads + threadIdx.x;
    const int i = 4 * i4;
    if (i >= n) return;
    if (i + 3 < n) {
        const int4 a = reinterpret_cast<const int4*>(anc)[i4];
#define PFB_GATHER_PLANE(P)                                                  \
    reinterpret_cast<float4*>(dst.P)[i4] =                                   \
        make_float4(src.P[a.x], src.P[a.y], src.P[a.z], src.P[a.w])
        PFB_GATHER_PLANE(px);
        PFB_GATHER_PLANE(py);
        PFB_GATHER_PLANE(pz);
        PFB_GATHER_PLANE(qw);
        PFB_GATHER_PLANE(qx);
        PFB_GATHER_PLANE(qy);
        PFB_GATHER_PLANE(qz);
#undef PFB_GATHER_PLANE
    } else {
        for (int o = i; o < n; ++o) {
            const int j = anc[o];
            dst.px[o] = src.px[j];
            dst.py[o] = src.py[j];
            dst.pz[o] = src.pz[j];
            dst.qw[o] = src.qw[j];
            dst.qx[o] = src.qx[j];
            dst.qy[o] = src.qy[j];
            dst.qz[o] = src.qz[j];
        }
    }
}

// Injection lists: head[idx] holds (epoch << 32 | last inserted j), next[j]
// chains the rest; entries of older epochs read as empty.
__global__ void k_inject_link(int n, int k, uint64_t gen, uint64_t* head,
                              int* next, CycleCtl* ctl, int cond,
                              unsigned epoch, const CycleArgs* ca) {
    pdl_wait();
    if (ca) {
        gen = ca->gen;
        epoch = ca->inj_epoch;
    }
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= k) return;
    const InjDraw d = inj_draw(ctl->lcg_next, gen, j, n);
    const uint64_t tag = ((uint64_t)epoch << 32) | (uint32_t)j;
    const uint64_t prev = atomicExch((unsigned long long*)&head[d.idx],
                                     (unsigned long long)tag);
    next[j] = ((uint32_t)(prev >> 32) == epoch) ? (int)(uint32_t)prev : -1;
}

__global__ void k_inject_apply(PlaneSet ps, int n, int k, uint64_t gen,
                               const uint64_t* head, const int* next,
                               CycleCtl* ctl, int cond, unsigned epoch,
                               const CycleArgs* ca) {
    pdl_wait();
    if (ca) {
        gen = ca->gen;
        epoch = ca->inj_epoch;
    }
    if (cond && !ctl->resample_now) return;
    if (!ctl->resample_valid) return;
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= k) return;
    const uint64_t lcg = ctl->lcg_next;
    const InjDraw d = inj_draw(lcg, gen, j, n);
    const uint64_t h = head[d.idx];
    if ((uint32_t)(h >> 32) != epoch || (int)(uint32_t)h != j) return;
    // This thread inserted last for particle d.idx: apply every draw of the
    // list in ascending j (selection over the short list).
    const Planes dst = pick_planes(ps, 1 - ctl->live);
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
    pdl_wait();
    if (!(cond && !ctl->resample_now)) {
        if (ctl->resample_valid) {
            ctl->live = 1 - ctl->live;
            ctl->resampled = 1;
            ctl->lcg = ctl->lcg_next;
        }
        ctl->wmode = WMODE_UNIFORM;
    }
    ctl->heavy_count = 0;
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

unsigned next_inj_epoch(PfHandle* h) {
    h->inj_epoch = h->inj_epoch + 1u;
    if (h->inj_epoch == 0u) h->inj_epoch = 1u;
    return h->inj_epoch;
}

// With dargs set (graph capture) the epochs and the generation come from
// device memory at replay time; the host counters are not advanced here.
int launch_resample(PfHandle* h, float inject_ratio, bool cond_on_ctl,
                    bool use_u01, double u01, const CycleArgs* dargs) {
    const int n = h->n;
    const int ntiles = ceil_div(n, kScanTile);
    // The weight total and the block prefixes come from the weight pass; run
    // one when the weights changed since the last.
    if (!h->prefix_valid && launch_weight_prefix(h, false, 0.0)) return -1;
    const int cond = cond_on_ctl ? 1 : 0;
    {
        KernelScope ks(h, KK_SCAN);
        PFB_CK(launch_pdl(k_resample, ntiles, kScanThreads, 0, h->stream, n, h->d_w,
                          h->d_ll, h->d_wprefix, h->d_anc, h->d_heavy, h->heavy_cap,
                          h->d_ctl, cond, use_u01 ? 1 : 0, u01));
    }
    PFB_KL();
    {
        KernelScope ks(h, KK_SCAN);
        PFB_CK(launch_pdl(k_expand_runs, 2 * 148, kThreads, 0, h->stream, h->d_heavy,
                          h->heavy_cap, h->d_anc, h->d_ctl, cond));
    }
    PFB_KL();
    {
        KernelScope ks(h, KK_GATHER);
        PFB_CK(launch_pdl(k_gather, ceil_div(n, 4 * kThreads), kThreads, 0, h->stream,
                          plane_set(h), n, h->d_anc, h->d_ctl, cond));
    }
    PFB_KL();
    // k = floor(ratio * n) with the reference's f32 product
    // (src/cuda/pf_kernels.cu:667-671).
    int k = (inject_ratio > 0.f) ? (int)(inject_ratio * (float)n) : 0;
    if (k > n) k = n;
    if (k > 0) {
        const unsigned iepoch = dargs ? 0u : next_inj_epoch(h);
        const int ig = ceil_div(k, kThreads);
        {
            KernelScope ks(h, KK_INJECT);
            PFB_CK(launch_pdl(k_inject_link, ig, kThreads, 0, h->stream, n, k, h->gen,
                              h->d_inj_head, h->d_inj_next, h->d_ctl, cond, iepoch,
                              dargs));
        }
        PFB_KL();
        {
            KernelScope ks(h, KK_INJECT);
            PFB_CK(launch_pdl(k_inject_apply, ig, kThreads, 0, h->stream, plane_set(h), n,
                              k, h->gen, h->d_inj_head, h->d_inj_next, h->d_ctl, cond,
                              iepoch, dargs));
        }
        PFB_KL();
    }
    {
        KernelScope ks(h, KK_COMMIT);
        PFB_CK(launch_pdl(k_commit, 1, 1, 0, h->stream, h->d_ctl, cond));
    }
    PFB_KL();
    h->anc_valid = true;
    // The weights are uniform afterwards; the next estimate pass recomputes
    // their fixed-point total.
    h->prefix_valid = false;
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
