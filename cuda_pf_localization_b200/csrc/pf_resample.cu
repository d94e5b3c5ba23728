// pf_resample.cu — systematic resampling with an exact fixed-point scan,
// fused with the ancestor gather, the injection and the estimate sums of the
// resampled cloud.
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
// exclusive fixed-point prefix of every block of kPrefixBlock particles.  Then
//   * k_mark (source-parallel, persistent): a tile scans its 2048 weights
//     from its block prefix; source j owns the outputs
//     [cnt(C_{j-1}), cnt(C_j)), cnt(X) = #{i : T_i <= X}, found in closed
//     form.  It writes j at the first output of its run and at every
//     output-tile boundary inside it (so every output tile starts with a
//     marker, and a source writes one marker plus one per tile its run
//     crosses), and adds its particle, weighted by its run length / n, to the
//     14 FP64 estimate sums of the new cloud (one partial per block);
//   * k_gather (output-parallel, persistent): block 0 combines k_mark's
//     partials in block order and runs the Markley mean (warp-parallel).
//     Blocks 1.. each load the markers of an output tile; a block-wide
//     running maximum (ancestors increase with the output index) gives every
//     output its ancestor, kept in shared memory.  A block resets the
//     markers it read, copies the seven planes of four outputs at a time
//     from the live set (16-byte stores) and adds the injection jitters of
//     the draws that landed in the tile; the last block to finish adds the
//     jitters' change to the position sums and commits the resample (live
//     set, LCG).
// No output needs a search and no block does more than its outputs or its
// sources, whatever the weights.  When the cycle does not resample (or the
// total is invalid), k_mark is the estimate pass over the cloud instead and
// k_gather does nothing.
//
// Injection uses the reference's splitmix64 streams
// (src/cuda/pf_kernels.cu:323-352).  k_mark files each draw under the output
// tile of its particle; k_gather applies a tile's draws per particle in
// ascending draw order, so the f32 result is deterministic (the reference's
// atomicAdd order is not).
#include <math.h>

#include "markley.h"
#include "pf_device.cuh"

namespace pfb {

namespace {

using namespace pfb::dev;

constexpr int kThreads = kBlk;
constexpr int kGroup = 4;                         // consecutive outputs per thread slot
constexpr int kTile = 2 * kGroup * kThreads;      // 2048 outputs per gather block
constexpr int kScanItems = 8;                     // sources per thread of k_mark
constexpr int kScanTile = kScanItems * kThreads;  // 2048 sources per k_mark block
constexpr int kInjChunk = kThreads;               // draws per round of the overflow scan
constexpr int kCorrN = 3;                         // position sums the injection changes
// persistent grids (multiples of the 148 SMs of a B200): k_mark at two
// blocks per SM, k_gather at four
constexpr int kMarkGrid = 2 * 148;
constexpr int kGatherGrid = 4 * 148;
static_assert(kScanTile % kPrefixBlock == 0, "scan tiles start on prefix blocks");

// The two particle sets as two base pointers and a plane stride (component
// k of set s is base[s] + k * stride): fewer registers than 14 pointers.
struct PlaneBase {
    float* base[2];
    long long stride;
};

PlaneBase plane_base(const PfHandle* h) {
    return {{h->d_state[0], h->d_state[1]}, (long long)h->n_pad};
}

__device__ __forceinline__ float* plane(const PlaneBase& pb, int set, int k) {
    return (set ? pb.base[1] : pb.base[0]) + (long long)k * pb.stride;
}

__device__ __forceinline__ uint64_t lcg_step(uint64_t x) {
    return x * 6364136223846793005ull + 1442695040888963407ull;
}

// Offsets of a resample from the control block (identical in every block).
struct Offsets {
    uint64_t T, lcg1;
    double total, step, u0;
};

__device__ __forceinline__ Offsets offsets(const CycleCtl* ctl, int n, int use_u01,
                                           double u01_arg) {
    Offsets o;
    o.T = ctl->w_total_fx;
    const uint64_t lcg0 = ctl->lcg;
    o.lcg1 = use_u01 ? lcg0 : lcg_step(lcg0);
    const double u01 =
        use_u01 ? u01_arg : (double)(o.lcg1 >> 11) * (1.0 / 9007199254740992.0);
    o.total = (double)o.T * 0x1p-62;
    o.step = o.total / (double)n;
    o.u0 = u01 * o.step;
    return o;
}

// Block sum of NV per-thread FP64 values (xor butterfly per warp, warps in
// order) into part[blockIdx.x * NV + q]; then whether this block was the last
// of the grid to finish (counter `done`).  Valid in every thread.
template <int NV>
__device__ __forceinline__ bool block_partial_last(const double (&acc)[NV], double* part,
                                                   unsigned* done) {
    __shared__ double s_w[NV][kThreads / 32];
    __shared__ bool s_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
#pragma unroll
    for (int q = 0; q < NV; ++q) {
        const double x = warp_sum_d(acc[q]);
        if (lane == 0) s_w[q][warp] = x;
    }
    __syncthreads();
    if (tid < NV) {
        double x = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) x += s_w[tid][k];
        part[(size_t)blockIdx.x * NV + tid] = x;
        __threadfence();
    }
    __syncthreads();
    if (tid == 0) s_last = atomicAdd(done, 1u) == gridDim.x - 1;
    __syncthreads();
    return s_last;
}

// The last block's combine: the G <= kMaxG partials of NV sums
// (part[b * NV + q]) staged in shared memory with one round of loads, then
// summed per component in block order (lanes strided, then a butterfly).
// Results in s_out[0, NV).
template <int NV, int kMaxG>
__device__ __forceinline__ void combine_staged(const double* part, int G, double* s_p,
                                               double* s_out) {
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int tot = G * NV;
    constexpr int kPer = (NV * kMaxG + kThreads - 1) / kThreads;
    constexpr int kBatch = 8;  // loads in flight per thread
#pragma unroll 1
    for (int r0 = 0; r0 < kPer; r0 += kBatch) {
        double v[kBatch];
#pragma unroll
        for (int r = 0; r < kBatch; ++r) {
            const int idx = tid + (r0 + r) * kThreads;
            v[r] = idx < tot ? __ldcg(&part[idx]) : 0.0;
        }
#pragma unroll
        for (int r = 0; r < kBatch; ++r) {
            const int idx = tid + (r0 + r) * kThreads;
            if (idx < tot) s_p[(idx % NV) * kMaxG + idx / NV] = v[r];
        }
    }
    __syncthreads();
    for (int q = warp; q < NV; q += kThreads / 32) {
        double x = 0.0;
        for (int b = lane; b < G; b += 32) x += s_p[q * kMaxG + b];
        x = warp_sum_d(x);
        if (lane == 0) s_out[q] = x;
    }
    __syncthreads();
}

// Injection draws of one tile, in shared memory: local output, draw index,
// jitter.
struct InjList {
    int loc[kThreads];
    int j[kThreads];
    float jx[kThreads], jy[kThreads], jz[kThreads];
    unsigned hit[kTile / 32];  // outputs of the tile hit by a listed draw
};

// Apply to the group of outputs [l0, l0 + kGroup), in ascending draw order,
// the listed draws (m entries, any order) that hit it; the exact change of
// every position value goes to d[0..2].
__device__ __forceinline__ void apply_draws(const InjList& L, int m, int l0,
                                            float (&x)[kGroup], float (&y)[kGroup],
                                            float (&z)[kGroup], double (&d)[kCorrN]) {
    int hits = 0;
    for (int e = 0; e < m; ++e) hits += (unsigned)(L.loc[e] - l0) < (unsigned)kGroup;
    int last = -1;
    for (int h = 0; h < hits; ++h) {
        int best = -1;
        for (int e = 0; e < m; ++e)
            if ((unsigned)(L.loc[e] - l0) < (unsigned)kGroup && L.j[e] > last &&
                (best < 0 || L.j[e] < L.j[best]))
                best = e;
        const int r = L.loc[best] - l0;
#pragma unroll
        for (int q = 0; q < kGroup; ++q)
            if (q == r) {
                const float nx = x[q] + L.jx[best], ny = y[q] + L.jy[best],
                            nz = z[q] + L.jz[best];
                // exact: differences of two f32 values
                d[0] += (double)nx - (double)x[q];
                d[1] += (double)ny - (double)y[q];
                d[2] += (double)nz - (double)z[q];
                x[q] = nx;
                y[q] = ny;
                z[q] = nz;
            }
        last = L.j[best];
    }
}

// The first pass of every cycle's end, on a persistent grid, in one of three
// modes:
//   * resample with a valid total: tiles of kScanTile sources (kScanItems per
//     thread) scanned from the weight pass's block prefix.  Source j writes j
//     at the first output of its run [cnt(C_{j-1}), cnt(C_j)) and at every
//     output tile boundary inside it (runs are disjoint, so no two sources
//     write the same marker), and adds (run length) x its particle with
//     weight 1/n to the 14 estimate sums.  The blocks first file the
//     injection draws under the output tile of their particle (any order
//     within a bucket; k_gather orders them and clears the counts);
//   * no resample: the estimate pass over the cloud and its weights;
//   * resample with an invalid total: the same over the unchanged cloud with
//     uniform weights, which the resample leaves.
// Each block leaves one partial of the 14 sums (the positions before the
// injection); block 0 of k_gather combines them.
__global__ void __launch_bounds__(kThreads, 2)
    k_mark(PlaneBase pb, int n, const float* __restrict__ w, const float* __restrict__ ll,
           const uint64_t* __restrict__ prefix, int* __restrict__ marker,
           int* __restrict__ inj_cnt, int* __restrict__ inj_bucket, int inj_cap, int k_inj,
           uint64_t gen, double* part_m, CycleCtl* ctl, int cond, int use_u01,
           double u01_arg, const CycleArgs* ca) {
    pdl_wait();
    if (ca) gen = ca->gen;
    const bool resample = !cond || ctl->resample_now;
    const bool valid = resample && ctl->w_total_fx != 0 && !ctl->w_bad;
    __shared__ uint64_t s_warp[kThreads / 32];
    __shared__ double s_w[kEstN][kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int wmode = ctl->wmode;
    const float M = ctl->ll_max, S = ctl->ll_sumexp;
    const int live = ctl->live;
    const float wuni = 1.0f / (float)n;
    const double wd = (double)wuni;  // the weight of a resampled particle
    double acc[kEstN];
#pragma unroll
    for (int q = 0; q < kEstN; ++q) acc[q] = 0.0;
    if (valid) {
        const Offsets of = offsets(ctl, n, use_u01, u01_arg);
        const double inv_step = 1.0 / of.step;
        for (int j = blockIdx.x * kThreads + tid; j < k_inj; j += gridDim.x * kThreads) {
            const InjDraw d = inj_draw(of.lcg1, gen, j, n);
            const int t = d.idx / kTile;
            const int slot = atomicAdd(&inj_cnt[t], 1);
            if (slot < inj_cap) inj_bucket[(size_t)t * inj_cap + slot] = j;
        }
        const int ntiles = ceil_div(n, kScanTile);
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
            // the tile's starting sum, fetched early (needed after the scan)
            const uint64_t tile_base =
                tid == 0 ? __ldcg(&prefix[(size_t)tile * (kScanTile / kPrefixBlock)]) : 0ull;
            const long long j0 = (long long)tile * kScanTile + (long long)tid * kScanItems;
            uint64_t W[kScanItems];
            if (wmode == WMODE_STORED && j0 + kScanItems <= n) {
                const float4* w4 = reinterpret_cast<const float4*>(w + j0);
#pragma unroll
                for (int q = 0; q < kScanItems / 4; ++q) {
                    const float4 a = w4[q];
                    W[4 * q] = weight_fx(a.x);
                    W[4 * q + 1] = weight_fx(a.y);
                    W[4 * q + 2] = weight_fx(a.z);
                    W[4 * q + 3] = weight_fx(a.w);
                }
            } else {
#pragma unroll
                for (int k = 0; k < kScanItems; ++k) {
                    const long long j = j0 + k;
                    W[k] = j < n ? weight_fx(weight_of(wmode, j, n, w, ll, M, S)) : 0ull;
                }
            }
            uint64_t run = 0;
#pragma unroll
            for (int k = 0; k < kScanItems; ++k) run += W[k];
            // block scan of the thread totals, from the tile's prefix
            uint64_t x = run;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint64_t y = shfl_up_u64(x, d);
                if (lane >= d) x += y;
            }
            if (lane == 31) s_warp[warp] = x;
            __syncthreads();
            if (tid == 0) {
                uint64_t a = tile_base;
                for (int k = 0; k < kThreads / 32; ++k) {
                    const uint64_t t = s_warp[k];
                    s_warp[k] = a;
                    a += t;
                }
            }
            __syncthreads();
            uint64_t C = s_warp[warp] + (x - run);  // C_{j0 - 1}
            __syncthreads();                        // s_warp is reused by the next tile
            long long s = (j0 == 0) ? 0 : count_le(C, n, of.u0, of.step, inv_step);
#pragma unroll
            for (int k = 0; k < kScanItems; ++k) {
                const long long j = j0 + k;
                if (j >= n) break;
                C += W[k];
                // a source without weight owns no output (the last takes the rest)
                const long long e =
                    (j == n - 1) ? n : (W[k] ? count_le(C, n, of.u0, of.step, inv_step) : s);
                if (e > s) {
                    marker[s] = (int)j;
                    for (long long t = (s / kTile + 1) * kTile; t < e; t += kTile)
                        marker[t] = (int)j;
                    // e - s copies of particle j, weight wd each: wd * (e - s)
                    // is exact (a 24-bit weight times a count below 2^29)
                    const double wc = wd * (double)(e - s);
                    const double px = plane(pb, live, 0)[j], py = plane(pb, live, 1)[j],
                                 pz = plane(pb, live, 2)[j];
                    const double qv[4] = {plane(pb, live, 3)[j], plane(pb, live, 4)[j],
                                          plane(pb, live, 5)[j], plane(pb, live, 6)[j]};
                    acc[0] += wc * px;
                    acc[1] += wc * py;
                    acc[2] += wc * pz;
                    int ei = 3;
#pragma unroll
                    for (int r = 0; r < 4; ++r)
#pragma unroll
                        for (int cc = r; cc < 4; ++cc) acc[ei++] += wc * qv[r] * qv[cc];
                    acc[13] += wc * wd;
                }
                s = e;
            }
        }
    } else {
        // estimate pass: kScanItems particles per thread, 16-byte loads
        const int em = resample ? (int)WMODE_UNIFORM : wmode;
        const int ntiles = ceil_div(n, kScanTile);
        for (int tile = blockIdx.x; tile < ntiles; tile += gridDim.x) {
#pragma unroll
            for (int h = 0; h < kScanItems / 4; ++h) {
                const long long i0 =
                    (long long)tile * kScanTile + (long long)h * 4 * kThreads + 4 * tid;
                if (i0 >= n) break;
                const long long v4 = i0 >> 2;  // planes are padded: in bounds
                const float4 X = reinterpret_cast<const float4*>(plane(pb, live, 0))[v4];
                const float4 Y = reinterpret_cast<const float4*>(plane(pb, live, 1))[v4];
                const float4 Z = reinterpret_cast<const float4*>(plane(pb, live, 2))[v4];
                const float4 QW = reinterpret_cast<const float4*>(plane(pb, live, 3))[v4];
                const float4 QX = reinterpret_cast<const float4*>(plane(pb, live, 4))[v4];
                const float4 QY = reinterpret_cast<const float4*>(plane(pb, live, 5))[v4];
                const float4 QZ = reinterpret_cast<const float4*>(plane(pb, live, 6))[v4];
                float4 Wv;
                if (em == WMODE_STORED)
                    Wv = reinterpret_cast<const float4*>(w)[v4];
                else if (em == WMODE_UNIFORM)
                    Wv = make_float4(wuni, wuni, wuni, wuni);
                else
                    Wv = make_float4(weight_of(em, i0, n, w, ll, M, S),
                                     weight_of(em, i0 + 1, n, w, ll, M, S),
                                     weight_of(em, i0 + 2, n, w, ll, M, S),
                                     weight_of(em, i0 + 3, n, w, ll, M, S));
#pragma unroll
                for (int c = 0; c < 4; ++c) {
                    if (i0 + c >= n) break;
                    est_add(acc, comp(Wv, c), comp(X, c), comp(Y, c), comp(Z, c),
                            comp(QW, c), comp(QX, c), comp(QY, c), comp(QZ, c));
                }
            }
        }
    }
    // block partial (xor butterfly per warp, warps in order); block 0 of
    // k_gather combines them
#pragma unroll
    for (int q = 0; q < kEstN; ++q) {
        const double v = warp_sum_d(acc[q]);
        if (lane == 0) s_w[q][warp] = v;
    }
    __syncthreads();
    if (tid < kEstN) {
        double v = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) v += s_w[tid][k];
        part_m[(size_t)blockIdx.x * kEstN + tid] = v;
    }
}

// Shared memory of k_gather: a tile's ancestors and injection list, or the
// partials a combine stages (used before or after the tiles).
union GatherSmem {
    struct {
        int anc[kTile];
        InjList inj;
    } t;
    double pm[kEstN * kMarkGrid];
    double pc[kCorrN * kGatherGrid];
};

// The end of a cycle's resample on a persistent grid.  Block 0 combines
// k_mark's partials in block order, runs the Markley mean and leaves the
// estimate sums in the control block (without a valid resample that is all
// the kernel does, and it records an invalid total).  Meanwhile blocks 1..
// take the output tiles of a resample (cond clear, or ctl->resample_now),
// kTile outputs at a time: the tile's ancestors (running maximum of its
// markers) go to shared memory, the particles are copied with 16-byte
// stores, the injection jitters of the tile's draws applied to x, y and z in
// ascending draw order.  The last block adds the jitters' change to the
// position sums and commits the resample.
__global__ void __launch_bounds__(kThreads, 4)
    k_gather(PlaneBase pb, int n, int* __restrict__ marker, int* __restrict__ anc,
             int record, int* __restrict__ inj_cnt, const int* __restrict__ inj_bucket,
             int inj_cap, int k_inj, uint64_t gen, const double* part_m, int mark_grid,
             double* part_c, unsigned* done, CycleCtl* ctl, int cond, int use_u01,
             double u01_arg, const CycleArgs* ca) {
    pdl_wait();
    if (ca) gen = ca->gen;
    __shared__ GatherSmem sm;
    __shared__ int s_wmax[kThreads / 32];
    __shared__ int s_m;
    __shared__ double s_out[kEstN];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const bool resample = !cond || ctl->resample_now;
    const bool valid = resample && ctl->w_total_fx != 0 && !ctl->w_bad;
    if (blockIdx.x == 0) {
        combine_staged<kEstN, kMarkGrid>(part_m, mark_grid, sm.pm, s_out);
        double qm[4];
        if (warp == 0) markley_mean_warp_call(&s_out[3], qm);
        if (tid == 0) {
            for (int q = 0; q < kEstN; ++q) ctl->est[q] = s_out[q];
            ctl->ess = s_out[13] > 0.0 ? 1.0 / s_out[13] : 0.0;
            ctl->est_partial = 0;
            for (int q = 0; q < 4; ++q) ctl->qmean[q] = qm[q];
            for (int q = 0; q < 3; ++q) ctl->cov_mean_p[q] = (float)s_out[q];
            for (int q = 0; q < 4; ++q) ctl->cov_mean_q[q] = (float)qm[q];
            if (resample && !valid) {
                ctl->resample_valid = 0;
                ctl->wmode = WMODE_UNIFORM;
            }
        }
        __syncthreads();  // sm is reused by the tiles
    }
    if (!valid) return;
    InjList& s_inj = sm.t.inj;
    int* s_anc = sm.t.anc;
    const int live = ctl->live;
    const Offsets of = offsets(ctl, n, use_u01, u01_arg);
    double corr[kCorrN] = {0.0, 0.0, 0.0};
    // the tiles go to blocks 1.. (block 0 combined the sums above), or to
    // block 0 when it is alone
    const int ntiles = ceil_div(n, kTile);
    const int workers = gridDim.x > 1 ? (int)gridDim.x - 1 : 1;
    const int first = gridDim.x > 1 ? (int)blockIdx.x - 1 : 0;
    for (int tile = first; tile >= 0 && tile < ntiles; tile += workers) {
        const long long o0 = (long long)tile * kTile;
        // the tile's injection draws: from its bucket, or (bucket overflow)
        // by scanning every draw in rounds below
        int m = 0;
        const int cnt = k_inj > 0 ? __ldcg(&inj_cnt[tile]) : 0;
        const bool overflow = cnt > inj_cap;
        if (tid < kTile / 32) s_inj.hit[tid] = 0u;
        __syncthreads();
        if (cnt > 0 && !overflow) {
            for (int e = tid; e < cnt; e += kThreads) {
                const int j = __ldcg(&inj_bucket[(size_t)tile * inj_cap + e]);
                const InjDraw d = inj_draw(of.lcg1, gen, j, n);
                const int loc = d.idx - (int)o0;
                s_inj.loc[e] = loc;
                s_inj.j[e] = j;
                s_inj.jx[e] = d.jx;
                s_inj.jy[e] = d.jy;
                s_inj.jz[e] = d.jz;
                atomicOr(&s_inj.hit[loc >> 5], 1u << (loc & 31));
            }
            m = cnt;
        }
        // ancestors of outputs [8t, 8t + 8): running maximum of the markers
        // (thread, then block); the markers read are reset for the next one
        const long long i0 = o0 + 8 * tid;
        int mk[8];
#pragma unroll
        for (int h = 0; h < 2; ++h) {
            int4 v4 = make_int4(-1, -1, -1, -1);
            const long long ib = i0 + 4 * h;
            if (ib + 4 <= n) {
                v4 = __ldcg(reinterpret_cast<const int4*>(marker + ib));
            } else {
                if (ib < n) v4.x = __ldcg(marker + ib);
                if (ib + 1 < n) v4.y = __ldcg(marker + ib + 1);
                if (ib + 2 < n) v4.z = __ldcg(marker + ib + 2);
            }
            mk[4 * h] = v4.x;
            mk[4 * h + 1] = v4.y;
            mk[4 * h + 2] = v4.z;
            mk[4 * h + 3] = v4.w;
        }
#pragma unroll
        for (int q = 0; q < 8; ++q)
            if (mk[q] >= 0) marker[i0 + q] = -1;
#pragma unroll
        for (int q = 1; q < 8; ++q) mk[q] = max(mk[q], mk[q - 1]);
        int x = mk[7];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const int y = __shfl_up_sync(~0u, x, d);
            if (lane >= d) x = max(x, y);
        }
        const int excl_w = __shfl_up_sync(~0u, x, 1);
        if (lane == 31) s_wmax[warp] = x;
        __syncthreads();  // also publishes the injection list
        int before = lane > 0 ? excl_w : -1;
        for (int k = 0; k < warp; ++k) before = max(before, s_wmax[k]);
#pragma unroll
        for (int q = 0; q < 8; ++q) s_anc[8 * tid + q] = min(max(max(mk[q], before), 0), n - 1);
        __syncthreads();
        if (record)
            for (int l = tid; l < kTile; l += kThreads)
                if (o0 + l < n) anc[o0 + l] = s_anc[l];
        // thread t copies outputs [4t, 4t + 4) and [1024 + 4t, 1024 + 4t + 4)
        // of the tile, the seven planes of four outputs at a time
#pragma unroll 1
        for (int h = 0; h < 2; ++h) {
            const int l0 = h * kGroup * kThreads + kGroup * tid;
            const long long ib = o0 + l0;
            float v[7][kGroup];
            int a[kGroup];
#pragma unroll
            for (int q = 0; q < kGroup; ++q) a[q] = s_anc[l0 + q];
#pragma unroll
            for (int c = 0; c < 7; ++c) {
                const float* sp = plane(pb, live, c);
#pragma unroll
                for (int q = 0; q < kGroup; ++q) v[c][q] = sp[a[q]];
            }
            // the tile's injection draws on these outputs (the bucket's, or
            // all draws in rounds on a bucket overflow)
            if (m > 0 && ((s_inj.hit[l0 >> 5] >> (l0 & 31)) & 0xFu))
                apply_draws(s_inj, m, l0, v[0], v[1], v[2], corr);
            if (overflow) {
                // rounds of kInjChunk draws, the round's hits on this tile
                // compacted in draw order and applied in that order
                // (block-uniform: every thread takes the same rounds)
                for (int base = 0; base < k_inj; base += kInjChunk) {
                    __syncthreads();
                    const int j = base + tid;
                    InjDraw d{};
                    bool hit = false;
                    if (j < k_inj) {
                        d = inj_draw(of.lcg1, gen, j, n);
                        hit = d.idx >= o0 && d.idx < o0 + kTile;
                    }
                    const unsigned bal = __ballot_sync(~0u, hit);
                    if (lane == 0) s_inj.j[warp] = __popc(bal);  // counts, then offsets
                    __syncthreads();
                    if (tid == 0) {
                        int off = 0;
                        for (int k = 0; k < kThreads / 32; ++k) {
                            const int cw = s_inj.j[k];
                            s_inj.j[k] = off;
                            off += cw;
                        }
                        s_m = off;
                    }
                    __syncthreads();
                    const int off = s_inj.j[warp] + __popc(bal & ((1u << lane) - 1u));
                    __syncthreads();
                    if (hit) {
                        s_inj.loc[off] = d.idx - (int)o0;
                        s_inj.j[off] = j;
                        s_inj.jx[off] = d.jx;
                        s_inj.jy[off] = d.jy;
                        s_inj.jz[off] = d.jz;
                    }
                    __syncthreads();
                    apply_draws(s_inj, s_m, l0, v[0], v[1], v[2], corr);
                }
                __syncthreads();
            }
            if (ib + kGroup <= n) {
#pragma unroll
                for (int c = 0; c < 7; ++c)
                    reinterpret_cast<float4*>(plane(pb, 1 - live, c))[ib >> 2] =
                        make_float4(v[c][0], v[c][1], v[c][2], v[c][3]);
            } else {
#pragma unroll
                for (int c = 0; c < 7; ++c)
#pragma unroll
                    for (int q = 0; q < kGroup; ++q)
                        if (ib + q < n) plane(pb, 1 - live, c)[ib + q] = v[c][q];
            }
        }
        if (tid == 0 && k_inj > 0) inj_cnt[tile] = 0;  // the bucket is consumed
        __syncthreads();  // s_anc and s_inj are reused by the next tile
    }
    if (!block_partial_last<kCorrN>(corr, part_c, done)) return;
    __threadfence();
    combine_staged<kCorrN, kGatherGrid>(part_c, gridDim.x, sm.pc, s_out);
    if (tid == 0) {
        const double wd = (double)(1.0f / (float)n);
        for (int q = 0; q < kCorrN; ++q) {
            // block 0's sums are visible: it finished before this block
            const double e = __ldcg(&ctl->est[q]) + wd * s_out[q];
            ctl->est[q] = e;
            ctl->cov_mean_p[q] = (float)e;
        }
        ctl->lcg_next = of.lcg1;
        ctl->total_fx = of.T;
        ctl->total = of.total;
        ctl->step = of.step;
        ctl->u0 = of.u0;
        ctl->live = 1 - live;
        ctl->resampled = 1;
        ctl->lcg = of.lcg1;
        ctl->resample_valid = 1;
        ctl->wmode = WMODE_UNIFORM;
        *done = 0u;
    }
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

int resample_tiles(int n) { return ceil_div(n, kTile); }

int resample_part_doubles(int) { return kEstN * kMarkGrid + kCorrN * kGatherGrid; }

int ensure_inject_buckets(PfHandle* h, int k) {
    if (k <= 0) return 0;
    const int tiles = resample_tiles(h->n);
    // expected draws per tile k * kTile / n; room for four times that
    const long long expect = ((long long)k * kTile + h->n - 1) / h->n;
    const int cap =
        (int)std::min<long long>(kThreads, std::max<long long>(64, 4 * expect + 32));
    if (h->d_inj_bucket && h->inj_cap >= cap) return 0;
    cudaFree(h->d_inj_bucket);
    h->d_inj_bucket = nullptr;
    h->inj_cap = 0;
    PFB_CK(cudaMalloc((void**)&h->d_inj_bucket, (size_t)tiles * cap * sizeof(int)));
    h->inj_cap = cap;
    return 0;
}

// With dargs set (graph capture) the generation comes from device memory at
// replay time.  The estimate sums of the cloud the call ends with (and its
// Markley mean) are in the control block afterwards, resample or not.
int launch_resample_est(PfHandle* h, float inject_ratio, bool cond_on_ctl, bool use_u01,
                        double u01, const CycleArgs* dargs) {
    const int n = h->n;
    // The weight total and the prefixes come from the weight pass; run one
    // when the weights changed since the last.
    if (!h->prefix_valid && launch_weight_prefix(h, false, 0.0)) return -1;
    const int cond = cond_on_ctl ? 1 : 0;
    // k = floor(ratio * n) with the reference's f32 product
    // (src/cuda/pf_kernels.cu:667-671).
    int k = (inject_ratio > 0.f) ? (int)(inject_ratio * (float)n) : 0;
    if (k > n) k = n;
    if (ensure_inject_buckets(h, k)) return -1;
    const int mark_grid = std::min(ceil_div(n, kScanTile), kMarkGrid);
    // one block more than the tiles it copies: block 0 combines the sums
    const int gather_grid = std::min(resample_tiles(n) + 1, kGatherGrid);
    double* part_m = h->d_part;
    double* part_c = h->d_part + (size_t)kEstN * kMarkGrid;
    {
        KernelScope ks(h, KK_SCAN);
        PFB_CK(launch_pdl(k_mark, mark_grid, kThreads, 0, h->stream, plane_base(h), n,
                          h->d_w, h->d_ll, h->d_wprefix, h->d_marker, h->d_inj_cnt,
                          h->d_inj_bucket, h->inj_cap, k, h->gen, part_m, h->d_ctl, cond,
                          use_u01 ? 1 : 0, u01, dargs));
    }
    PFB_KL();
    {
        KernelScope ks(h, KK_GATHER);
        PFB_CK(launch_pdl(k_gather, gather_grid, kThreads, 0, h->stream, plane_base(h), n,
                          h->d_marker, h->d_anc, h->record_anc ? 1 : 0, h->d_inj_cnt,
                          h->d_inj_bucket, h->inj_cap, k, h->gen, (const double*)part_m,
                          mark_grid, part_c, h->d_done + 4, h->d_ctl, cond,
                          use_u01 ? 1 : 0, u01, dargs));
    }
    PFB_KL();
    h->anc_valid = true;
    // The weights are uniform afterwards; the next weight pass recomputes
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
