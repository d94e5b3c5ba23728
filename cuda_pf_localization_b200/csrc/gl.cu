// gl.cu — CBGL-style global localization (Filotheou, arXiv:2307.14247) on
// the B200: uniform hypothesis dispersion, DDA raycast + CAER scoring, and
// bottom-k selection, behind the pfgl_* C-ABI.
//
// Device layout
//   grid  (W+2) x (H+2) bytes, row-major, row 0 = lowest y: 0 free,
//         1 occupied (any nonzero input byte), 2 = the one-cell border that
//         stands for "outside the map".  A ray that steps onto the border
//         returns rmax, exactly like the reference's bounds test after each
//         step (src/cuda/pf_kernels.cu:797-806), so the inner loop needs one
//         byte load and no bounds compares.
//   free  int2 list of free cells in row-major order (deterministic, the
//         order crates/pf_core/src/global_loc.rs:365-368 uses).
//   hyp   n x (x, y, theta) f32;  caer  n f32;  keys  n u64 composite keys.
//
// Scoring: persistent CTAs copy the padded grid and the real scan into shared
// memory once; each warp owns one hypothesis at a time and lanes cast
// consecutive rays (neighbouring rays have similar lengths, which keeps the
// DDA loops of a warp in step).  The DDA arithmetic is the reference's f32
// sequence (src/cuda/pf_kernels.cu:774-808) so per-ray distances agree bit
// for bit; only the order of the CAER sum differs (lane-sequential, then an
// xor butterfly).
//
// Early termination (pfgl_localize): the partial CAER of a hypothesis only
// grows (non-negative terms, monotone rounding), so a hypothesis whose
// partial sum already exceeds an upper bound of the final k-th best key can
// never enter the bottom-k.  The bound is the k-th best composite key of a
// fully scored seed batch, tightened after every chunk.  Selected results
// are identical to exhaustive scoring.
#include <limits.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <mutex>
#include <new>
#include <vector>

#include "gl_internal.h"

namespace pfb {

namespace {

constexpr int kThreads = 256;
constexpr int kWarps = kThreads / 32;
constexpr int kMaxSmem = 200 * 1024;

GlHandle* as_gl(void* h) { return static_cast<GlHandle*>(h); }

// ---------------------------------------------------------------- dispersion

// Uniform dispersion with the reference's mapping (src/cuda/pf_kernels.cu:
// 811-823): cell = free[floor(u3 * nfree)], in-cell offset (u0, u1), yaw
// -pi + 2 pi u2; the uniforms come from Philox4x32-10 keyed by the seed with
// counter (i, 0, 0, RNG_GL).
__global__ void k_gl_gen(int n, int n_yaw, int nfree, const int2* __restrict__ free_cells,
                         float ox, float oy, float res, uint64_t seed,
                         float* __restrict__ hyp, int p0) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= n) return;
    const int pl = i / n_yaw, j = i - pl * n_yaw;
    const int p = p0 + pl;  // global position index: the Philox counter
    const U4 r = philox4x32_10({(uint32_t)p, 0u, 0u, RNG_GL}, (uint32_t)seed,
                               (uint32_t)(seed >> 32));
    const float ux = u01_open(r.x), uy = u01_open(r.y), uz = u01_open(r.z),
                uw = u01_open(r.w);
    const int c = min((int)(uw * (float)nfree), nfree - 1);
    const int2 cell = free_cells[c];
    float th = -3.14159265f + 6.28318530f * uz;
    if (n_yaw > 1) th = th + (6.28318530f / (float)n_yaw) * (float)j;
    hyp[3 * i] = ox + ((float)cell.x + ux) * res;
    hyp[3 * i + 1] = oy + ((float)cell.y + uy) * res;
    hyp[3 * i + 2] = th;
}

// Dispersions of many queries: query q's n_pos x n_yaw hypotheses (k_gl_gen
// with seeds[q]) at [q * n_pos * n_yaw, ...).
__global__ void k_gl_gen_multi(int per_q, int n_yaw, int nfree,
                               const int2* __restrict__ free_cells, float ox, float oy,
                               float res, const uint64_t* __restrict__ seeds,
                               float* __restrict__ hyp) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i >= per_q) return;
    const int q = blockIdx.y;
    const uint64_t seed = seeds[q];
    const int p = i / n_yaw, j = i - p * n_yaw;
    const U4 r = philox4x32_10({(uint32_t)p, 0u, 0u, RNG_GL}, (uint32_t)seed,
                               (uint32_t)(seed >> 32));
    const float ux = u01_open(r.x), uy = u01_open(r.y), uz = u01_open(r.z),
                uw = u01_open(r.w);
    const int c = min((int)(uw * (float)nfree), nfree - 1);
    const int2 cell = free_cells[c];
    float th = -3.14159265f + 6.28318530f * uz;
    if (n_yaw > 1) th = th + (6.28318530f / (float)n_yaw) * (float)j;
    float* o = hyp + 3 * ((size_t)q * per_q + i);
    o[0] = ox + ((float)cell.x + ux) * res;
    o[1] = oy + ((float)cell.y + uy) * res;
    o[2] = th;
}

// ------------------------------------------------------------------ raycast

// CAER of one hypothesis by one warp, with rays handed out dynamically: a
// lane whose ray has ended takes the next unstarted ray of the hypothesis
// (restarts are batched until kRestart lanes are free), so the warp is not
// held by its longest ray.  The rays' crossing distances (ray_deltas: the
// sincos and the divisions) are computed first with all lanes busy, so a
// restart does neither; each ray's term |scan - raycast| then replaces them in
// the ray's shared-memory slot, and the total is summed in the fixed
// lane-sequential order
// (lane l adds rays l, l + 32, ..., then an xor butterfly), which does not
// depend on the assignment.
// With kPrune, the sum of the terms finished so far (any order) is compared
// with `bound` at every restart and -1 is returned once it exceeds it; the
// caller's bound includes a margin for the rounding difference between that
// partial order and the final one.
constexpr int kScoreThreads = 768;
constexpr int kScoreWarps = kScoreThreads / 32;
// a launch keeps at least this many hypotheses per block on average, so a
// small batch still reaches every SM without each block copying the grid
// for a handful of warps
constexpr int kMinScoreWarps = 8;
constexpr int kChunk = 12;   // DDA steps between warp votes
constexpr int kRestart = 8;  // free lanes that trigger a restart round

template <bool kPrune>
__device__ __forceinline__ float warp_caer(const unsigned char* __restrict__ g,
                                           const GridView& gv, int Hp, float x,
                                           float y, float th,
                                           const float* __restrict__ sc, int nrays,
                                           float rmax, float span,
                                           float* __restrict__ term,
                                           float2* __restrict__ dirs, float bound) {
    const int lane = threadIdx.x & 31;
    const unsigned lt = (1u << lane) - 1u;
    int start = 0;
    float frx = 0.f, fry = 0.f;
    if (!start_cell(gv, x, y, start, frx, fry)) {
        float acc = 0.f;
        for (int r = lane; r < nrays; r += 32) acc += fabsf(sc[r] - rmax);
        return warp_sum_f(acc);
    }
    const bool long_rays = gv.Wp + Hp > 8192;
    // ray directions of this hypothesis as signed crossing distances, all
    // lanes busy
    for (int r = lane; r < nrays; r += 32) {
        float dx, dy;
        sincosf(ray_angle(th, r, nrays, span), &dy, &dx);
        dirs[r] = ray_deltas(dx, dy, gv.res);
    }
    __syncwarp();
    Ray ray;
    int r = lane;
    bool active = r < nrays;
    ray.v = 1u;
    if (active) ray_init_deltas(ray, gv.Wp, start, frx, fry, dirs[r]);
    float lane_acc = 0.f;
    int next = 32;
    for (;;) {
#pragma unroll
        for (int k = 0; k < kChunk; ++k)
            if (ray.v == 0u) ray_step(ray, g);
        const unsigned done = __ballot_sync(~0u, active && ray.v != 0u);
        const unsigned moving = __ballot_sync(~0u, active && ray.v == 0u);
        if (moving != 0u && __popc(done) < kRestart) continue;
        if (active && ray.v != 0u) {
            const float t =
                fabsf(sc[r] - ray_result(ray, gv.Wp, start, rmax, long_rays));
            term[2 * r] = t;  // the ray's direction slot, no longer needed
            lane_acc += t;
            const int nr = next + __popc(done & lt);
            if (nr < nrays) {
                r = nr;
                ray_init_deltas(ray, gv.Wp, start, frx, fry, dirs[r]);
            } else {
                active = false;
            }
        }
        next += __popc(done);
        if (kPrune && warp_sum_f(lane_acc) > bound) return -1.0f;
        if (!__any_sync(~0u, active)) break;
    }
    __syncwarp();
    float acc = 0.f;
    for (int rr = lane; rr < nrays; rr += 32) acc += term[2 * rr];
    return warp_sum_f(acc);
}

// Shared memory of the scorers: [padded grid (kSmem)] [scan] [per-warp ray
// slots: the direction of each ray, then its CAER term once it has ended].
template <bool kSmem>
__device__ __forceinline__ void score_setup(const GridView& gv, int grid_bytes,
                                            const float* scan, int nrays,
                                            const unsigned char*& g,
                                            const float*& sc, float*& term,
                                            float2*& dirs) {
    extern __shared__ __align__(16) unsigned char smem[];
    const int gbytes = kSmem ? grid_bytes : 0;
    float* s_scan = reinterpret_cast<float*>(smem + gbytes);
    if (kSmem) {
        const int nv = grid_bytes / 16;
        const uint4* src = reinterpret_cast<const uint4*>(gv.cells);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (int k = threadIdx.x; k < nv; k += blockDim.x) dst[k] = __ldg(&src[k]);
    }
    for (int k = threadIdx.x; k < nrays; k += blockDim.x) s_scan[k] = scan[k];
    __syncthreads();
    g = kSmem ? smem : gv.cells;
    sc = s_scan;
    float2* slots = reinterpret_cast<float2*>(s_scan + ((nrays + 1) & ~1));
    dirs = slots + (size_t)(threadIdx.x >> 5) * nrays;
    term = reinterpret_cast<float*>(dirs);
}

// CAER of hypotheses [0, nh): one warp per hypothesis, static striding.
template <bool kSmem>
__global__ void __launch_bounds__(kScoreThreads, 2)
    k_gl_score(GridView gv, int grid_bytes, const float* __restrict__ hyp,
               int nh, const float* __restrict__ scan, int nrays, float rmax,
               float span, float* __restrict__ caer) {
    const unsigned char* g;
    const float* sc;
    float* term;
    float2* dirs;
    score_setup<kSmem>(gv, grid_bytes, scan, nrays, g, sc, term, dirs);
    const int Hp = gv.H + 2;
    // hypotheses striped across the blocks first (warp w of block b takes
    // b + w * gridDim.x, ...), so a batch smaller than the grid's warps is
    // spread evenly over the SMs
    const int gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int nw = gridDim.x * kScoreWarps;
    for (int h = gw; h < nh; h += nw) {
        const float c = warp_caer<false>(g, gv, Hp, hyp[3 * h], hyp[3 * h + 1],
                                         hyp[3 * h + 2], sc, nrays, rmax, span,
                                         term, dirs, 0.f);
        if ((threadIdx.x & 31) == 0) caer[h] = c;
        __syncwarp();
    }
}

// DDA cell visits of every (hypothesis, ray) pair, one thread each: the
// scorer's start cell, ray directions and stepping, so the count is exactly
// the number of cell steps the scorer takes for these hypotheses (the
// algorithmic work unit of CAER scoring).  Diagnostic, not timed.
__global__ void __launch_bounds__(kThreads)
    k_gl_count_visits(GridView gv, const float* __restrict__ hyp, int nh, int nrays,
                      float span, unsigned long long* total) {
    const long long t = (long long)blockIdx.x * kThreads + threadIdx.x;
    unsigned long long steps = 0;
    if (t < (long long)nh * nrays) {
        const int h = (int)(t / nrays), r = (int)(t % nrays);
        int start = 0;
        float frx = 0.f, fry = 0.f;
        if (start_cell(gv, hyp[3 * h], hyp[3 * h + 1], start, frx, fry)) {
            float dx, dy;
            sincosf(ray_angle(hyp[3 * h + 2], r, nrays, span), &dy, &dx);
            Ray ray;
            ray_init(ray, gv.Wp, start, frx, fry, dx, dy, gv.res);
            do {
                ray_step(ray, gv.cells);
                ++steps;
            } while (ray.v == 0u);
        }
    }
    __shared__ unsigned long long s_w[kWarps];
    unsigned long long v = steps;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = v;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long b = 0;
        for (int k = 0; k < kWarps; ++k) b += s_w[k];
        atomicAdd(total, b);
    }
}

// CAER value of a composite key (inverse of composite_key's high word).
__device__ __forceinline__ float key_to_float(uint64_t key) {
    const int o = (int)((uint32_t)(key >> 32) ^ 0x80000000u);
    return __int_as_float(o >= 0 ? o : (o ^ 0x7FFFFFFF));
}

// Pruned scorer for hypotheses [h0, h1).  A hypothesis is dropped once the
// sum of its finished terms exceeds tau_f (1 + margin): with n non-negative
// terms, any two summation orders agree to within about 2 n 2^-24 relative,
// so such a hypothesis ends above tau_f and can never enter the bottom-k.
// The CAER of every hypothesis that is not dropped is the exhaustive
// scorer's value; survivors (final key <= tau) are appended to cand.
template <bool kSmem>
__global__ void __launch_bounds__(kScoreThreads, 2)
    k_gl_score_pruned(GridView gv, int grid_bytes, const float* __restrict__ hyp,
                      int h0, int h1, const float* __restrict__ scan, int nrays,
                      float rmax, float span, float* __restrict__ caer,
                      uint64_t* __restrict__ cand, GlCtl* ctl, int cand_cap) {
    const unsigned char* g;
    const float* sc;
    float* term;
    float2* dirs;
    score_setup<kSmem>(gv, grid_bytes, scan, nrays, g, sc, term, dirs);
    const int Hp = gv.H + 2;
    const unsigned long long tau = ctl->tau;
    const float tau_f = key_to_float(tau);
    const float bound = tau_f * (1.0f + 4.0f * (float)nrays * 5.9604645e-8f + 1e-6f);
    const int lane = threadIdx.x & 31;
    // hypotheses striped across the blocks first (warp w of block b takes
    // b + w * gridDim.x, ...), so a batch smaller than the grid's warps is
    // spread evenly over the SMs
    const int gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int nw = gridDim.x * kScoreWarps;
    for (int h = h0 + gw; h < h1; h += nw) {
        const float total = warp_caer<true>(g, gv, Hp, hyp[3 * h], hyp[3 * h + 1],
                                            hyp[3 * h + 2], sc, nrays, rmax, span,
                                            term, dirs, bound);
        if (lane == 0) {
            caer[h] = total;  // -1 when dropped (not scored)
            if (total >= 0.f) {
                const uint64_t key = composite_key(total, (uint32_t)h);
                if (key <= tau) {
                    const unsigned slot = atomicAdd(&ctl->n_cand, 1u);
                    if ((int)slot < cand_cap) cand[slot] = key;
                }
            }
        }
        __syncwarp();
    }
}

// CAER of the hypotheses of many queries in one launch (exhaustive): the
// hypotheses of query q are [q * per_q, (q + 1) * per_q) and its scan is
// scans + q * nrays in global memory (each ray's term reads one scan value
// when the ray ends; the scan stays L1-resident).  Per hypothesis the same
// warp_caer as the single-query scorer, so every CAER equals the single-query
// scorer's value bit for bit.  Shared memory: [padded grid (kSmem)] [per-warp
// ray slots].
template <bool kSmem>
__global__ void __launch_bounds__(kScoreThreads, 2)
    k_gl_score_multi(GridView gv, int grid_bytes, const float* __restrict__ hyp,
                     int nh, int per_q, const float* __restrict__ scans, int nrays,
                     float rmax, float span, float* __restrict__ caer) {
    extern __shared__ __align__(16) unsigned char smem[];
    if (kSmem) {
        const int nv = grid_bytes / 16;
        const uint4* src = reinterpret_cast<const uint4*>(gv.cells);
        uint4* dst = reinterpret_cast<uint4*>(smem);
        for (int k = threadIdx.x; k < nv; k += blockDim.x) dst[k] = __ldg(&src[k]);
    }
    __syncthreads();
    const unsigned char* g = kSmem ? smem : gv.cells;
    float2* dirs = reinterpret_cast<float2*>(smem + (kSmem ? grid_bytes : 0)) +
                   (size_t)(threadIdx.x >> 5) * nrays;
    float* term = reinterpret_cast<float*>(dirs);
    const int Hp = gv.H + 2;
    const int gw = (threadIdx.x >> 5) * gridDim.x + blockIdx.x;
    const int nw = gridDim.x * kScoreWarps;
    for (int h = gw; h < nh; h += nw) {
        const float* sc = scans + (size_t)(h / per_q) * nrays;
        const float c = warp_caer<false>(g, gv, Hp, hyp[3 * h], hyp[3 * h + 1],
                                         hyp[3 * h + 2], sc, nrays, rmax, span, term,
                                         dirs, 0.f);
        if ((threadIdx.x & 31) == 0) caer[h] = c;
        __syncwarp();
    }
}

// ------------------------------------------------------------- radix sort
// Stable LSD radix sort of 64-bit composite keys on their high 32 bits
// (8-bit digits, 4 passes).  The low word is the hypothesis index and the
// input is in index order, so stability yields (CAER, index) order.

constexpr int kRsItems = 8;
constexpr int kRsTile = kThreads * kRsItems;  // 2048

__global__ void k_make_keys(const float* __restrict__ caer, int n,
                            uint64_t* __restrict__ keys) {
    const int i = blockIdx.x * kThreads + threadIdx.x;
    if (i < n) keys[i] = composite_key(caer[i], (uint32_t)i);
}

__global__ void __launch_bounds__(kThreads)
    k_rs_hist(const uint64_t* __restrict__ keys, int n, int shift,
              unsigned* __restrict__ hist, int nb) {
    __shared__ unsigned s_cnt[256];
    s_cnt[threadIdx.x] = 0;
    __syncthreads();
    const int base = blockIdx.x * kRsTile;
    for (int k = 0; k < kRsItems; ++k) {
        const int i = base + k * kThreads + threadIdx.x;
        if (i < n) atomicAdd(&s_cnt[(keys[i] >> shift) & 255u], 1u);
    }
    __syncthreads();
    hist[threadIdx.x * nb + blockIdx.x] = s_cnt[threadIdx.x];
}

// Exclusive scan of `total` counters in place, one block of 1024 threads.
__global__ void __launch_bounds__(1024) k_rs_scan(unsigned* hist, int total) {
    __shared__ unsigned s_w[32];
    __shared__ unsigned s_carry;
    if (threadIdx.x == 0) s_carry = 0;
    __syncthreads();
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    for (int base = 0; base < total; base += 1024) {
        const int i = base + threadIdx.x;
        const unsigned v = i < total ? hist[i] : 0u;
        unsigned x = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const unsigned y = __shfl_up_sync(~0u, x, d);
            if (lane >= d) x += y;
        }
        if (lane == 31) s_w[warp] = x;
        __syncthreads();
        if (warp == 0) {
            unsigned wv = s_w[lane];
            unsigned z = wv;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const unsigned y = __shfl_up_sync(~0u, z, d);
                if (lane >= d) z += y;
            }
            s_w[lane] = z - wv;
        }
        __syncthreads();
        const unsigned carry = s_carry;
        if (i < total) hist[i] = carry + s_w[warp] + x - v;
        __syncthreads();
        if (threadIdx.x == 1023) s_carry = carry + s_w[warp] + x;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(kThreads)
    k_rs_scatter(const uint64_t* __restrict__ in, uint64_t* __restrict__ out,
                 int n, int shift, const unsigned* __restrict__ hist, int nb) {
    __shared__ unsigned s_wc[kWarps][256];
    __shared__ unsigned s_base[256];
    __shared__ unsigned s_goff[256];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    s_base[tid] = 0;
    s_goff[tid] = hist[tid * nb + blockIdx.x];
    const unsigned lt = (1u << lane) - 1u;
    const int base = blockIdx.x * kRsTile;
    for (int k = 0; k < kRsItems; ++k) {
        for (int w = 0; w < kWarps; ++w) s_wc[w][tid] = 0;
        __syncthreads();
        const int i = base + k * kThreads + tid;
        const bool ok = i < n;
        const uint64_t key = ok ? in[i] : 0ull;
        const unsigned d = ok ? (unsigned)((key >> shift) & 255u) : 256u + lane;
        const unsigned peers = __match_any_sync(~0u, d);
        const unsigned rank = __popc(peers & lt);
        if (ok && rank == 0) s_wc[warp][d] = __popc(peers);
        __syncthreads();
        {
            unsigned run = s_base[tid];
            for (int w = 0; w < kWarps; ++w) {
                const unsigned c = s_wc[w][tid];
                s_wc[w][tid] = run;
                run += c;
            }
            s_base[tid] = run;
        }
        __syncthreads();
        if (ok) out[s_goff[d] + s_wc[warp][d] + rank] = key;
        __syncthreads();
    }
}

// Sort n composite keys held in d_keys.  index_bits > 0 also sorts the low
// (index) word over that many bits, for inputs that are not in index order.
// Returns the buffer that holds the sorted keys.
uint64_t* radix_sort_keys(GlHandle* h, int n, int index_bits) {
    const int nb = ceil_div(n, kRsTile);
    const int need = 256 * nb;
    if (need > h->hist_cap) {
        cudaFree(h->d_hist);
        h->d_hist = nullptr;
        if (cudaMalloc((void**)&h->d_hist, sizeof(unsigned) * (size_t)need) !=
            cudaSuccess) {
            set_error("pf_b200: radix sort histogram allocation failed");
            return nullptr;
        }
        h->hist_cap = need;
    }
    std::vector<int> shifts;
    for (int s = 0; s < 32 && s < index_bits; s += 8) shifts.push_back(s);
    for (int s = 32; s < 64; s += 8) shifts.push_back(s);
    uint64_t* a = h->d_keys;
    uint64_t* b = h->d_keys_alt;
    for (int shift : shifts) {
        k_rs_hist<<<nb, kThreads, 0, h->stream>>>(a, n, shift, h->d_hist, nb);
        k_rs_scan<<<1, 1024, 0, h->stream>>>(h->d_hist, need);
        k_rs_scatter<<<nb, kThreads, 0, h->stream>>>(a, b, n, shift, h->d_hist,
                                                     nb);
        std::swap(a, b);
    }
    if (cudaGetLastError() != cudaSuccess) {
        set_error("pf_b200: radix sort launch failed");
        return nullptr;
    }
    return a;
}

int index_bit_width(int n) {
    int b = 0;
    while (b < 32 && (1ull << b) < (unsigned long long)n) ++b;
    return b;
}

// ---------------------------------------------------------- small bottom-k
// For up to kSelMaxN keys and k <= kSelK, one block finds the k smallest
// composite keys by radix selection on the key range:
//   1. min and max of the keys (the max over scored keys only when dropped
//      hypotheses sort last and at least k are scored);
//   2. a 1024-bin histogram of (key - lo) >> sh over the current range
//      [lo, hi], with sh the smallest shift that maps the range onto 1024
//      bins; the prefix of the counts gives the bin b that holds the
//      remaining k-th smallest key;
//   3. when the keys of bins <= b (and those accepted at earlier levels) fit
//      the 2048-key buffer, they are sorted (bitonic network in shared
//      memory) and the first k written; otherwise the keys of bins < b are
//      accepted and the range narrows to bin b (at least 2^9 times smaller,
//      so at most eight levels: at shift 0 a bin holds one distinct key).
// The binning is monotone in the key, so the result is the k smallest keys
// in ascending order exactly, ties of CAER broken by the index word: the
// order the full radix sort gives, in one launch.

constexpr int kSelK = 128;
constexpr int kSelMaxN = 65536;
constexpr int kSelThreads = 1024;
constexpr int kSelBins = 1024;  // one per thread
constexpr int kSelCap = 2048;   // keys sorted at the end

// Ascending bitonic sort of m (a power of two) keys in shared memory, by the
// whole block.
__device__ void bitonic_sort_smem(uint64_t* s, int m) {
    for (int size = 2; size <= m; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            __syncthreads();
            for (int t = threadIdx.x; t < m / 2; t += blockDim.x) {
                const int i = 2 * t - (t & (stride - 1));
                const int j = i + stride;
                const bool up = (i & size) == 0;
                const uint64_t a = s[i], b = s[j];
                if ((a > b) == up) {
                    s[i] = b;
                    s[j] = a;
                }
            }
        }
    }
    __syncthreads();
}

// kFromCaer: the key of hypothesis i made from caer[i]; else keys[i].
// kDroppedLast: a negative CAER marks a hypothesis the pruned scorer dropped;
// its key sorts after every scored one (high word all ones, then index).
template <bool kFromCaer, bool kDroppedLast>
__device__ __forceinline__ uint64_t sel_key(const float* __restrict__ caer,
                                            const uint64_t* __restrict__ keys, int i) {
    if (kFromCaer) {
        const float c = caer[i];
        return (kDroppedLast && c < 0.f) ? (0xFFFFFFFFull << 32) | (uint32_t)i
                                         : composite_key(c, (uint32_t)i);
    }
    return keys[i];
}

// Exclusive prefix of one count per thread over a 1024-thread block.
__device__ __forceinline__ unsigned block_excl_scan(unsigned v, unsigned* s_w) {
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    unsigned x = v;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const unsigned y = __shfl_up_sync(~0u, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) s_w[w] = x;
    __syncthreads();
    if (w == 0) {
        unsigned t = s_w[lane];
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(~0u, t, o);
            if (lane >= o) t += y;
        }
        s_w[lane] = t;
    }
    __syncthreads();
    return (w > 0 ? s_w[w - 1] : 0u) + x - v;
}

__device__ __forceinline__ uint64_t warp_min_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = min(v, (uint64_t)__shfl_xor_sync(~0u, v, o));
    return v;
}

__device__ __forceinline__ uint64_t warp_max_u64(uint64_t v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = max(v, (uint64_t)__shfl_xor_sync(~0u, v, o));
    return v;
}

// The k smallest of n keys, ascending, into out[0, k) (out[j] = ~0 for
// j >= n).  n_dev (optional): the key count in device memory, at most n.
// Segmented form: block b selects from the segment starting at element
// b * seg_stride of caer / keys (counts n_dev[b]) into out[b * k, b * k + k);
// the index word of a key is the element's index within its segment.
template <bool kFromCaer, bool kDroppedLast>
__global__ void __launch_bounds__(kSelThreads)
    k_select_small(const float* __restrict__ caer, const uint64_t* __restrict__ keys,
                   int n, const unsigned* n_dev, int k, uint64_t* __restrict__ out,
                   int seg_stride) {
    __shared__ unsigned s_hist[kSelBins];
    __shared__ uint64_t s_list[kSelCap];
    __shared__ uint64_t s_red[3][32];
    __shared__ unsigned s_w[32], s_nv[32];
    __shared__ uint64_t s_lo, s_hi;
    __shared__ unsigned s_b, s_cb, s_hb, s_n;
    const size_t seg = blockIdx.x;
    if (caer) caer += seg * (size_t)seg_stride;
    if (keys) keys += seg * (size_t)seg_stride;
    out += seg * (size_t)k;
    if (n_dev) n = min(n, (int)min(n_dev[seg], 0x7FFFFFFFu));
    const int tid = threadIdx.x, lane = tid & 31, w = tid >> 5;
    const int kk = max(0, min(k, n));

    // 1. key range
    uint64_t mn = ~0ull, mx = 0, mxv = 0;
    unsigned nv = 0;
    for (int i = tid; i < n; i += kSelThreads) {
        const uint64_t key = sel_key<kFromCaer, kDroppedLast>(caer, keys, i);
        mn = min(mn, key);
        mx = max(mx, key);
        if (!kDroppedLast || (uint32_t)(key >> 32) != 0xFFFFFFFFu) {
            mxv = max(mxv, key);
            ++nv;
        }
    }
    mn = warp_min_u64(mn);
    mx = warp_max_u64(mx);
    mxv = warp_max_u64(mxv);
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) nv += __shfl_xor_sync(~0u, nv, o);
    if (lane == 0) {
        s_red[0][w] = mn;
        s_red[1][w] = mx;
        s_red[2][w] = mxv;
        s_nv[w] = nv;
    }
    __syncthreads();
    if (w == 0) {
        mn = warp_min_u64(s_red[0][lane]);
        mx = warp_max_u64(s_red[1][lane]);
        mxv = warp_max_u64(s_red[2][lane]);
        nv = s_nv[lane];
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) nv += __shfl_xor_sync(~0u, nv, o);
        if (lane == 0) {
            s_lo = mn;
            s_hi = nv >= (unsigned)kk ? mxv : mx;  // at least kk keys <= s_hi
        }
    }
    __syncthreads();

    // 2. narrow the range until the candidates fit the sort buffer
    uint64_t lo = s_lo, hi = s_hi;
    unsigned krem = (unsigned)kk, acc_n = 0, m = 0;
    bool done = kk == 0;
    for (int level = 0; level < 10 && !done; ++level) {
        const uint64_t range = hi - lo;
        const int sh = range < (uint64_t)kSelBins ? 0 : 54 - __clzll((long long)range);
        s_hist[tid] = 0u;
        __syncthreads();
        for (int i = tid; i < n; i += kSelThreads) {
            const uint64_t key = sel_key<kFromCaer, kDroppedLast>(caer, keys, i);
            if (key >= lo && key <= hi) atomicAdd(&s_hist[(unsigned)((key - lo) >> sh)], 1u);
        }
        __syncthreads();
        const unsigned hc = s_hist[tid];
        const unsigned cb = block_excl_scan(hc, s_w);
        if (cb < krem && krem <= cb + hc) {  // exactly one bin
            s_b = (unsigned)tid;
            s_cb = cb;
            s_hb = hc;
        }
        if (tid == 0) s_n = acc_n;
        __syncthreads();
        const unsigned b = s_b, cbb = s_cb, hb = s_hb;
        const bool last = acc_n + cbb + hb <= (unsigned)kSelCap;
        for (int i = tid; i < n; i += kSelThreads) {
            const uint64_t key = sel_key<kFromCaer, kDroppedLast>(caer, keys, i);
            if (key >= lo && key <= hi) {
                const unsigned bin = (unsigned)((key - lo) >> sh);
                if (bin < b || (last && bin == b)) s_list[atomicAdd(&s_n, 1u)] = key;
            }
        }
        __syncthreads();
        if (last) {
            m = acc_n + cbb + hb;
            done = true;
        } else {  // sh > 0 here: a bin of one key would have fitted
            acc_n += cbb;
            krem -= cbb;
            lo += (uint64_t)b << sh;
            const uint64_t top = lo + (((uint64_t)1 << sh) - 1);  // end of bin b
            if (top >= lo) hi = min(hi, top);  // else it wrapped: hi stays
        }
    }

    // 3. sort the candidates and write the first k
    int p = 2;
    while (p < (int)m) p <<= 1;
    for (int t = (int)m + tid; t < p; t += kSelThreads) s_list[t] = ~0ull;
    bitonic_sort_smem(s_list, p);
    for (int t = tid; t < k; t += kSelThreads)
        out[t] = (done && t < kk) ? s_list[t] : ~0ull;
}

bool small_select_ok(int n, int k) {
    return n > 0 && k > 0 && k <= kSelK && n <= kSelMaxN;
}

// The k smallest composite keys, ascending, in h->d_sel (needs
// small_select_ok(n, k)).  From caer[0, n) when keys is null.
// dropped_last: negative CAERs (hypotheses the pruned scorer dropped) last.
// n_dev: the key count in device memory (at most n), for keys only.
const uint64_t* small_select(GlHandle* h, const float* caer, const uint64_t* keys,
                             int n, int k, bool dropped_last = false,
                             const unsigned* n_dev = nullptr) {
    uint64_t* out = h->d_sel;
    if (keys)
        k_select_small<false, false><<<1, kSelThreads, 0, h->stream>>>(nullptr, keys, n,
                                                                      n_dev, k, out, 0);
    else if (dropped_last)
        k_select_small<true, true><<<1, kSelThreads, 0, h->stream>>>(caer, nullptr, n,
                                                                    nullptr, k, out, 0);
    else
        k_select_small<true, false><<<1, kSelThreads, 0, h->stream>>>(caer, nullptr, n,
                                                                     nullptr, k, out, 0);
    if (cudaGetLastError() != cudaSuccess) {
        set_error("pf_b200: bottom-k select launch failed");
        return nullptr;
    }
    return out;
}

__global__ void k_gather_topk(const uint64_t* __restrict__ keys, int k,
                              const float* __restrict__ hyp,
                              const float* __restrict__ caer, float* out3,
                              float* outc, int* outi) {
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j >= k) return;
    const int src = (int)(uint32_t)keys[j];
    out3[3 * j] = hyp[3 * src];
    out3[3 * j + 1] = hyp[3 * src + 1];
    out3[3 * j + 2] = hyp[3 * src + 2];
    outc[j] = caer[src];
    outi[j] = src;
}

// Bottom-k of many queries: out[q * k + j] from key q * k + j, whose index
// word is the hypothesis index within query q.  Keys beyond a query's count
// (all ones) give index -1 and CAER +inf.
__global__ void k_gather_topk_multi(const uint64_t* __restrict__ keys, int nq, int k,
                                    int per_q, const float* __restrict__ hyp,
                                    const float* __restrict__ caer, float* out3,
                                    float* outc, int* outi) {
    const int t = blockIdx.x * kThreads + threadIdx.x;
    if (t >= nq * k) return;
    const int q = t / k;
    const uint64_t key = keys[t];
    if (key == ~0ull) {
        out3[3 * t] = out3[3 * t + 1] = out3[3 * t + 2] = 0.f;
        outc[t] = INFINITY;
        outi[t] = -1;
        return;
    }
    const int loc = (int)(uint32_t)key;
    const size_t src = (size_t)q * per_q + loc;
    out3[3 * t] = hyp[3 * src];
    out3[3 * t + 1] = hyp[3 * src + 1];
    out3[3 * t + 2] = hyp[3 * src + 2];
    outc[t] = caer[src];
    outi[t] = loc;
}

// Start of the pruned passes: the k smallest keys of the seed batch (sorted)
// become the first k candidates and the k-th of them the pruning bound; the
// pruned scorer appends its survivors after them.
__global__ void k_seed_cand(const uint64_t* __restrict__ sorted, int k,
                            uint64_t* __restrict__ cand, GlCtl* ctl) {
    for (int t = threadIdx.x; t < k; t += blockDim.x) cand[t] = sorted[t];
    if (threadIdx.x == 0) {
        ctl->tau = sorted[k - 1];
        ctl->n_cand = (unsigned)k;
    }
}

// ------------------------------------------------------------ host helpers

int ensure_scan(GlHandle* h, const float* scan, int nrays) {
    if (nrays > h->scan_cap) {
        cudaFree(h->d_scan);
        h->d_scan = nullptr;
        PFB_CK(cudaMalloc((void**)&h->d_scan, sizeof(float) * (size_t)nrays));
        h->scan_cap = nrays;
    }
    PFB_CK(cudaMemcpyAsync(h->d_scan, scan, sizeof(float) * (size_t)nrays,
                           cudaMemcpyHostToDevice, h->stream));
    return 0;
}

template <bool kSmem>
int score_grid_size(size_t smem) {
    int per_sm = 0, sms = 0, dev = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gl_score<kSmem>,
                                                  kScoreThreads, smem);
    if (per_sm < 1) per_sm = 1;
    return sms * per_sm;
}

// Dynamic shared memory of a scorer launch; kSmem when the padded grid fits.
size_t score_smem(const GlHandle* h, int nrays, bool* grid_in_smem) {
    const size_t rest =
        sizeof(float) * (size_t)((nrays + 1) & ~1) + sizeof(float2) * (size_t)nrays * kScoreWarps;
    const size_t with_grid = (size_t)grid_bytes_padded(h) + rest;
    *grid_in_smem = with_grid <= (size_t)kMaxSmem;
    return *grid_in_smem ? with_grid : rest;
}

int launch_score(GlHandle* h, int nrays, float rmax, float span) {
    const int gb = grid_bytes_padded(h);
    bool in_smem = false;
    const size_t smem = score_smem(h, nrays, &in_smem);
    if (smem > (size_t)kMaxSmem) {
        set_error("pf_b200: pfgl_score: %d rays need too much shared memory", nrays);
        return -1;
    }
    const GridView gv = grid_view(h);
    const int warps_needed = h->nh;
    if (in_smem) {
        PFB_CK(cudaFuncSetAttribute(k_gl_score<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
        int grid = score_grid_size<true>(smem);
        grid = std::min(grid, ceil_div(warps_needed, kMinScoreWarps));
        k_gl_score<true><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, h->nh, h->d_scan, nrays, rmax, span, h->d_caer);
    } else {
        PFB_CK(cudaFuncSetAttribute(k_gl_score<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
        int grid = score_grid_size<false>(smem);
        grid = std::min(grid, ceil_div(warps_needed, kMinScoreWarps));
        k_gl_score<false><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, h->nh, h->d_scan, nrays, rmax, span, h->d_caer);
    }
    PFB_KL();
    return 0;
}

int launch_score_pruned(GlHandle* h, int h0, int h1, int nrays, float rmax,
                        float span) {
    const int gb = grid_bytes_padded(h);
    bool in_smem = false;
    const size_t smem = score_smem(h, nrays, &in_smem);
    if (smem > (size_t)kMaxSmem) {
        set_error("pf_b200: pfgl_localize: %d rays need too much shared memory", nrays);
        return -1;
    }
    const GridView gv = grid_view(h);
    const int warps_needed = h1 - h0;
    if (in_smem) {
        PFB_CK(cudaFuncSetAttribute(k_gl_score_pruned<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
        int grid = score_grid_size<true>(smem);
        grid = std::min(grid, ceil_div(warps_needed, kMinScoreWarps));
        k_gl_score_pruned<true><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, h0, h1, h->d_scan, nrays, rmax, span, h->d_caer,
            h->d_cand, h->d_ctl, h->cap_hyp);
    } else {
        PFB_CK(cudaFuncSetAttribute(k_gl_score_pruned<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize,
                                    (int)smem));
        int grid = score_grid_size<false>(smem);
        grid = std::min(grid, ceil_div(warps_needed, kMinScoreWarps));
        k_gl_score_pruned<false><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, h0, h1, h->d_scan, nrays, rmax, span, h->d_caer,
            h->d_cand, h->d_ctl, h->cap_hyp);
    }
    PFB_KL();
    return 0;
}

// Sort all current CAERs (index-ordered composite keys); returns the sorted
// buffer or nullptr.
uint64_t* sort_current(GlHandle* h) {
    k_make_keys<<<ceil_div(h->nh, kThreads), kThreads, 0, h->stream>>>(
        h->d_caer, h->nh, h->d_keys);
    return radix_sort_keys(h, h->nh, 0);
}

// Bound tightening between chunks of the pruned scorer: when the candidates
// (ctl->n_cand keys in cand) fit the block select, their k smallest (best)
// become the candidate list and the k-th of them the bound.  A hypothesis
// outside these k has k better ones and cannot reach the final bottom-k,
// and the new bound is still at least the final k-th best key.
__global__ void k_tighten(const uint64_t* __restrict__ best, int k,
                          uint64_t* __restrict__ cand, GlCtl* ctl, unsigned cap) {
    const unsigned nc = ctl->n_cand;
    __syncthreads();  // every thread has read n_cand before it changes
    if (nc > cap || nc < (unsigned)k) return;
    for (int t = threadIdx.x; t < k; t += blockDim.x) cand[t] = best[t];
    __syncthreads();
    if (threadIdx.x == 0) {
        ctl->n_cand = (unsigned)k;
        ctl->tau = best[k - 1];
    }
}

int tighten_bound(GlHandle* h, int k) {
    const int cap = std::min(kSelMaxN, h->cap_hyp);
    const uint64_t* best = small_select(h, nullptr, h->d_cand, cap, k, false,
                                        &h->d_ctl->n_cand);
    if (!best) return -1;
    k_tighten<<<1, 128, 0, h->stream>>>(best, k, h->d_cand, h->d_ctl, (unsigned)cap);
    PFB_KL();
    return 0;
}

// The k smallest (CAER, index) keys of the current CAERs, ascending: the
// block select when it applies, else the full sort.
const uint64_t* smallest_current(GlHandle* h, int k) {
    if (small_select_ok(h->nh, k)) return small_select(h, h->d_caer, nullptr, h->nh, k);
    return sort_current(h);
}

int copy_topk(GlHandle* h, const uint64_t* sorted, int k, float* out3k,
              float* caer_k, int* idx_k) {
    k_gather_topk<<<ceil_div(k, kThreads), kThreads, 0, h->stream>>>(
        sorted, k, h->d_hyp, h->d_caer, h->d_out, h->d_outc, h->d_outi);
    PFB_KL();
    h->last_k = k;
    if (out3k)
        PFB_CK(cudaMemcpyAsync(out3k, h->d_out, sizeof(float) * 3 * (size_t)k,
                               cudaMemcpyDeviceToHost, h->stream));
    if (caer_k)
        PFB_CK(cudaMemcpyAsync(caer_k, h->d_outc, sizeof(float) * (size_t)k,
                               cudaMemcpyDeviceToHost, h->stream));
    if (idx_k)
        PFB_CK(cudaMemcpyAsync(idx_k, h->d_outi, sizeof(int) * (size_t)k,
                               cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return k;
}


// Device scans of a batch of queries (grown on demand).
int ensure_scans(GlHandle* h, int count) {
    if (count > h->scans_cap) {
        cudaFree(h->d_scans);
        h->d_scans = nullptr;
        h->scans_cap = 0;
        PFB_CK(cudaMalloc((void**)&h->d_scans, sizeof(float) * (size_t)count));
        h->scans_cap = count;
    }
    return 0;
}

}  // namespace

// ------------------------------------------- entry points shared across units

int gl_upload_scan(GlHandle* h, const float* scan, int nrays) {
    return ensure_scan(h, scan, nrays);
}

int gl_topk_exhaustive(GlHandle* h, int nrays, float rmax, float span, int k,
                       float* out3k, float* caer_k, int* idx_k) {
    if (h->nh <= 0 || k <= 0) return -1;
    if (k > h->nh) k = h->nh;
    if (launch_score(h, nrays, rmax, span)) return -1;
    h->caer_valid = true;
    const uint64_t* sorted = smallest_current(h, k);
    if (!sorted) return -1;
    return copy_topk(h, sorted, k, out3k, caer_k, idx_k);
}

int gl_generate_range(GlHandle* h, int p0, int n_pos, int n_yaw, uint64_t seed) {
    if (h->nfree <= 0 || p0 < 0 || n_pos <= 0 || n_yaw <= 0) return -1;
    const long long n = (long long)n_pos * n_yaw;
    if (n > h->cap_hyp || (long long)p0 + n_pos > INT_MAX) return -1;
    h->nh = (int)n;
    k_gl_gen<<<ceil_div(h->nh, kThreads), kThreads, 0, h->stream>>>(
        h->nh, n_yaw, h->nfree, h->d_free, h->ox, h->oy, h->res, seed,
        h->d_hyp, p0);
    PFB_KL();
    h->caer_valid = false;
    return 0;
}

int gl_generate(GlHandle* h, int n_pos, int n_yaw, uint64_t seed) {
    return gl_generate_range(h, 0, n_pos, n_yaw, seed);
}

// Up to 64k hypotheses: a seed batch scored exhaustively, the bound set from
// its k-th best key on the device, the rest scored by the pruned scorer
// (dropped ones keep CAER -1), then the k smallest of the candidates: the
// seed's k best and the pruned scorer's survivors (key <= bound).  Every
// hypothesis whose CAER can reach the bottom-k is scored exactly and is a
// candidate (a hypothesis above the bound has the seed's k better ones), so
// the result equals exhaustive scoring.  Enqueued only; localize_small then
// copies the result with the one host synchronisation.
const uint64_t* gl_localize_small_keys(GlHandle* h, int nrays, float rmax,
                                       float ang_span, int k) {
    const int nh = h->nh;
    // seed batch: most of one round of the scorer grid's 7104 warps
    const int seed_n = std::min(nh, std::max(4 * k, 6144));
    h->nh = seed_n;
    const int rc = launch_score(h, nrays, rmax, ang_span);
    h->nh = nh;
    if (rc) return nullptr;
    if (seed_n == nh) {
        h->caer_valid = true;
        return small_select(h, h->d_caer, nullptr, nh, k);
    }
    const uint64_t* seed_sorted = small_select(h, h->d_caer, nullptr, seed_n, k);
    if (!seed_sorted) return nullptr;
    k_seed_cand<<<1, kSelK, 0, h->stream>>>(seed_sorted, k, h->d_cand, h->d_ctl);
    if (cudaGetLastError() != cudaSuccess) {
        set_error("pf_b200: bound launch failed");
        return nullptr;
    }
    if (launch_score_pruned(h, seed_n, nh, nrays, rmax, ang_span)) return nullptr;
    h->caer_valid = false;  // dropped hypotheses have no CAER
    // at most k + (nh - seed_n) <= nh candidates
    return small_select(h, nullptr, h->d_cand, nh, k, false, &h->d_ctl->n_cand);
}

bool gl_small_select_ok(int n, int k) { return small_select_ok(n, k); }

int gl_upload_scans(GlHandle* h, const float* scans, int nq, int nrays) {
    if (!scans || nq <= 0 || nrays <= 0) return -1;
    if (ensure_scans(h, nq * nrays)) return -1;
    PFB_CK(cudaMemcpyAsync(h->d_scans, scans, sizeof(float) * (size_t)nq * nrays,
                           cudaMemcpyHostToDevice, h->stream));
    return 0;
}

bool gl_batch_ok(const GlHandle* h, int nq, int per_q, int k) {
    return nq > 0 && per_q > 0 && k > 0 && k <= kSelK && per_q <= kSelMaxN &&
           (long long)nq * per_q <= h->cap_hyp && (long long)nq * k <= h->cap_hyp;
}

int gl_localize_batch_enqueue(GlHandle* h, int nq, int per_q, int nrays, float rmax,
                              float span, int k) {
    if (!gl_batch_ok(h, nq, per_q, k) || nq * nrays > h->scans_cap) {
        set_error("pf_b200: batch of %d queries x %d hypotheses (k %d) not supported", nq,
                  per_q, k);
        return -1;
    }
    const int nh = nq * per_q;
    h->nh = nh;
    const int gb = grid_bytes_padded(h);
    const size_t slots = sizeof(float2) * (size_t)nrays * kScoreWarps;
    const bool in_smem = (size_t)gb + slots <= (size_t)kMaxSmem;
    const size_t smem = in_smem ? gb + slots : slots;
    if (smem > (size_t)kMaxSmem) {
        set_error("pf_b200: %d rays need too much shared memory", nrays);
        return -1;
    }
    int dev = 0, sms = 0, per_sm = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const GridView gv = grid_view(h);
    if (in_smem) {
        PFB_CK(cudaFuncSetAttribute(k_gl_score_multi<true>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gl_score_multi<true>,
                                                      kScoreThreads, smem);
        const int grid = std::min(sms * std::max(per_sm, 1), ceil_div(nh, kMinScoreWarps));
        k_gl_score_multi<true><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, nh, per_q, h->d_scans, nrays, rmax, span, h->d_caer);
    } else {
        PFB_CK(cudaFuncSetAttribute(k_gl_score_multi<false>,
                                    cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_gl_score_multi<false>,
                                                      kScoreThreads, smem);
        const int grid = std::min(sms * std::max(per_sm, 1), ceil_div(nh, kMinScoreWarps));
        k_gl_score_multi<false><<<grid, kScoreThreads, smem, h->stream>>>(
            gv, gb, h->d_hyp, nh, per_q, h->d_scans, nrays, rmax, span, h->d_caer);
    }
    PFB_KL();
    h->caer_valid = true;
    k_select_small<true, false><<<nq, kSelThreads, 0, h->stream>>>(
        h->d_caer, nullptr, per_q, nullptr, k, h->d_keys, per_q);
    PFB_KL();
    k_gather_topk_multi<<<ceil_div(nq * k, kThreads), kThreads, 0, h->stream>>>(
        h->d_keys, nq, k, per_q, h->d_hyp, h->d_caer, h->d_out, h->d_outc, h->d_outi);
    PFB_KL();
    h->last_k = 0;  // d_out holds a batch, not one bottom-k
    return 0;
}

int gl_gather_topk(GlHandle* h, const uint64_t* sorted, int k) {
    k_gather_topk<<<ceil_div(k, kThreads), kThreads, 0, h->stream>>>(
        sorted, k, h->d_hyp, h->d_caer, h->d_out, h->d_outc, h->d_outi);
    PFB_KL();
    h->last_k = k;
    return 0;
}

int localize_small(GlHandle* h, int nrays, float rmax, float ang_span, int k,
                   float* out3k, float* caer_k, int* idx_k) {
    const uint64_t* sorted = gl_localize_small_keys(h, nrays, rmax, ang_span, k);
    if (!sorted) return -1;
    return copy_topk(h, sorted, k, out3k, caer_k, idx_k);
}

int gl_localize_loaded(GlHandle* h, int nrays, float rmax, float ang_span,
                       int k, float* out3k, float* caer_k, int* idx_k) {
    if (h->nh <= 0 || k <= 0) return -1;
    if (k > h->nh) k = h->nh;
    if (small_select_ok(h->nh, k))
        return localize_small(h, nrays, rmax, ang_span, k, out3k, caer_k, idx_k);
    const int nh = h->nh;
    // Seed batch scored exhaustively (two rounds of the scorer grid's 7104
    // warps on a 148-SM B200), then pruned chunks.
    const int seed_n = std::min(nh, std::max(4 * k, 14208));
    const int saved = h->nh;
    h->nh = seed_n;
    if (launch_score(h, nrays, rmax, ang_span)) return -1;
    const uint64_t* seed_sorted = smallest_current(h, k);
    h->nh = saved;
    if (!seed_sorted) return -1;
    if (seed_n == nh) {
        h->caer_valid = true;
        return copy_topk(h, seed_sorted, k, out3k, caer_k, idx_k);
    }
    // Pruning bound = k-th best key of the seed batch; candidates start with
    // the seed batch's best k.
    k_seed_cand<<<1, kSelK, 0, h->stream>>>(seed_sorted, k, h->d_cand, h->d_ctl);
    PFB_KL();
    // Chunks of the rest; between chunks the bound is tightened to the k-th
    // best key found so far (on the device, no host synchronisation).
    const int chunk = std::max(131072, ceil_div(nh - seed_n, 4));
    for (int c0 = seed_n; c0 < nh; c0 += chunk) {
        const int c1 = std::min(nh, c0 + chunk);
        if (launch_score_pruned(h, c0, c1, nrays, rmax, ang_span)) return -1;
        if (c1 < nh && k <= kSelK && tighten_bound(h, k)) return -1;
    }
    PFB_CK(cudaMemcpyAsync(h->h_ctl, h->d_ctl, sizeof(GlCtl),
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    int nc = (int)h->h_ctl->n_cand;
    if (nc > h->cap_hyp) {
        set_error("pf_b200: pfgl_localize candidate overflow");
        return -1;
    }
    // Sort the survivors (their keys already carry the index).
    PFB_CK(cudaMemcpyAsync(h->d_keys, h->d_cand, sizeof(uint64_t) * (size_t)nc,
                           cudaMemcpyDeviceToDevice, h->stream));
    const int kk2 = std::min(k, nc);
    const uint64_t* sorted = small_select_ok(nc, kk2)
                                 ? small_select(h, nullptr, h->d_keys, nc, kk2)
                                 : radix_sort_keys(h, nc, index_bit_width(nh));
    if (!sorted) return -1;
    h->caer_valid = false;  // pruned CAERs are not computed
    return copy_topk(h, sorted, std::min(k, nc), out3k, caer_k, idx_k);
}

}  // namespace pfb

using namespace pfb;

extern "C" {

void* pfgl_create(int W, int H, float res, float ox, float oy,
                  const unsigned char* occ, int cap_hyp) {
    clear_error();
    if (W <= 0 || H <= 0 || cap_hyp <= 0 || !occ) {
        set_error("pf_b200: pfgl_create: bad arguments");
        return nullptr;
    }
    GlHandle* h = new (std::nothrow) GlHandle();
    if (!h) return nullptr;
    h->W = W;
    h->H = H;
    h->Wp = W + 2;
    h->Hp = H + 2;
    h->res = res;
    h->ox = ox;
    h->oy = oy;
    h->cap_hyp = cap_hyp;
    // Host-side preparation: padded 0/1/2 grid and the row-major free list.
    std::vector<unsigned char> pad((size_t)h->Wp * h->Hp, 2);
    std::vector<int2> freel;
    h->host_grid.resize((size_t)W * H);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const unsigned char v = occ[(size_t)y * W + x] ? 1 : 0;
            h->host_grid[(size_t)y * W + x] = v;
            pad[(size_t)(y + 1) * h->Wp + (x + 1)] = v;
            if (!v) freel.push_back(make_int2(x, y));
        }
    h->nfree = (int)freel.size();
    const size_t gb = ((size_t)h->Wp * h->Hp + 15) / 16 * 16;
    bool ok = false;
    do {
        if (cudaGetDevice(&h->dev) != cudaSuccess) break;
        if (cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_grid, gb) != cudaSuccess) break;
        if (cudaMemset(h->d_grid, 2, gb) != cudaSuccess) break;
        if (cudaMemcpy(h->d_grid, pad.data(), pad.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_free,
                       sizeof(int2) * std::max<size_t>(1, freel.size())) !=
            cudaSuccess)
            break;
        if (!freel.empty() &&
            cudaMemcpy(h->d_free, freel.data(), sizeof(int2) * freel.size(),
                       cudaMemcpyHostToDevice) != cudaSuccess)
            break;
        const size_t c = (size_t)cap_hyp;
        if (cudaMalloc((void**)&h->d_hyp, 3 * c * sizeof(float)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_caer, c * sizeof(float)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_keys, c * sizeof(uint64_t)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_keys_alt, c * sizeof(uint64_t)) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_sel, (size_t)kSelK * sizeof(uint64_t)) !=
            cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_cand, c * sizeof(uint64_t)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_out, 3 * c * sizeof(float)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_outc, c * sizeof(float)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_outi, c * sizeof(int)) != cudaSuccess)
            break;
        if (cudaMalloc((void**)&h->d_ctl, sizeof(GlCtl)) != cudaSuccess) break;
        if (cudaMemset(h->d_ctl, 0, sizeof(GlCtl)) != cudaSuccess) break;
        if (cudaMallocHost((void**)&h->h_ctl, sizeof(GlCtl)) != cudaSuccess)
            break;
        ok = true;
    } while (0);
    if (!ok) {
        set_error("pf_b200: pfgl_create failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
        pfgl_destroy(h);
        return nullptr;
    }
    return h;
}

int pfgl_destroy(void* hv) {
    GlHandle* h = as_gl(hv);
    if (!h) return 0;
    if (h->stream) cudaStreamSynchronize(h->stream);
    cudaFree(h->d_grid);
    cudaFree(h->d_free);
    cudaFree(h->d_hyp);
    cudaFree(h->d_caer);
    cudaFree(h->d_keys);
    cudaFree(h->d_keys_alt);
    cudaFree(h->d_hist);
    cudaFree(h->d_scan);
    cudaFree(h->d_scans);
    cudaFree(h->d_out);
    cudaFree(h->d_outc);
    cudaFree(h->d_outi);
    cudaFree(h->d_cand);
    cudaFree(h->d_sel);
    cudaFree(h->d_ctl);
    cudaFreeHost(h->h_ctl);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return 0;
}

int pfgl_free_cells(void* hv) {
    GlHandle* h = as_gl(hv);
    return h ? h->nfree : -1;
}

int pfgl_generate(void* hv, int n, unsigned long long seed) {
    return pfgl_generate_yaws(hv, n, 1, seed);
}

int pfgl_generate_yaws(void* hv, int n_pos, int n_yaw, unsigned long long seed) {
    GlHandle* h = as_gl(hv);
    if (!h) return -1;
    return gl_generate(h, n_pos, n_yaw, seed);
}

int pfgl_generate_yaws_range(void* hv, int p0, int n_pos, int n_yaw,
                             unsigned long long seed) {
    GlHandle* h = as_gl(hv);
    if (!h) return -1;
    return gl_generate_range(h, p0, n_pos, n_yaw, seed);
}

int pfgl_localize_batch(void* hv, const float* scans, int nq, int nrays, float rmax,
                        float ang_span, int n_pos, int n_yaw,
                        const unsigned long long* seeds, int k, float* out3k,
                        float* caer_k, int* idx_k) {
    GlHandle* h = as_gl(hv);
    clear_error();
    if (!h || !scans || !seeds || nq <= 0 || nrays <= 0 || n_pos <= 0 || n_yaw <= 0 ||
        k <= 0 || h->nfree <= 0)
        return -1;
    const long long per = (long long)n_pos * n_yaw;
    if (per > INT_MAX) return -1;
    const int per_q = (int)per;
    if (k > per_q) k = per_q;
    const int chunk = (int)std::min<long long>(nq, h->cap_hyp / std::max(per_q, 1));
    if (!gl_batch_ok(h, std::max(chunk, 1), per_q, k) || chunk <= 0) {
        set_error("pf_b200: pfgl_localize_batch: %d hypotheses per query (k %d) exceed the "
                  "batch limits", per_q, k);
        return -1;
    }
    uint64_t* d_seeds = nullptr;
    PFB_CK(cudaMalloc((void**)&d_seeds, sizeof(uint64_t) * (size_t)chunk));
    int rc = 0;
    for (int q0 = 0; q0 < nq && rc == 0; q0 += chunk) {
        const int m = std::min(chunk, nq - q0);
        if (cudaMemcpyAsync(d_seeds, seeds + q0, sizeof(uint64_t) * (size_t)m,
                            cudaMemcpyHostToDevice, h->stream) != cudaSuccess ||
            gl_upload_scans(h, scans + (size_t)q0 * nrays, m, nrays)) {
            set_error("pf_b200: pfgl_localize_batch: input copy failed");
            rc = -1;
            break;
        }
        k_gl_gen_multi<<<dim3(ceil_div(per_q, kThreads), m), kThreads, 0, h->stream>>>(
            per_q, n_yaw, h->nfree, h->d_free, h->ox, h->oy, h->res, d_seeds, h->d_hyp);
        if (cudaGetLastError() != cudaSuccess) {
            set_error("pf_b200: pfgl_localize_batch: dispersion launch failed");
            rc = -1;
            break;
        }
        if (gl_localize_batch_enqueue(h, m, per_q, nrays, rmax, ang_span, k)) {
            rc = -1;
            break;
        }
        const size_t o = (size_t)q0 * k, mk = (size_t)m * k;
        if ((out3k && cudaMemcpyAsync(out3k + 3 * o, h->d_out, sizeof(float) * 3 * mk,
                                      cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) ||
            (caer_k && cudaMemcpyAsync(caer_k + o, h->d_outc, sizeof(float) * mk,
                                       cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) ||
            (idx_k && cudaMemcpyAsync(idx_k + o, h->d_outi, sizeof(int) * mk,
                                      cudaMemcpyDeviceToHost, h->stream) != cudaSuccess) ||
            cudaStreamSynchronize(h->stream) != cudaSuccess) {
            set_error("pf_b200: pfgl_localize_batch: %s",
                      cudaGetErrorString(cudaGetLastError()));
            rc = -1;
        }
    }
    cudaStreamSynchronize(h->stream);
    cudaFree(d_seeds);
    return rc ? -1 : k;
}

int pfgl_set_hyps(void* hv, const float* hyp3n, int n) {
    GlHandle* h = as_gl(hv);
    if (!h || !hyp3n || n <= 0 || n > h->cap_hyp) return -1;
    h->nh = n;
    PFB_CK(cudaMemcpyAsync(h->d_hyp, hyp3n, 3 * sizeof(float) * (size_t)n,
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    h->caer_valid = false;
    return 0;
}

int pfgl_get_hyps(void* hv, float* hyp3n) {
    GlHandle* h = as_gl(hv);
    if (!h || !hyp3n || h->nh <= 0) return -1;
    PFB_CK(cudaMemcpyAsync(hyp3n, h->d_hyp, 3 * sizeof(float) * (size_t)h->nh,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfgl_score(void* hv, const float* scan, int nrays, float rmax,
               float ang_span) {
    GlHandle* h = as_gl(hv);
    if (!h || h->nh <= 0 || !scan || nrays <= 0) return -1;
    if (ensure_scan(h, scan, nrays)) return -1;
    if (launch_score(h, nrays, rmax, ang_span)) return -1;
    h->caer_valid = true;
    return 0;
}

long long pfgl_count_visits(void* hv, int nrays, float ang_span) {
    GlHandle* h = as_gl(hv);
    if (!h || h->nh <= 0 || nrays <= 0) return -1;
    const GridView gv = grid_view(h);
    PFB_CK(cudaMemsetAsync(&h->d_ctl->visits, 0, sizeof(unsigned long long), h->stream));
    const long long pairs = (long long)h->nh * nrays;
    k_gl_count_visits<<<(unsigned)((pairs + kThreads - 1) / kThreads), kThreads, 0,
                        h->stream>>>(gv, h->d_hyp, h->nh, nrays, ang_span,
                                     &h->d_ctl->visits);
    PFB_KL();
    unsigned long long v = 0;
    PFB_CK(cudaMemcpyAsync(&v, &h->d_ctl->visits, sizeof v, cudaMemcpyDeviceToHost,
                           h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return (long long)v;
}

int pfgl_get_caer(void* hv, float* caer) {
    GlHandle* h = as_gl(hv);
    if (!h || !caer || h->nh <= 0 || !h->caer_valid) return -1;
    PFB_CK(cudaMemcpyAsync(caer, h->d_caer, sizeof(float) * (size_t)h->nh,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfgl_topk_ex(void* hv, int k, float* out3k, float* caer_k, int* idx_k) {
    GlHandle* h = as_gl(hv);
    if (!h || k <= 0 || h->nh <= 0 || !h->caer_valid) return -1;
    if (k > h->nh) k = h->nh;
    const uint64_t* sorted = smallest_current(h, k);
    if (!sorted) return -1;
    return copy_topk(h, sorted, k, out3k, caer_k, idx_k);
}

int pfgl_topk(void* hv, int k, float* out) {
    if (!out) return -1;
    return pfgl_topk_ex(hv, k, out, nullptr, nullptr);
}

int pfgl_topk_from_scores(void* hv, const float* caer, int n, int k,
                          int* idx_out) {
    GlHandle* h = as_gl(hv);
    if (!h || !caer || !idx_out || n <= 0 || k <= 0 || n > h->cap_hyp)
        return -1;
    if (k > n) k = n;
    PFB_CK(cudaMemcpyAsync(h->d_caer, caer, sizeof(float) * (size_t)n,
                           cudaMemcpyHostToDevice, h->stream));
    k_make_keys<<<ceil_div(n, kThreads), kThreads, 0, h->stream>>>(
        h->d_caer, n, h->d_keys);
    PFB_KL();
    const uint64_t* sorted = radix_sort_keys(h, n, 0);
    if (!sorted) return -1;
    std::vector<uint64_t> keys((size_t)k);
    PFB_CK(cudaMemcpyAsync(keys.data(), sorted, sizeof(uint64_t) * (size_t)k,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    for (int j = 0; j < k; ++j) idx_out[j] = (int)(uint32_t)keys[(size_t)j];
    h->caer_valid = false;  // d_caer now holds caller scores
    return k;
}

int pfgl_select_from_scores(void* hv, const float* caer, int n, int k,
                            int dropped_last, int* idx_out) {
    GlHandle* h = as_gl(hv);
    if (!h || !caer || !idx_out || n <= 0 || k <= 0 || n > h->cap_hyp) return -1;
    if (k > n) k = n;
    if (!small_select_ok(n, k)) {
        set_error("pf_b200: pfgl_select_from_scores: needs n <= %d and k <= %d",
                  kSelMaxN, kSelK);
        return -1;
    }
    PFB_CK(cudaMemcpyAsync(h->d_caer, caer, sizeof(float) * (size_t)n,
                           cudaMemcpyHostToDevice, h->stream));
    const uint64_t* sorted = small_select(h, h->d_caer, nullptr, n, k, dropped_last != 0);
    if (!sorted) return -1;
    std::vector<uint64_t> keys((size_t)k);
    PFB_CK(cudaMemcpyAsync(keys.data(), sorted, sizeof(uint64_t) * (size_t)k,
                           cudaMemcpyDeviceToHost, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    for (int j = 0; j < k; ++j) idx_out[j] = (int)(uint32_t)keys[(size_t)j];
    h->caer_valid = false;  // d_caer now holds caller scores
    return k;
}

int pfgl_localize(void* hv, const float* scan, int nrays, float rmax,
                  float ang_span, int k, float* out3k, float* caer_k,
                  int* idx_k) {
    GlHandle* h = as_gl(hv);
    if (!h || h->nh <= 0 || !scan || nrays <= 0 || k <= 0) return -1;
    if (gl_upload_scan(h, scan, nrays)) return -1;
    return gl_localize_loaded(h, nrays, rmax, ang_span, k, out3k, caer_k, idx_k);
}

const float* pfgl_topk_device(void* hv, int* k) {
    GlHandle* h = as_gl(hv);
    if (!h || h->last_k <= 0) return nullptr;
    if (k) *k = h->last_k;
    return h->d_out;
}

int pfgl_cell(void* hv, int cx, int cy) {
    GlHandle* h = as_gl(hv);
    if (!h || cx < 0 || cy < 0 || cx >= h->W || cy >= h->H) return -1;
    return h->host_grid[(size_t)cy * h->W + cx];
}

}  // extern "C"

// ------------------------------------------------ allocation-free bottom-k
//
// Some callers cannot allocate device memory at the time they need a
// bottom-k: a localization step inside a fixed-rate control loop (cudaMalloc
// and cudaFree can block for milliseconds and synchronise the device, which a
// real-time thread must not do), or an application that hands all device
// memory to its own pool allocator and forbids other allocations after
// start-up.  pfgl_topk_noalloc serves them: the caller passes the scores and
// the output buffer, and the working memory of the radix sort lives in the
// fixed array below, which is part of the library's device image.
//
// Limits and sharing:
//   * at most kNoAllocMaxN scores per call (larger inputs are rejected);
//   * every GPU that loads the library holds the array (1 MiB + 32 KiB)
//     until the process exits;
//   * all calls on a device share the array: calls whose work overlaps on the
//     GPU (different streams, or different host threads) race and corrupt
//     each other's results; serialise them on one stream;
//   * the array keeps the last call's contents; every word a call reads is
//     written earlier by the same call (keys, then each pass's histogram), so
//     nothing needs clearing between calls.
namespace pfb {
namespace noalloc {

constexpr int kNoAllocMaxN = 65536;
constexpr int kNoAllocBlocks = kNoAllocMaxN / kRsTile;  // 32 radix tiles
constexpr size_t kNoAllocKeyBytes = (size_t)kNoAllocMaxN * sizeof(uint64_t);
constexpr size_t kNoAllocBytes =
    2 * kNoAllocKeyBytes + 256 * (size_t)kNoAllocBlocks * sizeof(unsigned);

static __device__ __align__(256) unsigned char g_topk_scratch[kNoAllocBytes];

// Device address of g_topk_scratch per device, looked up once per device
// (host code must not use the symbol itself as a device pointer).
std::mutex g_scratch_mu;
std::vector<void*> g_scratch_addr;

void* scratch_address(int dev) {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if ((int)g_scratch_addr.size() <= dev) g_scratch_addr.resize(dev + 1, nullptr);
    if (!g_scratch_addr[dev]) {
        void* p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, g_topk_scratch);
        if (e != cudaSuccess) {
            set_error("pf_b200: pfgl_topk_noalloc: cudaGetSymbolAddress failed: %s",
                      cudaGetErrorString(e));
            return nullptr;
        }
        g_scratch_addr[dev] = p;
    }
    return g_scratch_addr[dev];
}

__global__ void k_keys_to_index(const uint64_t* __restrict__ sorted, int k,
                                int* __restrict__ idx) {
    const int j = blockIdx.x * kThreads + threadIdx.x;
    if (j < k) idx[j] = (int)(uint32_t)sorted[j];
}

}  // namespace noalloc
}  // namespace pfb

using namespace pfb::noalloc;

extern "C" int pfgl_topk_noalloc(const float* d_scores, int n, int k,
                                 int* d_idx, void* stream) {
    if (!d_scores || !d_idx || n <= 0 || k <= 0) {
        set_error("pf_b200: pfgl_topk_noalloc: bad arguments");
        return -1;
    }
    if (n > kNoAllocMaxN) {
        set_error("pf_b200: pfgl_topk_noalloc: n = %d exceeds the fixed scratch "
                  "capacity of %d scores", n, kNoAllocMaxN);
        return -1;
    }
    int dev = 0;
    PFB_CK(cudaGetDevice(&dev));
    unsigned char* base = static_cast<unsigned char*>(scratch_address(dev));
    if (!base) return -1;
    uint64_t* a = reinterpret_cast<uint64_t*>(base);
    uint64_t* b = reinterpret_cast<uint64_t*>(base + kNoAllocKeyBytes);
    unsigned* hist = reinterpret_cast<unsigned*>(base + 2 * kNoAllocKeyBytes);
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    if (k > n) k = n;
    const int nb = ceil_div(n, kRsTile);
    const int need = 256 * nb;
    k_make_keys<<<ceil_div(n, kThreads), kThreads, 0, s>>>(d_scores, n, a);
    for (int shift = 32; shift < 64; shift += 8) {
        k_rs_hist<<<nb, kThreads, 0, s>>>(a, n, shift, hist, nb);
        k_rs_scan<<<1, 1024, 0, s>>>(hist, need);
        k_rs_scatter<<<nb, kThreads, 0, s>>>(a, b, n, shift, hist, nb);
        std::swap(a, b);
    }
    k_keys_to_index<<<ceil_div(k, kThreads), kThreads, 0, s>>>(a, k, d_idx);
    PFB_KL();
    return k;
}
