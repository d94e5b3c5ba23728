// gl_internal.h — global-localization handle, the padded-grid raycaster and
// the entry points shared between the CBGL translation unit (gl.cu) and the
// learned proposal (gl_learned.cu).
//
// Device layout of a handle
//   grid  (W+2) x (H+2) bytes, row-major, row 0 = lowest y: 0 free,
//         1 occupied (any nonzero input byte), 2 = the one-cell border that
//         stands for "outside the map".
//   free  int2 list of free cells in row-major order.
//   hyp   cap_hyp x (x, y, theta) f32;  caer  cap_hyp f32;  keys  u64.
#pragma once

#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>

#include <vector>

#include "pf_common.cuh"

namespace pfb {

struct GlCtl {
    unsigned long long tau;   // pruning bound on the composite key
    unsigned n_cand;          // survivors appended by the pruned scorer
    unsigned err;
    unsigned long long visits;  // DDA cell visits counted by pfgl_count_visits
};

struct GlHandle {
    int dev = 0;
    cudaStream_t stream = nullptr;
    int W = 0, H = 0, Wp = 0, Hp = 0;
    float res = 0.05f, ox = 0.f, oy = 0.f;
    int cap_hyp = 0;
    int nfree = 0;
    int nh = 0;
    unsigned char* d_grid = nullptr;  // padded
    int2* d_free = nullptr;
    float* d_hyp = nullptr;
    float* d_caer = nullptr;
    uint64_t* d_keys = nullptr;
    uint64_t* d_keys_alt = nullptr;
    unsigned* d_hist = nullptr;
    int hist_cap = 0;
    float* d_scan = nullptr;
    int scan_cap = 0;
    float* d_scans = nullptr;  // a batch of queries' scans (nq x nrays)
    int scans_cap = 0;
    float* d_out = nullptr;   // k x 3 (cap_hyp)
    float* d_outc = nullptr;  // k CAER
    int* d_outi = nullptr;    // k indices
    uint64_t* d_cand = nullptr;  // pruned-scorer survivors (cap_hyp)
    uint64_t* d_sel = nullptr;   // small bottom-k select: the k smallest keys
    GlCtl* d_ctl = nullptr;
    GlCtl* h_ctl = nullptr;
    std::vector<unsigned char> host_grid;  // unpadded 0/1 copy
    bool caer_valid = false;
    int last_k = 0;  // entries of d_out written by the last bottom-k
};

struct GridView {
    const unsigned char* cells;  // padded grid
    int W, H, Wp;
    float res, ox, oy;
};

// 2-D DDA from the padded start index with in-cell fractions (frx, fry):
// distance to the first occupied cell, rmax when the ray passes rmax or
// leaves the map.  The f32 arithmetic follows src/cuda/pf_kernels.cu:784-808
// (tMax/tDelta stepping, x step on ties); stepping onto the border byte (2)
// is the reference's out-of-grid test.
//
// The reference tests dist > rmax and an 8192-step limit after every step.
// Both leave the loop here without changing any result: the step distances
// never decrease, so "the first hit, then rmax if its distance exceeds rmax"
// equals "rmax as soon as a step exceeds rmax"; the border ends every ray,
// and the number of steps taken (one cell in x or y per step) is recovered
// from the hit cell to apply the step limit.
struct Ray {
    float tmx, tmy, tdx, tdy, dist;
    int sx, sy, idx;
    unsigned v;  // 0 while the ray is travelling, else the cell value it hit
};

__device__ __forceinline__ void ray_init(Ray& r, int Wp, int start, float frx,
                                         float fry, float dirx, float diry,
                                         float res) {
    r.sx = dirx > 0 ? 1 : -1;
    r.sy = diry > 0 ? Wp : -Wp;
    const float adx = fabsf(dirx), ady = fabsf(diry);
    r.tdx = adx > 1e-9f ? res / adx : INFINITY;
    r.tdy = ady > 1e-9f ? res / ady : INFINITY;
    r.tmx = adx > 1e-9f ? ((dirx > 0 ? 1.f - frx : frx) * r.tdx) : INFINITY;
    r.tmy = ady > 1e-9f ? ((diry > 0 ? 1.f - fry : fry) * r.tdy) : INFINITY;
    r.idx = start;
    r.dist = 0.f;
    r.v = 0u;
}

// The distances between x and between y cell crossings of a ray, each signed
// by its step direction (+ for dirx > 0, resp. diry > 0; an axis the ray does
// not cross holds +-INFINITY): ray_init's divisions, done once per ray ahead
// of the stepping so that a lane restarting on a new ray does no division.
__device__ __forceinline__ float2 ray_deltas(float dirx, float diry, float res) {
    const float adx = fabsf(dirx), ady = fabsf(diry);
    const float tdx = adx > 1e-9f ? res / adx : INFINITY;
    const float tdy = ady > 1e-9f ? res / ady : INFINITY;
    return make_float2(dirx > 0 ? tdx : -tdx, diry > 0 ? tdy : -tdy);
}

// ray_init from ray_deltas: the same Ray, field for field (res / |dir| is
// finite exactly when |dir| > 1e-9, and its sign carries dir > 0).
__device__ __forceinline__ void ray_init_deltas(Ray& r, int Wp, int start, float frx,
                                                float fry, float2 d) {
    const bool px = d.x > 0.f, py = d.y > 0.f;
    r.sx = px ? 1 : -1;
    r.sy = py ? Wp : -Wp;
    r.tdx = fabsf(d.x);
    r.tdy = fabsf(d.y);
    r.tmx = r.tdx != INFINITY ? ((px ? 1.f - frx : frx) * r.tdx) : INFINITY;
    r.tmy = r.tdy != INFINITY ? ((py ? 1.f - fry : fry) * r.tdy) : INFINITY;
    r.idx = start;
    r.dist = 0.f;
    r.v = 0u;
}

__device__ __forceinline__ void ray_step(Ray& r, const unsigned char* __restrict__ g) {
    const bool px = r.tmx <= r.tmy;
    r.dist = px ? r.tmx : r.tmy;
    if (px)
        r.tmx += r.tdx;
    else
        r.tmy += r.tdy;
    r.idx += px ? r.sx : r.sy;
    r.v = g[r.idx];
}

// Result of an ended ray.  The step limit can only bind when a ray can take
// more than 8192 steps before reaching the border (Wp + Hp > 8192).
__device__ __forceinline__ float ray_result(const Ray& r, int Wp, int start,
                                            float rmax, bool long_rays = true) {
    if (r.v != 1u || r.dist > rmax) return rmax;
    if (!long_rays) return r.dist;
    const int dy = r.idx / Wp - start / Wp;  // cells moved in y
    const int dx = r.idx - start - dy * Wp;  // cells moved in x
    return (abs(dx) + abs(dy) > 8192) ? rmax : r.dist;
}

__device__ __forceinline__ float cast_ray(const unsigned char* __restrict__ g,
                                          int Wp, int start, float frx,
                                          float fry, float dirx, float diry,
                                          float res, float rmax) {
    Ray r;
    ray_init(r, Wp, start, frx, fry, dirx, diry, res);
    do {
        ray_step(r, g);
    } while (r.v == 0u);
    return ray_result(r, Wp, start, rmax);
}

// Start cell of a pose (floor of the f32 cell coordinate, as
// src/cuda/pf_kernels.cu:774-781); false when outside the map.
__device__ __forceinline__ bool start_cell(const GridView& gv, float x, float y,
                                           int& start, float& frx,
                                           float& fry) {
    const float fx = (x - gv.ox) / gv.res;
    const float fy = (y - gv.oy) / gv.res;
    const int cx = (int)floorf(fx), cy = (int)floorf(fy);
    if (!(cx >= 0 && cy >= 0 && cx < gv.W && cy < gv.H)) return false;
    frx = (x - gv.ox) / gv.res - (float)cx;
    fry = (y - gv.oy) / gv.res - (float)cy;
    start = (cy + 1) * gv.Wp + (cx + 1);
    return true;
}

// Angle of ray r: the reference spaces nrays rays over span with
// (nrays - 1) gaps (src/cuda/pf_kernels.cu:784).
__device__ __forceinline__ float ray_angle(float th, int r, int nrays,
                                           float span) {
    return th + (nrays > 1 ? span * (float)r / (float)(nrays - 1) : 0.f);
}

__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    return v;
}

inline GridView grid_view(const GlHandle* h) {
    return {h->d_grid, h->W, h->H, h->Wp, h->res, h->ox, h->oy};
}

inline int grid_bytes_padded(const GlHandle* h) {
    return (int)(((size_t)h->Wp * h->Hp + 15) / 16 * 16);
}

// ------------------------------------------- entry points shared across units
// Copy a host scan into the handle's device scan buffer (stream-ordered).
int gl_upload_scan(GlHandle* h, const float* scan, int nrays);
// Bottom-k of the h->nh hypotheses in d_hyp against the loaded scan, using the
// pruned scorer; results as pfgl_localize.  Returns k written or -1.
int gl_localize_loaded(GlHandle* h, int nrays, float rmax, float span, int k,
                       float* out3k, float* caer_k, int* idx_k);
// Exhaustive CAER of the h->nh hypotheses in d_hyp against the loaded scan,
// then the bottom-k (one host synchronisation).  Returns k written or -1.
int gl_topk_exhaustive(GlHandle* h, int nrays, float rmax, float span, int k,
                       float* out3k, float* caer_k, int* idx_k);
// Uniform dispersion of n_pos positions x n_yaw yaws into d_hyp.
int gl_generate(GlHandle* h, int n_pos, int n_yaw, uint64_t seed);
// The small-set localizer (n <= 65536 hypotheses, k <= 128, see
// gl_small_select_ok) enqueued without host synchronisation: returns the
// device buffer that will hold the k smallest (CAER, index) keys, or nullptr.
const uint64_t* gl_localize_small_keys(GlHandle* h, int nrays, float rmax, float span,
                                       int k);
bool gl_small_select_ok(int n, int k);
// Gathers the poses, CAERs and indices of the k keys into d_out / d_outc /
// d_outi (asynchronous).
int gl_gather_topk(GlHandle* h, const uint64_t* sorted, int k);
// Batches of queries.  gl_upload_scans copies nq host scans into d_scans;
// gl_localize_batch_enqueue scores the nq * per_q hypotheses in d_hyp
// (query q's at [q * per_q, (q + 1) * per_q)) exhaustively against their
// queries' scans in d_scans and writes each query's bottom-k (ascending,
// indices within the query) to d_out / d_outc / d_outi at [q * k, q * k + k)
// (asynchronous).  gl_batch_ok: the sizes this supports.
int gl_upload_scans(GlHandle* h, const float* scans, int nq, int nrays);
bool gl_batch_ok(const GlHandle* h, int nq, int per_q, int k);
int gl_localize_batch_enqueue(GlHandle* h, int nq, int per_q, int nrays, float rmax,
                              float span, int k);

}  // namespace pfb
