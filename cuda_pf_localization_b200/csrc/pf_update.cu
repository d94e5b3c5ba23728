// pf_update.cu — prior (reinit), motion update (predict) and landmark
// weighting kernels on the SoA particle planes.
//
// The weighting kernel optionally runs a deferred predict first, so one pass
// over HBM reads the old pose, writes the new pose and the log-likelihood,
// and leaves per-block softmax partials (block max, sum exp(ll - block max)
// in FP64).  The last block to finish combines the partials in block order,
// so M = max ll and S = sum exp(ll - M) are deterministic.
#include <math.h>

#include "pf_internal.h"

namespace pfb {

namespace {

constexpr int kThreads = 256;
constexpr int kObsChunk = 256;  // observations staged in shared memory at once


PlaneSet plane_set(const PfHandle* h) { return {h->planes(0), h->planes(1)}; }

__device__ __forceinline__ void load_pose(const Planes& s, int i, float3& p,
                                          Quat& q) {
    p = make_float3(s.px[i], s.py[i], s.pz[i]);
    q = {s.qw[i], s.qx[i], s.qy[i], s.qz[i]};
}

__device__ __forceinline__ void store_pose(const Planes& s, int i, float3 p,
                                           Quat q) {
    s.px[i] = p.x;
    s.py[i] = p.y;
    s.pz[i] = p.z;
    s.qw[i] = q.w;
    s.qx[i] = q.x;
    s.qy[i] = q.y;
    s.qz[i] = q.z;
}

// Motion model of the reference predict (src/cuda/pf_kernels.cu:198-222,
// semantics crates/pf_core/src/cpu.rs:197-218): body displacement t + sigma_t*n
// rotated into the world by q, then q <- (q * q_odo) * exp(sigma_r*w).  The
// quaternion is not renormalised, as in the reference.
__device__ __forceinline__ void apply_predict(const PredictArgs& pa,
                                              uint64_t seed, int i, float3& p,
                                              Quat& q) {
    float nz[6];
    pf_normals6(seed, pa.gen, (uint32_t)i, nz);
    float3 body = make_float3(pa.t[0] + pa.tstd[0] * nz[0],
                              pa.t[1] + pa.tstd[1] * nz[1],
                              pa.t[2] + pa.tstd[2] * nz[2]);
    float3 world = q_rotate(q, body);
    p.x += world.x;
    p.y += world.y;
    p.z += world.z;
    float3 axis = make_float3(pa.rstd[0] * nz[3], pa.rstd[1] * nz[4],
                              pa.rstd[2] * nz[5]);
    float ang = sqrtf(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
    Quat dq = q_from_axis_angle(axis, ang);
    Quat qo = {pa.q[0], pa.q[1], pa.q[2], pa.q[3]};
    q = q_product(q_product(q, qo), dq);
}

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
    float ang = sqrtf(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
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
    float ang = sqrtf(axis.x * axis.x + axis.y * axis.y + axis.z * axis.z);
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

// Observations staged in shared memory: the landmark resolved through the
// dense table and the observation, a = (lx, ly, lz, kind bits) with kind 1 =
// Cartesian, 2 = range + bearing; b = (dx, dy, dz, range).
struct GateConsts {
    float inv2rr, inv2bb, g2, cart_gate2, rng_gate2, brg_gate2, cart_out,
        half_out, gate;
};

// Same f32 expressions as the reference kernel prologue
// (src/cuda/pf_kernels.cu:229-234) so the gate thresholds are identical.
__device__ __forceinline__ GateConsts gate_consts(float sigma_r, float sigma_b,
                                                  float gate) {
    GateConsts g;
    g.inv2rr = 1.0f / (2.0f * sigma_r * sigma_r);
    g.inv2bb = 1.0f / (2.0f * sigma_b * sigma_b);
    g.g2 = gate * gate;
    g.cart_gate2 = g.g2 * 3.0f * sigma_r * sigma_r;
    g.rng_gate2 = g.g2 * sigma_r * sigma_r;
    g.brg_gate2 = g.g2 * sigma_b * sigma_b;
    g.cart_out = -0.5f * g.g2 * 3.0f;
    g.half_out = -0.5f * g.g2;
    g.gate = gate;
    return g;
}

// One particle against one observation, accumulated into acc in the
// reference's expression order (src/cuda/pf_kernels.cu:240-269; model
// crates/pf_core/src/cpu.rs:44-97): a range-bearing observation adds its range
// and bearing terms to acc one after the other.
__device__ __forceinline__ void obs_loglik(const GateConsts& g, float3 p,
                                           const Quat& qc, float4 a, float4 b,
                                           int kind, float& acc) {
    float3 d = make_float3(a.x - p.x, a.y - p.y, a.z - p.z);
    float3 pred = q_rotate(qc, d);  // landmark in the body frame
    if (kind == 1) {
        float ex = pred.x - b.x, ey = pred.y - b.y, ez = pred.z - b.z;
        float r2 = ex * ex + ey * ey + ez * ez;
        acc += (g.gate > 0.0f && r2 > g.cart_gate2) ? g.cart_out
                                                    : -r2 * g.inv2rr;
        return;
    }
    float rn = fmaxf(
        sqrtf(pred.x * pred.x + pred.y * pred.y + pred.z * pred.z), 1e-9f);
    float er = rn - b.w;
    float dot = -((pred.x * b.x + pred.y * b.y + pred.z * b.z) / rn);
    dot = fminf(fmaxf(dot, -1.0f), 1.0f);
    float eb = acosf(dot);
    acc += (g.gate > 0.0f && er * er > g.rng_gate2) ? g.half_out
                                                    : -er * er * g.inv2rr;
    acc += (g.gate > 0.0f && eb * eb > g.brg_gate2) ? g.half_out
                                                    : -eb * eb * g.inv2bb;
}

// Fixed-order block reductions (xor-butterfly inside warps, warps in index
// order) — results do not depend on scheduling.
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(~0u, v, o));
    return v;
}
__device__ __forceinline__ double warp_sum_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    return v;
}
__device__ __forceinline__ double warp_max_d(double v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(~0u, v, o));
    return v;
}

// Softmax partial of one block (two log-likelihoods per thread) + the
// last-block combine.
__device__ __forceinline__ void softmax_partials(float acc0, bool v0,
                                                 float acc1, bool v1,
                                                 double2* part,
                                                 unsigned* done,
                                                 CycleCtl* ctl) {
    __shared__ float s_m[kThreads / 32];
    __shared__ double s_s[kThreads / 32];
    __shared__ double s_bm;
    __shared__ bool s_last;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float m = warp_max_f(fmaxf(v0 ? acc0 : -INFINITY, v1 ? acc1 : -INFINITY));
    if (lane == 0) s_m[warp] = m;
    __syncthreads();
    if (tid == 0) {
        float bm = s_m[0];
        for (int k = 1; k < kThreads / 32; ++k) bm = fmaxf(bm, s_m[k]);
        s_bm = (double)bm;
    }
    __syncthreads();
    const double bm = s_bm;
    double e = (v0 ? exp((double)acc0 - bm) : 0.0) + (v1 ? exp((double)acc1 - bm) : 0.0);
    e = warp_sum_d(e);
    if (lane == 0) s_s[warp] = e;
    __syncthreads();
    if (tid == 0) {
        double sb = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) sb += s_s[k];
        part[blockIdx.x] = make_double2(bm, sb);
        __threadfence();
        s_last = (atomicAdd(done, 1u) == gridDim.x - 1);
    }
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    // Combine: M = max block max, S = sum_b exp(m_b - M) * s_b.
    const int G = gridDim.x;
    double mx = -INFINITY;
#pragma unroll 4
    for (int b = tid; b < G; b += kThreads) mx = fmax(mx, __ldcg(&part[b].x));
    mx = warp_max_d(mx);
    __shared__ double s_d[kThreads / 32];
    if (lane == 0) s_d[warp] = mx;
    __syncthreads();
    if (tid == 0) {
        double v = s_d[0];
        for (int k = 1; k < kThreads / 32; ++k) v = fmax(v, s_d[k]);
        s_bm = v;
    }
    __syncthreads();
    const double M = s_bm;
    double sum = 0.0;
#pragma unroll 4
    for (int b = tid; b < G; b += kThreads) {
        double2 pb = __ldcg(&part[b]);
        sum += exp(pb.x - M) * pb.y;
    }
    sum = warp_sum_d(sum);
    __syncthreads();
    if (lane == 0) s_d[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        double S = 0.0;
        for (int k = 0; k < kThreads / 32; ++k) S += s_d[k];
        ctl->ll_max = M;
        ctl->ll_sumexp = S;
        const int ok = (S > 0.0 && isfinite(S)) ? 1 : 0;
        ctl->weights_valid = ok;
        ctl->wmode = ok ? WMODE_LL : WMODE_UNIFORM;
        *done = 0u;
    }
}

// Stage observations [c0, c0 + cn) into shared memory, dropping the ones
// whose id is outside the landmark table (the reference skips them with
// `continue`, pf_kernels.cu:242) and keeping the order of the rest, so the
// f32 accumulation order is unchanged.  Returns the number kept; *all_cart
// is set when every kept observation is Cartesian.
__device__ __forceinline__ int stage_chunk(const CObservation* __restrict__ obs,
                                           const float* __restrict__ lm,
                                           int lm_count, int c0, int cn,
                                           float4* s_a, float4* s_b,
                                           float4* s_p, bool* all_cart) {
    __shared__ int s_wcount[kThreads / 32];
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    CObservation o;
    bool keep = false;
    if (tid < cn) {
        o = obs[c0 + tid];
        keep = o.id >= 0 && o.id < lm_count;
    }
    const unsigned ballot = __ballot_sync(~0u, keep);
    if (lane == 0) s_wcount[warp] = __popc(ballot);
    const int cart = __syncthreads_and(!keep || o.mode == 0);
    int off = 0, total = 0;
    for (int k = 0; k < kThreads / 32; ++k) {
        const int c = s_wcount[k];
        off += (k < warp) ? c : 0;
        total += c;
    }
    if (keep) {
        const int slot = off + __popc(ballot & ((1u << lane) - 1u));
        const float lx = lm[3 * o.id], ly = lm[3 * o.id + 1], lz = lm[3 * o.id + 2];
        s_a[slot] = make_float4(lx, ly, lz, __int_as_float(o.mode == 0 ? 1 : 2));
        s_b[slot] = make_float4(o.dx, o.dy, o.dz, o.range);
        // broadcast pairs for the packed two-particle path
        s_p[3 * slot] = make_float4(lx, lx, ly, ly);
        s_p[3 * slot + 1] = make_float4(lz, lz, -o.dx, -o.dx);
        s_p[3 * slot + 2] = make_float4(-o.dy, -o.dy, -o.dz, -o.dz);
    }
    *all_cart = cart != 0;
    __syncthreads();
    return total;
}

// Gated Cartesian term of the reference (pf_kernels.cu:247-252) for the
// specialised all-Cartesian loop; gate > 0 is hoisted out as kGated.
template <bool kGated>
__device__ __forceinline__ void cart_term(const GateConsts& g, float3 p,
                                          const Quat& qc, float4 a, float4 b,
                                          float& acc) {
    float3 d = make_float3(a.x - p.x, a.y - p.y, a.z - p.z);
    float3 pred = q_rotate(qc, d);
    float ex = pred.x - b.x, ey = pred.y - b.y, ez = pred.z - b.z;
    float r2 = ex * ex + ey * ey + ez * ez;
    // The reference rounds the product and the sum separately in both the
    // gated and the ungated case; the ungated form uses the intrinsics that
    // are never merged into a multiply-add.
    if (kGated)
        acc += (r2 > g.cart_gate2) ? g.cart_out : -r2 * g.inv2rr;
    else
        acc = __fadd_rn(acc, __fmul_rn(-r2, g.inv2rr));
}

// ---------------------------------------------------------- packed path
// The Cartesian term evaluated for two particles at once with packed f32x2
// arithmetic.  nvcc compiles the reference expression (q_rotate + squared
// residual) with these contractions, each operation rounded once:
//   t'  = fma(-q.z, v.y, q.y*v.z)  (likewise y, z);   t = 2 t' exactly
//   c.x = fma(-q.z, t.y, q.y*t.z)  (likewise y, z)
//   r.x = fma(q.w, t.x, v.x) + c.x;  e = r - o
//   r2  = fma(ez, ez, fma(ex, ex, ey*ey)),  term = -r2 * inv2rr
// (established by comparing candidate orderings against the compiled
// expression bit for bit).  Scaling by 2 is exact and commutes with rounding,
// so the products with t = 2t' are formed from t' and pre-doubled quaternion
// components, which removes the three multiplications by two; every rounded
// operation of the reference is still performed, so the log-likelihoods are
// identical.
struct PackedPose {
    float2 npx, npy, npz;      // -p
    float2 k1, k2, k3, k4, k5, k6;  // t' coefficients
    float2 m1, m2, m3, m4, m5, m6;  // c coefficients (doubled)
    float2 w2;                  // 2 q.w
};

__device__ __forceinline__ PackedPose pack_pose(float3 p0, const Quat& c0,
                                                float3 p1, const Quat& c1) {
    PackedPose k;
    k.npx = make_float2(-p0.x, -p1.x);
    k.npy = make_float2(-p0.y, -p1.y);
    k.npz = make_float2(-p0.z, -p1.z);
    k.k1 = make_float2(-c0.z, -c1.z);
    k.k2 = make_float2(c0.y, c1.y);
    k.k3 = make_float2(-c0.x, -c1.x);
    k.k4 = make_float2(c0.z, c1.z);
    k.k5 = make_float2(-c0.y, -c1.y);
    k.k6 = make_float2(c0.x, c1.x);
    k.m1 = make_float2(2.f * k.k1.x, 2.f * k.k1.y);
    k.m2 = make_float2(2.f * k.k2.x, 2.f * k.k2.y);
    k.m3 = make_float2(2.f * k.k3.x, 2.f * k.k3.y);
    k.m4 = make_float2(2.f * k.k4.x, 2.f * k.k4.y);
    k.m5 = make_float2(2.f * k.k5.x, 2.f * k.k5.y);
    k.m6 = make_float2(2.f * k.k6.x, 2.f * k.k6.y);
    k.w2 = make_float2(2.f * c0.w, 2.f * c1.w);
    return k;
}

// One observation (broadcast pairs A = (lx,lx,ly,ly), B = (lz,lz,-ox,-ox),
// C = (-oy,-oy,-oz,-oz)) against two particles; returns the packed term.
__device__ __forceinline__ float2 packed_r2(const PackedPose& k, float4 A,
                                            float4 B, float4 C) {
    const float2 dx = __fadd2_rn(make_float2(A.x, A.y), k.npx);
    const float2 dy = __fadd2_rn(make_float2(A.z, A.w), k.npy);
    const float2 dz = __fadd2_rn(make_float2(B.x, B.y), k.npz);
    const float2 tx = __ffma2_rn(k.k1, dy, __fmul2_rn(k.k2, dz));
    const float2 ty = __ffma2_rn(k.k3, dz, __fmul2_rn(k.k4, dx));
    const float2 tz = __ffma2_rn(k.k5, dx, __fmul2_rn(k.k6, dy));
    const float2 cx = __ffma2_rn(k.m1, ty, __fmul2_rn(k.m2, tz));
    const float2 cy = __ffma2_rn(k.m3, tz, __fmul2_rn(k.m4, tx));
    const float2 cz = __ffma2_rn(k.m5, tx, __fmul2_rn(k.m6, ty));
    const float2 rx = __fadd2_rn(__ffma2_rn(k.w2, tx, dx), cx);
    const float2 ry = __fadd2_rn(__ffma2_rn(k.w2, ty, dy), cy);
    const float2 rz = __fadd2_rn(__ffma2_rn(k.w2, tz, dz), cz);
    const float2 ex = __fadd2_rn(rx, make_float2(B.z, B.w));
    const float2 ey = __fadd2_rn(ry, make_float2(C.x, C.y));
    const float2 ez = __fadd2_rn(rz, make_float2(C.z, C.w));
    return __ffma2_rn(ez, ez, __ffma2_rn(ex, ex, __fmul2_rn(ey, ey)));
}

// Two particles per thread (i and i + 256): every staged observation read
// from shared memory serves both.
template <bool kPredict>
__global__ void __launch_bounds__(kThreads)
    k_weight(PlaneSet ps, int n, uint64_t seed, PredictArgs pa,
             const CObservation* __restrict__ obs, int nobs,
             const float* __restrict__ lm, int lm_count, float sigma_r,
             float sigma_b, float gate, float* __restrict__ ll,
             double2* part, unsigned* done, CycleCtl* ctl, int use_packed) {
    __shared__ float4 s_a[kObsChunk];
    __shared__ float4 s_b[kObsChunk];
    __shared__ float4 s_p[3 * kObsChunk];
    const Planes s = pick_planes(ps, ctl->live);
    const int i0 = blockIdx.x * (2 * kThreads) + threadIdx.x;
    const int i1 = i0 + kThreads;
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
    const GateConsts g = gate_consts(sigma_r, sigma_b, gate);
    const Quat qc0 = q_conjugate(q0), qc1 = q_conjugate(q1);
    const PackedPose pk = pack_pose(p0, qc0, p1, qc1);
    const float2 ninv = make_float2(-g.inv2rr, -g.inv2rr);
    float acc0 = 0.0f, acc1 = 0.0f;
    for (int c0 = 0; c0 < nobs; c0 += kObsChunk) {
        bool all_cart;
        __syncthreads();
        const int cn = stage_chunk(obs, lm, lm_count, c0, min(kObsChunk, nobs - c0),
                                   s_a, s_b, s_p, &all_cart);
        if (all_cart && use_packed) {
            float2 acc = make_float2(acc0, acc1);
            if (gate > 0.0f) {
#pragma unroll 2
                for (int k = 0; k < cn; ++k) {
                    const float2 r2 = packed_r2(pk, s_p[3 * k], s_p[3 * k + 1],
                                                s_p[3 * k + 2]);
                    const float2 t = __fmul2_rn(r2, ninv);
                    const float a0 = (r2.x > g.cart_gate2) ? g.cart_out : t.x;
                    const float a1 = (r2.y > g.cart_gate2) ? g.cart_out : t.y;
                    acc = __fadd2_rn(acc, make_float2(a0, a1));
                }
            } else {
#pragma unroll 2
                for (int k = 0; k < cn; ++k) {
                    const float2 r2 = packed_r2(pk, s_p[3 * k], s_p[3 * k + 1],
                                                s_p[3 * k + 2]);
                    // two roundings, as the reference (see cart_term)
                    acc.x = __fadd_rn(acc.x, __fmul_rn(r2.x, ninv.x));
                    acc.y = __fadd_rn(acc.y, __fmul_rn(r2.y, ninv.y));
                }
            }
            acc0 = acc.x;
            acc1 = acc.y;
        } else if (all_cart && gate > 0.0f) {
#pragma unroll 2
            for (int k = 0; k < cn; ++k) {
                const float4 a = s_a[k], b = s_b[k];
                cart_term<true>(g, p0, qc0, a, b, acc0);
                cart_term<true>(g, p1, qc1, a, b, acc1);
            }
        } else if (all_cart) {
#pragma unroll 2
            for (int k = 0; k < cn; ++k) {
                const float4 a = s_a[k], b = s_b[k];
                cart_term<false>(g, p0, qc0, a, b, acc0);
                cart_term<false>(g, p1, qc1, a, b, acc1);
            }
        } else {
            for (int k = 0; k < cn; ++k) {
                const float4 a = s_a[k], b = s_b[k];
                const int kind = __float_as_int(a.w);
                obs_loglik(g, p0, qc0, a, b, kind, acc0);
                obs_loglik(g, p1, qc1, a, b, kind, acc1);
            }
        }
    }
    if (v0) ll[i0] = acc0;
    if (v1) ll[i1] = acc1;
    softmax_partials(acc0, v0, acc1, v1, part, done, ctl);
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
                  int nobs, float sigma_r, float sigma_b, float gate) {
    const int grid = ceil_div(h->n, 2 * kThreads);
    double2* part = reinterpret_cast<double2*>(h->d_part);
    KernelScope ks(h, KK_WEIGHT);
    if (pa.enabled) {
        k_weight<true><<<grid, kThreads, 0, h->stream>>>(
            plane_set(h), h->n, h->seed, pa, d_obs, nobs, h->d_lm, h->lm_count,
            sigma_r, sigma_b, gate, h->d_ll, part, h->d_done + 0, h->d_ctl,
            h->weight_variant == 0 ? 1 : 0);
    } else {
        k_weight<false><<<grid, kThreads, 0, h->stream>>>(
            plane_set(h), h->n, h->seed, pa, d_obs, nobs, h->d_lm, h->lm_count,
            sigma_r, sigma_b, gate, h->d_ll, part, h->d_done + 0, h->d_ctl,
            h->weight_variant == 0 ? 1 : 0);
    }
    PFB_KL();
    return 0;
}

}  // namespace pfb
