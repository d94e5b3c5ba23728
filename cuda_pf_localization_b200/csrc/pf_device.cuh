// pf_device.cuh — per-particle device routines shared by the single-filter
// kernels (pf_update.cu, pf_estimate.cu, pf_resample.cu) and the batched
// multi-filter kernels (pf_batch.cu): motion model, gated weighting with the
// reference's roundings, fixed-order softmax partials, FP64 estimate and
// covariance accumulation, the fixed-point resampling thresholds, the
// decoupled look-back and the injection draws.  Sharing them is what makes a
// filter of a batch produce the same bits as the same filter run alone.
#pragma once

#include <math.h>

#include "pf_internal.h"

namespace pfb {
namespace dev {

constexpr int kBlk = 256;       // threads per block of the particle kernels (the
                                // weighting kernels use kWThreads)
// The staging, softmax-partial and combine helpers below run on weighting
// blocks of exactly kWThreads threads (pf_internal.h).
constexpr int kObsChunk = kWThreads;  // observations staged in shared memory at once

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
    float ang = norm3(axis);
    Quat dq = q_from_axis_angle(axis, ang);
    Quat qo = {pa.q[0], pa.q[1], pa.q[2], pa.q[3]};
    q = q_product(q_product(q, qo), dq);
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

// x^2 + y^2 + z^2 as nvcc contracts the reference's squared residual:
// fma(z, z, fma(x, x, y*y)).
__device__ __forceinline__ float sq3(float x, float y, float z) {
    return __fmaf_rn(z, z, __fmaf_rn(x, x, __fmul_rn(y, y)));
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
        const float ex = pred.x - b.x, ey = pred.y - b.y, ez = pred.z - b.z;
        const float r2 = sq3(ex, ey, ez);
        const float t = (g.gate > 0.0f && r2 > g.cart_gate2)
                            ? g.cart_out
                            : __fmul_rn(-r2, g.inv2rr);
        acc = __fadd_rn(acc, t);
        return;
    }
    // Same contraction shape as the squared residual: middle product first,
    // then the x and z terms fused; every other operation rounded alone.
    const float rn = fmaxf(sqrtf(sq3(pred.x, pred.y, pred.z)), 1e-9f);
    const float er = rn - b.w;
    const float dp = __fmaf_rn(pred.z, b.z, __fmaf_rn(pred.x, b.x, __fmul_rn(pred.y, b.y)));
    float dot = -__fdiv_rn(dp, rn);
    dot = fminf(fmaxf(dot, -1.0f), 1.0f);
    const float eb = acosf(dot);
    const float er2 = __fmul_rn(er, er), eb2 = __fmul_rn(eb, eb);
    const float tr = (g.gate > 0.0f && er2 > g.rng_gate2)
                         ? g.half_out
                         : __fmul_rn(__fmul_rn(-er, er), g.inv2rr);
    acc = __fadd_rn(acc, tr);
    const float tb = (g.gate > 0.0f && eb2 > g.brg_gate2)
                         ? g.half_out
                         : __fmul_rn(__fmul_rn(-eb, eb), g.inv2bb);
    acc = __fadd_rn(acc, tb);
}

// Fixed-order block reductions (xor-butterfly inside warps, warps in index
// order) — results do not depend on scheduling.
__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(~0u, v, o));
    return v;
}
__device__ __forceinline__ float warp_sum_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = __fadd_rn(v, __shfl_xor_sync(~0u, v, o));
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

__device__ __forceinline__ unsigned long long warp_sum_u64(unsigned long long v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(~0u, v, o);
    return v;
}

__device__ __forceinline__ float comp(const float4& v, int c) {
    return c == 0 ? v.x : (c == 1 ? v.y : (c == 2 ? v.z : v.w));
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
    __shared__ int s_wcount[kWThreads / 32];
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
    for (int k = 0; k < kWThreads / 32; ++k) {
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
    const float ex = pred.x - b.x, ey = pred.y - b.y, ez = pred.z - b.z;
    const float r2 = sq3(ex, ey, ez);
    // The reference rounds the product and the sum separately in both the
    // gated and the ungated case.
    if (kGated)
        acc = __fadd_rn(acc, (r2 > g.cart_gate2) ? g.cart_out : __fmul_rn(-r2, g.inv2rr));
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

// Softmax partial of one block of up to 2 * kWThreads log-likelihoods (two per
// thread): (block max, sum expf(ll - block max)) in f32, in a fixed order
// (xor butterfly inside warps, warps in index order).  Valid in every thread.
__device__ __forceinline__ float2 block_softmax_partial(float acc0, bool v0,
                                                        float acc1, bool v1) {
    __shared__ float s_m[kWThreads / 32];
    __shared__ float s_s[kWThreads / 32];
    __shared__ float s_bm, s_sb;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float m = warp_max_f(fmaxf(v0 ? acc0 : -INFINITY, v1 ? acc1 : -INFINITY));
    if (lane == 0) s_m[warp] = m;
    __syncthreads();
    if (tid == 0) {
        float bm = s_m[0];
        for (int k = 1; k < kWThreads / 32; ++k) bm = fmaxf(bm, s_m[k]);
        s_bm = bm;
    }
    __syncthreads();
    const float bm = s_bm;
    float e = __fadd_rn(v0 ? expf(__fsub_rn(acc0, bm)) : 0.0f,
                        v1 ? expf(__fsub_rn(acc1, bm)) : 0.0f);
    e = warp_sum_f(e);
    if (lane == 0) s_s[warp] = e;
    __syncthreads();
    if (tid == 0) {
        float sb = 0.0f;
        for (int k = 0; k < kWThreads / 32; ++k) sb = __fadd_rn(sb, s_s[k]);
        s_sb = sb;
    }
    __syncthreads();
    return make_float2(bm, s_sb);
}

// Combine G block partials (executed by a whole block of kWThreads threads):
// M = max of the block maxima, S = sum_b expf(m_b - M) * s_b in f32, each
// reduced thread-strided, then by xor butterfly, then over warps in order.
// The result is valid in every thread.
__device__ __forceinline__ float2 softmax_combine(const float2* part, int G) {
    __shared__ float s_d[kWThreads / 32];
    __shared__ float s_r;
    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    float mx = -INFINITY;
#pragma unroll 4
    for (int b = tid; b < G; b += kWThreads) mx = fmaxf(mx, __ldcg(&part[b].x));
    mx = warp_max_f(mx);
    if (lane == 0) s_d[warp] = mx;
    __syncthreads();
    if (tid == 0) {
        float v = s_d[0];
        for (int k = 1; k < kWThreads / 32; ++k) v = fmaxf(v, s_d[k]);
        s_r = v;
    }
    __syncthreads();
    const float M = s_r;
    float sum = 0.0f;
#pragma unroll 4
    for (int b = tid; b < G; b += kWThreads) {
        const float2 pb = __ldcg(&part[b]);
        sum = __fadd_rn(sum, __fmul_rn(expf(__fsub_rn(pb.x, M)), pb.y));
    }
    sum = warp_sum_f(sum);
    __syncthreads();
    if (lane == 0) s_d[warp] = sum;
    __syncthreads();
    if (tid == 0) {
        float S = 0.0f;
        for (int k = 0; k < kWThreads / 32; ++k) S = __fadd_rn(S, s_d[k]);
        s_r = S;
    }
    __syncthreads();
    return make_float2(M, s_r);
}

// Gated log-likelihoods of two particles (p0,q0) and (p1,q1) against nobs
// observations, staged kObsChunk at a time into shared memory (the whole
// block takes part).  use_packed selects the packed f32x2 path for
// all-Cartesian chunks; every path produces the reference's roundings.
__device__ __forceinline__ void weight_two(
    const CObservation* __restrict__ obs, int nobs, const float* __restrict__ lm,
    int lm_count, float sigma_r, float sigma_b, float gate, float3 p0, Quat q0,
    float3 p1, Quat q1, int use_packed, float& out0, float& out1) {
    __shared__ float4 s_a[kObsChunk];
    __shared__ float4 s_b[kObsChunk];
    __shared__ float4 s_p[3 * kObsChunk];
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
    out0 = acc0;
    out1 = acc1;
}

// Attitude residual of q about qm as a canonical rotation vector
// (w >= 0, angle = 2 atan2(|v|, w)), in FP64 (a series for angles below about
// 11 degrees, atan2 above) — the form of
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
    const double h2 = dx * dx + dy * dy + dz * dz;
    if (!(h2 > 1e-24)) {  // |v| <= 1e-12: no rotation
        aav[0] = aav[1] = aav[2] = 0.0;
        return;
    }
    double f;
    if (h2 < 0.01 * dw * dw) {
        // z = |v| / w < 0.1: 2 atan(z) / |v| = (2 / w) atan(z) / z with the
        // Taylor series of atan(z) / z in u = z^2 (terms to u^8; the
        // remainder is below u^9 / 19 < 1e-19), which needs neither the
        // square root nor atan2.
        const double r = 1.0 / dw;
        const double u = h2 * r * r;
        double p = 1.0 / 17.0;
        p = fma(p, u, -1.0 / 15.0);
        p = fma(p, u, 1.0 / 13.0);
        p = fma(p, u, -1.0 / 11.0);
        p = fma(p, u, 1.0 / 9.0);
        p = fma(p, u, -1.0 / 7.0);
        p = fma(p, u, 1.0 / 5.0);
        p = fma(p, u, -1.0 / 3.0);
        p = fma(p, u, 1.0);
        f = 2.0 * r * p;
    } else {
        const double hv = sqrt(h2);
        f = 2.0 * atan2(hv, dw) / hv;
    }
    aav[0] = dx * f;
    aav[1] = dy * f;
    aav[2] = dz * f;
}

// Accumulate one particle into the 14 estimate sums of the reference's
// pfc_est_sums layout (src/cuda/pf_kernels.cu:354-404), in FP64.
__device__ __forceinline__ void est_add(double (&acc)[kEstN], float wf, float x,
                                        float y, float z, float qw, float qx,
                                        float qy, float qz) {
    const double wd = (double)wf;
    acc[0] += wd * (double)x;
    acc[1] += wd * (double)y;
    acc[2] += wd * (double)z;
    const double q[4] = {(double)qw, (double)qx, (double)qy, (double)qz};
    int e = 3;
#pragma unroll
    for (int r = 0; r < 4; ++r)
#pragma unroll
        for (int cc = r; cc < 4; ++cc) acc[e++] += wd * q[r] * q[cc];
    acc[13] = __fma_rn(wd, wd, acc[13]);
}

// Accumulate one particle into the 12 covariance sums of the reference's
// pfc_covs layout (src/cuda/pf_kernels.cu:406-471) around (mp, qm), in FP64.
__device__ __forceinline__ void cov_add(double (&acc)[kCovN], double wd, float x,
                                        float y, float z, float qw, float qx,
                                        float qy, float qz, const double mp[3],
                                        const double qm[4]) {
    const double dp[3] = {(double)x - mp[0], (double)y - mp[1], (double)z - mp[2]};
    int e = 0;
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int cc = r; cc < 3; ++cc) acc[e++] += wd * dp[r] * dp[cc];
    const double q[4] = {(double)qw, (double)qx, (double)qy, (double)qz};
    double aav[3];
    att_residual(qm, q, aav);
#pragma unroll
    for (int r = 0; r < 3; ++r)
#pragma unroll
        for (int cc = r; cc < 3; ++cc) acc[e++] += wd * aav[r] * aav[cc];
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

__device__ __forceinline__ uint64_t shfl_up_u64(uint64_t v, int d) {
    unsigned lo = (unsigned)v, hi = (unsigned)(v >> 32);
    lo = __shfl_up_sync(~0u, lo, d);
    hi = __shfl_up_sync(~0u, hi, d);
    return ((uint64_t)hi << 32) | lo;
}


enum : unsigned { TILE_AGG = 1u, TILE_INCL = 2u };

// Fixed-point threshold of output i (see the specification above).
__device__ __forceinline__ uint64_t threshold_fx(long long i, double u0,
                                                 double step) {
    const double t = __dadd_rn(u0, __dmul_rn((double)i, step));
    const double s = t * 0x1p62;
    if (!(s > 0.0)) return 0ull;
    if (s >= 0x1p64) return ~0ull;
    return __double2ull_ru(s);
}

// cnt(X) = number of outputs i in [0, n) with threshold_fx(i) <= X.  The
// thresholds are non-decreasing in i, so this is one more than the last such
// index; it is estimated from the arithmetic sequence and then corrected
// against the exact thresholds.
// inv_step (optional, 1 / step): the estimate by a multiplication instead of
// a division; the corrections below make the count exact either way.
__device__ __forceinline__ long long count_le(uint64_t X, int n, double u0,
                                              double step, double inv_step = 0.0) {
    const double e = inv_step > 0.0 ? floor(((double)X * 0x1p-62 - u0) * inv_step)
                                     : floor(((double)X * 0x1p-62 - u0) / step);
    long long i;
    if (!(e >= -1.0))
        i = -1;
    else if (e > (double)(n - 1))
        i = n - 1;
    else
        i = (long long)e;
    while (i + 1 <= n - 1 && threshold_fx(i + 1, u0, step) <= X) ++i;
    while (i >= 0 && threshold_fx(i, u0, step) > X) --i;
    return i + 1;
}

// Warp-parallel look-back (run by warp 0 of a tile > 0): returns the sum of
// all predecessors' weights.  Lane l inspects tile base - l; the nearest
// predecessor that already knows its inclusive prefix ends the walk.  After
// `limit` polls without progress the wait gives up: ERR_SPIN_TIMEOUT is set
// and the partial sum returned (at most the true prefix, so every count the
// caller derives from it stays within [0, n]).
__device__ inline uint64_t look_back(const unsigned* flags, const uint64_t* vals,
                              int tile, unsigned epoch, unsigned* err,
                              int limit = kSpinLimit) {
    const int lane = threadIdx.x & 31;
    uint64_t prefix = 0;
    int base = tile - 1;
    int spins = 0;
    for (;;) {
        const int j = base - lane;
        unsigned f = 0;
        bool ready = true;
        if (j >= 0) {
            f = ld_acquire(&flags[j]);
            ready = (f >> 2) == epoch && (f & 3u) != 0u;
        }
        if (!__all_sync(~0u, ready)) {
            if (++spins > limit) {
                if (lane == 0) atomicOr(err, ERR_SPIN_TIMEOUT);
                return prefix;
            }
            continue;
        }
        const unsigned incl = __ballot_sync(~0u, j < 0 || (f & 3u) == TILE_INCL);
        const int first = incl ? __ffs(incl) - 1 : 31;
        uint64_t v = 0;
        if (lane <= first && j >= 0)
            v = (lane == first && incl) ? __ldcg(&vals[2 * (size_t)j + 1])
                                        : __ldcg(&vals[2 * (size_t)j]);
        prefix += warp_sum_u64(v);
        if (incl) return prefix;
        base -= 32;
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

}  // namespace dev
}  // namespace pfb
