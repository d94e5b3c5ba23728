// pf_common.cuh — device helpers shared by the particle-filter and
// global-localization kernels: counter-based Philox noise, Hamilton quaternion
// algebra in f32, order-preserving float keys, launch/error plumbing.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include "../../include/pfc_abi.h"

namespace pfb {

// ---------------------------------------------------------------- errors
// Thread-local last-error text, mirrored to stderr like the reference's
// CK/KL macros (src/cuda/pf_kernels.cu:37-67).
void set_error(const char* fmt, ...);
void clear_error();

#define PFB_CK(x)                                                           \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) {                                            \
            ::pfb::set_error("pf_b200 %s:%d %s: %s", __FILE__, __LINE__, #x, \
                             cudaGetErrorString(e_));                       \
            (void)cudaGetLastError(); /* do not leak into later checks */   \
            return -1;                                                      \
        }                                                                   \
    } while (0)

#define PFB_CK_NULL(x)                                                      \
    do {                                                                    \
        cudaError_t e_ = (x);                                               \
        if (e_ != cudaSuccess) {                                            \
            ::pfb::set_error("pf_b200 %s:%d %s: %s", __FILE__, __LINE__, #x, \
                             cudaGetErrorString(e_));                       \
            (void)cudaGetLastError(); /* do not leak into later checks */   \
            return nullptr;                                                 \
        }                                                                   \
    } while (0)

#define PFB_KL()                                                            \
    do {                                                                    \
        cudaError_t e_ = cudaGetLastError();                                \
        if (e_ != cudaSuccess) {                                            \
            ::pfb::set_error("pf_b200 %s:%d launch failed: %s", __FILE__,   \
                             __LINE__, cudaGetErrorString(e_));             \
            return -1;                                                      \
        }                                                                   \
    } while (0)

// Device-side error word bits (written by kernels, read by the host after a
// sync).  A bounded spin that runs out sets SPIN_TIMEOUT instead of hanging.
enum : unsigned {
    ERR_SPIN_TIMEOUT = 1u,
};

constexpr int kSpinLimit = 1 << 22;  // polls before a look-back gives up

// ---------------------------------------------------------------- Philox
// Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as easy
// as 1, 2, 3", SC'11): 10 rounds of two 32x32->64 multiplies with the published
// multipliers and Weyl key increments.  Stateless: noise for particle i in
// generation g is a pure function of (seed, i, g, block).
struct U4 {
    uint32_t x, y, z, w;
};

__host__ __device__ __forceinline__ void philox_mulhilo(uint32_t a, uint32_t b,
                                                        uint32_t& hi,
                                                        uint32_t& lo) {
#ifdef __CUDA_ARCH__
    hi = __umulhi(a, b);
    lo = a * b;
#else
    uint64_t p = (uint64_t)a * (uint64_t)b;
    hi = (uint32_t)(p >> 32);
    lo = (uint32_t)p;
#endif
}

__host__ __device__ __forceinline__ U4 philox4x32_10(U4 c, uint32_t k0,
                                                     uint32_t k1) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u;
    const uint32_t W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        if (r > 0) {
            k0 += W0;
            k1 += W1;
        }
        uint32_t hi0, lo0, hi1, lo1;
        philox_mulhilo(M0, c.x, hi0, lo0);
        philox_mulhilo(M1, c.z, hi1, lo1);
        U4 n;
        n.x = hi1 ^ c.y ^ k0;
        n.y = lo1;
        n.z = hi0 ^ c.w ^ k1;
        n.w = lo0;
        c = n;
    }
    return c;
}

// Uniform in the open interval (0,1): 23 random bits + 1/2, exact in f32.
__host__ __device__ __forceinline__ float u01_open(uint32_t x) {
    return ((float)(x >> 9) + 0.5f) * (1.0f / 8388608.0f);
}

// Box-Muller pair (Box & Muller 1958) from two open uniforms.
__device__ __forceinline__ float2 box_muller(float u1, float u2) {
    float r = sqrtf(-2.0f * logf(u1));
    float s, c;
    sincospif(2.0f * u2, &s, &c);
    return make_float2(r * c, r * s);
}

// Counter block ids: one Philox call per block, four uniforms each.
enum : uint32_t {
    RNG_PF_A = 0u,   // normals 0..3 of a particle update
    RNG_PF_B = 1u,   // normals 4..5
    RNG_GL = 2u,     // hypothesis dispersion
    RNG_LP_POSE = 3u,    // learned proposal: training / held-out poses
    RNG_LP_NOISE = 4u,   // learned proposal: range noise of rendered scans
    RNG_LP_SAMPLE = 5u,  // learned proposal: mixture samples
    RNG_LP_INIT = 6u,    // learned proposal: weight initialisation
};

// Six standard normals for particle i in generation gen: translation noise
// (n0,n1,n2) and rotation noise (n3,n4,n5).
__device__ __forceinline__ void pf_normals6(uint64_t seed, uint64_t gen,
                                            uint32_t i, float n[6]) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    U4 a = philox4x32_10({i, (uint32_t)gen, (uint32_t)(gen >> 32), RNG_PF_A},
                         k0, k1);
    U4 b = philox4x32_10({i, (uint32_t)gen, (uint32_t)(gen >> 32), RNG_PF_B},
                         k0, k1);
    float2 g0 = box_muller(u01_open(a.x), u01_open(a.y));
    float2 g1 = box_muller(u01_open(a.z), u01_open(a.w));
    float2 g2 = box_muller(u01_open(b.x), u01_open(b.y));
    n[0] = g0.x;
    n[1] = g0.y;
    n[2] = g1.x;
    n[3] = g1.y;
    n[4] = g2.x;
    n[5] = g2.y;
}

// ------------------------------------------------------- quaternion algebra
// Hamilton product and the rotation v' = v + 2w(u x v) + 2u x (u x v).
// Every rounding is written out with intrinsics, so the results do not
// depend on how the compiler contracts multiply-adds in the kernel they are
// inlined into (kernels that share these helpers produce the same bits).
// q_rotate spells out the contraction nvcc applies to the reference's
// expression (src/cuda/pf_kernels.cu:119-149), so rotated vectors equal the
// reference kernel's:
//   t = 2 fma(-q.z, v.y, q.y v.z) (likewise y, z)
//   c = fma(-q.z, t.y, q.y t.z)   (likewise y, z)
//   r = fma(q.w, t.x, v.x) + c.x  (likewise y, z)
struct Quat {
    float w, x, y, z;
};

__device__ __forceinline__ float3 q_rotate(const Quat& q, float3 v) {
    const float tx = __fmul_rn(2.f, __fmaf_rn(-q.z, v.y, __fmul_rn(q.y, v.z)));
    const float ty = __fmul_rn(2.f, __fmaf_rn(-q.x, v.z, __fmul_rn(q.z, v.x)));
    const float tz = __fmul_rn(2.f, __fmaf_rn(-q.y, v.x, __fmul_rn(q.x, v.y)));
    const float cx = __fmaf_rn(-q.z, ty, __fmul_rn(q.y, tz));
    const float cy = __fmaf_rn(-q.x, tz, __fmul_rn(q.z, tx));
    const float cz = __fmaf_rn(-q.y, tx, __fmul_rn(q.x, ty));
    return make_float3(__fadd_rn(__fmaf_rn(q.w, tx, v.x), cx),
                       __fadd_rn(__fmaf_rn(q.w, ty, v.y), cy),
                       __fadd_rn(__fmaf_rn(q.w, tz, v.z), cz));
}

__device__ __forceinline__ Quat q_conjugate(const Quat& q) {
    return {q.w, -q.x, -q.y, -q.z};
}

// Hamilton product, each component accumulated left to right from the
// first product.
__device__ __forceinline__ Quat q_product(const Quat& a, const Quat& b) {
    Quat r;
    r.w = __fmaf_rn(-a.z, b.z, __fmaf_rn(-a.y, b.y, __fmaf_rn(-a.x, b.x, __fmul_rn(a.w, b.w))));
    r.x = __fmaf_rn(-a.z, b.y, __fmaf_rn(a.y, b.z, __fmaf_rn(a.x, b.w, __fmul_rn(a.w, b.x))));
    r.y = __fmaf_rn(a.z, b.x, __fmaf_rn(a.y, b.w, __fmaf_rn(-a.x, b.z, __fmul_rn(a.w, b.y))));
    r.z = __fmaf_rn(a.z, b.w, __fmaf_rn(-a.y, b.x, __fmaf_rn(a.x, b.y, __fmul_rn(a.w, b.z))));
    return r;
}

// |v| with a fixed rounding sequence.
__device__ __forceinline__ float norm3(float3 v) {
    return sqrtf(__fmaf_rn(v.z, v.z, __fmaf_rn(v.y, v.y, __fmul_rn(v.x, v.x))));
}

// exp map of a rotation vector with the reference's guards (angle and axis
// norm must exceed 1e-12, else identity).
__device__ __forceinline__ Quat q_from_axis_angle(float3 axis, float angle) {
    const float nrm = norm3(axis);
    if (!(angle > 1e-12f) || !(nrm > 1e-12f)) return {1.f, 0.f, 0.f, 0.f};
    const float h = __fmul_rn(0.5f, angle);
    const float s = __fdiv_rn(sinf(h), nrm);
    return {cosf(h), __fmul_rn(axis.x, s), __fmul_rn(axis.y, s), __fmul_rn(axis.z, s)};
}

// ------------------------------------------------------------ float keys
// Signed-int image of a float whose integer order equals the float order
// (the reference's float_as_ordered, pf_kernels.cu:151-155).
__host__ __device__ __forceinline__ int ordered_key(float f) {
#ifdef __CUDA_ARCH__
    int i = __float_as_int(f);
#else
    int i;
    memcpy(&i, &f, 4);
#endif
    return (i >= 0) ? i : (i ^ 0x7FFFFFFF);
}

// 64-bit composite key: unsigned image of ordered_key in the high word,
// hypothesis index in the low word.  Sorting these ascending equals a stable
// sort by CAER (ties broken by lower index).
__host__ __device__ __forceinline__ uint64_t composite_key(float caer,
                                                           uint32_t idx) {
    uint32_t u = (uint32_t)ordered_key(caer) ^ 0x80000000u;
    return ((uint64_t)u << 32) | (uint64_t)idx;
}

// ------------------------------------------------------------------ sizes
__host__ __device__ __forceinline__ int ceil_div(int a, int b) {
    return (a + b - 1) / b;
}
__host__ __device__ __forceinline__ long long ceil_div_ll(long long a,
                                                          long long b) {
    return (a + b - 1) / b;
}

// ------------------------------------------------- programmatic dependent launch
// The kernels of a filter cycle are launched with programmatic stream
// serialisation: a kernel's blocks may be scheduled as soon as every block
// of its predecessor has exited, before the predecessor grid is retired, and
// wait at pdl_wait() until the predecessor grid has completed and its memory
// is visible.  Every such kernel calls pdl_wait() first, before any early
// return, so completion stays transitive along the chain (a kernel that ended
// without waiting could finish before the kernel two back).  A no-op for a
// plain launch.
__device__ __forceinline__ void pdl_wait() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
}

template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block,
                              size_t smem, cudaStream_t stream, Args... args) {
    cudaLaunchConfig_t cfg{};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    attr[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

}  // namespace pfb
