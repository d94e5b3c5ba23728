// gl_learned.cu — learned proposal for CBGL global localization.
//
// A per-map MLP maps a range scan (rays / rmax, zero padded to 384) to a
// 32-component Gaussian mixture over the pose (x_n, y_n, cos yaw, sin yaw),
// with x_n, y_n the position normalised to [-1, 1] over the map.  A query
// draws hypotheses from the mixture and scores them with the plain CAER
// scorer of gl.cu; when the best CAER is above a threshold calibrated on
// held-out poses, uniform hypotheses are scored as well (the fallback).
//
// Network (all widths padded to multiples of 128):
//   Z0 = X W0^T + b0     384 -> 1024,  H0 = relu(Z0)
//   Z1..Z3               1024 -> 1024, H_l = relu(Z_l)
//   Z4 = H3 W4^T + b4    1024 -> 384 (288 used: 32 logits, 32 x 4 means,
//                                    32 x 4 log-sigma pre-activations)
// Weights are kept as f32 masters (Adam state beside them) and as bf16
// copies in both orientations, W [out][in] and W^T [in][out], so that every
// GEMM of the forward and backward pass reads two K-major bf16 operands:
//   forward    Z_l  = H_{l-1} . W_l^T        A = H_{l-1} [B][in],  B = W_l [out][in]
//   input grad dZ_{l-1} = (dZ_l . W_l) * relu'  A = dZ_l [B][out], B = W_l^T [in][out]
//   weight grad dW_l = dZ_l^T . H_{l-1}      A = dZ_l^T [out][B], B = H_{l-1}^T [in][B]
// The forward and input-gradient epilogues write their bf16 result in both
// orientations, so no separate transposes are needed for the next GEMMs.
//
// GEMM kernel (sm_100a): persistent, one CTA per SM over 128 x BN output
// tiles (BN = 256 or 128), a 4- or 6-stage TMA ring of 64-element k-slices
// (128-byte swizzle), one thread issuing tcgen05.mma into two TMEM
// accumulators in turn, one thread issuing the TMA loads, and eight epilogue
// warps draining the idle accumulator through tcgen05.ld.  Every mbarrier
// wait is bounded; a wait that runs out sets an error word the host turns
// into -1.
#include <cuda.h>
#include <cuda_bf16.h>
#include <cuda_runtime.h>
#include <math.h>
#include <stdint.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <mutex>
#include <new>
#include <vector>

#include "gl_internal.h"
#include "umma.cuh"

namespace pfb {
namespace lp {

using bf16 = __nv_bfloat16;
using namespace pfb::umma;

constexpr int kIn = PFGL_LP_IN;
constexpr int kHid = PFGL_LP_HIDDEN;
constexpr int kOut = PFGL_LP_OUT;
constexpr int kComp = PFGL_LP_COMP;
constexpr int kLayers = PFGL_LP_LAYERS;
constexpr int kUsedOut = kComp * 9;           // 288
constexpr int kMeanOff = kComp;               // 32
constexpr int kSigOff = kComp + 4 * kComp;    // 160
constexpr float kLsLo = -5.5f, kLsHi = 0.0f;  // log-sigma range
constexpr float kHalfLog2Pi = 0.91893853320467274f;

constexpr int layer_in(int l) { return l == 0 ? kIn : kHid; }
constexpr int layer_out(int l) { return l == kLayers - 1 ? kOut : kHid; }

// ------------------------------------------------------------------ GEMM
constexpr int BM = 128, BK = 64;
// Output tile 128 x BN (BN = 128 or 256; the widest tcgen05 shape of one CTA
// is 128 x 256).  Per k-block of 64 a 128 x 256 tile moves 48 KiB of
// operands for 4.2 MFLOP, against 32 KiB for 2.1 MFLOP at 128 x 128: the
// wider tile needs 30 % fewer operand bytes per flop from L2.
constexpr uint32_t kWaitLimit = 1u << 24;

enum Epi : int {
    EPI_RELU_BF16 = 0,   // bf16 relu(acc + bias), row-major and transposed
    EPI_BIAS_F32 = 1,    // f32 acc + bias, row-major
    EPI_DRELU_BF16 = 2,  // bf16 acc * (mask > 0), row-major and transposed
    EPI_F32 = 3,         // f32 acc * scale, row-major
};

struct EpiArgs {
    void* out;
    void* outT;         // transposed copy (bf16 epilogues; may be null)
    const float* bias;  // [N]
    const bf16* mask;   // [M][ldm] activations whose sign gates the gradient
    int ldo, ldt, ldm;
    float scale;
    long long split_stride;  // f32 elements between split-K partial outputs
};

__device__ __forceinline__ uint32_t pack_bf16x2(float a, float b) {
    __nv_bfloat162 h = __floats2bfloat162_rn(a, b);
    return *reinterpret_cast<uint32_t*>(&h);
}

// Epilogue of 32 consecutive columns [col0, col0 + 32) of one output row.
template <int EPI>
__device__ __forceinline__ void epilogue_chunk(const uint32_t (&r)[32], int row,
                                               int col0, const float* bias,
                                               const EpiArgs& ep) {
    float v[32];
#pragma unroll
    for (int j = 0; j < 32; ++j) v[j] = __uint_as_float(r[j]);
    if (EPI == EPI_RELU_BF16 || EPI == EPI_BIAS_F32) {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] += bias[j];  // shared memory
    }
    if (EPI == EPI_RELU_BF16) {
#pragma unroll
        for (int j = 0; j < 32; ++j) v[j] = fmaxf(v[j], 0.0f);
    }
    if (EPI == EPI_DRELU_BF16) {
        const uint4* mp = reinterpret_cast<const uint4*>(
            ep.mask + (size_t)row * ep.ldm + col0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            const uint4 u = mp[q];
            const uint32_t w[4] = {u.x, u.y, u.z, u.w};
#pragma unroll
            for (int t = 0; t < 4; ++t) {
                // relu'(z) = 1 exactly when the stored activation is > 0:
                // a bf16 bit pattern in [1, 0x7fff].
                const int lo = (int)(short)(w[t] & 0xFFFFu);
                const int hi = (int)(short)(w[t] >> 16);
                if (lo <= 0) v[q * 8 + 2 * t] = 0.0f;
                if (hi <= 0) v[q * 8 + 2 * t + 1] = 0.0f;
            }
        }
    }
    if (EPI == EPI_BIAS_F32 || EPI == EPI_F32) {
        const float s = EPI == EPI_F32 ? ep.scale : 1.0f;
        float4* o = reinterpret_cast<float4*>(reinterpret_cast<float*>(ep.out) +
                                              (size_t)row * ep.ldo + col0);
#pragma unroll
        for (int q = 0; q < 8; ++q)
            o[q] = make_float4(v[4 * q] * s, v[4 * q + 1] * s, v[4 * q + 2] * s,
                               v[4 * q + 3] * s);
    } else {
        uint4* o = reinterpret_cast<uint4*>(reinterpret_cast<bf16*>(ep.out) +
                                            (size_t)row * ep.ldo + col0);
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            uint4 u;
            u.x = pack_bf16x2(v[8 * q], v[8 * q + 1]);
            u.y = pack_bf16x2(v[8 * q + 2], v[8 * q + 3]);
            u.z = pack_bf16x2(v[8 * q + 4], v[8 * q + 5]);
            u.w = pack_bf16x2(v[8 * q + 6], v[8 * q + 7]);
            o[q] = u;
        }
        if (ep.outT) {
            // Lanes hold consecutive rows: each store writes 64 contiguous
            // bytes of one transposed row.
            bf16* t = reinterpret_cast<bf16*>(ep.outT) + (size_t)col0 * ep.ldt + row;
#pragma unroll
            for (int j = 0; j < 32; ++j)
                t[(size_t)j * ep.ldt] = __float2bfloat16_rn(v[j]);
        }
    }
}

// D[M][N] = A[M][K] . B[N][K]^T, persistent and warp-specialised: one CTA
// per SM walks the output tiles t = blockIdx.x, blockIdx.x + gridDim.x, ...
// (tile t = split z, row block, column block; column blocks fastest so
// consecutive tiles share their A rows in L2).
//   warp 0 (one thread): TMA producer over a PTile<BN>::kStages-deep ring
//                        that runs on across tile boundaries;
//   warp 1 (one thread): MMA issuer into one of two TMEM accumulators
//                        (columns [0, BN) and [BN, 2 BN)), alternating per
//                        tile;
//   warps 2-9:           the epilogue of the other accumulator, so tile i's
//                        epilogue overlaps tile i + 1's MMAs.  Warp w reads
//                        TMEM lanes [32 (w % 4), 32 (w % 4) + 32), the lane
//                        quarter its warp may access; the two warps of a
//                        quarter take alternate 32-column chunks.
// Barriers: full/empty per ring stage, acc_full (MMA commit) and acc_empty
// (one arrival per epilogue warp, after its last chunk) per accumulator.  Every wait is bounded
// and gives up early once another role has failed; the producer then waits
// for its own loads in flight and the MMA thread for its MMAs before the
// TMEM is freed.
template <int BN>
struct PTile {
    static constexpr int kStages = BN == 256 ? 4 : 6;
    static constexpr int kABytes = BM * BK * 2;
    static constexpr int kBBytes = BN * BK * 2;
    static constexpr int kRing = kStages * (kABytes + kBBytes);
    static constexpr int kSmem = kRing + 1024 + 256;  // + alignment, barriers
};
constexpr int kEpiWarps = 8;  // two per TMEM lane quarter
constexpr int kPThreads = 64 + 32 * kEpiWarps;

struct TileGrid {
    int tn;      // column blocks (N / BN)
    int tmn;     // row blocks x column blocks
    int tiles;   // tmn x splits
    int splits;
};

template <int EPI, int BN>
__global__ void __launch_bounds__(kPThreads, 1)
    k_gemm_bf16_ws(const __grid_constant__ CUtensorMap tmA,
                   const __grid_constant__ CUtensorMap tmB, int K, int a_row0,
                   int a_k0, int b_row0, int b_k0, TileGrid tg, EpiArgs ep,
                   unsigned* __restrict__ err) {
    constexpr int S = PTile<BN>::kStages;
    constexpr int kABytes = PTile<BN>::kABytes, kBBytes = PTile<BN>::kBBytes;
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    const uint32_t s0 = smem_u32(smem_raw);
    unsigned char* base = smem_raw + ((1024u - (s0 & 1023u)) & 1023u);
    unsigned char* sA = base;
    unsigned char* sB = base + S * kABytes;
    uint64_t* full = reinterpret_cast<uint64_t*>(base + PTile<BN>::kRing);
    uint64_t* empty = full + S;
    uint64_t* acc_full = empty + S;   // [2]
    uint64_t* acc_empty = acc_full + 2;  // [2]
    uint64_t* fin = acc_empty + 2;
    uint32_t* tslot = reinterpret_cast<uint32_t*>(fin + 1);
    volatile int* abort = reinterpret_cast<volatile int*>(tslot + 1);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int nkb_all = K / BK;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&full[s], 1);
            mbar_init(&empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&acc_full[b], 1);
            mbar_init(&acc_empty[b], kEpiWarps);
        }
        mbar_init(fin, 1);
        *abort = 0;
        fence_mbar_init();
        tma_prefetch_map(&tmA);
        tma_prefetch_map(&tmB);
    }
    if (warp == 1) {
        tmem_alloc(tslot, 2 * BN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = *tslot;

    if (warp == 0) {
        if (lane == 0) {  // TMA producer
            uint32_t it = 0;  // k-slices issued so far (all tiles)
            bool ok = true;
            for (int t = blockIdx.x; ok && t < tg.tiles; t += gridDim.x) {
                const int z = t / tg.tmn, r = t - z * tg.tmn;
                const int m0 = (r / tg.tn) * BM, n0 = (r % tg.tn) * BN;
                const int kb0 = (int)(((long long)z * nkb_all) / tg.splits);
                const int kb1 = (int)(((long long)(z + 1) * nkb_all) / tg.splits);
                for (int kb = kb0; kb < kb1; ++kb, ++it) {
                    const uint32_t s = it % S, use = it / S;
                    if (use > 0 &&
                        !mbar_wait_abort(&empty[s], (use - 1) & 1, kWaitLimit, abort)) {
                        ok = false;
                        break;
                    }
                    mbar_expect_tx(&full[s], kABytes + kBBytes);
                    tma_load_2d(sA + s * kABytes, &tmA, &full[s], a_k0 + kb * BK,
                                a_row0 + m0);
                    tma_load_2d(sB + s * kBBytes, &tmB, &full[s], b_k0 + kb * BK,
                                b_row0 + n0);
                }
            }
            if (!ok) {
                *abort = 1;
                atomicOr(err, ERR_SPIN_TIMEOUT);
            }
            // Wait for the last load issued into each stage (already consumed
            // on the normal path), so no copy lands after the CTA ends.
            for (uint32_t s = 0; s < (uint32_t)S && s < it; ++s) {
                const uint32_t last_use = (it - 1 - s) / S;
                if (!mbar_wait(&full[s], last_use & 1, kWaitLimit))
                    atomicOr(err, ERR_SPIN_TIMEOUT);
            }
        }
        __syncwarp();
    } else if (warp == 1) {
        if (lane == 0) {  // MMA issuer
            constexpr uint32_t idesc = idesc_bf16_f32(BM, BN);
            uint32_t it = 0;
            int i = 0;  // tiles of this CTA so far
            bool ok = true;
            for (int t = blockIdx.x; ok && t < tg.tiles; t += gridDim.x, ++i) {
                const int z = t / tg.tmn;
                const int kb0 = (int)(((long long)z * nkb_all) / tg.splits);
                const int kb1 = (int)(((long long)(z + 1) * nkb_all) / tg.splits);
                const int b = i & 1, use = i >> 1;
                if (use > 0 &&
                    !mbar_wait_abort(&acc_empty[b], (use - 1) & 1, kWaitLimit, abort)) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                const uint32_t d = tmem + (uint32_t)(b * BN);
                for (int kb = kb0; kb < kb1; ++kb, ++it) {
                    const uint32_t s = it % S;
                    if (!mbar_wait_abort(&full[s], (it / S) & 1, kWaitLimit, abort)) {
                        ok = false;
                        break;
                    }
                    tc_fence_after();
                    const uint64_t ad = desc_kmajor_sw128(smem_u32(sA + s * kABytes));
                    const uint64_t bd = desc_kmajor_sw128(smem_u32(sB + s * kBBytes));
#pragma unroll
                    for (int k = 0; k < BK / 16; ++k)
                        mma_bf16(d, ad + 2 * k, bd + 2 * k, idesc,
                                 (kb != kb0 || k != 0) ? 1u : 0u);
                    mma_commit(&empty[s]);
                }
                if (ok) mma_commit(&acc_full[b]);
            }
            if (!ok) {
                *abort = 1;
                atomicOr(err, ERR_SPIN_TIMEOUT);
            }
            // Every MMA issued above has completed once fin's phase 0 ends.
            mma_commit(fin);
            if (!mbar_wait(fin, 0, kWaitLimit)) atomicOr(err, ERR_SPIN_TIMEOUT);
        }
        __syncwarp();
    } else {  // epilogue warps 2 .. kEpiWarps + 1
        const int q = warp & 3;
        constexpr int kPerQ = kEpiWarps / 4;  // warps sharing a lane quarter
        const int part = (warp - 2) / 4;      // which of them: chunks part, part + kPerQ, ...
        constexpr int kChunks = BN / 32;
        int i = 0;
        for (int t = blockIdx.x; t < tg.tiles; t += gridDim.x, ++i) {
            const int z = t / tg.tmn, r = t - z * tg.tmn;
            const int m0 = (r / tg.tn) * BM, n0 = (r % tg.tn) * BN;
            const int b = i & 1, use = i >> 1;
            const bool got = __all_sync(
                ~0u, mbar_wait_abort(&acc_full[b], use & 1, kWaitLimit, abort));
            if (!got) {
                if (lane == 0) {
                    *abort = 1;
                    atomicOr(err, ERR_SPIN_TIMEOUT);
                }
                break;
            }
            tc_fence_after();
            EpiArgs et = ep;
            if (EPI == EPI_F32)
                et.out = reinterpret_cast<float*>(ep.out) + (size_t)z * ep.split_stride;
            const int row = m0 + q * 32 + lane;
            const uint32_t trow = tmem + (uint32_t)(b * BN) + ((uint32_t)(q * 32) << 16);
#pragma unroll 1
            for (int c = part; c < kChunks; c += kPerQ) {
                uint32_t v[32];
                tmem_ld32(trow + (uint32_t)(c * 32), v);
                tmem_wait_ld();
                if (c + kPerQ >= kChunks) {  // this warp's last chunk: hand it back
                    tc_fence_before();
                    __syncwarp();
                    if (lane == 0) mbar_arrive(&acc_empty[b]);
                }
                epilogue_chunk<EPI>(v, row, n0 + c * 32,
                                    ep.bias ? ep.bias + n0 + c * 32 : nullptr, et);
            }
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tmem, 2 * BN);
    }
}

// ------------------------------------------------------------ tensor maps
typedef CUresult (*EncodeTiledFn)(CUtensorMap*, CUtensorMapDataType, cuuint32_t,
                                  void*, const cuuint64_t*, const cuuint64_t*,
                                  const cuuint32_t*, const cuuint32_t*,
                                  CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion,
                                  CUtensorMapFloatOOBfill);

EncodeTiledFn encode_fn() {
    static std::once_flag once;
    static EncodeTiledFn fn = nullptr;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p,
                                    cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    });
    return fn;
}

// Tensor map of a row-major rows x cols bf16 matrix with box_rows x 64 boxes
// and the 128-byte swizzle.
int make_map(CUtensorMap* m, const void* ptr, long long rows, long long cols,
             int box_rows) {
    EncodeTiledFn fn = encode_fn();
    if (!fn) {
        set_error("pf_b200: cuTensorMapEncodeTiled is unavailable");
        return -1;
    }
    if (((uintptr_t)ptr & 15u) || (cols * 2) % 16 || rows < BM || cols < BK) {
        set_error("pf_b200: tensor map: bad matrix %lld x %lld", rows, cols);
        return -1;
    }
    const cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    const cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    const cuuint32_t box[2] = {(cuuint32_t)BK, (cuuint32_t)box_rows};
    const cuuint32_t es[2] = {1, 1};
    const CUresult r =
        fn(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void*>(ptr), dims,
           strides, box, es, CU_TENSOR_MAP_INTERLEAVE_NONE,
           CU_TENSOR_MAP_SWIZZLE_128B, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
           CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) {
        set_error("pf_b200: cuTensorMapEncodeTiled failed (%d)", (int)r);
        return -1;
    }
    return 0;
}

// A bf16 matrix as a GEMM operand: tensor maps with 128-row and (when the
// matrix has at least 256 rows) 256-row boxes.
struct Mat {
    CUtensorMap m128, m256;
    bool has256 = false;
};

int make_mat(Mat* m, const void* ptr, long long rows, long long cols) {
    if (make_map(&m->m128, ptr, rows, cols, 128)) return -1;
    m->has256 = rows >= 256;
    if (m->has256 && make_map(&m->m256, ptr, rows, cols, 256)) return -1;
    return 0;
}

struct MapRef {
    const Mat* map;
    int row0;
    int k0;
};

int sm_count() {
    static std::once_flag once;
    static int n = 148;
    std::call_once(once, [] {
        int dev = 0, v = 0;
        if (cudaGetDevice(&dev) == cudaSuccess &&
            cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) ==
                cudaSuccess &&
            v > 0)
            n = v;
    });
    return n;
}

template <int EPI, int BN>
int gemm_bn(cudaStream_t s, MapRef a, MapRef b, int M, int N, int K,
            const EpiArgs& ep, unsigned* err, int splits) {
    constexpr int smem = PTile<BN>::kSmem;
    PFB_CK(cudaFuncSetAttribute(k_gemm_bf16_ws<EPI, BN>,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    TileGrid tg;
    tg.tn = N / BN;
    tg.tmn = (M / BM) * tg.tn;
    tg.tiles = tg.tmn * splits;
    tg.splits = splits;
    const int grid = std::min(tg.tiles, sm_count());
    const CUtensorMap& tb = BN == 256 ? b.map->m256 : b.map->m128;
    k_gemm_bf16_ws<EPI, BN><<<grid, kPThreads, smem, s>>>(
        a.map->m128, tb, K, a.row0, a.k0, b.row0, b.k0, tg, ep, err);
    PFB_KL();
    return 0;
}

// D = A B^T.  The 128 x 256 tile is used when N allows it and it still gives
// at least one CTA per SM; otherwise 128 x 128.
template <int EPI>
int gemm(cudaStream_t s, MapRef a, MapRef b, int M, int N, int K,
         const EpiArgs& ep, unsigned* err, int splits = 1) {
    if (M <= 0 || N <= 0 || K <= 0 || M % BM || N % 128 || K % BK ||
        (a.k0 % 8) || (b.k0 % 8) || splits < 1 || splits > K / BK ||
        (splits > 1 && EPI != EPI_F32)) {
        set_error("pf_b200: gemm shape %d x %d x %d (split %d) not tileable", M, N,
                  K, splits);
        return -1;
    }
    const bool wide = N % 256 == 0 && b.map->has256 &&
                      (long long)(M / BM) * (N / 256) * splits >= 148;
    return wide ? gemm_bn<EPI, 256>(s, a, b, M, N, K, ep, err, splits)
                : gemm_bn<EPI, 128>(s, a, b, M, N, K, ep, err, splits);
}

// ------------------------------------------------------- elementwise kernels

__device__ __forceinline__ float warp_max_f(float v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v = fmaxf(v, __shfl_xor_sync(~0u, v, o));
    return v;
}

__device__ __forceinline__ float sigmoidf_(float x) { return 1.0f / (1.0f + expf(-x)); }

// Mixture negative log-likelihood and its gradient with respect to the 288
// used outputs, one warp per sample (lane c = component c):
//   log pi_c = logit_c - LSE(logit)
//   ls_cd = LS_LO + (LS_HI - LS_LO) sigmoid(raw_cd),  sigma = exp(ls)
//   z_cd = (y_d - mu_cd) / sigma_cd
//   a_c = log pi_c - sum_d (z^2 / 2 + ls_cd + log(2 pi) / 2)
//   loss = -LSE(a),  r_c = exp(a_c + loss)   (responsibilities)
//   dloss/dlogit_c = pi_c - r_c;  dloss/dmu = -r z / sigma;
//   dloss/draw = r (1 - z^2) (LS_HI - LS_LO) s (1 - s)
// Gradients are scaled by inv_b (mean over the batch) and written as bf16
// (padding columns 288..383 zero).
__global__ void __launch_bounds__(256)
    k_gmm_loss(const float* __restrict__ Z, const float* __restrict__ Y, int y_row0,
               int rows, float inv_b, bf16* __restrict__ dZ, float* __restrict__ loss_acc) {
    __shared__ float s_loss[8];
    const int wid = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    float loss = 0.0f;
    if (wid < rows) {
        const float* z = Z + (size_t)wid * kOut;
        const float* y = Y + (size_t)(y_row0 + wid) * 4;
        const float logit = z[lane];
        const float yv[4] = {y[0], y[1], y[2], y[3]};
        // component `lane`: its 4 means and 4 log-sigma pre-activations are
        // consecutive (one 16-byte load each)
        const float4 mu4 = reinterpret_cast<const float4*>(z + kMeanOff)[lane];
        const float4 raw4 = reinterpret_cast<const float4*>(z + kSigOff)[lane];
        const float mu[4] = {mu4.x, mu4.y, mu4.z, mu4.w};
        const float raw[4] = {raw4.x, raw4.y, raw4.z, raw4.w};
        const float mx = warp_max_f(logit);
        const float lse_l = mx + logf(warp_sum_f(expf(logit - mx)));
        const float logpi = logit - lse_l;
        const float pi = expf(logpi);
        float zz[4], sg[4], sig[4];
        float nll = 4.0f * kHalfLog2Pi;
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            const float sgm = sigmoidf_(raw[d]);
            const float ls = kLsLo + (kLsHi - kLsLo) * sgm;
            sg[d] = sgm;
            sig[d] = expf(ls);
            zz[d] = (yv[d] - mu[d]) / sig[d];
            nll += 0.5f * zz[d] * zz[d] + ls;
        }
        const float a = logpi - nll;
        const float amx = warp_max_f(a);
        const float logp = amx + logf(warp_sum_f(expf(a - amx)));
        const float r = expf(a - logp);
        loss = -logp * inv_b;
        bf16* o = dZ + (size_t)wid * kOut;
        o[lane] = __float2bfloat16_rn((pi - r) * inv_b);
        bf16 gm[4], gs[4];
#pragma unroll
        for (int d = 0; d < 4; ++d) {
            gm[d] = __float2bfloat16_rn(-r * zz[d] / sig[d] * inv_b);
            gs[d] = __float2bfloat16_rn(r * (1.0f - zz[d] * zz[d]) * (kLsHi - kLsLo) *
                                        sg[d] * (1.0f - sg[d]) * inv_b);
        }
        uint2 pm, ps;
        pm.x = (uint32_t)__bfloat16_as_ushort(gm[0]) | ((uint32_t)__bfloat16_as_ushort(gm[1]) << 16);
        pm.y = (uint32_t)__bfloat16_as_ushort(gm[2]) | ((uint32_t)__bfloat16_as_ushort(gm[3]) << 16);
        ps.x = (uint32_t)__bfloat16_as_ushort(gs[0]) | ((uint32_t)__bfloat16_as_ushort(gs[1]) << 16);
        ps.y = (uint32_t)__bfloat16_as_ushort(gs[2]) | ((uint32_t)__bfloat16_as_ushort(gs[3]) << 16);
        reinterpret_cast<uint2*>(o + kMeanOff)[lane] = pm;
        reinterpret_cast<uint2*>(o + kSigOff)[lane] = ps;
        for (int p = kUsedOut + lane; p < kOut; p += 32) o[p] = __float2bfloat16_rn(0.0f);
    }
    // one atomic per block: the block's samples in warp order
    if (lane == 0) s_loss[threadIdx.x >> 5] = loss;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += s_loss[k];
        atomicAdd(loss_acc, t);
    }
}

// out[c][r] = in[r][c] for an R x C bf16 matrix, in 64 x 64 tiles through
// shared memory; tile rows are read and written as bf16 pairs (4-byte
// accesses, 128 bytes per warp) where the strides and base addresses allow.
__global__ void k_transpose_bf16(const bf16* __restrict__ in, long long ld_in,
                                 bf16* __restrict__ out, long long ld_out,
                                 long long R, long long C) {
    __shared__ bf16 t[64][66];
    const long long c0 = (long long)blockIdx.x * 64, r0 = (long long)blockIdx.y * 64;
    const int tx = threadIdx.x, ty = threadIdx.y;  // 32 x 8
    const bool vin = (ld_in & 1) == 0 && (reinterpret_cast<uintptr_t>(in) & 3) == 0;
    const bool vout = (ld_out & 1) == 0 && (reinterpret_cast<uintptr_t>(out) & 3) == 0;
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int i = ty + 8 * k;
        const long long r = r0 + i, c = c0 + 2 * tx;
        if (r >= R) continue;
        const bf16* src = in + r * ld_in + c;
        if (vin && c + 1 < C) {
            const __nv_bfloat162 v = *reinterpret_cast<const __nv_bfloat162*>(src);
            t[i][2 * tx] = v.x;
            t[i][2 * tx + 1] = v.y;
        } else {
            if (c < C) t[i][2 * tx] = src[0];
            if (c + 1 < C) t[i][2 * tx + 1] = src[1];
        }
    }
    __syncthreads();
#pragma unroll
    for (int k = 0; k < 8; ++k) {
        const int i = ty + 8 * k;
        const long long c = c0 + i, r = r0 + 2 * tx;
        if (c >= C) continue;
        bf16* dst = out + c * ld_out + r;
        if (vout && r + 1 < R) {
            __nv_bfloat162 v;
            v.x = t[2 * tx][i];
            v.y = t[2 * tx + 1][i];
            *reinterpret_cast<__nv_bfloat162*>(dst) = v;
        } else {
            if (r < R) dst[0] = t[2 * tx][i];
            if (r + 1 < R) dst[1] = t[2 * tx + 1][i];
        }
    }
}

// out[o] = sum over cols of in[o][*] (bf16 rows, f32 sum), one 256-thread
// block per row: thread t sums the 8-element chunks t, t + 256, ... (16-byte
// loads, all issued together), then the block adds the threads in a fixed
// order.
__device__ __forceinline__ float bf16x2_sum(uint32_t u) {
    const float2 f = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&u));
    return f.x + f.y;
}

__global__ void __launch_bounds__(256)
    k_rowsum_bf16(const bf16* __restrict__ in, int ld, int cols, int rows,
                  float* __restrict__ out) {
    __shared__ float s_w[8];
    const int row = blockIdx.x;
    if (row >= rows) return;
    const bf16* p = in + (size_t)row * ld;
    float acc = 0.0f;
    if ((cols & 7) == 0 && (reinterpret_cast<uintptr_t>(p) & 15) == 0) {
        const uint4* q = reinterpret_cast<const uint4*>(p);
        const int nq = cols >> 3;
#pragma unroll 4
        for (int c = threadIdx.x; c < nq; c += 256) {
            const uint4 u = q[c];
            acc += (bf16x2_sum(u.x) + bf16x2_sum(u.y)) + (bf16x2_sum(u.z) + bf16x2_sum(u.w));
        }
    } else {
        for (int c = threadIdx.x; c < cols; c += 256) acc += __bfloat162float(p[c]);
    }
    acc = warp_sum_f(acc);
    if ((threadIdx.x & 31) == 0) s_w[threadIdx.x >> 5] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        float t = 0.0f;
        for (int k = 0; k < 8; ++k) t += s_w[k];
        out[row] = t;
    }
}

// Adam on one weight matrix [out][in] (f32 master, moments) followed by the
// bf16 copies W [out][in] and W^T [in][out]; 32 x 32 tiles, 256 threads, one
// float4 of a tile row per thread (every load of the tile issued at once),
// the transposed copy through shared memory in 8-byte stores.  The blocks of
// tile column 0 also update the 32 biases of their rows (b, mb, vb from gb).
// With update == 0 only the bf16 copies are refreshed from the masters.
__device__ __forceinline__ void adam_one(float& w, float& m, float& v, float g, float lr,
                                         float b1, float b2, float eps, float bc1,
                                         float bc2) {
    m = b1 * m + (1.0f - b1) * g;
    v = b2 * v + (1.0f - b2) * g * g;
    w -= lr * (m / bc1) / (sqrtf(v / bc2) + eps);
}

__global__ void __launch_bounds__(256)
    k_adam_w(int out, int in, float* __restrict__ w, float* __restrict__ m,
             float* __restrict__ v, const float* __restrict__ g, int splits,
             bf16* __restrict__ wb, bf16* __restrict__ wtb, float* __restrict__ b,
             float* __restrict__ mb, float* __restrict__ vb, const float* __restrict__ gb,
             int update, float lr, float b1, float b2, float eps, float bc1, float bc2) {
    // g holds `splits` partial gradients of out*in floats each, summed in
    // split order.
    const size_t nw = (size_t)out * in;
    __shared__ bf16 t[32][36];
    const int i0 = blockIdx.x * 32, o0 = blockIdx.y * 32;
    const int rr = threadIdx.x >> 3, q = threadIdx.x & 7;
    const size_t idx = (size_t)(o0 + rr) * in + i0 + 4 * q;
    float4 ww = *reinterpret_cast<const float4*>(w + idx);
    if (update) {
        float4 gg = *reinterpret_cast<const float4*>(g + idx);
        for (int sp = 1; sp < splits; ++sp) {
            const float4 o = *reinterpret_cast<const float4*>(g + sp * nw + idx);
            gg.x += o.x;
            gg.y += o.y;
            gg.z += o.z;
            gg.w += o.w;
        }
        float4 mm = *reinterpret_cast<const float4*>(m + idx);
        float4 vv = *reinterpret_cast<const float4*>(v + idx);
        adam_one(ww.x, mm.x, vv.x, gg.x, lr, b1, b2, eps, bc1, bc2);
        adam_one(ww.y, mm.y, vv.y, gg.y, lr, b1, b2, eps, bc1, bc2);
        adam_one(ww.z, mm.z, vv.z, gg.z, lr, b1, b2, eps, bc1, bc2);
        adam_one(ww.w, mm.w, vv.w, gg.w, lr, b1, b2, eps, bc1, bc2);
        *reinterpret_cast<float4*>(m + idx) = mm;
        *reinterpret_cast<float4*>(v + idx) = vv;
        *reinterpret_cast<float4*>(w + idx) = ww;
        if (blockIdx.x == 0 && threadIdx.x < 32) {
            const int o = o0 + threadIdx.x;
            float bb = b[o], bm = mb[o], bv = vb[o];
            adam_one(bb, bm, bv, gb[o], lr, b1, b2, eps, bc1, bc2);
            b[o] = bb;
            mb[o] = bm;
            vb[o] = bv;
        }
    }
    const bf16 h[4] = {__float2bfloat16_rn(ww.x), __float2bfloat16_rn(ww.y),
                       __float2bfloat16_rn(ww.z), __float2bfloat16_rn(ww.w)};
    uint2 pk;
    pk.x = (uint32_t)__bfloat16_as_ushort(h[0]) | ((uint32_t)__bfloat16_as_ushort(h[1]) << 16);
    pk.y = (uint32_t)__bfloat16_as_ushort(h[2]) | ((uint32_t)__bfloat16_as_ushort(h[3]) << 16);
    *reinterpret_cast<uint2*>(wb + idx) = pk;
#pragma unroll
    for (int j = 0; j < 4; ++j) t[rr][4 * q + j] = h[j];
    __syncthreads();
    // transposed row i0 + c, columns o0 + 4 q .. + 3
    const int c = threadIdx.x >> 3;
    uint2 pt;
    pt.x = (uint32_t)__bfloat16_as_ushort(t[4 * q][c]) |
           ((uint32_t)__bfloat16_as_ushort(t[4 * q + 1][c]) << 16);
    pt.y = (uint32_t)__bfloat16_as_ushort(t[4 * q + 2][c]) |
           ((uint32_t)__bfloat16_as_ushort(t[4 * q + 3][c]) << 16);
    *reinterpret_cast<uint2*>(wtb + (size_t)(i0 + c) * out + o0 + 4 * q) = pt;
}

// Sum split-K partial gradients into split 0 (split order).
__global__ void k_sum_splits(float* __restrict__ g, int splits, long long nw) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= nw) return;
    float acc = g[i];
    for (int sp = 1; sp < splits; ++sp) acc += g[sp * nw + i];
    g[i] = acc;
}

// He-uniform initialisation from Philox (counter (i, layer, part, INIT)).
__global__ void k_init_uniform(float* __restrict__ p, long long n, float lo,
                               float hi, uint32_t layer, uint32_t part,
                               uint64_t seed) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const U4 r = philox4x32_10({(uint32_t)i, layer, part, RNG_LP_INIT},
                               (uint32_t)seed, (uint32_t)(seed >> 32));
    p[i] = lo + (hi - lo) * u01_open(r.x);
}

__global__ void k_f32_to_bf16(const float* __restrict__ in, bf16* __restrict__ out,
                              long long n) {
    const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __float2bfloat16_rn(in[i]);
}

// --------------------------------------------------------- scan rendering

struct RenderArgs {
    GridView gv;
    int grid_bytes;
    int nrays;
    float rmax, span, noise;
    uint64_t seed;
    float cx, cy, sx, sy;  // pose normalisation
};

// Scan of one pose by one warp: lanes take groups of 4 consecutive rays; the
// range noise of group q of sample `id` comes from Philox counter
// (id, q, 0, LP_NOISE).  Writes f32 ranges (out_f, may be null) and/or the
// network input row bf16(range / rmax) padded with zeros to kIn (out_x).
__device__ __forceinline__ void render_pose(const RenderArgs& a,
                                            const unsigned char* g, float x,
                                            float y, float th, uint32_t id,
                                            float* out_f, bf16* out_x) {
    const int lane = threadIdx.x & 31;
    int start = 0;
    float frx = 0.f, fry = 0.f;
    const bool inside = start_cell(a.gv, x, y, start, frx, fry);
    const float inv_rmax = 1.0f / a.rmax;
    const int ngroups = (a.nrays + 3) / 4;
    for (int q = lane; q < ngroups; q += 32) {
        const U4 u = philox4x32_10({id, (uint32_t)q, 0u, RNG_LP_NOISE},
                                   (uint32_t)a.seed, (uint32_t)(a.seed >> 32));
        const float2 n01 = box_muller(u01_open(u.x), u01_open(u.y));
        const float2 n23 = box_muller(u01_open(u.z), u01_open(u.w));
        const float nz[4] = {n01.x, n01.y, n23.x, n23.y};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const int r = 4 * q + t;
            if (r >= a.nrays) break;
            float d = a.rmax;
            if (inside) {
                float dx, dy;
                sincosf(ray_angle(th, r, a.nrays, a.span), &dy, &dx);
                d = cast_ray(g, a.gv.Wp, start, frx, fry, dx, dy, a.gv.res, a.rmax);
            }
            const float val = d + a.noise * nz[t];
            if (out_f) out_f[r] = val;
            if (out_x) out_x[r] = __float2bfloat16_rn(val * inv_rmax);
        }
    }
    if (out_x)
        for (int r = a.nrays + lane; r < kIn; r += 32)
            out_x[r] = __float2bfloat16_rn(0.0f);
}

// Uniform pose of sample id: free cell + in-cell offset, yaw in [0, 2 pi).
__device__ __forceinline__ void random_pose(const RenderArgs& a, int nfree,
                                            const int2* __restrict__ free_cells,
                                            uint32_t id, uint32_t stream,
                                            float& x, float& y, float& th) {
    const U4 u = philox4x32_10({id, stream, 0u, RNG_LP_POSE}, (uint32_t)a.seed,
                               (uint32_t)(a.seed >> 32));
    const int c = min((int)(u01_open(u.w) * (float)nfree), nfree - 1);
    const int2 cell = free_cells[c];
    x = a.gv.ox + ((float)cell.x + u01_open(u.x)) * a.gv.res;
    y = a.gv.oy + ((float)cell.y + u01_open(u.y)) * a.gv.res;
    th = 6.28318530f * (u01_open(u.z) - 0.5f / 8388608.0f);
}

__device__ __forceinline__ const unsigned char* stage_grid(const RenderArgs& a,
                                                           unsigned char* smem) {
    const int nv = a.grid_bytes / 16;
    const uint4* src = reinterpret_cast<const uint4*>(a.gv.cells);
    uint4* dst = reinterpret_cast<uint4*>(smem);
    for (int k = threadIdx.x; k < nv; k += blockDim.x) dst[k] = __ldg(&src[k]);
    __syncthreads();
    return smem;
}

// Training pairs [i0, i0 + n): random pose, rendered scan -> X row, target
// (x_n, y_n, cos, sin) -> Y row.  Persistent blocks, grid in shared memory.
__global__ void __launch_bounds__(256)
    k_make_pairs(RenderArgs a, int nfree, const int2* __restrict__ free_cells,
                 long long i0, long long n, bf16* __restrict__ X,
                 float* __restrict__ Y) {
    extern __shared__ __align__(16) unsigned char smem[];
    const unsigned char* g = stage_grid(a, smem);
    const int lane = threadIdx.x & 31;
    const long long nw = (long long)gridDim.x * (blockDim.x >> 5);
    for (long long w = (long long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
         w < n; w += nw) {
        const long long i = i0 + w;
        float x, y, th;
        random_pose(a, nfree, free_cells, (uint32_t)i, (uint32_t)(i >> 32), x, y, th);
        render_pose(a, g, x, y, th, (uint32_t)i, nullptr, X + (size_t)i * kIn);
        if (lane == 0) {
            float* t = Y + (size_t)i * 4;
            t[0] = (x - a.cx) / a.sx;
            t[1] = (y - a.cy) / a.sy;
            t[2] = cosf(th);
            t[3] = sinf(th);
        }
    }
}

// Scans at caller poses (one warp per pose).
__global__ void __launch_bounds__(256)
    k_render(RenderArgs a, const float* __restrict__ pose, int n,
             float* __restrict__ out) {
    extern __shared__ __align__(16) unsigned char smem[];
    const unsigned char* g = stage_grid(a, smem);
    const int nw = gridDim.x * (blockDim.x >> 5);
    for (int w = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5); w < n; w += nw)
        render_pose(a, g, pose[3 * w], pose[3 * w + 1], pose[3 * w + 2],
                    (uint32_t)w, out + (size_t)w * a.nrays, nullptr);
}

// Uniform held-out poses (same generator as the training pairs, own seed).
__global__ void k_random_poses(RenderArgs a, int nfree,
                               const int2* __restrict__ free_cells, int n,
                               float* __restrict__ pose) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    float x, y, th;
    random_pose(a, nfree, free_cells, (uint32_t)i, 0u, x, y, th);
    pose[3 * i] = x;
    pose[3 * i + 1] = y;
    pose[3 * i + 2] = th;
}

// Network input row 0 from a device scan: bf16(scan / rmax), zero padded.
__global__ void k_query_row(const float* __restrict__ scan, int nrays,
                            float inv_rmax, bf16* __restrict__ x) {
    for (int r = threadIdx.x; r < kIn; r += blockDim.x)
        x[r] = __float2bfloat16_rn(r < nrays ? scan[r] * inv_rmax : 0.0f);
}

// One row through one layer (a query's forward pass): warp w of the block
// computes output n = 8 blockIdx + w as the f32 dot product of the bf16
// weight row n (16-byte loads) with the bf16 input row, then the GEMM
// epilogue: bf16 relu(acc + bias) for hidden layers, f32 acc + bias for the
// output layer.  Same arithmetic as the tiled GEMM up to the f32 summation
// order; eight warps stream 16 KB of weights where a 128-row tcgen05 tile
// would run almost empty.
template <bool kRelu>
__global__ void __launch_bounds__(256)
    k_gemv_bf16(const bf16* __restrict__ W, const bf16* __restrict__ x,
                const float* __restrict__ b, int in, int out, bf16* __restrict__ yb,
                float* __restrict__ yf) {
    const int n = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (n >= out) return;
    const uint4* w4 = reinterpret_cast<const uint4*>(W + (size_t)n * in);
    const uint4* x4 = reinterpret_cast<const uint4*>(x);
    float acc = 0.f;
    for (int q = lane; q < in / 8; q += 32) {
        const uint4 a = __ldg(&w4[q]), c = x4[q];
        const uint32_t aw[4] = {a.x, a.y, a.z, a.w}, cw[4] = {c.x, c.y, c.z, c.w};
#pragma unroll
        for (int t = 0; t < 4; ++t) {
            const float2 fa = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&aw[t]));
            const float2 fc = __bfloat1622float2(*reinterpret_cast<const __nv_bfloat162*>(&cw[t]));
            acc = fmaf(fa.x, fc.x, acc);
            acc = fmaf(fa.y, fc.y, acc);
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_xor_sync(~0u, acc, o);
    if (lane == 0) {
        const float v = acc + b[n];
        if (kRelu)
            yb[n] = __float2bfloat16_rn(fmaxf(v, 0.0f));
        else
            yf[n] = v;
    }
}

// The mixture of one network output row Z in shared memory: cumulative
// component weights (softmax of the logits), means and standard deviations.
struct MixtureSmem {
    float cum[kComp];
    float mu[4 * kComp], sig[4 * kComp];
};

__device__ __forceinline__ void load_mixture(const float* __restrict__ Z, MixtureSmem& m) {
    const int t = threadIdx.x;
    if (t < 32) {
        const float l = Z[t];
        const float mx = warp_max_f(l);
        float e = expf(l - mx);
        float c = e;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const float o = __shfl_up_sync(~0u, c, d);
            if (t >= d) c += o;
        }
        const float tot = __shfl_sync(~0u, c, 31);
        m.cum[t] = c / tot;
    }
    if (t < 4 * kComp) {
        m.mu[t] = Z[kMeanOff + t];
        const float s = sigmoidf_(Z[kSigOff + t]);
        m.sig[t] = expf(kLsLo + (kLsHi - kLsLo) * s);
    }
    __syncthreads();
}

// Sample i of a query: component by inverse CDF, then a diagonal Gaussian
// draw in (x_n, y_n, c, s); yaw = atan2(s, c).  Philox counters (i, query,
// 0/1, LP_SAMPLE).
__device__ __forceinline__ void draw_sample(const MixtureSmem& m, int i, uint64_t seed,
                                            uint32_t query, float cx, float cy, float sx,
                                            float sy, float* __restrict__ out3) {
    const uint32_t k0 = (uint32_t)seed, k1 = (uint32_t)(seed >> 32);
    const U4 a = philox4x32_10({(uint32_t)i, query, 0u, RNG_LP_SAMPLE}, k0, k1);
    const U4 b = philox4x32_10({(uint32_t)i, query, 1u, RNG_LP_SAMPLE}, k0, k1);
    const float uc = u01_open(a.x);
    int c = kComp - 1;
    for (int j = 0; j < kComp; ++j)
        if (m.cum[j] >= uc) {
            c = j;
            break;
        }
    const float2 n01 = box_muller(u01_open(a.y), u01_open(a.z));
    const float2 n23 = box_muller(u01_open(a.w), u01_open(b.x));
    const float* mu = m.mu + 4 * c;
    const float* sg = m.sig + 4 * c;
    const float xn = mu[0] + sg[0] * n01.x;
    const float yn = mu[1] + sg[1] * n01.y;
    const float cc = mu[2] + sg[2] * n23.x;
    const float ss = mu[3] + sg[3] * n23.y;
    out3[0] = cx + sx * xn;
    out3[1] = cy + sy * yn;
    out3[2] = atan2f(ss, cc);
}

// n hypotheses from the mixture in Z row 0 (query counter `query`, or read
// from query_dev on a graph replay).
__global__ void k_lp_sample(const float* __restrict__ Z, int n, uint64_t seed,
                            uint32_t query, float cx, float cy, float sx,
                            float sy, float* __restrict__ hyp,
                            const uint32_t* __restrict__ query_dev) {
    if (query_dev) query = *query_dev;  // graph replay: this query's counter
    __shared__ MixtureSmem m;
    load_mixture(Z, m);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    draw_sample(m, i, seed, query, cx, cy, sx, sy, hyp + 3 * (size_t)i);
}

// A batch of queries: query q (blockIdx.y) draws its n samples from output
// row q of Z with counter query0 + q into hyp[q * n, (q + 1) * n).
__global__ void k_lp_sample_multi(const float* __restrict__ Z, int n, uint64_t seed,
                                  uint32_t query0, float cx, float cy, float sx, float sy,
                                  float* __restrict__ hyp) {
    const int q = blockIdx.y;
    __shared__ MixtureSmem m;
    load_mixture(Z + (size_t)q * kOut, m);
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    draw_sample(m, i, seed, query0 + (uint32_t)q, cx, cy, sx, sy,
                hyp + 3 * ((size_t)q * n + i));
}

// Network input rows [0, rows) from a batch of device scans: bf16(scan /
// rmax) zero padded to kIn columns; rows [nq, rows) all zero.
__global__ void k_query_rows(const float* __restrict__ scans, int nq, int nrays,
                             float inv_rmax, bf16* __restrict__ x, int rows) {
    const long long t = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= (long long)rows * kIn) return;
    const int r = (int)(t / kIn), c = (int)(t - (long long)r * kIn);
    x[t] = __float2bfloat16_rn(r < nq && c < nrays ? scans[(size_t)r * nrays + c] * inv_rmax
                                                   : 0.0f);
}

// ------------------------------------------------------------------ handle

struct Layer {
    int in = 0, out = 0;
    float* w = nullptr;   // [out][in] f32 master
    float* b = nullptr;   // [out]
    float* mw = nullptr;  // Adam moments
    float* vw = nullptr;
    float* mb = nullptr;
    float* vb = nullptr;
    float* gw = nullptr;  // weight gradient: `splits` partials of out*in
    int splits = 1;
    float* gb = nullptr;
    bf16* wb = nullptr;   // [out][in]
    bf16* wtb = nullptr;  // [in][out]
    Mat tm_w, tm_wt;
};

struct LpHandle {
    GlHandle* gl = nullptr;
    cudaStream_t stream = nullptr;
    int batch = 0;
    uint64_t seed = 0;
    Layer L[kLayers];
    bf16* H[kLayers - 1] = {};
    bf16* HT[kLayers - 1] = {};
    bf16* dZ[kLayers] = {};
    bf16* dZT[kLayers] = {};
    float* Z4 = nullptr;
    Mat tm_H[kLayers - 1], tm_HT[kLayers - 1], tm_dZ[kLayers], tm_dZT[kLayers];
    // training pairs
    bf16* X = nullptr;
    bf16* XT = nullptr;
    float* Y = nullptr;
    long long n_pairs = 0;
    Mat tm_X, tm_XT;
    int data_nrays = 360;
    float data_rmax = 10.0f;
    // caller inputs (gradient check, forward, queries): batch rows
    bf16* Xp = nullptr;
    bf16* XpT = nullptr;
    float* Xp_f = nullptr;
    float* Yp = nullptr;
    Mat tm_Xp, tm_XpT;
    // bookkeeping
    unsigned* d_err = nullptr;
    float* d_loss = nullptr;
    int loss_cap = 0;
    long long adam_t = 0;
    long long train_step = 0;
    float cx = 0, cy = 0, sx = 1, sy = 1;
    float tau = INFINITY;
    uint32_t query_count = 0;
    float* d_best = nullptr;
    // a query replayed from a CUDA graph: the query counter in device memory,
    // the results copied to pinned memory, the graph keyed on the query's
    // static parameters
    uint32_t* d_query = nullptr;
    float* h_res = nullptr;  // 3 kSelKMax poses, kSelKMax CAERs, kSelKMax indices
    cudaGraph_t q_graph = nullptr;
    cudaGraphExec_t q_exec = nullptr;
    int q_n = 0, q_k = 0, q_nrays = 0;
    float q_rmax = 0.f, q_span = 0.f;
    const float* q_scan = nullptr;
    bool q_caer_valid = false;
    bool q_off = false;  // capture failed once: direct launches from then on
};

constexpr int kSelKMax = 128;  // largest k of the small-set localizer

LpHandle* as_lp(void* p) { return static_cast<LpHandle*>(p); }

RenderArgs render_args_gl(const GlHandle* g, int nrays, float rmax, float span,
                          float noise, uint64_t seed) {
    RenderArgs a;
    a.gv = grid_view(g);
    a.grid_bytes = grid_bytes_padded(g);
    a.nrays = nrays;
    a.rmax = rmax;
    a.span = span;
    a.noise = noise;
    a.seed = seed;
    a.cx = g->ox + 0.5f * g->W * g->res;
    a.cy = g->oy + 0.5f * g->H * g->res;
    a.sx = 0.5f * g->W * g->res;
    a.sy = 0.5f * g->H * g->res;
    return a;
}

RenderArgs render_args(const LpHandle* h, int nrays, float rmax, float span,
                       float noise, uint64_t seed) {
    return render_args_gl(h->gl, nrays, rmax, span, noise, seed);
}

int check_err(LpHandle* h) {
    unsigned e = 0;
    PFB_CK(cudaMemcpyAsync(&e, h->d_err, sizeof(unsigned), cudaMemcpyDeviceToHost,
                           h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    if (e) {
        set_error("pf_b200: learned proposal kernel wait timed out (err %u)", e);
        cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->stream);
        return -1;
    }
    return 0;
}

// Refresh the bf16 weight copies of every layer from the f32 masters.
int round_weights(LpHandle* h) {
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        k_adam_w<<<dim3(L.in / 32, L.out / 32), 256, 0, h->stream>>>(
            L.out, L.in, L.w, L.mw, L.vw, L.gw, L.splits, L.wb, L.wtb, L.b, L.mb, L.vb,
            L.gb, 0, 0.f, 0.f, 0.f, 0.f, 1.f, 1.f);
    }
    PFB_KL();
    return 0;
}

// Forward pass over `rows` rows of the input map x (rows a multiple of 128).
int forward(LpHandle* h, MapRef x, int rows, bool write_t) {
    cudaStream_t s = h->stream;
    for (int l = 0; l < kLayers - 1; ++l) {
        EpiArgs ep{};
        ep.out = h->H[l];
        ep.outT = write_t ? h->HT[l] : nullptr;
        ep.bias = h->L[l].b;
        ep.ldo = h->L[l].out;
        ep.ldt = h->batch;
        const MapRef a = l == 0 ? x : MapRef{&h->tm_H[l - 1], 0, 0};
        if (gemm<EPI_RELU_BF16>(s, a, MapRef{&h->L[l].tm_w, 0, 0}, rows,
                                h->L[l].out, h->L[l].in, ep, h->d_err))
            return -1;
    }
    EpiArgs ep{};
    ep.out = h->Z4;
    ep.bias = h->L[kLayers - 1].b;
    ep.ldo = kOut;
    return gemm<EPI_BIAS_F32>(s, MapRef{&h->tm_H[kLayers - 2], 0, 0},
                              MapRef{&h->L[kLayers - 1].tm_w, 0, 0}, rows, kOut,
                              kHid, ep, h->d_err);
}

// Forward pass of the single query row in Xp row 0 (rows 0 of H[] and Z4).
int forward_one(LpHandle* h) {
    cudaStream_t s = h->stream;
    const bf16* x = h->Xp;
    for (int l = 0; l < kLayers - 1; ++l) {
        const Layer& L = h->L[l];
        k_gemv_bf16<true><<<ceil_div(L.out, 8), 256, 0, s>>>(L.wb, x, L.b, L.in, L.out,
                                                             h->H[l], nullptr);
        PFB_KL();
        x = h->H[l];
    }
    const Layer& L = h->L[kLayers - 1];
    k_gemv_bf16<false><<<ceil_div(L.out, 8), 256, 0, s>>>(L.wb, x, L.b, L.in, L.out,
                                                          nullptr, h->Z4);
    PFB_KL();
    return 0;
}

// Loss + backward over one batch (after forward); the loss is accumulated
// into *d_loss_slot.  xt: the transposed input rows (columns = samples); Y:
// the batch's targets.
int backward(LpHandle* h, MapRef xt, const float* Y, float* d_loss_slot) {
    cudaStream_t s = h->stream;
    const int B = h->batch;
    k_gmm_loss<<<ceil_div(B * 32, 256), 256, 0, s>>>(
        h->Z4, Y, 0, B, 1.0f / (float)B, h->dZ[kLayers - 1], d_loss_slot);
    PFB_KL();
    k_transpose_bf16<<<dim3(ceil_div(kOut, 64), ceil_div(B, 64)), dim3(32, 8), 0, s>>>(
        h->dZ[kLayers - 1], kOut, h->dZT[kLayers - 1], B, B, kOut);
    PFB_KL();
    for (int l = kLayers - 1; l >= 0; --l) {
        Layer& L = h->L[l];
        EpiArgs eg{};
        eg.out = L.gw;
        eg.ldo = L.in;
        eg.scale = 1.0f;
        eg.split_stride = (long long)L.out * L.in;
        const MapRef bt = l == 0 ? xt : MapRef{&h->tm_HT[l - 1], 0, 0};
        if (gemm<EPI_F32>(s, MapRef{&h->tm_dZT[l], 0, 0}, bt, L.out, L.in, B, eg,
                          h->d_err, L.splits))
            return -1;
        k_rowsum_bf16<<<L.out, 256, 0, s>>>(h->dZT[l], B, B, L.out, L.gb);
        PFB_KL();
        if (l > 0) {
            EpiArgs ed{};
            ed.out = h->dZ[l - 1];
            ed.outT = h->dZT[l - 1];
            ed.mask = h->H[l - 1];
            ed.ldo = L.in;
            ed.ldt = B;
            ed.ldm = L.in;
            if (gemm<EPI_DRELU_BF16>(s, MapRef{&h->tm_dZ[l], 0, 0},
                                     MapRef{&L.tm_wt, 0, 0}, B, L.in, L.out, ed,
                                     h->d_err))
                return -1;
        }
    }
    return 0;
}

int adam_update(LpHandle* h, float lr) {
    const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
    h->adam_t += 1;
    const float bc1 = 1.0f - powf(b1, (float)h->adam_t);
    const float bc2 = 1.0f - powf(b2, (float)h->adam_t);
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        // weights and biases of the layer in one launch
        k_adam_w<<<dim3(L.in / 32, L.out / 32), 256, 0, h->stream>>>(
            L.out, L.in, L.w, L.mw, L.vw, L.gw, L.splits, L.wb, L.wtb, L.b, L.mb, L.vb,
            L.gb, 1, lr, b1, b2, eps, bc1, bc2);
    }
    PFB_KL();
    return 0;
}

// Training pairs: the Y pointer passed to the loss kernel is already offset
// to the batch's first row.
int train_one(LpHandle* h, long long row0, float lr, float* d_loss_slot) {
    const MapRef x{&h->tm_X, (int)row0, 0};
    const MapRef xt{&h->tm_XT, 0, (int)row0};
    if (forward(h, x, h->batch, true)) return -1;
    if (backward(h, xt, h->Y + (size_t)row0 * 4, d_loss_slot)) return -1;
    return adam_update(h, lr);
}

void drop_query_graph(LpHandle* h);

void free_lp(LpHandle* h) {
    if (!h) return;
    if (h->stream) cudaStreamSynchronize(h->stream);
    drop_query_graph(h);
    cudaFree(h->d_query);
    if (h->h_res) cudaFreeHost(h->h_res);
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        cudaFree(L.w);
        cudaFree(L.b);
        cudaFree(L.mw);
        cudaFree(L.vw);
        cudaFree(L.mb);
        cudaFree(L.vb);
        cudaFree(L.gw);
        cudaFree(L.gb);
        cudaFree(L.wb);
        cudaFree(L.wtb);
        cudaFree(h->dZ[l]);
        cudaFree(h->dZT[l]);
    }
    for (int l = 0; l < kLayers - 1; ++l) {
        cudaFree(h->H[l]);
        cudaFree(h->HT[l]);
    }
    cudaFree(h->Z4);
    cudaFree(h->X);
    cudaFree(h->XT);
    cudaFree(h->Y);
    cudaFree(h->Xp);
    cudaFree(h->XpT);
    cudaFree(h->Xp_f);
    cudaFree(h->Yp);
    cudaFree(h->d_err);
    cudaFree(h->d_loss);
    cudaFree(h->d_best);
    delete h;
}

template <class T>
int dalloc(T** p, size_t count) {
    PFB_CK(cudaMalloc((void**)p, sizeof(T) * std::max<size_t>(count, 1)));
    return 0;
}

long long num_params() {
    long long n = 0;
    for (int l = 0; l < kLayers; ++l)
        n += (long long)layer_out(l) * layer_in(l) + layer_out(l);
    return n;
}

void drop_query_graph(LpHandle* h) {
    if (h->q_exec) cudaGraphExecDestroy(h->q_exec);
    if (h->q_graph) cudaGraphDestroy(h->q_graph);
    h->q_exec = nullptr;
    h->q_graph = nullptr;
}

// The kernels of a query up to the gathered bottom-k (asynchronous).  With
// query_dev the sampling counter is read from device memory.
int enqueue_query(LpHandle* h, int nrays, float rmax, float span, int n_samples,
                  int k, const uint32_t* query_dev, const uint64_t** sorted) {
    GlHandle* g = h->gl;
    k_query_row<<<1, 128, 0, h->stream>>>(g->d_scan, nrays, 1.0f / rmax, h->Xp);
    PFB_KL();
    if (forward_one(h)) return -1;
    k_lp_sample<<<ceil_div(n_samples, 256), 256, 0, h->stream>>>(
        h->Z4, n_samples, h->seed ^ 0x5DEECE66DULL, h->query_count, h->cx, h->cy,
        h->sx, h->sy, g->d_hyp, query_dev);
    PFB_KL();
    g->nh = n_samples;
    g->caer_valid = false;
    *sorted = gl_localize_small_keys(g, nrays, rmax, span, k);
    if (!*sorted) return -1;
    return gl_gather_topk(g, *sorted, k);
}

// A query of the small-set localizer replayed from a CUDA graph (captured on
// first use and again when n, k, the ray geometry or the scan buffer change):
// one launch and one synchronisation instead of about fifteen launches and
// pageable copies.  Same kernels and arguments as the direct path, so the
// same results.  Returns -2 when the graph cannot be used.
int learned_pass_graph(LpHandle* h, int nrays, float rmax, float span, int n_samples,
                       int k, float* out3k, float* caer_k, int* idx_k) {
    GlHandle* g = h->gl;
    if (h->q_off || !h->h_res || !gl_small_select_ok(n_samples, k) || k > kSelKMax)
        return -2;
    const bool same = h->q_exec && h->q_n == n_samples && h->q_k == k &&
                      h->q_nrays == nrays && h->q_rmax == rmax && h->q_span == span &&
                      h->q_scan == g->d_scan;
    if (!same) {
        drop_query_graph(h);
        if (cudaStreamBeginCapture(h->stream, cudaStreamCaptureModeRelaxed) !=
            cudaSuccess) {
            (void)cudaGetLastError();
            h->q_off = true;
            return -2;
        }
        const uint64_t* sorted = nullptr;
        int rc = enqueue_query(h, nrays, rmax, span, n_samples, k, h->d_query, &sorted);
        if (rc == 0) {
            const size_t kk = (size_t)k;
            rc |= cudaMemcpyAsync(h->h_res, g->d_out, sizeof(float) * 3 * kk,
                                  cudaMemcpyDeviceToHost, h->stream) != cudaSuccess;
            rc |= cudaMemcpyAsync(h->h_res + 3 * kSelKMax, g->d_outc, sizeof(float) * kk,
                                  cudaMemcpyDeviceToHost, h->stream) != cudaSuccess;
            rc |= cudaMemcpyAsync(h->h_res + 4 * kSelKMax, g->d_outi, sizeof(int) * kk,
                                  cudaMemcpyDeviceToHost, h->stream) != cudaSuccess;
        }
        cudaGraph_t gr = nullptr;
        const cudaError_t e = cudaStreamEndCapture(h->stream, &gr);
        if (rc || e != cudaSuccess || !gr ||
            cudaGraphInstantiate(&h->q_exec, gr, 0) != cudaSuccess) {
            if (gr) cudaGraphDestroy(gr);
            h->q_exec = nullptr;
            (void)cudaGetLastError();
            h->q_off = true;
            return -2;
        }
        h->q_graph = gr;
        h->q_n = n_samples;
        h->q_k = k;
        h->q_nrays = nrays;
        h->q_rmax = rmax;
        h->q_span = span;
        h->q_scan = g->d_scan;
        h->q_caer_valid = g->caer_valid;
    }
    // the counter is staged from pageable memory before the call returns
    PFB_CK(cudaMemcpyAsync(h->d_query, &h->query_count, sizeof(uint32_t),
                           cudaMemcpyHostToDevice, h->stream));
    PFB_CK(cudaGraphLaunch(h->q_exec, h->stream));
    PFB_CK(cudaStreamSynchronize(h->stream));
    h->query_count++;
    g->nh = n_samples;
    g->caer_valid = h->q_caer_valid;
    g->last_k = k;
    if (out3k) memcpy(out3k, h->h_res, sizeof(float) * 3 * (size_t)k);
    if (caer_k) memcpy(caer_k, h->h_res + 3 * kSelKMax, sizeof(float) * (size_t)k);
    if (idx_k) memcpy(idx_k, h->h_res + 4 * kSelKMax, sizeof(int) * (size_t)k);
    return k;
}

// Localize against the scan already in gl->d_scan with n learned samples.
int learned_pass(LpHandle* h, int nrays, float rmax, float span, int n_samples,
                 int k, float* out3k, float* caer_k, int* idx_k) {
    const int rg = learned_pass_graph(h, nrays, rmax, span, n_samples, k, out3k,
                                      caer_k, idx_k);
    if (rg != -2) return rg;
    GlHandle* g = h->gl;
    k_query_row<<<1, 128, 0, h->stream>>>(g->d_scan, nrays, 1.0f / rmax, h->Xp);
    PFB_KL();
    if (forward_one(h)) return -1;
    k_lp_sample<<<ceil_div(n_samples, 256), 256, 0, h->stream>>>(
        h->Z4, n_samples, h->seed ^ 0x5DEECE66DULL, h->query_count++, h->cx,
        h->cy, h->sx, h->sy, g->d_hyp, nullptr);
    PFB_KL();
    g->nh = n_samples;
    g->caer_valid = false;
    // the pruned localizer (one host synchronisation up to 64k samples)
    return gl_localize_loaded(g, nrays, rmax, span, k, out3k, caer_k, idx_k);
}

// A batch of nq queries whose scans are in gl->d_scans: the nq scan rows
// through the network with the tiled tcgen05 GEMM (rows padded to a multiple
// of 128), n_samples mixture samples per query (query counters query_count +
// q), exhaustive CAER of every sample and each query's bottom-k
// (gl_localize_batch_enqueue).  Asynchronous; query q's results land in
// gl->d_out / d_outc / d_outi at [q * k, q * k + k).
int learned_batch_enqueue(LpHandle* h, int nq, int nrays, float rmax, float span,
                          int n_samples, int k) {
    GlHandle* g = h->gl;
    const int rows = ceil_div(nq, BM) * BM;
    const long long nx = (long long)rows * kIn;
    k_query_rows<<<(unsigned)((nx + 255) / 256), 256, 0, h->stream>>>(
        g->d_scans, nq, nrays, 1.0f / rmax, h->Xp, rows);
    PFB_KL();
    if (forward(h, MapRef{&h->tm_Xp, 0, 0}, rows, false)) return -1;
    k_lp_sample_multi<<<dim3(ceil_div(n_samples, 256), nq), 256, 0, h->stream>>>(
        h->Z4, n_samples, h->seed ^ 0x5DEECE66DULL, h->query_count, h->cx, h->cy, h->sx,
        h->sy, g->d_hyp);
    PFB_KL();
    h->query_count += (uint32_t)nq;
    g->caer_valid = false;
    return gl_localize_batch_enqueue(g, nq, n_samples, nrays, rmax, span, k);
}

// Queries per chunk of a batch: the GEMM input rows, the hypothesis and
// result buffers of the map handle.
int batch_chunk(const LpHandle* h, int nq, int n_samples, int k) {
    const long long cap = h->gl->cap_hyp;
    long long c = std::min<long long>(nq, (h->batch / BM) * BM);
    c = std::min(c, cap / std::max(n_samples, 1));
    c = std::min(c, cap / std::max(k, 1));
    return (int)std::max(0LL, c);
}

// Learned localization of nq host scans in batches.  Query q's k best
// (poses, CAERs, sample indices) go to out3k/caer_k/idx_k at [q * k, ...);
// with n_fallback > 0 a query whose best CAER exceeds tau is localized again
// with n_fallback uniform hypotheses (the better bottom-k is kept; info[q]
// as pfgl_learned_localize).  best_out (optional): each query's best learned
// CAER before any fallback.  Returns k (clamped to n_samples) or -1.
int learned_localize_batch(LpHandle* h, const float* scans, int nq, int nrays, float rmax,
                           float span, int n_samples, int n_fallback, int k, float tau,
                           float* out3k, float* caer_k, int* idx_k, int* info,
                           float* best_out) {
    GlHandle* g = h->gl;
    if (k > n_samples) k = n_samples;
    const int chunk = batch_chunk(h, nq, n_samples, k);
    if (chunk <= 0 || !gl_batch_ok(g, chunk, n_samples, k)) {
        set_error("pf_b200: learned batch: %d samples per query (k %d) exceed the batch "
                  "limits", n_samples, k);
        return -1;
    }
    std::vector<float> o1(3 * (size_t)chunk * k), c1((size_t)chunk * k);
    std::vector<int> i1((size_t)chunk * k);
    for (int q0 = 0; q0 < nq; q0 += chunk) {
        const int m = std::min(chunk, nq - q0);
        const uint32_t qc0 = h->query_count;
        if (gl_upload_scans(g, scans + (size_t)q0 * nrays, m, nrays)) return -1;
        if (learned_batch_enqueue(h, m, nrays, rmax, span, n_samples, k)) return -1;
        const size_t mk = (size_t)m * k;
        PFB_CK(cudaMemcpyAsync(o1.data(), g->d_out, sizeof(float) * 3 * mk,
                               cudaMemcpyDeviceToHost, h->stream));
        PFB_CK(cudaMemcpyAsync(c1.data(), g->d_outc, sizeof(float) * mk,
                               cudaMemcpyDeviceToHost, h->stream));
        PFB_CK(cudaMemcpyAsync(i1.data(), g->d_outi, sizeof(int) * mk,
                               cudaMemcpyDeviceToHost, h->stream));
        if (check_err(h)) return -1;  // synchronises
        for (int q = 0; q < m; ++q) {
            const size_t o = (size_t)(q0 + q) * k, l = (size_t)q * k;
            const float best = c1[l];
            if (best_out) best_out[q0 + q] = best;
            int which = 0;
            const float* os = o1.data() + 3 * l;
            const float* cs = c1.data() + l;
            const int* is = i1.data() + l;
            std::vector<float> c2, o2;
            std::vector<int> i2;
            if (n_fallback > 0 && !(best <= tau)) {
                const int n_pos = std::max(1, n_fallback / 16);
                const int kk = std::min(k, n_pos * 16);
                c2.assign(k, INFINITY);
                o2.assign(3 * (size_t)k, 0.f);
                i2.assign(k, -1);
                if (gl_upload_scan(g, scans + (size_t)(q0 + q) * nrays, nrays) ||
                    gl_generate(g, n_pos, 16,
                                h->seed + 0x9E3779B97F4A7C15ULL * (qc0 + (uint64_t)q + 1)))
                    return -1;
                if (gl_localize_loaded(g, nrays, rmax, span, kk, o2.data(), c2.data(),
                                       i2.data()) <= 0)
                    return -1;
                which = 1;
                if (c2[0] < best) {
                    which = 2;
                    os = o2.data();
                    cs = c2.data();
                    is = i2.data();
                }
            }
            if (out3k) memcpy(out3k + 3 * o, os, sizeof(float) * 3 * (size_t)k);
            if (caer_k) memcpy(caer_k + o, cs, sizeof(float) * (size_t)k);
            if (idx_k) memcpy(idx_k + o, is, sizeof(int) * (size_t)k);
            if (info) info[q0 + q] = which;
        }
    }
    return k;
}

}  // namespace lp
}  // namespace pfb

using namespace pfb;
using namespace pfb::lp;

extern "C" {

long long pfgl_learned_num_params(void) { return num_params(); }

void* pfgl_learned_create(void* glv, int batch, unsigned long long seed) {
    clear_error();
    GlHandle* g = static_cast<GlHandle*>(glv);
    if (!g || batch < BM || batch % BM) {
        set_error("pf_b200: pfgl_learned_create: batch must be a positive multiple of 128");
        return nullptr;
    }
    LpHandle* h = new (std::nothrow) LpHandle();
    if (!h) return nullptr;
    h->gl = g;
    h->stream = g->stream;
    h->batch = batch;
    h->seed = seed;
    h->cx = g->ox + 0.5f * g->W * g->res;
    h->cy = g->oy + 0.5f * g->H * g->res;
    h->sx = 0.5f * g->W * g->res;
    h->sy = 0.5f * g->H * g->res;
    bool ok = false;
    do {
        bool bad = false;
        for (int l = 0; l < kLayers && !bad; ++l) {
            Layer& L = h->L[l];
            L.in = layer_in(l);
            L.out = layer_out(l);
            const size_t nw = (size_t)L.in * L.out;
            // split-K for the weight gradients, whose output has only
            // (out/128) x (in/128) tiles (24 or 64) while K is the batch:
            // enough splits to fill the SMs once the batch is long enough
            // for the partial products' extra traffic to pay
            const int tiles = (L.out / BM) * (L.in / 128);
            if (tiles < 64)
                L.splits = batch >= 4096 ? 6 : 4;
            else
                L.splits = batch >= 4096 ? 2 : 1;
            L.splits = std::max(1, std::min(batch / BK, L.splits));
            bad = dalloc(&L.w, nw) || dalloc(&L.b, L.out) || dalloc(&L.mw, nw) ||
                  dalloc(&L.vw, nw) || dalloc(&L.mb, L.out) ||
                  dalloc(&L.vb, L.out) || dalloc(&L.gw, nw * L.splits) ||
                  dalloc(&L.gb, L.out) || dalloc(&L.wb, nw) || dalloc(&L.wtb, nw) ||
                  dalloc(&h->dZ[l], (size_t)batch * L.out) ||
                  dalloc(&h->dZT[l], (size_t)batch * L.out);
            if (bad) break;
            bad = make_mat(&L.tm_w, L.wb, L.out, L.in) ||
                  make_mat(&L.tm_wt, L.wtb, L.in, L.out) ||
                  make_mat(&h->tm_dZ[l], h->dZ[l], batch, L.out) ||
                  make_mat(&h->tm_dZT[l], h->dZT[l], L.out, batch);
        }
        if (bad) break;
        for (int l = 0; l < kLayers - 1 && !bad; ++l) {
            bad = dalloc(&h->H[l], (size_t)batch * kHid) ||
                  dalloc(&h->HT[l], (size_t)batch * kHid) ||
                  make_mat(&h->tm_H[l], h->H[l], batch, kHid) ||
                  make_mat(&h->tm_HT[l], h->HT[l], kHid, batch);
        }
        if (bad) break;
        if (dalloc(&h->Z4, (size_t)batch * kOut) ||
            dalloc(&h->Xp, (size_t)batch * kIn) ||
            dalloc(&h->XpT, (size_t)batch * kIn) ||
            dalloc(&h->Xp_f, (size_t)batch * kIn) ||
            dalloc(&h->Yp, (size_t)batch * 4) || dalloc(&h->d_err, 1) ||
            dalloc(&h->d_best, 64) || dalloc(&h->d_query, 1))
            break;
        if (cudaMallocHost((void**)&h->h_res, sizeof(float) * 5 * kSelKMax) !=
            cudaSuccess) {
            h->h_res = nullptr;  // queries then use direct launches
            (void)cudaGetLastError();
        }
        if (make_mat(&h->tm_Xp, h->Xp, batch, kIn) ||
            make_mat(&h->tm_XpT, h->XpT, kIn, batch))
            break;
        if (cudaMemsetAsync(h->Xp, 0, sizeof(bf16) * (size_t)batch * kIn,
                            h->stream) != cudaSuccess ||
            cudaMemsetAsync(h->d_err, 0, sizeof(unsigned), h->stream) != cudaSuccess)
            break;
        // Initialisation: He-uniform hidden layers; small output layer with
        // spread mixture means.
        for (int l = 0; l < kLayers; ++l) {
            Layer& L = h->L[l];
            const long long nw = (long long)L.in * L.out;
            float bound = sqrtf(6.0f / (float)(l == 0 ? 360 : L.in));
            if (l == kLayers - 1) bound *= 0.1f;
            k_init_uniform<<<(unsigned)((nw + 255) / 256), 256, 0, h->stream>>>(
                L.w, nw, -bound, bound, (uint32_t)l, 0u, seed);
            cudaMemsetAsync(L.b, 0, sizeof(float) * L.out, h->stream);
            cudaMemsetAsync(L.mw, 0, sizeof(float) * nw, h->stream);
            cudaMemsetAsync(L.vw, 0, sizeof(float) * nw, h->stream);
            cudaMemsetAsync(L.mb, 0, sizeof(float) * L.out, h->stream);
            cudaMemsetAsync(L.vb, 0, sizeof(float) * L.out, h->stream);
        }
        {
            // Output layer: rows >= 288 (padding) zero; mean biases spread.
            Layer& L = h->L[kLayers - 1];
            cudaMemsetAsync(L.w + (size_t)kUsedOut * L.in, 0,
                            sizeof(float) * (size_t)(kOut - kUsedOut) * L.in,
                            h->stream);
            k_init_uniform<<<1, 128, 0, h->stream>>>(L.b + kMeanOff, 4 * kComp,
                                                     -0.8f, 0.8f,
                                                     (uint32_t)kLayers, 1u, seed);
        }
        if (cudaGetLastError() != cudaSuccess) break;
        if (round_weights(h)) break;
        if (cudaStreamSynchronize(h->stream) != cudaSuccess) break;
        ok = true;
    } while (0);
    if (!ok) {
        set_error("pf_b200: pfgl_learned_create failed: %s",
                  cudaGetErrorString(cudaGetLastError()));
        free_lp(h);
        return nullptr;
    }
    return h;
}

int pfgl_learned_destroy(void* p) {
    free_lp(as_lp(p));
    return 0;
}

int pfgl_learned_norm(void* p, float* c4) {
    LpHandle* h = as_lp(p);
    if (!h || !c4) return -1;
    c4[0] = h->cx;
    c4[1] = h->cy;
    c4[2] = h->sx;
    c4[3] = h->sy;
    return 0;
}

int pfgl_learned_get_params(void* p, float* out) {
    LpHandle* h = as_lp(p);
    if (!h || !out) return -1;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        const size_t nw = (size_t)L.in * L.out;
        PFB_CK(cudaMemcpyAsync(out + off, L.w, sizeof(float) * nw,
                               cudaMemcpyDeviceToHost, h->stream));
        off += nw;
        PFB_CK(cudaMemcpyAsync(out + off, L.b, sizeof(float) * L.out,
                               cudaMemcpyDeviceToHost, h->stream));
        off += L.out;
    }
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfgl_learned_set_params(void* p, const float* in) {
    LpHandle* h = as_lp(p);
    if (!h || !in) return -1;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        const size_t nw = (size_t)L.in * L.out;
        PFB_CK(cudaMemcpyAsync(L.w, in + off, sizeof(float) * nw,
                               cudaMemcpyHostToDevice, h->stream));
        off += nw;
        PFB_CK(cudaMemcpyAsync(L.b, in + off, sizeof(float) * L.out,
                               cudaMemcpyHostToDevice, h->stream));
        off += L.out;
    }
    if (round_weights(h)) return -1;
    PFB_CK(cudaStreamSynchronize(h->stream));
    return 0;
}

int pfgl_render_scans(void* glv, const float* pose3n, int n, int nrays,
                      float rmax, float ang_span, float noise_std,
                      unsigned long long seed, float* out) {
    GlHandle* g = static_cast<GlHandle*>(glv);
    if (!g || !pose3n || !out || n <= 0 || nrays <= 0) return -1;
    const RenderArgs a = render_args_gl(g, nrays, rmax, ang_span, noise_std, seed);
    float* d_pose = nullptr;
    float* d_out = nullptr;
    int rc = -1;
    do {
        if (cudaMalloc((void**)&d_pose, sizeof(float) * 3 * (size_t)n) != cudaSuccess ||
            cudaMalloc((void**)&d_out, sizeof(float) * (size_t)n * nrays) != cudaSuccess)
            break;
        if (cudaMemcpyAsync(d_pose, pose3n, sizeof(float) * 3 * (size_t)n,
                            cudaMemcpyHostToDevice, g->stream) != cudaSuccess)
            break;
        const size_t smem = (size_t)a.grid_bytes;
        if (smem > 200 * 1024) {
            set_error("pf_b200: pfgl_render_scans: map too large for shared memory");
            break;
        }
        if (cudaFuncSetAttribute(k_render, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)smem) != cudaSuccess)
            break;
        k_render<<<std::min(ceil_div(n, 8), 1184), 256, smem, g->stream>>>(a, d_pose, n,
                                                                         d_out);
        if (cudaGetLastError() != cudaSuccess) break;
        if (cudaMemcpyAsync(out, d_out, sizeof(float) * (size_t)n * nrays,
                            cudaMemcpyDeviceToHost, g->stream) != cudaSuccess)
            break;
        if (cudaStreamSynchronize(g->stream) != cudaSuccess) break;
        rc = 0;
    } while (0);
    if (rc) set_error("pf_b200: pfgl_render_scans failed: %s",
                      cudaGetErrorString(cudaGetLastError()));
    cudaFree(d_pose);
    cudaFree(d_out);
    return rc;
}

int pfgl_learned_make_data(void* p, long long n_pairs, int nrays, float rmax,
                           float ang_span, float noise_std,
                           unsigned long long seed) {
    LpHandle* h = as_lp(p);
    if (!h || n_pairs < h->batch || nrays <= 0 || nrays > kIn) {
        set_error("pf_b200: pfgl_learned_make_data: bad arguments");
        return -1;
    }
    if (h->gl->nfree <= 0) return -1;
    // Round to whole batches.
    n_pairs = n_pairs / h->batch * h->batch;
    if (n_pairs > (1ll << 31) - h->batch) return -1;
    cudaFree(h->X);
    cudaFree(h->XT);
    cudaFree(h->Y);
    h->X = h->XT = nullptr;
    h->Y = nullptr;
    h->n_pairs = 0;
    if (dalloc(&h->X, (size_t)n_pairs * kIn) || dalloc(&h->XT, (size_t)n_pairs * kIn) ||
        dalloc(&h->Y, (size_t)n_pairs * 4))
        return -1;
    const RenderArgs a = render_args(h, nrays, rmax, ang_span, noise_std, seed);
    const size_t smem = (size_t)a.grid_bytes;
    if (smem > 200 * 1024) {
        set_error("pf_b200: pfgl_learned_make_data: map too large for shared memory");
        return -1;
    }
    PFB_CK(cudaFuncSetAttribute(k_make_pairs,
                                cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    k_make_pairs<<<sms * 4, 256, smem, h->stream>>>(a, h->gl->nfree, h->gl->d_free, 0,
                                                    n_pairs, h->X, h->Y);
    PFB_KL();
    // XT[c][r] = X[r][c], in column chunks of at most 65535 * 32 rows.
    const long long chunk = 65535ll * 32;
    for (long long r0 = 0; r0 < n_pairs; r0 += chunk) {
        const long long rows = std::min(chunk, n_pairs - r0);
        k_transpose_bf16<<<dim3(ceil_div(kIn, 64), (unsigned)((rows + 63) / 64)), dim3(32, 8), 0,
                           h->stream>>>(h->X + (size_t)r0 * kIn, kIn, h->XT + r0,
                                        n_pairs, rows, kIn);
    }
    PFB_KL();
    if (make_mat(&h->tm_X, h->X, n_pairs, kIn) ||
        make_mat(&h->tm_XT, h->XT, kIn, n_pairs))
        return -1;
    PFB_CK(cudaStreamSynchronize(h->stream));
    h->n_pairs = n_pairs;
    h->data_nrays = nrays;
    h->data_rmax = rmax;
    return 0;
}

int pfgl_learned_train(void* p, int steps, int total_steps, float lr,
                       float* loss_out) {
    LpHandle* h = as_lp(p);
    if (!h || steps <= 0 || h->n_pairs < h->batch) {
        set_error("pf_b200: pfgl_learned_train: no training pairs");
        return -1;
    }
    if (total_steps < steps) total_steps = steps;
    if (steps > h->loss_cap) {
        cudaFree(h->d_loss);
        h->d_loss = nullptr;
        if (dalloc(&h->d_loss, (size_t)steps)) return -1;
        h->loss_cap = steps;
    }
    PFB_CK(cudaMemsetAsync(h->d_loss, 0, sizeof(float) * steps, h->stream));
    const long long nb = h->n_pairs / h->batch;
    const int warm = std::max(1, total_steps / 20);
    for (int i = 0; i < steps; ++i) {
        const long long t = h->train_step++;
        float lr_t;
        if (t < warm)
            lr_t = lr * (float)(t + 1) / (float)warm;
        else {
            const double f = std::min(1.0, (double)(t - warm) / std::max(1, total_steps - warm));
            lr_t = (float)(lr * (0.02 + 0.98 * 0.5 * (1.0 + std::cos(M_PI * f))));
        }
        const long long row0 = (t % nb) * h->batch;
        if (train_one(h, row0, lr_t, h->d_loss + i)) return -1;
    }
    if (loss_out)
        PFB_CK(cudaMemcpyAsync(loss_out, h->d_loss, sizeof(float) * steps,
                               cudaMemcpyDeviceToHost, h->stream));
    return check_err(h);
}

int pfgl_learned_grad(void* p, const float* x, const float* y, float* loss,
                      float* grad) {
    LpHandle* h = as_lp(p);
    if (!h || !x || !y || !grad) return -1;
    const int B = h->batch;
    const size_t nx = (size_t)B * kIn;
    PFB_CK(cudaMemcpyAsync(h->Xp_f, x, sizeof(float) * nx, cudaMemcpyHostToDevice,
                           h->stream));
    PFB_CK(cudaMemcpyAsync(h->Yp, y, sizeof(float) * 4 * B, cudaMemcpyHostToDevice,
                           h->stream));
    k_f32_to_bf16<<<(unsigned)((nx + 255) / 256), 256, 0, h->stream>>>(h->Xp_f, h->Xp,
                                                                      (long long)nx);
    k_transpose_bf16<<<dim3(ceil_div(kIn, 64), ceil_div(B, 64)), dim3(32, 8), 0, h->stream>>>(
        h->Xp, kIn, h->XpT, B, B, kIn);
    PFB_KL();
    if (h->loss_cap < 1) {
        if (dalloc(&h->d_loss, 1)) return -1;
        h->loss_cap = 1;
    }
    PFB_CK(cudaMemsetAsync(h->d_loss, 0, sizeof(float), h->stream));
    if (forward(h, MapRef{&h->tm_Xp, 0, 0}, B, true)) return -1;
    if (backward(h, MapRef{&h->tm_XpT, 0, 0}, h->Yp, h->d_loss))
        return -1;
    size_t off = 0;
    for (int l = 0; l < kLayers; ++l) {
        Layer& L = h->L[l];
        const size_t nw = (size_t)L.in * L.out;
        if (L.splits > 1) {
            k_sum_splits<<<(unsigned)((nw + 255) / 256), 256, 0, h->stream>>>(
                L.gw, L.splits, (long long)nw);
            PFB_KL();
        }
        PFB_CK(cudaMemcpyAsync(grad + off, L.gw, sizeof(float) * nw,
                               cudaMemcpyDeviceToHost, h->stream));
        off += nw;
        PFB_CK(cudaMemcpyAsync(grad + off, L.gb, sizeof(float) * L.out,
                               cudaMemcpyDeviceToHost, h->stream));
        off += L.out;
    }
    if (loss)
        PFB_CK(cudaMemcpyAsync(loss, h->d_loss, sizeof(float), cudaMemcpyDeviceToHost,
                               h->stream));
    return check_err(h);
}

int pfgl_learned_forward(void* p, const float* x, int rows, float* out) {
    LpHandle* h = as_lp(p);
    if (!h || !x || !out || rows <= 0 || rows > BM) return -1;
    const size_t nx = (size_t)BM * kIn;
    PFB_CK(cudaMemsetAsync(h->Xp_f, 0, sizeof(float) * nx, h->stream));
    PFB_CK(cudaMemcpyAsync(h->Xp_f, x, sizeof(float) * (size_t)rows * kIn,
                           cudaMemcpyHostToDevice, h->stream));
    k_f32_to_bf16<<<(unsigned)((nx + 255) / 256), 256, 0, h->stream>>>(h->Xp_f, h->Xp,
                                                                      (long long)nx);
    PFB_KL();
    if (forward(h, MapRef{&h->tm_Xp, 0, 0}, BM, false)) return -1;
    PFB_CK(cudaMemcpy2DAsync(out, sizeof(float) * kUsedOut, h->Z4,
                             sizeof(float) * kOut, sizeof(float) * kUsedOut, rows,
                             cudaMemcpyDeviceToHost, h->stream));
    return check_err(h);
}

int pfgl_learned_set_graph(void* p, int on) {
    LpHandle* h = as_lp(p);
    if (!h) return -1;
    h->q_off = on == 0;
    if (h->q_off) drop_query_graph(h);
    return 0;
}

int pfgl_learned_set_threshold(void* p, float tau) {
    LpHandle* h = as_lp(p);
    if (!h) return -1;
    h->tau = tau;
    return 0;
}

int pfgl_learned_localize(void* p, const float* scan, int nrays, float rmax,
                          float ang_span, int n_samples, int n_fallback, int k,
                          float* out3k, float* caer_k, int* idx_k, int* info) {
    LpHandle* h = as_lp(p);
    if (!h || !scan || nrays <= 0 || nrays > kIn || n_samples <= 0 || k <= 0 ||
        n_samples > h->gl->cap_hyp || n_fallback > h->gl->cap_hyp)
        return -1;
    GlHandle* g = h->gl;
    if (k > n_samples) k = n_samples;
    std::vector<float> c1((size_t)k), o1(3 * (size_t)k);
    std::vector<int> i1((size_t)k);
    if (gl_upload_scan(g, scan, nrays)) return -1;
    const int r1 = learned_pass(h, nrays, rmax, ang_span, n_samples, k, o1.data(),
                                c1.data(), i1.data());
    if (r1 <= 0) return -1;
    if (check_err(h)) return -1;
    int which = 0;
    int rk = r1;
    std::vector<float> c2, o2;
    std::vector<int> i2;
    if (n_fallback > 0 && !(c1[0] <= h->tau)) {
        const int n_pos = std::max(1, n_fallback / 16);
        if (gl_generate(g, n_pos, 16, h->seed + 0x9E3779B97F4A7C15ULL * (h->query_count + 1)))
            return -1;
        const int kk = std::min(k, n_pos * 16);
        c2.resize(kk);
        o2.resize(3 * (size_t)kk);
        i2.resize(kk);
        const int r2 = gl_localize_loaded(g, nrays, rmax, ang_span, kk, o2.data(),
                                          c2.data(), i2.data());
        if (r2 <= 0) return -1;
        which = 1;
        if (c2[0] < c1[0]) {
            which = 2;
            rk = r2;
        }
    }
    const std::vector<float>& cs = which == 2 ? c2 : c1;
    const std::vector<float>& os = which == 2 ? o2 : o1;
    const std::vector<int>& is = which == 2 ? i2 : i1;
    if (out3k) memcpy(out3k, os.data(), sizeof(float) * 3 * (size_t)rk);
    if (caer_k) memcpy(caer_k, cs.data(), sizeof(float) * (size_t)rk);
    if (idx_k) memcpy(idx_k, is.data(), sizeof(int) * (size_t)rk);
    if (info) *info = which;
    return rk;
}

int pfgl_learned_localize_batch(void* p, const float* scans, int nq, int nrays,
                                float rmax, float ang_span, int n_samples, int n_fallback,
                                int k, float* out3k, float* caer_k, int* idx_k, int* info) {
    LpHandle* h = as_lp(p);
    clear_error();
    if (!h || !scans || nq <= 0 || nrays <= 0 || nrays > kIn || n_samples <= 0 || k <= 0 ||
        n_fallback < 0 || n_fallback > h->gl->cap_hyp)
        return -1;
    return learned_localize_batch(h, scans, nq, nrays, rmax, ang_span, n_samples,
                                  n_fallback, k, h->tau, out3k, caer_k, idx_k, info,
                                  nullptr);
}

int pfgl_learned_calibrate(void* p, int n_queries, int nrays, float rmax,
                           float ang_span, float noise_std, int n_samples,
                           float quantile, unsigned long long seed,
                           float* tau_out, float* success_out) {
    LpHandle* h = as_lp(p);
    if (!h || n_queries <= 0 || nrays <= 0 || nrays > kIn || n_samples <= 0 ||
        n_samples > h->gl->cap_hyp)
        return -1;
    GlHandle* g = h->gl;
    const RenderArgs a = render_args(h, nrays, rmax, ang_span, noise_std, seed);
    std::vector<float> poses(3 * (size_t)n_queries), scans((size_t)n_queries * nrays);
    float* d_pose = nullptr;
    if (dalloc(&d_pose, 3 * (size_t)n_queries)) return -1;
    k_random_poses<<<ceil_div(n_queries, 128), 128, 0, h->stream>>>(
        a, g->nfree, g->d_free, n_queries, d_pose);
    const bool ok_launch = cudaGetLastError() == cudaSuccess &&
                           cudaMemcpyAsync(poses.data(), d_pose,
                                           sizeof(float) * poses.size(),
                                           cudaMemcpyDeviceToHost,
                                           h->stream) == cudaSuccess &&
                           cudaStreamSynchronize(h->stream) == cudaSuccess;
    cudaFree(d_pose);
    if (!ok_launch) return -1;
    if (pfgl_render_scans(g, poses.data(), n_queries, nrays, rmax, ang_span,
                          noise_std, seed ^ 0xA5A5A5A5ULL, scans.data()))
        return -1;
    // the held-out queries' best samples: through the batched path, or one
    // query at a time beyond its sample limit
    std::vector<float> best3(3 * (size_t)n_queries), bestc((size_t)n_queries);
    if (gl_batch_ok(g, 1, n_samples, 1)) {
        if (learned_localize_batch(h, scans.data(), n_queries, nrays, rmax, ang_span,
                                   n_samples, 0, 1, INFINITY, best3.data(), bestc.data(),
                                   nullptr, nullptr, nullptr) < 0)
            return -1;
    } else {
        for (int q = 0; q < n_queries; ++q) {
            int i0;
            if (gl_upload_scan(g, scans.data() + (size_t)q * nrays, nrays)) return -1;
            if (learned_pass(h, nrays, rmax, ang_span, n_samples, 1,
                             best3.data() + 3 * (size_t)q, bestc.data() + q, &i0) <= 0)
                return -1;
        }
        if (check_err(h)) return -1;
    }
    std::vector<float> good;
    int n_ok = 0;
    for (int q = 0; q < n_queries; ++q) {
        const float* t = poses.data() + 3 * (size_t)q;
        const float* out3 = best3.data() + 3 * (size_t)q;
        const double dp = std::hypot((double)out3[0] - t[0], (double)out3[1] - t[1]);
        double dth = std::fmod((double)out3[2] - t[2] + M_PI, 2 * M_PI);
        if (dth < 0) dth += 2 * M_PI;
        dth = std::fabs(dth - M_PI);
        if (dp <= 0.5 && dth <= 0.1) {
            ++n_ok;
            good.push_back(bestc[(size_t)q]);
        }
    }
    float tau = INFINITY;
    if (!good.empty()) {
        std::sort(good.begin(), good.end());
        // Nearest-rank quantile.
        const double qq = std::min(1.0, std::max(0.0, (double)quantile));
        long long idx = (long long)std::ceil(qq * (double)good.size()) - 1;
        idx = std::max(0ll, std::min((long long)good.size() - 1, idx));
        tau = good[(size_t)idx];
    }
    h->tau = tau;
    if (tau_out) *tau_out = tau;
    if (success_out) *success_out = (float)n_ok / (float)n_queries;
    return 0;
}

int pfgl_learned_gemm(int M, int N, int K, const unsigned short* A,
                      const unsigned short* B, float* D) {
    clear_error();
    if (!A || !B || !D || M <= 0 || N <= 0 || K <= 0 || M % BM || N % 128 || K % BK)
        return -1;
    bf16* dA = nullptr;
    bf16* dB = nullptr;
    float* dD = nullptr;
    unsigned* dErr = nullptr;
    int rc = -1;
    cudaStream_t s = nullptr;
    do {
        if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) break;
        if (cudaMalloc((void**)&dA, sizeof(bf16) * (size_t)M * K) != cudaSuccess ||
            cudaMalloc((void**)&dB, sizeof(bf16) * (size_t)N * K) != cudaSuccess ||
            cudaMalloc((void**)&dD, sizeof(float) * (size_t)M * N) != cudaSuccess ||
            cudaMalloc((void**)&dErr, sizeof(unsigned)) != cudaSuccess)
            break;
        if (cudaMemcpyAsync(dA, A, sizeof(bf16) * (size_t)M * K, cudaMemcpyHostToDevice,
                            s) != cudaSuccess ||
            cudaMemcpyAsync(dB, B, sizeof(bf16) * (size_t)N * K, cudaMemcpyHostToDevice,
                            s) != cudaSuccess ||
            cudaMemsetAsync(dErr, 0, sizeof(unsigned), s) != cudaSuccess)
            break;
        Mat ta, tb;
        if (make_mat(&ta, dA, M, K) || make_mat(&tb, dB, N, K)) break;
        EpiArgs ep{};
        ep.out = dD;
        ep.ldo = N;
        ep.scale = 1.0f;
        if (gemm<EPI_F32>(s, MapRef{&ta, 0, 0}, MapRef{&tb, 0, 0}, M, N, K, ep, dErr))
            break;
        unsigned e = 0;
        if (cudaMemcpyAsync(D, dD, sizeof(float) * (size_t)M * N, cudaMemcpyDeviceToHost,
                            s) != cudaSuccess ||
            cudaMemcpyAsync(&e, dErr, sizeof(unsigned), cudaMemcpyDeviceToHost, s) !=
                cudaSuccess ||
            cudaStreamSynchronize(s) != cudaSuccess)
            break;
        if (e) {
            set_error("pf_b200: pfgl_learned_gemm: pipeline wait timed out");
            break;
        }
        rc = 0;
    } while (0);
    if (rc && cudaGetLastError() != cudaSuccess)
        set_error("pf_b200: pfgl_learned_gemm failed");
    cudaFree(dA);
    cudaFree(dB);
    cudaFree(dD);
    cudaFree(dErr);
    if (s) cudaStreamDestroy(s);
    return rc;
}

}  // extern "C"
