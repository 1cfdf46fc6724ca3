// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Convolution layers of the learned super-stepper on tcgen05 tensor cores.
//
// One kernel template covers the forward layers and the input-gradient
// (transposed) layers: a CTA computes 128 consecutive pixels of one image row
// for all N output channels as an implicit GEMM (see lpbf_surrogate.cuh):
//   CIN = 32: K = 9 taps x 32 channels, one SW64 atom column per tap;
//   CIN = 4 or 1: K = 9 x CIN real entries padded to 64 (one SW128 atom).
// Zero padding at the image border.  Activations are NHWC bf16; weights are
// packed [N][K] bf16 (tap-major, then input channel).  Epilogues:
//   GELU   : out = gelu(acc + bias) (bf16), pre = acc + bias (bf16, optional)
//   LINEAR : y = acc[0] + bias[0] (fp32, one channel)
//   DGELU  : out = acc * gelu'(pre_in) (bf16): the gradient of the previous
//            layer's pre-activation when x is this layer's gradient and the
//            weights are packed flipped and transposed.
// ---------------------------------------------------------------------------
#include <cstring>

#include <algorithm>

#include "lpbf_host.hpp"
#include "lpbf_surrogate.cuh"
#include "lpbf_b200.h"

namespace lpbf_b200 {
namespace sg {

enum { EPI_GELU = 0, EPI_LINEAR = 1, EPI_DGELU = 2 };

struct ConvArgs {
    const void* x;          // input, NHWC bf16 with CIN channels
    const bf16* w;          // [N][K] packed weights
    const float* bias;      // [N] (GELU, LINEAR), or null
    const bf16* pre_in;     // DGELU: pre-activation of the target layer, [P][32]
    bf16* pre_out;          // GELU: pre-activation out, [P][N], or null
    void* out;              // GELU/DGELU: bf16 [P][N]; LINEAR: fp32 [P]
    int B, H, W;
    unsigned int* err;
};

template <int CIN> struct KOf { static constexpr int K = CIN == 32 ? 288 : 64;
                                static constexpr int KATOM = CIN == 32 ? 32 : 64; };

template <int CIN, int N>
constexpr size_t conv_smem_bytes() {
    return 1024 + size_t(128 + N) * KOf<CIN>::K * sizeof(bf16);
}

__device__ __forceinline__ uint8_t* align1024(uint8_t* p) {
    return reinterpret_cast<uint8_t*>((reinterpret_cast<uintptr_t>(p) + 1023) & ~uintptr_t(1023));
}

// Fill the im2col tile of pixels (b, y, x0 .. x0+127).
template <int CIN, class T>
__device__ __forceinline__ void fill_a(bf16* sA, const ConvArgs& a, int b, int y, int x0) {
    const int tid = threadIdx.x;
    if constexpr (CIN == 32) {
        const bf16* X = static_cast<const bf16*>(a.x);
        // unit u = ((tap * 128) + m) * 4 + c: 16 bytes = 8 channels
        for (int u = tid; u < 9 * 128 * 4; u += blockDim.x) {
            const int c = u & 3, m = (u >> 2) & 127, tap = u >> 9;
            const int yy = y + tap / 3 - 1, xx = x0 + m + tap % 3 - 1;
            uint4 v = make_uint4(0u, 0u, 0u, 0u);
            if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
                v = __ldg(reinterpret_cast<const uint4*>(
                    X + ((size_t(b) * a.H + yy) * a.W + xx) * 32 + c * 8));
            *reinterpret_cast<uint4*>(T::a_at(sA, m, tap * 32 + c * 8)) = v;
        }
    } else if constexpr (CIN == 4) {
        // K = 64: k = tap * 4 + ci; a 16-byte unit j holds taps 2j and 2j + 1
        // (one 8-byte pixel load each); units past tap 8 are zero
        const uint2* X = static_cast<const uint2*>(a.x);
        for (int u = tid; u < 128 * 8; u += blockDim.x) {
            const int m = u >> 3, j = u & 7;
            uint2 h[2] = {make_uint2(0u, 0u), make_uint2(0u, 0u)};
#pragma unroll
            for (int q = 0; q < 2; ++q) {
                const int tap = 2 * j + q;
                if (tap < 9) {
                    const int yy = y + tap / 3 - 1, xx = x0 + m + tap % 3 - 1;
                    if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
                        h[q] = __ldg(X + (size_t(b) * a.H + yy) * a.W + xx);
                }
            }
            *reinterpret_cast<uint4*>(T::a_at(sA, m, j * 8)) =
                make_uint4(h[0].x, h[0].y, h[1].x, h[1].y);
        }
    } else {
        // K = 64: k = tap * CIN + ci for k < 9 * CIN, zero beyond; unit = 8 k
        const uint16_t* X = static_cast<const uint16_t*>(a.x);
        for (int u = tid; u < 128 * 8; u += blockDim.x) {
            const int m = u >> 3, j = u & 7;
            uint16_t e[8];
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                const int k = j * 8 + q;
                uint16_t val = 0;
                if (k < 9 * CIN) {
                    const int tap = k / CIN, ci = k % CIN;
                    const int yy = y + tap / 3 - 1, xx = x0 + m + tap % 3 - 1;
                    if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W)
                        val = X[((size_t(b) * a.H + yy) * a.W + xx) * CIN + ci];
                }
                e[q] = val;
            }
            uint4 v;
            v.x = e[0] | (uint32_t(e[1]) << 16);
            v.y = e[2] | (uint32_t(e[3]) << 16);
            v.z = e[4] | (uint32_t(e[5]) << 16);
            v.w = e[6] | (uint32_t(e[7]) << 16);
            *reinterpret_cast<uint4*>(T::a_at(sA, m, j * 8)) = v;
        }
    }
}

template <int N, int K, class T>
__device__ __forceinline__ void fill_b(bf16* sB, const bf16* w) {
    for (int u = threadIdx.x; u < N * K / 8; u += blockDim.x) {
        const int n = u / (K / 8), k = (u % (K / 8)) * 8;
        *reinterpret_cast<uint4*>(T::b_at(sB, n, k)) =
            __ldg(reinterpret_cast<const uint4*>(w + size_t(n) * K + k));
    }
}

// Two floats as a bf16 pair (round to nearest even), one conversion
// instruction: lo in the low half.
__device__ __forceinline__ uint32_t pack_bf16(float lo, float hi) {
    uint32_t r;
    asm("cvt.rn.bf16x2.f32 %0, %1, %2;" : "=r"(r) : "f"(hi), "f"(lo));
    return r;
}
__device__ __forceinline__ float bf16_at(const bf16* p, size_t i) {
    return float(p[i]);
}

// One CTA of 128 threads per tile of 128 pixels of one image row: all
// threads fill the tile's im2col operand, one thread issues its MMAs, and
// thread m runs the epilogue of pixel m from accumulator lane m.  (A
// persistent form that walks tiles with the weights staged once measured
// slower: 112 against 70 us per 1024^2 input layer, its fill, MMA and
// epilogue phases no longer overlapping those of other CTAs.)
template <int CIN, int N, int EPI>
__global__ void __launch_bounds__(128) conv_kernel(const ConvArgs a) {
    using T = TileMma<N, KOf<CIN>::K, KOf<CIN>::KATOM>;
    constexpr int K = KOf<CIN>::K;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    bf16* sA = reinterpret_cast<bf16*>(align1024(smem_raw));
    bf16* sB = sA + T::A_ELEMS;
    static_assert((T::A_ELEMS * sizeof(bf16)) % 1024 == 0, "B tile 1024-byte aligned");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int x0 = blockIdx.x * 128, y = blockIdx.y, b = blockIdx.z;
    if (warp == 0) tmem_alloc(&tslot, T::TMEM_COLS);
    if (threadIdx.x == 32) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    fill_b<N, K, T>(sB, a.w);
    fill_a<CIN, T>(sA, a, b, y, x0);
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    if (warp == 0) T::issue(sA, sB, tmem, &bar);
    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bar, 0));
    tc_fence_after();
    if (ok) {
        const int m = warp * 32 + lane;
        const int x = x0 + m;
        float v[32];
        if constexpr (N == 32) tmem_ld32(tmem + (uint32_t(warp * 32) << 16), v);
        else tmem_ld16(tmem + (uint32_t(warp * 32) << 16), v);
        if (x < a.W) {
            const size_t p = (size_t(b) * a.H + y) * a.W + x;
            if constexpr (EPI == EPI_LINEAR) {
                static_cast<float*>(a.out)[p] = v[0] + (a.bias ? a.bias[0] : 0.0f);
            } else {
                uint32_t o[N / 2], pr[N / 2];
#pragma unroll
                for (int c = 0; c < N; c += 2) {
                    float v0 = v[c], v1 = v[c + 1];
                    if constexpr (EPI == EPI_GELU) {
                        v0 += __ldg(a.bias + c);
                        v1 += __ldg(a.bias + c + 1);
                        pr[c / 2] = pack_bf16(v0, v1);
                        o[c / 2] = pack_bf16(gelu(v0), gelu(v1));
                    } else {
                        const float g0 = gelu_grad(bf16_at(a.pre_in, p * N + c));
                        const float g1 = gelu_grad(bf16_at(a.pre_in, p * N + c + 1));
                        o[c / 2] = pack_bf16(v0 * g0, v1 * g1);
                    }
                }
                uint4* dst = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + p * N);
#pragma unroll
                for (int q = 0; q < N / 8; ++q)
                    dst[q] = make_uint4(o[4 * q], o[4 * q + 1], o[4 * q + 2], o[4 * q + 3]);
                if constexpr (EPI == EPI_GELU) {
                    if (a.pre_out) {
                        uint4* dp = reinterpret_cast<uint4*>(a.pre_out + p * N);
#pragma unroll
                        for (int q = 0; q < N / 8; ++q)
                            dp[q] = make_uint4(pr[4 * q], pr[4 * q + 1], pr[4 * q + 2], pr[4 * q + 3]);
                    }
                }
            }
        }
    } else if (threadIdx.x == 0 && a.err) {
        atomicOr(a.err, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, T::TMEM_COLS);
}

// Plain tile product C[128 x N] = A[128 x K] . B[N x K]^T (row-major, K
// contiguous): the tensor-core path on its own, for tests.
template <int N, int K>
__global__ void __launch_bounds__(128) gemm_bt_kernel(const bf16* A, const bf16* Bm, float* C,
                                                      unsigned int* err) {
    using T = TileMma<N, K, 32>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bar;
    __shared__ uint32_t tslot;
    bf16* sA = reinterpret_cast<bf16*>(align1024(smem_raw));
    bf16* sB = sA + T::A_ELEMS;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (warp == 0) tmem_alloc(&tslot, T::TMEM_COLS);
    if (threadIdx.x == 32) {
        mbar_init(&bar, 1);
        fence_mbar_init();
    }
    for (int u = threadIdx.x; u < 128 * K / 8; u += blockDim.x) {
        const int r = u / (K / 8), k = (u % (K / 8)) * 8;
        *reinterpret_cast<uint4*>(T::a_at(sA, r, k)) =
            *reinterpret_cast<const uint4*>(A + size_t(r) * K + k);
    }
    fill_b<N, K, T>(sB, Bm);
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    if (warp == 0) T::issue(sA, sB, tmem, &bar);
    const bool ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bar, 0));
    tc_fence_after();
    if (ok) {
        float v[32];
        if constexpr (N == 32) tmem_ld32(tmem + (uint32_t(warp * 32) << 16), v);
        else tmem_ld16(tmem + (uint32_t(warp * 32) << 16), v);
        const int m = warp * 32 + lane;
#pragma unroll
        for (int c = 0; c < N; ++c) C[size_t(m) * N + c] = v[c];
    } else if (threadIdx.x == 0 && err) {
        atomicOr(err, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, T::TMEM_COLS);
}

// ---- 32-channel layers: TMA-fed, warp-specialized, persistent --------------
//
// One CTA per SM walks the tiles (128 pixels of one row) of the layer.  Warp 0
// (one thread) loads each tile's nine tap tiles with TMA from a 4D tensor map
// over the NHWC activations: box {32 channels, 128 pixels}, 64-byte swizzle,
// i.e. exactly the tensor core's K-major SW64 operand layout; pixels off the
// image read as zero (the padding).  Warp 1 issues the 18 MMAs of a tile
// into one of two TMEM accumulators and commits to the stage's "empty" and
// the accumulator's "full" barriers.  Warps 2-9 (two per TMEM lane quarter,
// 16 accumulator columns each) read their accumulator lanes and run the
// epilogue, then release the accumulator.  Two shared
// memory stages and two accumulators overlap loads, MMAs and epilogues.
// Every wait is bounded; a timeout sets the error word and ends the CTA.
constexpr int CT_STAGES = 2;
constexpr int CT_TAP_ELEMS = 128 * 32;
constexpr int CT_STAGE_BYTES = 9 * CT_TAP_ELEMS * 2;
constexpr int CT_EPI_WARPS = 8;                        // two per TMEM lane quarter
constexpr int CT_THREADS = 32 * (2 + CT_EPI_WARPS);      // TMA warp, MMA warp, epilogue

__device__ __forceinline__ void tma_load_4d(void* dst, const CUtensorMap* map, int c0, int c1,
                                            int c2, int c3, uint64_t* bar) {
    asm volatile(
        "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
        " [%0], [%1, {%2, %3, %4, %5}], [%6];"
        :: "r"(smem_u32(dst)), "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2),
           "r"(c3), "r"(smem_u32(bar))
        : "memory");
}
__device__ __forceinline__ void mbar_arrive(uint64_t* bar) {
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" :: "r"(smem_u32(bar)) : "memory");
}

template <int N>
constexpr size_t ct_smem_bytes() {
    return 1024 + size_t(CT_STAGES) * CT_STAGE_BYTES + size_t(N) * 288 * 2;
}

template <int N, int EPI>
__global__ void __launch_bounds__(CT_THREADS, 1)
conv_tma_kernel(const __grid_constant__ CUtensorMap xmap, const ConvArgs a, int ntiles,
                int xtiles) {
    using T = TileMma<N, 288, 32>;
    constexpr int ACC_COLS = T::TMEM_COLS;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[CT_STAGES], empty[CT_STAGES], tfull[2], tempty[2];
    __shared__ uint32_t tslot;
    uint8_t* base = align1024(smem_raw);
    bf16* sA = reinterpret_cast<bf16*>(base);
    bf16* sB = reinterpret_cast<bf16*>(base + size_t(CT_STAGES) * CT_STAGE_BYTES);
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) tmem_alloc(&tslot, 2 * ACC_COLS);
    if (threadIdx.x == 0) {
        for (int i = 0; i < CT_STAGES; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
        for (int i = 0; i < 2; ++i) { mbar_init(&tfull[i], 1); mbar_init(&tempty[i], CT_EPI_WARPS); }
        fence_mbar_init();
    }
    fill_b<N, 288, T>(sB, a.w);
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
                const int s = i % CT_STAGES;
                const uint32_t ph = (i / CT_STAGES) & 1;
                if (!mbar_wait_bounded(&empty[s], ph ^ 1)) { ok = false; break; }
                const int xt = t % xtiles, row = t / xtiles;
                const int y = row % a.H, b = row / a.H, x0 = xt * 128;
                mbar_expect_tx(&full[s], CT_STAGE_BYTES);
                bf16* st = sA + size_t(s) * 9 * CT_TAP_ELEMS;
#pragma unroll 1
                for (int tap = 0; tap < 9; ++tap)
                    tma_load_4d(st + tap * CT_TAP_ELEMS, &xmap, 0, x0 + tap % 3 - 1,
                                y + tap / 3 - 1, b, &full[s]);
            }
        }
    } else if (warp == 1) {
        for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
            const int s = i % CT_STAGES;
            const uint32_t ph = (i / CT_STAGES) & 1;
            const int acc = i & 1;
            const uint32_t aph = (i >> 1) & 1;
            bool w = mbar_wait_bounded(&tempty[acc], aph ^ 1);
            w = w && mbar_wait_bounded(&full[s], ph);
            if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
            tc_fence_after();
            T::issue(sA + size_t(s) * 9 * CT_TAP_ELEMS, sB, tmem + acc * ACC_COLS, &empty[s]);
            cutlass::arch::umma_arrive(&tfull[acc]);
        }
    } else {
        // two warps per TMEM lane quarter, each with 16 of the accumulator's
        // columns (the LINEAR layer's one output channel sits in the first)
        const int q = warp & 3;                      // TMEM lane quarter of this warp
        const int h = (warp - 2) >> 2;               // column half: 0 or 1
        const bool active = N == 32 || h == 0;
        float bias[16];                              // this warp's 16 channels' biases
#pragma unroll
        for (int c = 0; c < 16; ++c)
            bias[c] = (EPI == EPI_GELU && active) ? __ldg(a.bias + 16 * h + c) : 0.0f;
        for (int i = 0, t = blockIdx.x; t < ntiles; ++i, t += gridDim.x) {
            const int acc = i & 1;
            const uint32_t aph = (i >> 1) & 1;
            if (!__all_sync(0xffffffffu, mbar_wait_bounded(&tfull[acc], aph))) { ok = false; break; }
            tc_fence_after();
            float v[16];
            if (active)
                tmem_ld16(tmem + acc * ACC_COLS + (uint32_t(q * 32) << 16) + 16 * h, v);
            tc_fence_before();
            __syncwarp();
            if (lane == 0) mbar_arrive(&tempty[acc]);
            const int xt = t % xtiles, row = t / xtiles;
            const int y = row % a.H, b = row / a.H;
            const int x = xt * 128 + q * 32 + lane;
            if (!active || x >= a.W) continue;
            const size_t p = (size_t(b) * a.H + y) * a.W + x;
            const int c0 = 16 * h;
            if constexpr (EPI == EPI_LINEAR) {
                static_cast<float*>(a.out)[p] = v[0] + (a.bias ? a.bias[0] : 0.0f);
            } else {
                uint32_t o[8], pr[8];
#pragma unroll
                for (int c = 0; c < 16; c += 2) {
                    float v0 = v[c], v1 = v[c + 1];
                    if constexpr (EPI == EPI_GELU) {
                        v0 += bias[c];
                        v1 += bias[c + 1];
                        pr[c / 2] = pack_bf16(v0, v1);
                        o[c / 2] = pack_bf16(gelu(v0), gelu(v1));
                    } else {
                        const float g0 = gelu_grad(bf16_at(a.pre_in, p * N + c0 + c));
                        const float g1 = gelu_grad(bf16_at(a.pre_in, p * N + c0 + c + 1));
                        o[c / 2] = pack_bf16(v0 * g0, v1 * g1);
                    }
                }
                uint4* dst = reinterpret_cast<uint4*>(static_cast<bf16*>(a.out) + p * N + c0);
                dst[0] = make_uint4(o[0], o[1], o[2], o[3]);
                dst[1] = make_uint4(o[4], o[5], o[6], o[7]);
                if constexpr (EPI == EPI_GELU) {
                    if (a.pre_out) {
                        uint4* dp = reinterpret_cast<uint4*>(a.pre_out + p * N + c0);
                        dp[0] = make_uint4(pr[0], pr[1], pr[2], pr[3]);
                        dp[1] = make_uint4(pr[4], pr[5], pr[6], pr[7]);
                    }
                }
            }
        }
    }
    if (!ok && a.err) atomicOr(a.err, 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_free(tmem, 2 * ACC_COLS);
}

template <int N, int EPI>
cudaError_t launch_conv_tma(const ConvArgs& a, cudaStream_t s) {
    CUtensorMap map;
    if (reinterpret_cast<uintptr_t>(a.x) % 16 != 0 ||
        !tensor_map_act_bf16(a.x, 32, a.W, a.H, a.B, 128, &map))
        return cudaErrorNotSupported;
    constexpr size_t smem = ct_smem_bytes<N>();
    auto kern = conv_tma_kernel<N, EPI>;
    static bool attr = false;
    if (!attr) {
        const cudaError_t e =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const int xtiles = (a.W + 127) / 128;
    const long long nt = (long long)xtiles * a.H * a.B;
    if (nt >= (1ll << 31)) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(nt, sm_count());
    kern<<<grid, CT_THREADS, smem, s>>>(map, a, (int)nt, xtiles);
    return cudaGetLastError();
}

template <int CIN, int N, int EPI>
cudaError_t launch_conv(const ConvArgs& a, cudaStream_t s) {
    constexpr size_t smem = conv_smem_bytes<CIN, N>();
    auto kern = conv_kernel<CIN, N, EPI>;
    static bool attr = false;
    if (!attr) {
        const cudaError_t e =
            cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
        attr = true;
    }
    const dim3 grid((a.W + 127) / 128, a.H, a.B);
    kern<<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

}  // namespace sg
}  // namespace lpbf_b200

using namespace lpbf_b200;
using namespace lpbf_b200::sg;

extern "C" {

int lpbf_b200_sg_conv(int kind, const lpbf_b200_sg_conv_args* p, cudaStream_t stream) {
    if (!p || !p->x || !p->w || !p->out || p->batch < 1 || p->height < 1 || p->width < 1 ||
        p->height > 65535 || p->batch > 65535)
        return LPBF_ERR_ARG;
    ConvArgs a;
    a.x = p->x;
    a.w = static_cast<const bf16*>(p->w);
    a.bias = p->bias;
    a.pre_in = static_cast<const bf16*>(p->pre_in);
    a.pre_out = static_cast<bf16*>(p->pre_out);
    a.out = p->out;
    a.B = p->batch;
    a.H = p->height;
    a.W = p->width;
    a.err = p->err;
    cudaError_t e;
    switch (kind) {
        case LPBF_SG_FWD_IN:
            if (!a.bias) return LPBF_ERR_ARG;
            e = launch_conv<4, 32, EPI_GELU>(a, stream); break;
        case LPBF_SG_FWD_HIDDEN:
            if (!a.bias) return LPBF_ERR_ARG;
            e = launch_conv_tma<32, EPI_GELU>(a, stream);
            if (e == cudaErrorNotSupported) e = launch_conv<32, 32, EPI_GELU>(a, stream);
            break;
        case LPBF_SG_FWD_OUT:
            e = launch_conv_tma<16, EPI_LINEAR>(a, stream);
            if (e == cudaErrorNotSupported) e = launch_conv<32, 16, EPI_LINEAR>(a, stream);
            break;
        case LPBF_SG_DX_OUT:
            if (!a.pre_in) return LPBF_ERR_ARG;
            e = launch_conv<1, 32, EPI_DGELU>(a, stream); break;
        case LPBF_SG_DX_HIDDEN:
            if (!a.pre_in) return LPBF_ERR_ARG;
            e = launch_conv_tma<32, EPI_DGELU>(a, stream);
            if (e == cudaErrorNotSupported) e = launch_conv<32, 32, EPI_DGELU>(a, stream);
            break;
        default:
            return LPBF_ERR_ARG;
    }
    return e == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_gemm_bt(const void* A, const void* B, float* C, int n, int k, unsigned int* err,
                         cudaStream_t stream) {
    if (!A || !B || !C) return LPBF_ERR_ARG;
    if (!((n == 32 || n == 16) && k == 288)) return LPBF_ERR_UNSUPPORTED;
    const bf16* a = static_cast<const bf16*>(A);
    const bf16* b = static_cast<const bf16*>(B);
    cudaError_t e;
    if (n == 32) {
        constexpr size_t smem = 1024 + size_t(128 + 32) * 288 * 2;
        cudaFuncSetAttribute(gemm_bt_kernel<32, 288>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        gemm_bt_kernel<32, 288><<<1, 128, smem, stream>>>(a, b, C, err);
    } else {
        constexpr size_t smem = 1024 + size_t(128 + 16) * 288 * 2;
        cudaFuncSetAttribute(gemm_bt_kernel<16, 288>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)smem);
        gemm_bt_kernel<16, 288><<<1, 128, smem, stream>>>(a, b, C, err);
    }
    e = cudaGetLastError();
    return e == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

}  // extern "C"
