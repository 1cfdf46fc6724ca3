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

// Form of the 32-channel layers and of the input layer (LPBF_SG_FORM_*):
// row-streaming, tap-tile (32-channel layers only) or plain; each form falls
// back to the next when it cannot run.
int g_conv_form = 0;
int g_conv_form_used = -1;          // form of the last FWD_IN or 32-channel launch

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

// Epilogue of 16 accumulator columns (channels c0 .. c0 + 15) of pixel p.
// GELU: bias, pre-activation and activation out (bf16); LINEAR: channel 0
// plus bias (fp32); DGELU: times gelu'(pre_in) (bf16).
template <int N, int EPI>
__device__ __forceinline__ void epilogue16(const ConvArgs& a, size_t p, int c0, const float* v,
                                           const float* bias) {
    if constexpr (EPI == EPI_LINEAR) {
        static_cast<float*>(a.out)[p] = v[0] + (a.bias ? a.bias[0] : 0.0f);
    } else {
        uint32_t o[8], pr[8];
        if constexpr (EPI == EPI_GELU) {
#pragma unroll
            for (int c = 0; c < 16; c += 2) {
                const float v0 = v[c] + bias[c], v1 = v[c + 1] + bias[c + 1];
                pr[c / 2] = pack_bf16(v0, v1);
                o[c / 2] = pack_bf16(gelu(v0), gelu(v1));
            }
        } else {
            const uint4* src = reinterpret_cast<const uint4*>(a.pre_in + p * N + c0);
            const uint4 u0 = __ldg(src), u1 = __ldg(src + 1);
            const uint32_t w[8] = {u0.x, u0.y, u0.z, u0.w, u1.x, u1.y, u1.z, u1.w};
#pragma unroll
            for (int c = 0; c < 16; c += 2) {
                const float g0 = __uint_as_float(w[c / 2] << 16);
                const float g1 = __uint_as_float(w[c / 2] & 0xffff0000u);
                o[c / 2] = pack_bf16(v[c] * gelu_grad(g0), v[c + 1] * gelu_grad(g1));
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
            epilogue16<N, EPI>(a, (size_t(b) * a.H + y) * a.W + x, 16 * h, v, bias);
        }
    }
    if (!ok && a.err) atomicOr(a.err, 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_free(tmem, 2 * ACC_COLS);
}

// ---- row-streaming form (32- and 4-channel inputs) --------------------------
//
// A CTA walks runs of CR_RUN output rows of one 128-pixel column tile, three
// CTAs per SM.  Warp 0 streams the run's input rows, plus one above and one
// below, by TMA into a ring of slots; each input row crosses from L2 once
// per run instead of once per tap.
//   32 channels: a slot holds 130 pixels (the tile and one either side) of
//     one row, 64 bytes each, with the 64-byte swizzle, which is the tensor
//     core's K-major SW64 operand layout.  The A operand of tap (dy, dx) is
//     the slot of input row y + dy - 1 from its pixel dx on: the start
//     address moves by 64 bytes per pixel (the swizzle follows the address
//     bits, so the shifted operand reads what TMA wrote), no im2col copy.
//     18 MMAs per output row (9 taps x 2 halves of 16 channels).
//   4 channels: TMA brings 132 pixels of a row (8 bytes each, as pixel
//     pairs: a TMA box row must be a multiple of 16 bytes) into a small raw
//     ring; the 32 lanes of warp 0 then write the row's three x-taps per
//     pixel, (x-1, x, x+1) x 4 channels plus 4 zeros, as a K = 16 no-swizzle
//     operand slot.  An output row is then 3 MMAs, one per input row dy.
// Warp 1 issues an output row's MMAs into one of two TMEM accumulators,
// releases the input slot that no later output of the run reads (all three
// after the run's last output) and commits to the accumulator's "full"
// barrier; warps 2-9 run the epilogue as in the tap-tile form.  Waits are
// bounded; after a timeout the CTA records the error, waits (bounded) for
// its copies and MMAs in flight, frees its TMEM and returns.
constexpr int CR_PX = 130;                         // pixels of a 32-channel slot
constexpr int CR_ROW_BYTES = CR_PX * 64;           // 8320 bytes loaded per row
constexpr int CR_PITCH32 = 8704;                   // slot pitch: 512-byte swizzle period
constexpr int CR_X3_BYTES = 2 * 128 * 16;          // 4-channel operand slot
constexpr int CR_RAW_PAIRS = 66;                   // 132 pixels of a 4-channel row
constexpr int CR_RAW_BYTES = CR_RAW_PAIRS * 16;   // loaded per 4-channel row
constexpr int CR_RAW_PITCH = 1152;                 // raw slot pitch
constexpr int CR_RAW = 4;                          // raw 4-channel row slots
constexpr int CR_SLOTS = 5;                        // operand slots
constexpr int CR_RUN = 32;                         // output rows per work unit
constexpr int CR_CTAS = 3;                         // CTAs per SM
constexpr int CR_NACC = 2;                         // TMEM accumulators
// a TMA tensor copy lands on a 128-byte boundary
static_assert(CR_PITCH32 % 512 == 0 && CR_X3_BYTES % 128 == 0 && CR_RAW_PITCH % 128 == 0 &&
                  CR_RAW_PITCH >= CR_RAW_BYTES && CR_PITCH32 >= CR_ROW_BYTES,
              "row slots");

template <int CIN, int N>
constexpr size_t cr_smem_bytes() {
    return CIN == 32 ? 1024 + size_t(CR_SLOTS) * CR_PITCH32 + size_t(N) * 288 * 2
                     : 1024 + size_t(CR_SLOTS) * CR_X3_BYTES + size_t(CR_RAW) * CR_RAW_PITCH +
                           3 * size_t(N) * 32;
}

// Work unit u: column tile xt, image b, output rows y0 .. y0 + n - 1.
struct RowUnit { int b, xt, y0, n; };
__device__ __forceinline__ RowUnit row_unit(int u, int xtiles, int runs, int H) {
    RowUnit r;
    r.xt = u % xtiles;
    const int t = u / xtiles;
    r.b = t / runs;
    r.y0 = (t % runs) * CR_RUN;
    r.n = min(CR_RUN, H - r.y0);
    return r;
}

// The input rows of a CTA's units in order: unit u, row L = 0 .. n + 1
// (field row y0 - 1 + L).
struct RowCursor {
    int u, L, nunits, xtiles, runs, H;
    RowUnit r;
    __device__ RowCursor(int u0, int nu, int xt, int ru, int h)
        : u(u0), L(0), nunits(nu), xtiles(xt), runs(ru), H(h) {
        if (u < nunits) r = row_unit(u, xtiles, runs, H);
    }
    __device__ bool valid() const { return u < nunits; }
    __device__ void next() {
        if (++L == r.n + 2) {
            L = 0;
            u += gridDim.x;
            if (u < nunits) r = row_unit(u, xtiles, runs, H);
        }
    }
};

// No-swizzle K-major operand layouts in bf16 elements, (rows, K = 16) of one
// MMA: rows 16 bytes apart in groups of 8 (128 bytes), the two 8-entry
// halves of K 128 rows (A, 4-channel slot) or N rows (weights) apart.
using LayX3 = cute::Layout<cute::Shape<cute::Shape<cute::_8, cute::_16>,
                                       cute::Shape<cute::_8, cute::_2>>,
                           cute::Stride<cute::Stride<cute::_8, cute::_64>,
                                        cute::Stride<cute::_1, cute::_1024>>>;
template <int N>
using LayRowB = cute::Layout<cute::Shape<cute::Shape<cute::_8, cute::Int<N / 8>>,
                                         cute::Shape<cute::_8, cute::_2>>,
                             cute::Stride<cute::Stride<cute::_8, cute::_64>,
                                          cute::Stride<cute::_1, cute::Int<N * 8>>>>;

template <int CIN, int N, int EPI>
__global__ void __launch_bounds__(CT_THREADS, CR_CTAS)
conv_row_kernel(const __grid_constant__ CUtensorMap xmap, const ConvArgs a, int nunits,
                int xtiles, int runs) {
    static_assert(CIN == 32 || (CIN == 4 && N == 32), "row-streaming layers");
    using Mma = cute::SM100_MMA_F16BF16_SS<bf16, bf16, float, 128, N, cute::UMMA::Major::K,
                                           cute::UMMA::Major::K>;
    constexpr int ACC_COLS = N < 32 ? 32 : N;
    constexpr uint32_t S = CR_SLOTS;
    constexpr int PITCH = CIN == 32 ? CR_PITCH32 : CR_X3_BYTES;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t full[CR_SLOTS], empty[CR_SLOTS], rfull[CR_RAW], tfull[CR_NACC],
        tempty[CR_NACC], drain;
    __shared__ uint32_t tslot;
    uint8_t* base = align1024(smem_raw);
    uint8_t* sRows = base;                           // operand slots
    uint8_t* sRaw = base + size_t(CR_SLOTS) * PITCH; // 4-channel raw rows
    uint8_t* sB = CIN == 32 ? sRaw : sRaw + size_t(CR_RAW) * CR_RAW_PITCH;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) tmem_alloc(&tslot, CR_NACC * ACC_COLS);
    if (threadIdx.x == 0) {
        for (int i = 0; i < CR_SLOTS; ++i) { mbar_init(&full[i], 1); mbar_init(&empty[i], 1); }
        for (int i = 0; i < CR_RAW; ++i) mbar_init(&rfull[i], 1);
        for (int i = 0; i < CR_NACC; ++i) {
            mbar_init(&tfull[i], 1);
            mbar_init(&tempty[i], CT_EPI_WARPS);
        }
        mbar_init(&drain, 1);
        fence_mbar_init();
    }
    if constexpr (CIN == 32) {
        // weights, K-major without swizzle: the 16-byte unit of output
        // channel n and input entries k .. k + 7 at (k / 8) * N * 16 + n * 16
        for (int u = threadIdx.x; u < N * 36; u += blockDim.x) {
            const int n = u % N, kc = u / N;
            *reinterpret_cast<uint4*>(sB + size_t(kc) * N * 16 + n * 16) =
                __ldg(reinterpret_cast<const uint4*>(a.w + size_t(n) * 288 + kc * 8));
        }
    } else {
        // one K = 16 weight tile per input row dy: entry k' = dx * 4 + ci is
        // packed entry (3 dy + dx) * 4 + ci = 12 dy + k' of [N][64]; 12..15 zero
        uint16_t* B16 = reinterpret_cast<uint16_t*>(sB);
        const uint16_t* w16 = reinterpret_cast<const uint16_t*>(a.w);
        for (int e = threadIdx.x; e < 3 * N * 16; e += blockDim.x) {
            const int kk = e & 15, n = (e >> 4) % N, dy = e / (16 * N);
            B16[(dy * 2 * N * 16 + (kk >> 3) * N * 16 + n * 16) / 2 + (kk & 7)] =
                kk < 12 ? w16[n * 64 + 12 * dy + kk] : uint16_t(0);
        }
    }
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    bool ok = true;

    if (warp == 0) {
        if constexpr (CIN == 32) {
            if (lane == 0) {
                uint32_t g = 0;                      // input rows issued
                for (RowCursor c(blockIdx.x, nunits, xtiles, runs, a.H); c.valid(); c.next(), ++g) {
                    const uint32_t s = g % S;
                    if (!mbar_wait_bounded(&empty[s], ((g / S) & 1) ^ 1)) { ok = false; break; }
                    mbar_expect_tx(&full[s], CR_ROW_BYTES);
                    tma_load_4d(sRows + size_t(s) * PITCH, &xmap, 0, c.r.xt * 128 - 1,
                                c.r.y0 - 1 + c.L, c.r.b, &full[s]);
                }
                // the last copy issued into each slot has landed
                for (uint32_t i = 0; i < S && i < g; ++i) {
                    const uint32_t gi = g - 1 - i;
                    if (!mbar_wait_bounded(&full[gi % S], (gi / S) & 1)) ok = false;
                }
            }
        } else {
            RowCursor c(blockIdx.x, nunits, xtiles, runs, a.H);
            uint32_t issued = 0, g = 0;
            auto issue = [&]() {                     // next raw row into its slot
                if (lane == 0) {
                    const uint32_t rs = issued % CR_RAW;
                    fence_smem_async();              // earlier reads of the slot first
                    mbar_expect_tx(&rfull[rs], CR_RAW_BYTES);
                    tma_load_4d(sRaw + size_t(rs) * CR_RAW_PITCH, &xmap, 0,
                                c.r.xt * 64 - 1, c.r.y0 - 1 + c.L, c.r.b, &rfull[rs]);
                }
                ++issued;
                c.next();
            };
            for (int i = 0; i < CR_RAW && c.valid(); ++i) issue();
            for (; g < issued; ++g) {
                const uint32_t rs = g % CR_RAW, s = g % S;
                bool w = mbar_wait_bounded(&rfull[rs], (g / CR_RAW) & 1);
                w = w && mbar_wait_bounded(&empty[s], ((g / S) & 1) ^ 1);
                if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
                // raw pixel i is field pixel xt * 128 - 2 + i; slot row m takes
                // pixels m - 1, m (first half of K) and m + 1 (second half)
                const uint8_t* rp = sRaw + size_t(rs) * CR_RAW_PITCH;
                uint8_t* xp = sRows + size_t(s) * PITCH;
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int m = lane + 32 * i;
                    const uint2 p0 = *reinterpret_cast<const uint2*>(rp + (m + 1) * 8);
                    const uint2 p1 = *reinterpret_cast<const uint2*>(rp + (m + 2) * 8);
                    const uint2 p2 = *reinterpret_cast<const uint2*>(rp + (m + 3) * 8);
                    *reinterpret_cast<uint4*>(xp + m * 16) = make_uint4(p0.x, p0.y, p1.x, p1.y);
                    *reinterpret_cast<uint4*>(xp + 2048 + m * 16) = make_uint4(p2.x, p2.y, 0u, 0u);
                }
                fence_smem_async();                  // visible to the tensor core
                __syncwarp();
                if (lane == 0) mbar_arrive(&full[s]);
                if (c.valid()) issue();
            }
            // copies issued and not consumed have landed
            for (uint32_t gi = g; gi < issued; ++gi)
                if (!mbar_wait_bounded(&rfull[gi % CR_RAW], (gi / CR_RAW) & 1)) ok = false;
        }
    } else if (warp == 1) {
        using namespace cute;
        const uint64_t idesc =
            UMMA::make_runtime_instr_desc<bf16, bf16, float, 128, N, UMMA::Major::K,
                                          UMMA::Major::K>();
        uint64_t dA0;
        if constexpr (CIN == 32) {
            // K-major, 64-byte swizzle: rows 64 bytes apart, 8-row groups 512
            UMMA::SmemDescriptor d;
            d.version_ = 1;
            d.lbo_mode_ = 0;
            d.layout_type_ = uint8_t(UMMA::LayoutType::SWIZZLE_64B);
            d.start_address_ = uint16_t(smem_u32(sRows) >> 4);
            d.base_offset_ = 0;
            d.leading_byte_offset_ = 1;
            d.stride_byte_offset_ = 512 >> 4;
            dA0 = d;
        } else {
            dA0 = UMMA::make_umma_desc<UMMA::Major::K>(
                make_tensor(make_smem_ptr(reinterpret_cast<bf16*>(sRows)), LayX3{}));
        }
        const uint64_t dB0 = UMMA::make_umma_desc<UMMA::Major::K>(
            make_tensor(make_smem_ptr(reinterpret_cast<bf16*>(sB)), LayRowB<N>{}));
        uint32_t g = 0, o = 0;                       // first input row of the unit; outputs
        for (int u = blockIdx.x; ok && u < nunits; u += gridDim.x) {
            const RowUnit r = row_unit(u, xtiles, runs, a.H);
            for (int j = 0; j < r.n; ++j, ++o) {
                const int acc = o % CR_NACC;
                bool w = mbar_wait_bounded(&tempty[acc], ((o / CR_NACC) & 1) ^ 1);
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
                    const uint32_t gi = g + j + dy;
                    w = w && mbar_wait_bounded(&full[gi % S], (gi / S) & 1);
                }
                if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
                tc_fence_after();
                const uint32_t d = tmem + acc * ACC_COLS;
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
                    // start addresses in 16-byte units
                    const uint64_t da = dA0 + ((g + j + dy) % S) * (PITCH >> 4);
                    if constexpr (CIN == 32) {
#pragma unroll
                        for (int dx = 0; dx < 3; ++dx) {
#pragma unroll
                            for (int h = 0; h < 2; ++h) {
                                const int tap = dy * 3 + dx;
                                Mma::fma(da + 4 * dx + 2 * h, dB0 + (tap * 4 + 2 * h) * N, d,
                                         (tap | h) != 0 ? 1u : 0u, idesc);
                            }
                        }
                    } else {
                        Mma::fma(da, dB0 + dy * 2 * N, d, dy != 0 ? 1u : 0u, idesc);
                    }
                }
                cutlass::arch::umma_arrive(&empty[(g + j) % S]);
                if (j == r.n - 1) {
                    cutlass::arch::umma_arrive(&empty[(g + j + 1) % S]);
                    cutlass::arch::umma_arrive(&empty[(g + j + 2) % S]);
                }
                cutlass::arch::umma_arrive(&tfull[acc]);
            }
            g += r.n + 2;
        }
        // every MMA issued has completed before the accumulators are freed
        cutlass::arch::umma_arrive(&drain);
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&drain, 0))) ok = false;
    } else {
        const int q = warp & 3;                      // TMEM lane quarter of this warp
        const int h = (warp - 2) >> 2;               // column half: 0 or 1
        const bool active = N == 32 || h == 0;
        float bias[16];
#pragma unroll
        for (int c = 0; c < 16; ++c)
            bias[c] = (EPI == EPI_GELU && active) ? __ldg(a.bias + 16 * h + c) : 0.0f;
        uint32_t o = 0;
        for (int u = blockIdx.x; ok && u < nunits; u += gridDim.x) {
            const RowUnit r = row_unit(u, xtiles, runs, a.H);
            for (int j = 0; j < r.n; ++j, ++o) {
                const int acc = o % CR_NACC;
                if (!__all_sync(0xffffffffu,
                                mbar_wait_bounded(&tfull[acc], (o / CR_NACC) & 1))) {
                    ok = false;
                    break;
                }
                tc_fence_after();
                float v[16];
                if (active)
                    tmem_ld16(tmem + acc * ACC_COLS + (uint32_t(q * 32) << 16) + 16 * h, v);
                tc_fence_before();
                __syncwarp();
                if (lane == 0) mbar_arrive(&tempty[acc]);
                const int x = r.xt * 128 + q * 32 + lane;
                if (!active || x >= a.W) continue;
                epilogue16<N, EPI>(a, (size_t(r.b) * a.H + r.y0 + j) * a.W + x, 16 * h, v, bias);
            }
        }
    }
    if (!ok && a.err) atomicOr(a.err, 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_free(tmem, CR_NACC * ACC_COLS);
}

// ---- weight gradient of the 32 -> 32 layers, row-streaming ---------------------
//
// dW[co][(dy, dx, ci)] = sum over pixels p of g[p][co] x[p + (dy - 1, dx - 1)][ci]
// and db[co] = sum of g[p][co].  The same runs of output rows as the
// forward form; warp 0 streams the run's input rows (130 pixels, 64-byte
// swizzle) and its gradient rows (128 pixels) by TMA.  Both operands are
// read MN-major straight from those slots: for input row dy the A operand
// is M = 128 = four 32-channel blocks 64 bytes apart (block dx is the row
// shifted by dx pixels; the fourth is computed and dropped), K = 16 pixels;
// B is the gradient row, N = 32 channels, K = 16 pixels.  Eight MMAs per
// output row and dy accumulate into one of three TMEM accumulators (one per
// dy) for the CTA's whole share; the eight epilogue warps sum the bias
// gradient from the gradient slots meanwhile, and at the end write the
// CTA's partial record, which a second kernel sums over CTAs in a fixed
// order (deterministic).
constexpr int WR_XS = 4;                           // input-row slots
constexpr int WR_GS = 3;                           // gradient-row slots
constexpr int WR_GBYTES = 128 * 64;                // one gradient row
constexpr int WR_REC = 3 * 96 * 32 + 32;           // floats per CTA record
constexpr int WR_MAX_CTAS = 1024;
static_assert(CR_PITCH32 >= 131 * 64, "the dropped fourth block reads pixel 130");

size_t wgrad_rows_scratch(long long P) {
    return size_t(std::min<long long>(P, WR_MAX_CTAS)) * WR_REC * sizeof(float);
}

__device__ __forceinline__ uint64_t sw64_desc(const void* p, uint32_t lbo, uint32_t sbo) {
    cute::UMMA::SmemDescriptor d;
    d.version_ = 1;
    d.lbo_mode_ = 0;
    d.layout_type_ = uint8_t(cute::UMMA::LayoutType::SWIZZLE_64B);
    d.start_address_ = uint16_t(smem_u32(p) >> 4);
    d.base_offset_ = 0;
    d.leading_byte_offset_ = uint16_t(lbo >> 4);
    d.stride_byte_offset_ = uint16_t(sbo >> 4);
    return d;
}

__global__ void __launch_bounds__(CT_THREADS, CR_CTAS)
wgrad_row_kernel(const __grid_constant__ CUtensorMap xmap, const __grid_constant__ CUtensorMap gmap,
                 const ConvArgs a, float* partial, int nunits, int xtiles, int runs) {
    using Mma = cute::SM100_MMA_F16BF16_SS<bf16, bf16, float, 128, 32, cute::UMMA::Major::MN,
                                           cute::UMMA::Major::MN>;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t xfull[WR_XS], xempty[WR_XS], gfull[WR_GS], gempty[WR_GS], done;
    __shared__ uint32_t tslot;
    __shared__ float sbias[CT_EPI_WARPS][32];
    uint8_t* base = align1024(smem_raw);
    uint8_t* sX = base;
    uint8_t* sG = base + size_t(WR_XS) * CR_PITCH32;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;

    if (warp == 1) tmem_alloc(&tslot, 128);
    if (threadIdx.x == 0) {
        for (int i = 0; i < WR_XS; ++i) { mbar_init(&xfull[i], 1); mbar_init(&xempty[i], 1); }
        for (int i = 0; i < WR_GS; ++i) {
            mbar_init(&gfull[i], 1);
            mbar_init(&gempty[i], 1 + CT_EPI_WARPS);   // the MMAs' commit, the bias warps
        }
        mbar_init(&done, 1);
        fence_mbar_init();
    }
    // the bytes past the loaded 130 pixels of each input slot (read by the
    // dropped fourth block only) hold zeros, not stale values
    for (int i = threadIdx.x; i < WR_XS * (CR_PITCH32 - CR_ROW_BYTES) / 16; i += blockDim.x) {
        const int s = i / ((CR_PITCH32 - CR_ROW_BYTES) / 16), o = i % ((CR_PITCH32 - CR_ROW_BYTES) / 16);
        *reinterpret_cast<uint4*>(sX + size_t(s) * CR_PITCH32 + CR_ROW_BYTES + o * 16) =
            make_uint4(0u, 0u, 0u, 0u);
    }
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    bool ok = true;

    if (warp == 0) {
        if (lane == 0) {
            uint32_t gx = 0, gg = 0;                 // rows issued into each ring
            for (int u = blockIdx.x; ok && u < nunits; u += gridDim.x) {
                const RowUnit r = row_unit(u, xtiles, runs, a.H);
                for (int L = 0; L < r.n + 2 && ok; ++L) {
                    uint32_t s = gx % WR_XS;
                    if (!mbar_wait_bounded(&xempty[s], ((gx / WR_XS) & 1) ^ 1)) { ok = false; break; }
                    mbar_expect_tx(&xfull[s], CR_ROW_BYTES);
                    tma_load_4d(sX + size_t(s) * CR_PITCH32, &xmap, 0, r.xt * 128 - 1,
                                r.y0 - 1 + L, r.b, &xfull[s]);
                    ++gx;
                    if (L < 2) continue;
                    s = gg % WR_GS;
                    if (!mbar_wait_bounded(&gempty[s], ((gg / WR_GS) & 1) ^ 1)) { ok = false; break; }
                    mbar_expect_tx(&gfull[s], WR_GBYTES);
                    tma_load_4d(sG + size_t(s) * WR_GBYTES, &gmap, 0, r.xt * 128, r.y0 + L - 2, r.b,
                                &gfull[s]);
                    ++gg;
                }
            }
            // the last copy issued into each slot has landed
            for (uint32_t i = 0; i < WR_XS && i < gx; ++i) {
                const uint32_t gi = gx - 1 - i;
                if (!mbar_wait_bounded(&xfull[gi % WR_XS], (gi / WR_XS) & 1)) ok = false;
            }
            for (uint32_t i = 0; i < WR_GS && i < gg; ++i) {
                const uint32_t gi = gg - 1 - i;
                if (!mbar_wait_bounded(&gfull[gi % WR_GS], (gi / WR_GS) & 1)) ok = false;
            }
        }
    } else if (warp == 1) {
        const uint64_t idesc =
            cute::UMMA::make_runtime_instr_desc<bf16, bf16, float, 128, 32, cute::UMMA::Major::MN,
                                                cute::UMMA::Major::MN>();
        // MN-major, 64-byte swizzle: 32-channel blocks 64 bytes apart (LBO),
        // 8-pixel groups 512 bytes apart (SBO); in 16-byte units below
        const uint64_t dX0 = sw64_desc(sX, 64, 512), dG0 = sw64_desc(sG, 64, 512);
        uint32_t gx = 0, gg = 0;
        bool first = true;
        for (int u = blockIdx.x; ok && u < nunits; u += gridDim.x) {
            const RowUnit r = row_unit(u, xtiles, runs, a.H);
            for (int j = 0; j < r.n; ++j, ++gg) {
                bool w = mbar_wait_bounded(&gfull[gg % WR_GS], (gg / WR_GS) & 1);
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
                    const uint32_t gi = gx + j + dy;
                    w = w && mbar_wait_bounded(&xfull[gi % WR_XS], (gi / WR_XS) & 1);
                }
                if (!__all_sync(0xffffffffu, w)) { ok = false; break; }
                tc_fence_after();
                const uint64_t dg = dG0 + (gg % WR_GS) * (WR_GBYTES >> 4);
#pragma unroll
                for (int dy = 0; dy < 3; ++dy) {
                    const uint64_t dx = dX0 + ((gx + j + dy) % WR_XS) * (CR_PITCH32 >> 4);
#pragma unroll
                    for (int kk = 0; kk < 8; ++kk)   // 16 pixels = 1024 bytes per step
                        Mma::fma(dx + kk * 64, dg + kk * 64, tmem + dy * 32,
                                 (first && kk == 0) ? 0u : 1u, idesc);
                }
                first = false;
                cutlass::arch::umma_arrive(&gempty[gg % WR_GS]);
                cutlass::arch::umma_arrive(&xempty[(gx + j) % WR_XS]);
                if (j == r.n - 1) {
                    cutlass::arch::umma_arrive(&xempty[(gx + j + 1) % WR_XS]);
                    cutlass::arch::umma_arrive(&xempty[(gx + j + 2) % WR_XS]);
                }
            }
            gx += r.n + 2;
        }
        // every MMA issued has completed before the accumulators are read or freed
        cutlass::arch::umma_arrive(&done);
        if (!__all_sync(0xffffffffu, mbar_wait_bounded(&done, 0))) ok = false;
    } else {
        const int e = warp - 2;                      // epilogue warp 0..7
        // bias gradient: warp e sums pixels 16e .. 16e + 15 of each gradient
        // row, lane = channel (the 16-byte chunk of channels c / 8 of pixel
        // px sits at chunk (c / 8) ^ ((px / 2) % 4) of its 64-byte row)
        float bsum = 0.0f;
        uint32_t gg = 0;
        for (int u = blockIdx.x; ok && u < nunits; u += gridDim.x) {
            const RowUnit r = row_unit(u, xtiles, runs, a.H);
            for (int j = 0; j < r.n; ++j, ++gg) {
                if (!__all_sync(0xffffffffu,
                                mbar_wait_bounded(&gfull[gg % WR_GS], (gg / WR_GS) & 1))) {
                    ok = false;
                    break;
                }
                const uint8_t* gs = sG + size_t(gg % WR_GS) * WR_GBYTES;
#pragma unroll
                for (int i = 0; i < 16; ++i) {
                    const int px = 16 * e + i;
                    const uint16_t v = *reinterpret_cast<const uint16_t*>(
                        gs + px * 64 + ((((lane >> 3) ^ (px >> 1)) & 3) << 4) + (lane & 7) * 2);
                    bsum += __uint_as_float(uint32_t(v) << 16);
                }
                __syncwarp();
                if (lane == 0) mbar_arrive(&gempty[gg % WR_GS]);
            }
        }
        sbias[e][lane] = bsum;
        // the CTA's record: rows dx * 32 + ci of accumulator dy (TMEM lane
        // quarter q = dx; the fourth quarter is the dropped block)
        const int q = warp & 3, h = e >> 2;
        const bool w = __all_sync(0xffffffffu, ok && mbar_wait_bounded(&done, 0));
        tc_fence_after();
        float* rec = partial + size_t(blockIdx.x) * WR_REC;
        if (w && q < 3) {
#pragma unroll
            for (int dy = 0; dy < 3; ++dy) {
                float v[16];
                tmem_ld16(tmem + dy * 32 + 16 * h + (uint32_t(q * 32) << 16), v);
                float4* dst = reinterpret_cast<float4*>(rec + (dy * 96 + q * 32 + lane) * 32 + 16 * h);
#pragma unroll
                for (int c = 0; c < 4; ++c)
                    dst[c] = make_float4(v[4 * c], v[4 * c + 1], v[4 * c + 2], v[4 * c + 3]);
            }
        }
        if (!w) ok = false;
        asm volatile("bar.sync 1, %0;" :: "r"(32 * CT_EPI_WARPS) : "memory");
        if (e == 0) {
            float s = 0.0f;
#pragma unroll
            for (int i = 0; i < CT_EPI_WARPS; ++i) s += sbias[i][lane];
            rec[9216 + lane] = s;
        }
    }
    if (!ok && a.err) atomicOr(a.err, 1u);
    tc_fence_before();
    __syncthreads();
    if (warp == 1) tmem_free(tmem, 128);
}

// dW[co][tap * 32 + ci] and db[co] from the CTA records, summed in CTA order.
__global__ void wgrad_row_reduce(const float* partial, int nrec, float* dw, float* db) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= WR_REC) return;
    float s = 0.0f;
    for (int r = 0; r < nrec; ++r) s += partial[size_t(r) * WR_REC + e];
    if (e < 9216) {
        const int co = e & 31, row = e >> 5, dy = row / 96, m = row % 96;
        dw[co * 288 + (dy * 3 + (m >> 5)) * 32 + (m & 31)] = s;
    } else {
        db[e - 9216] = s;
    }
}

cudaError_t launch_wgrad_rows(const bf16* x, const bf16* g, int B, int H, int W, float* dw,
                              float* db, float* partial, unsigned int* err, cudaStream_t s) {
    CUtensorMap xm, gm;
    if (reinterpret_cast<uintptr_t>(x) % 16 != 0 || reinterpret_cast<uintptr_t>(g) % 16 != 0 ||
        !tensor_map_act_bf16(x, 32, W, H, B, CR_PX, &xm) ||
        !tensor_map_act_bf16(g, 32, W, H, B, 128, &gm))
        return cudaErrorNotSupported;
    constexpr size_t smem = 1024 + size_t(WR_XS) * CR_PITCH32 + size_t(WR_GS) * WR_GBYTES;
    if (const cudaError_t e = smem_opt_in<wgrad_row_kernel>(smem); e != cudaSuccess) return e;
    const int xtiles = (W + 127) / 128;
    const int runs = (H + CR_RUN - 1) / CR_RUN;
    const long long nu = (long long)xtiles * runs * B;
    const long long P = (long long)B * H * W;
    if (nu >= (1ll << 31)) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(
        {nu, (long long)CR_CTAS * sm_count(), (long long)WR_MAX_CTAS, P});
    ConvArgs a{};
    a.B = B; a.H = H; a.W = W; a.err = err;
    wgrad_row_kernel<<<grid, CT_THREADS, smem, s>>>(xm, gm, a, partial, (int)nu, xtiles, runs);
    wgrad_row_reduce<<<(WR_REC + 255) / 256, 256, 0, s>>>(partial, grid, dw, db);
    return cudaGetLastError();
}

// ---- weight gradients of the 4 -> 32 and 32 -> 1 layers, CUDA cores ---------
//
// Too narrow for 128-row tensor-core tiles (36 and 1 real rows): each thread
// owns fixed sums over the pixels of its CTA's runs of rows, read from three
// input rows and one gradient row staged in shared memory.
//   32 -> 1 : 288 threads, one (tap, input channel) each; thread 0 also the
//             bias.  Per pixel: one input value, one (broadcast) gradient.
//   4 -> 32 : 148 of 160 threads, (tap, input channel) x 8 output channels,
//             and 4 threads the bias of 8 channels each.
// Each CTA writes its record in the gradient's own order (dW[co][tap][ci],
// then db); a second kernel sums the records in CTA order.
template <int CIN, int COUT>
struct WgSmall {
    static constexpr int NOUT = 9 * CIN * COUT + COUT;
    static constexpr int THREADS = CIN == 32 ? 288 : 160;
    static constexpr int RUN = 8;    // output rows per unit: enough CTAs to hide latency
};

template <int CIN, int COUT>
__global__ void __launch_bounds__((WgSmall<CIN, COUT>::THREADS))
wgrad_small_kernel(const bf16* __restrict__ x, const bf16* __restrict__ g, int H, int W,
                   int nunits, int xtiles, int runs, float* partial) {
    static_assert((CIN == 32 && COUT == 1) || (CIN == 4 && COUT == 32), "narrow layers");
    constexpr int NOUT = WgSmall<CIN, COUT>::NOUT;
    // input rows as bf16 (pixel p of a slot is column xt * 128 - 1 + p), the
    // gradient row as fp32
    __shared__ __align__(16) uint16_t sx[3][CR_PX][CIN];
    __shared__ __align__(16) float sg[128][COUT];
    const int t = threadIdx.x;
    // outputs of this thread
    int tap = 0, ci = 0, cb = 0;
    bool bias = false, active = true;
    if constexpr (CIN == 32) {
        tap = t >> 5;
        ci = t & 31;
        bias = t == 0;
    } else {
        const int tc = t >> 2;
        cb = (t & 3) * 8;
        active = tc <= 36;
        bias = tc == 36;
        tap = bias ? 0 : tc >> 2;
        ci = tc & 3;
    }
    const int dy = tap / 3, dx = tap % 3;
    float acc[COUT == 32 ? 8 : 1];
    float bacc = 0.0f;
#pragma unroll
    for (int c = 0; c < (COUT == 32 ? 8 : 1); ++c) acc[c] = 0.0f;

    auto stage_x = [&](int slot, int b, int y, int x0) {
        // 16-byte units of CIN channels: CIN = 32: 4 per pixel; CIN = 4: half
        // a unit per pixel, so 8-byte units
        if constexpr (CIN == 32) {
            for (int i = t; i < CR_PX * 4; i += blockDim.x) {
                const int p = i >> 2, q = i & 3, xx = x0 - 1 + p;
                uint4 v = make_uint4(0u, 0u, 0u, 0u);
                if (y >= 0 && y < H && xx >= 0 && xx < W)
                    v = __ldg(reinterpret_cast<const uint4*>(
                        x + ((size_t(b) * H + y) * W + xx) * 32 + q * 8));
                *reinterpret_cast<uint4*>(&sx[slot][p][q * 8]) = v;
            }
        } else {
            for (int p = t; p < CR_PX; p += blockDim.x) {
                const int xx = x0 - 1 + p;
                uint2 v = make_uint2(0u, 0u);
                if (y >= 0 && y < H && xx >= 0 && xx < W)
                    v = __ldg(reinterpret_cast<const uint2*>(x + ((size_t(b) * H + y) * W + xx) * 4));
                *reinterpret_cast<uint2*>(&sx[slot][p][0]) = v;
            }
        }
    };
    auto stage_g = [&](int b, int y, int x0) {
        for (int i = t; i < 128 * COUT; i += blockDim.x) {
            const int p = i / COUT, c = i % COUT, xx = x0 + p;
            float v = 0.0f;
            if (xx < W) {
                const uint16_t u = reinterpret_cast<const uint16_t*>(g)[((size_t(b) * H + y) * W + xx) * COUT + c];
                v = __uint_as_float(uint32_t(u) << 16);
            }
            sg[p][c] = v;
        }
    };

    constexpr int RUN = WgSmall<CIN, COUT>::RUN;
    for (int u = blockIdx.x; u < nunits; u += gridDim.x) {
        RowUnit r;
        r.xt = u % xtiles;
        r.b = (u / xtiles) / runs;
        r.y0 = ((u / xtiles) % runs) * RUN;
        r.n = min(RUN, H - r.y0);
        const int x0 = r.xt * 128;
        stage_x(0, r.b, r.y0 - 1, x0);
        stage_x(1, r.b, r.y0, x0);
        for (int j = 0; j < r.n; ++j) {
            stage_x((j + 2) % 3, r.b, r.y0 + j + 1, x0);
            stage_g(r.b, r.y0 + j, x0);
            __syncthreads();
            if (active) {
                const uint16_t* xr = &sx[(j + dy) % 3][dx][ci];
                if constexpr (COUT == 1) {
#pragma unroll 8
                    for (int p = 0; p < 128; ++p) {
                        const float gv = sg[p][0];
                        acc[0] = fmaf(__uint_as_float(uint32_t(xr[p * CIN]) << 16), gv, acc[0]);
                        if (bias) bacc += gv;
                    }
                } else {
#pragma unroll 4
                    for (int p = 0; p < 128; ++p) {
                        const float4 g0 = *reinterpret_cast<const float4*>(&sg[p][cb]);
                        const float4 g1 = *reinterpret_cast<const float4*>(&sg[p][cb + 4]);
                        const float xv = bias ? 1.0f : __uint_as_float(uint32_t(xr[p * CIN]) << 16);
                        acc[0] = fmaf(xv, g0.x, acc[0]); acc[1] = fmaf(xv, g0.y, acc[1]);
                        acc[2] = fmaf(xv, g0.z, acc[2]); acc[3] = fmaf(xv, g0.w, acc[3]);
                        acc[4] = fmaf(xv, g1.x, acc[4]); acc[5] = fmaf(xv, g1.y, acc[5]);
                        acc[6] = fmaf(xv, g1.z, acc[6]); acc[7] = fmaf(xv, g1.w, acc[7]);
                    }
                }
            }
            __syncthreads();
        }
    }
    float* rec = partial + size_t(blockIdx.x) * NOUT;
    if constexpr (COUT == 1) {
        rec[tap * 32 + ci] = acc[0];
        if (bias) rec[288] = bacc;
    } else if (active) {
#pragma unroll
        for (int c = 0; c < 8; ++c) {
            if (bias) rec[9 * 4 * 32 + cb + c] = acc[c];
            else      rec[(cb + c) * 36 + tap * 4 + ci] = acc[c];
        }
    }
}

template <int NOUT, int NW>
__global__ void wgrad_small_reduce(const float* partial, int nrec, float* dw, float* db) {
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= NOUT) return;
    float s = 0.0f;
    for (int r = 0; r < nrec; ++r) s += partial[size_t(r) * NOUT + e];
    if (e < NW) dw[e] = s;
    else        db[e - NW] = s;
}

template <int CIN, int COUT>
cudaError_t launch_wgrad_small(const bf16* x, const bf16* g, int B, int H, int W, float* dw,
                               float* db, float* partial, cudaStream_t s) {
    constexpr int NOUT = WgSmall<CIN, COUT>::NOUT;
    if (reinterpret_cast<uintptr_t>(x) % 16 != 0) return cudaErrorNotSupported;
    constexpr int RUN = WgSmall<CIN, COUT>::RUN;
    const int xtiles = (W + 127) / 128;
    const int runs = (H + RUN - 1) / RUN;
    const long long nu = (long long)xtiles * runs * B;
    const long long P = (long long)B * H * W;
    if (nu >= (1ll << 31)) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>({nu, 8ll * sm_count(), (long long)WR_MAX_CTAS, P});
    wgrad_small_kernel<CIN, COUT><<<grid, WgSmall<CIN, COUT>::THREADS, 0, s>>>(
        x, g, H, W, (int)nu, xtiles, runs, partial);
    wgrad_small_reduce<NOUT, 9 * CIN * COUT><<<(NOUT + 255) / 256, 256, 0, s>>>(partial, grid, dw, db);
    return cudaGetLastError();
}

cudaError_t launch_wgrad_in(const bf16* x, const bf16* g, int B, int H, int W, float* dw, float* db,
                            float* partial, cudaStream_t s) {
    return launch_wgrad_small<4, 32>(x, g, B, H, W, dw, db, partial, s);
}
cudaError_t launch_wgrad_out(const bf16* x, const bf16* g, int B, int H, int W, float* dw,
                             float* db, float* partial, cudaStream_t s) {
    return launch_wgrad_small<32, 1>(x, g, B, H, W, dw, db, partial, s);
}

template <int N, int EPI>
cudaError_t launch_conv_tma(const ConvArgs& a, cudaStream_t s) {
    CUtensorMap map;
    if (reinterpret_cast<uintptr_t>(a.x) % 16 != 0 ||
        !tensor_map_act_bf16(a.x, 32, a.W, a.H, a.B, 128, &map))
        return cudaErrorNotSupported;
    constexpr size_t smem = ct_smem_bytes<N>();
    auto kern = conv_tma_kernel<N, EPI>;
    if (const cudaError_t e = smem_opt_in<conv_tma_kernel<N, EPI>>(smem); e != cudaSuccess)
        return e;
    const int xtiles = (a.W + 127) / 128;
    const long long nt = (long long)xtiles * a.H * a.B;
    if (nt >= (1ll << 31)) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(nt, sm_count());
    kern<<<grid, CT_THREADS, smem, s>>>(map, a, (int)nt, xtiles);
    return cudaGetLastError();
}

template <int CIN, int N, int EPI>
cudaError_t launch_conv_row(const ConvArgs& a, cudaStream_t s) {
    CUtensorMap map;
    if (reinterpret_cast<uintptr_t>(a.x) % 16 != 0) return cudaErrorNotSupported;
    if (CIN == 32 ? !tensor_map_act_bf16(a.x, 32, a.W, a.H, a.B, CR_PX, &map)
                  : (a.W % 2 != 0 || !tensor_map_pixel_pairs_bf16(a.x, a.W, a.H, a.B,
                                                                   CR_RAW_PAIRS, &map)))
        return cudaErrorNotSupported;
    constexpr size_t smem = cr_smem_bytes<CIN, N>();
    auto kern = conv_row_kernel<CIN, N, EPI>;
    if (const cudaError_t e = smem_opt_in<conv_row_kernel<CIN, N, EPI>>(smem); e != cudaSuccess)
        return e;
    const int xtiles = (a.W + 127) / 128;
    const int runs = (a.H + CR_RUN - 1) / CR_RUN;
    const long long nu = (long long)xtiles * runs * a.B;
    if (nu >= (1ll << 31)) return cudaErrorInvalidValue;
    const int grid = (int)std::min<long long>(nu, (long long)CR_CTAS * sm_count());
    kern<<<grid, CT_THREADS, smem, s>>>(map, a, (int)nu, xtiles, runs);
    return cudaGetLastError();
}

template <int CIN, int N, int EPI>
cudaError_t launch_conv(const ConvArgs& a, cudaStream_t s) {
    constexpr size_t smem = conv_smem_bytes<CIN, N>();
    auto kern = conv_kernel<CIN, N, EPI>;
    if (const cudaError_t e = smem_opt_in<conv_kernel<CIN, N, EPI>>(smem); e != cudaSuccess)
        return e;
    const dim3 grid((a.W + 127) / 128, a.H, a.B);
    kern<<<grid, 128, smem, s>>>(a);
    return cudaGetLastError();
}

// Row-streaming form first, then the tap-tile form, then the plain one (each
// declines with cudaErrorNotSupported when its tensor map cannot be made).
template <int N, int EPI>
cudaError_t launch_conv32(const ConvArgs& a, cudaStream_t s) {
    g_conv_form_used = 0;
    cudaError_t e = g_conv_form == 0 ? launch_conv_row<32, N, EPI>(a, s) : cudaErrorNotSupported;
    if (e == cudaErrorNotSupported && g_conv_form <= 1) {
        g_conv_form_used = 1;
        e = launch_conv_tma<N, EPI>(a, s);
    }
    if (e == cudaErrorNotSupported) {
        g_conv_form_used = 2;
        e = launch_conv<32, N, EPI>(a, s);
    }
    return e;
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
            g_conv_form_used = 0;
            e = g_conv_form == 0 ? launch_conv_row<4, 32, EPI_GELU>(a, stream)
                                 : cudaErrorNotSupported;
            if (e == cudaErrorNotSupported) {
                g_conv_form_used = 2;
                e = launch_conv<4, 32, EPI_GELU>(a, stream);
            }
            break;
        case LPBF_SG_FWD_HIDDEN:
            if (!a.bias) return LPBF_ERR_ARG;
            e = launch_conv32<32, EPI_GELU>(a, stream); break;
        case LPBF_SG_FWD_OUT:
            e = launch_conv32<16, EPI_LINEAR>(a, stream); break;
        case LPBF_SG_DX_OUT:
            if (!a.pre_in) return LPBF_ERR_ARG;
            e = launch_conv<1, 32, EPI_DGELU>(a, stream); break;
        case LPBF_SG_DX_HIDDEN:
            if (!a.pre_in) return LPBF_ERR_ARG;
            e = launch_conv32<32, EPI_DGELU>(a, stream); break;
        default:
            return LPBF_ERR_ARG;
    }
    return e == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_set_form(int form) {
    if (form < LPBF_SG_FORM_ROWS || form > LPBF_SG_FORM_PLAIN) return LPBF_ERR_ARG;
    g_conv_form = form;
    return LPBF_OK;
}

int lpbf_b200_sg_form_used(void) { return g_conv_form_used; }

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
