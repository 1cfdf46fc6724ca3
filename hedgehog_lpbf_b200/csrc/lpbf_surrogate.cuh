// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Tensor-core building blocks of the learned super-stepper (sm_100a).
//
// Every layer of the network is a 3x3 convolution computed as an implicit
// GEMM on the 5th-generation tensor cores: a CTA owns M = 128 consecutive
// pixels of one image row; A is the im2col tile of those pixels (K = 9 taps
// x C_in channels, bf16, staged in shared memory in the K-major SW64/SW128
// canonical layouts), B the layer's weights (N output channels x K), and D
// (fp32, 128 lanes x N columns) accumulates in tensor memory.  One elected
// thread issues all tcgen05.mma of a tile; tcgen05.commit arrives on an
// mbarrier that the CTA waits on (bounded); each warp then reads its 32
// accumulator lanes with tcgen05.ld for the epilogue.  The shared-memory and
// instruction descriptors come from CuTe's UMMA helpers (their layouts are
// checked at compile time).
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <cute/tensor.hpp>
#include <cute/atom/mma_traits_sm100.hpp>
#include <cute/arch/mma_sm100_umma.hpp>
#include <cutlass/arch/barrier.h>
#include <cutlass/bfloat16.h>

#include "lpbf_device.cuh"

namespace lpbf_b200 {
namespace sg {

using bf16 = cutlass::bfloat16_t;

// A tile of M = 128 rows by N columns with K-reduction KTOT; KATOM is the
// K width of one swizzle atom (32 bf16 = SW64, 64 bf16 = SW128).
template <int N, int KTOT, int KATOM>
struct TileMma {
    static constexpr int M = 128;
    static_assert(N % 16 == 0 && N >= 16 && N <= 256, "UMMA N for M = 128");
    static_assert(KTOT % KATOM == 0 && KTOT % 16 == 0, "K in whole atoms");
    using Op = cute::SM100_MMA_F16BF16_SS<bf16, bf16, float, M, N, cute::UMMA::Major::K,
                                          cute::UMMA::Major::K>;
    using Atom = typename std::conditional<KATOM == 32, cute::UMMA::Layout_K_SW64_Atom<bf16>,
                                           cute::UMMA::Layout_K_SW128_Atom<bf16>>::type;
    using LayA = decltype(cute::tile_to_shape(Atom{}, cute::Shape<cute::Int<M>, cute::Int<KTOT>>{}));
    using LayB = decltype(cute::tile_to_shape(Atom{}, cute::Shape<cute::Int<N>, cute::Int<KTOT>>{}));
    static constexpr int A_ELEMS = M * KTOT;
    static constexpr int B_ELEMS = N * KTOT;
    static constexpr int TMEM_COLS = N < 32 ? 32 : N;   // allocation unit: 32 columns

    // Address of element (r, k) of an A- or B-shaped tile (swizzle applied);
    // 8 consecutive k (one 16-byte unit) stay contiguous.
    __device__ static bf16* a_at(bf16* base, int r, int k) {
        auto t = cute::make_tensor(cute::make_smem_ptr(base), LayA{});
        return &t(r, k);
    }
    __device__ static bf16* b_at(bf16* base, int r, int k) {
        auto t = cute::make_tensor(cute::make_smem_ptr(base), LayB{});
        return &t(r, k);
    }

    // Issue the whole K reduction into tensor memory at `tmem` and commit
    // to `bar`; `accumulate` adds to the accumulator instead of starting it.
    // Called by one full warp (the atom elects one thread).
    __device__ static void issue(bf16* sA, bf16* sB, uint32_t tmem, uint64_t* bar,
                                 bool accumulate = false) {
        using namespace cute;
        auto tiled = make_tiled_mma(Op{});
        Tensor tA = make_tensor(make_smem_ptr(sA), LayA{});
        Tensor tB = make_tensor(make_smem_ptr(sB), LayB{});
        auto thr = tiled.get_slice(0);
        Tensor tCsA = thr.partition_A(tA);
        Tensor tCsB = thr.partition_B(tB);
        Tensor tCrA = thr.make_fragment_A(tCsA);
        Tensor tCrB = thr.make_fragment_B(tCsB);
        Tensor gC = make_tensor(make_gmem_ptr(static_cast<float*>(nullptr)),
                                make_shape(Int<M>{}, Int<N>{}), LayoutRight{});
        Tensor tCtAcc = thr.make_fragment_C(thr.partition_C(gC));
        tCtAcc.data() = tmem;
        tiled.accumulate_ = accumulate ? UMMA::ScaleOut::One : UMMA::ScaleOut::Zero;
        CUTE_UNROLL
        for (int k = 0; k < size<2>(tCrA); ++k) {
            gemm(tiled, tCrA(_, _, k), tCrB(_, _, k), tCtAcc);
            tiled.accumulate_ = UMMA::ScaleOut::One;
        }
        cutlass::arch::umma_arrive(bar);
    }
};

// ---- tensor memory and ordering --------------------------------------------

// Allocate `cols` TMEM columns (one full warp); the address lands in *slot.
__device__ __forceinline__ void tmem_alloc(uint32_t* slot, int cols) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;"
                 :: "r"(smem_u32(slot)), "r"(cols) : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tmem_free(uint32_t addr, int cols) {
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;"
                 :: "r"(addr), "r"(cols) : "memory");
}
__device__ __forceinline__ void tc_fence_before() {
    asm volatile("tcgen05.fence::before_thread_sync;" ::: "memory");
}
__device__ __forceinline__ void tc_fence_after() {
    asm volatile("tcgen05.fence::after_thread_sync;" ::: "memory");
}
// Generic-proxy shared-memory writes become visible to the tensor core.
__device__ __forceinline__ void fence_smem_async() {
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
}

// Thread's accumulator row (lane = 32 * warp + lane id): 16 or 32 fp32 columns.
__device__ __forceinline__ void tmem_ld16(uint32_t addr, float* v) {
    uint32_t r[16];
    asm volatile("tcgen05.ld.sync.aligned.32x32b.x16.b32 "
                 "{%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];"
                 : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]),
                   "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]),
                   "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
                 : "r"(addr));
    asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
#pragma unroll
    for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_ld32(uint32_t addr, float* v) {
    tmem_ld16(addr, v);
    tmem_ld16(addr + 16, v + 16);
}

// ---- activation ---------------------------------------------------------------

// GELU in its tanh form (Hendrycks and Gimpel, "Gaussian Error Linear
// Units", 2016): gelu(x) = x/2 (1 + tanh(u)), u = sqrt(2/pi) (x + 0.044715
// x^3), and its derivative.  tanh is the hardware's tanh.approx.f32 (about
// 11 significant bits): the activations it feeds are stored in bf16 (8).
__device__ __forceinline__ float tanh_approx(float x) {
    float y;
    asm("tanh.approx.f32 %0, %1;" : "=f"(y) : "f"(x));
    return y;
}
constexpr float GELU_C = 0.7978845608028654f;      // sqrt(2 / pi)
constexpr float GELU_A = 0.044715f;
constexpr float GELU_CA = GELU_C * GELU_A;
// u = x (C + C A x^2); gelu = x/2 + x/2 t (five FP32 operations and a tanh)
__device__ __forceinline__ float gelu(float x) {
    const float u = x * fmaf(x * x, GELU_CA, GELU_C);
    const float hx = 0.5f * x;
    return fmaf(hx, tanh_approx(u), hx);
}
// gelu' = (1 + t)/2 + x/2 (1 - t^2) u', u' = C + 3 C A x^2
__device__ __forceinline__ float gelu_grad(float x) {
    const float x2 = x * x;
    const float t = tanh_approx(x * fmaf(x2, GELU_CA, GELU_C));
    const float du = fmaf(x2, 3.0f * GELU_CA, GELU_C);
    const float hx = 0.5f * x;
    return fmaf(hx * fmaf(-t, t, 1.0f), du, fmaf(0.5f, t, 0.5f));
}

// Opt kernel KERN in to `bytes` of dynamic shared memory on the current
// device, once per device (the attribute belongs to each device's context).
template <auto KERN>
inline cudaError_t smem_opt_in(size_t bytes) {
    static bool done[64] = {};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) dev = 0;
    if (done[dev]) return cudaSuccess;
    const cudaError_t e =
        cudaFuncSetAttribute(KERN, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess) done[dev] = true;
    return e;
}

// ---- entry points shared with the training code (lpbf_surrogate.cu) -----------

// Layer kernel form (LPBF_SG_FORM_*), set by lpbf_b200_sg_set_form.
extern int g_conv_form;
// Weight and bias gradients of a 32 -> 32 layer in the row-streaming form
// (x: layer input, g: pre-activation gradient, both NHWC bf16 with 32
// channels; dw [32][288], db [32]); cudaErrorNotSupported when its tensor
// maps cannot be made.  `partial` holds wgrad_rows_scratch(P) bytes.
cudaError_t launch_wgrad_rows(const bf16* x, const bf16* g, int B, int H, int W, float* dw,
                              float* db, float* partial, unsigned int* err, cudaStream_t s);
size_t wgrad_rows_scratch(long long P);
// Weight and bias gradients of the input (4 -> 32) and output (32 -> 1)
// layers on CUDA cores, the same runs of rows; partial: wgrad_rows_scratch
// bytes suffice.
cudaError_t launch_wgrad_in(const bf16* x, const bf16* g, int B, int H, int W, float* dw, float* db,
                            float* partial, cudaStream_t s);
cudaError_t launch_wgrad_out(const bf16* x, const bf16* g, int B, int H, int W, float* dw,
                             float* db, float* partial, cudaStream_t s);

}  // namespace sg
}  // namespace lpbf_b200
