// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Learned super-stepper: the network as a whole (forward, loss, backward,
// AdamW), its input features and its application to a field.
//
// Network: 5 layers of 3x3 convolutions (zero padding), 4 -> 32 -> 32 -> 32
// -> 32 -> 1 channels, GELU after the first four; bf16 weights and
// activations, fp32 accumulation (tcgen05 kernels of lpbf_surrogate.cu).
// Inputs per pixel (bf16): (T - T_amb) / 1000 K, the Gaussian source summed
// over the next 16 steps / 1000 K, and the pixel's position relative to the
// laser at the middle of those steps in units of 100 um (x and y, clamped to
// +-8).  Output: (T after 16 steps - T) / 100 K.
//
// Weight gradients are a tensor-core GEMM over pixels: rows are (tap, input
// channel) pairs plus one all-ones row (the bias), columns the output
// channels, and K runs over 64-pixel blocks staged transposed in shared
// memory (double-buffered, one mbarrier per stage); per-CTA partials are
// summed by a second kernel in a fixed order (deterministic).
//
// Network blob (device, caller-allocated, lpbf_b200_sg_net_bytes): fp32
// master parameters, gradients, AdamW moments m and v (each
// LPBF_SG_PARAMS floats, layer by layer W[c_out][9][c_in] then b[c_out]),
// then the bf16 packed forward and input-gradient weights.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <cstring>

#include "lpbf_host.hpp"
#include "lpbf_surrogate.cuh"
#include "lpbf_b200.h"

namespace lpbf_b200 {
namespace sg {

constexpr int CIN_OF[5] = {4, 32, 32, 32, 32};
constexpr int COUT_OF[5] = {32, 32, 32, 32, 1};

struct NetLayout {
    size_t w_off[5], b_off[5];       // in floats, into the parameter vector
    size_t np;                       // parameters
    size_t params, grads, m, v;      // byte offsets of the fp32 sections
    size_t fwd[5], dx[5];            // byte offsets of the bf16 packs (dx[0] unused)
    int fwd_n[5], fwd_k[5], dx_n[5], dx_k[5];
    size_t bytes;
};

inline size_t al256(size_t v) { return (v + 255) & ~size_t(255); }

inline NetLayout net_layout() {
    NetLayout L{};
    size_t o = 0;
    for (int l = 0; l < 5; ++l) {
        L.w_off[l] = o; o += size_t(COUT_OF[l]) * 9 * CIN_OF[l];
        L.b_off[l] = o; o += COUT_OF[l];
    }
    L.np = o;
    size_t b = 0;
    L.params = b; b = al256(b + 4 * o);
    L.grads = b;  b = al256(b + 4 * o);
    L.m = b;      b = al256(b + 4 * o);
    L.v = b;      b = al256(b + 4 * o);
    for (int l = 0; l < 5; ++l) {
        L.fwd_n[l] = COUT_OF[l] == 1 ? 16 : 32;
        L.fwd_k[l] = CIN_OF[l] == 32 ? 288 : 64;
        L.fwd[l] = b; b = al256(b + 2 * size_t(L.fwd_n[l]) * L.fwd_k[l]);
    }
    for (int l = 1; l < 5; ++l) {
        L.dx_n[l] = 32;                                   // = CIN_OF[l]
        L.dx_k[l] = COUT_OF[l] == 32 ? 288 : 64;
        L.dx[l] = b; b = al256(b + 2 * size_t(L.dx_n[l]) * L.dx_k[l]);
    }
    L.bytes = b;
    return L;
}

// ---- weight gradient ---------------------------------------------------------

constexpr int WG_BLOCKS = 32;        // 64-pixel blocks per CTA (2048 pixels)

struct WgArgs {
    const bf16* x;                   // layer input [P][CIN]
    const bf16* g;                   // pre-activation gradient [P][COUT]
    float* partial;                  // [mtiles][chunks][128][N]
    int B, H, W;
    long long P;
    int chunks;
    unsigned int* err;
};

template <int CIN, int N>
__global__ void __launch_bounds__(128) wgrad_kernel(const WgArgs a) {
    using T = TileMma<N, 64, 64>;
    constexpr int R = 9 * CIN + 1;                     // rows: taps x channels, then bias
    constexpr int COUT = N == 16 ? 1 : 32;
    extern __shared__ uint8_t smem_raw[];
    __shared__ uint64_t bar[2];
    __shared__ uint32_t tslot;
    bf16* sA0 = reinterpret_cast<bf16*>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    bf16* sA[2] = {sA0, sA0 + T::A_ELEMS};
    bf16* sB[2] = {sA0 + 2 * T::A_ELEMS, sA0 + 2 * T::A_ELEMS + T::B_ELEMS};
    static_assert((T::A_ELEMS * 2) % 1024 == 0 && (T::B_ELEMS * 2) % 1024 == 0, "alignment");

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, tid = threadIdx.x;
    const int mt = blockIdx.y, chunk = blockIdx.x;
    const int r0 = mt * 128;
    const long long p0 = (long long)chunk * WG_BLOCKS * 64;
    const int nblk = (int)std::min<long long>(WG_BLOCKS, (a.P - p0 + 63) / 64);

    if (warp == 0) tmem_alloc(&tslot, T::TMEM_COLS);
    if (tid == 32) {
        mbar_init(&bar[0], 1);
        mbar_init(&bar[1], 1);
        fence_mbar_init();
    }
    {   // rows outside this tile's real rows stay zero for the whole kernel
        uint4* z = reinterpret_cast<uint4*>(sA0);
        const int n16 = (2 * T::A_ELEMS + 2 * T::B_ELEMS) * 2 / 16;
        for (int i = tid; i < n16; i += blockDim.x) z[i] = make_uint4(0u, 0u, 0u, 0u);
    }
    fence_smem_async();
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tmem = tslot;
    bool ok = true;
    // taps whose rows fall in this tile
    const int tap_lo = r0 / CIN;
    const int tap_hi = std::min(9, (r0 + 128 + CIN - 1) / CIN);
    const int ntap = tap_hi - tap_lo;
    const bool bias_here = (R - 1) >= r0 && (R - 1) < r0 + 128;

    for (int kb = 0; kb < nblk; ++kb) {
        const int st = kb & 1;
        if (kb >= 2) {
            const bool w = mbar_wait_bounded(&bar[st], ((kb - 2) >> 1) & 1);
            ok = __syncthreads_and(w) && ok;
            if (!ok) break;
        }
        bf16* A = sA[st];
        bf16* Bm = sB[st];
        const long long pb = p0 + (long long)kb * 64;
        // A: (tap, channel) rows, pixel columns
        for (int it = tid; it < 64 * ntap; it += blockDim.x) {
            const int j = it & 63, tap = tap_lo + (it >> 6);
            const long long p = pb + j;
            float vals[CIN];
#pragma unroll
            for (int c = 0; c < CIN; ++c) vals[c] = 0.0f;
            if (p < a.P) {
                const int x = (int)(p % a.W);
                const long long q = p / a.W;
                const int y = (int)(q % a.H);
                const int b = (int)(q / a.H);
                const int yy = y + tap / 3 - 1, xx = x + tap % 3 - 1;
                if (yy >= 0 && yy < a.H && xx >= 0 && xx < a.W) {
                    const bf16* src = a.x + ((size_t(b) * a.H + yy) * a.W + xx) * CIN;
#pragma unroll
                    for (int c = 0; c < CIN; ++c) vals[c] = float(src[c]);
                }
            }
#pragma unroll
            for (int c = 0; c < CIN; ++c) {
                const int r = tap * CIN + c - r0;
                if (r >= 0 && r < 128) *T::a_at(A, r, j) = bf16(vals[c]);
            }
        }
        if (bias_here && tid < 64) {
            const long long p = pb + tid;
            *T::a_at(A, R - 1 - r0, tid) = bf16(p < a.P ? 1.0f : 0.0f);
        }
        // B: output-channel rows, pixel columns
        if (tid < 64) {
            const long long p = pb + tid;
#pragma unroll
            for (int c = 0; c < COUT; ++c)
                *T::b_at(Bm, c, tid) = p < a.P ? a.g[size_t(p) * COUT + c] : bf16(0.0f);
        }
        fence_smem_async();
        __syncthreads();
        if (warp == 0) T::issue(A, Bm, tmem, &bar[st], kb > 0);
    }
    if (ok) {
        const int last = nblk - 1;
        ok = __all_sync(0xffffffffu, mbar_wait_bounded(&bar[last & 1], (last >> 1) & 1));
    }
    tc_fence_after();
    if (ok) {
        float v[32];
        if constexpr (N == 32) tmem_ld32(tmem + (uint32_t(warp * 32) << 16), v);
        else tmem_ld16(tmem + (uint32_t(warp * 32) << 16), v);
        const int r = warp * 32 + lane;
        if (r0 + r < R) {
            float* dst = a.partial + ((size_t(mt) * a.chunks + chunk) * 128 + r) * N;
#pragma unroll
            for (int c = 0; c < N; ++c) dst[c] = v[c];
        }
    } else if (tid == 0 && a.err) {
        atomicOr(a.err, 1u);
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 0) tmem_free(tmem, T::TMEM_COLS);
}

// dW[co][r] (r = tap * CIN + ci) and db[co] from the per-CTA partials.
template <int CIN, int N>
__global__ void wgrad_reduce_kernel(const float* partial, int chunks, float* dw, float* db) {
    constexpr int R = 9 * CIN + 1;
    constexpr int COUT = N == 16 ? 1 : 32;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R * COUT) return;
    const int r = i / COUT, co = i % COUT;
    const int mt = r / 128, rl = r % 128;
    const float* src = partial + (size_t(mt) * chunks * 128 + rl) * N + co;
    float s = 0.0f;
    for (int c = 0; c < chunks; ++c) s += src[size_t(c) * 128 * N];
    if (r < R - 1) dw[size_t(co) * (R - 1) + r] = s;
    else db[co] = s;
}

template <int CIN, int N>
size_t wgrad_partial_bytes(long long P) {
    const long long chunks = (P + WG_BLOCKS * 64 - 1) / (WG_BLOCKS * 64);
    const int mtiles = (9 * CIN + 1 + 127) / 128;
    return size_t(mtiles) * chunks * 128 * N * sizeof(float);
}

template <int CIN, int N>
cudaError_t launch_wgrad(const bf16* x, const bf16* g, int B, int H, int W, float* dw, float* db,
                         float* partial, unsigned int* err, cudaStream_t s) {
    using T = TileMma<N, 64, 64>;
    constexpr size_t smem = 1024 + 2 * size_t(T::A_ELEMS + T::B_ELEMS) * 2;
    if (const cudaError_t e = smem_opt_in<wgrad_kernel<CIN, N>>(smem); e != cudaSuccess)
        return e;
    WgArgs a;
    a.x = x; a.g = g; a.partial = partial; a.B = B; a.H = H; a.W = W;
    a.P = (long long)B * H * W;
    a.chunks = (int)((a.P + WG_BLOCKS * 64 - 1) / (WG_BLOCKS * 64));
    a.err = err;
    const int mtiles = (9 * CIN + 1 + 127) / 128;
    wgrad_kernel<CIN, N><<<dim3(a.chunks, mtiles), 128, smem, s>>>(a);
    constexpr int R = 9 * CIN + 1;
    constexpr int COUT = N == 16 ? 1 : 32;
    wgrad_reduce_kernel<CIN, N><<<(R * COUT + 127) / 128, 128, 0, s>>>(partial, a.chunks, dw, db);
    return cudaGetLastError();
}

size_t wgrad_scratch(long long P) {
    return std::max({wgrad_partial_bytes<4, 32>(P), wgrad_partial_bytes<32, 32>(P),
                     wgrad_partial_bytes<32, 16>(P), wgrad_rows_scratch(P)});
}

// 32 -> 32 layers: the row-streaming form unless another form is selected
// or it cannot run.
cudaError_t launch_wgrad32(const bf16* x, const bf16* g, int B, int H, int W, float* dw, float* db,
                           float* partial, unsigned int* err, cudaStream_t s) {
    cudaError_t e = g_conv_form == 0 ? launch_wgrad_rows(x, g, B, H, W, dw, db, partial, err, s)
                                     : cudaErrorNotSupported;
    if (e == cudaErrorNotSupported) e = launch_wgrad<32, 32>(x, g, B, H, W, dw, db, partial, err, s);
    return e;
}

// ---- loss, AdamW, packing, features ---------------------------------------------

// g = scale * (y - t) (bf16); per-block sums of (y - t)^2.
__global__ void loss_kernel(const float* y, const float* t, bf16* g, long long P, float scale,
                            float* block_sums) {
    __shared__ float red[256];
    float s = 0.0f;
    for (long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x; i < P;
         i += (long long)gridDim.x * blockDim.x) {
        const float r = y[i] - t[i];
        g[i] = bf16(scale * r);
        s += r * r;
    }
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) block_sums[blockIdx.x] = red[0];
}
__global__ void sum_kernel(const float* v, int n, double inv, float* out) {
    __shared__ double red[256];
    double s = 0.0;
    for (int i = threadIdx.x; i < n; i += blockDim.x) s += v[i];
    red[threadIdx.x] = s;
    __syncthreads();
    for (int o = blockDim.x / 2; o > 0; o >>= 1) {
        if (threadIdx.x < o) red[threadIdx.x] += red[threadIdx.x + o];
        __syncthreads();
    }
    if (threadIdx.x == 0) out[0] = (float)(red[0] * inv);
}

__global__ void adamw_kernel(float* p, const float* g, float* m, float* v, size_t n, float lr,
                             float b1, float b2, float eps, float wd, float c1, float c2) {
    const size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x;
    if (i >= n) return;
    const float gi = g[i];
    const float mi = b1 * m[i] + (1.0f - b1) * gi;
    const float vi = b2 * v[i] + (1.0f - b2) * gi * gi;
    m[i] = mi;
    v[i] = vi;
    p[i] = p[i] - lr * ((mi / c1) / (sqrtf(vi / c2) + eps) + wd * p[i]);
}

struct PackArgs {
    const float* params;
    bf16* fwd[5];
    bf16* dx[5];
    size_t w_off[5];
};

// One thread per packed element of every layer (forward and input-gradient).
__global__ void pack_kernel(const PackArgs a) {
    const int l = blockIdx.y;
    const int cin = l == 0 ? 4 : 32, cout = l == 4 ? 1 : 32;
    const float* W = a.params + a.w_off[l];                // [cout][9][cin]
    const int fn = cout == 1 ? 16 : 32, fk = cin == 32 ? 288 : 64;
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < fn * fk) {
        const int n = i / fk, k = i % fk;
        const float v = (n < cout && k < 9 * cin) ? W[size_t(n) * 9 * cin + k] : 0.0f;
        a.fwd[l][i] = bf16(v);
    }
    if (l >= 1) {
        const int dk = cout == 32 ? 288 : 64;              // dn = cin = 32
        if (i < 32 * dk) {
            const int ci = i / dk, k = i % dk;
            float v = 0.0f;
            if (k < 9 * cout) {
                const int t = k / cout, co = k % cout;
                v = W[(size_t(co) * 9 + (8 - t)) * cin + ci];
            }
            a.dx[l][i] = bf16(v);
        }
    }
}

cudaError_t launch_pack(unsigned char* net, const NetLayout& L, cudaStream_t s) {
    PackArgs a;
    a.params = reinterpret_cast<const float*>(net + L.params);
    for (int l = 0; l < 5; ++l) {
        a.fwd[l] = reinterpret_cast<bf16*>(net + L.fwd[l]);
        a.dx[l] = l >= 1 ? reinterpret_cast<bf16*>(net + L.dx[l]) : nullptr;
        a.w_off[l] = L.w_off[l];
    }
    pack_kernel<<<dim3((32 * 288 + 255) / 256, 5), 256, 0, s>>>(a);
    return cudaGetLastError();
}

struct SgLaser { double x, y, cs; };
struct FeatArgs {
    const double* T;
    int nx, ny;
    double dx, dy, Tamb, m2r, r2_cut;
    SgLaser las[LPBF_SG_STEPS];
    double xm, ym;                   // laser position at the middle step
    bf16* out;                       // [ny][nx][4]
};

__global__ void features_kernel(const FeatArgs a) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i >= (long long)a.nx * a.ny) return;
    const int x = (int)(i % a.nx), y = (int)(i / a.nx);
    const double px = x * a.dx, py = y * a.dy;
    double S = 0.0;
#pragma unroll 4
    for (int s = 0; s < LPBF_SG_STEPS; ++s) {
        if (a.las[s].cs == 0.0) continue;
        const double ddx = px - a.las[s].x, ddy = py - a.las[s].y;
        const double r2 = ddx * ddx + ddy * ddy;
        if (r2 < a.r2_cut) S += a.las[s].cs * exp(a.m2r * r2);
    }
    const float f0 = (float)((a.T[i] - a.Tamb) * (1.0 / LPBF_SG_T_SCALE));
    const float f1 = (float)(S * (1.0 / LPBF_SG_S_SCALE));
    const float f2 = fminf(fmaxf((float)((px - a.xm) * (1.0 / LPBF_SG_POS_SCALE)), -8.f), 8.f);
    const float f3 = fminf(fmaxf((float)((py - a.ym) * (1.0 / LPBF_SG_POS_SCALE)), -8.f), 8.f);
    bf16* o = a.out + size_t(i) * 4;
    o[0] = bf16(f0); o[1] = bf16(f1); o[2] = bf16(f2); o[3] = bf16(f3);
}

// T += y * DT_SCALE (the super-step), or the target of a pair of snapshots.
__global__ void apply_kernel(double* T, const float* y, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) T[i] += (double)y[i] * LPBF_SG_DT_SCALE;
}
__global__ void target_kernel(const double* T0, const double* T1, float* t, long long n) {
    const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
    if (i < n) t[i] = (float)((T1[i] - T0[i]) * (1.0 / LPBF_SG_DT_SCALE));
}

// ---- work buffer ----------------------------------------------------------------

struct Work {
    bf16* act[4];
    bf16* pre[4];
    float* y;
    bf16* g5;
    bf16* ga;
    bf16* gb;
    float* partial;
    float* lsum;
    size_t bytes;
};

inline Work work_layout(unsigned char* base, long long P, bool train) {
    Work w{};
    size_t o = 0;
    auto take = [&](size_t n) { const size_t r = o; o = al256(o + n); return base ? base + r : nullptr; };
    const size_t act = size_t(P) * 32 * 2;
    const int nact = train ? 4 : 2;                  // inference ping-pongs two buffers
    for (int l = 0; l < 4; ++l)
        w.act[l] = reinterpret_cast<bf16*>(l < nact ? take(act) : nullptr);
    if (!train) { w.act[2] = w.act[0]; w.act[3] = w.act[1]; }
    for (int l = 0; l < 4; ++l) w.pre[l] = train ? reinterpret_cast<bf16*>(take(act)) : nullptr;
    w.y = reinterpret_cast<float*>(take(size_t(P) * 4));
    if (train) {
        w.g5 = reinterpret_cast<bf16*>(take(size_t(P) * 2));
        w.ga = reinterpret_cast<bf16*>(take(act));
        w.gb = reinterpret_cast<bf16*>(take(act));
        w.partial = reinterpret_cast<float*>(take(wgrad_scratch(P)));
        w.lsum = reinterpret_cast<float*>(take(1024 * 4));
    }
    w.bytes = o;
    return w;
}

int conv(int kind, const void* x, const bf16* w, const float* bias, const bf16* pre_in,
         bf16* pre_out, void* out, int B, int H, int W, unsigned int* err, cudaStream_t s) {
    lpbf_b200_sg_conv_args a;
    a.x = x; a.w = w; a.bias = bias; a.pre_in = pre_in; a.pre_out = pre_out; a.out = out;
    a.batch = B; a.height = H; a.width = W; a.err = err;
    return lpbf_b200_sg_conv(kind, &a, s);
}

// Forward through the 5 layers; y (fp32) into w.y.
int forward(const unsigned char* net, const NetLayout& L, const void* x4, const Work& w, int B,
            int H, int W, bool keep_pre, unsigned int* err, cudaStream_t s) {
    const float* P = reinterpret_cast<const float*>(net + L.params);
    auto fwd = [&](int l) { return reinterpret_cast<const bf16*>(net + L.fwd[l]); };
    int st = conv(LPBF_SG_FWD_IN, x4, fwd(0), P + L.b_off[0], nullptr,
                  keep_pre ? w.pre[0] : nullptr, w.act[0], B, H, W, err, s);
    for (int l = 1; l < 4 && st == LPBF_OK; ++l)
        st = conv(LPBF_SG_FWD_HIDDEN, w.act[l - 1], fwd(l), P + L.b_off[l], nullptr,
                  keep_pre ? w.pre[l] : nullptr, w.act[l], B, H, W, err, s);
    if (st == LPBF_OK)
        st = conv(LPBF_SG_FWD_OUT, w.act[3], fwd(4), P + L.b_off[4], nullptr, nullptr, w.y, B, H,
                  W, err, s);
    return st;
}

}  // namespace sg
}  // namespace lpbf_b200

using namespace lpbf_b200;
using namespace lpbf_b200::sg;

extern "C" {

int lpbf_b200_sg_param_count(void) { return (int)net_layout().np; }
size_t lpbf_b200_sg_net_bytes(void) { return net_layout().bytes; }

size_t lpbf_b200_sg_work_bytes(int batch, int height, int width, int train) {
    if (batch < 1 || height < 1 || width < 1) return 0;
    return work_layout(nullptr, (long long)batch * height * width, train != 0).bytes;
}

int lpbf_b200_sg_net_set(void* net, const float* params, cudaStream_t stream) {
    if (!net || !params) return LPBF_ERR_ARG;
    const NetLayout L = net_layout();
    unsigned char* n = static_cast<unsigned char*>(net);
    if (cudaMemcpyAsync(n + L.params, params, L.np * 4, cudaMemcpyDefault, stream) != cudaSuccess ||
        cudaMemsetAsync(n + L.m, 0, L.np * 4, stream) != cudaSuccess ||
        cudaMemsetAsync(n + L.v, 0, L.np * 4, stream) != cudaSuccess ||
        cudaMemsetAsync(n + L.grads, 0, L.np * 4, stream) != cudaSuccess)
        return LPBF_ERR_CUDA;
    return launch_pack(n, L, stream) == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_net_get(const void* net, float* params, float* grads, cudaStream_t stream) {
    if (!net) return LPBF_ERR_ARG;
    const NetLayout L = net_layout();
    const unsigned char* n = static_cast<const unsigned char*>(net);
    if (params && cudaMemcpyAsync(params, n + L.params, L.np * 4, cudaMemcpyDefault, stream) !=
                      cudaSuccess)
        return LPBF_ERR_CUDA;
    if (grads && cudaMemcpyAsync(grads, n + L.grads, L.np * 4, cudaMemcpyDefault, stream) !=
                     cudaSuccess)
        return LPBF_ERR_CUDA;
    return LPBF_OK;
}

int lpbf_b200_sg_forward(const void* net, const void* x4, float* y, int batch, int height,
                         int width, void* work, size_t work_bytes, unsigned int* err,
                         cudaStream_t stream) {
    NvtxRange nvtx_range("lpbf_b200_sg_forward");
    if (!net || !x4 || !y || batch < 1 || height < 1 || width < 1) return LPBF_ERR_ARG;
    const long long P = (long long)batch * height * width;
    Work w = work_layout(static_cast<unsigned char*>(work), P, false);
    if (!work || work_bytes < w.bytes) return LPBF_ERR_WORKSPACE;
    w.y = y;
    return forward(static_cast<const unsigned char*>(net), net_layout(), x4, w, batch, height,
                   width, false, err, stream);
}

int lpbf_b200_sg_gradients(void* net, const void* x4, const float* target, int batch, int height,
                           int width, void* work, size_t work_bytes, float* loss,
                           unsigned int* err, cudaStream_t stream) {
    if (!net || !x4 || !target || batch < 1 || height < 1 || width < 1) return LPBF_ERR_ARG;
    const long long P = (long long)batch * height * width;
    const Work w = work_layout(static_cast<unsigned char*>(work), P, true);
    if (!work || work_bytes < w.bytes) return LPBF_ERR_WORKSPACE;
    const NetLayout L = net_layout();
    unsigned char* n = static_cast<unsigned char*>(net);
    int st = forward(n, L, x4, w, batch, height, width, true, err, stream);
    if (st != LPBF_OK) return st;
    const int nb = (int)std::min<long long>(1024, (P + 255) / 256);
    loss_kernel<<<nb, 256, 0, stream>>>(w.y, target, w.g5, P, (float)(2.0 / P), w.lsum);
    if (loss) sum_kernel<<<1, 256, 0, stream>>>(w.lsum, nb, 1.0 / P, loss);
    float* G = reinterpret_cast<float*>(n + L.grads);
    auto dxw = [&](int l) { return reinterpret_cast<const bf16*>(n + L.dx[l]); };
    // layer 5 (32 -> 1): weight gradient, then the gradient into layer 4
    cudaError_t e = g_conv_form == 0
        ? launch_wgrad_out(w.act[3], w.g5, batch, height, width, G + L.w_off[4], G + L.b_off[4],
                           w.partial, stream)
        : cudaErrorNotSupported;
    if (e == cudaErrorNotSupported)
        e = launch_wgrad<32, 16>(w.act[3], w.g5, batch, height, width, G + L.w_off[4],
                                 G + L.b_off[4], w.partial, err, stream);
    if (e != cudaSuccess) return LPBF_ERR_CUDA;
    st = conv(LPBF_SG_DX_OUT, w.g5, dxw(4), nullptr, w.pre[3], nullptr, w.ga, batch, height,
              width, err, stream);
    bf16* g = w.ga;
    bf16* g2 = w.gb;
    for (int l = 3; l >= 0 && st == LPBF_OK; --l) {
        const bf16* xin = l == 0 ? static_cast<const bf16*>(x4) : w.act[l - 1];
        if (l == 0) {
            e = g_conv_form == 0 ? launch_wgrad_in(xin, g, batch, height, width, G + L.w_off[0],
                                                   G + L.b_off[0], w.partial, stream)
                                 : cudaErrorNotSupported;
            if (e == cudaErrorNotSupported)
                e = launch_wgrad<4, 32>(xin, g, batch, height, width, G + L.w_off[0],
                                        G + L.b_off[0], w.partial, err, stream);
        } else {
            e = launch_wgrad32(xin, g, batch, height, width, G + L.w_off[l], G + L.b_off[l],
                               w.partial, err, stream);
        }
        if (e != cudaSuccess) return LPBF_ERR_CUDA;
        if (l > 0) {
            st = conv(LPBF_SG_DX_HIDDEN, g, dxw(l), nullptr, w.pre[l - 1], nullptr, g2, batch,
                      height, width, err, stream);
            std::swap(g, g2);
        }
    }
    return st;
}

int lpbf_b200_sg_adamw(void* net, const lpbf_b200_sg_hyper* h, cudaStream_t stream) {
    if (!net || !h || h->step < 1) return LPBF_ERR_ARG;
    const NetLayout L = net_layout();
    unsigned char* n = static_cast<unsigned char*>(net);
    const float c1 = 1.0f - std::pow(h->beta1, (float)h->step);
    const float c2 = 1.0f - std::pow(h->beta2, (float)h->step);
    adamw_kernel<<<(unsigned)((L.np + 255) / 256), 256, 0, stream>>>(
        reinterpret_cast<float*>(n + L.params), reinterpret_cast<const float*>(n + L.grads),
        reinterpret_cast<float*>(n + L.m), reinterpret_cast<float*>(n + L.v), L.np, h->lr,
        h->beta1, h->beta2, h->eps, h->weight_decay, c1, c2);
    if (cudaGetLastError() != cudaSuccess) return LPBF_ERR_CUDA;
    return launch_pack(n, L, stream) == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_train_step(void* net, const void* x4, const float* target, int batch, int height,
                            int width, const lpbf_b200_sg_hyper* h, void* work, size_t work_bytes,
                            float* loss, unsigned int* err, cudaStream_t stream) {
    NvtxRange nvtx_range("lpbf_b200_sg_train_step");
    if (!h) return LPBF_ERR_ARG;
    const int st = lpbf_b200_sg_gradients(net, x4, target, batch, height, width, work, work_bytes,
                                          loss, err, stream);
    return st != LPBF_OK ? st : lpbf_b200_sg_adamw(net, h, stream);
}

int lpbf_b200_sg_features(const double* T, const StepConst* k, const lpbf_tick* plan,
                          void* x4, cudaStream_t stream) {
    if (!T || !k || !plan || !x4 || k->nx < 1 || k->ny < 1) return LPBF_ERR_ARG;
    FeatArgs a;
    a.T = T; a.nx = k->nx; a.ny = k->ny; a.dx = k->dx; a.dy = k->dy; a.Tamb = k->Tamb;
    const Coef c = make_coef(*k, 0, k->Tamb, 0.0);
    a.m2r = c.m2r;
    a.r2_cut = c.r2_cut;
    for (int s = 0; s < LPBF_SG_STEPS; ++s) {
        const LaserSub l = make_laser(*k, plan[s].x_l, plan[s].y_l, plan[s].q_scale);
        a.las[s] = SgLaser{l.x_l, l.y_l, l.cs};
    }
    a.xm = plan[LPBF_SG_STEPS / 2].x_l;
    a.ym = plan[LPBF_SG_STEPS / 2].y_l;
    a.out = static_cast<bf16*>(x4);
    const long long n = (long long)k->nx * k->ny;
    features_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(a);
    return cudaGetLastError() == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_apply(double* T, const float* y, long long n, cudaStream_t stream) {
    if (!T || !y || n < 0) return LPBF_ERR_ARG;
    if (n == 0) return LPBF_OK;
    apply_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(T, y, n);
    return cudaGetLastError() == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_sg_target(const double* T0, const double* T1, float* t, long long n,
                        cudaStream_t stream) {
    if (!T0 || !T1 || !t || n < 0) return LPBF_ERR_ARG;
    if (n == 0) return LPBF_OK;
    target_kernel<<<(unsigned)((n + 255) / 256), 256, 0, stream>>>(T0, T1, t, n);
    return cudaGetLastError() == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

}  // extern "C"
