// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Launch logic and C-ABI of the FP32 steps (lpbf_f32k.cuh): the compensated
// field (lpbf_b200_advance_f32k, lpbf_b200_f32k_split, lpbf_b200_f32k_join)
// and the plain f32 field (lpbf_b200_advance_f32).
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cstring>

#include "lpbf_f32k.cuh"
#include "lpbf_host.hpp"
#include "lpbf_b200.h"

namespace lpbf_b200 {
namespace {

FkCoef make_fk(const Coef& c, double T_edge) {
    FkCoef f;
    f.ax = (float)c.ax;
    f.ay = (float)c.ay;
    f.cls = (float)c.c_ls;
    f.crad = (float)c.c_rad;
    // radiation is referred to Tamb; the linear losses to the temperature
    // at which convection (Tamb) and substrate conduction (Tsub) cancel:
    // c_conv (T - Tamb) + c_sub (T - Tsub) = c_ls (T - Tlin)
    const float a_hi = (float)c.Tamb;
    f.Ta4 = fk_pow4(a_hi, (float)(c.Tamb - (double)a_hi));
    const double Tlin = (c.same_T || c.c_ls == 0.0)
                            ? c.Tamb : (c.c_conv * c.Tamb + c.c_sub * c.Tsub) / c.c_ls;
    f.Ta_hi = (float)Tlin;
    f.Ta_lo = (float)(Tlin - (double)f.Ta_hi);
    f.Tedge_hi = (float)T_edge;
    f.Tedge_lo = (float)(T_edge - (double)f.Tedge_hi);
    f.clsTa = (float)((double)f.cls * Tlin);
    return f;
}

// COMP: the compensated pair field; otherwise the plain f32 field (lo_in and
// lo_out unused).
template <int K, bool REDUCE, bool SQ, bool COMP>
cudaError_t launch_fk(const float* hi_in, const float* lo_in, float* hi_out, float* lo_out,
                      const Coef& c, const FkCoef& f, const LaserSub* las, Partial* ring,
                      Workspace* ws, int rows, cudaStream_t stream) {
    auto kern = advance_f32k_kernel<K, REDUCE, SQ, COMP>;
    constexpr size_t smem = fk_smem_bytes<COMP>();
    static int occ[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (occ[dev] == 0) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)smem);
        if (e != cudaSuccess) return e;
        int nb = 0;
        e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern, ADV_WARPS * 32, smem);
        if (e != cudaSuccess) return e;
        occ[dev] = std::max(1, nb);
    }
    const int resident = sm_count() * occ[dev];
    FkParams p;
    std::memset(&p, 0, sizeof(p));
    p.c = c;
    p.f = f;
    for (int t = 0; t < K; ++t) p.las[t] = las[t];
    laser_band(c, las, K, &p.band_lo, &p.band_hi, &p.bandx_lo, &p.bandx_hi);
    p.nstrips = (c.nx + ADV_WOUT - 1) / ADV_WOUT;
    int H = rows;
    if (H <= 0) {
        // about three tasks per resident warp, 12..48 rows (48 measured best
        // at 8192^2, depth 3, for both fields over the bench raster)
        const long long want = (long long)c.ny * p.nstrips / (3ll * resident * ADV_WARPS);
        H = (int)std::max(12ll, std::min(48ll, want));
    }
    p.H = std::max(std::min(H, c.ny), 1);
    // rows whose tasks (owned rows +- K) reach the source band: 8-row tasks
    p.Hb = p.H;
    if (p.band_lo <= p.band_hi) {
        const int b0 = std::max(0, p.band_lo - K);
        const int b1 = std::min(c.ny, p.band_hi + K + 1);
        if (b0 < b1) {
            p.Hb = std::min(p.H, ADV_BAND_ROWS);
            p.nA = b0 / p.H;
            p.Ya = p.nA * p.H;
            p.Yb = b1;
            p.nB = (p.Yb - p.Ya + p.Hb - 1) / p.Hb;
        }
    }
    p.nchunks = p.nA + p.nB + (c.ny - p.Yb + p.H - 1) / p.H;
    p.ntasks = p.nstrips * p.nchunks;
    const int grid = std::max(1, std::min({(p.ntasks + ADV_WARPS - 1) / ADV_WARPS, resident,
                                           MAX_CTAS}));
    p.Thi_out = hi_out;
    p.Tlo_out = lo_out;
    p.ring = ring;
    p.scratch = ws->parts;
    p.counter = &ws->counter;
    p.tasks = &ws->tasks;
    p.err = &ws->err;
    CUtensorMap mh, ml;
    if (!tensor_map_f32(hi_in, c.nx, c.ny, ADV_COLS, ADV_R, &mh)) return cudaErrorNotSupported;
    if (COMP) {
        if (!tensor_map_f32(lo_in, c.nx, c.ny, ADV_COLS, ADV_R, &ml)) return cudaErrorNotSupported;
    } else {
        ml = mh;     // not read by the plain kernel
    }
    kern<<<grid, ADV_WARPS * 32, smem, stream>>>(mh, ml, p);
    return cudaGetLastError();
}

template <bool COMP>
cudaError_t launch_fk_k(int K, bool reduce, const float* hi_in, const float* lo_in,
                        float* hi_out, float* lo_out, const Coef& c, const FkCoef& f,
                        const LaserSub* las, Partial* ring, Workspace* ws, int rows,
                        cudaStream_t s) {
    // square cells (the f32 coefficients equal) take the one-Laplacian form
    const bool sq = f.ax == f.ay;
#define LPBF_FK(KK)                                                                          \
    case KK:                                                                                 \
        if (sq)                                                                              \
            return reduce ? launch_fk<KK, true, true, COMP>(hi_in, lo_in, hi_out, lo_out, c, \
                                                            f, las, ring, ws, rows, s)       \
                          : launch_fk<KK, false, true, COMP>(hi_in, lo_in, hi_out, lo_out, c, \
                                                             f, las, ring, ws, rows, s);     \
        return reduce ? launch_fk<KK, true, false, COMP>(hi_in, lo_in, hi_out, lo_out, c, f,  \
                                                         las, ring, ws, rows, s)             \
                      : launch_fk<KK, false, false, COMP>(hi_in, lo_in, hi_out, lo_out, c, f, \
                                                          las, ring, ws, rows, s);
    switch (K) {
        LPBF_FK(1)
        LPBF_FK(2)
        LPBF_FK(3)
        LPBF_FK(4)
        default: return cudaErrorInvalidValue;
    }
#undef LPBF_FK
}

__global__ void split_kernel(const double* __restrict__ T, float* __restrict__ hi,
                             float* __restrict__ lo, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x) {
        const double t = T[i];
        const float h = (float)t;
        hi[i] = h;
        lo[i] = (float)(t - (double)h);
    }
}

__global__ void join_kernel(const float* __restrict__ hi, const float* __restrict__ lo,
                            double* __restrict__ T, size_t n) {
    for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n;
         i += (size_t)gridDim.x * blockDim.x)
        T[i] = (double)hi[i] + (double)lo[i];
}

bool aligned16(const void* p) { return reinterpret_cast<uintptr_t>(p) % 16 == 0; }

}  // namespace
}  // namespace lpbf_b200

using namespace lpbf_b200;

extern "C" {

int lpbf_b200_f32k_split(const double* T, float* hi, float* lo, size_t n, cudaStream_t s) {
    if (!T || !hi || !lo) return LPBF_ERR_ARG;
    if (n == 0) return LPBF_OK;
    const int grid = std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 8);
    split_kernel<<<grid, 256, 0, s>>>(T, hi, lo, n);
    return cudaGetLastError() == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_f32k_join(const float* hi, const float* lo, double* T, size_t n, cudaStream_t s) {
    if (!T || !hi || !lo) return LPBF_ERR_ARG;
    if (n == 0) return LPBF_OK;
    const int grid = std::min<size_t>((n + 255) / 256, (size_t)sm_count() * 8);
    join_kernel<<<grid, 256, 0, s>>>(hi, lo, T, n);
    return cudaGetLastError() == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_advance_f32k(float* hi_a, float* lo_a, float* hi_b, float* lo_b,
                           const StepConst* k, const lpbf_tick* plan, int n_steps,
                           const lpbf_b200_opts* opts, Partial* ring, void* work,
                           size_t work_bytes, cudaStream_t stream, int* result_in_b) {
    NvtxRange nvtx_range("lpbf_b200_advance_f32k");
    if (!k || k->nx < 2 || k->ny < 1 || !opts || !hi_a || !lo_a || !hi_b || !lo_b ||
        n_steps < 0 || (n_steps > 0 && !plan) || !result_in_b)
        return LPBF_ERR_ARG;
    if (opts->bc != 0 && opts->bc != 1) return LPBF_ERR_ARG;
    if (opts->phys != 0 && opts->phys != 1) return LPBF_ERR_ARG;
    if (opts->phys == 1) return LPBF_ERR_UNSUPPORTED;     // baseline physics only
    if (k->nx % 4 != 0 || !aligned16(hi_a) || !aligned16(lo_a) || !aligned16(hi_b) ||
        !aligned16(lo_b))
        return LPBF_ERR_UNSUPPORTED;
    const size_t N = (size_t)k->nx * k->ny;
    const float* bufs[4] = {hi_a, lo_a, hi_b, lo_b};
    for (int i = 0; i < 4; ++i)
        for (int j = i + 1; j < 4; ++j)
            if (bufs[i] < bufs[j] + N && bufs[j] < bufs[i] + N) return LPBF_ERR_ARG;
    Workspace* ws = static_cast<Workspace*>(work);
    if (!ws || work_bytes < sizeof(Workspace)) return LPBF_ERR_WORKSPACE;

    int depth = opts->depth;
    if (depth <= 0) {
        const long long n = (long long)N;
        depth = (n >= (1ll << 22)) ? 3 : (n >= (1ll << 18)) ? 2 : 1;
    }
    depth = std::min(std::max(depth, 1), 4);
    const Coef c = make_coef(*k, opts->bc, opts->T_edge, opts->Tm);
    const FkCoef f = make_fk(c, opts->T_edge);
    float *ch = hi_a, *cl = lo_a, *nh = hi_b, *nl = lo_b;
    int in_b = 0;
    for (int s0 = 0; s0 < n_steps; s0 += depth) {
        const int kk = std::min(depth, n_steps - s0);
        LaserSub las[KMAX];
        for (int t = 0; t < kk; ++t)
            las[t] = make_laser(*k, plan[s0 + t].x_l, plan[s0 + t].y_l, plan[s0 + t].q_scale);
        const cudaError_t e = launch_fk_k<true>(kk, ring != nullptr, ch, cl, nh, nl, c, f, las,
                                                ring ? ring + s0 : nullptr, ws, opts->rows,
                                                stream);
        if (e == cudaErrorNotSupported) return LPBF_ERR_TMA;
        if (e != cudaSuccess) return LPBF_ERR_CUDA;
        std::swap(ch, nh);
        std::swap(cl, nl);
        in_b ^= 1;
    }
    *result_in_b = in_b;
    return LPBF_OK;
}

int lpbf_b200_advance_f32(float* T_a, float* T_b, const StepConst* k, const lpbf_tick* plan,
                          int n_steps, const lpbf_b200_opts* opts, Partial* ring, void* work,
                          size_t work_bytes, cudaStream_t stream, int* result_in_b) {
    NvtxRange nvtx_range("lpbf_b200_advance_f32");
    if (!k || k->nx < 2 || k->ny < 1 || !opts || !T_a || !T_b || n_steps < 0 ||
        (n_steps > 0 && !plan) || !result_in_b)
        return LPBF_ERR_ARG;
    if (opts->bc != 0 && opts->bc != 1) return LPBF_ERR_ARG;
    if (opts->phys != 0 && opts->phys != 1) return LPBF_ERR_ARG;
    if (opts->phys == 1) return LPBF_ERR_UNSUPPORTED;     // baseline physics only
    if (k->nx % 4 != 0 || !aligned16(T_a) || !aligned16(T_b)) return LPBF_ERR_UNSUPPORTED;
    const size_t N = (size_t)k->nx * k->ny;
    if (T_a < T_b + N && T_b < T_a + N) return LPBF_ERR_ARG;
    Workspace* ws = static_cast<Workspace*>(work);
    if (!ws || work_bytes < sizeof(Workspace)) return LPBF_ERR_WORKSPACE;

    int depth = opts->depth;
    if (depth <= 0) {
        const long long n = (long long)N;
        depth = (n >= (1ll << 22)) ? 3 : (n >= (1ll << 18)) ? 2 : 1;
    }
    depth = std::min(std::max(depth, 1), 4);
    const Coef c = make_coef(*k, opts->bc, opts->T_edge, opts->Tm);
    const FkCoef f = make_fk(c, opts->T_edge);
    float *cur = T_a, *nxt = T_b;
    int in_b = 0;
    for (int s0 = 0; s0 < n_steps; s0 += depth) {
        const int kk = std::min(depth, n_steps - s0);
        LaserSub las[KMAX];
        for (int t = 0; t < kk; ++t)
            las[t] = make_laser(*k, plan[s0 + t].x_l, plan[s0 + t].y_l, plan[s0 + t].q_scale);
        const cudaError_t e = launch_fk_k<false>(kk, ring != nullptr, cur, nullptr, nxt, nullptr,
                                                 c, f, las, ring ? ring + s0 : nullptr, ws,
                                                 opts->rows, stream);
        if (e == cudaErrorNotSupported) return LPBF_ERR_TMA;
        if (e != cudaSuccess) return LPBF_ERR_CUDA;
        std::swap(cur, nxt);
        in_b ^= 1;
    }
    *result_in_b = in_b;
    return LPBF_OK;
}

}  // extern "C"
