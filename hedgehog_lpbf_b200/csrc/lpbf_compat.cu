// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// The reference's five launch wrappers (include/lpbf_kernels.hpp) on the
// B200 kernels, plus the extended-physics step.
//
//   lpbf_launch_step            -> temporally blocked kernel with K = 1,
//                                  no reduction (phys 0); ext kernel (phys 1)
//   lpbf_launch_step_reduce     -> same, with the reduction folded in: one
//                                  Partial per CTA, the remaining entries of
//                                  the caller's array set to the neutral
//                                  element so the caller's finalize over
//                                  ((nx+15)/16)*((ny+15)/16) entries is exact
//   lpbf_launch_reduce          -> row-parallel block reduce
//   lpbf_launch_reduce_finalize -> one 8-CTA cluster; partial results are
//                                  combined through distributed shared memory
//                                  (replaces the reference's <<<1,1>>> loop)
//   lpbf_launch_extract_col     -> one thread per row
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cooperative_groups.h>

#include "lpbf_host.hpp"
#include "lpbf_kernels.hpp"

namespace cg = cooperative_groups;

namespace lpbf_b200 {

// ---- extended physics (temperature-dependent IN718 properties) ------------
// Mills tables, include/params.hpp:67-73 (physical data, identical values).
__constant__ double c_T_PTS[9]  = {298, 473, 673, 873, 1073, 1273, 1473, 1533, 1609};
__constant__ double c_K_PTS[9]  = {8.9, 12.9, 15.8, 18.7, 21.9, 25.6, 28.6, 29.3, 29.6};
__constant__ double c_CP_PTS[9] = {435, 479, 515, 558, 580, 628, 670, 685, 720};
constexpr double T_SOL = 1533.0, T_LIQ = 1609.0, LATENT = 210.0e3;

// params.hpp:75-83: clamped piecewise-linear lookup.
__device__ __forceinline__ double tab_interp(double T, const double* ys) {
    if (T <= c_T_PTS[0]) return ys[0];
    if (T >= c_T_PTS[8]) return ys[8];
    int i = 1;
    while (T > c_T_PTS[i]) ++i;
    const double f = (T - c_T_PTS[i - 1]) / (c_T_PTS[i] - c_T_PTS[i - 1]);
    return ys[i - 1] + f * (ys[i] - ys[i - 1]);
}
__device__ __forceinline__ double k_eff_d(double T, double kmult) {
    const double k = tab_interp(T, c_K_PTS);
    if (kmult <= 1.0) return k;
    const double s = (T <= T_SOL) ? 0.0 : (T >= T_LIQ) ? 1.0 : (T - T_SOL) / (T_LIQ - T_SOL);
    return k * (1.0 + (kmult - 1.0) * s);
}
__device__ __forceinline__ double cp_eff_d(double T) {
    double c = tab_interp(T, c_CP_PTS);
    if (T >= T_SOL && T <= T_LIQ) c += LATENT / (T_LIQ - T_SOL);
    return c;
}

__global__ void reduce_rows_kernel(const double* __restrict__ T, int nx, int ny, double Tm,
                                   Partial* __restrict__ out);
constexpr int FIN_CTAS = 8;
constexpr int FIN_THREADS = 512;
__global__ void finalize_cluster_kernel(const Partial* __restrict__ parts, int nblocks, int nx, int ny,
                        Partial* __restrict__ out);

// Launch finalize_cluster_kernel as one cluster of FIN_CTAS CTAs.
inline cudaError_t launch_finalize(const Partial* parts, int nblocks, int nx, int ny,
                                   Partial* out, cudaStream_t stream) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(FIN_CTAS, 1, 1);
    cfg.blockDim = dim3(FIN_THREADS, 1, 1);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = stream;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeClusterDimension;
    attr[0].val.clusterDim.x = FIN_CTAS;
    attr[0].val.clusterDim.y = 1;
    attr[0].val.clusterDim.z = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, finalize_cluster_kernel, parts, nblocks, nx, ny, out);
}

struct ExtParams {
    StepConst k;
    int bc;
    double T_edge, Tm;
    Partial* ring;
    Partial* scratch;
    unsigned int* counter;
    Partial* ref_out;
    long long ref_nparts;
};

// One thread per cell, 16 x 16 blocks (the reference's layout, so the
// reference fused-reduce array has exactly one entry per block).  The cell
// arithmetic follows include/step_task.hpp:144-184.
template <bool REDUCE>
__global__ void __launch_bounds__(256)
ext_step_kernel(const double* __restrict__ Tin, double* __restrict__ Tout,
                const __grid_constant__ ExtParams p) {
    const StepConst& k = p.k;
    const int x = blockIdx.x * 16 + threadIdx.x;
    const int y = blockIdx.y * 16 + threadIdx.y;
    const int nx = k.nx, ny = k.ny;
    const long long N = (long long)nx * ny;
    double v = -1.0;
    bool inside = x < nx && y < ny;
    if (inside) {
        const long long c = (long long)y * nx + x;
        if (p.bc == 1 && (x == 0 || y == 0 || x == nx - 1 || y == ny - 1)) {
            v = p.T_edge;
        } else {
            const double T = Tin[c];
            const double Txm = (x == 0) ? T : Tin[c - 1];
            const double Txp = (x == nx - 1) ? T : Tin[c + 1];
            const double Tym = (y == 0) ? T : Tin[c - nx];
            const double Typ = (y == ny - 1) ? T : Tin[c + nx];
            const double kC = k_eff_d(T, k.kmult);
            const double kxm = 0.5 * (kC + k_eff_d(Txm, k.kmult));
            const double kxp = 0.5 * (kC + k_eff_d(Txp, k.kmult));
            const double kym = 0.5 * (kC + k_eff_d(Tym, k.kmult));
            const double kyp = 0.5 * (kC + k_eff_d(Typ, k.kmult));
            const double div = (kxp * (Txp - T) - kxm * (T - Txm)) * k.inv_dx2
                             + (kyp * (Typ - T) - kym * (T - Tym)) * k.inv_dy2;
            const double xd = __dsub_rn(__dmul_rn((double)x, k.dx), k.x_l);
            const double yd = __dsub_rn(__dmul_rn((double)y, k.dy), k.y_l);
            const double r2 = __dadd_rn(__dmul_rn(xd, xd), __dmul_rn(yd, yd));
            double q_in = 0.0;
            if (k.q_scale != 0.0 && r2 * k.inv_r0_sq < 0.5 * EXP_CUT)
                q_in = k.q_scale * k.peak_S * exp(__dmul_rn(-2.0 * r2, k.inv_r0_sq));
            double q_top = k.hConv * (T - k.Tamb);
            if (k.radiation) {
                const double T4 = T * T * T * T;
                const double Ta4 = k.Tamb * k.Tamb * k.Tamb * k.Tamb;
                q_top += k.eps * SIGMA_SB * (T4 - Ta4);
            }
            const double q_bot = (tab_interp(T, c_K_PTS) / k.dSub) * (T - k.Tsub);
            const double rhs = div + (q_in - q_top - q_bot) * k.inv_h;
            v = T + k.dt * rhs / (k.rho * cp_eff_d(T));
        }
        Tout[c] = v;
    }
    if constexpr (REDUCE) {
        double tm = inside ? v : -1.0;
        long long ag = inside ? (long long)y * nx + x : N;
        int mn = ny, mx = -1;
        if (inside && v > p.Tm) { mn = y; mx = y; }
        if (!(tm > -1.0)) { tm = -1.0; ag = N; }   // NaN and values <= -1 never win
        partial_warp_reduce(tm, ag, mn, mx);
        __shared__ Partial red[8];
        __shared__ unsigned int s_last;
        const int tid = threadIdx.y * 16 + threadIdx.x;
        if ((tid & 31) == 0) red[tid >> 5] = Partial{tm, ag, mn, mx};
        __syncthreads();
        const int bid = blockIdx.y * gridDim.x + blockIdx.x;
        const int nblk = gridDim.x * gridDim.y;
        if (tid == 0) {
            double a = -1.0; long long b = N; int c1 = ny, d1 = -1;
            for (int w = 0; w < 8; ++w)
                partial_take(a, b, c1, d1, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
            if (p.ref_out) p.ref_out[bid] = Partial{a, b, c1, d1};
            else p.scratch[bid] = Partial{a, b, c1, d1};
        }
        if (p.ref_out) return;
        __threadfence();
        __syncthreads();
        if (tid == 0) s_last = (atomicAdd(p.counter, 1u) == (unsigned)nblk - 1) ? 1u : 0u;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        double a = -1.0; long long b = N; int c1 = ny, d1 = -1;
        for (int i = tid; i < nblk; i += 256) {
            const Partial* q = &p.scratch[i];
            partial_take(a, b, c1, d1, __ldcg(&q->tmax), __ldcg(&q->arg), __ldcg(&q->ymin),
                         __ldcg(&q->ymax));
        }
        partial_warp_reduce(a, b, c1, d1);
        __syncthreads();
        if ((tid & 31) == 0) red[tid >> 5] = Partial{a, b, c1, d1};
        __syncthreads();
        if (tid == 0) {
            double a2 = -1.0; long long b2 = N; int c2 = ny, d2 = -1;
            for (int w = 0; w < 8; ++w)
                partial_take(a2, b2, c2, d2, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
            p.ring[0] = Partial{a2, b2, c2, d2};
            *p.counter = 0u;
        }
    }
}

cudaError_t launch_ext_step(const double* Tin, double* Tout, const StepConst& k, int bc,
                            double T_edge, double Tm, Partial* ring, Workspace* ws,
                            Partial* ref_out, long long ref_nparts, cudaStream_t stream) {
    ExtParams p{};
    p.k = k; p.bc = bc; p.T_edge = T_edge; p.Tm = Tm;
    p.ring = ring; p.ref_out = ref_out; p.ref_nparts = ref_nparts;
    const dim3 blk(16, 16);
    const dim3 grd((k.nx + 15) / 16, (k.ny + 15) / 16);
    const bool reduce = ring || ref_out;
    if (reduce && !ref_out) {
        if (!ws) return cudaErrorInvalidValue;
        if ((long long)grd.x * grd.y > (long long)MAX_CTAS * KMAX) {
            // more blocks than partial slots: step, then reduce rows separately
            ext_step_kernel<false><<<grd, blk, 0, stream>>>(Tin, Tout, p);
            const int nb = std::min(MAX_CTAS * KMAX, k.ny);
            reduce_rows_kernel<<<nb, 256, 0, stream>>>(Tout, k.nx, k.ny, Tm, ws->parts);
            return launch_finalize(ws->parts, nb, k.nx, k.ny, ring, stream);
        }
        p.scratch = ws->parts;
        p.counter = &ws->counter;
    }
    if (reduce) ext_step_kernel<true><<<grd, blk, 0, stream>>>(Tin, Tout, p);
    else        ext_step_kernel<false><<<grd, blk, 0, stream>>>(Tin, Tout, p);
    return cudaGetLastError();
}

// ---- standalone reduce --------------------------------------------------------
// Block b takes rows b, b + nblocks, ...; threads stride over the columns, so
// each thread meets its cells in increasing index order.
__global__ void __launch_bounds__(256)
reduce_rows_kernel(const double* __restrict__ T, int nx, int ny, double Tm,
                   Partial* __restrict__ out) {
    const long long N = (long long)nx * ny;
    double tm = -1.0; long long ag = N; int mn = ny, mx = -1;
    for (int y = blockIdx.x; y < ny; y += gridDim.x) {
        const double* row = T + (size_t)y * nx;
        bool molten = false;
        for (int x = threadIdx.x; x < nx; x += blockDim.x) {
            const double v = __ldg(row + x);
            if (v > tm) { tm = v; ag = (long long)y * nx + x; }
            molten |= (v > Tm);
        }
        if (molten) { mn = min(mn, y); mx = max(mx, y); }
    }
    partial_warp_reduce(tm, ag, mn, mx);
    __shared__ Partial red[8];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = Partial{tm, ag, mn, mx};
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = -1.0; long long b = N; int c = ny, d = -1;
        for (int w = 0; w < (int)(blockDim.x >> 5); ++w)
            partial_take(a, b, c, d, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
        out[blockIdx.x] = Partial{a, b, c, d};
    }
}

// ---- finalize: one cluster of FIN_CTAS CTAs ----------------------------------

__global__ void finalize_cluster_kernel(const Partial* __restrict__ parts, int nblocks, int nx, int ny,
                        Partial* __restrict__ out) {
    cg::cluster_group cluster = cg::this_cluster();
    __shared__ Partial red[FIN_THREADS / 32];
    __shared__ Partial cta_result;
    const long long N = (long long)nx * ny;
    double tm = -1.0; long long ag = N; int mn = ny, mx = -1;
    const int rank = (int)cluster.block_rank();
    for (int i = rank * FIN_THREADS + threadIdx.x; i < nblocks; i += FIN_CTAS * FIN_THREADS) {
        const Partial q = parts[i];
        partial_take(tm, ag, mn, mx, q.tmax, q.arg, q.ymin, q.ymax);
    }
    partial_warp_reduce(tm, ag, mn, mx);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = Partial{tm, ag, mn, mx};
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = -1.0; long long b = N; int c = ny, d = -1;
        for (int w = 0; w < FIN_THREADS / 32; ++w)
            partial_take(a, b, c, d, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
        cta_result = Partial{a, b, c, d};
    }
    cluster.sync();
    if (rank == 0 && threadIdx.x == 0) {
        double a = -1.0; long long b = N; int c = ny, d = -1;
        for (int r = 0; r < FIN_CTAS; ++r) {
            const Partial* q = cluster.map_shared_rank(&cta_result, r);
            partial_take(a, b, c, d, q->tmax, q->arg, q->ymin, q->ymax);
        }
        out[0] = Partial{a, b, c, d};
    }
    cluster.sync();   // keep every CTA's shared memory alive until rank 0 has read it
}

__global__ void extract_col_kernel(const double* __restrict__ T, int nx, int ny,
                                   const Partial* __restrict__ glob, double* __restrict__ col) {
    const int y = blockIdx.x * blockDim.x + threadIdx.x;
    if (y >= ny) return;
    const long long a = glob->arg;
    const int x = (int)(a % nx);
    col[y] = (a >= 0 && a < (long long)nx * ny) ? T[(size_t)y * nx + x] : 0.0;
}

}  // namespace lpbf_b200

using namespace lpbf_b200;

extern "C" {

void lpbf_launch_step(const double* Tin, double* Tout, const StepConst* k, int phys,
                      cudaStream_t stream) {
    if (phys == 0) {
        const Coef c = make_coef(*k, 0, 0.0, 0.0);
        const LaserSub las = make_laser(*k, k->x_l, k->y_l, k->q_scale);
        launch_advance(1, Tin, Tout, c, &las, nullptr, nullptr, nullptr, 0, 0, stream);
    } else {
        launch_ext_step(Tin, Tout, *k, 0, 0.0, 0.0, nullptr, nullptr, nullptr, 0, stream);
    }
}

void lpbf_launch_reduce(const double* T, int nx, int ny, double Tm, Partial* out,
                        int nblocks, cudaStream_t stream) {
    if (nblocks <= 0) return;
    reduce_rows_kernel<<<nblocks, 256, 0, stream>>>(T, nx, ny, Tm, out);
}

void lpbf_launch_step_reduce(const double* Tin, double* Tout, const StepConst* k, int phys,
                             double Tm, Partial* out, cudaStream_t stream) {
    const long long nparts = (long long)((k->nx + 15) / 16) * ((k->ny + 15) / 16);
    if (phys == 0) {
        const Coef c = make_coef(*k, 0, 0.0, Tm);
        const LaserSub las = make_laser(*k, k->x_l, k->y_l, k->q_scale);
        launch_advance(1, Tin, Tout, c, &las, nullptr, nullptr, out, nparts, 0, stream);
    } else {
        launch_ext_step(Tin, Tout, *k, 0, 0.0, Tm, nullptr, nullptr, out, nparts, stream);
    }
}

void lpbf_launch_reduce_finalize(const Partial* parts, int nblocks, int nx, int ny,
                                 Partial* out, cudaStream_t stream) {
    launch_finalize(parts, nblocks, nx, ny, out, stream);
}

void lpbf_launch_extract_col(const double* T, int nx, int ny, const Partial* glob,
                             double* out_col, cudaStream_t stream) {
    const int bs = 128;
    extract_col_kernel<<<(ny + bs - 1) / bs, bs, 0, stream>>>(T, nx, ny, glob, out_col);
}

}  // extern "C"
