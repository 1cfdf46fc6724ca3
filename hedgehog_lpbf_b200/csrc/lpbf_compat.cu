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
constexpr double INV_MUSHY = 1.0 / (T_LIQ - T_SOL);

// The tables in shared memory (lanes index them divergently): temperatures,
// k, cp, and the reciprocal segment widths.
struct ExtTab { double t[9], k[9], cp[9], inv[8]; };

// params.hpp:75-89: clamped piecewise-linear lookup.  The segment comes from
// seven compares instead of a search loop, and the segment width's
// reciprocal replaces the division (an ulp-level difference).
__device__ __forceinline__ int ext_seg(const ExtTab& tb, double T) {
    int i = 1;
#pragma unroll
    for (int j = 1; j < 8; ++j) i += (T > tb.t[j]) ? 1 : 0;
    return i;
}
__device__ __forceinline__ double ext_interp(const ExtTab& tb, const double* ys, double T, int i) {
    if (T <= tb.t[0]) return ys[0];
    if (T >= tb.t[8]) return ys[8];
    const double f = (T - tb.t[i - 1]) * tb.inv[i - 1];
    return ys[i - 1] + f * (ys[i] - ys[i - 1]);
}
// k_of(T) * k_enh(T, kmult)  (params.hpp:91-105)
__device__ __forceinline__ double ext_k(const ExtTab& tb, double T, double kmult, double* k_plain) {
    const double k = ext_interp(tb, tb.k, T, ext_seg(tb, T));
    if (k_plain) *k_plain = k;
    if (kmult <= 1.0) return k;
    const double s = (T <= T_SOL) ? 0.0 : (T >= T_LIQ) ? 1.0 : (T - T_SOL) * INV_MUSHY;
    return k * (1.0 + (kmult - 1.0) * s);
}
// cp_of(T) plus the latent heat spread over the mushy range (params.hpp:106-110)
__device__ __forceinline__ double ext_cp(const ExtTab& tb, double T) {
    double c = ext_interp(tb, tb.cp, T, ext_seg(tb, T));
    if (T >= T_SOL && T <= T_LIQ) c += LATENT * INV_MUSHY;
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

// Blocks of 16 x 16 threads over tiles of 16 x EXT_ROWS cells (each thread
// owns EXT_ROWS / 16 cells of one column).  The block stages the tile's T
// plus a one-cell ring (edge neighbours mirrored: the ghost is the centre)
// and the conductivities k_eff(T) of all of them in shared memory, so each
// cell's k_eff is evaluated once and read by its four neighbours.  The cell
// arithmetic follows include/step_task.hpp:144-184, with the divisions by
// dSub and by rho cp_eff(T) done as multiplications by correctly rounded
// reciprocals (ulp-level differences).  For the reference's fused-reduce
// layout (one Partial per 16 x 16 block) a tile writes its result into its
// first 16 x 16 entry and the neutral element into the others.
constexpr int EXT_ROWS = 64;
constexpr int EXT_RPT = EXT_ROWS / 16;          // cells per thread

template <bool REDUCE>
__global__ void __launch_bounds__(256)
ext_step_kernel(const double* __restrict__ Tin, double* __restrict__ Tout,
                const __grid_constant__ ExtParams p) {
    const StepConst& k = p.k;
    __shared__ double sT[EXT_ROWS + 2][18], sK[EXT_ROWS + 2][18];
    __shared__ ExtTab tb;
    const int tid = threadIdx.y * 16 + threadIdx.x;
    const int nx = k.nx, ny = k.ny;
    const long long N = (long long)nx * ny;
    if (tid < 9) {
        tb.t[tid] = c_T_PTS[tid];
        tb.k[tid] = c_K_PTS[tid];
        tb.cp[tid] = c_CP_PTS[tid];
        if (tid < 8) tb.inv[tid] = 1.0 / (c_T_PTS[tid + 1] - c_T_PTS[tid]);
    }
    __syncthreads();
    const int bx = blockIdx.x * 16, by = blockIdx.y * EXT_ROWS;
    for (int e = tid; e < (EXT_ROWS + 2) * 18; e += 256) {
        const int i = e % 18, j = e / 18;
        const int gx = min(max(bx + i - 1, 0), nx - 1);
        const int gy = min(max(by + j - 1, 0), ny - 1);
        const double T = __ldg(Tin + (size_t)gy * nx + gx);
        sT[j][i] = T;
        sK[j][i] = ext_k(tb, T, k.kmult, nullptr);
    }
    __syncthreads();
    const double r_dsub = __drcp_rn(k.dSub);
    const double Ta4 = k.Tamb * k.Tamb * k.Tamb * k.Tamb;
    const int tx = threadIdx.x;
    const int x = bx + tx;
    double tm = -1.0;
    long long ag = N;
    int mn = ny, mx = -1;
#pragma unroll 1
    for (int q = 0; q < EXT_RPT; ++q) {
        const int ty = threadIdx.y + 16 * q;            // rows of a thread step by 16
        const int y = by + ty;
        if (!(x < nx && y < ny)) continue;
        const long long c = (long long)y * nx + x;
        double v;
        if (p.bc == 1 && (x == 0 || y == 0 || x == nx - 1 || y == ny - 1)) {
            v = p.T_edge;
        } else {
            const double T = sT[ty + 1][tx + 1];
            const double Txm = sT[ty + 1][tx], Txp = sT[ty + 1][tx + 2];
            const double Tym = sT[ty][tx + 1], Typ = sT[ty + 2][tx + 1];
            const double kC = sK[ty + 1][tx + 1];
            const double kxm = 0.5 * (kC + sK[ty + 1][tx]);
            const double kxp = 0.5 * (kC + sK[ty + 1][tx + 2]);
            const double kym = 0.5 * (kC + sK[ty][tx + 1]);
            const double kyp = 0.5 * (kC + sK[ty + 2][tx + 1]);
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
                q_top += k.eps * SIGMA_SB * (T4 - Ta4);
            }
            // one table segment for the substrate conductivity (no kmult) and cp
            const int sg = ext_seg(tb, T);
            const double k_plain = k.kmult <= 1.0 ? kC : ext_interp(tb, tb.k, T, sg);
            double cp = ext_interp(tb, tb.cp, T, sg);
            if (T >= T_SOL && T <= T_LIQ) cp += LATENT * INV_MUSHY;
            const double q_bot = (k_plain * r_dsub) * (T - k.Tsub);
            const double rhs = div + (q_in - q_top - q_bot) * k.inv_h;
            v = T + (k.dt * rhs) * __drcp_rn(k.rho * cp);
        }
        Tout[c] = v;
        if constexpr (REDUCE) {
            // rows of this thread come in increasing order: strict '>' keeps
            // the first (smallest-index) maximum; NaN never wins
            if (v > tm) { tm = v; ag = c; }
            if (v > p.Tm) { mn = min(mn, y); mx = max(mx, y); }
        }
    }
    if constexpr (REDUCE) {
        partial_warp_reduce(tm, ag, mn, mx);
        __shared__ Partial red[8];
        __shared__ unsigned int s_last;
        if ((tid & 31) == 0) red[tid >> 5] = Partial{tm, ag, mn, mx};
        __syncthreads();
        const int nblk = gridDim.x * gridDim.y;
        if (tid == 0) {
            double a = -1.0; long long b = N; int c1 = ny, d1 = -1;
            for (int w = 0; w < 8; ++w)
                partial_take(a, b, c1, d1, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
            if (p.ref_out) {
                // reference layout: 16 x 16 blocks, row-major over the grid
                const int gx16 = (nx + 15) / 16, gy16 = (ny + 15) / 16;
                const Partial neutral{-1.0, N, ny, -1};
                for (int q = 0; q < EXT_RPT; ++q) {
                    const int yb = blockIdx.y * EXT_RPT + q;
                    if (yb >= gy16) break;
                    const long long idx = (long long)yb * gx16 + blockIdx.x;
                    if (idx < p.ref_nparts) p.ref_out[idx] = q == 0 ? Partial{a, b, c1, d1} : neutral;
                }
            } else {
                p.scratch[blockIdx.y * gridDim.x + blockIdx.x] = Partial{a, b, c1, d1};
            }
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
            const Partial* qq = &p.scratch[i];
            partial_take(a, b, c1, d1, __ldcg(&qq->tmax), __ldcg(&qq->arg), __ldcg(&qq->ymin),
                         __ldcg(&qq->ymax));
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
    const dim3 grd((k.nx + 15) / 16, (k.ny + EXT_ROWS - 1) / EXT_ROWS);
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
