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
#include <cstring>
#include <cooperative_groups.h>

#include "lpbf_host.hpp"
#include "lpbf_kernels.hpp"

namespace cg = cooperative_groups;

namespace lpbf_b200 {

// ---- extended physics (temperature-dependent IN718 properties) ------------
// Mills tables, include/params.hpp:67-73 (physical data, identical values).
constexpr double EXT_T_PTS[9]  = {298, 473, 673, 873, 1073, 1273, 1473, 1533, 1609};
constexpr double EXT_K_PTS[9]  = {8.9, 12.9, 15.8, 18.7, 21.9, 25.6, 28.6, 29.3, 29.6};
constexpr double EXT_CP_PTS[9] = {435, 479, 515, 558, 580, 628, 670, 685, 720};
constexpr double T_SOL = 1533.0, T_LIQ = 1609.0, LATENT = 210.0e3;
constexpr double INV_MUSHY = 1.0 / (T_LIQ - T_SOL);

// The clamped piecewise-linear tables of params.hpp:75-89 as ten straight
// lines y = a + b T, one per temperature segment: segment 0 (T <= 298) and 9
// (T > 1609) hold the clamped end values, segment j the chord between table
// points j-1 and j.  The reference evaluates the same chord as
// y[j-1] + (T - t[j-1]) / (t[j] - t[j-1]) (y[j] - y[j-1]); the line form
// agrees with it to a few ulp of y.  A cell's segment is the number of table
// temperatures below T, decided on a 32-bit key of T (ext_key): for T >= 0
// the key is twice the upper word of T's bit pattern plus one when the lower
// word is non-zero, and every table temperature (an integer of at most 11
// significant bits) has a zero lower word, so T > t_j exactly when
// key(T) > key(t_j); a negative T gets key 0, segment 0, like the
// reference's clamp, and a NaN the top segment.  The key's upper 16 bits
// (exponent and 5 mantissa bits) cut [256, 2048) K into 96 buckets of
// 8-32 K, none holding more than one table temperature (the closest two are
// 60 K apart): a bucket's base segment (table temperatures below it) plus
// one compare against the next table temperature gives the segment.
constexpr int EXT_BUCKET0 = 0x407 << 5;   // upper 16 key bits of 256.0
constexpr int EXT_BUCKETS = 96;           // up to 2048.0
struct ExtLines {
    double ak[10], bk[10], ac[10], bc[10];
    unsigned int tkey[10];             // keys of the table temperatures; [9] = no bound
    unsigned int sol_key, liq_key;     // of T_SOL and T_LIQ
    unsigned char bseg[EXT_BUCKETS];   // base segment of each bucket
};
static_assert(sizeof(ExtLines) % sizeof(double) == 0, "copied to shared memory as doubles");

inline unsigned int host_key(double v) {
    unsigned long long b;
    std::memcpy(&b, &v, sizeof(b));
    return (unsigned int)((b >> 32) << 1) | (unsigned int)((b & 0xffffffffull) != 0);
}

ExtLines make_ext_lines() {
    ExtLines L;
    L.ak[0] = EXT_K_PTS[0];  L.bk[0] = 0.0;
    L.ac[0] = EXT_CP_PTS[0]; L.bc[0] = 0.0;
    for (int j = 1; j < 9; ++j) {
        const double w = EXT_T_PTS[j] - EXT_T_PTS[j - 1];
        L.bk[j] = (EXT_K_PTS[j] - EXT_K_PTS[j - 1]) / w;
        L.ak[j] = EXT_K_PTS[j - 1] - L.bk[j] * EXT_T_PTS[j - 1];
        L.bc[j] = (EXT_CP_PTS[j] - EXT_CP_PTS[j - 1]) / w;
        L.ac[j] = EXT_CP_PTS[j - 1] - L.bc[j] * EXT_T_PTS[j - 1];
    }
    L.ak[9] = EXT_K_PTS[8];  L.bk[9] = 0.0;
    L.ac[9] = EXT_CP_PTS[8]; L.bc[9] = 0.0;
    for (int j = 0; j < 9; ++j) L.tkey[j] = host_key(EXT_T_PTS[j]);
    L.tkey[9] = 0xffffffffu;
    L.sol_key = host_key(T_SOL);
    L.liq_key = host_key(T_LIQ);
    for (int b = 0; b < EXT_BUCKETS; ++b) {
        // the bucket's lowest value: upper word (EXT_BUCKET0 + b) << 15
        const unsigned long long bits = (unsigned long long)(unsigned)(EXT_BUCKET0 + b) << 47;
        double lo;
        std::memcpy(&lo, &bits, sizeof(lo));
        int base = 0;
        while (base < 9 && EXT_T_PTS[base] < lo) ++base;
        L.bseg[b] = (unsigned char)base;
    }
    return L;
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

constexpr int EXT_WARPS = 8;       // warps per CTA
constexpr int EXT_V = 2;           // columns per lane
constexpr int EXT_OWN = 32 * EXT_V - 2;   // columns a warp owns (the first and last are halo)
constexpr int EXT_H = 64;          // rows per task
constexpr int EXT_PF = 8;          // rows loaded ahead of the one being updated

struct ExtParams {
    StepConst k;
    ExtLines L;
    double hx, hy;                 // inv_dx2 / 2, inv_dy2 / 2 (face averages folded in)
    double r_dsub, Ta4, esig;      // 1/dSub, Tamb^4, eps sigma (0 without radiation)
    double dt_rho;                 // dt / rho
    double r2_cut;                 // beyond this r^2 the source is below 2^-80 of its peak
    int band_lo, band_hi, bandx_lo, bandx_hi;   // cells the source can reach
    int nstrips, ntasks;
    int bc;
    double T_edge, Tm;
    Partial* ring;
    Partial* scratch;
    unsigned int* counter;
    Partial* ref_out;
    long long ref_nparts;
};

// 1/d for the positive, normal d = cp_eff(T) (435..3200): the hardware's
// approximate FP64 reciprocal refined by two Newton-Raphson steps,
// r <- r + r (1 - d r), each of which squares the relative error.
__device__ __forceinline__ double rcp_newton(double d) {
    double r;
    asm("rcp.approx.ftz.f64 %0, %1;" : "=d"(r) : "d"(d));
    double e = fma(-d, r, 1.0);
    r = fma(r, e, r);
    e = fma(-d, r, 1.0);
    return fma(r, e, r);
}

// The laser's heat input q_in at cell (x, y) (kernels.cu:141 order), zero
// where r^2 >= r2_cut (below 2^-80 of the peak).  Out of line: the exp code
// exists once in the binary and holds no registers in the row loop.
static __device__ __noinline__ double ext_source(int x, int y, const StepConst& k,
                                                 double r2_cut) {
    const double xd = __dsub_rn(__dmul_rn((double)x, k.dx), k.x_l);
    const double yd = __dsub_rn(__dmul_rn((double)y, k.dy), k.y_l);
    const double r2 = __dadd_rn(__dmul_rn(xd, xd), __dmul_rn(yd, yd));
    if (r2 >= r2_cut) return 0.0;
    return k.q_scale * k.peak_S * exp(__dmul_rn(-2.0 * r2, k.inv_r0_sq));
}

// The ordering key of T (see ExtLines).
__device__ __forceinline__ unsigned int ext_key(double T) {
    const unsigned int hi = (unsigned int)__double2hiint(T);
    const unsigned int lo = (unsigned int)__double2loint(T);
    const unsigned int k = (hi << 1) | (lo != 0u ? 1u : 0u);
    return (int)hi < 0 ? 0u : k;
}

// Segment of a key in the tables (bucket base plus one compare; see
// ExtLines), from the shared-memory copy of the tables.
__device__ __forceinline__ int ext_seg(unsigned int key, const ExtLines& L) {
    const int b = (int)(key >> 16) - EXT_BUCKET0;
    const int base = L.bseg[min(max(b, 0), EXT_BUCKETS - 1)];
    const int s = base + (key > L.tkey[base] ? 1 : 0);
    return b < 0 ? 0 : (b >= EXT_BUCKETS ? 9 : s);
}

// k_eff(T) = k_of(T) k_enh(T, kmult) (params.hpp:91-105); kp = k_of(T).
// L: the line tables in shared memory (indexed per lane); Lp: the same
// in the parameter space (uniform reads).
template <bool KM>
__device__ __forceinline__ double ext_keff(double T, unsigned int key, int s, const ExtLines& L,
                                           const ExtLines& Lp, double kmult, double& kp) {
    kp = fma(L.bk[s], T, L.ak[s]);
    if constexpr (!KM) {
        return kp;
    } else {
        const double f = (key <= Lp.sol_key) ? 0.0
                       : (key >= Lp.liq_key) ? 1.0 : (T - T_SOL) * INV_MUSHY;
        return kp * fma(kmult - 1.0, f, 1.0);
    }
}

// A cell as the row stream carries it: T, k_eff(T), k_of(T) (the substrate
// loss uses the conductivity without kmult), its ordering key and segment.
struct ExtCell { double T, k, kp; unsigned int key; int seg; };

template <bool KM>
__device__ __forceinline__ ExtCell ext_cell(double T, const ExtLines& L, const ExtLines& Lp,
                                            double kmult) {
    ExtCell c;
    c.T = T;
    c.key = ext_key(T);
    c.seg = ext_seg(c.key, L);
    c.k = ext_keff<KM>(T, c.key, c.seg, L, Lp, kmult, c.kp);
    return c;
}

// Flux through the face between cells a and b, (k_a + k_b)(T_b - T_a) (twice
// the arithmetic-mean face conductivity times the difference; the 1/2 is in
// hx, hy).
__device__ __forceinline__ double ext_flux(const ExtCell& a, const ExtCell& b) {
    return __dmul_rn(__dadd_rn(a.k, b.k), __dsub_rn(b.T, a.T));
}

// The new temperature of cell c from div(k grad T) and the source:
// T + dt (div + (q_in - q_top - q_bot) / h) / (rho cp_eff(T)).
__device__ __forceinline__ double ext_update(const ExtCell& c, double div, double q_in,
                                             const StepConst& k, const ExtParams& p,
                                             const ExtLines& L) {
    const double T = c.T;
    const double T2 = __dmul_rn(T, T);
    const double q_top = fma(p.esig, fma(T2, T2, -p.Ta4), k.hConv * (T - k.Tamb));
    const double q_bot = __dmul_rn(c.kp * p.r_dsub, T - k.Tsub);
    const double rhs = fma(q_in - (q_top + q_bot), k.inv_h, div);
    double cp = fma(L.bc[c.seg], T, L.ac[c.seg]);
    if (c.key >= p.L.sol_key && c.key <= p.L.liq_key) cp += LATENT * INV_MUSHY;
    return fma(__dmul_rn(rhs, p.dt_rho), rcp_newton(cp), T);
}

// One warp advances one (strip, chunk) task: 62 owned columns (lane l holds
// the two columns xs + 2l and xs + 2l + 1; lane 0's first and lane 31's
// second are the neighbours either side) down H rows.  Each cell's T and
// k_eff are loaded and evaluated once, when its row enters; a face's flux
// (k_a + k_b)(T_b - T_a) is computed once, inside the lane, by the lane to
// its left (passed on by a shuffle) or by the cell above it (y faces,
// carried to the next row in registers).  Loads of the
// cells just outside the field are clamped to the edge cell, which makes the
// edge faces' flux exactly zero: the reference's mirror ghost (ghost =
// centre).  The cell arithmetic follows include/step_task.hpp:144-184 and
// src/gpu/kernels.cu:125-147: div(k grad T) on arithmetic-mean faces, the
// source, convection, radiation and substrate losses, and the update
// T + dt rhs / (rho cp_eff(T)) with 1/cp_eff by rcp_newton.  Partials as in
// the baseline kernel: per lane over its owned cells, then warps, CTAs and
// the last CTA.
template <bool REDUCE, bool KM>
__global__ void __launch_bounds__(EXT_WARPS * 32, 2)
ext_step_kernel(const double* __restrict__ Tin, double* __restrict__ Tout,
                const __grid_constant__ ExtParams p) {
    const StepConst& k = p.k;
    __shared__ ExtLines L;
    __shared__ Partial red[EXT_WARPS];
    __shared__ unsigned int s_last;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    if (threadIdx.x < (int)(sizeof(ExtLines) / sizeof(double)))
        reinterpret_cast<double*>(&L)[threadIdx.x] =
            reinterpret_cast<const double*>(&p.L)[threadIdx.x];
    __syncthreads();
    const int nx = k.nx, ny = k.ny;
    const long long N = (long long)nx * ny;
    const double kmult = k.kmult;

    double tm = -1.0;
    long long ag = N;
    int mn = ny, mx = -1;
    for (int task = blockIdx.x * EXT_WARPS + wid; task < p.ntasks;
         task += gridDim.x * EXT_WARPS) {
        const int strip = task % p.nstrips, chunk = task / p.nstrips;
        // lane l holds columns xa = xs + 2l and xb = xa + 1; the warp owns
        // xs + 1 .. xs + EXT_OWN (lane 0's a and lane 31's b are its halo)
        const int xs = strip * EXT_OWN - 1;
        const int xa = xs + EXT_V * lane, xb = xa + 1;
        const int ca = min(max(xa, 0), nx - 1), cb = min(max(xb, 0), nx - 1);
        const bool own_a = lane >= 1 && xa < nx;
        const bool own_b = lane <= 30 && xb < nx;
        const int y0 = chunk * EXT_H, y1 = min(y0 + EXT_H, ny);
        const bool src_strip = !(xs + 1 + EXT_OWN <= p.bandx_lo || xs + 1 > p.bandx_hi);
        // rows y0 - 1 (up) and y0 (centre), clamped at the field's edges
        ExtCell ua, ub, a, b;
        {
            const size_t ru = (size_t)max(y0 - 1, 0) * nx, rc = (size_t)y0 * nx;
            ua = ext_cell<KM>(__ldg(Tin + ru + ca), L, p.L, kmult);
            ub = ext_cell<KM>(__ldg(Tin + ru + cb), L, p.L, kmult);
            a = ext_cell<KM>(__ldg(Tin + rc + ca), L, p.L, kmult);
            b = ext_cell<KM>(__ldg(Tin + rc + cb), L, p.L, kmult);
        }
        double Fua = ext_flux(ua, a), Fub = ext_flux(ub, b);
        // the next EXT_PF rows in flight (a global load's latency spans
        // several rows' arithmetic)
        double Qa[EXT_PF], Qb[EXT_PF];
#pragma unroll
        for (int i = 0; i < EXT_PF; ++i) {
            const size_t r = (size_t)min(y0 + 1 + i, ny - 1) * nx;
            Qa[i] = __ldg(Tin + r + ca);
            Qb[i] = __ldg(Tin + r + cb);
        }
#pragma unroll EXT_PF
        for (int y = y0; y < y1; ++y) {
            const double Tda = Qa[0], Tdb = Qb[0];
#pragma unroll
            for (int i = 0; i < EXT_PF - 1; ++i) { Qa[i] = Qa[i + 1]; Qb[i] = Qb[i + 1]; }
            // row y + EXT_PF + 1 is the lower neighbour of the task's row
            // y + EXT_PF: needed while that row is < y1
            if (y + EXT_PF < y1) {
                const size_t r = (size_t)min(y + EXT_PF + 1, ny - 1) * nx;
                Qa[EXT_PF - 1] = __ldg(Tin + r + ca);
                Qb[EXT_PF - 1] = __ldg(Tin + r + cb);
            }
            const ExtCell da = ext_cell<KM>(Tda, L, p.L, kmult);
            const ExtCell db = ext_cell<KM>(Tdb, L, p.L, kmult);
            // x faces: a|b inside the lane, b|next lane's a, and the previous
            // lane's b|a as this lane's left face; y faces: down, carried up
            const double Fab = ext_flux(a, b);
            const double TR = __shfl_down_sync(0xffffffffu, a.T, 1);
            const double kR = __shfl_down_sync(0xffffffffu, a.k, 1);
            const double FbR = __dmul_rn(__dadd_rn(b.k, kR), __dsub_rn(TR, b.T));
            const double FLa = __shfl_up_sync(0xffffffffu, FbR, 1);
            const double Fda = ext_flux(a, da), Fdb = ext_flux(b, db);
            const double diva = fma(__dsub_rn(Fda, Fua), p.hy, __dmul_rn(__dsub_rn(Fab, FLa), p.hx));
            const double divb = fma(__dsub_rn(Fdb, Fub), p.hy, __dmul_rn(__dsub_rn(FbR, Fab), p.hx));
            double qa = 0.0, qb = 0.0;
            if (src_strip && y >= p.band_lo && y <= p.band_hi && k.q_scale != 0.0) {
                qa = ext_source(xa, y, k, p.r2_cut);
                qb = ext_source(xb, y, k, p.r2_cut);
            }
            double va = ext_update(a, diva, qa, k, p, L);
            double vb = ext_update(b, divb, qb, k, p, L);
            if (p.bc == 1) {
                const bool ey = y == 0 || y == ny - 1;
                if (ey || xa == 0 || xa == nx - 1) va = p.T_edge;
                if (ey || xb == 0 || xb == nx - 1) vb = p.T_edge;
            }
            double* row = Tout + (size_t)y * nx;
            if (own_a) row[xa] = va;
            if (own_b) row[xb] = vb;
            if constexpr (REDUCE) {
                // a lane meets its cells in increasing index order (rows
                // down, a before b): strict '>' keeps the first maximum; NaN
                // never wins
                if (own_a && va > tm) { tm = va; ag = (long long)y * nx + xa; }
                if (own_b && vb > tm) { tm = vb; ag = (long long)y * nx + xb; }
                if (__any_sync(0xffffffffu, (own_a && va > p.Tm) || (own_b && vb > p.Tm)) &&
                    lane == 0) {
                    mn = min(mn, y);
                    mx = max(mx, y);
                }
            }
            // shift the rows
            Fua = Fda; Fub = Fdb;
            a = da; b = db;
        }
    }
    if constexpr (REDUCE) {
        mn = __shfl_sync(0xffffffffu, mn, 0);
        mx = __shfl_sync(0xffffffffu, mx, 0);
        partial_warp_reduce(tm, ag, mn, mx);
        if (lane == 0) red[wid] = Partial{tm, ag, mn, mx};
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = -1.0; long long b = N; int c1 = ny, d1 = -1;
            for (int w = 0; w < EXT_WARPS; ++w)
                partial_take(a, b, c1, d1, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
            if (p.ref_out) p.ref_out[blockIdx.x] = Partial{a, b, c1, d1};
            else p.scratch[blockIdx.x] = Partial{a, b, c1, d1};
        }
        if (p.ref_out) {
            // the rest of the caller's entries: the neutral element
            const Partial neutral{-1.0, N, ny, -1};
            for (long long i = gridDim.x + blockIdx.x * (long long)blockDim.x + threadIdx.x;
                 i < p.ref_nparts; i += (long long)gridDim.x * blockDim.x)
                p.ref_out[i] = neutral;
            return;
        }
        __threadfence();
        __syncthreads();
        if (threadIdx.x == 0)
            s_last = (atomicAdd(p.counter, 1u) == gridDim.x - 1) ? 1u : 0u;
        __syncthreads();
        if (!s_last) return;
        __threadfence();
        double a = -1.0; long long b = N; int c1 = ny, d1 = -1;
        for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
            const Partial* qq = &p.scratch[i];
            partial_take(a, b, c1, d1, __ldcg(&qq->tmax), __ldcg(&qq->arg), __ldcg(&qq->ymin),
                         __ldcg(&qq->ymax));
        }
        partial_warp_reduce(a, b, c1, d1);
        __syncthreads();
        if (lane == 0) red[wid] = Partial{a, b, c1, d1};
        __syncthreads();
        if (threadIdx.x == 0) {
            double a2 = -1.0; long long b2 = N; int c2 = ny, d2 = -1;
            for (int w = 0; w < EXT_WARPS; ++w)
                partial_take(a2, b2, c2, d2, red[w].tmax, red[w].arg, red[w].ymin, red[w].ymax);
            p.ring[0] = Partial{a2, b2, c2, d2};
            *p.counter = 0u;
        }
    }
}

template <bool REDUCE>
cudaError_t launch_ext_t(bool km, int grid, const double* Tin, double* Tout, const ExtParams& p,
                         cudaStream_t stream) {
    if (km) ext_step_kernel<REDUCE, true><<<grid, EXT_WARPS * 32, 0, stream>>>(Tin, Tout, p);
    else ext_step_kernel<REDUCE, false><<<grid, EXT_WARPS * 32, 0, stream>>>(Tin, Tout, p);
    return cudaGetLastError();
}

cudaError_t launch_ext_step(const double* Tin, double* Tout, const StepConst& k, int bc,
                            double T_edge, double Tm, Partial* ring, Workspace* ws,
                            Partial* ref_out, long long ref_nparts, cudaStream_t stream) {
    static const ExtLines lines = make_ext_lines();
    ExtParams p;
    std::memset(&p, 0, sizeof(p));
    p.k = k; p.L = lines;
    p.hx = 0.5 * k.inv_dx2;
    p.hy = 0.5 * k.inv_dy2;
    p.r_dsub = 1.0 / k.dSub;
    p.Ta4 = k.Tamb * k.Tamb * k.Tamb * k.Tamb;
    p.esig = k.radiation ? k.eps * SIGMA_SB : 0.0;
    p.dt_rho = k.dt / k.rho;
    p.bc = bc; p.T_edge = T_edge; p.Tm = Tm;
    p.ring = ring; p.ref_out = ref_out; p.ref_nparts = ref_nparts;
    // the source's reach: rows and columns where r^2 < r2_cut (a superset)
    const Coef c = make_coef(k, bc, T_edge, Tm);
    const LaserSub las = make_laser(k, k.x_l, k.y_l, k.q_scale);
    p.r2_cut = c.r2_cut;
    laser_band(c, &las, 1, &p.band_lo, &p.band_hi, &p.bandx_lo, &p.bandx_hi);
    p.nstrips = (k.nx + EXT_OWN - 1) / EXT_OWN;
    p.ntasks = p.nstrips * ((k.ny + EXT_H - 1) / EXT_H);
    int grid = (p.ntasks + EXT_WARPS - 1) / EXT_WARPS;
    const bool km = k.kmult > 1.0;
    const bool reduce = ring || ref_out;
    if (ref_out) {
        grid = (int)std::max<long long>(1, std::min<long long>(grid, ref_nparts));
        return launch_ext_t<true>(km, grid, Tin, Tout, p, stream);
    }
    if (reduce) {
        if (!ws) return cudaErrorInvalidValue;
        grid = std::min(grid, MAX_CTAS * KMAX);
        p.scratch = ws->parts;
        p.counter = &ws->counter;
        return launch_ext_t<true>(km, grid, Tin, Tout, p, stream);
    }
    return launch_ext_t<false>(km, grid, Tin, Tout, p, stream);
}

// ---- standalone reduce --------------------------------------------------------
// Block b takes rows b, b + nblocks, ... (the reference's API fixes the grid
// at nblocks Partials, 256 for large fields: under two CTAs per SM), so each
// CTA keeps many bytes in flight: 1024 threads, each loading RR_VEC
// independent 16-byte pairs of a row before examining them.  A thread meets
// its cells in increasing index order (pairs in order, then the next group
// of pairs, then the next row), so a strict '>' keeps its first maximal
// cell; the block's threads then combine by the same rule as every Partial.
constexpr int RR_THREADS = 1024;
constexpr int RR_VEC = 4;

__device__ __forceinline__ void rr_take(double v, long long i, double& tm, long long& ag,
                                        bool& molten, double Tm) {
    if (v > tm) { tm = v; ag = i; }
    molten |= (v > Tm);
}

__global__ void __launch_bounds__(RR_THREADS)
reduce_rows_kernel(const double* __restrict__ T, int nx, int ny, double Tm,
                   Partial* __restrict__ out) {
    const long long N = (long long)nx * ny;
    double tm = -1.0; long long ag = N; int mn = ny, mx = -1;
    // 16-byte pairs when every row starts on a 16-byte boundary
    const bool pairs = (nx % 2 == 0) && (reinterpret_cast<uintptr_t>(T) % 16 == 0);
    for (int y = blockIdx.x; y < ny; y += gridDim.x) {
        const double* row = T + (size_t)y * nx;
        const long long base = (long long)y * nx;
        bool molten = false;
        if (pairs) {
            const double2* r2 = reinterpret_cast<const double2*>(row);
            const int np = nx / 2;
            for (int p0 = threadIdx.x; p0 < np; p0 += RR_THREADS * RR_VEC) {
                double2 v[RR_VEC];
#pragma unroll
                for (int u = 0; u < RR_VEC; ++u) {
                    const int p = p0 + u * RR_THREADS;
                    v[u] = p < np ? __ldg(r2 + p) : make_double2(-INFINITY, -INFINITY);
                }
#pragma unroll
                for (int u = 0; u < RR_VEC; ++u) {
                    const long long i = base + 2ll * (p0 + u * RR_THREADS);
                    rr_take(v[u].x, i, tm, ag, molten, Tm);
                    rr_take(v[u].y, i + 1, tm, ag, molten, Tm);
                }
            }
        } else {
            for (int x0 = threadIdx.x; x0 < nx; x0 += RR_THREADS * RR_VEC) {
                double v[RR_VEC];
#pragma unroll
                for (int u = 0; u < RR_VEC; ++u) {
                    const int x = x0 + u * RR_THREADS;
                    v[u] = x < nx ? __ldg(row + x) : -INFINITY;
                }
#pragma unroll
                for (int u = 0; u < RR_VEC; ++u)
                    rr_take(v[u], base + x0 + u * RR_THREADS, tm, ag, molten, Tm);
            }
        }
        if (molten) { mn = min(mn, y); mx = max(mx, y); }
    }
    partial_warp_reduce(tm, ag, mn, mx);
    __shared__ Partial red[RR_THREADS / 32];
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = Partial{tm, ag, mn, mx};
    __syncthreads();
    if (threadIdx.x < 32) {
        Partial q = red[threadIdx.x];
        double a = q.tmax; long long b = q.arg; int c = q.ymin, d = q.ymax;
        partial_warp_reduce(a, b, c, d);
        if (threadIdx.x == 0) out[blockIdx.x] = Partial{a, b, c, d};
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
    reduce_rows_kernel<<<nblocks, RR_THREADS, 0, stream>>>(T, nx, ny, Tm, out);
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
