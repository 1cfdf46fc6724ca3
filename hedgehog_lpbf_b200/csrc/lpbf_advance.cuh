// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// The temporally blocked step kernel.
//
// Work decomposition.  The nx x ny field (row-major f64) is cut into column
// strips of WOUT owned columns and row chunks of H owned rows; one warp owns
// one (strip, chunk) task at a time.  A warp covers COLS = 64*NCH columns,
// i.e. its owned columns plus KH (= K rounded up to even) halo columns on each
// side, so it can advance its strip K time steps with no data from other
// warps: after level t the outermost t halo columns are stale, after K levels
// exactly the owned columns remain valid.
//
// Lane layout.  Lane l holds columns 64q + 2l + {0,1} of chunk q, so every
// row access is a conflict-free 512-byte vector access per chunk, and the x
// neighbours come from the adjacent lane by one warp shuffle each.
//
// Wavefront.  Rows stream top to bottom.  Level-0 rows arrive through a
// per-warp TMA pipeline (S stages of R rows, one mbarrier per stage, no CTA
// barrier anywhere in the stream).  At iteration j the warp loads level-0 row
// j and computes level-t row j-t for t = 1..K, each from the three rows of
// level t-1 held in registers.  Level-t row r lives in register slot r % 3;
// the row loop is unrolled by three so every slot index is a compile-time
// constant and no register is ever moved.  Level K rows are written straight
// to HBM as 16-byte stores.
//
// Reduction.  For every level (= time step) each lane keeps the peak T with
// its flat index and the molten row extent over its owned cells; warps,
// then CTAs combine them, and the last CTA to finish (atomic ticket, no
// waiting) reduces the per-CTA partials into one Partial per time step.
// ---------------------------------------------------------------------------
#pragma once
#include "lpbf_device.cuh"

namespace lpbf_b200 {

constexpr int ADV_WARPS = 4;       // warps per CTA
constexpr int ADV_NCH = 2;         // 64-column chunks per warp (COLS = 128)
constexpr int ADV_R = 4;           // rows per TMA box
constexpr int ADV_S = 4;           // TMA stages per warp

template <int K>
struct AdvGeo {
    static constexpr int KH = (K + 1) & ~1;
    static constexpr int COLS = 64 * ADV_NCH;
    static constexpr int WOUT = COLS - 2 * KH;
    static constexpr int V = 2 * ADV_NCH;
    static constexpr int STAGE_DOUBLES = ADV_R * COLS;
    static constexpr size_t SMEM_BYTES =
        size_t(ADV_WARPS) * ADV_S * STAGE_DOUBLES * sizeof(double)
        + size_t(ADV_WARPS) * ADV_S * sizeof(uint64_t);
};

struct AdvParams {
    Coef c;
    LaserSub las[KMAX];
    int nstrips, nchunks, H, ntasks;
    const double* Tin;             // source field (used by the direct-load path)
    double* Tout;                  // destination field (never aliases Tin)
    Partial* ring;                 // K finalized Partials (one per step), or null
    Partial* scratch;              // per-CTA partials, gridDim.x * K entries
    unsigned int* counter;         // last-CTA ticket, zero between launches
    unsigned int* err;             // error word (bit 0: TMA wait timed out)
    Partial* ref_out;              // reference fused-reduce layout (K == 1), or null
    long long ref_nparts;          // number of entries of ref_out to define
};

__host__ __device__ constexpr int mod3(int a) { return ((a % 3) + 3) % 3; }

// One warp advancing one task (strip, chunk) by K levels.
template <int K, bool TMA, bool REDUCE>
struct WarpStrip {
    using G = AdvGeo<K>;
    static constexpr int V = G::V;

    const AdvParams& p;
    const CUtensorMap* map;
    double* stages;                // this warp's S stages
    uint64_t* bars;                // this warp's S mbarriers
    uint32_t& gbox;                // running box counter of this warp (phase tracking)
    const int lane;

    int x0, xs, y0, y1, jy0, jend, nbox, issued;
    bool edge, failed;
    bool own[V];                   // lane's column is owned and inside the grid

    double w[K > 1 ? K : 1][3][V]; // level windows 0..K-1 (slot = row % 3)
    double tmx[K];
    long long targ[K];
    int ymn[K], ymx[K];

    __device__ WarpStrip(const AdvParams& p_, const CUtensorMap* m, double* st,
                         uint64_t* b, uint32_t& g, int ln)
        : p(p_), map(m), stages(st), bars(b), gbox(g), lane(ln), failed(false) {
        const long long N = (long long)p.c.nx * p.c.ny;
#pragma unroll
        for (int t = 0; t < K; ++t) { tmx[t] = -1.0; targ[t] = N; ymn[t] = p.c.ny; ymx[t] = -1; }
    }

    __device__ __forceinline__ void issue(int b) {
        const uint32_t g = gbox + b;
        const int st = g % ADV_S;
        double* dst = stages + st * G::STAGE_DOUBLES;
        mbar_expect_tx(&bars[st], G::STAGE_DOUBLES * sizeof(double));
        tma_load_2d(dst, map, xs, jy0 + b * ADV_R, &bars[st]);
        issued = b + 1;
    }

    __device__ __forceinline__ void run_task(int task) {
        const int nx = p.c.nx, ny = p.c.ny;
        const int strip = task % p.nstrips, chunk = task / p.nstrips;
        x0 = strip * G::WOUT;
        xs = x0 - G::KH;
        y0 = chunk * p.H;
        y1 = min(y0 + p.H, ny);
        jy0 = max(y0 - K, 0);
        jy0 -= jy0 % 3;
        jend = min(y1 + K, ny);
        nbox = (jend - jy0 + ADV_R - 1) / ADV_R;
        edge = (xs <= 0) || (xs + G::COLS > nx - 1);
#pragma unroll
        for (int v = 0; v < V; ++v) {
            const int x = xs + 64 * (v >> 1) + 2 * lane + (v & 1);
            own[v] = (x >= x0) && (x < x0 + G::WOUT) && (x < nx);
        }
        issued = 0;
        if constexpr (TMA) {
            if (lane == 0) {
                const int pre = min(ADV_S, nbox);
                for (int b = 0; b < pre; ++b) issue(b);
            }
        }
        const int jlast = y1 - 1 + K;
        for (int j = jy0; j <= jlast && !failed; j += 3) {
            row<0>(j);
            if (j + 1 <= jlast) row<1>(j + 1);
            if (j + 2 <= jlast) row<2>(j + 2);
        }
        if constexpr (TMA) {
            if (failed) drain();
            gbox += nbox;
        }
    }

    // After a timed-out wait: give the copies still in flight a bounded
    // chance to land before this warp stops touching its stages.
    __device__ __forceinline__ void drain() {
        const int last = __shfl_sync(0xffffffffu, issued, 0);
        for (int b = max(0, last - ADV_S); b < last; ++b) {
            const uint32_t g = gbox + b;
            mbar_wait_bounded(&bars[g % ADV_S], (g / ADV_S) & 1);
        }
    }

    __device__ __forceinline__ void load_row0(int jj, double* dst) {
        const int nx = p.c.nx;
        if constexpr (TMA) {
            const int rel = jj - jy0;
            const int b = rel / ADV_R, rr = rel % ADV_R;
            const uint32_t g = gbox + b;
            const int st = g % ADV_S;
            if (rr == 0) {
                const bool ok = mbar_wait_bounded(&bars[st], (g / ADV_S) & 1);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(p.err, 1u);
                    failed = true;
                    return;
                }
            }
            const double* src = stages + st * G::STAGE_DOUBLES + rr * G::COLS;
#pragma unroll
            for (int q = 0; q < ADV_NCH; ++q) {
                const double2 v = *reinterpret_cast<const double2*>(src + 64 * q + 2 * lane);
                dst[2 * q] = v.x;
                dst[2 * q + 1] = v.y;
            }
            if (rr == ADV_R - 1 || jj == jend - 1) {
                __syncwarp();
                if (lane == 0 && b + ADV_S < nbox) {
                    // order this warp's reads of the stage before the refill
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    issue(b + ADV_S);
                }
            }
        } else {
            const double* rowp = p.Tin + (size_t)jj * nx;
#pragma unroll
            for (int q = 0; q < ADV_NCH; ++q) {
#pragma unroll
                for (int e = 0; e < 2; ++e) {
                    const int x = xs + 64 * q + 2 * lane + e;
                    dst[2 * q + e] = (x >= 0 && x < nx) ? __ldg(rowp + x) : 0.0;
                }
            }
        }
    }

    template <int P>
    __device__ __forceinline__ void row(int jj) {
        if (jj < jend) {
            load_row0(jj, w[0][P]);
            if (failed) return;
        }
        level<P, 1>(jj);
    }

    template <int P, int T>
    __device__ __forceinline__ void level(int jj) {
        if constexpr (T <= K) {
            constexpr int su = mod3(P - T - 1), sc = mod3(P - T), sd = mod3(P - T + 1);
            const int ny = p.c.ny;
            const int r = jj - T;
            const int lo = max(y0 - K + T, 0);
            const int hi = min(y1 - 1 + K - T, ny - 1);
            if (r >= lo && r <= hi) {
                double (&win)[3][V] = w[T - 1];
                // Mirror edges: the ghost row is the centre row.  The slot of
                // row -1 (row 2) is not filled yet and the slot of row ny
                // (row ny-3) is no longer needed, so both can be overwritten.
                if (r == 0) {
#pragma unroll
                    for (int v = 0; v < V; ++v) win[su][v] = win[sc][v];
                }
                if (r == ny - 1) {
#pragma unroll
                    for (int v = 0; v < V; ++v) win[sd][v] = win[sc][v];
                }
                double nv[V];
                compute_row(win[su], win[sc], win[sd], r, p.las[T - 1], nv);
                if constexpr (T < K) {
#pragma unroll
                    for (int v = 0; v < V; ++v) w[T][sc][v] = nv[v];
                } else {
                    if (r >= y0 && r < y1) store_row(r, nv);
                }
                if constexpr (REDUCE) {
                    if (r >= y0 && r < y1) reduce_row<T - 1>(r, nv);
                }
            }
            level<P, T + 1>(jj);
        }
    }

    __device__ __forceinline__ void compute_row(const double* up, const double* ce,
                                                const double* dn, int r,
                                                const LaserSub& las, double* nv) {
        const Coef& c = p.c;
        const int nx = c.nx, ny = c.ny;
        if (c.bc == 1 && (r == 0 || r == ny - 1)) {
#pragma unroll
            for (int v = 0; v < V; ++v) nv[v] = c.T_edge;
            return;
        }
        // x neighbours across lanes: left of column 2l comes from lane l-1
        // (or chunk q-1's lane 31), right of column 2l+1 from lane l+1.
        double Lq[ADV_NCH], Rq[ADV_NCH];
#pragma unroll
        for (int q = 0; q < ADV_NCH; ++q) {
            const double lc = (q > 0 && lane == 31) ? ce[2 * (q - 1) + 1] : ce[2 * q + 1];
            const double rc = (q < ADV_NCH - 1 && lane == 0) ? ce[2 * (q + 1)] : ce[2 * q];
            Lq[q] = __shfl_sync(0xffffffffu, lc, (lane + 31) & 31);
            Rq[q] = __shfl_sync(0xffffffffu, rc, (lane + 1) & 31);
        }
        double L[V], R[V];
#pragma unroll
        for (int q = 0; q < ADV_NCH; ++q) {
            L[2 * q] = Lq[q];          R[2 * q] = ce[2 * q + 1];
            L[2 * q + 1] = ce[2 * q];  R[2 * q + 1] = Rq[q];
        }
        if (edge) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int x = xs + 64 * (v >> 1) + 2 * lane + (v & 1);
                if (x == 0) L[v] = ce[v];
                if (x == nx - 1) R[v] = ce[v];
            }
        }
        const double yd = __dsub_rn(__dmul_rn((double)r, c.dy), las.y_l);
        const double dy2 = __dmul_rn(yd, yd);
        if (las.cs != 0.0 && dy2 < c.r2_cut) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int x = xs + 64 * (v >> 1) + 2 * lane + (v & 1);
                const double S = source_dt(x, dy2, las, c);
                nv[v] = cell_update(ce[v], L[v], R[v], up[v], dn[v], S, c);
            }
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
                nv[v] = cell_update_nosrc(ce[v], L[v], R[v], up[v], dn[v], c);
        }
        if (edge && c.bc == 1) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int x = xs + 64 * (v >> 1) + 2 * lane + (v & 1);
                if (x == 0 || x == nx - 1) nv[v] = c.T_edge;
            }
        }
    }

    __device__ __forceinline__ void store_row(int r, const double* nv) {
        double* dst = p.Tout + (size_t)r * p.c.nx;
#pragma unroll
        for (int q = 0; q < ADV_NCH; ++q) {
            const int c0 = xs + 64 * q + 2 * lane;
            if constexpr (TMA) {
                // even nx and even c0: both cells of the pair share ownership
                if (own[2 * q])
                    *reinterpret_cast<double2*>(dst + c0) = make_double2(nv[2 * q], nv[2 * q + 1]);
            } else {
                if (own[2 * q]) dst[c0] = nv[2 * q];
                if (own[2 * q + 1]) dst[c0 + 1] = nv[2 * q + 1];
            }
        }
    }

    template <int T>
    __device__ __forceinline__ void reduce_row(int r, const double* nv) {
        // Row maximum over the lane's owned cells; fmax ignores NaN, as the
        // reference's strict '>' does.  Ties resolve to the lowest column.
        double m = -INFINITY;
#pragma unroll
        for (int v = 0; v < V; ++v)
            if (own[v]) m = fmax(m, nv[v]);
        if (m > tmx[T]) {
            int col = -1;
#pragma unroll
            for (int v = V - 1; v >= 0; --v)
                if (own[v] && nv[v] == m) col = xs + 64 * (v >> 1) + 2 * lane + (v & 1);
            tmx[T] = m;
            targ[T] = (long long)r * p.c.nx + col;
        }
        if (m > p.c.Tm) {
            ymn[T] = min(ymn[T], r);
            ymx[T] = max(ymx[T], r);
        }
    }
};

template <int K, bool TMA, bool REDUCE>
__global__ void __launch_bounds__(ADV_WARPS * 32, 3)
advance_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ AdvParams p) {
    using G = AdvGeo<K>;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ Partial red[ADV_WARPS][K];
    __shared__ unsigned int s_last;

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* stages = reinterpret_cast<double*>(smem) + wid * (ADV_S * G::STAGE_DOUBLES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        smem + size_t(ADV_WARPS) * ADV_S * G::STAGE_DOUBLES * sizeof(double)) + wid * ADV_S;

    if constexpr (TMA) {
        if (lane == 0) {
            for (int s = 0; s < ADV_S; ++s) mbar_init(&bars[s], 1);
            fence_mbar_init();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncwarp();
    }

    uint32_t gbox = 0;
    WarpStrip<K, TMA, REDUCE> ws(p, &map, stages, bars, gbox, lane);
    for (int task = blockIdx.x * ADV_WARPS + wid; task < p.ntasks;
         task += gridDim.x * ADV_WARPS) {
        ws.run_task(task);
        if (ws.failed) break;
    }

    if constexpr (REDUCE) {
#pragma unroll
        for (int t = 0; t < K; ++t) {
            partial_warp_reduce(ws.tmx[t], ws.targ[t], ws.ymn[t], ws.ymx[t]);
            if (lane == 0) red[wid][t] = Partial{ws.tmx[t], ws.targ[t], ws.ymn[t], ws.ymx[t]};
        }
        __syncthreads();
        const long long N = (long long)p.c.nx * p.c.ny;
        if (threadIdx.x < K) {
            const int t = threadIdx.x;
            double tm = -1.0; long long ag = N; int mn = p.c.ny, mx = -1;
            for (int w = 0; w < ADV_WARPS; ++w)
                partial_take(tm, ag, mn, mx, red[w][t].tmax, red[w][t].arg,
                             red[w][t].ymin, red[w][t].ymax);
            if (p.ref_out) p.ref_out[blockIdx.x] = Partial{tm, ag, mn, mx};
            else p.scratch[(size_t)blockIdx.x * K + t] = Partial{tm, ag, mn, mx};
        }
        if (p.ref_out) {
            // Reference layout: the caller finalizes ref_nparts entries, so
            // every entry past this grid's must hold the neutral element.
            const Partial neutral{-1.0, N, p.c.ny, -1};
            for (long long i = gridDim.x + (long long)blockIdx.x * blockDim.x + threadIdx.x;
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
        for (int t = 0; t < K; ++t) {
            double tm = -1.0; long long ag = N; int mn = p.c.ny, mx = -1;
            for (int i = threadIdx.x; i < (int)gridDim.x; i += blockDim.x) {
                const Partial* q = &p.scratch[(size_t)i * K + t];
                partial_take(tm, ag, mn, mx, __ldcg(&q->tmax), __ldcg(&q->arg),
                             __ldcg(&q->ymin), __ldcg(&q->ymax));
            }
            partial_warp_reduce(tm, ag, mn, mx);
            __syncthreads();
            if (lane == 0) red[wid][0] = Partial{tm, ag, mn, mx};
            __syncthreads();
            if (threadIdx.x == 0) {
                double a = -1.0; long long b = N; int c1 = p.c.ny, d1 = -1;
                for (int w = 0; w < ADV_WARPS; ++w)
                    partial_take(a, b, c1, d1, red[w][0].tmax, red[w][0].arg,
                                 red[w][0].ymin, red[w][0].ymax);
                p.ring[t] = Partial{a, b, c1, d1};
            }
        }
        if (threadIdx.x == 0) *p.counter = 0u;
    }
}

}  // namespace lpbf_b200
