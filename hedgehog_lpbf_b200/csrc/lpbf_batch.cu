// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Batched process map: many independent fields (scenarios) of uneven sizes,
// laser powers, speeds and scan paths advanced together, K time steps per
// launch, by one persistent kernel that pulls (scenario, strip, chunk) work
// items from a device queue.
//
// The reference runs such an ensemble as a serial loop, one GpuStepTask
// graph per manifest row (src/gpu/hh_gpu_main.cpp:162-270); small grids then
// leave most of the GPU idle.  Here every launch carries the whole batch:
//
//  * Queue.  Tasks are numbered scenario by scenario (largest scenarios
//    first, so the short tasks of small grids fill the tail); a warp draws
//    the next number with one atomic add, finds its scenario by binary search
//    over the per-scenario task offsets, copies that scenario's launch
//    parameters (a few hundred bytes) into its shared-memory slot and runs
//    the same WarpStrip as the single-field kernel.  Rows are staged either
//    by plain bulk copies (cp.async.bulk, one per row) or by tiled tensor-map
//    loads from per-scenario maps in the workspace; bulk copies read no
//    descriptor, which matters with hundreds of fields in flight.  Each
//    scenario's rows per task come from its size class (autotuned).
//  * Per-step results.  A warp carries its lane peaks across consecutive
//    tasks of one field (so its thresholds stay warm); after each task it
//    reduces its K per-step partials and stores them at the task's queue
//    position.  Tasks form
//    groups of 32: the warp that completes a group's last task (atomic
//    ticket, no waiting) folds the group's partials, one per lane, into a
//    group partial; the warp that completes a scenario's last group folds
//    the group partials into one Partial per step of the scenario's ring.
//    Each fold is a few loads per lane, so no single warp walks a large
//    scenario's thousands of task records.  Tickets re-arm themselves, and
//    the last CTA to exit re-arms the queue.
//  * Laser data.  Every substep's (x_l, y_l, cs) and source band for every
//    scenario is uploaded once for the whole plan, so launches differ only
//    in their first step and the buffer parity: a run is a fixed sequence of
//    launches that a CUDA graph replays.
//
// Every cell goes through the single-field kernel's cell functions, and the
// Partial combine is exact (max T, smallest index on ties), so each scenario
// is bit-identical to its own lpbf_b200_advance run whatever the batch, the
// depth or the rows per task.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <numeric>
#include <vector>

#include "lpbf_advance.cuh"
#include "lpbf_batch.hpp"
#include "lpbf_host.hpp"
#include "lpbf_b200.h"

namespace lpbf_b200 {

// ---- device kernel -----------------------------------------------------------

// Fold one finished task (local index i of scenario s) into its group and,
// when it completes the group, the group into the scenario; the warp that
// completes the scenario writes its K ring entries.  Called by a whole warp
// after lane 0 stored the task's K partials.
template <int K>
__device__ __forceinline__ void fold(const BatchLaunch& L, int s, int i, int base, int nt,
                                     int nx, int ny, Partial* ring, int lane) {
    const int g = i / BATCH_GROUP;
    const int gsz = min(BATCH_GROUP, nt - g * BATCH_GROUP);
    const int gb = __ldg(&L.group_base[s]);
    const int ng = __ldg(&L.group_base[s + 1]) - gb;
    const long long N = (long long)nx * ny;
    unsigned int last = 0;
    if (lane == 0) {
        __threadfence();
        last = (atomicAdd(&L.group_done[gb + g], 1u) == (unsigned int)(gsz - 1)) ? 1u : 0u;
    }
    if (!__shfl_sync(0xffffffffu, last, 0)) return;
    __threadfence();
#pragma unroll
    for (int t = 0; t < K; ++t) {
        double tm = -1.0; long long ag = N; int mn = ny, mx = -1;
        if (lane < gsz) {
            const Partial* q = &L.parts[(size_t)(base + g * BATCH_GROUP + lane) * K + t];
            partial_take(tm, ag, mn, mx, __ldcg(&q->tmax), __ldcg(&q->arg),
                         __ldcg(&q->ymin), __ldcg(&q->ymax));
        }
        partial_warp_reduce(tm, ag, mn, mx);
        if (lane == 0) L.gparts[(size_t)(gb + g) * K + t] = Partial{tm, ag, mn, mx};
    }
    last = 0;
    if (lane == 0) {
        L.group_done[gb + g] = 0u;
        __threadfence();
        last = (atomicAdd(&L.scen_done[s], 1u) == (unsigned int)(ng - 1)) ? 1u : 0u;
    }
    if (!__shfl_sync(0xffffffffu, last, 0)) return;
    __threadfence();
#pragma unroll 1
    for (int t = 0; t < K; ++t) {
        double tm = -1.0; long long ag = N; int mn = ny, mx = -1;
        for (int j = lane; j < ng; j += 32) {
            const Partial* q = &L.gparts[(size_t)(gb + j) * K + t];
            partial_take(tm, ag, mn, mx, __ldcg(&q->tmax), __ldcg(&q->arg),
                         __ldcg(&q->ymin), __ldcg(&q->ymax));
        }
        partial_warp_reduce(tm, ag, mn, mx);
        if (lane == 0 && ring) ring[L.step0 + t] = Partial{tm, ag, mn, mx};
    }
    if (lane == 0) L.scen_done[s] = 0u;
}

// Per-warp task context, kept in shared memory across the wavefront so that
// it holds no registers there.
struct TaskCtx { int tq, s, base, nt; };

// ST: 0 direct loads, 1 bulk row copies, 2 tensor-map tiles (BATCH_STAGE_*).
// SQM: 1 every field has square cells (one form of the cell update), 2 each
// field takes its own form per task (the WarpStrip modes).
template <int K, int ST, int SQM>
__global__ void __launch_bounds__(ADV_WARPS * 32, AdvOcc<K>::min_ctas)
batch_kernel(const __grid_constant__ BatchLaunch L) {
    constexpr bool STAGED = ST != BATCH_STAGE_DIRECT;
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ __align__(16) RedSmem<K> s_red[ADV_WARPS];
    __shared__ __align__(16) AdvParams s_par[ADV_WARPS];
    __shared__ TaskCtx s_ctx[ADV_WARPS];
    __shared__ unsigned int s_last;

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* stages = reinterpret_cast<double*>(smem) + wid * (ADV_S * ADV_STAGE_DOUBLES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        smem + size_t(ADV_WARPS) * ADV_S * ADV_STAGE_DOUBLES * sizeof(double)) + wid * ADV_S;
    if constexpr (STAGED) {
        if (lane == 0) {
            for (int s = 0; s < ADV_S; ++s) mbar_init(&bars[s], 1);
            fence_mbar_init();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncwarp();
    }

    AdvParams& par = s_par[wid];
    {   // neutral contents until the first task binds a scenario
        unsigned long long* d = reinterpret_cast<unsigned long long*>(&par);
        for (int i = lane; i < (int)(sizeof(AdvParams) / 8); i += 32) d[i] = 0ull;
        __syncwarp();
    }
    WarpStrip<K, STAGED, true, ST == BATCH_STAGE_BULK, SQM> ws(par, nullptr, stages, bars, lane,
                                                         &s_red[wid]);
    volatile TaskCtx* ctx = &s_ctx[wid];
    int bound = -1;                // scenario whose parameters sit in `par`

    for (;;) {
        unsigned int tq = 0;
        if (lane == 0) tq = atomicAdd(&L.hdr->queue, 1u);
        tq = __shfl_sync(0xffffffffu, tq, 0);
        if (tq >= (unsigned int)L.ntasks) break;

        // scenario of queue position tq: largest s with task_base[s] <= tq
        int lo = 0, hi = L.nscen - 1;
        while (lo < hi) {
            const int mid = (lo + hi + 1) >> 1;
            if ((unsigned int)__ldg(&L.task_base[mid]) <= tq) lo = mid; else hi = mid - 1;
        }
        const int s = lo;
        const int base = __ldg(&L.task_base[s]);
        const BatchScen* sc = L.scen + s;
        if (lane == 0) {
            ctx->tq = (int)tq; ctx->s = s; ctx->base = base;
            ctx->nt = __ldg(&L.task_base[s + 1]) - base;
        }

        // bind: the scenario's static parameters, then this launch's substeps
        // (the same for every task of the scenario in this launch)
        if (s != bound) {
            bound = s;
            __syncwarp();
            const unsigned long long* src = reinterpret_cast<const unsigned long long*>(&sc->par);
            unsigned long long* d = reinterpret_cast<unsigned long long*>(&par);
            for (int i = lane; i < (int)(sizeof(AdvParams) / 8); i += 32) d[i] = __ldg(src + i);
            __syncwarp();
            if (lane == 0) {
                int blo = 1 << 30, bhi = -(1 << 30), bxlo = 1 << 30, bxhi = -(1 << 30);
#pragma unroll
                for (int t = 0; t < K; ++t) {
                    const BatchStep& st = L.steps[(size_t)(L.step0 + t) * L.nscen + s];
                    par.las[t] = st.las;
                    blo = min(blo, st.band_lo); bhi = max(bhi, st.band_hi);
                    bxlo = min(bxlo, st.bandx_lo); bxhi = max(bxhi, st.bandx_hi);
                }
                par.band_lo = blo; par.band_hi = bhi; par.bandx_lo = bxlo; par.bandx_hi = bxhi;
                // this launch's chunks: the band split of steps [step0, step0 +
                // kfull), as the host's task tables count them
                int ulo = 1 << 30, uhi = -(1 << 30);
                const int tend = __ldg(&sc->split) ? min(L.step0 + L.kfull, L.nsteps) : 0;
                for (int t = L.step0; t < tend; ++t) {
                    const BatchStep& st = L.steps[(size_t)t * L.nscen + s];
                    ulo = min(ulo, st.band_lo); uhi = max(uhi, st.band_hi);
                }
                band_chunks(par.H, 0, par.c.ny, L.kfull, ulo, uhi, &par.nA, &par.nB, &par.Hb,
                            &par.Ya, &par.Yb, &par.nchunks);
                par.ntasks = par.nstrips * par.nchunks;
                par.Tin = sc->buf[L.parity];
                par.Tout = sc->buf[L.parity ^ 1];
                par.err = &L.hdr->err;
            }
            __syncwarp();
            ws.reload_coef();
            ws.reset_red();        // lane peaks are carried only within one field
        }
        __syncwarp();
        if constexpr (ST == BATCH_STAGE_TMAP) ws.map = &sc->map[L.parity];
        ws.run_task((int)tq - base);
        if (ws.failed) break;
        const int c_tq = ctx->tq, c_s = ctx->s, c_base = ctx->base, c_nt = ctx->nt;

        // The warp's K partials so far for this field (this task and the
        // field's earlier tasks of this warp: max and min are idempotent),
        // at the task's queue position.
        __syncwarp();
#pragma unroll
        for (int t = 0; t < K; ++t) {
            double tm = s_red[wid].tmx[t][lane];
            long long ag = s_red[wid].arg[t][lane];
            int mn = s_red[wid].ymn[t], mx = s_red[wid].ymx[t];
            partial_warp_reduce(tm, ag, mn, mx);
            if (lane == 0) L.parts[(size_t)c_tq * K + t] = Partial{tm, ag, mn, mx};
        }
        fold<K>(L, c_s, c_tq - c_base, c_base, c_nt, par.c.nx, par.c.ny, L.scen[c_s].ring, lane);
    }

    // the last CTA to leave re-arms the queue for the next launch
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        s_last = (atomicAdd(&L.hdr->ctas, 1u) == gridDim.x - 1) ? 1u : 0u;
    }
    __syncthreads();
    if (s_last && threadIdx.x == 0) {
        L.hdr->queue = 0u;
        L.hdr->ctas = 0u;
    }
}

// ---- launch ------------------------------------------------------------------

namespace {

template <int K, int ST>
struct BatchKernelInfo {
    static constexpr bool STAGED = ST != BATCH_STAGE_DIRECT;
    static int resident_per_sm() {
        static int occ[64] = {0};
        int dev = 0;
        cudaGetDevice(&dev);
        if (dev < 0 || dev >= 64) dev = 0;
        if (occ[dev] == 0) {
            const size_t smem = STAGED ? ADV_SMEM_BYTES : 0;
            int nb = 1 << 30;
            for (auto kern : {batch_kernel<K, ST, 1>, batch_kernel<K, ST, 2>}) {
                if (smem > 48 * 1024 &&
                    cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem) != cudaSuccess)
                    return 0;
                int n = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kern, ADV_WARPS * 32,
                                                                  smem) != cudaSuccess)
                    return 0;
                nb = std::min(nb, n);
            }
            occ[dev] = std::max(1, nb);
        }
        return occ[dev];
    }
    static cudaError_t launch(const BatchLaunch& L, int ctas_per_sm, cudaStream_t s) {
        const int occ = resident_per_sm();
        if (occ <= 0) return cudaErrorInvalidConfiguration;
        const int per_sm = ctas_per_sm > 0 ? std::min(ctas_per_sm, occ) : occ;
        int grid = std::min(sm_count() * per_sm, (L.ntasks + ADV_WARPS - 1) / ADV_WARPS);
        grid = std::max(grid, 1);
        const size_t smem = STAGED ? ADV_SMEM_BYTES : 0;
        if (L.sq_all) batch_kernel<K, ST, 1><<<grid, ADV_WARPS * 32, smem, s>>>(L);
        else          batch_kernel<K, ST, 2><<<grid, ADV_WARPS * 32, smem, s>>>(L);
        return cudaGetLastError();
    }
};

template <int ST>
cudaError_t launch_batch_t(int K, const BatchLaunch& L, int ctas_per_sm, cudaStream_t s) {
    switch (K) {
        case 1: return BatchKernelInfo<1, ST>::launch(L, ctas_per_sm, s);
        case 2: return BatchKernelInfo<2, ST>::launch(L, ctas_per_sm, s);
        case 3: return BatchKernelInfo<3, ST>::launch(L, ctas_per_sm, s);
        case 4: return BatchKernelInfo<4, ST>::launch(L, ctas_per_sm, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int ST>
int resident_t(int K) {
    switch (K) {
        case 1: return BatchKernelInfo<1, ST>::resident_per_sm();
        case 2: return BatchKernelInfo<2, ST>::resident_per_sm();
        case 3: return BatchKernelInfo<3, ST>::resident_per_sm();
        case 4: return BatchKernelInfo<4, ST>::resident_per_sm();
        default: return 0;
    }
}

}  // namespace

cudaError_t launch_batch(int K, int stage, const BatchLaunch& L, int ctas_per_sm,
                         cudaStream_t s) {
    switch (stage) {
        case BATCH_STAGE_DIRECT: return launch_batch_t<BATCH_STAGE_DIRECT>(K, L, ctas_per_sm, s);
        case BATCH_STAGE_BULK: return launch_batch_t<BATCH_STAGE_BULK>(K, L, ctas_per_sm, s);
        case BATCH_STAGE_TMAP: return launch_batch_t<BATCH_STAGE_TMAP>(K, L, ctas_per_sm, s);
        default: return cudaErrorInvalidValue;
    }
}

int batch_resident_per_sm(int K, int stage) {
    switch (stage) {
        case BATCH_STAGE_DIRECT: return resident_t<BATCH_STAGE_DIRECT>(K);
        case BATCH_STAGE_BULK: return resident_t<BATCH_STAGE_BULK>(K);
        case BATCH_STAGE_TMAP: return resident_t<BATCH_STAGE_TMAP>(K);
        default: return 0;
    }
}

// ---- host layout -------------------------------------------------------------

int size_class(int nx, int ny) {
    const int side = std::max(nx, ny);
    return side < 512 ? 0 : side < 1024 ? 1 : side < 2048 ? 2 : 3;
}

namespace {

size_t align_up(size_t v, size_t a) { return (v + a - 1) / a * a; }

int resolve_rows(const lpbf_b200_batch_opts& o, int cls, int K, int ny) {
    int H = o.rows[cls] > 0 ? o.rows[cls] : 24;
    H = std::max(H, std::max(8, 4 * K));
    return std::min(H, ny);
}

}  // namespace

bool batch_layout(const lpbf_b200_scenario* sc, int n, int n_steps,
                  const lpbf_b200_batch_opts& o, BatchLayout* out) {
    BatchLayout Lo;
    Lo.K = o.depth > 0 ? std::min(o.depth, 4) : 3;
    Lo.order.resize(n);
    std::iota(Lo.order.begin(), Lo.order.end(), 0);
    // largest scenarios first; ties keep the caller's order
    std::stable_sort(Lo.order.begin(), Lo.order.end(), [&](int a, int b) {
        return (long long)sc[a].k->nx * sc[a].k->ny > (long long)sc[b].k->nx * sc[b].k->ny;
    });
    Lo.H.assign(n, 0);
    Lo.split.assign(n, 0);
    std::vector<int> nstrips(n), ny(n);
    long long total = 0;
    for (int i = 0; i < n; ++i) total += (long long)sc[i].k->nx * sc[i].k->ny;
    bool plans = n_steps > 0;
    for (int i = 0; i < n; ++i) {
        const StepConst& k = *sc[Lo.order[i]].k;
        Lo.H[i] = resolve_rows(o, size_class(k.nx, k.ny), Lo.K, k.ny);
        nstrips[i] = (k.nx + ADV_WOUT - 1) / ADV_WOUT;
        ny[i] = k.ny;
        Lo.split[i] = batch_split_field((long long)k.nx * k.ny, total) ? 1 : 0;
        plans = plans && sc[Lo.order[i]].plan != nullptr;
    }
    // per-step laser data and source bands, by stored position
    if (plans) {
        Lo.steps.resize((size_t)n * n_steps);
        for (int i = 0; i < n; ++i) {
            const lpbf_b200_scenario& s = sc[Lo.order[i]];
            const StepConst& k = *s.k;
            const Coef c = make_coef(k, s.bc, s.T_edge, s.Tm);
            for (int t = 0; t < n_steps; ++t) {
                BatchStep& st = Lo.steps[(size_t)t * n + i];
                st.las = make_laser(k, s.plan[t].x_l, s.plan[t].y_l, s.plan[t].q_scale);
                laser_band(c, &st.las, 1, &st.band_lo, &st.band_hi, &st.bandx_lo, &st.bandx_hi);
            }
        }
    }
    // task and group offsets of every scenario for a launch starting at each
    // plan step: the band split of the band over [r, r + K)
    Lo.rows_t = std::max(n_steps, 1);
    Lo.task_base.assign((size_t)Lo.rows_t * (n + 1), 0);
    Lo.group_base.assign((size_t)Lo.rows_t * (n + 1), 0);
    long long tmax = 0, gmax = 0;
    for (int r = 0; r < Lo.rows_t; ++r) {
        long long tot = 0, gtot = 0;
        int* tb = &Lo.task_base[(size_t)r * (n + 1)];
        int* gb = &Lo.group_base[(size_t)r * (n + 1)];
        for (int i = 0; i < n; ++i) {
            int lo = 1 << 30, hi = -(1 << 30);
            if (plans && Lo.split[i]) {
                for (int t = r; t < std::min(r + Lo.K, n_steps); ++t) {
                    const BatchStep& st = Lo.steps[(size_t)t * n + i];
                    lo = std::min(lo, st.band_lo);
                    hi = std::max(hi, st.band_hi);
                }
            }
            int nA, nB, Hb, Ya, Yb, nch;
            band_chunks(Lo.H[i], 0, ny[i], Lo.K, lo, hi, &nA, &nB, &Hb, &Ya, &Yb, &nch);
            long long nt = (long long)nstrips[i] * nch;
            if (!plans) {
                // sizing without the plans: every chunk of at most
                // min(H, ADV_BAND_ROWS) rows bounds any launch's count
                const int hb = std::min(Lo.H[i], ADV_BAND_ROWS);
                nt = std::max(nt, (long long)nstrips[i] * ((ny[i] + hb - 1) / hb + 2));
            }
            tb[i] = (int)tot;
            gb[i] = (int)gtot;
            tot += nt;
            gtot += (nt + BATCH_GROUP - 1) / BATCH_GROUP;
            if (tot >= (1ll << 30)) return false;
        }
        tb[n] = (int)tot;
        gb[n] = (int)gtot;
        tmax = std::max(tmax, tot);
        gmax = std::max(gmax, gtot);
    }
    Lo.ntasks = (int)tmax;
    Lo.ngroups = (int)gmax;
    const size_t tables = sizeof(int) * (size_t)Lo.rows_t * (n + 1);
    size_t off = sizeof(BatchHeader);
    Lo.off_done = off;   off = align_up(off + sizeof(unsigned int) * n, 256);
    Lo.off_scen = off;   off = align_up(off + sizeof(BatchScen) * n, 256);
    Lo.off_base = off;   off = align_up(off + tables, 256);
    Lo.off_gbase = off;  off = align_up(off + tables, 256);
    Lo.off_gdone = off;  off = align_up(off + sizeof(unsigned int) * gmax, 256);
    Lo.off_steps = off;  off = align_up(off + sizeof(BatchStep) * (size_t)n * n_steps, 256);
    Lo.off_parts = off;  off = align_up(off + sizeof(Partial) * (size_t)tmax * Lo.K, 256);
    Lo.off_gparts = off; off = align_up(off + sizeof(Partial) * (size_t)gmax * Lo.K, 256);
    Lo.bytes = off;
    *out = std::move(Lo);
    return true;
}

}  // namespace lpbf_b200

namespace lpbf_b200 {

// ---- sub-grid melt width on the hot column ------------------------------------

// Per scenario (one CTA each), after plan step `step` wrote its Partial and
// the field now sits in buf[par]: the melt width through the column of the
// step's hottest cell, interpolating the two T = Tm crossings linearly (the
// rule of the reference's MetricsTask, include/gpu_step_task.hpp:380-395),
// where cruise[step][user] is set and the peak exceeds Tm; 0 elsewhere.
__global__ void wsub_kernel(const BatchScen* scen, int step, int n_steps, int par,
                            const unsigned char* cruise, double* w_sub, int nscen) {
    __shared__ int s_a, s_b;
    const BatchScen& sc = scen[blockIdx.x];
    const int user = sc.user;
    const int nx = sc.par.c.nx, ny = sc.par.c.ny;
    const double Tm = sc.par.c.Tm, dy = sc.par.c.dy;
    const bool has = sc.ring != nullptr && cruise[(size_t)step * nscen + user] != 0;
    const Partial r = has ? sc.ring[step] : Partial{-1.0, 0, 0, -1};
    if (!(has && r.tmax > Tm)) {
        if (threadIdx.x == 0) w_sub[(size_t)step * nscen + user] = 0.0;
        return;
    }
    const int x = (int)(r.arg % nx);
    const double* col = sc.buf[par] + x;
    if (threadIdx.x == 0) { s_a = ny; s_b = -1; }
    __syncthreads();
    int a = ny, b = -1;
    for (int y = threadIdx.x; y < ny; y += blockDim.x)
        if (col[(size_t)y * nx] > Tm) { a = min(a, y); b = max(b, y); }
    atomicMin(&s_a, a);
    atomicMax(&s_b, b);
    __syncthreads();
    if (threadIdx.x != 0) return;
    a = s_a;
    b = s_b;
    double w = 0.0;
    if (b >= 0) {
        double lo = __dmul_rn((double)a, dy), hi = __dmul_rn((double)b, dy);
        if (a > 0) {
            const double c0 = col[(size_t)(a - 1) * nx], c1 = col[(size_t)a * nx];
            lo = __dmul_rn(__dadd_rn((double)(a - 1), __ddiv_rn(__dsub_rn(Tm, c0), __dsub_rn(c1, c0))), dy);
        }
        if (b < ny - 1) {
            const double c0 = col[(size_t)b * nx], c1 = col[(size_t)(b + 1) * nx];
            hi = __dmul_rn(__dadd_rn((double)b, __ddiv_rn(__dsub_rn(Tm, c0), __dsub_rn(c1, c0))), dy);
        }
        w = __dmul_rn(__dsub_rn(hi, lo), 1e6);
    }
    w_sub[(size_t)step * nscen + user] = w;
}

}  // namespace lpbf_b200

// ===========================================================================
// C-ABI
// ===========================================================================
using namespace lpbf_b200;

struct lpbf_b200_batch {
    int nscen = 0, n_steps = 0, K = 3, ctas_per_sm = 0;
    int stage = BATCH_STAGE_BULK;
    BatchLayout lay;
    unsigned char* work = nullptr;
    int cur = 0;                   // buffer holding the current fields (0: T_a, 1: T_b)
    bool all_rings = false;        // every scenario has a ring
    bool sq_all = false;           // every scenario has square cells
    int device = 0;
    // cached graphs, keyed by (first_step, n_steps, starting parity)
    struct Graph { cudaGraphExec_t exec = nullptr; int first = -1, n = -1, par = -1; };
    Graph graphs[2];
    int next_graph = 0;
    cudaStream_t cap = nullptr;

    BatchLaunch launch_params(int step0, int parity) const {
        BatchLaunch L;
        // the task tables of a launch starting at step0
        const size_t row = (size_t)std::min(std::max(step0, 0), lay.rows_t - 1) * (nscen + 1);
        L.scen = reinterpret_cast<const BatchScen*>(work + lay.off_scen);
        L.task_base = reinterpret_cast<const int*>(work + lay.off_base) + row;
        L.steps = reinterpret_cast<const BatchStep*>(work + lay.off_steps);
        L.hdr = reinterpret_cast<BatchHeader*>(work);
        L.scen_done = reinterpret_cast<unsigned int*>(work + lay.off_done);
        L.group_base = reinterpret_cast<const int*>(work + lay.off_gbase) + row;
        L.group_done = reinterpret_cast<unsigned int*>(work + lay.off_gdone);
        L.parts = reinterpret_cast<Partial*>(work + lay.off_parts);
        L.gparts = reinterpret_cast<Partial*>(work + lay.off_gparts);
        L.nscen = nscen;
        L.ntasks = lay.task_base[row + nscen];
        L.parity = parity;
        L.step0 = step0;
        L.sq_all = sq_all ? 1 : 0;
        L.kfull = K;
        L.nsteps = n_steps;
        return L;
    }

    // Issue the launches of steps [first, first + n) on `s`, starting from
    // buffer parity `par`; *par_out receives the parity after them.
    cudaError_t issue(int first, int n, int par, cudaStream_t s, int* par_out) const {
        for (int s0 = first; s0 < first + n; s0 += K) {
            const int kk = std::min(K, first + n - s0);
            const cudaError_t e = launch_batch(kk, stage, launch_params(s0, par), ctas_per_sm, s);
            if (e != cudaSuccess) return e;
            par ^= 1;
        }
        *par_out = par;
        return cudaSuccess;
    }

    void drop_graphs() {
        for (auto& g : graphs) {
            if (g.exec) cudaGraphExecDestroy(g.exec);
            g = Graph{};
        }
    }
};

namespace {

bool valid_scenario(const lpbf_b200_scenario& s) {
    if (!s.k || !s.T_a || !s.T_b || s.T_a == s.T_b) return false;
    const StepConst& k = *s.k;
    if (k.nx < 2 || k.ny < 1 || (long long)k.nx * k.ny >= (1ll << 40)) return false;
    if (s.bc != 0 && s.bc != 1) return false;
    const size_t N = (size_t)k.nx * k.ny;
    return !(s.T_a < s.T_b + N && s.T_b < s.T_a + N);
}

bool valid_opts(const lpbf_b200_batch_opts* o) {
    if (!o) return true;
    if (o->depth < 0 || o->depth > 4 || o->ctas_per_sm < 0) return false;
    if (o->staging < 0 || o->staging > 2) return false;
    for (int i = 0; i < 4; ++i)
        if (o->rows[i] < 0) return false;
    return true;
}

lpbf_b200_batch_opts opts_or_default(const lpbf_b200_batch_opts* o) {
    lpbf_b200_batch_opts d;
    std::memset(&d, 0, sizeof(d));
    return o ? *o : d;
}

}  // namespace

extern "C" {

int lpbf_b200_batch_size_class(int nx, int ny) { return size_class(nx, ny); }

size_t lpbf_b200_batch_workspace_bytes(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                                       const lpbf_b200_batch_opts* opts) {
    if (!sc || n_scen <= 0 || n_steps < 0 || !valid_opts(opts)) return 0;
    for (int i = 0; i < n_scen; ++i)
        if (!sc[i].k) return 0;
    BatchLayout lay;
    if (!batch_layout(sc, n_scen, n_steps, opts_or_default(opts), &lay)) return 0;
    return lay.bytes;
}

int lpbf_b200_batch_create(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                           const lpbf_b200_batch_opts* opts, void* work, size_t work_bytes,
                           cudaStream_t stream, lpbf_b200_batch** out) {
    NvtxRange nvtx_range("lpbf_b200_batch_create");
    if (!out) return LPBF_ERR_ARG;
    *out = nullptr;
    if (!sc || n_scen <= 0 || n_steps < 0 || !valid_opts(opts)) return LPBF_ERR_ARG;
    for (int i = 0; i < n_scen; ++i)
        if (!valid_scenario(sc[i]) || (n_steps > 0 && !sc[i].plan)) return LPBF_ERR_ARG;
    const lpbf_b200_batch_opts o = opts_or_default(opts);
    BatchLayout lay;
    if (!batch_layout(sc, n_scen, n_steps, o, &lay)) return LPBF_ERR_ARG;
    if (!work || work_bytes < lay.bytes || reinterpret_cast<uintptr_t>(work) % 256 != 0)
        return LPBF_ERR_WORKSPACE;

    // Staged loads need even rows and 16-byte aligned fields; one field
    // without them switches the batch to direct loads.  Automatic staging:
    // bulk row copies, unless the batch holds few fields (then one tensor
    // map per buffer stays resident in the copy engine's descriptor cache).
    bool can_stage = true;
    for (int i = 0; i < n_scen; ++i)
        can_stage = can_stage && tma_ok(sc[i].T_a, sc[i].k->nx) && tma_ok(sc[i].T_b, sc[i].k->nx);
    int stage = o.staging == 0 ? (n_scen <= 4 ? BATCH_STAGE_TMAP : BATCH_STAGE_BULK) : o.staging;
    if (!can_stage) stage = BATCH_STAGE_DIRECT;

    // Warm the per-device occupancy cache now: a later run may be captured
    // into a graph, where these queries are best avoided.
    for (int kk = 1; kk <= 4; ++kk)
        if (batch_resident_per_sm(kk, stage) <= 0) return LPBF_ERR_CUDA;

    // host image of the descriptor sections, uploaded in one copy
    const size_t img_bytes = lay.off_steps;
    std::vector<BatchHeader> img_store(img_bytes / sizeof(BatchHeader));
    unsigned char* img = reinterpret_cast<unsigned char*>(img_store.data());
    std::memset(img, 0, img_bytes);
    const std::vector<BatchStep>& steps = lay.steps;
    std::vector<BatchScen> scen(n_scen);
    bool sq_all = true;
    for (int i = 0; i < n_scen; ++i) {
        const lpbf_b200_scenario& s = sc[lay.order[i]];
        const StepConst& k = *s.k;
        BatchScen& b = scen[i];
        std::memset(&b, 0, sizeof(b));
        AdvParams& p = b.par;
        p.c = make_coef(k, s.bc, s.T_edge, s.Tm);
        sq_all = sq_all && p.c.ax == p.c.ay;
        p.nstrips = (k.nx + ADV_WOUT - 1) / ADV_WOUT;
        p.H = lay.H[i];
        p.nchunks = (k.ny + p.H - 1) / p.H;
        p.ntasks = p.nstrips * p.nchunks;
        p.row0 = 0;
        p.gny = k.ny;
        p.row_lo = 0;
        p.row_hi = k.ny;
        p.st256 = (k.nx % 4 == 0) && reinterpret_cast<uintptr_t>(s.T_a) % 32 == 0 &&
                  reinterpret_cast<uintptr_t>(s.T_b) % 32 == 0;
        b.buf[0] = s.T_a;
        b.buf[1] = s.T_b;
        b.ring = s.ring;
        b.user = lay.order[i];
        b.split = lay.split[i];
        if (stage == BATCH_STAGE_TMAP &&
            (!tensor_map_f64(s.T_a, k.nx, k.ny, ADV_COLS, ADV_R, &b.map[0]) ||
             !tensor_map_f64(s.T_b, k.nx, k.ny, ADV_COLS, ADV_R, &b.map[1])))
            return LPBF_ERR_TMA;
    }
    std::memcpy(img + lay.off_scen, scen.data(), sizeof(BatchScen) * n_scen);
    std::memcpy(img + lay.off_base, lay.task_base.data(), sizeof(int) * lay.task_base.size());
    std::memcpy(img + lay.off_gbase, lay.group_base.data(), sizeof(int) * lay.group_base.size());

    int dev = 0;
    cudaGetDevice(&dev);
    unsigned char* w = static_cast<unsigned char*>(work);
    if (cudaMemcpyAsync(w, img, img_bytes, cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return LPBF_ERR_CUDA;
    if (!steps.empty() &&
        cudaMemcpyAsync(w + lay.off_steps, steps.data(), sizeof(BatchStep) * steps.size(),
                        cudaMemcpyHostToDevice, stream) != cudaSuccess)
        return LPBF_ERR_CUDA;
    // the host images are freed on return
    if (cudaStreamSynchronize(stream) != cudaSuccess) return LPBF_ERR_CUDA;

    lpbf_b200_batch* b = new lpbf_b200_batch();
    b->nscen = n_scen;
    b->n_steps = n_steps;
    b->K = lay.K;
    b->ctas_per_sm = o.ctas_per_sm;
    b->stage = stage;
    b->all_rings = true;
    b->sq_all = sq_all;
    for (int i = 0; i < n_scen; ++i) b->all_rings = b->all_rings && sc[i].ring != nullptr;
    b->lay = std::move(lay);
    b->work = w;
    b->device = dev;
    *out = b;
    return LPBF_OK;
}

int lpbf_b200_batch_launches(const lpbf_b200_batch* b, int n_steps) {
    if (!b || n_steps < 0) return LPBF_ERR_ARG;
    return (n_steps + b->K - 1) / b->K;
}

int lpbf_b200_batch_tasks(const lpbf_b200_batch* b) {
    return b ? b->lay.ntasks : LPBF_ERR_ARG;
}

}  // extern "C"

namespace {

// The cached graph of steps [first, first + n) from buffer parity `par`,
// captured now if missing; null on failure.
lpbf_b200_batch::Graph* batch_graph(lpbf_b200_batch* b, int first, int n, int par) {
    for (auto& c : b->graphs)
        if (c.exec && c.first == first && c.n == n && c.par == par) return &c;
    if (!b->cap && cudaStreamCreateWithFlags(&b->cap, cudaStreamNonBlocking) != cudaSuccess)
        return nullptr;
    lpbf_b200_batch::Graph* g = &b->graphs[b->next_graph];
    b->next_graph ^= 1;
    if (g->exec) cudaGraphExecDestroy(g->exec);
    *g = lpbf_b200_batch::Graph{};
    cudaGraph_t graph = nullptr;
    if (cudaStreamBeginCapture(b->cap, cudaStreamCaptureModeThreadLocal) != cudaSuccess)
        return nullptr;
    int par_end = par;
    const cudaError_t e1 = b->issue(first, n, par, b->cap, &par_end);
    const cudaError_t e2 = cudaStreamEndCapture(b->cap, &graph);
    if (e1 != cudaSuccess || e2 != cudaSuccess) {
        if (graph) cudaGraphDestroy(graph);
        return nullptr;
    }
    const cudaError_t e3 = cudaGraphInstantiate(&g->exec, graph, 0);
    cudaGraphDestroy(graph);
    if (e3 != cudaSuccess) { g->exec = nullptr; return nullptr; }
    g->first = first; g->n = n; g->par = par;
    return g;
}

bool valid_range(const lpbf_b200_batch* b, int first_step, int n_steps) {
    return b && first_step >= 0 && n_steps >= 0 && first_step <= b->n_steps &&
           n_steps <= b->n_steps - first_step;
}

}  // namespace

extern "C" {

int lpbf_b200_batch_run(lpbf_b200_batch* b, int first_step, int n_steps, int use_graph,
                        cudaStream_t stream) {
    NvtxRange nvtx_range("lpbf_b200_batch_run");
    if (!valid_range(b, first_step, n_steps)) return LPBF_ERR_ARG;
    if (n_steps == 0) return LPBF_OK;
    int par = b->cur;
    if (!use_graph) {
        if (b->issue(first_step, n_steps, par, stream, &par) != cudaSuccess) return LPBF_ERR_CUDA;
        b->cur = par;
        return LPBF_OK;
    }
    lpbf_b200_batch::Graph* g = batch_graph(b, first_step, n_steps, par);
    if (!g) return LPBF_ERR_CUDA;
    if (cudaGraphLaunch(g->exec, stream) != cudaSuccess) return LPBF_ERR_CUDA;
    b->cur = par ^ (((n_steps + b->K - 1) / b->K) & 1);
    return LPBF_OK;
}

int lpbf_b200_batch_run_wsub(lpbf_b200_batch* b, int first_step, int n_steps,
                             const unsigned char* cruise, double* w_sub, cudaStream_t stream) {
    NvtxRange nvtx_range("lpbf_b200_batch_run_wsub");
    if (!valid_range(b, first_step, n_steps) || !cruise || !w_sub || !b->all_rings)
        return LPBF_ERR_ARG;
    const BatchScen* scen = reinterpret_cast<const BatchScen*>(b->work + b->lay.off_scen);
    for (int s = first_step; s < first_step + n_steps; ++s) {
        int par = b->cur;
        if (b->issue(s, 1, par, stream, &par) != cudaSuccess) return LPBF_ERR_CUDA;
        b->cur = par;
        wsub_kernel<<<b->nscen, 128, 0, stream>>>(scen, s, b->n_steps, par, cruise, w_sub,
                                                  b->nscen);
        if (cudaGetLastError() != cudaSuccess) return LPBF_ERR_CUDA;
    }
    return LPBF_OK;
}

int lpbf_b200_batch_capture(lpbf_b200_batch* b, int first_step, int n_steps) {
    if (!valid_range(b, first_step, n_steps)) return LPBF_ERR_ARG;
    if (n_steps == 0) return LPBF_OK;
    return batch_graph(b, first_step, n_steps, b->cur) ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_batch_result_in_b(const lpbf_b200_batch* b) {
    return b ? b->cur : LPBF_ERR_ARG;
}

int lpbf_b200_batch_read_error(const lpbf_b200_batch* b, cudaStream_t stream, unsigned int* err) {
    if (!b || !err) return LPBF_ERR_ARG;
    const BatchHeader* h = reinterpret_cast<const BatchHeader*>(b->work);
    if (cudaMemcpyAsync(err, &h->err, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream) !=
        cudaSuccess)
        return LPBF_ERR_CUDA;
    return cudaStreamSynchronize(stream) == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_batch_scenario_rows(const lpbf_b200_batch* b, int scenario) {
    if (!b || scenario < 0 || scenario >= b->nscen) return LPBF_ERR_ARG;
    for (int i = 0; i < b->nscen; ++i)
        if (b->lay.order[i] == scenario) return b->lay.H[i];
    return LPBF_ERR_ARG;
}

void lpbf_b200_batch_destroy(lpbf_b200_batch* b) {
    if (!b) return;
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev != b->device) cudaSetDevice(b->device);
    b->drop_graphs();
    if (b->cap) cudaStreamDestroy(b->cap);
    if (dev != b->device) cudaSetDevice(dev);
    delete b;
}

}  // extern "C"
