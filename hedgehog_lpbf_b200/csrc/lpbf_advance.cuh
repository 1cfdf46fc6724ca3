// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// The temporally blocked step kernel.
//
// Work decomposition.  The nx x ny field (row-major f64) is cut into column
// strips of WOUT = 120 owned columns and row chunks of H owned rows; a warp
// advances one (strip, chunk) task at a time by K time steps.  A warp covers
// COLS = 128 columns: its owned columns plus KH = 4 halo columns per side, so
// it needs no data from other warps (after level t the outermost t halo
// columns are stale; after K <= 4 levels the owned columns are still exact).
// Warps take tasks from an atomic counter (balanced: the laser rows cost
// more) when a workspace is given, round-robin otherwise.
//
// Lane layout.  Lane l holds the four consecutive columns 4l..4l+3 of the
// strip: lanes 1..30 own all their cells, lanes 0 and 31 are halo.  The x
// neighbours of a lane's first and last cell come from the adjacent lanes by
// one warp shuffle each.
//
// Wavefront.  Rows stream top to bottom in boxes of three rows, each box one
// TMA load into a per-warp stage ring (S stages, one mbarrier per stage, no
// CTA barrier anywhere in the stream).  At iteration j the warp takes level-0
// row j from the stage and computes level-t row j-t for t = 1..K from the
// three rows of level t-1 held in registers.  Level-t row r lives in register
// slot r % 3; a box is exactly one turn of the slot rotation, so every slot
// index is a compile-time constant and no register is moved.  Level-K rows
// go straight to HBM as 32-byte stores.
//
// Fast and general boxes.  A box whose rows, over all K levels, are interior
// to the domain and carry no source runs a branch-free body, in strips away
// from the x edges and in strips at a mirror x edge alike (there the lane
// just off the field holds its neighbour's cells in reverse order); rows of
// the chunk's own halo are computed there too and only masked out of the
// store and the reduction (a value outside a level's valid range only ever
// feeds rows that are themselves outside the next level's range).  Every
// other box runs the general body, which handles the top and bottom edges,
// fixed-value boundaries, partial ownership and the Gaussian source
// (evaluated out of line, so exp is not replicated).  Both bodies evaluate
// every cell with the same function, so results depend neither on the body
// nor on K, H or the task order.
//
// Reduction.  For every level (= time step) each lane keeps the peak T with
// its flat index, and each warp the molten row extent (warp vote), over owned
// cells; warps, then CTAs combine them, and the last CTA to finish (atomic
// ticket, no waiting) reduces the per-CTA partials into one Partial per step
// and re-arms the counters for the next launch.
// ---------------------------------------------------------------------------
#pragma once
#include <stddef.h>

#include "lpbf_device.cuh"

namespace lpbf_b200 {

constexpr int ADV_WARPS = 4;       // warps per CTA
constexpr int ADV_COLS = 128;      // columns per warp strip
constexpr int ADV_KH = 4;          // halo columns per side (supports K <= 4)
constexpr int ADV_WOUT = ADV_COLS - 2 * ADV_KH;
constexpr int ADV_V = 4;           // values per lane per row
constexpr int ADV_R = 3;           // rows per TMA box (= the register slot rotation)
constexpr int ADV_S = 4;           // TMA stages per warp
constexpr int ADV_BAND_ROWS = 8;   // rows per task where tasks reach the source band
constexpr int ADV_STAGE_DOUBLES = ADV_R * ADV_COLS;
constexpr size_t ADV_SMEM_BYTES =
    size_t(ADV_WARPS) * ADV_S * ADV_STAGE_DOUBLES * sizeof(double)
    + size_t(ADV_WARPS) * ADV_S * sizeof(uint64_t);

struct AdvParams {
    Coef c;
    LaserSub las[KMAX];
    int band_lo, band_hi;          // rows any substep's source can reach (union)
    int bandx_lo, bandx_hi;        // columns any substep's source can reach (union)
    int nstrips, nchunks, H, ntasks;
    const double* Tin;             // source field (used by the direct-load path)
    double* Tout;                  // destination field (never aliases Tin)
    Partial* ring;                 // K finalized Partials (one per step), or null
    Partial* scratch;              // per-CTA partials, gridDim.x * K entries
    unsigned int* counter;         // last-CTA ticket, zero between launches
    unsigned int* tasks;           // task counter (dynamic scheduling), or null
    unsigned int* err;             // error word (bit 0: TMA wait timed out)
    Partial* ref_out;              // reference fused-reduce layout (K == 1), or null
    long long ref_nparts;          // number of entries of ref_out to define
    int st256;                     // 32-byte aligned rows: 256-bit stores
    // Row window: the launch advances buffer rows [row_lo, row_hi) (the rest
    // are input halo); buffer row 0 is row row0 of a field of gny rows, which
    // places the source and numbers the cells in the reductions.  A whole
    // field: row0 = 0, gny = ny, [0, ny).
    int row0, gny, row_lo, row_hi;
    // Chunks: nA of H rows from row_lo, then nB of Hb rows from Ya up to Yb
    // (the rows whose tasks reach the source band: short tasks, so that
    // none of these slow ones is left long at the end of a launch), then
    // H-row chunks from Yb.  No band split: nA = nB = 0, Ya = Yb = row_lo.
    int nA, nB, Hb, Ya, Yb;
};

__host__ __device__ constexpr int mod3(int a) { return ((a % 3) + 3) % 3; }

// Chunk layout of rows [row_lo, row_hi) for tasks of H rows at depth K
// (AdvParams's nA, nB, Hb, Ya, Yb, nchunks): the rows whose tasks (owned
// rows +- K) reach the source band [band_lo, band_hi] go in chunks of at
// most ADV_BAND_ROWS rows, so that none of these slow tasks is left long at
// the end of a launch; H-row chunks before and after.  An empty band
// (band_lo > band_hi) gives H-row chunks only.
__host__ __device__ inline void band_chunks(int H, int row_lo, int row_hi, int K, int band_lo,
                                            int band_hi, int* nA, int* nB, int* Hb, int* Ya,
                                            int* Yb, int* nchunks) {
    *nA = 0; *nB = 0; *Hb = H; *Ya = row_lo; *Yb = row_lo;
    if (band_lo <= band_hi) {
        const int b0 = band_lo - K > row_lo ? band_lo - K : row_lo;
        const int b1 = band_hi + K + 1 < row_hi ? band_hi + K + 1 : row_hi;
        if (b0 < b1) {
            *Hb = H < ADV_BAND_ROWS ? H : ADV_BAND_ROWS;
            *nA = (b0 - row_lo) / H;
            *Ya = row_lo + *nA * H;
            *Yb = b1;
            *nB = (*Yb - *Ya + *Hb - 1) / *Hb;
        }
    }
    *nchunks = *nA + *nB + (row_hi - *Yb + H - 1) / H;
}

// Hot coefficients, held in registers for the whole kernel (clsTa is
// c_ls * Tamb, rounded once; sq: ax == ay, square cells).
struct HotCoef {
    double ax, ay, cls, crad, clsTa, Ta4;
    bool sq;
};
__device__ __forceinline__ HotCoef hot_coef(const Coef& c) {
    return HotCoef{c.ax, c.ay, c.c_ls, c.c_rad, __dmul_rn(c.c_ls, c.Tamb), c.Tamb4,
                   c.ax == c.ay};
}

// The update of one cell from its four neighbours (Tamb == Tsub form).
// T^4 - Tamb^4 and c_ls (T - Tamb) are each one fused multiply-add and the
// loss enters the increment's fused chain: 11 FP64 operations, or 10 when
// ax == ay (SQ: one Laplacian (R + L) + (U + D) - 4T).  Which form a field
// uses depends only on its coefficients, so every path computes a cell
// bit-identically.  The Laplacian is exactly zero for a uniform field, and
// the loss at Tamb is only a last rounding (|loss| ~ 1e-16 K), below half an
// ulp of T, so a uniform field at Tamb stays exactly uniform.
template <bool SQ>
__device__ __forceinline__ double cell_net(double T, double L, double R, double U, double D,
                                           const HotCoef& h) {
    const double t2 = __dmul_rn(T, T);
    const double e4 = fma(t2, t2, -h.Ta4);
    const double loss = fma(h.crad, e4, fma(h.cls, T, -h.clsTa));
    if constexpr (SQ) {
        const double lap = fma(-4.0, T, __dadd_rn(R + L, U + D));
        return fma(h.ax, lap, -loss);
    } else {
        const double lx = fma(-2.0, T, R + L);
        const double ly = fma(-2.0, T, U + D);
        return fma(h.ax, lx, fma(h.ay, ly, -loss));
    }
}
template <bool SQ>
__device__ __forceinline__ double cell_core(double T, double L, double R, double U, double D,
                                            const HotCoef& h) {
    return __dadd_rn(T, cell_net<SQ>(T, L, R, U, D, h));
}
template <bool SQ>
__device__ __forceinline__ double cell_core_src(double T, double L, double R, double U, double D,
                                                double S, const HotCoef& h) {
    return __dadd_rn(T, __dadd_rn(cell_net<SQ>(T, L, R, U, D, h), S));
}

// Gaussian source increment of a lane's four cells starting at column x0
// (out of line: the exp code exists once in the binary).
static __device__ __noinline__ double4 source4(int x0, double dy2, double x_l, double cs, double dx,
                                        double m2r, double r2_cut) {
    double S[4];
#pragma unroll
    for (int v = 0; v < 4; ++v) {
        const double xd = __dsub_rn(__dmul_rn((double)(x0 + v), dx), x_l);
        const double r2 = __dadd_rn(__dmul_rn(xd, xd), dy2);
        S[v] = (r2 < r2_cut) ? cs * exp(__dmul_rn(m2r, r2)) : 0.0;
    }
    return make_double4(S[0], S[1], S[2], S[3]);
}

// 32-byte stores of level-K values.  They carry no "memory" clobber: the
// kernel never reads the destination field back (the exact reduction reads
// staged copies), and a clobber would make the compiler reload every
// parameter it keeps in memory after each store.
__device__ __forceinline__ void st_global_v4(double* p, double a, double b, double c, double d) {
    asm volatile("st.global.v4.f64 [%0], {%1, %2, %3, %4};"
                 :: "l"(p), "d"(a), "d"(b), "d"(c), "d"(d));
}
// 32-byte store issued under a predicate (no branch).
__device__ __forceinline__ void st_global_v4_pred(double* p, const double* v, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t"
                 "@q st.global.v4.f64 [%0], {%1, %2, %3, %4};\n\t}"
                 :: "l"(p), "d"(v[0]), "d"(v[1]), "d"(v[2]), "d"(v[3]), "r"((int)pred));
}

// Per-warp reduction state in shared memory: lane peaks and their flat
// indices per level, the molten row extent per level, and a staging area for
// one level's three box rows.
template <int K>
struct alignas(16) RedSmem {
    double tmx[K][32];
    long long arg[K][32];
    int ymn[K], ymx[K];
    alignas(16) double box[3][32][ADV_V];   // written as 16-byte vectors
};
static_assert(offsetof(RedSmem<1>, box) % 16 == 0 && sizeof(RedSmem<1>) % 16 == 0, "align");
static_assert(offsetof(RedSmem<3>, box) % 16 == 0 && sizeof(RedSmem<3>) % 16 == 0, "align");

// TMA: rows are staged in shared memory by the copy engine (otherwise each
// lane loads its cells directly).  BULK: the staging copies are plain bulk
// copies, one per row, instead of tensor-map loads: no descriptor is read per
// copy, which matters when warps work on many different fields at once (a
// tensor map in global memory is fetched by the copy engine); requires an
// even row length and a 16-byte aligned field.
// SQM: which cell_net form the strip uses — 0 the general one, 1 the
// square-cell one, 2 the field's own (h.sq), chosen per task (the batched
// kernel, whose fields differ).
template <int K, bool TMA, bool REDUCE, bool BULK = false, int SQM = 0>
struct WarpStrip {
    static constexpr int V = ADV_V;

    const AdvParams& p;
    const CUtensorMap* map;
    double* stages;                // this warp's S stages
    uint64_t* bars;                // this warp's S mbarriers
    uint32_t gbox;                 // running box counter (mbarrier phase tracking)
    const int lane;
    HotCoef h;

    int x0, xs, xl, y0, y1, jy0, jend, nbox, issued;
    int last_chunk;                      // row chunk of this warp's previous task (-1: none)
    bool edge, failed, own_all, src_strip;
    // Mirror-edge strips on the fast body: the lane just off the field
    // (columns -4..-1, or nx..nx+3) holds the reversed cells of its field
    // neighbour, so the field's edge cell sees itself as its outer neighbour
    // through the ordinary shuffle.
    bool mir;                            // this task keeps mirror lanes (warp-uniform)
    bool mlane;                          // this lane is a mirror lane
    int msrc;                            // lane whose cells this lane mirrors (own lane if none)
    bool fast_ok;                        // the task may use the fast body at all
    bool incl;                           // this task also examines values equal to the lane peak

    double w0[3][V];                     // level-0 window (slot = row % 3)
    double w[K > 1 ? K - 1 : 1][3][V];   // windows of levels 1..K-1
    // Reduction state per level: the lane's resolved peak, this box's peak
    // (resolved once per box, so no row carries a branch), the warp's molten
    // row extent, and in shared memory the flat index of the lane's peak.
    double thr[K];                       // per-box trigger: min(peak, Tm), +inf off-strip
    bool hit[K];                         // a cell of this box crossed thr
    unsigned kmask;                      // level-K rows of this box staged in rs->box
    RedSmem<K>* rs;                      // this warp's reduction state (shared memory)

    // gbox0: boxes this warp has already consumed through its stage ring
    // (mbarrier phases continue across WarpStrip instances of one warp).
    __device__ __forceinline__ WarpStrip(const AdvParams& p_, const CUtensorMap* m,
                                         double* st, uint64_t* b, int ln, RedSmem<K>* rs_,
                                         uint32_t gbox0 = 0)
        : p(p_), map(m), stages(st), bars(b), gbox(gbox0), lane(ln),
          h(hot_coef(p_.c)),
          last_chunk(-1), failed(false), incl(false), kmask(0u), rs(rs_) {
        reset_red();
    }

    // Re-read the hot coefficients after the parameters behind `p` changed
    // (the batched kernel rebinds one WarpStrip to another field per task).
    __device__ __forceinline__ void reload_coef() {
        h = hot_coef(p.c);
    }

    // Neutral reduction state for every level (a new field for this warp).
    __device__ __forceinline__ void reset_red() {
        const long long N = (long long)p.c.nx * p.gny;
        last_chunk = -1;
        if constexpr (REDUCE) {
#pragma unroll
            for (int t = 0; t < K; ++t) {
                hit[t] = false;
                rs->tmx[t][lane] = -1.0;
                rs->arg[t][lane] = N;
                if (lane == 0) { rs->ymn[t] = p.gny; rs->ymx[t] = -1; }
            }
        }
        __syncwarp();
    }

    __device__ __forceinline__ void issue(int b) {
        const uint32_t g = gbox + b;
        const int st = g % ADV_S;
        double* dst = stages + st * ADV_STAGE_DOUBLES;
        if constexpr (BULK) {
            // The rows of the box that exist, columns clipped to the field;
            // stage words outside stay stale and are never used (rows past
            // the end are not read, columns off the field are mirror-edge
            // halo whose values reach no owned cell).
            const int nx = p.c.nx;
            const int r0 = jy0 + b * ADV_R;
            const int nr = min(ADV_R, p.c.ny - r0);
            const int c0 = max(xs, 0);
            const int c1 = min(xs + ADV_COLS, nx);
            const uint32_t bytes = (uint32_t)(c1 - c0) * (uint32_t)sizeof(double);
            mbar_expect_tx(&bars[st], bytes * (uint32_t)nr);
            for (int i = 0; i < nr; ++i)
                bulk_load(dst + i * ADV_COLS + (c0 - xs), p.Tin + (size_t)(r0 + i) * nx + c0,
                          bytes, &bars[st]);
        } else {
            mbar_expect_tx(&bars[st], ADV_STAGE_DOUBLES * sizeof(double));
            tma_load_2d(dst, map, xs, jy0 + b * ADV_R, &bars[st]);
        }
        issued = b + 1;
    }

    __device__ __forceinline__ void run_task(int task) {
        const int nx = p.c.nx, ny = p.c.ny;
        const int strip = task % p.nstrips, chunk = task / p.nstrips;
        // A warp draws tasks in increasing order, so its earlier tasks lie in
        // lower row chunks (every cell there has a smaller flat index than
        // every cell here: an equal peak here cannot be the first one) or in
        // this same chunk, where it can: then equal values are examined too.
        incl = chunk == last_chunk;
        last_chunk = chunk;
        x0 = strip * ADV_WOUT;
        xs = x0 - ADV_KH;
        xl = xs + 4 * lane;
        if (chunk < p.nA) {
            y0 = p.row_lo + chunk * p.H;
            y1 = y0 + p.H;
        } else if (chunk < p.nA + p.nB) {
            y0 = p.Ya + (chunk - p.nA) * p.Hb;
            y1 = min(y0 + p.Hb, p.Yb);
        } else {
            y0 = p.Yb + (chunk - p.nA - p.nB) * p.H;
            y1 = min(y0 + p.H, p.row_hi);
        }
        jy0 = max(y0 - K, 0);
        jy0 -= jy0 % 3;
        jend = min(y1 + K, ny);
        nbox = (jend - jy0 + ADV_R - 1) / ADV_R;
        edge = (xs <= 0) || (xs + ADV_COLS > nx - 1);
        own_all = owned_lane();
        // With nx a multiple of 4 every lane lies wholly on or off the field;
        // the mirror lanes are the lane before column 0 and the lane at nx.
        mir = edge && p.st256 && p.c.bc == 0;
        mlane = mir && (xl == -V || xl == nx);
        msrc = !mlane ? lane : (xl < 0 ? lane + 1 : lane - 1);
        fast_ok = (!edge || mir) && p.st256 && p.c.same_T;
        src_strip = !(xs + ADV_COLS <= p.bandx_lo || xs > p.bandx_hi);
        issued = 0;
        if constexpr (TMA) {
            if (lane == 0) {
                const int pre = min(ADV_S, nbox);
                for (int b = 0; b < pre; ++b) issue(b);
            }
        }
        const int jlast = y1 - 1 + K;
        // per-box thresholds change only when an exact pass moves a peak
        if constexpr (REDUCE) set_thresholds();
        for (int b = 0, j = jy0; j <= jlast && !failed; ++b, j += ADV_R) {
            const double* st = nullptr;
            if (j < jend) {
                st = wait_box(b);
                if (failed) break;
            }
            // computed rows of this box: j-K .. j+1 over all levels
            const bool fast = fast_ok && j - K >= 1 && j + 1 <= ny - 2 &&
                              (!src_strip || j + 1 < p.band_lo || j - K > p.band_hi);
            if (fast && j < jend) {
                if constexpr (SQM == 2) {
                    if (h.sq) fast_box<true>(j, st);
                    else      fast_box<false>(j, st);
                } else {
                    fast_box<SQM == 1>(j, st);
                }
            } else {
                general_row<0>(j, st, jlast);
                general_row<1>(j + 1, st, jlast);
                general_row<2>(j + 2, st, jlast);
            }
            if constexpr (REDUCE) resolve_box(j);
            if constexpr (TMA) {
                if (j < jend) {
                    __syncwarp();
                    if (lane == 0 && b + ADV_S < nbox) {
                        // order this warp's reads of the stage before the refill
                        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                        issue(b + ADV_S);
                    }
                }
            }
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

    // Wait for box b; returns its stage (TMA) or null (direct loads).
    __device__ __forceinline__ const double* wait_box(int b) {
        if constexpr (TMA) {
            const uint32_t g = gbox + b;
            const int st = g % ADV_S;
            const bool ok = mbar_wait_bounded(&bars[st], (g / ADV_S) & 1);
            if (!__all_sync(0xffffffffu, ok)) {
                if (lane == 0 && p.err) atomicOr(p.err, 1u);
                failed = true;
                return nullptr;
            }
            return stages + st * ADV_STAGE_DOUBLES;
        } else {
            return nullptr;
        }
    }

    // Level-0 row jj (row P of the current box) into dst.
    template <int P>
    __device__ __forceinline__ void load_row0(int jj, const double* st, double* dst) {
        if constexpr (TMA) {
            const double* src = st + P * ADV_COLS + 4 * lane;
            const double2 a = *reinterpret_cast<const double2*>(src);
            const double2 b2 = *reinterpret_cast<const double2*>(src + 2);
            dst[0] = a.x; dst[1] = a.y; dst[2] = b2.x; dst[3] = b2.y;
        } else {
            const int nx = p.c.nx;
            const double* rowp = p.Tin + (size_t)jj * nx;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const int x = xl + v;
                dst[v] = (x >= 0 && x < nx) ? __ldg(rowp + x) : 0.0;
            }
        }
    }

    // Window of level t (t = 0..K-1).
    template <int T>
    __device__ __forceinline__ double (&win())[3][V] {
        if constexpr (T == 0) return w0;
        else return w[T - 1];
    }

    // x neighbours of the lane's first and last cell.
    __device__ __forceinline__ void neighbours(const double* ce, double& Lo, double& Ro) {
        Lo = __shfl_up_sync(0xffffffffu, ce[V - 1], 1);
        Ro = __shfl_down_sync(0xffffffffu, ce[0], 1);
    }

    // ---- fast body -------------------------------------------------------
    // A mirror lane takes its neighbour lane's cells in reverse order (the
    // mirror image about the field edge); other lanes keep theirs.
    __device__ __forceinline__ void mirror_fix(double* v) {
        double m[V];
#pragma unroll
        for (int i = 0; i < V; ++i) m[i] = __shfl_sync(0xffffffffu, v[i], msrc);
        if (mlane) {
#pragma unroll
            for (int i = 0; i < V; ++i) v[i] = m[V - 1 - i];
        }
    }

    template <bool SQ>
    __device__ __forceinline__ void fast_box(int j, const double* st) {
        fast_row<0, SQ>(j, st);
        fast_row<1, SQ>(j + 1, st);
        fast_row<2, SQ>(j + 2, st);
    }

    template <int P, bool SQ>
    __device__ __forceinline__ void fast_row(int jj, const double* st) {
        load_row0<P>(jj, st, win<0>()[P]);
        if (mir) mirror_fix(win<0>()[P]);
        fast_level<P, 1, SQ>(jj);
    }

    template <int P, int T, bool SQ>
    __device__ __forceinline__ void fast_level(int jj) {
        if constexpr (T <= K) {
            constexpr int su = mod3(P - T - 1), sc = mod3(P - T), sd = mod3(P - T + 1);
            double (&wn)[3][V] = win<T - 1>();
            const double* up = wn[su];
            const double* ce = wn[sc];
            const double* dn = wn[sd];
            double Lo, Ro;
            neighbours(ce, Lo, Ro);
            double nv[V];
            nv[0] = cell_core<SQ>(ce[0], Lo, ce[1], up[0], dn[0], h);
            nv[1] = cell_core<SQ>(ce[1], ce[0], ce[2], up[1], dn[1], h);
            nv[2] = cell_core<SQ>(ce[2], ce[1], ce[3], up[2], dn[2], h);
            nv[3] = cell_core<SQ>(ce[3], ce[2], Ro, up[3], dn[3], h);
            const int r = jj - T;
            // Rows outside [y0, y1) are this chunk's halo: computed (their
            // values only ever feed other halo rows) but not stored or reduced.
            const bool owned_row = r >= y0 && r < y1;
            if constexpr (T < K) {
                double (&wo)[3][V] = win<T>();
#pragma unroll
                for (int v = 0; v < V; ++v) wo[sc][v] = nv[v];
            } else {
                st_global_v4_pred(p.Tout + (size_t)r * p.c.nx + xl, nv, owned_row && own_all);
            }
            // Only owned rows are tested (an infinite threshold elsewhere, so
            // no branch splits the box): the first halo rows of a task are
            // computed from window slots that still hold the warp's previous
            // task (values of no use here, which would only trigger empty
            // exact passes).
            if constexpr (REDUCE) row_stats_fast<T - 1, P>(nv, owned_row);
            fast_level<P, T + 1, SQ>(jj);
        }
    }

    // ---- general body ----------------------------------------------------
    template <int P>
    __device__ __forceinline__ void general_row(int jj, const double* st, int jlast) {
        if (jj > jlast) return;
        if (jj < jend) {
            load_row0<P>(jj, st, win<0>()[P]);
            if (mir) mirror_fix(win<0>()[P]);
        }
        general_level<P, 1>(jj);
    }

    template <int P, int T>
    __device__ __forceinline__ void general_level(int jj) {
        if constexpr (T <= K) {
            constexpr int su = mod3(P - T - 1), sc = mod3(P - T), sd = mod3(P - T + 1);
            const int ny = p.c.ny;
            const int r = jj - T;
            const int lo = max(y0 - K + T, 0);
            const int hi = min(y1 - 1 + K - T, ny - 1);
            if (r >= lo && r <= hi) {
                double (&wn)[3][V] = win<T - 1>();
                // Mirror edges: the ghost row is the centre row.  The slot of
                // row -1 (row 2) is not filled yet and the slot of row ny
                // (row ny-3) is no longer needed, so both can be overwritten.
                if (r == 0) {
#pragma unroll
                    for (int v = 0; v < V; ++v) wn[su][v] = wn[sc][v];
                }
                if (r == ny - 1) {
#pragma unroll
                    for (int v = 0; v < V; ++v) wn[sd][v] = wn[sc][v];
                }
                double nv[V];
                compute_row_general(wn[su], wn[sc], wn[sd], r, p.las[T - 1], nv);
                // keep the mirror lanes exact for later fast boxes (the source
                // term and the edge patch are not mirror-symmetric off the field)
                if constexpr (T < K) {
                    if (mir) mirror_fix(nv);
                }
                const bool owned_row = r >= y0 && r < y1;
                if constexpr (T < K) {
                    double (&wo)[3][V] = win<T>();
#pragma unroll
                    for (int v = 0; v < V; ++v) wo[sc][v] = nv[v];
                } else {
                    if (owned_row) store_row(r, nv);
                }
                if constexpr (REDUCE) {
                    if (owned_row) row_stats<T - 1, P>(r, nv, owned_lane(), !edge);
                }
            }
            general_level<P, T + 1>(jj);
        }
    }

    // The general body's cell update in this strip's form.
    __device__ __forceinline__ double gcore(double T, double L, double R, double U, double D) {
        if constexpr (SQM == 2) return h.sq ? cell_core<true>(T, L, R, U, D, h)
                                            : cell_core<false>(T, L, R, U, D, h);
        else return cell_core<SQM == 1>(T, L, R, U, D, h);
    }
    __device__ __forceinline__ double gcore_src(double T, double L, double R, double U, double D,
                                                double S) {
        if constexpr (SQM == 2) return h.sq ? cell_core_src<true>(T, L, R, U, D, S, h)
                                            : cell_core_src<false>(T, L, R, U, D, S, h);
        else return cell_core_src<SQM == 1>(T, L, R, U, D, S, h);
    }

    __device__ __forceinline__ bool owned_lane() const {
        return xl >= x0 && xl < x0 + ADV_WOUT && xl < p.c.nx;
    }

    __device__ __forceinline__ void compute_row_general(const double* up, const double* ce,
                                                        const double* dn, int r,
                                                        const LaserSub& las, double* nv) {
        const Coef& c = p.c;
        const int nx = c.nx, ny = c.ny;
        if (c.bc == 1 && (r == 0 || r == ny - 1)) {
#pragma unroll
            for (int v = 0; v < V; ++v) nv[v] = c.T_edge;
            return;
        }
        double Lo, Ro;
        neighbours(ce, Lo, Ro);
        double L[V] = {Lo, ce[0], ce[1], ce[2]};
        double R[V] = {ce[1], ce[2], ce[3], Ro};
        if (edge) {
#pragma unroll
            for (int v = 0; v < V; ++v) {
                if (xl + v == 0) L[v] = ce[v];
                if (xl + v == nx - 1) R[v] = ce[v];
            }
        }
        const double yd = __dsub_rn(__dmul_rn((double)(r + p.row0), c.dy), las.y_l);
        const double dy2 = __dmul_rn(yd, yd);
        const bool src = las.cs != 0.0 && dy2 < c.r2_cut && src_strip;
        double4 S4 = make_double4(0.0, 0.0, 0.0, 0.0);
        if (src) S4 = source4(xl, dy2, las.x_l, las.cs, c.dx, c.m2r, c.r2_cut);
        const double S[V] = {S4.x, S4.y, S4.z, S4.w};
        if (c.same_T) {
#pragma unroll
            for (int v = 0; v < V; ++v)
                nv[v] = src ? gcore_src(ce[v], L[v], R[v], up[v], dn[v], S[v])
                            : gcore(ce[v], L[v], R[v], up[v], dn[v]);
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
                nv[v] = cell_update(ce[v], L[v], R[v], up[v], dn[v], S[v], c);
        }
        if (edge && c.bc == 1) {
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (xl + v == 0 || xl + v == nx - 1) nv[v] = c.T_edge;
        }
    }

    __device__ __forceinline__ void store_row(int r, const double* nv) {
        double* dst = p.Tout + (size_t)r * p.c.nx + xl;
        if constexpr (TMA) {
            // even nx and a 4-aligned lane start: pairs share ownership
            if (xl >= x0 && xl < x0 + ADV_WOUT) {
                if (p.st256 && xl + 4 <= p.c.nx) {
                    st_global_v4(dst, nv[0], nv[1], nv[2], nv[3]);
                } else {
                    if (xl < p.c.nx) *reinterpret_cast<double2*>(dst) = make_double2(nv[0], nv[1]);
                    if (xl + 2 < p.c.nx)
                        *reinterpret_cast<double2*>(dst + 2) = make_double2(nv[2], nv[3]);
                }
            }
        } else {
#pragma unroll
            for (int v = 0; v < V; ++v)
                if (xl + v >= x0 && xl + v < x0 + ADV_WOUT && xl + v < p.c.nx) dst[v] = nv[v];
        }
    }

    // Reduction, two tiers.  Every cell is tested against a per-box threshold
    // thr = min(lane peak, Tm) (+inf for lanes owning no cell): one FP64
    // compare folded into a predicate, no select.  Only a box in which some
    // lane crossed its threshold -- the first box of a lane, or cells near
    // the laser -- runs the exact pass: the crossed levels' rows are staged in
    // shared memory and one compact routine updates the lane peak, its index
    // and the molten rows.  NaN never crosses (strict '>'), as in the
    // reference.
    __device__ __forceinline__ void set_thresholds() {
        const bool ol = owned_lane();
#pragma unroll
        for (int t = 0; t < K; ++t) {
            double tm = rs->tmx[t][lane];
            // inclusive task: the largest double below the peak, so that
            // equal values cross too (peaks are positive temperatures; a
            // non-positive peak leaves the threshold where it is)
            if (incl && tm > 0.0) tm = __longlong_as_double(__double_as_longlong(tm) - 1);
            const double a = (tm < p.c.Tm) ? tm : p.c.Tm;
            thr[t] = ol ? a : INFINITY;
        }
    }

    // full: the lane's four cells are all inside the grid.  A last-level
    // (T == K-1) row that crosses the threshold on owned cells is staged in
    // shared memory (box row P) for the exact pass: the last level has no
    // register window to stage from, and a row that does not cross can hold
    // neither a new peak nor a molten cell.
    template <int T, int P>
    __device__ __forceinline__ void row_stats(int r, const double* nv, bool own, bool full) {
        bool rh = false;
#pragma unroll
        for (int v = 0; v < V; ++v) {
            // !(v <= thr): the same test as v > thr for numbers, and true for
            // NaN, so a non-finite cell reaches the exact pass (which flags it)
            if (full) rh = rh | !(nv[v] <= thr[T]);
            else      rh = rh | (own && xl + v < p.c.nx && !(nv[v] <= thr[T]));
        }
        hit[T] = hit[T] | rh;
        if constexpr (T == K - 1) {
            if (rh && own) {
                double2* d = reinterpret_cast<double2*>(&rs->box[P][lane][0]);
                d[0] = make_double2(nv[0], nv[1]);
                d[1] = make_double2(nv[2], nv[3]);
                kmask |= 1u << P;
            }
        }
    }

    // The fast body's test: whole lanes, rows outside the task's own rows
    // against an infinite threshold.
    template <int T, int P>
    __device__ __forceinline__ void row_stats_fast(const double* nv, bool owned_row) {
        const double th = owned_row ? thr[T] : INFINITY;
        bool rh = false;
#pragma unroll
        for (int v = 0; v < V; ++v) rh = rh | !(nv[v] <= th);
        hit[T] = hit[T] | rh;
        if constexpr (T == K - 1) {
            if (rh && own_all && owned_row) {
                double2* d = reinterpret_cast<double2*>(&rs->box[P][lane][0]);
                d[0] = make_double2(nv[0], nv[1]);
                d[1] = make_double2(nv[2], nv[3]);
                kmask |= 1u << P;
            }
        }
    }

    // Exact update of level T (1..K) from three of its rows (row j + P - T
    // in x[P]; only rows set in `rows` take part): the lane's first maximal
    // owned cell in flat-index order, the molten-row extent, non-finite
    // cells.  Each lane reads only its own values, so no warp barrier is
    // needed around the scan.
    template <int T>
    __device__ __forceinline__ void exact_rows(const double (&x)[3][V], int j, unsigned rows) {
        const int nx = p.c.nx;
        const bool ol = owned_lane();
        double m = -INFINITY;
        long long a = -1;
        bool nonfinite = false;
#pragma unroll
        for (int P = 0; P < 3; ++P) {
            const int r = j + P - T;
            const bool cand = ((rows >> P) & 1u) && r >= y0 && r < y1 && ol;
            bool hot = false;
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const bool ok = cand && xl + v < nx;
                const double val = x[P][v];
                // rows, then columns, ascend: the first maximum has the
                // smallest flat index (NaN never wins)
                const bool take = ok && val > m;
                m = take ? val : m;
                a = take ? (long long)(r + p.row0) * nx + xl + v : a;
                hot |= ok && val > p.c.Tm;
                nonfinite |= ok && !(fabs(val) < INFINITY);
            }
            if (__any_sync(0xffffffffu, hot) && lane == 0) {
                rs->ymn[T - 1] = min(rs->ymn[T - 1], r + p.row0);
                rs->ymx[T - 1] = max(rs->ymx[T - 1], r + p.row0);
            }
        }
        // a NaN or infinite temperature is reported, never trapped on; the
        // peak keeps the reference rule (NaN never wins)
        if (__any_sync(0xffffffffu, nonfinite) && lane == 0 && p.err) atomicOr(p.err, 2u);
        const double pk = rs->tmx[T - 1][lane];
        // an equal peak (inclusive task) moves only to a smaller index
        if (m > pk || (incl && m == pk && a < rs->arg[T - 1][lane])) {
            rs->tmx[T - 1][lane] = m;
            rs->arg[T - 1][lane] = a;
        }
    }

    // Levels 1..K-1 straight from their register windows (the box's three
    // rows of level T sit in slots mod3(P - T)).
    template <int T>
    __device__ __forceinline__ void resolve_levels(unsigned bits, int j) {
        if constexpr (T < K) {
            if ((bits >> (T - 1)) & 1u) {
                const double (&wn)[3][V] = win<T>();
                double x[3][V];
#pragma unroll
                for (int P = 0; P < 3; ++P)
#pragma unroll
                    for (int v = 0; v < V; ++v) x[P][v] = wn[mod3(P - T)][v];
                exact_rows<T>(x, j, 7u);
            }
            resolve_levels<T + 1>(bits, j);
        }
    }

    __device__ __forceinline__ void resolve_box(int j) {
        unsigned bits = 0;
#pragma unroll
        for (int t = 0; t < K; ++t) {
            bits |= hit[t] ? (1u << t) : 0u;
            hit[t] = false;
        }
        bits = __reduce_or_sync(0xffffffffu, bits);
        if (bits == 0u) { kmask = 0u; return; }
        // the last level from the rows that row_stats staged (those of kmask:
        // the others crossed no threshold, so every value there is at most
        // the lane's peak so far and none is molten)
        if ((bits >> (K - 1)) & 1u) {
            double x[3][V];
#pragma unroll
            for (int P = 0; P < 3; ++P) {
                const double2* b = reinterpret_cast<const double2*>(&rs->box[P][lane][0]);
                const double2 u = b[0], w2 = b[1];
                x[P][0] = u.x; x[P][1] = u.y; x[P][2] = w2.x; x[P][3] = w2.y;
            }
            exact_rows<K>(x, j, kmask);
        }
        kmask = 0u;
        resolve_levels<1>(bits, j);
        __syncwarp();
        set_thresholds();
    }
};

// Resident CTAs per SM the register budget is sized for.  The staged kernels
// hold 48 KB of stages plus 15-21 KB of reduction state per CTA, so shared
// memory admits three CTAs whatever K is; a tighter register cap would only
// spill.
template <int K>
struct AdvOcc { static constexpr int min_ctas = 3; };

template <int K, bool TMA, bool REDUCE, bool SQ>
__global__ void __launch_bounds__(ADV_WARPS * 32, AdvOcc<K>::min_ctas)
advance_kernel(const __grid_constant__ CUtensorMap map, const __grid_constant__ AdvParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ Partial red[ADV_WARPS][K];
    __shared__ unsigned int s_last;
    __shared__ __align__(16) RedSmem<K> s_red[REDUCE ? ADV_WARPS : 1];

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    double* stages = reinterpret_cast<double*>(smem) + wid * (ADV_S * ADV_STAGE_DOUBLES);
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        smem + size_t(ADV_WARPS) * ADV_S * ADV_STAGE_DOUBLES * sizeof(double)) + wid * ADV_S;

    if constexpr (TMA) {
        if (lane == 0) {
            for (int s = 0; s < ADV_S; ++s) mbar_init(&bars[s], 1);
            fence_mbar_init();
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncwarp();
    }

    WarpStrip<K, TMA, REDUCE, false, SQ ? 1 : 0> ws(p, &map, stages, bars, lane,
                                                    &s_red[REDUCE ? wid : 0]);
    if (p.tasks) {
        // dynamic: lane 0 draws the next task for the warp
        for (;;) {
            unsigned int t = 0;
            if (lane == 0) t = atomicAdd(p.tasks, 1u);
            t = __shfl_sync(0xffffffffu, t, 0);
            if (t >= (unsigned int)p.ntasks) break;
            ws.run_task((int)t);
            if (ws.failed) break;
        }
    } else {
        for (int task = blockIdx.x * ADV_WARPS + wid; task < p.ntasks;
             task += gridDim.x * ADV_WARPS) {
            ws.run_task(task);
            if (ws.failed) break;
        }
    }

    const long long N = (long long)p.c.nx * p.gny;
    if constexpr (REDUCE) {
#pragma unroll
        __syncwarp();
        for (int t = 0; t < K; ++t) {
            double tm = s_red[wid].tmx[t][lane];
            long long ag = s_red[wid].arg[t][lane];
            int mn = s_red[wid].ymn[t], mx = s_red[wid].ymx[t];
            partial_warp_reduce(tm, ag, mn, mx);
            if (lane == 0) red[wid][t] = Partial{tm, ag, mn, mx};
        }
        __syncthreads();
        if (threadIdx.x < K) {
            const int t = threadIdx.x;
            double tm = -1.0; long long ag = N; int mn = p.gny, mx = -1;
            for (int w = 0; w < ADV_WARPS; ++w)
                partial_take(tm, ag, mn, mx, red[w][t].tmax, red[w][t].arg,
                             red[w][t].ymin, red[w][t].ymax);
            if (p.ref_out) p.ref_out[blockIdx.x] = Partial{tm, ag, mn, mx};
            else if (p.ring) p.scratch[(size_t)blockIdx.x * K + t] = Partial{tm, ag, mn, mx};
        }
        if (p.ref_out) {
            // Reference layout: the caller finalizes ref_nparts entries, so
            // every entry past this grid's must hold the neutral element.
            const Partial neutral{-1.0, N, p.gny, -1};
            for (long long i = gridDim.x + (long long)blockIdx.x * blockDim.x + threadIdx.x;
                 i < p.ref_nparts; i += (long long)gridDim.x * blockDim.x)
                p.ref_out[i] = neutral;
        }
    }
    if (!p.counter) return;
    // Last CTA: finalize the per-step Partials and re-arm the counters.
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0)
        s_last = (atomicAdd(p.counter, 1u) == gridDim.x - 1) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if constexpr (REDUCE) {
        if (p.ring) {
            // The whole GPU waits on this CTA: every thread issues the loads
            // of all its CTA records (FIN_U CTAs x K levels) before combining
            // any, so the pass costs about one L2 round trip per FIN_U
            // records, not one per record.  The combine is commutative (ties
            // to the smaller index), so the order does not change the result.
            constexpr int FIN_U = 4;
            double tm[K]; long long ag[K]; int mn[K], mx[K];
#pragma unroll
            for (int t = 0; t < K; ++t) { tm[t] = -1.0; ag[t] = N; mn[t] = p.gny; mx[t] = -1; }
            for (int i0 = threadIdx.x; i0 < (int)gridDim.x; i0 += blockDim.x * FIN_U) {
                Partial q[FIN_U][K];
#pragma unroll
                for (int u = 0; u < FIN_U; ++u) {
                    const int i = i0 + u * (int)blockDim.x;
#pragma unroll
                    for (int t = 0; t < K; ++t) {
                        if (i < (int)gridDim.x) {
                            const Partial* r = &p.scratch[(size_t)i * K + t];
                            q[u][t] = Partial{__ldcg(&r->tmax), __ldcg(&r->arg),
                                              __ldcg(&r->ymin), __ldcg(&r->ymax)};
                        } else {
                            q[u][t] = Partial{-1.0, N, p.gny, -1};
                        }
                    }
                }
#pragma unroll
                for (int u = 0; u < FIN_U; ++u)
#pragma unroll
                    for (int t = 0; t < K; ++t)
                        partial_take(tm[t], ag[t], mn[t], mx[t], q[u][t].tmax, q[u][t].arg,
                                     q[u][t].ymin, q[u][t].ymax);
            }
            __syncthreads();
#pragma unroll
            for (int t = 0; t < K; ++t) {
                partial_warp_reduce(tm[t], ag[t], mn[t], mx[t]);
                if (lane == 0) red[wid][t] = Partial{tm[t], ag[t], mn[t], mx[t]};
            }
            __syncthreads();
            if (threadIdx.x < K) {
                const int t = threadIdx.x;
                double a = -1.0; long long b = N; int c1 = p.gny, d1 = -1;
                for (int w = 0; w < ADV_WARPS; ++w)
                    partial_take(a, b, c1, d1, red[w][t].tmax, red[w][t].arg,
                                 red[w][t].ymin, red[w][t].ymax);
                p.ring[t] = Partial{a, b, c1, d1};
            }
        }
    }
    if (threadIdx.x == 0) {
        *p.counter = 0u;
        if (p.tasks) *p.tasks = 0u;
    }
}

}  // namespace lpbf_b200
