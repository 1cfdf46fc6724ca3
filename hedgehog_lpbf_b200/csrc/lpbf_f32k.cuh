// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// FP32 compensated variant of the temporally blocked step.
//
// The field is held as two f32 arrays, hi and lo, with the temperature
// T = hi + lo (lo the rounding remainder of hi, |lo| <= ulp(hi)/2).  Per cell
// and step:
//   * neighbour differences are formed on the pairs,
//       (R - T) = (R.hi - T.hi) + (R.lo - T.lo),
//     the hi difference being exact for neighbours within a factor of two,
//     so the Laplacian keeps ~48 significant bits;
//   * the loss terms and the increment are f32; the Gaussian source is
//     evaluated in FP64 (as in the FP64 path) and rounded once;
//   * the increment is added with an error-free sum (Fast2Sum: the
//     increment is never larger than T), and the rounding error is carried
//     in lo (Kahan-compensated accumulation).
// Memory traffic per cell-update equals the FP64 path's (hi + lo = 8 bytes).
//
// Structure (warp tasks, lanes, TMA pipeline, wavefront, fast/general boxes,
// two-tier reduction) follows lpbf_advance.cuh; the per-step Partials are
// computed on T = (double)hi + (double)lo, which is exact.
//
// The same kernel with COMP = false is the plain FP32 field: one f32 array,
// each step's update rounded once (the FP64 step's fused form in f32, the
// source still evaluated in FP64), 8 bytes per cell-update; no lo array is
// loaded, staged, shuffled or stored.
// ---------------------------------------------------------------------------
#pragma once
#include <stddef.h>

#include "lpbf_advance.cuh"

namespace lpbf_b200 {

// floats per TMA stage: the hi box, then (compensated field) the lo box
template <bool COMP>
constexpr int fk_stage_floats() { return (COMP ? 2 : 1) * ADV_R * ADV_COLS; }
template <bool COMP>
constexpr size_t fk_smem_bytes() {
    return size_t(ADV_WARPS) * ADV_S * fk_stage_floats<COMP>() * sizeof(float)
           + size_t(ADV_WARPS) * ADV_S * sizeof(uint64_t);
}

// 16-byte store issued under a predicate (no branch).  It carries a
// "memory" clobber: the exact reduction reads level-K values back from the
// output field, and those loads must stay after the stores.
__device__ __forceinline__ void st_global_v4f_pred(float* p, const float* v, bool pred) {
    asm volatile("{\n\t.reg .pred q;\n\tsetp.ne.b32 q, %5, 0;\n\t"
                 "@q st.global.v4.f32 [%0], {%1, %2, %3, %4};\n\t}"
                 :: "l"(p), "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "r"((int)pred)
                 : "memory");
}

struct FkCoef {
    float ax, ay, cls, crad;
    float Ta_hi, Ta_lo, Ta4;       // linear-loss reference T as a pair; Ta4 = f4(Tamb)
    float Tedge_hi, Tedge_lo;
    float clsTa;                   // c_ls * (linear-loss reference T), rounded once
};

struct FkParams {
    Coef c;                        // geometry, source and reduction constants
    FkCoef f;
    LaserSub las[KMAX];
    int band_lo, band_hi, bandx_lo, bandx_hi;
    int nstrips, nchunks, H, ntasks;
    int nA, nB, Hb, Ya, Yb;        // band-split chunks, as in AdvParams
    float* Thi_out;
    float* Tlo_out;
    Partial* ring;
    Partial* scratch;
    unsigned int* counter;
    unsigned int* tasks;
    unsigned int* err;
};

// T^4 of a pair, in f32 (the same expression for cells and for Tamb, so the
// radiation difference is exactly zero at equilibrium).
__device__ __host__ __forceinline__ float fk_pow4(float hi, float lo) {
    const float t = hi + lo;
    const float t2 = t * t;
    return t2 * t2;
}

// One compensated cell update.  (th, tl) centre; neighbour pairs; S_dt the
// dt-scaled FP64 source rounded to f32.  SQ (ax == ay): one Laplacian of the
// hi parts plus one of the lo parts, the source and loss in the same fused
// chain; otherwise the x and y terms apart.  T^4 - Ta^4 is one fused
// multiply-add.
template <bool SQ>
__device__ __forceinline__ void fk_cell(float th, float tl, float Lh, float Ll, float Rh,
                                        float Rl, float Uh, float Ul, float Dh, float Dl,
                                        float S, const FkCoef& f, float& oh, float& ol) {
    const float da = __fsub_rn(th, f.Ta_hi) + (tl - f.Ta_lo);
    const float t = th + tl;
    const float t2 = t * t;
    const float e4 = fmaf(t2, t2, -f.Ta4);
    const float loss = fmaf(f.crad, e4, __fmul_rn(f.cls, da));
    float d;
    if constexpr (SQ) {
        const float lh = (__fsub_rn(Rh, th) + __fsub_rn(Lh, th)) +
                         (__fsub_rn(Dh, th) + __fsub_rn(Uh, th));
        const float ll = fmaf(-4.0f, tl, (Rl + Ll) + (Dl + Ul));
        d = fmaf(f.ax, lh + ll, __fsub_rn(S, loss));
    } else {
        const float lx = ((__fsub_rn(Rh, th) + __fsub_rn(Lh, th)) + ((Rl - tl) + (Ll - tl)));
        const float ly = ((__fsub_rn(Dh, th) + __fsub_rn(Uh, th)) + ((Dl - tl) + (Ul - tl)));
        d = fmaf(f.ax, lx, fmaf(f.ay, ly, __fsub_rn(S, loss)));
    }
    // th + d with its rounding error (Fast2Sum, exact for |d| <= |th|: a
    // step's increment is far smaller than the temperature), the error
    // folded into lo, then renormalised
    const float s = __fadd_rn(th, d);
    const float err = __fsub_rn(d, __fsub_rn(s, th));
    const float lo = __fadd_rn(tl, err);
    oh = __fadd_rn(s, lo);
    ol = __fsub_rn(lo, __fsub_rn(oh, s));
}

// One plain f32 cell update: the FP64 step's form in f32.  T^4 - Ta^4 and
// c_ls T - c_ls Ta are each one fused multiply-add and the loss enters the
// increment's fused chain (SQ: one Laplacian (R + L) + (U + D) - 4T).  The
// Laplacian of a uniform field is exactly zero and its loss at Tamb far below
// half an ulp of T, so a uniform field at Tamb stays exactly uniform.
// SRC: the cell's source increment S is added to the net change before T.
template <bool SQ, bool SRC>
__device__ __forceinline__ float f32_cell(float t, float L, float R, float U, float D, float S,
                                          const FkCoef& f) {
    const float t2 = __fmul_rn(t, t);
    const float e4 = fmaf(t2, t2, -f.Ta4);
    const float loss = fmaf(f.crad, e4, fmaf(f.cls, t, -f.clsTa));
    float net;
    if constexpr (SQ) {
        const float lap = fmaf(-4.0f, t, __fadd_rn(__fadd_rn(R, L), __fadd_rn(U, D)));
        net = fmaf(f.ax, lap, -loss);
    } else {
        const float lx = fmaf(-2.0f, t, __fadd_rn(R, L));
        const float ly = fmaf(-2.0f, t, __fadd_rn(U, D));
        net = fmaf(f.ax, lx, fmaf(f.ay, ly, -loss));
    }
    if constexpr (SRC) net = __fadd_rn(net, S);
    return __fadd_rn(t, net);
}

// (a.hi, a.lo) > (b.hi, b.lo) for canonical pairs.
__device__ __forceinline__ bool fk_gt(float ah, float al, float bh, float bl) {
    return ah > bh || (ah == bh && al > bl);
}

template <int K, bool REDUCE, bool SQ, bool COMP>
struct FkStrip {
    static constexpr int V = ADV_V;
    static constexpr int STAGE = fk_stage_floats<COMP>();

    const FkParams& p;
    const CUtensorMap* map_hi;
    const CUtensorMap* map_lo;
    float* stages;
    uint64_t* bars;
    uint32_t gbox;
    const int lane;

    int x0, xs, xl, y0, y1, jy0, jend, nbox, issued;
    bool edge, failed, src_strip;

    float wh0[3][V], wl0[3][V];
    float wh[K > 1 ? K - 1 : 1][3][V], wl[K > 1 ? K - 1 : 1][3][V];
    float thr_h[K], thr_l[K];
    bool hit[K];
    double (*s_tmx)[32];
    long long (*s_arg)[32];
    int* s_ymn;
    int* s_ymx;
    float (*s_box)[32][2 * ADV_V];     // [3][32][hi0..3, lo0..3]

    __device__ __forceinline__ FkStrip(const FkParams& p_, const CUtensorMap* mh,
                                       const CUtensorMap* ml, float* st, uint64_t* b, int ln,
                                       double (*tm)[32], long long (*ar)[32], int* mn, int* mx,
                                       float (*bx)[32][2 * ADV_V])
        : p(p_), map_hi(mh), map_lo(ml), stages(st), bars(b), gbox(0), lane(ln), failed(false),
          s_tmx(tm), s_arg(ar), s_ymn(mn), s_ymx(mx), s_box(bx) {
        if constexpr (REDUCE) {
            const long long N = (long long)p.c.nx * p.c.ny;
#pragma unroll
            for (int t = 0; t < K; ++t) {
                hit[t] = false;
                s_tmx[t][lane] = -1.0;
                s_arg[t][lane] = N;
                if (lane == 0) { s_ymn[t] = p.c.ny; s_ymx[t] = -1; }
            }
        }
        __syncwarp();
    }

    __device__ __forceinline__ void issue(int b) {
        const uint32_t g = gbox + b;
        const int st = g % ADV_S;
        float* dst = stages + st * STAGE;
        mbar_expect_tx(&bars[st], STAGE * sizeof(float));
        tma_load_2d(dst, map_hi, xs, jy0 + b * ADV_R, &bars[st]);
        if constexpr (COMP)
            tma_load_2d(dst + ADV_R * ADV_COLS, map_lo, xs, jy0 + b * ADV_R, &bars[st]);
        issued = b + 1;
    }

    __device__ __forceinline__ bool owned_lane() const {
        return xl >= x0 && xl < x0 + ADV_WOUT && xl < p.c.nx;
    }

    __device__ __forceinline__ void run_task(int task) {
        const int nx = p.c.nx, ny = p.c.ny;
        const int strip = task % p.nstrips, chunk = task / p.nstrips;
        x0 = strip * ADV_WOUT;
        xs = x0 - ADV_KH;
        xl = xs + 4 * lane;
        if (chunk < p.nA) {
            y0 = chunk * p.H;
            y1 = y0 + p.H;
        } else if (chunk < p.nA + p.nB) {
            y0 = p.Ya + (chunk - p.nA) * p.Hb;
            y1 = min(y0 + p.Hb, p.Yb);
        } else {
            y0 = p.Yb + (chunk - p.nA - p.nB) * p.H;
            y1 = min(y0 + p.H, ny);
        }
        jy0 = max(y0 - K, 0);
        jy0 -= jy0 % 3;
        jend = min(y1 + K, ny);
        nbox = (jend - jy0 + ADV_R - 1) / ADV_R;
        edge = (xs <= 0) || (xs + ADV_COLS > nx - 1);
        src_strip = !(xs + ADV_COLS <= p.bandx_lo || xs > p.bandx_hi);
        issued = 0;
        if (lane == 0) {
            const int pre = min(ADV_S, nbox);
            for (int b = 0; b < pre; ++b) issue(b);
        }
        const int jlast = y1 - 1 + K;
        // per-box thresholds change only when an exact pass moves a peak
        if constexpr (REDUCE) set_thresholds();
        for (int b = 0, j = jy0; j <= jlast && !failed; ++b, j += ADV_R) {
            const float* st = nullptr;
            if (j < jend) {
                const uint32_t g = gbox + b;
                const int sidx = g % ADV_S;
                const bool ok = mbar_wait_bounded(&bars[sidx], (g / ADV_S) & 1);
                if (!__all_sync(0xffffffffu, ok)) {
                    if (lane == 0) atomicOr(p.err, 1u);
                    failed = true;
                    break;
                }
                st = stages + sidx * STAGE;
            }
            // mirror-edge strips too: row_update patches the edge cells'
            // outer neighbours itself (nx a multiple of 4: whole lanes)
            const bool fast = (!edge || (p.c.bc == 0 && (p.c.nx & 3) == 0)) &&
                              j - K >= 1 && j + 1 <= ny - 2 &&
                              (!src_strip || j + 1 < p.band_lo || j - K > p.band_hi);
            if (fast && j < jend) {
                fast_row<0>(j, st);
                fast_row<1>(j + 1, st);
                fast_row<2>(j + 2, st);
            } else {
                general_row<0>(j, st, jlast);
                general_row<1>(j + 1, st, jlast);
                general_row<2>(j + 2, st, jlast);
            }
            if constexpr (REDUCE) resolve_box(j);
            if (j < jend) {
                __syncwarp();
                if (lane == 0 && b + ADV_S < nbox) {
                    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
                    issue(b + ADV_S);
                }
            }
        }
        if (failed) {
            const int last = __shfl_sync(0xffffffffu, issued, 0);
            for (int b = max(0, last - ADV_S); b < last; ++b) {
                const uint32_t g = gbox + b;
                mbar_wait_bounded(&bars[g % ADV_S], (g / ADV_S) & 1);
            }
        }
        gbox += nbox;
    }

    template <int P>
    __device__ __forceinline__ void load_row0(const float* st) {
        const float4 h = *reinterpret_cast<const float4*>(st + P * ADV_COLS + 4 * lane);
        wh0[P][0] = h.x; wh0[P][1] = h.y; wh0[P][2] = h.z; wh0[P][3] = h.w;
        if constexpr (COMP) {
            const float4 l =
                *reinterpret_cast<const float4*>(st + (ADV_R + P) * ADV_COLS + 4 * lane);
            wl0[P][0] = l.x; wl0[P][1] = l.y; wl0[P][2] = l.z; wl0[P][3] = l.w;
        }
    }

    template <int T>
    __device__ __forceinline__ float (&winh())[3][V] {
        if constexpr (T == 0) return wh0; else return wh[T - 1];
    }
    template <int T>
    __device__ __forceinline__ float (&winl())[3][V] {
        if constexpr (T == 0) return wl0; else return wl[T - 1];
    }

    // One row of level T from the three rows (up, centre, down) of level T-1
    // (plain field: the lo rows are not read and ol is not written).
    __device__ __forceinline__ void row_update(const float* uh, const float* ul, const float* ch,
                                               const float* cl, const float* dh, const float* dl,
                                               const float* S, float* oh, float* ol) {
        if constexpr (!COMP) {
            const float L0 = __shfl_up_sync(0xffffffffu, ch[V - 1], 1);
            const float R3 = __shfl_down_sync(0xffffffffu, ch[0], 1);
            float L[V] = {L0, ch[0], ch[1], ch[2]};
            float R[V] = {ch[1], ch[2], ch[3], R3};
            if (edge) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    if (xl + v == 0) L[v] = ch[v];
                    if (xl + v == p.c.nx - 1) R[v] = ch[v];
                }
            }
#pragma unroll
            for (int v = 0; v < V; ++v)
                oh[v] = S ? f32_cell<SQ, true>(ch[v], L[v], R[v], uh[v], dh[v], S[v], p.f)
                          : f32_cell<SQ, false>(ch[v], L[v], R[v], uh[v], dh[v], 0.0f, p.f);
        } else {
            const float Lh0 = __shfl_up_sync(0xffffffffu, ch[V - 1], 1);
            const float Ll0 = __shfl_up_sync(0xffffffffu, cl[V - 1], 1);
            const float Rh3 = __shfl_down_sync(0xffffffffu, ch[0], 1);
            const float Rl3 = __shfl_down_sync(0xffffffffu, cl[0], 1);
            float Lh[V] = {Lh0, ch[0], ch[1], ch[2]}, Ll[V] = {Ll0, cl[0], cl[1], cl[2]};
            float Rh[V] = {ch[1], ch[2], ch[3], Rh3}, Rl[V] = {cl[1], cl[2], cl[3], Rl3};
            if (edge) {
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    if (xl + v == 0) { Lh[v] = ch[v]; Ll[v] = cl[v]; }
                    if (xl + v == p.c.nx - 1) { Rh[v] = ch[v]; Rl[v] = cl[v]; }
                }
            }
#pragma unroll
            for (int v = 0; v < V; ++v)
                fk_cell<SQ>(ch[v], cl[v], Lh[v], Ll[v], Rh[v], Rl[v], uh[v], ul[v], dh[v],
                            dl[v], S ? S[v] : 0.0f, p.f, oh[v], ol[v]);
        }
    }

    template <int P>
    __device__ __forceinline__ void fast_row(int jj, const float* st) {
        load_row0<P>(st);
        fast_level<P, 1>(jj);
    }

    template <int P, int T>
    __device__ __forceinline__ void fast_level(int jj) {
        if constexpr (T <= K) {
            constexpr int su = mod3(P - T - 1), sc = mod3(P - T), sd = mod3(P - T + 1);
            float (&ah)[3][V] = winh<T - 1>();
            float (&al)[3][V] = winl<T - 1>();
            float oh[V], ol[V];
            row_update(ah[su], al[su], ah[sc], al[sc], ah[sd], al[sd], nullptr, oh, ol);
            const int r = jj - T;
            const bool owned_row = r >= y0 && r < y1;
            finish_level<T, sc>(r, oh, ol, owned_row, true);
            fast_level<P, T + 1>(jj);
        }
    }

    template <int P>
    __device__ __forceinline__ void general_row(int jj, const float* st, int jlast) {
        if (jj > jlast) return;
        if (jj < jend) load_row0<P>(st);
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
                float (&ah)[3][V] = winh<T - 1>();
                float (&al)[3][V] = winl<T - 1>();
                if (r == 0) {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        ah[su][v] = ah[sc][v];
                        if constexpr (COMP) al[su][v] = al[sc][v];
                    }
                }
                if (r == ny - 1) {
#pragma unroll
                    for (int v = 0; v < V; ++v) {
                        ah[sd][v] = ah[sc][v];
                        if constexpr (COMP) al[sd][v] = al[sc][v];
                    }
                }
                float oh[V], ol[V];
                if (p.c.bc == 1 && (r == 0 || r == ny - 1)) {
#pragma unroll
                    for (int v = 0; v < V; ++v) { oh[v] = p.f.Tedge_hi; ol[v] = p.f.Tedge_lo; }
                } else {
                    const LaserSub& las = p.las[T - 1];
                    const double yd = __dsub_rn(__dmul_rn((double)r, p.c.dy), las.y_l);
                    const double dy2 = __dmul_rn(yd, yd);
                    float S[V] = {0.f, 0.f, 0.f, 0.f};
                    if (las.cs != 0.0 && dy2 < p.c.r2_cut && src_strip) {
                        const double4 s4 = source4(xl, dy2, las.x_l, las.cs, p.c.dx, p.c.m2r,
                                                   p.c.r2_cut);
                        S[0] = (float)s4.x; S[1] = (float)s4.y; S[2] = (float)s4.z; S[3] = (float)s4.w;
                    }
                    row_update(ah[su], al[su], ah[sc], al[sc], ah[sd], al[sd], S, oh, ol);
                    if (edge && p.c.bc == 1) {
#pragma unroll
                        for (int v = 0; v < V; ++v)
                            if (xl + v == 0 || xl + v == p.c.nx - 1) {
                                oh[v] = p.f.Tedge_hi; ol[v] = p.f.Tedge_lo;
                            }
                    }
                }
                finish_level<T, sc>(r, oh, ol, r >= y0 && r < y1, !edge);
            }
            general_level<P, T + 1>(jj);
        }
    }

    // Keep the new row in level T's window slot SC (T < K) or store it
    // (T == K), and test it against the box threshold.
    template <int T, int SC>
    __device__ __forceinline__ void finish_level(int r, const float* oh, const float* ol,
                                                 bool owned_row, bool full) {
        if constexpr (T < K) {
            float (&bh)[3][V] = winh<T>();
            float (&bl)[3][V] = winl<T>();
#pragma unroll
            for (int v = 0; v < V; ++v) {
                bh[SC][v] = oh[v];
                if constexpr (COMP) bl[SC][v] = ol[v];
            }
        } else {
            // nx is a multiple of 4 (checked on entry): an owned lane's four
            // cells are in the field and 16-byte aligned; the stores are
            // predicated, so no branch splits the box
            const size_t off = (size_t)r * p.c.nx + xl;
            const bool st = owned_row && owned_lane();
            st_global_v4f_pred(p.Thi_out + off, oh, st);
            if constexpr (COMP) st_global_v4f_pred(p.Tlo_out + off, ol, st);
        }
        if constexpr (REDUCE) {
            bool h = hit[T - 1];
            const bool ol_ok = owned_row && owned_lane();
#pragma unroll
            for (int v = 0; v < V; ++v) {
                const bool ok = ol_ok && (full || xl + v < p.c.nx);
                if constexpr (COMP)
                    h = h | (ok && fk_gt(oh[v], ol[v], thr_h[T - 1], thr_l[T - 1]));
                else
                    h = h | (ok && oh[v] > thr_h[T - 1]);
            }
            hit[T - 1] = h;
        }
    }

    // ---- two-tier reduction on T = hi + lo ------------------------------
    __device__ __forceinline__ void set_thresholds() {
        const bool ol = owned_lane();
#pragma unroll
        for (int t = 0; t < K; ++t) {
            double a = s_tmx[t][lane];
            a = (a < p.c.Tm) ? a : p.c.Tm;
            if constexpr (COMP) {
                // the largest pair not above a: compare strictly against it
                const float h = (float)a;
                const float l = (float)(a - (double)h);
                thr_h[t] = ol ? h : INFINITY;
                thr_l[t] = ol ? l : 0.0f;
            } else {
                // the largest float not above a: a float cell exceeds it
                // exactly when it exceeds a
                thr_h[t] = ol ? __double2float_rd(a) : INFINITY;
            }
        }
    }

    template <int T>
    __device__ __forceinline__ void stage_level() {
        if constexpr (T >= 1 && T < K) {
#pragma unroll
            for (int P = 0; P < 3; ++P) {
                constexpr int dummy = 0;
                (void)dummy;
                const int s = ((P - T) % 3 + 3) % 3;
                float* d = s_box[P][lane];
#pragma unroll
                for (int v = 0; v < V; ++v) {
                    d[v] = (s == 0) ? winh<T>()[0][v] : (s == 1) ? winh<T>()[1][v] : winh<T>()[2][v];
                    if constexpr (COMP)
                        d[V + v] = (s == 0) ? winl<T>()[0][v]
                                 : (s == 1) ? winl<T>()[1][v] : winl<T>()[2][v];
                }
            }
        }
    }

    __device__ __forceinline__ double value_at(int t, int P, int r, int v) const {
        const size_t off = (size_t)r * p.c.nx + xl + v;
        if constexpr (COMP) {
            if (t < K) return (double)s_box[P][lane][v] + (double)s_box[P][lane][V + v];
            return (double)p.Thi_out[off] + (double)p.Tlo_out[off];
        } else {
            if (t < K) return (double)s_box[P][lane][v];
            return (double)p.Thi_out[off];
        }
    }

    __device__ __forceinline__ void exact_level(int t, int j) {
        const int nx = p.c.nx;
        const bool ol = owned_lane();
        double m = -INFINITY;
        for (int P = 0; P < 3; ++P) {
            const int r = j + P - t;
            const bool cand = r >= y0 && r < y1 && ol;
            bool hot = false;
            for (int v = 0; v < V; ++v) {
                const bool ok = cand && xl + v < nx;
                const double x = ok ? value_at(t, P, r, v) : 0.0;
                m = (ok && x > m) ? x : m;
                hot |= ok && x > p.c.Tm;
            }
            if (__any_sync(0xffffffffu, hot) && lane == 0) {
                s_ymn[t - 1] = min(s_ymn[t - 1], r);
                s_ymx[t - 1] = max(s_ymx[t - 1], r);
            }
        }
        if (m > s_tmx[t - 1][lane]) {
            long long arg = -1;
            for (int P = 0; P < 3 && arg < 0; ++P) {
                const int r = j + P - t;
                if (!(r >= y0 && r < y1 && ol)) continue;
                for (int v = 0; v < V && xl + v < nx; ++v)
                    if (value_at(t, P, r, v) == m) { arg = (long long)r * nx + xl + v; break; }
            }
            s_tmx[t - 1][lane] = m;
            s_arg[t - 1][lane] = arg;
        }
    }

    __device__ __forceinline__ void resolve_box(int j) {
        unsigned bits = 0;
#pragma unroll
        for (int t = 0; t < K; ++t) { bits |= hit[t] ? (1u << t) : 0u; hit[t] = false; }
        bits = __reduce_or_sync(0xffffffffu, bits);
        if (bits == 0u) return;
        for (int t = 1; t <= K; ++t) {
            if (!((bits >> (t - 1)) & 1u)) continue;
            switch (t) {
                case 1: stage_level<1>(); break;
                case 2: stage_level<2>(); break;
                case 3: stage_level<3>(); break;
                default: break;
            }
            __syncwarp();
            exact_level(t, j);
            __syncwarp();
        }
        set_thresholds();
    }
};

template <int K, bool REDUCE, bool SQ, bool COMP>
__global__ void __launch_bounds__(ADV_WARPS * 32, AdvOcc<K>::min_ctas)
advance_f32k_kernel(const __grid_constant__ CUtensorMap map_hi,
                    const __grid_constant__ CUtensorMap map_lo,
                    const __grid_constant__ FkParams p) {
    extern __shared__ __align__(128) unsigned char smem[];
    __shared__ Partial red[ADV_WARPS][K];
    __shared__ unsigned int s_last;
    __shared__ double s_tmx[ADV_WARPS][K][32];
    __shared__ long long s_arg[ADV_WARPS][K][32];
    __shared__ int s_ymn[ADV_WARPS][K], s_ymx[ADV_WARPS][K];
    __shared__ __align__(16) float s_box[ADV_WARPS][3][32][2 * ADV_V];

    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    constexpr int STAGE = fk_stage_floats<COMP>();
    float* stages = reinterpret_cast<float*>(smem) + wid * (ADV_S * STAGE);
    uint64_t* bars = reinterpret_cast<uint64_t*>(
        smem + size_t(ADV_WARPS) * ADV_S * STAGE * sizeof(float)) + wid * ADV_S;
    if (lane == 0) {
        for (int s = 0; s < ADV_S; ++s) mbar_init(&bars[s], 1);
        fence_mbar_init();
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    }
    __syncwarp();

    FkStrip<K, REDUCE, SQ, COMP> ws(p, &map_hi, &map_lo, stages, bars, lane, s_tmx[wid], s_arg[wid],
                          s_ymn[wid], s_ymx[wid], s_box[wid]);
    for (;;) {
        unsigned int t = 0;
        if (lane == 0) t = atomicAdd(p.tasks, 1u);
        t = __shfl_sync(0xffffffffu, t, 0);
        if (t >= (unsigned int)p.ntasks) break;
        ws.run_task((int)t);
        if (ws.failed) break;
    }

    const long long N = (long long)p.c.nx * p.c.ny;
    if constexpr (REDUCE) {
        __syncwarp();
        for (int t = 0; t < K; ++t) {
            double tm = s_tmx[wid][t][lane];
            long long ag = s_arg[wid][t][lane];
            int mn = s_ymn[wid][t], mx = s_ymx[wid][t];
            partial_warp_reduce(tm, ag, mn, mx);
            if (lane == 0) red[wid][t] = Partial{tm, ag, mn, mx};
        }
        __syncthreads();
        if (threadIdx.x < K) {
            const int t = threadIdx.x;
            double tm = -1.0; long long ag = N; int mn = p.c.ny, mx = -1;
            for (int w = 0; w < ADV_WARPS; ++w)
                partial_take(tm, ag, mn, mx, red[w][t].tmax, red[w][t].arg,
                             red[w][t].ymin, red[w][t].ymax);
            p.scratch[(size_t)blockIdx.x * K + t] = Partial{tm, ag, mn, mx};
        }
    }
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) s_last = (atomicAdd(p.counter, 1u) == gridDim.x - 1) ? 1u : 0u;
    __syncthreads();
    if (!s_last) return;
    __threadfence();
    if constexpr (REDUCE) {
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
    }
    if (threadIdx.x == 0) { *p.counter = 0u; *p.tasks = 0u; }
}

}  // namespace lpbf_b200
