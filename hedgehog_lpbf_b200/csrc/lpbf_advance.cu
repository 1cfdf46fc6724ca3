// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Launch logic of the temporally blocked baseline step and the extended C-ABI
// entry points of include/lpbf_b200.h.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <cmath>
#include <cstring>
#include <mutex>

#include "lpbf_advance.cuh"
#include "lpbf_host.hpp"
#include "lpbf_b200.h"

namespace lpbf_b200 {

// ---- device properties ----------------------------------------------------
int sm_count() {
    static int cache[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (cache[dev] == 0) {
        int n = 0;
        cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev);
        cache[dev] = n > 0 ? n : 1;
    }
    return cache[dev];
}

// ---- tensor maps ------------------------------------------------------------
namespace {

using EncodeFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*,
                              const cuuint64_t*, const cuuint64_t*, const cuuint32_t*,
                              const cuuint32_t*, CUtensorMapInterleave, CUtensorMapSwizzle,
                              CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

EncodeFn encode_fn() {
    static EncodeFn fn = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess && q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeFn>(p);
    });
    return fn;
}

struct MapKey {
    const void* base; int nx, ny, bc, br, dt;
    bool operator==(const MapKey& o) const {
        return base == o.base && nx == o.nx && ny == o.ny && bc == o.bc && br == o.br && dt == o.dt;
    }
};
struct MapEntry { MapKey key; CUtensorMap map; bool used; };
constexpr int MAP_CACHE = 32;
MapEntry g_maps[MAP_CACHE];
int g_next = 0;
std::mutex g_map_mu;

bool tensor_map(const void* base, int nx, int ny, int box_cols, int box_rows, int esize,
                CUtensorMapDataType dtype, int dtag, CUtensorMap* out) {
    const MapKey key{base, nx, ny, box_cols, box_rows, dtag};
    std::lock_guard<std::mutex> lk(g_map_mu);
    for (auto& e : g_maps)
        if (e.used && e.key == key) { *out = e.map; return true; }
    EncodeFn fn = encode_fn();
    if (!fn) return false;
    cuuint64_t gdim[2] = {(cuuint64_t)nx, (cuuint64_t)ny};
    cuuint64_t gstride[1] = {(cuuint64_t)nx * esize};
    cuuint32_t box[2] = {(cuuint32_t)box_cols, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    CUtensorMap m;
    std::memset(&m, 0, sizeof(m));
    const CUresult r = fn(&m, dtype, 2, const_cast<void*>(base), gdim, gstride, box, estr,
                          CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                          CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
                          CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
    if (r != CUDA_SUCCESS) return false;
    MapEntry& e = g_maps[g_next];
    g_next = (g_next + 1) % MAP_CACHE;
    e.key = key; e.map = m; e.used = true;
    *out = m;
    return true;
}

}  // namespace

bool tensor_map_f64(const void* base, int nx, int ny, int box_cols, int box_rows,
                    CUtensorMap* out) {
    return tensor_map(base, nx, ny, box_cols, box_rows, 8, CU_TENSOR_MAP_DATA_TYPE_FLOAT64,
                      64, out);
}
bool tensor_map_f32(const void* base, int nx, int ny, int box_cols, int box_rows,
                    CUtensorMap* out) {
    return tensor_map(base, nx, ny, box_cols, box_rows, 4, CU_TENSOR_MAP_DATA_TYPE_FLOAT32,
                      32, out);
}

// NHWC bf16 activations (C channels per pixel) as a 4D tensor (c, x, y, b):
// boxes of {C, box_px, 1, 1} with the 64-byte swizzle that the tensor core's
// K-major SW64 operand layout expects; out-of-range pixels read as zero.
bool tensor_map_act_bf16(const void* base, int C, int W, int H, int B, int box_px,
                         CUtensorMap* out) {
    EncodeFn fn = encode_fn();
    if (!fn || C * 2 > 64 || (C * 2) % 16 != 0) return false;
    cuuint64_t gdim[4] = {(cuuint64_t)C, (cuuint64_t)W, (cuuint64_t)H, (cuuint64_t)B};
    cuuint64_t gstride[3] = {(cuuint64_t)C * 2, (cuuint64_t)C * 2 * W, (cuuint64_t)C * 2 * W * H};
    cuuint32_t box[4] = {(cuuint32_t)C, (cuuint32_t)box_px, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    std::memset(out, 0, sizeof(*out));
    return fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), gdim, gstride,
              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_64B,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// NHWC bf16 activations with 4 channels (8 bytes per pixel) as a 4D tensor
// of pixel pairs (8 values, W / 2 pairs, H, B; W even): a box {8, box_pairs,
// 1, 1} brings 2 box_pairs consecutive pixels of one row, unswizzled (a TMA
// box row must hold a multiple of 16 bytes).  Pixels and rows off the image
// read as zero.
bool tensor_map_pixel_pairs_bf16(const void* base, int W, int H, int B, int box_pairs,
                                 CUtensorMap* out) {
    EncodeFn fn = encode_fn();
    if (!fn || W % 2 != 0 || box_pairs < 1 || box_pairs > 256) return false;
    cuuint64_t gdim[4] = {8, (cuuint64_t)W / 2, (cuuint64_t)H, (cuuint64_t)B};
    cuuint64_t gstride[3] = {16, (cuuint64_t)8 * W, (cuuint64_t)8 * W * H};
    cuuint32_t box[4] = {8, (cuuint32_t)box_pairs, 1, 1};
    cuuint32_t estr[4] = {1, 1, 1, 1};
    std::memset(out, 0, sizeof(*out));
    return fn(out, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 4, const_cast<void*>(base), gdim, gstride,
              box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

// ---- launch of one temporally blocked step ---------------------------------
namespace {

template <int K, bool TMA, bool REDUCE, bool SQ>
cudaError_t launch_t(const double* Tin, double* Tout, const Coef& c, const LaserSub* las,
                     Partial* ring, Workspace* ws, Partial* ref_out, long long ref_nparts,
                     int rows, cudaStream_t stream, const RowWindow* win, int parts_cap) {
    auto kern = advance_kernel<K, TMA, REDUCE, SQ>;
    const size_t smem = TMA ? ADV_SMEM_BYTES : 0;

    static int occ[64] = {0};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 64) dev = 0;
    if (occ[dev] == 0) {
        if (smem > 48 * 1024) {
            cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                 (int)smem);
            if (e != cudaSuccess) return e;
        }
        int nb = 0;
        cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&nb, kern,
                                                                      ADV_WARPS * 32, smem);
        if (e != cudaSuccess) return e;
        occ[dev] = std::max(1, nb);
    }
    const int resident = sm_count() * occ[dev];

    AdvParams p;
    std::memset(&p, 0, sizeof(p));
    p.c = c;
    for (int t = 0; t < K; ++t) p.las[t] = las[t];
    p.row0 = win ? win->row0 : 0;
    p.gny = win ? win->gny : c.ny;
    p.row_lo = win ? win->lo : 0;
    p.row_hi = win ? win->hi : c.ny;
    const int nrows = p.row_hi - p.row_lo;
    if (win) {
        // the source band in the field's rows, then in this buffer's
        Coef g = c;
        g.ny = p.gny;
        laser_band(g, las, K, &p.band_lo, &p.band_hi, &p.bandx_lo, &p.bandx_hi);
        p.band_lo = std::max(-2, std::min(p.band_lo - p.row0, c.ny + 2));
        p.band_hi = std::max(-2, std::min(p.band_hi - p.row0, c.ny + 2));
    } else {
        laser_band(c, las, K, &p.band_lo, &p.band_hi, &p.bandx_lo, &p.bandx_hi);
    }
    p.nstrips = (c.nx + ADV_WOUT - 1) / ADV_WOUT;
    // Dynamic scheduling (workspace given): several tasks per warp from the
    // atomic queue.  Static: about one task per resident warp.
    const bool dynamic = ws != nullptr;
    int H = rows;
    if (H <= 0) {
        if (dynamic) {
            // 12..64 rows.  The queue deals tasks to the resident warps in
            // waves, so the launch lasts about (waves) x (rows a task
            // computes, its own plus about 2K of halo): take the height with
            // the least of that, the taller on a tie.  Tall tasks cost less
            // halo; a last wave that is nearly empty costs a whole task (a
            // 2048-row strip of an 8192-wide field: 41 rows, two waves,
            // instead of 26 rows and a fourth wave of 7 % of the warps).
            // The band split keeps the slow source-band tasks short
            // whatever H is.
            const long long warps = (long long)resident * ADV_WARPS;
            long long best = -1;
            for (int h = 12; h <= 64; ++h) {
                const long long tasks = (long long)((nrows + h - 1) / h) * p.nstrips;
                const long long cost = ((tasks + warps - 1) / warps) * (h + 2 * K);
                if (best < 0 || cost <= best) { best = cost; H = h; }
            }
        } else {
            const int want = std::max(1, (resident * ADV_WARPS) / p.nstrips);
            H = (nrows + want - 1) / want;
        }
        H = std::max(H, std::max(8, 4 * K));
    }
    p.H = std::min(H, nrows);
    // the band split needs the dynamic queue (static scheduling: H-row chunks)
    band_chunks(p.H, p.row_lo, p.row_hi, K, dynamic ? p.band_lo : 1, dynamic ? p.band_hi : 0,
                &p.nA, &p.nB, &p.Hb, &p.Ya, &p.Yb, &p.nchunks);
    p.ntasks = p.nstrips * p.nchunks;
    int grid = std::min((p.ntasks + ADV_WARPS - 1) / ADV_WARPS, resident);
    if (REDUCE && !ref_out) grid = std::min(grid, std::min(MAX_CTAS, parts_cap / K));
    if (ref_out) grid = (int)std::min<long long>(grid, ref_nparts);
    grid = std::max(grid, 1);
    // every CTA of a reducing launch writes K records into ws->parts
    if (REDUCE && !ref_out && (long long)grid * K > parts_cap) return cudaErrorInvalidValue;
    p.Tin = Tin;
    p.Tout = Tout;
    p.ring = ring;
    p.ref_out = ref_out;
    p.ref_nparts = ref_nparts;
    p.st256 = (c.nx % 4 == 0) && (reinterpret_cast<uintptr_t>(Tout) % 32 == 0);
    if (ws) {
        p.scratch = ws->parts;
        p.counter = &ws->counter;
        p.tasks = &ws->tasks;
        p.err = &ws->err;
    }
    CUtensorMap map;
    std::memset(&map, 0, sizeof(map));
    if (TMA && !tensor_map_f64(Tin, c.nx, c.ny, ADV_COLS, ADV_R, &map))
        return cudaErrorNotSupported;
    kern<<<grid, ADV_WARPS * 32, smem, stream>>>(map, p);
    return cudaGetLastError();
}

template <int K, bool SQ>
cudaError_t launch_k2(bool tma, bool reduce, const double* Tin, double* Tout, const Coef& c,
                      const LaserSub* las, Partial* ring, Workspace* ws, Partial* ref_out,
                      long long ref_nparts, int rows, cudaStream_t s, const RowWindow* w,
                      int cap) {
    if (tma) {
        const cudaError_t e = reduce
            ? launch_t<K, true, true, SQ>(Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows,
                                          s, w, cap)
            : launch_t<K, true, false, SQ>(Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows,
                                           s, w, cap);
        if (e != cudaErrorNotSupported) return e;
        // tensor map unavailable: fall through to the direct-load kernel
    }
    return reduce
        ? launch_t<K, false, true, SQ>(Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, s, w,
                                       cap)
        : launch_t<K, false, false, SQ>(Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, s,
                                        w, cap);
}

// Square cells (ax == ay, the same comparison the kernels make) take the
// one-Laplacian form of the cell update.
template <int K>
cudaError_t launch_k(bool tma, bool reduce, const double* Tin, double* Tout, const Coef& c,
                     const LaserSub* las, Partial* ring, Workspace* ws, Partial* ref_out,
                     long long ref_nparts, int rows, cudaStream_t s, const RowWindow* w,
                     int cap) {
    return c.ax == c.ay
        ? launch_k2<K, true>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows,
                             s, w, cap)
        : launch_k2<K, false>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows,
                              s, w, cap);
}

}  // namespace

cudaError_t launch_advance(int K, const double* Tin, double* Tout, const Coef& c,
                           const LaserSub* las, Partial* ring, Workspace* ws,
                           Partial* ref_out, long long ref_nparts, int rows,
                           cudaStream_t stream, const RowWindow* win, int parts_cap) {
    const bool tma = tma_ok(Tin, c.nx) && tma_ok(Tout, c.nx);
    const bool reduce = (ring != nullptr) || (ref_out != nullptr);
    if (reduce && !ref_out && !ws) return cudaErrorInvalidValue;
    switch (K) {
        case 1: return launch_k<1>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, stream, win, parts_cap);
        case 2: return launch_k<2>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, stream, win, parts_cap);
        case 3: return launch_k<3>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, stream, win, parts_cap);
        case 4: return launch_k<4>(tma, reduce, Tin, Tout, c, las, ring, ws, ref_out, ref_nparts, rows, stream, win, parts_cap);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace lpbf_b200

// ===========================================================================
// Extended C-ABI (include/lpbf_b200.h)
// ===========================================================================
using namespace lpbf_b200;

namespace {

// Measured on B200 at 8192^2 with the per-step reduction: depth 3 is the
// fastest (depth 4 is register-bound); small grids fit in L2 and gain little.
int auto_depth(int nx, int ny) {
    const long long n = (long long)nx * ny;
    if (n >= (1ll << 22)) return 3;
    if (n >= (1ll << 18)) return 2;
    return 1;
}

int resolve_depth(const lpbf_b200_opts* o, int nx, int ny) {
    if (o->phys != 0) return 1;
    int d = o->depth > 0 ? o->depth : auto_depth(nx, ny);
    return std::min(std::max(d, 1), 4);
}

bool valid_const(const StepConst* k) {
    return k && k->nx >= 2 && k->ny >= 1 && (long long)k->nx * k->ny < (1ll << 40);
}

}  // namespace

extern "C" {

int lpbf_b200_version(void) { return 1; }

const char* lpbf_b200_status_string(int status) {
    switch (status) {
        case LPBF_OK: return "ok";
        case LPBF_ERR_ARG: return "invalid argument";
        case LPBF_ERR_UNSUPPORTED: return "unsupported request";
        case LPBF_ERR_WORKSPACE: return "workspace missing or too small";
        case LPBF_ERR_CUDA: return "CUDA runtime error";
        case LPBF_ERR_TMA: return "tensor-map encoding failed";
        default: return "unknown status";
    }
}

size_t lpbf_b200_workspace_bytes(void) { return sizeof(Workspace); }

int lpbf_b200_workspace_init(void* work, size_t work_bytes, cudaStream_t stream) {
    if (!work || work_bytes < sizeof(Workspace)) return LPBF_ERR_WORKSPACE;
    return cudaMemsetAsync(work, 0, 256, stream) == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_advance_launches(int nx, int ny, int n_steps, const lpbf_b200_opts* opts) {
    if (!opts || n_steps < 0) return LPBF_ERR_ARG;
    const int d = resolve_depth(opts, nx, ny);
    return (n_steps + d - 1) / d;
}

int lpbf_b200_advance(double* T_a, double* T_b, const StepConst* k, const lpbf_tick* plan,
                      int n_steps, const lpbf_b200_opts* opts, Partial* ring, void* work,
                      size_t work_bytes, cudaStream_t stream, int* result_in_b) {
    NvtxRange nvtx_range("lpbf_b200_advance");
    if (!valid_const(k) || !opts || !T_a || !T_b || T_a == T_b || n_steps < 0 ||
        (n_steps > 0 && !plan) || !result_in_b)
        return LPBF_ERR_ARG;
    if (opts->bc != 0 && opts->bc != 1) return LPBF_ERR_ARG;
    if (opts->phys != 0 && opts->phys != 1) return LPBF_ERR_ARG;
    const size_t N = (size_t)k->nx * k->ny;
    const double* a_end = T_a + N;
    const double* b_end = T_b + N;
    if (T_a < b_end && T_b < a_end) return LPBF_ERR_ARG;
    Workspace* ws = static_cast<Workspace*>(work);
    if (ring && (!ws || work_bytes < sizeof(Workspace))) return LPBF_ERR_WORKSPACE;

    const int depth = resolve_depth(opts, k->nx, k->ny);
    const Coef c = make_coef(*k, opts->bc, opts->T_edge, opts->Tm);
    double* cur = T_a;
    double* nxt = T_b;
    int in_b = 0;
    for (int s0 = 0; s0 < n_steps; s0 += depth) {
        const int kk = std::min(depth, n_steps - s0);
        cudaError_t e;
        if (opts->phys == 0) {
            LaserSub las[KMAX];
            for (int t = 0; t < kk; ++t)
                las[t] = make_laser(*k, plan[s0 + t].x_l, plan[s0 + t].y_l, plan[s0 + t].q_scale);
            e = launch_advance(kk, cur, nxt, c, las, ring ? ring + s0 : nullptr, ws, nullptr, 0,
                               opts->rows, stream);
        } else {
            StepConst ks = *k;
            ks.x_l = plan[s0].x_l; ks.y_l = plan[s0].y_l; ks.q_scale = plan[s0].q_scale;
            e = launch_ext_step(cur, nxt, ks, opts->bc, opts->T_edge, opts->Tm,
                                ring ? ring + s0 : nullptr, ws, nullptr, 0, stream);
        }
        if (e != cudaSuccess) return LPBF_ERR_CUDA;
        std::swap(cur, nxt);
        in_b ^= 1;
    }
    *result_in_b = in_b;
    return LPBF_OK;
}

int lpbf_b200_advance_rows(const double* T_in, double* T_out, const StepConst* k,
                           const lpbf_tick* plan, int n_steps, const lpbf_b200_opts* opts,
                           const lpbf_b200_rows* rows, Partial* ring, void* work,
                           size_t work_bytes, cudaStream_t stream) {
    NvtxRange nvtx_range("lpbf_b200_advance_rows");
    if (!valid_const(k) || !opts || !rows || !T_in || !T_out || n_steps < 1 || n_steps > 4 ||
        !plan)
        return LPBF_ERR_ARG;
    if (opts->bc != 0 && opts->bc != 1) return LPBF_ERR_ARG;
    if (opts->phys != 0) return LPBF_ERR_UNSUPPORTED;
    const size_t N = (size_t)k->nx * k->ny;
    if ((const double*)T_out < T_in + N && T_in < (const double*)T_out + N) return LPBF_ERR_ARG;
    const RowWindow w{rows->row0, rows->global_ny, rows->lo, rows->hi};
    if (w.row0 < 0 || w.gny < 1 || (long long)w.row0 + k->ny > w.gny ||
        (long long)k->nx * w.gny >= (1ll << 40) || w.lo < 0 || w.lo >= w.hi || w.hi > k->ny)
        return LPBF_ERR_ARG;
    // the values of the advanced rows depend on n_steps rows either side
    if (w.row0 > 0 && w.lo < n_steps) return LPBF_ERR_ARG;
    if (w.row0 + k->ny < w.gny && k->ny - w.hi < n_steps) return LPBF_ERR_ARG;
    Workspace* ws = static_cast<Workspace*>(work);
    if (ring && (!ws || work_bytes < sizeof(Workspace))) return LPBF_ERR_WORKSPACE;
    const Coef c = make_coef(*k, opts->bc, opts->T_edge, opts->Tm);
    LaserSub las[KMAX];
    for (int t = 0; t < n_steps; ++t)
        las[t] = make_laser(*k, plan[t].x_l, plan[t].y_l, plan[t].q_scale);
    const cudaError_t e = launch_advance(n_steps, T_in, T_out, c, las, ring, ws, nullptr, 0,
                                         opts->rows, stream, &w);
    return e == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

int lpbf_b200_read_error(const void* work, cudaStream_t stream, unsigned int* err) {
    if (!work || !err) return LPBF_ERR_ARG;
    const Workspace* ws = static_cast<const Workspace*>(work);
    if (cudaMemcpyAsync(err, &ws->err, sizeof(unsigned int), cudaMemcpyDeviceToHost, stream) !=
        cudaSuccess)
        return LPBF_ERR_CUDA;
    return cudaStreamSynchronize(stream) == cudaSuccess ? LPBF_OK : LPBF_ERR_CUDA;
}

}  // extern "C"
