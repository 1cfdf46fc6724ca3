// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Host-side helpers shared by the translation units of liblpbf_b200.so:
// device properties, the workspace layout, TMA tensor-map encoding (through
// the driver entry point, so the library does not link libcuda directly) and
// the launch functions each unit exports to the others.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

#include <algorithm>
#include <cmath>

#include <nvtx3/nvToolsExt.h>

#include "lpbf_device.cuh"

namespace lpbf_b200 {

// NVTX range over a host entry point (visible in Nsight timelines; a no-op
// without a tool attached).
struct NvtxRange {
    explicit NvtxRange(const char* name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange&) = delete;
    NvtxRange& operator=(const NvtxRange&) = delete;
};

constexpr int MAX_CTAS = 2048;     // most CTAs a reducing launch may use

// Device workspace.  The counter and error word sit in the first 256 bytes;
// per-CTA partials follow.
struct Workspace {
    unsigned int counter;          // last-CTA ticket
    unsigned int err;              // error word
    unsigned int tasks;            // dynamic task counter
    unsigned int pad[61];
    Partial parts[MAX_CTAS * KMAX];
};
static_assert(offsetof(Workspace, parts) == 256, "workspace header");

int sm_count();                    // of the current device

// Encode (or fetch from a small cache) a 2D f64 tensor map over a row-major
// nx x ny field with box {box_cols, box_rows}.  Returns false on failure.
bool tensor_map_f64(const void* base, int nx, int ny, int box_cols, int box_rows,
                    CUtensorMap* out);
bool tensor_map_f32(const void* base, int nx, int ny, int box_cols, int box_rows,
                    CUtensorMap* out);
bool tensor_map_pixel_pairs_bf16(const void* base, int W, int H, int B, int box_pairs,
                                 CUtensorMap* out);
bool tensor_map_act_bf16(const void* base, int C, int W, int H, int B, int box_px,
                         CUtensorMap* out);

// Rows whose source term can be non-zero in any of the K substeps (a
// superset: the kernel decides exactly, this only routes rows to the general
// body).  Empty when every substep has the beam off.
inline void laser_band(const Coef& c, const LaserSub* las, int K, int* lo, int* hi, int* xlo,
                int* xhi) {
    int blo = 1 << 30, bhi = -(1 << 30), cxlo = 1 << 30, cxhi = -(1 << 30);
    const double R = std::sqrt(c.r2_cut);
    for (int t = 0; t < K; ++t) {
        if (las[t].cs == 0.0) continue;
        const double y = las[t].y_l, x = las[t].x_l;
        if (!std::isfinite(y) || !std::isfinite(x) || !std::isfinite(R) || c.dy <= 0.0 ||
            c.dx <= 0.0) {
            blo = -2; bhi = c.ny + 2; cxlo = -2; cxhi = c.nx + 2;
            break;
        }
        auto clampi = [](double v, double a, double b) { return (int)std::max(a, std::min(v, b)); };
        blo = std::min(blo, clampi(std::floor((y - R) / c.dy) - 2.0, -2.0, c.ny + 2.0));
        bhi = std::max(bhi, clampi(std::ceil((y + R) / c.dy) + 2.0, -2.0, c.ny + 2.0));
        cxlo = std::min(cxlo, clampi(std::floor((x - R) / c.dx) - 2.0, -2.0, c.nx + 2.0));
        cxhi = std::max(cxhi, clampi(std::ceil((x + R) / c.dx) + 2.0, -2.0, c.nx + 2.0));
    }
    *lo = blo; *hi = bhi; *xlo = cxlo; *xhi = cxhi;
}

// True when `p` suits the TMA path (16-byte aligned base, even row length).
inline bool tma_ok(const void* p, int nx) {
    return (reinterpret_cast<uintptr_t>(p) % 16 == 0) && (nx % 2 == 0);
}

// Baseline-physics advance of `K` steps in one launch (K = 1..4).
//   ring   : K finalized Partials (null: no reduction)
//   ref_out: reference fused-reduce layout (K == 1 only), ref_nparts entries
//   win    : row window of a row-strip shard (null: the whole field; c.ny is
//            then the buffer's rows and win->gny the field's)
//   parts_cap: per-CTA partial records ws->parts can hold; a reducing launch
//            uses at most parts_cap / K CTAs (and at most MAX_CTAS)
// Returns a CUDA error code.
struct RowWindow { int row0, gny, lo, hi; };
cudaError_t launch_advance(int K, const double* Tin, double* Tout, const Coef& c,
                           const LaserSub* las, Partial* ring, Workspace* ws,
                           Partial* ref_out, long long ref_nparts, int rows,
                           cudaStream_t stream, const RowWindow* win = nullptr,
                           int parts_cap = MAX_CTAS * KMAX);

// Extended-physics (phys == 1) single step, one thread per cell, with the
// same reduction outputs as launch_advance.
cudaError_t launch_ext_step(const double* Tin, double* Tout, const StepConst& k,
                            int bc, double T_edge, double Tm, Partial* ring,
                            Workspace* ws, Partial* ref_out, long long ref_nparts,
                            cudaStream_t stream);

}  // namespace lpbf_b200
