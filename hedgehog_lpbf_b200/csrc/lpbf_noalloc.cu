// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// lpbf_b200_advance_noalloc: the multi-step advance for callers that cannot
// allocate device memory.
//
// lpbf_b200_advance needs a caller-owned workspace (per-CTA partial results,
// a ticket counter, a task counter and an error word).  Some callers cannot
// provide one: code that runs inside a device-memory budget fixed at start-up
// (a task graph whose buffers were all reserved in its initialisation step),
// language bindings that only pass raw device pointers through and own no
// allocator (cgo, JNI), and hosts where a cudaMalloc would synchronize the
// device at a point where that is not allowed.  This entry point needs no
// workspace: its scratch is a fixed array in the library's own device memory.
//
// The array below is a file-scope __device__ variable.  In host code its name
// is only a host-side stand-in, not a device address; the device address is
// looked up with cudaGetSymbolAddress once per device (on the first call made
// with that device current) and cached.  Nothing here calls cudaMalloc,
// cudaFree or any allocating routine.
// ---------------------------------------------------------------------------
#include <algorithm>
#include <mutex>

#include "lpbf_host.hpp"
#include "lpbf_b200.h"

namespace lpbf_b200 {
namespace {

// Most per-CTA partial records the scratch holds (grid size x steps per
// launch): 4096 records = 98,560 bytes with the 256-byte counter header.
// The launch path sizes the grid from the occupancy query and then clamps it
// to NOALLOC_PARTIALS / depth CTAs (>= 1024 for depth <= 4), so the records
// of one launch always fit, on any GPU and for either load path.
constexpr int NOALLOC_PARTIALS = 4096;
constexpr size_t NOALLOC_BYTES = 256 + size_t(NOALLOC_PARTIALS) * sizeof(Partial);
static_assert(NOALLOC_BYTES == LPBF_B200_NOALLOC_SCRATCH_BYTES, "header constant");

// Same layout as Workspace's header followed by NOALLOC_PARTIALS partials.
// Held by every GPU that loads the library, for the life of the process.
static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_BYTES];

std::mutex g_mu;
void* g_addr[64] = {nullptr};

// Device address of g_noalloc_scratch on the current device (cached).
int scratch_address(void** out) {
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return LPBF_ERR_CUDA;
    std::lock_guard<std::mutex> lk(g_mu);
    if (!g_addr[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p)
            return LPBF_ERR_CUDA;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return LPBF_OK;
}

}  // namespace
}  // namespace lpbf_b200

using namespace lpbf_b200;

extern "C" int lpbf_b200_advance_noalloc(double* T_a, double* T_b, const StepConst* k,
                                         const lpbf_tick* plan, int n_steps,
                                         const lpbf_b200_opts* opts, Partial* ring,
                                         cudaStream_t stream, int* result_in_b,
                                         unsigned int* err) {
    if (!k || k->nx < 2 || k->ny < 1 || (long long)k->nx * k->ny >= (1ll << 40) || !opts ||
        !T_a || !T_b || T_a == T_b || n_steps < 0 || (n_steps > 0 && !plan) || !result_in_b)
        return LPBF_ERR_ARG;
    if (opts->bc != 0 && opts->bc != 1) return LPBF_ERR_ARG;
    if (opts->phys != 0 && opts->phys != 1) return LPBF_ERR_ARG;
    if (opts->phys == 1) return LPBF_ERR_UNSUPPORTED;     // baseline physics only
    const size_t N = (size_t)k->nx * k->ny;
    if (T_a < T_b + N && T_b < T_a + N) return LPBF_ERR_ARG;

    int depth = opts->depth;
    if (depth <= 0) {
        const long long n = (long long)k->nx * k->ny;
        depth = (n >= (1ll << 22)) ? 3 : (n >= (1ll << 18)) ? 2 : 1;
    }
    depth = std::min(std::max(depth, 1), 4);

    void* scratch = nullptr;
    const int st = scratch_address(&scratch);
    if (st != LPBF_OK) return st;
    // Every call shares the array: clear the counters and the error word.
    if (cudaMemsetAsync(scratch, 0, 256, stream) != cudaSuccess) return LPBF_ERR_CUDA;
    Workspace* ws = static_cast<Workspace*>(scratch);

    const Coef c = make_coef(*k, opts->bc, opts->T_edge, opts->Tm);
    double* cur = T_a;
    double* nxt = T_b;
    int in_b = 0;
    for (int s0 = 0; s0 < n_steps; s0 += depth) {
        const int kk = std::min(depth, n_steps - s0);
        LaserSub las[KMAX];
        for (int t = 0; t < kk; ++t)
            las[t] = make_laser(*k, plan[s0 + t].x_l, plan[s0 + t].y_l, plan[s0 + t].q_scale);
        const cudaError_t e = launch_advance(kk, cur, nxt, c, las, ring ? ring + s0 : nullptr,
                                             ws, nullptr, 0, opts->rows, stream, nullptr,
                                             NOALLOC_PARTIALS);
        // a launch needing more per-CTA records than the scratch holds
        if (e == cudaErrorInvalidValue) return LPBF_ERR_WORKSPACE;
        if (e != cudaSuccess) return LPBF_ERR_CUDA;
        std::swap(cur, nxt);
        in_b ^= 1;
    }
    // The error word lives in the shared scratch, which the caller cannot
    // address: copy it out behind this call's launches.
    if (err && cudaMemcpyAsync(err, &ws->err, sizeof(unsigned int), cudaMemcpyDeviceToHost,
                               stream) != cudaSuccess)
        return LPBF_ERR_CUDA;
    *result_in_b = in_b;
    return LPBF_OK;
}
