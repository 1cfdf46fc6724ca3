// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Device-side layout of a batched process map (see lpbf_batch.cu).
//
// Workspace (one caller-owned device block, 256-byte aligned sections):
//   BatchHeader                 queue counter, CTA exit ticket, error word
//   unsigned int done[n]        per-scenario group tickets
//   BatchScen scen[n]           per-scenario static parameters (and tensor maps)
//   int task_base[R][n + 1]     first queue position of each scenario, for a
//                               launch starting at plan step r (R = n_steps)
//   int group_base[R][n + 1]    first task group of each scenario, likewise
//   unsigned int gdone[ngroups] per-group task tickets
//   BatchStep steps[n_steps][n] per-step laser of every scenario
//   Partial parts[ntasks][K]    per-task, per-step partials
//   Partial gparts[ngroups][K]  per-group, per-step partials
// A group is BATCH_GROUP consecutive tasks of one scenario.  A scenario's
// tasks in a launch follow the single-field kernel's band split for that
// launch's source band (band_chunks), so task and group counts depend on
// the launch's first step; ntasks and ngroups are their maxima.
// Scenarios are stored largest first; `order` maps that position back to the
// caller's index.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>
#include <stddef.h>

#include <vector>

#include "lpbf_advance.cuh"
#include "lpbf_b200.h"

namespace lpbf_b200 {

constexpr int BATCH_GROUP = 32;   // tasks folded together by the group's last warp

// How a batch stages rows in shared memory (lpbf_b200_batch_opts.staging).
constexpr int BATCH_STAGE_DIRECT = 0;   // no staging: each lane loads its cells
constexpr int BATCH_STAGE_BULK = 1;     // one cp.async.bulk per row
constexpr int BATCH_STAGE_TMAP = 2;     // one tiled tensor-map load per 3-row box

struct BatchHeader {
    unsigned int queue;            // next queue position
    unsigned int ctas;             // CTA exit ticket
    unsigned int err;              // error word (bit 0: a copy wait timed out)
    unsigned int pad[61];
};
static_assert(sizeof(BatchHeader) == 256, "batch header");

struct alignas(128) BatchScen {
    CUtensorMap map[2];            // tiled maps over buf[0], buf[1] (tensor-map staging only)
    AdvParams par;                 // static launch parameters (laser, band, buffers patched per task)
    double* buf[2];                // the ping-pong pair
    Partial* ring;                 // one Partial per plan step, or null
    int user;                      // the caller's index of this scenario
    int split;                     // its rows near the laser go in short tasks (band split)
};
static_assert(offsetof(BatchScen, par) % 8 == 0 && sizeof(AdvParams) % 8 == 0, "8-byte words");

struct BatchStep {
    LaserSub las;                  // x_l, y_l, dt-scaled source amplitude
    int band_lo, band_hi;          // rows the source can reach (empty: lo > hi)
    int bandx_lo, bandx_hi;        // columns the source can reach
};

struct BatchLaunch {
    const BatchScen* scen;
    const int* task_base;
    const BatchStep* steps;
    BatchHeader* hdr;
    unsigned int* scen_done;
    const int* group_base;
    unsigned int* group_done;
    Partial* parts;
    Partial* gparts;
    int nscen, ntasks;
    int parity;                    // fields are read from buf[parity], written to buf[parity ^ 1]
    int sq_all;                    // every scenario has square cells (ax == ay)
    int step0;                     // plan step of this launch's first substep
    int kfull;                     // the batch's depth: the band split covers steps
                                   // [step0, step0 + kfull) whatever this launch's depth
    int nsteps;                    // steps of the plan
};

struct BatchLayout {
    int K = 3;
    int ntasks = 0, ngroups = 0;   // maxima over launch start steps
    int rows_t = 1;                // rows of the task and group tables (max(n_steps, 1))
    std::vector<int> split;        // band split on, by stored position (batch_split_field)
    std::vector<int> order;        // stored position -> caller's scenario index
    std::vector<int> task_base;    // rows_t x (n + 1) entries
    std::vector<int> group_base;   // rows_t x (n + 1) entries
    std::vector<int> H;            // rows per task, by stored position
    std::vector<BatchStep> steps;  // n_steps x n, by stored position
    size_t off_done = 0, off_scen = 0, off_base = 0, off_gbase = 0, off_gdone = 0,
           off_steps = 0, off_parts = 0, off_gparts = 0, bytes = 0;
};

// Size class of a grid: 0 side < 512, 1 < 1024, 2 < 2048, 3 larger (side = max(nx, ny)).
int size_class(int nx, int ny);

// Whether a field of `cells` cells in a batch of `total` cells splits its
// source-band rows into short tasks.  The split pays when the field is a
// large share of the batch: then a slow band task left at a launch's end
// would set the launch's length (one 8192^2 field: 463 -> 752 GCell/s).  In
// a batch of many fields the large fields' band tasks come early in the
// queue, the small fields' tasks fill the tail, and the split only adds
// tasks and halo rows (256 mixed scenarios: 466 without it, 416 with it on
// the 2048^2 fields alone).
inline bool batch_split_field(long long cells, long long total) { return cells * 16 >= total; }

// Layout of a batch; with the scenarios' plans (n_steps > 0) it also fills
// the per-step laser data and the per-start-step task tables.
bool batch_layout(const lpbf_b200_scenario* sc, int n, int n_steps,
                  const lpbf_b200_batch_opts& o, BatchLayout* out);

// One launch of `K` steps over the whole batch (stage: BATCH_STAGE_*).
cudaError_t launch_batch(int K, int stage, const BatchLaunch& L, int ctas_per_sm,
                         cudaStream_t s);

// Resident CTAs per SM of the batch kernel (0 on failure).
int batch_resident_per_sm(int K, int stage);

}  // namespace lpbf_b200
