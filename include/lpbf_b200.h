/* SPDX-License-Identifier: 0BSD
 * ---------------------------------------------------------------------------
 * liblpbf_b200 extended C-ABI: multi-step, status-returning entry points.
 *
 * Plain C (usable from C, C++, ctypes, cgo, JNI): pointers, sizes, POD
 * structs whose layouts equal the reference's StepConst / Partial / Tick.
 * Every entry point is asynchronous on `stream` unless noted, allocates no
 * device memory (the autotuner excepted, as noted), and returns LPBF_OK (0)
 * or a negative status (lpbf_b200_status_string).
 *
 * Reference interfaces these replace or extend:
 *   lpbf_b200_advance   the per-step loop of GpuStepTask::execute
 *                       (include/gpu_step_task.hpp:149-197): step + reduce +
 *                       finalize for `n_steps` Ticks of a plan, in
 *                       ceil(n_steps / depth) launches instead of 2-4
 *                       launches per step.
 * ---------------------------------------------------------------------------
 */
#ifndef LPBF_B200_H
#define LPBF_B200_H

#include <stddef.h>
#include <cuda_runtime.h>

#ifdef __cplusplus
#include "lpbf_step_const.hpp"
#include "gpu_messages.hpp"
typedef lpbf::Tick lpbf_tick;
extern "C" {
#else
#include <stdbool.h>
typedef struct StepConst {
    int nx, ny;
    double dx, dy, inv_dx2, inv_dy2, inv_r0_sq;
    double alpha, K, rho, cp, rho_cp, inv_h, h, dt;
    double peak_S, eta, P;
    double hConv, Tamb, Tsub, dSub, eps;
    bool radiation;
    double kmult;
    double x_l, y_l;
    double q_scale;
} StepConst;
typedef struct Partial { double tmax; long long arg; int ymin; int ymax; } Partial;
typedef struct lpbf_tick {
    int step; double t; double x_l, y_l; double q_scale; double x_laser_csv;
    bool wrapped; bool dump;
} lpbf_tick;
#endif

enum {
    LPBF_OK = 0,
    LPBF_ERR_ARG = -1,          /* invalid argument */
    LPBF_ERR_UNSUPPORTED = -2,  /* valid request this build does not implement */
    LPBF_ERR_WORKSPACE = -3,    /* workspace missing or too small */
    LPBF_ERR_CUDA = -4,         /* a CUDA runtime call or launch failed */
    LPBF_ERR_TMA = -5           /* tensor-map encoding failed */
};

/* Options of a multi-step advance. */
typedef struct lpbf_b200_opts {
    int    phys;     /* 0 constant properties (baseline); 1 extended (Mills k(T), cp(T)) */
    int    bc;       /* 0 zero-flux mirror edges (the reference's); 1 fixed-value edges */
    double T_edge;   /* edge temperature for bc == 1 [K] */
    double Tm;       /* melt threshold of the per-step Partial [K] */
    int    depth;    /* time steps per launch (temporal blocking, 1..4); 0 = automatic */
    int    rows;     /* rows per warp task; 0 = automatic */
} lpbf_b200_opts;

int         lpbf_b200_version(void);
const char* lpbf_b200_status_string(int status);

/* Device workspace (per-launch partials, a ticket counter and an error word).
 * Size is independent of the grid.  Zero it once with
 * lpbf_b200_workspace_init before its first use; advance leaves it ready for
 * the next call.  Calls that share one workspace must be stream-ordered. */
size_t lpbf_b200_workspace_bytes(void);
int    lpbf_b200_workspace_init(void* work, size_t work_bytes, cudaStream_t stream);

/* Advance the field by n_steps time steps along plan[0..n_steps) (host array;
 * each step uses plan[i].x_l, y_l, q_scale and k->dt).  The field starts in
 * T_a; T_a and T_b are a ping-pong pair of nx*ny doubles (row-major, must not
 * overlap).  On return *result_in_b tells which buffer holds the final field
 * (this is known on the host at once: the launch count's parity).  ring
 * (device, nullable) receives one finalized Partial per step, ring[i] for
 * step i.  Capturable in a CUDA graph (no host synchronization). */
int lpbf_b200_advance(double* T_a, double* T_b, const StepConst* k,
                      const lpbf_tick* plan, int n_steps, const lpbf_b200_opts* opts,
                      Partial* ring, void* work, size_t work_bytes,
                      cudaStream_t stream, int* result_in_b);

/* Number of launches lpbf_b200_advance issues for these arguments. */
int lpbf_b200_advance_launches(int nx, int ny, int n_steps, const lpbf_b200_opts* opts);

/* A row strip of a larger field: the buffers hold rows row0 .. row0+k->ny-1
 * of a field of global_ny rows (k->ny is the buffer's row count, every other
 * StepConst member is the field's), and the call advances buffer rows
 * [lo, hi); the rows outside are halo, read but not written. */
typedef struct lpbf_b200_rows {
    int row0;        /* field row of buffer row 0 */
    int global_ny;   /* rows of the whole field */
    int lo, hi;      /* buffer rows advanced */
} lpbf_b200_rows;

/* One launch of n_steps (1..4) baseline steps over a row strip, T_in ->
 * T_out (rows [lo, hi) of T_out written, nothing else).  The results of
 * rows [lo, hi) equal those of lpbf_b200_advance on the whole field bit for
 * bit, provided the halo rows hold the field's values: at least n_steps halo
 * rows above lo unless row0 == 0 (buffer row 0 is the field's top edge),
 * at least n_steps below hi unless row0 + k->ny == global_ny (the bottom
 * edge); otherwise LPBF_ERR_ARG.  ring (device, nullable) receives one
 * Partial per step over rows [lo, hi) in the field's numbering (flat index
 * (row0 + r) * nx + x, molten rows as field rows, neutral elements from
 * global_ny); the Partials of all strips combine by the reduction's rule
 * into the whole field's.  Row-strip sharding across GPUs: each rank
 * advances its strip, then exchanges n_steps halo rows with its neighbours.
 * No counterpart in the reference, which advances whole fields only. */
int lpbf_b200_advance_rows(const double* T_in, double* T_out, const StepConst* k,
                           const lpbf_tick* plan, int n_steps, const lpbf_b200_opts* opts,
                           const lpbf_b200_rows* rows, Partial* ring, void* work,
                           size_t work_bytes, cudaStream_t stream);

/* Copy the workspace error word to *err (synchronizes `stream`); bit 0 means
 * a TMA wait exceeded its time limit and the launch stopped early; bit 1
 * means a computed temperature was NaN or infinite (baseline FP64 advance
 * with a ring; the Partials ignore NaN as the reference does).  The word
 * accumulates until lpbf_b200_workspace_init clears it. */
int lpbf_b200_read_error(const void* work, cudaStream_t stream, unsigned int* err);

/* FP32 compensated variant (no reference counterpart; the reference path is
 * FP64 only).  The field is two f32 arrays, hi and lo, with T = hi + lo; each
 * step adds its increment with an error-free two-sum and keeps the rounding
 * error in lo, the Gaussian source is evaluated in FP64, and per-step Partials
 * are reduced on hi + lo in FP64.  (hi_a, lo_a) holds the start field,
 * (hi_b, lo_b) the other half of the ping-pong pair; *result_in_b as for
 * lpbf_b200_advance.  Requires nx % 4 == 0 and 16-byte aligned arrays
 * (LPBF_ERR_UNSUPPORTED otherwise) and baseline physics.  Needs a workspace. */
int lpbf_b200_advance_f32k(float* hi_a, float* lo_a, float* hi_b, float* lo_b,
                           const StepConst* k, const lpbf_tick* plan, int n_steps,
                           const lpbf_b200_opts* opts, Partial* ring, void* work,
                           size_t work_bytes, cudaStream_t stream, int* result_in_b);
/* hi = (float)T, lo = (float)(T - hi), and back: T = (double)hi + (double)lo. */
int lpbf_b200_f32k_split(const double* T, float* hi, float* lo, size_t n, cudaStream_t stream);
int lpbf_b200_f32k_join(const float* hi, const float* lo, double* T, size_t n,
                        cudaStream_t stream);

/* Plain FP32 field (no reference counterpart): one f32 array, each step's
 * update rounded once (the FP64 step's operations in f32; the Gaussian source
 * evaluated in FP64 and rounded), 8 bytes per cell-update against 16 for the
 * FP64 and compensated fields.  Per-step Partials are reduced on the f32
 * values (exactly, in FP64).  T_a holds the start field, T_b the other half
 * of the ping-pong pair; *result_in_b, requirements and workspace as for
 * lpbf_b200_advance_f32k. */
int lpbf_b200_advance_f32(float* T_a, float* T_b, const StepConst* k, const lpbf_tick* plan,
                          int n_steps, const lpbf_b200_opts* opts, Partial* ring, void* work,
                          size_t work_bytes, cudaStream_t stream, int* result_in_b);

/* No counterpart in the reference.  lpbf_b200_advance without a workspace,
 * for callers that cannot allocate device memory: code running inside a
 * device-memory budget fixed at start-up, bindings that only pass raw device
 * pointers (cgo, JNI) and own no allocator, hosts where a cudaMalloc would
 * synchronize the device at a forbidden point.  Its scratch is a fixed
 * LPBF_B200_NOALLOC_SCRATCH_BYTES array in the library's device memory, held
 * by every GPU that loads the library until the process exits.
 *  - The first call on a device looks up that array's device address
 *    (cudaGetSymbolAddress) and caches it; make that first call before any
 *    stream capture.
 *  - Every call clears and reuses the same array: calls that overlap on the
 *    GPU (other streams, other threads) race and must not be issued.
 *  - Baseline physics only (phys == 1 returns LPBF_ERR_UNSUPPORTED, other
 *    phys values LPBF_ERR_ARG, as lpbf_b200_advance).
 *  - The array holds 4096 per-CTA partial records.  Each launch is clamped
 *    to 4096 / depth CTAs, so every field size fits; a launch that would
 *    still need more records is rejected with LPBF_ERR_WORKSPACE.
 *  - err (host, nullable) receives the call's error word, which otherwise
 *    stays inside the shared array: bit 0 = a bounded wait for a row copy
 *    ran out and the field is incomplete, bit 1 = a NaN or infinite
 *    temperature was seen by the per-step reduction (needs ring).  It is
 *    copied behind the call's launches on `stream`: read it after the
 *    stream has been synchronized.
 * Inputs, outputs and results are otherwise as for lpbf_b200_advance. */
#define LPBF_B200_NOALLOC_SCRATCH_BYTES 98560
int lpbf_b200_advance_noalloc(double* T_a, double* T_b, const StepConst* k,
                              const lpbf_tick* plan, int n_steps,
                              const lpbf_b200_opts* opts, Partial* ring,
                              cudaStream_t stream, int* result_in_b,
                              unsigned int* err);

/* ---- Batched process map ---------------------------------------------------
 * Replaces the reference's serial ensemble loop, one GpuStepTask graph per
 * manifest row (src/gpu/hh_gpu_main.cpp:162-270 run_one_row/run_manifest):
 * many independent fields of any sizes, lasers and plans advance together,
 * `depth` time steps per launch, in one persistent kernel per launch that
 * pulls (scenario, tile) items from a device queue.  Every scenario's field
 * and ring are bit-identical to its own lpbf_b200_advance run.
 *
 * A batch is built once (lpbf_b200_batch_create: descriptors and the whole
 * plan of every scenario go to the workspace) and run any number of times;
 * runs are stream-ordered, allocate nothing on the device, and with
 * use_graph != 0 replay one CUDA graph per (first step, step count, buffer
 * parity), captured on the first such run. */
typedef struct lpbf_b200_scenario {
    const StepConst* k;     /* host: grid, material, dt, laser peak (x_l/y_l/q_scale unused) */
    const lpbf_tick* plan;  /* host: the batch's n_steps Ticks (x_l, y_l, q_scale per step) */
    double* T_a;            /* device: start field, nx*ny f64 row-major */
    double* T_b;            /* device: the other buffer of the ping-pong pair */
    Partial* ring;          /* device, nullable: ring[i] = Partial of plan step i */
    int    bc;              /* 0 mirror edges, 1 fixed edges at T_edge */
    double T_edge;          /* [K] */
    double Tm;              /* melt threshold of the Partials [K] */
} lpbf_b200_scenario;

typedef struct lpbf_b200_batch_opts {
    int depth;              /* time steps per launch, 1..4; 0 = 3 */
    int ctas_per_sm;        /* CTAs per SM of the persistent grid; 0 = as many as fit */
    int rows[4];            /* rows per task by size class (lpbf_b200_batch_size_class); 0 = 24 */
    int staging;            /* rows into shared memory by 1 bulk row copies, 2 per-field tensor
                               maps; 0 = automatic (maps for <= 4 fields, else bulk copies);
                               fields with odd nx or 16-byte misalignment use direct loads */
} lpbf_b200_batch_opts;

typedef struct lpbf_b200_batch lpbf_b200_batch;   /* opaque host object */

/* Size class of a grid for the per-class tile shape: 0 for max(nx, ny) < 512,
 * 1 for < 1024, 2 for < 2048, 3 above. */
int lpbf_b200_batch_size_class(int nx, int ny);
/* Device workspace bytes of a batch (0 for invalid arguments).  With every
 * scenario's plan set this is exact; without plans it is an upper bound
 * that holds whatever plans lpbf_b200_batch_create is later given. */
size_t lpbf_b200_batch_workspace_bytes(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                                       const lpbf_b200_batch_opts* opts);
/* Build a batch of n_scen scenarios sharing a step count.  work: 256-byte
 * aligned device block of lpbf_b200_batch_workspace_bytes; it belongs to the
 * batch until lpbf_b200_batch_destroy.  Uploads the descriptors on `stream`
 * and synchronizes it (a set-up call, not capturable).  All fields start in
 * T_a.  *out receives a host object (host heap memory). */
int lpbf_b200_batch_create(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                           const lpbf_b200_batch_opts* opts, void* work, size_t work_bytes,
                           cudaStream_t stream, lpbf_b200_batch** out);
/* Advance every scenario through plan steps [first_step, first_step + n_steps)
 * from the buffer that holds its current field; ring entries of those steps
 * are written.  Asynchronous on `stream`. */
int lpbf_b200_batch_run(lpbf_b200_batch* b, int first_step, int n_steps, int use_graph,
                        cudaStream_t stream);
/* Capture (without launching) the graph that lpbf_b200_batch_run with
 * use_graph != 0 would replay for these steps from the current buffers, so
 * that the first such run pays no capture.  Not itself capturable. */
int lpbf_b200_batch_capture(lpbf_b200_batch* b, int first_step, int n_steps);
/* Advance steps [first_step, first_step + n_steps) one step per launch and,
 * after each step s, write w_sub[s * n_scen + i] (device f64, caller order):
 * scenario i's sub-grid melt width [um] through the column of that step's
 * hottest cell, from the two linearly interpolated T = Tm crossings (the
 * reference MetricsTask rule, include/gpu_step_task.hpp:380-395), where
 * cruise[s * n_scen + i] (device bytes) is non-zero and the step's peak
 * exceeds Tm, else 0.  Every scenario needs a ring. */
int lpbf_b200_batch_run_wsub(lpbf_b200_batch* b, int first_step, int n_steps,
                             const unsigned char* cruise, double* w_sub, cudaStream_t stream);
/* 1 when the current fields are in the T_b buffers, 0 for T_a. */
int lpbf_b200_batch_result_in_b(const lpbf_b200_batch* b);
/* Launches that a run of n_steps issues; queue items of the largest launch
 * (a scenario's rows near its laser go in shorter tasks, so the count
 * follows the laser); rows per task chosen for a scenario (caller's index). */
int lpbf_b200_batch_launches(const lpbf_b200_batch* b, int n_steps);
int lpbf_b200_batch_tasks(const lpbf_b200_batch* b);
int lpbf_b200_batch_scenario_rows(const lpbf_b200_batch* b, int scenario);
/* Error word (synchronizes `stream`): bit 0 = a copy wait exceeded its time
 * limit (the batch's counters are then undefined: destroy and re-create it);
 * bit 1 = a scenario computed a NaN or infinite temperature. */
int lpbf_b200_batch_read_error(const lpbf_b200_batch* b, cudaStream_t stream, unsigned int* err);
/* Frees the host object and its graphs; the workspace is the caller's again. */
void lpbf_b200_batch_destroy(lpbf_b200_batch* b);

/* Autotuner (no reference counterpart).  Chooses rows per size class, depth,
 * CTAs per SM and staging for this batch by timing short graph-replayed
 * runs (trial_steps steps, <= n_steps, of the scenarios' own plans) on a
 * subset of the scenarios (up to 2^27 cells per size class) in scratch
 * device memory that it allocates and frees itself: a set-up call, to be
 * made outside any stream capture, that synchronizes the device.  With
 * cache_path non-null the result is looked up first and stored after in
 * that JSON file, keyed by lpbf_b200_batch_tune_key.  T_a/T_b/ring of `sc`
 * are not touched. */
int lpbf_b200_batch_autotune(const lpbf_b200_scenario* sc, int n_scen, int n_steps,
                             const char* cache_path, int trial_steps, lpbf_b200_batch_opts* out);
/* Cache key of a batch: GPU name, SM count and the size-class histogram
 * (counts rounded up to powers of two).  Host-only. */
int lpbf_b200_batch_tune_key(const lpbf_b200_scenario* sc, int n_scen, char* buf, size_t len);
/* The tuner's JSON cache (host-only): get returns LPBF_OK and fills *out
 * when `key` is present, 1 when it is not, LPBF_ERR_ARG on a malformed
 * file; put adds or replaces `key` (atomic rename). */
int lpbf_b200_tune_cache_get(const char* path, const char* key, lpbf_b200_batch_opts* out);
int lpbf_b200_tune_cache_put(const char* path, const char* key, const lpbf_b200_batch_opts* o,
                             double gcells);

/* ---- Learned super-stepper: convolution layers on tcgen05 tensor cores ------
 * No reference counterpart (the reference has no learned component).  Each
 * call runs one 3x3 convolution layer (zero padding) over `batch` images of
 * height x width pixels as an implicit GEMM on the tensor cores: bf16
 * operands, fp32 accumulation in tensor memory.  Activations are NHWC bf16;
 * weights are packed [N][K] bf16 with K = 9 taps x C_in (tap-major, taps in
 * row-major 3x3 order, (dy, dx) = (tap / 3 - 1, tap % 3 - 1)), padded with
 * zeros to 64 when 9 x C_in < 64; N = 32, or 16 for the output layer (row 0
 * real, the rest zero).
 *   LPBF_SG_FWD_IN     C_in 4 -> 32, out = gelu(conv + bias), pre_out = conv + bias
 *   LPBF_SG_FWD_HIDDEN C_in 32 -> 32, same epilogue
 *   LPBF_SG_FWD_OUT    C_in 32 -> 1 (N = 16), out (fp32) = conv[0] + bias[0]
 *   LPBF_SG_DX_OUT     C_in 1 -> 32, out = conv * gelu'(pre_in)
 *   LPBF_SG_DX_HIDDEN  C_in 32 -> 32, out = conv * gelu'(pre_in)
 * The DX kinds give the gradient of the previous layer's pre-activation
 * when x is this layer's pre-activation gradient and the weights are packed
 * transposed with the taps flipped.  err (nullable): bit 0 set when a
 * tensor-core completion wait ran out of time. */
enum {
    LPBF_SG_FWD_IN = 0, LPBF_SG_FWD_HIDDEN = 1, LPBF_SG_FWD_OUT = 2,
    LPBF_SG_DX_OUT = 3, LPBF_SG_DX_HIDDEN = 4
};
typedef struct lpbf_b200_sg_conv_args {
    const void*  x;        /* input activations, NHWC bf16 */
    const void*  w;        /* packed weights, bf16 [N][K] */
    const float* bias;     /* [N] fp32 (forward kinds) */
    const void*  pre_in;   /* DX kinds: pre-activation of the target layer, bf16 [P][32] */
    void*        pre_out;  /* FWD_IN/FWD_HIDDEN: pre-activation out, bf16 [P][32], nullable */
    void*        out;      /* bf16 [P][32], or fp32 [P] for FWD_OUT */
    int batch, height, width;
    unsigned int* err;
} lpbf_b200_sg_conv_args;
int lpbf_b200_sg_conv(int kind, const lpbf_b200_sg_conv_args* args, cudaStream_t stream);
/* Kernel form of the 32-channel kinds (FWD_HIDDEN, FWD_OUT, DX_HIDDEN) and
 * of FWD_IN for this process, default LPBF_SG_FORM_ROWS:
 *   ROWS   input rows streamed by TMA once per run of output rows; 32
 *          channels: taps as pixel-shifted tensor-core operands; FWD_IN
 *          (even widths): each row's three x-taps written once, three MMAs
 *          per output row;
 *   TILES  32-channel kinds: nine TMA tap tiles per 128-pixel tile;
 *   PLAIN  im2col tile gathered by all threads.
 * A form that cannot run (its tensor map cannot be encoded, an odd FWD_IN
 * width) falls back to the next.  The 32-channel forms give identical
 * results; FWD_IN's forms sum the taps in other groupings (fp32).  Not
 * thread-safe against concurrent launches. */
enum { LPBF_SG_FORM_ROWS = 0, LPBF_SG_FORM_TILES = 1, LPBF_SG_FORM_PLAIN = 2 };
int lpbf_b200_sg_set_form(int form);
/* Form that ran the last FWD_IN or 32-channel launch of this process (-1:
 * none yet). */
int lpbf_b200_sg_form_used(void);
/* ---- The network: parameters, training, features ----------------------------
 * 5 layers (4 -> 32 -> 32 -> 32 -> 32 -> 1 channels, GELU after the first
 * four).  Inputs per pixel, bf16 NHWC: (T - T_amb) / LPBF_SG_T_SCALE, the
 * Gaussian source summed over the next LPBF_SG_STEPS steps / LPBF_SG_S_SCALE,
 * and the pixel's x and y offset from the laser at the middle of those steps
 * / LPBF_SG_POS_SCALE (clamped to +-8).  Output (fp32): the field's change
 * over those steps / LPBF_SG_DT_SCALE.
 * The network blob (lpbf_b200_sg_net_bytes, caller-allocated device memory)
 * holds fp32 parameters (LPBF_SG_PARAMS = lpbf_b200_sg_param_count(), layer
 * by layer W[c_out][9][c_in] then b[c_out]), their gradients, the AdamW
 * moments and the packed bf16 weights. */
#define LPBF_SG_STEPS 16
#define LPBF_SG_T_SCALE 1000.0
#define LPBF_SG_S_SCALE 1000.0
#define LPBF_SG_DT_SCALE 100.0
#define LPBF_SG_POS_SCALE 100e-6
typedef struct lpbf_b200_sg_hyper {
    float lr, beta1, beta2, eps, weight_decay;
    int step;                 /* 1-based AdamW step (bias correction) */
} lpbf_b200_sg_hyper;
int    lpbf_b200_sg_param_count(void);
size_t lpbf_b200_sg_net_bytes(void);
/* Activation workspace for batch x height x width pixels (train != 0: the
 * training step, which keeps every layer's activations and gradients). */
size_t lpbf_b200_sg_work_bytes(int batch, int height, int width, int train);
/* Set the parameters from fp32 `params` (host or device), zero the AdamW
 * moments and gradients, pack the bf16 weights. */
int lpbf_b200_sg_net_set(void* net, const float* params, cudaStream_t stream);
/* Copy parameters and/or gradients (fp32, host or device; nullable). */
int lpbf_b200_sg_net_get(const void* net, float* params, float* grads, cudaStream_t stream);
/* y (fp32, batch x height x width) from inputs x4 (bf16 [P][4]). */
int lpbf_b200_sg_forward(const void* net, const void* x4, float* y, int batch, int height,
                         int width, void* work, size_t work_bytes, unsigned int* err,
                         cudaStream_t stream);
/* Mean squared error against `target` (fp32 [P]) into *loss (device,
 * nullable) and its gradients into the blob's gradient section. */
int lpbf_b200_sg_gradients(void* net, const void* x4, const float* target, int batch, int height,
                           int width, void* work, size_t work_bytes, float* loss,
                           unsigned int* err, cudaStream_t stream);
/* One AdamW step (decoupled weight decay) from the stored gradients; repacks
 * the bf16 weights. */
int lpbf_b200_sg_adamw(void* net, const lpbf_b200_sg_hyper* h, cudaStream_t stream);
/* gradients + adamw. */
int lpbf_b200_sg_train_step(void* net, const void* x4, const float* target, int batch, int height,
                            int width, const lpbf_b200_sg_hyper* h, void* work, size_t work_bytes,
                            float* loss, unsigned int* err, cudaStream_t stream);
/* Network inputs for the field T (device, nx x ny f64) before plan[0 ..
 * LPBF_SG_STEPS) (host Ticks) into x4 (device bf16 [ny][nx][4]). */
int lpbf_b200_sg_features(const double* T, const StepConst* k, const lpbf_tick* plan,
                          void* x4, cudaStream_t stream);
/* T += y * LPBF_SG_DT_SCALE (one super-step), and the training target
 * t = (T1 - T0) / LPBF_SG_DT_SCALE. */
int lpbf_b200_sg_apply(double* T, const float* y, long long n, cudaStream_t stream);
int lpbf_b200_sg_target(const double* T0, const double* T1, float* t, long long n,
                        cudaStream_t stream);
/* C[128 x n] (fp32, row-major) = A[128 x k] . B[n x k]^T, bf16 row-major
 * operands, on the tensor cores (one CTA; n = 16 or 32, k = 288): the
 * matrix core of the layers alone, for diagnostics. */
int lpbf_b200_sg_gemm_bt(const void* A, const void* B, float* C, int n, int k,
                         unsigned int* err, cudaStream_t stream);

#ifdef __cplusplus
}  /* extern "C" */
#endif
#endif /* LPBF_B200_H */
