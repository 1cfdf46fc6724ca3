// SPDX-License-Identifier: 0BSD
// ---------------------------------------------------------------------------
// Drop-in C-ABI of liblpbf_b200.so for code written against hedgehog_lpbf.
//
// The five launch wrappers of the reference's include/lpbf_kernels.hpp:24-53,
// same names, same signatures, same contract: asynchronous on `stream`, no
// allocation (the caller owns every buffer), `*k` read on the host at launch,
// Tin/Tout must not alias, errors reported through cudaGetLastError().
// Linking liblpbf_b200.so instead of the reference's kernels.cu object is the
// whole integration step for the reference's drivers.
// ---------------------------------------------------------------------------
#pragma once
#include <cuda_runtime.h>
#include "lpbf_step_const.hpp"

extern "C" {

// One explicit-Euler step of the whole grid (phys 0 baseline, 1 extended).
// Replaces the reference lpbf_launch_step, include/lpbf_kernels.hpp:24-25.
void lpbf_launch_step(const double* Tin, double* Tout,
                      const StepConst* k, int phys, cudaStream_t stream);

// Writes `nblocks` per-block Partials (peak T, argmax with smallest-index
// ties, molten row extent); finalizing them gives the global Partial.
// Replaces the reference lpbf_launch_reduce, include/lpbf_kernels.hpp:30-31.
void lpbf_launch_reduce(const double* T, int nx, int ny, double Tm,
                        Partial* out, int nblocks, cudaStream_t stream);

// Fused step + reduce; defines all ((nx+15)/16)*((ny+15)/16) entries of
// `out` so that finalizing that many entries gives the global Partial of
// the new field.  Replaces the reference lpbf_launch_step_reduce,
// include/lpbf_kernels.hpp:37-39.
void lpbf_launch_step_reduce(const double* Tin, double* Tout,
                             const StepConst* k, int phys, double Tm,
                             Partial* out, cudaStream_t stream);

// Reduces `nblocks` Partials into out[0] on the device.  Replaces the
// reference lpbf_launch_reduce_finalize, include/lpbf_kernels.hpp:44-46.
void lpbf_launch_reduce_finalize(const Partial* parts, int nblocks,
                                 int nx, int ny, Partial* out,
                                 cudaStream_t stream);

// Copies column x_hot = glob->arg % nx of T into out_col (ny doubles).
// Replaces the reference lpbf_launch_extract_col, include/lpbf_kernels.hpp:51-53.
void lpbf_launch_extract_col(const double* T, int nx, int ny,
                             const Partial* glob, double* out_col,
                             cudaStream_t stream);

}  // extern "C"
