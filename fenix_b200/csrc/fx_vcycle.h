// Weighted-Jacobi V-cycle pressure solver with FP64 norms (fx_vcycle.cu).
//
// An extension with no counterpart in the reference, whose solve is the fixed
// schedule of PressureSolvePass.ts:68-84. It uses the reference's level sizes
// (buffers.ts:10-16) and its prolongation sample position. It stops when
// ||div - A p||_2 <= tolerance * ||div||_2, both norms in FP64 on the device, or
// after max_cycles. A is the reference's unscaled 7-point operator with zero
// boundary voxels.
#pragma once

#include <cuda_runtime.h>

#include "fx_kernels.h"

namespace fx {

constexpr int kMaxVLevels = 6;
// Blocks of a norm kernel: one FP64 partial sum each.
constexpr int kNormParts = 2048;

// Device-side solver state and statistics (FP64).
struct SolverDev {
  double rhs2;                     // sum of div^2
  double res2;                     // sum of residual^2 of the latest iterate
  unsigned long long maxdiv_bits;  // max |div u| after projection (bits of a non-negative double)
  int cycles;
  int converged;
  int cont;  // 1 while another V-cycle is due
  int pad;
  double part_rhs[kNormParts];  // per-block partial sums of the norm kernels,
  double part_res[kNormParts];  // added in a fixed order by the finalize kernel
};

struct VCycleConfig {
  int levels;  // 2..kMaxVLevels
  int pre, post, coarse, max_cycles;
  float omega;
  bool omega_one;
  double tol;
  bool warm;
  bool plain;  // one-voxel kernels only (the plain path's V-cycle), never the marching ones
};

// Level k: rhs in `div`, iterate in p[0]/p[1]; level 0 is the fine pressure.
struct VCycleLevels {
  LevelBuf lv[kMaxVLevels];
};

// Before the loop: zero the statistics, clear the fine iterate unless warm
// starting, the norm of div and of the initial residual, and the first
// continue decision (sets `cond` when non-zero).
cudaError_t vcycle_prologue(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                            cudaGraphConditionalHandle cond);

// One V-cycle from fine buffer `start` (ends in the same buffer), then the
// residual norm and the continue decision (sets `cond` when non-zero).
// *launches counts the kernels.
cudaError_t vcycle_body(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                        cudaGraphConditionalHandle cond, uint32_t* launches);

// FP64 norms of the reference solve's result (no cycles): rhs, residual, decision.
cudaError_t solver_norms(cudaStream_t s, Dims dm, const float* div, const float* p, double tol, SolverDev* st);

// max |0.5 (central differences of v)| over interior voxels, in FP64.
cudaError_t max_divergence(cudaStream_t s, Dims dm, VelField v, SolverDev* st);
// Once per device before the first V-cycle (the tail kernel's shared memory).
cudaError_t vcycle_init();

}  // namespace fx
