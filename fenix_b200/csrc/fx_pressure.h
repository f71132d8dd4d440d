// Fine-level pressure passes of the fused path (fx_pressure.cu).
#pragma once

#include <cuda_runtime.h>

#include "fx_kernels.h"

namespace fx {

// Per-voxel kernels of the fine pressure passes.
cudaError_t lean_div_first(cudaStream_t s, Dims dm, VelField v, float* div, float* p1, Dims mid, float* mid_div, bool restrict_mid);
cudaError_t lean_sweep(cudaStream_t s, Dims dm, const float* div, const float* src, float* dst, Dims mid, const float* mid_p);

// Sweep kernel variants (all give the same bits): one x per thread with z-depth
// 2, 4 or 8, two x per thread (even widths) with z-depth 2 or 4, four x per
// thread (widths divisible by 4) with z-depth 2, 4 or 1, or four x per thread
// marching runs of planes with the next plane's loads in flight. An invalid
// variant (-1, or a vector variant on a width it does not divide) takes the
// default.
enum SweepVariant {
  SWEEP_Z2 = 0,
  SWEEP_Z4 = 1,
  SWEEP_Z8 = 2,
  SWEEP_VEC_Z2 = 3,   // two x per thread (even widths)
  SWEEP_VEC_Z4 = 4,
  SWEEP_VEC4_Z2 = 5,  // four x per thread (widths divisible by 4)
  SWEEP_VEC4_Z4 = 6,
  SWEEP_VEC4_Z1 = 7,
  SWEEP_VEC4_MARCH = 8,  // four x per thread, one wave of blocks marching in z
  kSweepVariants = 9
};
// Planes per block of a marching kernel (host arithmetic; `slots` = resident
// blocks of the kernel on the device). One wave over 128 x 8 row tiles: the
// tiles times the runs fill the slots once (at most one run per plane).
int march_plan_one_wave(Dims dm, int slots);
// The same with runs of an even number of planes (dm.d even), for kernels that
// pair planes.
int march_plan_pairs(Dims dm, int slots);
// Over tx x ty tiles: the run count (at most one per 8 planes) whose blocks fill
// whole waves of the slots best, the fewest runs among equals.
int march_plan_waves(Dims dm, int tx, int ty, int slots);

// The V-cycle's weighted sweep (dst = src + w (J(src) - src); J(src) itself
// when `one`) as the marching four-x kernel: same bits as the V-cycle's
// one-x kernel. cudaErrorNotSupported where the width is not a multiple of 4.
cudaError_t march_wsweep(cudaStream_t s, Dims dm, const float* rhs, const float* src, float* dst, float w, bool one);
// march_wsweep that also writes the FP64 squared residual norm of src, one
// partial per block, into part (at most *nparts; *nparts gets the count).
// cudaErrorNotSupported where march_wsweep refuses or the blocks outnumber *nparts.
cudaError_t march_wsweep_norm(cudaStream_t s, Dims dm, const float* rhs, const float* src, float* dst, float w, bool one,
                              double* part, int* nparts);

bool sweep_variant_valid(int variant, Dims dm);
int sweep_variant_default(Dims dm);
// slot_pct < 100 plans the marching sweep for that share of the resident blocks
// (longer runs, the rest of each SM free for another stream's kernels); the
// results are the same bits.
cudaError_t lean_sweep_variant(cudaStream_t s, int variant, Dims dm, const float* div, const float* src, float* dst, Dims mid,
                               const float* mid_p, int slot_pct = 100);
// The share of the resident blocks for the fine sweeps that run beside the mid
// and coarse levels (FENIX_MARCH_SHARE, percent; default 50).
int march_share_pct();
cudaError_t lean_prolong_zero(cudaStream_t s, Dims dm, float* dst, Dims mid, const float* mid_p);

// Counts the floats x (all 2^32 bit patterns, NaNs excluded) for which the
// pressure kernels' division by 6 differs from the IEEE quotient x / 6.0f.
cudaError_t div6_exhaustive_check(unsigned long long* host_bad);

}  // namespace fx
