// Fine-level pressure passes of the fused path (fx_pressure.cu).
#pragma once

#include <cuda_runtime.h>

#include "fx_kernels.h"

namespace fx {

// Stage-0 input of a pass.
enum ZInput {
  ZIN_ZERO = 0,          // the cleared buffer: the first sweep is (0 - div) / 6
  ZIN_BUF = 1,           // p_in
  ZIN_BUF_PROLONG = 2,   // p_in + prolongation of mid_p (boundary 0)
  ZIN_ZERO_PROLONG = 3,  // 0 + prolongation of mid_p (boundary 0)
};

struct ZPass {
  Dims dm;
  Dims mid;
  int zchunk;            // planes per block (0 = default)
  int sweeps;            // 0..4
  ZInput input;
  bool div_from_velocity;  // compute the divergence of vfin (and write div_out, mid_div)
  bool project;            // finish with the projection of vfin into vcur
  int restrict_mid;        // with div_from_velocity: also write the fine->mid restriction
  const float* p_in;
  const float* div_in;
  float* div_out;
  float* mid_div;
  const float* mid_p;
  float* p_out;
  VelField vfin;
  VelField vcur;
  float* vmag;
  int write_vmag;
};

cudaError_t zpass_launch(cudaStream_t s, const ZPass& p);

// Tuning of the fine passes: sweeps fused per pass (1..4) and planes per block.
// Defaults come from measurement; FENIX_ZPASS_SWEEPS / FENIX_ZPASS_ZCHUNK override.
int zpass_max_sweeps();
int zpass_zchunk();

// Lean per-voxel kernels of the default pressure plan.
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

bool sweep_variant_valid(int variant, Dims dm);
int sweep_variant_default(Dims dm);
cudaError_t lean_sweep_variant(cudaStream_t s, int variant, Dims dm, const float* div, const float* src, float* dst, Dims mid,
                               const float* mid_p);
cudaError_t lean_prolong_zero(cudaStream_t s, Dims dm, float* dst, Dims mid, const float* mid_p);

// The mid/coarse part of the solve in one cooperative launch. `bar` is 96
// zeroed device words: [0] arrivals, [32] generation, [64] error flag (set when
// a grid barrier times out). *mid_result gets the id of the mid buffer
// holding the result.
cudaError_t mg_lower_launch(cudaStream_t s, const LevelBuf& mid, const LevelBuf& coarse, int mid_pre, int coarse_n, int mid_post,
                            unsigned* bar, int* mid_result);

// Mid/coarse levels: 0 = kernel per sweep (default), 1 = one cooperative launch (FENIX_MG_PLAN=1).
int multigrid_plan();

// 0: per-voxel sweeps (default); 1: z-march passes (FENIX_PRESSURE_PLAN=1).
int pressure_plan();

// Counts the floats x (all 2^32 bit patterns, NaNs excluded) for which the
// pressure kernels' division by 6 differs from the IEEE quotient x / 6.0f.
cudaError_t div6_exhaustive_check(unsigned long long* host_bad);

}  // namespace fx
