// Host-side declarations of the kernel launchers used by the simulation object.
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "fx_math.cuh"

namespace fx {

struct ScalarSet {
  float* f[4];  // density, temperature, fuel, reaction
};

struct VelField {
  float* c[3];  // x, y, z planes
};

struct LevelBuf {
  Dims dm;
  float* div;
  float* p[2];  // pressureA, pressureB
};

// ---------------------------------------------------------------- plain path
// One launcher per reference WGSL pass (shaders/passes/*.wgsl.ts).
void plain_inject_scalar(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet set);
void plain_inject_velocity(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, VelField v);
void plain_inject_igniter(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet set);
void plain_active_bricks(cudaStream_t s, Dims dm, uint3 bricks, ScalarSet set, uint32_t* flags);
void plain_advect_velocity(cudaStream_t s, Dims dm, const Params* P, VelField src, VelField dst);
void plain_advect_scalars(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, int mode, ScalarSet src, VelField vel,
                          const uint32_t* flags, ScalarSet dst);
void plain_combustion(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet snapshot, const uint32_t* flags,
                      ScalarSet dst);
void plain_buoyancy(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet set, const uint32_t* flags, VelField v);
void plain_vorticity(cudaStream_t s, Dims dm, VelField v, VelField w, float* wmag);
void plain_confinement(cudaStream_t s, Dims dm, const Params* P, VelField w, const float* wmag, ScalarSet set, VelField v,
                       float* fmag);
void plain_divergence(cudaStream_t s, Dims dm, VelField v, float* div);
void plain_jacobi(cudaStream_t s, Dims dm, const float* div, const float* src, float* dst);
void plain_restrict(cudaStream_t s, Dims fine, Dims coarse, const float* src, float* dst);
void plain_prolong(cudaStream_t s, Dims coarse, Dims fine, const float* coarse_p, float* fine_pa);
void plain_project(cudaStream_t s, Dims dm, VelField vsrc, const float* p, VelField vdst);
void plain_velocity_magnitude(cudaStream_t s, Dims dm, VelField v, float* out);

// The inflow patch of the differentiable rollout (an extension with no
// counterpart in the reference): velocity.y at (x0 + i, y, z0 + k) is set to
// values[i + nx k] after inject-velocity (fx_adjoint.cu).
struct InflowPatch {
  uint32_t x0, y, z0, nx, nz;
};
void plain_inflow(cudaStream_t s, Dims dm, InflowPatch p, const float* values, VelField v);

// Streaming multiprocessors of the current device (queried once per device).
int device_sm_count();

// The library's device and pinned-host allocations go through these two, so a
// test can make the n-th of them fail as an exhausted memory would
// (fx_test_fail_allocations): the call then returns cudaErrorMemoryAllocation
// without reaching CUDA.
cudaError_t device_alloc(void** ptr, size_t bytes);
cudaError_t host_alloc(void** ptr, size_t bytes);

// Stochastic binary16 rounding over an array: out[i] = sr_half(x[i], sr_draw(i, site, step)).
cudaError_t sr_half_array(const float* x, float* out, uint32_t n, uint32_t site, uint32_t step);

// Pinned sin/cos over an array (tests compare it with the oracle bit for bit).
void pinned_sincos_array(cudaStream_t s, const float* x, float* out, uint32_t n, int cosine);

}  // namespace fx
