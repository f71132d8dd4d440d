// Reverse-mode (adjoint) kernels of the plain FP32 step, and the inflow control
// of the differentiable rollout.
//
// Each adj_* launcher maps the adjoint (lambda) of a pass's outputs to the
// adjoint of its inputs, given the inputs the forward pass read. Brick flags,
// emitter sources and the step uniform are constants of the differentiation.
// A branch (min, max, clamp, the MacCormack limiter) passes the adjoint of the
// operand it selected in the forward pass.
#pragma once

#include "fx_kernels.h"

namespace fx {


// loss += sum (d - target)^2 in FP64 (loss is a device double; each difference is
// formed in FP64); lam_d = 2 (d - target) rounded to f32 (when lam_d is not NULL).
void adj_loss(cudaStream_t s, uint32_t n, const float* d, const float* target, float* lam_d, double* loss);

// project-velocity: lam_c = lambda of the projected velocity at interior voxels
// (0 on the boundary); lam_p = its pressure part (both assigned).
void adj_project(cudaStream_t s, Dims dm, VelField lam_v, VelField lam_c, float* lam_p);
// pressure-jacobi (src -> dst): lam_src += J^T lam_dst, lam_div += -lam_dst / 6.
// accumulate false: lam_src is taken as zero and written whole (lam_src = J^T lam_dst).
void adj_jacobi(cudaStream_t s, Dims dm, const float* lam_dst, float* lam_src, float* lam_div, bool accumulate);
// pressure-restriction (fine.div -> coarse.div): lam_fine += scatter (atomics).
void adj_restrict(cudaStream_t s, Dims fine, Dims coarse, const float* lam_coarse, float* lam_fine);
// pressure-prolongation (coarse p -> fine pressureA +=): lam_cp += scatter
// (atomics); lam_fpa is zeroed on the fine boundary.
void adj_prolong(cudaStream_t s, Dims coarse, Dims fine, float* lam_fpa, float* lam_cp);
// compute-divergence: lam_c += D^T lam_div.
void adj_divergence(cudaStream_t s, Dims dm, const float* lam_div, VelField lam_c);
// apply-vorticity-confinement: lam_v (in: after, out: before) in place; writes
// lam_w, lam_wmag (local part) and lam_g (the |w| gradient), adds the scalar
// parts to lam_set (density, temperature, reaction).
void adj_confinement(cudaStream_t s, Dims dm, const Params* P, VelField w, const float* wmag, ScalarSet set, VelField v,
                     VelField lam_v, VelField lam_w, float* lam_wmag, VelField lam_g, ScalarSet lam_set);
// compute-vorticity: lam_v += curl^T (lam_w + lam_wmag w / |w|), with the |w|
// gradient part of lam_wmag gathered from lam_g.
void adj_vorticity(cudaStream_t s, Dims dm, VelField w, const float* wmag, VelField lam_w, const float* lam_wmag, VelField lam_g,
                   VelField lam_v);
// apply-buoyancy (masked by flags): lam_v in place; lam_set += scalar parts.
// hot, dens: zeroed scratch fields of n floats.
void adj_buoyancy(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet set, const uint32_t* flags, VelField v,
                  VelField lam_v, ScalarSet lam_set, float* hot, float* dens);
// combustion-update (masked by flags, reading the snapshot `snap`): lam_set in
// place from the outputs' to the inputs'. hot: a zeroed scratch field.
void adj_combustion(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet snap, const uint32_t* flags, ScalarSet lam_set,
                    float* hot);
// advect-scalar-maccormack (masked by flags): from lam_out (the advected set)
// to lam_src += (atomics, zeroed by the caller) and lam_vel += (atomics).
void adj_advect_scalars(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet src, VelField vel, const uint32_t* flags,
                        ScalarSet lam_out, ScalarSet lam_src, VelField lam_vel);
// advect-velocity-semilagrangian: lam_src += (atomics, zeroed by the caller).
void adj_advect_velocity(cudaStream_t s, Dims dm, const Params* P, VelField src, VelField lam_dst, VelField lam_src);
// inject-igniter: lam_set in place (temperature, fuel, reaction) given the
// temperature and reaction before the pass and the fuel it read.
void adj_inject_igniter(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, const float* t_before,
                        const float* fuel, const float* r_before, ScalarSet lam_set);
// The inflow patch: grad += lam_v.y at the patch; lam_v.y there is zeroed.
void adj_inflow(cudaStream_t s, Dims dm, InflowPatch p, VelField lam_v, float* grad);
// inject-velocity (with the speed clamp): lam_v in place given the velocity before.
void adj_inject_velocity(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, VelField v_before, VelField lam_v);
// inject-scalar: lam_set in place (density, temperature, fuel) given the set before.
void adj_inject_scalar(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet before, ScalarSet lam_set);

}  // namespace fx
