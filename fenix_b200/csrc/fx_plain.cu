// The plain FP32 CUDA step: one kernel per reference WGSL pass, one thread per
// voxel (or per brick for the flag pass), dense over the grid exactly like the
// reference's dispatches (runtime/shared/createVolumeDispatch.ts:5-21). This path
// is kept as the measured "plain FP32" baseline of the fused path; both produce
// the same bits.
#include "fx_kernels.h"

namespace fx {
namespace {

constexpr dim3 kBlock(32, 4, 2);

inline dim3 grid_for(Dims d) { return dim3((d.w + kBlock.x - 1) / kBlock.x, (d.h + kBlock.y - 1) / kBlock.y, (d.d + kBlock.z - 1) / kBlock.z); }

#define FX_VOXEL_PROLOGUE(dm)                                  \
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;    \
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;    \
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z;    \
  if (x >= (dm).w || y >= (dm).h || z >= (dm).d) return;       \
  const uint32_t i = flat(dm, x, y, z)

FX_DEV void voxel_pos(const Dims& dm, uint32_t x, uint32_t y, uint32_t z, float& px, float& py, float& pz) {
  px = ((float)x + 0.5f) / (float)dm.w;
  py = ((float)y + 0.5f) / (float)dm.h;
  pz = ((float)z + 0.5f) / (float)dm.d;
}

// shaders/passes/inject-scalar.wgsl.ts:32-70
__global__ void k_inject_scalar(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc, ScalarSet set) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  float d = set.f[0][i], t = set.f[1][i], f = set.f[2][i];
  inject_scalar_voxel(P, src, nsrc, px, py, pz, d, t, f);
  set.f[0][i] = d;
  set.f[1][i] = t;
  set.f[2][i] = f;
}

// shaders/passes/inject-velocity.wgsl.ts:46-96
__global__ void k_inject_velocity(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc, VelField v) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  float vx = v.c[0][i], vy = v.c[1][i], vz = v.c[2][i];
  inject_velocity_voxel(P, src, nsrc, px, py, pz, vx, vy, vz);
  const float lim = speed_limit(P);
  v.c[0][i] = clampv(vx, -lim, lim);
  v.c[1][i] = clampv(vy, -lim, lim);
  v.c[2][i] = clampv(vz, -lim, lim);
}

// shaders/passes/inject-igniter.wgsl.ts:32-66
__global__ void k_inject_igniter(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc, ScalarSet set) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  float r = set.f[3][i], t = set.f[1][i];
  inject_igniter_voxel(P, src, nsrc, px, py, pz, set.f[2][i], r, t);
  set.f[3][i] = r;
  set.f[1][i] = t;
}

// shaders/passes/compute-active-bricks.wgsl.ts:24-79 (one thread per brick)
__global__ void k_active_bricks(Dims dm, uint3 bc, ScalarSet set, uint32_t* __restrict__ flags) {
  const uint32_t bx = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t by = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t bz = blockIdx.z * blockDim.z + threadIdx.z;
  if (bx >= bc.x || by >= bc.y || bz >= bc.z) return;
  const uint32_t x0 = bx * 8u, y0 = by * 8u, z0 = bz * 8u;
  bool active = false;
  float peak = 0.0f;
  for (uint32_t zz = 0; zz < 8u; zz += 2u)
    for (uint32_t yy = 0; yy < 8u; yy += 2u)
      for (uint32_t xx = 0; xx < 8u; xx += 2u) {
        const uint32_t cx = x0 + xx, cy = y0 + yy, cz = z0 + zz;
        if (cx < dm.w && cy < dm.h && cz < dm.d) {
          const uint32_t j = flat(dm, cx, cy, cz);
          const float e = set.f[0][j] + set.f[1][j] * 0.7f + set.f[3][j] * 0.9f;
          peak = mx(peak, e);
          if (e > 0.012f) active = true;
        }
      }
  const uint32_t ccx = min(x0 + 4u, dm.w - 1u), ccy = min(y0 + 4u, dm.h - 1u), ccz = min(z0 + 4u, dm.d - 1u);
  const uint32_t cj = flat(dm, ccx, ccy, ccz);
  const float ce = set.f[0][cj] + set.f[1][cj] * 0.7f + set.f[3][cj] * 0.9f;
  peak = mx(peak, ce);
  if (ce > 0.012f) active = true;
  if (!active) return;
  const int rad = (peak > 0.05f || ce > 0.035f) ? 1 : 0;
  for (int dz = -rad; dz <= rad; ++dz)
    for (int dy = -rad; dy <= rad; ++dy)
      for (int dx = -rad; dx <= rad; ++dx) {
        const uint32_t nx = (uint32_t)min(max((int)bx + dx, 0), (int)bc.x - 1);
        const uint32_t ny = (uint32_t)min(max((int)by + dy, 0), (int)bc.y - 1);
        const uint32_t nz = (uint32_t)min(max((int)bz + dz, 0), (int)bc.z - 1);
        flags[nx + bc.x * (ny + bc.y * nz)] = 1u;
      }
}

FX_DEV bool is_active_coord(const uint32_t* __restrict__ flags, uint3 bc, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t bx = min(x >> 3, bc.x - 1u), by = min(y >> 3, bc.y - 1u), bz = min(z >> 3, bc.z - 1u);
  return __ldg(flags + bx + bc.x * (by + bc.y * bz)) != 0u;
}

// shaders/passes/advect-velocity-semilagrangian.wgsl.ts:23-41
__global__ void k_advect_velocity(Dims dm, const Params* __restrict__ Pp, VelField src, VelField dst) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    dst.c[0][i] = 0.0f;
    dst.c[1][i] = 0.0f;
    dst.c[2][i] = 0.0f;
    return;
  }
  const float dt = Pp->dt;
  const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
  const Tri c0 = tri_corners(dm, cx - 0.5f, cy - 0.5f, cz - 0.5f);
  const float v0x = tri_interp(src.c[0], c0), v0y = tri_interp(src.c[1], c0), v0z = tri_interp(src.c[2], c0);
  const float bx = cx - v0x * dt, by = cy - v0y * dt, bz = cz - v0z * dt;
  const Tri c1 = tri_corners(dm, bx - 0.5f, by - 0.5f, bz - 0.5f);
  const float damp = 1.0f - dt * 0.025f;
  dst.c[0][i] = tri_interp(src.c[0], c1) * damp;
  dst.c[1][i] = tri_interp(src.c[1], c1) * damp;
  dst.c[2][i] = tri_interp(src.c[2], c1) * damp;
}

// shaders/passes/advect-scalar-maccormack.wgsl.ts:33-101 (mode 1) and
// advect-scalar-semilagrangian.wgsl.ts:26-44,76-104 (mode 0)
__global__ void k_advect_scalars(Dims dm, uint3 bc, const Params* __restrict__ Pp, int mode, ScalarSet src, VelField vel,
                                 const uint32_t* __restrict__ flags, ScalarSet dst) {
  FX_VOXEL_PROLOGUE(dm);
  if (!is_active_coord(flags, bc, x, y, z)) {
    dst.f[0][i] = 0.0f;
    dst.f[1][i] = 0.0f;
    dst.f[2][i] = 0.0f;
    dst.f[3][i] = 0.0f;
    return;
  }
  const Params P = *Pp;
  const float dt = P.dt;
  const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
  const Tri c0 = tri_corners(dm, cx - 0.5f, cy - 0.5f, cz - 0.5f);
  const float vx = tri_interp(vel.c[0], c0), vy = tri_interp(vel.c[1], c0), vz = tri_interp(vel.c[2], c0);
  const float bx = cx - vx * dt, by = cy - vy * dt, bz = cz - vz * dt;
  const float spx = bx - 0.5f, spy = by - 0.5f, spz = bz - 0.5f;
  const Tri cs = tri_corners(dm, spx, spy, spz);
  float out[4];
  float noise;
  if (mode == 1) {
    const float fvx = tri_interp(vel.c[0], cs), fvy = tri_interp(vel.c[1], cs), fvz = tri_interp(vel.c[2], cs);
    const float rx = bx + fvx * dt, ry = by + fvy * dt, rz = bz + fvz * dt;
    const Tri cr = tri_corners(dm, rx - 0.5f, ry - 0.5f, rz - 0.5f);
#pragma unroll
    for (int f = 0; f < 4; ++f) {
      const float predicted = tri_interp(src.f[f], cs);
      const float recovered = tri_interp(src.f[f], cr);
      const float original = tri_interp(src.f[f], c0);
      const float corrected = predicted + 0.5f * (original - recovered);
      out[f] = clampv(corrected, mn(original, predicted), mx(original, predicted));
    }
    noise = thermal_noise(P, cx, cy, cz);
  } else {
#pragma unroll
    for (int f = 0; f < 4; ++f) out[f] = tri_interp(src.f[f], cs);
    noise = thermal_noise(P, spx, spy, spz);
  }
  const float ny = ((float)y + 0.5f) / (float)dm.h;
  decay_scalars(P, ny, noise, out[0], out[1], out[2], out[3]);
  dst.f[0][i] = out[0];
  dst.f[1][i] = out[1];
  dst.f[2][i] = out[2];
  dst.f[3][i] = out[3];
}

// shaders/passes/combustion-update.wgsl.ts:42-93 reading every neighbour from
// `snap`, a copy of the set taken before the pass.
__global__ void k_combustion(Dims dm, uint3 bc, const Params* __restrict__ Pp, ScalarSet snap, const uint32_t* __restrict__ flags,
                             ScalarSet dst) {
  FX_VOXEL_PROLOGUE(dm);
  if (!is_active_coord(flags, bc, x, y, z)) return;
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  auto hot = [&](uint32_t xx, uint32_t yy, uint32_t zz) {
    const uint32_t j = flat(dm, xx, yy, zz);
    return comb_hot(__ldg(snap.f[1] + j), __ldg(snap.f[2] + j), __ldg(snap.f[3] + j));
  };
  const float nsum = hot(inc(x, W1), y, z) + hot(dec(x), y, z) + hot(x, inc(y, H1), z) + hot(x, dec(y), z) + hot(x, y, inc(z, D1)) +
                     hot(x, y, dec(z));
  float d = snap.f[0][i], t = snap.f[1][i], f = snap.f[2][i], r = snap.f[3][i];
  const float ny = ((float)y + 0.5f) / (float)dm.h;
  combustion_voxel(P, x, y, z, ny, nsum, d, t, f, r);
  dst.f[0][i] = d;
  dst.f[1][i] = t;
  dst.f[2][i] = f;
  dst.f[3][i] = r;
}

// shaders/passes/apply-buoyancy.wgsl.ts:37-110
__global__ void k_buoyancy(Dims dm, uint3 bc, const Params* __restrict__ Pp, ScalarSet set, const uint32_t* __restrict__ flags, VelField v) {
  FX_VOXEL_PROLOGUE(dm);
  if (!is_active_coord(flags, bc, x, y, z)) return;
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float* D = set.f[0];
  auto hot = [&](uint32_t xx, uint32_t yy, uint32_t zz) {
    const uint32_t j = flat(dm, xx, yy, zz);
    return buoy_hot(set.f[1][j], set.f[3][j]);
  };
  const float hot_gas = hot(x, y, z);
  const float tgx = (hot(inc(x, W1), y, z) - hot(dec(x), y, z)) * 0.5f;
  const float tgy = (hot(x, inc(y, H1), z) - hot(x, dec(y), z)) * 0.5f;
  const float tgz = (hot(x, y, inc(z, D1)) - hot(x, y, dec(z))) * 0.5f;
  const float dgx = (D[flat(dm, inc(x, W1), y, z)] - D[flat(dm, dec(x), y, z)]) * 0.5f;
  const float dgy = (D[flat(dm, x, inc(y, H1), z)] - D[flat(dm, x, dec(y), z)]) * 0.5f;
  const float dgz = (D[flat(dm, x, y, inc(z, D1))] - D[flat(dm, x, y, dec(z))]) * 0.5f;
  float vx = v.c[0][i], vy = v.c[1][i], vz = v.c[2][i];
  buoyancy_voxel(P, dm, x, y, z, D[i], hot_gas, tgx, tgy, tgz, dgx, dgy, dgz, vx, vy, vz);
  v.c[0][i] = vx;
  v.c[1][i] = vy;
  v.c[2][i] = vz;
}

// shaders/passes/compute-vorticity.wgsl.ts:23-50
__global__ void k_vorticity(Dims dm, VelField v, VelField w, float* __restrict__ wmag) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    w.c[0][i] = 0.0f;
    w.c[1][i] = 0.0f;
    w.c[2][i] = 0.0f;
    wmag[i] = 0.0f;
    return;
  }
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const uint32_t x0 = flat(dm, dec(x), y, z), x1 = flat(dm, inc(x, W1), y, z);
  const uint32_t y0 = flat(dm, x, dec(y), z), y1 = flat(dm, x, inc(y, H1), z);
  const uint32_t z0 = flat(dm, x, y, dec(z)), z1 = flat(dm, x, y, inc(z, D1));
  const float cx = ((v.c[2][y1] - v.c[2][y0]) - (v.c[1][z1] - v.c[1][z0])) * 0.5f;
  const float cy = ((v.c[0][z1] - v.c[0][z0]) - (v.c[2][x1] - v.c[2][x0])) * 0.5f;
  const float cz = ((v.c[1][x1] - v.c[1][x0]) - (v.c[0][y1] - v.c[0][y0])) * 0.5f;
  w.c[0][i] = cx;
  w.c[1][i] = cy;
  w.c[2][i] = cz;
  wmag[i] = length3(cx, cy, cz);
}

// shaders/passes/apply-vorticity-confinement.wgsl.ts:30-66
__global__ void k_confinement(Dims dm, const Params* __restrict__ Pp, VelField w, const float* __restrict__ wmag, ScalarSet set, VelField v,
                              float* __restrict__ fmag) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    fmag[i] = 0.0f;
    return;
  }
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float gx = (wmag[flat(dm, inc(x, W1), y, z)] - wmag[flat(dm, dec(x), y, z)]) * 0.5f;
  const float gy = (wmag[flat(dm, x, inc(y, H1), z)] - wmag[flat(dm, x, dec(y), z)]) * 0.5f;
  const float gz = (wmag[flat(dm, x, y, inc(z, D1))] - wmag[flat(dm, x, y, dec(z))]) * 0.5f;
  float vx = v.c[0][i], vy = v.c[1][i], vz = v.c[2][i];
  fmag[i] = confinement_voxel(P, gx, gy, gz, w.c[0][i], w.c[1][i], w.c[2][i], wmag[i], set.f[0][i], set.f[1][i], set.f[3][i], vx, vy, vz);
  v.c[0][i] = vx;
  v.c[1][i] = vy;
  v.c[2][i] = vz;
}

// shaders/passes/compute-divergence.wgsl.ts:22-42
__global__ void k_divergence(Dims dm, VelField v, float* __restrict__ div) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    div[i] = 0.0f;
    return;
  }
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float ddx = v.c[0][flat(dm, inc(x, W1), y, z)] - v.c[0][flat(dm, dec(x), y, z)];
  const float ddy = v.c[1][flat(dm, x, inc(y, H1), z)] - v.c[1][flat(dm, x, dec(y), z)];
  const float ddz = v.c[2][flat(dm, x, y, inc(z, D1))] - v.c[2][flat(dm, x, y, dec(z))];
  div[i] = (ddx + ddy + ddz) * 0.5f;
}

// shaders/passes/pressure-jacobi.wgsl.ts:15-36
__global__ void k_jacobi(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    dst[i] = 0.0f;
    return;
  }
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float s = src[flat(dm, inc(x, W1), y, z)] + src[flat(dm, dec(x), y, z)] + src[flat(dm, x, inc(y, H1), z)] +
                  src[flat(dm, x, dec(y), z)] + src[flat(dm, x, y, inc(z, D1))] + src[flat(dm, x, y, dec(z))];
  dst[i] = (s - div[i]) / 6.0f;
}

// shaders/passes/pressure-restriction.wgsl.ts:27-50
__global__ void k_restrict(Dims fine, Dims dm, const float* __restrict__ src, float* __restrict__ dst) {
  FX_VOXEL_PROLOGUE(dm);
  if (x == 0u || y == 0u || z == 0u || x == dm.w - 1u || y == dm.h - 1u || z == dm.d - 1u) {
    dst[i] = 0.0f;
    return;
  }
  float sum = 0.0f;
  for (uint32_t dz = 0; dz < 2u; ++dz)
    for (uint32_t dy = 0; dy < 2u; ++dy)
      for (uint32_t dx = 0; dx < 2u; ++dx) {
        const uint32_t sx = min(2u * x + dx, fine.w - 1u), sy = min(2u * y + dy, fine.h - 1u), sz = min(2u * z + dz, fine.d - 1u);
        sum += src[flat(fine, sx, sy, sz)];
      }
  dst[i] = sum * 0.125f;
}

// shaders/passes/pressure-prolongation.wgsl.ts:29-44
__global__ void k_prolong(Dims coarse, Dims dm, const float* __restrict__ cp, float* __restrict__ fine_pa) {
  FX_VOXEL_PROLOGUE(dm);
  if (x == 0u || y == 0u || z == 0u || x == dm.w - 1u || y == dm.h - 1u || z == dm.d - 1u) {
    fine_pa[i] = 0.0f;
    return;
  }
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  fine_pa[i] += tri_interp(cp, tri_corners(coarse, px, py, pz));
}

// shaders/passes/project-velocity.wgsl.ts:21-43
__global__ void k_project(Dims dm, VelField vs, const float* __restrict__ p, VelField vd) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
    vd.c[0][i] = 0.0f;
    vd.c[1][i] = 0.0f;
    vd.c[2][i] = 0.0f;
    return;
  }
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float gx = (p[flat(dm, inc(x, W1), y, z)] - p[flat(dm, dec(x), y, z)]) * 0.5f;
  const float gy = (p[flat(dm, x, inc(y, H1), z)] - p[flat(dm, x, dec(y), z)]) * 0.5f;
  const float gz = (p[flat(dm, x, y, inc(z, D1))] - p[flat(dm, x, y, dec(z))]) * 0.5f;
  vd.c[0][i] = vs.c[0][i] - gx;
  vd.c[1][i] = vs.c[1][i] - gy;
  vd.c[2][i] = vs.c[2][i] - gz;
}

// shaders/passes/compute-debug-fields.wgsl.ts:18-25
__global__ void k_velocity_magnitude(Dims dm, VelField v, float* __restrict__ out) {
  FX_VOXEL_PROLOGUE(dm);
  out[i] = length3(v.c[0][i], v.c[1][i], v.c[2][i]);
}

__global__ void k_sr_half(const float* __restrict__ x, float* __restrict__ out, uint32_t n, uint32_t site, uint32_t step) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = sr_half(x[i], sr_draw(i, site, step));
}

__global__ void k_pinned_sincos(const float* __restrict__ x, float* __restrict__ out, uint32_t n, int cosine) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) out[i] = cosine ? pcos(x[i]) : psin(x[i]);
}

}  // namespace

void plain_inject_scalar(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet set) {
  k_inject_scalar<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, set);
}
void plain_inject_velocity(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, VelField v) {
  k_inject_velocity<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, v);
}
void plain_inject_igniter(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet set) {
  k_inject_igniter<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, set);
}
void plain_active_bricks(cudaStream_t s, Dims dm, uint3 bricks, ScalarSet set, uint32_t* flags) {
  const dim3 blk(8, 4, 4);
  const dim3 grd((bricks.x + blk.x - 1) / blk.x, (bricks.y + blk.y - 1) / blk.y, (bricks.z + blk.z - 1) / blk.z);
  k_active_bricks<<<grd, blk, 0, s>>>(dm, bricks, set, flags);
}
void plain_advect_velocity(cudaStream_t s, Dims dm, const Params* P, VelField src, VelField dst) {
  k_advect_velocity<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, dst);
}
void plain_advect_scalars(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, int mode, ScalarSet src, VelField vel,
                          const uint32_t* flags, ScalarSet dst) {
  k_advect_scalars<<<grid_for(dm), kBlock, 0, s>>>(dm, bricks, P, mode, src, vel, flags, dst);
}
void plain_combustion(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet snapshot, const uint32_t* flags, ScalarSet dst) {
  k_combustion<<<grid_for(dm), kBlock, 0, s>>>(dm, bricks, P, snapshot, flags, dst);
}
void plain_buoyancy(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet set, const uint32_t* flags, VelField v) {
  k_buoyancy<<<grid_for(dm), kBlock, 0, s>>>(dm, bricks, P, set, flags, v);
}
void plain_vorticity(cudaStream_t s, Dims dm, VelField v, VelField w, float* wmag) {
  k_vorticity<<<grid_for(dm), kBlock, 0, s>>>(dm, v, w, wmag);
}
void plain_confinement(cudaStream_t s, Dims dm, const Params* P, VelField w, const float* wmag, ScalarSet set, VelField v, float* fmag) {
  k_confinement<<<grid_for(dm), kBlock, 0, s>>>(dm, P, w, wmag, set, v, fmag);
}
void plain_divergence(cudaStream_t s, Dims dm, VelField v, float* div) { k_divergence<<<grid_for(dm), kBlock, 0, s>>>(dm, v, div); }
void plain_jacobi(cudaStream_t s, Dims dm, const float* div, const float* src, float* dst) {
  k_jacobi<<<grid_for(dm), kBlock, 0, s>>>(dm, div, src, dst);
}
void plain_restrict(cudaStream_t s, Dims fine, Dims coarse, const float* src, float* dst) {
  k_restrict<<<grid_for(coarse), kBlock, 0, s>>>(fine, coarse, src, dst);
}
void plain_prolong(cudaStream_t s, Dims coarse, Dims fine, const float* coarse_p, float* fine_pa) {
  k_prolong<<<grid_for(fine), kBlock, 0, s>>>(coarse, fine, coarse_p, fine_pa);
}
void plain_project(cudaStream_t s, Dims dm, VelField vsrc, const float* p, VelField vdst) {
  k_project<<<grid_for(dm), kBlock, 0, s>>>(dm, vsrc, p, vdst);
}
void plain_velocity_magnitude(cudaStream_t s, Dims dm, VelField v, float* out) {
  k_velocity_magnitude<<<grid_for(dm), kBlock, 0, s>>>(dm, v, out);
}
void pinned_sincos_array(cudaStream_t s, const float* x, float* out, uint32_t n, int cosine) {
  if (n == 0) return;
  k_pinned_sincos<<<(n + 255) / 256, 256, 0, s>>>(x, out, n, cosine);
}

cudaError_t sr_half_array(const float* x, float* out, uint32_t n, uint32_t site, uint32_t step) {
  if (n == 0) return cudaSuccess;
  k_sr_half<<<(n + 255) / 256, 256>>>(x, out, n, site, step);
  return cudaGetLastError();
}

}  // namespace fx
