// Reverse-mode kernels of the plain FP32 step (see fx_adjoint.h).
//
// Layout and order follow the forward kernels of fx_plain.cu: one thread per
// voxel over the dense grid. Pointwise source terms (injection, the decay block,
// combustion, buoyancy, confinement) get their local Jacobian by evaluating the
// forward's own per-voxel function (fx_math.cuh) on dual numbers, so each branch
// is the one the forward took. Trilinear gathers scatter their adjoint to the
// eight corners with atomics (the transposed trilinear scatter) and add the
// position term through the sample position's clamp. Linear stencils
// (divergence, the pressure schedule, projection, vorticity) are transposed as
// gathers over the interior voxels that read a given voxel; an interior voxel's
// neighbours are never clamped, so the gathers are exact.
#include <cuda_runtime.h>

#include "fx_adjoint.h"
#include "fx_dual.cuh"

namespace fx {
namespace {

constexpr dim3 kBlock(32, 4, 2);

inline dim3 grid_for(Dims d) { return dim3((d.w + kBlock.x - 1) / kBlock.x, (d.h + kBlock.y - 1) / kBlock.y, (d.d + kBlock.z - 1) / kBlock.z); }

#define FX_VOXEL_PROLOGUE(dm)                               \
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x; \
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y; \
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z; \
  if (x >= (dm).w || y >= (dm).h || z >= (dm).d) return;    \
  const uint32_t i = flat(dm, x, y, z)

FX_DEV void voxel_pos(const Dims& dm, uint32_t x, uint32_t y, uint32_t z, float& px, float& py, float& pz) {
  px = ((float)x + 0.5f) / (float)dm.w;
  py = ((float)y + 0.5f) / (float)dm.h;
  pz = ((float)z + 0.5f) / (float)dm.d;
}

FX_DEV bool active_coord(const uint32_t* __restrict__ flags, uint3 bc, uint32_t x, uint32_t y, uint32_t z) {
  const uint32_t bx = min(x >> 3, bc.x - 1u), by = min(y >> 3, bc.y - 1u), bz = min(z >> 3, bc.z - 1u);
  return flags[bx + bc.x * (by + bc.y * bz)] != 0u;
}

FX_DEV bool interior_at(const Dims& dm, int x, int y, int z) {
  return x > 0 && y > 0 && z > 0 && x < (int)dm.w - 1 && y < (int)dm.h - 1 && z < (int)dm.d - 1;
}
// f at (x, y, z) when that voxel is interior, else 0.
FX_DEV float interior_val(const float* f, const Dims& dm, int x, int y, int z) {
  return interior_at(dm, x, y, z) ? f[flat(dm, (uint32_t)x, (uint32_t)y, (uint32_t)z)] : 0.0f;
}

// Derivative of clamp_pos(p, hi) with respect to p: 1 where the sample
// position passes through, 0 where it is clamped.
FX_DEV float pass_mask(float p, float hi) { return (p > 0.0f && p < hi) ? 1.0f : 0.0f; }

// lam[corner] += g * d(tri_interp)/d(corner value), for the eight corners.
FX_DEV void tri_scatter(float* lam, const Tri& c, float g) {
  if (g == 0.0f) return;
  const float ax = 1.0f - c.fx, ay = 1.0f - c.fy, az = 1.0f - c.fz;
  atomicAdd(lam + c.i000, g * (ax * ay * az));
  atomicAdd(lam + c.i100, g * (c.fx * ay * az));
  atomicAdd(lam + c.i010, g * (ax * c.fy * az));
  atomicAdd(lam + c.i110, g * (c.fx * c.fy * az));
  atomicAdd(lam + c.i001, g * (ax * ay * c.fz));
  atomicAdd(lam + c.i101, g * (c.fx * ay * c.fz));
  atomicAdd(lam + c.i011, g * (ax * c.fy * c.fz));
  atomicAdd(lam + c.i111, g * (c.fx * c.fy * c.fz));
}

// d(tri_interp(f, c))/d(fx, fy, fz).
FX_DEV void tri_dpos(const float* __restrict__ f, const Tri& c, float& gx, float& gy, float& gz) {
  const float f000 = f[c.i000], f100 = f[c.i100], f010 = f[c.i010], f110 = f[c.i110];
  const float f001 = f[c.i001], f101 = f[c.i101], f011 = f[c.i011], f111 = f[c.i111];
  const float ax = 1.0f - c.fx, ay = 1.0f - c.fy, az = 1.0f - c.fz;
  const float x00 = f000 * ax + f100 * c.fx, x10 = f010 * ax + f110 * c.fx;
  const float x01 = f001 * ax + f101 * c.fx, x11 = f011 * ax + f111 * c.fx;
  gz = (x01 * ay + x11 * c.fy) - (x00 * ay + x10 * c.fy);
  gy = az * (x10 - x00) + c.fz * (x11 - x01);
  gx = az * (ay * (f100 - f000) + c.fy * (f110 - f010)) + c.fz * (ay * (f101 - f001) + c.fy * (f111 - f011));
}

// A trilinear sample position with its clamp masks.
struct Sample {
  Tri t;
  float mx, my, mz;
  int bx, by, bz, ux, uy, uz;  // the lower and upper corner coordinates (tri_corners')
};
FX_DEV Sample sample_at(const Dims& dm, float px, float py, float pz) {
  Sample s;
  s.t = tri_corners(dm, px, py, pz);
  s.bx = (int)floorf(clamp_pos(px, (float)(dm.w - 1u)));
  s.by = (int)floorf(clamp_pos(py, (float)(dm.h - 1u)));
  s.bz = (int)floorf(clamp_pos(pz, (float)(dm.d - 1u)));
  s.ux = min(s.bx + 1, (int)dm.w - 1);
  s.uy = min(s.by + 1, (int)dm.h - 1);
  s.uz = min(s.bz + 1, (int)dm.d - 1);
  s.mx = pass_mask(px, (float)(dm.w - 1u));
  s.my = pass_mask(py, (float)(dm.h - 1u));
  s.mz = pass_mask(pz, (float)(dm.d - 1u));
  return s;
}
// g += w * d(tri_interp(f, s))/d(position).
FX_DEV void add_dpos(const float* __restrict__ f, const Sample& s, float w, float g[3]) {
  float gx, gy, gz;
  tri_dpos(f, s.t, gx, gy, gz);
  g[0] += w * gx * s.mx;
  g[1] += w * gy * s.my;
  g[2] += w * gz * s.mz;
}

// Brick-local accumulation of the advections' transposed trilinear scatters.
// A block owns one 8^3 brick (two voxels per thread) and keeps, per adjoint
// field, a shared-memory tile of the brick with a halo of kAccHalo voxels. A
// sample whose eight corners lie in the tile adds to it with shared-memory
// atomics; any other goes to global memory directly. At the end the block adds
// each touched tile cell to global memory once, instead of one global atomic
// per (sample, corner): a back-traced sample lies within a voxel or two of its
// voxel wherever the flow is slow, so neighbouring voxels hit the same cells.
constexpr int kAccHalo = 2;
constexpr int kAccEdge = 8 + 2 * kAccHalo;
constexpr int kAccCells = kAccEdge * kAccEdge * kAccEdge;
constexpr int kAccThreads = 256;
static_assert(7 * kAccCells * sizeof(float) <= 48 * 1024, "the scalar adjoint's tiles fit the default shared memory");

struct TileOrigin {
  int x, y, z;
};

FX_DEV TileOrigin brick_tile(uint3 bc, uint32_t b) {
  const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
  return {(int)(bx * 8u) - kAccHalo, (int)(by * 8u) - kAccHalo, (int)(bz * 8u) - kAccHalo};
}

FX_DEV void tile_clear(float* sh, int fields) {
  for (int j = threadIdx.x; j < fields * kAccCells; j += blockDim.x) sh[j] = 0.0f;
  __syncthreads();
}

// tri_scatter of g at sample s into the field's tile `sh` (or `lam` when a
// corner lies outside the tile).
FX_DEV void tile_scatter(const TileOrigin& o, float* sh, float* lam, const Sample& s, float g) {
  if (g == 0.0f) return;
  const int lx = s.bx - o.x, ly = s.by - o.y, lz = s.bz - o.z;
  const int hx = s.ux - o.x, hy = s.uy - o.y, hz = s.uz - o.z;
  if (lx < 0 || ly < 0 || lz < 0 || hx >= kAccEdge || hy >= kAccEdge || hz >= kAccEdge) {
    tri_scatter(lam, s.t, g);
    return;
  }
  const Tri& c = s.t;
  const float ax = 1.0f - c.fx, ay = 1.0f - c.fy, az = 1.0f - c.fz;
  const int r00 = kAccEdge * (ly + kAccEdge * lz), r10 = kAccEdge * (hy + kAccEdge * lz);
  const int r01 = kAccEdge * (ly + kAccEdge * hz), r11 = kAccEdge * (hy + kAccEdge * hz);
  atomicAdd(sh + lx + r00, g * (ax * ay * az));
  atomicAdd(sh + hx + r00, g * (c.fx * ay * az));
  atomicAdd(sh + lx + r10, g * (ax * c.fy * az));
  atomicAdd(sh + hx + r10, g * (c.fx * c.fy * az));
  atomicAdd(sh + lx + r01, g * (ax * ay * c.fz));
  atomicAdd(sh + hx + r01, g * (c.fx * ay * c.fz));
  atomicAdd(sh + lx + r11, g * (ax * c.fy * c.fz));
  atomicAdd(sh + hx + r11, g * (c.fx * c.fy * c.fz));
}

// v added at voxel (x, y, z) of the block's own brick.
FX_DEV void tile_point(const TileOrigin& o, float* sh, uint32_t x, uint32_t y, uint32_t z, float v) {
  if (v != 0.0f) atomicAdd(sh + ((int)x - o.x) + kAccEdge * (((int)y - o.y) + kAccEdge * ((int)z - o.z)), v);
}

// Adds the block's tiles to their global fields (after a barrier).
FX_DEV void tile_flush(const Dims& dm, const TileOrigin& o, const float* sh, float* const* lam, int fields) {
  __syncthreads();
  for (int j = threadIdx.x; j < kAccCells; j += blockDim.x) {
    const int x = o.x + j % kAccEdge, y = o.y + (j / kAccEdge) % kAccEdge, z = o.z + j / (kAccEdge * kAccEdge);
    if (x < 0 || y < 0 || z < 0 || x >= (int)dm.w || y >= (int)dm.h || z >= (int)dm.d) continue;
    const uint32_t gi = flat(dm, (uint32_t)x, (uint32_t)y, (uint32_t)z);
    for (int f = 0; f < fields; ++f) {
      const float v = sh[f * kAccCells + j];
      if (v != 0.0f) atomicAdd(lam[f] + gi, v);
    }
  }
}

// ------------------------------------------------------------------ kernels
__global__ void k_inflow(Dims dm, InflowPatch p, const float* __restrict__ values, VelField v) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.nx * p.nz) return;
  const uint32_t ix = t % p.nx, iz = t / p.nx;
  v.c[1][flat(dm, p.x0 + ix, p.y, p.z0 + iz)] = values[t];
}

__global__ void k_adj_loss(uint32_t n, const float* __restrict__ d, const float* __restrict__ target, float* __restrict__ lam_d,
                           double* __restrict__ loss) {
  double acc = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double diff = (double)d[i] - (double)target[i];
    if (lam_d) lam_d[i] = (float)(2.0 * diff);
    acc += diff * diff;
  }
  for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
  __shared__ double part[32];
  if ((threadIdx.x & 31) == 0) part[threadIdx.x >> 5] = acc;
  __syncthreads();
  if (threadIdx.x < 32) {
    acc = threadIdx.x < blockDim.x / 32 ? part[threadIdx.x] : 0.0;
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (threadIdx.x == 0) atomicAdd(loss, acc);
  }
}

// project-velocity.wgsl.ts:21-43: v = vs - 0.5 grad p at interior voxels, 0 on the boundary.
__global__ void k_adj_project(Dims dm, VelField lam_v, VelField lam_c, float* __restrict__ lam_p) {
  FX_VOXEL_PROLOGUE(dm);
  const bool in = !is_boundary(dm, x, y, z);
#pragma unroll
  for (int c = 0; c < 3; ++c) lam_c.c[c][i] = in ? lam_v.c[c][i] : 0.0f;
  const int X = (int)x, Y = (int)y, Z = (int)z;
  const float ax = interior_val(lam_v.c[0], dm, X + 1, Y, Z) - interior_val(lam_v.c[0], dm, X - 1, Y, Z);
  const float ay = interior_val(lam_v.c[1], dm, X, Y + 1, Z) - interior_val(lam_v.c[1], dm, X, Y - 1, Z);
  const float az = interior_val(lam_v.c[2], dm, X, Y, Z + 1) - interior_val(lam_v.c[2], dm, X, Y, Z - 1);
  lam_p[i] = 0.5f * (ax + ay + az);
}

// pressure-jacobi.wgsl.ts:15-36: dst = (sum of the 6 neighbours of src - div) / 6.
// ACCUMULATE false: lam_src holds no adjoint yet (it is treated as zero and
// written whole), which gives the accumulated bits: 0 + q is q, or +0 for a
// q that is -0.
template <bool ACCUMULATE>
__global__ void k_adj_jacobi(Dims dm, const float* __restrict__ lam_dst, float* __restrict__ lam_src, float* __restrict__ lam_div) {
  FX_VOXEL_PROLOGUE(dm);
  const int X = (int)x, Y = (int)y, Z = (int)z;
  const float acc = interior_val(lam_dst, dm, X + 1, Y, Z) + interior_val(lam_dst, dm, X - 1, Y, Z) + interior_val(lam_dst, dm, X, Y + 1, Z) +
                    interior_val(lam_dst, dm, X, Y - 1, Z) + interior_val(lam_dst, dm, X, Y, Z + 1) + interior_val(lam_dst, dm, X, Y, Z - 1);
  if (ACCUMULATE) {
    if (acc != 0.0f) lam_src[i] += acc / 6.0f;
  } else {
    lam_src[i] = acc != 0.0f ? 0.0f + acc / 6.0f : 0.0f;
  }
  if (!is_boundary(dm, x, y, z)) {
    const float l = lam_dst[i];
    if (l != 0.0f) lam_div[i] += -l / 6.0f;
  }
}

// pressure-restriction.wgsl.ts:27-50: coarse = 0.125 x the sum of 8 clamped children.
__global__ void k_adj_restrict(Dims fine, Dims dm, const float* __restrict__ lam_coarse, float* __restrict__ lam_fine) {
  FX_VOXEL_PROLOGUE(dm);
  if (x == 0u || y == 0u || z == 0u || x == dm.w - 1u || y == dm.h - 1u || z == dm.d - 1u) return;
  const float g = lam_coarse[i] * 0.125f;
  if (g == 0.0f) return;
  for (uint32_t dz = 0; dz < 2u; ++dz)
    for (uint32_t dy = 0; dy < 2u; ++dy)
      for (uint32_t dx = 0; dx < 2u; ++dx) {
        const uint32_t sx = min(2u * x + dx, fine.w - 1u), sy = min(2u * y + dy, fine.h - 1u), sz = min(2u * z + dz, fine.d - 1u);
        atomicAdd(lam_fine + flat(fine, sx, sy, sz), g);
      }
}

// pressure-prolongation.wgsl.ts:29-44: fine pA += trilinear(coarse p) inside, 0 on the boundary.
__global__ void k_adj_prolong(Dims coarse, Dims dm, float* __restrict__ lam_fpa, float* __restrict__ lam_cp) {
  FX_VOXEL_PROLOGUE(dm);
  if (x == 0u || y == 0u || z == 0u || x == dm.w - 1u || y == dm.h - 1u || z == dm.d - 1u) {
    lam_fpa[i] = 0.0f;
    return;
  }
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  tri_scatter(lam_cp, tri_corners(coarse, px, py, pz), lam_fpa[i]);
}

// compute-divergence.wgsl.ts:22-42: div = 0.5 (sum of central differences) inside.
__global__ void k_adj_divergence(Dims dm, const float* __restrict__ lam_div, VelField lam_c) {
  FX_VOXEL_PROLOGUE(dm);
  const int X = (int)x, Y = (int)y, Z = (int)z;
  lam_c.c[0][i] += 0.5f * (interior_val(lam_div, dm, X - 1, Y, Z) - interior_val(lam_div, dm, X + 1, Y, Z));
  lam_c.c[1][i] += 0.5f * (interior_val(lam_div, dm, X, Y - 1, Z) - interior_val(lam_div, dm, X, Y + 1, Z));
  lam_c.c[2][i] += 0.5f * (interior_val(lam_div, dm, X, Y, Z - 1) - interior_val(lam_div, dm, X, Y, Z + 1));
}

// apply-vorticity-confinement.wgsl.ts:30-66 at interior voxels.
__global__ void k_adj_confinement(Dims dm, const Params* __restrict__ Pp, VelField w, const float* __restrict__ wmag, ScalarSet set,
                                  VelField v, VelField lam_v, VelField lam_w, float* __restrict__ lam_wmag, VelField lam_g,
                                  ScalarSet lam_set) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) {
#pragma unroll
    for (int c = 0; c < 3; ++c) {
      lam_g.c[c][i] = 0.0f;
      lam_w.c[c][i] = 0.0f;
    }
    lam_wmag[i] = 0.0f;
    return;
  }
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  using D = Dn<13>;
  const float gx = (wmag[flat(dm, inc(x, W1), y, z)] - wmag[flat(dm, dec(x), y, z)]) * 0.5f;
  const float gy = (wmag[flat(dm, x, inc(y, H1), z)] - wmag[flat(dm, x, dec(y), z)]) * 0.5f;
  const float gz = (wmag[flat(dm, x, y, inc(z, D1))] - wmag[flat(dm, x, y, dec(z))]) * 0.5f;
  D vx = D::var(v.c[0][i], 0), vy = D::var(v.c[1][i], 1), vz = D::var(v.c[2][i], 2);
  confinement_voxel<D>(P, D::var(gx, 3), D::var(gy, 4), D::var(gz, 5), D::var(w.c[0][i], 6), D::var(w.c[1][i], 7), D::var(w.c[2][i], 8),
                       D::var(wmag[i], 9), D::var(set.f[0][i], 10), D::var(set.f[1][i], 11), D::var(set.f[3][i], 12), vx, vy, vz);
  const float l0 = lam_v.c[0][i], l1 = lam_v.c[1][i], l2 = lam_v.c[2][i];
  float lin[13];
#pragma unroll
  for (int k = 0; k < 13; ++k) lin[k] = l0 * vx.g[k] + l1 * vy.g[k] + l2 * vz.g[k];
#pragma unroll
  for (int c = 0; c < 3; ++c) {
    lam_v.c[c][i] = lin[c];
    lam_g.c[c][i] = lin[3 + c];
    lam_w.c[c][i] = lin[6 + c];
  }
  lam_wmag[i] = lin[9];
  lam_set.f[0][i] += lin[10];
  lam_set.f[1][i] += lin[11];
  lam_set.f[3][i] += lin[12];
}

// |w| = length(w) and the confinement's |w| gradient, folded into lam_w.
__global__ void k_adj_wmag(Dims dm, VelField w, const float* __restrict__ wmag, VelField lam_w, const float* __restrict__ lam_wmag,
                           VelField lam_g) {
  FX_VOXEL_PROLOGUE(dm);
  if (is_boundary(dm, x, y, z)) return;  // lam_w is 0 there
  const int X = (int)x, Y = (int)y, Z = (int)z;
  // g_x(m) = 0.5 (|w|(m + x) - |w|(m - x)) at interior m
  const float lm = lam_wmag[i] + 0.5f * (interior_val(lam_g.c[0], dm, X - 1, Y, Z) - interior_val(lam_g.c[0], dm, X + 1, Y, Z)) +
                   0.5f * (interior_val(lam_g.c[1], dm, X, Y - 1, Z) - interior_val(lam_g.c[1], dm, X, Y + 1, Z)) +
                   0.5f * (interior_val(lam_g.c[2], dm, X, Y, Z - 1) - interior_val(lam_g.c[2], dm, X, Y, Z + 1));
  const float m = wmag[i];
  if (lm == 0.0f || !(m > 0.0f)) return;
  const float h = lm / m;
#pragma unroll
  for (int c = 0; c < 3; ++c) lam_w.c[c][i] += h * w.c[c][i];
}

// compute-vorticity.wgsl.ts:23-50: w = 0.5 curl(v) at interior voxels.
__global__ void k_adj_curl(Dims dm, VelField lam_w, VelField lam_v) {
  FX_VOXEL_PROLOGUE(dm);
  const int X = (int)x, Y = (int)y, Z = (int)z;
  auto W = [&](int c, int xx, int yy, int zz) { return interior_val(lam_w.c[c], dm, xx, yy, zz); };
  lam_v.c[0][i] += 0.5f * (W(1, X, Y, Z - 1) - W(1, X, Y, Z + 1) - W(2, X, Y - 1, Z) + W(2, X, Y + 1, Z));
  lam_v.c[1][i] += 0.5f * (-W(0, X, Y, Z - 1) + W(0, X, Y, Z + 1) + W(2, X - 1, Y, Z) - W(2, X + 1, Y, Z));
  lam_v.c[2][i] += 0.5f * (W(0, X, Y - 1, Z) - W(0, X, Y + 1, Z) - W(1, X - 1, Y, Z) + W(1, X + 1, Y, Z));
}

// apply-buoyancy.wgsl.ts:37-110 at active voxels: local parts, and the neighbour
// parts of the hot-gas and density differences into the scratch fields.
__global__ void k_adj_buoyancy(Dims dm, uint3 bc, const Params* __restrict__ Pp, ScalarSet set, const uint32_t* __restrict__ flags,
                               VelField v, VelField lam_v, ScalarSet lam_set, float* __restrict__ hot, float* __restrict__ dens) {
  FX_VOXEL_PROLOGUE(dm);
  if (!active_coord(flags, bc, x, y, z)) return;
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  const float* Dv = set.f[0];
  auto hotf = [&](uint32_t xx, uint32_t yy, uint32_t zz) {
    const uint32_t j = flat(dm, xx, yy, zz);
    return buoy_hot(set.f[1][j], set.f[3][j]);
  };
  const uint32_t xp = flat(dm, inc(x, W1), y, z), xm = flat(dm, dec(x), y, z);
  const uint32_t yp = flat(dm, x, inc(y, H1), z), ym = flat(dm, x, dec(y), z);
  const uint32_t zp = flat(dm, x, y, inc(z, D1)), zm = flat(dm, x, y, dec(z));
  const float hot_gas = hotf(x, y, z);
  const float tgx = (hotf(inc(x, W1), y, z) - hotf(dec(x), y, z)) * 0.5f;
  const float tgy = (hotf(x, inc(y, H1), z) - hotf(x, dec(y), z)) * 0.5f;
  const float tgz = (hotf(x, y, inc(z, D1)) - hotf(x, y, dec(z))) * 0.5f;
  const float dgx = (Dv[xp] - Dv[xm]) * 0.5f;
  const float dgy = (Dv[yp] - Dv[ym]) * 0.5f;
  const float dgz = (Dv[zp] - Dv[zm]) * 0.5f;
  using D = Dn<11>;
  D vx = D::var(v.c[0][i], 0), vy = D::var(v.c[1][i], 1), vz = D::var(v.c[2][i], 2);
  buoyancy_voxel<D>(P, dm, x, y, z, D::var(Dv[i], 3), D::var(hot_gas, 4), D::var(tgx, 5), D::var(tgy, 6), D::var(tgz, 7), D::var(dgx, 8),
                    D::var(dgy, 9), D::var(dgz, 10), vx, vy, vz);
  const float l0 = lam_v.c[0][i], l1 = lam_v.c[1][i], l2 = lam_v.c[2][i];
  float lin[11];
#pragma unroll
  for (int k = 0; k < 11; ++k) lin[k] = l0 * vx.g[k] + l1 * vy.g[k] + l2 * vz.g[k];
#pragma unroll
  for (int c = 0; c < 3; ++c) lam_v.c[c][i] = lin[c];
  lam_set.f[0][i] += lin[3];
  const Dn<2> h = buoy_hot(Dn<2>::var(set.f[1][i], 0), Dn<2>::var(set.f[3][i], 1));
  lam_set.f[1][i] += lin[4] * h.g[0];
  lam_set.f[3][i] += lin[4] * h.g[1];
  if (lin[5] != 0.0f) {
    atomicAdd(hot + xp, 0.5f * lin[5]);
    atomicAdd(hot + xm, -0.5f * lin[5]);
  }
  if (lin[6] != 0.0f) {
    atomicAdd(hot + yp, 0.5f * lin[6]);
    atomicAdd(hot + ym, -0.5f * lin[6]);
  }
  if (lin[7] != 0.0f) {
    atomicAdd(hot + zp, 0.5f * lin[7]);
    atomicAdd(hot + zm, -0.5f * lin[7]);
  }
  if (lin[8] != 0.0f) {
    atomicAdd(dens + xp, 0.5f * lin[8]);
    atomicAdd(dens + xm, -0.5f * lin[8]);
  }
  if (lin[9] != 0.0f) {
    atomicAdd(dens + yp, 0.5f * lin[9]);
    atomicAdd(dens + ym, -0.5f * lin[9]);
  }
  if (lin[10] != 0.0f) {
    atomicAdd(dens + zp, 0.5f * lin[10]);
    atomicAdd(dens + zm, -0.5f * lin[10]);
  }
}

// The scratch fields of k_adj_buoyancy into lam_set; clears them.
__global__ void k_adj_buoyancy_fold(Dims dm, ScalarSet set, ScalarSet lam_set, float* __restrict__ hot, float* __restrict__ dens) {
  FX_VOXEL_PROLOGUE(dm);
  const float hd = dens[i], hh = hot[i];
  if (hd != 0.0f) {
    lam_set.f[0][i] += hd;
    dens[i] = 0.0f;
  }
  if (hh != 0.0f) {
    const Dn<2> h = buoy_hot(Dn<2>::var(set.f[1][i], 0), Dn<2>::var(set.f[3][i], 1));
    lam_set.f[1][i] += hh * h.g[0];
    lam_set.f[3][i] += hh * h.g[1];
    hot[i] = 0.0f;
  }
}

// combustion-update.wgsl.ts:42-93 at active voxels, reading the snapshot.
__global__ void k_adj_combustion(Dims dm, uint3 bc, const Params* __restrict__ Pp, ScalarSet snap, const uint32_t* __restrict__ flags,
                                 ScalarSet lam_set, float* __restrict__ hot) {
  FX_VOXEL_PROLOGUE(dm);
  if (!active_coord(flags, bc, x, y, z)) return;
  const Params P = *Pp;
  const uint32_t W1 = dm.w - 1u, H1 = dm.h - 1u, D1 = dm.d - 1u;
  auto hotf = [&](uint32_t j) { return comb_hot(snap.f[1][j], snap.f[2][j], snap.f[3][j]); };
  const uint32_t nb[6] = {flat(dm, inc(x, W1), y, z), flat(dm, dec(x), y, z), flat(dm, x, inc(y, H1), z),
                          flat(dm, x, dec(y), z),     flat(dm, x, y, inc(z, D1)), flat(dm, x, y, dec(z))};
  const float nsum = hotf(nb[0]) + hotf(nb[1]) + hotf(nb[2]) + hotf(nb[3]) + hotf(nb[4]) + hotf(nb[5]);
  using D = Dn<5>;
  D d = D::var(snap.f[0][i], 0), t = D::var(snap.f[1][i], 1), f = D::var(snap.f[2][i], 2), r = D::var(snap.f[3][i], 3);
  const float ny = ((float)y + 0.5f) / (float)dm.h;
  combustion_voxel<D>(P, x, y, z, ny, D::var(nsum, 4), d, t, f, r);
  const float ld = lam_set.f[0][i], lt = lam_set.f[1][i], lf = lam_set.f[2][i], lr = lam_set.f[3][i];
  float lin[5];
#pragma unroll
  for (int k = 0; k < 5; ++k) lin[k] = ld * d.g[k] + lt * t.g[k] + lf * f.g[k] + lr * r.g[k];
#pragma unroll
  for (int k = 0; k < 4; ++k) lam_set.f[k][i] = lin[k];
  if (lin[4] != 0.0f)
#pragma unroll
    for (int k = 0; k < 6; ++k) atomicAdd(hot + nb[k], lin[4]);
}

__global__ void k_adj_combustion_fold(Dims dm, ScalarSet snap, ScalarSet lam_set, float* __restrict__ hot) {
  FX_VOXEL_PROLOGUE(dm);
  const float hh = hot[i];
  if (hh == 0.0f) return;
  const Dn<3> h = comb_hot(Dn<3>::var(snap.f[1][i], 0), Dn<3>::var(snap.f[2][i], 1), Dn<3>::var(snap.f[3][i], 2));
  lam_set.f[1][i] += hh * h.g[0];
  lam_set.f[2][i] += hh * h.g[1];
  lam_set.f[3][i] += hh * h.g[2];
  hot[i] = 0.0f;
}

// advect-scalar-maccormack.wgsl.ts:33-101 at one voxel of an active brick
// (velocity = vel). Tiles 0-3: lam_src's fields; 4-6: lam_vel's components.
FX_DEV void adj_advect_scalars_voxel(const Dims& dm, const Params& P, const ScalarSet& src, const VelField& vel, const ScalarSet& lam_out,
                                     const ScalarSet& lam_src, const VelField& lam_vel, uint32_t x, uint32_t y, uint32_t z,
                                     const TileOrigin& o, float* sh) {
  const uint32_t i = flat(dm, x, y, z);
  const float dt = P.dt;
  const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
  const Tri c0 = tri_corners(dm, cx - 0.5f, cy - 0.5f, cz - 0.5f);
  const float vx = tri_interp(vel.c[0], c0), vy = tri_interp(vel.c[1], c0), vz = tri_interp(vel.c[2], c0);
  const float bx = cx - vx * dt, by = cy - vy * dt, bz = cz - vz * dt;
  const float spx = bx - 0.5f, spy = by - 0.5f, spz = bz - 0.5f;
  const Sample cs = sample_at(dm, spx, spy, spz);
  const float fvx = tri_interp(vel.c[0], cs.t), fvy = tri_interp(vel.c[1], cs.t), fvz = tri_interp(vel.c[2], cs.t);
  const float rx = bx + fvx * dt, ry = by + fvy * dt, rz = bz + fvz * dt;
  const Sample cr = sample_at(dm, rx - 0.5f, ry - 0.5f, rz - 0.5f);
  // The limiter's selection: 0 corrected, 1 predicted, 2 original.
  int sel[4];
  Dn<4> out[4];
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float predicted = tri_interp(src.f[f], cs.t);
    const float recovered = tri_interp(src.f[f], cr.t);
    const float original = tri_interp(src.f[f], c0);
    const float corrected = predicted + 0.5f * (original - recovered);
    const float lo = mn(original, predicted), hi = mx(original, predicted);
    const float a = mx(corrected, lo);
    if (hi < a) sel[f] = original < predicted ? 1 : 2;
    else if (!(corrected < lo)) sel[f] = 0;
    else sel[f] = predicted < original ? 1 : 2;
    out[f] = Dn<4>::var(mn(a, hi), f);
  }
  const float noise = thermal_noise(P, cx, cy, cz);
  const float ny = ((float)y + 0.5f) / (float)dm.h;
  decay_scalars<Dn<4>>(P, ny, noise, out[0], out[1], out[2], out[3]);
  float lo4[4];
#pragma unroll
  for (int k = 0; k < 4; ++k)
    lo4[k] = lam_out.f[0][i] * out[0].g[k] + lam_out.f[1][i] * out[1].g[k] + lam_out.f[2][i] * out[2].g[k] + lam_out.f[3][i] * out[3].g[k];
  float gsp[3] = {0.0f, 0.0f, 0.0f}, gb[3] = {0.0f, 0.0f, 0.0f}, gfv[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float l = lo4[f];
    if (l == 0.0f) continue;
    float lpred = 0.0f, lorig = 0.0f, lrec = 0.0f;
    if (sel[f] == 0) {
      lpred = l;
      lorig = 0.5f * l;
      lrec = -0.5f * l;
    } else if (sel[f] == 1) {
      lpred = l;
    } else {
      lorig = l;
    }
    if (lpred != 0.0f) {
      tile_scatter(o, sh + f * kAccCells, lam_src.f[f], cs, lpred);
      add_dpos(src.f[f], cs, lpred, gsp);
    }
    if (lrec != 0.0f) {
      tile_scatter(o, sh + f * kAccCells, lam_src.f[f], cr, lrec);
      float gr[3] = {0.0f, 0.0f, 0.0f};
      add_dpos(src.f[f], cr, lrec, gr);
#pragma unroll
      for (int k = 0; k < 3; ++k) {
        gb[k] += gr[k];
        gfv[k] += gr[k] * dt;
      }
    }
    tile_point(o, sh + f * kAccCells, x, y, z, lorig);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (gfv[k] == 0.0f) continue;
    tile_scatter(o, sh + (4 + k) * kAccCells, lam_vel.c[k], cs, gfv[k]);
    add_dpos(vel.c[k], cs, gfv[k], gsp);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    const float g = -dt * (gb[k] + gsp[k]);
    tile_point(o, sh + (4 + k) * kAccCells, x, y, z, g);
  }
}

__global__ void __launch_bounds__(kAccThreads) k_adj_advect_scalars(Dims dm, uint3 bc, const Params* __restrict__ Pp, ScalarSet src,
                                                                    VelField vel, const uint32_t* __restrict__ flags, ScalarSet lam_out,
                                                                    ScalarSet lam_src, VelField lam_vel) {
  extern __shared__ float sh[];
  const uint32_t b = blockIdx.x;
  if (flags[b] == 0u) return;
  const TileOrigin o = brick_tile(bc, b);
  tile_clear(sh, 7);
  const Params P = *Pp;
  for (uint32_t v = threadIdx.x; v < 512u; v += kAccThreads) {
    const uint32_t x = (uint32_t)(o.x + kAccHalo) + (v & 7u), y = (uint32_t)(o.y + kAccHalo) + ((v >> 3) & 7u),
                   z = (uint32_t)(o.z + kAccHalo) + (v >> 6);
    if (x < dm.w && y < dm.h && z < dm.d) adj_advect_scalars_voxel(dm, P, src, vel, lam_out, lam_src, lam_vel, x, y, z, o, sh);
  }
  float* const lam[7] = {lam_src.f[0], lam_src.f[1], lam_src.f[2], lam_src.f[3], lam_vel.c[0], lam_vel.c[1], lam_vel.c[2]};
  tile_flush(dm, o, sh, lam, 7);
}

// advect-velocity-semilagrangian.wgsl.ts:23-41 at one interior voxel; tiles
// 0-2: lam_src's components.
FX_DEV void adj_advect_velocity_voxel(const Dims& dm, float dt, const VelField& src, const VelField& lam_dst, const VelField& lam_src,
                                      uint32_t x, uint32_t y, uint32_t z, const TileOrigin& o, float* sh) {
  if (is_boundary(dm, x, y, z)) return;
  const uint32_t i = flat(dm, x, y, z);
  const float damp = 1.0f - dt * 0.025f;
  float la[3];
  bool any = false;
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    la[k] = lam_dst.c[k][i] * damp;
    any |= la[k] != 0.0f;
  }
  if (!any) return;
  const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
  const Tri c0 = tri_corners(dm, cx - 0.5f, cy - 0.5f, cz - 0.5f);
  const float v0x = tri_interp(src.c[0], c0), v0y = tri_interp(src.c[1], c0), v0z = tri_interp(src.c[2], c0);
  const float bx = cx - v0x * dt, by = cy - v0y * dt, bz = cz - v0z * dt;
  const Sample c1 = sample_at(dm, bx - 0.5f, by - 0.5f, bz - 0.5f);
  float gp[3] = {0.0f, 0.0f, 0.0f};
#pragma unroll
  for (int k = 0; k < 3; ++k) {
    if (la[k] == 0.0f) continue;
    tile_scatter(o, sh + k * kAccCells, lam_src.c[k], c1, la[k]);
    add_dpos(src.c[k], c1, la[k], gp);
  }
#pragma unroll
  for (int k = 0; k < 3; ++k) tile_point(o, sh + k * kAccCells, x, y, z, -dt * gp[k]);
}

__global__ void __launch_bounds__(kAccThreads) k_adj_advect_velocity(Dims dm, uint3 bc, const Params* __restrict__ Pp, VelField src,
                                                                     VelField lam_dst, VelField lam_src) {
  extern __shared__ float sh[];
  const TileOrigin o = brick_tile(bc, blockIdx.x);
  tile_clear(sh, 3);
  const float dt = Pp->dt;
  for (uint32_t v = threadIdx.x; v < 512u; v += kAccThreads) {
    const uint32_t x = (uint32_t)(o.x + kAccHalo) + (v & 7u), y = (uint32_t)(o.y + kAccHalo) + ((v >> 3) & 7u),
                   z = (uint32_t)(o.z + kAccHalo) + (v >> 6);
    if (x < dm.w && y < dm.h && z < dm.d) adj_advect_velocity_voxel(dm, dt, src, lam_dst, lam_src, x, y, z, o, sh);
  }
  float* const lam[3] = {lam_src.c[0], lam_src.c[1], lam_src.c[2]};
  tile_flush(dm, o, sh, lam, 3);
}

// inject-igniter.wgsl.ts:32-66.
__global__ void k_adj_inject_igniter(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc,
                                     const float* __restrict__ t_before, const float* __restrict__ fuel, const float* __restrict__ r_before,
                                     ScalarSet lam_set) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  using D = Dn<3>;
  D t = D::var(t_before[i], 0), f = D::var(fuel[i], 1), r = D::var(r_before[i], 2);
  inject_igniter_voxel<D>(P, src, nsrc, px, py, pz, f, r, t);
  const float lt = lam_set.f[1][i], lf = lam_set.f[2][i], lr = lam_set.f[3][i];
  lam_set.f[1][i] = lt * t.g[0] + lr * r.g[0];
  lam_set.f[2][i] = lf + lt * t.g[1] + lr * r.g[1];
  lam_set.f[3][i] = lt * t.g[2] + lr * r.g[2];
}

__global__ void k_adj_inflow(Dims dm, InflowPatch p, VelField lam_v, float* __restrict__ grad) {
  const uint32_t t = blockIdx.x * blockDim.x + threadIdx.x;
  if (t >= p.nx * p.nz) return;
  const uint32_t ix = t % p.nx, iz = t / p.nx;
  const uint32_t j = flat(dm, p.x0 + ix, p.y, p.z0 + iz);
  grad[t] += lam_v.c[1][j];
  lam_v.c[1][j] = 0.0f;
}

// inject-velocity.wgsl.ts:46-96 with the speed clamp.
__global__ void k_adj_inject_velocity(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc, VelField vb,
                                      VelField lam_v) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  using D = Dn<3>;
  D vx = D::var(vb.c[0][i], 0), vy = D::var(vb.c[1][i], 1), vz = D::var(vb.c[2][i], 2);
  inject_velocity_voxel<D>(P, src, nsrc, px, py, pz, vx, vy, vz);
  const float lim = speed_limit(P);
  vx = clampv(vx, -lim, lim);
  vy = clampv(vy, -lim, lim);
  vz = clampv(vz, -lim, lim);
  const float l0 = lam_v.c[0][i], l1 = lam_v.c[1][i], l2 = lam_v.c[2][i];
#pragma unroll
  for (int k = 0; k < 3; ++k) lam_v.c[k][i] = l0 * vx.g[k] + l1 * vy.g[k] + l2 * vz.g[k];
}

// inject-scalar.wgsl.ts:32-70.
__global__ void k_adj_inject_scalar(Dims dm, const Params* __restrict__ Pp, const float* __restrict__ src, uint32_t nsrc, ScalarSet before,
                                    ScalarSet lam_set) {
  FX_VOXEL_PROLOGUE(dm);
  const Params P = *Pp;
  float px, py, pz;
  voxel_pos(dm, x, y, z, px, py, pz);
  using D = Dn<3>;
  D d = D::var(before.f[0][i], 0), t = D::var(before.f[1][i], 1), f = D::var(before.f[2][i], 2);
  inject_scalar_voxel<D>(P, src, nsrc, px, py, pz, d, t, f);
  const float ld = lam_set.f[0][i], lt = lam_set.f[1][i], lf = lam_set.f[2][i];
#pragma unroll
  for (int k = 0; k < 3; ++k) lam_set.f[k][i] = ld * d.g[k] + lt * t.g[k] + lf * f.g[k];
}

}  // namespace

void plain_inflow(cudaStream_t s, Dims dm, InflowPatch p, const float* values, VelField v) {
  const uint32_t n = p.nx * p.nz;
  if (n) k_inflow<<<(n + 127) / 128, 128, 0, s>>>(dm, p, values, v);
}
void adj_loss(cudaStream_t s, uint32_t n, const float* d, const float* target, float* lam_d, double* loss) {
  k_adj_loss<<<592, 256, 0, s>>>(n, d, target, lam_d, loss);
}
void adj_project(cudaStream_t s, Dims dm, VelField lam_v, VelField lam_c, float* lam_p) {
  k_adj_project<<<grid_for(dm), kBlock, 0, s>>>(dm, lam_v, lam_c, lam_p);
}
void adj_jacobi(cudaStream_t s, Dims dm, const float* lam_dst, float* lam_src, float* lam_div, bool accumulate) {
  if (accumulate)
    k_adj_jacobi<true><<<grid_for(dm), kBlock, 0, s>>>(dm, lam_dst, lam_src, lam_div);
  else
    k_adj_jacobi<false><<<grid_for(dm), kBlock, 0, s>>>(dm, lam_dst, lam_src, lam_div);
}
void adj_restrict(cudaStream_t s, Dims fine, Dims coarse, const float* lam_coarse, float* lam_fine) {
  k_adj_restrict<<<grid_for(coarse), kBlock, 0, s>>>(fine, coarse, lam_coarse, lam_fine);
}
void adj_prolong(cudaStream_t s, Dims coarse, Dims fine, float* lam_fpa, float* lam_cp) {
  k_adj_prolong<<<grid_for(fine), kBlock, 0, s>>>(coarse, fine, lam_fpa, lam_cp);
}
void adj_divergence(cudaStream_t s, Dims dm, const float* lam_div, VelField lam_c) {
  k_adj_divergence<<<grid_for(dm), kBlock, 0, s>>>(dm, lam_div, lam_c);
}
void adj_confinement(cudaStream_t s, Dims dm, const Params* P, VelField w, const float* wmag, ScalarSet set, VelField v, VelField lam_v,
                     VelField lam_w, float* lam_wmag, VelField lam_g, ScalarSet lam_set) {
  k_adj_confinement<<<grid_for(dm), kBlock, 0, s>>>(dm, P, w, wmag, set, v, lam_v, lam_w, lam_wmag, lam_g, lam_set);
}
void adj_vorticity(cudaStream_t s, Dims dm, VelField w, const float* wmag, VelField lam_w, const float* lam_wmag, VelField lam_g,
                   VelField lam_v) {
  k_adj_wmag<<<grid_for(dm), kBlock, 0, s>>>(dm, w, wmag, lam_w, lam_wmag, lam_g);
  k_adj_curl<<<grid_for(dm), kBlock, 0, s>>>(dm, lam_w, lam_v);
}
void adj_buoyancy(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet set, const uint32_t* flags, VelField v, VelField lam_v,
                  ScalarSet lam_set, float* hot, float* dens) {
  k_adj_buoyancy<<<grid_for(dm), kBlock, 0, s>>>(dm, bricks, P, set, flags, v, lam_v, lam_set, hot, dens);
  k_adj_buoyancy_fold<<<grid_for(dm), kBlock, 0, s>>>(dm, set, lam_set, hot, dens);
}
void adj_combustion(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet snap, const uint32_t* flags, ScalarSet lam_set,
                    float* hot) {
  k_adj_combustion<<<grid_for(dm), kBlock, 0, s>>>(dm, bricks, P, snap, flags, lam_set, hot);
  k_adj_combustion_fold<<<grid_for(dm), kBlock, 0, s>>>(dm, snap, lam_set, hot);
}
void adj_advect_scalars(cudaStream_t s, Dims dm, uint3 bricks, const Params* P, ScalarSet src, VelField vel, const uint32_t* flags,
                        ScalarSet lam_out, ScalarSet lam_src, VelField lam_vel) {
  const size_t smem = 7 * kAccCells * sizeof(float);  // 48,384 B: within the default 48 KiB
  k_adj_advect_scalars<<<bricks.x * bricks.y * bricks.z, kAccThreads, smem, s>>>(dm, bricks, P, src, vel, flags, lam_out, lam_src, lam_vel);
}
void adj_advect_velocity(cudaStream_t s, Dims dm, const Params* P, VelField src, VelField lam_dst, VelField lam_src) {
  const uint3 bc = make_uint3((dm.w + 7) / 8, (dm.h + 7) / 8, (dm.d + 7) / 8);
  const size_t smem = 3 * kAccCells * sizeof(float);
  k_adj_advect_velocity<<<bc.x * bc.y * bc.z, kAccThreads, smem, s>>>(dm, bc, P, src, lam_dst, lam_src);
}
void adj_inject_igniter(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, const float* t_before, const float* fuel,
                        const float* r_before, ScalarSet lam_set) {
  k_adj_inject_igniter<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, t_before, fuel, r_before, lam_set);
}
void adj_inflow(cudaStream_t s, Dims dm, InflowPatch p, VelField lam_v, float* grad) {
  const uint32_t n = p.nx * p.nz;
  if (n) k_adj_inflow<<<(n + 127) / 128, 128, 0, s>>>(dm, p, lam_v, grad);
}
void adj_inject_velocity(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, VelField v_before, VelField lam_v) {
  k_adj_inject_velocity<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, v_before, lam_v);
}
void adj_inject_scalar(cudaStream_t s, Dims dm, const Params* P, const float* src, uint32_t nsrc, ScalarSet before, ScalarSet lam_set) {
  k_adj_inject_scalar<<<grid_for(dm), kBlock, 0, s>>>(dm, P, src, nsrc, before, lam_set);
}

}  // namespace fx
