// Weighted-Jacobi V-cycle pressure solver with FP64 norms (see fx_vcycle.h).
//
// Per level k the cycle runs `pre` weighted sweeps, restricts 4 x the mean of
// the 8 fine residuals under each coarse voxel (the mean and the clamped
// children of pressure-restriction.wgsl.ts:27-50; the 4 rescales the unscaled
// 7-point operator to the doubled spacing), solves the coarse correction from
// zero, adds its trilinear prolongation (the sample position of
// pressure-prolongation.wgsl.ts:29-44) and runs `post` sweeps. The coarsest
// level runs `coarse` sweeps. Values are f32 and computed in the same order as
// the oracle, so the iterates agree bit for bit; the norms are FP64 sums whose
// order differs between the two, which matters only for a residual within
// rounding of the tolerance.
//
// The loop runs as a WHILE conditional node of the step's CUDA graph: the
// finalize kernel sets the condition from the FP64 residual, and it is 0 once
// max_cycles cycles have run, so the loop always ends.
//
// On levels whose width is a multiple of 4 the sweeps, the residual restriction
// and the prolongation run as marching kernels (four x per thread, a run of z
// planes per thread, the next plane's loads in flight), with the same
// operations in the same order as the one-voxel kernels, so the iterates are the
// same bits. The FP64 norms are reduced deterministically: every block writes one
// partial sum and the finalize kernel adds the partials in a fixed order, so the
// cycle count and the statistics repeat from run to run.
#include <algorithm>
#include <cmath>

#include "fx_pressure.h"
#include "fx_vcycle.h"

namespace fx {
namespace {

constexpr int kVZ = 4;

// dst = src + w ((sum of the 6 neighbours - rhs) / 6 - src) at interior voxels
// (dst = the Jacobi value when w is 1), 0 on the boundary. Warp layout of the
// fine sweep kernel: 32 consecutive x per warp, x neighbours by shuffles, z
// neighbours from a register column; the sum keeps the order +x, -x, +y, -y, +z, -z.
__global__ void __launch_bounds__(256) k_wjacobi(Dims dm, const float* __restrict__ rhs, const float* __restrict__ src, float* __restrict__ dst,
                                                 float w, int one) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x = blockIdx.x * 32 + lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * kVZ;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x < dm.w;
  const uint32_t base = (xin ? x : dm.w - 1) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const bool xint = x > 0 && x < dm.w - 1;
  const int nz = min(kVZ, (int)dm.d - (int)z0);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst[base + sz * (z0 + k)] = 0.0f;
    return;
  }
  float c[kVZ + 2], yp[kVZ], ym[kVZ], dv[kVZ], xe[kVZ];
  const bool left_end = lane == 0 && x > 0, right_end = (lane == 31 || x == dm.w - 1) && x + 1 < dm.w;
#pragma unroll
  for (int k = 0; k < kVZ + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (z >= 0 && z < (int)dm.d) ? __ldg(src + base + sz * (uint32_t)z) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < kVZ; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(rhs + i);
    yp[k] = __ldg(src + i + sy);
    ym[k] = __ldg(src + i - sy);
    xe[k] = 0.0f;
    if (left_end) xe[k] = __ldg(src + i - 1);
    if (right_end) xe[k] = __ldg(src + i + 1);
  }
#pragma unroll
  for (int k = 0; k < kVZ; ++k) {
    const float cm = c[k + 1];
    float xr = __shfl_down_sync(0xffffffffu, cm, 1);
    float xl = __shfl_up_sync(0xffffffffu, cm, 1);
    if (right_end) xr = xe[k];
    if (left_end) xl = xe[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float v = 0.0f;
    if (xint && z > 0 && z < dm.d - 1) {
      const float s = xr + xl + yp[k] + ym[k] + c[k + 2] + c[k];
      const float j = div6(s - dv[k]);
      v = one ? j : cm + w * (j - cm);
    }
    dst[base + sz * z] = v;
  }
}

FX_DEV float resid_at(const Dims& f, const float* __restrict__ rhs, const float* __restrict__ e, uint32_t x, uint32_t y, uint32_t z) {
  if (is_boundary(f, x, y, z)) return 0.0f;
  const uint32_t W1 = f.w - 1u, H1 = f.h - 1u, D1 = f.d - 1u;
  const uint32_t i = flat(f, x, y, z);
  const float s = __ldg(e + flat(f, inc(x, W1), y, z)) + __ldg(e + flat(f, dec(x), y, z)) + __ldg(e + flat(f, x, inc(y, H1), z)) +
                  __ldg(e + flat(f, x, dec(y), z)) + __ldg(e + flat(f, x, y, inc(z, D1))) + __ldg(e + flat(f, x, y, dec(z)));
  const float lap = s - __ldg(e + i) * 6.0f;
  return __ldg(rhs + i) - lap;
}

__global__ void __launch_bounds__(256) k_resid_restrict(Dims f, const float* __restrict__ rhs_f, const float* __restrict__ e_f, Dims c,
                                                        float* __restrict__ rhs_c) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
                 z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= c.w || y >= c.h || z >= c.d) return;
  const uint32_t i = flat(c, x, y, z);
  if (x == 0u || y == 0u || z == 0u || x == c.w - 1u || y == c.h - 1u || z == c.d - 1u) {
    rhs_c[i] = 0.0f;
    return;
  }
  float sum = 0.0f;
#pragma unroll
  for (uint32_t dz = 0; dz < 2; ++dz)
#pragma unroll
    for (uint32_t dy = 0; dy < 2; ++dy)
#pragma unroll
      for (uint32_t dx = 0; dx < 2; ++dx)
        sum += resid_at(f, rhs_f, e_f, min(2u * x + dx, f.w - 1u), min(2u * y + dy, f.h - 1u), min(2u * z + dz, f.d - 1u));
  rhs_c[i] = (sum * 0.125f) * 4.0f;
}

// dst = src + trilinear(ec) at interior fine voxels, dst = src on the boundary
// (src and dst may be the same buffer).
__global__ void __launch_bounds__(256) k_prolong_add(Dims c, const float* __restrict__ ec, Dims f, const float* src, float* dst) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y * blockDim.y + threadIdx.y,
                 z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= f.w || y >= f.h || z >= f.d) return;
  const uint32_t i = flat(f, x, y, z);
  const float v = src[i];
  if (x == 0u || y == 0u || z == 0u || x == f.w - 1u || y == f.h - 1u || z == f.d - 1u) {
    dst[i] = v;
    return;
  }
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  dst[i] = v + tri_interp(ec, tri_corners(c, px, py, pz));
}

// Block sum of one double per thread (fixed tree order) written to part[block].
FX_DEV void block_sum_to(double v, double* part) {
  __shared__ double wsum[32];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  const int nthreads = blockDim.x * blockDim.y;
  const int t = threadIdx.x + blockDim.x * threadIdx.y;
  const int warp = t >> 5, lane = t & 31;
  if (lane == 0) wsum[warp] = v;
  __syncthreads();
  if (warp == 0) {
    const int nw = nthreads >> 5;
    v = lane < nw ? wsum[lane] : 0.0;
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    if (lane == 0) part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = v;
  }
}

// Sum of part[0..n) by one block of 256 threads in a fixed order.
FX_DEV double sum_parts(const double* part, int n) {
  __shared__ double wsum[8];
  double v = 0.0;
  for (int i = threadIdx.x; i < n; i += 256) v += part[i];
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  if ((threadIdx.x & 31) == 0) wsum[threadIdx.x >> 5] = v;
  __syncthreads();
  double t = 0.0;
  for (int w = 0; w < 8; ++w) t += wsum[w];
  __syncthreads();
  return t;
}

// k_resid_restrict for a fine level that is exactly twice its coarse level
// (widths divisible by 4), marching runs of an even number of planes with four
// fine x per thread: the residual of each fine voxel is resid_at's (same
// operations, same order), and the 2x2x2 sums follow k_resid_restrict's
// dz, dy, dx order. The even row's warp adds plane 2m (its row, then the odd
// row's from shared memory) and carries the partial sum to plane 2m + 1. The
// children of every interior coarse cell are interior fine voxels, so no
// neighbour is clamped.
__global__ void __launch_bounds__(256, 4) k_resid_restrict_march(Dims f, const float* __restrict__ rhs, const float* __restrict__ e, Dims c,
                                                                 float* __restrict__ rhs_c, int run) {
  __shared__ float4 srow[2][8][32];  // this plane's residual rows of the block, double-buffered by plane parity
  const uint32_t lane = threadIdx.x, ty = threadIdx.y;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + ty;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)f.d);
  if (zb >= ze) return;  // whole block
  const int D = (int)f.d;
  const uint32_t sy = f.w, sz = f.w * f.h;
  const bool yin = y < f.h;
  const bool xin = x0 < f.w;  // f.w % 4 == 0: x0 + 3 < f.w too
  const uint32_t base = (xin ? x0 : f.w - 4) + f.w * (yin ? y : f.h - 1);
  const bool yint = yin && y > 0 && y < f.h - 1;
  const bool int0 = x0 > 0, int3 = x0 + 3 < f.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < f.w;
  const float4* __restrict__ e4 = reinterpret_cast<const float4*>(e);
  const float4* __restrict__ rhs4 = reinterpret_cast<const float4*>(rhs);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  auto erow = [&](int z) { return (yint && z >= 0 && z < D) ? __ldg(e4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 cm = erow(zb - 1), c0 = erow(zb), cp = erow(zb + 1);
  float4 dv = zero4, yp = zero4, ym = zero4;
  float xle = 0.0f, xre = 0.0f;
  if (yint) {
    const uint32_t i = base + sz * (uint32_t)zb;
    dv = __ldg(rhs4 + (i >> 2));
    yp = __ldg(e4 + ((i + sy) >> 2));
    ym = __ldg(e4 + ((i - sy) >> 2));
    if (left_end) xle = __ldg(e + i - 1);
    if (right_end) xre = __ldg(e + i + 4);
  }
  float part0 = 0.0f, part1 = 0.0f;  // sums of coarse x = x0/2 and x0/2 + 1 (even rows)
  for (int z = zb; z < ze; ++z) {
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    const float4 n_c = erow(z + 2);
    float4 n_dv = zero4, n_yp = zero4, n_ym = zero4;
    float n_xle = 0.0f, n_xre = 0.0f;
    if (yint) {
      n_dv = __ldg(rhs4 + (in >> 2));
      n_yp = __ldg(e4 + ((in + sy) >> 2));
      n_ym = __ldg(e4 + ((in - sy) >> 2));
      if (left_end) n_xle = __ldg(e + in - 1);
      if (right_end) n_xre = __ldg(e + in + 4);
    }
    float left = __shfl_up_sync(0xffffffffu, c0.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, c0.x, 1);  // x0 + 4
    if (left_end) left = xle;
    if (right_end) right = xre;
    float4 r = zero4;
    if (yint && z > 0 && z < D - 1) {
      if (int0) r.x = dv.x - ((c0.y + left + yp.x + ym.x + cp.x + cm.x) - c0.x * 6.0f);
      r.y = dv.y - ((c0.z + c0.x + yp.y + ym.y + cp.y + cm.y) - c0.y * 6.0f);
      r.z = dv.z - ((c0.w + c0.y + yp.z + ym.z + cp.z + cm.z) - c0.z * 6.0f);
      if (int3) r.w = dv.w - ((right + c0.z + yp.w + ym.w + cp.w + cm.w) - c0.w * 6.0f);
    }
    const int b = z & 1;
    srow[b][ty][lane] = r;
    __syncthreads();
    if ((ty & 1) == 0) {
      const float4 o = srow[b][ty + 1][lane];  // row y + 1
      if (b == 0) {
        part0 = 0.0f;
        part1 = 0.0f;
      }
      part0 += r.x;
      part0 += r.y;
      part0 += o.x;
      part0 += o.y;
      part1 += r.z;
      part1 += r.w;
      part1 += o.z;
      part1 += o.w;
      if (b == 1 && xin && yin) {
        const uint32_t cy = y >> 1, cz = (uint32_t)z >> 1;
        for (int h = 0; h < 2; ++h) {
          const uint32_t cx = (x0 >> 1) + (uint32_t)h;
          const bool cb = cx == 0u || cy == 0u || cz == 0u || cx == c.w - 1u || cy == c.h - 1u || cz == c.d - 1u;
          rhs_c[flat(c, cx, cy, cz)] = cb ? 0.0f : ((h ? part1 : part0) * 0.125f) * 4.0f;
        }
      }
    }
    cm = c0;
    c0 = cp;
    cp = n_c;
    dv = n_dv;
    yp = n_yp;
    ym = n_ym;
    xle = n_xle;
    xre = n_xre;
  }
}

// k_prolong_add for a fine level that is exactly twice its coarse level
// (widths divisible by 4), marching runs of planes with four fine x per thread.
// At an interior fine voxel the sample position needs no clamp, its corners are
// coarse cells (c - 1) >> 1 and one more per axis, and its weights are exactly
// 0.75 (even c) or 0.25 (odd c); consecutive fine planes share coarse planes, so
// the thread keeps the two coarse planes of the current fine plane (a float2
// per row, the outer columns by warp shuffle). The mixes are tri_interp's in
// its order, so the values are the same bits. src and dst may be one buffer.
__global__ void __launch_bounds__(256, 4) k_prolong_add_march(Dims c, const float* __restrict__ ec, Dims f, const float* src, float* dst,
                                                              int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)f.d);
  if (y >= f.h || zb >= ze) return;  // whole warp
  const uint32_t sz = f.w * f.h;
  const bool xin = x0 < f.w;
  const uint32_t xb = xin ? x0 : f.w - 4;
  const uint32_t base = xb + f.w * y;
  const float4* src4 = reinterpret_cast<const float4*>(src);
  float4* dst4 = reinterpret_cast<float4*>(dst);
  const bool yint = y > 0 && y < f.h - 1;
  if (!yint) {  // boundary row: dst = src
    if (xin)
      for (int z = zb; z < ze; ++z) {
        const uint32_t q = (base + sz * (uint32_t)z) >> 2;
        dst4[q] = src4[q];
      }
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < f.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < f.w;
  const int D = (int)f.d;
  const uint32_t mc = xb >> 1;
  const uint32_t mby = (y - 1u) >> 1, muy = mby + 1u;
  const float fy = (y & 1u) ? 0.25f : 0.75f;
  const float2* __restrict__ c2 = reinterpret_cast<const float2*>(ec);
  struct Plane {
    float v[2][4];
  };
  auto load_plane = [&](int pz) {
    const uint32_t pc = (uint32_t)max(0, min(pz, (int)c.d - 1));
    const uint32_t i0 = mc + c.w * (mby + c.h * pc), i1 = mc + c.w * (muy + c.h * pc);
    const float2 r0 = __ldg(c2 + (i0 >> 1)), r1 = __ldg(c2 + (i1 >> 1));
    float a = __shfl_up_sync(0xffffffffu, r0.y, 1), b = __shfl_down_sync(0xffffffffu, r0.x, 1);
    float d0 = __shfl_up_sync(0xffffffffu, r1.y, 1), d1 = __shfl_down_sync(0xffffffffu, r1.x, 1);
    if (left_end) {
      a = __ldg(ec + i0 - 1);
      d0 = __ldg(ec + i1 - 1);
    }
    if (right_end) {
      b = __ldg(ec + i0 + 2);
      d1 = __ldg(ec + i1 + 2);
    }
    Plane p;
    p.v[0][0] = a;
    p.v[0][1] = r0.x;
    p.v[0][2] = r0.y;
    p.v[0][3] = b;
    p.v[1][0] = d0;
    p.v[1][1] = r1.x;
    p.v[1][2] = r1.y;
    p.v[1][3] = d1;
    return p;
  };
  auto sample = [&](const Plane& A, const Plane& B, int k, float fx, float fz) {
    const float x00 = mixv(A.v[0][k], A.v[0][k + 1], fx);
    const float x10 = mixv(A.v[1][k], A.v[1][k + 1], fx);
    const float x01 = mixv(B.v[0][k], B.v[0][k + 1], fx);
    const float x11 = mixv(B.v[1][k], B.v[1][k + 1], fx);
    return mixv(mixv(x00, x10, fy), mixv(x01, x11, fy), fz);
  };
  int cbz = (zb - 1) >> 1;
  Plane A = load_plane(cbz), B = load_plane(cbz + 1);
  for (int z = zb; z < ze; ++z) {
    const int bz = (z - 1) >> 1;
    if (bz != cbz) {  // warp-uniform
      A = B;
      cbz = bz;
      B = load_plane(cbz + 1);
    }
    if (!xin) continue;
    const uint32_t q = (base + sz * (uint32_t)z) >> 2;
    float4 v = src4[q];
    if (z > 0 && z < D - 1) {
      const float fz = (z & 1) ? 0.25f : 0.75f;
      if (int0) v.x = v.x + sample(A, B, 0, 0.75f, fz);
      v.y = v.y + sample(A, B, 1, 0.25f, fz);
      v.z = v.z + sample(A, B, 1, 0.75f, fz);
      if (int3) v.w = v.w + sample(A, B, 2, 0.25f, fz);
    }
    dst4[q] = v;
  }
}

// k_resid_norm with four x per thread marching runs of planes (widths divisible
// by 4): each residual term is computed as there, in double from the stored f32
// values; one partial sum per block.
__global__ void __launch_bounds__(256, 4) k_resid_norm_march(Dims f, const float* __restrict__ rhs, const float* __restrict__ p,
                                                             double* part, int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)f.d);
  const int D = (int)f.d;
  const uint32_t sy = f.w, sz = f.w * f.h;
  const bool yin = y < f.h;
  const bool xin = x0 < f.w;
  const uint32_t base = (xin ? x0 : f.w - 4) + f.w * (yin ? y : f.h - 1);
  const bool act = yin && xin && y > 0 && y < f.h - 1;
  const bool int0 = x0 > 0, int3 = x0 + 3 < f.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < f.w;
  const float4* __restrict__ p4 = reinterpret_cast<const float4*>(p);
  const float4* __restrict__ rhs4 = reinterpret_cast<const float4*>(rhs);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  auto prow = [&](int z) { return (act && z >= 0 && z < D) ? __ldg(p4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  double s2 = 0.0;
  if (zb < ze) {
    float4 cm = prow(zb - 1), c0 = prow(zb), cp = prow(zb + 1);
    for (int z = zb; z < ze; ++z) {
      const uint32_t i = base + sz * (uint32_t)z;
      float4 dv = zero4, yp = zero4, ym = zero4;
      float xle = 0.0f, xre = 0.0f;
      if (act) {
        dv = __ldg(rhs4 + (i >> 2));
        yp = __ldg(p4 + ((i + sy) >> 2));
        ym = __ldg(p4 + ((i - sy) >> 2));
        if (left_end) xle = __ldg(p + i - 1);
        if (right_end) xre = __ldg(p + i + 4);
      }
      const float4 n_c = prow(z + 2);
      float left = __shfl_up_sync(0xffffffffu, c0.w, 1);
      float right = __shfl_down_sync(0xffffffffu, c0.x, 1);
      if (left_end) left = xle;
      if (right_end) right = xre;
      if (act && z > 0 && z < D - 1) {
        auto term = [&](float xp, float xm, float ypv, float ymv, float zp, float zm, float c, float rh) {
          const double s = (double)xp + (double)xm + (double)ypv + (double)ymv + (double)zp + (double)zm;
          const double r = (double)rh - (s - 6.0 * (double)c);
          return r * r;
        };
        if (int0) s2 += term(c0.y, left, yp.x, ym.x, cp.x, cm.x, c0.x, dv.x);
        s2 += term(c0.z, c0.x, yp.y, ym.y, cp.y, cm.y, c0.y, dv.y);
        s2 += term(c0.w, c0.y, yp.z, ym.z, cp.z, cm.z, c0.z, dv.z);
        if (int3) s2 += term(right, c0.z, yp.w, ym.w, cp.w, cm.w, c0.w, dv.w);
      }
      cm = c0;
      c0 = cp;
      cp = n_c;
    }
  }
  block_sum_to(s2, part);
}

// The lower part of a V-cycle in one block of 1024 threads: from level k0 (its
// right-hand side restricted and its p[0] cleared by the caller) down to the
// coarsest level and back, as level_cycle runs it: pre-sweeps, residual
// restriction, clearing, the coarsest sweeps, prolongation and post-sweeps, with a
// block barrier between passes. Each voxel is computed as in k_wjacobi,
// k_resid_restrict and k_prolong_add, in their operation order, so the results
// are the same bits. Small levels are bound by launch latency when every pass is
// its own kernel; here they cost one launch. Buffers written in the kernel are
// read with plain loads (never the read-only path) after the barrier.
// A level at most this large runs in the tail kernel: at most 8 voxels per
// thread, whose loads are issued together (one block has too few warps to hide
// the latency of longer chains; 32^3 levels measured slower there than launched).
constexpr uint32_t kTailVoxels = 8192;
constexpr int kTailThreads = 1024;
constexpr int kTailVox = 4;  // voxels per thread per round, loads issued before the arithmetic

FX_DEV void tail_sweep(const LevelBuf& B, const float* src, float* dst, float w, bool one) {
  const Dims d = B.dm;
  const uint32_t n = d.w * d.h * d.d, sy = d.w, sz = d.w * d.h;
  for (uint32_t i0 = threadIdx.x; i0 < n; i0 += kTailThreads * kTailVox) {
    float nb[kTailVox][7];
    bool in[kTailVox];
#pragma unroll
    for (int k = 0; k < kTailVox; ++k) {
      const uint32_t i = i0 + (uint32_t)k * kTailThreads;
      const uint32_t x = i % d.w, y = (i / d.w) % d.h, z = i / sz;
      in[k] = i < n && !is_boundary(d, x, y, z);
      if (in[k]) {
        nb[k][0] = src[i + 1];
        nb[k][1] = src[i - 1];
        nb[k][2] = src[i + sy];
        nb[k][3] = src[i - sy];
        nb[k][4] = src[i + sz];
        nb[k][5] = src[i - sz];
        nb[k][6] = B.div[i];
      }
    }
#pragma unroll
    for (int k = 0; k < kTailVox; ++k) {
      const uint32_t i = i0 + (uint32_t)k * kTailThreads;
      if (i >= n) continue;
      float v = 0.0f;
      if (in[k]) {
        const float s = nb[k][0] + nb[k][1] + nb[k][2] + nb[k][3] + nb[k][4] + nb[k][5];
        const float j = div6(s - nb[k][6]);
        const float cm = src[i];
        v = one ? j : cm + w * (j - cm);
      }
      dst[i] = v;
    }
  }
}

FX_DEV float tail_resid_at(const Dims& f, const float* rhs, const float* e, uint32_t x, uint32_t y, uint32_t z) {
  if (is_boundary(f, x, y, z)) return 0.0f;
  const uint32_t W1 = f.w - 1u, H1 = f.h - 1u, D1 = f.d - 1u;
  const uint32_t i = flat(f, x, y, z);
  const float s = e[flat(f, inc(x, W1), y, z)] + e[flat(f, dec(x), y, z)] + e[flat(f, x, inc(y, H1), z)] + e[flat(f, x, dec(y), z)] +
                  e[flat(f, x, y, inc(z, D1))] + e[flat(f, x, y, dec(z))];
  const float lap = s - e[i] * 6.0f;
  return rhs[i] - lap;
}

FX_DEV void tail_resid_restrict(const LevelBuf& B, const float* e, const LevelBuf& C) {
  const Dims f = B.dm, c = C.dm;
  const uint32_t n = c.w * c.h * c.d;
  for (uint32_t i = threadIdx.x; i < n; i += kTailThreads) {
    const uint32_t x = i % c.w, y = (i / c.w) % c.h, z = i / (c.w * c.h);
    if (x == 0u || y == 0u || z == 0u || x == c.w - 1u || y == c.h - 1u || z == c.d - 1u) {
      C.div[i] = 0.0f;
      continue;
    }
    float sum = 0.0f;
    for (uint32_t dz = 0; dz < 2; ++dz)
      for (uint32_t dy = 0; dy < 2; ++dy)
        for (uint32_t dx = 0; dx < 2; ++dx)
          sum += tail_resid_at(f, B.div, e, min(2u * x + dx, f.w - 1u), min(2u * y + dy, f.h - 1u), min(2u * z + dz, f.d - 1u));
    C.div[i] = (sum * 0.125f) * 4.0f;
  }
}

FX_DEV float tail_interp(const float* f, const Tri& c) {
  const float x00 = mixv(f[c.i000], f[c.i100], c.fx);
  const float x10 = mixv(f[c.i010], f[c.i110], c.fx);
  const float x01 = mixv(f[c.i001], f[c.i101], c.fx);
  const float x11 = mixv(f[c.i011], f[c.i111], c.fx);
  return mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
}

FX_DEV void tail_prolong_add(const LevelBuf& C, const float* ec, const LevelBuf& B, const float* src, float* dst) {
  const Dims f = B.dm;
  const uint32_t n = f.w * f.h * f.d;
  for (uint32_t i = threadIdx.x; i < n; i += kTailThreads) {
    const uint32_t x = i % f.w, y = (i / f.w) % f.h, z = i / (f.w * f.h);
    const float v = src[i];
    if (x == 0u || y == 0u || z == 0u || x == f.w - 1u || y == f.h - 1u || z == f.d - 1u) {
      dst[i] = v;
      continue;
    }
    const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
    const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
    const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
    dst[i] = v + tail_interp(ec, tri_corners(C.dm, px, py, pz));
  }
}

FX_DEV int tail_smooth(const LevelBuf& B, int sweeps, int start, const VCycleConfig& c) {
  int a = start;
  for (int k = 0; k < sweeps; ++k) {
    tail_sweep(B, B.p[a], B.p[a ^ 1], c.omega, c.omega_one);
    __syncthreads();
    a ^= 1;
  }
  return a;
}

// The coarsest level's sweeps with its two buffers and right-hand side held in
// shared memory (up to kTailSharedVox voxels): each thread's voxel indices and
// boundary tests are worked out once, and a sweep reads only shared memory. Each
// voxel is computed as in tail_sweep, in its operation order, so the results are
// the same bits; both buffers are written back, as the ping-pong leaves them.
constexpr uint32_t kTailSharedVox = 8192;
constexpr int kTailSharedPer = (int)(kTailSharedVox / kTailThreads);

FX_DEV int tail_smooth_shared(const LevelBuf& B, int sweeps, int start, const VCycleConfig& c, float* sm) {
  const Dims d = B.dm;
  const uint32_t n = d.w * d.h * d.d, sy = d.w, sz = d.w * d.h;
  float* P[2] = {sm, sm + n};
  float* R = sm + 2 * n;
  for (uint32_t i = threadIdx.x; i < n; i += kTailThreads) {
    P[0][i] = B.p[start][i];
    P[1][i] = B.p[start ^ 1][i];
    R[i] = B.div[i];
  }
  bool valid[kTailSharedPer], inner[kTailSharedPer];
#pragma unroll
  for (int k = 0; k < kTailSharedPer; ++k) {
    const uint32_t i = threadIdx.x + (uint32_t)k * kTailThreads;
    valid[k] = i < n;
    const uint32_t x = i % d.w, y = (i / d.w) % d.h, z = i / sz;
    inner[k] = valid[k] && !is_boundary(d, x, y, z);
  }
  __syncthreads();
  int a = 0;
  for (int it = 0; it < sweeps; ++it) {
    const float* src = P[a];
    float* dst = P[a ^ 1];
#pragma unroll
    for (int k = 0; k < kTailSharedPer; ++k) {
      if (!valid[k]) continue;
      const uint32_t i = threadIdx.x + (uint32_t)k * kTailThreads;
      float v = 0.0f;
      if (inner[k]) {
        const float t = src[i + 1] + src[i - 1] + src[i + sy] + src[i - sy] + src[i + sz] + src[i - sz];
        const float j = div6(t - R[i]);
        const float cm = src[i];
        v = c.omega_one ? j : cm + c.omega * (j - cm);
      }
      dst[i] = v;
    }
    __syncthreads();
    a ^= 1;
  }
  for (uint32_t i = threadIdx.x; i < n; i += kTailThreads) {
    B.p[start][i] = P[0][i];
    B.p[start ^ 1][i] = P[1][i];
  }
  __syncthreads();
  return start ^ (sweeps & 1);
}

__global__ void __launch_bounds__(kTailThreads) k_vcycle_tail(VCycleLevels L, VCycleConfig c, int k0, int coarse_shared) {
  int a[kMaxVLevels];
  for (int k = k0; k < c.levels - 1; ++k) {
    const LevelBuf& B = L.lv[k];
    const LevelBuf& C = L.lv[k + 1];
    a[k] = tail_smooth(B, c.pre, 0, c);
    tail_resid_restrict(B, B.p[a[k]], C);
    const uint32_t nc = C.dm.w * C.dm.h * C.dm.d;
    for (uint32_t i = threadIdx.x; i < nc; i += kTailThreads) C.p[0][i] = 0.0f;
    __syncthreads();
  }
  extern __shared__ float tail_sm[];
  int e = coarse_shared ? tail_smooth_shared(L.lv[c.levels - 1], c.coarse, 0, c, tail_sm)
                        : tail_smooth(L.lv[c.levels - 1], c.coarse, 0, c);
  for (int k = c.levels - 2; k >= k0; --k) {
    const LevelBuf& B = L.lv[k];
    const LevelBuf& C = L.lv[k + 1];
    const int b = ((c.pre + c.post) & 1) ? a[k] ^ 1 : a[k];
    tail_prolong_add(C, C.p[e], B, B.p[a[k]], B.p[b]);
    __syncthreads();
    e = tail_smooth(B, c.post, b, c);
  }
}

__global__ void __launch_bounds__(256) k_fill0(float* __restrict__ p, uint32_t n) {
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0.0f;
}

__global__ void __launch_bounds__(256) k_sumsq(const float* __restrict__ a, uint32_t n, double* part) {
  double s = 0.0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
    const double v = (double)__ldg(a + i);
    s += v * v;
  }
  block_sum_to(s, part);
}

// Sum over interior voxels of (rhs - (sum of the 6 neighbours - 6 p))^2, each
// term in double from the stored f32 values.
__global__ void __launch_bounds__(256) k_resid_norm(Dims f, const float* __restrict__ rhs, const float* __restrict__ p, double* part) {
  const uint32_t iw = f.w - 2u, ih = f.h - 2u, id = f.d - 2u;
  const uint32_t n = iw * ih * id;
  const uint32_t sy = f.w, sz = f.w * f.h;
  double s2 = 0.0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t x = 1u + t % iw, y = 1u + (t / iw) % ih, z = 1u + t / (iw * ih);
    const uint32_t i = flat(f, x, y, z);
    const double s = (double)__ldg(p + i + 1) + (double)__ldg(p + i - 1) + (double)__ldg(p + i + sy) + (double)__ldg(p + i - sy) +
                     (double)__ldg(p + i + sz) + (double)__ldg(p + i - sz);
    const double r = (double)__ldg(rhs + i) - (s - 6.0 * (double)__ldg(p + i));
    s2 += r * r;
  }
  block_sum_to(s2, part);
}

// Adds the residual partials (and, with nrhs > 0, the right-hand side's),
// counts the cycle, decides whether another cycle is due and hands the decision
// to the graph's WHILE node. One block of 256 threads.
__global__ void __launch_bounds__(256) k_finalize(SolverDev* st, double tol, int max_cycles, int count, int nres, int nrhs,
                                                  cudaGraphConditionalHandle cond) {
  const double res2 = sum_parts(st->part_res, nres);
  const double rhs2 = nrhs > 0 ? sum_parts(st->part_rhs, nrhs) : 0.0;
  if (threadIdx.x != 0) return;
  if (nrhs > 0) st->rhs2 = rhs2;
  if (count) st->cycles += 1;
  st->res2 = res2;
  const bool done = sqrt(st->res2) <= tol * sqrt(st->rhs2);
  st->converged = done ? 1 : 0;
  const int cont = (!done && st->cycles < max_cycles) ? 1 : 0;
  st->cont = cont;
  if (cond) cudaGraphSetConditional(cond, (unsigned)cont);
}

__global__ void __launch_bounds__(256) k_maxdiv(Dims dm, VelField v, unsigned long long* bits) {
  const uint32_t iw = dm.w - 2u, ih = dm.h - 2u, id = dm.d - 2u;
  const uint32_t n = iw * ih * id;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  double m = 0.0;
  for (uint32_t t = blockIdx.x * blockDim.x + threadIdx.x; t < n; t += gridDim.x * blockDim.x) {
    const uint32_t x = 1u + t % iw, y = 1u + (t / iw) % ih, z = 1u + t / (iw * ih);
    const uint32_t i = flat(dm, x, y, z);
    const double ddx = (double)__ldg(v.c[0] + i + 1) - (double)__ldg(v.c[0] + i - 1);
    const double ddy = (double)__ldg(v.c[1] + i + sy) - (double)__ldg(v.c[1] + i - sy);
    const double ddz = (double)__ldg(v.c[2] + i + sz) - (double)__ldg(v.c[2] + i - sz);
    m = fmax(m, fabs(0.5 * (ddx + ddy + ddz)));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmax(m, __shfl_down_sync(0xffffffffu, m, o));
  // non-negative doubles order like their bit patterns
  if ((threadIdx.x & 31) == 0 && m > 0.0) atomicMax(bits, (unsigned long long)__double_as_longlong(m));
}

inline uint32_t reduce_blocks() { return std::min<uint32_t>((uint32_t)device_sm_count() * 4u, (uint32_t)kNormParts); }

inline dim3 vz_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 7) / 8, (d.d + kVZ - 1) / kVZ); }
inline dim3 pt_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 3) / 4, (d.d + 1) / 2); }
const dim3 kPtBlock(32, 4, 2);
const dim3 kMarchBlock(32, 8, 1);

inline uint32_t count_of(Dims d) { return d.w * d.h * d.d; }

// Resident 256-thread blocks of `kernel` on the current device, cached per device.
int resident_slots(const void* kernel, int* cache) {
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return device_sm_count();
  if (cache[dev] <= 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0) != cudaSuccess) per_sm = 1;
    cache[dev] = std::max(1, per_sm) * device_sm_count();
  }
  return cache[dev];
}

// Four-x marching kernels need widths divisible by 4 (and at least 8).
inline bool marchable(Dims d) { return d.w % 4 == 0 && d.w >= 8; }
// The fine level is exactly twice the coarse one on every axis.
inline bool halves(Dims f, Dims c) { return marchable(f) && f.w == 2 * c.w && f.h == 2 * c.h && f.d == 2 * c.d; }
inline dim3 march_grid(Dims d, int run) { return dim3((d.w + 127) / 128, (d.h + 7) / 8, (d.d + run - 1) / run); }

void fill0(cudaStream_t s, float* p, Dims d) {
  const uint32_t n = count_of(d);
  k_fill0<<<std::min<uint32_t>((n + 255) / 256, reduce_blocks() * 2), 256, 0, s>>>(p, n);
}

int smooth(cudaStream_t s, const LevelBuf& B, int sweeps, int start, const VCycleConfig& c, uint32_t* launches) {
  int a = start;
  for (int k = 0; k < sweeps; ++k) {
    if (c.plain || march_wsweep(s, B.dm, B.div, B.p[a], B.p[a ^ 1], c.omega, c.omega_one) != cudaSuccess) {
      (void)cudaGetLastError();  // cudaErrorNotSupported is a host-side refusal, nothing was launched
      k_wjacobi<<<vz_grid(B.dm), dim3(32, 8, 1), 0, s>>>(B.dm, B.div, B.p[a], B.p[a ^ 1], c.omega, c.omega_one ? 1 : 0);
    }
    a ^= 1;
    ++*launches;
  }
  return a;
}

void resid_restrict(cudaStream_t s, const LevelBuf& B, const float* e, const LevelBuf& C, bool plain) {
  if (!plain && halves(B.dm, C.dm)) {
    static int cache[64];
    const int run = march_plan_pairs(B.dm, resident_slots((const void*)k_resid_restrict_march, cache));
    k_resid_restrict_march<<<march_grid(B.dm, run), kMarchBlock, 0, s>>>(B.dm, B.div, e, C.dm, C.div, run);
  } else {
    k_resid_restrict<<<pt_grid(C.dm), kPtBlock, 0, s>>>(B.dm, B.div, e, C.dm, C.div);
  }
}

void prolong_add(cudaStream_t s, const LevelBuf& C, const float* ec, const LevelBuf& B, const float* src, float* dst, bool plain) {
  if (!plain && halves(B.dm, C.dm)) {
    static int cache[64];
    const int run = march_plan_one_wave(B.dm, resident_slots((const void*)k_prolong_add_march, cache));
    k_prolong_add_march<<<march_grid(B.dm, run), kMarchBlock, 0, s>>>(C.dm, ec, B.dm, src, dst, run);
  } else {
    k_prolong_add<<<pt_grid(B.dm), kPtBlock, 0, s>>>(C.dm, ec, B.dm, src, dst);
  }
}

// The FP64 residual norm's partials into part; returns how many.
int resid_norm(cudaStream_t s, Dims dm, const float* rhs, const float* p, double* part, bool plain) {
  if (!plain && marchable(dm)) {
    static int cache[64];
    const int run = march_plan_one_wave(dm, resident_slots((const void*)k_resid_norm_march, cache));
    const dim3 g = march_grid(dm, run);
    const uint32_t blocks = g.x * g.y * g.z;
    if (blocks <= (uint32_t)kNormParts) {
      k_resid_norm_march<<<g, kMarchBlock, 0, s>>>(dm, rhs, p, part, run);
      return (int)blocks;
    }
  }
  k_resid_norm<<<reduce_blocks(), 256, 0, s>>>(dm, rhs, p, part);
  return (int)reduce_blocks();
}

// The buffer id that level_cycle(k, start) ends in (host arithmetic).
int cycle_end_id(const VCycleConfig& c, int k, int start) {
  if (k == c.levels - 1) return start ^ (c.coarse & 1);
  const int a = start ^ (c.pre & 1);
  const int b = ((c.pre + c.post) & 1) ? a ^ 1 : a;
  return b ^ (c.post & 1);
}

// first_done: the level's first pre-sweep has already run (fused with the
// residual norm, see fused_norm_sweep), from p[start] into p[start ^ 1].
int level_cycle(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int k, int start, uint32_t* launches,
                bool first_done = false) {
  const LevelBuf& B = L.lv[k];
  // A small level and everything below it: one block, one launch (the caller has
  // restricted its right-hand side and cleared p[0], so start is 0).
  if (!c.plain && k > 0 && start == 0 && count_of(B.dm) <= kTailVoxels) {
    const uint32_t nc = count_of(L.lv[c.levels - 1].dm);
    const int shared = nc <= kTailSharedVox ? 1 : 0;
    k_vcycle_tail<<<1, kTailThreads, shared ? 3 * nc * sizeof(float) : 0, s>>>(L, c, k, shared);
    ++*launches;
    return cycle_end_id(c, k, 0);
  }
  if (k == c.levels - 1) return smooth(s, B, c.coarse, start, c, launches);
  const int a = first_done ? smooth(s, B, c.pre - 1, start ^ 1, c, launches) : smooth(s, B, c.pre, start, c, launches);
  const LevelBuf& C = L.lv[k + 1];
  resid_restrict(s, B, B.p[a], C, c.plain);
  fill0(s, C.p[0], C.dm);
  *launches += 2;
  const int ce = level_cycle(s, L, c, k + 1, 0, launches);
  const int b = ((c.pre + c.post) & 1) ? a ^ 1 : a;
  prolong_add(s, C, C.p[ce], B, B.p[a], B.p[b], c.plain);
  ++*launches;
  return smooth(s, B, c.post, b, c, launches);
}

}  // namespace

// Whether the fine level's residual norm rides on the next cycle's first
// pre-sweep: the marching kernels, at least one pre-sweep and a fine level with
// more than one level below it (a cycle's fine pre-smoothing starts from p[start]).
bool fuse_norm(const VCycleLevels& L, const VCycleConfig& c) {
  return !c.plain && c.pre >= 1 && c.levels >= 2 && L.lv[0].dm.w % 4 == 0 && L.lv[0].dm.w >= 8;
}

// The residual norm of p[start] (its partials into st->part_res) and, in the same
// pass, the first pre-sweep of the next cycle from p[start] into p[start ^ 1]:
// both read the same neighbours. When the norm stops the loop, the sweep's output
// is left unused in p[start ^ 1] (the result stays in p[start]). Returns the
// partial count, or 0 where the fused kernel refuses.
int fused_norm_sweep(cudaStream_t s, const LevelBuf& F, const VCycleConfig& c, int start, SolverDev* st) {
  int n = kNormParts;
  if (march_wsweep_norm(s, F.dm, F.div, F.p[start], F.p[start ^ 1], c.omega, c.omega_one, st->part_res, &n) != cudaSuccess) {
    (void)cudaGetLastError();  // a host-side refusal: nothing was launched
    return 0;
  }
  return n;
}

// The fused pass, or where the kernel refuses, the norm and the first pre-sweep
// apart (the next cycle expects that sweep done either way).
int norm_and_first_sweep(cudaStream_t s, const LevelBuf& F, const VCycleConfig& c, int start, SolverDev* st, uint32_t* launches) {
  int n = fused_norm_sweep(s, F, c, start, st);
  if (n > 0) return n;
  n = resid_norm(s, F.dm, F.div, F.p[start], st->part_res, c.plain);
  smooth(s, F, 1, start, c, launches);
  return n;
}

cudaError_t vcycle_prologue(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                            cudaGraphConditionalHandle cond) {
  const LevelBuf& F = L.lv[0];
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(SolverDev), s);
  if (e != cudaSuccess) return e;
  if (!c.warm) fill0(s, F.p[start], F.dm);
  k_sumsq<<<reduce_blocks(), 256, 0, s>>>(F.div, count_of(F.dm), st->part_rhs);
  uint32_t extra = 0;
  const int nres = fuse_norm(L, c) ? norm_and_first_sweep(s, F, c, start, st, &extra) : resid_norm(s, F.dm, F.div, F.p[start], st->part_res, c.plain);
  k_finalize<<<1, 256, 0, s>>>(st, c.tol, c.max_cycles, 0, nres, (int)reduce_blocks(), cond);
  return cudaGetLastError();
}

cudaError_t vcycle_body(cudaStream_t s, const VCycleLevels& L, const VCycleConfig& c, int start, SolverDev* st,
                        cudaGraphConditionalHandle cond, uint32_t* launches) {
  const LevelBuf& F = L.lv[0];
  // The prologue and every body end with the fused norm and first pre-sweep
  // whenever fuse_norm holds (the host decides both the same way).
  const bool fused = fuse_norm(L, c);
  const int fin = level_cycle(s, L, c, 0, start, launches, fused);
  (void)fin;  // == start: the fine level ends in the buffer it started from
  const int nres = fused ? norm_and_first_sweep(s, F, c, start, st, launches) : resid_norm(s, F.dm, F.div, F.p[start], st->part_res, c.plain);
  k_finalize<<<1, 256, 0, s>>>(st, c.tol, c.max_cycles, 1, nres, 0, cond);
  *launches += 2;
  return cudaGetLastError();
}

cudaError_t solver_norms(cudaStream_t s, Dims dm, const float* div, const float* p, double tol, SolverDev* st) {
  cudaError_t e = cudaMemsetAsync(st, 0, sizeof(SolverDev), s);
  if (e != cudaSuccess) return e;
  k_sumsq<<<reduce_blocks(), 256, 0, s>>>(div, count_of(dm), st->part_rhs);
  const int nres = resid_norm(s, dm, div, p, st->part_res, false);
  k_finalize<<<1, 256, 0, s>>>(st, tol, 0, 0, nres, (int)reduce_blocks(), 0);
  return cudaGetLastError();
}

cudaError_t vcycle_init() {
  return cudaFuncSetAttribute(k_vcycle_tail, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)(3 * kTailSharedVox * sizeof(float)));
}

cudaError_t max_divergence(cudaStream_t s, Dims dm, VelField v, SolverDev* st) {
  k_maxdiv<<<reduce_blocks(), 256, 0, s>>>(dm, v, &st->maxdiv_bits);
  return cudaGetLastError();
}

}  // namespace fx
