// Fine-level pressure passes of the fused path: the Jacobi sweep
// (pressure-jacobi.wgsl.ts:15-36) in several bit-identical thread layouts, the
// divergence (compute-divergence.wgsl.ts:22-42) fused with the first sweep and
// the fine->mid restriction (pressure-restriction.wgsl.ts:27-50), and the
// mid->fine prolongation (pressure-prolongation.wgsl.ts:29-44) fused with the
// first post-sweep.
//
// Every value is computed with the reference's operations in its order: the
// result equals the sweep-by-sweep evaluation of the reference bit for bit. The
// division by 6 is the exact IEEE quotient (div6, fx_math.cuh).
#include <algorithm>
#include <cstdlib>

#include "fx_fused.h"
#include "fx_pressure.h"

namespace fx {
namespace {

// Integer tuning knob from the environment (defaults come from measurement).
int env_int(const char* name, int dflt, int lo, int hi) {
  const char* v = std::getenv(name);
  if (!v || !*v) return dflt;
  const int x = std::atoi(v);
  return (x >= lo && x <= hi) ? x : dflt;
}

// Prolongation term of pressure-prolongation.wgsl.ts:42-43 at fine voxel (x,y,z).
FX_DEV float prolong_sample(const Dims& mid, const float* __restrict__ mp, int x, int y, int z) {
  const float px = ((float)x + 0.5f) * 0.5f - 0.5f;
  const float py = ((float)y + 0.5f) * 0.5f - 0.5f;
  const float pz = ((float)z + 0.5f) * 0.5f - 0.5f;
  return tri_interp(mp, tri_corners(mid, px, py, pz));
}

// ---------------------------------------------------------------------------
// Lean per-voxel kernels (one thread per voxel, blocks of 32 x 4 x 2).
// ---------------------------------------------------------------------------

// Divergence (compute-divergence.wgsl.ts:22-42) with, pointwise, the first
// Jacobi sweep from the cleared buffer, (0 - div) / 6, and the fine->mid
// restriction (pressure-restriction.wgsl.ts:27-50) of each 2x2x2 group of the
// block through shared memory. The restriction needs every fine dimension >= 16.
__global__ void __launch_bounds__(256) k_div_first(Dims dm, VelField v, float* __restrict__ div, float* __restrict__ p1, Dims mid,
                                                   float* __restrict__ mid_div, int restrict_mid) {
  __shared__ float sd[2][4][32];
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 4 + threadIdx.y, z = blockIdx.z * 2 + threadIdx.z;
  const bool in = x < dm.w && y < dm.h && z < dm.d;
  float d = 0.0f;
  if (in) {
    const uint32_t i = flat(dm, x, y, z);
    if (!is_boundary(dm, x, y, z)) {
      const uint32_t sy = dm.w, sz = dm.w * dm.h;
      const float ddx = __ldg(v.c[0] + i + 1) - __ldg(v.c[0] + i - 1);
      const float ddy = __ldg(v.c[1] + i + sy) - __ldg(v.c[1] + i - sy);
      const float ddz = __ldg(v.c[2] + i + sz) - __ldg(v.c[2] + i - sz);
      d = (ddx + ddy + ddz) * 0.5f;
      if (p1) p1[i] = div6(0.0f - d);
    } else if (p1) {
      p1[i] = 0.0f;
    }
    div[i] = d;
  }
  if (!restrict_mid) return;
  sd[threadIdx.z][threadIdx.y][threadIdx.x] = d;
  __syncthreads();
  if (threadIdx.z == 0 && (threadIdx.y & 1) == 0 && (threadIdx.x & 1) == 0) {
    const uint32_t mx_ = x >> 1, my_ = y >> 1, mz_ = z >> 1;
    if (mx_ < mid.w && my_ < mid.h && mz_ < mid.d) {
      float out = 0.0f;
      if (!(mx_ == 0 || my_ == 0 || mz_ == 0 || mx_ == mid.w - 1 || my_ == mid.h - 1 || mz_ == mid.d - 1)) {
        const int tx = threadIdx.x, ty = threadIdx.y;
        float sum = 0.0f;
        sum += sd[0][ty][tx];
        sum += sd[0][ty][tx + 1];
        sum += sd[0][ty + 1][tx];
        sum += sd[0][ty + 1][tx + 1];
        sum += sd[1][ty][tx];
        sum += sd[1][ty][tx + 1];
        sum += sd[1][ty + 1][tx];
        sum += sd[1][ty + 1][tx + 1];
        out = sum * 0.125f;
      }
      mid_div[flat(mid, mx_, my_, mz_)] = out;
    }
  }
}

// k_div_first with four x per thread marching runs of planes (widths divisible
// by 4, even heights and depths; runs of even length starting on even planes).
// Per plane a thread loads one float4 of vx (the x neighbours by warp shuffle,
// the row ends load theirs), two of vy (rows y - 1 and y + 1) and one of vz
// (plane z + 1; planes z - 1 and z are held from the earlier planes), issuing
// the next plane's loads before it computes the current one. The restriction
// adds each 2x2x2 group in k_div_first's order: the even row's warp sums plane
// 2m (its row, then the odd row's from shared memory) and carries the partial
// sum to plane 2m + 1. Every value is computed with the same operations in the
// same order, so the results are the same bits.
__global__ void __launch_bounds__(256, 4) k_div_march(Dims dm, VelField v, float* __restrict__ div, float* __restrict__ p1, Dims mid,
                                                      float* __restrict__ mid_div, int restrict_mid, int run) {
  __shared__ float4 srow[2][8][32];  // this plane's divergence rows of the block, double-buffered by plane parity
  const uint32_t lane = threadIdx.x, ty = threadIdx.y;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + ty;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (zb >= ze) return;  // whole block
  const int D = (int)dm.d;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool yin = y < dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * (yin ? y : dm.h - 1);
  const bool yint = yin && y > 0 && y < dm.h - 1;
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are interior in x
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const float4* __restrict__ vx4 = reinterpret_cast<const float4*>(v.c[0]);
  const float4* __restrict__ vy4 = reinterpret_cast<const float4*>(v.c[1]);
  const float4* __restrict__ vz4 = reinterpret_cast<const float4*>(v.c[2]);
  const float* __restrict__ vx = v.c[0];
  float4* __restrict__ div4 = reinterpret_cast<float4*>(div);
  float4* __restrict__ p14 = reinterpret_cast<float4*>(p1);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  // vz row at a plane (zero outside the grid and on boundary rows, which never use it)
  auto vzrow = [&](int z) { return (yint && z >= 0 && z < D) ? __ldg(vz4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 vzm = vzrow(zb - 1), vzc = vzrow(zb), vzp = vzrow(zb + 1);
  float4 X = zero4, YP = zero4, YM = zero4;
  float XL = 0.0f, XR = 0.0f;
  {
    const uint32_t i = base + sz * (uint32_t)zb;
    if (yint) {
      X = __ldg(vx4 + (i >> 2));
      YP = __ldg(vy4 + ((i + sy) >> 2));
      YM = __ldg(vy4 + ((i - sy) >> 2));
      if (left_end) XL = __ldg(vx + i - 1);
      if (right_end) XR = __ldg(vx + i + 4);
    }
  }
  float part0 = 0.0f, part1 = 0.0f;  // restriction sums of mid x = x0/2 and x0/2 + 1 (even rows)
  for (int z = zb; z < ze; ++z) {
    // next plane's loads (clamped in range on the last plane, values then unused)
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    float4 nX = zero4, nYP = zero4, nYM = zero4;
    float nXL = 0.0f, nXR = 0.0f;
    if (yint) {
      nX = __ldg(vx4 + (in >> 2));
      nYP = __ldg(vy4 + ((in + sy) >> 2));
      nYM = __ldg(vy4 + ((in - sy) >> 2));
      if (left_end) nXL = __ldg(vx + in - 1);
      if (right_end) nXR = __ldg(vx + in + 4);
    }
    const float4 nvz = vzrow(z + 2);
    float left = __shfl_up_sync(0xffffffffu, X.w, 1);     // vx at x0 - 1
    float right = __shfl_down_sync(0xffffffffu, X.x, 1);  // vx at x0 + 4
    if (left_end) left = XL;
    if (right_end) right = XR;
    float4 d = zero4;
    const bool plane_int = yint && z > 0 && z < D - 1;
    if (plane_int) {
      if (int0) d.x = ((X.y - left) + (YP.x - YM.x) + (vzp.x - vzm.x)) * 0.5f;
      d.y = ((X.z - X.x) + (YP.y - YM.y) + (vzp.y - vzm.y)) * 0.5f;
      d.z = ((X.w - X.y) + (YP.z - YM.z) + (vzp.z - vzm.z)) * 0.5f;
      if (int3) d.w = ((right - X.z) + (YP.w - YM.w) + (vzp.w - vzm.w)) * 0.5f;
    }
    const uint32_t i = base + sz * (uint32_t)z;
    if (yin && xin) {
      div4[i >> 2] = d;
      if (p1) {
        float4 q = zero4;
        if (plane_int) {
          if (int0) q.x = div6(0.0f - d.x);
          q.y = div6(0.0f - d.y);
          q.z = div6(0.0f - d.z);
          if (int3) q.w = div6(0.0f - d.w);
        }
        p14[i >> 2] = q;
      }
    }
    if (restrict_mid) {
      const int b = z & 1;
      srow[b][ty][lane] = d;
      __syncthreads();
      if ((ty & 1) == 0) {
        const float4 o = srow[b][ty + 1][lane];  // row y + 1 (zero beyond the grid)
        if (b == 0) {
          part0 = 0.0f;
          part1 = 0.0f;
        }
        part0 += d.x;
        part0 += d.y;
        part0 += o.x;
        part0 += o.y;
        part1 += d.z;
        part1 += d.w;
        part1 += o.z;
        part1 += o.w;
        if (b == 1 && xin && yin) {
          const uint32_t my_ = y >> 1, mz_ = (uint32_t)z >> 1;
          for (int h = 0; h < 2; ++h) {
            const uint32_t mx_ = (x0 >> 1) + (uint32_t)h;
            if (mx_ < mid.w && my_ < mid.h && mz_ < mid.d) {
              const bool mb = mx_ == 0 || my_ == 0 || mz_ == 0 || mx_ == mid.w - 1 || my_ == mid.h - 1 || mz_ == mid.d - 1;
              mid_div[flat(mid, mx_, my_, mz_)] = mb ? 0.0f : (h ? part1 : part0) * 0.125f;
            }
          }
        }
      }
    }
    vzm = vzc;
    vzc = vzp;
    vzp = nvz;
    X = nX;
    YP = nYP;
    YM = nYM;
    XL = nXL;
    XR = nXR;
  }
}

// One Jacobi sweep (pressure-jacobi.wgsl.ts:15-36). With `mid_p`, the result
// then gets the prolongation added (pressure-prolongation.wgsl.ts:36-43: the
// boundary stays 0, the interior becomes p + sample), as when the reference
// prolongs into the buffer this sweep wrote. With `src` NULL the input is the
// cleared buffer.
//
// A thread computes a column of ZB voxels along z, reusing the z neighbours in
// registers; all loads of the column are independent, which keeps enough bytes
// in flight per SM to stream HBM.
// A warp holds 32 consecutive x of one row. The x neighbours come from the
// coalesced centre row by shuffles (the two row ends load their outer
// neighbour), the z neighbours from the column in registers; every load of the
// column is issued before the arithmetic. The sum keeps the reference order
// +x, -x, +y, -y, +z, -z.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                               Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x = blockIdx.x * 32 + lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x < dm.w;
  const uint32_t base = (xin ? x : dm.w - 1) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const bool xint = x > 0 && x < dm.w - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst[base + sz * (z0 + k)] = 0.0f;
    return;
  }
  float c[ZB + 2], yp[ZB], ym[ZB], dv[ZB], xe[ZB];
  const bool left_end = lane == 0 && x > 0, right_end = (lane == 31 || x == dm.w - 1) && x + 1 < dm.w;
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src + base + sz * (uint32_t)z) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div + i);
    yp[k] = src ? __ldg(src + i + sy) : 0.0f;
    ym[k] = src ? __ldg(src + i - sy) : 0.0f;
    xe[k] = 0.0f;
    if (src && left_end) xe[k] = __ldg(src + i - 1);
    if (src && right_end) xe[k] = __ldg(src + i + 1);
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float cm = c[k + 1];
    float xr = __shfl_down_sync(0xffffffffu, cm, 1);
    float xl = __shfl_up_sync(0xffffffffu, cm, 1);
    if (right_end) xr = xe[k];
    if (left_end) xl = xe[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float v = 0.0f;
    if (xint && z > 0 && z < dm.d - 1) {
      if (src) {
        const float s = xr + xl + yp[k] + ym[k] + c[k + 2] + c[k];
        v = div6(s - dv[k]);
      } else {
        v = div6(0.0f - dv[k]);
      }
      if (mid_p) v = v + prolong_sample(mid, mid_p, (int)x, (int)y, (int)z);
    }
    dst[base + sz * z] = v;
  }
}

// k_sweep with two consecutive x per thread (even widths): a warp covers 64 x,
// the column loads are float2, and one shuffle per voxel brings the outer x
// neighbour of each pair from the next lane. Each voxel's sum, division and
// prolongation are those of k_sweep, in the same order, so the results are the
// same bits.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep_v2(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                                  Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 64 + 2 * lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w is even: x0 + 1 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 2) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  const float2* __restrict__ src2 = reinterpret_cast<const float2*>(src);
  const float2* __restrict__ div2 = reinterpret_cast<const float2*>(div);
  float2* __restrict__ dst2 = reinterpret_cast<float2*>(dst);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst2[(base + sz * (z0 + k)) >> 1] = make_float2(0.0f, 0.0f);
    return;
  }
  const bool int0 = x0 > 0 && x0 < dm.w - 1, int1 = x0 + 1 < dm.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 2 < dm.w;
  float2 c[ZB + 2], yp[ZB], ym[ZB], dv[ZB];
  float xl_e[ZB], xr_e[ZB];
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src2 + ((base + sz * (uint32_t)z) >> 1)) : make_float2(0.0f, 0.0f);
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div2 + (i >> 1));
    yp[k] = src ? __ldg(src2 + ((i + sy) >> 1)) : make_float2(0.0f, 0.0f);
    ym[k] = src ? __ldg(src2 + ((i - sy) >> 1)) : make_float2(0.0f, 0.0f);
    xl_e[k] = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
    xr_e[k] = (src && right_end) ? __ldg(src + i + 2) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float2 cm = c[k + 1];
    float left = __shfl_up_sync(0xffffffffu, cm.y, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, cm.x, 1);  // x0 + 2
    if (left_end) left = xl_e[k];
    if (right_end) right = xr_e[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    const bool zint = z > 0 && z < dm.d - 1;
    float v0 = 0.0f, v1 = 0.0f;
    if (zint && int0) {
      v0 = src ? div6(cm.y + left + yp[k].x + ym[k].x + c[k + 2].x + c[k].x - dv[k].x) : div6(0.0f - dv[k].x);
      if (mid_p) v0 = v0 + prolong_sample(mid, mid_p, (int)x0, (int)y, (int)z);
    }
    if (zint && int1) {
      v1 = src ? div6(right + cm.x + yp[k].y + ym[k].y + c[k + 2].y + c[k].y - dv[k].y) : div6(0.0f - dv[k].y);
      if (mid_p) v1 = v1 + prolong_sample(mid, mid_p, (int)x0 + 1, (int)y, (int)z);
    }
    dst2[(base + sz * z) >> 1] = make_float2(v0, v1);
  }
}

// k_sweep with four consecutive x per thread (widths divisible by 4): a warp
// covers 128 x, the column loads are float4, and one shuffle each way per voxel
// row brings the outer x neighbours from the adjacent lanes. Each voxel's sum,
// division and prolongation are those of k_sweep, in the same order, so the
// results are the same bits.
template <int ZB>
__global__ void __launch_bounds__(256) k_sweep_v4(Dims dm, const float* __restrict__ div, const float* __restrict__ src, float* __restrict__ dst,
                                                  Dims mid, const float* __restrict__ mid_p) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const int nz = min(ZB, (int)dm.d - (int)z0);
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  if (!yint) {
    if (xin)
      for (int k = 0; k < nz; ++k) dst4[(base + sz * (z0 + k)) >> 2] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  float4 c[ZB + 2], yp[ZB], ym[ZB], dv[ZB];
  float xl_e[ZB], xr_e[ZB];
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
#pragma unroll
  for (int k = 0; k < ZB + 2; ++k) {
    const int z = (int)z0 + k - 1;
    c[k] = (src && z >= 0 && z < (int)dm.d) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = min(z0 + k, dm.d - 1);
    const uint32_t i = base + sz * z;
    dv[k] = __ldg(div4 + (i >> 2));
    yp[k] = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
    ym[k] = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
    xl_e[k] = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
    xr_e[k] = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  }
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const float4 cm = c[k + 1];
    float left = __shfl_up_sync(0xffffffffu, cm.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, cm.x, 1);  // x0 + 4
    if (left_end) left = xl_e[k];
    if (right_end) right = xr_e[k];
    const uint32_t z = z0 + k;
    if (k >= nz || !xin) continue;
    float4 v = zero4;
    if (z > 0 && z < dm.d - 1) {
      if (src) {
        if (int0) v.x = div6(cm.y + left + yp[k].x + ym[k].x + c[k + 2].x + c[k].x - dv[k].x);
        v.y = div6(cm.z + cm.x + yp[k].y + ym[k].y + c[k + 2].y + c[k].y - dv[k].y);
        v.z = div6(cm.w + cm.y + yp[k].z + ym[k].z + c[k + 2].z + c[k].z - dv[k].z);
        if (int3) v.w = div6(right + cm.z + yp[k].w + ym[k].w + c[k + 2].w + c[k].w - dv[k].w);
      } else {
        if (int0) v.x = div6(0.0f - dv[k].x);
        v.y = div6(0.0f - dv[k].y);
        v.z = div6(0.0f - dv[k].z);
        if (int3) v.w = div6(0.0f - dv[k].w);
      }
      if (mid_p) {
        if (int0) v.x = v.x + prolong_sample(mid, mid_p, (int)x0, (int)y, (int)z);
        v.y = v.y + prolong_sample(mid, mid_p, (int)x0 + 1, (int)y, (int)z);
        v.z = v.z + prolong_sample(mid, mid_p, (int)x0 + 2, (int)y, (int)z);
        if (int3) v.w = v.w + prolong_sample(mid, mid_p, (int)x0 + 3, (int)y, (int)z);
      }
    }
    dst4[(base + sz * z) >> 2] = v;
  }
}

// k_sweep_v4 marching in z: a thread owns four x of one row and walks a run of
// `run` planes, holding the rows at z - 1, z and z + 1 in registers and issuing
// the loads of plane z + 1 before it computes plane z, so a warp always has one
// plane of loads in flight. The host sizes the runs so the grid is one wave of
// resident blocks. Each voxel's sum and division are those of k_sweep, in the
// same order, so the results are the same bits. The sweep with the fused
// prolongation has its own marching kernel, k_sweep_march_prolong, which also
// shares the prolongation's mid-level corners between voxels.
//
// WEIGHTED is the V-cycle's weighted sweep (an extension, fx_vcycle.cu): each
// interior value becomes c + w (j - c), with j the Jacobi value above and c the
// source value, in that operation order; the boundary stays 0.
// With NORM the kernel also adds up, in FP64, the squared residual
// rhs - (sum of the 6 neighbours - 6 p) of its source over the interior voxels it
// visits (the residual norm of k_resid_norm_march, per voxel in the same
// operations), one deterministic partial per block into norm_part.
FX_DEV void block_sum_double(double v, double* part) {
  for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
  __shared__ double warp_sums[8];  // blocks of 32 x 8 threads
  if (threadIdx.x == 0) warp_sums[threadIdx.y] = v;
  __syncthreads();
  if (threadIdx.x == 0 && threadIdx.y == 0) {
    double t = 0.0;
    for (int k = 0; k < 8; ++k) t += warp_sums[k];
    part[blockIdx.x + gridDim.x * (blockIdx.y + gridDim.y * blockIdx.z)] = t;
  }
}

FX_DEV double resid_sq(float xp, float xm, float yp, float ym, float zp, float zm, float c, float rh) {
  const double s = (double)xp + (double)xm + (double)yp + (double)ym + (double)zp + (double)zm;
  const double r = (double)rh - (s - 6.0 * (double)c);
  return r * r;
}

template <bool WEIGHTED, bool NORM = false>
__global__ void __launch_bounds__(256, 4) k_sweep_march(Dims dm, const float* __restrict__ div, const float* __restrict__ src,
                                                        float* __restrict__ dst, int run, float w, double* norm_part = nullptr) {
  double s2 = 0.0;
  [&]() {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (y >= dm.h || zb >= ze) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t base = (xin ? x0 : dm.w - 4) + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!yint) {
    if (xin)
      for (int z = zb; z < ze; ++z) dst4[(base + sz * (uint32_t)z) >> 2] = zero4;
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const int D = (int)dm.d;
  // Rows of the source at a plane, zero outside the grid (only the interior
  // planes 1..D-2 read them, and those reach 0..D-1).
  auto crow = [&](int z) { return (src && z >= 0 && z < D) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 cm = crow(zb - 1), c0 = crow(zb), cp = crow(zb + 1);
  // Plane zb's own rows; every later plane's are loaded one iteration ahead.
  const uint32_t i = base + sz * (uint32_t)zb;
  float4 dv = __ldg(div4 + (i >> 2));
  float4 yp = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
  float4 ym = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
  float xle = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
  float xre = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  for (int z = zb; z < ze; ++z) {
    // Loads for plane z + 1 (its z + 1 row is plane z + 2), clamped in range on
    // the last plane, whose values are then never used.
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    const float4 n_c = crow(z + 2);
    const float4 n_dv = __ldg(div4 + (in >> 2));
    const float4 n_yp = src ? __ldg(src4 + ((in + sy) >> 2)) : zero4;
    const float4 n_ym = src ? __ldg(src4 + ((in - sy) >> 2)) : zero4;
    const float n_xle = (src && left_end) ? __ldg(src + in - 1) : 0.0f;
    const float n_xre = (src && right_end) ? __ldg(src + in + 4) : 0.0f;
    float left = __shfl_up_sync(0xffffffffu, c0.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, c0.x, 1);  // x0 + 4
    if (left_end) left = xle;
    if (right_end) right = xre;
    if (xin) {
      float4 v = zero4;
      if (z > 0 && z < D - 1) {
        if (src) {
          if (int0) v.x = div6(c0.y + left + yp.x + ym.x + cp.x + cm.x - dv.x);
          v.y = div6(c0.z + c0.x + yp.y + ym.y + cp.y + cm.y - dv.y);
          v.z = div6(c0.w + c0.y + yp.z + ym.z + cp.z + cm.z - dv.z);
          if (int3) v.w = div6(right + c0.z + yp.w + ym.w + cp.w + cm.w - dv.w);
        } else {
          if (int0) v.x = div6(0.0f - dv.x);
          v.y = div6(0.0f - dv.y);
          v.z = div6(0.0f - dv.z);
          if (int3) v.w = div6(0.0f - dv.w);
        }
        if (WEIGHTED) {
          if (int0) v.x = c0.x + w * (v.x - c0.x);
          v.y = c0.y + w * (v.y - c0.y);
          v.z = c0.z + w * (v.z - c0.z);
          if (int3) v.w = c0.w + w * (v.w - c0.w);
        }
        if (NORM) {
          if (int0) s2 += resid_sq(c0.y, left, yp.x, ym.x, cp.x, cm.x, c0.x, dv.x);
          s2 += resid_sq(c0.z, c0.x, yp.y, ym.y, cp.y, cm.y, c0.y, dv.y);
          s2 += resid_sq(c0.w, c0.y, yp.z, ym.z, cp.z, cm.z, c0.z, dv.z);
          if (int3) s2 += resid_sq(right, c0.z, yp.w, ym.w, cp.w, cm.w, c0.w, dv.w);
        }
      }
      dst4[(base + sz * (uint32_t)z) >> 2] = v;
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
  }();
  if constexpr (NORM) block_sum_double(s2, norm_part);
}

// k_sweep_march with the prolongation of mid_p added (the first fine post-sweep),
// for even fine grids with widths divisible by 4 whose mid level is exactly half
// their size. There, at an interior fine voxel, prolong_sample's position
// ((c + 0.5) * 0.5 - 0.5 per axis) needs no clamp, its corners are mid cells
// (c - 1) >> 1 and one more, and its weights are exactly 0.75 for even c and
// 0.25 for odd c. A thread's four x then read mid columns x0/2 - 1 .. x0/2 + 2 of
// two mid rows, and consecutive fine planes share mid planes: the kernel holds
// the two mid planes of the current fine plane (8 values each: a float2 load
// per row, the outer columns by warp shuffle) and loads the next one, from L2,
// when fine z reaches it. Each sample is tri_interp's mix of the same corner values with the
// same weights in the same order, so the results are the same bits.
__global__ void __launch_bounds__(256, 3) k_sweep_march_prolong(Dims dm, const float* __restrict__ div, const float* __restrict__ src,
                                                                float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p, int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (y >= dm.h || zb >= ze) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t xb = xin ? x0 : dm.w - 4;
  const uint32_t base = xb + dm.w * y;
  const bool yint = y > 0 && y < dm.h - 1;
  const float4* __restrict__ src4 = reinterpret_cast<const float4*>(src);
  const float4* __restrict__ div4 = reinterpret_cast<const float4*>(div);
  float4* __restrict__ dst4 = reinterpret_cast<float4*>(dst);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  if (!yint) {
    if (xin)
      for (int z = zb; z < ze; ++z) dst4[(base + sz * (uint32_t)z) >> 2] = zero4;
    return;
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;  // x0 + 1 and x0 + 2 are always interior
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const int D = (int)dm.d;
  // mid rows and row weight of this fine row (interior, so unclamped)
  const uint32_t mc = xb >> 1;  // even; the thread's mid columns are mc - 1 .. mc + 2
  const uint32_t mby = (y - 1u) >> 1, muy = mby + 1u;
  const float fy = (y & 1u) ? 0.25f : 0.75f;
  const float2* __restrict__ mid2 = reinterpret_cast<const float2*>(mid_p);
  // Raw loads of one mid plane: the float2 (mc, mc + 1) of each row, and at the
  // row ends of the warp the outer column the shuffle cannot bring.
  struct Raw {
    float2 r0, r1;
    float l0, l1, q0, q1;
  };
  auto mid_raw = [&](int pz) {
    Raw o;
    const uint32_t pc = (uint32_t)max(0, min(pz, (int)mid.d - 1));
    const uint32_t i0 = mc + mid.w * (mby + mid.h * pc), i1 = mc + mid.w * (muy + mid.h * pc);
    o.r0 = __ldg(mid2 + (i0 >> 1));
    o.r1 = __ldg(mid2 + (i1 >> 1));
    o.l0 = left_end ? __ldg(mid_p + i0 - 1) : 0.0f;
    o.l1 = left_end ? __ldg(mid_p + i1 - 1) : 0.0f;
    o.q0 = right_end ? __ldg(mid_p + i0 + 2) : 0.0f;
    o.q1 = right_end ? __ldg(mid_p + i1 + 2) : 0.0f;
    return o;
  };
  // The 8 values of a mid plane: [row][column mc - 1 + k]
  struct Plane {
    float v[2][4];
  };
  auto expand = [&](const Raw& r) {
    Plane p;
    float a = __shfl_up_sync(0xffffffffu, r.r0.y, 1), b = __shfl_down_sync(0xffffffffu, r.r0.x, 1);
    float c = __shfl_up_sync(0xffffffffu, r.r1.y, 1), d = __shfl_down_sync(0xffffffffu, r.r1.x, 1);
    if (left_end) {
      a = r.l0;
      c = r.l1;
    }
    if (right_end) {
      b = r.q0;
      d = r.q1;
    }
    p.v[0][0] = a;
    p.v[0][1] = r.r0.x;
    p.v[0][2] = r.r0.y;
    p.v[0][3] = b;
    p.v[1][0] = c;
    p.v[1][1] = r.r1.x;
    p.v[1][2] = r.r1.y;
    p.v[1][3] = d;
    return p;
  };
  // tri_interp over mid columns (k, k + 1) of planes A (z corner b) and B (u)
  auto sample = [&](const Plane& A, const Plane& B, int k, float fx, float fz) {
    const float x00 = mixv(A.v[0][k], A.v[0][k + 1], fx);
    const float x10 = mixv(A.v[1][k], A.v[1][k + 1], fx);
    const float x01 = mixv(B.v[0][k], B.v[0][k + 1], fx);
    const float x11 = mixv(B.v[1][k], B.v[1][k + 1], fx);
    return mixv(mixv(x00, x10, fy), mixv(x01, x11, fy), fz);
  };
  int cbz = (zb - 1) >> 1;  // the mid plane held in A (B holds cbz + 1)
  Plane A = expand(mid_raw(cbz)), B = expand(mid_raw(cbz + 1));

  auto crow = [&](int z) { return (src && z >= 0 && z < D) ? __ldg(src4 + ((base + sz * (uint32_t)z) >> 2)) : zero4; };
  float4 cm = crow(zb - 1), c0 = crow(zb), cp = crow(zb + 1);
  const uint32_t i = base + sz * (uint32_t)zb;
  float4 dv = __ldg(div4 + (i >> 2));
  float4 yp = src ? __ldg(src4 + ((i + sy) >> 2)) : zero4;
  float4 ym = src ? __ldg(src4 + ((i - sy) >> 2)) : zero4;
  float xle = (src && left_end) ? __ldg(src + i - 1) : 0.0f;
  float xre = (src && right_end) ? __ldg(src + i + 4) : 0.0f;
  for (int z = zb; z < ze; ++z) {
    const int bz = (z - 1) >> 1;
    if (bz != cbz) {  // warp-uniform: fine z moved on to the next mid plane pair (an L2 hit)
      A = B;
      cbz = bz;
      B = expand(mid_raw(cbz + 1));
    }
    const int zn = min(z + 1, D - 1);
    const uint32_t in = base + sz * (uint32_t)zn;
    const float4 n_c = crow(z + 2);
    const float4 n_dv = __ldg(div4 + (in >> 2));
    const float4 n_yp = src ? __ldg(src4 + ((in + sy) >> 2)) : zero4;
    const float4 n_ym = src ? __ldg(src4 + ((in - sy) >> 2)) : zero4;
    const float n_xle = (src && left_end) ? __ldg(src + in - 1) : 0.0f;
    const float n_xre = (src && right_end) ? __ldg(src + in + 4) : 0.0f;
    float left = __shfl_up_sync(0xffffffffu, c0.w, 1);     // x0 - 1
    float right = __shfl_down_sync(0xffffffffu, c0.x, 1);  // x0 + 4
    if (left_end) left = xle;
    if (right_end) right = xre;
    if (xin) {
      float4 v = zero4;
      if (z > 0 && z < D - 1) {
        if (src) {
          if (int0) v.x = div6(c0.y + left + yp.x + ym.x + cp.x + cm.x - dv.x);
          v.y = div6(c0.z + c0.x + yp.y + ym.y + cp.y + cm.y - dv.y);
          v.z = div6(c0.w + c0.y + yp.z + ym.z + cp.z + cm.z - dv.z);
          if (int3) v.w = div6(right + c0.z + yp.w + ym.w + cp.w + cm.w - dv.w);
        } else {
          if (int0) v.x = div6(0.0f - dv.x);
          v.y = div6(0.0f - dv.y);
          v.z = div6(0.0f - dv.z);
          if (int3) v.w = div6(0.0f - dv.w);
        }
        const float fz = (z & 1) ? 0.25f : 0.75f;
        if (int0) v.x = v.x + sample(A, B, 0, 0.75f, fz);
        v.y = v.y + sample(A, B, 1, 0.25f, fz);
        v.z = v.z + sample(A, B, 1, 0.75f, fz);
        if (int3) v.w = v.w + sample(A, B, 2, 0.25f, fz);
      }
      dst4[(base + sz * (uint32_t)z) >> 2] = v;
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

// The cleared buffer plus the prolongation (finePre = 0): boundary 0, interior 0 + sample.
__global__ void __launch_bounds__(256) k_prolong_zero(Dims dm, float* __restrict__ dst, Dims mid, const float* __restrict__ mid_p) {
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 4 + threadIdx.y, z = blockIdx.z * 2 + threadIdx.z;
  if (x >= dm.w || y >= dm.h || z >= dm.d) return;
  const uint32_t i = flat(dm, x, y, z);
  dst[i] = is_boundary(dm, x, y, z) ? 0.0f : 0.0f + prolong_sample(mid, mid_p, (int)x, (int)y, (int)z);
}

inline dim3 lean_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 3) / 4, (d.d + 1) / 2); }

__global__ void k_div6_check(uint32_t hi_base, unsigned long long* bad) {
  const uint32_t u = hi_base + blockIdx.x * blockDim.x + threadIdx.x;
  const float x = __uint_as_float(u);
  if (x != x) return;
  const float a = div6(x), b = x / 6.0f;
  if (__float_as_uint(a) != __float_as_uint(b)) atomicAdd(bad, 1ull);
}

}  // namespace

// k_div_march where the grid allows it (FENIX_DIV_MARCH=0 keeps k_div_first):
// widths divisible by 4, even heights and depths. Runs of an even number of
// planes such that the row tiles times the runs fill the resident blocks once.
cudaError_t lean_div_first(cudaStream_t s, Dims dm, VelField v, float* div, float* p1, Dims mid, float* mid_div, bool restrict_mid) {
  static const int march = env_int("FENIX_DIV_MARCH", 1, 0, 1);
  if (march && dm.w % 4 == 0 && dm.w >= 8 && dm.h % 2 == 0 && dm.d % 2 == 0) {
    static int slots[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
    if (n <= 0) {
      int per_sm = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_div_march, 256, 0);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      n = std::max(1, per_sm) * std::max(1, sms);
      if (dev >= 0 && dev < 64) slots[dev] = n;
    }
    const int run = march_plan_pairs(dm, n);
    const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
    k_div_march<<<g, dim3(32, 8, 1), 0, s>>>(dm, v, div, p1, mid, mid_div, restrict_mid ? 1 : 0, run);
    return cudaGetLastError();
  }
  k_div_first<<<lean_grid(dm), dim3(32, 4, 2), 0, s>>>(dm, v, div, p1, mid, mid_div, restrict_mid ? 1 : 0);
  return cudaGetLastError();
}

bool sweep_variant_valid(int variant, Dims dm) {
  if (variant < 0 || variant >= kSweepVariants) return false;
  if (variant >= SWEEP_VEC4_Z2) return dm.w % 4 == 0 && dm.w >= 8;
  return variant < SWEEP_VEC_Z2 || (dm.w % 2 == 0 && dm.w >= 4);
}

int march_plan_one_wave(Dims dm, int slots) {
  const int tiles = (int)(((dm.w + 127) / 128) * ((dm.h + 7) / 8));
  const int runs = std::max(1, std::min((int)dm.d, std::max(slots, 1) / std::max(tiles, 1)));
  return ((int)dm.d + runs - 1) / runs;
}

int march_plan_pairs(Dims dm, int slots) {
  const int tiles = (int)(((dm.w + 127) / 128) * ((dm.h + 7) / 8));
  const int pairs = std::max(1, (int)dm.d / 2);
  const int runs = std::max(1, std::min(pairs, std::max(slots, 1) / std::max(tiles, 1)));
  return 2 * ((pairs + runs - 1) / runs);
}

int march_plan_waves(Dims dm, int tx, int ty, int slots) {
  const long n = std::max(slots, 1);
  const long tiles = (long)((dm.w + tx - 1) / tx) * (long)((dm.h + ty - 1) / ty);
  int best = 1;
  double best_eff = -1.0;
  for (int r = 1; r <= std::max(1, (int)dm.d / 8); ++r) {
    const int len = ((int)dm.d + r - 1) / r;
    const int runs = ((int)dm.d + len - 1) / len;
    const long blocks = tiles * runs;
    const long waves = (blocks + n - 1) / n;
    const double eff = (double)blocks / (double)(waves * n);
    if (eff > best_eff + 1e-9) {
      best_eff = eff;
      best = len;
    }
  }
  return best;
}

static cudaError_t march_run(Dims dm, int* run, int slot_pct = 100);

// The variant used when none was chosen: four x per thread marching in z where
// the width allows and a thread marches at least 8 planes (the 256^3 level of
// plume_256, 39.8 against 49.8 us per sweep), else four x per thread at z-depth
// 2 where the width allows (on the 128^3 and 64^3 levels the marching kernel
// gets 4 and 1 planes per thread and ties with it), else two x, else one.
// FENIX_SWEEP_VEC (0, 1, 2) caps the x per thread at 1, 2 or 4, and 2 also
// leaves out the marching kernel.
int sweep_variant_default(Dims dm) {
  static const int zb = env_int("FENIX_SWEEP_ZB", 4, 1, 8);
  static const int vec = env_int("FENIX_SWEEP_VEC", 3, 0, 3);
  static const int vzb = env_int("FENIX_SWEEP_VEC_ZB", 2, 2, 4);
  int run = 0;
  if (vec >= 3 && sweep_variant_valid(SWEEP_VEC4_MARCH, dm) && march_run(dm, &run) == cudaSuccess && run >= 8) return SWEEP_VEC4_MARCH;
  if (vec >= 2 && sweep_variant_valid(SWEEP_VEC4_Z2, dm)) return vzb <= 2 ? SWEEP_VEC4_Z2 : SWEEP_VEC4_Z4;
  if (vec >= 1 && sweep_variant_valid(SWEEP_VEC_Z2, dm)) return vzb <= 2 ? SWEEP_VEC_Z2 : SWEEP_VEC_Z4;
  return zb <= 2 ? SWEEP_Z2 : (zb <= 4 ? SWEEP_Z4 : SWEEP_Z8);
}

// Resident blocks of k_sweep_march on the current device (SMs x blocks per SM),
// looked up once per device.
static cudaError_t march_slots(int* slots) {
  static int cached[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && cached[dev] > 0) {
    *slots = cached[dev];
    return cudaSuccess;
  }
  int per_sm = 0, sms = 0;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_march<false>, 256, 0);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  *slots = std::max(1, per_sm) * std::max(1, sms);
  if (dev >= 0 && dev < 64) cached[dev] = *slots;
  return cudaSuccess;
}

// Planes per thread of k_sweep_march on a level: runs of planes such that the
// row tiles times the runs fill the resident slots once.
static cudaError_t march_run(Dims dm, int* run, int slot_pct) {
  int slots = 0;
  const cudaError_t e = march_slots(&slots);
  if (e != cudaSuccess) return e;
  *run = march_plan_one_wave(dm, std::max(1, slots * slot_pct / 100));
  return cudaSuccess;
}

// march_run for another marching kernel of 256-thread blocks over 128 x 8 row
// tiles (its own resident blocks, looked up once per device).
template <typename K>
static cudaError_t march_run_of(K kernel, Dims dm, int* run) {
  static int cached[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int slots = (dev >= 0 && dev < 64) ? cached[dev] : 0;
  if (slots <= 0) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    slots = std::max(1, per_sm) * std::max(1, sms);
    if (dev >= 0 && dev < 64) cached[dev] = slots;
  }
  *run = march_plan_one_wave(dm, slots);
  return cudaSuccess;
}

int march_share_pct() {
  static const int pct = env_int("FENIX_MARCH_SHARE", 50, 10, 100);
  return pct;
}

cudaError_t lean_sweep_variant(cudaStream_t s, int variant, Dims dm, const float* div, const float* src, float* dst, Dims mid,
                               const float* mid_p, int slot_pct) {
  if (!sweep_variant_valid(variant, dm)) variant = sweep_variant_default(dm);
  auto grid = [&](int x_per_block, int z) { return dim3((dm.w + x_per_block - 1) / x_per_block, (dm.h + 7) / 8, (dm.d + z - 1) / z); };
  const dim3 block(32, 8, 1);
  switch (variant) {
    case SWEEP_Z2: k_sweep<2><<<grid(32, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_Z4: k_sweep<4><<<grid(32, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_Z8: k_sweep<8><<<grid(32, 8), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC_Z2: k_sweep_v2<2><<<grid(64, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC_Z4: k_sweep_v2<4><<<grid(64, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z2: k_sweep_v4<2><<<grid(128, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z4: k_sweep_v4<4><<<grid(128, 4), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    case SWEEP_VEC4_Z1: k_sweep_v4<1><<<grid(128, 1), block, 0, s>>>(dm, div, src, dst, mid, mid_p); break;
    default: {
      int run = 0;
      const cudaError_t e = march_run(dm, &run, slot_pct);
      if (e != cudaSuccess) return e;
      // FENIX_PROLONG_MARCH=0 keeps k_sweep_v4<2> for the sweep with the prolongation
      static const bool prolong_march = env_int("FENIX_PROLONG_MARCH", 1, 0, 1) == 1;
      int prun = 0;
      const bool pm_ok = mid_p && dm.h % 2 == 0 && dm.d % 2 == 0 && mid.w * 2 == dm.w && mid.h * 2 == dm.h && mid.d * 2 == dm.d;
      if (pm_ok && prolong_march && march_run_of(k_sweep_march_prolong, dm, &prun) == cudaSuccess) {
        const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + prun - 1) / prun);
        k_sweep_march_prolong<<<g, block, 0, s>>>(dm, div, src, dst, mid, mid_p, prun);
      } else if (mid_p) {
        k_sweep_v4<2><<<grid(128, 2), block, 0, s>>>(dm, div, src, dst, mid, mid_p);
      } else {
        const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
        k_sweep_march<false><<<g, block, 0, s>>>(dm, div, src, dst, run, 1.0f);
      }
      break;
    }
  }
  return cudaGetLastError();
}

cudaError_t march_wsweep(cudaStream_t s, Dims dm, const float* rhs, const float* src, float* dst, float w, bool one) {
  if (dm.w % 4 != 0 || dm.w < 8 || !src) return cudaErrorNotSupported;
  static int slots[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
  if (n <= 0) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_march<true>, 256, 0);
    if (e != cudaSuccess) return e;
    n = std::max(1, per_sm) * device_sm_count();
    if (dev >= 0 && dev < 64) slots[dev] = n;
  }
  const int run = march_plan_one_wave(dm, n);
  const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
  if (one)
    k_sweep_march<false><<<g, dim3(32, 8, 1), 0, s>>>(dm, rhs, src, dst, run, 1.0f);
  else
    k_sweep_march<true><<<g, dim3(32, 8, 1), 0, s>>>(dm, rhs, src, dst, run, w);
  return cudaGetLastError();
}

cudaError_t march_wsweep_norm(cudaStream_t s, Dims dm, const float* rhs, const float* src, float* dst, float w, bool one,
                              double* part, int* nparts) {
  if (dm.w % 4 != 0 || dm.w < 8 || !src) return cudaErrorNotSupported;
  static int slots[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
  if (n <= 0) {
    int per_sm = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_sweep_march<true, true>, 256, 0);
    if (e != cudaSuccess) return e;
    n = std::max(1, per_sm) * device_sm_count();
    if (dev >= 0 && dev < 64) slots[dev] = n;
  }
  const int run = march_plan_one_wave(dm, n);
  const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
  if ((int)(g.x * g.y * g.z) > *nparts) return cudaErrorNotSupported;
  *nparts = (int)(g.x * g.y * g.z);
  if (one)
    k_sweep_march<false, true><<<g, dim3(32, 8, 1), 0, s>>>(dm, rhs, src, dst, run, 1.0f, part);
  else
    k_sweep_march<true, true><<<g, dim3(32, 8, 1), 0, s>>>(dm, rhs, src, dst, run, w, part);
  return cudaGetLastError();
}

cudaError_t lean_sweep(cudaStream_t s, Dims dm, const float* div, const float* src, float* dst, Dims mid, const float* mid_p) {
  return lean_sweep_variant(s, -1, dm, div, src, dst, mid, mid_p);
}

cudaError_t lean_prolong_zero(cudaStream_t s, Dims dm, float* dst, Dims mid, const float* mid_p) {
  k_prolong_zero<<<lean_grid(dm), dim3(32, 4, 2), 0, s>>>(dm, dst, mid, mid_p);
  return cudaGetLastError();
}

cudaError_t div6_exhaustive_check(unsigned long long* host_bad) {
  unsigned long long* d = nullptr;
  cudaError_t e = cudaMalloc(&d, sizeof(unsigned long long));
  if (e != cudaSuccess) return e;
  cudaMemset(d, 0, sizeof(unsigned long long));
  // 2^32 inputs in 256 launches of 2^24 (65536 blocks of 256 threads)
  for (uint32_t k = 0; k < 256; ++k) k_div6_check<<<65536, 256>>>(k << 24, d);
  e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaMemcpy(host_bad, d, sizeof(unsigned long long), cudaMemcpyDeviceToHost);
  cudaFree(d);
  return e;
}

}  // namespace fx
