// Fused kernel path (see fx_fused.h).
//
// The step is the reference's (runtime/createCombustionVolumeSimulation.ts:270-301)
// with the same per-voxel arithmetic as the plain path, reorganised for B200:
//  - Injection visits only the bricks that intersect an emitter's reach (host-culled
//    list). The reference clamps the whole velocity field to +-80/dx inside its
//    velocity-injection pass (inject-velocity.wgsl.ts:94-95); the only reader of
//    that field before projection rewrites it is velocity advection, so the clamp
//    is applied there, on every value read, which gives identical results.
//  - Brick flags (compute-active-bricks.wgsl.ts) are built from per-brick summaries
//    (bit 0: a sample is above 0.012, bit 1: the brick dilates) that the kernels
//    writing a scalar set emit as a by-product, then dilated in gather form:
//    flag[b] = active[b] OR any neighbour n (Chebyshev distance 1) with
//    active[n] AND dilate[n]. That is the reference's clamped scatter.
//  - Scalar advection, combustion and buoyancy run over compacted brick lists.
//    Per-brick "may be non-zero" bits of each scalar buffer let the kernels skip
//    bricks that are already zero where the reference rewrites zeros.
//  - Combustion writes the next set from the advected scratch set, so every
//    neighbour read sees the state before the pass.
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <vector>

#include <cuda_fp16.h>

#include "fx_fused.h"
#include "fx_pressure.h"

namespace fx {
namespace {

inline size_t align256(size_t b) { return (b + 255) & ~(size_t)255; }

constexpr int kBrickThreads = 256;

// ------------------------------------------------------------- scalar storage
// The scalar sets (density, temperature, fuel, reaction) are stored as float or,
// with FP16 storage, as binary16. The kernels compute in f32 either way. Each
// value the reference stores into one of those buffers goes through qS_at first
// (round to the storage type and back), so everything read afterwards (the
// brick summaries, the non-zero bits, later fields) sees the stored value.
template <typename S>
struct SSet {
  S* f[4];
};

template <typename S>
SSet<S> sset(const ScalarSet& s) {
  SSet<S> o;
  for (int k = 0; k < 4; ++k) o.f[k] = reinterpret_cast<S*>(s.f[k]);
  return o;
}

FX_DEV float ldS(const float* p, uint32_t i) { return __ldg(p + i); }
FX_DEV float ldS(const __half* p, uint32_t i) { return __half2float(__ldg(p + i)); }
FX_DEV float rdS(const float* p, uint32_t i) { return p[i]; }
FX_DEV float rdS(const __half* p, uint32_t i) { return __half2float(p[i]); }
FX_DEV void stS(float* p, uint32_t i, float v) { p[i] = v; }
FX_DEV void stS(__half* p, uint32_t i, float v) { p[i] = __float2half_rn(v); }

// The value a pass stores for voxel i at store site `site` (numbered as the
// oracle's Sim::qs_at): itself in f32 storage; in binary16 storage rounded to
// nearest, or stochastically (sr_half) when the step's uniform asks for it.
template <typename S>
FX_DEV float qS_at(float v, const Params& P, uint32_t i, uint32_t site);
template <>
FX_DEV float qS_at<float>(float v, const Params&, uint32_t, uint32_t) {
  return v;
}
template <>
FX_DEV float qS_at<__half>(float v, const Params& P, uint32_t i, uint32_t site) {
  return P.half_round ? sr_half(v, sr_draw(i, site, P.step_index)) : __half2float(__float2half_rn(v));
}

// tri_interp (sampling-scalar.wgsl.ts:11-34) over a stored scalar field.
template <typename S>
FX_DEV float tri_interp_s(const S* __restrict__ f, const Tri& c) {
  const float x00 = mixv(ldS(f, c.i000), ldS(f, c.i100), c.fx);
  const float x10 = mixv(ldS(f, c.i010), ldS(f, c.i110), c.fx);
  const float x01 = mixv(ldS(f, c.i001), ldS(f, c.i101), c.fx);
  const float x11 = mixv(ldS(f, c.i011), ldS(f, c.i111), c.fx);
  return mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
}

// The interleaved copy of a scalar set: per voxel (d, t, f, r) as a float4, or
// as four binary16 values in a uint2 (d and t in .x, f and r in .y, low half
// first).
template <typename S>
struct Aos;
template <>
struct Aos<float> {
  using T = float4;
  static FX_DEV T pack(const SSet<float>& s, uint32_t i) {
    return make_float4(__ldg(s.f[0] + i), __ldg(s.f[1] + i), __ldg(s.f[2] + i), __ldg(s.f[3] + i));
  }
  static FX_DEV T zero() { return make_float4(0.f, 0.f, 0.f, 0.f); }
  static FX_DEV void unpack(const T* __restrict__ a, uint32_t i, float (&o)[4]) {
    const float4 v = __ldg(a + i);
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
    o[3] = v.w;
  }
};
template <>
struct Aos<__half> {
  using T = uint2;
  static FX_DEV T pack(const SSet<__half>& s, uint32_t i) {
    const uint32_t d = __half_as_ushort(__ldg(s.f[0] + i)), t = __half_as_ushort(__ldg(s.f[1] + i));
    const uint32_t f = __half_as_ushort(__ldg(s.f[2] + i)), r = __half_as_ushort(__ldg(s.f[3] + i));
    return make_uint2(d | (t << 16), f | (r << 16));
  }
  static FX_DEV T zero() { return make_uint2(0u, 0u); }
  static FX_DEV void unpack(const T* __restrict__ a, uint32_t i, float (&o)[4]) {
    const uint2 v = __ldg(a + i);
    o[0] = __half2float(__ushort_as_half((unsigned short)(v.x & 0xFFFFu)));
    o[1] = __half2float(__ushort_as_half((unsigned short)(v.x >> 16)));
    o[2] = __half2float(__ushort_as_half((unsigned short)(v.y & 0xFFFFu)));
    o[3] = __half2float(__ushort_as_half((unsigned short)(v.y >> 16)));
  }
};

// tri_interp_s of all four fields at once from the interleaved copy: the same
// corner values, mixed per field in tri_interp's order.
template <typename S>
FX_DEV void tri_interp_aos(const typename Aos<S>::T* __restrict__ a, const Tri& c, float (&out)[4]) {
  float v000[4], v100[4], v010[4], v110[4], v001[4], v101[4], v011[4], v111[4];
  Aos<S>::unpack(a, c.i000, v000);
  Aos<S>::unpack(a, c.i100, v100);
  Aos<S>::unpack(a, c.i010, v010);
  Aos<S>::unpack(a, c.i110, v110);
  Aos<S>::unpack(a, c.i001, v001);
  Aos<S>::unpack(a, c.i101, v101);
  Aos<S>::unpack(a, c.i011, v011);
  Aos<S>::unpack(a, c.i111, v111);
#pragma unroll
  for (int f = 0; f < 4; ++f) {
    const float x00 = mixv(v000[f], v100[f], c.fx);
    const float x10 = mixv(v010[f], v110[f], c.fx);
    const float x01 = mixv(v001[f], v101[f], c.fx);
    const float x11 = mixv(v011[f], v111[f], c.fx);
    out[f] = mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
  }
}

// Calls f(tag) where decltype(tag)::type is the storage type (float or __half).
template <typename S>
struct StorageTag {
  using type = S;
};
template <typename F>
void by_storage(bool half, F&& f) {
  if (half) f(StorageTag<__half>{});
  else f(StorageTag<float>{});
}

__global__ void k_count_flags(const uint32_t* __restrict__ flags, uint32_t nb, uint32_t* __restrict__ out) {
  uint32_t local = 0;
  for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < nb; i += gridDim.x * blockDim.x) local += flags[i] != 0u;
  for (int o = 16; o > 0; o >>= 1) local += __shfl_down_sync(0xffffffffu, local, o);
  if ((threadIdx.x & 31) == 0 && local) atomicAdd(out, local);
}

// One thread per brick; block-level sums, one atomic pair per block.
__global__ void k_accumulate_active(Dims dm, uint3 bc, const uint32_t* __restrict__ flags, unsigned long long* __restrict__ acc) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  unsigned long long bricks = 0, voxels = 0;
  for (uint32_t b = blockIdx.x * blockDim.x + threadIdx.x; b < nb; b += gridDim.x * blockDim.x) {
    if (flags[b] == 0u) continue;
    const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
    const uint32_t ex = min(8u, dm.w - 8u * bx), ey = min(8u, dm.h - 8u * by), ez = min(8u, dm.d - 8u * bz);
    bricks += 1;
    voxels += (unsigned long long)ex * ey * ez;
  }
  for (int o = 16; o > 0; o >>= 1) {
    bricks += __shfl_down_sync(0xffffffffu, bricks, o);
    voxels += __shfl_down_sync(0xffffffffu, voxels, o);
  }
  __shared__ unsigned long long sb[32], sv[32];
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  if (lane == 0) {
    sb[warp] = bricks;
    sv[warp] = voxels;
  }
  __syncthreads();
  if (warp == 0) {
    const int nw = blockDim.x >> 5;
    bricks = lane < nw ? sb[lane] : 0;
    voxels = lane < nw ? sv[lane] : 0;
    for (int o = 16; o > 0; o >>= 1) {
      bricks += __shfl_down_sync(0xffffffffu, bricks, o);
      voxels += __shfl_down_sync(0xffffffffu, voxels, o);
    }
    if (lane == 0 && bricks) {
      atomicAdd(acc, bricks);
      atomicAdd(acc + 1, voxels);
    }
  }
}

// The six neighbours of voxel (x, y, z) at flat index i, clamped as the
// reference's inc/dec (clamp-utils.wgsl.ts:12-22): i -+ 1, i -+ sy, i -+ sz, or
// i itself at the grid edge.
struct Nbr {
  uint32_t xp, xm, yp, ym, zp, zm;
};

FX_DEV Nbr neighbours(const Dims& dm, uint32_t x, uint32_t y, uint32_t z, uint32_t i) {
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  Nbr n;
  n.xp = x + 1u < dm.w ? i + 1u : i;
  n.xm = x > 0u ? i - 1u : i;
  n.yp = y + 1u < dm.h ? i + sy : i;
  n.ym = y > 0u ? i - sy : i;
  n.zp = z + 1u < dm.d ? i + sz : i;
  n.zm = z > 0u ? i - sz : i;
  return n;
}

// Brick geometry of a list entry and the two voxels each thread owns.
struct BrickCtx {
  uint32_t bx, by, bz;
  uint32_t x0, y0, z0;
  uint32_t cx, cy, cz;  // flag centre (compute-active-bricks.wgsl.ts:52)
};

FX_DEV BrickCtx brick_ctx(const Dims& dm, uint3 bc, uint32_t b) {
  BrickCtx c;
  c.bx = b % bc.x;
  c.by = (b / bc.x) % bc.y;
  c.bz = b / (bc.x * bc.y);
  c.x0 = c.bx * 8u;
  c.y0 = c.by * 8u;
  c.z0 = c.bz * 8u;
  c.cx = min(c.x0 + 4u, dm.w - 1u);
  c.cy = min(c.y0 + 4u, dm.h - 1u);
  c.cz = min(c.z0 + 4u, dm.d - 1u);
  return c;
}

// Sample-point test of compute-active-bricks.wgsl.ts:35-58 for one voxel of a
// brick: local coordinates all even are samples, plus the brick's flag centre.
struct Energy {
  bool over_active;  // some sample or the centre > 0.012
  bool over_peak;    // peak > 0.05 (over samples and centre)
  bool center_hot;   // centre > 0.035
};

FX_DEV void energy_vote(const BrickCtx& c, uint32_t x, uint32_t y, uint32_t z, bool inside, float d, float t, float r, Energy& e) {
  if (!inside) return;
  const bool sample = ((x - c.x0) & 1u) == 0u && ((y - c.y0) & 1u) == 0u && ((z - c.z0) & 1u) == 0u;
  const bool center = x == c.cx && y == c.cy && z == c.cz;
  if (!sample && !center) return;
  const float en = d + t * 0.7f + r * 0.9f;
  if (en > 0.012f) e.over_active = true;
  if (en > 0.05f) e.over_peak = true;
  if (center && en > 0.035f) e.center_hot = true;
}

// Block-wide OR of the votes into the brick summary (bit 0 active, bit 1 dilate).
FX_DEV uint8_t summary_of(const Energy& e) {
  const int a = __syncthreads_or(e.over_active ? 1 : 0);
  const int p = __syncthreads_or(e.over_peak ? 1 : 0);
  const int h = __syncthreads_or(e.center_hot ? 1 : 0);
  if (!a) return 0;
  return (uint8_t)(1u | ((p || h) ? 2u : 0u));
}

// ------------------------------------------------------------------ injection
template <typename S>
__global__ void __launch_bounds__(kBrickThreads) k_inject(Dims dm, uint3 bc, const Params* __restrict__ Pp, const float* __restrict__ src,
                                                          uint32_t nsrc, const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                                          SSet<S> set, VelField v, uint8_t* __restrict__ summary, uint8_t* __restrict__ nz,
                                                          float* __restrict__ tape_t1, float* __restrict__ tape_r1) {
  const Params P = *Pp;
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t b = list[li];
    const BrickCtx c = brick_ctx(dm, bc, b);
    Energy e{false, false, false};
    bool any = false;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t lv = threadIdx.x + kBrickThreads * j;
      const uint32_t x = c.x0 + (lv & 7u), y = c.y0 + ((lv >> 3) & 7u), z = c.z0 + (lv >> 6);
      const bool inside = x < dm.w && y < dm.h && z < dm.d;
      float d = 0.f, t = 0.f, f = 0.f, r = 0.f;
      if (inside) {
        const uint32_t i = flat(dm, x, y, z);
        const float px = ((float)x + 0.5f) / (float)dm.w, py = ((float)y + 0.5f) / (float)dm.h, pz = ((float)z + 0.5f) / (float)dm.d;
        d = rdS(set.f[0], i);
        t = rdS(set.f[1], i);
        f = rdS(set.f[2], i);
        r = rdS(set.f[3], i);
        inject_scalar_voxel(P, src, nsrc, px, py, pz, d, t, f);
        // inject-scalar stores d, T, f here; inject-igniter reads them back
        d = qS_at<S>(d, P, i, 0);
        t = qS_at<S>(t, P, i, 1);
        f = qS_at<S>(f, P, i, 2);
        if (tape_t1) {  // the rollout's tape: after the scalar injection, before the igniter
          tape_t1[i] = t;
          tape_r1[i] = r;
        }
        float vx = v.c[0][i], vy = v.c[1][i], vz = v.c[2][i];
        inject_velocity_voxel(P, src, nsrc, px, py, pz, vx, vy, vz);
        const float lim = speed_limit(P);
        v.c[0][i] = clampv(vx, -lim, lim);
        v.c[1][i] = clampv(vy, -lim, lim);
        v.c[2][i] = clampv(vz, -lim, lim);
        inject_igniter_voxel(P, src, nsrc, px, py, pz, f, r, t);
        r = qS_at<S>(r, P, i, 3);
        t = qS_at<S>(t, P, i, 4);
        stS(set.f[0], i, d);
        stS(set.f[1], i, t);
        stS(set.f[2], i, f);
        stS(set.f[3], i, r);
        any = any || d != 0.f || t != 0.f || f != 0.f || r != 0.f;
      }
      energy_vote(c, x, y, z, inside, d, t, r, e);
    }
    const uint8_t s = summary_of(e);
    const int nzb = __syncthreads_or(any ? 1 : 0);
    if (threadIdx.x == 0) {
      summary[b] = s;
      if (nzb) nz[b] = 1;
    }
  }
}

// ------------------------------------------------------------------- dilation
// flags[b] = active[b] || any neighbour within Chebyshev distance 1 that is
// active and dilates. Appends to `list` every brick with a flag or with any of
// the given "may be non-zero" bits set.
__global__ void k_dilate(uint3 bc, const uint8_t* __restrict__ summary, uint32_t* __restrict__ flags, const uint8_t* __restrict__ nz_a,
                         const uint8_t* __restrict__ nz_b, uint32_t* __restrict__ list, uint32_t* __restrict__ count) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  const uint32_t b = blockIdx.x * blockDim.x + threadIdx.x;
  bool take = false;
  if (b < nb) {
    const uint32_t bx = b % bc.x, by = (b / bc.x) % bc.y, bz = b / (bc.x * bc.y);
    bool flag = (summary[b] & 1u) != 0u;
    if (!flag) {
      const uint32_t zlo = bz ? bz - 1 : 0, zhi = min(bz + 1, bc.z - 1);
      const uint32_t ylo = by ? by - 1 : 0, yhi = min(by + 1, bc.y - 1);
      const uint32_t xlo = bx ? bx - 1 : 0, xhi = min(bx + 1, bc.x - 1);
      for (uint32_t z = zlo; z <= zhi && !flag; ++z)
        for (uint32_t y = ylo; y <= yhi && !flag; ++y)
          for (uint32_t x = xlo; x <= xhi; ++x)
            if (summary[x + bc.x * (y + bc.y * z)] == 3u) {
              flag = true;
              break;
            }
    }
    flags[b] = flag ? 1u : 0u;
    take = flag || (nz_a && nz_a[b]) || (nz_b && nz_b[b]);
  }
  const unsigned mask = __ballot_sync(0xffffffffu, take);
  if (mask) {
    const int lane = threadIdx.x & 31;
    uint32_t base = 0;
    if (lane == __ffs(mask) - 1) base = atomicAdd(count, (uint32_t)__popc(mask));
    base = __shfl_sync(0xffffffffu, base, __ffs(mask) - 1);
    if (take) list[base + __popc(mask & ((1u << lane) - 1u))] = b;
  }
}

FX_DEV bool flag_at(const uint32_t* __restrict__ flags, uint3 bc, uint32_t b) { return __ldg(flags + b) != 0u; }

// Planes per thread for a kernel of 256-thread blocks marching runs of z over
// tx x ty row tiles: the number of runs (at most one per 8 planes) that fills
// whole waves of the kernel's resident blocks best, the fewest runs among equals.
template <typename K>
cudaError_t march_runs(K kernel, Dims dm, int tx, int ty, int* run) {
  static int slots[64] = {};
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
  if (n <= 0) {
    int per_sm = 0, sms = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, 256, 0);
    if (e != cudaSuccess) return e;
    e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return e;
    n = std::max(1, per_sm) * std::max(1, sms);
    if (dev >= 0 && dev < 64) slots[dev] = n;
  }
  *run = march_plan_waves(dm, tx, ty, n);
  return cudaSuccess;
}

// ------------------------------------------------------------ velocity advection
// advect-velocity-semilagrangian.wgsl.ts:23-41 over vCurrent clamped to +-lim on read.
FX_DEV float tri_interp_clamped(const float* __restrict__ f, const Tri& c, float lim) {
  const float x00 = mixv(clampv(__ldg(f + c.i000), -lim, lim), clampv(__ldg(f + c.i100), -lim, lim), c.fx);
  const float x10 = mixv(clampv(__ldg(f + c.i010), -lim, lim), clampv(__ldg(f + c.i110), -lim, lim), c.fx);
  const float x01 = mixv(clampv(__ldg(f + c.i001), -lim, lim), clampv(__ldg(f + c.i101), -lim, lim), c.fx);
  const float x11 = mixv(clampv(__ldg(f + c.i011), -lim, lim), clampv(__ldg(f + c.i111), -lim, lim), c.fx);
  return mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
}

// The start sample of the back-trace sits on the voxel centre: every weight of
// the trilinear mix is 0, so the mix equals the voxel's own (clamped) value up to
// the sign of a zero, and c - v*dt comes out the same (c >= 0.5). For fields
// without NaN this reads one value instead of eight.
// Voxels per thread along z (one: measured fastest on the 256^3 plume, 170 against
// 179 us for four; FENIX_ADV_Z = 2, 4 or 8 selects the others, with the same bits).
constexpr int kAdvZ = 1;

// The clamp is the identity on every value when the largest |v| of the field is
// within the limit: `vmax` holds that bound (float bits, written by the
// projection that produced the field; all ones when unknown), and the kernel
// then reads the values as they are, with the same results.
template <bool CLAMP, int ZB>
FX_DEV void advect_velocity_column(Dims dm, uint32_t x, uint32_t y, uint32_t z0, float dt, float lim, float damp, bool xyint,
                                   const VelField& src, const VelField& dst) {
#pragma unroll
  for (int k = 0; k < ZB; ++k) {
    const uint32_t z = z0 + k;
    if (z >= dm.d) break;
    const uint32_t i = flat(dm, x, y, z);
    if (!xyint || z == 0 || z == dm.d - 1) {
      dst.c[0][i] = 0.0f;
      dst.c[1][i] = 0.0f;
      dst.c[2][i] = 0.0f;
      continue;
    }
    const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
    float v0x = __ldg(src.c[0] + i), v0y = __ldg(src.c[1] + i), v0z = __ldg(src.c[2] + i);
    if (CLAMP) {
      v0x = clampv(v0x, -lim, lim);
      v0y = clampv(v0y, -lim, lim);
      v0z = clampv(v0z, -lim, lim);
    }
    const float bx = cx - v0x * dt, by = cy - v0y * dt, bz = cz - v0z * dt;
    const Tri c1 = tri_corners(dm, bx - 0.5f, by - 0.5f, bz - 0.5f);
    if (CLAMP) {
      dst.c[0][i] = tri_interp_clamped(src.c[0], c1, lim) * damp;
      dst.c[1][i] = tri_interp_clamped(src.c[1], c1, lim) * damp;
      dst.c[2][i] = tri_interp_clamped(src.c[2], c1, lim) * damp;
    } else {
      dst.c[0][i] = tri_interp(src.c[0], c1) * damp;
      dst.c[1][i] = tri_interp(src.c[1], c1) * damp;
      dst.c[2][i] = tri_interp(src.c[2], c1) * damp;
    }
  }
}

template <int ZB>
__global__ void __launch_bounds__(256) k_advect_velocity(Dims dm, const Params* __restrict__ Pp, VelField src, VelField dst,
                                                         const unsigned* __restrict__ vmax) {
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * ZB;
  if (x >= dm.w || y >= dm.h) return;
  const float dt = Pp->dt;
  const float lim = speed_limit(*Pp);
  const float damp = 1.0f - dt * 0.025f;
  const bool xyint = x > 0 && y > 0 && x < dm.w - 1 && y < dm.h - 1;
  if (__uint_as_float(__ldg(vmax)) <= lim) advect_velocity_column<false, ZB>(dm, x, y, z0, dt, lim, damp, xyint, src, dst);
  else advect_velocity_column<true, ZB>(dm, x, y, z0, dt, lim, damp, xyint, src, dst);
}

// k_advect_velocity with each thread marching a run of z planes of one (x, y)
// column: the velocity at plane z + 1 (the start of its back-trace) is loaded
// before the 24 gathers of plane z are issued, so a voxel waits for one memory
// latency instead of two. Each voxel's back-trace, samples and damping are
// advect_velocity_column's, in the same order, so the results are the same bits.
template <bool CLAMP>
FX_DEV void advect_velocity_march(Dims dm, uint32_t x, uint32_t y, int zb, int ze, float dt, float lim, float damp, const VelField& src,
                                  const VelField& dst) {
  const uint32_t sz = dm.w * dm.h;
  const uint32_t base = x + dm.w * y;
  const int D = (int)dm.d;
  uint32_t i = base + sz * (uint32_t)zb;
  float v0x = __ldg(src.c[0] + i), v0y = __ldg(src.c[1] + i), v0z = __ldg(src.c[2] + i);
  for (int z = zb; z < ze; ++z) {
    const uint32_t in = base + sz * (uint32_t)min(z + 1, D - 1);
    const float nx = __ldg(src.c[0] + in), ny = __ldg(src.c[1] + in), nz = __ldg(src.c[2] + in);
    if (z == 0 || z == D - 1) {
      dst.c[0][i] = 0.0f;
      dst.c[1][i] = 0.0f;
      dst.c[2][i] = 0.0f;
    } else {
      const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
      float ax = v0x, ay = v0y, az = v0z;
      if (CLAMP) {
        ax = clampv(ax, -lim, lim);
        ay = clampv(ay, -lim, lim);
        az = clampv(az, -lim, lim);
      }
      const float bx = cx - ax * dt, by = cy - ay * dt, bz = cz - az * dt;
      const Tri c1 = tri_corners(dm, bx - 0.5f, by - 0.5f, bz - 0.5f);
      if (CLAMP) {
        dst.c[0][i] = tri_interp_clamped(src.c[0], c1, lim) * damp;
        dst.c[1][i] = tri_interp_clamped(src.c[1], c1, lim) * damp;
        dst.c[2][i] = tri_interp_clamped(src.c[2], c1, lim) * damp;
      } else {
        dst.c[0][i] = tri_interp(src.c[0], c1) * damp;
        dst.c[1][i] = tri_interp(src.c[1], c1) * damp;
        dst.c[2][i] = tri_interp(src.c[2], c1) * damp;
      }
    }
    v0x = nx;
    v0y = ny;
    v0z = nz;
    i = in;
  }
}

__global__ void __launch_bounds__(256) k_advect_velocity_march(Dims dm, const Params* __restrict__ Pp, VelField src, VelField dst,
                                                               const unsigned* __restrict__ vmax, int run) {
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y;
  const int zb = (int)blockIdx.z * run, ze = min(zb + run, (int)dm.d);
  if (x >= dm.w || y >= dm.h || zb >= ze) return;
  const float dt = Pp->dt;
  const float lim = speed_limit(*Pp);
  const float damp = 1.0f - dt * 0.025f;
  const bool xyint = x > 0 && y > 0 && x < dm.w - 1 && y < dm.h - 1;
  if (!xyint) {
    for (int z = zb; z < ze; ++z) {
      const uint32_t i = flat(dm, x, y, (uint32_t)z);
      dst.c[0][i] = 0.0f;
      dst.c[1][i] = 0.0f;
      dst.c[2][i] = 0.0f;
    }
    return;
  }
  if (__uint_as_float(__ldg(vmax)) <= lim) advect_velocity_march<false>(dm, x, y, zb, ze, dt, lim, damp, src, dst);
  else advect_velocity_march<true>(dm, x, y, zb, ze, dt, lim, damp, src, dst);
}

// ------------------------------------------------------------ interleaved copy
// Mirrors the current scalar set into the interleaved copy the scalar advection
// gathers from: every brick that may be non-zero in the set is packed, and every
// brick whose copy may still hold values of an earlier step is cleared; nz_aos
// then marks the bricks where the copy may be non-zero. Elsewhere the copy and
// the set are both zero, so the copy equals the set everywhere.
//
// One warp per brick; a lane packs two 8-voxel x rows. Where the width is a
// multiple of 8, a row of a field is one 16-byte load (binary16) or two (f32),
// and the row's interleaved values are 64 or 128 contiguous bytes.
template <typename S>
FX_DEV void pack_row(const SSet<S>& set, uint32_t i, uint32_t nx, bool live, bool vec, typename Aos<S>::T* __restrict__ aos) {
  using A = Aos<S>;
  if (vec) {
    if constexpr (sizeof(S) == 2) {
      uint4 out[4] = {};  // 8 voxels x 8 bytes
      if (live) {
        uint4 f[4];
#pragma unroll
        for (int k = 0; k < 4; ++k) f[k] = __ldg(reinterpret_cast<const uint4*>(set.f[k] + i));
        const uint32_t* d = reinterpret_cast<const uint32_t*>(&f[0]);
        const uint32_t* t = reinterpret_cast<const uint32_t*>(&f[1]);
        const uint32_t* fu = reinterpret_cast<const uint32_t*>(&f[2]);
        const uint32_t* r = reinterpret_cast<const uint32_t*>(&f[3]);
        uint32_t* o = reinterpret_cast<uint32_t*>(out);
#pragma unroll
        for (int v = 0; v < 8; ++v) {
          const int w = v >> 1, sh = (v & 1) * 16;
          const uint32_t dv = (d[w] >> sh) & 0xFFFFu, tv = (t[w] >> sh) & 0xFFFFu;
          const uint32_t fv = (fu[w] >> sh) & 0xFFFFu, rv = (r[w] >> sh) & 0xFFFFu;
          o[2 * v] = dv | (tv << 16);
          o[2 * v + 1] = fv | (rv << 16);
        }
      }
      uint4* dst = reinterpret_cast<uint4*>(aos + i);
#pragma unroll
      for (int k = 0; k < 4; ++k) dst[k] = out[k];
    } else {
      float4 out[8];
      if (live) {
        float4 f[4][2];
#pragma unroll
        for (int k = 0; k < 4; ++k) {
          f[k][0] = __ldg(reinterpret_cast<const float4*>(set.f[k] + i));
          f[k][1] = __ldg(reinterpret_cast<const float4*>(set.f[k] + i) + 1);
        }
        auto at = [&](int k, int v) {
          const float4 q = f[k][v >> 2];
          const int c = v & 3;
          return c == 0 ? q.x : c == 1 ? q.y : c == 2 ? q.z : q.w;
        };
#pragma unroll
        for (int v = 0; v < 8; ++v) out[v] = make_float4(at(0, v), at(1, v), at(2, v), at(3, v));
      } else {
#pragma unroll
        for (int v = 0; v < 8; ++v) out[v] = A::zero();
      }
      float4* dst = reinterpret_cast<float4*>(aos + i);
#pragma unroll
      for (int v = 0; v < 8; ++v) dst[v] = out[v];
    }
  } else {
    for (uint32_t v = 0; v < nx; ++v) aos[i + v] = live ? A::pack(set, i + v) : A::zero();
  }
}

template <typename S>
__global__ void __launch_bounds__(256) k_pack_aos(Dims dm, uint3 bc, SSet<S> set, const uint8_t* __restrict__ nz_set,
                                                  uint8_t* __restrict__ nz_aos, typename Aos<S>::T* __restrict__ aos) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  const uint32_t b = blockIdx.x * 8 + threadIdx.y;  // one warp per brick
  if (b >= nb) return;
  const bool live = __ldg(nz_set + b) != 0, stale = nz_aos[b] != 0;
  if (!live && !stale) return;  // the same for the whole warp
  const BrickCtx c = brick_ctx(dm, bc, b);
  const uint32_t nx = min(8u, dm.w - c.x0);
  const bool vec = nx == 8u && dm.w % 8u == 0u;
#pragma unroll
  for (int j = 0; j < 2; ++j) {
    const uint32_t row = threadIdx.x + 32u * j;  // 64 rows: y = row & 7, z = row >> 3
    const uint32_t y = c.y0 + (row & 7u), z = c.z0 + (row >> 3);
    if (y < dm.h && z < dm.d) pack_row<S>(set, flat(dm, c.x0, y, z), nx, live, vec, aos);
  }
  __syncwarp();  // every lane has read nz_aos[b] before it changes
  if (threadIdx.x == 0) nz_aos[b] = live ? 1 : 0;
}

// -------------------------------------------------------------- scalar advection
// advect-scalar-maccormack.wgsl.ts:33-101 / advect-scalar-semilagrangian.wgsl.ts
// over the bricks of list_adv: flagged bricks are advected into T, the others
// (T may hold old values there) are zeroed. Emits T's brick summary and non-zero bit.
template <typename S>
__global__ void __launch_bounds__(kBrickThreads) k_advect_scalars(Dims dm, uint3 bc, const Params* __restrict__ Pp, int mode,
                                                                  const typename Aos<S>::T* __restrict__ src, VelField vel,
                                                                  const uint32_t* __restrict__ flags,
                                                                  const uint32_t* __restrict__ list, const uint32_t* __restrict__ count,
                                                                  SSet<S> dst, uint8_t* __restrict__ summary, uint8_t* __restrict__ nz) {
  const Params P = *Pp;
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t b = list[li];
    const BrickCtx c = brick_ctx(dm, bc, b);
    const bool active = flag_at(flags, bc, b);
    Energy e{false, false, false};
    bool any = false;
    // the thread's two voxels share x and y (z and z + 4), hence the row weight
    // and the y-only sine of the thermal noise at the voxel centre
    const uint32_t x = c.x0 + (threadIdx.x & 7u), y = c.y0 + ((threadIdx.x >> 3) & 7u);
    float ny = 0.0f, ysin = 0.0f;
    if (active) {
      ny = ((float)y + 0.5f) / (float)dm.h;
      if (mode == 1) ysin = thermal_noise_ysin(P, (float)y + 0.5f);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t z = c.z0 + ((threadIdx.x + kBrickThreads * j) >> 6);
      const bool inside = x < dm.w && y < dm.h && z < dm.d;
      float out[4] = {0.f, 0.f, 0.f, 0.f};
      if (inside && active) {
        const float dt = P.dt;
        const float cx = (float)x + 0.5f, cy = (float)y + 0.5f, cz = (float)z + 0.5f;
        // Samples at the voxel centre (the back-trace start and `original`) equal the
        // voxel's values up to the sign of a zero, which neither c - v*dt nor the
        // max(0, .) of every output can see (NaN-free fields).
        const uint32_t ic = flat(dm, x, y, z);
        const float vx = __ldg(vel.c[0] + ic), vy = __ldg(vel.c[1] + ic), vz = __ldg(vel.c[2] + ic);
        const float bxp = cx - vx * dt, byp = cy - vy * dt, bzp = cz - vz * dt;
        const float spx = bxp - 0.5f, spy = byp - 0.5f, spz = bzp - 0.5f;
        const Tri cs = tri_corners(dm, spx, spy, spz);
        float noise;
        if (mode == 1) {
          const float fvx = tri_interp(vel.c[0], cs), fvy = tri_interp(vel.c[1], cs), fvz = tri_interp(vel.c[2], cs);
          const float rx = bxp + fvx * dt, ry = byp + fvy * dt, rz = bzp + fvz * dt;
          const Tri cr = tri_corners(dm, rx - 0.5f, ry - 0.5f, rz - 0.5f);
          float predicted[4], recovered[4], original[4];
          tri_interp_aos<S>(src, cs, predicted);
          tri_interp_aos<S>(src, cr, recovered);
          Aos<S>::unpack(src, ic, original);
#pragma unroll
          for (int f = 0; f < 4; ++f) {
            const float corrected = predicted[f] + 0.5f * (original[f] - recovered[f]);
            out[f] = clampv(corrected, mn(original[f], predicted[f]), mx(original[f], predicted[f]));
          }
          noise = thermal_noise_ys(P, cx, cy, cz, ysin);
        } else {
          tri_interp_aos<S>(src, cs, out);
          noise = thermal_noise(P, spx, spy, spz);
        }
        decay_scalars(P, ny, noise, out[0], out[1], out[2], out[3]);
        const uint32_t iv = flat(dm, x, y, z);
#pragma unroll
        for (int f = 0; f < 4; ++f) out[f] = qS_at<S>(out[f], P, iv, 5u + (uint32_t)f);
        any = any || out[0] != 0.f || out[1] != 0.f || out[2] != 0.f || out[3] != 0.f;
      }
      if (inside) {
        const uint32_t i = flat(dm, x, y, z);
        stS(dst.f[0], i, out[0]);
        stS(dst.f[1], i, out[1]);
        stS(dst.f[2], i, out[2]);
        stS(dst.f[3], i, out[3]);
      }
      energy_vote(c, x, y, z, inside, out[0], out[1], out[3], e);
    }
    const uint8_t s = summary_of(e);
    const int nzb = __syncthreads_or(any ? 1 : 0);
    if (threadIdx.x == 0) {
      summary[b] = s;
      nz[b] = nzb ? 1 : 0;
    }
  }
}

// -------------------------------------------------------------------- combustion
// combustion-update.wgsl.ts:42-93 from T into the next set over list_next:
// flagged bricks get the combustion update, the others copy T. Emits the next
// set's brick summary and non-zero bit.
template <typename S>
__global__ void __launch_bounds__(kBrickThreads) k_combustion(Dims dm, uint3 bc, const Params* __restrict__ Pp, SSet<S> tset,
                                                              const uint32_t* __restrict__ flags, const uint32_t* __restrict__ list,
                                                              const uint32_t* __restrict__ count, const uint8_t* __restrict__ nz_t,
                                                              const uint8_t* __restrict__ summary_t, SSet<S> dst,
                                                              uint8_t* __restrict__ summary, uint8_t* __restrict__ nz) {
  const Params P = *Pp;
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t b = list[li];
    const BrickCtx c = brick_ctx(dm, bc, b);
    const bool active = flag_at(flags, bc, b);
    const bool t_nonzero = nz_t[b] != 0;
    Energy e{false, false, false};
    bool any = false;
    // the thread's two voxels share x and y (z and z + 4), hence the row weight
    // and the y-only sine of the thermal cluster
    const uint32_t x = c.x0 + (threadIdx.x & 7u), y = c.y0 + ((threadIdx.x >> 3) & 7u);
    float ny = 0.0f, ysin = 0.0f;
    if (active) {
      ny = ((float)y + 0.5f) / (float)dm.h;
      ysin = thermal_cluster_ysin(P, (float)y);
    }
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t z = c.z0 + ((threadIdx.x + kBrickThreads * j) >> 6);
      const bool inside = x < dm.w && y < dm.h && z < dm.d;
      if (!inside) continue;
      const uint32_t i = flat(dm, x, y, z);
      float d = 0.f, t = 0.f, f = 0.f, r = 0.f;
      if (t_nonzero || active) {
        d = ldS(tset.f[0], i);
        t = ldS(tset.f[1], i);
        f = ldS(tset.f[2], i);
        r = ldS(tset.f[3], i);
      }
      if (active) {
        auto hot = [&](uint32_t k) { return comb_hot(ldS(tset.f[1], k), ldS(tset.f[2], k), ldS(tset.f[3], k)); };
        const Nbr n = neighbours(dm, x, y, z, i);
        const float nsum = hot(n.xp) + hot(n.xm) + hot(n.yp) + hot(n.ym) + hot(n.zp) + hot(n.zm);
        combustion_voxel_c(P, thermal_cluster_ys(P, (float)x, (float)y, (float)z, ysin), ny, nsum, d, t, f, r);
        d = qS_at<S>(d, P, i, 11);
        t = qS_at<S>(t, P, i, 10);
        f = qS_at<S>(f, P, i, 9);
        r = qS_at<S>(r, P, i, 12);
        energy_vote(c, x, y, z, true, d, t, r, e);
      }
      stS(dst.f[0], i, d);
      stS(dst.f[1], i, t);
      stS(dst.f[2], i, f);
      stS(dst.f[3], i, r);
      any = any || d != 0.f || t != 0.f || f != 0.f || r != 0.f;
    }
    const uint8_t s = summary_of(e);
    const int nzb = __syncthreads_or(any ? 1 : 0);
    if (threadIdx.x == 0) {
      summary[b] = active ? s : summary_t[b];
      nz[b] = nzb ? 1 : 0;
    }
  }
}

// ---------------------------------------------------------------------- buoyancy
// apply-buoyancy.wgsl.ts:37-110 over the flagged bricks of list_next.
template <typename S>
__global__ void __launch_bounds__(kBrickThreads) k_buoyancy(Dims dm, uint3 bc, const Params* __restrict__ Pp, SSet<S> set,
                                                            const uint32_t* __restrict__ flags, const uint32_t* __restrict__ list,
                                                            const uint32_t* __restrict__ count, VelField v) {
  const Params P = *Pp;
  const uint32_t n = *count;
  for (uint32_t li = blockIdx.x; li < n; li += gridDim.x) {
    const uint32_t b = list[li];
    if (!flag_at(flags, bc, b)) continue;
    const BrickCtx c = brick_ctx(dm, bc, b);
    // the thread's two voxels share x and y (z and z + 4)
    const uint32_t x = c.x0 + (threadIdx.x & 7u), y = c.y0 + ((threadIdx.x >> 3) & 7u);
    const BuoyXY q = buoy_xy(P, dm, x, y);
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t z = c.z0 + ((threadIdx.x + kBrickThreads * j) >> 6);
      if (x >= dm.w || y >= dm.h || z >= dm.d) continue;
      const uint32_t i = flat(dm, x, y, z);
      const S* D = set.f[0];
      auto hot = [&](uint32_t k) { return buoy_hot(ldS(set.f[1], k), ldS(set.f[3], k)); };
      const Nbr n = neighbours(dm, x, y, z, i);
      const float hot_gas = hot(i);
      const float tgx = (hot(n.xp) - hot(n.xm)) * 0.5f;
      const float tgy = (hot(n.yp) - hot(n.ym)) * 0.5f;
      const float tgz = (hot(n.zp) - hot(n.zm)) * 0.5f;
      const float dgx = (ldS(D, n.xp) - ldS(D, n.xm)) * 0.5f;
      const float dgy = (ldS(D, n.yp) - ldS(D, n.ym)) * 0.5f;
      const float dgz = (ldS(D, n.zp) - ldS(D, n.zm)) * 0.5f;
      float vx = v.c[0][i], vy = v.c[1][i], vz = v.c[2][i];
      buoyancy_voxel_xy(P, dm, q, x, y, z, ldS(D, i), hot_gas, tgx, tgy, tgz, dgx, dgy, dgz, vx, vy, vz);
      v.c[0][i] = vx;
      v.c[1][i] = vy;
      v.c[2][i] = vz;
    }
  }
}

// ------------------------------------------------------------ vorticity magnitude
// compute-vorticity.wgsl.ts:23-50: |w| for every voxel (w itself only when the
// debug fields are wanted; the confinement kernel recomputes w at its voxel).
// At an interior voxel i the reference's clamped neighbours (clamp-utils.wgsl.ts
// dec/inc) are i -+ 1, i -+ sy, i -+ sz: the curl and gradients there read
// them directly.
FX_DEV void curl_at(const VelField& v, uint32_t i, uint32_t sy, uint32_t sz, float& cx, float& cy, float& cz) {
  const uint32_t x0 = i - 1u, x1 = i + 1u, y0 = i - sy, y1 = i + sy, z0 = i - sz, z1 = i + sz;
  cx = ((__ldg(v.c[2] + y1) - __ldg(v.c[2] + y0)) - (__ldg(v.c[1] + z1) - __ldg(v.c[1] + z0))) * 0.5f;
  cy = ((__ldg(v.c[0] + z1) - __ldg(v.c[0] + z0)) - (__ldg(v.c[2] + x1) - __ldg(v.c[2] + x0))) * 0.5f;
  cz = ((__ldg(v.c[1] + x1) - __ldg(v.c[1] + x0)) - (__ldg(v.c[0] + y1) - __ldg(v.c[0] + y0))) * 0.5f;
}

__global__ void __launch_bounds__(256) k_vorticity(Dims dm, VelField v, float* __restrict__ wmag, VelField w, int write_w) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= dm.w || y >= dm.h || z >= dm.d) return;
  const uint32_t i = flat(dm, x, y, z);
  float cx = 0.f, cy = 0.f, cz = 0.f;
  if (!is_boundary(dm, x, y, z)) curl_at(v, i, dm.w, dm.w * dm.h, cx, cy, cz);
  wmag[i] = is_boundary(dm, x, y, z) ? 0.0f : length3(cx, cy, cz);
  if (write_w) {
    w.c[0][i] = cx;
    w.c[1][i] = cy;
    w.c[2][i] = cz;
  }
}

// k_vorticity with four x per thread (widths divisible by 4), one plane per
// thread: the rows it needs are float4 loads (vx at y -+ 1 and z -+ 1, vy at its
// row and z -+ 1, vz at its row and y -+ 1), the x neighbours of vy and vz come
// by warp shuffle (the row ends load theirs), and all of them are issued before
// the arithmetic. Each component and |w| are curl_at's operations in its order,
// so the results are the same bits.
__global__ void __launch_bounds__(256) k_vorticity_v4(Dims dm, VelField v, float* __restrict__ wmag, VelField w, int write_w) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y, z = blockIdx.z;
  if (y >= dm.h) return;  // whole warp
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const bool xin = x0 < dm.w;  // dm.w % 4 == 0: x0 + 3 < dm.w too
  const uint32_t i = (xin ? x0 : dm.w - 4) + dm.w * (y + dm.h * z);
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  auto ld4 = [&](const float* f, uint32_t k) { return __ldg(reinterpret_cast<const float4*>(f) + (k >> 2)); };
  auto st4 = [&](float* f, float4 val) { reinterpret_cast<float4*>(f)[i >> 2] = val; };
  const bool inner = y > 0 && y < dm.h - 1 && z > 0 && z < dm.d - 1;
  if (!inner) {
    if (xin) {
      st4(wmag, zero4);
      if (write_w) {
        st4(w.c[0], zero4);
        st4(w.c[1], zero4);
        st4(w.c[2], zero4);
      }
    }
    return;  // the whole warp shares y and z
  }
  const bool int0 = x0 > 0, int3 = x0 + 3 < dm.w - 1;
  const bool left_end = lane == 0 && x0 > 0, right_end = lane == 31 && x0 + 4 < dm.w;
  const float4 XU = ld4(v.c[0], i + sy), XD = ld4(v.c[0], i - sy), XP = ld4(v.c[0], i + sz), XM = ld4(v.c[0], i - sz);
  const float4 Y = ld4(v.c[1], i), YP = ld4(v.c[1], i + sz), YM = ld4(v.c[1], i - sz);
  const float4 Z = ld4(v.c[2], i), ZU = ld4(v.c[2], i + sy), ZD = ld4(v.c[2], i - sy);
  float yl = __shfl_up_sync(0xffffffffu, Y.w, 1), yr = __shfl_down_sync(0xffffffffu, Y.x, 1);
  float zl = __shfl_up_sync(0xffffffffu, Z.w, 1), zr = __shfl_down_sync(0xffffffffu, Z.x, 1);
  if (left_end) {
    yl = __ldg(v.c[1] + i - 1);
    zl = __ldg(v.c[2] + i - 1);
  }
  if (right_end) {
    yr = __ldg(v.c[1] + i + 4);
    zr = __ldg(v.c[2] + i + 4);
  }
  if (!xin) return;
  float4 cx = zero4, cy = zero4, cz = zero4, m = zero4;
  if (int0) {
    cx.x = ((ZU.x - ZD.x) - (YP.x - YM.x)) * 0.5f;
    cy.x = ((XP.x - XM.x) - (Z.y - zl)) * 0.5f;
    cz.x = ((Y.y - yl) - (XU.x - XD.x)) * 0.5f;
    m.x = length3(cx.x, cy.x, cz.x);
  }
  cx.y = ((ZU.y - ZD.y) - (YP.y - YM.y)) * 0.5f;
  cy.y = ((XP.y - XM.y) - (Z.z - Z.x)) * 0.5f;
  cz.y = ((Y.z - Y.x) - (XU.y - XD.y)) * 0.5f;
  m.y = length3(cx.y, cy.y, cz.y);
  cx.z = ((ZU.z - ZD.z) - (YP.z - YM.z)) * 0.5f;
  cy.z = ((XP.z - XM.z) - (Z.w - Z.y)) * 0.5f;
  cz.z = ((Y.w - Y.y) - (XU.z - XD.z)) * 0.5f;
  m.z = length3(cx.z, cy.z, cz.z);
  if (int3) {
    cx.w = ((ZU.w - ZD.w) - (YP.w - YM.w)) * 0.5f;
    cy.w = ((XP.w - XM.w) - (zr - Z.z)) * 0.5f;
    cz.w = ((yr - Y.z) - (XU.w - XD.w)) * 0.5f;
    m.w = length3(cx.w, cy.w, cz.w);
  }
  st4(wmag, m);
  if (write_w) {
    st4(w.c[0], cx);
    st4(w.c[1], cy);
    st4(w.c[2], cz);
  }
}

// apply-vorticity-confinement.wgsl.ts:30-66 from vScratch into vScratch2, with w
// recomputed at the voxel and the scalars read only from bricks that may be
// non-zero.
template <typename S, bool FMAG>
__global__ void __launch_bounds__(256) k_confinement(Dims dm, uint3 bc, const Params* __restrict__ Pp, VelField v, const float* __restrict__ wmag,
                                                     SSet<S> set, const uint8_t* __restrict__ nz, VelField out, float* __restrict__ fmag) {
  const uint32_t x = blockIdx.x * blockDim.x + threadIdx.x;
  const uint32_t y = blockIdx.y * blockDim.y + threadIdx.y;
  const uint32_t z = blockIdx.z * blockDim.z + threadIdx.z;
  if (x >= dm.w || y >= dm.h || z >= dm.d) return;
  const uint32_t i = flat(dm, x, y, z);
  float vx = __ldg(v.c[0] + i), vy = __ldg(v.c[1] + i), vz = __ldg(v.c[2] + i);
  if (is_boundary(dm, x, y, z)) {
    out.c[0][i] = vx;
    out.c[1][i] = vy;
    out.c[2][i] = vz;
    if (FMAG) fmag[i] = 0.0f;
    return;
  }
  const Params P = *Pp;
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const float gx = (__ldg(wmag + i + 1u) - __ldg(wmag + i - 1u)) * 0.5f;
  const float gy = (__ldg(wmag + i + sy) - __ldg(wmag + i - sy)) * 0.5f;
  const float gz = (__ldg(wmag + i + sz) - __ldg(wmag + i - sz)) * 0.5f;
  float wx, wy, wz;
  curl_at(v, i, sy, sz, wx, wy, wz);
  const uint32_t b = (x >> 3) + bc.x * ((y >> 3) + bc.y * (z >> 3));
  float d = 0.f, t = 0.f, r = 0.f;
  if (__ldg(nz + b)) {
    d = ldS(set.f[0], i);
    t = ldS(set.f[1], i);
    r = ldS(set.f[3], i);
  }
  // |F| (a length and a square root) only when the debug fields want it
  if (FMAG) {
    fmag[i] = confinement_voxel(P, gx, gy, gz, wx, wy, wz, __ldg(wmag + i), d, t, r, vx, vy, vz);
  } else {
    confinement_voxel_v(P, gx, gy, gz, wx, wy, wz, __ldg(wmag + i), d, t, r, vx, vy, vz);
  }
  out.c[0][i] = vx;
  out.c[1][i] = vy;
  out.c[2][i] = vz;
}

// Projection (project-velocity.wgsl.ts:21-43) with |v|
// (compute-debug-fields.wgsl.ts:18-25) fused when it is due. A thread computes
// a column of kProjZ voxels and reuses the z neighbours of the pressure.
constexpr int kProjZ = 8;

FX_DEV void project_column(Dims dm, uint32_t x, uint32_t y, uint32_t z0, const VelField& vs, const float* __restrict__ p, const VelField& vd,
                           float* __restrict__ vmag, int write_vmag, float& m) {
  const uint32_t sy = dm.w, sz = dm.w * dm.h;
  const uint32_t base = x + dm.w * y;
  const bool xyint = x > 0 && y > 0 && x < dm.w - 1 && y < dm.h - 1;
  float pz[kProjZ + 2];
  if (xyint) {
#pragma unroll
    for (int k = 0; k < kProjZ + 2; ++k) {
      const int z = (int)z0 + k - 1;
      pz[k] = (z >= 0 && z < (int)dm.d) ? __ldg(p + base + sz * (uint32_t)z) : 0.0f;
    }
  }
#pragma unroll
  for (int k = 0; k < kProjZ; ++k) {
    const uint32_t z = z0 + k;
    if (z >= dm.d) break;
    const uint32_t i = base + sz * z;
    float ox = 0.f, oy = 0.f, oz = 0.f;
    if (xyint && z > 0 && z < dm.d - 1) {
      const float gx = (__ldg(p + i + 1) - __ldg(p + i - 1)) * 0.5f;
      const float gy = (__ldg(p + i + sy) - __ldg(p + i - sy)) * 0.5f;
      const float gz = (pz[k + 2] - pz[k]) * 0.5f;
      ox = __ldg(vs.c[0] + i) - gx;
      oy = __ldg(vs.c[1] + i) - gy;
      oz = __ldg(vs.c[2] + i) - gz;
    }
    vd.c[0][i] = ox;
    vd.c[1][i] = oy;
    vd.c[2][i] = oz;
    if (write_vmag) vmag[i] = length3(ox, oy, oz);
    m = fmaxf(m, fmaxf(fabsf(ox), fmaxf(fabsf(oy), fabsf(oz))));
  }
}

// Also records max |v| of the result in *vmax (float bits; reset to 0 before
// the launch) for the next step's velocity advection.
__global__ void __launch_bounds__(256) k_project(Dims dm, VelField vs, const float* __restrict__ p, VelField vd, float* __restrict__ vmag,
                                                 int write_vmag, unsigned* __restrict__ vmax) {
  const uint32_t x = blockIdx.x * 32 + threadIdx.x, y = blockIdx.y * 8 + threadIdx.y, z0 = blockIdx.z * kProjZ;
  const bool live = x < dm.w && y < dm.h;
  float m = 0.0f;
  if (live) project_column(dm, x, y, z0, vs, p, vd, vmag, write_vmag, m);
  // block maximum, then one atomic per block when it raises the bound
  unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
  __shared__ unsigned part[8];
  const int warp = threadIdx.y;
  if (threadIdx.x == 0) part[warp] = bits;
  __syncthreads();
  if (threadIdx.x == 0 && warp == 0) {
    for (int k = 1; k < 8; ++k) bits = max(bits, part[k]);
    if (bits > __ldcg(vmax)) atomicMax(vmax, bits);
  }
}

inline dim3 proj_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 7) / 8, (d.d + kProjZ - 1) / kProjZ); }

// k_project with four x per thread marching runs of planes (widths divisible by
// 4). A thread holds the pressure rows at z - 1, z and z + 1, takes the x
// neighbours of its row by warp shuffle (the row ends load theirs) and reads the
// rows y -+ 1, which its neighbour warps loaded a plane earlier, from cache. The
// loads only it makes from DRAM (the three velocity rows of plane z + 1 and the
// pressure row of plane z + 2) are issued before it computes plane z. Each
// component, |v| and the running maximum are computed with project_column's
// operations in its order, so the results are the same bits.
template <bool VMAG>
__global__ void __launch_bounds__(256, 4) k_project_march(Dims dm, VelField vs, const float* __restrict__ p, VelField vd,
                                                          float* __restrict__ vmag, unsigned* __restrict__ vmax, int run) {
  const uint32_t lane = threadIdx.x;
  const uint32_t x0 = blockIdx.x * 128 + 4 * lane, y = blockIdx.y * 8 + threadIdx.y;
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
  const float4 zero4 = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
  auto ld4 = [&](const float* f, uint32_t i) { return __ldg(reinterpret_cast<const float4*>(f) + (i >> 2)); };
  auto st4 = [&](float* f, uint32_t i, float4 v) { reinterpret_cast<float4*>(f)[i >> 2] = v; };
  auto prow = [&](int z) { return (yint && z >= 0 && z < D) ? ld4(p, base + sz * (uint32_t)z) : zero4; };
  float4 pm = prow(zb - 1), pc = prow(zb), pp = prow(zb + 1);
  float4 VX = zero4, VY = zero4, VZ = zero4;
  {
    const uint32_t i = base + sz * (uint32_t)zb;
    if (yint) {
      VX = ld4(vs.c[0], i);
      VY = ld4(vs.c[1], i);
      VZ = ld4(vs.c[2], i);
    }
  }
  float m = 0.0f;
  for (int z = zb; z < ze; ++z) {
    const uint32_t i = base + sz * (uint32_t)z;
    const uint32_t in = base + sz * (uint32_t)min(z + 1, D - 1);
    float4 nVX = zero4, nVY = zero4, nVZ = zero4;
    if (yint) {
      nVX = ld4(vs.c[0], in);
      nVY = ld4(vs.c[1], in);
      nVZ = ld4(vs.c[2], in);
    }
    const float4 npp = prow(z + 2);
    const bool zint = yint && z > 0 && z < D - 1;
    float4 PU = zero4, PD = zero4;
    float pl = 0.0f, pr = 0.0f;
    if (zint) {
      PU = ld4(p, i + sy);
      PD = ld4(p, i - sy);
      if (left_end) pl = __ldg(p + i - 1);
      if (right_end) pr = __ldg(p + i + 4);
    }
    float left = __shfl_up_sync(0xffffffffu, pc.w, 1);     // p at x0 - 1
    float right = __shfl_down_sync(0xffffffffu, pc.x, 1);  // p at x0 + 4
    if (left_end) left = pl;
    if (right_end) right = pr;
    if (yin && xin) {
      // each component is stored as soon as it is formed (fewer live registers);
      // the running maximum is exact in any order
      float4 ox = zero4;
      if (zint) {
        if (int0) ox.x = VX.x - (pc.y - left) * 0.5f;
        ox.y = VX.y - (pc.z - pc.x) * 0.5f;
        ox.z = VX.z - (pc.w - pc.y) * 0.5f;
        if (int3) ox.w = VX.w - (right - pc.z) * 0.5f;
      }
      st4(vd.c[0], i, ox);
      float4 oy = zero4;
      if (zint) {
        if (int0) oy.x = VY.x - (PU.x - PD.x) * 0.5f;
        oy.y = VY.y - (PU.y - PD.y) * 0.5f;
        oy.z = VY.z - (PU.z - PD.z) * 0.5f;
        if (int3) oy.w = VY.w - (PU.w - PD.w) * 0.5f;
      }
      st4(vd.c[1], i, oy);
      float4 oz = zero4;
      if (zint) {
        if (int0) oz.x = VZ.x - (pp.x - pm.x) * 0.5f;
        oz.y = VZ.y - (pp.y - pm.y) * 0.5f;
        oz.z = VZ.z - (pp.z - pm.z) * 0.5f;
        if (int3) oz.w = VZ.w - (pp.w - pm.w) * 0.5f;
      }
      st4(vd.c[2], i, oz);
      if (VMAG)
        st4(vmag, i, make_float4(length3(ox.x, oy.x, oz.x), length3(ox.y, oy.y, oz.y), length3(ox.z, oy.z, oz.z), length3(ox.w, oy.w, oz.w)));
      m = fmaxf(m, fmaxf(fabsf(ox.x), fmaxf(fabsf(oy.x), fabsf(oz.x))));
      m = fmaxf(m, fmaxf(fabsf(ox.y), fmaxf(fabsf(oy.y), fabsf(oz.y))));
      m = fmaxf(m, fmaxf(fabsf(ox.z), fmaxf(fabsf(oy.z), fabsf(oz.z))));
      m = fmaxf(m, fmaxf(fabsf(ox.w), fmaxf(fabsf(oy.w), fabsf(oz.w))));
    }
    pm = pc;
    pc = pp;
    pp = npp;
    VX = nVX;
    VY = nVY;
    VZ = nVZ;
  }
  // block maximum, then one atomic per block when it raises the bound
  unsigned bits = __reduce_max_sync(0xffffffffu, __float_as_uint(m));
  __shared__ unsigned part[8];
  const int warp = threadIdx.y;
  if (threadIdx.x == 0) part[warp] = bits;
  __syncthreads();
  if (threadIdx.x == 0 && warp == 0) {
    for (int k = 1; k < 8; ++k) bits = max(bits, part[k]);
    if (bits > __ldcg(vmax)) atomicMax(vmax, bits);
  }
}

// The projection launch: k_project_march where the width allows it
// (FENIX_PROJ_MARCH=0 keeps k_project), with runs of planes such that the
// 128 x 8 row tiles times the runs fill the resident blocks once.
cudaError_t launch_project(cudaStream_t s, Dims dm, const VelField& vs, const float* p, const VelField& vd, float* vmag, int write_vmag,
                           unsigned* vmax) {
  static const bool march = [] {
    const char* v = std::getenv("FENIX_PROJ_MARCH");
    return !(v && *v == '0');
  }();
  if (march && dm.w % 4 == 0 && dm.w >= 8) {
    static int slots[64] = {};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    int n = (dev >= 0 && dev < 64) ? slots[dev] : 0;
    if (n <= 0) {
      int per_sm = 0, sms = 0;
      e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_project_march<true>, 256, 0);
      if (e != cudaSuccess) return e;
      e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
      if (e != cudaSuccess) return e;
      n = std::max(1, per_sm) * std::max(1, sms);
      if (dev >= 0 && dev < 64) slots[dev] = n;
    }
    const int run = march_plan_one_wave(dm, n);
    const dim3 g((dm.w + 127) / 128, (dm.h + 7) / 8, (dm.d + run - 1) / run);
    if (write_vmag)
      k_project_march<true><<<g, dim3(32, 8, 1), 0, s>>>(dm, vs, p, vd, vmag, vmax, run);
    else
      k_project_march<false><<<g, dim3(32, 8, 1), 0, s>>>(dm, vs, p, vd, vmag, vmax, run);
  } else {
    k_project<<<proj_grid(dm), dim3(32, 8, 1), 0, s>>>(dm, vs, p, vd, vmag, write_vmag, vmax);
  }
  return cudaGetLastError();
}

// Rebuilds the per-brick bookkeeping after the fields were written from the host:
// the non-zero bits of the three scalar buffers and the summary of the current set.
template <typename S>
__global__ void __launch_bounds__(kBrickThreads) k_rebuild(Dims dm, uint3 bc, SSet<S> cur, SSet<S> other, SSet<S> tset,
                                                           uint8_t* __restrict__ summary_cur, uint8_t* __restrict__ nz_cur,
                                                           uint8_t* __restrict__ nz_other, uint8_t* __restrict__ nz_t) {
  const uint32_t nb = bc.x * bc.y * bc.z;
  for (uint32_t b = blockIdx.x; b < nb; b += gridDim.x) {
    const BrickCtx c = brick_ctx(dm, bc, b);
    Energy e{false, false, false};
    bool a0 = false, a1 = false, a2 = false;
#pragma unroll
    for (int j = 0; j < 2; ++j) {
      const uint32_t lv = threadIdx.x + kBrickThreads * j;
      const uint32_t x = c.x0 + (lv & 7u), y = c.y0 + ((lv >> 3) & 7u), z = c.z0 + (lv >> 6);
      const bool inside = x < dm.w && y < dm.h && z < dm.d;
      float d = 0.f, t = 0.f, r = 0.f;
      if (inside) {
        const uint32_t i = flat(dm, x, y, z);
        d = rdS(cur.f[0], i);
        t = rdS(cur.f[1], i);
        r = rdS(cur.f[3], i);
        a0 = a0 || d != 0.f || t != 0.f || rdS(cur.f[2], i) != 0.f || r != 0.f;
        a1 = a1 || rdS(other.f[0], i) != 0.f || rdS(other.f[1], i) != 0.f || rdS(other.f[2], i) != 0.f || rdS(other.f[3], i) != 0.f;
        a2 = a2 || rdS(tset.f[0], i) != 0.f || rdS(tset.f[1], i) != 0.f || rdS(tset.f[2], i) != 0.f || rdS(tset.f[3], i) != 0.f;
      }
      energy_vote(c, x, y, z, inside, d, t, r, e);
    }
    const uint8_t s = summary_of(e);
    const int n0 = __syncthreads_or(a0 ? 1 : 0);
    const int n1 = __syncthreads_or(a1 ? 1 : 0);
    const int n2 = __syncthreads_or(a2 ? 1 : 0);
    if (threadIdx.x == 0) {
      summary_cur[b] = s;
      nz_cur[b] = n0 ? 1 : 0;
      nz_other[b] = n1 ? 1 : 0;
      nz_t[b] = n2 ? 1 : 0;
    }
  }
}

inline dim3 dense_grid(Dims d) { return dim3((d.w + 31) / 32, (d.h + 3) / 4, (d.d + 1) / 2); }
const dim3 kDenseBlock(32, 4, 2);

#include "fx_fused_sparse.cuh"

// Host: bricks whose voxels an emitter can reach this step (conservative).
void injection_bricks(const FusedStep& st, std::vector<uint8_t>& mark, std::vector<uint32_t>& out) {
  out.clear();
  if (!st.host_sources || st.host_nsrc == 0) return;
  const Dims dm = st.dm;
  const uint3 bc = st.bricks;
  mark.assign((size_t)bc.x * bc.y * bc.z, 0);
  const double dxw = (double)st.host_params.dx / std::max((double)st.host_params.world_size, 1e-4);
  const double t = st.host_params.time;
  for (uint32_t e = 0; e < st.host_nsrc; ++e) {
    const float* s = st.host_sources + 32 * (size_t)e;
    const double start = s[4], duration = s[5];
    const double age = t - start;
    // activeGate (inject-source-common.wgsl.ts:24-27) with a margin for f32 rounding
    if (!(age >= -1e-3 * (1.0 + std::fabs(t)) && age <= duration + 1e-3 * (1.0 + std::fabs(duration)))) {
      if (std::isfinite(age) && std::isfinite(duration)) continue;
    }
    const double r = s[3];
    double reach = r + std::max(r * 0.24, dxw * 3.0);
    if (!std::isfinite(reach)) reach = 4.0;
    reach = std::max(reach, 0.0) * 1.0001 + 1e-6;
    uint32_t lo[3], hi[3];
    const uint32_t dims[3] = {dm.w, dm.h, dm.d};
    bool empty = false;
    for (int a = 0; a < 3; ++a) {
      const double c = s[a];
      double l = std::floor((c - reach) * dims[a] - 0.5) - 1.0, h = std::ceil((c + reach) * dims[a] - 0.5) + 1.0;
      if (!std::isfinite(l)) l = 0;
      if (!std::isfinite(h)) h = dims[a] - 1.0;
      l = std::max(l, 0.0);
      h = std::min(h, dims[a] - 1.0);
      if (h < l) {
        empty = true;
        break;
      }
      lo[a] = (uint32_t)l;
      hi[a] = (uint32_t)h;
    }
    if (empty) continue;
    for (uint32_t bz = lo[2] / 8; bz <= hi[2] / 8; ++bz)
      for (uint32_t by = lo[1] / 8; by <= hi[1] / 8; ++by)
        for (uint32_t bx = lo[0] / 8; bx <= hi[0] / 8; ++bx) {
          const uint32_t b = bx + bc.x * (by + bc.y * bz);
          if (!mark[b]) {
            mark[b] = 1;
            out.push_back(b);
          }
        }
  }
}

}  // namespace

size_t fused_work_bytes(Dims dm, uint3 bricks, size_t aos_voxel_bytes) {
  const size_t nb = (size_t)bricks.x * bricks.y * bricks.z;
  const size_t n = (size_t)dm.w * dm.h * dm.d;
  return 12 * align256(nb) + 7 * align256(nb * 4) + align256(16 * 4) + align256(sizeof(SolverDev)) + align256(4) +
         align256(n * aos_voxel_bytes);
}

void fused_work_carve(FusedWork& w, char* base, Dims dm, uint3 bricks, size_t aos_voxel_bytes) {
  w.dm = dm;
  w.bricks = bricks;
  w.nb = bricks.x * bricks.y * bricks.z;
  size_t off = 0;
  auto take = [&](size_t bytes) {
    char* p = base + off;
    off += align256(bytes);
    return p;
  };
  w.summary_set[0] = (uint8_t*)take(w.nb);
  w.summary_set[1] = (uint8_t*)take(w.nb);
  w.summary_t = (uint8_t*)take(w.nb);
  w.nz_set[0] = (uint8_t*)take(w.nb);
  w.nz_set[1] = (uint8_t*)take(w.nb);
  w.nz_t = (uint8_t*)take(w.nb);
  w.nz_aos = (uint8_t*)take(w.nb);
  take(w.nb);
  w.list_adv = (uint32_t*)take((size_t)w.nb * 4);
  w.list_next = (uint32_t*)take((size_t)w.nb * 4);
  w.list_inj = (uint32_t*)take((size_t)w.nb * 4);
  for (auto& b : w.nz_sp) b = (uint8_t*)take(w.nb);
  for (auto& l : w.list_sp) l = (uint32_t*)take((size_t)w.nb * 4);
  w.counters = (uint32_t*)take(16 * 4);
  w.dev_err = w.counters + 8;
  w.solver = (SolverDev*)take(sizeof(SolverDev));
  w.vmax = (unsigned*)take(4);
  w.aos = take((size_t)dm.w * dm.h * dm.d * aos_voxel_bytes);
}

fx_status fused_init(FusedWork& w, cudaStream_t) {
  if (cudaEventCreateWithFlags(&w.inj_event, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (host_alloc((void**)&w.host_list_inj, ((size_t)w.nb + 1) * 4) != cudaSuccess) return FX_ERR_OUT_OF_MEMORY;
  if (host_alloc((void**)&w.host_cont, sizeof(int)) != cudaSuccess) return FX_ERR_OUT_OF_MEMORY;
  if (cudaStreamCreateWithFlags(&w.aux, cudaStreamNonBlocking) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&w.aux2, cudaStreamNonBlocking) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.fork_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.join_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaStreamCreateWithFlags(&w.aux3, cudaStreamNonBlocking) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.fork2_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.join2_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.prep_fork_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaEventCreateWithFlags(&w.prep_join_ev, cudaEventDisableTiming) != cudaSuccess) return FX_ERR_CUDA;
  if (vcycle_init() != cudaSuccess) return FX_ERR_CUDA;
  w.valid = true;  // the arena starts cleared: every brick is zero
  return FX_OK;
}

fx_status fused_reset(FusedWork& w, cudaStream_t) {
  // The arena was cleared: every brick is zero, and the device copy of the
  // injection list is gone.
  w.valid = true;
  w.sp_known = true;
  w.uploaded_list.clear();
  return FX_OK;
}

fx_status fused_invalidate(FusedWork& w, cudaStream_t) {
  w.valid = false;
  w.sp_known = false;
  return FX_OK;
}

void fused_release(FusedWork& w) {
  for (auto& kv : w.graphs) cudaGraphExecDestroy(kv.second.exec);
  w.graphs.clear();
  if (w.inj_event) cudaEventDestroy(w.inj_event);
  w.inj_event = nullptr;
  if (w.host_list_inj) cudaFreeHost(w.host_list_inj);
  w.host_list_inj = nullptr;
  if (w.host_cont) cudaFreeHost(w.host_cont);
  w.host_cont = nullptr;
  if (w.aux) cudaStreamDestroy(w.aux);
  w.aux = nullptr;
  if (w.aux2) cudaStreamDestroy(w.aux2);
  w.aux2 = nullptr;
  if (w.fork_ev) cudaEventDestroy(w.fork_ev);
  if (w.join_ev) cudaEventDestroy(w.join_ev);
  w.fork_ev = w.join_ev = nullptr;
  if (w.aux3) cudaStreamDestroy(w.aux3);
  w.aux3 = nullptr;
  if (w.fork2_ev) cudaEventDestroy(w.fork2_ev);
  if (w.join2_ev) cudaEventDestroy(w.join2_ev);
  w.fork2_ev = w.join2_ev = nullptr;
  if (w.prep_fork_ev) cudaEventDestroy(w.prep_fork_ev);
  if (w.prep_join_ev) cudaEventDestroy(w.prep_join_ev);
  w.prep_fork_ev = w.prep_join_ev = nullptr;
  for (auto& ev : w.timing_events) cudaEventDestroy(ev);
  w.timing_events.clear();
}

void fused_set_timing(FusedWork& w, bool on) { w.timing = on; }

void fused_drain_timing(FusedWork& w, const std::function<void(const char*, uint32_t, double)>& sink) {
  for (auto& p : w.timing_pending) {
    float ms = 0.f;
    cudaEventElapsedTime(&ms, w.timing_events[p.a], w.timing_events[p.b]);
    sink(p.name, 1, ms);
  }
  w.timing_pending.clear();
  w.timing_next = 0;
}

namespace {

struct Timed {
  FusedWork& w;
  cudaStream_t s;
  int a = -1;
  const char* name;
  Timed(FusedWork& w_, cudaStream_t s_, const char* n) : w(w_), s(s_), name(n) {
    if (!w.timing) return;
    a = w.next_event();
    cudaEventRecord(w.timing_events[a], s);
  }
  ~Timed() {
    if (!w.timing) return;
    const int b = w.next_event();
    cudaEventRecord(w.timing_events[b], s);
    w.timing_pending.push_back({name, a, b});
  }
};

}  // namespace

int FusedWork::next_event() {
  if (timing_next >= (int)timing_events.size()) {
    cudaEvent_t e = nullptr;
    cudaEventCreate(&e);
    timing_events.push_back(e);
  }
  return timing_next++;
}

#define FX_CK(call)                              \
  do {                                           \
    cudaError_t e_ = (call);                     \
    if (e_ != cudaSuccess) {                     \
      out.error = std::string(#call) + ": " + cudaGetErrorString(e_); \
      return FX_ERR_CUDA;                        \
    }                                            \
  } while (0)

fx_status fused_sequence(FusedWork& w, const FusedStep& st, uint32_t ninj, FusedResult& out);

// The grid of brick kernel k: SMs x its CTAs per SM, at most one block per brick.
uint32_t brick_grid_of(const FusedStep& st, uint32_t nb, BrickKernel k) {
  const uint32_t m = st.brick_ctas[k] ? st.brick_ctas[k] : (uint32_t)kBrickCtasDefault;
  return std::max<uint32_t>(1, std::min<uint32_t>(nb, (uint32_t)device_sm_count() * m));
}

fx_status fused_prepare(FusedWork& w, const FusedStep& st, uint32_t* ninj_out, FusedResult& out) {
  cudaStream_t s = st.stream;
  const Dims dm = st.dm;
  const uint3 bc = st.bricks;
  const uint32_t nb = w.nb;
  const int cur = st.cur_index, next = cur ^ 1;
  uint32_t launches = 0;
  const uint32_t brick_grid = std::max<uint32_t>(1, std::min<uint32_t>(nb, (uint32_t)device_sm_count() * 8u));
  uint32_t* c_inj = w.counters + 3;

  if (!w.valid) {
    // the fields came from the host: their largest |v| is unknown
    FX_CK(cudaMemsetAsync(w.vmax, 0xFF, sizeof(unsigned), s));
    Timed tm(w, s, "fused_rebuild");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_rebuild<S><<<brick_grid, kBrickThreads, 0, s>>>(dm, bc, sset<S>(st.cur), sset<S>(st.next), sset<S>(st.scratch), w.summary_set[cur],
                                                        w.nz_set[cur], w.nz_set[next], w.nz_t);
    });
    ++launches;
    w.valid = true;
  }

  // Sparse mode keeps per-brick non-zero bits of the velocity buffers; after a
  // dense step or a host write every brick may be non-zero.
  if (st.sparse && !w.sp_known) {
    for (auto* b : w.nz_sp) FX_CK(cudaMemsetAsync(b, 1, nb, s));
    w.sp_known = true;
  }
  if (!st.sparse) w.sp_known = false;

  // 1. injection over the reachable bricks: the list is built on the host and
  // uploaded only when it changes.
  injection_bricks(st, w.host_mark, w.host_list);
  const uint32_t ninj = (uint32_t)w.host_list.size();
  if (ninj && w.host_list != w.uploaded_list) {
    FX_CK(cudaEventSynchronize(w.inj_event));
    std::memcpy(w.host_list_inj, w.host_list.data(), ninj * 4);
    w.host_list_inj[nb] = ninj;
    FX_CK(cudaMemcpyAsync(w.list_inj, w.host_list_inj, ninj * 4, cudaMemcpyHostToDevice, s));
    FX_CK(cudaMemcpyAsync(c_inj, w.host_list_inj + nb, 4, cudaMemcpyHostToDevice, s));
    FX_CK(cudaEventRecord(w.inj_event, s));
    w.uploaded_list = w.host_list;
  }
  *ninj_out = ninj;
  out.launches = launches;
  return FX_OK;
}

constexpr size_t kMaxTapedGraphs = 64;

uint64_t fused_key(const FusedStep& st, uint32_t ninj) {
  uint64_t key = 0;
  auto mix_key = [&](uint64_t v) { key = (key ^ v) * 0x100000001b3ull; };
  key = 0xcbf29ce484222325ull;
  mix_key((uint64_t)st.cur_index);
  mix_key(ninj > 0);
  mix_key((uint64_t)(uintptr_t)st.sources);
  mix_key(st.nsrc);
  mix_key((uint64_t)st.advect_mode);
  mix_key(st.vort_on);
  mix_key(st.pressure_on);
  mix_key(st.debug_on);
  mix_key(st.debug_fields);
  mix_key((uint64_t)st.last_p);
  for (int k = 0; k < 7; ++k) mix_key((uint64_t)st.q[k]);
  mix_key((uint64_t)st.solver_mode);
  for (int l = 0; l < 3; ++l) mix_key((uint64_t)(st.sweep_variant[l] + 1));
  mix_key(st.solver_norms);
  mix_key(st.sparse);
  for (int k = 0; k < kBrickKernels; ++k) mix_key(st.brick_ctas[k]);
  for (const void* p : {(const void*)st.tape_t1, (const void*)st.tape_r1, (const void*)st.tape_v1.c[0], (const void*)st.tape_a.c[0],
                        (const void*)st.tape_b.c[0]})
    mix_key((uint64_t)(uintptr_t)p);
  mix_key((uint64_t)(uintptr_t)st.inflow);
  if (st.inflow)
    for (uint32_t v : {st.inflow_patch.x0, st.inflow_patch.y, st.inflow_patch.z0, st.inflow_patch.nx, st.inflow_patch.nz}) mix_key(v);
  if (st.solver_mode == 1) {
    const VCycleConfig& c = st.vc;
    for (int v : {c.levels, c.pre, c.post, c.coarse, c.max_cycles, (int)c.warm, (int)c.omega_one}) mix_key((uint64_t)v);
    uint32_t wb;
    std::memcpy(&wb, &c.omega, 4);
    uint64_t tb;
    std::memcpy(&tb, &c.tol, 8);
    mix_key(wb);
    mix_key(tb);
  }
  return key;
}

fx_status fused_step(FusedWork& w, const FusedStep& st, FusedResult& out) {
  cudaStream_t s = st.stream;
  uint32_t ninj = 0;
  FusedResult prep;
  const fx_status ps = fused_prepare(w, st, &ninj, prep);
  if (ps != FX_OK) {
    out.error = prep.error;
    return ps;
  }
  const uint32_t launches = prep.launches;

  // The device part of the step, captured once per configuration and replayed.
  const bool graphs = w.use_graphs && !w.timing;
  const uint64_t key = fused_key(st, ninj);
  if (graphs) {
    auto it = w.graphs.find(key);
    if (it == w.graphs.end()) {
      cudaGraph_t g = nullptr;
      FX_CK(cudaStreamBeginCapture(s, cudaStreamCaptureModeRelaxed));
      FusedResult tmp;
      const fx_status cst = fused_sequence(w, st, ninj, tmp);
      const cudaError_t ce = cudaStreamEndCapture(s, &g);
      if (cst != FX_OK || ce != cudaSuccess) {
        if (g) cudaGraphDestroy(g);
        cudaGetLastError();
        w.use_graphs = false;  // capture unsupported here: launch directly from now on
        w.graph_note = "capture failed: " + (cst != FX_OK ? tmp.error : std::string(cudaGetErrorString(ce)));
        return fused_sequence(w, st, ninj, out);
      }
      cudaGraphExec_t ex = nullptr;
      const cudaError_t ie = cudaGraphInstantiate(&ex, g, 0);
      cudaGraphDestroy(g);
      if (ie != cudaSuccess) {
        cudaGetLastError();
        w.use_graphs = false;
        w.graph_note = std::string("instantiate failed: ") + cudaGetErrorString(ie);
        return fused_sequence(w, st, ninj, out);
      }
      const bool taped = st.tape_t1 != nullptr;
      if (taped) {
        // Every rollout records its tapes at its own addresses: keep the taped
        // graphs of a few rollouts, not of every rollout ever made.
        size_t count = 0;
        for (const auto& kv : w.graphs) count += kv.second.taped;
        if (count >= kMaxTapedGraphs)
          for (auto g = w.graphs.begin(); g != w.graphs.end();) {
            if (g->second.taped) {
              cudaGraphExecDestroy(g->second.exec);
              g = w.graphs.erase(g);
            } else {
              ++g;
            }
          }
      }
      it = w.graphs.emplace(key, FusedWork::GraphEntry{ex, tmp, taped}).first;
    }
    FX_CK(cudaGraphLaunch(it->second.exec, s));
    out = it->second.result;
    out.launches += launches;
    out.graph = true;
    return FX_OK;
  }
  const fx_status r = fused_sequence(w, st, ninj, out);
  out.launches += launches;
  return r;
}

// The V-cycle solve: the divergence, the prologue (norms, first decision) and
// the loop. Under stream capture the loop is a WHILE conditional node whose
// body graph (one cycle + norm + decision) is captured on the auxiliary stream;
// without capture the host reads the decision after every cycle.
fx_status vcycle_solve(FusedWork& w, const FusedStep& st, const VelField& vfin, uint32_t& launches, FusedResult& out) {
  cudaStream_t s = st.stream;
  const LevelBuf& F = st.lv[0];
  {
    Timed tm(w, s, "fused_divergence");
    FX_CK(lean_div_first(s, st.dm, vfin, F.div, nullptr, st.lv[1].dm, st.lv[1].div, false));
    ++launches;
  }
  VCycleLevels L;
  for (int k = 0; k < 3; ++k) {
    L.lv[k] = st.lv[k];
    L.lv[3 + k] = st.xlv[k];
  }
  const int start = st.last_p;
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  FX_CK(cudaStreamIsCapturing(s, &cs));
  if (cs == cudaStreamCaptureStatusActive) {
    cudaGraph_t g = nullptr;
    const cudaGraphNode_t* deps = nullptr;
    size_t ndeps = 0;
    FX_CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphConditionalHandle h = 0;
    FX_CK(cudaGraphConditionalHandleCreate(&h, g, 0, cudaGraphCondAssignDefault));
    FX_CK(vcycle_prologue(s, L, st.vc, start, w.solver, h));
    launches += 3;
    FX_CK(cudaStreamGetCaptureInfo(s, &cs, nullptr, &g, &deps, &ndeps));
    cudaGraphNodeParams cp = {};
    cp.type = cudaGraphNodeTypeConditional;
    cp.conditional.handle = h;
    cp.conditional.type = cudaGraphCondTypeWhile;
    cp.conditional.size = 1;
    cudaGraphNode_t node = nullptr;
    FX_CK(cudaGraphAddNode(&node, g, deps, ndeps, &cp));
    cudaGraph_t body = cp.conditional.phGraph_out[0];
    FX_CK(cudaStreamBeginCaptureToGraph(w.aux, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed));
    uint32_t body_launches = 0;
    const cudaError_t be = vcycle_body(w.aux, L, st.vc, start, w.solver, h, &body_launches);
    cudaGraph_t body_out = nullptr;
    const cudaError_t ee = cudaStreamEndCapture(w.aux, &body_out);
    FX_CK(be);
    FX_CK(ee);
    FX_CK(cudaStreamUpdateCaptureDependencies(s, &node, 1, cudaStreamSetCaptureDependencies));
    out.cycle_launches = body_launches;
  } else {
    {
      Timed tm(w, s, "fused_vcycle_prologue");
      FX_CK(vcycle_prologue(s, L, st.vc, start, w.solver, 0));
      launches += 3;
    }
    uint32_t body_launches = 0;
    for (int c = 0; c < st.vc.max_cycles; ++c) {
      FX_CK(cudaMemcpyAsync(w.host_cont, &w.solver->cont, sizeof(int), cudaMemcpyDeviceToHost, s));
      FX_CK(cudaStreamSynchronize(s));
      if (!*w.host_cont) break;
      Timed tm(w, s, "fused_vcycle");
      body_launches = 0;
      FX_CK(vcycle_body(s, L, st.vc, start, w.solver, 0, &body_launches));
    }
    out.cycle_launches = body_launches;
  }
  return FX_OK;
}

fx_status fused_sequence(FusedWork& w, const FusedStep& st, uint32_t ninj, FusedResult& out) {
  cudaStream_t s = st.stream;
  const Dims dm = st.dm;
  const uint3 bc = st.bricks;
  const uint32_t nb = w.nb;
  const int cur = st.cur_index, next = cur ^ 1;
  uint32_t launches = 0;
  uint32_t* c_adv = w.counters + 0;
  uint32_t* c_next = w.counters + 1;
  uint32_t* c_inj = w.counters + 3;
  // The mid and coarse part of PressureSolvePass.solve (:73-82), sweep by sweep
  // (inside the step's CUDA graph the launch gaps are short): mid pre-smoothing,
  // restriction to coarse, coarse smoothing, prolongation into mid pressureA,
  // mid post-smoothing. The first sweep of a level reads the cleared buffer, so
  // it is computed from the divergence alone. With `side`, the chain runs on the
  // second stream, forked after the restriction into the mid level and joined by
  // join_ev; *mid gets the mid buffer holding the result.
  auto lower_levels = [&](bool side, int& mid) -> cudaError_t {
    const LevelBuf& M = st.lv[1];
    const LevelBuf& C = st.lv[2];
    cudaStream_t ls = s;
    if (side) {
      cudaError_t e = cudaEventRecord(w.fork_ev, s);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(w.aux2, w.fork_ev, 0);
      if (e != cudaSuccess) return e;
      ls = w.aux2;
    }
    // The coarse level needs the restricted divergence, not the mid
    // pre-sweeps: beside the fine sweeps it runs on a third stream next to
    // them, and the prolongation into the mid level waits for both.
    cudaStream_t cs = ls;
    if (side) {
      cudaError_t e = cudaEventRecord(w.fork2_ev, ls);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(w.aux3, w.fork2_ev, 0);
      if (e != cudaSuccess) return e;
      cs = w.aux3;
    }
    int a = 0;
    for (int k = 0; k < st.q[4]; ++k) {
      Timed tm(w, ls, "fused_sweep_mid");
      cudaError_t e = lean_sweep_variant(ls, st.sweep_variant[1], M.dm, M.div, k == 0 ? nullptr : M.p[a], M.p[a ^ 1], M.dm, nullptr);
      if (e != cudaSuccess) return e;
      a ^= 1;
      ++launches;
    }
    const int mid_pre = a;
    {
      Timed tm(w, cs, "fused_restrict");
      plain_restrict(cs, M.dm, C.dm, M.div, C.div);
      ++launches;
    }
    int coarse = 0;
    for (int k = 0; k < st.q[6]; ++k) {
      Timed tm(w, cs, "fused_sweep_coarse");
      cudaError_t e = lean_sweep_variant(cs, st.sweep_variant[2], C.dm, C.div, k == 0 ? nullptr : C.p[coarse], C.p[coarse ^ 1], C.dm, nullptr);
      if (e != cudaSuccess) return e;
      coarse ^= 1;
      ++launches;
    }
    if (side) {
      cudaError_t e = cudaEventRecord(w.join2_ev, cs);
      if (e == cudaSuccess) e = cudaStreamWaitEvent(ls, w.join2_ev, 0);
      if (e != cudaSuccess) return e;
    }
    {
      Timed tm(w, ls, "fused_prolong");
      plain_prolong(ls, C.dm, M.dm, C.p[coarse], M.p[0]);
      ++launches;
    }
    mid = mid_pre;
    for (int k = 0; k < st.q[5]; ++k) {
      Timed tm(w, ls, "fused_sweep_mid");
      cudaError_t e = lean_sweep_variant(ls, st.sweep_variant[1], M.dm, M.div, M.p[mid], M.p[mid ^ 1], M.dm, nullptr);
      if (e != cudaSuccess) return e;
      mid ^= 1;
      ++launches;
    }
    if (side) return cudaEventRecord(w.join_ev, w.aux2);
    return cudaGetLastError();
  };
  // The rollout's tape (f32 storage): copies of the velocity at three points of
  // the step, and temperature and reaction before the igniter, which equal the
  // fields before the injection outside the emitters' reach and are written by the
  // injection kernel inside it.
  const bool taped = st.tape_t1 != nullptr && !st.half_storage;
  const size_t field_bytes = (size_t)dm.w * dm.h * dm.d * sizeof(float);
  auto tape_vel = [&](const VelField& dst, const VelField& src) -> cudaError_t {
    for (int k = 0; k < 3 && dst.c[0]; ++k) {
      const cudaError_t e = cudaMemcpyAsync(dst.c[k], src.c[k], field_bytes, cudaMemcpyDeviceToDevice, s);
      if (e != cudaSuccess) return e;
    }
    return cudaSuccess;
  };
  if (taped) {
    FX_CK(cudaMemcpyAsync(st.tape_t1, st.cur.f[1], field_bytes, cudaMemcpyDeviceToDevice, s));
    FX_CK(cudaMemcpyAsync(st.tape_r1, st.cur.f[3], field_bytes, cudaMemcpyDeviceToDevice, s));
  }
  if (ninj) {
    Timed tm(w, s, "fused_inject");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_inject<S><<<brick_grid_of(st, nb, BK_INJECT), kBrickThreads, 0, s>>>(dm, bc, st.params, st.sources, st.nsrc, w.list_inj, c_inj, sset<S>(st.cur), st.vcur,
                                                       w.summary_set[cur], w.nz_set[cur], taped ? st.tape_t1 : nullptr,
                                                       taped ? st.tape_r1 : nullptr);
    });
    ++launches;
  }

  // Sparse mode: the injected velocity may be non-zero in the injected bricks.
  if (st.sparse && ninj) {
    k_sp_mark<<<std::max<uint32_t>(1, std::min<uint32_t>((ninj + 255) / 256, 256)), 256, 0, s>>>(w.list_inj, c_inj, w.nz_sp[SP_VCUR]);
    ++launches;
  }

  // The inflow patch after injection; its values are not bounded by the recorded
  // max |v|, so the velocity advection clamps on read in this step.
  if (st.inflow) {
    plain_inflow(s, dm, st.inflow_patch, st.inflow, st.vcur);
    FX_CK(cudaMemsetAsync(w.vmax, 0xFF, sizeof(unsigned), s));
    ++launches;
  }
  if (taped) FX_CK(tape_vel(st.tape_v1, st.vcur));

  // The interleaved copy, and in dense mode the current flags too, do not feed
  // the velocity advection: they run on the second stream beside it, joined
  // before the scalar advection. (Sparse mode's velocity advection walks the
  // current flags, so there they stay on the step's stream.)
  FX_CK(cudaEventRecord(w.prep_fork_ev, s));
  FX_CK(cudaStreamWaitEvent(w.aux2, w.prep_fork_ev, 0));
  const cudaStream_t ps = w.aux2;
  const cudaStream_t fs = st.sparse ? s : w.aux2;
  // the interleaved copy of the current set for the scalar advection
  {
    Timed tm(w, ps, "fused_pack_aos");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_pack_aos<S><<<(nb + 7) / 8, dim3(32, 8), 0, ps>>>(dm, bc, sset<S>(st.cur), w.nz_set[cur], w.nz_aos,
                                                          static_cast<typename Aos<S>::T*>(w.aos));
    });
    ++launches;
  }

  // 2. flags of the current set, list of bricks for scalar advection
  FX_CK(cudaMemsetAsync(w.counters, 0, 3 * sizeof(uint32_t), fs));
  if (st.sparse) FX_CK(cudaMemsetAsync(w.counters + 4, 0, 4 * sizeof(uint32_t), fs));
  {
    Timed tm(w, fs, "fused_dilate");
    k_dilate<<<(nb + 255) / 256, 256, 0, fs>>>(bc, w.summary_set[cur], st.flags_cur, w.nz_t, nullptr, w.list_adv, c_adv);
    ++launches;
  }
  FX_CK(cudaEventRecord(w.prep_join_ev, ps));
  // 3. velocity advection (dense; sparse mode: over the current flags)
  if (st.sparse) {
    if (st.solver_mode != 0) return FX_ERR_UNSUPPORTED;
    SpLists L{};
    L.list[0] = w.list_sp[SP_VSCR];
    L.count[0] = w.counters + 4 + SP_VSCR;
    L.nz[0] = w.nz_sp[SP_VSCR];
    {
      Timed tm(w, s, "sparse_lists");
      k_sp_lists<<<(nb + 255) / 256, 256, 0, s>>>(bc, nb, st.flags_cur, nullptr, L, nullptr);
      ++launches;
    }
    Timed tm(w, s, "sparse_advect_velocity");
    k_sp_advect_velocity<<<brick_grid_of(st, nb, BK_SP_ADVECT_VELOCITY), kBrickThreads, 0, s>>>(dm, bc, st.params, st.vcur, st.vscr, L.list[0], L.count[0]);
    ++launches;
  } else {
    Timed tm(w, s, "fused_advect_velocity");
    static const int zb = [] {
      const char* v = std::getenv("FENIX_ADV_Z");
      return v && *v ? std::atoi(v) : kAdvZ;
    }();
    const dim3 blk(32, 8, 1);
    auto grid = [&](int z) { return dim3((dm.w + 31) / 32, (dm.h + 7) / 8, (dm.d + z - 1) / z); };
    static const bool march = [] {
      const char* v = std::getenv("FENIX_ADV_MARCH");
      return !(v && *v == '0');
    }();
    int run = 0;
    if (march && std::getenv("FENIX_ADV_Z") == nullptr && march_runs(k_advect_velocity_march, dm, 32, 8, &run) == cudaSuccess) {
      k_advect_velocity_march<<<grid(run), blk, 0, s>>>(dm, st.params, st.vcur, st.vscr, w.vmax, run);
    } else switch (zb) {
      case 2: k_advect_velocity<2><<<grid(2), blk, 0, s>>>(dm, st.params, st.vcur, st.vscr, w.vmax); break;
      case 8: k_advect_velocity<8><<<grid(8), blk, 0, s>>>(dm, st.params, st.vcur, st.vscr, w.vmax); break;
      case 4: k_advect_velocity<4><<<grid(4), blk, 0, s>>>(dm, st.params, st.vcur, st.vscr, w.vmax); break;
      default: k_advect_velocity<kAdvZ><<<grid(kAdvZ), blk, 0, s>>>(dm, st.params, st.vcur, st.vscr, w.vmax); break;
    }
    ++launches;
  }
  // 4. scalar advection over the list
  if (taped) FX_CK(tape_vel(st.tape_a, st.vscr));
  FX_CK(cudaStreamWaitEvent(s, w.prep_join_ev, 0));
  FX_CK(cudaMemsetAsync(w.summary_t, 0, nb, s));
  {
    Timed tm(w, s, "fused_advect_scalars");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_advect_scalars<S><<<brick_grid_of(st, nb, BK_ADVECT_SCALARS), kBrickThreads, 0, s>>>(dm, bc, st.params, st.advect_mode,
                                                               static_cast<const typename Aos<S>::T*>(w.aos), st.vscr, st.flags_cur,
                                                               w.list_adv, c_adv, sset<S>(st.scratch), w.summary_t, w.nz_t);
    });
    ++launches;
  }
  // 5. flags of the advected set
  {
    Timed tm(w, s, "fused_dilate");
    k_dilate<<<(nb + 255) / 256, 256, 0, s>>>(bc, w.summary_t, st.flags_next, w.nz_t, w.nz_set[next], w.list_next, c_next);
    ++launches;
  }
  // Sparse mode: U = current | next flags; the lists of the curl, pressure and
  // velocity buffers (U plus the bricks where they may hold earlier values), and
  // the velocity scratch is non-zero in U only once buoyancy has run.
  auto sp_list = [&](int f) { return w.list_sp[f]; };
  auto sp_count = [&](int f) { return w.counters + 4 + f; };
  if (st.sparse) {
    SpLists L{};
    const int fams[3] = {SP_CURL, SP_PRESSURE, SP_VCUR};
    const bool due[3] = {st.vort_on, st.pressure_on, true};
    for (int k = 0; k < 3; ++k) {
      if (!due[k]) continue;
      L.list[k] = sp_list(fams[k]);
      L.count[k] = sp_count(fams[k]);
      L.nz[k] = w.nz_sp[fams[k]];
    }
    Timed tm(w, s, "sparse_lists");
    k_sp_lists<<<(nb + 255) / 256, 256, 0, s>>>(bc, nb, st.flags_cur, st.flags_next, L, w.nz_sp[SP_VSCR]);
    ++launches;
  }
  // 6. combustion T -> next set, 7. buoyancy
  FX_CK(cudaMemsetAsync(w.summary_set[next], 0, nb, s));
  {
    Timed tm(w, s, "fused_combustion");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_combustion<S><<<brick_grid_of(st, nb, BK_COMBUSTION), kBrickThreads, 0, s>>>(dm, bc, st.params, sset<S>(st.scratch), st.flags_next, w.list_next, c_next, w.nz_t,
                                                           w.summary_t, sset<S>(st.next), w.summary_set[next], w.nz_set[next]);
    });
    ++launches;
  }
  {
    Timed tm(w, s, "fused_buoyancy");
    by_storage(st.half_storage, [&](auto tag) {
      using S = typename decltype(tag)::type;
      k_buoyancy<S><<<brick_grid_of(st, nb, BK_BUOYANCY), kBrickThreads, 0, s>>>(dm, bc, st.params, sset<S>(st.next), st.flags_next, w.list_next, c_next, st.vscr);
    });
    ++launches;
  }
  if (taped) FX_CK(tape_vel(st.tape_b, st.vscr));
  // 8. vorticity confinement
  const VelField* vfinal = &st.vscr;
  if (st.vort_on && st.sparse) {
    {
      Timed tm(w, s, "sparse_vorticity");
      k_sp_vorticity<<<brick_grid_of(st, nb, BK_SP_VORTICITY), kBrickThreads, 0, s>>>(dm, bc, st.vscr, st.vort_mag, st.vort, st.debug_fields ? 1 : 0, sp_list(SP_CURL),
                                                          sp_count(SP_CURL));
      ++launches;
    }
    {
      Timed tm(w, s, "sparse_confinement");
      by_storage(st.half_storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        if (st.debug_fields)
          k_sp_confinement<S, true><<<brick_grid_of(st, nb, BK_SP_CONFINEMENT), kBrickThreads, 0, s>>>(dm, bc, st.params, st.vscr, st.vort_mag, sset<S>(st.next), w.nz_set[next],
                                                                         st.vscr2, st.conf_mag, sp_list(SP_CURL), sp_count(SP_CURL));
        else
          k_sp_confinement<S, false><<<brick_grid_of(st, nb, BK_SP_CONFINEMENT), kBrickThreads, 0, s>>>(dm, bc, st.params, st.vscr, st.vort_mag, sset<S>(st.next),
                                                                          w.nz_set[next], st.vscr2, st.conf_mag, sp_list(SP_CURL),
                                                                          sp_count(SP_CURL));
      });
      ++launches;
    }
    vfinal = &st.vscr2;
  } else if (st.vort_on) {
    {
      Timed tm(w, s, "fused_vorticity");
      static const bool v4 = [] {
        const char* e = std::getenv("FENIX_VORT_V4");
        return !(e && *e == '0');
      }();
      if (v4 && dm.w % 4 == 0 && dm.w >= 8)
        k_vorticity_v4<<<dim3((dm.w + 127) / 128, (dm.h + 7) / 8, dm.d), dim3(32, 8, 1), 0, s>>>(dm, st.vscr, st.vort_mag, st.vort,
                                                                                               st.debug_fields ? 1 : 0);
      else
        k_vorticity<<<dense_grid(dm), kDenseBlock, 0, s>>>(dm, st.vscr, st.vort_mag, st.vort, st.debug_fields ? 1 : 0);
      ++launches;
    }
    {
      Timed tm(w, s, "fused_confinement");
      by_storage(st.half_storage, [&](auto tag) {
        using S = typename decltype(tag)::type;
        if (st.debug_fields)
          k_confinement<S, true><<<dense_grid(dm), kDenseBlock, 0, s>>>(dm, bc, st.params, st.vscr, st.vort_mag, sset<S>(st.next),
                                                                        w.nz_set[next], st.vscr2, st.conf_mag);
        else
          k_confinement<S, false><<<dense_grid(dm), kDenseBlock, 0, s>>>(dm, bc, st.params, st.vscr, st.vort_mag, sset<S>(st.next),
                                                                         w.nz_set[next], st.vscr2, st.conf_mag);
      });
      ++launches;
    }
    vfinal = &st.vscr2;
  }
  // 9. pressure (PressureSolvePass.solve, :68-84) and 10. projection
  int last_p = st.last_p;
  if (st.pressure_on && st.solver_mode == 1) {
    const fx_status vs = vcycle_solve(w, st, *vfinal, launches, out);
    if (vs != FX_OK) return vs;
    Timed tm(w, s, "fused_project");
    FX_CK(cudaMemsetAsync(w.vmax, 0, sizeof(unsigned), s));
    FX_CK(launch_project(s, dm, *vfinal, st.lv[0].p[last_p], st.vcur, st.vel_mag, st.debug_on ? 1 : 0, w.vmax));
    ++launches;
  } else if (st.pressure_on && st.sparse) {
    // The reference schedule with the fine passes over the sparse lists (the
    // dense path's buffer ids and fusions; the restriction rides on the
    // divergence kernel).
    const int m = st.q[2], n = st.q[3];
    const LevelBuf& F = st.lv[0];
    const LevelBuf& M = st.lv[1];
    const LevelBuf& C = st.lv[2];
    last_p = (m & 1) ^ (n & 1);
    FX_CK(cudaMemsetAsync(M.p[0], 0, (size_t)M.dm.w * M.dm.h * M.dm.d * sizeof(float), s));
    FX_CK(cudaMemsetAsync(C.p[0], 0, (size_t)C.dm.w * C.dm.h * C.dm.d * sizeof(float), s));
    const bool prolong_live = (m & 1) == 0;
    const int nwrites = std::max(m, 0) + (m == 0 ? 1 : 0) + n;
    std::vector<float*> outs(nwrites);
    for (int i = nwrites; i-- > 0;)
      outs[i] = (i + 1 == nwrites) ? F.p[last_p] : (outs[i + 1] == F.p[last_p] ? F.p[last_p ^ 1] : F.p[last_p]);
    int wi = 0;
    const float* chain = nullptr;
    const uint32_t* pl = sp_list(SP_PRESSURE);
    const uint32_t* pc = sp_count(SP_PRESSURE);
    {
      Timed tm(w, s, "sparse_div_first_sweep");
      k_sp_div_first<<<brick_grid_of(st, nb, BK_SP_DIV_FIRST), kBrickThreads, 0, s>>>(dm, bc, *vfinal, F.div, m >= 1 ? outs[0] : nullptr, M.dm, M.div, pl, pc);
      ++launches;
    }
    if (m >= 1) chain = outs[wi++];
    const bool overlap = prolong_live && m >= 3;
    int mid = 0;
    if (prolong_live) FX_CK(lower_levels(overlap, mid));
    // The fine sweeps: TMA-staged where tensor maps of the buffers exist.
    static const bool use_tma = [] {
      const char* v = std::getenv("FENIX_SPARSE_TMA");
      return !(v && *v == '0');
    }();
    if (use_tma && (w.tmap_base[0] != F.p[0] || w.tmap_base[1] != F.p[1] || w.tmap_base[2] != F.div)) {
      w.tmaps_ok = field_tensor_map(&w.tmap_p[0], F.p[0], dm, 16, 10, 10) && field_tensor_map(&w.tmap_p[1], F.p[1], dm, 16, 10, 10) &&
                   field_tensor_map(&w.tmap_div, F.div, dm, 8, 8, 8);
      w.tmap_base[0] = F.p[0];
      w.tmap_base[1] = F.p[1];
      w.tmap_base[2] = F.div;
    }
    auto sweep = [&](const float* src, float* dst, const float* mid_p, const char* name) {
      Timed tm(w, s, name);
      if (use_tma && w.tmaps_ok && src) {
        const CUtensorMap& sm = src == F.p[0] ? w.tmap_p[0] : w.tmap_p[1];
        const uint32_t sweep_grid = brick_grid_of(st, nb, BK_SP_SWEEP);
        k_sp_sweep_tma<<<sweep_grid, kSpSweepThreads, 0, s>>>(sm, w.tmap_div, dm, bc, dst, M.dm, mid_p, pl, pc, w.dev_err, w.tma_wait_ns,
                                                              w.tma_extra_tx);
      } else {
        k_sp_sweep<<<brick_grid_of(st, nb, BK_SP_SWEEP), kBrickThreads, 0, s>>>(dm, bc, F.div, src, dst, M.dm, mid_p, 0, pl, pc);
      }
      ++launches;
    };
    for (int k = 2; k <= m; ++k) {
      const bool add = prolong_live && k == m;
      if (add && overlap) FX_CK(cudaStreamWaitEvent(s, w.join_ev, 0));
      sweep(chain, outs[wi], add ? M.p[mid] : nullptr, add ? "sparse_sweep_prolong" : "sparse_sweep");
      chain = outs[wi++];
    }
    if (m == 0) {
      Timed tm(w, s, "sparse_prolong_fine");
      k_sp_sweep<<<brick_grid_of(st, nb, BK_SP_PROLONG_FINE), kBrickThreads, 0, s>>>(dm, bc, F.div, nullptr, outs[wi], M.dm, M.p[mid], 1, pl, pc);
      chain = outs[wi++];
      ++launches;
    }
    for (int k = 1; k <= n; ++k) {
      sweep(chain, outs[wi], nullptr, "sparse_sweep");
      chain = outs[wi++];
    }
    {
      Timed tm(w, s, "sparse_project");
      k_sp_project<<<brick_grid_of(st, nb, BK_SP_PROJECT), kBrickThreads, 0, s>>>(dm, bc, *vfinal, F.p[last_p], st.vcur, sp_list(SP_VCUR), sp_count(SP_VCUR));
      ++launches;
    }
  } else if (st.pressure_on) {
    const int m = st.q[2], n = st.q[3];
    const LevelBuf& F = st.lv[0];
    const LevelBuf& M = st.lv[1];
    const LevelBuf& C = st.lv[2];
    const bool fuse_restrict = dm.w >= 16 && dm.h >= 16 && dm.d >= 16;
    // The reference's buffer ids: the pre-smoothed pressure ends in 'a' after an
    // even number of sweeps, and the post smoothing flips it once per sweep.
    const int fine_pre_id = m & 1;
    last_p = fine_pre_id ^ (n & 1);
    // Mid and coarse start from cleared pressureA (PressureSolvePass.clear). The
    // fine passes never read the cleared fine buffer, so it is not cleared.
    FX_CK(cudaMemsetAsync(M.p[0], 0, (size_t)M.dm.w * M.dm.h * M.dm.d * sizeof(float), s));
    FX_CK(cudaMemsetAsync(C.p[0], 0, (size_t)C.dm.w * C.dm.h * C.dm.d * sizeof(float), s));

    // Per-voxel plan. Fine writes in order: the first sweep (fused into the
    // divergence kernel), the remaining pre sweeps (the last one adds the
    // prolongation when the reference prolongs into it), the prolongation alone
    // when there is no pre sweep, then the post sweeps. The last write lands in
    // p[last]; going backwards the writes alternate with the other buffer, so no
    // sweep reads the buffer it writes.
    const bool prolong_live = (m & 1) == 0;  // odd m: the correction lands in a buffer never read
    const int nwrites = std::max(m, 0) + (m == 0 ? 1 : 0) + n;
    std::vector<float*> outs(nwrites);
    for (int i = nwrites; i-- > 0;)
      outs[i] = (i + 1 == nwrites) ? F.p[last_p] : (outs[i + 1] == F.p[last_p] ? F.p[last_p ^ 1] : F.p[last_p]);
    int wi = 0;
    const float* chain = nullptr;
    {
      Timed tm(w, s, "fused_div_first_sweep");
      FX_CK(lean_div_first(s, dm, *vfinal, F.div, m >= 1 ? outs[0] : nullptr, M.dm, M.div, fuse_restrict));
      ++launches;
    }
    if (m >= 1) chain = outs[wi++];
    if (!fuse_restrict) {
      Timed tm(w, s, "fused_restrict");
      plain_restrict(s, F.dm, M.dm, F.div, M.div);
      ++launches;
    }
    // The mid and coarse levels run on a second stream while the fine
    // pre-sweeps before the last one (which adds their prolongation) run here.
    const bool overlap = prolong_live && m >= 3;
    int mid = 0;
    if (prolong_live) FX_CK(lower_levels(overlap, mid));
    for (int k = 2; k <= m; ++k) {
      const bool add = prolong_live && k == m;
      if (add && overlap) FX_CK(cudaStreamWaitEvent(s, w.join_ev, 0));
      Timed tm(w, s, add ? "fused_sweep_prolong" : (overlap ? "fused_sweep_shared" : "fused_sweep"));
      // The sweeps beside the lower levels take part of each SM: at 64
      // registers four marching blocks fill an SM's register file, and the
      // second stream's small sweeps would otherwise wait for a whole sweep to
      // drain. Half the blocks (longer runs) cost the fine sweep less than the
      // lower chain gains (plume_256: 1.2673 -> 1.2398 ms per step).
      FX_CK(lean_sweep_variant(s, st.sweep_variant[0], dm, F.div, chain, outs[wi], M.dm, add ? M.p[mid] : nullptr,
                               overlap && !add ? march_share_pct() : 100));
      chain = outs[wi++];
      ++launches;
    }
    if (m == 0) {
      Timed tm(w, s, "fused_prolong_fine");
      FX_CK(lean_prolong_zero(s, dm, outs[wi], M.dm, M.p[mid]));
      chain = outs[wi++];
      ++launches;
    }
    for (int k = 1; k <= n; ++k) {
      Timed tm(w, s, "fused_sweep");
      FX_CK(lean_sweep_variant(s, st.sweep_variant[0], dm, F.div, chain, outs[wi], M.dm, nullptr));
      chain = outs[wi++];
      ++launches;
    }
    {
      Timed tm(w, s, "fused_project");
      FX_CK(cudaMemsetAsync(w.vmax, 0, sizeof(unsigned), s));
      FX_CK(launch_project(s, dm, *vfinal, F.p[last_p], st.vcur, st.vel_mag, st.debug_on ? 1 : 0, w.vmax));
      ++launches;
    }
  } else if (st.sparse) {
    Timed tm(w, s, "sparse_project");
    k_sp_project<<<brick_grid_of(st, nb, BK_SP_PROJECT), kBrickThreads, 0, s>>>(dm, bc, *vfinal, st.lv[0].p[last_p], st.vcur, sp_list(SP_VCUR), sp_count(SP_VCUR));
    ++launches;
  } else {
    // 10. projection with the pressure of the last solve (+ |v|)
    Timed tm(w, s, "fused_project");
    FX_CK(cudaMemsetAsync(w.vmax, 0, sizeof(unsigned), s));
    FX_CK(launch_project(s, dm, *vfinal, st.lv[0].p[last_p], st.vcur, st.vel_mag, st.debug_on ? 1 : 0, w.vmax));
    ++launches;
  }
  if (st.sparse) {
    // the sparse projection records no max |v|; |v| for the debug fields over the grid
    FX_CK(cudaMemsetAsync(w.vmax, 0xFF, sizeof(unsigned), s));
    if (st.debug_on) {
      Timed tm(w, s, "sparse_velocity_magnitude");
      k_sp_velocity_magnitude<<<(uint32_t)device_sm_count() * 8u, 256, 0, s>>>(dm, st.vcur, st.vel_mag);
      ++launches;
    }
  }
  // FP64 statistics of the solve: ||div||, ||div - A p|| (the V-cycle has them
  // already) and max |div u| of the projected velocity.
  if (st.pressure_on && (st.solver_mode == 1 || st.solver_norms)) {
    Timed tm(w, s, "fused_solver_norms");
    if (st.solver_mode == 0) {
      FX_CK(solver_norms(s, dm, st.lv[0].div, st.lv[0].p[last_p], st.vc.tol, w.solver));
      launches += 3;
    }
    FX_CK(max_divergence(s, dm, st.vcur, w.solver));
    ++launches;
  }
  FX_CK(cudaGetLastError());
  out.last_p = last_p;
  out.final_vscr_is_2 = st.vort_on;
  out.launches = launches;
  return FX_OK;
}

fx_status fused_check_device_error(FusedWork& w, cudaStream_t s) {
  uint32_t h = 0;
  if (cudaMemcpyAsync(&h, w.dev_err, sizeof h, cudaMemcpyDeviceToHost, s) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FX_ERR_CUDA;
  return h ? FX_ERR_TIMEOUT : FX_OK;
}

void fused_set_tma_test(FusedWork& w, uint64_t wait_ns, uint32_t extra_tx) {
  w.tma_wait_ns = wait_ns;
  w.tma_extra_tx = extra_tx;
  for (auto& kv : w.graphs) cudaGraphExecDestroy(kv.second.exec);  // the values are captured in the graphs
  w.graphs.clear();
}

fx_status fused_count_active(FusedWork& w, cudaStream_t s, const uint32_t* flags, uint32_t nb, uint32_t* out) {
  uint32_t* c = w.counters + 2;
  if (cudaMemsetAsync(c, 0, 4, s) != cudaSuccess) return FX_ERR_CUDA;
  k_count_flags<<<device_sm_count(), 256, 0, s>>>(flags, nb, c);
  uint32_t h = 0;
  if (cudaMemcpyAsync(&h, c, 4, cudaMemcpyDeviceToHost, s) != cudaSuccess) return FX_ERR_CUDA;
  if (cudaStreamSynchronize(s) != cudaSuccess) return FX_ERR_CUDA;
  *out = h;
  return FX_OK;
}

cudaError_t fused_accumulate_active(cudaStream_t s, Dims dm, uint3 bricks, const uint32_t* flags, unsigned long long* acc) {
  const uint32_t nb = bricks.x * bricks.y * bricks.z;
  const uint32_t blocks = std::min<uint32_t>((nb + 255) / 256, (uint32_t)device_sm_count());
  k_accumulate_active<<<blocks, 256, 0, s>>>(dm, bricks, flags, acc);
  return cudaGetLastError();
}

}  // namespace fx
