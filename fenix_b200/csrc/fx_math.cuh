// Device-side WGSL builtins and shared types for the fenix combustion-volume
// kernels.
//
// Every kernel evaluates the reference's f32 expressions in source order with no
// FMA contraction (the library is compiled with -fmad=false, IEEE division and
// square root). sin and cos use the project's pinned f32 algorithm below, which
// the CPU oracle implements with the same operations. As a result the CUDA step
// and the oracle agree bit for bit.
#pragma once

#include <cstdint>

#include <cuda_fp16.h>

#define FX_DEV __device__ __forceinline__

namespace fx {

// ---------------------------------------------------------------------------
// Pinned f32 sin/cos: the argument is reduced in double by a three-part
// Cody-Waite split of pi/2 (33 + 33 + 53 significant bits), then Taylor
// polynomials with coefficients 1/k! are evaluated in f32 on |r| <= pi/4 with
// fused multiply-adds.
// ---------------------------------------------------------------------------
FX_DEV float poly_sin(float r) {
  const float r2 = r * r;
  float p = fmaf(r2, -0x1.ae6456p-26f, 0x1.71de3ap-19f);
  p = fmaf(p, r2, -0x1.a01a02p-13f);
  p = fmaf(p, r2, 0x1.111112p-7f);
  p = fmaf(p, r2, -0x1.555556p-3f);
  const float r3 = r2 * r;
  return fmaf(r3, p, r);
}

FX_DEV float poly_cos(float r) {
  const float r2 = r * r;
  float p = fmaf(r2, 0x1.1eed8ep-29f, -0x1.27e4fcp-22f);
  p = fmaf(p, r2, 0x1.a01a02p-16f);
  p = fmaf(p, r2, -0x1.6c16c2p-10f);
  p = fmaf(p, r2, 0x1.555556p-5f);
  p = fmaf(p, r2, -0.5f);
  return fmaf(p, r2, 1.0f);
}

// Below |x| = 8192 the reduction runs in f32 (four fused multiply-adds with a
// Cody-Waite split of pi/2 into three 12-bit parts and the rounded rest; Cody and
// Waite, "Software Manual for the Elementary Functions", 1980): with |k| < 2^13
// the first two steps are exact and the split's error stays below 2^-50, so the
// reduced argument is within about one unit in the last place. Larger and
// non-finite arguments take the double reduction.
FX_DEV float pinned_quadrant(float r, int q) {
  const float s = (q & 1) ? poly_cos(r) : poly_sin(r);
  return (q & 2) ? -s : s;
}

FX_DEV float pinned_sincos(float x, int quadrant_offset) {
  if (fabsf(x) < 8192.0f) {
    const float kf = rintf(x * 0x1.45f306p-1f);
    float r = fmaf(-kf, 0x1.92p+0f, x);
    r = fmaf(-kf, 0x1.fb4p-12f, r);
    r = fmaf(-kf, 0x1.444p-24f, r);
    r = fmaf(-kf, 0x1.68c234p-39f, r);
    return pinned_quadrant(r, (int)kf + quadrant_offset);
  }
  const double xd = (double)x;
  const double k = rint(xd * 0x1.45f306dc9c883p-1);
  double r = fma(-k, 0x1.921fb544p+0, xd);
  r = fma(-k, 0x1.0b4611a6p-34, r);
  r = fma(-k, 0x1.3198a2e037073p-69, r);
  const double kq = k - 4.0 * floor(k * 0.25);
  int q = (int)kq;
  if (!(q >= 0 && q <= 3)) q = 0;
  q = (q + quadrant_offset) & 3;
  const float rf = (float)r;
  const float s = (q & 1) ? poly_cos(rf) : poly_sin(rf);
  return (q & 2) ? -s : s;
}

// The fast-arithmetic build (FX_FAST_MATH; libfenixcuda_fast.so, compiled with
// contraction into FMA and approximate division and square root) calls CUDA's
// sinf/cosf instead: not the oracle's bits, a stated error against f64.
#ifdef FX_FAST_MATH
FX_DEV float psin(float x) { return sinf(x); }
FX_DEV float pcos(float x) { return cosf(x); }
#else
FX_DEV float psin(float x) { return pinned_sincos(x, 0); }
FX_DEV float pcos(float x) { return pinned_sincos(x, 1); }
#endif

// ---------------------------------------------------------------------------
// WGSL builtins (spec formulas), written as the same comparisons and operations
// as the oracle so NaN and signed-zero behaviour matches too.
// ---------------------------------------------------------------------------
FX_DEV float mn(float a, float b) { return b < a ? b : a; }
FX_DEV float mx(float a, float b) { return a < b ? b : a; }
FX_DEV float clampv(float x, float lo, float hi) { return mn(mx(x, lo), hi); }
FX_DEV float clamp01(float x) { return clampv(x, 0.0f, 1.0f); }
FX_DEV float mixv(float a, float b, float t) { return a * (1.0f - t) + b * t; }
FX_DEV float fractv(float x) { return x - floorf(x); }
FX_DEV float stepv(float e, float x) { return x >= e ? 1.0f : 0.0f; }
// x / c rounded to nearest for a constant divisor c, by Markstein's correction
// of the product with r = RN(1/c) ("IA-64 and Elementary Functions", 2000):
// q0 = x r, q = fma(fma(-q0, c, x), r, q0). For every divisor smoothstepv meets
// in these kernels (the difference of its two literal edges), an exhaustive
// check over 2^-100 <= |x| <= 2^100 shows q equals the IEEE quotient
// (tests/native/divconst_check.c, run by tests/test_exact_division.py); other x
// take the IEEE division. With literal edges c and r fold at compile time.
FX_DEV float div_const(float x, float c) {
#ifdef FX_FAST_MATH
  return x * (1.0f / c);
#endif
  const float r = 1.0f / c;
  const float ax = fabsf(x);
  if (ax >= 0x1p-100f && ax <= 0x1p100f) {
    const float q0 = x * r;
    return fmaf(fmaf(-q0, c, x), r, q0);
  }
  return x / c;
}
// smoothstep with literal edges (their difference is a verified divisor).
FX_DEV float smoothstepv(float e0, float e1, float x) {
  const float t = clampv(div_const(x - e0, e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
// smoothstep with edges computed at run time (IEEE division).
FX_DEV float smoothstep_dyn(float e0, float e1, float x) {
  const float t = clampv((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
FX_DEV float length3(float x, float y, float z) { return sqrtf(x * x + y * y + z * z); }

// Grid geometry. Flat index x + W*(y + H*z) as in
// shaders/common/indexing.wgsl.ts:2-4 (32-bit: grids below 2^32 voxels).
struct Dims {
  uint32_t w, h, d;
};

FX_DEV uint32_t flat(const Dims& dm, uint32_t x, uint32_t y, uint32_t z) { return x + dm.w * (y + dm.h * z); }
FX_DEV uint32_t dec(uint32_t v) { return v == 0u ? 0u : v - 1u; }
FX_DEV uint32_t inc(uint32_t v, uint32_t m) { return min(v + 1u, m); }
// x / 6 rounded to nearest, for every float x, without a division. For |x| in
// [2^-125, FLT_MAX] the quotient is q0 = x * RN(1/6) corrected once by its exact
// residual (Markstein, "IA-64 and Elementary Functions", 2000):
// e = fma(-q0, 6, x), q = fma(e, RN(1/6), q0). Nonzero |x| below 2^-125 runs the
// same correction in f64, where x is far from the subnormal range, and rounds the
// f64 quotient to float once; rounding twice, first to 53 bits, gives the same
// float because 53 >= 2 * 24 + 2 (Figueroa, "When is double rounding
// innocuous?", 1995). For +-0, +-inf and NaN, q0 itself is the quotient. An
// exhaustive check over all 2^32 inputs compares the result with the IEEE
// quotient. Having no division keeps a slow path and its call out of the sweep
// kernels, whose pressure tails reach the subnormal range.
FX_DEV float div6(float x) {
#ifdef FX_FAST_MATH
  return x * 0x1.555556p-3f;
#endif
  const float ax = fabsf(x);
  const float r6 = 0x1.555556p-3f;  // RN(1/6)
  const float q0 = x * r6;
  if (ax >= 0x1p-125f && ax <= 0x1.fffffep127f) return fmaf(fmaf(-q0, 6.0f, x), r6, q0);
  if (!(ax > 0.0f && ax < 0x1p-125f)) return q0;  // +-0, +-inf, NaN
  const double r = 0x1.5555555555555p-3;  // RN(1/6) in f64
  const double xd = (double)x;
  const double p0 = xd * r;
  return (float)fma(fma(-p0, 6.0, xd), r, p0);
}

FX_DEV bool is_boundary(const Dims& dm, uint32_t x, uint32_t y, uint32_t z) {
  return x == 0u || y == 0u || z == 0u || x == dm.w - 1u || y == dm.h - 1u || z == dm.d - 1u;
}

// The 80-byte uniform of shaders/common/simulation-params.wgsl.ts:2-14, then two
// words the reference does not have: the step index and the rounding of binary16
// scalar stores (0 to nearest, 1 stochastic; see sr_half).
struct Params {
  float time, dt, prev_time, scalar_set;
  float wind[4];
  float gravity[4];
  float buoyancy, vorticity_strength, dx, world_size;
  float vmask[4];
  uint32_t step_index;
  uint32_t half_round;
};

// Stochastic rounding to binary16 (an extension for FP16 scalar storage).
// sr_draw is a 32-bit hash of a voxel index (one per voxel, shared by its store
// sites) plus the store site times 0x85EBCA77 plus the step index times
// 0x9E3779B9 (2^32 / golden ratio: a rank-1 sequence in time); sr_half
// rounds a finite |v| < 65504 to the binary16 value below it (toward zero) or
// the next one up, up when the distance from the lower one, in units of their
// spacing, exceeds the top 24 bits of r read as a fraction. Every operation is
// exact. A value that changes by less than half a binary16 spacing per step moves
// by the right amount on average instead of staying put, which is the bias of
// round-to-nearest on slowly decaying smoke. Other values round to nearest.
FX_DEV uint32_t sr_draw(uint32_t i, uint32_t site, uint32_t step) {
  uint32_t h = i * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h + site * 0x85EBCA77u + step * 0x9E3779B9u;
}

//
// Computed here without a division: in the binary16 normal range the distance
// from the lower value in units of the spacing is the 13 low significand bits of
// the float over 2^13, so "frac > u" is the integer test (bits << 11) > (r >> 8),
// and the upper value is the lower one's bit pattern plus 2^13 (a carry into the
// exponent gives the next binade's first value, as it should). Below 2^-14 the
// spacing is 2^-24 and a * 2^24 and its truncation are exact. The results equal
// the oracle's formulation bit for bit.
FX_DEV float sr_half(float v, uint32_t r) {
  const float a = fabsf(v);
  if (!(a < 65504.0f)) return __half2float(__float2half_rn(v));
  const uint32_t rb = r >> 8;
  if (a >= 0x1p-14f) {
    const uint32_t b = __float_as_uint(a);
    const uint32_t lo = b & ~0x1FFFu;
    const uint32_t m = ((b & 0x1FFFu) << 11) > rb ? lo + 0x2000u : lo;
    return copysignf(__uint_as_float(m), v);
  }
  const float q = a * 0x1p24f;
  const float t = truncf(q);
  const float u = (float)rb * 0x1p-24f;
  return copysignf(((q - t) > u ? t + 1.0f : t) * 0x1p-24f, v);
}

// Trilinear sampler of shaders/common/sampling-scalar.wgsl.ts:11-34. A NaN
// position is sent to 0, like the oracle.
FX_DEV float clamp_pos(float p, float hi) { return !(p > 0.0f) ? 0.0f : (p < hi ? p : hi); }

struct Tri {
  uint32_t i000, i100, i010, i110, i001, i101, i011, i111;
  float fx, fy, fz;
};

FX_DEV Tri tri_corners(const Dims& dm, float px, float py, float pz) {
  const float cx = clamp_pos(px, (float)(dm.w - 1u));
  const float cy = clamp_pos(py, (float)(dm.h - 1u));
  const float cz = clamp_pos(pz, (float)(dm.d - 1u));
  const float flx = floorf(cx), fly = floorf(cy), flz = floorf(cz);
  const uint32_t bx = (uint32_t)flx, by = (uint32_t)fly, bz = (uint32_t)flz;
  const uint32_t ux = min(bx + 1u, dm.w - 1u), uy = min(by + 1u, dm.h - 1u), uz = min(bz + 1u, dm.d - 1u);
  Tri t;
  t.fx = cx - flx;
  t.fy = cy - fly;
  t.fz = cz - flz;
  const uint32_t row_b = dm.w * (by + dm.h * bz), row_uy = dm.w * (uy + dm.h * bz);
  const uint32_t row_uz = dm.w * (by + dm.h * uz), row_uyz = dm.w * (uy + dm.h * uz);
  t.i000 = bx + row_b;
  t.i100 = ux + row_b;
  t.i010 = bx + row_uy;
  t.i110 = ux + row_uy;
  t.i001 = bx + row_uz;
  t.i101 = ux + row_uz;
  t.i011 = bx + row_uyz;
  t.i111 = ux + row_uyz;
  return t;
}

FX_DEV float tri_interp(const float* __restrict__ f, const Tri& c) {
  const float x00 = mixv(__ldg(f + c.i000), __ldg(f + c.i100), c.fx);
  const float x10 = mixv(__ldg(f + c.i010), __ldg(f + c.i110), c.fx);
  const float x01 = mixv(__ldg(f + c.i001), __ldg(f + c.i101), c.fx);
  const float x11 = mixv(__ldg(f + c.i011), __ldg(f + c.i111), c.fx);
  return mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
}

// ---------------------------------------------------------------------------
// Emitter helpers: shaders/passes/inject-source-common.wgsl.ts. A source is 32
// floats (sim/emitters/packEmitterSources.ts:13-77).
// ---------------------------------------------------------------------------
struct Src {
  float px, py, pz, radius, start, duration, yd, yt, yf, speed, mode, falloff, tight, dirx, diry, dirz;
  float noise_scale, noise_mix, intensity, kind, seed;
};

FX_DEV Src load_src(const float* __restrict__ s) {
  Src o;
  o.px = s[0]; o.py = s[1]; o.pz = s[2]; o.radius = s[3];
  o.start = s[4]; o.duration = s[5];
  o.yd = s[8]; o.yt = s[9]; o.yf = s[10];
  o.speed = s[12]; o.mode = s[13]; o.falloff = s[14]; o.tight = s[15];
  o.dirx = s[16]; o.diry = s[17]; o.dirz = s[18];
  o.noise_scale = s[20]; o.noise_mix = s[21]; o.intensity = s[22];
  o.kind = s[28]; o.seed = s[29];
  return o;
}

FX_DEV float active_gate(const Params& P, const Src& s) {
  const float age = P.time - s.start;
  return stepv(0.0f, age) * stepv(age, s.duration);
}
FX_DEV float source_age(const Params& P, const Src& s) { return mx(P.time - s.start, 0.0f); }
FX_DEV float source_duration(const Src& s) { return mx(s.duration, 0.0001f); }
FX_DEV float sphere_falloff(float dist, float radius, float falloff) {
  const float t = clampv(1.0f - dist / mx(radius, 0.0001f), 0.0f, 1.0f);
  return mixv(stepv(0.0f, t - 0.0001f), t * t, falloff);
}
FX_DEV float source_feather(const Params& P, float r) {
  const float voxel_width = P.dx / mx(P.world_size, 0.0001f);
  return mx(r * 0.24f, voxel_width * 3.0f);
}
FX_DEV float source_outer_limit(const Params& P, float r) { return r + source_feather(P, r); }
// The emitter hash fract(sin(dot(p, (127.1, 311.7, 74.7))) * 43758.5453) turns
// the last bit of its sine into about 2^-9 of output, so it is always evaluated
// with the pinned sine and with products and sums that are never contracted into
// FMA (the _rn intrinsics): the fast-arithmetic build keeps the same hash values
// (the same lattice noise) as the parity build and the oracle.
FX_DEV float hash31(float x, float y, float z) {
  const float d = __fadd_rn(__fadd_rn(__fmul_rn(x, 127.1f), __fmul_rn(y, 311.7f)), __fmul_rn(z, 74.7f));
  const float v = __fmul_rn(pinned_sincos(d, 0), 43758.5453123f);
  return __fsub_rn(v, floorf(v));
}
FX_DEV float value_noise3(float px, float py, float pz) {
  const float cx = floorf(px), cy = floorf(py), cz = floorf(pz);
  const float fx = fractv(px), fy = fractv(py), fz = fractv(pz);
  const float ux = fx * fx * (3.0f - 2.0f * fx);
  const float uy = fy * fy * (3.0f - 2.0f * fy);
  const float uz = fz * fz * (3.0f - 2.0f * fz);
  const float cx1 = cx + 1.0f, cy1 = cy + 1.0f, cz1 = cz + 1.0f;
  return mixv(mixv(mixv(hash31(cx, cy, cz), hash31(cx1, cy, cz), ux), mixv(hash31(cx, cy1, cz), hash31(cx1, cy1, cz), ux), uy),
              mixv(mixv(hash31(cx, cy, cz1), hash31(cx1, cy, cz1), ux), mixv(hash31(cx, cy1, cz1), hash31(cx1, cy1, cz1), ux), uy),
              uz);
}
FX_DEV float emitter_noise(float px, float py, float pz, float scale, float seed) {
  const float s = mx(scale, 0.1f);
  return value_noise3(px * s + seed * 0.137f, py * s + seed * 0.271f, pz * s + (-seed) * 0.193f);
}
FX_DEV float eruptive_falloff(const Params& P, float px, float py, float pz, float dist, const Src& s, float falloff) {
  const float target = s.radius;
  const float growth_seconds = clampv(target * 5.5f, 0.1f, 0.75f);
  const float age = source_age(P, s);
  const float growth = smoothstepv(0.0f, 1.0f, clampv(age / growth_seconds, 0.0f, 1.0f));
  const float feather = source_feather(P, target);
  const float seed = s.seed;
  const float coarse = emitter_noise(px + age * 0.17f, py + (-age) * 0.11f, pz + age * 0.07f, 6.0f, seed);
  const float fine = emitter_noise(px + (-age) * 0.33f, py + age * 0.21f, pz + (-age) * 0.15f, 18.0f, seed + 41.0f);
  const float lobe = clampv(coarse * 0.72f + fine * 0.28f, 0.0f, 1.0f);
  const float reach = target * growth * mixv(0.62f, 1.0f, smoothstepv(0.2f, 0.92f, lobe));
  const float front = 1.0f - smoothstep_dyn(reach - feather, reach + feather, dist);
  const float core_radius = mx(target * (0.18f + growth * 0.38f), feather);
  const float core = sphere_falloff(dist, core_radius, falloff) * (1.0f - growth * 0.35f);
  const float body = sphere_falloff(dist, mx(reach + feather, feather), falloff) * front;
  return clampv(mx(core, body) * mixv(0.72f, 1.2f, lobe), 0.0f, 1.0f);
}
FX_DEV void turbulent_dir(float px, float py, float pz, float seed, float& ox, float& oy, float& oz) {
  const float nx = emitter_noise(px, py, pz, 4.0f, seed);
  const float ny = emitter_noise(px, py, pz, 4.0f, seed + 17.3f);
  const float nz = emitter_noise(px, py, pz, 4.0f, seed + 31.7f);
  const float vx = nx - 0.5f, vy = ny - 0.5f, vz = nz - 0.5f;
  const float l = length3(vx, vy, vz);
  ox = vx / l;
  oy = vy / l;
  oz = vz / l;
}

// The per-voxel emitter loops of inject-scalar.wgsl.ts:44-65,
// inject-velocity.wgsl.ts:56-95 and inject-igniter.wgsl.ts:43-62.
//
// These and the per-voxel source terms below are templates over the number
// type of the state values: the kernels use float; the adjoint kernels evaluate
// the same code with dual numbers (fx_dual.cuh) to obtain its local Jacobian.
template <class T>
FX_DEV void inject_scalar_voxel(const Params& P, const float* __restrict__ src, uint32_t nsrc, float px, float py, float pz, T& dd,
                                T& tt, T& ff) {
  for (uint32_t e = 0; e < nsrc; ++e) {
    const Src s = load_src(src + 32u * e);
    const bool burst = s.kind == 3.0f;
    if (!(s.kind == 0.0f || burst)) continue;
    if (active_gate(P, s) < 0.0001f) continue;
    const float ox = px - s.px, oy = py - s.py, oz = pz - s.pz;
    const float dist = length3(ox, oy, oz);
    const float radius = s.radius;
    if (dist > (burst ? source_outer_limit(P, radius) : radius)) continue;
    const float weight = burst ? eruptive_falloff(P, px, py, pz, dist, s, 0.5f) : sphere_falloff(dist, radius, 0.5f);
    const float noise = emitter_noise(px, py, pz, s.noise_scale, s.seed);
    const float modulation = mixv(1.0f, noise, clampv(s.noise_mix, 0.0f, 1.0f));
    const float release = burst ? 1.0f / source_duration(s) : 1.0f;
    const float contribution = weight * modulation * release * P.dt;
    dd = clamp01(dd + s.yd * contribution);
    tt = clamp01(tt + s.yt * contribution);
    ff = clamp01(ff + s.yf * contribution);
  }
}

template <class T>
FX_DEV void inject_velocity_voxel(const Params& P, const float* __restrict__ src, uint32_t nsrc, float px, float py, float pz, T& vx,
                                  T& vy, T& vz) {
  for (uint32_t e = 0; e < nsrc; ++e) {
    const Src s = load_src(src + 32u * e);
    const bool burst = s.kind == 3.0f;
    if (!(s.kind == 1.0f || burst)) continue;
    if (active_gate(P, s) < 0.0001f) continue;
    const float ox = px - s.px, oy = py - s.py, oz = pz - s.pz;
    const float dist = length3(ox, oy, oz);
    const float radius = s.radius;
    if (dist > (burst ? source_outer_limit(P, radius) : radius)) continue;
    const float weight = burst ? eruptive_falloff(P, px, py, pz, dist, s, s.falloff) : sphere_falloff(dist, radius, s.falloff);
    const float speed = s.speed;
    float dx = 0.0f, dy = 0.0f, dz = 0.0f;
    if (burst) {
      float rx = 0.0f, ry = 1.0f, rz = 0.0f;
      if (dist > 0.0001f) {
        const float m = mx(dist, 0.0001f);
        rx = ox / m;
        ry = oy / m;
        rz = oz / m;
      }
      const float t = P.time;
      float tx, ty, tz;
      turbulent_dir(px + t * 0.19f, py + (-t) * 0.13f, pz + t * 0.07f, s.seed + 83.0f, tx, ty, tz);
      const float bx = rx * speed + 0.0f + tx * s.tight;
      const float by = ry * speed + s.mode + ty * s.tight;
      const float bz = rz * speed + 0.0f + tz * s.tight;
      const float dur = source_duration(s);
      vx += bx * weight * P.dt / dur;
      vy += by * weight * P.dt / dur;
      vz += bz * weight * P.dt / dur;
      continue;
    } else if (s.mode == 0.0f) {
      dy = 1.0f;
      if (dist > 0.0001f) {
        const float m = mx(dist, 0.0001f);
        dx = ox / m;
        dy = oy / m;
        dz = oz / m;
      }
    } else if (s.mode == 1.0f) {
      dy = 1.0f;
      if (s.dirx * s.dirx + s.diry * s.diry + s.dirz * s.dirz > 0.0001f) {
        const float l = length3(s.dirx, s.diry, s.dirz);
        dx = s.dirx / l;
        dy = s.diry / l;
        dz = s.dirz / l;
      }
    } else {
      turbulent_dir(px, py, pz, s.seed, dx, dy, dz);
    }
    const float fx = dx * speed * weight * P.dt;
    const float fy = dy * speed * weight * P.dt;
    const float fz = dz * speed * weight * P.dt;
    const float tightness = clampv(s.tight, 0.0f, 1.0f) * weight;
    vx = mixv(vx + fx, dx * speed, tightness);
    vy = mixv(vy + fy, dy * speed, tightness);
    vz = mixv(vz + fz, dz * speed, tightness);
  }
}

FX_DEV float speed_limit(const Params& P) { return 80.0f / mx(P.dx, 0.001f); }

template <class T>
FX_DEV void inject_igniter_voxel(const Params& P, const float* __restrict__ src, uint32_t nsrc, float px, float py, float pz, T fuel,
                                 T& rr, T& tt) {
  for (uint32_t e = 0; e < nsrc; ++e) {
    const Src s = load_src(src + 32u * e);
    const bool burst = s.kind == 3.0f;
    if (!(s.kind == 2.0f || burst)) continue;
    if (active_gate(P, s) < 0.0001f) continue;
    const float dist = length3(px - s.px, py - s.py, pz - s.pz);
    const float radius = s.radius;
    if (dist > (burst ? source_outer_limit(P, radius) : radius)) continue;
    const float weight = burst ? eruptive_falloff(P, px, py, pz, dist, s, 0.6f) : sphere_falloff(dist, radius, 0.6f);
    const float intensity = s.intensity;
    const T fuel_avail = burst ? T(1.0f) : smoothstepv(0.02f, 0.22f, fuel);
    const float release = burst ? 1.0f / source_duration(s) : 1.6f;
    const T seed = intensity * weight * fuel_avail * P.dt * release;
    rr = clamp01(rr + seed);
    tt = clamp01(tt + intensity * weight * P.dt * 4.0f);
  }
}

// ---------------------------------------------------------------------------
// Per-voxel source terms shared by the plain and fused kernels.
// ---------------------------------------------------------------------------

// scalarThermalNoise, advect-scalar-maccormack.wgsl.ts:52-57.
// thermal_noise's inner sine, which depends on y only.
FX_DEV float thermal_noise_ysin(const Params& P, float py) {
  const float y = py + (-P.time) * 3.1f;
  return psin(y * 0.079f);
}
// thermal_noise given its inner sine (thermal_noise_ysin(P, py)).
FX_DEV float thermal_noise_ys(const Params& P, float px, float py, float pz, float ysin) {
  const float t = P.time;
  const float x = px + t * 1.7f, y = py + (-t) * 3.1f, z = pz + t * 1.1f;
  const float a = 0.5f + 0.5f * psin(x * 0.097f + y * 0.061f + z * -0.083f);
  const float b = 0.5f + 0.5f * psin(x * -0.043f + y * 0.137f + z * 0.071f + ysin * 1.6f);
  return clampv(a * 0.58f + b * 0.42f, 0.0f, 1.0f);
}
FX_DEV float thermal_noise(const Params& P, float px, float py, float pz) {
  const float t = P.time;
  const float x = px + t * 1.7f, y = py + (-t) * 3.1f, z = pz + t * 1.1f;
  const float a = 0.5f + 0.5f * psin(x * 0.097f + y * 0.061f + z * -0.083f);
  const float b = 0.5f + 0.5f * psin(x * -0.043f + y * 0.137f + z * 0.071f + psin(y * 0.079f) * 1.6f);
  return clampv(a * 0.58f + b * 0.42f, 0.0f, 1.0f);
}

// The decay block of advect-scalar-maccormack.wgsl.ts:80-100.
template <class T>
FX_DEV void decay_scalars(const Params& P, float ny, float noise, T& density, T& temperature, T& fuel, T& reaction) {
  const float dt = P.dt;
  const T hot = smoothstepv(0.22f, 0.78f, temperature + fuel * 0.2f + reaction * 0.26f);
  const T cooling_pocket = smoothstepv(0.44f, 0.9f, 1.0f - noise) * smoothstepv(0.08f, 0.74f, density) * (1.0f - hot * 0.72f);
  const T cooling = dt * (0.016f + ny * 0.052f) * mixv(1.28f, 0.58f, hot) * mixv(0.86f, 1.9f, cooling_pocket);
  const float smoke_loss = dt * (0.008f + ny * 0.026f) * mixv(0.75f, 1.38f, noise);
  const T cold_breakup = dt * density * (1.0f - smoothstepv(0.2f, 0.86f, hot)) * smoothstepv(0.18f, 0.72f, density) *
                         smoothstepv(0.34f, 0.92f, noise) * 0.34f;
  const T clearing = dt * density * hot * mixv(0.1f, 0.72f, noise);
  const T d = clamp01(mx(0.0f, density * (1.0f - smoke_loss) - clearing - cold_breakup));
  const T t = clamp01(mx(0.0f, temperature - cooling));
  const T f = clamp01(mx(0.0f, fuel - dt * mixv(0.012f, 0.034f, noise)));
  const T r = clamp01(mx(0.0f, reaction - dt * mixv(0.46f, 0.82f, noise)));
  density = d;
  temperature = t;
  fuel = f;
  reaction = r;
}

// thermalCluster, combustion-update.wgsl.ts:27-34.
// thermal_cluster's inner sine, which depends on y only.
FX_DEV float thermal_cluster_ysin(const Params& P, float py) {
  const float y = py + P.time * 5.2f;
  return psin(y * 0.057f);
}
// thermal_cluster given its inner sine (thermal_cluster_ysin(P, py)).
FX_DEV float thermal_cluster_ys(const Params& P, float px, float py, float pz, float ysin) {
  const float t = P.time;
  const float x = px + t * 2.2f, y = py + t * 5.2f, z = pz + (-t) * 1.7f;
  const float body = 0.5f + 0.5f * psin(x * 0.071f + y * 0.093f + z * -0.064f + ysin * 1.8f);
  const float pocket = 0.5f + 0.5f * psin(x * 0.143f + y * -0.081f + z * 0.119f + psin(x * 0.11f + z * 0.07f) * 1.2f);
  const float rising = 0.5f + 0.5f * psin(x * 0.18f + y * 0.13f - z * 0.16f + t * 1.4f);
  return clampv(body * 0.46f + pocket * 0.34f + rising * 0.2f, 0.0f, 1.0f);
}
FX_DEV float thermal_cluster(const Params& P, float px, float py, float pz) {
  const float t = P.time;
  const float x = px + t * 2.2f, y = py + t * 5.2f, z = pz + (-t) * 1.7f;
  const float body = 0.5f + 0.5f * psin(x * 0.071f + y * 0.093f + z * -0.064f + psin(y * 0.057f) * 1.8f);
  const float pocket = 0.5f + 0.5f * psin(x * 0.143f + y * -0.081f + z * 0.119f + psin(x * 0.11f + z * 0.07f) * 1.2f);
  const float rising = 0.5f + 0.5f * psin(x * 0.18f + y * 0.13f - z * 0.16f + t * 1.4f);
  return clampv(body * 0.46f + pocket * 0.34f + rising * 0.2f, 0.0f, 1.0f);
}

// localHotGas of combustion-update.wgsl.ts:36-40.
template <class T>
FX_DEV T comb_hot(T t, T f, T r) {
  return clampv(t * 1.55f + f * 0.26f + r * 0.44f, 0.0f, 1.0f);
}

// combustion-update.wgsl.ts:52-92, given the six neighbour hot-gas values summed
// in the reference order (+x, -x, +y, -y, +z, -z).
template <class T>
FX_DEV void combustion_voxel_c(const Params& P, float cluster, float ny, T neighbor_sum, T& d, T& t, T& f, T& r);

template <class T>
FX_DEV void combustion_voxel(const Params& P, uint32_t x, uint32_t y, uint32_t z, float ny, T neighbor_sum, T& d, T& t, T& f, T& r) {
  combustion_voxel_c(P, thermal_cluster(P, (float)x, (float)y, (float)z), ny, neighbor_sum, d, t, f, r);
}

// combustion_voxel given the voxel's thermal cluster value.
template <class T>
FX_DEV void combustion_voxel_c(const Params& P, float cluster, float ny, T neighbor_sum, T& d, T& t, T& f, T& r) {
  const float dt = P.dt;
  const T neighbor = neighbor_sum * 0.16666667f;
  const T local_before = comb_hot(t, f, r);
  const T radiative =
      mx(neighbor - local_before * 0.55f, 0.0f) * smoothstepv(0.04f, 0.76f, d) * (0.45f + (1.0f - cluster) * 0.55f) * dt * 2.6f;
  const T hot_pocket = smoothstepv(0.58f, 0.92f, cluster + r * 0.22f);
  const T cooling_pocket =
      smoothstepv(0.42f, 0.82f, 1.0f - cluster) * smoothstepv(0.08f, 0.68f, d) * (1.0f - smoothstepv(0.54f, 0.94f, r));
  const T ignition = smoothstepv(0.1f, 0.55f, t);
  const T burn = mn(f, f * ignition * dt * mixv(4.2f, 8.6f, hot_pocket));
  const T hot_soot = smoothstepv(0.24f, 0.88f, t + r * 0.2f) * smoothstepv(0.36f, 0.9f, 1.0f - cluster + d * 0.18f);
  const T smoke_yield = burn * mixv(0.16f, 0.58f, cooling_pocket + (1.0f - ignition) * 0.5f + hot_soot * 0.45f);
  const T hot_cooling = mixv(1.3f, 0.62f, hot_pocket);
  const T heat_loss = dt * (0.018f + ny * 0.052f) * hot_cooling * mixv(1.0f, 2.25f, cooling_pocket);
  const T density_loss = dt * d * (0.02f + ny * 0.07f);
  const T clearing = d * smoothstepv(0.18f, 0.82f, t + r * 0.22f + f * 0.1f) * dt * mixv(0.55f, 2.45f, hot_pocket);
  const T cooling_smoke = d * t * (cooling_pocket + hot_soot * 0.32f) * dt * 0.16f;
  const T reaction_decay = r * (1.0f - dt * mixv(0.68f, 0.22f, hot_pocket));
  const T nf = clamp01(f - burn);
  const T nt = clamp01(t + burn * mixv(2.1f, 3.25f, hot_pocket) + radiative - heat_loss);
  const T nd = clamp01(mx(0.0f, d + smoke_yield + cooling_smoke - density_loss - clearing * 0.72f));
  const T nr = clamp01(mx(reaction_decay, burn * mixv(4.0f, 7.5f, hot_pocket) + radiative * 1.8f));
  f = nf;
  t = nt;
  d = nd;
  r = nr;
}

// hotGasAt of apply-buoyancy.wgsl.ts:31-35.
template <class T>
FX_DEV T buoy_hot(T t, T r) {
  return clampv(t * 1.0f + r * 0.85f, 0.0f, 1.0f);
}

// apply-buoyancy.wgsl.ts:47-109 given the voxel's own density/hot gas, the
// central differences of hot gas (tg*) and density (dg*), and its velocity.
// The terms of buoyancy_voxel that depend on x and y only (a brick thread's two
// voxels share them).
struct BuoyXY {
  float ny, shear_y, s1, s3;
};
FX_DEV BuoyXY buoy_xy(const Params& P, const Dims& dm, uint32_t x, uint32_t y) {
  const float t = P.time;
  const float fxv = (float)x, fyv = (float)y;
  BuoyXY o;
  o.ny = ((float)y + 0.5f) / (float)dm.h;
  o.shear_y = psin(fyv * 0.073f + t * 0.9f);
  o.s1 = psin(fyv * 0.117f + t * 1.9f);
  o.s3 = pcos(fxv * 0.061f + fyv * 0.049f - t * 1.6f);
  return o;
}

template <class T>
FX_DEV void buoyancy_voxel_xy(const Params& P, const Dims& dm, const BuoyXY& q, uint32_t x, uint32_t y, uint32_t z, T d, T hot_gas, T tgx,
                              T tgy, T tgz, T dgx, T dgy, T dgz, T& vx, T& vy, T& vz);

template <class T>
FX_DEV void buoyancy_voxel(const Params& P, const Dims& dm, uint32_t x, uint32_t y, uint32_t z, T d, T hot_gas, T tgx, T tgy, T tgz,
                           T dgx, T dgy, T dgz, T& vx, T& vy, T& vz) {
  buoyancy_voxel_xy(P, dm, buoy_xy(P, dm, x, y), x, y, z, d, hot_gas, tgx, tgy, tgz, dgx, dgy, dgz, vx, vy, vz);
}

// apply-buoyancy.wgsl.ts:37-110 given the voxel's (x, y) terms.
template <class T>
FX_DEV void buoyancy_voxel_xy(const Params& P, const Dims& dm, const BuoyXY& q, uint32_t x, uint32_t y, uint32_t z, T d, T hot_gas, T tgx,
                              T tgy, T tgz, T dgx, T dgy, T dgz, T& vx, T& vy, T& vz) {
  const float dt = P.dt;
  const float b = P.buoyancy;
  const float response = b * (1.0f + smoothstepv(6.0f, 24.0f, fabsf(b)) * 0.38f);
  const T lift = hot_gas * response;
  const float gw = P.gravity[3];
  const T gfx = P.gravity[0] * d * gw, gfy = P.gravity[1] * d * gw, gfz = P.gravity[2] * d * gw;
  const T entrain = d * smoothstepv(0.04f, 0.3f, hot_gas);
  const float ny = q.ny;
  const float t = P.time;
  const float fxv = (float)x, fzv = (float)z;
  const float shear = q.shear_y * 0.35f + psin(fxv * 0.041f - fzv * 0.052f + t * 0.43f) * 0.22f;
  const float ww = P.wind[3];
  const float wx = P.wind[0], wy = P.wind[1], wz = P.wind[2];
  const T amount = ww * (0.18f + d * 0.55f + ny * 0.45f);
  const T windx = wx * amount + (-wz) * amount * shear;
  const T windy = wy * amount + 0.0f * amount * shear;
  const T windz = wz * amount + wx * amount * shear;
  const T dgl = mx(length3(dgx, dgy, dgz), 0.0001f);
  const T cold = d * (1.0f - smoothstepv(0.12f, 0.72f, hot_gas));
  const T breakup = smoothstepv(0.008f, 0.06f, dgl) * cold;
  const float s1 = q.s1;
  const float s2 = psin(fxv * 0.071f - fzv * 0.083f + t * 1.35f) * 0.35f;
  const float s3 = q.s3;
  const float sl = length3(s1, s2, s3);
  const float shx = s1 / sl, shy = s2 / sl, shz = s3 / sl;
  const T collapse = d * (1.0f - smoothstepv(0.16f, 0.64f, hot_gas));
  const T drag = d * smoothstepv(0.03f, 0.45f, hot_gas);
  const float keep = 1.0f - dt * 0.08f;
  vx = vx * keep;
  vy = vy * keep;
  vz = vz * keep;
  vx += windx * dt; vy += windy * dt; vz += windz * dt;
  vx += gfx * dt; vy += gfy * dt; vz += gfz * dt;
  const float tk = 3.2f + fabsf(b) * 0.08f;
  vx += tgx * collapse * dt * tk; vy += tgy * collapse * dt * tk; vz += tgz * collapse * dt * tk;
  vx += (-dgx) / dgl * breakup * dt * 2.8f;
  vy += (-dgy) / dgl * breakup * dt * 2.8f;
  vz += (-dgz) / dgl * breakup * dt * 2.8f;
  const T sk = 0.72f + breakup * 2.4f;
  vx += shx * cold * dt * sk; vy += shy * cold * dt * sk; vz += shz * cold * dt * sk;
  vx += wx * cold * ww * dt * 0.9f; vy += wy * cold * ww * dt * 0.9f; vz += wz * cold * ww * dt * 0.9f;
  vx += 0.0f * dt; vy += drag * response * 0.55f * dt; vz += 0.0f * dt;
  const float lim = speed_limit(P);
  vy = clampv(vy + (lift + entrain * response * 0.24f) * dt, -lim, lim);
  if (x == 0u || x == dm.w - 1u || z == 0u || z == dm.d - 1u) {
    vx = 0.0f;
    vz = 0.0f;
  }
  if (y == 0u) vy = mx(vy, 0.0f);
}

// apply-vorticity-confinement.wgsl.ts:42-65 given the |w| central differences,
// the voxel's w, |w| and scalars: applies the force to v and returns it in f.
template <class T>
FX_DEV void confinement_force(const Params& P, T gx, T gy, T gz, T wx, T wy, T wz, T wmag, T d, T t, T r, T& vx, T& vy, T& vz, T& fx, T& fy,
                              T& fz) {
  const T gl = mx(length3(gx, gy, gz), 0.0001f);
  const T nx = gx / gl, ny = gy / gl, nz = gz / gl;
  const T hot_gas = clampv(t + r * 0.85f, 0.0f, 1.0f);
  const T mask = clampv(P.vmask[0] + smoothstepv(0.02f, 0.38f, wmag) * P.vmask[1] + smoothstepv(0.04f, 0.7f, hot_gas) * P.vmask[2] +
                            smoothstepv(0.04f, 0.65f, d) * P.vmask[3],
                        0.0f, 4.0f);
  const float k = P.vorticity_strength;
  fx = (ny * wz - nz * wy) * k * mask * 1.45f;
  fy = (nz * wx - nx * wz) * k * mask * 1.45f;
  fz = (nx * wy - ny * wx) * k * mask * 1.45f;
  const float lim = speed_limit(P);
  vx = clampv(vx + fx * P.dt, -lim, lim);
  vy = clampv(vy + fy * P.dt, -lim, lim);
  vz = clampv(vz + fz * P.dt, -lim, lim);
}

// The same, returning |F|.
template <class T>
FX_DEV T confinement_voxel(const Params& P, T gx, T gy, T gz, T wx, T wy, T wz, T wmag, T d, T t, T r, T& vx, T& vy, T& vz) {
  T fx, fy, fz;
  confinement_force(P, gx, gy, gz, wx, wy, wz, wmag, d, t, r, vx, vy, vz, fx, fy, fz);
  return length3(fx, fy, fz);
}

// The same, without |F|.
template <class T>
FX_DEV void confinement_voxel_v(const Params& P, T gx, T gy, T gz, T wx, T wy, T wz, T wmag, T d, T t, T r, T& vx, T& vy, T& vz) {
  T fx, fy, fz;
  confinement_force(P, gx, gy, gz, wx, wy, wz, wmag, d, t, r, vx, vy, vz, fx, fy, fz);
}

}  // namespace fx
