// Volume raymarch of the simulation's render buffers into a headless RGBA
// device buffer: the reference's VolumeRaymarchPass
// (render/passes/createVolumeRaymarchPass.ts), whose fragment shader
// (:300-726) runs here as one CUDA thread per pixel.
//
// The reference draws a full-screen triangle into a cleared target with
// premultiplied blending (one, one-minus-src-alpha), so a pixel is the fragment
// output or (0, 0, 0, 0) where the fragment discards. The fragment's uv is the
// rasterizer's interpolation at the pixel centre: u = (x + 0.5) / W,
// v = 1 - (y + 0.5) / H, row 0 at the top.
//
// Arithmetic: f32 in the shader's operation order (no contraction), WGSL
// builtins by their spec formulas, round() half to even, float->u32 conversions
// saturating. exp and pow use the project's pinned algorithms below (FP64
// cores, rounded once to f32), which the CPU oracle implements with the same
// operations, so images agree bit for bit.
#include <cuda_fp16.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <string>

#include "../../include/fenix_cuda.h"
#include "fx_math.cuh"

namespace fx {

void set_last_error(const std::string& msg);

// The simulation state a render reads (fx_sim.cu).
struct SimView {
  Dims dm;
  uint3 bricks;
  const void* f[4];  // density, temperature, fuel, reaction of the current set
  const uint32_t* flags;
  bool half;
  cudaStream_t stream;
  int device;
};
bool sim_view(fx_sim* s, SimView* out);

namespace {

// ------------------------------------------------------------ pinned exp/log
// exp: Cody-Waite reduction x = k ln2 + r with ln2 split into 32 + 53 bits (k ln2_hi
// exact for |k| < 2^21), then the Taylor polynomial of degree 12 (coefficients 1/k!)
// on |r| <= ln2/2 by Horner with fused multiply-adds, scaled by 2^k.
// log: x = m 2^e with m in [sqrt(1/2), sqrt(2)), s = (m - 1)/(m + 1),
// log m = 2 s (1 + s^2/3 + ... + s^22/23) (the atanh series), log x = e ln2 + log m.
__device__ __forceinline__ double exp_core(double x) {
  if (x != x) return x;
  if (x > 709.0) return INFINITY;
  if (x < -745.5) return 0.0;
  const double k = rint(x * 0x1.71547652b82fep+0);
  const double r = (x - k * 0x1.62e42fee00000p-1) - k * 0x1.a39ef35793c76p-33;
  double p = 0x1.1eed8eff8d898p-29;
  p = fma(p, r, 0x1.ae64567f544e4p-26);
  p = fma(p, r, 0x1.27e4fb7789f5cp-22);
  p = fma(p, r, 0x1.71de3a556c734p-19);
  p = fma(p, r, 0x1.a01a01a01a01ap-16);
  p = fma(p, r, 0x1.a01a01a01a01ap-13);
  p = fma(p, r, 0x1.6c16c16c16c17p-10);
  p = fma(p, r, 0x1.1111111111111p-7);
  p = fma(p, r, 0x1.5555555555555p-5);
  p = fma(p, r, 0x1.5555555555555p-3);
  p = fma(p, r, 0x1.0000000000000p-1);
  p = fma(p, r, 1.0);
  p = fma(p, r, 1.0);
  return scalbn(p, (int)k);
}

__device__ __forceinline__ double log_core(double x) {  // x > 0, finite
  int e = 0;
  double m = frexp(x, &e);
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = m * 2.0;
    e -= 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  double p = 0x1.642c8590b2164p-5;
  p = fma(p, s2, 0x1.8618618618618p-5);
  p = fma(p, s2, 0x1.af286bca1af28p-5);
  p = fma(p, s2, 0x1.e1e1e1e1e1e1ep-5);
  p = fma(p, s2, 0x1.1111111111111p-4);
  p = fma(p, s2, 0x1.3b13b13b13b14p-4);
  p = fma(p, s2, 0x1.745d1745d1746p-4);
  p = fma(p, s2, 0x1.c71c71c71c71cp-4);
  p = fma(p, s2, 0x1.2492492492492p-3);
  p = fma(p, s2, 0x1.999999999999ap-3);
  p = fma(p, s2, 0x1.5555555555555p-2);
  p = fma(p, s2, 1.0);
  return (double)e * 0x1.62e42fefa39efp-1 + 2.0 * s * p;
}

__device__ __forceinline__ float pexp(float x) { return (float)exp_core((double)x); }

// pow(x, y) for the shader's exponents: NaN for x < 0 or NaN input, 0 for x = 0
// and y > 0, else exp(y log x) in FP64 rounded once.
__device__ __forceinline__ float ppow(float x, float y) {
  if (x != x || y != y || x < 0.0f) return __int_as_float(0x7fc00000);
  if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
  if (isinf(x)) return y > 0.0f ? INFINITY : (y == 0.0f ? 1.0f : 0.0f);
  return (float)exp_core((double)y * log_core((double)x));
}

// ------------------------------------------------------------------ vectors
struct V3 {
  float x, y, z;
};
FX_DEV V3 v3(float x, float y, float z) { return V3{x, y, z}; }
FX_DEV V3 add(V3 a, V3 b) { return v3(a.x + b.x, a.y + b.y, a.z + b.z); }
FX_DEV V3 sub(V3 a, V3 b) { return v3(a.x - b.x, a.y - b.y, a.z - b.z); }
FX_DEV V3 mul(V3 a, V3 b) { return v3(a.x * b.x, a.y * b.y, a.z * b.z); }
FX_DEV V3 mulf(V3 a, float s) { return v3(a.x * s, a.y * s, a.z * s); }
FX_DEV V3 fmulv(float s, V3 a) { return v3(s * a.x, s * a.y, s * a.z); }
FX_DEV V3 divv(V3 a, V3 b) { return v3(a.x / b.x, a.y / b.y, a.z / b.z); }
FX_DEV V3 divf(V3 a, float s) { return v3(a.x / s, a.y / s, a.z / s); }
FX_DEV V3 neg(V3 a) { return v3(-a.x, -a.y, -a.z); }
FX_DEV float dot3(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
FX_DEV float len3(V3 a) { return sqrtf(a.x * a.x + a.y * a.y + a.z * a.z); }
FX_DEV V3 norm3(V3 a) { return divf(a, len3(a)); }
FX_DEV V3 mixv3(V3 a, V3 b, float t) { return v3(mixv(a.x, b.x, t), mixv(a.y, b.y, t), mixv(a.z, b.z, t)); }
FX_DEV V3 mixv3v(V3 a, V3 b, V3 t) { return v3(mixv(a.x, b.x, t.x), mixv(a.y, b.y, t.y), mixv(a.z, b.z, t.z)); }
FX_DEV V3 clamp3(V3 a, V3 lo, V3 hi) { return v3(clampv(a.x, lo.x, hi.x), clampv(a.y, lo.y, hi.y), clampv(a.z, lo.z, hi.z)); }
FX_DEV V3 exp3(V3 a) { return v3(pexp(a.x), pexp(a.y), pexp(a.z)); }

// f32 -> u32 as WGSL converts: toward zero, saturated (NaN -> 0).
FX_DEV uint32_t to_u32(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967040.0f) return 0xffffffffu;
  return (uint32_t)f;
}

// The uniform of render() (createVolumeRaymarchPass.ts:195-250): the 80-float
// camera block, the resolution uniform and the packed brick layout.
struct Uniform {
  float cam[80];
  float res[4];
  uint32_t brick[8];
};

// Camera block offsets (CameraData, :300-314)
constexpr int C_POS = 0, C_RIGHT = 4, C_UP = 8, C_FWD = 12, C_VCENTER = 16, C_HALF = 20, C_RINFO = 24, C_RMODE = 28, C_SCATTER = 40,
              C_LIGHTS = 44;

template <typename S>
struct Fields {
  const S* f[4];
  const uint32_t* flags;
};

FX_DEV float ld(const float* p, uint32_t i) { return __ldg(p + i); }
FX_DEV float ld(const __half* p, uint32_t i) { return __half2float(__ldg(p + i)); }

template <typename S>
struct Ctx {
  const Uniform& U;
  Fields<S> F;
  uint32_t W, H;  // u32(resolution.width / height)
  V3 dims;        // sampleBounds()

  FX_DEV V3 cv(int o) const { return v3(U.cam[o], U.cam[o + 1], U.cam[o + 2]); }
  FX_DEV uint32_t flatten(uint32_t x, uint32_t y, uint32_t z) const { return x + W * (y + H * z); }
  FX_DEV uint32_t brick_size() const { return max(U.brick[4], 1u); }

  FX_DEV bool is_active(V3 p) const {
    const V3 c = clamp3(p, v3(0.0f, 0.0f, 0.0f), dims);
    const uint32_t cx = to_u32(floorf(c.x)), cy = to_u32(floorf(c.y)), cz = to_u32(floorf(c.z));
    const uint32_t bs = brick_size();
    const uint32_t bx = min(cx / bs, U.brick[0] - 1u), by = min(cy / bs, U.brick[1] - 1u), bz = min(cz / bs, U.brick[2] - 1u);
    return __ldg(F.flags + bx + U.brick[0] * (by + U.brick[1] * bz)) != 0u;
  }

  FX_DEV float dist_to_next_brick(V3 p, V3 d) const {
    const float far = 1e9f;
    const float be = (float)brick_size();
    const V3 bc = v3(floorf(p.x / be), floorf(p.y / be), floorf(p.z / be));
    const V3 b = v3(d.x > 0.0f ? (bc.x + 1.0f) * be : bc.x * be, d.y > 0.0f ? (bc.y + 1.0f) * be : bc.y * be,
                    d.z > 0.0f ? (bc.z + 1.0f) * be : bc.z * be);
    const float tx = fabsf(d.x) > 0.00001f ? (b.x - p.x) / d.x : far;
    const float ty = fabsf(d.y) > 0.00001f ? (b.y - p.y) / d.y : far;
    const float tz = fabsf(d.z) > 0.00001f ? (b.z - p.z) / d.z : far;
    return mn(tx, mn(ty, tz)) * len3(d) + 0.5f;
  }

  FX_DEV void sample_all(V3 p, float out[4]) const {
    const V3 c = clamp3(p, v3(0.0f, 0.0f, 0.0f), dims);
    const uint32_t bx = to_u32(floorf(c.x)), by = to_u32(floorf(c.y)), bz = to_u32(floorf(c.z));
    const uint32_t mxx = to_u32(dims.x), mxy = to_u32(dims.y), mxz = to_u32(dims.z);
    const uint32_t ux = min(bx + 1u, mxx), uy = min(by + 1u, mxy), uz = min(bz + 1u, mxz);
    const float fx = c.x - floorf(c.x), fy = c.y - floorf(c.y), fz = c.z - floorf(c.z);
    const uint32_t i000 = flatten(bx, by, bz), i100 = flatten(ux, by, bz), i010 = flatten(bx, uy, bz), i110 = flatten(ux, uy, bz);
    const uint32_t i001 = flatten(bx, by, uz), i101 = flatten(ux, by, uz), i011 = flatten(bx, uy, uz), i111 = flatten(ux, uy, uz);
#pragma unroll
    for (int k = 0; k < 4; ++k) {
      const S* f = F.f[k];
      const float x00 = mixv(ld(f, i000), ld(f, i100), fx);
      const float x10 = mixv(ld(f, i010), ld(f, i110), fx);
      const float x01 = mixv(ld(f, i001), ld(f, i101), fx);
      const float x11 = mixv(ld(f, i011), ld(f, i111), fx);
      out[k] = mixv(mixv(x00, x10, fy), mixv(x01, x11, fy), fz);
    }
  }

  FX_DEV float density_nearest(V3 p) const {
    const uint32_t mxx = to_u32(dims.x), mxy = to_u32(dims.y), mxz = to_u32(dims.z);
    const uint32_t x = min(to_u32(floorf(p.x)), mxx), y = min(to_u32(floorf(p.y)), mxy), z = min(to_u32(floorf(p.z)), mxz);
    return ld(F.f[0], flatten(x, y, z));
  }

  FX_DEV V3 density_gradient(V3 p) const {
    const uint32_t mxx = to_u32(dims.x), mxy = to_u32(dims.y), mxz = to_u32(dims.z);
    const uint32_t x = min(to_u32(rintf(p.x)), mxx), y = min(to_u32(rintf(p.y)), mxy), z = min(to_u32(rintf(p.z)), mxz);
    const S* d = F.f[0];
    const uint32_t xp = flatten(min(x + 1u, mxx), y, z), xn = flatten(x == 0u ? 0u : x - 1u, y, z);
    const uint32_t yp = flatten(x, min(y + 1u, mxy), z), yn = flatten(x, y == 0u ? 0u : y - 1u, z);
    const uint32_t zp = flatten(x, y, min(z + 1u, mxz)), zn = flatten(x, y, z == 0u ? 0u : z - 1u);
    return v3(ld(d, xp) - ld(d, xn), ld(d, yp) - ld(d, yn), ld(d, zp) - ld(d, zn));
  }

  FX_DEV V3 light_direction(int i, V3 wp) const {
    const int o = C_LIGHTS + 12 * i;
    if (U.cam[o + 3] > 0.5f) return norm3(sub(cv(o + 4), wp));
    const V3 raw = cv(o);
    return norm3(dot3(raw, raw) > 0.0001f ? raw : v3(-0.34f, 0.88f, 0.31f));
  }

  FX_DEV float light_attenuation(int i, V3 wp) const {
    const int o = C_LIGHTS + 12 * i;
    if (U.cam[o + 3] <= 0.5f) return 1.0f;
    const float d = len3(sub(cv(o + 4), wp));
    return 1.0f / (1.0f + d * 0.09f + d * d * 0.02f);
  }

  FX_DEV float light_intensity(int i) const { return mx(U.cam[C_LIGHTS + 12 * i + 7], 0.0f); }
  FX_DEV V3 light_color(int i) const { return cv(C_LIGHTS + 12 * i + 8); }
};

FX_DEV V3 fire_palette(float t) {
  const V3 ember = v3(0.18f, 0.018f, 0.0f), red = v3(1.0f, 0.075f, 0.012f), orange = v3(1.0f, 0.42f, 0.035f),
           white_hot = v3(1.0f, 0.86f, 0.56f);
  const float red_mix = smoothstepv(0.01f, 0.11f, t);
  const float orange_mix = smoothstepv(0.09f, 0.38f, t);
  const float white_mix = smoothstepv(0.58f, 0.92f, t);
  return mixv3(mixv3(mixv3(ember, red, red_mix), orange, orange_mix), white_hot, white_mix);
}

FX_DEV V3 smoke_albedo(float density, float temperature, float hot_gas) {
  const float warm_tint = clampv(temperature * 0.38f, 0.0f, 1.0f);
  const float soot = smoothstepv(0.16f, 0.9f, density) * (1.0f - smoothstepv(0.2f, 0.74f, hot_gas));
  const V3 cool = v3(0.26f, 0.275f, 0.295f), dense_soot = v3(0.04f, 0.041f, 0.045f), warm = v3(0.36f, 0.27f, 0.18f);
  return mixv3(mixv3(cool, dense_soot, soot * 0.86f), warm, warm_tint * (0.35f + hot_gas * 0.45f));
}

FX_DEV float phase_hg(float cos_theta, float g) {
  const float g2 = g * g;
  const float denom = ppow(mx(1.0f + g2 - 2.0f * g * cos_theta, 0.001f), 1.5f);
  return (1.0f - g2) / (12.566370614359172f * denom);
}

FX_DEV V3 thermal_scatter(float temperature, float fuel, float reaction, float density) {
  const float heat = clampv(temperature * 1.25f + fuel * 0.18f + reaction * 0.34f, 0.0f, 1.0f);
  const float flame = clampv(temperature * 0.9f + fuel * 0.12f + reaction * 0.18f, 0.0f, 1.0f);
  const float smoke_catch = smoothstepv(0.012f, 0.38f, density);
  return mulf(mulf(mulf(mulf(fire_palette(flame), heat), heat), smoke_catch), 0.18f);
}

template <typename S>
FX_DEV float primary_transmittance(const Ctx<S>& c, V3 sp, V3 light_step, float density, float hot_gas) {
  const V3 zero = v3(0.0f, 0.0f, 0.0f);
  const V3 p1 = clamp3(add(sp, mulf(light_step, 0.9f)), zero, c.dims);
  const V3 p2 = clamp3(add(sp, mulf(light_step, 2.0f)), zero, c.dims);
  const V3 p3 = clamp3(add(sp, mulf(light_step, 3.6f)), zero, c.dims);
  const float d1 = mx(c.density_nearest(p1) - 0.004f, 0.0f);
  const float d2 = mx(c.density_nearest(p2) - 0.004f, 0.0f);
  const float d3 = mx(c.density_nearest(p3) - 0.004f, 0.0f);
  const float optical = density * 0.34f + d1 * 1.15f + d2 * 0.72f + d3 * 0.4f - hot_gas * 0.06f;
  return pexp(-mx(optical, 0.0f) * 2.15f);
}

// fsMain (:587-724) for one pixel; returns false where the fragment discards.
template <typename S>
FX_DEV bool shade(const Ctx<S>& c, float u, float v, float out[4]) {
  const Uniform& U = c.U;
  const float ndcx = u * 2.0f - 1.0f, ndcy = v * 2.0f - 1.0f;
  const float aspect = U.cam[C_RINFO + 2], tanh_ = U.cam[C_RINFO + 3];
  const V3 ray = norm3(add(add(c.cv(C_FWD), mulf(mulf(mulf(c.cv(C_RIGHT), ndcx), aspect), tanh_)), mulf(mulf(c.cv(C_UP), ndcy), tanh_)));
  const V3 cam = c.cv(C_POS);
  const V3 box_min = sub(c.cv(C_VCENTER), c.cv(C_HALF)), box_max = add(c.cv(C_VCENTER), c.cv(C_HALF));
  // intersectBox (:466-476)
  const V3 inv = divv(v3(1.0f, 1.0f, 1.0f), ray);
  const V3 t0 = mul(sub(box_min, cam), inv), t1 = mul(sub(box_max, cam), inv);
  const V3 tmin = v3(mn(t0.x, t1.x), mn(t0.y, t1.y), mn(t0.z, t1.z)), tmax = v3(mx(t0.x, t1.x), mx(t0.y, t1.y), mx(t0.z, t1.z));
  float bx = mx(tmin.x, mx(tmin.y, tmin.z));
  const float by = mn(tmax.x, mn(tmax.y, tmax.z));
  if (bx > by) return false;
  bx = mx(bx, 0.0f);

  const uint32_t steps = to_u32(U.cam[C_RMODE + 1]);
  const V3 inv_extent = divv(v3(1.0f, 1.0f, 1.0f), mulf(c.cv(C_HALF), 2.0f));
  const V3 dims = c.dims;
  const V3 vox_dir = mul(mul(ray, inv_extent), dims);
  const float steps_f = mx((float)steps, 1.0f);
  const float vox_delta = len3(vox_dir) * (by - bx) / steps_f;
  const float world_delta = (by - bx) / steps_f;
  const uint32_t lights = to_u32(clampv(U.cam[C_SCATTER + 2], 0.0f, 3.0f));
  const V3 primary_dir = lights > 0u ? c.light_direction(0, cam) : v3(0.0f, 1.0f, 0.0f);
  const V3 light_step = mulf(mul(primary_dir, dims), 0.036f);

  V3 pos = mul(mul(sub(add(cam, mulf(ray, bx)), box_min), inv_extent), dims);
  float travelled = 0.0f;
  const float ray_len = len3(vox_dir) * (by - bx);
  const V3 dir_unit = norm3(vox_dir);
  const V3 mray = neg(ray);
  V3 acc = v3(0.0f, 0.0f, 0.0f);
  float alpha = 0.0f;
  const float mode = U.cam[C_RMODE];

  for (uint32_t index = 0; index < steps && travelled <= ray_len; ++index) {
    if (alpha > 0.985f) break;
    float step = vox_delta;
    const V3 sp = pos;
    const V3 uvw = divv(sp, dims);
    if (c.is_active(sp)) {
      float smp[4];
      c.sample_all(sp, smp);
      const float density = mx(smp[0] - 0.004f, 0.0f);
      const float temperature = smp[1], fuel = smp[2], reaction = smp[3];
      const float hot_gas = clampv(temperature * 1.45f + fuel * 0.22f + reaction * 0.38f, 0.0f, 1.0f);
      if (density > 0.001f || hot_gas > 0.018f) {
        if (density < 0.012f && hot_gas < 0.04f) {
          step = vox_delta * 1.8f;
        } else {
          const V3 grad = c.density_gradient(sp);
          const float grad_len = mx(len3(grad), 0.0001f);
          const V3 normal = grad_len > 0.00011f ? divf(neg(grad), grad_len) : v3(0.0f, 1.0f, 0.0f);
          const float detail = clampv(grad_len * 5.2f + hot_gas * 0.28f + reaction * 0.18f, 0.0f, 1.0f);
          const float dd = mx(ppow(density, 0.96f) * mixv(0.82f, 1.42f, detail), 0.0f);
          const V3 wp = mixv3v(box_min, box_max, uvw);
          const float top_fade = 1.0f - smoothstepv(0.9f, 0.995f, uvw.y);
          V3 total = v3(0.0f, 0.0f, 0.0f);
          const float primary_t = lights > 0u ? primary_transmittance(c, sp, light_step, dd, hot_gas) : 1.0f;
          for (uint32_t li = 0; li < 3u; ++li) {
            if (li >= lights) break;
            const V3 to_light = c.light_direction((int)li, wp);
            const float raw_power = c.light_intensity((int)li) * c.light_attenuation((int)li, wp);
            const float power = raw_power / (1.0f + raw_power * 0.18f);
            const V3 color = c.light_color((int)li);
            const float view_cos = clampv(dot3(to_light, mray), -1.0f, 1.0f);
            const float fwd = phase_hg(view_cos, U.cam[C_SCATTER]) * 5.2f * power;
            const float back = phase_hg(view_cos, U.cam[C_SCATTER + 1]) * 1.55f * power;
            const float facing = clampv(dot3(normal, to_light) * 0.5f + 0.5f, 0.0f, 1.0f);
            const float surface = ppow(facing, 1.35f) * mixv(1.0f, 0.56f, smoothstepv(0.16f, 0.9f, dd));
            const float rim = ppow(1.0f - fabsf(dot3(normal, mray)), 2.4f) * ppow(clampv(dot3(to_light, mray) * 0.5f + 0.5f, 0.0f, 1.0f), 1.2f);
            const float directional = (surface * 0.42f + rim * 0.22f) * power;
            const float scatter = (fwd + back) * mixv(0.36f, 0.74f, hot_gas);
            const float transmission = li > 0u ? 1.0f : primary_t;
            total = add(total, mulf(mulf(color, transmission), directional + scatter));
          }
          const V3 tone = sub(v3(1.0f, 1.0f, 1.0f), exp3(mulf(neg(total), 0.72f)));
          const V3 ambient = v3(0.045f, 0.048f, 0.052f);
          const V3 smoke = smoke_albedo(dd, temperature, hot_gas);
          const float absorption = mixv(0.92f, 0.34f, smoothstepv(0.26f, 1.05f, dd));
          const V3 heat = thermal_scatter(temperature, fuel, reaction, dd);
          const V3 lit = add(add(add(mul(smoke, ambient), mulf(mul(smoke, tone), absorption)), mulf(mulf(tone, smoothstepv(0.018f, 0.22f, dd)), 0.18f)),
                             heat);
          const float flame_heat = clampv(temperature * 0.9f + fuel * 0.14f + reaction * 0.16f, 0.0f, 1.0f);
          const V3 emissive = mulf(mulf(fire_palette(flame_heat), hot_gas), 0.48f + fuel * 0.16f + reaction * 0.24f);
          const float contribution = clampv(dd * 1.35f + hot_gas * 1.25f, 0.0f, 1.0f);
          const float step_distance = world_delta * mixv(1.02f, 0.76f, contribution);
          step = vox_delta * mixv(1.02f, 0.76f, contribution);
          V3 composite = add(lit, emissive);
          float opacity = (1.0f - pexp(-(dd * 4.75f + hot_gas * 0.42f) * step_distance)) * top_fade;
          if (mode > 0.5f && mode < 1.5f) {
            composite = mixv3(v3(0.01f, 0.01f, 0.012f), v3(0.88f, 0.9f, 0.94f), clampv(dd * 1.4f, 0.0f, 1.0f));
            opacity = 1.0f - pexp(-dd * step_distance * 8.6f);
          } else if (mode >= 1.5f) {
            composite = mixv3(v3(0.04f, 0.012f, 0.0f), v3(1.0f, 0.72f, 0.22f), clampv(fuel * 1.3f, 0.0f, 1.0f));
            opacity = 1.0f - pexp(-fuel * step_distance * 7.0f);
          }
          acc = add(acc, mulf(fmulv(1.0f - alpha, composite), opacity));
          alpha = alpha + (1.0f - alpha) * opacity;
        }
      } else {
        step = vox_delta * 1.35f;
      }
    } else {
      step = mx(c.dist_to_next_brick(sp, vox_dir), vox_delta);
    }
    pos = add(pos, mulf(dir_unit, step));
    travelled = travelled + step;
  }
  if (alpha < 0.01f) return false;
  out[0] = acc.x;
  out[1] = acc.y;
  out[2] = acc.z;
  out[3] = alpha;
  return true;
}

template <typename S, typename P>
__global__ void __launch_bounds__(128) k_raymarch(Uniform U, Fields<S> F, uint32_t width, uint32_t height, P* __restrict__ pixels) {
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= width || py >= height) return;
  Ctx<S> c{U, F, to_u32(U.res[0]), to_u32(U.res[1]), v3(U.res[0] - 1.0f, U.res[1] - 1.0f, U.res[2] - 1.0f)};
  const float u = ((float)px + 0.5f) / (float)width;
  const float v = 1.0f - ((float)py + 0.5f) / (float)height;
  float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
  shade(c, u, v, o);
  const size_t i = ((size_t)py * width + px) * 4;
#pragma unroll
  for (int k = 0; k < 4; ++k) {
    if constexpr (sizeof(P) == 2) {
      pixels[i + k] = __float2half_rn(o[k]);
    } else {
      pixels[i + k] = o[k];
    }
  }
}

// ---------------------------------------------------------------------- bloom
// createBloomPass.ts: soft threshold into a half-resolution texture, a 9-tap
// gaussian blur along x then y, and the composite with pow(., 0.92) into the
// canvas (:224-297). Textures are RGBA16F (values rounded to nearest); a
// textureSample with the linear sampler is bilinear with exact f32 weights and
// clamp-to-edge addressing; the fragment uv at pixel (x, y) of a W x H target
// is ((x + 0.5) / W, (y + 0.5) / H).
struct Px4 {
  float v[4];
};

template <typename T>
FX_DEV float texel(const T* t, uint32_t i) {
  if constexpr (sizeof(T) == 2) return __half2float(t[i]);
  else return t[i];
}

template <typename T>
FX_DEV Px4 sample_bilinear(const T* tex, uint32_t tw, uint32_t th, float u, float v) {
  const float x = u * (float)tw - 0.5f, y = v * (float)th - 0.5f;
  const float x0 = floorf(x), y0 = floorf(y);
  const float fx = x - x0, fy = y - y0;
  const int ix = (int)x0, iy = (int)y0;
  const uint32_t xa = (uint32_t)min(max(ix, 0), (int)tw - 1), xb = (uint32_t)min(max(ix + 1, 0), (int)tw - 1);
  const uint32_t ya = (uint32_t)min(max(iy, 0), (int)th - 1), yb = (uint32_t)min(max(iy + 1, 0), (int)th - 1);
  Px4 o;
#pragma unroll
  for (int c = 0; c < 4; ++c) {
    const float t00 = texel(tex, (ya * tw + xa) * 4 + c), t10 = texel(tex, (ya * tw + xb) * 4 + c);
    const float t01 = texel(tex, (yb * tw + xa) * 4 + c), t11 = texel(tex, (yb * tw + xb) * 4 + c);
    o.v[c] = mixv(mixv(t00, t10, fx), mixv(t01, t11, fx), fy);
  }
  return o;
}

struct BloomU {
  float threshold, strength, radius;
  float texel_hx, texel_hy;  // 1 / half width, 1 / half height (paramsData[4..5])
};

template <typename T>
__global__ void k_bloom_threshold(const T* __restrict__ src, uint32_t w, uint32_t h, uint32_t hw, uint32_t hh, BloomU U, __half* __restrict__ out) {
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= hw || py >= hh) return;
  const float u = ((float)px + 0.5f) / (float)hw, v = ((float)py + 0.5f) / (float)hh;
  const Px4 c = sample_bilinear(src, w, h, u, v);
  const float lum = c.v[0] * 0.2126f + c.v[1] * 0.7152f + c.v[2] * 0.0722f;
  const float knee = U.threshold * 0.5f;
  const float rq = clampv(lum - U.threshold + knee, 0.0f, 2.0f * knee);
  const float wgt = (rq * rq) / (4.0f * knee * knee + 0.00001f);
  const float mask = mx(wgt, stepv(U.threshold, lum));
  const size_t o = ((size_t)py * hw + px) * 4;
  out[o + 0] = __float2half_rn(c.v[0] * mask * c.v[3]);
  out[o + 1] = __float2half_rn(c.v[1] * mask * c.v[3]);
  out[o + 2] = __float2half_rn(c.v[2] * mask * c.v[3]);
  out[o + 3] = __float2half_rn(c.v[3] * mask);
}

__global__ void k_bloom_blur(const __half* __restrict__ src, uint32_t hw, uint32_t hh, float sx, float sy, __half* __restrict__ out) {
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= hw || py >= hh) return;
  const float u = ((float)px + 0.5f) / (float)hw, v = ((float)py + 0.5f) / (float)hh;
  const float wts[5] = {0.2270270270f, 0.1945945946f, 0.1216216216f, 0.0540540541f, 0.0162162162f};
  Px4 col = sample_bilinear(src, hw, hh, u, v);
#pragma unroll
  for (int c = 0; c < 4; ++c) col.v[c] = col.v[c] * wts[0];
#pragma unroll
  for (int k = 1; k <= 4; ++k) {
    const float ox = sx * (float)k, oy = sy * (float)k;
    const Px4 a = sample_bilinear(src, hw, hh, u + ox, v + oy);
    const Px4 b = sample_bilinear(src, hw, hh, u - ox, v - oy);
#pragma unroll
    for (int c = 0; c < 4; ++c) col.v[c] = col.v[c] + a.v[c] * wts[k];
#pragma unroll
    for (int c = 0; c < 4; ++c) col.v[c] = col.v[c] + b.v[c] * wts[k];
  }
  const size_t o = ((size_t)py * hw + px) * 4;
#pragma unroll
  for (int c = 0; c < 4; ++c) out[o + c] = __float2half_rn(col.v[c]);
}

FX_DEV uint8_t unorm8(float x) { return (uint8_t)rintf(clampv(x, 0.0f, 1.0f) * 255.0f); }

template <typename T, typename P>
__global__ void k_bloom_composite(const T* __restrict__ src, uint32_t w, uint32_t h, const __half* __restrict__ glow_tex, uint32_t hw,
                                  uint32_t hh, BloomU U, int enabled, P* __restrict__ out) {
  const uint32_t px = blockIdx.x * blockDim.x + threadIdx.x, py = blockIdx.y * blockDim.y + threadIdx.y;
  if (px >= w || py >= h) return;
  const float u = ((float)px + 0.5f) / (float)w, v = ((float)py + 0.5f) / (float)h;
  const Px4 base = sample_bilinear(src, w, h, u, v);
  float r[4];
  if (enabled) {
    const Px4 glow = sample_bilinear(glow_tex, hw, hh, u, v);
    for (int c = 0; c < 3; ++c) r[c] = ppow(mx(base.v[c] + mx(glow.v[c], 0.0f) * U.strength, 0.0f), 0.92f);
    const float glow_alpha = clampv(glow.v[3] * U.strength, 0.0f, 1.0f);
    r[3] = clampv(base.v[3] + glow_alpha * (1.0f - base.v[3]), 0.0f, 1.0f);
  } else {  // the blit shader (:284-296)
    for (int c = 0; c < 3; ++c) r[c] = ppow(mx(base.v[c], 0.0f), 0.92f);
    r[3] = clampv(base.v[3], 0.0f, 1.0f);
  }
  const size_t o = ((size_t)py * w + px) * 4;
  for (int c = 0; c < 4; ++c) {
    if constexpr (sizeof(P) == 1) out[o + c] = unorm8(r[c]);
    else out[o + c] = r[c];
  }
}

__global__ void k_exp_pow(const float* x, const float* y, float* oe, float* op, uint32_t n) {
  const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  oe[i] = pexp(x[i]);
  op[i] = ppow(x[i], y[i]);
}

// ------------------------------------------------------------------ host side
double clampd(double v, double lo, double hi) { return std::max(lo, std::min(hi, v)); }

// sanitizeRenderLights (:47-80): normalised direction (the default light when
// shorter than 1e-4), non-negative colour and intensity, at most 3 lights.
void sanitize_light(const fx_render_light& in, fx_render_light& out) {
  out = in;
  const double l = std::sqrt(in.direction[0] * in.direction[0] + in.direction[1] * in.direction[1] + in.direction[2] * in.direction[2]);
  if (l <= 0.0001) {
    out.direction[0] = -0.34;
    out.direction[1] = 0.88;
    out.direction[2] = 0.31;
  } else {
    for (int k = 0; k < 3; ++k) out.direction[k] = in.direction[k] / l;
  }
  for (int k = 0; k < 3; ++k) out.color[k] = std::max(in.color[k], 0.0);
  out.intensity = std::max(in.intensity, 0.0);
}

}  // namespace
}  // namespace fx

using namespace fx;

struct fx_bloom {
  int device = 0;
  uint32_t hw = 0, hh = 0;
  __half* tex[3] = {nullptr, nullptr, nullptr};  // bright, blur x, blur y (half resolution)
};

struct fx_raymarch {
  uint32_t w, h, d;
  double center_y, half[3];
  int step_count;
  fx_render_light lights[FX_MAX_RENDER_LIGHTS];
  uint32_t light_count;
  double scatter_forward = 0.32, scatter_back = -0.18;
};

namespace {

fx_status rm_fail(fx_status code, const std::string& msg) {
  fx::set_last_error(msg);
  return code;
}

fx_render_light default_light() {
  fx_render_light l{};
  l.type = FX_LIGHT_DIRECTIONAL;
  l.direction[0] = -0.34;
  l.direction[1] = 0.88;
  l.direction[2] = 0.31;
  l.color[0] = 1.0;
  l.color[1] = 0.95;
  l.color[2] = 0.88;
  l.intensity = 1.25;
  return l;
}

int js_round_int(double v) { return (int)std::floor(v + 0.5); }

}  // namespace

extern "C" {

fx_status fx_raymarch_create(uint32_t width, uint32_t height, uint32_t depth, fx_raymarch** out) {
  if (!out) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_create: out is NULL");
  *out = nullptr;
  if (width < 2 || height < 2 || depth < 2) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_create: every dimension must be >= 2");
  fx_raymarch* r = new (std::nothrow) fx_raymarch;
  if (!r) return rm_fail(FX_ERR_OUT_OF_MEMORY, "fx_raymarch_create: host allocation failed");
  r->w = width;
  r->h = height;
  r->d = depth;
  // getVolumeWorldBounds (render/volumetrics/volumeWorldBounds.ts:17-33)
  const double scale = 13.5, mh = (double)std::max(width, depth);
  r->half[0] = 2.05 * scale * (width / mh);
  r->half[1] = 2.05 * scale * (height / mh);
  r->half[2] = 2.05 * scale * (depth / mh);
  r->center_y = r->half[1] - 0.25;
  // createVolumeRaymarchPass.ts:87
  const double voxels = (double)width * height * depth;
  r->step_count = (int)clampd(js_round_int(std::max({width, height, depth}) * 1.5), 180, voxels >= 4000000.0 ? 720 : 560);
  sanitize_light(default_light(), r->lights[0]);
  r->light_count = 1;
  *out = r;
  return FX_OK;
}

void fx_raymarch_destroy(fx_raymarch* r) { delete r; }

fx_status fx_raymarch_set_params(fx_raymarch* r, const fx_raymarch_params* p) {
  if (!r || !p) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_set_params: NULL argument");
  if (p->mask & ~(uint32_t)(FX_RM_STEP_COUNT | FX_RM_LIGHTS | FX_RM_SCATTER_FORWARD | FX_RM_SCATTER_BACK))
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_set_params: unknown mask bits");
  // setRenderParams (:268-281)
  if (p->mask & FX_RM_STEP_COUNT) {
    if (!std::isfinite(p->step_count)) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_set_params: step_count must be finite");
    // setRenderParams keeps max(32, round(n)); the upper bound of 4096 keeps one launch short
    r->step_count = std::min(4096, std::max(32, js_round_int(std::min(std::max(p->step_count, -1e6), 1e6))));
  }
  if (p->mask & FX_RM_LIGHTS) {
    r->light_count = std::min<uint32_t>(p->light_count, FX_MAX_RENDER_LIGHTS);
    for (uint32_t k = 0; k < r->light_count; ++k) sanitize_light(p->lights[k], r->lights[k]);
  }
  if (p->mask & FX_RM_SCATTER_FORWARD) r->scatter_forward = clampd(p->scattering_forward, 0.0, 0.98);
  if (p->mask & FX_RM_SCATTER_BACK) r->scatter_back = clampd(p->scattering_back, -0.98, 0.0);
  return FX_OK;
}

fx_status fx_raymarch_render(fx_raymarch* r, fx_sim* sim, const fx_camera* cam, int32_t display_mode, uint32_t width, uint32_t height,
                             double elapsed_seconds, void* pixels, int32_t pixel_format) {
  if (!r || !sim || !cam || !pixels) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_render: NULL argument");
  if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28))
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_render: image size out of range");
  if (display_mode < FX_DISPLAY_TEMPERATURE || display_mode > FX_DISPLAY_FUEL)
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_render: unknown display mode");
  if (pixel_format != FX_PIXELS_RGBA16F && pixel_format != FX_PIXELS_RGBA32F)
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_render: unknown pixel format");
  SimView sv;
  if (!sim_view(sim, &sv)) return rm_fail(FX_ERR_STATE, "fx_raymarch_render: the simulation has an error");
  if (sv.dm.w != r->w || sv.dm.h != r->h || sv.dm.d != r->d)
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_raymarch_render: the simulation's resolution differs from the pass's");
  // render() (:195-250): the camera block as f32
  Uniform U;
  std::memset(&U, 0, sizeof U);
  float* c = U.cam;
  for (int k = 0; k < 3; ++k) {
    c[C_POS + k] = (float)cam->position[k];
    c[C_RIGHT + k] = (float)cam->right[k];
    c[C_UP + k] = (float)cam->up[k];
    c[C_FWD + k] = (float)cam->forward[k];
    c[C_HALF + k] = (float)r->half[k];
    c[32 + k] = (float)cam->target[k];
  }
  c[C_VCENTER + 1] = (float)r->center_y;
  c[C_RINFO + 0] = (float)width;
  c[C_RINFO + 1] = (float)height;
  c[C_RINFO + 2] = (float)cam->aspect;
  c[C_RINFO + 3] = (float)cam->tan_half_fov_y;
  c[C_RMODE + 0] = (float)display_mode;
  c[C_RMODE + 1] = (float)r->step_count;
  c[C_RMODE + 2] = (float)elapsed_seconds;
  c[C_SCATTER + 0] = (float)r->scatter_forward;
  c[C_SCATTER + 1] = (float)r->scatter_back;
  c[C_SCATTER + 2] = (float)r->light_count;
  for (uint32_t k = 0; k < r->light_count; ++k) {
    const fx_render_light& l = r->lights[k];
    float* b = c + C_LIGHTS + 12 * k;
    for (int a = 0; a < 3; ++a) {
      b[a] = (float)l.direction[a];
      b[4 + a] = (float)l.position[a];
      b[8 + a] = (float)l.color[a];
    }
    b[3] = l.type == FX_LIGHT_POINT ? 1.0f : 0.0f;
    b[7] = (float)l.intensity;
  }
  U.res[0] = (float)r->w;
  U.res[1] = (float)r->h;
  U.res[2] = (float)r->d;
  U.brick[0] = sv.bricks.x;
  U.brick[1] = sv.bricks.y;
  U.brick[2] = sv.bricks.z;
  U.brick[3] = sv.bricks.x * sv.bricks.y * sv.bricks.z;
  U.brick[4] = 8;
  if (cudaSetDevice(sv.device) != cudaSuccess) return rm_fail(FX_ERR_CUDA, "fx_raymarch_render: cudaSetDevice failed");
  const dim3 block(16, 8, 1), grid((width + 15) / 16, (height + 7) / 8, 1);
  auto launch = [&](auto stag) {
    using S = decltype(stag);
    Fields<S> F;
    for (int k = 0; k < 4; ++k) F.f[k] = static_cast<const S*>(sv.f[k]);
    F.flags = sv.flags;
    if (pixel_format == FX_PIXELS_RGBA16F)
      k_raymarch<S, __half><<<grid, block, 0, sv.stream>>>(U, F, width, height, static_cast<__half*>(pixels));
    else
      k_raymarch<S, float><<<grid, block, 0, sv.stream>>>(U, F, width, height, static_cast<float*>(pixels));
  };
  if (sv.half) launch(__half{});
  else launch(float{});
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rm_fail(FX_ERR_CUDA, std::string("fx_raymarch_render: launch failed: ") + cudaGetErrorString(e));
  return FX_OK;
}

fx_status fx_bloom_create(fx_bloom** out) {
  if (!out) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_bloom_create: out is NULL");
  *out = new (std::nothrow) fx_bloom;
  if (!*out) return rm_fail(FX_ERR_OUT_OF_MEMORY, "fx_bloom_create: host allocation failed");
  if (cudaGetDevice(&(*out)->device) != cudaSuccess) (*out)->device = 0;
  return FX_OK;
}

void fx_bloom_destroy(fx_bloom* b) {
  if (!b) return;
  cudaSetDevice(b->device);
  for (auto& t : b->tex)
    if (t) cudaFree(t);
  delete b;
}

fx_status fx_bloom_render(fx_bloom* b, const void* hdr, int32_t hdr_format, uint32_t width, uint32_t height, const fx_bloom_params* p,
                          void* out, int32_t out_format, void* stream) {
  if (!b || !hdr || !p || !out) return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_bloom_render: NULL argument");
  if (width == 0 || height == 0 || (uint64_t)width * height > (1ull << 28))
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_bloom_render: image size out of range");
  if ((hdr_format != FX_PIXELS_RGBA16F && hdr_format != FX_PIXELS_RGBA32F) || (out_format != FX_PIXELS_RGBA8 && out_format != FX_PIXELS_RGBA32F))
    return rm_fail(FX_ERR_INVALID_ARGUMENT, "fx_bloom_render: unknown pixel format");
  if (cudaSetDevice(b->device) != cudaSuccess) return rm_fail(FX_ERR_CUDA, "fx_bloom_render: cudaSetDevice failed");
  // rebuildTextures (:84-94): half resolution, at least 1 x 1
  const uint32_t hw = std::max(1u, width / 2), hh = std::max(1u, height / 2);
  if (hw != b->hw || hh != b->hh) {
    b->hw = b->hh = 0;  // a failed allocation leaves no size that matches
    for (auto& t : b->tex) {
      if (t) cudaFree(t);
      t = nullptr;
    }
    for (auto& t : b->tex)
      if (cudaMalloc(&t, (size_t)hw * hh * 4 * sizeof(__half)) != cudaSuccess)
        return rm_fail(FX_ERR_OUT_OF_MEMORY, "fx_bloom_render: texture allocation failed");
    b->hw = hw;
    b->hh = hh;
  }
  // paramsData (:103-111), as f32
  BloomU U;
  U.threshold = (float)p->threshold;
  U.strength = (float)p->strength;
  U.radius = (float)p->radius;
  U.texel_hx = (float)(1.0 / hw);
  U.texel_hy = (float)(1.0 / hh);
  const cudaStream_t s = static_cast<cudaStream_t>(stream);
  const dim3 block(16, 16, 1), half_grid((hw + 15) / 16, (hh + 15) / 16, 1), full_grid((width + 15) / 16, (height + 15) / 16, 1);
  // blur step: texel * (1 + radius * 2) along one axis (:247)
  const float spread = 1.0f + U.radius * 2.0f;
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const T* src = static_cast<const T*>(hdr);
    if (p->enabled) {
      k_bloom_threshold<T><<<half_grid, block, 0, s>>>(src, width, height, hw, hh, U, b->tex[0]);
      k_bloom_blur<<<half_grid, block, 0, s>>>(b->tex[0], hw, hh, U.texel_hx * spread, 0.0f * spread, b->tex[1]);
      k_bloom_blur<<<half_grid, block, 0, s>>>(b->tex[1], hw, hh, 0.0f * spread, U.texel_hy * spread, b->tex[2]);
    }
    if (out_format == FX_PIXELS_RGBA8)
      k_bloom_composite<T, uint8_t><<<full_grid, block, 0, s>>>(src, width, height, b->tex[2], hw, hh, U, p->enabled ? 1 : 0,
                                                                 static_cast<uint8_t*>(out));
    else
      k_bloom_composite<T, float><<<full_grid, block, 0, s>>>(src, width, height, b->tex[2], hw, hh, U, p->enabled ? 1 : 0,
                                                               static_cast<float*>(out));
  };
  if (hdr_format == FX_PIXELS_RGBA16F) run(__half{});
  else run(float{});
  const cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rm_fail(FX_ERR_CUDA, std::string("fx_bloom_render: launch failed: ") + cudaGetErrorString(e));
  return FX_OK;
}

// Test hook: the pinned f32 exp and pow on the device, for n inputs (pow reads
// y[i]; exp ignores y).
fx_status fx_test_pinned_exp_pow(const float* x, const float* y, float* out_exp, float* out_pow, uint32_t n);

}  // extern "C"

extern "C" fx_status fx_test_pinned_exp_pow(const float* x, const float* y, float* out_exp, float* out_pow, uint32_t n) {
  if (!x || !y || !out_exp || !out_pow) return FX_ERR_INVALID_ARGUMENT;
  float *dx = nullptr, *dy = nullptr, *de = nullptr, *dp = nullptr;
  const size_t b = (size_t)n * sizeof(float);
  fx_status st = FX_OK;
  if (cudaMalloc(&dx, b) != cudaSuccess || cudaMalloc(&dy, b) != cudaSuccess || cudaMalloc(&de, b) != cudaSuccess ||
      cudaMalloc(&dp, b) != cudaSuccess)
    st = FX_ERR_OUT_OF_MEMORY;
  if (st == FX_OK && (cudaMemcpy(dx, x, b, cudaMemcpyHostToDevice) != cudaSuccess || cudaMemcpy(dy, y, b, cudaMemcpyHostToDevice) != cudaSuccess))
    st = FX_ERR_CUDA;
  if (st == FX_OK && n) {
    k_exp_pow<<<(n + 255) / 256, 256>>>(dx, dy, de, dp, n);
    if (cudaMemcpy(out_exp, de, b, cudaMemcpyDeviceToHost) != cudaSuccess || cudaMemcpy(out_pow, dp, b, cudaMemcpyDeviceToHost) != cudaSuccess)
      st = FX_ERR_CUDA;
  }
  cudaFree(dx);
  cudaFree(dy);
  cudaFree(de);
  cudaFree(dp);
  return st;
}
