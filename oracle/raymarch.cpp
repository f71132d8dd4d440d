// ORACLE — test infrastructure, not product code.
//
// CPU restatement of fenix's volume raymarch, the fragment shader of
// src/engine/render/passes/createVolumeRaymarchPass.ts (:300-726), with the host
// packing of its render() (:184-266), setRenderParams (:268-281), the light
// sanitizing (:47-80) and the world bounds of
// src/engine/render/volumetrics/volumeWorldBounds.ts:17-33.
//
// Parity status: unpinned against the reference itself (its WGSL cannot run
// here: no WebGPU adapter). The product's CUDA raymarch is compared with this
// restatement bit for bit; the choices both share are written below.
//  - A pixel is the fragment output, or (0, 0, 0, 0) where the fragment
//    discards: the reference clears the target to 0 and blends with
//    (one, one-minus-src-alpha).
//  - The fragment uv at pixel (x, y) of a W x H image is u = (x + 0.5) / W,
//    v = 1 - (y + 0.5) / H (row 0 at the top).
//  - f32 arithmetic in the shader's order without contraction (build with
//    -ffp-contract=off); WGSL builtins by their spec formulas; round() half to
//    even; float -> u32 saturating; min/max as b < a ? b : a and a < b ? b : a.
//  - exp and pow: the project's pinned algorithms (FP64 cores below, rounded once
//    to f32). The step count is clamped to [32, 4096].
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

// exp: x = k ln2 + r (Cody-Waite, ln2 in 32 + 53 bits), Taylor polynomial of
// degree 12 (1/k!) by Horner with fused multiply-adds, times 2^k.
double exp_core(double x) {
  if (x != x) return x;
  if (x > 709.0) return INFINITY;
  if (x < -745.5) return 0.0;
  const double k = std::nearbyint(x * 0x1.71547652b82fep+0);
  const double r = (x - k * 0x1.62e42fee00000p-1) - k * 0x1.a39ef35793c76p-33;
  static const double c[13] = {0x1.1eed8eff8d898p-29, 0x1.ae64567f544e4p-26, 0x1.27e4fb7789f5cp-22, 0x1.71de3a556c734p-19,
                               0x1.a01a01a01a01ap-16, 0x1.a01a01a01a01ap-13, 0x1.6c16c16c16c17p-10, 0x1.1111111111111p-7,
                               0x1.5555555555555p-5,  0x1.5555555555555p-3,  0x1.0000000000000p-1,  1.0,
                               1.0};
  double p = c[0];
  for (int i = 1; i < 13; ++i) p = std::fma(p, r, c[i]);
  return std::scalbn(p, (int)k);
}

// log: x = m 2^e, m in [sqrt(1/2), sqrt(2)), s = (m-1)/(m+1), log m = 2 s sum s^2k/(2k+1).
double log_core(double x) {
  int e = 0;
  double m = std::frexp(x, &e);
  if (m < 0x1.6a09e667f3bcdp-1) {
    m = m * 2.0;
    e -= 1;
  }
  const double s = (m - 1.0) / (m + 1.0);
  const double s2 = s * s;
  static const double c[12] = {0x1.642c8590b2164p-5, 0x1.8618618618618p-5, 0x1.af286bca1af28p-5, 0x1.e1e1e1e1e1e1ep-5,
                               0x1.1111111111111p-4, 0x1.3b13b13b13b14p-4, 0x1.745d1745d1746p-4, 0x1.c71c71c71c71cp-4,
                               0x1.2492492492492p-3, 0x1.999999999999ap-3, 0x1.5555555555555p-2, 1.0};
  double p = c[0];
  for (int i = 1; i < 12; ++i) p = std::fma(p, s2, c[i]);
  return (double)e * 0x1.62e42fefa39efp-1 + 2.0 * s * p;
}

float fexp(float x) { return (float)exp_core((double)x); }

float fpow(float x, float y) {
  if (std::isnan(x) || std::isnan(y) || x < 0.0f) return std::nanf("");
  if (x == 0.0f) return y > 0.0f ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
  if (std::isinf(x)) return y > 0.0f ? INFINITY : (y == 0.0f ? 1.0f : 0.0f);
  return (float)exp_core((double)y * log_core((double)x));
}

float fmin_(float a, float b) { return b < a ? b : a; }
float fmax_(float a, float b) { return a < b ? b : a; }
float fclamp(float x, float lo, float hi) { return fmin_(fmax_(x, lo), hi); }
float fmix(float a, float b, float t) { return a * (1.0f - t) + b * t; }
float fsmooth(float e0, float e1, float x) {
  const float t = fclamp((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
uint32_t u32of(float f) {
  if (!(f > 0.0f)) return 0u;
  if (f >= 4294967040.0f) return 0xffffffffu;
  return (uint32_t)f;
}

struct Vec {
  float x, y, z;
};
Vec vec(float x, float y, float z) { return Vec{x, y, z}; }
Vec operator+(Vec a, Vec b) { return vec(a.x + b.x, a.y + b.y, a.z + b.z); }
Vec operator-(Vec a, Vec b) { return vec(a.x - b.x, a.y - b.y, a.z - b.z); }
Vec operator*(Vec a, Vec b) { return vec(a.x * b.x, a.y * b.y, a.z * b.z); }
Vec operator*(Vec a, float s) { return vec(a.x * s, a.y * s, a.z * s); }
Vec operator*(float s, Vec a) { return vec(s * a.x, s * a.y, s * a.z); }
Vec operator/(Vec a, Vec b) { return vec(a.x / b.x, a.y / b.y, a.z / b.z); }
Vec operator/(Vec a, float s) { return vec(a.x / s, a.y / s, a.z / s); }
Vec operator-(Vec a) { return vec(-a.x, -a.y, -a.z); }
float dot(Vec a, Vec b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
float length(Vec a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
Vec normalize(Vec a) { return a / length(a); }
Vec mixs(Vec a, Vec b, float t) { return vec(fmix(a.x, b.x, t), fmix(a.y, b.y, t), fmix(a.z, b.z, t)); }
Vec mixv(Vec a, Vec b, Vec t) { return vec(fmix(a.x, b.x, t.x), fmix(a.y, b.y, t.y), fmix(a.z, b.z, t.z)); }
Vec clampv(Vec a, Vec lo, Vec hi) { return vec(fclamp(a.x, lo.x, hi.x), fclamp(a.y, lo.y, hi.y), fclamp(a.z, lo.z, hi.z)); }
Vec expv(Vec a) { return vec(fexp(a.x), fexp(a.y), fexp(a.z)); }

struct Light {
  Vec dir;
  float kind;
  Vec pos;
  float intensity;
  Vec color;
};

struct Shader {
  // uniforms (f32 as the reference's Float32Array holds them)
  Vec cam_pos, right, up, fwd, vcenter, half;
  float aspect, tanh_, mode, step_count, scat_f, scat_b, light_count;
  Light lights[3];
  float res[3];
  uint32_t bricks[3], brick_size;
  const float* d;
  const float* t;
  const float* fu;
  const float* re;
  const uint32_t* flags;

  Vec bounds() const { return vec(res[0], res[1], res[2]) - vec(1.0f, 1.0f, 1.0f); }
  uint32_t flatten(uint32_t x, uint32_t y, uint32_t z) const { return x + u32of(res[0]) * (y + u32of(res[1]) * z); }

  bool active_sample(Vec p) const {
    const Vec c = clampv(p, vec(0, 0, 0), bounds());
    const uint32_t bs = std::max(brick_size, 1u);
    const uint32_t bx = std::min(u32of(std::floor(c.x)) / bs, bricks[0] - 1), by = std::min(u32of(std::floor(c.y)) / bs, bricks[1] - 1),
                   bz = std::min(u32of(std::floor(c.z)) / bs, bricks[2] - 1);
    return flags[bx + bricks[0] * (by + bricks[1] * bz)] != 0u;
  }

  float next_brick(Vec p, Vec dir) const {
    const float far = 1e9f;
    const float ext = (float)std::max(brick_size, 1u);
    const Vec bc = vec(std::floor(p.x / ext), std::floor(p.y / ext), std::floor(p.z / ext));
    const Vec b = vec(dir.x > 0.0f ? (bc.x + 1.0f) * ext : bc.x * ext, dir.y > 0.0f ? (bc.y + 1.0f) * ext : bc.y * ext,
                      dir.z > 0.0f ? (bc.z + 1.0f) * ext : bc.z * ext);
    const float tx = std::fabs(dir.x) > 0.00001f ? (b.x - p.x) / dir.x : far;
    const float ty = std::fabs(dir.y) > 0.00001f ? (b.y - p.y) / dir.y : far;
    const float tz = std::fabs(dir.z) > 0.00001f ? (b.z - p.z) / dir.z : far;
    return fmin_(tx, fmin_(ty, tz)) * length(dir) + 0.5f;
  }

  void sample(Vec p, float out[4]) const {
    const Vec dims = bounds();
    const Vec c = clampv(p, vec(0, 0, 0), dims);
    const uint32_t x0 = u32of(std::floor(c.x)), y0 = u32of(std::floor(c.y)), z0 = u32of(std::floor(c.z));
    const uint32_t x1 = std::min(x0 + 1, u32of(dims.x)), y1 = std::min(y0 + 1, u32of(dims.y)), z1 = std::min(z0 + 1, u32of(dims.z));
    const float fx = c.x - std::floor(c.x), fy = c.y - std::floor(c.y), fz = c.z - std::floor(c.z);
    const float* fields[4] = {d, t, fu, re};
    for (int k = 0; k < 4; ++k) {
      const float* f = fields[k];
      const float a = fmix(f[flatten(x0, y0, z0)], f[flatten(x1, y0, z0)], fx);
      const float b = fmix(f[flatten(x0, y1, z0)], f[flatten(x1, y1, z0)], fx);
      const float cc = fmix(f[flatten(x0, y0, z1)], f[flatten(x1, y0, z1)], fx);
      const float e = fmix(f[flatten(x0, y1, z1)], f[flatten(x1, y1, z1)], fx);
      out[k] = fmix(fmix(a, b, fy), fmix(cc, e, fy), fz);
    }
  }

  float nearest_density(Vec p) const {
    const Vec dims = bounds();
    return d[flatten(std::min(u32of(std::floor(p.x)), u32of(dims.x)), std::min(u32of(std::floor(p.y)), u32of(dims.y)),
                     std::min(u32of(std::floor(p.z)), u32of(dims.z)))];
  }

  Vec gradient(Vec p) const {
    const Vec dims = bounds();
    const uint32_t mx = u32of(dims.x), my = u32of(dims.y), mz = u32of(dims.z);
    const uint32_t x = std::min(u32of(std::nearbyint(p.x)), mx), y = std::min(u32of(std::nearbyint(p.y)), my),
                   z = std::min(u32of(std::nearbyint(p.z)), mz);
    return vec(d[flatten(std::min(x + 1, mx), y, z)] - d[flatten(x == 0 ? 0 : x - 1, y, z)],
               d[flatten(x, std::min(y + 1, my), z)] - d[flatten(x, y == 0 ? 0 : y - 1, z)],
               d[flatten(x, y, std::min(z + 1, mz))] - d[flatten(x, y, z == 0 ? 0 : z - 1)]);
  }

  Vec light_dir(int i, Vec wp) const {
    if (lights[i].kind > 0.5f) return normalize(lights[i].pos - wp);
    const Vec raw = lights[i].dir;
    return normalize(dot(raw, raw) > 0.0001f ? raw : vec(-0.34f, 0.88f, 0.31f));
  }
  float light_att(int i, Vec wp) const {
    if (lights[i].kind <= 0.5f) return 1.0f;
    const float dist = length(lights[i].pos - wp);
    return 1.0f / (1.0f + dist * 0.09f + dist * dist * 0.02f);
  }

  static Vec fire(float temperature) {
    const Vec ember = vec(0.18f, 0.018f, 0.0f), red = vec(1.0f, 0.075f, 0.012f), orange = vec(1.0f, 0.42f, 0.035f),
              white = vec(1.0f, 0.86f, 0.56f);
    return mixs(mixs(mixs(ember, red, fsmooth(0.01f, 0.11f, temperature)), orange, fsmooth(0.09f, 0.38f, temperature)), white,
                fsmooth(0.58f, 0.92f, temperature));
  }
  static Vec albedo(float density, float temperature, float hot) {
    const float warm_tint = fclamp(temperature * 0.38f, 0.0f, 1.0f);
    const float soot = fsmooth(0.16f, 0.9f, density) * (1.0f - fsmooth(0.2f, 0.74f, hot));
    return mixs(mixs(vec(0.26f, 0.275f, 0.295f), vec(0.04f, 0.041f, 0.045f), soot * 0.86f), vec(0.36f, 0.27f, 0.18f),
                warm_tint * (0.35f + hot * 0.45f));
  }
  static float hg(float cos_theta, float g) {
    const float g2 = g * g;
    const float denom = fpow(fmax_(1.0f + g2 - 2.0f * g * cos_theta, 0.001f), 1.5f);
    return (1.0f - g2) / (12.566370614359172f * denom);
  }
  float transmittance(Vec sp, Vec dims, Vec step, float density, float hot) const {
    const Vec p1 = clampv(sp + step * 0.9f, vec(0, 0, 0), dims);
    const Vec p2 = clampv(sp + step * 2.0f, vec(0, 0, 0), dims);
    const Vec p3 = clampv(sp + step * 3.6f, vec(0, 0, 0), dims);
    const float d1 = fmax_(nearest_density(p1) - 0.004f, 0.0f);
    const float d2 = fmax_(nearest_density(p2) - 0.004f, 0.0f);
    const float d3 = fmax_(nearest_density(p3) - 0.004f, 0.0f);
    const float depth = density * 0.34f + d1 * 1.15f + d2 * 0.72f + d3 * 0.4f - hot * 0.06f;
    return fexp(-fmax_(depth, 0.0f) * 2.15f);
  }
  static Vec thermal(float temperature, float fuel, float reaction, float density) {
    const float heat = fclamp(temperature * 1.25f + fuel * 0.18f + reaction * 0.34f, 0.0f, 1.0f);
    const float flame = fclamp(temperature * 0.9f + fuel * 0.12f + reaction * 0.18f, 0.0f, 1.0f);
    return fire(flame) * heat * heat * fsmooth(0.012f, 0.38f, density) * 0.18f;
  }

  // fsMain; false where the fragment discards
  bool fragment(float u, float v, float out[4]) const {
    const float nx = u * 2.0f - 1.0f, ny = v * 2.0f - 1.0f;
    const Vec ray = normalize(fwd + right * nx * aspect * tanh_ + up * ny * tanh_);
    const Vec bmin = vcenter - half, bmax = vcenter + half;
    const Vec inv = vec(1.0f, 1.0f, 1.0f) / ray;
    const Vec a = (bmin - cam_pos) * inv, b = (bmax - cam_pos) * inv;
    const Vec lo = vec(fmin_(a.x, b.x), fmin_(a.y, b.y), fmin_(a.z, b.z)), hi = vec(fmax_(a.x, b.x), fmax_(a.y, b.y), fmax_(a.z, b.z));
    float t0 = fmax_(lo.x, fmax_(lo.y, lo.z));
    const float t1 = fmin_(hi.x, fmin_(hi.y, hi.z));
    if (t0 > t1) return false;
    t0 = fmax_(t0, 0.0f);
    const uint32_t steps = u32of(step_count);
    const Vec inv_ext = vec(1.0f, 1.0f, 1.0f) / (half * 2.0f);
    const Vec dims = bounds();
    const Vec vdir = ray * inv_ext * dims;
    const float vdelta = length(vdir) * (t1 - t0) / fmax_((float)steps, 1.0f);
    const float wdelta = (t1 - t0) / fmax_((float)steps, 1.0f);
    const uint32_t nl = u32of(fclamp(light_count, 0.0f, 3.0f));
    const Vec primary = nl > 0 ? light_dir(0, cam_pos) : vec(0.0f, 1.0f, 0.0f);
    const Vec lstep = primary * dims * 0.036f;
    Vec pos = (cam_pos + ray * t0 - bmin) * inv_ext * dims;
    float travelled = 0.0f;
    const float ray_len = length(vdir) * (t1 - t0);
    Vec color = vec(0, 0, 0);
    float alpha = 0.0f;
    for (uint32_t i = 0; i < steps && travelled <= ray_len; ++i) {
      if (alpha > 0.985f) break;
      float vstep = vdelta;
      const Vec sp = pos;
      const Vec uvw = sp / dims;
      if (active_sample(sp)) {
        float s[4];
        sample(sp, s);
        const float density = fmax_(s[0] - 0.004f, 0.0f);
        const float temperature = s[1], fuel = s[2], reaction = s[3];
        const float hot = fclamp(temperature * 1.45f + fuel * 0.22f + reaction * 0.38f, 0.0f, 1.0f);
        if (density > 0.001f || hot > 0.018f) {
          if (density < 0.012f && hot < 0.04f) {
            vstep = vdelta * 1.8f;
          } else {
            const Vec g = gradient(sp);
            const float glen = fmax_(length(g), 0.0001f);
            const Vec normal = glen > 0.00011f ? -g / glen : vec(0.0f, 1.0f, 0.0f);
            const float detail = fclamp(glen * 5.2f + hot * 0.28f + reaction * 0.18f, 0.0f, 1.0f);
            const float dd = fmax_(fpow(density, 0.96f) * fmix(0.82f, 1.42f, detail), 0.0f);
            const Vec wp = mixv(bmin, bmax, uvw);
            const float fade = 1.0f - fsmooth(0.9f, 0.995f, uvw.y);
            Vec light = vec(0, 0, 0);
            const float primary_t = nl > 0 ? transmittance(sp, dims, lstep, dd, hot) : 1.0f;
            for (uint32_t li = 0; li < 3; ++li) {
              if (li >= nl) break;
              const Vec to = light_dir((int)li, wp);
              const float raw = std::max(lights[li].intensity, 0.0f) * light_att((int)li, wp);
              const float power = raw / (1.0f + raw * 0.18f);
              const float vc = fclamp(dot(to, -ray), -1.0f, 1.0f);
              const float fwd_s = hg(vc, scat_f) * 5.2f * power;
              const float back_s = hg(vc, scat_b) * 1.55f * power;
              const float facing = fclamp(dot(normal, to) * 0.5f + 0.5f, 0.0f, 1.0f);
              const float surface = fpow(facing, 1.35f) * fmix(1.0f, 0.56f, fsmooth(0.16f, 0.9f, dd));
              const float rim = fpow(1.0f - std::fabs(dot(normal, -ray)), 2.4f) * fpow(fclamp(dot(to, -ray) * 0.5f + 0.5f, 0.0f, 1.0f), 1.2f);
              const float directional = (surface * 0.42f + rim * 0.22f) * power;
              const float scatter = (fwd_s + back_s) * fmix(0.36f, 0.74f, hot);
              const float trans = li > 0 ? 1.0f : primary_t;
              light = light + lights[li].color * trans * (directional + scatter);
            }
            const Vec tone = vec(1.0f, 1.0f, 1.0f) - expv(-light * 0.72f);
            const Vec smoke = albedo(dd, temperature, hot);
            const float absorb = fmix(0.92f, 0.34f, fsmooth(0.26f, 1.05f, dd));
            const Vec lit = smoke * vec(0.045f, 0.048f, 0.052f) + smoke * tone * absorb + tone * fsmooth(0.018f, 0.22f, dd) * 0.18f +
                            thermal(temperature, fuel, reaction, dd);
            const float flame_heat = fclamp(temperature * 0.9f + fuel * 0.14f + reaction * 0.16f, 0.0f, 1.0f);
            const Vec emissive = fire(flame_heat) * hot * (0.48f + fuel * 0.16f + reaction * 0.24f);
            const float contribution = fclamp(dd * 1.35f + hot * 1.25f, 0.0f, 1.0f);
            const float sdist = wdelta * fmix(1.02f, 0.76f, contribution);
            vstep = vdelta * fmix(1.02f, 0.76f, contribution);
            Vec composite = lit + emissive;
            float opacity = (1.0f - fexp(-(dd * 4.75f + hot * 0.42f) * sdist)) * fade;
            if (mode > 0.5f && mode < 1.5f) {
              composite = mixs(vec(0.01f, 0.01f, 0.012f), vec(0.88f, 0.9f, 0.94f), fclamp(dd * 1.4f, 0.0f, 1.0f));
              opacity = 1.0f - fexp(-dd * sdist * 8.6f);
            } else if (mode >= 1.5f) {
              composite = mixs(vec(0.04f, 0.012f, 0.0f), vec(1.0f, 0.72f, 0.22f), fclamp(fuel * 1.3f, 0.0f, 1.0f));
              opacity = 1.0f - fexp(-fuel * sdist * 7.0f);
            }
            color = color + (1.0f - alpha) * composite * opacity;
            alpha = alpha + (1.0f - alpha) * opacity;
          }
        } else {
          vstep = vdelta * 1.35f;
        }
      } else {
        vstep = fmax_(next_brick(sp, vdir), vdelta);
      }
      pos = pos + normalize(vdir) * vstep;
      travelled = travelled + vstep;
    }
    if (alpha < 0.01f) return false;
    out[0] = color.x;
    out[1] = color.y;
    out[2] = color.z;
    out[3] = alpha;
    return true;
  }
};

double clampd(double v, double lo, double hi) { return std::max(lo, std::min(hi, v)); }
int jsround(double v) { return (int)std::floor(v + 0.5); }

}  // namespace

extern "C" {

// camera: position[3], target[3], forward[3], right[3], up[3], aspect, tanHalfFovY.
// settings: has_step, step_count, has_forward, forward, has_back, back.
// lights: light_count x {type, direction[3], position[3], color[3], intensity};
// light_count < 0 keeps the default light. rgba: width x height x 4 floats.
void orc_raymarch(const float* density, const float* temperature, const float* fuel, const float* reaction, const uint32_t* flags,
                  uint32_t w, uint32_t h, uint32_t d, const double* camera, int display_mode, uint32_t width, uint32_t height,
                  double elapsed, const double* settings, int light_count, const double* lights, float* rgba) {
  (void)elapsed;
  Shader s;
  std::memset(&s, 0, sizeof s);
  const double scale = 13.5, mh = (double)std::max(w, d);
  const double half[3] = {2.05 * scale * (w / mh), 2.05 * scale * (h / mh), 2.05 * scale * (d / mh)};
  const double voxels = (double)w * h * d;
  int steps = (int)clampd(jsround(std::max({w, h, d}) * 1.5), 180, voxels >= 4000000.0 ? 720 : 560);
  if (settings[0] != 0.0) steps = std::min(4096, std::max(32, jsround(std::min(std::max(settings[1], -1e6), 1e6))));
  const double sf = settings[2] != 0.0 ? clampd(settings[3], 0.0, 0.98) : 0.32;
  const double sb = settings[4] != 0.0 ? clampd(settings[5], -0.98, 0.0) : -0.18;
  double L[3][11];
  int nl = light_count;
  if (nl < 0) {
    const double dflt[11] = {0, -0.34, 0.88, 0.31, 0, 0, 0, 1.0, 0.95, 0.88, 1.25};
    std::memcpy(L[0], dflt, sizeof dflt);
    nl = 1;
  } else {
    nl = std::min(nl, 3);
    for (int i = 0; i < nl; ++i) std::memcpy(L[i], lights + 11 * i, sizeof L[i]);
  }
  for (int i = 0; i < nl; ++i) {  // sanitizeRenderLights
    double* l = L[i];
    const double len = std::sqrt(l[1] * l[1] + l[2] * l[2] + l[3] * l[3]);
    if (len <= 0.0001) {
      l[1] = -0.34;
      l[2] = 0.88;
      l[3] = 0.31;
    } else {
      l[1] /= len;
      l[2] /= len;
      l[3] /= len;
    }
    for (int k = 7; k < 10; ++k) l[k] = std::max(l[k], 0.0);
    l[10] = std::max(l[10], 0.0);
    s.lights[i].dir = vec((float)l[1], (float)l[2], (float)l[3]);
    s.lights[i].kind = l[0] == 1.0 ? 1.0f : 0.0f;
    s.lights[i].pos = vec((float)l[4], (float)l[5], (float)l[6]);
    s.lights[i].intensity = (float)l[10];
    s.lights[i].color = vec((float)l[7], (float)l[8], (float)l[9]);
  }
  auto fv = [&](int o) { return vec((float)camera[o], (float)camera[o + 1], (float)camera[o + 2]); };
  s.cam_pos = fv(0);
  s.fwd = fv(6);
  s.right = fv(9);
  s.up = fv(12);
  s.vcenter = vec(0.0f, (float)(half[1] - 0.25), 0.0f);
  s.half = vec((float)half[0], (float)half[1], (float)half[2]);
  s.aspect = (float)camera[15];
  s.tanh_ = (float)camera[16];
  s.mode = (float)display_mode;
  s.step_count = (float)steps;
  s.scat_f = (float)sf;
  s.scat_b = (float)sb;
  s.light_count = (float)nl;
  s.res[0] = (float)w;
  s.res[1] = (float)h;
  s.res[2] = (float)d;
  s.bricks[0] = (w + 7) / 8;
  s.bricks[1] = (h + 7) / 8;
  s.bricks[2] = (d + 7) / 8;
  s.brick_size = 8;
  s.d = density;
  s.t = temperature;
  s.fu = fuel;
  s.re = reaction;
  s.flags = flags;
#pragma omp parallel for schedule(dynamic, 4)
  for (int64_t py = 0; py < (int64_t)height; ++py)
    for (uint32_t px = 0; px < width; ++px) {
      const float u = ((float)px + 0.5f) / (float)width;
      const float v = 1.0f - ((float)py + 0.5f) / (float)height;
      float o[4] = {0.0f, 0.0f, 0.0f, 0.0f};
      s.fragment(u, v, o);
      std::memcpy(rgba + ((size_t)py * width + px) * 4, o, sizeof o);
    }
}

// Bloom: createBloomPass.ts (:216-297) with render() (:93-130). `hdr` holds
// width x height RGBA f32 pixels (an RGBA16F source converted exactly), row 0 at
// the top; the three half-resolution textures are RGBA16F (each value rounded to
// nearest f16 on store). The fragment uv at pixel (x, y) of a W x H target is
// ((x + 0.5) / W, (y + 0.5) / H); textureSample with the linear sampler is
// bilinear with exact f32 weights, clamp-to-edge. Writes out_f32 (RGBA f32) and,
// when non-NULL, out_u8 (round(clamp(x, 0, 1) * 255), half to even).
void orc_bloom(const float* hdr, uint32_t width, uint32_t height, int enabled, double threshold, double strength, double radius,
               float* out_f32, uint8_t* out_u8) {
  struct Tex {
    const float* px;
    uint32_t w, h;
    float at(int x, int y, int c) const {
      x = std::min(std::max(x, 0), (int)w - 1);
      y = std::min(std::max(y, 0), (int)h - 1);
      return px[((size_t)y * w + x) * 4 + c];
    }
    void sample(float u, float v, float o[4]) const {
      const float fx = u * (float)w - 0.5f, fy = v * (float)h - 0.5f;
      const float bx = std::floor(fx), by = std::floor(fy);
      const float tx = fx - bx, ty = fy - by;
      const int x = (int)bx, y = (int)by;
      for (int c = 0; c < 4; ++c) {
        const float top = fmix(at(x, y, c), at(x + 1, y, c), tx);
        const float bottom = fmix(at(x, y + 1, c), at(x + 1, y + 1, c), tx);
        o[c] = fmix(top, bottom, ty);
      }
    }
  };
  auto f16 = [](float x) { return (float)(_Float16)x; };
  const float thr = (float)threshold, str = (float)strength, rad = (float)radius;
  const uint32_t hw = std::max(1u, width / 2), hh = std::max(1u, height / 2);
  const Tex src{hdr, width, height};
  std::vector<float> bright((size_t)hw * hh * 4), blur_h(bright.size()), blur_v(bright.size());
  if (enabled) {
    for (uint32_t y = 0; y < hh; ++y)  // threshold (:224-233)
      for (uint32_t x = 0; x < hw; ++x) {
        float c[4];
        src.sample(((float)x + 0.5f) / (float)hw, ((float)y + 0.5f) / (float)hh, c);
        const float lum = c[0] * 0.2126f + c[1] * 0.7152f + c[2] * 0.0722f;
        const float knee = thr * 0.5f;
        const float rq = fclamp(lum - thr + knee, 0.0f, 2.0f * knee);
        const float wq = (rq * rq) / (4.0f * knee * knee + 0.00001f);
        const float mask = fmax_(wq, lum >= thr ? 1.0f : 0.0f);
        float* o = &bright[((size_t)y * hw + x) * 4];
        for (int k = 0; k < 3; ++k) o[k] = f16(c[k] * mask * c[3]);
        o[3] = f16(c[3] * mask);
      }
    static const float g[5] = {0.2270270270f, 0.1945945946f, 0.1216216216f, 0.0540540541f, 0.0162162162f};
    const float spread = 1.0f + rad * 2.0f;
    for (int pass = 0; pass < 2; ++pass) {  // blur along x, then y (:246-263)
      const Tex in{pass == 0 ? bright.data() : blur_h.data(), hw, hh};
      std::vector<float>& outv = pass == 0 ? blur_h : blur_v;
      const float step_x = (pass == 0 ? 1.0f / (float)hw : 0.0f) * spread, step_y = (pass == 0 ? 0.0f : 1.0f / (float)hh) * spread;
      for (uint32_t y = 0; y < hh; ++y)
        for (uint32_t x = 0; x < hw; ++x) {
          const float u = ((float)x + 0.5f) / (float)hw, v = ((float)y + 0.5f) / (float)hh;
          float acc[4], t[4];
          in.sample(u, v, t);
          for (int c = 0; c < 4; ++c) acc[c] = t[c] * g[0];
          for (int k = 1; k <= 4; ++k)
            for (int sign = 1; sign >= -1; sign -= 2) {
              const float du = step_x * (float)k, dv = step_y * (float)k;
              in.sample(sign > 0 ? u + du : u - du, sign > 0 ? v + dv : v - dv, t);
              for (int c = 0; c < 4; ++c) acc[c] = acc[c] + t[c] * g[k];
            }
          for (int c = 0; c < 4; ++c) outv[((size_t)y * hw + x) * 4 + c] = f16(acc[c]);
        }
    }
  }
  const Tex glow_tex{blur_v.data(), hw, hh};
  for (uint32_t y = 0; y < height; ++y)  // composite (:290-297) or blit (:273-277)
    for (uint32_t x = 0; x < width; ++x) {
      const float u = ((float)x + 0.5f) / (float)width, v = ((float)y + 0.5f) / (float)height;
      float base[4], r[4];
      src.sample(u, v, base);
      if (enabled) {
        float glow[4];
        glow_tex.sample(u, v, glow);
        for (int c = 0; c < 3; ++c) r[c] = fpow(fmax_(base[c] + fmax_(glow[c], 0.0f) * str, 0.0f), 0.92f);
        const float ga = fclamp(glow[3] * str, 0.0f, 1.0f);
        r[3] = fclamp(base[3] + ga * (1.0f - base[3]), 0.0f, 1.0f);
      } else {
        for (int c = 0; c < 3; ++c) r[c] = fpow(fmax_(base[c], 0.0f), 0.92f);
        r[3] = fclamp(base[3], 0.0f, 1.0f);
      }
      const size_t o = ((size_t)y * width + x) * 4;
      for (int c = 0; c < 4; ++c) {
        if (out_f32) out_f32[o + c] = r[c];
        if (out_u8) out_u8[o + c] = (uint8_t)std::nearbyint(fclamp(r[c], 0.0f, 1.0f) * 255.0f);
      }
    }
}

// The pinned f32 exp and pow, for tests.
void orc_pinned_exp_pow(const float* x, const float* y, float* oe, float* op, long n) {
  for (long i = 0; i < n; ++i) {
    oe[i] = fexp(x[i]);
    op[i] = fpow(x[i], y[i]);
  }
}

}  // extern "C"
