// ORACLE — test infrastructure, not product code.
//
// A CPU restatement of fenix's per-frame combustion-volume step, written pass by
// pass from the reference's WGSL kernels and its TypeScript host schedule. Only the
// test suite, the smoke check and the CPU-baseline leg of the benchmark load this
// library; the CUDA product never links or calls it.
//
// Parity status: UNPINNED against the reference itself. The reference is a
// TypeScript/WebGPU app with no CPU implementation of this step, no tests and no
// golden vectors, and its WGSL cannot run in this environment (no JS runtime, no
// WebGPU adapter). This file is therefore pinned only by (1) analytic known-answer
// tests and (2) an independent numpy restatement of the stencil passes, both under
// tests/.
//
// Two instantiations:
//   Real = float  : the reference's f32 arithmetic, evaluated strictly in source
//                   order with no FMA contraction (build with -ffp-contract=off).
//                   sin/cos use the project's pinned f32 algorithm (below), which
//                   the CUDA kernels implement identically, so CUDA == oracle bit
//                   for bit. This instantiation is also the timed CPU baseline.
//   Real = double : the accuracy reference (libm sin/cos), used to state the f32
//                   and f16-storage error of the CUDA path.
//   Real = Tan, Tan32 : tangent numbers (FP64 values, or f32 values on the f32
//                   trajectory bit for bit, each with an FP64 directional
//                   derivative): the exact derivative of the restatement along a
//                   seeded direction, the reference for the CUDA adjoint.
// Either instantiation can store the scalar sets in binary16 (orc_set_half_storage):
// each value a reference pass writes to density, temperature, fuel or reaction is
// rounded to the nearest binary16, ties to even, as the CUDA FP16-storage path does.
//
// WGSL builtin semantics used throughout (WGSL spec formulas):
//   mix(a,b,t) = a*(1-t) + b*t;  smoothstep(e0,e1,x) = t*t*(3-2t), t=clamp((x-e0)/(e1-e0),0,1)
//   fract(x) = x - floor(x);  step(e,x) = x >= e;  clamp(x,lo,hi) = min(max(x,lo),hi)
//   length(v) = sqrt(x*x + y*y + z*z);  normalize(v) = v / length(v)
//
// File map (reference paths relative to src/engine/simulation/):
//   shaders/common/indexing.wgsl.ts:2-19         flatten / clampCoord / isBoundary
//   shaders/common/clamp-utils.wgsl.ts:2-22      clamp01 / insideVolume / dec / inc
//   shaders/common/sampling-*.wgsl.ts            trilinear samplers
//   shaders/passes/*.wgsl.ts                      one function per pass below
//   runtime/createCombustionVolumeSimulation.ts:230-305   step schedule
//   runtime/passes/PressureSolvePass.ts:62-158             multilevel schedule
//   runtime/passes/SourceInjectionPass.ts:13-23           128-byte minimum source buffer

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <type_traits>
#include <vector>

#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

// ---------------------------------------------------------------------------
// Pinned f32 sin/cos. Range reduction in double by a three-part Cody-Waite split
// of pi/2 (each part with <= 33 significant bits, so k*P1 is exact for the
// quotient range that occurs), then Taylor polynomials (coefficients 1/k!) on
// |r| <= pi/4 evaluated in f32 with fused multiply-adds. Deterministic IEEE
// operations only, so gcc and nvcc produce identical bits.
// ---------------------------------------------------------------------------
constexpr double kTwoOverPi = 0x1.45f306dc9c883p-1;
constexpr double kPio2_1 = 0x1.921fb544p+0;
constexpr double kPio2_2 = 0x1.0b4611a6p-34;
constexpr double kPio2_3 = 0x1.3198a2e037073p-69;

inline float poly_sin(float r) {
  const float r2 = r * r;
  float p = std::fma(r2, -0x1.ae6456p-26f, 0x1.71de3ap-19f);
  p = std::fma(p, r2, -0x1.a01a02p-13f);
  p = std::fma(p, r2, 0x1.111112p-7f);
  p = std::fma(p, r2, -0x1.555556p-3f);
  const float r3 = r2 * r;
  return std::fma(r3, p, r);
}

inline float poly_cos(float r) {
  const float r2 = r * r;
  float p = std::fma(r2, 0x1.1eed8ep-29f, -0x1.27e4fcp-22f);
  p = std::fma(p, r2, 0x1.a01a02p-16f);
  p = std::fma(p, r2, -0x1.6c16c2p-10f);
  p = std::fma(p, r2, 0x1.555556p-5f);
  p = std::fma(p, r2, -0.5f);
  return std::fma(p, r2, 1.0f);
}

// Below |x| = 8192 the reduction runs in f32: k = rint(x * RN(2/pi)), then
// r = x - k*P1 - k*P2 - k*P3 - k*P4 by four fused multiply-adds with a Cody-Waite
// split of pi/2 into three 12-bit parts and the rounded rest (pi/2 - sum < 2^-63).
// With |k| < 2^13 the first two steps are exact (x and the products share a
// 2^-24 grid and the differences are below 1), the third is exact whenever
// |r| < 2^-11, and the split's error k * 2^-63 stays below 2^-50; the reduced
// argument is within about one unit in the last place, as in Cody and Waite,
// "Software Manual for the Elementary Functions" (1980). k may be off by one
// at quadrant boundaries; |r| then slightly exceeds pi/4, where the polynomials
// are still accurate. Larger and non-finite arguments take the double path.
constexpr float kTwoOverPiF = 0x1.45f306p-1f;
constexpr float kPio2F_1 = 0x1.92p+0f;
constexpr float kPio2F_2 = 0x1.fb4p-12f;
constexpr float kPio2F_3 = 0x1.444p-24f;
constexpr float kPio2F_4 = 0x1.68c234p-39f;

inline float poly_quadrant(float r, int q) {
  switch (q & 3) {
    case 0: return poly_sin(r);
    case 1: return poly_cos(r);
    case 2: return -poly_sin(r);
    default: return -poly_cos(r);
  }
}

// quadrant_offset: 0 for sin, 1 for cos (cos x = sin(x + pi/2)).
inline float pinned_sincos(float x, int quadrant_offset) {
  if (std::fabs(x) < 8192.0f) {
    const float kf = std::rint(x * kTwoOverPiF);
    float r = std::fma(-kf, kPio2F_1, x);
    r = std::fma(-kf, kPio2F_2, r);
    r = std::fma(-kf, kPio2F_3, r);
    r = std::fma(-kf, kPio2F_4, r);
    return poly_quadrant(r, (int)kf + quadrant_offset);
  }
  const double xd = (double)x;
  const double k = std::rint(xd * kTwoOverPi);
  double r = std::fma(-k, kPio2_1, xd);
  r = std::fma(-k, kPio2_2, r);
  r = std::fma(-k, kPio2_3, r);
  const double kq = k - 4.0 * std::floor(k * 0.25);
  int q = (int)kq;
  if (!(q >= 0 && q <= 3)) q = 0;  // non-finite input: r is NaN already
  q = (q + quadrant_offset) & 3;
  const float rf = (float)r;
  switch (q) {
    case 0: return poly_sin(rf);
    case 1: return poly_cos(rf);
    case 2: return -poly_sin(rf);
    default: return -poly_cos(rf);
  }
}

// Tangent numbers: a value (V = double for the FP64 restatement, V = float
// for the f32 one) with one directional derivative in FP64. Sim<Tan> and
// Sim<Tan32> evaluate the restatement in forward mode, which gives the exact
// derivative of its output along a chosen input direction (the check of the
// product's hand-written adjoint); Sim<Tan32> follows the f32 trajectory bit for
// bit. A branch (min, max, clamp, select) follows the value and carries the
// derivative of the branch taken; floor has derivative 0; sqrt has derivative 0
// at 0.
template <class V>
struct TanT {
  V v = 0;
  double d = 0.0;
  TanT() = default;
  TanT(double x) : v((V)x), d(0.0) {}
  TanT(V x, double dx, int) : v(x), d(dx) {}
  explicit operator double() const { return (double)v; }
  explicit operator float() const { return (float)v; }
  explicit operator uint32_t() const { return (uint32_t)v; }
  TanT operator-() const { return TanT(-v, -d, 0); }
  TanT& operator+=(TanT b) { v += b.v; d += b.d; return *this; }
  TanT& operator-=(TanT b) { v -= b.v; d -= b.d; return *this; }
  TanT& operator*=(TanT b) { d = d * (double)b.v + (double)v * b.d; v *= b.v; return *this; }
};
template <class V> inline TanT<V> operator+(TanT<V> a, TanT<V> b) { return TanT<V>(a.v + b.v, a.d + b.d, 0); }
template <class V> inline TanT<V> operator-(TanT<V> a, TanT<V> b) { return TanT<V>(a.v - b.v, a.d - b.d, 0); }
template <class V> inline TanT<V> operator*(TanT<V> a, TanT<V> b) {
  return TanT<V>(a.v * b.v, a.d * (double)b.v + (double)a.v * b.d, 0);
}
template <class V> inline TanT<V> operator/(TanT<V> a, TanT<V> b) {
  const V q = a.v / b.v;
  return TanT<V>(q, (a.d - (double)q * b.d) / (double)b.v, 0);
}
#define FX_TAN_MIXED(op)                                                                          \
  template <class V> inline auto operator op(TanT<V> a, double b) { return a op TanT<V>(b); }    \
  template <class V> inline auto operator op(double a, TanT<V> b) { return TanT<V>(a) op b; }
FX_TAN_MIXED(+)
FX_TAN_MIXED(-)
FX_TAN_MIXED(*)
FX_TAN_MIXED(/)
#undef FX_TAN_MIXED
template <class V> inline bool operator<(TanT<V> a, TanT<V> b) { return a.v < b.v; }
template <class V> inline bool operator>(TanT<V> a, TanT<V> b) { return a.v > b.v; }
template <class V> inline bool operator<=(TanT<V> a, TanT<V> b) { return a.v <= b.v; }
template <class V> inline bool operator>=(TanT<V> a, TanT<V> b) { return a.v >= b.v; }
template <class V> inline bool operator==(TanT<V> a, TanT<V> b) { return a.v == b.v; }
template <class V> inline bool operator!=(TanT<V> a, TanT<V> b) { return a.v != b.v; }
using Tan = TanT<double>;
using Tan32 = TanT<float>;

template <class R> struct is_tan : std::false_type {};
template <class V> struct is_tan<TanT<V>> : std::true_type {};
// Instantiations whose values are f32 (f32 literals and the pinned sin/cos).
template <class R> struct is_f32 : std::is_same<R, float> {};
template <> struct is_f32<Tan32> : std::true_type {};

// floor, sqrt and |x| for every instantiation.
inline float flr(float x) { return std::floor(x); }
inline double flr(double x) { return std::floor(x); }
template <class V> inline TanT<V> flr(TanT<V> x) { return TanT<V>(std::floor(x.v), 0.0, 0); }
inline float sqr(float x) { return std::sqrt(x); }
inline double sqr(double x) { return std::sqrt(x); }
template <class V> inline TanT<V> sqr(TanT<V> x) {
  const V r = std::sqrt(x.v);
  return TanT<V>(r, r > 0 ? x.d / (2.0 * (double)r) : 0.0, 0);
}
inline float absr(float x) { return std::fabs(x); }
inline double absr(double x) { return std::fabs(x); }
template <class V> inline TanT<V> absr(TanT<V> x) { return x.v < 0 ? -x : x; }

template <class R> struct Mth;
template <> struct Mth<float> {
  static float sin(float x) { return pinned_sincos(x, 0); }
  static float cos(float x) { return pinned_sincos(x, 1); }
};
template <> struct Mth<double> {
  static double sin(double x) { return std::sin(x); }
  static double cos(double x) { return std::cos(x); }
};
template <> struct Mth<Tan> {
  static Tan sin(Tan x) { return Tan(std::sin(x.v), std::cos(x.v) * x.d, 0); }
  static Tan cos(Tan x) { return Tan(std::cos(x.v), -std::sin(x.v) * x.d, 0); }
};
template <> struct Mth<Tan32> {
  static Tan32 sin(Tan32 x) { return Tan32(pinned_sincos(x.v, 0), (double)pinned_sincos(x.v, 1) * x.d, 0); }
  static Tan32 cos(Tan32 x) { return Tan32(pinned_sincos(x.v, 1), -(double)pinned_sincos(x.v, 0) * x.d, 0); }
};

// A literal in the precision of the instantiation: the f32 literal for float
// (matching WGSL's f32 constants), the f64 literal for double.
#define K(x) (static_cast<R>(is_f32<R>::value ? static_cast<double>(x##f) : static_cast<double>(x)))

template <class R> inline R mn(R a, R b) { return b < a ? b : a; }
template <class R> inline R mx(R a, R b) { return a < b ? b : a; }
template <class R> inline R clampv(R x, R lo, R hi) { return mn(mx(x, lo), hi); }
template <class R> inline R clamp01(R x) { return clampv(x, R(0), R(1)); }
template <class R> inline R mixv(R a, R b, R t) { return a * (R(1) - t) + b * t; }
template <class R> inline R fractv(R x) { return x - flr(x); }
template <class R> inline R stepv(R e, R x) { return x >= e ? R(1) : R(0); }
template <class R> inline R smoothstepv(R e0, R e1, R x) {
  const R t = clampv((x - e0) / (e1 - e0), R(0), R(1));
  return t * t * (R(3) - R(2) * t);
}
template <class R> inline R length3(R x, R y, R z) { return sqr(x * x + y * y + z * z); }

template <class R> struct V3 {
  R x, y, z;
};

struct Dims {
  uint32_t w = 0, h = 0, d = 0;
  size_t n = 0;
};

inline Dims make_dims(uint32_t w, uint32_t h, uint32_t d) {
  Dims r;
  r.w = w;
  r.h = h;
  r.d = d;
  r.n = (size_t)w * h * d;
  return r;
}

// runtime/combustion-volume-simulation/buffers.ts:10-16
inline Dims halve(const Dims& a) {
  return make_dims(std::max<uint32_t>(4, a.w / 2), std::max<uint32_t>(4, a.h / 2), std::max<uint32_t>(4, a.d / 2));
}

inline size_t flat(const Dims& dm, uint32_t x, uint32_t y, uint32_t z) {
  return (size_t)x + (size_t)dm.w * ((size_t)y + (size_t)dm.h * z);
}
inline uint32_t dec(uint32_t v) { return v == 0 ? 0 : v - 1; }
inline uint32_t inc(uint32_t v, uint32_t m) { return std::min(v + 1, m); }
inline bool is_boundary(const Dims& dm, uint32_t x, uint32_t y, uint32_t z) {
  return x == 0 || y == 0 || z == 0 || x == dm.w - 1 || y == dm.h - 1 || z == dm.d - 1;
}

// The uniform block of shaders/common/simulation-params.wgsl.ts:2-14 (all f32).
struct Params {
  float time, dt, prev_time, scalar_set;
  float wind[4];
  float gravity[4];
  float buoyancy, vorticity_strength, dx, world_size;
  float vmask[4];
};

// Trilinear sample with the clamp-to-[0, dim-1] rule of
// shaders/common/sampling-scalar.wgsl.ts:11-34. A NaN position is sent to 0
// (the rule is otherwise identical; the CUDA sampler does the same).
template <class R> inline R clamp_pos(R p, R hi) { return !(p > R(0)) ? R(0) : (p < hi ? p : hi); }

template <class R> struct Corners {
  size_t i000, i100, i010, i110, i001, i101, i011, i111;
  R fx, fy, fz;
};

template <class R> inline Corners<R> corners(const Dims& dm, R px, R py, R pz) {
  const R mxp = R(dm.w - 1), myp = R(dm.h - 1), mzp = R(dm.d - 1);
  const R cx = clamp_pos(px, mxp), cy = clamp_pos(py, myp), cz = clamp_pos(pz, mzp);
  const R flx = flr(cx), fly = flr(cy), flz = flr(cz);
  const uint32_t bx = (uint32_t)flx, by = (uint32_t)fly, bz = (uint32_t)flz;
  const uint32_t ux = std::min(bx + 1, dm.w - 1), uy = std::min(by + 1, dm.h - 1), uz = std::min(bz + 1, dm.d - 1);
  Corners<R> c;
  c.fx = cx - flx;
  c.fy = cy - fly;
  c.fz = cz - flz;
  c.i000 = flat(dm, bx, by, bz);
  c.i100 = flat(dm, ux, by, bz);
  c.i010 = flat(dm, bx, uy, bz);
  c.i110 = flat(dm, ux, uy, bz);
  c.i001 = flat(dm, bx, by, uz);
  c.i101 = flat(dm, ux, by, uz);
  c.i011 = flat(dm, bx, uy, uz);
  c.i111 = flat(dm, ux, uy, uz);
  return c;
}

template <class R> inline R interp(const R* f, const Corners<R>& c) {
  const R x00 = mixv(f[c.i000], f[c.i100], c.fx);
  const R x10 = mixv(f[c.i010], f[c.i110], c.fx);
  const R x01 = mixv(f[c.i001], f[c.i101], c.fx);
  const R x11 = mixv(f[c.i011], f[c.i111], c.fx);
  return mixv(mixv(x00, x10, c.fy), mixv(x01, x11, c.fy), c.fz);
}

template <class R> struct Level {
  Dims dm;
  std::vector<R> div, pa, pb;
};

// Field ids shared with the product's C ABI (include/fenix_cuda.h, FX_FIELD_*).
enum FieldId {
  F_DENSITY = 0, F_TEMPERATURE, F_FUEL, F_REACTION,
  F_PREV_DENSITY, F_PREV_TEMPERATURE, F_PREV_FUEL, F_PREV_REACTION,
  F_VEL_X, F_VEL_Y, F_VEL_Z,
  F_VSCR_X, F_VSCR_Y, F_VSCR_Z,
  F_VORT_X, F_VORT_Y, F_VORT_Z,
  F_VORT_MAG, F_CONF_MAG, F_VEL_MAG,
  F_FLAGS, F_PREV_FLAGS,
  F_FINE_DIV, F_FINE_PA, F_FINE_PB,
  F_MID_DIV, F_MID_PA, F_MID_PB,
  F_COARSE_DIV, F_COARSE_PA, F_COARSE_PB,
  F_PRESSURE,
  F_COUNT
};

struct Quality {
  int pressure_interval = 1, vorticity_interval = 1;
  int fine_pre = 2, fine_post = 3, mid_pre = 2, mid_post = 3, coarse = 10;
};

// Pressure solver selection. mode 0 is the reference's fixed schedule
// (PressureSolvePass.ts:68-84). mode 1 is an extension with no counterpart in the
// reference: a weighted-Jacobi V-cycle over `levels` levels (the reference's
// level sizes, buffers.ts:10-16) that runs until ||div - A p||_2 <= tol * ||div||_2
// in FP64, or max_cycles.
struct SolverSettings {
  int mode = 0, levels = 5, pre = 4, post = 4, coarse = 20, max_cycles = 30, warm = 1;
  double omega = 2.0 / 3.0, tol = 1e-5;
};

// FP64 diagnostics of the last solve: squared norms of the divergence and of the
// final residual, the max |div u| of the projected velocity, and the V-cycles run.
struct SolverStats {
  double rhs2 = 0, res2 = 0, maxdiv = 0;
  int cycles = 0, converged = 0;
};

// Stochastic rounding to binary16 (extension). sr_draw is a 32-bit hash of a
// voxel index plus the store site times 0x85EBCA77 plus the step index times
// 0x9E3779B9 (2^32 / golden ratio); sr_half rounds a finite |v| < 65504 to the binary16 value below
// it (toward zero) or the next one up, up when the distance from the lower one,
// in units of their spacing, exceeds the top 24 bits of r read as a fraction.
// Every operation is exact, so the CUDA kernels reproduce it bit for bit. Other
// values round to nearest.
inline uint32_t sr_draw(uint32_t i, uint32_t site, uint32_t step) {
  uint32_t h = i * 0x9E3779B1u;
  h ^= h >> 16;
  h *= 0x7FEB352Du;
  h ^= h >> 15;
  h *= 0x846CA68Bu;
  h ^= h >> 16;
  return h + site * 0x85EBCA77u + step * 0x9E3779B9u;
}

inline float sr_half(float v, uint32_t r) {
  const float a = std::fabs(v);
  if (!(a < 65504.0f)) return (float)(_Float16)v;
  float lo, ulp;
  if (a >= 0x1p-14f) {
    uint32_t b;
    std::memcpy(&b, &a, 4);
    const uint32_t lb = b & ~0x1FFFu, ub = (((b >> 23) & 0xFFu) - 10u) << 23;
    std::memcpy(&lo, &lb, 4);
    std::memcpy(&ulp, &ub, 4);
  } else {
    lo = std::trunc(a * 0x1p24f) * 0x1p-24f;
    ulp = 0x1p-24f;
  }
  const float frac = (a - lo) / ulp;
  const float u = (float)(r >> 8) * 0x1p-24f;
  return std::copysign(frac > u ? lo + ulp : lo, v);
}

template <class R> class Sim {
 public:
  Dims dm;
  uint32_t bcx, bcy, bcz, nb;
  static constexpr uint32_t kBrick = 8;
  std::vector<R> sc[2][4];  // [set][density, temperature, fuel, reaction]
  std::vector<R> vc[3], vs[3], vort[3], vort_mag, conf_mag, vel_mag;
  std::vector<uint32_t> flags[2];
  Level<R> lv[3];
  Level<R> xl[3];  // V-cycle levels 3..5
  SolverSettings sv;
  SolverStats stats;
  bool norms = false;  // compute SolverStats in the reference mode too
  std::vector<float> sources;  // packed, >= 32 floats (phantom emitter when empty)
  Quality q;
  int advect_mode = 1;         // 0 semi-lagrangian, 1 maccormack
  bool emit_dead_residual = false;
  // FP16 storage of the scalar sets (density, temperature, fuel, reaction): every
  // value a reference pass stores into one of those buffers is rounded to the
  // nearest binary16 (ties to even) and read back as R. Arithmetic stays in R.
  bool half_storage = false;
  // Sparse mode (extension; orc_set_sparse). The velocity passes run on a set of
  // bricks and are zero outside it, where the reference runs them on the whole
  // grid (createCombustionVolumeSimulation.ts:270-296):
  //  - velocity advection computes vScratch in the bricks flagged in the current
  //    set (the reference's flags, compute-active-bricks.wgsl.ts) and writes 0
  //    elsewhere;
  //  - after the flags of the next set, U = current flags | next flags; curl,
  //    |curl|, confinement, divergence, every fine Jacobi sweep and the fine
  //    prolongation compute as the reference inside U and write 0 outside it,
  //    and the projection writes the new velocity inside U and 0 outside it.
  // Scalar passes, injection, the mid and coarse pressure levels and the
  // restriction are the reference's. So velocity and the fine pressure are zero
  // outside U, and stencils at U's edge read those zeros.
  bool sparse = false;
  std::vector<uint8_t> uset;  // per brick: in U this step
  bool in_set(const std::vector<uint8_t>& m, uint32_t x, uint32_t y, uint32_t z) const {
    const uint32_t bx = std::min(x / kBrick, bcx - 1), by = std::min(y / kBrick, bcy - 1), bz = std::min(z / kBrick, bcz - 1);
    return m[bx + bcx * (by + bcy * bz)] != 0;
  }
  bool outside_u(uint32_t x, uint32_t y, uint32_t z) const { return sparse && !in_set(uset, x, y, z); }
  R qs(R v) const {
    if constexpr (is_tan<R>::value) return v;
    else return half_storage ? (R)(_Float16)v : v;
  }
  // Stochastic rounding of the binary16 stores (extension; orc_set_half_rounding):
  // a pass's store of voxel i rounds to one of the two neighbouring binary16
  // values, up with probability equal to the distance from the lower one in
  // units of their spacing. The draw is the voxel's and store site's hash plus
  // the step index times 2^32 / golden ratio (a rank-1 sequence in time): a value
  // that changes by less than half a binary16 spacing per step then moves by the
  // right amount on average over a few steps, where round-to-nearest would hold
  // it still every step.
  bool half_sr = false;
  R qs_at(R v, size_t i, uint32_t site) const {
    if constexpr (is_tan<R>::value) return v;
    else {
      if (!half_storage) return v;
      if (!half_sr) return (R)(_Float16)v;
      return (R)sr_half((float)v, sr_draw((uint32_t)i, site, (uint32_t)step_index));
    }
  }
  // Extension with no reference counterpart: a patch of per-voxel inflow
  // velocity. After inject-velocity, velocity.y at (x0 + i, y, z0 + k) is set to
  // inflow[i + nx * k] (the control of the differentiable rollout).
  uint32_t in_x0 = 0, in_y = 0, in_z0 = 0, in_nx = 0, in_nz = 0;
  std::vector<R> inflow;
  void apply_inflow() {
    for (uint32_t k = 0; k < in_nz; ++k)
      for (uint32_t i = 0; i < in_nx; ++i) vc[1][flat(dm, in_x0 + i, in_y, in_z0 + k)] = inflow[i + in_nx * k];
  }
  // runtime params (createCombustionVolumeSimulation.ts:194-204)
  double wind[3] = {0, 0, 0}, wind_strength = 0, gravity[3] = {0, -1, 0}, gravity_strength = 0.45;
  double buoyancy = 3.6, vorticity_strength = 2.15;
  double vmask[4] = {1.0, 0.4, 0.8, 0.35};
  double world_size = 10.0;
  // host state
  int cur = 0;
  long step_index = 0;
  bool initialized = false;
  double start_s = 0, last_elapsed_s = 0;
  int last_p = 0;  // 0 = 'a', 1 = 'b'
  bool debug_requested = false;
  Params P{};

  Sim(uint32_t w, uint32_t h, uint32_t d) {
    dm = make_dims(w, h, d);
    bcx = (w + kBrick - 1) / kBrick;
    bcy = (h + kBrick - 1) / kBrick;
    bcz = (d + kBrick - 1) / kBrick;
    nb = bcx * bcy * bcz;
    for (auto& s : sc)
      for (auto& f : s) f.assign(dm.n, R(0));
    for (int c = 0; c < 3; ++c) {
      vc[c].assign(dm.n, R(0));
      vs[c].assign(dm.n, R(0));
      vort[c].assign(dm.n, R(0));
    }
    vort_mag.assign(dm.n, R(0));
    conf_mag.assign(dm.n, R(0));
    vel_mag.assign(dm.n, R(0));
    flags[0].assign(nb, 0);
    flags[1].assign(nb, 0);
    lv[0].dm = dm;
    lv[1].dm = halve(dm);
    lv[2].dm = halve(lv[1].dm);
    for (auto& l : lv) {
      l.div.assign(l.dm.n, R(0));
      l.pa.assign(l.dm.n, R(0));
      l.pb.assign(l.dm.n, R(0));
    }
    xl[0].dm = halve(lv[2].dm);
    xl[1].dm = halve(xl[0].dm);
    xl[2].dm = halve(xl[1].dm);
    for (auto& l : xl) {
      l.div.assign(l.dm.n, R(0));
      l.pa.assign(l.dm.n, R(0));
      l.pb.assign(l.dm.n, R(0));
    }
    sources.assign(32, 0.0f);
    uset.assign(nb, 0);
  }

  // createCombustionVolumeSimulation.ts:206-226
  void reset() {
    for (auto& l : xl) {
      std::fill(l.div.begin(), l.div.end(), R(0));
      std::fill(l.pa.begin(), l.pa.end(), R(0));
      std::fill(l.pb.begin(), l.pb.end(), R(0));
    }
    stats = SolverStats{};
    cur = 0;
    step_index = 0;
    last_p = 0;
    initialized = false;
    start_s = last_elapsed_s;
    for (auto& s : sc)
      for (auto& f : s) std::fill(f.begin(), f.end(), R(0));
    for (int c = 0; c < 3; ++c) {
      std::fill(vc[c].begin(), vc[c].end(), R(0));
      std::fill(vs[c].begin(), vs[c].end(), R(0));
      std::fill(vort[c].begin(), vort[c].end(), R(0));
    }
    std::fill(vort_mag.begin(), vort_mag.end(), R(0));
    std::fill(conf_mag.begin(), conf_mag.end(), R(0));
    std::fill(vel_mag.begin(), vel_mag.end(), R(0));
    std::fill(flags[0].begin(), flags[0].end(), 0u);
    std::fill(flags[1].begin(), flags[1].end(), 0u);
    std::fill(uset.begin(), uset.end(), 0);
    for (auto& l : lv) std::fill(l.pa.begin(), l.pa.end(), R(0));
  }

  // ---------------------------------------------------------------- emitters
  // shaders/passes/inject-source-common.wgsl.ts
  struct Src {
    R px, py, pz, radius, start, duration, yd, yt, yf, speed, mode, falloff, tight, dirx, diry, dirz;
    R noise_scale, noise_mix, intensity, kind, seed;
  };
  static Src unpack(const float* s) {
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
  R active_gate(const Src& s) const {  // :24-27
    const R age = R(P.time) - s.start;
    return stepv(R(0), age) * stepv(age, s.duration);
  }
  R source_age(const Src& s) const { return mx(R(P.time) - s.start, R(0)); }  // :57-59
  static R source_duration(const Src& s) { return mx(s.duration, K(0.0001)); }  // :61-63
  static R sphere_falloff(R dist, R radius, R falloff) {  // :65-68
    const R t = clampv(R(1) - dist / mx(radius, K(0.0001)), R(0), R(1));
    return mixv(stepv(R(0), t - K(0.0001)), t * t, falloff);
  }
  R source_feather(R r) const {  // :70-73
    const R voxel_width = R(P.dx) / mx(R(P.world_size), K(0.0001));
    return mx(r * K(0.24), voxel_width * K(3.0));
  }
  R source_outer_limit(R r) const { return r + source_feather(r); }
  // hash31 (:102-104). The hash is a discrete pseudo-random function of integer
  // lattice points, not a physical quantity: both instantiations evaluate it in
  // f32 so that they produce the same noise pattern (an f64 evaluation of
  // fract(sin(.) * 43758.5) gives unrelated values, not more accurate ones).
  static R hash31(R x, R y, R z) {
    const float xf = (float)x, yf = (float)y, zf = (float)z;
    const float d = xf * 127.1f + yf * 311.7f + zf * 74.7f;
    return (R)fractv(pinned_sincos(d, 0) * 43758.5453123f);
  }
  static R value_noise3(R px, R py, R pz) {  // :106-117
    const R cx = flr(px), cy = flr(py), cz = flr(pz);
    const R fx = fractv(px), fy = fractv(py), fz = fractv(pz);
    const R ux = fx * fx * (R(3) - R(2) * fx);
    const R uy = fy * fy * (R(3) - R(2) * fy);
    const R uz = fz * fz * (R(3) - R(2) * fz);
    const R cx1 = cx + R(1), cy1 = cy + R(1), cz1 = cz + R(1);
    return mixv(mixv(mixv(hash31(cx, cy, cz), hash31(cx1, cy, cz), ux),
                     mixv(hash31(cx, cy1, cz), hash31(cx1, cy1, cz), ux), uy),
                mixv(mixv(hash31(cx, cy, cz1), hash31(cx1, cy, cz1), ux),
                     mixv(hash31(cx, cy1, cz1), hash31(cx1, cy1, cz1), ux), uy),
                uz);
  }
  static R emitter_noise(R px, R py, R pz, R scale, R seed) {  // :119-121
    const R s = mx(scale, K(0.1));
    return value_noise3(px * s + seed * K(0.137), py * s + seed * K(0.271), pz * s + (-seed) * K(0.193));
  }
  R eruptive_falloff(R px, R py, R pz, R dist, const Src& s, R falloff) const {  // :79-97
    const R target = s.radius;
    const R growth_seconds = clampv(target * K(5.5), K(0.1), K(0.75));
    const R age = source_age(s);
    const R growth = smoothstepv(R(0), R(1), clampv(age / growth_seconds, R(0), R(1)));
    const R feather = source_feather(target);
    const R seed = s.seed;
    const R coarse = emitter_noise(px + age * K(0.17), py + (-age) * K(0.11), pz + age * K(0.07), K(6.0), seed);
    const R fine = emitter_noise(px + (-age) * K(0.33), py + age * K(0.21), pz + (-age) * K(0.15), K(18.0), seed + K(41.0));
    const R lobe = clampv(coarse * K(0.72) + fine * K(0.28), R(0), R(1));
    const R reach = target * growth * mixv(K(0.62), R(1), smoothstepv(K(0.2), K(0.92), lobe));
    const R front = R(1) - smoothstepv(reach - feather, reach + feather, dist);
    const R core_radius = mx(target * (K(0.18) + growth * K(0.38)), feather);
    const R core = sphere_falloff(dist, core_radius, falloff) * (R(1) - growth * K(0.35));
    const R body = sphere_falloff(dist, mx(reach + feather, feather), falloff) * front;
    return clampv(mx(core, body) * mixv(K(0.72), K(1.2), lobe), R(0), R(1));
  }
  V3<R> turbulent_dir(R px, R py, R pz, R seed) const {  // inject-velocity.wgsl.ts:39-44
    const R nx = emitter_noise(px, py, pz, K(4.0), seed);
    const R ny = emitter_noise(px, py, pz, K(4.0), seed + K(17.3));
    const R nz = emitter_noise(px, py, pz, K(4.0), seed + K(31.7));
    const R vx = nx - K(0.5), vy = ny - K(0.5), vz = nz - K(0.5);
    const R l = length3(vx, vy, vz);
    return {vx / l, vy / l, vz / l};
  }
  size_t source_count() const { return sources.size() / 32; }

  template <class F> void for_voxels(const Dims& d, F f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (uint32_t z = 0; z < d.d; ++z)
      for (uint32_t y = 0; y < d.h; ++y)
        for (uint32_t x = 0; x < d.w; ++x) f(x, y, z);
  }

  V3<R> voxel_pos(uint32_t x, uint32_t y, uint32_t z) const {
    return {(R(x) + K(0.5)) / R(dm.w), (R(y) + K(0.5)) / R(dm.h), (R(z) + K(0.5)) / R(dm.d)};
  }

  // shaders/passes/inject-scalar.wgsl.ts:32-70
  void inject_scalar(int set) {
    auto& D = sc[set][0];
    auto& T = sc[set][1];
    auto& Fu = sc[set][2];
    const size_t ns = source_count();
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      const V3<R> p = voxel_pos(x, y, z);
      R dd = D[i], tt = T[i], ff = Fu[i];
      for (size_t e = 0; e < ns; ++e) {
        const Src s = unpack(&sources[e * 32]);
        const bool burst = s.kind == R(3);
        if (!(s.kind == R(0) || burst)) continue;
        if (active_gate(s) < K(0.0001)) continue;
        const R ox = p.x - s.px, oy = p.y - s.py, oz = p.z - s.pz;
        const R dist = length3(ox, oy, oz);
        const R radius = s.radius;
        if (dist > (burst ? source_outer_limit(radius) : radius)) continue;
        const R weight = burst ? eruptive_falloff(p.x, p.y, p.z, dist, s, K(0.5)) : sphere_falloff(dist, radius, K(0.5));
        const R noise = emitter_noise(p.x, p.y, p.z, s.noise_scale, s.seed);
        const R modulation = mixv(R(1), noise, clampv(s.noise_mix, R(0), R(1)));
        const R release = burst ? R(1) / source_duration(s) : R(1);
        const R contribution = weight * modulation * release * R(P.dt);
        dd = clamp01(dd + s.yd * contribution);
        tt = clamp01(tt + s.yt * contribution);
        ff = clamp01(ff + s.yf * contribution);
      }
      D[i] = qs_at(dd, i, 0);
      T[i] = qs_at(tt, i, 1);
      Fu[i] = qs_at(ff, i, 2);
    });
  }

  // shaders/passes/inject-velocity.wgsl.ts:46-96 (writes velocityCurrent)
  void inject_velocity() {
    const size_t ns = source_count();
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      const V3<R> p = voxel_pos(x, y, z);
      R vx = vc[0][i], vy = vc[1][i], vz = vc[2][i];
      for (size_t e = 0; e < ns; ++e) {
        const Src s = unpack(&sources[e * 32]);
        const bool burst = s.kind == R(3);
        if (!(s.kind == R(1) || burst)) continue;
        if (active_gate(s) < K(0.0001)) continue;
        const R ox = p.x - s.px, oy = p.y - s.py, oz = p.z - s.pz;
        const R dist = length3(ox, oy, oz);
        const R radius = s.radius;
        if (dist > (burst ? source_outer_limit(radius) : radius)) continue;
        const R weight = burst ? eruptive_falloff(p.x, p.y, p.z, dist, s, s.falloff) : sphere_falloff(dist, radius, s.falloff);
        const R speed = s.speed;
        const R mode = s.mode;
        V3<R> dir{R(0), R(0), R(0)};
        if (burst) {
          V3<R> radial{R(0), R(1), R(0)};
          if (dist > K(0.0001)) {
            const R m = mx(dist, K(0.0001));
            radial = {ox / m, oy / m, oz / m};
          }
          const R t = R(P.time);
          const V3<R> turb = turbulent_dir(p.x + t * K(0.19), p.y + (-t) * K(0.13), p.z + t * K(0.07), s.seed + K(83.0));
          const R bx = radial.x * speed + R(0) + turb.x * s.tight;
          const R by = radial.y * speed + s.mode + turb.y * s.tight;
          const R bz = radial.z * speed + R(0) + turb.z * s.tight;
          const R dur = source_duration(s);
          vx += bx * weight * R(P.dt) / dur;
          vy += by * weight * R(P.dt) / dur;
          vz += bz * weight * R(P.dt) / dur;
          continue;
        } else if (mode == R(0)) {
          dir = {R(0), R(1), R(0)};
          if (dist > K(0.0001)) {
            const R m = mx(dist, K(0.0001));
            dir = {ox / m, oy / m, oz / m};
          }
        } else if (mode == R(1)) {
          const R dx = s.dirx, dy = s.diry, dz = s.dirz;
          dir = {R(0), R(1), R(0)};
          if (dx * dx + dy * dy + dz * dz > K(0.0001)) {
            const R l = length3(dx, dy, dz);
            dir = {dx / l, dy / l, dz / l};
          }
        } else {
          dir = turbulent_dir(p.x, p.y, p.z, s.seed);
        }
        const R fx = dir.x * speed * weight * R(P.dt);
        const R fy = dir.y * speed * weight * R(P.dt);
        const R fz = dir.z * speed * weight * R(P.dt);
        const R tightness = clampv(s.tight, R(0), R(1)) * weight;
        vx = mixv(vx + fx, dir.x * speed, tightness);
        vy = mixv(vy + fy, dir.y * speed, tightness);
        vz = mixv(vz + fz, dir.z * speed, tightness);
      }
      const R lim = K(80.0) / mx(R(P.dx), K(0.001));
      vc[0][i] = clampv(vx, -lim, lim);
      vc[1][i] = clampv(vy, -lim, lim);
      vc[2][i] = clampv(vz, -lim, lim);
    });
  }

  // shaders/passes/inject-igniter.wgsl.ts:32-66
  void inject_igniter(int set) {
    auto& T = sc[set][1];
    auto& Fu = sc[set][2];
    auto& Re = sc[set][3];
    const size_t ns = source_count();
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      const V3<R> p = voxel_pos(x, y, z);
      R rr = Re[i], tt = T[i];
      for (size_t e = 0; e < ns; ++e) {
        const Src s = unpack(&sources[e * 32]);
        const bool burst = s.kind == R(3);
        if (!(s.kind == R(2) || burst)) continue;
        if (active_gate(s) < K(0.0001)) continue;
        const R dist = length3(p.x - s.px, p.y - s.py, p.z - s.pz);
        const R radius = s.radius;
        if (dist > (burst ? source_outer_limit(radius) : radius)) continue;
        const R weight = burst ? eruptive_falloff(p.x, p.y, p.z, dist, s, K(0.6)) : sphere_falloff(dist, radius, K(0.6));
        const R intensity = s.intensity;
        const R fuel_avail = burst ? R(1) : smoothstepv(K(0.02), K(0.22), Fu[i]);
        const R release = burst ? R(1) / source_duration(s) : K(1.6);
        const R seed = intensity * weight * fuel_avail * R(P.dt) * release;
        rr = clamp01(rr + seed);
        tt = clamp01(tt + intensity * weight * R(P.dt) * K(4.0));
      }
      Re[i] = qs_at(rr, i, 3);
      T[i] = qs_at(tt, i, 4);
    });
  }

  // ------------------------------------------------------------ brick flags
  // shaders/passes/compute-active-bricks.wgsl.ts:24-79 (flags cleared first,
  // createCombustionVolumeSimulation.ts:271,280)
  void active_bricks(int set) {
    std::vector<uint32_t>& fl = flags[set];
    std::fill(fl.begin(), fl.end(), 0u);
    const auto& D = sc[set][0];
    const auto& T = sc[set][1];
    const auto& Re = sc[set][3];
    const uint32_t bs = kBrick, stride = std::max<uint32_t>(bs / 4, 1);
    // Dilation stores are idempotent (always 1), so the parallel loop writes the
    // same result in any order.
#pragma omp parallel for collapse(2) schedule(static)
    for (uint32_t bz = 0; bz < bcz; ++bz)
      for (uint32_t by = 0; by < bcy; ++by)
        for (uint32_t bx = 0; bx < bcx; ++bx) {
          const uint32_t x0 = bx * bs, y0 = by * bs, z0 = bz * bs;
          bool active = false;
          R peak = R(0);
          for (uint32_t z = 0; z < bs; z += stride)
            for (uint32_t y = 0; y < bs; y += stride)
              for (uint32_t x = 0; x < bs; x += stride) {
                const uint32_t cx = x0 + x, cy = y0 + y, cz = z0 + z;
                if (cx < dm.w && cy < dm.h && cz < dm.d) {
                  const size_t i = flat(dm, cx, cy, cz);
                  const R e = D[i] + T[i] * K(0.7) + Re[i] * K(0.9);
                  peak = mx(peak, e);
                  if (e > K(0.012)) active = true;
                }
              }
          const uint32_t ccx = std::min(x0 + bs / 2, dm.w - 1), ccy = std::min(y0 + bs / 2, dm.h - 1),
                         ccz = std::min(z0 + bs / 2, dm.d - 1);
          const size_t ci = flat(dm, ccx, ccy, ccz);
          const R ce = D[ci] + T[ci] * K(0.7) + Re[ci] * K(0.9);
          peak = mx(peak, ce);
          if (ce > K(0.012)) active = true;
          if (!active) continue;
          const int rad = (peak > K(0.05) || ce > K(0.035)) ? 1 : 0;
          for (int dz = -rad; dz <= rad; ++dz)
            for (int dy = -rad; dy <= rad; ++dy)
              for (int dx = -rad; dx <= rad; ++dx) {
                const uint32_t nx = (uint32_t)std::clamp((int)bx + dx, 0, (int)bcx - 1);
                const uint32_t ny = (uint32_t)std::clamp((int)by + dy, 0, (int)bcy - 1);
                const uint32_t nz = (uint32_t)std::clamp((int)bz + dz, 0, (int)bcz - 1);
                fl[nx + bcx * (ny + bcy * nz)] = 1u;
              }
        }
  }

  bool is_active_coord(const std::vector<uint32_t>& fl, uint32_t x, uint32_t y, uint32_t z) const {
    // shaders/common/active-brick-mask.wgsl.ts:13-18
    const uint32_t bx = std::min(x / kBrick, bcx - 1), by = std::min(y / kBrick, bcy - 1), bz = std::min(z / kBrick, bcz - 1);
    return fl[bx + bcx * (by + bcy * bz)] != 0u;
  }

  // ---------------------------------------------------------- advection
  V3<R> sample_vel(const std::vector<R>* v, R px, R py, R pz) const {
    const Corners<R> c = corners(dm, px, py, pz);
    return {interp(v[0].data(), c), interp(v[1].data(), c), interp(v[2].data(), c)};
  }

  // shaders/passes/advect-velocity-semilagrangian.wgsl.ts:23-41 (vCurrent -> vScratch)
  void advect_velocity() {
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (is_boundary(dm, x, y, z) || (sparse && !is_active_coord(flags[cur], x, y, z))) {
        vs[0][i] = vs[1][i] = vs[2][i] = R(0);
        return;
      }
      const R cx = R(x) + K(0.5), cy = R(y) + K(0.5), cz = R(z) + K(0.5);
      const R dt = R(P.dt);
      const V3<R> v0 = sample_vel(vc, cx - K(0.5), cy - K(0.5), cz - K(0.5));
      const R bx = cx - v0.x * dt, by = cy - v0.y * dt, bz = cz - v0.z * dt;
      const V3<R> a = sample_vel(vc, bx - K(0.5), by - K(0.5), bz - K(0.5));
      const R damp = R(1) - dt * K(0.025);
      vs[0][i] = a.x * damp;
      vs[1][i] = a.y * damp;
      vs[2][i] = a.z * damp;
    });
  }

  R thermal_noise(R px, R py, R pz) const {  // advect-scalar-maccormack.wgsl.ts:52-57
    const R t = R(P.time);
    const R x = px + t * K(1.7), y = py + (-t) * K(3.1), z = pz + t * K(1.1);
    const R a = K(0.5) + K(0.5) * Mth<R>::sin(x * K(0.097) + y * K(0.061) + z * K(-0.083));
    const R b = K(0.5) + K(0.5) * Mth<R>::sin(x * K(-0.043) + y * K(0.137) + z * K(0.071) + Mth<R>::sin(y * K(0.079)) * K(1.6));
    return clampv(a * K(0.58) + b * K(0.42), R(0), R(1));
  }

  // The decay block shared by both scalar advection kernels
  // (advect-scalar-maccormack.wgsl.ts:80-100, advect-scalar-semilagrangian.wgsl.ts:83-103).
  void write_decayed(int dst, size_t i, uint32_t y, R density, R temperature, R fuel, R reaction, R noise) {
    const R dt = R(P.dt);
    const R ny = (R(y) + K(0.5)) / R(dm.h);
    const R hot = smoothstepv(K(0.22), K(0.78), temperature + fuel * K(0.2) + reaction * K(0.26));
    const R cooling_pocket = smoothstepv(K(0.44), K(0.9), R(1) - noise) * smoothstepv(K(0.08), K(0.74), density) *
                             (R(1) - hot * K(0.72));
    const R cooling = dt * (K(0.016) + ny * K(0.052)) * mixv(K(1.28), K(0.58), hot) * mixv(K(0.86), K(1.9), cooling_pocket);
    const R smoke_loss = dt * (K(0.008) + ny * K(0.026)) * mixv(K(0.75), K(1.38), noise);
    const R cold_breakup = dt * density * (R(1) - smoothstepv(K(0.2), K(0.86), hot)) * smoothstepv(K(0.18), K(0.72), density) *
                           smoothstepv(K(0.34), K(0.92), noise) * K(0.34);
    const R clearing = dt * density * hot * mixv(K(0.1), K(0.72), noise);
    sc[dst][0][i] = qs_at(clamp01(mx(R(0), density * (R(1) - smoke_loss) - clearing - cold_breakup)), i, 5);
    sc[dst][1][i] = qs_at(clamp01(mx(R(0), temperature - cooling)), i, 6);
    sc[dst][2][i] = qs_at(clamp01(mx(R(0), fuel - dt * mixv(K(0.012), K(0.034), noise))), i, 7);
    sc[dst][3][i] = qs_at(clamp01(mx(R(0), reaction - dt * mixv(K(0.46), K(0.82), noise))), i, 8);
  }

  // shaders/passes/advect-scalar-maccormack.wgsl.ts:33-101 (set src -> set dst,
  // masked by flags[src]; velocity = vScratch)
  void advect_scalars_maccormack(int src, int dst) {
    const std::vector<uint32_t>& fl = flags[src];
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (!is_active_coord(fl, x, y, z)) {
        for (int f = 0; f < 4; ++f) sc[dst][f][i] = R(0);
        return;
      }
      const R dt = R(P.dt);
      const R cx = R(x) + K(0.5), cy = R(y) + K(0.5), cz = R(z) + K(0.5);
      R out[4];
      for (int f = 0; f < 4; ++f) {
        const R* S = sc[src][f].data();
        const V3<R> v = sample_vel(vs, cx - K(0.5), cy - K(0.5), cz - K(0.5));
        const R bx = cx - v.x * dt, by = cy - v.y * dt, bz = cz - v.z * dt;
        const R spx = bx - K(0.5), spy = by - K(0.5), spz = bz - K(0.5);
        const R predicted = interp(S, corners(dm, spx, spy, spz));
        const V3<R> fv = sample_vel(vs, spx, spy, spz);
        const R rx = bx + fv.x * dt, ry = by + fv.y * dt, rz = bz + fv.z * dt;
        const R recovered = interp(S, corners(dm, rx - K(0.5), ry - K(0.5), rz - K(0.5)));
        const R original = interp(S, corners(dm, cx - K(0.5), cy - K(0.5), cz - K(0.5)));
        const R corrected = predicted + K(0.5) * (original - recovered);
        out[f] = clampv(corrected, mn(original, predicted), mx(original, predicted));
      }
      const R noise = thermal_noise(cx, cy, cz);
      write_decayed(dst, i, y, out[0], out[1], out[2], out[3], noise);
    });
  }

  // shaders/passes/advect-scalar-semilagrangian.wgsl.ts:26-44,76-104
  void advect_scalars_semilagrangian(int src, int dst) {
    const std::vector<uint32_t>& fl = flags[src];
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (!is_active_coord(fl, x, y, z)) {
        for (int f = 0; f < 4; ++f) sc[dst][f][i] = R(0);
        return;
      }
      const R dt = R(P.dt);
      const R cx = R(x) + K(0.5), cy = R(y) + K(0.5), cz = R(z) + K(0.5);
      const V3<R> v = sample_vel(vs, cx - K(0.5), cy - K(0.5), cz - K(0.5));
      const R bx = cx - v.x * dt, by = cy - v.y * dt, bz = cz - v.z * dt;
      const R spx = bx - K(0.5), spy = by - K(0.5), spz = bz - K(0.5);
      const Corners<R> c = corners(dm, spx, spy, spz);
      R out[4];
      for (int f = 0; f < 4; ++f) out[f] = interp(sc[src][f].data(), c);
      const R noise = thermal_noise(spx, spy, spz);
      write_decayed(dst, i, y, out[0], out[1], out[2], out[3], noise);
    });
  }

  // --------------------------------------------------------- combustion
  R thermal_cluster(R px, R py, R pz) const {  // combustion-update.wgsl.ts:27-34
    const R t = R(P.time);
    const R x = px + t * K(2.2), y = py + t * K(5.2), z = pz + (-t) * K(1.7);
    const R body = K(0.5) + K(0.5) * Mth<R>::sin(x * K(0.071) + y * K(0.093) + z * K(-0.064) + Mth<R>::sin(y * K(0.057)) * K(1.8));
    const R pocket = K(0.5) + K(0.5) * Mth<R>::sin(x * K(0.143) + y * K(-0.081) + z * K(0.119) +
                                                    Mth<R>::sin(x * K(0.11) + z * K(0.07)) * K(1.2));
    const R rising = K(0.5) + K(0.5) * Mth<R>::sin(x * K(0.18) + y * K(0.13) - z * K(0.16) + t * K(1.4));
    return clampv(body * K(0.46) + pocket * K(0.34) + rising * K(0.2), R(0), R(1));
  }

  // shaders/passes/combustion-update.wgsl.ts:42-93, masked by flags[set]. The
  // reference updates the set in place while neighbouring invocations read it;
  // WebGPU gives no order between invocations, so the result there depends on
  // scheduling. This restatement (and the CUDA kernels) read every neighbour
  // from the state before the pass.
  void combustion(int set) {
    const std::vector<uint32_t>& fl = flags[set];
    std::vector<R> D0 = sc[set][0], T0 = sc[set][1], F0 = sc[set][2], R0 = sc[set][3];
    auto hot = [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t j = flat(dm, x, y, z);
      return clampv(T0[j] * K(1.55) + F0[j] * K(0.26) + R0[j] * K(0.44), R(0), R(1));
    };
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      if (!is_active_coord(fl, x, y, z)) return;
      const size_t i = flat(dm, x, y, z);
      const R dt = R(P.dt);
      const R ny = (R(y) + K(0.5)) / R(dm.h);
      const R cluster = thermal_cluster(R(x), R(y), R(z));
      const R neighbor = (hot(inc(x, W1), y, z) + hot(dec(x), y, z) + hot(x, inc(y, H1), z) + hot(x, dec(y), z) +
                          hot(x, y, inc(z, D1)) + hot(x, y, dec(z))) *
                         K(0.16666667);
      const R local_before = hot(x, y, z);
      const R d = D0[i], t = T0[i], f = F0[i], r = R0[i];
      const R radiative = mx(neighbor - local_before * K(0.55), R(0)) * smoothstepv(K(0.04), K(0.76), d) *
                          (K(0.45) + (R(1) - cluster) * K(0.55)) * dt * K(2.6);
      const R hot_pocket = smoothstepv(K(0.58), K(0.92), cluster + r * K(0.22));
      const R cooling_pocket = smoothstepv(K(0.42), K(0.82), R(1) - cluster) * smoothstepv(K(0.08), K(0.68), d) *
                               (R(1) - smoothstepv(K(0.54), K(0.94), r));
      const R ignition = smoothstepv(K(0.1), K(0.55), t);
      const R burn = mn(f, f * ignition * dt * mixv(K(4.2), K(8.6), hot_pocket));
      const R hot_soot = smoothstepv(K(0.24), K(0.88), t + r * K(0.2)) * smoothstepv(K(0.36), K(0.9), R(1) - cluster + d * K(0.18));
      const R smoke_yield = burn * mixv(K(0.16), K(0.58), cooling_pocket + (R(1) - ignition) * K(0.5) + hot_soot * K(0.45));
      const R hot_cooling = mixv(K(1.3), K(0.62), hot_pocket);
      const R heat_loss = dt * (K(0.018) + ny * K(0.052)) * hot_cooling * mixv(R(1), K(2.25), cooling_pocket);
      const R density_loss = dt * d * (K(0.02) + ny * K(0.07));
      const R clearing = d * smoothstepv(K(0.18), K(0.82), t + r * K(0.22) + f * K(0.1)) * dt * mixv(K(0.55), K(2.45), hot_pocket);
      const R cooling_smoke = d * t * (cooling_pocket + hot_soot * K(0.32)) * dt * K(0.16);
      const R reaction_decay = r * (R(1) - dt * mixv(K(0.68), K(0.22), hot_pocket));
      sc[set][2][i] = qs_at(clamp01(f - burn), i, 9);
      sc[set][1][i] = qs_at(clamp01(t + burn * mixv(K(2.1), K(3.25), hot_pocket) + radiative - heat_loss), i, 10);
      sc[set][0][i] = qs_at(clamp01(mx(R(0), d + smoke_yield + cooling_smoke - density_loss - clearing * K(0.72))), i, 11);
      sc[set][3][i] = qs_at(clamp01(mx(reaction_decay, burn * mixv(K(4.0), K(7.5), hot_pocket) + radiative * K(1.8))), i, 12);
    });
  }

  // shaders/passes/apply-buoyancy.wgsl.ts:37-110, masked by flags[set]; updates vScratch
  void buoyancy_pass(int set) {
    const std::vector<uint32_t>& fl = flags[set];
    const auto& D = sc[set][0];
    const auto& T = sc[set][1];
    const auto& Re = sc[set][3];
    auto hot = [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t j = flat(dm, x, y, z);
      return clampv(T[j] * K(1.0) + Re[j] * K(0.85), R(0), R(1));
    };
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      if (!is_active_coord(fl, x, y, z)) return;
      const size_t i = flat(dm, x, y, z);
      const R dt = R(P.dt);
      const R b = R(P.buoyancy);
      const R response = b * (R(1) + smoothstepv(K(6.0), K(24.0), absr(b)) * K(0.38));
      const R hot_gas = hot(x, y, z);
      const R lift = hot_gas * response;
      const R d = D[i];
      const R gw = R(P.gravity[3]);
      const R gfx = R(P.gravity[0]) * d * gw, gfy = R(P.gravity[1]) * d * gw, gfz = R(P.gravity[2]) * d * gw;
      const R entrain = d * smoothstepv(K(0.04), K(0.3), hot_gas);
      const R ny = (R(y) + K(0.5)) / R(dm.h);
      const R t = R(P.time);
      const R shear = Mth<R>::sin(R(y) * K(0.073) + t * K(0.9)) * K(0.35) +
                      Mth<R>::sin(R(x) * K(0.041) - R(z) * K(0.052) + t * K(0.43)) * K(0.22);
      const R ww = R(P.wind[3]);
      const R wx = R(P.wind[0]), wy = R(P.wind[1]), wz = R(P.wind[2]);
      const R amount = ww * (K(0.18) + d * K(0.55) + ny * K(0.45));
      const R windx = wx * amount + (-wz) * amount * shear;
      const R windy = wy * amount + R(0) * amount * shear;
      const R windz = wz * amount + wx * amount * shear;
      const R tgx = (hot(inc(x, W1), y, z) - hot(dec(x), y, z)) * K(0.5);
      const R tgy = (hot(x, inc(y, H1), z) - hot(x, dec(y), z)) * K(0.5);
      const R tgz = (hot(x, y, inc(z, D1)) - hot(x, y, dec(z))) * K(0.5);
      const R dgx = (D[flat(dm, inc(x, W1), y, z)] - D[flat(dm, dec(x), y, z)]) * K(0.5);
      const R dgy = (D[flat(dm, x, inc(y, H1), z)] - D[flat(dm, x, dec(y), z)]) * K(0.5);
      const R dgz = (D[flat(dm, x, y, inc(z, D1))] - D[flat(dm, x, y, dec(z))]) * K(0.5);
      const R dgl = mx(length3(dgx, dgy, dgz), K(0.0001));
      const R cold = d * (R(1) - smoothstepv(K(0.12), K(0.72), hot_gas));
      const R breakup = smoothstepv(K(0.008), K(0.06), dgl) * cold;
      const R s1 = Mth<R>::sin(R(y) * K(0.117) + t * K(1.9));
      const R s2 = Mth<R>::sin(R(x) * K(0.071) - R(z) * K(0.083) + t * K(1.35)) * K(0.35);
      const R s3 = Mth<R>::cos(R(x) * K(0.061) + R(y) * K(0.049) - t * K(1.6));
      const R sl = length3(s1, s2, s3);
      const R shx = s1 / sl, shy = s2 / sl, shz = s3 / sl;
      const R collapse = d * (R(1) - smoothstepv(K(0.16), K(0.64), hot_gas));
      const R drag = d * smoothstepv(K(0.03), K(0.45), hot_gas);
      const R keep = R(1) - dt * K(0.08);
      R vx = vs[0][i] * keep, vy = vs[1][i] * keep, vz = vs[2][i] * keep;
      vx += windx * dt; vy += windy * dt; vz += windz * dt;
      vx += gfx * dt; vy += gfy * dt; vz += gfz * dt;
      const R tk = K(3.2) + absr(b) * K(0.08);
      vx += tgx * collapse * dt * tk; vy += tgy * collapse * dt * tk; vz += tgz * collapse * dt * tk;
      vx += (-dgx) / dgl * breakup * dt * K(2.8);
      vy += (-dgy) / dgl * breakup * dt * K(2.8);
      vz += (-dgz) / dgl * breakup * dt * K(2.8);
      const R sk = K(0.72) + breakup * K(2.4);
      vx += shx * cold * dt * sk; vy += shy * cold * dt * sk; vz += shz * cold * dt * sk;
      vx += wx * cold * ww * dt * K(0.9); vy += wy * cold * ww * dt * K(0.9); vz += wz * cold * ww * dt * K(0.9);
      vx += R(0) * dt; vy += drag * response * K(0.55) * dt; vz += R(0) * dt;
      const R lim = K(80.0) / mx(R(P.dx), K(0.001));
      vy = clampv(vy + (lift + entrain * response * K(0.24)) * dt, -lim, lim);
      if (x == 0 || x == W1 || z == 0 || z == D1) {
        vx = R(0);
        vz = R(0);
      }
      if (y == 0) vy = mx(vy, R(0));
      vs[0][i] = vx;
      vs[1][i] = vy;
      vs[2][i] = vz;
    });
  }

  // shaders/passes/compute-vorticity.wgsl.ts:23-50
  void vorticity_pass() {
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (is_boundary(dm, x, y, z) || outside_u(x, y, z)) {
        vort[0][i] = vort[1][i] = vort[2][i] = R(0);
        vort_mag[i] = R(0);
        return;
      }
      const size_t x0 = flat(dm, dec(x), y, z), x1 = flat(dm, inc(x, W1), y, z);
      const size_t y0 = flat(dm, x, dec(y), z), y1 = flat(dm, x, inc(y, H1), z);
      const size_t z0 = flat(dm, x, y, dec(z)), z1 = flat(dm, x, y, inc(z, D1));
      const R cx = ((vs[2][y1] - vs[2][y0]) - (vs[1][z1] - vs[1][z0])) * K(0.5);
      const R cy = ((vs[0][z1] - vs[0][z0]) - (vs[2][x1] - vs[2][x0])) * K(0.5);
      const R cz = ((vs[1][x1] - vs[1][x0]) - (vs[0][y1] - vs[0][y0])) * K(0.5);
      vort[0][i] = cx;
      vort[1][i] = cy;
      vort[2][i] = cz;
      vort_mag[i] = length3(cx, cy, cz);
    });
  }

  // shaders/passes/apply-vorticity-confinement.wgsl.ts:30-66 (scalars of set)
  void confinement_pass(int set) {
    const auto& D = sc[set][0];
    const auto& T = sc[set][1];
    const auto& Re = sc[set][3];
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (is_boundary(dm, x, y, z) || outside_u(x, y, z)) {  // vScratch is 0 outside U already
        conf_mag[i] = R(0);
        return;
      }
      const R gx = (vort_mag[flat(dm, inc(x, W1), y, z)] - vort_mag[flat(dm, dec(x), y, z)]) * K(0.5);
      const R gy = (vort_mag[flat(dm, x, inc(y, H1), z)] - vort_mag[flat(dm, x, dec(y), z)]) * K(0.5);
      const R gz = (vort_mag[flat(dm, x, y, inc(z, D1))] - vort_mag[flat(dm, x, y, dec(z))]) * K(0.5);
      const R gl = mx(length3(gx, gy, gz), K(0.0001));
      const R nx = gx / gl, ny = gy / gl, nz = gz / gl;
      const R hot_gas = clampv(T[i] + Re[i] * K(0.85), R(0), R(1));
      const R mask = clampv(R(P.vmask[0]) + smoothstepv(K(0.02), K(0.38), vort_mag[i]) * R(P.vmask[1]) +
                                smoothstepv(K(0.04), K(0.7), hot_gas) * R(P.vmask[2]) +
                                smoothstepv(K(0.04), K(0.65), D[i]) * R(P.vmask[3]),
                            R(0), R(4));
      const R wx = vort[0][i], wy = vort[1][i], wz = vort[2][i];
      const R k = R(P.vorticity_strength);
      const R fx = (ny * wz - nz * wy) * k * mask * K(1.45);
      const R fy = (nz * wx - nx * wz) * k * mask * K(1.45);
      const R fz = (nx * wy - ny * wx) * k * mask * K(1.45);
      const R dt = R(P.dt);
      const R lim = K(80.0) / mx(R(P.dx), K(0.001));
      vs[0][i] = clampv(vs[0][i] + fx * dt, -lim, lim);
      vs[1][i] = clampv(vs[1][i] + fy * dt, -lim, lim);
      vs[2][i] = clampv(vs[2][i] + fz * dt, -lim, lim);
      conf_mag[i] = length3(fx, fy, fz);
    });
  }

  // shaders/passes/compute-divergence.wgsl.ts:22-42 (vScratch -> fine.div)
  void divergence_pass() {
    auto& div = lv[0].div;
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (is_boundary(dm, x, y, z) || outside_u(x, y, z)) {
        div[i] = R(0);
        return;
      }
      const R ddx = vs[0][flat(dm, inc(x, W1), y, z)] - vs[0][flat(dm, dec(x), y, z)];
      const R ddy = vs[1][flat(dm, x, inc(y, H1), z)] - vs[1][flat(dm, x, dec(y), z)];
      const R ddz = vs[2][flat(dm, x, y, inc(z, D1))] - vs[2][flat(dm, x, y, dec(z))];
      div[i] = (ddx + ddy + ddz) * K(0.5);
    });
  }

  // shaders/passes/pressure-jacobi.wgsl.ts:15-36
  void jacobi(Level<R>& L, const std::vector<R>& src, std::vector<R>& dst) {
    const Dims& d = L.dm;
    const uint32_t W1 = d.w - 1, H1 = d.h - 1, D1 = d.d - 1;
    const bool fine = &L == &lv[0];
    for_voxels(d, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(d, x, y, z);
      if (is_boundary(d, x, y, z) || (fine && outside_u(x, y, z))) {
        dst[i] = R(0);
        return;
      }
      const R s = src[flat(d, inc(x, W1), y, z)] + src[flat(d, dec(x), y, z)] + src[flat(d, x, inc(y, H1), z)] +
                  src[flat(d, x, dec(y), z)] + src[flat(d, x, y, inc(z, D1))] + src[flat(d, x, y, dec(z))];
      dst[i] = (s - L.div[i]) / R(6);
    });
  }

  // shaders/passes/pressure-residual.wgsl.ts:16-38 (output never read; kept for the
  // dead-store test)
  void residual(Level<R>& L, const std::vector<R>& src, std::vector<R>& dst) {
    const Dims& d = L.dm;
    const uint32_t W1 = d.w - 1, H1 = d.h - 1, D1 = d.d - 1;
    for_voxels(d, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(d, x, y, z);
      if (is_boundary(d, x, y, z)) {
        dst[i] = R(0);
        return;
      }
      const R s = src[flat(d, inc(x, W1), y, z)] + src[flat(d, dec(x), y, z)] + src[flat(d, x, inc(y, H1), z)] +
                  src[flat(d, x, dec(y), z)] + src[flat(d, x, y, inc(z, D1))] + src[flat(d, x, y, dec(z))];
      const R lap = s - src[i] * R(6);
      dst[i] = L.div[i] - lap;
    });
  }

  // shaders/passes/pressure-restriction.wgsl.ts:27-50 (fine.div -> coarse.div)
  void restrict_div(const Level<R>& F, Level<R>& C) {
    const Dims& s = F.dm;
    const Dims& t = C.dm;
    for_voxels(t, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(t, x, y, z);
      if (x == 0 || y == 0 || z == 0 || x == t.w - 1 || y == t.h - 1 || z == t.d - 1) {
        C.div[i] = R(0);
        return;
      }
      R sum = R(0);
      for (uint32_t dz = 0; dz < 2; ++dz)
        for (uint32_t dy = 0; dy < 2; ++dy)
          for (uint32_t dx = 0; dx < 2; ++dx) {
            const uint32_t sx = std::min(2 * x + dx, s.w - 1), sy = std::min(2 * y + dy, s.h - 1), sz = std::min(2 * z + dz, s.d - 1);
            sum += F.div[flat(s, sx, sy, sz)];
          }
      C.div[i] = sum * K(0.125);
    });
  }

  // shaders/passes/pressure-prolongation.wgsl.ts:29-44 (fine.pressureA += coarse)
  void prolong(const Level<R>& C, const std::vector<R>& coarse_p, Level<R>& F) {
    const Dims& t = F.dm;
    const bool fine = &F == &lv[0];
    for_voxels(t, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(t, x, y, z);
      if (x == 0 || y == 0 || z == 0 || x == t.w - 1 || y == t.h - 1 || z == t.d - 1 || (fine && outside_u(x, y, z))) {
        F.pa[i] = R(0);
        return;
      }
      const R px = (R(x) + K(0.5)) * K(0.5) - K(0.5);
      const R py = (R(y) + K(0.5)) * K(0.5) - K(0.5);
      const R pz = (R(z) + K(0.5)) * K(0.5) - K(0.5);
      F.pa[i] += interp(coarse_p.data(), corners(C.dm, px, py, pz));
    });
  }

  // PressureSolvePass.ts:129-143
  int smooth(Level<R>& L, int iters, int start) {
    int active = start;
    for (int k = 0; k < iters; ++k) {
      if (active == 0) jacobi(L, L.pa, L.pb);
      else jacobi(L, L.pb, L.pa);
      active ^= 1;
    }
    return active;
  }
  std::vector<R>& pbuf(Level<R>& L, int id) { return id == 0 ? L.pa : L.pb; }

  // PressureSolvePass.ts:68-84
  int solve() {
    const int fine_pre = smooth(lv[0], q.fine_pre, 0);
    if (emit_dead_residual) residual(lv[0], pbuf(lv[0], fine_pre), pbuf(lv[0], fine_pre ^ 1));
    restrict_div(lv[0], lv[1]);
    const int mid_pre = smooth(lv[1], q.mid_pre, 0);
    if (emit_dead_residual) residual(lv[1], pbuf(lv[1], mid_pre), pbuf(lv[1], mid_pre ^ 1));
    restrict_div(lv[1], lv[2]);
    const int coarse = smooth(lv[2], q.coarse, 0);
    prolong(lv[2], pbuf(lv[2], coarse), lv[1]);
    const int mid = smooth(lv[1], q.mid_post, mid_pre);
    prolong(lv[1], pbuf(lv[1], mid), lv[0]);
    return smooth(lv[0], q.fine_post, fine_pre);
  }

  // ------------------------------------------------ V-cycle solver (extension)
  // Level k of the V-cycle: the reference's fine, mid and coarse levels, then
  // three more halvings. `div` holds the level's right-hand side, pa/pb its
  // iterate (the pressure on level 0, a correction below).
  Level<R>& vlev(int k) { return k < 3 ? lv[k] : xl[k - 3]; }

  // Weighted Jacobi: j = (sum of the 6 neighbours - rhs) / 6 in the reference's
  // order, dst = src + w (j - src) (dst = j when w is 1); boundary voxels 0.
  void wjacobi(Level<R>& L, const std::vector<R>& src, std::vector<R>& dst) {
    const Dims& d = L.dm;
    const uint32_t W1 = d.w - 1, H1 = d.h - 1, D1 = d.d - 1;
    const R w = R(sv.omega);
    const bool one = sv.omega == 1.0;
    for_voxels(d, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(d, x, y, z);
      if (is_boundary(d, x, y, z)) {
        dst[i] = R(0);
        return;
      }
      const R s = src[flat(d, inc(x, W1), y, z)] + src[flat(d, dec(x), y, z)] + src[flat(d, x, inc(y, H1), z)] +
                  src[flat(d, x, dec(y), z)] + src[flat(d, x, y, inc(z, D1))] + src[flat(d, x, y, dec(z))];
      const R j = (s - L.div[i]) / R(6);
      dst[i] = one ? j : src[i] + w * (j - src[i]);
    });
  }

  int wsmooth(Level<R>& L, int iters, int start) {
    int a = start;
    for (int k = 0; k < iters; ++k) {
      wjacobi(L, pbuf(L, a), pbuf(L, a ^ 1));
      a ^= 1;
    }
    return a;
  }

  // rhs - (sum of the 6 neighbours - 6 e) at an interior voxel, 0 on the boundary.
  R resid_at(const Level<R>& L, const std::vector<R>& e, uint32_t x, uint32_t y, uint32_t z) const {
    const Dims& d = L.dm;
    if (is_boundary(d, x, y, z)) return R(0);
    const uint32_t W1 = d.w - 1, H1 = d.h - 1, D1 = d.d - 1;
    const size_t i = flat(d, x, y, z);
    const R s = e[flat(d, inc(x, W1), y, z)] + e[flat(d, dec(x), y, z)] + e[flat(d, x, inc(y, H1), z)] + e[flat(d, x, dec(y), z)] +
                e[flat(d, x, y, inc(z, D1))] + e[flat(d, x, y, dec(z))];
    const R lap = s - e[i] * R(6);
    return L.div[i] - lap;
  }

  // Coarse right-hand side: 4 x the mean of the 8 fine residuals under a coarse
  // voxel (children clamped as in pressure-restriction.wgsl.ts:27-50); the 4
  // rescales the unscaled 7-point operator to the doubled spacing.
  void restrict_residual(const Level<R>& F, const std::vector<R>& e, Level<R>& C) {
    const Dims& s = F.dm;
    const Dims& t = C.dm;
    for_voxels(t, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(t, x, y, z);
      if (x == 0 || y == 0 || z == 0 || x == t.w - 1 || y == t.h - 1 || z == t.d - 1) {
        C.div[i] = R(0);
        return;
      }
      R sum = R(0);
      for (uint32_t dz = 0; dz < 2; ++dz)
        for (uint32_t dy = 0; dy < 2; ++dy)
          for (uint32_t dx = 0; dx < 2; ++dx)
            sum += resid_at(F, e, std::min(2 * x + dx, s.w - 1), std::min(2 * y + dy, s.h - 1), std::min(2 * z + dz, s.d - 1));
      C.div[i] = (sum * K(0.125)) * R(4);
    });
  }

  // dst = src + trilinear(coarse e) at interior fine voxels (the sample position
  // of pressure-prolongation.wgsl.ts:29-44); boundary voxels copy src.
  void prolong_add(const Level<R>& C, const std::vector<R>& ec, const Level<R>& F, const std::vector<R>& src, std::vector<R>& dst) {
    const Dims& t = F.dm;
    for_voxels(t, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(t, x, y, z);
      if (x == 0 || y == 0 || z == 0 || x == t.w - 1 || y == t.h - 1 || z == t.d - 1) {
        dst[i] = src[i];
        return;
      }
      const R px = (R(x) + K(0.5)) * K(0.5) - K(0.5);
      const R py = (R(y) + K(0.5)) * K(0.5) - K(0.5);
      const R pz = (R(z) + K(0.5)) * K(0.5) - K(0.5);
      dst[i] = src[i] + interp(ec.data(), corners(C.dm, px, py, pz));
    });
  }

  // One V-cycle on level k from buffer `start`; returns the buffer of the result.
  // When pre + post is odd the prolongation writes the other buffer, so the fine
  // level always ends in the buffer it started from.
  int vcycle(int k, int start) {
    Level<R>& L = vlev(k);
    if (k == sv.levels - 1) return wsmooth(L, sv.coarse, start);
    const int a = wsmooth(L, sv.pre, start);
    Level<R>& C = vlev(k + 1);
    restrict_residual(L, pbuf(L, a), C);
    std::fill(C.pa.begin(), C.pa.end(), R(0));
    const int ce = vcycle(k + 1, 0);
    const int b = ((sv.pre + sv.post) & 1) ? a ^ 1 : a;
    prolong_add(C, pbuf(C, ce), L, pbuf(L, a), pbuf(L, b));
    return wsmooth(L, sv.post, b);
  }

  // Squared FP64 norms: sum of div^2, and of the residual computed in double from
  // the stored values (neighbour sum in the reference's order).
  double rhs_norm2() const {
    double acc = 0;
    for (const R v : lv[0].div) acc += (double)v * (double)v;
    return acc;
  }
  double residual_norm2(const std::vector<R>& p) const {
    const Dims& d = lv[0].dm;
    const auto& div = lv[0].div;
    const uint32_t W1 = d.w - 1, H1 = d.h - 1, D1 = d.d - 1;
    double acc = 0;
#pragma omp parallel for collapse(2) reduction(+ : acc) schedule(static)
    for (uint32_t z = 1; z < d.d - 1; ++z)
      for (uint32_t y = 1; y < d.h - 1; ++y)
        for (uint32_t x = 1; x + 1 < d.w; ++x) {
          const size_t i = flat(d, x, y, z);
          const double s = (double)p[flat(d, inc(x, W1), y, z)] + (double)p[flat(d, dec(x), y, z)] + (double)p[flat(d, x, inc(y, H1), z)] +
                           (double)p[flat(d, x, dec(y), z)] + (double)p[flat(d, x, y, inc(z, D1))] + (double)p[flat(d, x, y, dec(z))];
          const double r = (double)div[i] - (s - 6.0 * (double)p[i]);
          acc += r * r;
        }
    return acc;
  }
  // max |0.5 (central differences of v)| over interior voxels, in FP64.
  double max_abs_divergence() const {
    double m = 0;
#pragma omp parallel for collapse(2) reduction(max : m) schedule(static)
    for (uint32_t z = 1; z < dm.d - 1; ++z)
      for (uint32_t y = 1; y < dm.h - 1; ++y)
        for (uint32_t x = 1; x + 1 < dm.w; ++x) {
          const double ddx = (double)vc[0][flat(dm, x + 1, y, z)] - (double)vc[0][flat(dm, x - 1, y, z)];
          const double ddy = (double)vc[1][flat(dm, x, y + 1, z)] - (double)vc[1][flat(dm, x, y - 1, z)];
          const double ddz = (double)vc[2][flat(dm, x, y, z + 1)] - (double)vc[2][flat(dm, x, y, z - 1)];
          m = std::max(m, std::fabs(0.5 * (ddx + ddy + ddz)));
        }
    return m;
  }

  bool vcycle_done() const { return std::sqrt(stats.res2) <= sv.tol * std::sqrt(stats.rhs2); }

  int solve_vcycle() {
    Level<R>& F = lv[0];
    int pid = last_p;
    if (!sv.warm) std::fill(pbuf(F, pid).begin(), pbuf(F, pid).end(), R(0));
    stats = SolverStats{};
    stats.rhs2 = rhs_norm2();
    stats.res2 = residual_norm2(pbuf(F, pid));
    while (!vcycle_done() && stats.cycles < sv.max_cycles) {
      pid = vcycle(0, pid);
      stats.cycles += 1;
      stats.res2 = residual_norm2(pbuf(F, pid));
    }
    stats.converged = vcycle_done() ? 1 : 0;
    return pid;
  }

  // shaders/passes/project-velocity.wgsl.ts:21-43 (vScratch, p -> vCurrent)
  void project(const std::vector<R>& p) {
    const uint32_t W1 = dm.w - 1, H1 = dm.h - 1, D1 = dm.d - 1;
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      if (is_boundary(dm, x, y, z) || outside_u(x, y, z)) {
        vc[0][i] = vc[1][i] = vc[2][i] = R(0);
        return;
      }
      const R gx = (p[flat(dm, inc(x, W1), y, z)] - p[flat(dm, dec(x), y, z)]) * K(0.5);
      const R gy = (p[flat(dm, x, inc(y, H1), z)] - p[flat(dm, x, dec(y), z)]) * K(0.5);
      const R gz = (p[flat(dm, x, y, inc(z, D1))] - p[flat(dm, x, y, dec(z))]) * K(0.5);
      vc[0][i] = vs[0][i] - gx;
      vc[1][i] = vs[1][i] - gy;
      vc[2][i] = vs[2][i] - gz;
    });
  }

  // shaders/passes/compute-debug-fields.wgsl.ts:18-25
  void debug_fields() {
    for_voxels(dm, [&](uint32_t x, uint32_t y, uint32_t z) {
      const size_t i = flat(dm, x, y, z);
      vel_mag[i] = length3(vc[0][i], vc[1][i], vc[2][i]);
    });
  }

  // The uniform of createCombustionVolumeSimulation.ts:237-266 (doubles rounded to f32).
  void prepare_params(double elapsed, double step_s) {
    const double effective = std::min(step_s, 1.0 / 15.0);
    const double local_time = elapsed - start_s;
    const double prev_local = last_elapsed_s - start_s;
    const double dx = world_size / (double)std::max(dm.w, dm.d);
    P.time = (float)local_time;
    P.dt = (float)effective;
    P.prev_time = (float)prev_local;
    P.scalar_set = (float)cur;
    for (int k = 0; k < 3; ++k) P.wind[k] = (float)wind[k];
    P.wind[3] = (float)wind_strength;
    for (int k = 0; k < 3; ++k) P.gravity[k] = (float)gravity[k];
    P.gravity[3] = (float)gravity_strength;
    P.buoyancy = (float)buoyancy;
    P.vorticity_strength = (float)vorticity_strength;
    P.dx = (float)dx;
    P.world_size = (float)world_size;
    for (int k = 0; k < 4; ++k) P.vmask[k] = (float)vmask[k];
  }

  // createCombustionVolumeSimulation.ts:230-305
  void step(double elapsed, double step_s) {
    if (!initialized) {
      initialized = true;
      start_s = elapsed;
      last_elapsed_s = elapsed;
    }
    prepare_params(elapsed, step_s);
    const int next = cur == 0 ? 1 : 0;
    inject_scalar(cur);
    inject_velocity();
    apply_inflow();
    inject_igniter(cur);
    active_bricks(cur);
    advect_velocity();
    if (advect_mode == 0) advect_scalars_semilagrangian(cur, next);
    else advect_scalars_maccormack(cur, next);
    active_bricks(next);
    if (sparse)
      for (uint32_t b = 0; b < nb; ++b) uset[b] = (flags[cur][b] | flags[next][b]) != 0u ? 1 : 0;
    combustion(next);
    buoyancy_pass(next);
    if (step_index % q.vorticity_interval == 0) {
      vorticity_pass();
      confinement_pass(next);
    }
    const bool solved = step_index % q.pressure_interval == 0;
    if (solved && sv.mode == 1) {
      divergence_pass();
      last_p = solve_vcycle();
    } else if (solved) {
      for (auto& l : lv) std::fill(l.pa.begin(), l.pa.end(), R(0));
      divergence_pass();
      last_p = solve();
      if (norms) {
        stats = SolverStats{};
        stats.rhs2 = rhs_norm2();
        stats.res2 = residual_norm2(pbuf(lv[0], last_p));
        stats.converged = vcycle_done() ? 1 : 0;
      }
    }
    project(pbuf(lv[0], last_p));
    if (solved && (sv.mode == 1 || norms)) stats.maxdiv = max_abs_divergence();
    if (dm.n < 1800000 || debug_requested) {
      debug_fields();
      debug_requested = false;
    }
    cur = next;
    last_elapsed_s = elapsed;
    step_index += 1;
  }

  // Field access by FX_FIELD_* id; *n receives the element count (0 on a bad id).
  R* field_ptr(int id, size_t* n) {
    const int prev = cur ^ 1;
    *n = dm.n;
    switch (id) {
      case F_DENSITY: case F_TEMPERATURE: case F_FUEL: case F_REACTION: return sc[cur][id - F_DENSITY].data();
      case F_PREV_DENSITY: case F_PREV_TEMPERATURE: case F_PREV_FUEL: case F_PREV_REACTION: return sc[prev][id - F_PREV_DENSITY].data();
      case F_VEL_X: case F_VEL_Y: case F_VEL_Z: return vc[id - F_VEL_X].data();
      case F_VSCR_X: case F_VSCR_Y: case F_VSCR_Z: return vs[id - F_VSCR_X].data();
      case F_VORT_X: case F_VORT_Y: case F_VORT_Z: return vort[id - F_VORT_X].data();
      case F_VORT_MAG: return vort_mag.data();
      case F_CONF_MAG: return conf_mag.data();
      case F_VEL_MAG: return vel_mag.data();
      case F_FINE_DIV: case F_FINE_PA: case F_FINE_PB:
      case F_MID_DIV: case F_MID_PA: case F_MID_PB:
      case F_COARSE_DIV: case F_COARSE_PA: case F_COARSE_PB: {
        const int l = (id - F_FINE_DIV) / 3, k = (id - F_FINE_DIV) % 3;
        *n = lv[l].dm.n;
        return k == 0 ? lv[l].div.data() : (k == 1 ? lv[l].pa.data() : lv[l].pb.data());
      }
      case F_PRESSURE: return pbuf(lv[0], last_p).data();
      default: *n = 0; return nullptr;
    }
  }
  uint32_t* flags_ptr(int id, size_t* n) {
    *n = nb;
    if (id == F_FLAGS) return flags[cur].data();
    if (id == F_PREV_FLAGS) return flags[cur ^ 1].data();
    *n = 0;
    return nullptr;
  }
};

struct Handle {
  int precision;
  void* sim;
};

template <class R> Sim<R>* as(Handle* h) { return static_cast<Sim<R>*>(h->sim); }

// precision 32 (f32), 64 (f64), 65 (f64 tangent numbers) or 66 (f32 values
// with FP64 tangents)
template <class F> auto dispatch(Handle* h, F f) {
  if (h->precision == 32) return f(as<float>(h));
  if (h->precision == 65) return f(as<Tan>(h));
  if (h->precision == 66) return f(as<Tan32>(h));
  return f(as<double>(h));
}

}  // namespace

extern "C" {

// Creates an oracle simulation (precision 32 or 64) of the given resolution with
// the reference defaults (createCombustionVolumeSimulation.ts:54,194-204).
// precisions 65 (FP64) and 66 (f32 values, the f32 trajectory) carry tangent
// numbers: every field has a directional derivative in FP64
// (orc_write_tangent seeds it, orc_read_tangent reads it).
void* orc_create(int precision, uint32_t w, uint32_t h, uint32_t d) {
  if ((precision != 32 && precision != 64 && precision != 65 && precision != 66) || w < 2 || h < 2 || d < 2) return nullptr;
  Handle* hd = new Handle;
  hd->precision = precision;
  if (precision == 32) hd->sim = new Sim<float>(w, h, d);
  else if (precision == 65) hd->sim = new Sim<Tan>(w, h, d);
  else if (precision == 66) hd->sim = new Sim<Tan32>(w, h, d);
  else hd->sim = new Sim<double>(w, h, d);
  return hd;
}

void orc_destroy(void* hv) {
  Handle* h = static_cast<Handle*>(hv);
  if (!h) return;
  if (h->precision == 32) delete as<float>(h);
  else if (h->precision == 65) delete as<Tan>(h);
  else if (h->precision == 66) delete as<Tan32>(h);
  else delete as<double>(h);
  delete h;
}

// values: wind[3], windStrength, gravity[3], gravityStrength, buoyancy,
// vorticityStrength, vorticityConstantMask, vorticityVelocityMask,
// vorticityHeatMask, vorticityDensityMask, worldSize (15 doubles).
void orc_set_runtime_params(void* hv, const double* v) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    for (int k = 0; k < 3; ++k) s->wind[k] = v[k];
    s->wind_strength = v[3];
    for (int k = 0; k < 3; ++k) s->gravity[k] = v[4 + k];
    s->gravity_strength = v[7];
    s->buoyancy = v[8];
    s->vorticity_strength = v[9];
    for (int k = 0; k < 4; ++k) s->vmask[k] = v[10 + k];
    s->world_size = v[14];
    return 0;
  });
}

// q: pressureInterval, vorticityInterval, finePre, finePost, midPre, midPost,
// coarse — already clamped by the caller.
void orc_set_quality(void* hv, const int* q) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    s->q.pressure_interval = q[0];
    s->q.vorticity_interval = q[1];
    s->q.fine_pre = q[2];
    s->q.fine_post = q[3];
    s->q.mid_pre = q[4];
    s->q.mid_post = q[5];
    s->q.coarse = q[6];
    return 0;
  });
}

void orc_set_advection_mode(void* hv, int mode) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) { s->advect_mode = mode; return 0; });
}

void orc_set_emit_dead_residual(void* hv, int on) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) { s->emit_dead_residual = on != 0; return 0; });
}

// packed: count * 32 floats (packEmitterSources layout). With count == 0 the
// injection kernels see one all-zero source, like the 128-byte minimum buffer
// of SourceInjectionPass.ts:13-23.
void orc_update_sources(void* hv, const float* packed, uint32_t count) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    if (count == 0) s->sources.assign(32, 0.0f);
    else s->sources.assign(packed, packed + (size_t)count * 32);
    return 0;
  });
}

// Sets the step uniform for (elapsed, step) without running a step.
void orc_prepare_params(void* hv, double elapsed, double step_s) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    if (!s->initialized) {
      s->initialized = true;
      s->start_s = elapsed;
      s->last_elapsed_s = elapsed;
    }
    s->prepare_params(elapsed, step_s);
    return 0;
  });
}

// Runs one pass on the current state (tests). Scalar sets are addressed by
// index 0/1, levels by 0 (fine), 1 (mid), 2 (coarse). Returns 0, or -1 for an
// unknown pass.
//   0 inject-scalar(set a)   1 inject-velocity          2 inject-igniter(set a)
//   3 active-bricks(set a)   4 advect-velocity          5 maccormack(a -> b)
//   6 semi-lagrangian(a -> b) 7 combustion(set a)       8 buoyancy(set a)
//   9 vorticity             10 confinement(set a)      11 divergence
//  12 jacobi(level a, p[b] -> p[1-b])                   13 restrict(level a -> a+1)
//  14 prolong(level a+1 p[b] -> level a pA)             15 project(fine p[a])
//  16 velocity magnitude    17 pressure solve (returns the final buffer id)
int orc_run_pass(void* hv, int pass, int a, int b) {
  return dispatch(static_cast<Handle*>(hv), [&](auto* s) -> int {
    switch (pass) {
      case 0: s->inject_scalar(a); return 0;
      case 1: s->inject_velocity(); return 0;
      case 2: s->inject_igniter(a); return 0;
      case 3: s->active_bricks(a); return 0;
      case 4: s->advect_velocity(); return 0;
      case 5: s->advect_scalars_maccormack(a, b); return 0;
      case 6: s->advect_scalars_semilagrangian(a, b); return 0;
      case 7: s->combustion(a); return 0;
      case 8: s->buoyancy_pass(a); return 0;
      case 9: s->vorticity_pass(); return 0;
      case 10: s->confinement_pass(a); return 0;
      case 11: s->divergence_pass(); return 0;
      case 12: s->jacobi(s->lv[a], s->pbuf(s->lv[a], b), s->pbuf(s->lv[a], b ^ 1)); return 0;
      case 13: s->restrict_div(s->lv[a], s->lv[a + 1]); return 0;
      case 14: s->prolong(s->lv[a + 1], s->pbuf(s->lv[a + 1], b), s->lv[a]); return 0;
      case 15: s->project(s->pbuf(s->lv[0], a)); return 0;
      case 16: s->debug_fields(); return 0;
      case 17: return s->solve();
      default: return -1;
    }
  });
}

void orc_step(void* hv, double elapsed, double step_s) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) { s->step(elapsed, step_s); return 0; });
}

void orc_reset(void* hv) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) { s->reset(); return 0; });
}

void orc_request_debug(void* hv) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) { s->debug_requested = true; return 0; });
}

// out: cur set, step index, last pressure buffer (0 a, 1 b), brick count.
void orc_get_state(void* hv, long* out) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    out[0] = s->cur;
    out[1] = s->step_index;
    out[2] = s->last_p;
    out[3] = s->nb;
    return 0;
  });
}

// Copies field `id` out as float64 (exact for both precisions). Returns the
// element count, 0 on a bad id, or -(needed) when `cap` is too small.
long orc_read_field(void* hv, int id, double* dst, long cap) {
  return dispatch(static_cast<Handle*>(hv), [&](auto* s) -> long {
    size_t n = 0;
    if (id == F_FLAGS || id == F_PREV_FLAGS) {
      uint32_t* p = s->flags_ptr(id, &n);
      if (!p) return 0;
      if ((long)n > cap) return -(long)n;
      for (size_t i = 0; i < n; ++i) dst[i] = (double)p[i];
      return (long)n;
    }
    auto* p = s->field_ptr(id, &n);
    if (!p) return 0;
    if ((long)n > cap) return -(long)n;
    for (size_t i = 0; i < n; ++i) dst[i] = (double)p[i];
    return (long)n;
  });
}

// Pressure solver: iv = mode, levels, pre, post, coarse, max_cycles, warm_start;
// dv = omega, tolerance. norms = 1 computes the FP64 statistics in mode 0 too.
void orc_set_solver(void* hv, const int* iv, const double* dv, int norms) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    s->sv.mode = iv[0];
    s->sv.levels = iv[1];
    s->sv.pre = iv[2];
    s->sv.post = iv[3];
    s->sv.coarse = iv[4];
    s->sv.max_cycles = iv[5];
    s->sv.warm = iv[6];
    s->sv.omega = dv[0];
    s->sv.tol = dv[1];
    s->norms = norms != 0;
    return 0;
  });
}

// out: rhs_l2, residual_l2, relative residual, max |div u|; iout: cycles, converged.
void orc_get_solver_stats(void* hv, double* out, int* iout) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    const double rhs = std::sqrt(s->stats.rhs2), res = std::sqrt(s->stats.res2);
    out[0] = rhs;
    out[1] = res;
    out[2] = rhs > 0 ? res / rhs : (res > 0 ? INFINITY : 0.0);
    out[3] = s->stats.maxdiv;
    iout[0] = s->stats.cycles;
    iout[1] = s->stats.converged;
    return 0;
  });
}

// Switches sparse mode (see Sim::sparse) on (1) or off (0); it takes effect at
// the next step. Returns -1 with the V-cycle solver, which has no sparse form.
int orc_set_sparse(void* hv, int on) {
  return dispatch(static_cast<Handle*>(hv), [&](auto* s) -> int {
    if (on && s->sv.mode == 1) return -1;
    s->sparse = on != 0;
    return 0;
  });
}

// The host clock of a simulation (createCombustionVolumeSimulation.ts:180-204):
// the elapsed time of its first step, of its latest step and the step index, so
// a fresh oracle can take a step in the middle of another simulation's run.
void orc_set_clock(void* hv, double start_s, double last_elapsed_s, long step_index) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    s->initialized = true;
    s->start_s = start_s;
    s->last_elapsed_s = last_elapsed_s;
    s->step_index = step_index;
    return 0;
  });
}

// sr_half(x[i], sr_draw(i, site, step)) for i < n (tests compare it with the CUDA one).
void orc_sr_half_array(const float* x, float* out, long n, uint32_t site, uint32_t step) {
  for (long i = 0; i < n; ++i) out[i] = sr_half(x[i], sr_draw((uint32_t)i, site, step));
}

// Rounding of the binary16 stores: 0 to nearest (ties to even), 1 stochastic
// (see Sim::qs_at).
void orc_set_half_rounding(void* hv, int mode) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    s->half_sr = mode == 1;
    return 0;
  });
}

// Switches FP16 storage of the scalar sets on (1) or off (0); set it before the
// first step or field write.
void orc_set_half_storage(void* hv, int on) {
  dispatch(static_cast<Handle*>(hv), [&](auto* s) {
    s->half_storage = on != 0;
    return 0;
  });
}

// Overwrites field `id` from float64 values (rounded to the oracle precision,
// and to binary16 for scalar fields under FP16 storage).
long orc_write_field(void* hv, int id, const double* src, long count) {
  return dispatch(static_cast<Handle*>(hv), [&](auto* s) -> long {
    size_t n = 0;
    using R = std::remove_reference_t<decltype(*s->field_ptr(0, &n))>;
    if (id == F_FLAGS || id == F_PREV_FLAGS) {
      uint32_t* p = s->flags_ptr(id, &n);
      if (!p || (long)n != count) return 0;
      for (size_t i = 0; i < n; ++i) p[i] = (uint32_t)src[i];
      return (long)n;
    }
    auto* p = s->field_ptr(id, &n);
    if (!p || (long)n != count) return 0;
    const bool scalar = id >= F_DENSITY && id <= F_PREV_REACTION;
    for (size_t i = 0; i < n; ++i) p[i] = scalar ? s->qs((R)src[i]) : (R)src[i];
    return (long)n;
  });
}

// The inflow patch (extension): nx * nz values (row x fastest) of velocity.y at
// (x0 .. x0+nx-1, y, z0 .. z0+nz-1), set after inject-velocity every step;
// nx * nz == 0 turns it off. `tangents` (nullable) seeds their derivatives in a
// precision-65 simulation. Returns 0, or -1 when the patch leaves the grid.
int orc_set_inflow(void* hv, uint32_t x0, uint32_t y, uint32_t z0, uint32_t nx, uint32_t nz, const double* values,
                   const double* tangents) {
  return dispatch(static_cast<Handle*>(hv), [&](auto* s) -> int {
    using R = typename std::remove_reference_t<decltype(s->inflow)>::value_type;
    if ((uint64_t)x0 + nx > s->dm.w || y >= s->dm.h || (uint64_t)z0 + nz > s->dm.d) return -1;
    s->in_x0 = x0;
    s->in_y = y;
    s->in_z0 = z0;
    s->in_nx = nx;
    s->in_nz = nz;
    s->inflow.assign((size_t)nx * nz, R(0));
    for (size_t k = 0; k < s->inflow.size(); ++k) {
      if constexpr (is_tan<R>::value) s->inflow[k] = R((typename std::remove_reference_t<decltype(s->inflow[k].v)>)values[k], tangents ? tangents[k] : 0.0, 0);
      else s->inflow[k] = (R)values[k];
    }
    return 0;
  });
}

// Tangent parts of a field in a precision-65 simulation: read into dst (returns
// the count, 0 for another precision or a bad id, -(needed) when cap is too
// small) or overwrite them from src (values stay).
long orc_read_tangent(void* hv, int id, double* dst, long cap) {
  Handle* h = static_cast<Handle*>(hv);
  if ((h->precision != 65 && h->precision != 66) || id == F_FLAGS || id == F_PREV_FLAGS) return 0;
  return dispatch(h, [&](auto* s) -> long {
    using R = typename std::remove_reference_t<decltype(s->inflow)>::value_type;
    if constexpr (is_tan<R>::value) {
      size_t n = 0;
      R* p = s->field_ptr(id, &n);
      if (!p) return 0;
      if ((long)n > cap) return -(long)n;
      for (size_t i = 0; i < n; ++i) dst[i] = p[i].d;
      return (long)n;
    } else {
      return 0;
    }
  });
}
long orc_write_tangent(void* hv, int id, const double* src, long count) {
  Handle* h = static_cast<Handle*>(hv);
  if ((h->precision != 65 && h->precision != 66) || id == F_FLAGS || id == F_PREV_FLAGS) return 0;
  return dispatch(h, [&](auto* s) -> long {
    using R = typename std::remove_reference_t<decltype(s->inflow)>::value_type;
    if constexpr (is_tan<R>::value) {
      size_t n = 0;
      R* p = s->field_ptr(id, &n);
      if (!p || (long)n != count) return 0;
      for (size_t i = 0; i < n; ++i) p[i].d = src[i];
      return (long)n;
    } else {
      return 0;
    }
  });
}

// The pinned f32 sine/cosine, exported so tests can compare the CUDA
// implementation and libm against it.
void orc_pinned_sin(const float* x, float* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = pinned_sincos(x[i], 0);
}
void orc_pinned_cos(const float* x, float* out, long n) {
  for (long i = 0; i < n; ++i) out[i] = pinned_sincos(x[i], 1);
}

int orc_num_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

void orc_set_num_threads(int n) {
#ifdef _OPENMP
  if (n > 0) omp_set_num_threads(n);
#else
  (void)n;
#endif
}

}  // extern "C"
