// Forward-mode dual numbers for the adjoint kernels.
//
// Dn<N> holds an f32 value and its derivatives with respect to N local inputs.
// Every operation computes the value with the same single f32 operation as the
// plain float code (the library is built without FMA contraction), so a
// per-voxel function evaluated on Dn takes exactly the branches the forward
// kernel took, and the derivatives are those of the branch taken: min, max and
// clamp select the derivative of the chosen operand, floor-like steps have
// derivative 0, and sqrt has derivative 0 at 0.
#pragma once

#include <type_traits>

#include "fx_math.cuh"

namespace fx {

template <int N>
struct Dn {
  float v;
  float g[N];
  FX_DEV Dn() {}
  FX_DEV Dn(float x) : v(x) {
#pragma unroll
    for (int k = 0; k < N; ++k) g[k] = 0.0f;
  }
  FX_DEV static Dn var(float x, int k) {
    Dn r(x);
    r.g[k] = 1.0f;
    return r;
  }
  FX_DEV Dn operator-() const {
    Dn r;
    r.v = -v;
#pragma unroll
    for (int k = 0; k < N; ++k) r.g[k] = -g[k];
    return r;
  }
};

template <class T>
struct is_dn : std::false_type {};
template <int N>
struct is_dn<Dn<N>> : std::true_type {};

// The dual type among the arguments (all duals in one call share N).
template <class... A>
struct dn_of;
template <class A>
struct dn_of<A> {
  using type = typename std::conditional<is_dn<A>::value, A, void>::type;
};
template <class A, class... B>
struct dn_of<A, B...> {
  using type = typename std::conditional<is_dn<A>::value, A, typename dn_of<B...>::type>::type;
};
template <class... A>
using dn_t = typename std::enable_if<!std::is_void<typename dn_of<A...>::type>::value, typename dn_of<A...>::type>::type;

template <int N>
FX_DEV Dn<N> operator+(const Dn<N>& a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a.v + b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a.g[k] + b.g[k];
  return r;
}
template <int N>
FX_DEV Dn<N> operator-(const Dn<N>& a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a.v - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a.g[k] - b.g[k];
  return r;
}
template <int N>
FX_DEV Dn<N> operator*(const Dn<N>& a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a.v * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a.g[k] * b.v + a.v * b.g[k];
  return r;
}
template <int N>
FX_DEV Dn<N> operator/(const Dn<N>& a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a.v / b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = (a.g[k] - r.v * b.g[k]) / b.v;
  return r;
}
template <int N>
FX_DEV Dn<N> operator+(const Dn<N>& a, float b) {
  Dn<N> r = a;
  r.v = a.v + b;
  return r;
}
template <int N>
FX_DEV Dn<N> operator+(float a, const Dn<N>& b) {
  Dn<N> r = b;
  r.v = a + b.v;
  return r;
}
template <int N>
FX_DEV Dn<N> operator-(const Dn<N>& a, float b) {
  Dn<N> r = a;
  r.v = a.v - b;
  return r;
}
template <int N>
FX_DEV Dn<N> operator-(float a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a - b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = -b.g[k];
  return r;
}
template <int N>
FX_DEV Dn<N> operator*(const Dn<N>& a, float b) {
  Dn<N> r;
  r.v = a.v * b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a.g[k] * b;
  return r;
}
template <int N>
FX_DEV Dn<N> operator*(float a, const Dn<N>& b) {
  Dn<N> r;
  r.v = a * b.v;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a * b.g[k];
  return r;
}
template <int N>
FX_DEV Dn<N> operator/(const Dn<N>& a, float b) {
  Dn<N> r;
  r.v = a.v / b;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = a.g[k] / b;
  return r;
}
template <int N>
FX_DEV Dn<N> operator/(float a, const Dn<N>& b) {
  return Dn<N>(a) / b;
}
template <int N, class B>
FX_DEV Dn<N>& operator+=(Dn<N>& a, const B& b) {
  a = a + b;
  return a;
}
template <int N, class B>
FX_DEV Dn<N>& operator-=(Dn<N>& a, const B& b) {
  a = a - b;
  return a;
}

FX_DEV float val(float x) { return x; }
template <int N>
FX_DEV float val(const Dn<N>& x) {
  return x.v;
}

template <class A, class B, class D = dn_t<A, B>>
FX_DEV bool operator<(const A& a, const B& b) {
  return val(a) < val(b);
}
template <class A, class B, class D = dn_t<A, B>>
FX_DEV bool operator>(const A& a, const B& b) {
  return val(a) > val(b);
}
template <class A, class B, class D = dn_t<A, B>>
FX_DEV bool operator>=(const A& a, const B& b) {
  return val(a) >= val(b);
}

// WGSL builtins on duals, with the same comparisons as the float versions.
template <class A, class B, class D = dn_t<A, B>>
FX_DEV D mn(const A& a, const B& b) {
  return val(b) < val(a) ? D(b) : D(a);
}
template <class A, class B, class D = dn_t<A, B>>
FX_DEV D mx(const A& a, const B& b) {
  return val(a) < val(b) ? D(b) : D(a);
}
template <class X, class L, class H, class D = dn_t<X, L, H>>
FX_DEV D clampv(const X& x, const L& lo, const H& hi) {
  return mn(mx(D(x), D(lo)), D(hi));
}
template <int N>
FX_DEV Dn<N> clamp01(const Dn<N>& x) {
  return clampv(x, 0.0f, 1.0f);
}
template <class A, class B, class C, class D = dn_t<A, B, C>>
FX_DEV D mixv(const A& a, const B& b, const C& t) {
  return D(a) * (1.0f - D(t)) + D(b) * D(t);
}
template <int N>
FX_DEV Dn<N> smoothstepv(float e0, float e1, const Dn<N>& x) {
  const Dn<N> t = clampv((x - e0) / (e1 - e0), 0.0f, 1.0f);
  return t * t * (3.0f - 2.0f * t);
}
template <int N>
FX_DEV Dn<N> length3(const Dn<N>& x, const Dn<N>& y, const Dn<N>& z) {
  const Dn<N> s = x * x + y * y + z * z;
  Dn<N> r;
  r.v = sqrtf(s.v);
  const float h = r.v > 0.0f ? 0.5f / r.v : 0.0f;
#pragma unroll
  for (int k = 0; k < N; ++k) r.g[k] = s.g[k] * h;
  return r;
}

}  // namespace fx
