// ORACLE — test infrastructure, not product code.
// Runtime for the C++ that oracle/wgsl2cpp.py translates from the reference's
// WGSL: WGSL scalar/vector types and built-ins with WGSL semantics, abstract
// float literals, and a dispatcher that runs workgroups (threads in lockstep
// at workgroupBarrier when a kernel uses one). Compile with -ffp-contract=off.
#pragma once
#include <barrier>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <type_traits>
#include <vector>

namespace wgsl {

// ---------------------------------------------------------------- abstract float literals
// A WGSL float literal is an AbstractFloat: evaluated exactly (double here) until
// it meets an f32, where it converts to the nearest f32.
struct AF {
  double v;
  constexpr explicit AF(double x) : v(x) {}
  operator float() const { return (float)v; }
};
inline AF operator-(AF a) { return AF(-a.v); }
inline AF operator+(AF a, AF b) { return AF(a.v + b.v); }
inline AF operator-(AF a, AF b) { return AF(a.v - b.v); }
inline AF operator*(AF a, AF b) { return AF(a.v * b.v); }
inline AF operator/(AF a, AF b) { return AF(a.v / b.v); }
inline float operator+(AF a, float b) { return (float)a.v + b; }
inline float operator-(AF a, float b) { return (float)a.v - b; }
inline float operator*(AF a, float b) { return (float)a.v * b; }
inline float operator/(AF a, float b) { return (float)a.v / b; }
inline float operator+(float a, AF b) { return a + (float)b.v; }
inline float operator-(float a, AF b) { return a - (float)b.v; }
inline float operator*(float a, AF b) { return a * (float)b.v; }
inline float operator/(float a, AF b) { return a / (float)b.v; }
inline bool operator<(float a, AF b) { return a < (float)b.v; }
inline bool operator>(float a, AF b) { return a > (float)b.v; }
inline bool operator<=(float a, AF b) { return a <= (float)b.v; }
inline bool operator>=(float a, AF b) { return a >= (float)b.v; }
inline bool operator<(AF a, float b) { return (float)a.v < b; }
inline bool operator>(AF a, float b) { return (float)a.v > b; }

inline float F(float x) { return x; }
inline float F(AF x) { return (float)x.v; }
inline float F(int32_t x) { return (float)x; }
inline float F(uint32_t x) { return (float)x; }

// let/var concretisation: AbstractFloat -> f32, everything else unchanged
inline float conc(AF a) { return (float)a.v; }
template <class T> inline T conc(T x) { return x; }

// ---------------------------------------------------------------- vectors
struct vec2f {
  float x, y;
  vec2f() = default;
  vec2f(const vec2f&) = default;
  template <class A> explicit vec2f(A a) : x(F(a)), y(F(a)) {}
  template <class A, class B> vec2f(A a, B b) : x(F(a)), y(F(b)) {}
};
struct vec3f {
  float x, y, z;
  vec3f() = default;
  vec3f(const vec3f&) = default;
  template <class A> explicit vec3f(A a) : x(F(a)), y(F(a)), z(F(a)) {}
  template <class A, class B, class C> vec3f(A a, B b, C c) : x(F(a)), y(F(b)), z(F(c)) {}
  float operator[](int32_t i) const { return i == 0 ? x : i == 1 ? y : z; }
};
struct vec4f {
  float x, y, z, w;
  vec4f() = default;
  vec4f(const vec4f&) = default;
  template <class A> explicit vec4f(A a) : x(F(a)), y(F(a)), z(F(a)), w(F(a)) {}
  template <class A, class B, class C, class D> vec4f(A a, B b, C c, D d) : x(F(a)), y(F(b)), z(F(c)), w(F(d)) {}
  template <class A> vec4f(vec3f v, A a) : x(v.x), y(v.y), z(v.z), w(F(a)) {}
  float operator[](uint32_t i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
  float operator[](int32_t i) const { return (*this)[(uint32_t)i]; }
};
struct vec2i {
  int32_t x, y;
  vec2i() = default;
  vec2i(int32_t a, int32_t b) : x(a), y(b) {}
  explicit vec2i(vec2f v);   // i32(f32) per component: truncating, saturating
};
struct vec3u { uint32_t x, y, z; };
struct bvec2 { bool x, y; };
struct bvec3 { bool x, y, z; };
struct bvec4 { bool x, y, z, w; };

inline vec2f operator+(vec2f a, vec2f b) { return {a.x + b.x, a.y + b.y}; }
inline vec2f operator-(vec2f a, vec2f b) { return {a.x - b.x, a.y - b.y}; }
inline vec2f operator*(vec2f a, vec2f b) { return {a.x * b.x, a.y * b.y}; }
inline vec2f operator/(vec2f a, vec2f b) { return {a.x / b.x, a.y / b.y}; }
template <class S> inline vec2f operator*(S s, vec2f a) { const float f = F(s); return {f * a.x, f * a.y}; }
template <class S> inline vec2f operator*(vec2f a, S s) { const float f = F(s); return {a.x * f, a.y * f}; }
template <class S> inline vec2f operator/(vec2f a, S s) { const float f = F(s); return {a.x / f, a.y / f}; }
template <class S> inline vec2f operator/(S s, vec2f a) { const float f = F(s); return {f / a.x, f / a.y}; }
inline vec2f operator-(vec2f a) { return {-a.x, -a.y}; }
inline vec4f operator+(vec4f a, vec4f b) { return {a.x + b.x, a.y + b.y, a.z + b.z, a.w + b.w}; }
inline vec4f operator-(vec4f a, vec4f b) { return {a.x - b.x, a.y - b.y, a.z - b.z, a.w - b.w}; }
inline vec4f operator*(vec4f a, vec4f b) { return {a.x * b.x, a.y * b.y, a.z * b.z, a.w * b.w}; }
template <class S> inline vec4f operator*(S s, vec4f a) { const float f = F(s); return {f * a.x, f * a.y, f * a.z, f * a.w}; }
template <class S> inline vec4f operator*(vec4f a, S s) { const float f = F(s); return {a.x * f, a.y * f, a.z * f, a.w * f}; }
template <class S> inline vec4f operator/(vec4f a, S s) { const float f = F(s); return {a.x / f, a.y / f, a.z / f, a.w / f}; }
inline vec4f& operator+=(vec4f& a, vec4f b) { a = a + b; return a; }
inline vec4f operator-(vec4f a) { return {-a.x, -a.y, -a.z, -a.w}; }
template <class S> inline vec2f operator-(S s, vec2f a) { const float f = F(s); return {f - a.x, f - a.y}; }
// vec3f (the renderer's colours)
inline vec3f operator+(vec3f a, vec3f b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline vec3f operator-(vec3f a, vec3f b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline vec3f operator*(vec3f a, vec3f b) { return {a.x * b.x, a.y * b.y, a.z * b.z}; }
inline vec3f operator/(vec3f a, vec3f b) { return {a.x / b.x, a.y / b.y, a.z / b.z}; }
template <class S> inline vec3f operator*(S s, vec3f a) { const float f = F(s); return {f * a.x, f * a.y, f * a.z}; }
template <class S> inline vec3f operator*(vec3f a, S s) { const float f = F(s); return {a.x * f, a.y * f, a.z * f}; }
template <class S> inline vec3f operator/(vec3f a, S s) { const float f = F(s); return {a.x / f, a.y / f, a.z / f}; }
template <class S> inline vec3f operator+(vec3f a, S s) { const float f = F(s); return {a.x + f, a.y + f, a.z + f}; }
template <class S> inline vec3f operator-(vec3f a, S s) { const float f = F(s); return {a.x - f, a.y - f, a.z - f}; }
template <class S> inline vec3f operator+(S s, vec3f a) { const float f = F(s); return {f + a.x, f + a.y, f + a.z}; }
inline vec3f operator-(vec3f a) { return {-a.x, -a.y, -a.z}; }
inline vec3f& operator+=(vec3f& a, vec3f b) { a = a + b; return a; }
inline bvec3 operator<=(vec3f a, vec3f b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z}; }
inline vec2f& operator+=(vec2f& a, vec2f b) { a = a + b; return a; }
inline bvec2 operator<(vec2f a, vec2f b) { return {a.x < b.x, a.y < b.y}; }
inline bvec4 operator>=(vec4f a, vec4f b) { return {a.x >= b.x, a.y >= b.y, a.z >= b.z, a.w >= b.w}; }
inline bvec4 operator<=(vec4f a, vec4f b) { return {a.x <= b.x, a.y <= b.y, a.z <= b.z, a.w <= b.w}; }
inline bool all(bvec4 b) { return b.x && b.y && b.z && b.w; }
inline bool all(bvec2 b) { return b.x && b.y; }

// ---------------------------------------------------------------- built-ins (WGSL semantics)
template <class A, class B> struct Common { using type = float; };
template <> struct Common<AF, AF> { using type = AF; };
template <> struct Common<int, int> { using type = int; };
template <> struct Common<uint32_t, uint32_t> { using type = uint32_t; };
template <class T> inline T as(float x) { return (T)x; }
template <class T> inline T cv(T x) { return x; }
inline float cv(AF x) { return (float)x.v; }

// min(e1, e2): e2 if e2 < e1, else e1; max likewise
inline float min(float a, float b) { return b < a ? b : a; }
inline float max(float a, float b) { return a < b ? b : a; }
inline int min(int a, int b) { return b < a ? b : a; }
inline int max(int a, int b) { return a < b ? b : a; }
inline float min(AF a, float b) { return min((float)a.v, b); }
inline float min(float a, AF b) { return min(a, (float)b.v); }
inline float max(AF a, float b) { return max((float)a.v, b); }
inline float max(float a, AF b) { return max(a, (float)b.v); }
inline vec2f min(vec2f a, vec2f b) { return {min(a.x, b.x), min(a.y, b.y)}; }
inline vec2f max(vec2f a, vec2f b) { return {max(a.x, b.x), max(a.y, b.y)}; }
inline vec4f min(vec4f a, vec4f b) { return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z), min(a.w, b.w)}; }
inline vec3f min(vec3f a, vec3f b) { return {min(a.x, b.x), min(a.y, b.y), min(a.z, b.z)}; }
inline vec3f max(vec3f a, vec3f b) { return {max(a.x, b.x), max(a.y, b.y), max(a.z, b.z)}; }
inline vec4f max(vec4f a, vec4f b) { return {max(a.x, b.x), max(a.y, b.y), max(a.z, b.z), max(a.w, b.w)}; }
template <class E, class L, class H> inline auto clamp(E e, L lo, H hi) { return min(max(e, lo), hi); }
inline float clamp(float e, AF lo, AF hi) { return min(max(e, (float)lo.v), (float)hi.v); }

// select(f, t, cond)
inline AF select(AF f, AF t, bool c) { return c ? t : f; }
inline float select(AF f, float t, bool c) { return c ? t : (float)f.v; }
inline float select(float f, AF t, bool c) { return c ? (float)t.v : f; }
inline float select(float f, float t, bool c) { return c ? t : f; }
inline int select(int f, int t, bool c) { return c ? t : f; }
inline uint32_t select(uint32_t f, uint32_t t, bool c) { return c ? t : f; }
inline vec2f select(vec2f f, vec2f t, bvec2 c) { return {c.x ? t.x : f.x, c.y ? t.y : f.y}; }
inline vec2f select(vec2f f, vec2f t, bool c) { return c ? t : f; }
inline vec3f select(vec3f f, vec3f t, bvec3 c) { return {c.x ? t.x : f.x, c.y ? t.y : f.y, c.z ? t.z : f.z}; }

inline float abs(float x) { return std::fabs(x); }
inline vec2f abs(vec2f v) { return {std::fabs(v.x), std::fabs(v.y)}; }
inline float floor(float x) { return std::floor(x); }
inline vec2f floor(vec2f v) { return {std::floor(v.x), std::floor(v.y)}; }
inline float ceil(float x) { return std::ceil(x); }
inline float fract(float x) { return x - std::floor(x); }
inline float exp(float x) { return std::exp(x); }
inline float log(float x) { return std::log(x); }
inline float pow(float a, float b) { return std::pow(a, b); }
inline float pow(float a, AF b) { return std::pow(a, (float)b.v); }
inline float cos(float x) { return std::cos(x); }
inline float sin(float x) { return std::sin(x); }
inline float atan2(float y, float x) { return std::atan2(y, x); }
inline float sqrt(float x) { return std::sqrt(x); }
inline float length(vec2f v) { return std::sqrt(v.x * v.x + v.y * v.y); }
inline vec2f fract(vec2f v) { return {fract(v.x), fract(v.y)}; }
inline vec3f exp(vec3f v) { return {exp(v.x), exp(v.y), exp(v.z)}; }
inline vec4f exp(vec4f v) { return {exp(v.x), exp(v.y), exp(v.z), exp(v.w)}; }
inline vec3f pow(vec3f a, vec3f b) { return {pow(a.x, b.x), pow(a.y, b.y), pow(a.z, b.z)}; }
inline float dot(vec2f a, vec2f b) { return a.x * b.x + a.y * b.y; }
inline float dot(vec3f a, vec3f b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
// smoothstep(low, high, x) = t * t * (3 - 2 t), t = clamp((x - low) / (high - low), 0, 1)
inline float smoothstep(float lo, float hi, float x) {
  const float t = min(max((x - lo) / (hi - lo), 0.f), 1.f);
  return t * t * (3.f - 2.f * t);
}
inline float round(float x) { return std::nearbyint(x); }
// mix(a, b, t) = a * (1 - t) + b * t
inline float mix(float a, float b, float t) { return a * (1.f - t) + b * t; }
inline vec4f mix(vec4f a, vec4f b, float t) { return {mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t), mix(a.w, b.w, t)}; }
inline vec3f mix(vec3f a, vec3f b, float t) { return {mix(a.x, b.x, t), mix(a.y, b.y, t), mix(a.z, b.z, t)}; }

// conversions: f32 -> i32/u32 truncate toward zero and saturate
inline int32_t conv_i32(float v) {
  if (!(v == v)) return 0;
  if (v >= 2147483647.f) return INT32_MAX;
  if (v <= -2147483648.f) return INT32_MIN;
  return (int32_t)v;
}
inline int32_t conv_i32(int32_t v) { return v; }
inline int32_t conv_i32(uint32_t v) { return (int32_t)v; }
inline uint32_t conv_u32(float v) {
  if (!(v == v) || v <= 0.f) return 0u;
  if (v >= 4294967295.f) return 0xffffffffu;
  return (uint32_t)v;
}
inline uint32_t conv_u32(int32_t v) { return (uint32_t)v; }
inline uint32_t conv_u32(uint32_t v) { return v; }
inline float conv_f32(float v) { return v; }
inline float conv_f32(int32_t v) { return (float)v; }
inline float conv_f32(uint32_t v) { return (float)v; }
inline float conv_f32(AF v) { return (float)v.v; }
inline vec2i::vec2i(vec2f v) : x(conv_i32(v.x)), y(conv_i32(v.y)) {}
template <class T, class V> inline T conv(V v) { return (T)cv(v); }
inline uint32_t bitcast_uint32_t(float f) { uint32_t u; std::memcpy(&u, &f, 4); return u; }
inline float bitcast_float(uint32_t u) { float f; std::memcpy(&f, &u, 4); return f; }

inline int32_t atomicAdd(int32_t* p, int32_t v) { return __atomic_fetch_add(p, v, __ATOMIC_RELAXED); }
inline int32_t atomicMax(int32_t* p, int32_t v) {
  int32_t cur = __atomic_load_n(p, __ATOMIC_RELAXED);
  while (cur < v && !__atomic_compare_exchange_n(p, &cur, v, false, __ATOMIC_RELAXED, __ATOMIC_RELAXED)) {}
  return cur;
}

// ---------------------------------------------------------------- dispatch
inline thread_local std::barrier<>* tl_barrier = nullptr;
inline void workgroupBarrier() { tl_barrier->arrive_and_wait(); }

// Runs a dispatch of (wx, wy, wz) workgroups of size (sx, sy, sz). Kernels without
// barriers run their invocations in order on this thread; kernels with barriers
// run each workgroup's invocations as threads meeting at workgroupBarrier.
template <class Fn>
void dispatch(uint32_t sx, uint32_t sy, uint32_t sz, uint32_t wx, uint32_t wy, uint32_t wz, bool barrier, Fn f) {
  const uint32_t n = sx * sy * sz;
  for (uint32_t gz = 0; gz < wz; gz++)
    for (uint32_t gy = 0; gy < wy; gy++)
      for (uint32_t gx = 0; gx < wx; gx++) {
        const vec3u wg{gx, gy, gz};
        auto inv = [&](uint32_t lx, uint32_t ly, uint32_t lz) {
          const vec3u lid{lx, ly, lz};
          const vec3u gid{gx * sx + lx, gy * sy + ly, gz * sz + lz};
          f(gid, wg, lid, lx + sx * (ly + sy * lz));
        };
        if (!barrier) {
          for (uint32_t lz = 0; lz < sz; lz++)
            for (uint32_t ly = 0; ly < sy; ly++)
              for (uint32_t lx = 0; lx < sx; lx++) inv(lx, ly, lz);
        } else {
          std::barrier<> bar((std::ptrdiff_t)n);
          std::vector<std::thread> th;
          th.reserve(n);
          for (uint32_t lz = 0; lz < sz; lz++)
            for (uint32_t ly = 0; ly < sy; ly++)
              for (uint32_t lx = 0; lx < sx; lx++)
                th.emplace_back([&, lx, ly, lz] { tl_barrier = &bar; inv(lx, ly, lz); });
          for (auto& t : th) t.join();
        }
      }
}

}  // namespace wgsl
