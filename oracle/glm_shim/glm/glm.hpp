// Minimal GLSL-style vector/matrix header, written for this project so that the
// reference trainer's FP64 CPU twin (src/train/reference.cpp) and its two
// headers (src/render/camera.hpp, src/splat/gaussian_cloud.hpp) compile
// unmodified. glm itself is not installed and the reference does not vendor it
// (vcpkg.json lists it unpinned), so this header restates only the GLSL
// semantics those files use:
//   * vectors of 2-4 components with x/y/z/w and r/g/b/a names and operator[];
//   * column-major matrices with m[column][row]; matCxR has C columns of R rows;
//   * mat * vec, mat * mat, transpose, determinant (2x2), componentwise vector
//     arithmetic, dot, length, normalize, mix, sign, max.
// It is test infrastructure (the oracle), never part of the product.
#pragma once

#include <cmath>
#include <cstddef>
#include <type_traits>

namespace glm {

template <int N, class T> struct vec;

template <class T> struct vec<2, T> {
  union { T x, r; };
  union { T y, g; };
  constexpr vec() : x(0), y(0) {}
  constexpr explicit vec(T s) : x(s), y(s) {}
  constexpr vec(T a, T b) : x(a), y(b) {}
  template <class U> constexpr explicit vec(const vec<2, U> &o) : x(T(o.x)), y(T(o.y)) {}
  constexpr T &operator[](int i) { return i == 0 ? x : y; }
  constexpr const T &operator[](int i) const { return i == 0 ? x : y; }
};

template <class T> struct vec<3, T> {
  union { T x, r; };
  union { T y, g; };
  union { T z, b; };
  constexpr vec() : x(0), y(0), z(0) {}
  constexpr explicit vec(T s) : x(s), y(s), z(s) {}
  template <class A, class B, class C> constexpr vec(A a, B b, C c) : x(T(a)), y(T(b)), z(T(c)) {}
  template <class U> constexpr explicit vec(const vec<3, U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  template <class U> constexpr explicit vec(const vec<4, U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)) {}
  constexpr T &operator[](int i) { return i == 0 ? x : i == 1 ? y : z; }
  constexpr const T &operator[](int i) const { return i == 0 ? x : i == 1 ? y : z; }
};

template <class T> struct vec<4, T> {
  union { T x, r; };
  union { T y, g; };
  union { T z, b; };
  union { T w, a; };
  constexpr vec() : x(0), y(0), z(0), w(0) {}
  constexpr explicit vec(T s) : x(s), y(s), z(s), w(s) {}
  template <class A, class B, class C, class D> constexpr vec(A a, B b, C c, D d) : x(T(a)), y(T(b)), z(T(c)), w(T(d)) {}
  template <class U, class S> constexpr vec(const vec<3, U> &v, S s) : x(T(v.x)), y(T(v.y)), z(T(v.z)), w(T(s)) {}
  template <class U> constexpr explicit vec(const vec<4, U> &o) : x(T(o.x)), y(T(o.y)), z(T(o.z)), w(T(o.w)) {}
  constexpr T &operator[](int i) { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
  constexpr const T &operator[](int i) const { return i == 0 ? x : i == 1 ? y : i == 2 ? z : w; }
};

// Componentwise arithmetic.
#define GLM_SHIM_VEC_OP(op)                                                                  \
  template <int N, class T> constexpr vec<N, T> operator op(const vec<N, T> &a, const vec<N, T> &b) { \
    vec<N, T> out;                                                                           \
    for (int i = 0; i < N; ++i) out[i] = a[i] op b[i];                                       \
    return out;                                                                              \
  }                                                                                          \
  template <int N, class T> constexpr vec<N, T> operator op(const vec<N, T> &a, T s) {        \
    vec<N, T> out;                                                                           \
    for (int i = 0; i < N; ++i) out[i] = a[i] op s;                                          \
    return out;                                                                              \
  }                                                                                          \
  template <int N, class T> constexpr vec<N, T> operator op(T s, const vec<N, T> &a) {        \
    vec<N, T> out;                                                                           \
    for (int i = 0; i < N; ++i) out[i] = s op a[i];                                          \
    return out;                                                                              \
  }                                                                                          \
  template <int N, class T> constexpr vec<N, T> &operator op##=(vec<N, T> &a, const vec<N, T> &b) { \
    for (int i = 0; i < N; ++i) a[i] = a[i] op b[i];                                         \
    return a;                                                                                \
  }                                                                                          \
  template <int N, class T> constexpr vec<N, T> &operator op##=(vec<N, T> &a, T s) {          \
    for (int i = 0; i < N; ++i) a[i] = a[i] op s;                                            \
    return a;                                                                                \
  }
GLM_SHIM_VEC_OP(+)
GLM_SHIM_VEC_OP(-)
GLM_SHIM_VEC_OP(*)
GLM_SHIM_VEC_OP(/)
#undef GLM_SHIM_VEC_OP

template <int N, class T> constexpr vec<N, T> operator-(const vec<N, T> &a) {
  vec<N, T> out;
  for (int i = 0; i < N; ++i) out[i] = -a[i];
  return out;
}
template <int N, class T> constexpr bool operator==(const vec<N, T> &a, const vec<N, T> &b) {
  for (int i = 0; i < N; ++i)
    if (!(a[i] == b[i])) return false;
  return true;
}

template <int N, class T> constexpr T dot(const vec<N, T> &a, const vec<N, T> &b) {
  T s = a[0] * b[0];
  for (int i = 1; i < N; ++i) s += a[i] * b[i];
  return s;
}
template <int N, class T> T length(const vec<N, T> &a) { return std::sqrt(dot(a, a)); }
template <int N, class T> vec<N, T> normalize(const vec<N, T> &a) { return a / length(a); }
template <int N, class T> constexpr vec<N, T> mix(const vec<N, T> &x, const vec<N, T> &y, T t) {
  return x * (T(1) - t) + y * t;
}
template <int N, class T> constexpr vec<N, T> sign(const vec<N, T> &a) {
  vec<N, T> out;
  for (int i = 0; i < N; ++i) out[i] = a[i] > T(0) ? T(1) : (a[i] < T(0) ? T(-1) : T(0));
  return out;
}
template <int N, class T> constexpr vec<N, T> max(const vec<N, T> &a, const vec<N, T> &b) {
  vec<N, T> out;
  for (int i = 0; i < N; ++i) out[i] = a[i] < b[i] ? b[i] : a[i];
  return out;
}

// C columns of R rows, column-major.
template <int C, int R, class T> struct mat {
  vec<R, T> col[C];
  constexpr mat() {}
  // Diagonal matrix.
  constexpr explicit mat(T s) {
    for (int c = 0; c < C; ++c)
      for (int r = 0; r < R; ++r) col[c][r] = c == r ? s : T(0);
  }
  // Column vectors.
  template <class... V, class = decltype(sizeof...(V))>
  constexpr mat(const vec<R, T> &c0, const vec<R, T> &c1, const V &...rest) : col{c0, c1, rest...} {}
  // Scalars, column by column.
  template <class... S>
    requires(sizeof...(S) == C * R && (... && !std::is_class_v<S>))
  constexpr mat(S... s) {
    const T values[] = {T(s)...};
    for (int c = 0; c < C; ++c)
      for (int r = 0; r < R; ++r) col[c][r] = values[c * R + r];
  }
  // From another shape or type: the overlapping upper-left block, identity elsewhere.
  template <int C2, int R2, class U>
    requires(C2 != C || R2 != R || !std::is_same_v<U, T>)
  constexpr explicit mat(const mat<C2, R2, U> &o) {
    for (int c = 0; c < C; ++c)
      for (int r = 0; r < R; ++r) col[c][r] = (c < C2 && r < R2) ? T(o.col[c][r]) : (c == r ? T(1) : T(0));
  }
  constexpr vec<R, T> &operator[](int c) { return col[c]; }
  constexpr const vec<R, T> &operator[](int c) const { return col[c]; }
};

template <int C, int R, class T> constexpr vec<R, T> operator*(const mat<C, R, T> &m, const vec<C, T> &v) {
  vec<R, T> out;
  for (int r = 0; r < R; ++r) {
    T s = m[0][r] * v[0];
    for (int c = 1; c < C; ++c) s += m[c][r] * v[c];
    out[r] = s;
  }
  return out;
}
// (R x K) * (K x C2) with m[c][r] indexing.
template <int K, int R, int C2, class T> constexpr mat<C2, R, T> operator*(const mat<K, R, T> &a, const mat<C2, K, T> &b) {
  mat<C2, R, T> out;
  for (int c = 0; c < C2; ++c)
    for (int r = 0; r < R; ++r) {
      T s = a[0][r] * b[c][0];
      for (int k = 1; k < K; ++k) s += a[k][r] * b[c][k];
      out[c][r] = s;
    }
  return out;
}
template <int C, int R, class T> constexpr mat<C, R, T> operator*(T s, const mat<C, R, T> &m) {
  mat<C, R, T> out;
  for (int c = 0; c < C; ++c) out[c] = s * m[c];
  return out;
}
template <int C, int R, class T> constexpr mat<C, R, T> operator*(const mat<C, R, T> &m, T s) { return s * m; }
template <int C, int R, class T> constexpr mat<C, R, T> operator/(const mat<C, R, T> &m, T s) {
  mat<C, R, T> out;
  for (int c = 0; c < C; ++c) out[c] = m[c] / s;
  return out;
}
template <int C, int R, class T> constexpr mat<C, R, T> operator+(const mat<C, R, T> &a, const mat<C, R, T> &b) {
  mat<C, R, T> out;
  for (int c = 0; c < C; ++c) out[c] = a[c] + b[c];
  return out;
}
template <int C, int R, class T> constexpr mat<C, R, T> operator-(const mat<C, R, T> &a, const mat<C, R, T> &b) {
  mat<C, R, T> out;
  for (int c = 0; c < C; ++c) out[c] = a[c] - b[c];
  return out;
}
template <int C, int R, class T> constexpr mat<C, R, T> &operator+=(mat<C, R, T> &a, const mat<C, R, T> &b) {
  a = a + b;
  return a;
}
template <int C, int R, class T> constexpr mat<R, C, T> transpose(const mat<C, R, T> &m) {
  mat<R, C, T> out;
  for (int c = 0; c < C; ++c)
    for (int r = 0; r < R; ++r) out[r][c] = m[c][r];
  return out;
}
template <class T> constexpr T determinant(const mat<2, 2, T> &m) { return m[0][0] * m[1][1] - m[1][0] * m[0][1]; }

using vec2 = vec<2, float>;
using vec3 = vec<3, float>;
using vec4 = vec<4, float>;
using dvec2 = vec<2, double>;
using dvec3 = vec<3, double>;
using dvec4 = vec<4, double>;
using mat3 = mat<3, 3, float>;
using mat4 = mat<4, 4, float>;
using dmat2 = mat<2, 2, double>;
using dmat3 = mat<3, 3, double>;
using dmat4 = mat<4, 4, double>;
using dmat2x3 = mat<2, 3, double>;
using dmat3x2 = mat<3, 2, double>;

} // namespace glm
