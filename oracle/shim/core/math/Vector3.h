// Project-written stand-in for waLBerla's Vector3: a three-component value type, enough
// for the conversion helpers in the reference's PointND header. Test infrastructure only.
#pragma once
namespace walberla { namespace math {
template <typename T> struct Vector3 {
  T v[3];
  Vector3() : v{T(0), T(0), T(0)} {}
  Vector3(T a, T b, T c) : v{a, b, c} {}
  T& operator[](int i) { return v[i]; }
  const T& operator[](int i) const { return v[i]; }
};
}}  // namespace walberla::math
