/* Minimal fixed-size vector standing in for Peano's tarch::la::Vector
 * (the reference snapshot does not ship Peano's tarch). */
#pragma once
namespace tarch { namespace la {
template <int Size, typename Scalar> class Vector {
  Scalar _v[Size];
 public:
  Vector() {}
  Vector(const Scalar& s) { for (int i = 0; i < Size; i++) _v[i] = s; }
  Vector(const Scalar& a, const Scalar& b) { _v[0] = a; if (Size > 1) _v[1] = b; }
  Vector(const Scalar& a, const Scalar& b, const Scalar& c) { _v[0] = a; if (Size > 1) _v[1] = b; if (Size > 2) _v[2] = c; }
  Scalar& operator[](int i) { return _v[i]; }
  const Scalar& operator[](int i) const { return _v[i]; }
  Scalar& operator()(int i) { return _v[i]; }
  const Scalar& operator()(int i) const { return _v[i]; }
  Scalar* data() { return _v; }
  const Scalar* data() const { return _v; }
  int size() const { return Size; }
};
template <int Size, typename Scalar>
Vector<Size, Scalar> operator-(const Vector<Size, Scalar>& a, const Vector<Size, Scalar>& b) {
  Vector<Size, Scalar> r; for (int i = 0; i < Size; i++) r[i] = a[i] - b[i]; return r;
}
template <int Size, typename Scalar>
Vector<Size, Scalar> operator+(const Vector<Size, Scalar>& a, const Vector<Size, Scalar>& b) {
  Vector<Size, Scalar> r; for (int i = 0; i < Size; i++) r[i] = a[i] + b[i]; return r;
}
template <int Size, typename Scalar>
Vector<Size, Scalar> operator/(const Vector<Size, Scalar>& a, const Scalar& s) {
  Vector<Size, Scalar> r; for (int i = 0; i < Size; i++) r[i] = a[i] / s; return r;
}
template <int Size, typename Scalar>
Vector<Size, Scalar> operator*(const Vector<Size, Scalar>& a, const Scalar& s) {
  Vector<Size, Scalar> r; for (int i = 0; i < Size; i++) r[i] = a[i] * s; return r;
}
template <int Size, typename Scalar>
Vector<Size, Scalar> operator*(const Scalar& s, const Vector<Size, Scalar>& a) { return a * s; }
template <int Size, typename Scalar> Scalar volume(const Vector<Size, Scalar>& v) {
  Scalar r = 1; for (int i = 0; i < Size; i++) r *= v[i]; return r;
}
}}
