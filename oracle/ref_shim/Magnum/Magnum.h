/* Minimal stand-in for the Magnum math types used by the reference's engine
 * headers (the Magnum submodule is absent from the reference checkout).
 * Semantics follow Magnum's: component-wise IEEE arithmetic in the vector's
 * own element type (a scalar operand is converted to that type first),
 * dot(a,b) = a0*b0 + a1*b1 + a2*b2 evaluated left to right. */
#pragma once
#include <cmath>
#include <cstddef>
#include <algorithm>
namespace Magnum {
namespace Math {
template <std::size_t N, class T> struct Vector {
    T _d[N];
    Vector() : _d{} {}
    T &operator[](std::size_t i) { return _d[i]; }
    const T &operator[](std::size_t i) const { return _d[i]; }
    T *data() { return _d; }
    const T *data() const { return _d; }
};
#define MXSHIM_VEC_OPS(NAME, N)                                                                     \
    NAME operator+(const NAME &o) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] + o._d[i]; return r; } \
    NAME operator-(const NAME &o) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] - o._d[i]; return r; } \
    NAME operator*(const NAME &o) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] * o._d[i]; return r; } \
    NAME operator/(const NAME &o) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] / o._d[i]; return r; } \
    NAME operator-() const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = -this->_d[i]; return r; }  \
    NAME operator*(T s) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] * s; return r; } \
    NAME operator/(T s) const { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = this->_d[i] / s; return r; } \
    NAME &operator+=(const NAME &o) { for (std::size_t i = 0; i < N; ++i) this->_d[i] += o._d[i]; return *this; } \
    NAME &operator-=(const NAME &o) { for (std::size_t i = 0; i < N; ++i) this->_d[i] -= o._d[i]; return *this; } \
    NAME &operator*=(T s) { for (std::size_t i = 0; i < N; ++i) this->_d[i] *= s; return *this; }            \
    NAME &operator/=(T s) { for (std::size_t i = 0; i < N; ++i) this->_d[i] /= s; return *this; }            \
    friend NAME operator*(T s, const NAME &v) { NAME r; for (std::size_t i = 0; i < N; ++i) r._d[i] = s * v._d[i]; return r; } \
    T sum() const { T s = this->_d[0]; for (std::size_t i = 1; i < N; ++i) s += this->_d[i]; return s; }      \
    T dot() const { return ((*this) * (*this)).sum(); }                                                       \
    T length() const { return std::sqrt(dot()); }                                                            \
    NAME normalized() const { return (*this) / length(); }                                                    \
    bool operator==(const NAME &o) const { for (std::size_t i = 0; i < N; ++i) if (this->_d[i] != o._d[i]) return false; return true; } \
    bool operator!=(const NAME &o) const { return !(*this == o); }

template <class T> struct Vector2 : Vector<2, T> {
    Vector2() {}
    Vector2(T a, T b) { this->_d[0] = a; this->_d[1] = b; }
    explicit Vector2(T a) { this->_d[0] = this->_d[1] = a; }
    MXSHIM_VEC_OPS(Vector2, 2)
};
template <class T> struct Vector3 : Vector<3, T> {
    Vector3() {}
    Vector3(T a, T b, T c) { this->_d[0] = a; this->_d[1] = b; this->_d[2] = c; }
    explicit Vector3(T a) { this->_d[0] = this->_d[1] = this->_d[2] = a; }
    template <class U> explicit Vector3(const Vector3<U> &o) { for (int i = 0; i < 3; ++i) this->_d[i] = T(o[i]); }
    T &x() { return this->_d[0]; }
    T &y() { return this->_d[1]; }
    T &z() { return this->_d[2]; }
    T x() const { return this->_d[0]; }
    T y() const { return this->_d[1]; }
    T z() const { return this->_d[2]; }
    static Vector3 xAxis(T v = T(1)) { return {v, T(0), T(0)}; }
    static Vector3 yAxis(T v = T(1)) { return {T(0), v, T(0)}; }
    static Vector3 zAxis(T v = T(1)) { return {T(0), T(0), v}; }
    MXSHIM_VEC_OPS(Vector3, 3)
};
template <class T> struct Vector4 : Vector<4, T> {
    Vector4() {}
    Vector4(T a, T b, T c, T d) { this->_d[0] = a; this->_d[1] = b; this->_d[2] = c; this->_d[3] = d; }
    Vector4(const Vector3<T> &v, T d) { this->_d[0] = v[0]; this->_d[1] = v[1]; this->_d[2] = v[2]; this->_d[3] = d; }
    Vector3<T> xyz() const { return {this->_d[0], this->_d[1], this->_d[2]}; }
    MXSHIM_VEC_OPS(Vector4, 4)
};
template <class T> T ceil(T v) { return std::ceil(v); }
template <class T> T min(T a, T b) { return std::min(a, b); }
template <class T> T max(T a, T b) { return std::max(a, b); }
template <class T> T dot(const Vector3<T> &a, const Vector3<T> &b) { return (a * b).sum(); }
template <class T> Vector3<T> cross(const Vector3<T> &a, const Vector3<T> &b) {
    return {a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2], a[0] * b[1] - a[1] * b[0]};
}
template <class T> struct Range3D {
    Vector3<T> _min, _max;
    Vector3<T> &min() { return _min; }
    Vector3<T> &max() { return _max; }
    const Vector3<T> &min() const { return _min; }
    const Vector3<T> &max() const { return _max; }
    Vector3<T> size() const { return _max - _min; }
    Vector3<T> center() const { return (_min + _max) * T(0.5); }
};
template <class T> struct Matrix3 {
    Vector3<T> c[3];
    Vector3<T> &operator[](std::size_t i) { return c[i]; }
    const Vector3<T> &operator[](std::size_t i) const { return c[i]; }
};
template <class T> struct Matrix4 { Vector4<T> c[4]; };
template <class T> struct Quaternion {
    Vector3<T> _v; T _w;
    Quaternion() : _w(1) {}
    Quaternion(const Vector3<T> &a, T b) : _v(a), _w(b) {}
    const Vector3<T> &vector() const { return _v; }
    T scalar() const { return _w; }
    Quaternion operator*(const Quaternion &o) const {
        return Quaternion(o._v * _w + _v * o._w + cross(_v, o._v), _w * o._w - dot(_v, o._v));
    }
    Quaternion conjugated() const { return Quaternion(-_v, _w); }
    Vector3<T> transformVector(const Vector3<T> &v) const {
        Quaternion p(v, T(0));
        return ((*this) * p * conjugated())._v;
    }
    Vector3<T> transformVectorNormalized(const Vector3<T> &v) const { return transformVector(v); }
};
}
typedef Math::Vector2<float> Vector2;
typedef Math::Vector3<float> Vector3;
typedef Math::Vector4<float> Vector4;
typedef Math::Vector3<double> Vector3d;
typedef Math::Vector2<double> Vector2d;
typedef Math::Vector4<double> Vector4d;
typedef Math::Vector2<int> Vector2i;
typedef Math::Vector3<int> Vector3i;
typedef Math::Vector4<int> Vector4i;
typedef Math::Matrix3<float> Matrix3;
typedef Math::Matrix3<double> Matrix3d;
typedef Math::Matrix4<float> Matrix4;
typedef Math::Quaternion<float> Quaternion;
typedef Math::Vector3<float> Color3;
typedef Math::Vector4<float> Color4;
typedef Math::Range3D<float> Range3D;
typedef float Float;
typedef double Double;
typedef int Int;
typedef unsigned int UnsignedInt;
}
