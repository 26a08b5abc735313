// Test infrastructure only: a project-written stand-in for the subset of the
// OpenEXR 2.x Imath vector API (pinned by the reference at openexr/[>=2.5.3 <3],
// conanfile.py:19) that the emerald sph2d_box / sph_common / z_index sources
// use. It exists so those unmodified reference sources compile in the oracle
// build (oracle/_ref); it is never linked into the product library.
//
// Arithmetic follows Imath's published definitions operator by operator:
// component-wise +,-,*,/ ; dot = x*u.x + y*u.y ; length() = sqrt(dot) unless
// dot < 2*FLT_MIN, in which case the components are rescaled by the larger
// magnitude first (Imath's lengthTiny).
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>
#include <ostream>

namespace Imath {

template <class T>
struct Math {
    static T sqrt(T x) { return std::sqrt(x); }
    static T fabs(T x) { return std::fabs(x); }
};

template <class T>
struct limits {
    static T smallest() { return std::numeric_limits<T>::min(); }
    static T min() { return std::numeric_limits<T>::lowest(); }
    static T max() { return std::numeric_limits<T>::max(); }
};

template <class T>
struct Vec2 {
    T x, y;

    Vec2() {}
    explicit Vec2(T a) : x(a), y(a) {}
    Vec2(T a, T b) : x(a), y(b) {}
    template <class S>
    explicit Vec2(Vec2<S> const& v) : x(T(v.x)), y(T(v.y)) {}

    T& operator[](int i) { return (&x)[i]; }
    T const& operator[](int i) const { return (&x)[i]; }

    static unsigned int dimensions() { return 2; }
    static T baseTypeMin() { return limits<T>::min(); }
    static T baseTypeMax() { return limits<T>::max(); }
    static T baseTypeSmallest() { return limits<T>::smallest(); }

    template <class S>
    bool operator==(Vec2<S> const& v) const { return x == v.x && y == v.y; }
    template <class S>
    bool operator!=(Vec2<S> const& v) const { return x != v.x || y != v.y; }

    T dot(Vec2 const& v) const { return x * v.x + y * v.y; }
    T cross(Vec2 const& v) const { return x * v.y - y * v.x; }

    Vec2 const& operator+=(Vec2 const& v) { x += v.x; y += v.y; return *this; }
    Vec2 operator+(Vec2 const& v) const { return Vec2(x + v.x, y + v.y); }
    Vec2 const& operator-=(Vec2 const& v) { x -= v.x; y -= v.y; return *this; }
    Vec2 operator-(Vec2 const& v) const { return Vec2(x - v.x, y - v.y); }
    Vec2 operator-() const { return Vec2(-x, -y); }
    Vec2 const& operator*=(Vec2 const& v) { x *= v.x; y *= v.y; return *this; }
    Vec2 const& operator*=(T a) { x *= a; y *= a; return *this; }
    Vec2 operator*(Vec2 const& v) const { return Vec2(x * v.x, y * v.y); }
    Vec2 operator*(T a) const { return Vec2(x * a, y * a); }
    Vec2 const& operator/=(Vec2 const& v) { x /= v.x; y /= v.y; return *this; }
    Vec2 const& operator/=(T a) { x /= a; y /= a; return *this; }
    Vec2 operator/(Vec2 const& v) const { return Vec2(x / v.x, y / v.y); }
    Vec2 operator/(T a) const { return Vec2(x / a, y / a); }

    T lengthTiny() const {
        T absX = (x >= T(0)) ? x : -x;
        T absY = (y >= T(0)) ? y : -y;
        T mx = absX;
        if (mx < absY) mx = absY;
        if (mx == T(0)) return T(0);
        absX /= mx;
        absY /= mx;
        return mx * Math<T>::sqrt(absX * absX + absY * absY);
    }
    T length() const {
        T l2 = dot(*this);
        if (l2 < T(2) * limits<T>::smallest()) return lengthTiny();
        return Math<T>::sqrt(l2);
    }
    T length2() const { return dot(*this); }
    Vec2 normalized() const {
        T l = length();
        if (l == T(0)) return Vec2(T(0));
        return Vec2(x / l, y / l);
    }
};

template <class T>
inline Vec2<T> operator*(T a, Vec2<T> const& v) {
    return Vec2<T>(a * v.x, a * v.y);
}

template <class T>
struct Vec3 {
    T x, y, z;

    Vec3() {}
    explicit Vec3(T a) : x(a), y(a), z(a) {}
    Vec3(T a, T b, T c) : x(a), y(b), z(c) {}
    template <class S>
    explicit Vec3(Vec3<S> const& v) : x(T(v.x)), y(T(v.y)), z(T(v.z)) {}

    T& operator[](int i) { return (&x)[i]; }
    T const& operator[](int i) const { return (&x)[i]; }

    static unsigned int dimensions() { return 3; }
    static T baseTypeMin() { return limits<T>::min(); }
    static T baseTypeMax() { return limits<T>::max(); }

    template <class S>
    bool operator==(Vec3<S> const& v) const { return x == v.x && y == v.y && z == v.z; }
    template <class S>
    bool operator!=(Vec3<S> const& v) const { return !(*this == v); }

    T dot(Vec3 const& v) const { return x * v.x + y * v.y + z * v.z; }
    Vec3 cross(Vec3 const& v) const {
        return Vec3(y * v.z - z * v.y, z * v.x - x * v.z, x * v.y - y * v.x);
    }
    Vec3 const& operator+=(Vec3 const& v) { x += v.x; y += v.y; z += v.z; return *this; }
    Vec3 operator+(Vec3 const& v) const { return Vec3(x + v.x, y + v.y, z + v.z); }
    Vec3 const& operator-=(Vec3 const& v) { x -= v.x; y -= v.y; z -= v.z; return *this; }
    Vec3 operator-(Vec3 const& v) const { return Vec3(x - v.x, y - v.y, z - v.z); }
    Vec3 operator-() const { return Vec3(-x, -y, -z); }
    Vec3 const& operator*=(T a) { x *= a; y *= a; z *= a; return *this; }
    Vec3 operator*(T a) const { return Vec3(x * a, y * a, z * a); }
    Vec3 operator*(Vec3 const& v) const { return Vec3(x * v.x, y * v.y, z * v.z); }
    Vec3 const& operator/=(T a) { x /= a; y /= a; z /= a; return *this; }
    Vec3 operator/(T a) const { return Vec3(x / a, y / a, z / a); }
    T length2() const { return dot(*this); }
    T length() const { return Math<T>::sqrt(dot(*this)); }
};

template <class T>
inline Vec3<T> operator*(T a, Vec3<T> const& v) {
    return Vec3<T>(a * v.x, a * v.y, a * v.z);
}

template <class T>
struct Vec4 {
    T x, y, z, w;
    Vec4() {}
    Vec4(T a, T b, T c, T d) : x(a), y(b), z(c), w(d) {}
    T& operator[](int i) { return (&x)[i]; }
    T const& operator[](int i) const { return (&x)[i]; }
};

template <class T>
std::ostream& operator<<(std::ostream& s, Vec2<T> const& v) {
    return s << '(' << v.x << ' ' << v.y << ')';
}
template <class T>
std::ostream& operator<<(std::ostream& s, Vec3<T> const& v) {
    return s << '(' << v.x << ' ' << v.y << ' ' << v.z << ')';
}

typedef Vec2<short> V2s;
typedef Vec2<int> V2i;
typedef Vec2<float> V2f;
typedef Vec2<double> V2d;
typedef Vec3<short> V3s;
typedef Vec3<int> V3i;
typedef Vec3<float> V3f;
typedef Vec3<double> V3d;
typedef Vec4<short> V4s;
typedef Vec4<int> V4i;
typedef Vec4<float> V4f;
typedef Vec4<double> V4d;

}  // namespace Imath
