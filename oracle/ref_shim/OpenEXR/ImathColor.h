// Test infrastructure only: stand-in for Imath::Color3 / Color4 (OpenEXR 2.x).
#pragma once

#include <OpenEXR/ImathVec.h>

namespace Imath {

template <class T>
struct Color3 : public Vec3<T> {
    Color3() {}
    Color3(T a, T b, T c) : Vec3<T>(a, b, c) {}
};

template <class T>
struct Color4 {
    T r, g, b, a;
    Color4() {}
    Color4(T x, T y, T z, T w) : r(x), g(y), b(z), a(w) {}
    T& operator[](int i) { return (&r)[i]; }
    T const& operator[](int i) const { return (&r)[i]; }
};

typedef Color3<float> C3f;
typedef Color3<unsigned char> C3c;
typedef Color4<float> C4f;
typedef Color4<unsigned char> C4c;

}  // namespace Imath
