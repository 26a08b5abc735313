// Test infrastructure only: the emerald sources name Imath matrix and
// quaternion types in typedefs but never use them on the SPH path.
#pragma once

#include <OpenEXR/ImathVec.h>

namespace Imath {
template <class T>
struct Matrix33 { T x[3][3]; };
template <class T>
struct Matrix44 { T x[4][4]; };
template <class T>
struct Quat { T r; Vec3<T> v; };
typedef Matrix33<float> M33f;
typedef Matrix33<double> M33d;
typedef Matrix44<float> M44f;
typedef Matrix44<double> M44d;
}  // namespace Imath
