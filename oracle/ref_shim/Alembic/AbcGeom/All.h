// Test infrastructure only: emerald/util/foundation.h imports Imath-based type
// aliases through Alembic::AbcGeom. This stand-in supplies those aliases from
// the Imath stand-in so the reference sources compile without Alembic.
#pragma once

#include <OpenEXR/ImathBox.h>
#include <OpenEXR/ImathColor.h>
#include <OpenEXR/ImathMatrix.h>
#include <OpenEXR/ImathVec.h>
#include <OpenEXR/half.h>

#include <cstdint>

namespace Alembic {
namespace AbcGeom {
typedef bool bool_t;
typedef std::uint8_t byte_t;
typedef double chrono_t;
typedef ::half float16_t;
typedef float float32_t;
typedef double float64_t;
typedef std::int64_t index_t;
using std::int16_t;
using std::int32_t;
using std::int64_t;
using std::int8_t;
using std::uint16_t;
using std::uint32_t;
using std::uint64_t;
using std::uint8_t;
using Imath::V2d;
using Imath::V2f;
using Imath::V2i;
using Imath::V2s;
using Imath::V3d;
using Imath::V3f;
using Imath::V3i;
using Imath::V3s;
using Imath::Box2d;
using Imath::Box2f;
using Imath::Box2i;
using Imath::Box2s;
using Imath::Box3d;
using Imath::Box3f;
using Imath::Box3i;
using Imath::Box3s;
using Imath::M33d;
using Imath::M33f;
using Imath::M44d;
using Imath::M44f;
typedef Imath::Quat<double> Quatd;
typedef Imath::Quat<float> Quatf;
typedef Imath::Color3<unsigned char> C3c;
typedef Imath::Color3<float> C3f;
typedef Imath::Color3<::half> C3h;
typedef Imath::Color4<unsigned char> C4c;
typedef Imath::Color4<float> C4f;
typedef Imath::Color4<::half> C4h;
typedef Imath::Vec3<double> N3d;
typedef Imath::Vec3<float> N3f;
}  // namespace AbcGeom
}  // namespace Alembic
