// Test infrastructure only: stand-in for Imath::Box (OpenEXR 2.x) as used by
// the emerald reference sources (default-empty box, extendBy, size, isEmpty).
#pragma once

#include <OpenEXR/ImathVec.h>

namespace Imath {

template <class V>
struct Box {
    V min;
    V max;

    Box() { makeEmpty(); }
    explicit Box(V const& p) : min(p), max(p) {}
    Box(V const& a, V const& b) : min(a), max(b) {}

    void makeEmpty() {
        for (unsigned int i = 0; i < V::dimensions(); ++i) {
            min[i] = V::baseTypeMax();
            max[i] = V::baseTypeMin();
        }
    }
    void extendBy(V const& p) {
        for (unsigned int i = 0; i < V::dimensions(); ++i) {
            if (p[i] < min[i]) min[i] = p[i];
            if (p[i] > max[i]) max[i] = p[i];
        }
    }
    void extendBy(Box const& b) {
        for (unsigned int i = 0; i < V::dimensions(); ++i) {
            if (b.min[i] < min[i]) min[i] = b.min[i];
            if (b.max[i] > max[i]) max[i] = b.max[i];
        }
    }
    bool isEmpty() const {
        for (unsigned int i = 0; i < V::dimensions(); ++i) {
            if (max[i] < min[i]) return true;
        }
        return false;
    }
    V size() const {
        if (isEmpty()) {
            V z;
            for (unsigned int i = 0; i < V::dimensions(); ++i) z[i] = 0;
            return z;
        }
        return max - min;
    }
    bool operator==(Box const& b) const { return min == b.min && max == b.max; }
    bool operator!=(Box const& b) const { return !(*this == b); }
};

typedef Box<V2s> Box2s;
typedef Box<V2i> Box2i;
typedef Box<V2f> Box2f;
typedef Box<V2d> Box2d;
typedef Box<V3s> Box3s;
typedef Box<V3i> Box3i;
typedef Box<V3f> Box3f;
typedef Box<V3d> Box3d;

}  // namespace Imath
