// Per-particle arithmetic of the 2D SPH step, shared by every kernel.
//
// Each helper restates one reference operation in the same IEEE
// single-precision operator order; the library is compiled with
// --fmad=false (no contraction), IEEE division and square root, and
// denormals preserved, so device results are bit-identical to the
// reference's CPU results for the same inputs.
#pragma once

#include <cmath>
#include <cstdint>
#include <limits>

#include <cuda_runtime.h>

namespace emerald {

#define EMLD_HD __host__ __device__ __forceinline__

EMLD_HD float2 mk2(float x, float y) { return make_float2(x, y); }
EMLD_HD float2 add2(float2 a, float2 b) { return mk2(a.x + b.x, a.y + b.y); }
EMLD_HD float2 sub2(float2 a, float2 b) { return mk2(a.x - b.x, a.y - b.y); }
EMLD_HD float2 neg2(float2 a) { return mk2(-a.x, -a.y); }
EMLD_HD float2 scl2(float s, float2 a) { return mk2(s * a.x, s * a.y); }
EMLD_HD float2 div2(float2 a, float s) { return mk2(a.x / s, a.y / s); }
EMLD_HD float dot2(float2 a, float2 b) { return a.x * b.x + a.y * b.y; }
EMLD_HD float sqrf(float a) { return a * a; }

// std::max(0.0f, x) and std::max(x, 0.0f): they differ for NaN and -0.0.
EMLD_HD float max_0x(float x) { return (0.0f < x) ? x : 0.0f; }
EMLD_HD float max_x0(float x) { return (x < 0.0f) ? 0.0f : x; }

// mix(a, b, t) = a*(1-t) + b*t (emerald/util/functions.h:45-49).
EMLD_HD float mix1(float a, float b, float t) { return (a * (1.0f - t)) + (b * t); }

constexpr float kFltMin = 1.17549435082228750797e-38f;  // FLT_MIN
constexpr double kDblMin = 2.2250738585072013831e-308;  // DBL_MIN

// is_safe_divide for float and for Vec2 (emerald/util/safe_divide.h:20-31, 48-59).
EMLD_HD bool safe_f(float n, float d) {
    if (d == 0.0f) return false;
    if (fabsf(d) >= 1.0f) return true;
    return (fabsf(d) / kFltMin) > fabsf(n);
}
EMLD_HD bool safe_v(float2 n, float d) {
    if (d == 0.0f) return false;
    if (fabsf(d) >= 1.0f) return true;
    float const mr = fabsf(d) / kFltMin;
    return (mr > fabsf(n.x)) && (mr > fabsf(n.y));
}
EMLD_HD bool safe_d(double n, double d) {
    if (d == 0.0) return false;
    if (fabs(d) >= 1.0) return true;
    return (fabs(d) / kDblMin) > fabs(n);
}

// Imath Vec2<float>::length(): sqrt of the dot product, rescaled by the
// larger component when the dot product is below 2*FLT_MIN.
EMLD_HD float length2f(float2 a) {
    float const l2 = dot2(a, a);
    if (l2 < 2.0f * kFltMin) {
        float ax = (a.x >= 0.0f) ? a.x : -a.x;
        float ay = (a.y >= 0.0f) ? a.y : -a.y;
        float m = ax;
        if (m < ay) m = ay;
        if (m == 0.0f) return 0.0f;
        ax /= m;
        ay /= m;
        return m * sqrtf(ax * ax + ay * ay);
    }
    return sqrtf(l2);
}

// Kahan-compensated running sums (Kahan 1965): s holds the sum, c the
// low-order part lost by the last addition. Exact under IEEE arithmetic
// without contraction, which these sources are compiled for.
struct KahanF {
    float s, c;
};
struct KahanF2 {
    KahanF x, y;
};
EMLD_HD void kahan_add(KahanF& k, float v) {
    float const y = v - k.c;
    float const t = k.s + y;
    k.c = (t - k.s) - y;
    k.s = t;
}
EMLD_HD void kahan_add(KahanF2& k, float2 v) {
    kahan_add(k.x, v.x);
    kahan_add(k.y, v.y);
}

// A running sum of float (SumF) or float2 (SumF2) terms: with K = false
// exactly the reference's s += t, with K = true Kahan-compensated.
template <bool K>
struct SumF {
    float s;
    EMLD_HD explicit SumF(float init = 0.0f) : s(init) {}
    EMLD_HD void add(float v) { s += v; }
    EMLD_HD float get() const { return s; }
};
template <>
struct SumF<true> {
    KahanF k;
    EMLD_HD explicit SumF(float init = 0.0f) : k{init, 0.0f} {}
    EMLD_HD void add(float v) { kahan_add(k, v); }
    EMLD_HD float get() const { return k.s; }
};
template <bool K>
struct SumF2 {
    float2 s;
    EMLD_HD SumF2() : s{0.0f, 0.0f} {}
    EMLD_HD void add(float2 v) {
        s.x += v.x;
        s.y += v.y;
    }
    EMLD_HD float2 get() const { return s; }
};
template <>
struct SumF2<true> {
    KahanF2 k;
    EMLD_HD SumF2() : k{{0.0f, 0.0f}, {0.0f, 0.0f}} {}
    EMLD_HD void add(float2 v) { kahan_add(k, v); }
    EMLD_HD float2 get() const { return float2{k.x.s, k.y.s}; }
};

// Cubic spline with the reference's 3D normalisation 1/(pi h^3), support 2h
// (emerald/sph_common/kernels.h:12-64).
constexpr float kPi = 3.14159274101257324218750f;

EMLD_HD float kernel_w(float r, float h) {
    float const q = r / h;
    float const k = h * h * h * kPi;
    if (q <= 1.0f) return (1.0f + q * q * (q * 0.75f - 1.5f)) / k;
    if (q <= 2.0f) {
        float const t = 2.0f - q;
        return ((t * t * t) / 4.0f) / k;
    }
    return 0.0f;
}

EMLD_HD float kernel_dw(float r, float h) {
    float const q = r / h;
    float const k = h * h * h * kPi;
    if (q <= 1.0f) return (-3.0f * r / (h * h) + 2.25f * r * r / (h * h * h)) / k;
    if (q <= 2.0f) return (-3.0f * sqrf(2.0f - (r / h)) / (4.0f * h)) / k;
    return 0.0f;
}

// W and dW of the same r, sharing q = r / h (the same value either function
// computes on its own).
EMLD_HD void kernel_w_dw(float r, float h, float& w, float& dw) {
    float const q = r / h;
    float const k = h * h * h * kPi;
    if (q <= 1.0f) {
        w = (1.0f + q * q * (q * 0.75f - 1.5f)) / k;
        dw = (-3.0f * r / (h * h) + 2.25f * r * r / (h * h * h)) / k;
    } else if (q <= 2.0f) {
        float const t = 2.0f - q;
        w = ((t * t * t) / 4.0f) / k;
        dw = (-3.0f * sqrf(2.0f - q) / (4.0f * h)) / k;
    } else {
        w = 0.0f;
        dw = 0.0f;
    }
}

EMLD_HD float2 kernel_grad_w(float2 dp, float h) {
    float const r = length2f(dp);
    if (safe_v(dp, r)) {
        float const d = kernel_dw(r, h);
        float2 const u = div2(dp, r);
        return mk2(u.x * d, u.y * d);
    }
    return mk2(0.0f, 0.0f);
}

// safe_divide(p, sqr(rho)).value_or(0) (emerald/sph_common/pressure.cpp:21-23).
EMLD_HD float p_over_rho2(float p, float rho) {
    float const d = sqrf(rho);
    return safe_f(p, d) ? p / d : 0.0f;
}

// Morton key of a grid cell: 32-bit x in the even bits, y in the odd bits
// (emerald/z_index/z_index.cpp:8-10, 17-48). Negative cells are taken as
// their uint32 bit patterns, as the reference's int32 -> uint32 conversion.
EMLD_HD uint64_t spread_bits(uint32_t v) {
    uint64_t x = v;
    x = (x | (x << 16)) & 0x0000FFFF0000FFFFull;
    x = (x | (x << 8)) & 0x00FF00FF00FF00FFull;
    x = (x | (x << 4)) & 0x0F0F0F0F0F0F0F0Full;
    x = (x | (x << 2)) & 0x3333333333333333ull;
    x = (x | (x << 1)) & 0x5555555555555555ull;
    return x;
}
EMLD_HD uint64_t morton2(uint32_t x, uint32_t y) { return spread_bits(x) | (spread_bits(y) << 1); }

// compute_grid_coord with bounds_min (0,0) (emerald/sph_common/common.cpp:43-56).
EMLD_HD void grid_coord(float2 p, float cell, int32_t& gx, int32_t& gy) {
    float2 const q = div2(sub2(p, mk2(0.0f, 0.0f)), cell);
    gx = static_cast<int32_t>(floorf(q.x));
    gy = static_cast<int32_t>(floorf(q.y));
}

// Smallest float t with sqrtf(t) >= d (host side): x*x + y*y >= t holds
// exactly when the correctly rounded length of (x, y) is >= d.
inline float reject_threshold(float d) {
    float const inf = std::numeric_limits<float>::infinity();
    if (!(d > 0.0f)) return 0.0f;
    if (!(d < 1.8e19f)) return inf;
    float t = d * d;
    while (t > 0.0f && std::sqrt(std::nextafter(t, 0.0f)) >= d) t = std::nextafter(t, 0.0f);
    while (std::sqrt(t) < d) t = std::nextafter(t, inf);
    return t;
}

}  // namespace emerald
