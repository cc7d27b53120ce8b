// detmath.h -- float3 arithmetic and fixed-definition transcendentals shared by
// the host scene builder and the sm_100a kernels.
//
// Rounding contract: every translation unit that includes this header is built
// without FMA contraction (nvcc --fmad=false, g++ -ffp-contract=off) and
// without fast-math, so a*b+c rounds twice exactly as the reference's source
// expressions read (core/vector.cuh).  Explicit fmaf() is used where a fused
// multiply-add is intended.  Division and square root are IEEE round-to-nearest
// on both host and device.  The reference's rsqrtf/sinf/cosf/expf/logf/powf
// (vector.cuh:222-283, sample.cuh, nee.cuh, render.cuh:58-73, config.cuh:3)
// are replaced by the fixed definitions below so that results do not depend on
// which machine computes them:
//   sin/cos: Cody-Waite reduction by pi/2 (three-part split), Taylor series to
//            x^11 / x^10 on [-pi/4, pi/4];
//   exp:     reduction by ln 2 (two-part split), Taylor series to r^8, ldexpf;
//   log:     frexp into [sqrt(1/2), sqrt(2)), 2*atanh((m-1)/(m+1)) series to s^11;
//   pow:     exp(y * log x);   rsqrt: 1/sqrt.
#pragma once

#include <cfloat>
#include <cmath>
#include <cstdint>

#ifdef __CUDACC__
#define AR_HD __host__ __device__ __forceinline__
#else
#define AR_HD inline
#endif

namespace ar {

struct f3 { float x, y, z; };

AR_HD bool isnan_(float x) { return x != x; }
AR_HD bool isinf_(float x) { return fabsf(x) == INFINITY; }
AR_HD f3 mk(float x, float y, float z) { f3 r; r.x = x; r.y = y; r.z = z; return r; }
AR_HD f3 operator+(f3 a, f3 b) { return mk(a.x + b.x, a.y + b.y, a.z + b.z); }
AR_HD f3 operator-(f3 a, f3 b) { return mk(a.x - b.x, a.y - b.y, a.z - b.z); }
AR_HD f3 operator-(f3 a) { return mk(-a.x, -a.y, -a.z); }
AR_HD f3 operator*(f3 a, f3 b) { return mk(a.x * b.x, a.y * b.y, a.z * b.z); }
AR_HD f3 operator*(f3 a, float b) { return mk(a.x * b, a.y * b, a.z * b); }
AR_HD f3 operator/(f3 a, float b) { return mk(a.x / b, a.y / b, a.z / b); }
AR_HD f3 operator/(f3 a, f3 b) { return mk(a.x / b.x, a.y / b.y, a.z / b.z); }
AR_HD float dot(f3 a, f3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
AR_HD f3 cross(f3 a, f3 b) { return mk(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x); }
AR_HD float length(f3 a) { return sqrtf(dot(a, a)); }
AR_HD f3 vmin(f3 a, f3 b) { return mk(fminf(a.x, b.x), fminf(a.y, b.y), fminf(a.z, b.z)); }
AR_HD f3 vmax(f3 a, f3 b) { return mk(fmaxf(a.x, b.x), fmaxf(a.y, b.y), fmaxf(a.z, b.z)); }
AR_HD f3 vmaxs(f3 a, float b) { return mk(fmaxf(a.x, b), fmaxf(a.y, b), fmaxf(a.z, b)); }
AR_HD float max3(f3 a) { return fmaxf(a.x, fmaxf(a.y, a.z)); }
AR_HD f3 vabs(f3 a) { return mk(fabsf(a.x), fabsf(a.y), fabsf(a.z)); }
AR_HD bool all_zero(f3 a) { return a.x == 0.0f && a.y == 0.0f && a.z == 0.0f; }
AR_HD float rsqrt_ieee(float x) { return 1.0f / sqrtf(x); }
// normalize (vector.cuh:222-231) with rsqrtf -> 1/sqrtf
AR_HD f3 normalize(f3 v)
{
    const float l2 = dot(v, v);
    if (l2 <= 1e-20f) return mk(0.0f, 0.0f, 0.0f);
    return v * rsqrt_ieee(l2);
}
AR_HD float clampf(float v, float a, float b) { return isnan_(v) ? 0.0f : fminf(fmaxf(v, a), b); }
AR_HD float saturate(float v) { return isnan_(v) ? 0.0f : fminf(fmaxf(v, 0.0f), 1.0f); }
AR_HD float signf(float a) { return a > 0.0f ? 1.0f : (a < 0.0f ? -1.0f : 0.0f); }
AR_HD float lerpf(float a, float b, float v) { return a * (1.0f - v) + b * v; }
AR_HD f3 lerp3(f3 a, f3 b, float v) { return mk(lerpf(a.x, b.x, v), lerpf(a.y, b.y, v), lerpf(a.z, b.z, v)); }
AR_HD float luminance(f3 c) { return dot(c, mk(0.2126f, 0.7152f, 0.0722f)); }
AR_HD f3 reflect(f3 v, f3 n) { return v - n * (2.0f * dot(v, n)); }
AR_HD f3 refract(f3 in, f3 normal, float eta)
{
    const f3 n = (dot(normal, in) > 0.0f) ? -normal : normal;
    const float cosI = -dot(n, in);
    const float k = 1.0f - (eta * eta) * fmaxf(0.0f, 1.0f - cosI * cosI);
    const float cosT = sqrtf(fmaxf(0.0f, k));
    return in * eta + n * (eta * cosI - cosT);
}
AR_HD float inv_safe(float x) { return (x == 0.0f) ? (x >= 0 ? FLT_MAX : -FLT_MAX) : 1.0f / x; }

// Row-major 3x3 (float3x3, vector.cuh:320-420)
struct m3 { f3 x, y, z; };
AR_HD f3 mul(const m3& m, f3 v) { return mk(dot(m.x, v), dot(m.y, v), dot(m.z, v)); }

constexpr float kPi = 3.14159265358979f;  // CUDART_PI_F

// ---------------------------------------------------------------- sin / cos
AR_HD void sincos_det(float x, float* s, float* c)
{
    if (isnan_(x) || isinf_(x)) { *s = NAN; *c = NAN; return; }
    const float k = rintf(x * 0x1.45f306p-1f);
    float r = fmaf(-k, 0x1.921fb6p+0f, x);
    r = fmaf(-k, -0x1.777a5cp-25f, r);
    r = fmaf(-k, -0x1.ee59dap-50f, r);
    const float z = r * r;
    float ps = fmaf(z, -0x1.ae6456p-26f, 0x1.71de3ap-19f);
    ps = fmaf(z, ps, -0x1.a01a02p-13f);
    ps = fmaf(z, ps, 0x1.111112p-7f);
    ps = fmaf(z, ps, -0x1.555556p-3f);
    const float sr = fmaf(r * z, ps, r);
    float pc = fmaf(z, -0x1.27e4fcp-22f, 0x1.a01a02p-16f);
    pc = fmaf(z, pc, -0x1.6c16c2p-10f);
    pc = fmaf(z, pc, 0x1.555556p-5f);
    pc = fmaf(z, pc, -0.5f);
    const float cr = fmaf(z, pc, 1.0f);
    const int q = static_cast<int>(static_cast<long long>(k) & 3);
    if (q == 0) { *s = sr; *c = cr; }
    else if (q == 1) { *s = cr; *c = -sr; }
    else if (q == 2) { *s = -sr; *c = -cr; }
    else { *s = -cr; *c = sr; }
}
AR_HD float tan_det(float x) { float s, c; sincos_det(x, &s, &c); return s / c; }

// ---------------------------------------------------------------- exp / log / pow
AR_HD float exp_det(float x)
{
    if (isnan_(x)) return x;
    if (x > 88.72f) return INFINITY;
    if (x < -103.98f) return 0.0f;
    const float k = rintf(x * 0x1.715476p+0f);
    float r = fmaf(-k, 0x1.62e430p-1f, x);
    r = fmaf(-k, -0x1.05c610p-29f, r);
    float p = 0x1.a01a02p-16f;
    p = fmaf(p, r, 0x1.a01a02p-13f);
    p = fmaf(p, r, 0x1.6c16c2p-10f);
    p = fmaf(p, r, 0x1.111112p-7f);
    p = fmaf(p, r, 0x1.555556p-5f);
    p = fmaf(p, r, 0x1.555556p-3f);
    p = fmaf(p, r, 0.5f);
    p = fmaf(p, r, 1.0f);
    p = fmaf(p, r, 1.0f);
    return ldexpf(p, static_cast<int>(k));
}
AR_HD float log_det(float x)
{
    if (isnan_(x) || x < 0.0f) return NAN;
    if (x == 0.0f) return -INFINITY;
    if (isinf_(x)) return x;
    int e;
    float m = frexpf(x, &e);
    if (m < 0x1.6a09e6p-1f) { m = m * 2.0f; e = e - 1; }
    const float s = (m - 1.0f) / (m + 1.0f);
    const float z = s * s;
    float p = fmaf(z, 0x1.745d18p-4f, 0x1.c71c72p-4f);
    p = fmaf(z, p, 0x1.24924ap-3f);
    p = fmaf(z, p, 0x1.99999ap-3f);
    p = fmaf(z, p, 0x1.555556p-2f);
    const float t = 2.0f * s;
    const float logm = fmaf(t * z, p, t);
    const float ef = static_cast<float>(e);
    return fmaf(ef, 0x1.62e430p-1f, fmaf(ef, -0x1.05c610p-29f, logm));
}
AR_HD float pow_det(float x, float y)
{
    if (x == 0.0f) return (y > 0.0f) ? 0.0f : (y == 0.0f ? 1.0f : INFINITY);
    if (x == 1.0f || y == 0.0f) return 1.0f;
    if (x < 0.0f || isnan_(x) || isnan_(y)) return NAN;
    return exp_det(y * log_det(x));
}

}  // namespace ar
