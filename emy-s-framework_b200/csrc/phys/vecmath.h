// Vector / matrix / quaternion / transform arithmetic for the arena kernels.
//
// The reference simulator runs Bullet 3.24 with its x86 SSE code paths
// (LinearMath/btVector3.h, btMatrix3x3.h, btQuaternion.h, btTransform.h).  The
// routines below evaluate the same expressions with the same association order,
// so that single-precision results equal the reference's: normalisation starts its
// Newton step from the CPU's rsqrtss estimate and sin / cos / atan2 / asin return
// the reference C library's bits (refmath.h).
//
// Conventions follow Bullet: a Mat3 is stored as three rows; `m * v` is three row
// dot products; `v * m` (tmul) is the transposed product.
//
// ALTERED SOURCE: this file is not the original Bullet code.  It restates the algorithms of
// the Bullet 3.24 files named above (as patched in RocketSim) for a CUDA device and a host
// build, with its own data layout, naming and control flow; the original's notice follows.
//
// Bullet Continuous Collision Detection and Physics Library
// Copyright (c) 2003-2006 Erwin Coumans  https://bulletphysics.org
//
// This software is provided 'as-is', without any express or implied warranty.
// In no event will the authors be held liable for any damages arising from the use of this software.
// Permission is granted to anyone to use this software for any purpose,
// including commercial applications, and to alter it and redistribute it freely,
// subject to the following restrictions:
//
// 1. The origin of this software must not be misrepresented; you must not claim that you wrote the original software. If you use this software in a product, an acknowledgment in the product documentation would be appreciated but is not required.
// 2. Altered source versions must be plainly marked as such, and must not be misrepresented as being the original software.
// 3. This notice may not be removed or altered from any source distribution.
#pragma once
#include "hd.h"
#include "refmath.h"

namespace rsb {

struct V3 {
    float x, y, z;
    RSB_HD float operator[](int i) const { return i == 0 ? x : (i == 1 ? y : z); }
    RSB_HD float& operator[](int i) { return i == 0 ? x : (i == 1 ? y : z); }
};

RSB_HD V3 v3(float x, float y, float z) { return V3{x, y, z}; }
RSB_HD V3 v3zero() { return V3{0.f, 0.f, 0.f}; }
RSB_HD V3 operator+(V3 a, V3 b) { return V3{a.x + b.x, a.y + b.y, a.z + b.z}; }
RSB_HD V3 operator-(V3 a, V3 b) { return V3{a.x - b.x, a.y - b.y, a.z - b.z}; }
RSB_HD V3 operator-(V3 a) { return V3{-a.x, -a.y, -a.z}; }
RSB_HD V3 operator*(V3 a, V3 b) { return V3{a.x * b.x, a.y * b.y, a.z * b.z}; }
RSB_HD V3 operator*(V3 a, float s) { return V3{a.x * s, a.y * s, a.z * s}; }
RSB_HD V3 operator*(float s, V3 a) { return V3{a.x * s, a.y * s, a.z * s}; }
// Bullet divides a vector by a scalar as a multiply by the reciprocal.
RSB_HD V3 bdiv(V3 a, float s) { float r = 1.f / s; return a * r; }
// RocketSim's own Vec type divides component-wise.
RSB_HD V3 vdiv(V3 a, float s) { return V3{a.x / s, a.y / s, a.z / s}; }
RSB_HD V3& operator+=(V3& a, V3 b) { a = a + b; return a; }
RSB_HD V3& operator-=(V3& a, V3 b) { a = a - b; return a; }
RSB_HD V3& operator*=(V3& a, float s) { a = a * s; return a; }
RSB_HD bool operator==(V3 a, V3 b) { return a.x == b.x && a.y == b.y && a.z == b.z; }

RSB_HD float dot(V3 a, V3 b) { return (a.x * b.x + a.y * b.y) + a.z * b.z; }
// Association of the solver's SSE2 row kernels (btSimdDot3): x + (y + z).
RSB_HD float dot_simd(V3 a, V3 b) {
    float px = a.x * b.x, py = a.y * b.y, pz = a.z * b.z;
    return px + (py + pz);
}
RSB_HD V3 cross(V3 a, V3 b) {
    return V3{a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}
RSB_HD float length2(V3 a) { return dot(a, a); }
RSB_HD float length(V3 a) { return fsqrt(length2(a)); }
RSB_HD float dist2(V3 a, V3 b) { return length2(b - a); }
RSB_HD bool isZero(V3 a) { return a.x == 0.f && a.y == 0.f && a.z == 0.f; }
RSB_HD bool fuzzyZero(V3 a) { return length2(a) < kEpsilon * kEpsilon; }
RSB_HD V3 vabs(V3 a) { return V3{fabsf(a.x), fabsf(a.y), fabsf(a.z)}; }
// _mm_min_ps / _mm_max_ps semantics (first operand kept only if strictly smaller / larger)
RSB_HD V3 vmin(V3 a, V3 b) { return V3{a.x < b.x ? a.x : b.x, a.y < b.y ? a.y : b.y, a.z < b.z ? a.z : b.z}; }
RSB_HD V3 vmax(V3 a, V3 b) { return V3{a.x > b.x ? a.x : b.x, a.y > b.y ? a.y : b.y, a.z > b.z ? a.z : b.z}; }

// btVector3::normalize (SSE path): one Newton-Raphson step on 1/sqrt(|v|^2) from the
// rsqrtss estimate.
RSB_HD V3 normalized(V3 a) {
    float l2 = length2(a);
    float y0 = rsqrtEstimate(l2);
    float vd = l2 * 0.5f;
    vd = vd * y0;
    vd = vd * y0;
    float z = 1.5f - vd;
    float y = y0 * z;
    return a * y;
}
// btVector3::safeNormalize
RSB_HD V3 safeNormalized(V3 a) {
    float l2 = length2(a);
    if (l2 >= kEpsilon * kEpsilon) return bdiv(a, fsqrt(l2));
    return V3{1.f, 0.f, 0.f};
}
// RocketSim Vec::Normalized (MathTypes.h:88-95): true component division, zero below
// a length of FLT_EPSILON squared
RSB_HD V3 rsNormalized(V3 a) {
    float l = length(a);
    if (l > kEpsilon * kEpsilon) return vdiv(a, l);
    return v3zero();
}
RSB_HD int maxAxis(V3 a) { return a.x < a.y ? (a.y < a.z ? 2 : 1) : (a.x < a.z ? 2 : 0); }

// ------------------------------------------------------------------ Mat3 (rows)
struct M3 {
    V3 r[3];
    RSB_HD const V3& operator[](int i) const { return r[i]; }
    RSB_HD V3& operator[](int i) { return r[i]; }
    RSB_HD V3 col(int j) const { return V3{r[0][j], r[1][j], r[2][j]}; }
};

RSB_HD M3 m3(float a, float b, float c, float d, float e, float f, float g, float h, float i) {
    M3 m;
    m.r[0] = V3{a, b, c};
    m.r[1] = V3{d, e, f};
    m.r[2] = V3{g, h, i};
    return m;
}
RSB_HD M3 m3identity() { return m3(1, 0, 0, 0, 1, 0, 0, 0, 1); }
RSB_HD V3 operator*(const M3& m, V3 v) { return V3{dot(m.r[0], v), dot(m.r[1], v), dot(m.r[2], v)}; }
// v^T * m  (Bullet operator*(btVector3, btMatrix3x3))
RSB_HD V3 tmul(V3 v, const M3& m) {
    return V3{(m.r[0].x * v.x + m.r[1].x * v.y) + m.r[2].x * v.z,
              (m.r[0].y * v.x + m.r[1].y * v.y) + m.r[2].y * v.z,
              (m.r[0].z * v.x + m.r[1].z * v.y) + m.r[2].z * v.z};
}
RSB_HD M3 operator*(const M3& a, const M3& b) {
    M3 o;
    for (int i = 0; i < 3; i++) {
        V3 r = a.r[i];
        o.r[i] = V3{(r.x * b.r[0].x + r.y * b.r[1].x) + r.z * b.r[2].x,
                    (r.x * b.r[0].y + r.y * b.r[1].y) + r.z * b.r[2].y,
                    (r.x * b.r[0].z + r.y * b.r[1].z) + r.z * b.r[2].z};
    }
    return o;
}
RSB_HD M3 transpose(const M3& m) {
    return m3(m.r[0].x, m.r[1].x, m.r[2].x, m.r[0].y, m.r[1].y, m.r[2].y, m.r[0].z, m.r[1].z, m.r[2].z);
}
// this^T * m
RSB_HD M3 transposeTimes(const M3& a, const M3& m) {
    M3 o;
    for (int i = 0; i < 3; i++) {
        o.r[i] = V3{(a.r[0][i] * m.r[0].x + a.r[1][i] * m.r[1].x) + a.r[2][i] * m.r[2].x,
                    (a.r[0][i] * m.r[0].y + a.r[1][i] * m.r[1].y) + a.r[2][i] * m.r[2].y,
                    (a.r[0][i] * m.r[0].z + a.r[1][i] * m.r[1].z) + a.r[2][i] * m.r[2].z};
    }
    return o;
}
// rows scaled component-wise (btMatrix3x3::scaled)
RSB_HD M3 scaled(const M3& m, V3 s) { return M3{{m.r[0] * s, m.r[1] * s, m.r[2] * s}}; }
RSB_HD M3 mabs(const M3& m) { return M3{{vabs(m.r[0]), vabs(m.r[1]), vabs(m.r[2])}}; }
RSB_HD float cofac(const M3& m, int r1, int c1, int r2, int c2) {
    return m.r[r1][c1] * m.r[r2][c2] - m.r[r1][c2] * m.r[r2][c1];
}
RSB_HD M3 inverse(const M3& m) {
    V3 co = V3{cofac(m, 1, 1, 2, 2), cofac(m, 1, 2, 2, 0), cofac(m, 1, 0, 2, 1)};
    float det = dot(m.r[0], co);
    float s = 1.f / det;
    return m3(co.x * s, cofac(m, 0, 2, 2, 1) * s, cofac(m, 0, 1, 1, 2) * s,
              co.y * s, cofac(m, 0, 0, 2, 2) * s, cofac(m, 0, 2, 1, 0) * s,
              co.z * s, cofac(m, 0, 1, 2, 0) * s, cofac(m, 0, 0, 1, 1) * s);
}

// ------------------------------------------------------------------ Quaternion
struct Quat {
    float x, y, z, w;
};

// btQuaternion operator* (SSE path)
RSB_HD Quat qmul(Quat a, Quat b) {
    float a1x = a.x * b.w, a1y = a.y * b.w, a1z = a.z * b.w, a1w = a.x * b.x;
    float a2x = a.y * b.z, a2y = a.z * b.x, a2z = a.x * b.y, a2w = a.y * b.y;
    float b1x = a.z * b.y, b1y = a.x * b.z, b1z = a.y * b.x, b1w = a.z * b.z;
    float a0x = a.w * b.x, a0y = a.w * b.y, a0z = a.w * b.z, a0w = a.w * b.w;
    float s1x = a1x + a2x, s1y = a1y + a2y, s1z = a1z + a2z, s1w = -(a1w + a2w);
    float d0x = a0x - b1x, d0y = a0y - b1y, d0z = a0z - b1z, d0w = a0w - b1w;
    return Quat{d0x + s1x, d0y + s1y, d0z + s1z, d0w + s1w};
}
// btQuaternion * btVector3 (SSE path)
RSB_HD Quat qmulv(Quat q, V3 v) {
    float a1x = q.w * v.x, a1y = q.w * v.y, a1z = q.w * v.z, a1w = q.x * v.x;
    float a2x = q.y * v.z, a2y = q.z * v.x, a2z = q.x * v.y, a2w = q.y * v.y;
    float a3x = q.z * v.y, a3y = q.x * v.z, a3z = q.y * v.x, a3w = q.z * v.z;
    float sx = a1x + a2x, sy = a1y + a2y, sz = a1z + a2z, sw = -(a1w + a2w);
    return Quat{sx - a3x, sy - a3y, sz - a3z, sw - a3w};
}
RSB_HD Quat qinverse(Quat q) { return Quat{-q.x, -q.y, -q.z, q.w}; }
RSB_HD float qlength2(Quat q) {
    float xx = q.x * q.x, yy = q.y * q.y, zz = q.z * q.z, ww = q.w * q.w;
    return (xx + zz) + (yy + ww);
}
RSB_HD Quat qnormalized(Quat q) {
    float s = 1.f / fsqrt(qlength2(q));
    return Quat{q.x * s, q.y * s, q.z * s, q.w * s};
}
RSB_HD Quat qsafeNormalized(Quat q) {
    if (qlength2(q) > kEpsilon) return qnormalized(q);
    return q;
}
// btQuaternion(axis, angle)
RSB_HD Quat qaxisAngle(V3 axis, float angle) {
    float d = length(axis);
    float s = rsSinf(angle * 0.5f) / d;
    return Quat{axis.x * s, axis.y * s, axis.z * s, rsCosf(angle * 0.5f)};
}
// quatRotate(rotation, v)
RSB_HD V3 quatRotate(Quat r, V3 v) {
    Quat q = qmulv(r, v);
    q = qmul(q, qinverse(r));
    return V3{q.x, q.y, q.z};
}
// btMatrix3x3::setRotation (SSE path)
RSB_HD M3 m3fromQuat(Quat q) {
    float d = qlength2(q);
    float s = 2.f / d;
    float x = q.x, y = q.y, z = q.z, w = q.w;
    float xx = x * x, yy = y * y, zz = z * z, xy = x * y, zx = z * x, yz = y * z;
    float wz = w * z, wy = w * y, wx = w * x;
    // rows as produced by the shuffles of the SSE implementation
    float r00 = -yy + -zz, r01 = xy + -wz, r02 = zx + y * w;
    float r10 = xy + z * w, r11 = -xx + -zz, r12 = yz + -wx;
    float r20 = zx + -wy, r21 = yz + w * x, r22 = -xx + -yy;
    (void)wy;
    return m3(r00 * s + 1.f, r01 * s, r02 * s,
              r10 * s, r11 * s + 1.f, r12 * s,
              r20 * s, r21 * s, r22 * s + 1.f);
}
// btMatrix3x3::getRotation (SSE path)
RSB_HD Quat quatFromM3(const M3& m) {
    float trace = m.r[0].x + m.r[1].y + m.r[2].z;
    float t[4];
    float x;
    if (trace > 0.f) {
        x = trace + 1.f;
        t[0] = m.r[2].y - m.r[1].z;
        t[1] = m.r[0].z - m.r[2].x;
        t[2] = m.r[1].x - m.r[0].y;
        t[3] = x;
    } else {
        int i, j, k;
        if (m.r[0].x < m.r[1].y) {
            if (m.r[1].y < m.r[2].z) { i = 2; j = 0; k = 1; }
            else { i = 1; j = 2; k = 0; }
        } else {
            if (m.r[0].x < m.r[2].z) { i = 2; j = 0; k = 1; }
            else { i = 0; j = 1; k = 2; }
        }
        x = m.r[i][i] - m.r[j][j] - m.r[k][k] + 1.f;
        t[3] = m.r[k][j] - m.r[j][k];
        t[j] = m.r[j][i] + m.r[i][j];
        t[k] = m.r[k][i] + m.r[i][k];
        t[i] = x;
    }
    float s = fsqrt(x);
    s = 0.5f / s;
    return Quat{t[0] * s, t[1] * s, t[2] * s, t[3] * s};
}

// btMatrix3x3::setEulerZYX(eulerX, eulerY, eulerZ)
RSB_HD M3 m3fromEulerZYX(float ex, float ey, float ez) {
    float ci = rsCosf(ex), cj = rsCosf(ey), ch = rsCosf(ez);
    float si = rsSinf(ex), sj = rsSinf(ey), sh = rsSinf(ez);
    float cc = ci * ch, cs = ci * sh, sc = si * ch, ss = si * sh;
    return m3(cj * ch, sj * sc - cs, sj * cc + ss,
              cj * sh, sj * ss + cc, sj * cs - sc,
              -sj, cj * si, cj * ci);
}

// ------------------------------------------------------------------ Transform
struct Xf {
    M3 b;
    V3 o;
};
RSB_HD Xf xfIdentity() { return Xf{m3identity(), v3zero()}; }
RSB_HD V3 xfPoint(const Xf& t, V3 p) { return (t.b * p) + t.o; }
RSB_HD V3 xfInvPoint(const Xf& t, V3 p) { V3 v = p - t.o; return transpose(t.b) * v; }
RSB_HD Xf xfMul(const Xf& a, const Xf& c) { return Xf{a.b * c.b, xfPoint(a, c.o)}; }
RSB_HD Xf xfInverse(const Xf& t) { M3 inv = transpose(t.b); return Xf{inv, inv * (-t.o)}; }
// this^-1 * t
RSB_HD Xf xfInverseTimes(const Xf& a, const Xf& t) {
    V3 v = t.o - a.o;
    return Xf{transposeTimes(a.b, t.b), tmul(v, a.b)};
}

// btPlaneSpace1
RSB_HD void planeSpace1(V3 n, V3& p, V3& q) {
    if (fabsf(n.z) > kSqrt12) {
        float a = n.y * n.y + n.z * n.z;
        float k = 1.f / fsqrt(a);
        p = V3{0.f, -n.z * k, n.y * k};
        q = V3{a * k, -n.x * p.z, n.x * p.y};
    } else {
        float a = n.x * n.x + n.y * n.y;
        float k = 1.f / fsqrt(a);
        p = V3{-n.y * k, n.x * k, 0.f};
        q = V3{-n.z * p.y, n.z * p.x, a * k};
    }
}

// btTransformAabb(localAabbMin, localAabbMax, margin, trans, ...)
RSB_HD void transformAabb(V3 lmin, V3 lmax, float margin, const Xf& t, V3& omin, V3& omax) {
    V3 he = (lmax - lmin) * 0.5f;
    he = he + V3{margin, margin, margin};
    V3 lc = (lmax + lmin) * 0.5f;
    M3 ab = mabs(t.b);
    V3 c = xfPoint(t, lc);
    V3 e = V3{dot(ab.r[0], he), dot(ab.r[1], he), dot(ab.r[2], he)};
    omin = c - e;
    omax = c + e;
}
// btTransformAabb(halfExtents, margin, trans, ...)
RSB_HD void transformAabbHalf(V3 halfExtents, float margin, const Xf& t, V3& omin, V3& omax) {
    V3 he = halfExtents + V3{margin, margin, margin};
    M3 ab = mabs(t.b);
    V3 e = V3{dot(ab.r[0], he), dot(ab.r[1], he), dot(ab.r[2], he)};
    omin = t.o - e;
    omax = t.o + e;
}
// TestAabbAgainstAabb2
RSB_HD bool aabbOverlap(V3 mn1, V3 mx1, V3 mn2, V3 mx2) {
    bool overlap = true;
    overlap = (mn1.x > mx2.x || mx1.x < mn2.x) ? false : overlap;
    overlap = (mn1.z > mx2.z || mx1.z < mn2.z) ? false : overlap;
    overlap = (mn1.y > mx2.y || mx1.y < mn2.y) ? false : overlap;
    return overlap;
}
// TestTriangleAgainstAabb2
RSB_HD bool triAabbOverlap(const V3* v, V3 mn, V3 mx) {
    if (fmin_(fmin_(v[0].x, v[1].x), v[2].x) > mx.x) return false;
    if (fmax_(fmax_(v[0].x, v[1].x), v[2].x) < mn.x) return false;
    if (fmin_(fmin_(v[0].z, v[1].z), v[2].z) > mx.z) return false;
    if (fmax_(fmax_(v[0].z, v[1].z), v[2].z) < mn.z) return false;
    if (fmin_(fmin_(v[0].y, v[1].y), v[2].y) > mx.y) return false;
    if (fmax_(fmax_(v[0].y, v[1].y), v[2].y) < mn.y) return false;
    return true;
}

// btTransformUtil::integrateTransform (exponential map) and its no-rotation variant
constexpr float kAngularMotionThreshold = 0.5f * kHalfPi;
RSB_HD Xf integrateTransform(const Xf& cur, V3 linvel, V3 angvel, float dt) {
    Xf out;
    out.o = cur.o + linvel * dt;
    float a2 = length2(angvel);
    float ang = 0.f;
    if (a2 > kEpsilon) ang = fsqrt(a2);
    if (ang * dt > kAngularMotionThreshold) ang = kAngularMotionThreshold / dt;
    V3 axis;
    if (ang < 0.001f) {
        axis = angvel * (0.5f * dt - (dt * dt * dt) * (0.020833333333f) * ang * ang);
    } else {
        axis = angvel * (rsSinf(0.5f * ang * dt) / ang);
    }
    Quat dorn = Quat{axis.x, axis.y, axis.z, rsCosf(ang * dt * 0.5f)};
    Quat orn0 = quatFromM3(cur.b);
    Quat pred = qmul(dorn, orn0);
    pred = qsafeNormalized(pred);
    if (qlength2(pred) > kEpsilon) out.b = m3fromQuat(pred);
    else out.b = cur.b;
    return out;
}
RSB_HD Xf integrateTransformNoRot(const Xf& cur, V3 linvel, float dt) {
    return Xf{cur.b, cur.o + linvel * dt};
}

}  // namespace rsb
