// Convex shapes that meet in the narrowphase: the car's hitbox box, a mesh triangle and
// the ball sphere, with the support and bounding-box queries Bullet's algorithms call.
//
//   supportNoMargin ... btConvexShape::localGetSupportVertexWithoutMarginNonVirtual
//                       (btConvexShape.cpp:287-360)
//   supportMarginN .... btConvexShape::localGetSupportVertexNonVirtual (.cpp:362-375):
//                       direction normalised, then the margin added along it
//   supportVirtual .... the virtual localGetSupportingVertex of each shape:
//                       btBoxShape.h:58-68 (margin added per axis, no normalisation),
//                       btSphereShape.cpp:33-49, btConvexInternalShape.cpp:47-70 (triangle)
//   shapeAabb ......... btBoxShape::getAabb (btTransformAabb), btSphereShape::getAabb,
//                       btTriangleShape::getAabb -> getAabbSlow (btConvexInternalShape.cpp:74-92)
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
#include "vecmath.h"

namespace rsb {

enum : int32_t { SH_BOX = 0, SH_TRI = 1, SH_SPHERE = 2 };

struct ConvexShape {
    int32_t type;
    float margin;  // box: collision margin; sphere: radius; triangle: mesh margin (0)
    V3 he;         // box: implicit half extents (half extents without the margin)
    V3 v[3];       // triangle vertices in the shape's local frame
};

RSB_HD ConvexShape makeBox(V3 implicitHalfExtents, float margin) {
    ConvexShape s;
    s.type = SH_BOX;
    s.margin = margin;
    s.he = implicitHalfExtents;
    s.v[0] = s.v[1] = s.v[2] = v3zero();
    return s;
}
RSB_HD ConvexShape makeSphere(float radius) {
    ConvexShape s;
    s.type = SH_SPHERE;
    s.margin = radius;
    s.he = v3zero();
    s.v[0] = s.v[1] = s.v[2] = v3zero();
    return s;
}
RSB_HD ConvexShape makeTri(const V3* v, float margin) {
    ConvexShape s;
    s.type = SH_TRI;
    s.margin = margin;
    s.he = v3zero();
    s.v[0] = v[0];
    s.v[1] = v[1];
    s.v[2] = v[2];
    return s;
}

// btFsels(a, b, c): a >= 0 ? b : c
RSB_HD float fsels(float a, float b, float c) { return a >= 0.f ? b : c; }

RSB_HD V3 triSupport(const ConvexShape& s, V3 dir) {
    V3 dots = V3{dot(dir, s.v[0]), dot(dir, s.v[1]), dot(dir, s.v[2])};
    return s.v[maxAxis(dots)];
}

RSB_HD V3 supportNoMargin(const ConvexShape& s, V3 dir) {
    if (s.type == SH_BOX) return V3{fsels(dir.x, s.he.x, -s.he.x), fsels(dir.y, s.he.y, -s.he.y), fsels(dir.z, s.he.z, -s.he.z)};
    if (s.type == SH_TRI) return triSupport(s, dir);
    return v3zero();
}

RSB_HD V3 dirNormalized(V3 d) {
    if (length2(d) < kEpsilon * kEpsilon) d = V3{-1.f, -1.f, -1.f};
    return normalized(d);
}

RSB_HD V3 supportMarginN(const ConvexShape& s, V3 dir) {
    V3 n = dirNormalized(dir);
    return supportNoMargin(s, n) + n * s.margin;
}

RSB_HD V3 supportVirtual(const ConvexShape& s, V3 dir) {
    if (s.type == SH_BOX) {
        V3 h = s.he + V3{s.margin, s.margin, s.margin};
        return V3{fsels(dir.x, h.x, -h.x), fsels(dir.y, h.y, -h.y), fsels(dir.z, h.z, -h.z)};
    }
    if (s.type == SH_SPHERE) {
        V3 n = dirNormalized(dir);
        return v3zero() + n * s.margin;
    }
    V3 sv = triSupport(s, dir);
    if (s.margin != 0.f) sv = sv + dirNormalized(dir) * s.margin;
    return sv;
}

RSB_HD void shapeAabb(const ConvexShape& s, const Xf& t, V3& mn, V3& mx) {
    if (s.type == SH_BOX) {
        transformAabbHalf(s.he, s.margin, t, mn, mx);
    } else if (s.type == SH_SPHERE) {
        float m = s.margin + 0.08f;  // RocketSim widens sphere AABBs (btSphereShape.cpp:52-59)
        V3 e{m, m, m};
        mn = t.o - e;
        mx = t.o + e;
    } else {
        for (int i = 0; i < 3; i++) {
            V3 vec = v3zero();
            vec[i] = 1.f;
            V3 sv = supportVirtual(s, tmul(vec, t.b));
            V3 tmp = xfPoint(t, sv);
            mx[i] = tmp[i] + s.margin;
            vec[i] = -1.f;
            tmp = xfPoint(t, supportVirtual(s, tmul(vec, t.b)));
            mn[i] = tmp[i] - s.margin;
        }
    }
}

}  // namespace rsb
