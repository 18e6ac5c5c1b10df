// Host construction of the static soccar arena (meshes, BVHs, edge info, grids).
//
// Each step restates what RocketSim does at RocketSim::Init / Arena construction, so
// that the device traversals visit triangles and statics in the reference's order:
//   CMF parsing ............ CollisionMeshFile.cpp:11-73 (int32 tri/vert counts, then
//                            int32[3] triangles, then float[3] vertices, Bullet units)
//   mesh local AABB ........ btTriangleMeshShape::recalcLocalAabb (support vertices)
//   quantized BVH .......... btOptimizedBvh::build + btQuantizedBvh::buildTree /
//                            sortAndCalcSplittingIndex / calcSplittingAxis /
//                            updateSubtreeHeaders (btQuantizedBvh.cpp:76-305)
//   internal edge info ..... btGenerateInternalEdgeInfo (btInternalEdgeUtility.cpp:40-330)
//   broadphase static cells  btRSBroadphase::_UpdateCellsStatic (btRSBroadphase.cpp:93-170)
//   static planes .......... Arena::_SetupArenaCollisionShapes (Arena.cpp:1055-1120) and
//                            btStaticPlaneShape::getAabb (btStaticPlaneShape.cpp:40-54)
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
#include "arena_build.h"
#include "phys/consts.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <fstream>
#include <map>

namespace rsb {

namespace {

struct MeshBuild {
    std::vector<int32_t> idx;   // 3 per triangle
    std::vector<V3> verts;
    V3 localMin, localMax;
    MeshDesc desc;
    std::vector<BvhNode> leaves;     // quantized leaf nodes during the build
    std::vector<BvhNode> nodes;      // contiguous nodes
    std::vector<BvhSubtree> subs;
    int curNode = 0;
};

bool readFile(const std::string& path, std::vector<char>& data) {
    std::ifstream f(path, std::ios::binary);
    if (!f) return false;
    data.assign(std::istreambuf_iterator<char>(f), std::istreambuf_iterator<char>());
    return true;
}

bool parseCmf(const std::vector<char>& d, MeshBuild& m, std::string& err) {
    if (d.size() < 8) { err = "truncated mesh file"; return false; }
    int32_t nt, nv;
    std::memcpy(&nt, d.data(), 4);
    std::memcpy(&nv, d.data() + 4, 4);
    const int32_t kMax = 1000 * 1000;
    if (nt <= 0 || nv <= 0 || nt > kMax || nv > kMax) { err = "bad triangle/vertex count"; return false; }
    size_t need = 8 + (size_t)nt * 12 + (size_t)nv * 12;
    if (d.size() < need) { err = "mesh file shorter than its counts"; return false; }
    m.idx.resize((size_t)nt * 3);
    std::memcpy(m.idx.data(), d.data() + 8, (size_t)nt * 12);
    m.verts.resize(nv);
    const char* vp = d.data() + 8 + (size_t)nt * 12;
    for (int i = 0; i < nv; i++) {
        float f[3];
        std::memcpy(f, vp + (size_t)i * 12, 12);
        m.verts[i] = V3{f[0], f[1], f[2]};
    }
    for (int32_t v : m.idx)
        if (v < 0 || v >= nv) { err = "bad triangle vertex index"; return false; }
    return true;
}

V3 triV(const MeshBuild& m, int t, int j) { return m.verts[m.idx[3 * t + j]]; }

// btTriangleMeshShape::recalcLocalAabb via localGetSupportingVertex (margin 0)
void computeLocalAabb(MeshBuild& m) {
    int nt = (int)m.idx.size() / 3;
    for (int axis = 0; axis < 3; axis++) {
        for (int sgn = 0; sgn < 2; sgn++) {
            V3 dir = v3zero();
            dir[axis] = sgn == 0 ? 1.f : -1.f;
            float maxDot = -kLargeFloat;
            V3 sup = v3zero();
            for (int t = 0; t < nt; t++)
                for (int j = 0; j < 3; j++) {
                    V3 p = triV(m, t, j);
                    float d = dot(dir, p);
                    if (d > maxDot) { maxDot = d; sup = p; }
                }
            if (sgn == 0) m.localMax[axis] = sup[axis] + 0.f;
            else m.localMin[axis] = sup[axis] - 0.f;
        }
    }
}

// btQuantizedBvh::setQuantizationValues (margin 1.0)
void setQuantization(MeshDesc& d, V3 bmin, V3 bmax) {
    V3 clampValue{1.f, 1.f, 1.f};
    d.bvhMin = bmin - clampValue;
    d.bvhMax = bmax + clampValue;
    V3 size = d.bvhMax - d.bvhMin;
    V3 k{65533.f, 65533.f, 65533.f};
    d.quant = V3{k.x / size.x, k.y / size.y, k.z / size.z};
    uint16_t q[3];
    bvhQuantize(d, d.bvhMin, 0, q);
    V3 v = bvhUnquantize(d, q);
    d.bvhMin = vmin(d.bvhMin, v - clampValue);
    size = d.bvhMax - d.bvhMin;
    d.quant = V3{k.x / size.x, k.y / size.y, k.z / size.z};
    bvhQuantize(d, d.bvhMax, 1, q);
    v = bvhUnquantize(d, q);
    d.bvhMax = vmax(d.bvhMax, v + clampValue);
    size = d.bvhMax - d.bvhMin;
    d.quant = V3{k.x / size.x, k.y / size.y, k.z / size.z};
}

V3 leafMin(const MeshBuild& m, int i) { return bvhUnquantize(m.desc, m.leaves[i].qmin); }
V3 leafMax(const MeshBuild& m, int i) { return bvhUnquantize(m.desc, m.leaves[i].qmax); }

int calcSplittingAxis(const MeshBuild& m, int s, int e) {
    V3 means = v3zero(), var = v3zero();
    int n = e - s;
    for (int i = s; i < e; i++) means += (leafMax(m, i) + leafMin(m, i)) * 0.5f;
    means *= (1.f / (float)n);
    for (int i = s; i < e; i++) {
        V3 c = (leafMax(m, i) + leafMin(m, i)) * 0.5f;
        V3 d2 = c - means;
        d2 = d2 * d2;
        var += d2;
    }
    var *= (1.f / ((float)n - 1));
    return maxAxis(var);
}

int sortAndSplit(MeshBuild& m, int s, int e, int axis) {
    int split = s, n = e - s;
    V3 means = v3zero();
    for (int i = s; i < e; i++) means += (leafMax(m, i) + leafMin(m, i)) * 0.5f;
    means *= (1.f / (float)n);
    float splitValue = means[axis];
    for (int i = s; i < e; i++) {
        V3 c = (leafMax(m, i) + leafMin(m, i)) * 0.5f;
        if (c[axis] > splitValue) {
            std::swap(m.leaves[i], m.leaves[split]);
            split++;
        }
    }
    int balanced = n / 3;
    bool unbalanced = (split <= (s + balanced)) || (split >= (e - 1 - balanced));
    if (unbalanced) split = s + (n >> 1);
    return split;
}

bool isLeaf(const BvhNode& n) { return n.data >= 0; }
int escapeOf(const BvhNode& n) { return -n.data; }

void addSubtree(MeshBuild& m, int nodeIndex, int size) {
    BvhSubtree st;
    std::memcpy(st.qmin, m.nodes[nodeIndex].qmin, sizeof(st.qmin));
    std::memcpy(st.qmax, m.nodes[nodeIndex].qmax, sizeof(st.qmax));
    st.root = nodeIndex;
    st.size = size;
    m.subs.push_back(st);
}

void buildTree(MeshBuild& m, int s, int e) {
    const int kMaxSubtreeBytes = 2048, kNodeBytes = 16;
    int n = e - s;
    int curIndex = m.curNode;
    if (n == 1) {
        m.nodes[m.curNode] = m.leaves[s];
        m.curNode++;
        return;
    }
    int axis = calcSplittingAxis(m, s, e);
    int split = sortAndSplit(m, s, e, axis);
    int internal = m.curNode;
    bvhQuantize(m.desc, m.desc.bvhMax, 0, m.nodes[internal].qmin);
    bvhQuantize(m.desc, m.desc.bvhMin, 1, m.nodes[internal].qmax);
    for (int i = s; i < e; i++) {
        uint16_t qmn[3], qmx[3];
        bvhQuantize(m.desc, leafMin(m, i), 0, qmn);
        bvhQuantize(m.desc, leafMax(m, i), 1, qmx);
        for (int a = 0; a < 3; a++) {
            if (m.nodes[internal].qmin[a] > qmn[a]) m.nodes[internal].qmin[a] = qmn[a];
            if (m.nodes[internal].qmax[a] < qmx[a]) m.nodes[internal].qmax[a] = qmx[a];
        }
    }
    m.curNode++;
    int left = m.curNode;
    buildTree(m, s, split);
    int right = m.curNode;
    buildTree(m, split, e);
    int escape = m.curNode - curIndex;
    if (escape * kNodeBytes > kMaxSubtreeBytes) {
        const BvhNode& ln = m.nodes[left];
        int lsize = isLeaf(ln) ? 1 : escapeOf(ln);
        const BvhNode& rn = m.nodes[right];
        int rsize = isLeaf(rn) ? 1 : escapeOf(rn);
        if (lsize * kNodeBytes <= kMaxSubtreeBytes) addSubtree(m, left, lsize);
        if (rsize * kNodeBytes <= kMaxSubtreeBytes) addSubtree(m, right, rsize);
    }
    m.nodes[internal].data = -escape;
}

void buildBvh(MeshBuild& m) {
    int nt = (int)m.idx.size() / 3;
    setQuantization(m.desc, m.localMin, m.localMax);
    m.leaves.resize(nt);
    for (int t = 0; t < nt; t++) {
        V3 mn{kLargeFloat, kLargeFloat, kLargeFloat}, mx{-kLargeFloat, -kLargeFloat, -kLargeFloat};
        for (int j = 0; j < 3; j++) {
            mn = vmin(mn, triV(m, t, j));
            mx = vmax(mx, triV(m, t, j));
        }
        const float kMinDim = 0.002f, kMinHalf = 0.001f;
        for (int a = 0; a < 3; a++) {
            if (mx[a] - mn[a] < kMinDim) {
                mx[a] = mx[a] + kMinHalf;
                mn[a] = mn[a] - kMinHalf;
            }
        }
        bvhQuantize(m.desc, mn, 0, m.leaves[t].qmin);
        bvhQuantize(m.desc, mx, 1, m.leaves[t].qmax);
        m.leaves[t].data = t;
    }
    m.nodes.assign(2 * nt, BvhNode{});
    m.curNode = 0;
    buildTree(m, 0, nt);
    if (m.subs.empty()) addSubtree(m, 0, isLeaf(m.nodes[0]) ? 1 : escapeOf(m.nodes[0]));
    m.nodes.resize(m.curNode);
}

}  // namespace

// Squared Euclidean distance (in voxels) from every voxel centre to the nearest centre of a
// voxel with a mesh bit: three one-dimensional passes, each the lower envelope of parabolas
// (Felzenszwalb and Huttenlocher, "Distance Transforms of Sampled Functions", 2012).
static void edt1d(const double* f, int n, double* d, std::vector<int>& v, std::vector<double>& z) {
    const double inf = 1e20;
    int k = 0;
    v[0] = 0;
    z[0] = -inf;
    z[1] = inf;
    for (int q = 1; q < n; q++) {
        double s;
        while (true) {
            s = ((f[q] + (double)q * q) - (f[v[k]] + (double)v[k] * v[k])) / (2.0 * (q - v[k]));
            if (s <= z[k] && k > 0) k--;
            else break;
        }
        if (s <= z[k]) {  // k == 0: the new parabola replaces the first
            v[0] = q;
            z[0] = -inf;
            z[1] = inf;
            continue;
        }
        k++;
        v[k] = q;
        z[k] = s;
        z[k + 1] = inf;
    }
    k = 0;
    for (int q = 0; q < n; q++) {
        while (z[k + 1] < (double)q) k++;
        const double dq = (double)(q - v[k]);
        d[q] = dq * dq + f[v[k]];
    }
}

static void occupiedDistance2(const std::vector<uint16_t>& occ, int X, int Y, int Z, std::vector<double>& out) {
    const double inf = 1e20;
    const size_t nv = (size_t)X * Y * Z;
    out.assign(nv, inf);
    for (size_t v = 0; v < nv; v++)
        if (occ[v]) out[v] = 0.0;
    const int nmax = std::max(X, std::max(Y, Z));
    std::vector<double> f(nmax), d(nmax), z(nmax + 1);
    std::vector<int> vv(nmax);
    auto at = [&](int x, int y, int zz) -> double& { return out[((size_t)x * Y + y) * Z + zz]; };
    for (int x = 0; x < X; x++)  // along z
        for (int y = 0; y < Y; y++) {
            for (int q = 0; q < Z; q++) f[q] = at(x, y, q);
            edt1d(f.data(), Z, d.data(), vv, z);
            for (int q = 0; q < Z; q++) at(x, y, q) = d[q];
        }
    for (int x = 0; x < X; x++)  // along y
        for (int zz = 0; zz < Z; zz++) {
            for (int q = 0; q < Y; q++) f[q] = at(x, q, zz);
            edt1d(f.data(), Y, d.data(), vv, z);
            for (int q = 0; q < Y; q++) at(x, q, zz) = d[q];
        }
    for (int y = 0; y < Y; y++)  // along x
        for (int zz = 0; zz < Z; zz++) {
            for (int q = 0; q < X; q++) f[q] = at(q, y, zz);
            edt1d(f.data(), X, d.data(), vv, z);
            for (int q = 0; q < X; q++) at(q, y, zz) = d[q];
        }
}

bool buildArenaStatic(const std::string& folder, ArenaStaticHost& out) {
    std::vector<MeshBuild> meshes;
    for (int i = 0; i < MAX_MESHES; i++) {
        std::string path = folder + "/soccar/mesh_" + std::to_string(i) + ".cmf";
        std::vector<char> data;
        if (!readFile(path, data)) break;
        MeshBuild m;
        std::string err;
        if (!parseCmf(data, m, err)) {
            out.error = path + ": " + err;
            return false;
        }
        meshes.push_back(std::move(m));
    }
    if (meshes.empty()) {
        out.error = "no soccar/mesh_<i>.cmf files under " + folder;
        return false;
    }

    // ---- meshes, BVHs, flat arrays
    ArenaStatic& S = out.view;
    std::memset(&S, 0, sizeof(S));
    S.numMeshes = (int)meshes.size();
    for (size_t mi = 0; mi < meshes.size(); mi++) {
        MeshBuild& m = meshes[mi];
        computeLocalAabb(m);
        buildBvh(m);
        MeshDesc& d = m.desc;
        d.nodeOff = (int)out.nodes.size();
        d.nodeCount = (int)m.nodes.size();
        d.subOff = (int)out.subs.size();
        d.subCount = (int)m.subs.size();
        d.triOff = (int)out.triVerts.size() / 3;
        d.triCount = (int)m.idx.size() / 3;
        out.nodes.insert(out.nodes.end(), m.nodes.begin(), m.nodes.end());
        out.subs.insert(out.subs.end(), m.subs.begin(), m.subs.end());
        for (int t = 0; t < d.triCount; t++)
            for (int j = 0; j < 3; j++) out.triVerts.push_back(triV(m, t, j));
        // broadphase AABB: btTriangleMeshShape::getAabb(identity) +- 0.02
        Xf id = xfIdentity();
        V3 mn, mx;
        transformAabb(m.localMin, m.localMax, 0.f, id, mn, mx);
        d.shapeMin = mn;
        d.shapeMax = mx;
        V3 thr{0.02f, 0.02f, 0.02f};
        d.bpMin = mn - thr;
        d.bpMax = mx + thr;
        S.meshes[mi] = d;
    }
    out.triInfo.assign(out.triVerts.size() / 3, TriEdgeInfo{kTwoPi, kTwoPi, kTwoPi, 0});

    // temporary host view for the BVH queries below
    S.nodes = out.nodes.data();
    S.subs = out.subs.data();
    S.triVerts = out.triVerts.data();

    // ---- internal edge info (btGenerateInternalEdgeInfo)
    const float kEqualVertex = 0.0001f * 0.0001f, kPlanarEps = 0.0001f;
    for (int mi = 0; mi < S.numMeshes; mi++) {
        const MeshDesc& d = S.meshes[mi];
        for (int ta = 0; ta < d.triCount; ta++) {
            V3 A[3];
            triVerts(S, mi, ta, A);
            V3 amn{kLargeFloat, kLargeFloat, kLargeFloat}, amx{-kLargeFloat, -kLargeFloat, -kLargeFloat};
            for (int j = 0; j < 3; j++) { amn = vmin(amn, A[j]); amx = vmax(amx, A[j]); }
            bvhQueryAabb(S, mi, amn, amx, [&](int tb) {
                if (tb == ta) return true;
                V3 B[3];
                triVerts(S, mi, tb, B);
                if (length2(cross(B[1] - B[0], B[2] - B[0])) < kEqualVertex) return true;
                if (length2(cross(A[1] - A[0], A[2] - A[0])) < kEqualVertex) return true;
                int sa[3] = {-1, -1, -1}, sb[3] = {-1, -1, -1}, ns = 0;
                for (int i = 0; i < 3; i++) {
                    for (int j = 0; j < 3; j++) {
                        if (length2(A[i] - B[j]) < kEqualVertex) {
                            sa[ns] = i;
                            sb[ns] = j;
                            ns++;
                            if (ns >= 3) return true;
                        }
                    }
                    if (ns >= 3) return true;
                }
                if (ns != 2) return true;
                if (sa[0] == 0 && sa[1] == 2) {
                    sa[0] = 2; sa[1] = 0;
                    int tmp = sb[1]; sb[1] = sb[0]; sb[0] = tmp;
                }
                TriEdgeInfo& info = out.triInfo[d.triOff + ta];
                info.flags |= TRI_INFO_PRESENT;
                int sumA = sa[0] + sa[1];
                int otherA = 3 - sumA;
                V3 edge = A[sa[1]] - A[sa[0]];
                int otherB = 3 - (sb[0] + sb[1]);
                V3 tB[3] = {B[sb[1]], B[sb[0]], B[otherB]};
                V3 nA = normalized(cross(A[1] - A[0], A[2] - A[0]));
                V3 nB = normalized(cross(tB[1] - tB[0], tB[2] - tB[0]));
                edge = normalized(edge);
                V3 ecA = normalized(cross(edge, nA));
                if (dot(ecA, A[otherA] - A[sa[0]]) < 0) ecA *= -1.f;
                V3 ecB = normalized(cross(edge, nB));
                if (dot(ecB, B[otherB] - B[sb[0]]) < 0) ecB *= -1.f;
                V3 calcEdge = cross(ecA, ecB);
                float len2 = length2(calcEdge);
                float corrected = 0.f;
                bool isConvex = false;
                if (!(len2 < kPlanarEps)) {
                    calcEdge = normalized(calcEdge);
                    V3 calcNA = normalized(cross(calcEdge, ecA));
                    float angle2 = atan2f(dot(ecB, calcNA), dot(ecB, ecA));
                    float ang4 = kPi - angle2;
                    isConvex = dot(nA, ecB) < 0.f;
                    corrected = isConvex ? ang4 : -ang4;
                }
                V3 e2;
                int swapFlag, convexFlag;
                float* slot;
                switch (sumA) {
                    case 1: e2 = A[0] - A[1]; swapFlag = TRI_INFO_V0V1_SWAP_NORMALB; convexFlag = TRI_INFO_V0V1_CONVEX; slot = &info.a01; break;
                    case 2: e2 = A[2] - A[0]; swapFlag = TRI_INFO_V2V0_SWAP_NORMALB; convexFlag = TRI_INFO_V2V0_CONVEX; slot = &info.a20; break;
                    default: e2 = A[1] - A[2]; swapFlag = TRI_INFO_V1V2_SWAP_NORMALB; convexFlag = TRI_INFO_V1V2_CONVEX; slot = &info.a12; break;
                }
                Quat orn = qaxisAngle(e2, -corrected);
                V3 cnB = quatRotate(orn, nA);
                if (dot(cnB, nB) < 0) info.flags |= swapFlag;
                *slot = -corrected;
                if (isConvex) info.flags |= convexFlag;
                return true;
            });
        }
    }

    // ---- static planes: floor, ceiling, -x wall, +x wall
    {
        const V3 normals[4] = {{0, 0, 1}, {0, 0, -1}, {1, 0, 0}, {-1, 0, 0}};
        const V3 origins[4] = {V3{0, 0, 0}, V3{0, 0, ARENA_HEIGHT} * kUuToBt,
                               V3{-ARENA_EXTENT_X, 0, ARENA_HEIGHT / 2} * kUuToBt,
                               V3{ARENA_EXTENT_X, 0, ARENA_HEIGHT / 2} * kUuToBt};
        for (int p = 0; p < NUM_PLANES; p++) {
            V3 n = normalized(normals[p]);
            S.planeNormal[p] = n;
            S.planeOrigin[p] = origins[p];
            V3 mn{-kLargeFloat, -kLargeFloat, -kLargeFloat}, mx{kLargeFloat, kLargeFloat, kLargeFloat};
            int axis = n.x != 0.f ? 0 : (n.y != 0.f ? 1 : 2);
            const float kOff = 0.2f;
            float c = 0.f;  // plane constant
            mn[axis] = origins[p][axis] + (c - kOff);
            mx[axis] = origins[p][axis] + (c + kOff);
            if (n[axis] < 0) mx[axis] = kLargeFloat;
            else mn[axis] = -kLargeFloat;
            S.planeShapeMin[p] = mn;
            S.planeShapeMax[p] = mx;
            V3 thr{0.02f, 0.02f, 0.02f};
            S.planeBpMin[p] = mn - thr;
            S.planeBpMax[p] = mx + thr;
        }
    }

    // ---- broadphase static cells (btRSBroadphase, ArenaConfig defaults)
    {
        BpGrid& g = S.bp;
        V3 minPos = V3{-4500, -6000, 0} * kUuToBt, maxPos = V3{4500, 6000, 2500} * kUuToBt;
        g.minPos = minPos;
        g.cellSize = 370.f * kUuToBt * 1.f;
        V3 range = maxPos - minPos;
        g.cellsX = imax_(1, (int)std::ceil(range.x / g.cellSize));
        g.cellsY = imax_(1, (int)std::ceil(range.y / g.cellSize));
        g.cellsZ = imax_(1, (int)std::ceil(range.z / g.cellSize));
        out.bpCells.assign((size_t)g.cellsX * g.cellsY * g.cellsZ, 0u);
        auto cellIdx3 = [&](V3 pos, int& i, int& j, int& k) {
            V3 f = bdiv(pos - g.minPos, g.cellSize);
            // float -> int of out-of-range values behaves as x86 cvttss2si (INT_MIN)
            auto toInt = [](float x) -> int {
                if (!(x > -2147483648.f && x < 2147483648.f)) return INT32_MIN;
                return (int)x;
            };
            i = imin_(imax_(toInt(f.x), 0), g.cellsX - 1);
            j = imin_(imax_(toInt(f.y), 0), g.cellsY - 1);
            k = imin_(imax_(toInt(f.z), 0), g.cellsZ - 1);
        };
        for (int s = 0; s < NUM_STATICS; s++) {
            bool isMesh = s < MAX_MESHES;
            if (isMesh && s >= S.numMeshes) continue;
            V3 amin = isMesh ? S.meshes[s].bpMin : S.planeBpMin[s - MAX_MESHES];
            V3 amax = isMesh ? S.meshes[s].bpMax : S.planeBpMax[s - MAX_MESHES];
            amax = V3{fmin_(amax.x, maxPos.x), fmin_(amax.y, maxPos.y), fmin_(amax.z, maxPos.z)};
            int i0, j0, k0, i1, j1, k1;
            cellIdx3(amin, i0, j0, k0);
            cellIdx3(amax, i1, j1, k1);
            for (int i = i0; i <= i1; i++)
                for (int j = j0; j <= j1; j++)
                    for (int k = k0; k <= k1; k++) {
                        if (isMesh) {
                            V3 cmn = g.minPos + V3{(float)i, (float)j, (float)k} * g.cellSize;
                            V3 cmx = cmn + V3{g.cellSize, g.cellSize, g.cellSize};
                            bool hit = false;
                            bvhQueryAabb(S, s, cmn, cmx, [&](int) { hit = true; return false; });
                            if (!hit) continue;
                        }
                        for (int a = -1; a <= 1; a++)
                            for (int b = -1; b <= 1; b++)
                                for (int c = -1; c <= 1; c++) {
                                    int ci = i + a, cj = j + b, ck = k + c;
                                    if (ci < 0 || cj < 0 || ck < 0) continue;
                                    if (ci >= g.cellsX || cj >= g.cellsY || ck >= g.cellsZ) continue;
                                    out.bpCells[(size_t)ci * g.cellsY * g.cellsZ + (size_t)cj * g.cellsZ + ck] |= 1u << s;
                                }
                    }
        }
    }

    S.triInfo = out.triInfo.data();
    S.bpCells = out.bpCells.data();

    // ---- mesh occupancy grid (see ArenaStatic::occ): 64 uu voxels over the arena, a mesh bit each
    {
        const float cell = 64.f * kUuToBt, tol = 2.f * kUuToBt;
        const V3 gmn = V3{-4400.f, -6300.f, -200.f} * kUuToBt, gmx = V3{4400.f, 6300.f, 2300.f} * kUuToBt;
        S.occMin = gmn;
        S.occInvCell = 1.f / cell;
        S.occX = (int)std::ceil((gmx.x - gmn.x) / cell);
        S.occY = (int)std::ceil((gmx.y - gmn.y) / cell);
        S.occZ = (int)std::ceil((gmx.z - gmn.z) / cell);
        const size_t nv = (size_t)S.occX * S.occY * S.occZ;
        out.occ.assign(nv, 0);
        const float halfDiag = 0.5f * cell * std::sqrt(3.f);
        const size_t ntri = out.triVerts.size() / 3;
        std::vector<int> meshOf(ntri, 0);
        for (int m = 0; m < S.numMeshes; m++)
            for (int t = 0; t < S.meshes[m].triCount; t++) meshOf[S.meshes[m].triOff + t] = m;
        // the BVH leaf (node index within its mesh) of every triangle; the voxel keys hold
        // 12 bits of leaf index and 10 bits of triangle index
        for (int m = 0; m < S.numMeshes; m++)
            if (S.meshes[m].nodeCount > 4096 || S.meshes[m].triCount > 1024) {
                out.error = "mesh too large for the voxel triangle lists";
                return false;
            }
        std::vector<int> leafOf(ntri, -1);
        for (int m = 0; m < S.numMeshes; m++)
            for (int k = 0; k < S.meshes[m].nodeCount; k++) {
                const BvhNode& nd = out.nodes[(size_t)S.meshes[m].nodeOff + k];
                if (nd.data >= 0) leafOf[(size_t)S.meshes[m].triOff + nd.data] = k;
            }
        std::vector<std::pair<uint32_t, uint32_t>> lists;  // (voxel, key)
        for (size_t t = 0; t < ntri; t++) {
            const V3 a = out.triVerts[3 * t], b = out.triVerts[3 * t + 1], c = out.triVerts[3 * t + 2];
            const V3 mn = vmin(vmin(a, b), c) - V3{tol, tol, tol}, mx = vmax(vmax(a, b), c) + V3{tol, tol, tol};
            V3 n = cross(b - a, c - a);
            const float nl = std::sqrt(dot(n, n));
            const bool flat = nl > 0.f;
            if (flat) n = n * (1.f / nl);
            auto idx = [&](float v, float o, int hi) {
                int i = (int)std::floor((v - o) / cell);
                return i < 0 ? 0 : (i >= hi ? hi - 1 : i);
            };
            for (int x = idx(mn.x, gmn.x, S.occX); x <= idx(mx.x, gmn.x, S.occX); x++)
                for (int y = idx(mn.y, gmn.y, S.occY); y <= idx(mx.y, gmn.y, S.occY); y++)
                    for (int z = idx(mn.z, gmn.z, S.occZ); z <= idx(mx.z, gmn.z, S.occZ); z++) {
                        const V3 centre = gmn + V3{(x + 0.5f) * cell, (y + 0.5f) * cell, (z + 0.5f) * cell};
                        // the triangle's plane must come within the voxel's half diagonal
                        if (flat && std::fabs(dot(n, centre - a)) > halfDiag + tol) continue;
                        const size_t v = ((size_t)x * S.occY + y) * S.occZ + z;
                        out.occ[v] |= (uint16_t)(1u << meshOf[t]);
                        const int m = meshOf[t], lt = (int)t - S.meshes[m].triOff;
                        lists.emplace_back((uint32_t)v, voxKey(m, leafOf[t], lt));
                    }
        }
        S.occ = out.occ.data();
        // per-voxel triangle lists, each sorted by (mesh, BVH leaf): the order in which the
        // meshes' BVH walks would report them
        std::sort(lists.begin(), lists.end());
        out.voxOff.assign(nv + 1, 0u);
        out.voxList.resize(lists.size());
        for (size_t i = 0; i < lists.size(); i++) {
            out.voxOff[lists[i].first + 1]++;
            out.voxList[i] = lists[i].second;
        }
        for (size_t v = 0; v < nv; v++) out.voxOff[v + 1] += out.voxOff[v];
        S.voxOff = out.voxOff.data();
        S.voxList = out.voxList.data();
        // distance bound of every voxel (see ArenaStatic::occDist)
        std::vector<double> d2;
        occupiedDistance2(out.occ, S.occX, S.occY, S.occZ, d2);
        out.occDist.resize(nv);
        const float cellUu = 64.f;
        for (size_t v = 0; v < nv; v++) {
            const double d = (std::sqrt(d2[v]) - std::sqrt(3.0)) * cellUu;
            out.occDist[v] = (uint16_t)std::min(65535.0, std::max(0.0, std::floor(d)));
        }
        S.occDist = out.occDist.data();
    }
    return true;
}

ArenaStatic deviceView(const ArenaStaticHost& h, const BvhNode* nodes, const BvhSubtree* subs,
                       const V3* triVerts, const TriEdgeInfo* triInfo, const uint32_t* bpCells,
                       const uint16_t* occ, const uint32_t* voxOff, const uint32_t* voxList,
                       const uint16_t* occDist) {
    ArenaStatic v = h.view;
    v.occ = occ;
    v.occDist = occDist;
    v.voxOff = voxOff;
    v.voxList = voxList;
    v.nodes = nodes;
    v.subs = subs;
    v.triVerts = triVerts;
    v.triInfo = triInfo;
    v.bpCells = bpCells;
    return v;
}

}  // namespace rsb
