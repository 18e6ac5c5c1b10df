// Static soccar arena data: triangle meshes with their quantized BVHs, per-triangle
// internal-edge information and the broadphase static-cell table.  Built once on the host (arena_build.cpp) and read by the
// kernels from device memory; the whole set is ~0.5 MB and stays L2-resident.
//
// Layouts restate the structures RocketSim builds at init time:
//   - BvhNode / BvhSubtree: btQuantizedBvhNode / btBvhSubtreeInfo (btQuantizedBvh.h),
//     16-byte nodes, stackless escape-index order, subtree headers in build order.
//   - TriEdgeInfo: btTriangleInfo (btTriangleInfoMap.h) for triangles that have one.
//   - bp cells: which static objects btRSBroadphase registered in each cell.
#pragma once
#include "vecmath.h"

namespace rsb {

constexpr int MAX_MESHES = 16;
constexpr int NUM_PLANES = 4;
constexpr int NUM_STATICS = MAX_MESHES + NUM_PLANES;  // collision objects 0..19

struct BvhNode {
    uint16_t qmin[3];
    uint16_t qmax[3];
    int32_t data;  // >= 0: leaf triangle index; < 0: internal node, escape = -data
};

struct BvhSubtree {
    uint16_t qmin[3];
    uint16_t qmax[3];
    int32_t root;
    int32_t size;
};

// btTriangleInfo flags (btTriangleInfoMap.h)
enum : int32_t {
    TRI_INFO_V0V1_CONVEX = 1,
    TRI_INFO_V1V2_CONVEX = 2,
    TRI_INFO_V2V0_CONVEX = 4,
    TRI_INFO_V0V1_SWAP_NORMALB = 8,
    TRI_INFO_V1V2_SWAP_NORMALB = 16,
    TRI_INFO_V2V0_SWAP_NORMALB = 32,
    TRI_INFO_PRESENT = 1 << 30
};

struct TriEdgeInfo {
    float a01, a12, a20;  // m_edgeV0V1Angle, m_edgeV1V2Angle, m_edgeV2V0Angle
    int32_t flags;
};

struct MeshDesc {
    int32_t nodeOff, nodeCount;
    int32_t subOff, subCount;
    int32_t triOff, triCount;
    V3 bvhMin, bvhMax, quant;  // quantization frame (btQuantizedBvh m_bvhAabbMin/Max/Quantization)
    V3 bpMin, bpMax;           // broadphase AABB (shape AABB +- gContactBreakingThreshold)
    V3 shapeMin, shapeMax;     // btTriangleMeshShape::getAabb at the identity transform
};

// btRSBroadphase grid (Arena.cpp:459-471 with ArenaConfig defaults)
struct BpGrid {
    V3 minPos;
    float cellSize;
    int cellsX, cellsY, cellsZ;
};

struct ArenaStatic {
    const BvhNode* nodes;
    const BvhSubtree* subs;
    const V3* triVerts;        // 3 per triangle, Bullet units
    const TriEdgeInfo* triInfo;
    const uint32_t* bpCells;   // bit s set: static object s registered in the cell
    // Mesh occupancy grid (Bullet units): bit m of voxel v set when some triangle of mesh
    // m may pass through the voxel (the triangle's AABB overlaps the voxel and its plane
    // crosses it, both tested with a tolerance).  A mesh with no bit in the voxels of a
    // region holds no triangle there, so its queries confined to the region cannot find
    // anything and are skipped.
    const uint16_t* occ;
    // Per voxel (CSR: voxOff[v] .. voxOff[v + 1] into voxList), the mesh triangles marked in
    // it as voxKey(mesh, BVH leaf node, triangle), sorted: the order the meshes' BVH walks
    // visit them.
    const uint32_t* voxOff;
    const uint32_t* voxList;
    // Per voxel, a lower bound (uu, rounded down) on the distance from any point of the voxel
    // to any mesh triangle: the distance between its centre and the nearest voxel with a mesh
    // bit, less the voxel diagonal (64 * sqrt(3) uu).
    const uint16_t* occDist;
    V3 occMin;
    float occInvCell;
    int occX, occY, occZ;
    MeshDesc meshes[MAX_MESHES];
    int32_t numMeshes;
    BpGrid bp;
    // static planes: normal and world origin (Arena.cpp:1060-1100), broadphase AABB
    V3 planeNormal[NUM_PLANES];
    V3 planeOrigin[NUM_PLANES];
    V3 planeBpMin[NUM_PLANES], planeBpMax[NUM_PLANES];
    V3 planeShapeMin[NUM_PLANES], planeShapeMax[NUM_PLANES];  // btStaticPlaneShape::getAabb
};

RSB_HD uint32_t voxKey(int mesh, int leaf, int tri) {
    return ((uint32_t)mesh << 22) | ((uint32_t)leaf << 10) | (uint32_t)tri;
}

// The meshes that may have a triangle in a voxel overlapped by the box [mn, mx] (boxes
// reaching outside the grid get every mesh).
RSB_HD uint32_t occMask(const ArenaStatic& S, V3 mn, V3 mx) {
    const float f = S.occInvCell;
    int x0 = (int)floorf((mn.x - S.occMin.x) * f), x1 = (int)floorf((mx.x - S.occMin.x) * f);
    int y0 = (int)floorf((mn.y - S.occMin.y) * f), y1 = (int)floorf((mx.y - S.occMin.y) * f);
    int z0 = (int)floorf((mn.z - S.occMin.z) * f), z1 = (int)floorf((mx.z - S.occMin.z) * f);
    if (!(x0 >= 0 && y0 >= 0 && z0 >= 0 && x1 < S.occX && y1 < S.occY && z1 < S.occZ)) return 0xffffffffu;
    uint32_t m = 0;
    for (int x = x0; x <= x1; x++)
        for (int y = y0; y <= y1; y++)
            for (int z = z0; z <= z1; z++) m |= S.occ[(x * S.occY + y) * S.occZ + z];
    return m;
}

// ------------------------------------------------------------ BVH queries (device)

RSB_HD void bvhQuantize(const MeshDesc& m, V3 p, int isMax, uint16_t* out) {
    V3 v = (p - m.bvhMin) * m.quant;
    if (isMax) {
        out[0] = (uint16_t)(((uint16_t)(v.x + 1.f)) | 1);
        out[1] = (uint16_t)(((uint16_t)(v.y + 1.f)) | 1);
        out[2] = (uint16_t)(((uint16_t)(v.z + 1.f)) | 1);
    } else {
        out[0] = (uint16_t)(((uint16_t)(v.x)) & 0xfffe);
        out[1] = (uint16_t)(((uint16_t)(v.y)) & 0xfffe);
        out[2] = (uint16_t)(((uint16_t)(v.z)) & 0xfffe);
    }
}
RSB_HD void bvhQuantizeClamp(const MeshDesc& m, V3 p, int isMax, uint16_t* out) {
    V3 c = vmax(p, m.bvhMin);
    c = vmin(c, m.bvhMax);
    bvhQuantize(m, c, isMax, out);
}
RSB_HD V3 bvhUnquantize(const MeshDesc& m, const uint16_t* q) {
    V3 v = V3{(float)q[0] / m.quant.x, (float)q[1] / m.quant.y, (float)q[2] / m.quant.z};
    return v + m.bvhMin;
}
RSB_HD bool qOverlap(const uint16_t* mn1, const uint16_t* mx1, const uint16_t* mn2, const uint16_t* mx2) {
    return (mn1[0] <= mx2[0]) & (mx1[0] >= mn2[0]) & (mn1[2] <= mx2[2]) & (mx1[2] >= mn2[2]) &
           (mn1[1] <= mx2[1]) & (mx1[1] >= mn2[1]);
}

// btQuantizedBvh::reportAabbOverlappingNodex -> walkStacklessQuantizedTreeCacheFriendly:
// visits the leaves whose quantized box overlaps the query, subtree by subtree, in the
// reference's order.  fn(triIndex) returns false to stop early.
template <class F>
RSB_HD void bvhQueryAabb(const ArenaStatic& S, int mesh, V3 aabbMin, V3 aabbMax, F&& fn) {
    const MeshDesc& m = S.meshes[mesh];
    uint16_t qmn[3], qmx[3];
    bvhQuantizeClamp(m, aabbMin, 0, qmn);
    bvhQuantizeClamp(m, aabbMax, 1, qmx);
    for (int s = 0; s < m.subCount; s++) {
        const BvhSubtree& st = S.subs[m.subOff + s];
        if (!qOverlap(qmn, qmx, st.qmin, st.qmax)) continue;
        int cur = st.root, end = st.root + st.size;
        while (cur < end) {
            const BvhNode& n = S.nodes[m.nodeOff + cur];
            bool ov = qOverlap(qmn, qmx, n.qmin, n.qmax);
            bool leaf = n.data >= 0;
            if (leaf && ov) {
                if (!fn(n.data)) return;
            }
            if (ov || leaf) cur++;
            else cur += -n.data;
        }
    }
}

// btRayAabb2 (btAabbUtil2.h)
RSB_HD bool rayAabb2(V3 src, V3 invDir, const unsigned* sign, const V3* bounds, float& tmin, float lmin, float lmax) {
    float txmin = (bounds[sign[0]].x - src.x) * invDir.x;
    float txmax = (bounds[1 - sign[0]].x - src.x) * invDir.x;
    float tymin = (bounds[sign[1]].y - src.y) * invDir.y;
    float tymax = (bounds[1 - sign[1]].y - src.y) * invDir.y;
    if ((txmin > tymax) || (tymin > txmax)) return false;
    if (tymin > txmin) txmin = tymin;
    if (tymax < txmax) txmax = tymax;
    float tzmin = (bounds[sign[2]].z - src.z) * invDir.z;
    float tzmax = (bounds[1 - sign[2]].z - src.z) * invDir.z;
    if ((txmin > tzmax) || (tzmin > txmax)) return false;
    if (tzmin > txmin) txmin = tzmin;
    if (tzmax < txmax) txmax = tzmax;
    tmin = txmin;
    return ((txmin < lmax) && (txmax > lmin));
}

// btQuantizedBvh::walkStacklessQuantizedTreeAgainstRay over the whole tree (no box extents)
template <class F>
RSB_HD void bvhQueryRay(const ArenaStatic& S, int mesh, V3 src, V3 dst, F&& fn) {
    const MeshDesc& m = S.meshes[mesh];
    V3 rayDir = safeNormalized(dst - src);
    float lambdaMax = dot(rayDir, dst - src);
    V3 inv;
    inv.x = rayDir.x == 0.f ? kLargeFloat : 1.f / rayDir.x;
    inv.y = rayDir.y == 0.f ? kLargeFloat : 1.f / rayDir.y;
    inv.z = rayDir.z == 0.f ? kLargeFloat : 1.f / rayDir.z;
    unsigned sign[3] = {inv.x < 0.f, inv.y < 0.f, inv.z < 0.f};
    V3 rmn = vmin(src, dst), rmx = vmax(src, dst);
    uint16_t qmn[3], qmx[3];
    bvhQuantizeClamp(m, rmn, 0, qmn);
    bvhQuantizeClamp(m, rmx, 1, qmx);
    int cur = 0, end = m.nodeCount;
    while (cur < end) {
        const BvhNode& n = S.nodes[m.nodeOff + cur];
        float param = 1.f;
        bool rayOv = false;
        bool leaf = n.data >= 0;
        if (qOverlap(qmn, qmx, n.qmin, n.qmax)) {
            V3 bounds[2];
            bounds[0] = bvhUnquantize(m, n.qmin);
            bounds[1] = bvhUnquantize(m, n.qmax);
            rayOv = rayAabb2(src, inv, sign, bounds, param, 0.f, lambdaMax);
        }
        if (leaf && rayOv) {
            if (!fn(n.data)) return;
        }
        if (rayOv || leaf) cur++;
        else cur += -n.data;
    }
}

RSB_HD void triVerts(const ArenaStatic& S, int mesh, int tri, V3* v) {
    const V3* p = S.triVerts + 3 * (S.meshes[mesh].triOff + tri);
    v[0] = p[0];
    v[1] = p[1];
    v[2] = p[2];
}

}  // namespace rsb
