// Host-side construction of the static soccar arena data (see phys/arena_static.h).
#pragma once
#include <string>
#include <vector>

#include "phys/arena_static.h"

namespace rsb {

struct ArenaStaticHost {
    std::vector<BvhNode> nodes;
    std::vector<BvhSubtree> subs;
    std::vector<V3> triVerts;
    std::vector<TriEdgeInfo> triInfo;
    std::vector<uint32_t> bpCells;
    std::vector<uint16_t> occ;
    std::vector<uint32_t> voxOff, voxList;
    std::vector<uint16_t> occDist;
    ArenaStatic view;  // pointers into the vectors above (host addresses)
    std::string error;
};

// Loads mesh_0.cmf .. mesh_<n-1>.cmf from <folder>/soccar in numeric order and builds
// every structure.  Returns false (with `error` set) when the folder holds no meshes or
// a file is malformed.
bool buildArenaStatic(const std::string& folder, ArenaStaticHost& out);

// Re-points out.view at a device copy whose buffers are given.
ArenaStatic deviceView(const ArenaStaticHost& h, const BvhNode* nodes, const BvhSubtree* subs,
                       const V3* triVerts, const TriEdgeInfo* triInfo, const uint32_t* bpCells,
                       const uint16_t* occ, const uint32_t* voxOff, const uint32_t* voxList,
                       const uint16_t* occDist);

}  // namespace rsb
