// GPU BVH builder: binned SAH (32 bins) binary build, then a collapse
// (SAH-optimal by default, or the reference's greedy rule) to the 8-wide
// quantised layout of bvh.cuh. Replaces the reference's CPU build
// (src/accelerators/bvh_common.cpp:185-391 binned SAH with 9 bins and
// src/accelerators/wide_bvh.cpp:200-243 collapse + 290-356 flatten).
#pragma once

#include "bvh.cuh"

#include <vector>

namespace ag {

struct BuildStats {
    uint32_t binaryNodes = 0;
    uint32_t binaryLevels = 0;
    uint32_t wideNodes = 0;
    uint32_t wideDepth = 0;
    uint32_t triCount = 0;
    float sahCost = 0.0f;  // SAH cost of the wide tree (node + triangle tests per unit root area)
    float buildMs = 0.0f;  // device time of the whole build
    uint32_t childSlots = 0;  // filled slots over all wide nodes
    uint32_t bigLevels = 0;   // leading binary levels with tasks above kSmallMax references
};

// Which binary nodes fill the slots of a wide node.
constexpr uint32_t kCollapseSah = 0;     // SAH-optimal (dynamic program over the binary tree)
constexpr uint32_t kCollapseGreedy = 1;  // largest-area child first (src/accelerators/wide_bvh.cpp:200-243)
constexpr float kCollapseTriCost = 1.0f;  // default SAH cost of a triangle test per wide-node visit

// Device buffers owned by a builder; grown on demand and reused across builds.
class Builder {
public:
    Builder() = default;
    ~Builder();
    Builder(const Builder&) = delete;
    Builder& operator=(const Builder&) = delete;

    // verts: float[3 * nverts] (device), idx: uint32[3 * ntris] (device),
    // spheres: float4[nspheres] centre + radius (device, may be null when 0).
    // Primitives are the triangles, then the spheres. Outputs: nodes
    // (capacity >= ntris + nspheres + 1), tris (ntris + nspheres records).
    // Returns 0 on success, a negative code on failure (message in err).
    int build(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres, uint32_t nspheres,
              WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t stream, BuildStats* stats,
              char* err, size_t errLen);

    // Device-driven build: the same tree as build(), bit for bit, with every
    // count kept in device memory, so that nothing waits on the host and the
    // sequence of launches is fixed. It runs maxLevels binary levels and
    // maxWideLevels collapse levels (a level past the tree's depth costs a
    // few short launches), captured in a CUDA graph on the first call and
    // replayed until the arguments change or a build() records new per-level
    // counts (they size the grids and pick the levels that run the big-task
    // kernels). Needs buffers for ntris + nspheres primitives (a build() of
    // at least that size first). A tree deeper than the binary cap, or a big
    // task below the big-task levels, leaves the previous tree in place; one
    // deeper than the wide cap leaves it partly rewritten; all three set
    // kErrBuildDepth in deviceStatus. Returns 0, or a negative code with a
    // message in err.
    int enqueue(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres, uint32_t nspheres,
                WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t stream, uint32_t maxLevels,
                uint32_t maxWideLevels, char* err, size_t errLen);
    // Statistics of the last enqueue(), read from device memory (synchronous).
    int enqueued_stats(cudaStream_t stream, BuildStats* stats, char* err, size_t errLen);
    uint32_t graph_captures() const { return graphCaptures_; }
    uint32_t graph_launches() const { return graphLaunches_; }

    // Collapse rule and the SAH cost of a triangle test relative to a
    // wide-node visit (used by kCollapseSah); applied at the next build.
    void set_collapse(uint32_t rule, float triCost)
    {
        collapse_ = rule;
        triCost_ = triCost;
    }
    uint32_t collapse() const { return collapse_; }
    float triangle_cost() const { return triCost_; }

private:
    int reserve(uint32_t ntris, char* err, size_t errLen);
    void release();
    void enqueue_launches(const float* verts, const uint32_t* idx, uint32_t ntris, const float4* spheres, uint32_t n,
                          WideNode* nodes, TriRecord* tris, uint32_t* deviceStatus, cudaStream_t stream,
                          uint32_t maxLevels, uint32_t maxWideLevels);

    uint32_t cap_ = 0;
    uint32_t collapse_ = kCollapseSah;
    float triCost_ = kCollapseTriCost;
    void* mem_ = nullptr;  // one allocation carved into the arrays below
    size_t memBytes_ = 0;
    float4* primLo_ = nullptr;
    float4* primHi_ = nullptr;
    uint32_t* refs_[2] = {nullptr, nullptr};
    uint32_t* order_ = nullptr;
    BinNode* bnodes_ = nullptr;
    void* tasks_[2] = {nullptr, nullptr};
    void* cands_ = nullptr;
    uint32_t* candFlag_ = nullptr;
    uint32_t* candPos_ = nullptr;
    uint32_t* bigFlag_ = nullptr;
    uint32_t* bigPos_ = nullptr;
    uint32_t* bigList_ = nullptr;
    uint32_t* bigChunks_ = nullptr;
    uint32_t* chunkOffSparse_ = nullptr;
    uint32_t* chunkOff_ = nullptr;
    uint32_t* chunkTask_ = nullptr;
    uint32_t* chunkLeft_ = nullptr;
    uint32_t* chunkLeftOff_ = nullptr;
    uint32_t* bigBins_ = nullptr;
    void* bigSplit_ = nullptr;
    uint32_t* items_[2] = {nullptr, nullptr};
    uint32_t* slots_ = nullptr;
    std::vector<uint32_t> levelStart_;   // first binary node id of each level (host)
    float* collapseCost_ = nullptr;      // 8 per binary node (k_collapse_cost)
    uint32_t* collapseChoice_ = nullptr; // 1 per binary node
    uint32_t* intCount_ = nullptr;
    uint32_t* intOff_ = nullptr;
    uint32_t* triCount_ = nullptr;
    uint32_t* triOff_ = nullptr;
    uint32_t* counters_ = nullptr;  // small device scalars
    uint32_t* hostCounters_ = nullptr;  // pinned mirror
    uint32_t* scanScratch_ = nullptr;
    float* sahAccum_ = nullptr;
    cudaEvent_t ev0_ = nullptr, ev1_ = nullptr;
    uint32_t* levelStartDev_ = nullptr;  // first binary node id of each level (device-driven build)
    uint32_t bigLevels_ = 0;             // leading binary levels with big tasks in the last build()
    struct LevelCounts {
        uint32_t tasks, big, chunks;
    };
    std::vector<LevelCounts> levelCounts_;  // per binary level of the last build(): sizes enqueue()'s grids
    std::vector<uint32_t> wideCounts_;      // wide nodes per collapse level of the last build()
    uint64_t buildGeneration_ = 0;          // build() calls so far (part of the graph key)
    cudaGraphExec_t graphExec_ = nullptr;  // the captured device-driven build
    std::vector<uint64_t> graphKey_;
    uint32_t graphCaptures_ = 0, graphLaunches_ = 0;
};

}  // namespace ag
