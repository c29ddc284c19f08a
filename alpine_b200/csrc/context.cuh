// The context behind the C ABI: device memory, streams, scene state.
#pragma once

#include "../../include/alpine_gpu.h"
#include "build.cuh"

#include <string>
#include <vector>

namespace ag {

// A growable device buffer.
struct DeviceBuffer {
    void* ptr = nullptr;
    size_t bytes = 0;
    ~DeviceBuffer() { release(); }
    void release()
    {
        if (ptr) cudaFree(ptr);
        ptr = nullptr;
        bytes = 0;
    }
    // Returns false when the allocation fails. Contents are not preserved.
    bool reserve(size_t n)
    {
        if (n <= bytes && ptr) return true;
        release();
        size_t want = n < 256 ? 256 : n;
        if (cudaMalloc(&ptr, want) != cudaSuccess) {
            cudaGetLastError();
            ptr = nullptr;
            return false;
        }
        bytes = want;
        return true;
    }
    template <typename T>
    T* as() const { return static_cast<T*>(ptr); }
};

constexpr int kCopyStreams = 4;

}  // namespace ag

struct alpine_gpu_ctx {
    int device = 0;
    alpine_gpu_config cfg{};
    cudaStream_t stream = nullptr;
    cudaStream_t copyStreams[ag::kCopyStreams] = {};
    std::string error;

    // scene geometry (host mirror + device copy)
    std::vector<float> verts;       // 3 per vertex, all meshes
    std::vector<uint32_t> idx;      // 3 per triangle, global vertex indices
    std::vector<uint32_t> shapeVertBase, shapeVertCount, shapeTriBase, shapeTriCount;
    bool geometryDirty = true;      // device vertex/index copy out of date
    bool bvhDirty = true;           // BVH out of date w.r.t. geometry
    ag::DeviceBuffer dVerts, dIdx;

    // acceleration structure
    ag::Builder builder;
    ag::DeviceBuffer dNodes, dTris;
    uint32_t nodeCount = 0, triCount = 0;
    alpine_gpu_bvh_stats stats{};

    // device status word (DeviceError bits) and its pinned host mirror
    uint32_t* dStatus = nullptr;
    uint32_t* hStatus = nullptr;

    // staging for host-memory queries
    ag::DeviceBuffer dRays, dOut;

    int fail(int code, const std::string& msg)
    {
        error = msg;
        return code;
    }
};
