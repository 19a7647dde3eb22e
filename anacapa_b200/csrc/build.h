// Device build of a scene's triangle sections (build.cu).
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

#include <string>

#include "../../include/anacapa_b200.h"
#include "layout.h"

namespace ana {

// The triangle sections of one scene built on the device: 4-wide nodes,
// leaf-ordered intersection records and mesh-ordered shading records, the
// same bytes prepare_scene's host path produces for them.
struct DeviceTris {
    Bvh4Node* nodes = nullptr;  // num_nodes
    float4* isect = nullptr;    // 3 per triangle, leaf order
    float4* shade = nullptr;    // 4 per triangle, mesh order
    uint32_t num_nodes = 0, num_tris = 0;
    float ms[4] = {0.f, 0.f, 0.f, 0.f};  // setup, SAH levels, small subtrees, collapse
    uint32_t levels = 0;
    DeviceTris() = default;
    DeviceTris(const DeviceTris&) = delete;
    DeviceTris& operator=(const DeviceTris&) = delete;
    ~DeviceTris();
};

// BVHBackend::commit's triangle setup, its binned SAH build and the 4-wide
// collapse, run on the current device on stream `s` for the meshes of `d`
// (num_meshes > 0 and at least one triangle). Returns ANA_OK, or an error
// code with a message: invalid meshes, a device failure, a tree deeper than
// the traversal stack.
int build_tris_on_device(const ana_scene_desc& d, uint32_t maxLeaf, cudaStream_t s, DeviceTris& out,
                         std::string& err);

}  // namespace ana
