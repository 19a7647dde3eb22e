// Host-side scene preparation: validates an ana_scene_desc, builds the BVHs
// and flattens everything into the device layout of layout.h.
#pragma once
#include <stdint.h>

#include <string>
#include <vector>

#include "../../include/anacapa_b200.h"
#include "layout.h"

namespace ana {

struct HostEnv {
    std::vector<float> rgb, cond_func, cond_cdf, cond_int, marg_func, marg_cdf;
    float marg_int = 0.f;
    float intensity = 1.f;
    uint32_t width = 0, height = 0;
    float radiance[3] = {0.f, 0.f, 0.f};
    bool present = false;
};

struct Prepared {
    std::vector<Bvh4Node> tri_nodes;
    std::vector<float4> tri_isect;   // 3 per triangle, leaf order
    std::vector<float4> tri_shade;   // 4 per triangle, mesh order
    bool tri_root_is_empty = true;
    std::vector<Bvh4Node> seg_nodes;
    std::vector<float4> segs;        // 5 per segment, leaf order
    std::vector<float> strand_color;
    std::vector<DevMaterial> materials;
    std::vector<int32_t> slot_material;
    std::vector<DevLight> lights;
    HostEnv env;
    ana_camera camera{};
    uint32_t num_tris = 0, num_segs = 0;
    bool has_emitters = false;
    bool has_transmit = false;  // a slot's material has a non-black shadow tint
    // Triangle sections built on the device (build_tris_on_device): tri_nodes,
    // tri_isect and tri_shade stay empty, num_tris is set and the node count
    // is filled in once the device build has run.
    bool tris_on_device = false;
    uint32_t dev_tri_nodes = 0;
    // motion meshes: (first key, key count) per motion mesh, 5 float4 per key
    std::vector<uint2> mesh_motion;
    std::vector<float4> motion_keys;
    uint64_t bytes() const;
};

// The roughness-derived fields of a standard_surface material (rough, metal,
// spec and transmission set): GGX alpha2 of sample/evaluate, the unclamped
// alpha2 of the transmission lobe, flags() and isDelta()
// (StandardSurface.h:152-181, 384).
void derive_standard(DevMaterial& m);

// One ana_material in the device layout with its derived constants; returns
// nullptr, or the reason it is rejected.
const char* make_material(const ana_material& m, DevMaterial& o);

// Returns ANA_OK or an error code with a message in err. With
// tris_on_device the triangle sections are left to the device build (the
// mesh offsets are still validated here).
int prepare_scene(const ana_scene_desc& d, Prepared& out, std::string& err, bool tris_on_device = false);

// Camera::makePinhole (include/anacapa/integrator/IIntegrator.h:49-74) for a film size.
DevCamera make_camera(const ana_camera& c, uint32_t width, uint32_t height);

}  // namespace ana
