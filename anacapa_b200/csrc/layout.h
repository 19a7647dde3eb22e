// Device-resident scene layout shared by the host preparation code and the
// sm_100a kernels. Plain POD, no CUDA runtime calls.
//
// HBM layout (all arrays 16-byte aligned, read with 16-byte vector loads):
//   tri_nodes   4-wide BVH nodes, 128 B each (Bvh4Node): the four children's
//               boxes live in the parent so one node fetch tests four boxes.
//   tri_isect   48 B per triangle in leaf order: (v0, orig index) (e1) (e2),
//               i.e. BVHTriangle::v0/e1/e2 (src/accel/BVHBackend.h:49-59).
//   tri_shade   64 B per triangle in mesh order: (ng, meshID) (sn0, primID)
//               (sn1) (sn2), read once per shaded hit.
//   seg_nodes   4-wide BVH nodes over cubic Bezier segments (same 128 B format).
//   segs        80 B per segment in leaf order: P0..P3 with the two half
//               widths and the strand-parameter offset/scale, then ids.
#pragma once
#include <stdint.h>
#include <vector_types.h>

namespace ana {

// 4-wide BVH node (128 bytes, one L2 line): the four children's
// boxes as structure of arrays (child k in component k) and their references
// (an interior node index, a leaf entry: bit 31 | (count-1) << 25 | first
// triangle, or kEmptyChild). The nodes are the reference's binary SAH tree
// collapsed: every child box is a box of that tree, bit for bit.
struct Bvh4Node {
    float4 lox, hix, loy, hiy, loz, hiz;
    uint4 ref;
    uint4 pad;
};
static_assert(sizeof(Bvh4Node) == 128, "Bvh4Node must be 128 bytes");
constexpr uint32_t kEmptyChild = 0xFFFFFFFFu;
// Triangle traversal stack: a 4-wide step pushes up to three entries, so the
// build bounds the worst root-to-leaf sum of pushes by this (prepare_scene
// rejects a deeper tree).
constexpr uint32_t kMaxStack4 = 128;

// Material, flattened with the derived constants each reference class
// precomputes in its constructor.
struct DevMaterial {
    uint32_t type;       // ANA_MAT_*
    uint32_t flags;      // BSDFFlags of IMaterial::flags()
    uint32_t is_delta;   // IMaterial::isDelta()
    uint32_t hair_mode;
    float3 albedo;       // Lambert albedo / standard base_color
    float3 emission;     // Le (Emissive) or emission_color * emission (standard)
    // standard_surface
    float base, metal, rough, spec;
    float3 spec_color;
    float coat;
    float alpha2;        // max(1e-4, r^2)^2
    float coat_alpha2;
    float f0_dielectric; // F0_fromIOR(specular_IOR)
    float coat_f0;       // F0_fromIOR(1.5)
    // hair
    float eta;
    float3 sigma_a;
    float v[3];          // longitudinal variances R, TT, TRT
    float s;             // azimuthal logistic scale
    float alpha_shift[3];// lobe shift angles (radians)
    float beta_m;
    // standard_surface glass and alpha (StandardSurface.h:197-218, 245-414)
    float transmission;  // Params::transmission
    float ior;           // Params::specular_IOR (eta of the glass lobes)
    float alpha2_t;      // (r^2)^2 unclamped: evaluate()'s transmission lobe
    float opacity;       // evalOpacity: opacity when alphaMask, else 1
    float3 tint;         // transmittanceColor (black: opaque to shadow rays)
    float pad0;
};

struct DevLight {
    uint32_t type;       // ANA_LIGHT_*
    uint32_t pad[3];
    float3 center, u, v, normal, Le;
    float area;
    float uLen2, vLen2;  // |u|^2, |v|^2 as AreaLight::pdf computes them
    float cos_cone;      // directional: cos of the angular radius (normal = direction to it)
};

// Equirect dome with its 2-D piecewise-constant distribution
// (Distribution1D per row + marginal, src/shading/lights/DomeLight.h:146-182, 355-386).
struct DevEnv {
    const float* rgb;        // W*H*3, row 0 = zenith
    const float* cond_func;  // H rows of W
    const float* cond_cdf;   // H rows of W+1
    const float* cond_int;   // H
    const float* marg_func;  // H
    const float* marg_cdf;   // H+1
    float marg_int;
    float intensity;
    uint32_t width, height;
    float3 radiance;         // constant background when rgb == nullptr
    uint32_t present;        // 1 if a dome exists
};

struct DevCamera {
    float3 origin, lower_left, horizontal, vertical, basis_u, basis_v;
    float aperture, focal_distance, shutter_open, shutter_close;
    uint32_t width, height;
};

// Per-scene record of a batch (a plain render is a batch of one). Global
// arrays hold every scene's data; a scene's BVH roots and its slot / light
// ranges index into them.
constexpr uint32_t kNoRoot = 0xFFFFFFFFu;

struct DevSceneRec {
    uint32_t tri_root, seg_root;     // interior root node, or kNoRoot
    uint32_t slot_base, num_slots;   // SceneView::materials of this scene
    uint32_t light_base, num_lights; // SceneView::lights of this scene
    uint32_t spp, sample_start;
    uint32_t max_depth, min_depth;
    uint32_t film_offset;            // first pixel of this scene's film in the batch film
    uint32_t path_offset;            // first global path id of this scene
    uint64_t seed;                   // HaltonSampler seed
    float3 env_radiance;             // SceneView::envRadiance (no dome)
    uint32_t has_dome;
    DevCamera cam;                   // includes the film size
    // The item's pixels: a rect_w-wide rectangle at (rect_x0, rect_y0) of a
    // film_w-wide film (a TileRequest; a whole frame is the full rectangle).
    uint32_t rect_x0, rect_y0, rect_w, film_w;
    // ceil(2^64 / spp) and ceil(2^64 / rect_w), 0 for a divisor of 1: the
    // kernels divide path and pixel indices by multiply-high
    uint64_t spp_div, rect_w_div;
};

// Material and light classes present in an uploaded scene (DevScene::features).
// Shading kernels are also compiled for subsets of them, so a batch that
// lacks a class runs a kernel without its code.
constexpr uint32_t kFeatLambert = 1;   // Lambertian and emissive materials
constexpr uint32_t kFeatStandard = 2;  // standard_surface
constexpr uint32_t kFeatArea = 4;      // area lights
constexpr uint32_t kFeatDome = 8;      // dome lights
constexpr uint32_t kFeatDir = 16;      // directional lights
constexpr uint32_t kFeatAll = 31;

struct DevScene {
    const Bvh4Node* tri_nodes;
    const float4* tri_isect;
    const float4* tri_shade;
    const Bvh4Node* seg_nodes;  // the curve segments' 4-wide BVH
    const float4* segs;
    const float* strand_color;   // 3 per strand
    const DevMaterial* materials;
    const int32_t* slot_material;
    const DevLight* lights;
    const DevSceneRec* scenes;
    const uint32_t* scene_path_offset;  // num_scenes + 1 (global path id ranges)
    uint32_t num_scenes;
    uint32_t has_curves;    // any scene has curve segments
    uint32_t has_emitters;  // any material reachable from a slot emits (Le != 0)
    uint32_t has_fibers;    // curve segments or hair materials: shading needs the fiber code
    uint32_t has_transmit;  // a material passes shadow rays (non-black transmittanceColor):
                            // shadow and MIS rays step through surfaces
    // Motion blur: an object-space triangle has bit 31 set in its tri_isect
    // index word and its motion mesh in the e1 record's w; mesh_motion[m] =
    // (first key, key count), each key 5 float4 in motion_keys: (time, -, -,
    // -) and the object-to-world rows.
    const uint2* mesh_motion;
    const float4* motion_keys;
    uint32_t has_motion;
    uint32_t has_extra_shading;  // glass, alpha masks or motion: the shading kernel with their code
    uint32_t features;           // kFeat* bits of the materials and lights present
    DevEnv env;             // the (single) dome of the batch
};

}  // namespace ana
