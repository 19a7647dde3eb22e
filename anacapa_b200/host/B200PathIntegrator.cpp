// B200PathIntegrator: SceneView -> ana_scene_desc flattening and the
// renderFrame bridge (see B200PathIntegrator.h).
#include "B200PathIntegrator.h"

#include <anacapa/accel/CurvePool.h>
#include <anacapa/accel/GeometryPool.h>
#include <anacapa/accel/IAccelerationStructure.h>
#include <anacapa/shading/ILight.h>
#include <anacapa/shading/IMaterial.h>
#include <anacapa/shading/ShadingContext.h>

#include <cmath>
#include <cstring>
#include <stdexcept>
#include <unordered_map>
#include <vector>

#include "accel/CurveBrute.h"
#include "shading/Lambertian.h"
#include "shading/MarschnerHair.h"
#include "shading/StandardSurface.h"
#include "shading/lights/AreaLight.h"
#include "shading/lights/DirectionalLight.h"
#include "shading/lights/DomeLight.h"

namespace anacapa_b200 {

using namespace anacapa;

namespace {

void put3(float* o, Vec3f v) {
    o[0] = v.x;
    o[1] = v.y;
    o[2] = v.z;
}

// A shading context at a flat, front-facing surface point with a white strand
// colour: the probe used to read constant reflectances and emissions.
ShadingContext probe_ctx() {
    SurfaceInteraction si;
    si.p = {};
    si.n = {0.f, 0.f, 1.f};
    si.ng = si.n;
    si.color = {1.f, 1.f, 1.f};
    return ShadingContext(si, Vec3f{0.f, 0.f, -1.f});
}

// AreaLight keeps its quad private; sampleLe places uPos on it at
// center + uAxis (2 uPos.x - 1) + vAxis (2 uPos.y - 1) (AreaLight.h:81-105).
// uPos = (0.5, 0.5) returns the centre exactly, but centre + axis - centre is
// not the axis once rounded, and light samples then land an ulp away from the
// reference's. Instead uPos.x = 2^(k-1) with k >= 25 makes 2 uPos.x - 1 round to
// 2^k, so the position is uAxis 2^k (exact) plus a centre far below half an ulp
// of it, i.e. exactly uAxis 2^k; scaling back by 2^-k gives uAxis bit for bit. A
// component is accepted when two values of k agree; a zero component never
// agrees (it leaves the centre's component, divided by different powers of two).
void area_axis(const AreaLight& a, bool vAxis, float* out) {
    auto scaled = [&](int k, int i) {
        const float x = std::ldexp(1.f, k - 1);
        const Vec3f p = a.sampleLe(vAxis ? Vec2f{0.5f, x} : Vec2f{x, 0.5f}, {0.5f, 0.5f}).pos;
        return std::ldexp(i == 0 ? p.x : i == 1 ? p.y : p.z, -k);
    };
    for (int i = 0; i < 3; ++i) {
        out[i] = 0.f;
        for (int k = 40; k <= 88; k += 16) {
            const float lo = scaled(k, i), hi = scaled(k + 16, i);
            if (std::isfinite(lo) && lo == hi) {
                out[i] = lo;
                break;
            }
        }
    }
}

// Flattened scene arrays kept alive for the ana_scene_desc pointing at them.
struct Flat {
    std::vector<uint32_t> meshVert, meshTri, indices, strandCp, strandWidth, strandSlot;
    std::vector<uint8_t> hasN;
    std::vector<float> pos, nrm, cps, widths, strandColor, env;
    std::vector<ana_material> mats;
    std::vector<int32_t> slots;
    std::vector<ana_light> lights;
    std::vector<uint32_t> meshMotion;  // key offsets per mesh (+1)
    std::vector<ana_motion_key> keys;
    ana_scene_desc d{};
};

bool material_of(const IMaterial* m, ana_material& o, std::string& err) {
    std::memset(&o, 0, sizeof(o));
    const ShadingContext ctx = probe_ctx();
    if (auto* em = dynamic_cast<const EmissiveMaterial*>(m)) {
        o.type = ANA_MAT_EMISSIVE;
        put3(o.albedo, em->reflectance(ctx));
        put3(o.emission, em->Le(ctx, Vec3f{0.f, 0.f, 1.f}));
        return true;
    }
    if (auto* lm = dynamic_cast<const LambertianMaterial*>(m)) {
        o.type = ANA_MAT_LAMBERT;
        put3(o.albedo, lm->reflectance(ctx));
        return true;
    }
    if (auto* sm = dynamic_cast<const StandardSurfaceMaterial*>(m)) {
        const auto& p = sm->params();
        if (p.base_color.hasTexture() || p.metalness.hasTexture() || p.roughness.hasTexture() ||
            p.specular.hasTexture() || p.opacity.hasTexture() || p.emission_color.hasTexture() ||
            (p.has_normal_map && p.normal_map.hasTexture())) {
            err = "standard_surface with image textures is not supported";
            return false;
        }
        o.type = ANA_MAT_STANDARD;
        put3(o.base_color, p.base_color.value);
        o.base = p.base;
        o.metalness = p.metalness.value;
        o.roughness = p.roughness.value;
        o.specular = p.specular.value;
        put3(o.specular_color, p.specular_color);
        o.specular_ior = p.specular_IOR;
        o.coat = p.coat;
        o.coat_roughness = p.coat_roughness;
        o.transmission = p.transmission;
        o.emission_weight = p.emission;
        put3(o.emission_color, p.emission_color.value);
        o.alpha_mask = p.alphaMask ? 1u : 0u;
        o.opacity = p.opacity.value;
        return true;
    }
    if (auto* hm = dynamic_cast<const MarschnerHairMaterial*>(m)) {
        // MarschnerHairMaterial keeps its Params private. What the reference
        // executes (Kajiya-Kay, MarschnerHair.h:240, 267-282) reads only the
        // absorption, recovered from reflectance() = exp(-sigma_a) at a white
        // strand colour; beta_m is roughness(). The remaining Marschner
        // parameters are set to the class defaults (MarschnerHair.h:192-198).
        Vec3f r = hm->reflectance(ctx);
        o.type = ANA_MAT_HAIR;
        o.hair_mode = ANA_HAIR_KAJIYA_KAY;
        o.sigma_a[0] = -std::log(r.x);
        o.sigma_a[1] = -std::log(r.y);
        o.sigma_a[2] = -std::log(r.z);
        o.eta = 1.55f;
        o.beta_m = hm->roughness();
        o.beta_n = 0.3f;
        o.alpha_deg = 2.f;
        return true;
    }
    err = "unsupported material class";
    return false;
}

bool flatten(const SceneView& scene, uint32_t width, uint32_t height, Flat& F, std::string& err) {
    if (!scene.accel) {
        err = "SceneView has no acceleration structure";
        return false;
    }
    // ---- meshes (GeometryPool) ----
    const GeometryPool& pool = scene.accel->pool();
    F.meshVert.push_back(0);
    F.meshTri.push_back(0);
    F.meshMotion.push_back(0);
    for (const MeshDesc& m : pool.meshes()) {
        for (const MotionKey& k : m.motionKeys) {  // object-space positions, keys by time
            ana_motion_key mk;
            mk.time = k.time;
            for (int i = 0; i < 4; ++i)
                for (int j = 0; j < 4; ++j) mk.object_to_world[4 * i + j] = k.objectToWorld.m[i][j];
            F.keys.push_back(mk);
        }
        F.meshMotion.push_back(uint32_t(F.keys.size()));
        for (const Vec3f& p : m.positions) F.pos.insert(F.pos.end(), {p.x, p.y, p.z});
        bool hasN = m.normals.size() >= m.positions.size() && !m.normals.empty();
        F.hasN.push_back(hasN ? 1 : 0);
        for (size_t i = 0; i < m.positions.size(); ++i) {
            Vec3f n = hasN ? m.normals[i] : Vec3f{};
            F.nrm.insert(F.nrm.end(), {n.x, n.y, n.z});
        }
        F.indices.insert(F.indices.end(), m.indices.begin(), m.indices.begin() + 3 * m.numTriangles());
        F.meshVert.push_back(uint32_t(F.pos.size() / 3));
        F.meshTri.push_back(uint32_t(F.indices.size() / 3));
    }
    // ---- strands (CurvePool of a CurveBrute accel) ----
    F.strandCp.push_back(0);
    F.strandWidth.push_back(0);
    if (auto* cb = dynamic_cast<const CurveBrute*>(scene.accel)) {
        for (const StrandDesc& s : cb->curvePool().strands()) {
            // CurveBrute intersects the control points as stored, with or
            // without motion keys (CurveBrute.cpp:332-396 read no key)
            for (const Vec3f& p : s.controlPoints) F.cps.insert(F.cps.end(), {p.x, p.y, p.z});
            F.widths.insert(F.widths.end(), s.widths.begin(), s.widths.end());
            F.strandCp.push_back(uint32_t(F.cps.size() / 3));
            F.strandWidth.push_back(uint32_t(F.widths.size()));
            F.strandSlot.push_back(s.materialIndex);
            F.strandColor.insert(F.strandColor.end(), {s.color.x, s.color.y, s.color.z});
        }
    }
    // ---- materials: SceneView::materials, deduplicated by object ----
    std::unordered_map<const IMaterial*, int32_t> index;
    for (const IMaterial* m : scene.materials) {
        if (!m) {
            F.slots.push_back(-1);
            continue;
        }
        auto it = index.find(m);
        if (it == index.end()) {
            ana_material am;
            if (!material_of(m, am, err)) return false;
            it = index.emplace(m, int32_t(F.mats.size())).first;
            F.mats.push_back(am);
        }
        F.slots.push_back(it->second);
    }
    // ---- lights, in SceneView::lights order ----
    const DomeLight* dome = scene.envLight ? dynamic_cast<const DomeLight*>(scene.envLight) : nullptr;
    if (scene.envLight && !dome) {
        err = "unsupported environment light class";
        return false;
    }
    for (const ILight* l : scene.lights) {
        ana_light al;
        std::memset(&al, 0, sizeof(al));
        if (auto* a = dynamic_cast<const AreaLight*>(l)) {
            al.type = ANA_LIGHT_AREA;
            put3(al.center, a->sampleLe({0.5f, 0.5f}, {0.5f, 0.5f}).pos);
            area_axis(*a, false, al.u);
            area_axis(*a, true, al.v);
            put3(al.Le, a->sampleLe({0.5f, 0.5f}, {0.5f, 0.5f}).Le);
        } else if (auto* sun = dynamic_cast<const DirectionalLight*>(l)) {
            // DirectionalLight keeps its direction and cone private. sample()
            // returns the direction itself for u.x = 0 (the whole cone
            // collapses to it; for a hard light exactly, DirectionalLight.h:
            // 60-62) and a direction on the cone's edge for u.x = 1.
            const LightSample s0 = sun->sample({}, {}, {0.f, 0.f});
            const LightSample s1 = sun->sample({}, {}, {1.f, 0.f});
            const float c = std::min(1.f, dot(s0.wi, s1.wi));
            al.type = ANA_LIGHT_DIRECTIONAL;
            put3(al.u, s0.wi);
            put3(al.Le, s0.Li);
            al.half_angle_deg = c >= 1.f - 1e-6f ? 0.f : std::acos(c) * 180.f / 3.14159265358979323846f;
        } else if (auto* dl = dynamic_cast<const DomeLight*>(l)) {
            if (dl != dome) {
                err = "a dome light in SceneView::lights must be SceneView::envLight";
                return false;
            }
            al.type = ANA_LIGHT_DOME;
        } else {
            err = "unsupported light class";
            return false;
        }
        F.lights.push_back(al);
    }
    ana_scene_desc& d = F.d;
    std::memset(&d, 0, sizeof(d));
    if (dome) {
        Vec3f r0, r1, r2;
        dome->getRotation(r0, r1, r2);
        if (!(r0 == Vec3f{1, 0, 0} && r1 == Vec3f{0, 1, 0} && r2 == Vec3f{0, 0, 1})) {
            err = "a rotated dome light is not supported";
            return false;
        }
        size_t n = size_t(dome->envWidth()) * dome->envHeight() * 3;
        F.env.assign(dome->pixels(), dome->pixels() + n);
        d.env_rgb = F.env.data();
        d.env_width = dome->envWidth();
        d.env_height = dome->envHeight();
        d.env_intensity = dome->intensity();
    }
    put3(d.env_radiance, scene.envRadiance);
    // ---- camera (PathIntegrator::renderTile's default when none is set) ----
    ana_camera& cam = d.camera;
    if (scene.camera) {
        const Camera& c = *scene.camera;
        if (c.imageWidth != width || c.imageHeight != height) {
            err = "the scene camera was built for another film size";
            return false;
        }
        cam.explicit_basis = 1;
        put3(cam.origin, c.origin);
        put3(cam.lower_left, c.lowerLeftCorner);
        put3(cam.horizontal, c.horizontal);
        put3(cam.vertical, c.vertical);
        put3(cam.basis_u, c.basisU);
        put3(cam.basis_v, c.basisV);
        cam.aperture_radius = c.apertureRadius;
        cam.focal_distance = c.focalDistance;
        cam.shutter_open = c.shutterOpen;
        cam.shutter_close = c.shutterClose;
    } else {
        const float from[3] = {0.f, 0.f, -2.5f}, at[3] = {0.f, 0.f, 1.f}, up[3] = {0.f, 1.f, 0.f};
        std::memcpy(cam.from, from, sizeof(from));
        std::memcpy(cam.at, at, sizeof(at));
        std::memcpy(cam.up, up, sizeof(up));
        cam.vfov_deg = 50.f;
    }
    d.num_meshes = uint32_t(F.hasN.size());
    d.mesh_vert_offset = F.meshVert.data();
    d.mesh_tri_offset = F.meshTri.data();
    d.mesh_has_normals = F.hasN.data();
    d.positions = F.pos.data();
    d.normals = F.nrm.data();
    d.indices = F.indices.data();
    if (!F.keys.empty()) {
        d.mesh_motion_offset = F.meshMotion.data();
        d.motion_keys = F.keys.data();
    }
    d.num_strands = uint32_t(F.strandSlot.size());
    d.strand_cp_offset = F.strandCp.data();
    d.control_points = F.cps.data();
    d.strand_width_offset = F.strandWidth.data();
    d.widths = F.widths.data();
    d.strand_slot = F.strandSlot.data();
    d.strand_color = F.strandColor.data();
    d.num_materials = uint32_t(F.mats.size());
    d.materials = F.mats.data();
    d.num_slots = uint32_t(F.slots.size());
    d.slot_material = F.slots.data();
    d.num_lights = uint32_t(F.lights.size());
    d.lights = F.lights.data();
    return true;
}

std::string ana_message(ana_ctx* ctx) {
    char buf[512];
    ana_last_error(ctx, buf, sizeof(buf));
    return buf;
}

}  // namespace

B200PathIntegrator::B200PathIntegrator(uint32_t maxDepth, uint32_t minDepth, int device)
    : m_maxDepth(maxDepth), m_minDepth(minDepth) {
    ana_device_opts o{};
    o.device = device;
    if (ana_create(&m_ctx, &o) != ANA_OK) {
        m_ctx = nullptr;
        m_err = ana_message(nullptr);
    }
}

B200PathIntegrator::~B200PathIntegrator() { ana_destroy(m_ctx); }

bool B200PathIntegrator::fail(const std::string& what) {
    m_err = what;
    return false;
}

ana_stats B200PathIntegrator::stats() const {
    ana_stats s{};
    if (m_ctx) ana_get_stats(m_ctx, &s);
    return s;
}

ana_prepared* B200PathIntegrator::prepareHost(const SceneView& scene, uint32_t filmWidth, uint32_t filmHeight,
                                              std::string& err) {
    Flat F;
    if (!flatten(scene, filmWidth, filmHeight, F, err)) {
        err = "B200PathIntegrator: " + err;
        return nullptr;
    }
    ana_prepared* p = nullptr;
    if (ana_prepare_scene(&F.d, &p) != ANA_OK) {
        err = ana_message(nullptr);
        return nullptr;
    }
    return p;
}

bool B200PathIntegrator::upload(const SceneView& scene) {
    // film size: the scene camera's, or (without one) the default pinhole is
    // rebuilt per frame from the film size
    uint32_t w = scene.camera ? scene.camera->imageWidth : 1, h = scene.camera ? scene.camera->imageHeight : 1;
    std::string err;
    Flat F;
    if (!flatten(scene, w, h, F, err)) return fail("B200PathIntegrator: " + err);
    // triangle setup and SAH build on the device: the bytes prepareHost's
    // layout would upload, without the host build (BVHBackend::commit)
    if (ana_upload_scene_device(m_ctx, &F.d) != ANA_OK) return fail(ana_message(m_ctx));
    m_prepared = &scene;
    return true;
}

void B200PathIntegrator::prepare(const SceneView& scene) {
    m_prepared = nullptr;
    if (!m_ctx) return;
    upload(scene);
}

void B200PathIntegrator::renderTile(const SceneView&, const TileRequest&, uint32_t, uint32_t, ISampler&,
                                    TileBuffer&) {
    throw std::runtime_error("B200PathIntegrator renders whole frames (renderFrame); tiles are not supported");
}

bool B200PathIntegrator::renderFrame(const SceneView& scene, uint32_t filmWidth, uint32_t filmHeight,
                                     uint32_t sampleStart, uint32_t sampleCount, Film& film) {
    if (!m_ctx) return fail(m_err.empty() ? "B200PathIntegrator: no CUDA device" : m_err);
    if (scene.camera && (scene.camera->imageWidth != filmWidth || scene.camera->imageHeight != filmHeight))
        return fail("B200PathIntegrator: the scene camera was built for another film size");
    if (m_prepared != &scene && !upload(scene)) return false;
    ana_render_desc r{};
    r.width = filmWidth;
    r.height = filmHeight;
    r.sample_start = sampleStart;
    r.sample_count = sampleCount;
    r.max_depth = m_maxDepth;
    r.min_depth = m_minDepth;
    r.seed = 0;  // HaltonSampler's default seed (RenderSession.cpp:465)
    r.flags = ANA_RENDER_CLEAR_FILM | ANA_RENDER_AOVS;
    if (ana_render(m_ctx, &r) != ANA_OK) return fail(ana_message(m_ctx));
    const size_t n = size_t(filmWidth) * filmHeight;
    std::vector<ana_film_pixel> px(n);
    if (ana_film_read(m_ctx, px.data(), n) != ANA_OK) return fail(ana_message(m_ctx));
    // this pass's denoising AOVs (the device film was cleared: weight 1)
    std::vector<float> albedo(3 * n), normal(3 * n);
    if (ana_aov_read(m_ctx, albedo.data(), normal.data(), n) != ANA_OK) return fail(ana_message(m_ctx));
    // one full-frame TileBuffer, merged as the tile loop would (Film.cpp:34-73)
    TileBuffer tile(0, 0, filmWidth, filmHeight);
    for (size_t i = 0; i < n; ++i) {
        tile.pixels[i].r = px[i].r;
        tile.pixels[i].g = px[i].g;
        tile.pixels[i].b = px[i].b;
        tile.pixels[i].weight = px[i].w;
        tile.sumLumSq[i] = px[i].sum_lum_sq;
        tile.albedo[i] = {albedo[3 * i], albedo[3 * i + 1], albedo[3 * i + 2], 1u};
        tile.normals[i] = {normal[3 * i], normal[3 * i + 1], normal[3 * i + 2], 1u};
    }
    film.mergeTile(tile);
    return true;
}

}  // namespace anacapa_b200
