// ============================================================================
// TEST INFRASTRUCTURE — NOT PART OF THE PRODUCT.
//
// A C harness over the reference renderer's own hot-path classes. It is linked
// with the reference's unmodified sources (src/accel/BVHBackend.cpp,
// src/accel/CurveBrute.cpp, src/integrator/PathIntegrator.cpp and the
// header-only materials, lights, sampler and thread pool) by oracle/Makefile
// into oracle/_ref/. Only tests/, __graft_entry__.smoke() and bench.py's CPU
// baseline leg load it, as the checker and as the timed CPU baseline.
//
// What this file supplies on its own:
//   * evalTOV (src/shading/Texture.cpp:126-136): the constant-value branch
//     only; image textures need OpenImageIO, which is absent, and no workload
//     uses them.
//   * DomeLight::loadImage (src/shading/lights/DomeLight.cpp:15-107): instead
//     of reading a file it copies an in-memory RGB float equirect that the
//     caller registered; DomeLight::buildDistribution then runs unchanged.
//   * the frame driver: RenderSession::render's non-adaptive CPU branch
//     (src/render/RenderSession.cpp:465-547) — HaltonSampler(spp, seed 0),
//     ThreadPool, 64x64 tiles, PathIntegrator::renderTile, and a merge of each
//     TileBuffer into plain arrays with Film::mergeTile's arithmetic
//     (src/film/Film.cpp:34-73; Film.cpp itself needs OpenImageIO).
// ============================================================================
#include <anacapa/core/Types.h>
#include <anacapa/accel/GeometryPool.h>
#include <anacapa/accel/CurvePool.h>
#include <anacapa/integrator/IIntegrator.h>
#include <anacapa/shading/ShadingContext.h>

#include "accel/BVHBackend.h"
#include "accel/CurveBrute.h"
#include "integrator/PathIntegrator.h"
#include "render/ThreadPool.h"
#include "sampling/HaltonSampler.h"
#include "sampling/PCGRng.h"
#include "shading/Lambertian.h"
#include "shading/MarschnerHair.h"
#include "shading/StandardSurface.h"
#include "shading/Texture.h"
#include "shading/lights/AreaLight.h"
#include "shading/lights/DirectionalLight.h"
#include "shading/lights/DomeLight.h"

#include <chrono>
#include <cstdint>
#include <cstring>
#include <memory>
#include <mutex>
#include <vector>

namespace anacapa {

Spectrum evalTOV(const SpectrumTOV& t, Vec2f) { return t.value; }
float evalTOV(const FloatTOV& t, Vec2f) { return t.value; }

namespace {
const float* g_pendingEnv = nullptr;
uint32_t g_pendingW = 0, g_pendingH = 0;
}  // namespace

void DomeLight::loadImage(const std::string&) {
    if (!g_pendingEnv || g_pendingW == 0 || g_pendingH == 0) return;
    m_width = g_pendingW;
    m_height = g_pendingH;
    m_pixels.assign(g_pendingEnv, g_pendingEnv + size_t(m_width) * m_height * 3);
}

}  // namespace anacapa

using namespace anacapa;

namespace {

struct RefScene {
    GeometryPool geom;
    CurvePool curves;
    std::vector<std::unique_ptr<IMaterial>> mats;
    std::vector<std::unique_ptr<ILight>> lights;
    std::unique_ptr<CurveBrute> accel;
    SceneView view;
    bool committed = false;
};

Vec3f v3(const float* p) { return {p[0], p[1], p[2]}; }
void put3(float* o, Vec3f v) { o[0] = v.x; o[1] = v.y; o[2] = v.z; }

// Records the order in which the integrator draws sampler dimensions.
class LoggingSampler : public ISampler {
public:
    explicit LoggingSampler(uint32_t spp) : m_inner(spp, 0) {}
    std::unique_ptr<ISampler> clone() const override {
        return std::make_unique<LoggingSampler>(*this);
    }
    void startPixelSample(uint32_t x, uint32_t y, uint32_t s) override {
        m_inner.startPixelSample(x, y, s);
        m_dim = 0;
    }
    float get1D() override {
        log.push_back(int32_t(m_dim++));
        return m_inner.get1D();
    }
    Vec2f get2D() override {
        // Dimensions of one 2-D draw are logged as negative pairs so the
        // caller can tell 1-D draws from 2-D draws.
        log.push_back(-1 - int32_t(m_dim));
        m_dim += 2;
        return m_inner.get2D();
    }
    SamplerState getState() const override { return m_inner.getState(); }
    std::vector<int32_t> log;

private:
    HaltonSampler m_inner;
    uint32_t m_dim = 0;
};

StandardSurfaceMaterial::Params ssParams(const float* p) {
    // Packed layout (20 floats): base_color[3], base, metalness, roughness,
    // specular, specular_color[3], specular_IOR, coat, coat_roughness,
    // transmission, emission, emission_color[3], alphaMask (0/1), opacity
    StandardSurfaceMaterial::Params q;
    q.base_color = SpectrumTOV(Vec3f{p[0], p[1], p[2]});
    q.base = p[3];
    q.metalness = FloatTOV(p[4]);
    q.roughness = FloatTOV(p[5]);
    q.specular = FloatTOV(p[6]);
    q.specular_color = {p[7], p[8], p[9]};
    q.specular_IOR = p[10];
    q.coat = p[11];
    q.coat_roughness = p[12];
    q.transmission = p[13];
    q.emission = p[14];
    q.emission_color = SpectrumTOV(Vec3f{p[15], p[16], p[17]});
    q.alphaMask = p[18] != 0.f;
    q.opacity = FloatTOV(p[19]);
    return q;
}

// ---------------------------------------------------------------------------
// The Marschner R/TT/TRT code of MarschnerHairMaterial (MarschnerHair.h:242-257
// in evaluate, 284-375 in sample, helpers and evalLobes/evalPdf at 430-556) is
// unreachable through the public interface: evaluate and sample return the
// Kajiya-Kay lobe first (MarschnerHair.h:240, 267-282), and the helpers are
// private. An explicit instantiation may name private members ([temp.spec]),
// so the templates below hand out pointers to them without editing the
// reference's sources; the functions called are the reference's own code.
// ---------------------------------------------------------------------------
template <class Tag, typename Tag::type M>
struct Expose {
    friend typename Tag::type member(Tag) { return M; }
};
struct MhLobes {
    using type = Spectrum (MarschnerHairMaterial::*)(float, float, float, float, float, float, Spectrum) const;
    friend type member(MhLobes);
};
struct MhPdf {
    using type = float (MarschnerHairMaterial::*)(float, float, float, float, float, float, Spectrum) const;
    friend type member(MhPdf);
};
struct MhSigma {
    using type = Spectrum (MarschnerHairMaterial::*)(const ShadingContext&) const;
    friend type member(MhSigma);
};
struct MhLong {
    using type = void (*)(Vec3f, Vec3f, float&, float&);
    friend type member(MhLong);
};
struct MhPhiOf {
    using type = float (*)(Vec3f, Vec3f, Vec3f, float, float);
    friend type member(MhPhiOf);
};
struct MhImpact {
    using type = float (*)(Vec3f, Vec3f, Vec3f, float);
    friend type member(MhImpact);
};
struct MhParams {
    using type = MarschnerHairMaterial::Params MarschnerHairMaterial::*;
    friend type member(MhParams);
};
struct MhVar {
    using type = float (MarschnerHairMaterial::*)[3];
    friend type member(MhVar);
};
struct MhScale {
    using type = float MarschnerHairMaterial::*;
    friend type member(MhScale);
};
struct MhAlpha {
    using type = float (MarschnerHairMaterial::*)[3];
    friend type member(MhAlpha);
};
template struct Expose<MhLobes, &MarschnerHairMaterial::evalLobes>;
template struct Expose<MhPdf, &MarschnerHairMaterial::evalPdf>;
template struct Expose<MhSigma, &MarschnerHairMaterial::effectiveSigmaA>;
template struct Expose<MhLong, &MarschnerHairMaterial::hairLongitudinal>;
template struct Expose<MhPhiOf, &MarschnerHairMaterial::hairPhi>;
template struct Expose<MhImpact, &MarschnerHairMaterial::hairImpactParam>;
template struct Expose<MhParams, &MarschnerHairMaterial::m_p>;
template struct Expose<MhVar, &MarschnerHairMaterial::m_v>;
template struct Expose<MhScale, &MarschnerHairMaterial::m_s>;
template struct Expose<MhAlpha, &MarschnerHairMaterial::m_alpha>;

// MarschnerHairMaterial::evaluate's Marschner branch (MarschnerHair.h:242-257),
// composed of the reference's private helpers. out: f[3], pdf, pdfRev.
void mhEvaluate(const MarschnerHairMaterial& m, const ShadingContext& ctx, Vec3f wo, Vec3f wi, float* out) {
    float sinThetaO, cosThetaO, sinThetaI, cosThetaI;
    member(MhLong{})(wo, ctx.t, sinThetaO, cosThetaO);
    member(MhLong{})(wi, ctx.t, sinThetaI, cosThetaI);
    float phi = member(MhPhiOf{})(wo, wi, ctx.t, sinThetaO, sinThetaI);
    float h = member(MhImpact{})(wo, ctx.t, ctx.n, sinThetaO);
    Spectrum sigA = (m.*member(MhSigma{}))(ctx);
    Spectrum f = (m.*member(MhLobes{}))(sinThetaO, cosThetaO, sinThetaI, cosThetaI, phi, h, sigA);
    float pd = (m.*member(MhPdf{}))(sinThetaO, cosThetaO, sinThetaI, cosThetaI, phi, h, sigA);
    out[0] = f.x;
    out[1] = f.y;
    out[2] = f.z;
    out[3] = pd;
    out[4] = (m.*member(MhPdf{}))(sinThetaI, cosThetaI, sinThetaO, cosThetaO, -phi, h, sigA);
}

// MarschnerHairMaterial::sample's Marschner branch (MarschnerHair.h:284-375).
// The statements between the calls are restated here in the reference's order
// (they sit inside sample() after its early return and cannot be called);
// every function they call is the reference's own. out: f[3], wi[3], pdf,
// valid (0/1).
void mhSample(const MarschnerHairMaterial& m, const ShadingContext& ctx, Vec3f wo, Vec2f u, float uComp,
              float* out) {
    for (int k = 0; k < 8; ++k) out[k] = 0.f;
    const MarschnerHairMaterial::Params& P = m.*member(MhParams{});
    const float* V = m.*member(MhVar{});
    const float S = m.*member(MhScale{});
    const float* A = m.*member(MhAlpha{});
    float sinThetaO, cosThetaO;
    member(MhLong{})(wo, ctx.t, sinThetaO, cosThetaO);
    float h = member(MhImpact{})(wo, ctx.t, ctx.n, sinThetaO);
    Spectrum sigA = (m.*member(MhSigma{}))(ctx);
    auto ap = mh_Ap(cosThetaO, P.eta, h, sigA);
    float weights[3];
    for (int p = 0; p < 3; ++p) weights[p] = luminance(ap[p]);
    float total = weights[0] + weights[1] + weights[2];
    if (total < 1e-8f) return;
    float invTotal = 1.f / total;
    float cdf[3];
    cdf[0] = weights[0] * invTotal;
    cdf[1] = cdf[0] + weights[1] * invTotal;
    cdf[2] = 1.f;
    int lobe = 0;
    float uRemapped = uComp;
    if (uComp < cdf[0]) {
        uRemapped = uComp / cdf[0];
    } else if (uComp < cdf[1]) {
        lobe = 1;
        uRemapped = (uComp - cdf[0]) / (cdf[1] - cdf[0]);
    } else {
        lobe = 2;
        uRemapped = (uComp - cdf[1]) / (cdf[2] - cdf[1]);
    }
    float thetaO = std::asin(std::clamp(sinThetaO, -1.f + 1e-5f, 1.f - 1e-5f));
    float z = mh_sampleGaussian(u.x, u.y);
    float thetaI = thetaO + A[lobe] + z * std::sqrt(V[lobe]);
    thetaI = std::clamp(thetaI, -kMH_Pi * 0.5f, kMH_Pi * 0.5f);
    float sinThetaI = std::sin(thetaI);
    float cosThetaI = std::cos(thetaI);
    float sin2ThetaO = 1.f - cosThetaO * cosThetaO;
    float etaP = std::sqrt(std::max(0.f, P.eta * P.eta - sin2ThetaO)) / cosThetaO;
    float gammaO = std::asin(std::clamp(h, -1.f + 1e-5f, 1.f - 1e-5f));
    float sinGammaT = std::clamp(h / (etaP > 1e-5f ? etaP : 1e-5f), -1.f + 1e-5f, 1.f - 1e-5f);
    float gammaT = std::asin(sinGammaT);
    float phiSampled = mh_sampleTrimmedLogistic(uRemapped, S) + mh_Phi(lobe, gammaO, gammaT);
    Vec3f woPerp = safeNormalize(wo - ctx.t * sinThetaO);
    if (woPerp.lengthSq() < 1e-8f) {
        Vec3f dummy;
        buildOrthonormalBasis(ctx.t, woPerp, dummy);
    }
    Vec3f ctPerp = cross(ctx.t, woPerp);
    Vec3f wi = ctx.t * sinThetaI + woPerp * (cosThetaI * std::cos(phiSampled)) +
               ctPerp * (cosThetaI * std::sin(phiSampled));
    wi = safeNormalize(wi);
    float sinThetaIa, cosThetaIa;
    member(MhLong{})(wi, ctx.t, sinThetaIa, cosThetaIa);
    float phiActual = member(MhPhiOf{})(wo, wi, ctx.t, sinThetaO, sinThetaIa);
    Spectrum f = (m.*member(MhLobes{}))(sinThetaO, cosThetaO, sinThetaIa, cosThetaIa, phiActual, h, sigA);
    float pd = (m.*member(MhPdf{}))(sinThetaO, cosThetaO, sinThetaIa, cosThetaIa, phiActual, h, sigA);
    if (pd < 1e-8f) return;
    float cosSurf = std::abs(dot(wi, ctx.n));
    f = f * cosSurf;
    put3(out, f);
    put3(out + 3, wi);
    out[6] = pd;
    out[7] = 1.f;
}

SurfaceInteraction makeSI(const float* s) {
    // s: p[3], n[3], ng[3], dpdu[3], color[3], isCurve
    SurfaceInteraction si;
    si.p = v3(s + 0);
    si.n = v3(s + 3);
    si.ng = v3(s + 6);
    si.dpdu = v3(s + 9);
    si.color = v3(s + 12);
    si.isCurve = s[15] != 0.f;
    return si;
}

}  // namespace

extern "C" {

void* ref_scene_new() { return new RefScene(); }
void ref_scene_free(void* s) { delete static_cast<RefScene*>(s); }

int ref_add_mesh(void* sp, const float* pos, const float* nrm, const float* uv,
                 uint32_t nv, const uint32_t* idx, uint32_t ntri) {
    auto* s = static_cast<RefScene*>(sp);
    MeshDesc m;
    m.positions.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) m.positions[i] = v3(pos + 3 * i);
    if (nrm) {
        m.normals.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) m.normals[i] = v3(nrm + 3 * i);
    }
    if (uv) {
        m.uvs.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) m.uvs[i] = {uv[2 * i], uv[2 * i + 1]};
    }
    m.indices.assign(idx, idx + size_t(ntri) * 3);
    return int(s->geom.addMesh(std::move(m)));
}

// A motion-blurred mesh: positions in object space and nkeys MotionKeys of
// 17 floats each (time, objectToWorld row-major); worldToObject is the
// inverse, as the scene loaders precompute it.
int ref_add_mesh_motion(void* sp, const float* pos, const float* nrm, const float* uv, uint32_t nv,
                        const uint32_t* idx, uint32_t ntri, const float* keys, uint32_t nkeys) {
    auto* s = static_cast<RefScene*>(sp);
    MeshDesc m;
    m.positions.resize(nv);
    for (uint32_t i = 0; i < nv; ++i) m.positions[i] = v3(pos + 3 * i);
    if (nrm) {
        m.normals.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) m.normals[i] = v3(nrm + 3 * i);
    }
    if (uv) {
        m.uvs.resize(nv);
        for (uint32_t i = 0; i < nv; ++i) m.uvs[i] = {uv[2 * i], uv[2 * i + 1]};
    }
    m.indices.assign(idx, idx + size_t(ntri) * 3);
    for (uint32_t k = 0; k < nkeys; ++k) {
        MotionKey mk;
        mk.time = keys[17 * k];
        for (int i = 0; i < 4; ++i)
            for (int j = 0; j < 4; ++j) mk.objectToWorld.m[i][j] = keys[17 * k + 1 + 4 * i + j];
        mk.worldToObject = mk.objectToWorld.inverse();
        m.motionKeys.push_back(mk);
    }
    return int(s->geom.addMesh(std::move(m)));
}

int ref_add_strand(void* sp, const float* cps, uint32_t ncp, const float* widths,
                   uint32_t nw, uint32_t matSlot, const float* color) {
    auto* s = static_cast<RefScene*>(sp);
    StrandDesc d;
    d.controlPoints.resize(ncp);
    for (uint32_t i = 0; i < ncp; ++i) d.controlPoints[i] = v3(cps + 3 * i);
    d.widths.assign(widths, widths + nw);
    d.materialIndex = matSlot;
    if (color) d.color = v3(color);
    return int(s->curves.addStrand(std::move(d)));
}

int ref_mat_lambert(void* sp, const float* albedo) {
    auto* s = static_cast<RefScene*>(sp);
    s->mats.push_back(std::make_unique<LambertianMaterial>(v3(albedo)));
    return int(s->mats.size() - 1);
}

int ref_mat_emissive(void* sp, const float* albedo, const float* emission) {
    auto* s = static_cast<RefScene*>(sp);
    s->mats.push_back(std::make_unique<EmissiveMaterial>(v3(albedo), v3(emission)));
    return int(s->mats.size() - 1);
}

int ref_mat_standard(void* sp, const float* packed20) {
    auto* s = static_cast<RefScene*>(sp);
    s->mats.push_back(std::make_unique<StandardSurfaceMaterial>(ssParams(packed20)));
    return int(s->mats.size() - 1);
}

int ref_mat_marschner(void* sp, float eta, const float* sigma_a, float beta_m,
                      float beta_n, float alpha_deg) {
    auto* s = static_cast<RefScene*>(sp);
    MarschnerHairMaterial::Params p;
    p.eta = eta;
    p.sigma_a = v3(sigma_a);
    p.beta_m = beta_m;
    p.beta_n = beta_n;
    p.alpha = alpha_deg;
    s->mats.push_back(std::make_unique<MarschnerHairMaterial>(p));
    return int(s->mats.size() - 1);
}

// SceneView::materials is indexed by meshID (and by StrandDesc::materialIndex).
void ref_set_slot(void* sp, uint32_t slot, int matHandle) {
    auto* s = static_cast<RefScene*>(sp);
    if (s->view.materials.size() <= slot) s->view.materials.resize(slot + 1, nullptr);
    s->view.materials[slot] = matHandle >= 0 ? s->mats[size_t(matHandle)].get() : nullptr;
}

int ref_light_area(void* sp, const float* c, const float* u, const float* v, const float* Le) {
    auto* s = static_cast<RefScene*>(sp);
    s->lights.push_back(std::make_unique<AreaLight>(v3(c), v3(u), v3(v), v3(Le)));
    s->view.lights.push_back(s->lights.back().get());
    return int(s->lights.size() - 1);
}

// DirectionalLight (its scene radius and centre only place BDPT's emission disk).
int ref_light_directional(void* sp, const float* dir, const float* Le, float halfAngleDeg) {
    auto* s = static_cast<RefScene*>(sp);
    s->lights.push_back(std::make_unique<DirectionalLight>(v3(dir), v3(Le), 10.f, Vec3f{}, halfAngleDeg));
    s->view.lights.push_back(s->lights.back().get());
    return int(s->lights.size() - 1);
}

// Dome light: registered as SceneView::envLight and appended to the light list,
// as RenderSession::render does (src/render/RenderSession.cpp:407-422).
int ref_light_dome(void* sp, const float* rgb, uint32_t w, uint32_t h, float intensity,
                   int inLightList) {
    auto* s = static_cast<RefScene*>(sp);
    g_pendingEnv = rgb;
    g_pendingW = w;
    g_pendingH = h;
    auto dome = std::make_unique<DomeLight>(rgb ? std::string("mem") : std::string(),
                                            intensity, 10.f, Vec3f{});
    g_pendingEnv = nullptr;
    s->view.envLight = dome.get();
    if (inLightList) s->view.lights.push_back(dome.get());
    s->lights.push_back(std::move(dome));
    return int(s->lights.size() - 1);
}

void ref_set_env_radiance(void* sp, const float* rgb) {
    static_cast<RefScene*>(sp)->view.envRadiance = v3(rgb);
}

void ref_set_camera(void* sp, const float* from, const float* at, const float* up,
                    float vfov, uint32_t w, uint32_t h) {
    auto* s = static_cast<RefScene*>(sp);
    s->view.camera = Camera::makePinhole(v3(from), v3(at), v3(up), vfov, w, h);
}

void ref_set_shutter(void* sp, float open, float close) {
    auto* s = static_cast<RefScene*>(sp);
    if (!s->view.camera) return;
    s->view.camera->shutterOpen = open;
    s->view.camera->shutterClose = close;
}

int ref_commit(void* sp) {
    auto* s = static_cast<RefScene*>(sp);
    s->accel = std::make_unique<CurveBrute>(s->geom, s->curves);
    s->accel->commit();
    s->view.accel = s->accel.get();
    s->committed = true;
    return 0;
}

// rays: n x 8 floats (ox, oy, oz, tmin, dx, dy, dz, tmax)
// out_ids: n x 4 int32 (hit, meshID, primID, strandID); out_t: n floats
// times: one Ray::time per ray, or NULL (time 0)
void ref_trace(void* sp, const float* rays, const float* times, uint64_t n, int32_t* out_ids, float* out_t,
               int nthreads) {
    auto* s = static_cast<RefScene*>(sp);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    const uint64_t chunk = 4096;
    uint32_t nChunks = uint32_t((n + chunk - 1) / chunk);
    pool.parallelFor(nChunks, [&](uint32_t c) {
        uint64_t b = uint64_t(c) * chunk, e = std::min<uint64_t>(n, b + chunk);
        for (uint64_t i = b; i < e; ++i) {
            const float* r = rays + 8 * i;
            Ray ray{v3(r), v3(r + 4), r[3], r[7]};
            if (times) ray.time = times[i];
            TraceResult tr = s->accel->trace(ray);
            out_ids[4 * i + 0] = tr.hit ? 1 : 0;
            out_ids[4 * i + 1] = tr.hit ? int32_t(tr.si.meshID) : -1;
            out_ids[4 * i + 2] = tr.hit ? int32_t(tr.si.primID) : -1;
            out_ids[4 * i + 3] = tr.hit && tr.si.isCurve ? int32_t(tr.si.strandID) : -1;
            out_t[i] = tr.hit ? tr.si.t : 0.f;
        }
    });
}

void ref_occluded(void* sp, const float* rays, const float* times, uint64_t n, uint8_t* out, int nthreads) {
    auto* s = static_cast<RefScene*>(sp);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    const uint64_t chunk = 4096;
    uint32_t nChunks = uint32_t((n + chunk - 1) / chunk);
    pool.parallelFor(nChunks, [&](uint32_t c) {
        uint64_t b = uint64_t(c) * chunk, e = std::min<uint64_t>(n, b + chunk);
        for (uint64_t i = b; i < e; ++i) {
            const float* r = rays + 8 * i;
            Ray ray{v3(r), v3(r + 4), r[3], r[7]};
            if (times) ray.time = times[i];
            out[i] = s->accel->occluded(ray) ? 1 : 0;
        }
    });
}

// Non-adaptive frame render of the pixel rectangle [x0,x1) x [y0,y1) through the
// reference's ThreadPool and PathIntegrator::renderTile, 64x64 tiles.
// out_rgbw: W*H*4 (pre-weighted r,g,b and weight, as Film's accumulators hold),
// out_lumsq: W*H. Only pixels inside the rectangle are written (added to).
// Returns the render wall time in seconds (scene build excluded).
double ref_render(void* sp, uint32_t W, uint32_t H, uint32_t spp, uint32_t sampleStart,
                  uint32_t maxDepth, int nthreads, uint32_t x0, uint32_t y0, uint32_t x1,
                  uint32_t y1, float* out_rgbw, float* out_lumsq) {
    auto* s = static_cast<RefScene*>(sp);
    PathIntegrator integ(maxDepth);
    integ.prepare(s->view);
    HaltonSampler base(spp);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    std::vector<TileRequest> tiles;
    const uint32_t ts = 64;
    for (uint32_t y = y0; y < y1; y += ts)
        for (uint32_t x = x0; x < x1; x += ts)
            tiles.push_back({x, y, std::min(ts, x1 - x), std::min(ts, y1 - y), sampleStart, spp});
    std::mutex mu;
    auto t0 = std::chrono::steady_clock::now();
    pool.parallelFor(uint32_t(tiles.size()), [&](uint32_t ti) {
        const TileRequest& t = tiles[ti];
        auto sampler = base.clone();
        TileBuffer tb(t.x0, t.y0, t.width, t.height);
        integ.renderTile(s->view, t, W, H, *sampler, tb);
        std::lock_guard<std::mutex> lk(mu);
        for (uint32_t ty = 0; ty < t.height; ++ty)
            for (uint32_t tx = 0; tx < t.width; ++tx) {
                size_t fi = size_t(t.y0 + ty) * W + (t.x0 + tx);
                size_t li = size_t(ty) * t.width + tx;
                const auto& px = tb.pixels[li];
                if (px.weight > 0.f) {
                    out_rgbw[4 * fi + 0] += px.r;
                    out_rgbw[4 * fi + 1] += px.g;
                    out_rgbw[4 * fi + 2] += px.b;
                    out_rgbw[4 * fi + 3] += px.weight;
                    out_lumsq[fi] += tb.sumLumSq[li];
                }
            }
    });
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// ref_render over several full-width row bands [rows[2k], rows[2k+1]) of the
// frame at once: the 64x64 tiles of every band (cut as RenderSession's
// scheduleTiles cuts a frame, clipped to the band) go to one
// ThreadPool::parallelFor, so the pool stays busy across bands. Returns the
// seconds of the parallelFor.
double ref_render_rows(void* sp, uint32_t W, uint32_t H, uint32_t spp, uint32_t sampleStart, uint32_t maxDepth,
                       int nthreads, const uint32_t* rows, uint32_t nbands, float* out_rgbw, float* out_lumsq) {
    auto* s = static_cast<RefScene*>(sp);
    PathIntegrator integ(maxDepth);
    integ.prepare(s->view);
    HaltonSampler base(spp);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    std::vector<TileRequest> tiles;
    const uint32_t ts = 64;
    for (uint32_t b = 0; b < nbands; ++b) {
        const uint32_t y0 = std::min(rows[2 * b], H), y1 = std::min(rows[2 * b + 1], H);
        for (uint32_t y = y0; y < y1; y += ts)
            for (uint32_t x = 0; x < W; x += ts)
                tiles.push_back({x, y, std::min(ts, W - x), std::min(ts, y1 - y), sampleStart, spp});
    }
    std::mutex mu;
    auto t0 = std::chrono::steady_clock::now();
    pool.parallelFor(uint32_t(tiles.size()), [&](uint32_t ti) {
        const TileRequest& t = tiles[ti];
        auto sampler = base.clone();
        TileBuffer tb(t.x0, t.y0, t.width, t.height);
        integ.renderTile(s->view, t, W, H, *sampler, tb);
        std::lock_guard<std::mutex> lk(mu);
        for (uint32_t ty = 0; ty < t.height; ++ty)
            for (uint32_t tx = 0; tx < t.width; ++tx) {
                size_t fi = size_t(t.y0 + ty) * W + (t.x0 + tx);
                size_t li = size_t(ty) * t.width + tx;
                const auto& px = tb.pixels[li];
                if (px.weight > 0.f) {
                    out_rgbw[4 * fi + 0] += px.r;
                    out_rgbw[4 * fi + 1] += px.g;
                    out_rgbw[4 * fi + 2] += px.b;
                    out_rgbw[4 * fi + 3] += px.weight;
                    out_lumsq[fi] += tb.sumLumSq[li];
                }
            }
    });
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

// The denoising AOVs of a frame: the 64x64 tiles of ref_render, each merged
// into plain albedo (rgbw) and normal (xyzw) accumulators with
// Film::mergeTile's arithmetic (Film.cpp:58-70): the tile's per-pixel average
// over its count, added with weight 1.
void ref_render_aov(void* sp, uint32_t W, uint32_t H, uint32_t spp, uint32_t sampleStart, uint32_t maxDepth,
                    int nthreads, float* out_albedo, float* out_normal) {
    auto* s = static_cast<RefScene*>(sp);
    PathIntegrator integ(maxDepth);
    integ.prepare(s->view);
    HaltonSampler base(spp);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    std::vector<TileRequest> tiles;
    const uint32_t ts = 64;
    for (uint32_t y = 0; y < H; y += ts)
        for (uint32_t x = 0; x < W; x += ts)
            tiles.push_back({x, y, std::min(ts, W - x), std::min(ts, H - y), sampleStart, spp});
    std::mutex mu;
    pool.parallelFor(uint32_t(tiles.size()), [&](uint32_t ti) {
        const TileRequest& t = tiles[ti];
        auto sampler = base.clone();
        TileBuffer tb(t.x0, t.y0, t.width, t.height);
        integ.renderTile(s->view, t, W, H, *sampler, tb);
        std::lock_guard<std::mutex> lk(mu);
        for (uint32_t ty = 0; ty < t.height; ++ty)
            for (uint32_t tx = 0; tx < t.width; ++tx) {
                size_t fi = size_t(t.y0 + ty) * W + (t.x0 + tx);
                size_t li = size_t(ty) * t.width + tx;
                const auto& a = tb.albedo[li];
                if (a.count > 0) {
                    float inv = 1.f / static_cast<float>(a.count);
                    out_albedo[4 * fi + 0] += a.r * inv;
                    out_albedo[4 * fi + 1] += a.g * inv;
                    out_albedo[4 * fi + 2] += a.b * inv;
                    out_albedo[4 * fi + 3] += 1.f;
                }
                const auto& n = tb.normals[li];
                if (n.count > 0) {
                    float inv = 1.f / static_cast<float>(n.count);
                    out_normal[4 * fi + 0] += n.r * inv;
                    out_normal[4 * fi + 1] += n.g * inv;
                    out_normal[4 * fi + 2] += n.b * inv;
                    out_normal[4 * fi + 3] += 1.f;
                }
            }
    });
}

// Radiance of single camera samples (pixel px,py, sample index s), through a
// 1x1 tile with sampleCount 1: the tile holds exactly the sample (0 if it was
// not finite). out: n x 3.
void ref_li(void* sp, uint32_t W, uint32_t H, uint32_t maxDepth, const uint32_t* pxy_s,
            uint64_t n, float* out, int nthreads) {
    auto* s = static_cast<RefScene*>(sp);
    PathIntegrator integ(maxDepth);
    integ.prepare(s->view);
    HaltonSampler base(1);
    ThreadPool pool(uint32_t(nthreads > 0 ? nthreads : 0));
    pool.parallelFor(uint32_t(n), [&](uint32_t i) {
        auto sampler = base.clone();
        TileRequest t{pxy_s[3 * i], pxy_s[3 * i + 1], 1, 1, pxy_s[3 * i + 2], 1};
        TileBuffer tb(t.x0, t.y0, 1, 1);
        integ.renderTile(s->view, t, W, H, *sampler, tb);
        out[3 * i + 0] = tb.pixels[0].r;
        out[3 * i + 1] = tb.pixels[0].g;
        out[3 * i + 2] = tb.pixels[0].b;
    });
}

// Order of sampler draws for one camera sample. Entries >= 0 are 1-D draws of
// that dimension; entries < 0 encode a 2-D draw starting at dimension -1-e.
int ref_dim_log(void* sp, uint32_t W, uint32_t H, uint32_t maxDepth, uint32_t px, uint32_t py,
                uint32_t sIdx, int32_t* out, int cap) {
    auto* s = static_cast<RefScene*>(sp);
    PathIntegrator integ(maxDepth);
    integ.prepare(s->view);
    LoggingSampler ls(1);
    TileRequest t{px, py, 1, 1, sIdx, 1};
    TileBuffer tb(px, py, 1, 1);
    integ.renderTile(s->view, t, W, H, ls, tb);
    int n = int(std::min<size_t>(ls.log.size(), size_t(cap)));
    for (int i = 0; i < n; ++i) out[i] = ls.log[size_t(i)];
    return int(ls.log.size());
}

// Camera rays exactly as PathIntegrator::renderTile builds them.
void ref_camera_rays(void* sp, uint32_t W, uint32_t H, const uint32_t* pxy_s, uint64_t n,
                     float* out /* n x 6 */) {
    auto* s = static_cast<RefScene*>(sp);
    Camera cam = s->view.camera.value_or(
        Camera::makePinhole({0.f, 0.f, -2.5f}, {0.f, 0.f, 1.f}, {0.f, 1.f, 0.f}, 50.f, W, H));
    HaltonSampler smp(1);
    for (uint64_t i = 0; i < n; ++i) {
        smp.startPixelSample(pxy_s[3 * i], pxy_s[3 * i + 1], pxy_s[3 * i + 2]);
        Vec2f j = smp.get2D();
        Vec2f l = smp.get2D();
        float tu = smp.get1D();
        Ray r = cam.generateRay(pxy_s[3 * i], pxy_s[3 * i + 1], j.x, j.y, l.x, l.y, tu);
        put3(out + 6 * i, r.origin);
        put3(out + 6 * i + 3, r.direction);
    }
}

// The scene's Camera as this build of the reference computed it: origin,
// lowerLeftCorner, horizontal, vertical, basisU, basisV, apertureRadius,
// focalDistance, shutterOpen, shutterClose (22 floats).
void ref_camera_basis(void* sp, uint32_t W, uint32_t H, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    Camera cam = s->view.camera.value_or(
        Camera::makePinhole({0.f, 0.f, -2.5f}, {0.f, 0.f, 1.f}, {0.f, 1.f, 0.f}, 50.f, W, H));
    put3(out, cam.origin);
    put3(out + 3, cam.lowerLeftCorner);
    put3(out + 6, cam.horizontal);
    put3(out + 9, cam.vertical);
    put3(out + 12, cam.basisU);
    put3(out + 15, cam.basisV);
    out[18] = cam.apertureRadius;
    out[19] = cam.focalDistance;
    out[20] = cam.shutterOpen;
    out[21] = cam.shutterClose;
}

// ---- sampler -------------------------------------------------------------
void ref_halton(uint32_t px, uint32_t py, uint32_t sampleIndex, uint64_t seed, uint32_t ndims,
                float* out) {
    HaltonSampler s(1, seed);
    s.startPixelSample(px, py, sampleIndex);
    for (uint32_t d = 0; d < ndims; ++d) out[d] = s.get1D();
}

void ref_pcg(uint64_t seed, uint32_t n, uint32_t* out) {
    PCGRng r{seed};
    for (uint32_t i = 0; i < n; ++i) out[i] = r.nextUint32();
}

// ---- materials (single evaluations) ----------------------------------------
// si: see makeSI. out: f[3], pdf, pdfRev
void ref_mat_evaluate(void* sp, int h, const float* si, const float* rayDir, const float* wo,
                      const float* wi, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    ShadingContext ctx(makeSI(si), v3(rayDir));
    BSDFEval e = s->mats[size_t(h)]->evaluate(ctx, v3(wo), v3(wi));
    put3(out, e.f);
    out[3] = e.pdf;
    out[4] = e.pdfRev;
}

// out: f[3], wi[3], pdf, flags
void ref_mat_sample(void* sp, int h, const float* si, const float* rayDir, const float* wo,
                    const float* u2, float uc, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    ShadingContext ctx(makeSI(si), v3(rayDir));
    BSDFSample b = s->mats[size_t(h)]->sample(ctx, v3(wo), Vec2f{u2[0], u2[1]}, uc);
    put3(out, b.f);
    put3(out + 3, b.wi);
    out[6] = b.pdf;
    out[7] = float(b.flags);
}

void ref_mat_le(void* sp, int h, const float* si, const float* rayDir, const float* wo,
                float* out) {
    auto* s = static_cast<RefScene*>(sp);
    ShadingContext ctx(makeSI(si), v3(rayDir));
    put3(out, s->mats[size_t(h)]->Le(ctx, v3(wo)));
}

float ref_ggx_D(float cosH, float alpha2) { return D_GGX(cosH, alpha2); }

// ---- Marschner hair lobes (MarschnerHair.h) ------------------------------------
// Evaluation and sampling through the Marschner branches (see mhEvaluate /
// mhSample) of material handle h, which must be a MarschnerHairMaterial.
// si: see makeSI. eval out: f[3], pdf, pdfRev; sample out: f[3], wi[3], pdf, valid.
int ref_mh_evaluate(void* sp, int h, const float* si, const float* rayDir, const float* wo, const float* wi,
                    float* out) {
    auto* s = static_cast<RefScene*>(sp);
    auto* m = dynamic_cast<const MarschnerHairMaterial*>(s->mats[size_t(h)].get());
    if (!m) return 1;
    ShadingContext ctx(makeSI(si), v3(rayDir));
    mhEvaluate(*m, ctx, v3(wo), v3(wi), out);
    return 0;
}

int ref_mh_sample(void* sp, int h, const float* si, const float* rayDir, const float* wo, const float* u2,
                  float uc, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    auto* m = dynamic_cast<const MarschnerHairMaterial*>(s->mats[size_t(h)].get());
    if (!m) return 1;
    ShadingContext ctx(makeSI(si), v3(rayDir));
    mhSample(*m, ctx, v3(wo), Vec2f{u2[0], u2[1]}, uc, out);
    return 0;
}

// The public lobe functions (MarschnerHair.h:88-187) over n inputs of 10
// floats: cosI, sinI, cosR, sinR, v, x, s, u, h, cosO (eta and sigma_a shared).
// out per input, 16 floats: mh_Mp(cosI, sinI, cosR, sinR, v),
// mh_trimmedLogistic(x, s), mh_sampleTrimmedLogistic(u, s),
// mh_Np(x, p, s, asin(h), 0.3 h) for p = 0..2, mh_Ap(cosO, eta, h, sigma_a)
// (3 x rgb), mh_sampleGaussian(u, x / 2pi + 0.5).
void ref_mh_functions(const float* in, uint32_t n, float eta, const float* sigma_a, float* out) {
    const Spectrum sa = v3(sigma_a);
    for (uint32_t k = 0; k < n; ++k) {
        const float* q = in + 10 * size_t(k);
        float* o = out + 16 * size_t(k);
        o[0] = mh_Mp(q[0], q[1], q[2], q[3], q[4]);
        o[1] = mh_trimmedLogistic(q[5], q[6]);
        o[2] = mh_sampleTrimmedLogistic(q[7], q[6]);
        const float gO = std::asin(q[8]), gT = 0.3f * q[8];
        for (int p = 0; p < 3; ++p) o[3 + p] = mh_Np(q[5], p, q[6], gO, gT);
        auto ap = mh_Ap(q[9], eta, q[8], sa);
        for (int p = 0; p < 3; ++p) put3(o + 6 + 3 * p, ap[size_t(p)]);
        o[15] = mh_sampleGaussian(q[7], q[5] * 0.15915494f + 0.5f);
    }
}

// ---- lights ----------------------------------------------------------------
// out: Li[3], wi[3], pdf, dist
void ref_light_sample(void* sp, int h, const float* p, const float* n, const float* u2,
                      float* out) {
    auto* s = static_cast<RefScene*>(sp);
    LightSample ls = s->lights[size_t(h)]->sample(v3(p), v3(n), Vec2f{u2[0], u2[1]});
    put3(out, ls.Li);
    put3(out + 3, ls.wi);
    out[6] = ls.pdf;
    out[7] = ls.dist;
}

float ref_light_pdf(void* sp, int h, const float* p, const float* wi) {
    auto* s = static_cast<RefScene*>(sp);
    return s->lights[size_t(h)]->pdf(v3(p), v3(wi));
}

void ref_light_le(void* sp, int h, const float* wo, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    put3(out, s->lights[size_t(h)]->Le({}, {}, v3(wo)));
}

// out: pdfPos, pdfDir, dot(dir, normal), Le[3]
void ref_light_sample_le(void* sp, int h, const float* uPos, const float* uDir, float* out) {
    auto* s = static_cast<RefScene*>(sp);
    LightLeSample ls = s->lights[size_t(h)]->sampleLe({uPos[0], uPos[1]}, {uDir[0], uDir[1]});
    out[0] = ls.pdfPos;
    out[1] = ls.pdfDir;
    out[2] = dot(ls.dir, ls.normal);
    put3(out + 3, ls.Le);
}

// ---- Distribution1D ---------------------------------------------------------
// out per u: idx, pdf, uRemapped
void ref_dist1d(const float* vals, uint32_t n, const float* us, uint32_t nu, float* out,
                float* integral) {
    Distribution1D d;
    d.build(vals, n);
    *integral = d.integral;
    for (uint32_t i = 0; i < nu; ++i) {
        float pdf, ur;
        uint32_t idx = d.sample(us[i], pdf, ur);
        out[3 * i] = float(idx);
        out[3 * i + 1] = pdf;
        out[3 * i + 2] = ur;
    }
}

}  // extern "C"

// ============================================================================
// Drop-in check (built only into oracle/_ref/libanacapa_ref_dropin.so, which
// also links this repository's B200PathIntegrator and CUDA library): the
// reference's SceneView and Film driven through IIntegrator::prepare /
// renderFrame exactly as RenderSession::render's non-adaptive branch does
// (src/render/RenderSession.cpp:468, 541-547).
// ============================================================================
#ifdef ANA_DROPIN
#include "B200PathIntegrator.h"

namespace anacapa {
// Film.cpp needs OpenImageIO; the check supplies Film's accumulation members
// with the arithmetic of src/film/Film.cpp:18-90, and its EXR / PNG writers
// through this repository's (ana_image_write_exr / _png) with the layers
// Film::writeEXR resolves; denoising (OIDN) reports failure.
Film::Film(uint32_t width, uint32_t height)
    : m_width(width), m_height(height), m_pixels(width * height), m_albedo(width * height),
      m_normals(width * height) {}
void Film::splatPixel(float x, float y, Spectrum value) {
    if (!value.isFinite()) return;
    int px = int(x), py = int(y);
    if (!inBounds(px, py)) return;
    m_pixels[py * m_width + px].add(value.x, value.y, value.z, 1.f);
}
void Film::mergeTile(const TileBuffer& tile) {
    m_dirty.store(true, std::memory_order_relaxed);
    for (uint32_t ty = 0; ty < tile.height; ++ty)
        for (uint32_t tx = 0; tx < tile.width; ++tx) {
            uint32_t fx = tile.x0 + tx, fy = tile.y0 + ty;
            if (!inBounds(int(fx), int(fy))) continue;
            uint32_t fi = fy * m_width + fx, ti = ty * tile.width + tx;
            const auto& s = tile.pixels[ti];
            if (s.weight > 0.f) {
                m_pixels[fi].r.fetch_add(s.r, std::memory_order_relaxed);
                m_pixels[fi].g.fetch_add(s.g, std::memory_order_relaxed);
                m_pixels[fi].b.fetch_add(s.b, std::memory_order_relaxed);
                m_pixels[fi].weight.fetch_add(s.weight, std::memory_order_relaxed);
                m_pixels[fi].sumLumSq.fetch_add(tile.sumLumSq[ti], std::memory_order_relaxed);
            }
            const auto& a = tile.albedo[ti];
            if (a.count > 0) {
                float inv = 1.f / static_cast<float>(a.count);
                m_albedo[fi].add(a.r * inv, a.g * inv, a.b * inv, 1.f);
            }
            const auto& n = tile.normals[ti];
            if (n.count > 0) {
                float inv = 1.f / static_cast<float>(n.count);
                m_normals[fi].add(n.r * inv, n.g * inv, n.b * inv, 1.f);
            }
        }
}
Spectrum Film::getPixel(uint32_t x, uint32_t y) const { return m_pixels[y * m_width + x].resolve(); }
float Film::varianceAt(uint32_t x, uint32_t y) const {
    const auto& p = m_pixels[y * m_width + x];
    float w = p.weight.load(std::memory_order_relaxed);
    if (w <= 0.f) return 0.f;
    float invW = 1.f / w;
    float meanL = (p.r.load() * 0.2126f + p.g.load() * 0.7152f + p.b.load() * 0.0722f) * invW;
    float eLsq = p.sumLumSq.load() * invW;
    return std::max(0.f, eLsq - meanL * meanL);
}
bool Film::denoise() { return false; }
static void resolve_layer(const std::vector<PixelAccumulator>& acc, std::vector<float>& out) {
    out.resize(acc.size() * 3);
    for (size_t i = 0; i < acc.size(); ++i) {
        const Spectrum s = acc[i].resolve();
        out[3 * i] = s.x;
        out[3 * i + 1] = s.y;
        out[3 * i + 2] = s.z;
    }
}
bool Film::writeEXR(const std::string& path, const DenoiseOptions& opts) const {
    std::vector<float> rgb, al, nr;
    resolve_layer(m_pixels, rgb);
    if (opts.writeAOVs) {
        resolve_layer(m_albedo, al);
        resolve_layer(m_normals, nr);
    }
    return ana_image_write_exr(path.c_str(), m_width, m_height, rgb.data(), opts.writeAOVs ? al.data() : nullptr,
                               opts.writeAOVs ? nr.data() : nullptr) == ANA_OK;
}
bool Film::writePNG(const std::string& path, float exposure) const {
    std::vector<float> rgb;
    resolve_layer(m_pixels, rgb);
    return ana_image_write_png(path.c_str(), m_width, m_height, rgb.data(), exposure) == ANA_OK;
}
}  // namespace anacapa

extern "C" int ref_dropin_render(void* sp, uint32_t W, uint32_t H, uint32_t spp, uint32_t maxDepth,
                                 int passes, float* out_rgb, float* out_var, char* err, int errlen) {
    auto* s = static_cast<RefScene*>(sp);
    anacapa_b200::B200PathIntegrator integ(maxDepth);
    if (!integ.isValid()) {
        std::snprintf(err, size_t(errlen), "%s", integ.lastError().c_str());
        return 1;
    }
    integ.prepare(s->view);
    Film film(W, H);
    // `passes` renderFrame calls of spp samples each continue the sample
    // indices (progressive accumulation into the same Film)
    for (int k = 0; k < passes; ++k)
        if (!integ.renderFrame(s->view, W, H, uint32_t(k) * spp, spp, film)) {
            std::snprintf(err, size_t(errlen), "%s", integ.lastError().c_str());
            return 2;
        }
    for (uint32_t y = 0; y < H; ++y)
        for (uint32_t x = 0; x < W; ++x) {
            Spectrum c = film.getPixel(x, y);
            size_t i = size_t(y) * W + x;
            out_rgb[3 * i] = c.x;
            out_rgb[3 * i + 1] = c.y;
            out_rgb[3 * i + 2] = c.z;
            out_var[i] = film.varianceAt(x, y);
        }
    return 0;
}
// The drop-in's frames written by the reference Film's writers: `passes`
// renderFrame calls, then Film::writeEXR (with the AOV layers) and
// Film::writePNG.
extern "C" int ref_dropin_write(void* sp, uint32_t W, uint32_t H, uint32_t spp, uint32_t maxDepth, int passes,
                                const char* exr, const char* png, float exposure, char* err, int errlen) {
    auto* s = static_cast<RefScene*>(sp);
    anacapa_b200::B200PathIntegrator integ(maxDepth);
    if (!integ.isValid()) {
        std::snprintf(err, size_t(errlen), "%s", integ.lastError().c_str());
        return 1;
    }
    integ.prepare(s->view);
    Film film(W, H);
    for (int k = 0; k < passes; ++k)
        if (!integ.renderFrame(s->view, W, H, uint32_t(k) * spp, spp, film)) {
            std::snprintf(err, size_t(errlen), "%s", integ.lastError().c_str());
            return 2;
        }
    DenoiseOptions o;
    o.writeAOVs = true;
    if (!film.writeEXR(exr, o)) return 3;
    if (!film.writePNG(png, exposure)) return 4;
    return 0;
}

// The host half of the drop-in's prepare (no device needed): the prepared
// layout built from the reference's SceneView, for comparison with the layout
// the C ABI builds from the same scene description. Free with
// ana_prepared_free.
extern "C" void* ref_dropin_prepare(void* sp, uint32_t W, uint32_t H, char* err, int errlen) {
    auto* s = static_cast<RefScene*>(sp);
    std::string e;
    ana_prepared* p = anacapa_b200::B200PathIntegrator::prepareHost(s->view, W, H, e);
    if (!p) std::snprintf(err, size_t(errlen), "%s", e.c_str());
    return p;
}
#endif  // ANA_DROPIN
