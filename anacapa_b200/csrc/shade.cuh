// Materials, lights and the shading frame on the device. Each function
// restates the reference's float code (cited per function); results agree with
// the reference statistically (device transcendental functions differ from
// glibc's by a few ulps), while control flow, sample-dimension use and every
// branch condition follow the reference exactly.
#pragma once
#include "../../include/anacapa_b200.h"
#include "dmath.cuh"
#include "layout.h"

namespace ana {

constexpr float kPi = 3.14159265358979323846f;
constexpr float kInvPi = 0.31830988618379067154f;
constexpr float k2Pi = 6.28318530717958647692f;

constexpr uint32_t kFlagDiffuse = 1u, kFlagGlossy = 2u, kFlagSpecular = 4u;
constexpr uint32_t kFlagTransmission = 8u, kFlagReflection = 16u;

// SurfaceInteraction (include/anacapa/accel/IAccelerationStructure.h:12-30),
// the fields shading reads.
struct SurfInt {
    float3 p, n, ng, dpdu, color;
    uint32_t slot;
    bool is_curve;
};

// ShadingContext (include/anacapa/shading/ShadingContext.h:15-60).
struct ShadeCtx {
    float3 p, n, ng, t, bt, color;
    bool front;
    __device__ float3 to_local(float3 v) const { return f3(dot(v, t), dot(v, bt), dot(v, n)); }
    __device__ float3 to_world(float3 v) const { return t * v.x + bt * v.y + n * v.z; }
};

// buildOrthonormalBasis (Types.h:108-114)
__device__ __forceinline__ void onb(float3 n, float3& t, float3& b) {
    float sign = copysignf(1.f, n.z);
    float a = -1.f / (sign + n.z);
    float bb = n.x * n.y * a;
    t = f3(1.f + sign * n.x * n.x * a, sign * bb, -sign * n.x);
    b = f3(bb, sign + n.y * n.y * a, -n.y);
}

__device__ __forceinline__ ShadeCtx make_ctx(const SurfInt& si, float3 rayDir) {
    ShadeCtx c;
    c.p = si.p;
    c.color = si.color;
    c.front = dot(-rayDir, si.ng) > 0.f;
    c.n = c.front ? si.n : -si.n;
    c.ng = c.front ? si.ng : -si.ng;
    if (si.is_curve) {
        c.t = si.dpdu;
        c.bt = safe_normalize(cross(c.n, c.t));
    } else {
        onb(c.n, c.t, c.bt);
    }
    return c;
}

struct BsdfSample {
    float3 f, wi;  // f includes |cos theta_i| (IMaterial.h:26)
    float pdf;
    uint32_t flags;
    __device__ bool valid() const { return pdf > 0.f && !is_black(f); }
    __device__ bool delta() const { return (flags & kFlagSpecular) != 0; }
};

struct BsdfEval {
    float3 f;  // without the cosine
    float pdf;
};

__device__ __forceinline__ BsdfSample no_sample() {
    BsdfSample s;
    s.f = f3(0.f, 0.f, 0.f);
    s.wi = f3(0.f, 0.f, 0.f);
    s.pdf = 0.f;
    s.flags = 0;
    return s;
}

// ---- GGX helpers (StandardSurface.h:20-76) ------------------------------------
__device__ __forceinline__ float d_ggx(float cosH, float a2) {
    if (cosH <= 0.f) return 0.f;
    float denom = cosH * cosH * (a2 - 1.f) + 1.f;
    return a2 / (kPi * denom * denom);
}
__device__ __forceinline__ float g1_smith(float absCos, float a2) {
    if (absCos <= 0.f) return 0.f;
    float c2 = absCos * absCos;
    return 2.f * absCos / (absCos + sqrtf(a2 + (1.f - a2) * c2));
}
__device__ __forceinline__ float g2_sep(float cosO, float cosI, float a2) {
    return g1_smith(fabsf(cosO), a2) * g1_smith(fabsf(cosI), a2);
}
__device__ __forceinline__ float3 sample_ggx_h(float ux, float uy, float a2) {
    float phi = 2.f * kPi * ux;
    float cosH2 = (1.f - uy) / fmaxf(1.f + (a2 - 1.f) * uy, 1e-10f);
    float cosH = sqrtf(fmaxf(0.f, cosH2));
    float sinH = sqrtf(fmaxf(0.f, 1.f - cosH2));
    float sp, cp;
    sincosf(phi, &sp, &cp);
    return f3(sinH * cp, sinH * sp, cosH);
}
__device__ __forceinline__ float pdf_ggx_refl(float cosH, float a2, float dotVH) {
    if (cosH <= 0.f || dotVH <= 0.f) return 0.f;
    return d_ggx(cosH, a2) * cosH / (4.f * dotVH);
}
__device__ __forceinline__ float schlick_d(float c, float f0) {
    float x = 1.f - fabsf(c);
    float x5 = x * x * x * x * x;
    return f0 + (1.f - f0) * x5;
}
__device__ __forceinline__ float3 schlick_c(float c, float3 f0) {
    float x = 1.f - fabsf(c);
    float x5 = x * x * x * x * x;
    return f0 + (f3(1.f, 1.f, 1.f) - f0) * x5;
}
__device__ __forceinline__ float fresnel_dielectric(float cosI, float eta) {
    float sin2I = fmaxf(0.f, 1.f - cosI * cosI);
    float sin2T = sin2I / (eta * eta);
    if (sin2T >= 1.f) return 1.f;
    float cosT = sqrtf(1.f - sin2T);
    float Rs = (cosI - eta * cosT) / (cosI + eta * cosT);
    float Rp = (eta * cosI - cosT) / (eta * cosI + cosT);
    return 0.5f * (Rs * Rs + Rp * Rp);
}

// ---- Lambert (Lambertian.h:12-82) -----------------------------------------------
__device__ __forceinline__ BsdfSample lambert_sample(const DevMaterial& m, const ShadeCtx& c, float3 wo,
                                                     float ux, float uy) {
    float r = sqrtf(ux);
    float phi = 2.f * kPi * uy;
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float3 wl = f3(r * cp, r * sp, sqrtf(fmaxf(0.f, 1.f - ux)));
    if (c.to_local(wo).z < 0.f) wl.z = -wl.z;
    BsdfSample s;
    s.wi = c.to_world(wl);
    s.pdf = fmaxf(0.f, fabsf(wl.z)) * kInvPi;
    s.f = m.albedo * (kInvPi * fabsf(wl.z));
    s.flags = kFlagDiffuse | kFlagReflection;
    return s;
}
__device__ __forceinline__ BsdfEval lambert_eval(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    float3 wil = c.to_local(wi), wol = c.to_local(wo);
    BsdfEval e{f3(0.f, 0.f, 0.f), 0.f};
    if (!(wil.z * wol.z > 0.f)) return e;
    e.f = m.albedo * kInvPi;
    e.pdf = fmaxf(0.f, fabsf(wil.z)) * kInvPi;
    return e;
}

// ---- standard_surface, opaque branch (StandardSurface.h:231-661) -------------
struct LobeWeights {
    float coat, metal, spec, diff;
};

__device__ __forceinline__ bool ss_weights(const DevMaterial& m, float cosO, LobeWeights& w) {
    float coatF = schlick_d(cosO, m.coat_f0);
    float specF = schlick_d(cosO, m.f0_dielectric);
    w.coat = m.coat * coatF;
    w.metal = m.metal * (1.f - w.coat);
    w.spec = m.spec * (1.f - m.metal) * specF * (1.f - w.coat);
    w.diff = m.base * (1.f - m.metal) * (1.f - m.spec * specF) * (1.f - w.coat);
    float sum = w.coat + w.metal + w.spec + w.diff;
    if (sum <= 0.f) return false;
    float inv = 1.f / sum;
    w.coat *= inv;
    w.metal *= inv;
    w.spec *= inv;
    w.diff *= inv;
    return true;
}

// evalGGX: BSDF value without cosine and forward pdf.
__device__ __forceinline__ float3 eval_ggx(float3 wol, float3 wil, float a2, float3 F0, float& pdf) {
    pdf = 0.f;
    if (wol.z <= 0.f || wil.z <= 0.f) return f3(0.f, 0.f, 0.f);
    float3 wh = safe_normalize(wol + wil);
    if (wh.z <= 0.f) return f3(0.f, 0.f, 0.f);
    float dotVH = fmaxf(0.f, dot(wol, wh));
    float3 F = schlick_c(dotVH, F0);
    float D = d_ggx(wh.z, a2);
    float G2 = g2_sep(wol.z, wil.z, a2);
    float cosO = fabsf(wol.z), cosI = fabsf(wil.z);
    if (cosO < 1e-6f || cosI < 1e-6f) return f3(0.f, 0.f, 0.f);
    float3 bsdf = F * (D * G2 / (4.f * cosO * cosI));
    pdf = pdf_ggx_refl(wh.z, a2, dotVH);
    return bsdf;
}

__device__ __forceinline__ float3 ss_combined(const DevMaterial& m, float3 wol, float3 wil, const LobeWeights& w,
                                              float& pdf) {
    float3 f = f3(0.f, 0.f, 0.f);
    pdf = 0.f;
    if (!(wol.z * wil.z > 0.f)) return f;
    if (w.coat > 0.f) {
        float p;
        float3 fc = eval_ggx(wol, wil, m.coat_alpha2, f3(m.coat_f0, m.coat_f0, m.coat_f0), p);
        f = f + fc * w.coat;
        pdf += p * w.coat;
    }
    if (w.metal > 0.f) {
        float p;
        float3 fm = eval_ggx(wol, wil, m.alpha2, m.albedo * m.base, p);
        f = f + fm * w.metal;
        pdf += p * w.metal;
    }
    if (w.spec > 0.f) {
        float p;
        float3 fs = eval_ggx(wol, wil, m.alpha2, m.spec_color * (m.spec * m.f0_dielectric), p);
        f = f + fs * w.spec;
        pdf += p * w.spec;
    }
    if (w.diff > 0.f) {
        float cosI = fabsf(wil.z);
        f = f + (m.albedo * m.base * kInvPi) * w.diff;
        pdf += cosI * kInvPi * w.diff;
    }
    return f;
}

// sampleGGX (StandardSurface.h:516-549): direction and validity.
__device__ __forceinline__ bool ss_sample_ggx(float3 wol, float ux, float uy, float a2, float3 F0,
                                              float3& wil) {
    float3 wh = sample_ggx_h(ux, uy, a2);
    if (wh.z <= 0.f) return false;
    float dotVH = dot(wol, wh);
    if (dotVH <= 0.f) return false;
    wil = wh * (2.f * dotVH) - wol;
    if (wil.z <= 0.f) return false;
    float3 F = schlick_c(dotVH, F0);
    float D = d_ggx(wh.z, a2);
    float G2 = g2_sep(wol.z, wil.z, a2);
    float cosO = fabsf(wol.z), cosI = fabsf(wil.z);
    if (cosO < 1e-6f || cosI < 1e-6f) return false;
    float3 f = F * (D * G2 / (4.f * cosO)) * cosI;
    float pdf = pdf_ggx_refl(wh.z, a2, dotVH);
    return pdf > 0.f && !is_black(f);
}

// ---- standard_surface glass (StandardSurface.h:245-340) --------------------
// The sample path of a transmissive non-metal: Fresnel chooses between mirror
// reflection and Snell refraction (roughness < 0.001, delta), or between GGX
// reflection and Walter et al. microfacet refraction about a sampled
// half-vector. eta = IOR entering the front face, 1/IOR leaving; f carries
// |cos| (importance transport, no eta^2).
__device__ __forceinline__ bool ss_glass(const DevMaterial& m) { return m.transmission > 0.001f && m.metal < 0.001f; }

__device__ __forceinline__ BsdfSample glass_sample(const DevMaterial& m, const ShadeCtx& c, float3 wol, float ux,
                                                   float uy, float uc) {
    const float eta = c.front ? m.ior : (1.f / m.ior);
    BsdfSample s;
    if (m.rough < 0.001f) {
        const float cosI = wol.z;
        const float Fr = fresnel_dielectric(cosI, eta);
        if (uc < Fr) {
            s.wi = c.to_world(f3(-wol.x, -wol.y, wol.z));
            s.f = m.albedo * Fr;
            s.pdf = Fr;
            s.flags = kFlagSpecular | kFlagReflection;
        } else {
            const float sin2T = fmaxf(0.f, 1.f - cosI * cosI) / (eta * eta);
            const float cosT = sqrtf(fmaxf(0.f, 1.f - sin2T));
            s.wi = c.to_world(f3(-wol.x / eta, -wol.y / eta, -cosT));
            s.f = m.albedo * (1.f - Fr);
            s.pdf = 1.f - Fr;
            s.flags = kFlagSpecular | kFlagTransmission;
        }
        return s;
    }
    const float a2 = m.alpha2;
    const float3 wh = sample_ggx_h(ux, uy, a2);
    if (wh.z <= 0.f) return no_sample();
    const float cosIH = fmaxf(0.f, dot(wol, wh));
    if (cosIH <= 0.f) return no_sample();
    const float Fr = fresnel_dielectric(cosIH, eta);
    if (uc < Fr) {
        const float3 wil = wh * (2.f * cosIH) - wol;
        if (wil.z <= 0.f) return no_sample();
        const float D = d_ggx(wh.z, a2);
        const float G2 = g2_sep(wol.z, wil.z, a2);
        s.wi = c.to_world(wil);
        s.f = f3(Fr, Fr, Fr) * (D * G2 / (4.f * wol.z)) * m.albedo;
        s.pdf = Fr * pdf_ggx_refl(wh.z, a2, cosIH);
        s.flags = kFlagGlossy | kFlagReflection;
        return s;
    }
    const float sin2T = fmaxf(0.f, 1.f - cosIH * cosIH) / (eta * eta);
    if (sin2T >= 1.f) return no_sample();  // total internal reflection
    const float cosTH = sqrtf(1.f - sin2T);
    const float3 wil = wol * (-1.f / eta) + wh * (cosIH / eta - cosTH);
    if (wil.z >= 0.f) return no_sample();
    const float cosO = wol.z;
    const float D = d_ggx(wh.z, a2);
    const float G2 = g2_sep(cosO, fabsf(wil.z), a2);
    const float denom = cosIH + eta * fabsf(dot(wil, wh));
    if (denom < 1e-6f) return no_sample();
    const float absT = fabsf(dot(wil, wh));
    const float jac = eta * eta * absT / (denom * denom);
    s.wi = c.to_world(wil);
    s.f = m.albedo * ((1.f - Fr) * D * G2 * cosIH * absT / (cosO * denom * denom));
    s.pdf = (1.f - Fr) * (D * wh.z) * jac;
    s.flags = kFlagGlossy | kFlagTransmission;
    return s;
}

// evaluate() of glass (StandardSurface.h:380-438): the microfacet
// transmission lobe for directions on opposite sides (its alpha2 unclamped),
// Fresnel-weighted GGX reflection on the same side; smooth glass has no
// finite density.
__device__ __forceinline__ BsdfEval glass_eval_t(const DevMaterial& m, const ShadeCtx& c, float3 wol, float3 wil) {
    BsdfEval e{f3(0.f, 0.f, 0.f), 0.f};
    if (m.transmission < 0.001f || m.rough < 0.001f || m.metal > 0.001f) return e;
    const float eta = c.front ? m.ior : (1.f / m.ior);
    const float a2 = m.alpha2_t;
    float3 wh = safe_normalize(wol + wil * eta);
    if (wh.z < 0.f) wh = -wh;
    const float cosIH = fmaxf(0.f, dot(wol, wh));
    const float cosTH = fabsf(dot(wil, wh));
    const float Fr = fresnel_dielectric(cosIH, eta);
    const float D = d_ggx(wh.z, a2);
    const float G2 = g2_sep(wol.z, fabsf(wil.z), a2);
    const float denom = cosIH + eta * cosTH;
    if (denom < 1e-6f) return e;
    const float bsdf = (1.f - Fr) * D * G2 * cosIH * cosTH / (wol.z * fabsf(wil.z) * denom * denom);
    const float jac = eta * eta * cosTH / (denom * denom);
    e.f = m.albedo * bsdf;
    e.pdf = (1.f - Fr) * D * wh.z * jac;
    return e;
}
__device__ __forceinline__ BsdfEval glass_eval_r(const DevMaterial& m, const ShadeCtx& c, float3 wol, float3 wil) {
    BsdfEval e{f3(0.f, 0.f, 0.f), 0.f};
    if (m.rough < 0.001f) return e;
    const float eta = c.front ? m.ior : (1.f / m.ior);
    const float a2 = m.alpha2;
    const float3 wh = safe_normalize(wol + wil);
    if (wh.z < 0.f) return e;
    const float cosIH = fmaxf(0.f, dot(wol, wh));
    const float Fr = fresnel_dielectric(cosIH, eta);
    const float D = d_ggx(wh.z, a2);
    const float G2 = g2_sep(wol.z, wil.z, a2);
    const float cosR = wil.z;
    e.pdf = Fr > 0.f ? Fr * pdf_ggx_refl(wh.z, a2, cosIH) : 0.f;
    e.f = m.albedo * (Fr * D * G2 / (4.f * wol.z * cosR));
    return e;
}

// kGlass = false compiles the glass lobes out (batches without transmission).
template <bool kGlass = true>
__device__ __forceinline__ BsdfSample ss_sample(const DevMaterial& m, const ShadeCtx& c, float3 wo, float ux,
                                                float uy, float uc) {
    float3 wol = c.to_local(wo);
    if (wol.z <= 0.f) return no_sample();
    if (kGlass && ss_glass(m)) return glass_sample(m, c, wol, ux, uy, uc);
    LobeWeights w;
    if (!ss_weights(m, wol.z, w)) return no_sample();
    float3 wil;
    bool ok;
    if (uc < w.coat) {
        ok = ss_sample_ggx(wol, ux, uy, m.coat_alpha2, f3(m.coat_f0, m.coat_f0, m.coat_f0), wil);
    } else if (uc < w.coat + w.metal) {
        ok = ss_sample_ggx(wol, ux, uy, m.alpha2, m.albedo * m.base, wil);
    } else if (uc < w.coat + w.metal + w.spec) {
        ok = ss_sample_ggx(wol, ux, uy, m.alpha2, m.spec_color * (m.spec * m.f0_dielectric), wil);
    } else {
        // sampleDiffuse (StandardSurface.h:554-573)
        float phi = 2.f * kPi * ux;
        float r = sqrtf(uy);
        float z = sqrtf(fmaxf(0.f, 1.f - uy));
        float sp, cp;
        sincosf(phi, &sp, &cp);
        wil = f3(r * cp, r * sp, z);
        if (wol.z < 0.f) wil.z = -wil.z;
        float cosI = fabsf(wil.z);
        float p = cosI * kInvPi;
        float3 f = m.albedo * m.base * (kInvPi * cosI);
        ok = p > 0.f && !is_black(f);
    }
    if (!ok) return no_sample();
    BsdfSample s;
    s.wi = c.to_world(wil);
    float3 wl2 = c.to_local(s.wi);
    float pdf;
    float3 fc = ss_combined(m, wol, wl2, w, pdf);
    s.f = fc * fabsf(wl2.z);
    s.pdf = pdf;
    s.flags = m.flags;
    return s;
}

template <bool kGlass = true>
__device__ __forceinline__ BsdfEval ss_eval(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    float3 wol = c.to_local(wo), wil = c.to_local(wi);
    BsdfEval e{f3(0.f, 0.f, 0.f), 0.f};
    if (!(wol.z * wil.z > 0.f)) return kGlass ? glass_eval_t(m, c, wol, wil) : e;  // opaque: black
    if (kGlass && ss_glass(m)) return glass_eval_r(m, c, wol, wil);
    LobeWeights w;
    if (!ss_weights(m, wol.z, w)) return e;
    e.f = ss_combined(m, wol, wil, w, e.pdf);
    return e;
}

// ---- hair (MarschnerHair.h) ------------------------------------------------------
// effectiveSigmaA (MarschnerHair.h:430-450)
__device__ __forceinline__ float3 hair_sigma(const DevMaterial& m, float3 c) {
    if (c.x > 0.98f && c.y > 0.98f && c.z > 0.98f) return m.sigma_a;
    float lr = powf(fmaxf(c.x, 0.f), 2.2f), lg = powf(fmaxf(c.y, 0.f), 2.2f),
          lb = powf(fmaxf(c.z, 0.f), 2.2f);
    if (lr < 0.01f && lg < 0.01f && lb < 0.01f) return m.sigma_a;
    return f3(-logf(fmaxf(lr, 0.001f)), -logf(fmaxf(lg, 0.001f)), -logf(fmaxf(lb, 0.001f)));
}

// kajiyaKayEval (MarschnerHair.h:395-422)
__device__ __forceinline__ BsdfEval kk_eval(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    float3 sa = hair_sigma(m, c.color);
    float3 alb = f3(expf(-sa.x), expf(-sa.y), expf(-sa.z));
    float dTL = dot(c.t, wi), dTV = dot(c.t, wo);
    float sTL = sqrtf(fmaxf(0.f, 1.f - dTL * dTL)), sTV = sqrtf(fmaxf(0.f, 1.f - dTV * dTV));
    float3 f = alb * kInvPi;
    float spec = dTL * dTV + sTL * sTV;
    if (spec > 0.f) f = f + f3(0.15f, 0.15f, 0.15f) * (powf(spec, 20.f) * kInvPi);
    BsdfEval e;
    e.f = f;
    e.pdf = fmaxf(0.f, dot(wi, c.n)) * kInvPi;
    return e;
}

// Kajiya-Kay sample about the ribbon normal (MarschnerHair.h:267-282)
__device__ __forceinline__ BsdfSample kk_sample(const DevMaterial& m, const ShadeCtx& c, float3 wo, float ux,
                                                float uy) {
    float3 t, b;
    onb(c.n, t, b);
    float phi = k2Pi * ux;
    float cT = sqrtf(uy), sT = sqrtf(1.0f - uy);
    float sp, cp;
    sincosf(phi, &sp, &cp);
    float3 wi = safe_normalize(t * (sT * cp) + b * (sT * sp) + c.n * cT);
    BsdfEval ev = kk_eval(m, c, wo, wi);
    BsdfSample s;
    s.wi = wi;
    s.f = ev.f * cT;
    s.pdf = cT * kInvPi;
    s.flags = kFlagDiffuse | kFlagReflection;
    return s;
}

// -- Marschner R/TT/TRT lobes (MarschnerHair.h:49-185, 284-375, 457-556) --
__device__ __forceinline__ float mh_I0(float x) {
    float sum = 0.f, x2i = 1.f, den = 1.f;
    for (int i = 0; i < 12; ++i) {
        if (i > 0) {
            x2i *= x * x;
            den *= float(i) * float(i) * 4.f;
        }
        sum += x2i / den;
    }
    return sum;
}
__device__ __forceinline__ float mh_logI0(float x) {
    if (x > 12.f) return x + 0.5f * (-logf(k2Pi) + logf(1.f / x) + 1.f / (8.f * x));
    return logf(mh_I0(x));
}
__device__ __forceinline__ float mh_Mp(float cosI, float sinI, float cosR, float sinR, float v) {
    if (v < 1e-5f) v = 1e-5f;
    float a = cosI * cosR / v, b = sinI * sinR / v;
    if (v <= 0.1f) return expf(mh_logI0(a) - b - 1.f / v + 0.6931472f + logf(0.5f / v));
    return expf(-b) * mh_I0(a) / (2.f * v * sinhf(1.f / v));
}
__device__ __forceinline__ float mh_logistic(float x, float s) {
    float ex = expf(-fabsf(x) / s);
    return ex / (s * (1.f + ex) * (1.f + ex));
}
__device__ __forceinline__ float mh_logistic_cdf(float x, float s) { return 1.f / (1.f + expf(-x / s)); }
__device__ __forceinline__ float mh_trimmed(float x, float s) {
    float norm = mh_logistic_cdf(kPi, s) - mh_logistic_cdf(-kPi, s);
    return mh_logistic(x, s) / norm;
}
__device__ __forceinline__ float mh_sample_trimmed(float u, float s) {
    float a = mh_logistic_cdf(-kPi, s), b = mh_logistic_cdf(kPi, s);
    float x = -s * logf(1.f / (a + u * (b - a)) - 1.f);
    return fminf(fmaxf(x, -kPi), kPi);
}
__device__ __forceinline__ float mh_Phi(int p, float gO, float gT) {
    return 2.f * float(p) * gT - 2.f * gO + float(p) * kPi;
}
__device__ __forceinline__ float mh_wrap(float x) {
    for (int i = 0; i < 64 && x > kPi; ++i) x -= k2Pi;
    for (int i = 0; i < 64 && x < -kPi; ++i) x += k2Pi;
    return x;
}
__device__ __forceinline__ float mh_Np(float phi, int p, float s, float gO, float gT) {
    return mh_trimmed(mh_wrap(phi - mh_Phi(p, gO, gT)), s);
}
__device__ __forceinline__ void mh_Ap(float cosO, float eta, float h, float3 sa, float3 ap[3]) {
    float sin2O = fmaxf(0.f, 1.f - cosO * cosO);
    float etaP = sqrtf(fmaxf(0.f, eta * eta - sin2O)) / cosO;
    float sGT = fminf(fmaxf(h / (etaP > 1e-5f ? etaP : 1e-5f), -1.f + 1e-5f), 1.f - 1e-5f);
    float cGT = sqrtf(fmaxf(0.f, 1.f - sGT * sGT));
    float3 T = f3(expf(-sa.x * 2.f * cGT), expf(-sa.y * 2.f * cGT), expf(-sa.z * 2.f * cGT));
    float cGO = sqrtf(fmaxf(0.f, 1.f - h * h));
    float cosA = fmaxf(0.f, cosO * cGO);
    float fr = fresnel_dielectric(cosA, eta);
    ap[0] = f3(fr, fr, fr);
    ap[1] = T * ((1.f - fr) * (1.f - fr));
    ap[2] = ap[1] * T * fr;
}
__device__ __forceinline__ void hair_long(float3 d, float3 t, float& s, float& c) {
    s = dot(d, t);
    c = sqrtf(fmaxf(0.f, 1.f - s * s));
}
__device__ __forceinline__ float hair_phi(float3 wo, float3 wi, float3 t, float sO, float sI) {
    float3 op = wo - t * sO, ip = wi - t * sI;
    float lo = length(op), li = length(ip);
    if (lo < 1e-5f || li < 1e-5f) return 0.f;
    op = op * (1.f / lo);
    ip = ip * (1.f / li);
    float c = fminf(fmaxf(dot(op, ip), -1.f), 1.f);
    float s = dot(cross(ip, op), t);
    return atan2f(s, c);
}
__device__ __forceinline__ float hair_h(float3 wo, float3 t, float3 n, float sO) {
    float3 op = wo - t * sO;
    float lp = length(op);
    if (lp < 1e-5f) return 0.f;
    return fminf(fmaxf(dot(op * (1.f / lp), n), -1.f + 1e-5f), 1.f - 1e-5f);
}
__device__ __forceinline__ void mh_gammas(const DevMaterial& m, float cosO, float h, float& gO, float& gT) {
    float sin2O = 1.f - cosO * cosO;
    float etaP = sqrtf(fmaxf(0.f, m.eta * m.eta - sin2O)) / cosO;
    gO = asinf(fminf(fmaxf(h, -1.f + 1e-5f), 1.f - 1e-5f));
    float sGT = fminf(fmaxf(h / (etaP > 1e-5f ? etaP : 1e-5f), -1.f + 1e-5f), 1.f - 1e-5f);
    gT = asinf(sGT);
}
// The R/TT/TRT lobe sum and its sampling pdf for the same directions
// (evalLobes and evalPdf, MarschnerHair.h:490-556) in one pass: the gammas,
// the attenuations and each lobe's Mp and Np are computed once for both, with
// the reference's operations for each (two separate functions measured 84.0
// against 48.1 ms for the shade stage of the 1280x720x32 hair frame in
// Marschner mode).
__device__ __forceinline__ float3 mh_lobes_pdf(const DevMaterial& m, float sO, float cO, float sI, float cI,
                                               float phi, float h, float3 sa, float& pdfOut) {
    float cD = sqrtf(fmaxf(0.f, 0.5f * (1.f + cO * cI + sO * sI)));
    float den = fmaxf(0.25f, cD * cD);
    float gO, gT;
    mh_gammas(m, cO, h, gO, gT);
    float3 ap[3];
    mh_Ap(cO, m.eta, h, sa, ap);
    float w[3] = {luminance(ap[0]), luminance(ap[1]), luminance(ap[2])};
    float tot = w[0] + w[1] + w[2];
    float3 fs = f3(0.f, 0.f, 0.f);
    float pdf = 0.f;
    for (int p = 0; p < 3; ++p) {
        float sOs = sO * cosf(2.f * m.alpha_shift[p]) + cO * sinf(2.f * m.alpha_shift[p]);
        float cOs = sqrtf(fmaxf(0.f, 1.f - sOs * sOs));
        float mp = mh_Mp(cI, sI, cOs, sOs, m.v[p]);
        float np = mh_Np(phi, p, m.s, gO, gT);
        fs = fs + ap[p] * (mp * np);
        float mpc = mp * cI;
        pdf += (w[p] / tot) * mpc * np;
    }
    pdfOut = tot < 1e-8f ? 0.f : fmaxf(0.f, pdf);
    return fs * (1.f / den);
}
__device__ __forceinline__ BsdfEval marschner_eval(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    float sO, cO, sI, cI;
    hair_long(wo, c.t, sO, cO);
    hair_long(wi, c.t, sI, cI);
    float phi = hair_phi(wo, wi, c.t, sO, sI);
    float h = hair_h(wo, c.t, c.n, sO);
    float3 sa = hair_sigma(m, c.color);
    BsdfEval e;
    e.f = mh_lobes_pdf(m, sO, cO, sI, cI, phi, h, sa, e.pdf);
    return e;
}
__device__ __forceinline__ BsdfSample marschner_sample(const DevMaterial& m, const ShadeCtx& c, float3 wo,
                                                       float ux, float uy, float uc) {
    float sO, cO;
    hair_long(wo, c.t, sO, cO);
    float h = hair_h(wo, c.t, c.n, sO);
    float3 sa = hair_sigma(m, c.color);
    float3 ap[3];
    mh_Ap(cO, m.eta, h, sa, ap);
    float w[3] = {luminance(ap[0]), luminance(ap[1]), luminance(ap[2])};
    float tot = w[0] + w[1] + w[2];
    if (tot < 1e-8f) return no_sample();
    float inv = 1.f / tot;
    float cdf0 = w[0] * inv, cdf1 = cdf0 + w[1] * inv, cdf2 = 1.f;
    int lobe = 0;
    float ur = uc;
    if (uc < cdf0) {
        ur = uc / cdf0;
    } else if (uc < cdf1) {
        lobe = 1;
        ur = (uc - cdf0) / (cdf1 - cdf0);
    } else {
        lobe = 2;
        ur = (uc - cdf1) / (cdf2 - cdf1);
    }
    float thO = asinf(fminf(fmaxf(sO, -1.f + 1e-5f), 1.f - 1e-5f));
    float u1 = fmaxf(ux, 1e-6f);
    float z = sqrtf(-2.f * logf(u1)) * cosf(k2Pi * uy);
    float thI = thO + m.alpha_shift[lobe] + z * sqrtf(m.v[lobe]);
    thI = fminf(fmaxf(thI, -kPi * 0.5f), kPi * 0.5f);
    float sI = sinf(thI), cI = cosf(thI);
    float gO, gT;
    mh_gammas(m, cO, h, gO, gT);
    float phiS = mh_sample_trimmed(ur, m.s) + mh_Phi(lobe, gO, gT);
    float3 wop = safe_normalize(wo - c.t * sO);
    if (length_sq(wop) < 1e-8f) {
        float3 d;
        onb(c.t, wop, d);
    }
    float3 ctp = cross(c.t, wop);
    float sp, cp;
    sincosf(phiS, &sp, &cp);
    float3 wi = safe_normalize(c.t * sI + wop * (cI * cp) + ctp * (cI * sp));
    float sIa, cIa;
    hair_long(wi, c.t, sIa, cIa);
    float phA = hair_phi(wo, wi, c.t, sO, sIa);
    float pd;
    float3 f = mh_lobes_pdf(m, sO, cO, sIa, cIa, phA, h, sa, pd);
    if (pd < 1e-8f) return no_sample();
    BsdfSample s;
    s.wi = wi;
    s.f = f * fabsf(dot(wi, c.n));
    s.pdf = pd;
    s.flags = kFlagGlossy | kFlagReflection | kFlagTransmission;
    return s;
}

// ---- material dispatch (IMaterial.h:53-114) ------------------------------------
// kHair = false compiles the hair BSDFs out, for batches without hair
// materials (smaller shading kernels: fewer registers, fewer i-cache misses).
// kFeat: the kFeat* material classes compiled in (the others return no sample
// / a zero BSDF; the host picks a kernel whose set covers the scene's).
template <bool kHair = true, bool kGlass = true, uint32_t kFeat = kFeatAll>
__device__ __forceinline__ BsdfSample mat_sample(const DevMaterial& m, const ShadeCtx& c, float3 wo, float ux,
                                                 float uy, float uc) {
    switch (m.type) {
        case ANA_MAT_LAMBERT:
        case ANA_MAT_EMISSIVE:
            if constexpr ((kFeat & kFeatLambert) != 0) return lambert_sample(m, c, wo, ux, uy);
            else return no_sample();
        case ANA_MAT_STANDARD:
            if constexpr ((kFeat & kFeatStandard) != 0) return ss_sample<kGlass>(m, c, wo, ux, uy, uc);
            else return no_sample();
        default:
            if constexpr (kHair)
                return m.hair_mode == ANA_HAIR_MARSCHNER ? marschner_sample(m, c, wo, ux, uy, uc)
                                                         : kk_sample(m, c, wo, ux, uy);
            else
                return no_sample();
    }
}
template <bool kHair = true, bool kGlass = true, uint32_t kFeat = kFeatAll>
__device__ __forceinline__ BsdfEval mat_eval(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    switch (m.type) {
        case ANA_MAT_LAMBERT:
        case ANA_MAT_EMISSIVE:
            if constexpr ((kFeat & kFeatLambert) != 0) return lambert_eval(m, c, wo, wi);
            else return BsdfEval{f3(0.f, 0.f, 0.f), 0.f};
        case ANA_MAT_STANDARD:
            if constexpr ((kFeat & kFeatStandard) != 0) return ss_eval<kGlass>(m, c, wo, wi);
            else return BsdfEval{f3(0.f, 0.f, 0.f), 0.f};
        default:
            if constexpr (kHair)
                return m.hair_mode == ANA_HAIR_MARSCHNER ? marschner_eval(m, c, wo, wi) : kk_eval(m, c, wo, wi);
            else
                return BsdfEval{f3(0.f, 0.f, 0.f), 0.f};
    }
}
// IMaterial::Le: Emissive returns its emission on both sides; standard_surface
// returns emission_color * emission; Lambert and hair emit nothing.
__device__ __forceinline__ float3 mat_le(const DevMaterial& m) { return m.emission; }

// ---- parameter derivatives of the BSDF value (path-replay adjoint) -------------
// The pieces of eval_ggx that depend on alpha2: the Schlick weight
// x5 = (1 - dot(wo, h))^5, dg = D G2 / (4 cosO cosI), and d(dg)/d(alpha2) from
//   dD/da2  = (den - 2 a2 cosH^2) / (pi den^3),  den = cosH^2 (a2 - 1) + 1
//   dG1/da2 = -c (1 - c^2) / (s (c + s)^2),       s = sqrt(a2 + (1 - a2) c^2)
// under the same validity tests as eval_ggx (false where it returns zero).
__device__ __forceinline__ bool ggx_parts(float3 wol, float3 wil, float a2, float& x5, float& dg, float& ddg) {
    if (wol.z <= 0.f || wil.z <= 0.f) return false;
    float3 wh = safe_normalize(wol + wil);
    if (wh.z <= 0.f) return false;
    const float dotVH = fmaxf(0.f, dot(wol, wh));
    const float cosO = fabsf(wol.z), cosI = fabsf(wil.z);
    if (cosO < 1e-6f || cosI < 1e-6f) return false;
    const float x = 1.f - dotVH;
    x5 = x * x * x * x * x;
    const float c2 = wh.z * wh.z;
    const float den = c2 * (a2 - 1.f) + 1.f;
    const float D = a2 / (kPi * den * den);
    const float dD = (den - 2.f * a2 * c2) / (kPi * den * den * den);
    auto g1 = [a2](float c, float& g, float& dgc) {
        const float cc = c * c, s = sqrtf(a2 + (1.f - a2) * cc);
        g = 2.f * c / (c + s);
        dgc = -c * (1.f - cc) / (s * (c + s) * (c + s));
    };
    float gO, dgO, gI, dgI;
    g1(cosO, gO, dgO);
    g1(cosI, gI, dgI);
    const float inv = 1.f / (4.f * cosO * cosI);
    dg = D * gO * gI * inv;
    ddg = (dD * gO * gI + D * (dgO * gI + gO * dgI)) * inv;
    return true;
}

// f(wo, wi) as mat_eval returns it (no cosine), with its derivatives by the
// material's albedo (per channel: f_c depends on albedo_c alone) and by its
// GGX roughness r. Lambert / emissive: f = albedo / pi. standard_surface: the
// lobe weights depend on neither parameter; the metal lobe's Schlick F0 =
// albedo * base and the diffuse lobe are affine in albedo; r enters the metal
// and dielectric-specular lobes through alpha2 = max(1e-4, r^2)^2, so
// d alpha2 / dr = 4 r^3 above the clamp and 0 below it. Hair has no
// differentiable parameter here: both derivatives are zero.
struct BsdfGrad {
    float3 f, dfda, dfdr;
};
template <bool kHair = true>
__device__ __forceinline__ BsdfGrad mat_grad(const DevMaterial& m, const ShadeCtx& c, float3 wo, float3 wi) {
    BsdfGrad g{f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f), f3(0.f, 0.f, 0.f)};
    const float3 wol = c.to_local(wo), wil = c.to_local(wi);
    if (m.type == ANA_MAT_HAIR) {
        g.f = mat_eval<kHair>(m, c, wo, wi).f;
        return g;
    }
    if (!(wol.z * wil.z > 0.f)) return g;
    if (m.type != ANA_MAT_STANDARD) {
        g.f = m.albedo * kInvPi;
        g.dfda = f3(kInvPi, kInvPi, kInvPi);
        return g;
    }
    LobeWeights w;
    if (!ss_weights(m, wol.z, w)) return g;
    float pdf;
    g.f = ss_combined(m, wol, wil, w, pdf);
    const float r = m.rough;
    const float dA2 = r * r > 1e-4f ? 4.f * r * r * r : 0.f;
    float x5, dg, ddg;
    if ((w.metal > 0.f || w.spec > 0.f) && ggx_parts(wol, wil, m.alpha2, x5, dg, ddg)) {
        const float3 one = f3(1.f, 1.f, 1.f);
        if (w.metal > 0.f) {
            const float3 F0 = m.albedo * m.base;
            const float3 F = F0 + (one - F0) * x5;
            g.dfda = g.dfda + one * (w.metal * m.base * (1.f - x5) * dg);
            g.dfdr = g.dfdr + F * (w.metal * ddg * dA2);
        }
        if (w.spec > 0.f) {
            const float3 F0 = m.spec_color * (m.spec * m.f0_dielectric);
            const float3 F = F0 + (one - F0) * x5;
            g.dfdr = g.dfdr + F * (w.spec * ddg * dA2);
        }
    }
    if (w.diff > 0.f) {
        const float k = m.base * kInvPi * w.diff;
        g.dfda = g.dfda + f3(k, k, k);
    }
    return g;
}

// ---- lights ------------------------------------------------------------------------
struct LightSample {
    float3 Li, wi;
    float pdf, dist;
    bool delta;  // LightSample::isDelta: MIS weight 1
};

// Distribution1D::sample (DomeLight.h:167-181): lower_bound over the cdf.
__device__ __forceinline__ uint32_t dist_sample(const float* func, const float* cdf, uint32_t n, float integral,
                                                float u, float& pdf, float& ur) {
    // first index i in [0, n] with cdf[i] >= u
    uint32_t lo = 0, cnt = n + 1;
    while (cnt > 0) {
        uint32_t step = cnt >> 1;
        uint32_t mid = lo + step;
        if (__ldg(cdf + mid) < u) {
            lo = mid + 1;
            cnt -= step + 1;
        } else {
            cnt = step;
        }
    }
    int idx = int(lo) - 1;
    idx = max(0, min(idx, int(n) - 1));
    float c0 = __ldg(cdf + idx), c1 = __ldg(cdf + idx + 1);
    float bw = c1 - c0;
    ur = bw > 1e-12f ? (u - c0) / bw : 0.f;
    ur = fmaxf(0.f, fminf(ur, 1.f - 1e-7f));
    pdf = integral > 0.f ? __ldg(func + idx) / integral : 0.f;
    return uint32_t(idx);
}

// DomeLight::evalEnvmap (DomeLight.h:453-491), identity rotation.
__device__ __forceinline__ float3 env_eval(const DevEnv& E, float3 wo) {
    if (!E.rgb) return E.radiance;
    float theta = acosf(fmaxf(-1.f, fminf(1.f, wo.y)));
    float phi = atan2f(wo.x, wo.z);
    if (phi < 0.f) phi += k2Pi;
    float uu = phi / k2Pi, v = theta / kPi;
    float fc = uu * float(E.width) - 0.5f, fr = v * float(E.height) - 0.5f;
    int c0 = int(floorf(fc)), r0 = int(floorf(fr));
    float tc = fc - float(c0), tr = fr - float(r0);
    int W = int(E.width), H = int(E.height);
    // c0 is in [-1, W - 1] and c0 + 1 in [0, W]: one add or subtract wraps
    // them as ((c % W) + W) % W does; the clamp only keeps a non-finite
    // direction's index in bounds
    auto wrapc = [&](int c) { return uint32_t(max(0, min(c < 0 ? c + W : (c >= W ? c - W : c), W - 1))); };
    auto clampr = [&](int r) { return uint32_t(max(0, min(r, H - 1))); };
    uint32_t c1 = wrapc(c0 + 1), c0u = wrapc(c0), r1u = clampr(r0 + 1), r0u = clampr(r0);
    const float* p00 = E.rgb + (size_t(r0u) * E.width + c0u) * 3;
    const float* p01 = E.rgb + (size_t(r0u) * E.width + c1) * 3;
    const float* p10 = E.rgb + (size_t(r1u) * E.width + c0u) * 3;
    const float* p11 = E.rgb + (size_t(r1u) * E.width + c1) * 3;
    float s[3];
#pragma unroll
    for (int ch = 0; ch < 3; ++ch) {
        s[ch] = (1.f - tr) * ((1.f - tc) * __ldg(p00 + ch) + tc * __ldg(p01 + ch)) +
                tr * ((1.f - tc) * __ldg(p10 + ch) + tc * __ldg(p11 + ch));
        s[ch] = fmaxf(0.f, s[ch]);
    }
    return f3(s[0], s[1], s[2]) * E.intensity;
}

// Environment radiance seen along a direction that leaves the scene:
// SceneView::envLight->Le or envRadiance (PathIntegrator.cpp:83-90, 244-247).
__device__ __forceinline__ float3 env_le(const DevEnv& E, float3 d) {
    return E.present ? env_eval(E, d) : E.radiance;
}

// DomeLight::evalPdf (DomeLight.h:427-448)
__device__ __forceinline__ float env_pdf(const DevEnv& E, float3 wo) {
    float theta = acosf(fmaxf(-1.f, fminf(1.f, wo.y)));
    float phi = atan2f(wo.x, wo.z);
    if (phi < 0.f) phi += k2Pi;
    float uu = phi / k2Pi, v = theta / kPi;
    uint32_t col = min(uint32_t(uu * float(E.width)), E.width - 1u);
    uint32_t row = min(uint32_t(v * float(E.height)), E.height - 1u);
    float sinT = fmaxf(sinf(theta), 1e-6f);
    float pr = E.marg_int > 0.f ? __ldg(E.marg_func + row) / E.marg_int : 0.f;
    float ci = __ldg(E.cond_int + row);
    float pc = ci > 0.f ? __ldg(E.cond_func + size_t(row) * E.width + col) / ci : 0.f;
    return (pr * pc * float(E.width * E.height)) / (k2Pi * kPi * sinT);
}

// DomeLight::sample / sampleDirection (DomeLight.h:244-256, 391-422)
__device__ __forceinline__ LightSample env_sample(const DevEnv& E, float ux, float uy) {
    LightSample ls;
    ls.pdf = 0.f;
    float pR, pC, urR, urC;
    uint32_t row = dist_sample(E.marg_func, E.marg_cdf, E.height, E.marg_int, uy, pR, urR);
    uint32_t col = dist_sample(E.cond_func + size_t(row) * E.width, E.cond_cdf + size_t(row) * (E.width + 1),
                               E.width, __ldg(E.cond_int + row), ux, pC, urC);
    float v = (float(row) + urR) / float(E.height);
    float uu = (float(col) + urC) / float(E.width);
    float theta = v * kPi, phi = uu * k2Pi;
    float st, ct, sp, cp;
    sincosf(theta, &st, &ct);
    sincosf(phi, &sp, &cp);
    float3 dir = f3(st * sp, ct, st * cp);
    float sa = fmaxf(st, 1e-6f);
    float pdf = (pR * pC * float(E.width * E.height)) / (k2Pi * kPi * sa);
    if (pdf <= 0.f) pdf = 0.f;
    if (pdf <= 0.f) return ls;
    ls.Li = env_eval(E, dir);
    ls.wi = dir;
    ls.pdf = pdf;
    ls.dist = 1e10f;
    return ls;
}

// AreaLight::sample (AreaLight.h:32-56)
__device__ __forceinline__ LightSample area_sample(const DevLight& L, float3 p, float ux, float uy) {
    LightSample ls;
    ls.pdf = 0.f;
    float3 pos = L.center + L.u * (2.f * ux - 1.f) + L.v * (2.f * uy - 1.f);
    float3 tl = pos - p;
    float d2 = length_sq(tl);
    float d = sqrtf(d2);
    float3 wi = tl * (1.f / d);
    float cosL = dot(-wi, L.normal);
    if (cosL <= 0.f) return ls;
    ls.Li = L.Le;
    ls.wi = wi;
    ls.pdf = d2 / (cosL * L.area);
    ls.dist = d * (1.f - 1e-4f);
    return ls;
}

// AreaLight::pdf (AreaLight.h:58-79)
__device__ __forceinline__ float area_pdf(const DevLight& L, float3 p, float3 wi) {
    float3 mn = -L.normal;
    float denom = dot(wi, mn);
    if (denom < 1e-6f) return 0.f;
    float t = dot(L.center - p, mn) / denom;
    if (t <= 0.f) return 0.f;
    float3 off = (p + wi * t) - L.center;
    float up = dot(off, L.u) / L.uLen2, vp = dot(off, L.v) / L.vLen2;
    if (fabsf(up) > 1.f || fabsf(vp) > 1.f) return 0.f;
    return (t * t) / (denom * L.area);
}

// DirectionalLight::sample (DirectionalLight.h:52-78): the direction toward the
// light, jittered inside its cone when it has an angular radius; pdf 1 and
// delta either way, so Li / pdf = Le.
__device__ __forceinline__ LightSample dir_sample(const DevLight& L, float ux, float uy) {
    LightSample s;
    s.Li = L.Le;
    s.pdf = 1.f;
    s.dist = 1e10f;
    s.delta = true;
    if (L.cos_cone >= 1.f - 1e-6f) {
        s.wi = L.normal;
    } else {
        const float cosT = 1.f - ux * (1.f - L.cos_cone);
        const float sinT = sqrtf(fmaxf(0.f, 1.f - cosT * cosT));
        const float phi = 2.f * kPi * uy;
        float sp, cp;
        sincosf(phi, &sp, &cp);
        float3 t, bt;
        onb(L.normal, t, bt);
        s.wi = safe_normalize(t * (sinT * cp) + bt * (sinT * sp) + L.normal * cosT);
    }
    return s;
}

// kFeat: the kFeat* light classes compiled in (the others give a zero sample).
template <uint32_t kFeat = kFeatAll>
__device__ __forceinline__ LightSample light_sample(const DevScene& S, const DevLight& L, float3 p, float ux,
                                                    float uy) {
    if constexpr ((kFeat & kFeatDir) != 0)
        if (L.type == ANA_LIGHT_DIRECTIONAL) return dir_sample(L, ux, uy);
    LightSample s;
    s.Li = f3(0.f, 0.f, 0.f);
    s.wi = f3(0.f, 0.f, 1.f);
    s.pdf = 0.f;
    s.dist = 0.f;
    if constexpr ((kFeat & kFeatArea) != 0 && (kFeat & kFeatDome) != 0)
        s = L.type == ANA_LIGHT_AREA ? area_sample(L, p, ux, uy) : env_sample(S.env, ux, uy);
    else if constexpr ((kFeat & kFeatArea) != 0)
        s = area_sample(L, p, ux, uy);
    else if constexpr ((kFeat & kFeatDome) != 0)
        s = env_sample(S.env, ux, uy);
    s.delta = false;
    return s;
}
// IMaterial::reflectance, the first-hit albedo AOV: Lambertian.h:76-78 (an
// emitter keeps its Lambertian albedo), StandardSurface.h:186-192,
// MarschnerHair.h:224-232.
__device__ __forceinline__ float3 mat_reflectance(const DevMaterial& m, const ShadeCtx& c) {
    if (m.type == ANA_MAT_STANDARD) {
        const float diff = (1.f - m.metal) * (1.f - m.spec * 0.5f);
        return (m.albedo * m.base) * (diff + m.metal);
    }
    if (m.type == ANA_MAT_HAIR) {
        const float3 sa = hair_sigma(m, c.color);
        return f3(expf(-sa.x), expf(-sa.y), expf(-sa.z));
    }
    return m.albedo;
}

// ILight::pdf; a directional light is delta (DirectionalLight::pdf returns 0).
template <uint32_t kFeat = kFeatAll>
__device__ __forceinline__ float light_pdf(const DevScene& S, const DevLight& L, float3 p, float3 wi) {
    if constexpr ((kFeat & kFeatDir) != 0)
        if (L.type == ANA_LIGHT_DIRECTIONAL) return 0.f;
    if constexpr ((kFeat & kFeatArea) != 0 && (kFeat & kFeatDome) != 0)
        return L.type == ANA_LIGHT_AREA ? area_pdf(L, p, wi) : env_pdf(S.env, wi);
    else if constexpr ((kFeat & kFeatArea) != 0)
        return area_pdf(L, p, wi);
    else if constexpr ((kFeat & kFeatDome) != 0)
        return env_pdf(S.env, wi);
    else
        return 0.f;
}

// spawnRay / spawnRayTo (Types.h:269-284)
__device__ __forceinline__ float3 spawn_origin(float3 p, float3 n, float3 d) {
    float3 off = n * 1e-4f;
    if (dot(d, n) < 0.f) off = -off;
    return p + off;
}

__device__ __forceinline__ float power_heuristic(float f, float g) { return (f * f) / (f * f + g * g); }

}  // namespace ana
