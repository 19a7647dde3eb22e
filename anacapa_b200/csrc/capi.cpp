// C ABI of the B200 path-tracing hot path (include/anacapa_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <memory>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/anacapa_b200.h"
#include "build.h"
#include "kernels.h"
#include "prepare.h"

namespace {

std::mutex g_err_mu;
std::string g_last_err;

// ceil(2^64 / d), 0 for d <= 1: the kernels' div_magic gives floor(n / d) for
// every 32-bit n from it (M*d = 2^64 + e with e < d, so n*e < 2^64).
uint64_t magic_div(uint32_t d) { return d <= 1 ? 0 : ~0ULL / d + 1; }

void set_global_err(const std::string& m) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_err = m;
}

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

inline float fbits(uint32_t u) {
    float f;
    std::memcpy(&f, &u, 4);
    return f;
}
inline uint32_t ubits(float f) {
    uint32_t u;
    std::memcpy(&u, &f, 4);
    return u;
}

// Per-scene facts of a blob that the per-render scene records need.
struct SceneStatic {
    uint32_t tri_root = ana::kNoRoot, seg_root = ana::kNoRoot;
    uint32_t slot_base = 0, num_slots = 0, light_base = 0, num_lights = 0;
    bool has_dome = false;
    float env_radiance[3] = {0.f, 0.f, 0.f};
    ana_camera camera{};
};

// One or more prepared scenes laid out as a single device arena in pinned
// host memory (256-byte aligned sections), so an upload is one copy.
struct Blob {
    unsigned char* mem = nullptr;  // host copy of [host_base, size)
    size_t size = 0;
    size_t host_base = 0;  // > 0: the triangle sections come from a device build
    bool pinned = false;
    size_t o_tri_nodes = 0, o_tri_isect = 0, o_tri_shade = 0, o_seg_nodes = 0, o_segs = 0, o_scol = 0, o_mats = 0,
           o_slots = 0, o_lights = 0, o_env_rgb = 0, o_cf = 0, o_cc = 0, o_ci = 0, o_mf = 0, o_mc = 0,
           o_motion = 0, o_keys = 0;
    std::vector<SceneStatic> scenes;
    bool has_curves = false, has_emitters = false, has_transmit = false, has_motion = false;
    size_t n_mats = 0, n_lights = 0;
    ana::HostEnv env_meta;  // scalars only
    unsigned char* at(size_t off) const { return mem + (off - host_base); }
    Blob() = default;
    Blob(const Blob&) = delete;
    Blob& operator=(const Blob&) = delete;
    ~Blob() {
        if (!mem) return;
        if (pinned) cudaFreeHost(mem);
        else std::free(mem);
    }
};

int build_blob(const ana::Prepared* const* list, uint32_t n, Blob& B, std::string& err) {
    size_t nNodes = 0, nTris = 0, nSegNodes = 0, nSegs = 0, nStr = 0, nMats = 0, nSlots = 0, nLights = 0,
           nMotion = 0, nKeyVec = 0;
    const ana::Prepared* dome = nullptr;
    for (uint32_t k = 0; k < n; ++k) {
        const ana::Prepared& P = *list[k];
        if (P.tris_on_device && n != 1) {
            err = "a scene built on the device is uploaded on its own";
            return ANA_ERR_INVALID_ARG;
        }
        nNodes += P.tris_on_device ? size_t(P.dev_tri_nodes) : P.tri_nodes.size();
        nTris += P.num_tris;
        nSegNodes += P.seg_nodes.size();
        nSegs += P.num_segs;
        nStr += P.strand_color.size() / 3;
        nMats += P.materials.size();
        nSlots += P.slot_material.size();
        nLights += P.lights.size();
        nMotion += P.mesh_motion.size();
        nKeyVec += P.motion_keys.size();
        if (P.env.present) {
            if (dome) {
                err = "a batch may hold at most one dome light";
                return ANA_ERR_UNSUPPORTED;
            }
            dome = &P;
        }
    }
    if (nTris >= (1u << 25) || nSegs >= (1u << 25)) {
        err = "more than 2^25 triangles or curve segments in the batch";
        return ANA_ERR_INVALID_ARG;
    }
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes);
        return o;
    };
    B.o_tri_nodes = take(nNodes * sizeof(ana::Bvh4Node));
    B.o_tri_isect = take(nTris * 48);
    B.o_tri_shade = take(nTris * 64);
    B.o_seg_nodes = take(nSegNodes * sizeof(ana::Bvh4Node));
    B.o_segs = take(nSegs * 80);
    B.o_scol = take(nStr * 12);
    B.o_mats = take(nMats * sizeof(ana::DevMaterial));
    B.o_slots = take(nSlots * 4);
    B.o_lights = take(nLights * sizeof(ana::DevLight));
    B.n_mats = nMats;
    B.n_lights = nLights;
    B.o_env_rgb = take(dome ? dome->env.rgb.size() * 4 : 0);
    B.o_cf = take(dome ? dome->env.cond_func.size() * 4 : 0);
    B.o_cc = take(dome ? dome->env.cond_cdf.size() * 4 : 0);
    B.o_ci = take(dome ? dome->env.cond_int.size() * 4 : 0);
    B.o_mf = take(dome ? dome->env.marg_func.size() * 4 : 0);
    B.o_mc = take(dome ? dome->env.marg_cdf.size() * 4 : 0);
    B.o_motion = take(nMotion * sizeof(uint2));
    B.o_keys = take(nKeyVec * 16);
    B.size = std::max<size_t>(off, kAlign);
    bool devTris = false;
    for (uint32_t k = 0; k < n; ++k) devTris = devTris || list[k]->tris_on_device;
    B.host_base = devTris ? B.o_seg_nodes : 0;
    const size_t hostBytes = std::max<size_t>(B.size - B.host_base, kAlign);
    void* mem = nullptr;
    if (cudaHostAlloc(&mem, hostBytes, cudaHostAllocPortable) == cudaSuccess) {
        B.pinned = true;
    } else {
        cudaGetLastError();
        mem = std::aligned_alloc(kAlign, hostBytes);
        B.pinned = false;
        if (!mem) {
            err = "host allocation failed";
            return ANA_ERR_OOM;
        }
    }
    B.mem = static_cast<unsigned char*>(mem);
    std::memset(B.mem, 0, hostBytes);
    auto* nodes = devTris ? nullptr : reinterpret_cast<ana::Bvh4Node*>(B.at(B.o_tri_nodes));
    auto* isect = devTris ? nullptr : reinterpret_cast<float4*>(B.at(B.o_tri_isect));
    auto* shade = devTris ? nullptr : reinterpret_cast<float4*>(B.at(B.o_tri_shade));
    auto* snodes = reinterpret_cast<ana::Bvh4Node*>(B.at(B.o_seg_nodes));
    auto* segs = reinterpret_cast<float4*>(B.at(B.o_segs));
    auto* scol = reinterpret_cast<float*>(B.at(B.o_scol));
    auto* mats = reinterpret_cast<ana::DevMaterial*>(B.at(B.o_mats));
    auto* slots = reinterpret_cast<int32_t*>(B.at(B.o_slots));
    auto* lights = reinterpret_cast<ana::DevLight*>(B.at(B.o_lights));
    auto* motion = reinterpret_cast<uint2*>(B.at(B.o_motion));
    auto* keys = reinterpret_cast<float4*>(B.at(B.o_keys));
    // 4-wide nodes (triangles and curve segments): interior refs shift by the
    // scene's node base, the first-primitive field of leaf entries (bits 0..24)
    // by its primitive base
    auto fix_node4 = [](ana::Bvh4Node nd, uint32_t nodeBase, uint32_t primBase) {
        uint32_t* ref = &nd.ref.x;
        for (int k = 0; k < 4; ++k) {
            if (ref[k] == ana::kEmptyChild) continue;
            ref[k] += (ref[k] & 0x80000000u) ? primBase : nodeBase;
        }
        return nd;
    };
    size_t iN = 0, iT = 0, iSN = 0, iS = 0, iStr = 0, iM = 0, iSl = 0, iL = 0, iMo = 0, iK = 0;
    B.scenes.assign(n, SceneStatic{});
    B.has_motion = nMotion > 0;
    B.has_curves = false;
    B.has_emitters = false;
    B.has_transmit = false;
    for (uint32_t k = 0; k < n; ++k) {
        const ana::Prepared& P = *list[k];
        SceneStatic& st = B.scenes[k];
        const uint32_t nodeBase = uint32_t(iN), triBase = uint32_t(iT), sNodeBase = uint32_t(iSN),
                       segBase = uint32_t(iS), strBase = uint32_t(iStr), matBase = uint32_t(iM);
        if (P.tris_on_device) {  // sections copied from the device build
            st.tri_root = nodeBase;
            iN += P.dev_tri_nodes;
        } else {
            st.tri_root = (P.num_tris && !P.tri_nodes.empty()) ? nodeBase : ana::kNoRoot;
        }
        for (const ana::Bvh4Node& nd : P.tri_nodes) nodes[iN++] = fix_node4(nd, nodeBase, triBase);
        const uint32_t motionBase = uint32_t(iMo), keyBase = uint32_t(iK / 5);
        for (uint32_t t = 0; t < (P.tris_on_device ? 0u : P.num_tris); ++t) {
            float4 a = P.tri_isect[3 * size_t(t)];
            float4 e1 = P.tri_isect[3 * size_t(t) + 1];
            a.w = fbits(ubits(a.w) + triBase);  // index into the batch's shading array (bit 31 kept)
            if (ubits(a.w) & 0x80000000u) e1.w = fbits(ubits(e1.w) + motionBase);  // batch motion mesh
            isect[3 * (size_t(triBase) + t)] = a;
            isect[3 * (size_t(triBase) + t) + 1] = e1;
            isect[3 * (size_t(triBase) + t) + 2] = P.tri_isect[3 * size_t(t) + 2];
            for (int j = 0; j < 4; ++j) shade[4 * (size_t(triBase) + t) + j] = P.tri_shade[4 * size_t(t) + j];
        }
        iT += P.num_tris;
        for (const uint2& mo : P.mesh_motion) motion[iMo++] = make_uint2(mo.x + keyBase, mo.y);
        for (const float4& k4 : P.motion_keys) keys[iK++] = k4;
        st.seg_root = (P.num_segs && !P.seg_nodes.empty()) ? sNodeBase : ana::kNoRoot;
        if (P.num_segs) B.has_curves = true;
        for (const ana::Bvh4Node& nd : P.seg_nodes) snodes[iSN++] = fix_node4(nd, sNodeBase, segBase);
        for (uint32_t s = 0; s < P.num_segs; ++s) {
            for (int j = 0; j < 4; ++j) segs[5 * (size_t(segBase) + s) + j] = P.segs[5 * size_t(s) + j];
            float4 r = P.segs[5 * size_t(s) + 4];
            r.x = fbits(ubits(r.x) + strBase);  // batch strand index
            r.w = fbits(strBase);               // strand - w is the scene-local strand index
            segs[5 * (size_t(segBase) + s) + 4] = r;
        }
        iS += P.num_segs;
        for (size_t i = 0; i < P.strand_color.size(); ++i) scol[3 * size_t(strBase) + i] = P.strand_color[i];
        iStr += P.strand_color.size() / 3;
        for (const ana::DevMaterial& m : P.materials) mats[iM++] = m;
        st.slot_base = uint32_t(iSl);
        st.num_slots = uint32_t(P.slot_material.size());
        for (int32_t s : P.slot_material) slots[iSl++] = s >= 0 ? s + int32_t(matBase) : -1;
        st.light_base = uint32_t(iL);
        st.num_lights = uint32_t(P.lights.size());
        for (const ana::DevLight& l : P.lights) lights[iL++] = l;
        st.has_dome = P.env.present;
        std::memcpy(st.env_radiance, P.env.radiance, sizeof(st.env_radiance));
        st.camera = P.camera;
        if (P.has_emitters) B.has_emitters = true;
        if (P.has_transmit) B.has_transmit = true;
    }
    if (dome) {
        std::memcpy(B.at(B.o_env_rgb), dome->env.rgb.data(), dome->env.rgb.size() * 4);
        std::memcpy(B.at(B.o_cf), dome->env.cond_func.data(), dome->env.cond_func.size() * 4);
        std::memcpy(B.at(B.o_cc), dome->env.cond_cdf.data(), dome->env.cond_cdf.size() * 4);
        std::memcpy(B.at(B.o_ci), dome->env.cond_int.data(), dome->env.cond_int.size() * 4);
        std::memcpy(B.at(B.o_mf), dome->env.marg_func.data(), dome->env.marg_func.size() * 4);
        std::memcpy(B.at(B.o_mc), dome->env.marg_cdf.data(), dome->env.marg_cdf.size() * 4);
        B.env_meta.present = true;
        B.env_meta.width = dome->env.width;
        B.env_meta.height = dome->env.height;
        B.env_meta.intensity = dome->env.intensity;
        B.env_meta.marg_int = dome->env.marg_int;
    }
    return ANA_OK;
}

}  // namespace

// A prepared scene: the host-built device layout (BVHs, flattened materials,
// dome distribution) and its single-scene pinned blob.
struct ana_prepared {
    ana::Prepared P;
    Blob blob;
};

struct ana_batch {
    std::vector<const ana_prepared*> items;
    Blob blob;
};

struct GraphCache {
    cudaGraphExec_t exec = nullptr;
    std::vector<unsigned char> key;
};

struct ana_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    ana_device_opts opts{};
    // scenes
    unsigned char* d_scene = nullptr;
    size_t d_scene_size = 0;
    size_t scene_bytes = 0;  // bytes of the uploaded arena in use
    ana::DevScene ds{};
    std::vector<SceneStatic> scenes;
    bool has_scene = false;
    uint64_t upload_serial = 0;
    // per-render tables: scene records, path offsets, chunk pixel runs
    unsigned char* d_tables = nullptr;
    size_t d_tables_size = 0;
    std::vector<unsigned char> h_tables;
    // film (all items of the last render, back to back)
    unsigned char* film = nullptr;
    size_t film_bytes = 0, film_pixels = 0;
    // AOV film (8 floats per pixel) and per-path first-hit AOVs (6 floats)
    unsigned char* aov_film = nullptr;
    size_t aov_film_bytes = 0;
    unsigned char* path_aov = nullptr;
    size_t path_aov_bytes = 0;
    bool aov_valid = false;  // the AOV film matches the beauty film's passes
    std::vector<size_t> item_film_offset, item_film_pixels;
    // wavefront buffers
    ana::Queues q{};
    unsigned char* d_queues = nullptr;
    uint32_t cap = 0;
    unsigned char* d_counters = nullptr;
    size_t counters_bytes = 0;
    uint32_t* d_err = nullptr;
    unsigned long long* d_work = nullptr;
    std::vector<uint32_t> h_counters;
    std::vector<cudaEvent_t> stage_ev;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    GraphCache graph;
    ana_stats stats{};
    int num_sms = 148;
    // differentiable rendering: host copies of the uploaded material and
    // light tables (parameters are written into them and copied back), the
    // last ana_forward's frame (its seeds determine every path), and the
    // adjoint replay's buffers
    std::vector<ana::DevMaterial> h_mats;
    std::vector<ana::DevLight> h_lights;
    size_t o_mats = 0, o_lights = 0;
    bool fwd_valid = false;
    ana_render_desc fwd_desc{};
    ana::AdjQueues aq{};
    unsigned char* d_adj = nullptr;
    size_t adj_size = 0;
    uint32_t adj_cap = 0;
    float* adj_L = nullptr;
    unsigned char* d_adj_io = nullptr;  // adjoint image + gradient accumulators
    size_t adj_io_size = 0;
    ana_film_pixel* film_px() const { return reinterpret_cast<ana_film_pixel*>(film); }
};

namespace {

int fail(ana_ctx* c, int code, const std::string& m) {
    if (c) c->err = m;
    set_global_err(m);
    return code;
}

int cuda_fail(ana_ctx* c, cudaError_t e, const char* what) {
    std::string m = std::string(what) + ": " + cudaGetErrorString(e);
    cudaGetLastError();
    return fail(c, e == cudaErrorMemoryAllocation ? ANA_ERR_OOM : ANA_ERR_CUDA, m);
}

#define CK(call, what)                                        \
    do {                                                      \
        cudaError_t e_ = (call);                              \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

void drop_graph(ana_ctx* c) {
    if (c->graph.exec) cudaGraphExecDestroy(c->graph.exec);
    c->graph.exec = nullptr;
    c->graph.key.clear();
}

// Grows a device buffer (contents are not kept). Any cached graph refers to
// the old address, so it is dropped.
int ensure_buffer(ana_ctx* c, unsigned char** p, size_t* have, size_t need, const char* what) {
    if (*have >= need && *p) return ANA_OK;
    if (*p) {
        CK(cudaStreamSynchronize(c->stream), "sync");
        cudaFree(*p);
        *p = nullptr;
        *have = 0;
    }
    drop_graph(c);
    void* mem = nullptr;
    CK(cudaMalloc(&mem, need), what);
    *p = static_cast<unsigned char*>(mem);
    *have = need;
    return ANA_OK;
}

// Wavefront buffers for `cap` paths.
int ensure_queues(ana_ctx* c, uint32_t cap) {
    if (c->cap >= cap && c->d_queues) return ANA_OK;
    size_t f4 = size_t(cap) * 16;
    size_t total = 14 * align_up(f4) + align_up(size_t(cap) * 12);
    size_t have = c->d_queues ? size_t(1) : 0;  // force reallocation
    if (c->d_queues) {
        CK(cudaStreamSynchronize(c->stream), "sync");
        cudaFree(c->d_queues);
        c->d_queues = nullptr;
        have = 0;
    }
    int rc = ensure_buffer(c, &c->d_queues, &have, total, "cudaMalloc(wavefront queues)");
    if (rc) return rc;
    unsigned char* b = c->d_queues;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* p = b + off;
        off += align_up(bytes);
        return p;
    };
    for (int k = 0; k < 2; ++k) {
        c->q.ext_o[k] = reinterpret_cast<float4*>(take(f4));
        c->q.ext_d[k] = reinterpret_cast<float4*>(take(f4));
        c->q.ext_b[k] = reinterpret_cast<float4*>(take(f4));
    }
    c->q.hit0 = reinterpret_cast<float4*>(take(f4));
    c->q.hit1 = reinterpret_cast<float4*>(take(f4));
    c->q.sh_o = reinterpret_cast<float4*>(take(f4));
    c->q.sh_d = reinterpret_cast<float4*>(take(f4));
    c->q.sh_c = reinterpret_cast<float4*>(take(f4));
    c->q.mis_o = reinterpret_cast<float4*>(take(f4));
    c->q.mis_d = reinterpret_cast<float4*>(take(f4));
    c->q.mis_c = reinterpret_cast<float4*>(take(f4));
    c->q.L = reinterpret_cast<float*>(take(size_t(cap) * 12));
    c->cap = cap;
    return ANA_OK;
}

// Copies a blob into the device arena. With `dt` the triangle sections come
// from a device build (device-to-device) and the blob holds the rest.
int upload_blob(ana_ctx* c, const Blob& B, const ana::DeviceTris* dt = nullptr) {
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    int rc = ensure_buffer(c, &c->d_scene, &c->d_scene_size, B.size, "cudaMalloc(scene)");
    if (rc) return rc;
    if (dt) {
        CK(cudaMemsetAsync(c->d_scene, 0, B.o_seg_nodes, c->stream), "scene clear");
        CK(cudaMemcpyAsync(c->d_scene + B.o_tri_nodes, dt->nodes, size_t(dt->num_nodes) * sizeof(ana::Bvh4Node),
                           cudaMemcpyDeviceToDevice, c->stream),
           "triangle nodes D2D");
        CK(cudaMemcpyAsync(c->d_scene + B.o_tri_isect, dt->isect, size_t(dt->num_tris) * 48, cudaMemcpyDeviceToDevice,
                           c->stream),
           "triangle records D2D");
        CK(cudaMemcpyAsync(c->d_scene + B.o_tri_shade, dt->shade, size_t(dt->num_tris) * 64, cudaMemcpyDeviceToDevice,
                           c->stream),
           "triangle shading D2D");
        CK(cudaMemcpyAsync(c->d_scene + B.o_seg_nodes, B.at(B.o_seg_nodes), B.size - B.o_seg_nodes,
                           cudaMemcpyHostToDevice, c->stream),
           "scene upload");
    } else {
        if (B.host_base) return fail(c, ANA_ERR_STATE, "scene upload: the triangle sections are missing");
        CK(cudaMemcpyAsync(c->d_scene, B.mem, B.size, cudaMemcpyHostToDevice, c->stream), "scene upload");
    }
    c->scene_bytes = B.size;
    unsigned char* b = c->d_scene;
    ana::DevScene& S = c->ds;
    S = ana::DevScene{};
    S.tri_nodes = reinterpret_cast<const ana::Bvh4Node*>(b + B.o_tri_nodes);
    S.tri_isect = reinterpret_cast<const float4*>(b + B.o_tri_isect);
    S.tri_shade = reinterpret_cast<const float4*>(b + B.o_tri_shade);
    S.seg_nodes = reinterpret_cast<const ana::Bvh4Node*>(b + B.o_seg_nodes);
    S.segs = reinterpret_cast<const float4*>(b + B.o_segs);
    S.strand_color = reinterpret_cast<const float*>(b + B.o_scol);
    S.materials = reinterpret_cast<const ana::DevMaterial*>(b + B.o_mats);
    S.slot_material = reinterpret_cast<const int32_t*>(b + B.o_slots);
    S.lights = reinterpret_cast<const ana::DevLight*>(b + B.o_lights);
    S.has_curves = B.has_curves ? 1 : 0;
    S.has_emitters = B.has_emitters ? 1 : 0;
    S.has_transmit = B.has_transmit ? 1 : 0;
    S.mesh_motion = reinterpret_cast<const uint2*>(b + B.o_motion);
    S.motion_keys = reinterpret_cast<const float4*>(b + B.o_keys);
    S.has_motion = B.has_motion ? 1 : 0;
    S.has_fibers = S.has_curves;
    S.has_extra_shading = S.has_motion;
    {
        const auto* mats = reinterpret_cast<const ana::DevMaterial*>(B.at(B.o_mats));
        for (size_t i = 0; i < B.n_mats; ++i) {
            if (mats[i].type == ANA_MAT_HAIR) S.has_fibers = 1;
            if (mats[i].transmission > 0.001f || mats[i].opacity < 1.f) S.has_extra_shading = 1;
            if (mats[i].type == ANA_MAT_LAMBERT || mats[i].type == ANA_MAT_EMISSIVE) S.features |= ana::kFeatLambert;
            if (mats[i].type == ANA_MAT_STANDARD) S.features |= ana::kFeatStandard;
        }
        const auto* lights = reinterpret_cast<const ana::DevLight*>(B.at(B.o_lights));
        for (size_t i = 0; i < B.n_lights; ++i) {
            if (lights[i].type == ANA_LIGHT_AREA) S.features |= ana::kFeatArea;
            else if (lights[i].type == ANA_LIGHT_DOME) S.features |= ana::kFeatDome;
            else S.features |= ana::kFeatDir;
        }
    }
    ana::DevEnv& E = S.env;
    E.present = B.env_meta.present ? 1 : 0;
    E.rgb = E.present ? reinterpret_cast<const float*>(b + B.o_env_rgb) : nullptr;
    E.cond_func = reinterpret_cast<const float*>(b + B.o_cf);
    E.cond_cdf = reinterpret_cast<const float*>(b + B.o_cc);
    E.cond_int = reinterpret_cast<const float*>(b + B.o_ci);
    E.marg_func = reinterpret_cast<const float*>(b + B.o_mf);
    E.marg_cdf = reinterpret_cast<const float*>(b + B.o_mc);
    E.marg_int = B.env_meta.marg_int;
    E.intensity = B.env_meta.intensity;
    E.width = B.env_meta.width;
    E.height = B.env_meta.height;
    c->scenes = B.scenes;
    c->has_scene = true;
    c->upload_serial++;
    const auto* hm = reinterpret_cast<const ana::DevMaterial*>(B.at(B.o_mats));
    const auto* hl = reinterpret_cast<const ana::DevLight*>(B.at(B.o_lights));
    c->h_mats.assign(hm, hm + B.n_mats);
    c->h_lights.assign(hl, hl + B.n_lights);
    c->o_mats = B.o_mats;
    c->o_lights = B.o_lights;
    c->fwd_valid = false;
    drop_graph(c);
    return ANA_OK;
}

struct ChunkPlan {
    uint32_t first_path, paths, pixels, seg_begin, seg_count;
};

// Adjoint replay buffers for `cap` paths, next to the forward queues.
int ensure_adjoint(ana_ctx* c, uint32_t cap) {
    if (c->adj_cap >= cap && c->d_adj) return ANA_OK;
    const size_t f4 = size_t(cap) * 16;
    const size_t total = 9 * align_up(f4) + align_up(size_t(cap) * 4) + 2 * align_up(size_t(cap) * 12);
    int rc = ensure_buffer(c, &c->d_adj, &c->adj_size, total, "cudaMalloc(adjoint queues)");
    if (rc) return rc;
    unsigned char* b = c->d_adj;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        unsigned char* q = b + off;
        off += align_up(bytes);
        return q;
    };
    ana::AdjQueues& a = c->aq;
    for (int k = 0; k < 2; ++k) {
        a.ext_g0[k] = reinterpret_cast<float4*>(take(f4));
        a.ext_g1[k] = reinterpret_cast<float4*>(take(f4));
    }
    a.sh_g0 = reinterpret_cast<float4*>(take(f4));
    a.sh_g1 = reinterpret_cast<float4*>(take(f4));
    a.mis_g0 = reinterpret_cast<float4*>(take(f4));
    a.mis_g1 = reinterpret_cast<float4*>(take(f4));
    a.mis_res = reinterpret_cast<float4*>(take(f4));
    a.sh_vis = reinterpret_cast<uint32_t*>(take(size_t(cap) * 4));
    a.dL = reinterpret_cast<float*>(take(size_t(cap) * 12));
    // the adjoint replay's running radiance (the primal's lives in the queues' L)
    c->adj_L = reinterpret_cast<float*>(take(size_t(cap) * 12));
    c->adj_cap = cap;
    return ANA_OK;
}

// The batch render: descs[k] renders uploaded scene k into its film.
// With adj_image (host, 3 floats per film pixel: dLoss / d pixel) it runs the
// path-replay adjoint instead: per chunk a primal replay of the same paths
// (their radiance L) and an adjoint replay that accumulates dLoss / d theta
// into adj_grad (host, 8 floats per material then 4 per light).
// One render item: the pixels [x0, x0 + rw) x [y0, y0 + rh) of the width x
// height film of uploaded scene `scene`, sample indices [sample_start,
// sample_start + spp), accumulated at film_offset of the context's film. A
// frame is one item covering its film; PathIntegrator::renderTile's tiles
// are items that share one film.
struct Item {
    uint32_t scene, width, height, x0, y0, rw, rh, sample_start, spp, max_depth, min_depth;
    uint64_t seed, film_offset;
};

// The batch render of `items` into a film of totalPixels pixels.
int render_items(ana_ctx* c, const std::vector<Item>& items, uint64_t totalPixels, uint32_t flags,
                 const float* adj_image = nullptr, float* adj_grad = nullptr) {
    const bool backward = adj_image != nullptr;
    if (backward) flags &= ~uint32_t(ANA_RENDER_GRAPH | ANA_RENDER_COUNT_WORK);
    const uint32_t n = uint32_t(items.size());
    if (n == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: no items");
    uint64_t totalPaths = 0;
    uint32_t maxSpp = 0, maxDepth = 0;
    for (const Item& it : items) {
        if (it.rw == 0 || it.rh == 0 || it.spp == 0)
            return fail(c, ANA_ERR_INVALID_ARG, "ana_render: empty frame or zero samples");
        if (it.max_depth > 255) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: max_depth > 255");
        totalPaths += uint64_t(it.rw) * it.rh * it.spp;
        maxSpp = std::max(maxSpp, it.spp);
        maxDepth = std::max(maxDepth, it.max_depth);
    }
    if (totalPaths >= (1ull << 32))
        return fail(c, ANA_ERR_INVALID_ARG, "ana_render: total width*height*sample_count must be < 2^32");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const bool count_work = (flags & ANA_RENDER_COUNT_WORK) != 0;
    const bool use_graph = (flags & ANA_RENDER_GRAPH) != 0 && !count_work;
    const bool timing = c->opts.timing != 0 && !use_graph;
    // default chunk: 32M paths in flight (~8 GB of queues). Smaller chunks
    // leave the late, sparse bounces of each chunk too few rays to fill the
    // GPU (throughput scene: 772 ms/frame at 4M paths, 537 ms at 32M).
    uint32_t cap = c->opts.chunk_paths ? c->opts.chunk_paths : (1u << 25);
    cap = std::max(cap, maxSpp);
    if (uint64_t(cap) > totalPaths) cap = uint32_t(totalPaths);
    int rc = ensure_queues(c, cap);
    if (rc) return rc;
    const size_t nparams = 8 * c->h_mats.size() + 4 * c->h_lights.size();
    const size_t oGrad = align_up(size_t(totalPixels) * 12);
    if (backward) {
        rc = ensure_adjoint(c, cap);
        if (rc) return rc;
        rc = ensure_buffer(c, &c->d_adj_io, &c->adj_io_size, oGrad + std::max<size_t>(nparams, 1) * 4,
                           "cudaMalloc(adjoint image)");
        if (rc) return rc;
        CK(cudaMemcpyAsync(c->d_adj_io, adj_image, size_t(totalPixels) * 12, cudaMemcpyHostToDevice, c->stream),
           "adjoint image H2D");
    }
    // film: all items back to back
    rc = ensure_buffer(c, &c->film, &c->film_bytes, totalPixels * sizeof(ana_film_pixel), "cudaMalloc(film)");
    if (rc) return rc;
    if (c->film_pixels != totalPixels) flags |= ANA_RENDER_CLEAR_FILM;
    c->film_pixels = totalPixels;
    const bool aovs = (flags & ANA_RENDER_AOVS) != 0 && !backward;
    if (aovs) {
        rc = ensure_buffer(c, &c->aov_film, &c->aov_film_bytes, totalPixels * 32, "cudaMalloc(AOV film)");
        if (rc) return rc;
        rc = ensure_buffer(c, &c->path_aov, &c->path_aov_bytes, size_t(cap) * 24, "cudaMalloc(path AOVs)");
        if (rc) return rc;
        if (!c->aov_valid && !(flags & ANA_RENDER_CLEAR_FILM))
            return fail(c, ANA_ERR_STATE, "AOVs need a cleared film or AOVs in every pass since the last clear");
    }
    c->aov_valid = aovs && (c->aov_valid || (flags & ANA_RENDER_CLEAR_FILM));
    // scene records, path offsets, chunk plan
    std::vector<ana::DevSceneRec> recs(n);
    std::vector<uint32_t> pathOff(n + 1, 0);
    uint64_t path = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const Item& r = items[k];
        const SceneStatic& st = c->scenes[r.scene];
        ana::DevSceneRec& R = recs[k];
        std::memset(&R, 0, sizeof(R));
        R.tri_root = st.tri_root;
        R.seg_root = st.seg_root;
        R.slot_base = st.slot_base;
        R.num_slots = st.num_slots;
        R.light_base = st.light_base;
        R.num_lights = st.num_lights;
        R.spp = r.spp;
        R.sample_start = r.sample_start;
        R.max_depth = r.max_depth;
        R.min_depth = r.min_depth;
        R.film_offset = uint32_t(r.film_offset);
        R.path_offset = uint32_t(path);
        R.seed = r.seed;
        R.env_radiance = make_float3(st.env_radiance[0], st.env_radiance[1], st.env_radiance[2]);
        R.has_dome = st.has_dome ? 1 : 0;
        R.cam = ana::make_camera(st.camera, r.width, r.height);
        R.rect_x0 = r.x0;
        R.rect_y0 = r.y0;
        R.rect_w = r.rw;
        R.film_w = r.width;
        R.spp_div = magic_div(r.spp);
        R.rect_w_div = magic_div(r.rw);
        pathOff[k] = uint32_t(path);
        path += uint64_t(r.rw) * r.rh * r.spp;
    }
    pathOff[n] = uint32_t(path);
    // chunks: cut the global path space at pixel boundaries, `cap` paths each
    std::vector<ana::ChunkSeg> segs;
    std::vector<ChunkPlan> chunks;
    {
        ChunkPlan cp{0, 0, 0, 0, 0};
        uint32_t gpath = 0;
        for (uint32_t k = 0; k < n; ++k) {
            const uint32_t spp = items[k].spp;
            const uint32_t npx = items[k].rw * items[k].rh;
            uint32_t px = 0;
            while (px < npx) {
                uint32_t fit = std::min(npx - px, (cap - cp.paths) / spp);
                if (fit == 0) {  // chunk full
                    chunks.push_back(cp);
                    cp = ChunkPlan{gpath, 0, 0, uint32_t(segs.size()), 0};
                    continue;
                }
                ana::ChunkSeg sg{};
                sg.scene = k;
                sg.first_pixel = px;
                sg.num_pixels = fit;
                sg.local_pixel = cp.pixels;
                sg.local_path = cp.paths;
                segs.push_back(sg);
                cp.seg_count++;
                cp.paths += fit * spp;
                cp.pixels += fit;
                px += fit;
                gpath += fit * spp;
            }
        }
        if (cp.paths) chunks.push_back(cp);
    }
    const uint32_t nchunks = uint32_t(chunks.size());
    // tables: records | path offsets | chunk pixel runs
    const size_t oRec = 0, oOff = align_up(n * sizeof(ana::DevSceneRec)), oSeg = oOff + align_up((n + 1) * 4);
    const size_t tbytes = oSeg + segs.size() * sizeof(ana::ChunkSeg);
    std::vector<unsigned char> tables(tbytes, 0);
    std::memcpy(tables.data() + oRec, recs.data(), n * sizeof(ana::DevSceneRec));
    std::memcpy(tables.data() + oOff, pathOff.data(), (n + 1) * 4);
    std::memcpy(tables.data() + oSeg, segs.data(), segs.size() * sizeof(ana::ChunkSeg));
    rc = ensure_buffer(c, &c->d_tables, &c->d_tables_size, tbytes, "cudaMalloc(tables)");
    if (rc) return rc;
    if (tables != c->h_tables) {
        c->h_tables = tables;
        CK(cudaMemcpyAsync(c->d_tables, c->h_tables.data(), tbytes, cudaMemcpyHostToDevice, c->stream),
           "tables H2D");
    }
    const uint32_t rows = maxDepth + 2;
    const size_t ncount = size_t(nchunks) * rows * ana::kCountersPerBounce;
    // the backward pass keeps the adjoint replay's counters after the primal's
    const size_t ncountAll = (backward ? 2 : 1) * ncount;
    rc = ensure_buffer(c, &c->d_counters, &c->counters_bytes, ncountAll * 4, "cudaMalloc(counters)");
    if (rc) return rc;
    uint32_t* counters = reinterpret_cast<uint32_t*>(c->d_counters);
    ana::Params p{};
    p.S = c->ds;
    p.S.scenes = reinterpret_cast<const ana::DevSceneRec*>(c->d_tables + oRec);
    p.S.scene_path_offset = reinterpret_cast<const uint32_t*>(c->d_tables + oOff);
    p.S.num_scenes = n;
    p.q = c->q;
    p.film = c->film_px();
    p.aov = aovs ? reinterpret_cast<float*>(c->aov_film) : nullptr;
    p.q.aov = aovs ? reinterpret_cast<float*>(c->path_aov) : nullptr;
    p.err = c->d_err;
    p.work = c->d_work;
    ana::LaunchCfg cfg;
    cfg.block = c->opts.block_size ? int(c->opts.block_size) : 256;
    cfg.persistent = c->opts.traversal == ANA_TRAVERSAL_PER_RAY ? 0 : 1;
    const long long gcap = ((long long)cap + cfg.block - 1) / cfg.block;
    cfg.grid_cap = int(std::max<long long>(1, std::min<long long>(gcap, 1 << 20)));
    cfg.stage_grid = std::max(1, 4 * c->num_sms * (2048 / cfg.block));
    const size_t launches = backward ? size_t(nchunks) * (3 + 9 * size_t(maxDepth + 1))
                                     : size_t(nchunks) * (2 + 4 * size_t(maxDepth + 1));
    if (timing && c->stage_ev.size() < 2 * launches) {
        size_t old = c->stage_ev.size();
        c->stage_ev.resize(2 * launches);
        for (size_t i = old; i < c->stage_ev.size(); ++i) CK(cudaEventCreate(&c->stage_ev[i]), "event create");
    }
    std::vector<int> stage_of;
    size_t ev_i = 0;
    cudaError_t first_launch_err = cudaSuccess;
    const char* first_launch_stage = "";
    static const char* kStageNames[5] = {"extend", "shade", "shadow", "mis", "generate/film"};
    auto timed = [&](int stage, auto&& launch) {
        if (timing) cudaEventRecord(c->stage_ev[2 * ev_i], c->stream);
        launch();
        cudaError_t le = cudaGetLastError();
        if (le != cudaSuccess && first_launch_err == cudaSuccess) {
            first_launch_err = le;
            first_launch_stage = kStageNames[stage];
        }
        if (timing) {
            cudaEventRecord(c->stage_ev[2 * ev_i + 1], c->stream);
            stage_of.push_back(stage);
            ++ev_i;
        }
    };
    // the launch sequence (captured into a graph when requested)
    const bool clear = (flags & ANA_RENDER_CLEAR_FILM) != 0;
    auto enqueue_backward = [&]() {
        cudaMemsetAsync(c->d_counters, 0, ncountAll * 4, c->stream);
        cudaMemsetAsync(c->d_err, 0, 4, c->stream);
        cudaMemsetAsync(c->d_adj_io + oGrad, 0, nparams * 4, c->stream);
        ana::Params pa = p;
        // the emission gradient of MIS hits needs the emissive material hit,
        // which the any-hit MIS query of emitter-free scenes does not find
        for (const ana::DevMaterial& m : c->h_mats)
            if (m.type == ANA_MAT_EMISSIVE) pa.S.has_emitters = 1;
        pa.a = c->aq;
        pa.a.Lp = c->q.L;
        pa.a.d_image = reinterpret_cast<const float*>(c->d_adj_io);
        pa.a.grad = reinterpret_cast<float*>(c->d_adj_io + oGrad);
        pa.a.num_materials = uint32_t(c->h_mats.size());
        for (uint32_t k = 0; k < nchunks; ++k) {
            const ChunkPlan& cp = chunks[k];
            pa.chunk_first_path = cp.first_path;
            pa.chunk_paths = cp.paths;
            pa.chunk_pixels = cp.pixels;
            pa.segs = reinterpret_cast<const ana::ChunkSeg*>(c->d_tables + oSeg) + cp.seg_begin;
            pa.num_segs = cp.seg_count;
            // primal replay: the forward pass's paths, their radiance into q.L
            pa.q.L = c->q.L;
            pa.counters = counters + size_t(k) * rows * ana::kCountersPerBounce;
            pa.bounce = 0;
            timed(4, [&] { ana::launch_generate(pa, cfg, c->stream); });
            for (uint32_t b = 0; b <= maxDepth; ++b) {
                pa.bounce = b;
                timed(0, [&] { ana::launch_extend(pa, cfg, c->stream, false); });
                timed(1, [&] { ana::launch_shade(pa, cfg, c->stream); });
                timed(2, [&] { ana::launch_shadow(pa, cfg, c->stream); });
                timed(3, [&] { ana::launch_mis(pa, cfg, c->stream); });
            }
            // adjoint replay: the same paths again, gathering radiance into
            // adj_L so that L - adj_L is the radiance still to come
            pa.q.L = c->adj_L;
            pa.counters = counters + ncount + size_t(k) * rows * ana::kCountersPerBounce;
            pa.bounce = 0;
            timed(4, [&] { ana::launch_generate(pa, cfg, c->stream); });
            timed(4, [&] { ana::launch_adj_init(pa, cfg, c->stream); });
            for (uint32_t b = 0; b <= maxDepth; ++b) {
                pa.bounce = b;
                timed(0, [&] { ana::launch_extend(pa, cfg, c->stream, false); });
                timed(1, [&] { ana::launch_shade_adj(pa, cfg, c->stream); });
                timed(2, [&] { ana::launch_shadow_adj(pa, cfg, c->stream); });
                timed(3, [&] { ana::launch_mis_adj(pa, cfg, c->stream); });
                timed(4, [&] { ana::launch_adj_direct(pa, cfg, c->stream); });
            }
        }
    };
    auto enqueue = [&]() {
        if (clear) cudaMemsetAsync(c->film, 0, totalPixels * sizeof(ana_film_pixel), c->stream);
        if (clear && aovs) cudaMemsetAsync(c->aov_film, 0, totalPixels * 32, c->stream);
        cudaMemsetAsync(c->d_counters, 0, ncount * 4, c->stream);
        cudaMemsetAsync(c->d_err, 0, 4, c->stream);
        if (count_work) cudaMemsetAsync(c->d_work, 0, 4 * sizeof(unsigned long long), c->stream);
        for (uint32_t k = 0; k < nchunks; ++k) {
            const ChunkPlan& cp = chunks[k];
            p.chunk_first_path = cp.first_path;
            p.chunk_paths = cp.paths;
            p.chunk_pixels = cp.pixels;
            p.segs = reinterpret_cast<const ana::ChunkSeg*>(c->d_tables + oSeg) + cp.seg_begin;
            p.num_segs = cp.seg_count;
            p.counters = counters + size_t(k) * rows * ana::kCountersPerBounce;
            p.bounce = 0;
            timed(4, [&] { ana::launch_generate(p, cfg, c->stream); });
            for (uint32_t b = 0; b <= maxDepth; ++b) {
                p.bounce = b;
                timed(0, [&] { ana::launch_extend(p, cfg, c->stream, count_work); });
                timed(1, [&] { ana::launch_shade(p, cfg, c->stream); });
                timed(2, [&] { ana::launch_shadow(p, cfg, c->stream); });
                timed(3, [&] { ana::launch_mis(p, cfg, c->stream); });
            }
            timed(4, [&] { ana::launch_film(p, cfg, c->stream); });
        }
    };
    CK(cudaEventRecord(c->ev0, c->stream), "event");
    if (use_graph) {
        // the graph is reused while the tables, flags, launch configuration,
        // buffers and uploaded scene are unchanged
        std::vector<unsigned char> key = c->h_tables;
        auto put = [&](const void* x, size_t nb) {
            const unsigned char* bb = static_cast<const unsigned char*>(x);
            key.insert(key.end(), bb, bb + nb);
        };
        put(&clear, sizeof(clear));
        put(&p.aov, sizeof(p.aov));
        put(&p.q.aov, sizeof(p.q.aov));
        put(&cfg, sizeof(cfg));
        put(&cap, sizeof(cap));
        put(&c->upload_serial, sizeof(c->upload_serial));
        if (!c->graph.exec || c->graph.key != key) {
            drop_graph(c);
            cudaGraph_t g = nullptr;
            CK(cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeThreadLocal), "begin capture");
            enqueue();
            cudaError_t e = cudaStreamEndCapture(c->stream, &g);
            if (first_launch_err != cudaSuccess) {
                if (g) cudaGraphDestroy(g);
                std::string what = std::string("graph capture: ") + first_launch_stage + " launch";
                return cuda_fail(c, first_launch_err, what.c_str());
            }
            if (e != cudaSuccess) return cuda_fail(c, e, "end capture");
            e = cudaGraphInstantiate(&c->graph.exec, g, 0);
            cudaGraphDestroy(g);
            if (e != cudaSuccess) {
                c->graph.exec = nullptr;
                return cuda_fail(c, e, "graph instantiate");
            }
            c->graph.key = key;
        }
        CK(cudaGraphLaunch(c->graph.exec, c->stream), "graph launch");
    } else {
        if (backward) enqueue_backward();
        else enqueue();
        if (first_launch_err != cudaSuccess) {
            std::string what = std::string(first_launch_stage) + " launch";
            return cuda_fail(c, first_launch_err, what.c_str());
        }
    }
    CK(cudaGetLastError(), "kernel launch");
    CK(cudaEventRecord(c->ev1, c->stream), "event");
    unsigned long long hwork[4] = {0, 0, 0, 0};
    if (count_work)
        CK(cudaMemcpyAsync(hwork, c->d_work, sizeof(hwork), cudaMemcpyDeviceToHost, c->stream), "work D2H");
    c->h_counters.resize(ncountAll);
    CK(cudaMemcpyAsync(c->h_counters.data(), counters, ncountAll * 4, cudaMemcpyDeviceToHost, c->stream),
       "counters D2H");
    if (backward && nparams)
        CK(cudaMemcpyAsync(adj_grad, c->d_adj_io + oGrad, nparams * 4, cudaMemcpyDeviceToHost, c->stream),
           "gradient D2H");
    uint32_t herr = 0;
    CK(cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream), "err D2H");
    CK(cudaStreamSynchronize(c->stream), "render sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    ana_stats& st = c->stats;
    const ana_stats up = st;  // the upload fields describe the last upload
    st = ana_stats{};
    st.upload_ms = up.upload_ms;
    for (int k = 0; k < 4; ++k) st.build_ms[k] = up.build_ms[k];
    st.build_levels = up.build_levels;
    st.paths = totalPaths;
    for (uint32_t k = 0; k < nchunks * (backward ? 2u : 1u); ++k)
        for (uint32_t b = 0; b < rows; ++b) {
            const uint32_t* cc = c->h_counters.data() + (size_t(k) * rows + b) * ana::kCountersPerBounce;
            if (b <= maxDepth) st.extend_rays += cc[0];
            st.shadow_rays += cc[1];
            st.mis_rays += cc[2];
            if (cc[0]) st.bounces = std::max(st.bounces, b + 1);
        }
    st.render_ms = ms;
    st.chunks = nchunks;
    st.kernel_launches = launches;
    st.extend_launches = size_t(nchunks) * (maxDepth + 1);
    st.node_fetches = hwork[0];
    st.tri_tests = hwork[1];
    st.seg_tests = hwork[2];
    st.curve_node_fetches = hwork[3];
    if (timing) {
        float acc[5] = {0, 0, 0, 0, 0};
        for (size_t i = 0; i < ev_i; ++i) {
            float e = 0.f;
            cudaEventElapsedTime(&e, c->stage_ev[2 * i], c->stage_ev[2 * i + 1]);
            acc[stage_of[i]] += e;
        }
        st.extend_ms = acc[0];
        st.shade_ms = acc[1];
        st.shadow_ms = acc[2];
        st.mis_ms = acc[3];
        st.film_ms = acc[4];
    }
    if (herr) return fail(c, ANA_ERR_DEVICE_CHECK, "ana_render: traversal stack overflow on the device");
    return ANA_OK;
}

// Whole frames: descs[k] renders uploaded scene k into its own film, the
// films back to back.
int render_descs(ana_ctx* c, const ana_render_desc* descs, uint32_t n, uint32_t flags,
                 const float* adj_image = nullptr, float* adj_grad = nullptr) {
    if (!c || !descs || n == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: NULL argument or no items");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_render: no scene uploaded");
    if (n != c->scenes.size())
        return fail(c, ANA_ERR_INVALID_ARG, "ana_render_batch: one desc per uploaded scene is required");
    std::vector<Item> items(n);
    std::vector<size_t> offs(n), pixels(n);
    uint64_t pix = 0;
    for (uint32_t k = 0; k < n; ++k) {
        const ana_render_desc& r = descs[k];
        items[k] = Item{k, r.width, r.height, 0, 0, r.width, r.height, r.sample_start, r.sample_count,
                        r.max_depth, r.min_depth, r.seed, pix};
        offs[k] = pix;
        pixels[k] = size_t(r.width) * r.height;
        pix += uint64_t(r.width) * r.height;
    }
    const int rc = render_items(c, items, pix, flags, adj_image, adj_grad);
    if (rc == ANA_OK) {
        c->item_film_offset = offs;
        c->item_film_pixels = pixels;
    }
    return rc;
}

// Writes differentiable parameters into the host material / light tables and
// copies both tables to the device. Derived fields follow prepare_scene
// (derive_standard: GGX alpha2, flags, isDelta).
int apply_params(ana_ctx* c, const ana_diff_params* P) {
    const size_t nm = c->h_mats.size(), nl = c->h_lights.size();
    for (size_t i = 0; i < nm; ++i) {
        ana::DevMaterial& m = c->h_mats[i];
        if (P->albedo) m.albedo = make_float3(P->albedo[3 * i], P->albedo[3 * i + 1], P->albedo[3 * i + 2]);
        if (P->roughness && m.type == ANA_MAT_STANDARD) {
            m.rough = P->roughness[i];
            ana::derive_standard(m);
        }
        if (P->emission && m.type == ANA_MAT_EMISSIVE)
            m.emission = make_float3(P->emission[3 * i], P->emission[3 * i + 1], P->emission[3 * i + 2]);
    }
    for (size_t i = 0; i < nl; ++i)
        if (P->light_le && c->h_lights[i].type == ANA_LIGHT_AREA)
            c->h_lights[i].Le = make_float3(P->light_le[3 * i], P->light_le[3 * i + 1], P->light_le[3 * i + 2]);
    bool emitters = false;
    for (const ana::DevMaterial& m : c->h_mats)
        if (m.emission.x != 0.f || m.emission.y != 0.f || m.emission.z != 0.f) emitters = true;
    c->ds.has_emitters = emitters ? 1 : 0;
    if (nm)
        CK(cudaMemcpyAsync(c->d_scene + c->o_mats, c->h_mats.data(), nm * sizeof(ana::DevMaterial),
                           cudaMemcpyHostToDevice, c->stream),
           "materials H2D");
    if (nl)
        CK(cudaMemcpyAsync(c->d_scene + c->o_lights, c->h_lights.data(), nl * sizeof(ana::DevLight),
                           cudaMemcpyHostToDevice, c->stream),
           "lights H2D");
    CK(cudaStreamSynchronize(c->stream), "parameter upload");
    drop_graph(c);
    return ANA_OK;
}

}  // namespace

extern "C" {

int ana_version(void) { return 100; }

int ana_create(ana_ctx** out, const ana_device_opts* opts) {
    if (!out) return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_create: out is NULL");
    *out = nullptr;
    ana_ctx* c = new (std::nothrow) ana_ctx();
    if (!c) return fail(nullptr, ANA_ERR_OOM, "ana_create: host allocation failed");
    if (opts) c->opts = *opts;
    c->device = c->opts.device;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        std::string m = std::string("ana_create: no CUDA device (") + cudaGetErrorString(e) + ")";
        cudaGetLastError();
        delete c;
        return fail(nullptr, ANA_ERR_CUDA, m);
    }
    if (c->device < 0 || c->device >= n) {
        delete c;
        return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_create: device ordinal out of range");
    }
    if (c->opts.block_size && (c->opts.block_size % 32 || c->opts.block_size > 512)) {
        delete c;
        return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_create: block_size must be a multiple of 32, <= 512");
    }
    if (c->opts.traversal > ANA_TRAVERSAL_PER_RAY) {
        delete c;
        return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_create: unknown traversal schedule");
    }
    auto bail = [&](cudaError_t err, const char* what) {
        std::string m = std::string(what) + ": " + cudaGetErrorString(err);
        cudaGetLastError();
        delete c;
        return fail(nullptr, err == cudaErrorMemoryAllocation ? ANA_ERR_OOM : ANA_ERR_CUDA, m);
    };
    if ((e = cudaSetDevice(c->device)) != cudaSuccess) return bail(e, "cudaSetDevice");
    if ((e = cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking)) != cudaSuccess)
        return bail(e, "cudaStreamCreate");
    void* ep = nullptr;
    if ((e = cudaMalloc(&ep, 256)) != cudaSuccess) return bail(e, "cudaMalloc(error word)");
    c->d_err = static_cast<uint32_t*>(ep);
    c->d_work = reinterpret_cast<unsigned long long*>(static_cast<unsigned char*>(ep) + 64);
    cudaMemset(c->d_err, 0, 256);
    cudaEventCreate(&c->ev0);
    cudaEventCreate(&c->ev1);
    cudaDeviceGetAttribute(&c->num_sms, cudaDevAttrMultiProcessorCount, c->device);
    ana::prime_kernels();
    if ((e = cudaGetLastError()) != cudaSuccess) return bail(e, "kernel load");
    *out = c;
    return ANA_OK;
}

void ana_destroy(ana_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    drop_graph(c);
    cudaFree(c->d_scene);
    cudaFree(c->d_tables);
    cudaFree(c->film);
    cudaFree(c->aov_film);
    cudaFree(c->path_aov);
    cudaFree(c->d_queues);
    cudaFree(c->d_counters);
    cudaFree(c->d_err);
    cudaFree(c->d_adj);
    cudaFree(c->d_adj_io);
    for (cudaEvent_t e : c->stage_ev) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int ana_prepare_scene(const ana_scene_desc* d, ana_prepared** out) {
    if (!d || !out) return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_prepare_scene: NULL argument");
    *out = nullptr;
    ana_prepared* pp = new (std::nothrow) ana_prepared();
    if (!pp) return fail(nullptr, ANA_ERR_OOM, "ana_prepare_scene: host allocation failed");
    std::string err;
    int rc;
    try {
        rc = ana::prepare_scene(*d, pp->P, err);
        if (rc == ANA_OK) {
            const ana::Prepared* one = &pp->P;
            rc = build_blob(&one, 1, pp->blob, err);
        }
    } catch (const std::bad_alloc&) {
        delete pp;
        return fail(nullptr, ANA_ERR_OOM, "ana_prepare_scene: host allocation failed");
    }
    if (rc != ANA_OK) {
        delete pp;
        return fail(nullptr, rc, "ana_prepare_scene: " + err);
    }
    *out = pp;
    return ANA_OK;
}

uint64_t ana_prepared_bytes(const ana_prepared* p) { return p ? p->blob.size : 0; }

uint64_t ana_prepared_digest(const ana_prepared* p) {
    if (!p || !p->blob.mem) return 0;
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < p->blob.size; ++i) {
        h ^= p->blob.mem[i];
        h *= 1099511628211ULL;
    }
    return h;
}
void ana_prepared_free(ana_prepared* p) { delete p; }

int ana_upload_prepared(ana_ctx* c, const ana_prepared* p) {
    if (!c || !p) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_prepared: NULL argument");
    return upload_blob(c, p->blob);
}

int ana_upload_scene(ana_ctx* c, const ana_scene_desc* d) {
    if (!c || !d) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_scene: NULL argument");
    const auto t0 = std::chrono::steady_clock::now();
    ana_prepared* p = nullptr;
    int rc = ana_prepare_scene(d, &p);
    if (rc != ANA_OK) {
        std::lock_guard<std::mutex> lk(g_err_mu);
        c->err = g_last_err;
        return rc;
    }
    rc = ana_upload_prepared(c, p);
    if (rc == ANA_OK) {
        cudaError_t e = cudaStreamSynchronize(c->stream);
        if (e != cudaSuccess) rc = cuda_fail(c, e, "scene upload sync");
    }
    ana_prepared_free(p);
    for (int k = 0; k < 4; ++k) c->stats.build_ms[k] = 0.f;
    c->stats.build_levels = 0;
    c->stats.upload_ms =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

int ana_upload_scene_device(ana_ctx* c, const ana_scene_desc* d) {
    if (!c || !d) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_scene_device: NULL argument");
    const auto t0 = std::chrono::steady_clock::now();
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    std::unique_ptr<ana_prepared> pp(new (std::nothrow) ana_prepared());
    if (!pp) return fail(c, ANA_ERR_OOM, "ana_upload_scene_device: host allocation failed");
    std::string err;
    ana::DeviceTris dt;
    int rc;
    try {
        rc = ana::prepare_scene(*d, pp->P, err, true);
        if (rc == ANA_OK && pp->P.tris_on_device) {
            const uint32_t maxLeaf = d->max_leaf_tris ? d->max_leaf_tris : 4;
            rc = ana::build_tris_on_device(*d, maxLeaf, c->stream, dt, err);
            pp->P.dev_tri_nodes = dt.num_nodes;
        }
        if (rc == ANA_OK) {
            const ana::Prepared* one = &pp->P;
            rc = build_blob(&one, 1, pp->blob, err);
        }
    } catch (const std::bad_alloc&) {
        return fail(c, ANA_ERR_OOM, "ana_upload_scene_device: host allocation failed");
    }
    if (rc != ANA_OK) {
        cudaStreamSynchronize(c->stream);
        return fail(c, rc, "ana_upload_scene_device: " + err);
    }
    rc = upload_blob(c, pp->blob, pp->P.tris_on_device ? &dt : nullptr);
    cudaError_t e = cudaStreamSynchronize(c->stream);  // before the build buffers are freed
    if (rc == ANA_OK && e != cudaSuccess) rc = cuda_fail(c, e, "scene upload sync");
    for (int k = 0; k < 4; ++k) c->stats.build_ms[k] = dt.ms[k];
    c->stats.build_levels = dt.levels;
    c->stats.upload_ms =
        std::chrono::duration<float, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return rc;
}

static uint64_t fnv1a(const unsigned char* p, size_t n) {
    uint64_t h = 1469598103934665603ULL;
    for (size_t i = 0; i < n; ++i) {
        h ^= p[i];
        h *= 1099511628211ULL;
    }
    return h;
}

int ana_scene_digest(ana_ctx* c, uint64_t* out) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_scene_digest: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_scene_digest: no scene uploaded");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    std::vector<unsigned char> h(c->scene_bytes);
    CK(cudaMemcpyAsync(h.data(), c->d_scene, h.size(), cudaMemcpyDeviceToHost, c->stream), "scene D2H");
    CK(cudaStreamSynchronize(c->stream), "scene D2H sync");
    *out = fnv1a(h.data(), h.size());
    return ANA_OK;
}

int ana_batch_create(const ana_prepared* const* scenes, uint32_t count, ana_batch** out) {
    if (!scenes || !out || count == 0) return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_batch_create: bad arguments");
    *out = nullptr;
    std::vector<const ana::Prepared*> list(count);
    for (uint32_t k = 0; k < count; ++k) {
        if (!scenes[k]) return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_batch_create: NULL scene");
        list[k] = &scenes[k]->P;
    }
    ana_batch* b = new (std::nothrow) ana_batch();
    if (!b) return fail(nullptr, ANA_ERR_OOM, "ana_batch_create: host allocation failed");
    std::string err;
    int rc = build_blob(list.data(), count, b->blob, err);
    if (rc != ANA_OK) {
        delete b;
        return fail(nullptr, rc, "ana_batch_create: " + err);
    }
    b->items.assign(scenes, scenes + count);
    *out = b;
    return ANA_OK;
}

void ana_batch_free(ana_batch* b) { delete b; }
uint64_t ana_batch_bytes(const ana_batch* b) { return b ? b->blob.size : 0; }

int ana_upload_batch(ana_ctx* c, const ana_batch* b) {
    if (!c || !b) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_batch: NULL argument");
    return upload_blob(c, b->blob);
}

int ana_render(ana_ctx* c, const ana_render_desc* r) {
    if (!c || !r) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: NULL argument");
    if (c->has_scene && c->scenes.size() != 1)
        return fail(c, ANA_ERR_STATE, "ana_render: a batch is uploaded; use ana_render_batch");
    return render_descs(c, r, 1, r->flags);
}

int ana_render_batch(ana_ctx* c, const ana_render_desc* descs, uint32_t count, uint32_t flags) {
    return render_descs(c, descs, count, flags);
}

int ana_render_tiles(ana_ctx* c, const ana_render_desc* f, const ana_tile* tiles, uint32_t n) {
    if (!c || !f || (!tiles && n)) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_tiles: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_render_tiles: no scene uploaded");
    if (c->scenes.size() != 1)
        return fail(c, ANA_ERR_UNSUPPORTED, "ana_render_tiles: tiles render one uploaded scene, not a batch");
    const uint32_t W = f->width, H = f->height;
    if (W == 0 || H == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_tiles: empty frame");
    std::vector<uint8_t> cover(size_t(W) * H, 0);
    std::vector<Item> items;
    items.reserve(n);
    for (uint32_t i = 0; i < n; ++i) {
        const ana_tile& t = tiles[i];
        if (uint64_t(t.x0) + t.width > W || uint64_t(t.y0) + t.height > H)
            return fail(c, ANA_ERR_INVALID_ARG, "ana_render_tiles: tile " + std::to_string(i) + " outside the frame");
        if (t.width == 0 || t.height == 0 || t.sample_count == 0) continue;  // nothing to render
        for (uint32_t y = t.y0; y < t.y0 + t.height; ++y)
            for (uint32_t x = t.x0; x < t.x0 + t.width; ++x) {
                uint8_t& m = cover[size_t(y) * W + x];
                if (m) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_tiles: tiles overlap");
                m = 1;
            }
        items.push_back(Item{0, W, H, t.x0, t.y0, t.width, t.height, t.sample_start, t.sample_count, f->max_depth,
                             f->min_depth, f->seed, 0});
    }
    const uint32_t flags = f->flags & (ANA_RENDER_CLEAR_FILM | ANA_RENDER_COUNT_WORK | ANA_RENDER_AOVS);
    if (items.empty()) return (flags & ANA_RENDER_CLEAR_FILM) ? ana_film_clear(c, W, H) : ANA_OK;
    const int rc = render_items(c, items, uint64_t(W) * H, flags);
    if (rc == ANA_OK) {
        c->item_film_offset.assign(1, 0);
        c->item_film_pixels.assign(1, size_t(W) * H);
    }
    return rc;
}

int ana_render_adaptive(ana_ctx* c, const ana_render_desc* f, uint32_t ts, uint32_t baseSpp, uint32_t* extraOut,
                        uint32_t extraCap) {
    if (!c || !f) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_adaptive: NULL argument");
    if (ts == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_adaptive: tile_size is 0");
    const uint32_t W = f->width, H = f->height, total = f->sample_count;
    if (W == 0 || H == 0 || total == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_render_adaptive: empty frame");
    uint32_t base = baseSpp > 0 ? baseSpp : std::min(32u, std::max(16u, total / 16));
    base = std::min(base, total);
    const uint32_t extra = total - base;
    // scheduleTiles: row-major tiles of ts x ts pixels, clipped at the frame
    std::vector<ana_tile> tiles;
    for (uint32_t y = 0; y < H; y += ts)
        for (uint32_t x = 0; x < W; x += ts) tiles.push_back(ana_tile{x, y, std::min(ts, W - x), std::min(ts, H - y), 0, 0});
    const uint32_t nt = uint32_t(tiles.size());
    // base pass over every pixel (the base tiles cover the frame exactly)
    ana_render_desc b = *f;
    b.sample_start = 0;
    b.sample_count = base;
    b.flags = ANA_RENDER_CLEAR_FILM | (f->flags & ANA_RENDER_AOVS);  // renderTile's AOVs, as the tile loop merges them
    int rc = render_descs(c, &b, 1, b.flags);
    if (rc) return rc;
    std::vector<uint32_t> extraPerTile(nt, 0);
    if (extra > 0) {
        std::vector<ana_film_pixel> px(size_t(W) * H);
        CK(cudaMemcpyAsync(px.data(), c->film, px.size() * sizeof(ana_film_pixel), cudaMemcpyDeviceToHost,
                           c->stream),
           "film D2H");
        CK(cudaStreamSynchronize(c->stream), "film D2H");
        // Film::varianceAt: the mean luminance with Rec.709 weights against the
        // sum of squared integrator luminances, both per unit weight
        auto variance_at = [&](uint32_t x, uint32_t y) {
            const ana_film_pixel& p = px[size_t(y) * W + x];
            const float w = p.w;
            if (w <= 0.f) return 0.f;
            const float invW = 1.f / w;
            const float meanL = (p.r * 0.2126f + p.g * 0.7152f + p.b * 0.0722f) * invW;
            const float eLsq = p.sum_lum_sq * invW;
            return std::max(0.f, eLsq - meanL * meanL);
        };
        std::vector<float> logWeight(nt);
        for (uint32_t i = 0; i < nt; ++i) {
            const ana_tile& t = tiles[i];
            float sum = 0.f;
            for (uint32_t ty = 0; ty < t.height; ++ty)
                for (uint32_t tx = 0; tx < t.width; ++tx) sum += variance_at(t.x0 + tx, t.y0 + ty);
            const float tileVar = sum / static_cast<float>(t.width * t.height);
            logWeight[i] = std::log(1.f + tileVar);
        }
        float totalW = 0.f;
        for (float v : logWeight) totalW += v;
        const uint32_t uniformHalf = extra / 2, bonusHalf = extra - uniformHalf;
        for (uint32_t i = 0; i < nt; ++i) {
            uint32_t bonus = 0;
            if (totalW > 1e-6f) {
                const float frac = logWeight[i] / totalW;
                bonus = static_cast<uint32_t>(std::round(frac * static_cast<float>(bonusHalf * nt)));
            }
            extraPerTile[i] = std::min(uniformHalf + bonus, extra);
        }
        for (uint32_t i = 0; i < nt; ++i) {
            tiles[i].sample_start = base;
            tiles[i].sample_count = extraPerTile[i];
        }
        ana_render_desc e = *f;
        e.flags = f->flags & ANA_RENDER_AOVS;
        rc = ana_render_tiles(c, &e, tiles.data(), nt);
        if (rc) return rc;
    }
    if (extraOut)
        for (uint32_t i = 0; i < std::min(nt, extraCap); ++i) extraOut[i] = extraPerTile[i];
    return ANA_OK;
}

int ana_film_clear(ana_ctx* c, uint32_t w, uint32_t h) {
    if (!c || w == 0 || h == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_clear: bad size");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    size_t n = size_t(w) * h;
    int rc = ensure_buffer(c, &c->film, &c->film_bytes, n * sizeof(ana_film_pixel), "cudaMalloc(film)");
    if (rc) return rc;
    c->film_pixels = n;
    CK(cudaMemsetAsync(c->film, 0, n * sizeof(ana_film_pixel), c->stream), "memset film");
    rc = ensure_buffer(c, &c->aov_film, &c->aov_film_bytes, n * 32, "cudaMalloc(AOV film)");
    if (rc) return rc;
    CK(cudaMemsetAsync(c->aov_film, 0, n * 32, c->stream), "memset AOV film");
    c->aov_valid = true;
    return ANA_OK;
}

int ana_film_read(ana_ctx* c, ana_film_pixel* out, size_t count) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_read: NULL argument");
    if (!c->film || c->film_pixels == 0) return fail(c, ANA_ERR_STATE, "ana_film_read: no film");
    if (count != c->film_pixels)
        return fail(c, ANA_ERR_INVALID_ARG, "ana_film_read: count != pixels of the last render");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(out, c->film, count * sizeof(ana_film_pixel), cudaMemcpyDeviceToHost, c->stream), "film D2H");
    CK(cudaStreamSynchronize(c->stream), "film sync");
    return ANA_OK;
}

int ana_batch_film_read(ana_ctx* c, uint32_t item, ana_film_pixel* out, size_t count) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_batch_film_read: NULL argument");
    if (item >= c->item_film_offset.size()) return fail(c, ANA_ERR_INVALID_ARG, "ana_batch_film_read: bad item");
    if (count != c->item_film_pixels[item])
        return fail(c, ANA_ERR_INVALID_ARG, "ana_batch_film_read: count != the item's pixels");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(out, c->film_px() + c->item_film_offset[item], count * sizeof(ana_film_pixel),
                       cudaMemcpyDeviceToHost, c->stream),
       "film D2H");
    CK(cudaStreamSynchronize(c->stream), "film sync");
    return ANA_OK;
}

int ana_aov_read(ana_ctx* c, float* albedo, float* normal, size_t count) {
    if (!c) return ANA_ERR_INVALID_ARG;
    if (!c->aov_valid || !c->aov_film) return fail(c, ANA_ERR_STATE, "ana_aov_read: no AOVs in the film");
    if (count != c->film_pixels)
        return fail(c, ANA_ERR_INVALID_ARG, "ana_aov_read: count != pixels of the last render");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    std::vector<float> h(count * 8);
    CK(cudaMemcpyAsync(h.data(), c->aov_film, h.size() * 4, cudaMemcpyDeviceToHost, c->stream), "AOV D2H");
    CK(cudaStreamSynchronize(c->stream), "AOV sync");
    for (size_t i = 0; i < count; ++i)  // PixelAccumulator::resolve
        for (int l = 0; l < 2; ++l) {
            float* out = l ? normal : albedo;
            if (!out) continue;
            const float* a = h.data() + 8 * i + 4 * l;
            const float w = a[3];
            const float inv = w > 0.f ? 1.f / w : 0.f;
            for (int k = 0; k < 3; ++k) out[3 * i + k] = w > 0.f ? a[k] * inv : 0.f;
        }
    return ANA_OK;
}

// The resolved beauty film (PixelAccumulator::resolve: r * (1 / weight)).
static int resolved_film(ana_ctx* c, uint32_t w, uint32_t h, std::vector<float>& rgb) {
    if (!c->film || size_t(w) * h != c->film_pixels)
        return fail(c, ANA_ERR_INVALID_ARG, "film write: width * height != pixels of the last render");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    std::vector<ana_film_pixel> px(c->film_pixels);
    CK(cudaMemcpyAsync(px.data(), c->film, px.size() * sizeof(ana_film_pixel), cudaMemcpyDeviceToHost, c->stream),
       "film D2H");
    CK(cudaStreamSynchronize(c->stream), "film sync");
    rgb.assign(px.size() * 3, 0.f);
    for (size_t i = 0; i < px.size(); ++i) {
        if (!(px[i].w > 0.f)) continue;
        const float inv = 1.f / px[i].w;
        rgb[3 * i] = px[i].r * inv;
        rgb[3 * i + 1] = px[i].g * inv;
        rgb[3 * i + 2] = px[i].b * inv;
    }
    return ANA_OK;
}

int ana_film_write_exr(ana_ctx* c, uint32_t w, uint32_t h, const char* path, int write_aovs) {
    if (!c || !path) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_write_exr: NULL argument");
    std::vector<float> rgb, al, nr;
    int rc = resolved_film(c, w, h, rgb);
    if (rc) return rc;
    if (write_aovs) {
        al.resize(rgb.size());
        nr.resize(rgb.size());
        rc = ana_aov_read(c, al.data(), nr.data(), size_t(w) * h);
        if (rc) return rc;
    }
    rc = ana_image_write_exr(path, w, h, rgb.data(), write_aovs ? al.data() : nullptr,
                             write_aovs ? nr.data() : nullptr);
    if (rc) return fail(c, rc, std::string("ana_film_write_exr: cannot write ") + path);
    return ANA_OK;
}

int ana_film_write_png(ana_ctx* c, uint32_t w, uint32_t h, const char* path, float exposure) {
    if (!c || !path) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_write_png: NULL argument");
    std::vector<float> rgb;
    int rc = resolved_film(c, w, h, rgb);
    if (rc) return rc;
    rc = ana_image_write_png(path, w, h, rgb.data(), exposure);
    if (rc) return fail(c, rc, std::string("ana_film_write_png: cannot write ") + path);
    return ANA_OK;
}

int ana_film_device_ptr(ana_ctx* c, void** dptr) {
    if (!c || !dptr) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_device_ptr: NULL argument");
    if (!c->film) return fail(c, ANA_ERR_STATE, "ana_film_device_ptr: no film");
    *dptr = c->film;
    return ANA_OK;
}

// ana_trace_batch with optional per-ray times (host or device like the rays).
static int trace_batch(ana_ctx* c, const float* rays, const float* times, size_t n, ana_hit* out, int occlusion,
                       int on_device) {
    if (!c || (!rays && n) || (!out && n)) return fail(c, ANA_ERR_INVALID_ARG, "ana_trace_batch: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_trace_batch: no scene uploaded");
    if (n == 0) return ANA_OK;
    if (n >= (size_t(1) << 32) - 64) return fail(c, ANA_ERR_INVALID_ARG, "ana_trace_batch: n >= 2^32");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    // one scene record (scene 0: its roots) ahead of the rays
    ana::DevSceneRec R{};
    R.tri_root = c->scenes[0].tri_root;
    R.seg_root = c->scenes[0].seg_root;
    const size_t recBytes = align_up(sizeof(R));
    const size_t tmpBytes = recBytes + (on_device ? 0 : n * 32 + n * sizeof(ana_hit) + (times ? n * 4 : 0));
    void* tmp = nullptr;
    CK(cudaMalloc(&tmp, tmpBytes), "cudaMalloc(trace batch)");
    unsigned char* tb = static_cast<unsigned char*>(tmp);
    const float* d_rays = rays;
    const float* d_times = times;
    ana_hit* d_out = out;
    cudaError_t e = cudaMemcpyAsync(tb, &R, sizeof(R), cudaMemcpyHostToDevice, c->stream);
    if (!on_device) {
        d_rays = reinterpret_cast<const float*>(tb + recBytes);
        d_out = reinterpret_cast<ana_hit*>(tb + recBytes + n * 32);
        if (e == cudaSuccess) e = cudaMemcpyAsync(tb + recBytes, rays, n * 32, cudaMemcpyHostToDevice, c->stream);
        if (times) {
            float* t = reinterpret_cast<float*>(tb + recBytes + n * 32 + n * sizeof(ana_hit));
            d_times = t;
            if (e == cudaSuccess) e = cudaMemcpyAsync(t, times, n * 4, cudaMemcpyHostToDevice, c->stream);
        }
    }
    uint32_t* d_fetch = c->d_err + 32;  // fetch counter of the persistent kernel
    if (e == cudaSuccess) e = cudaMemsetAsync(c->d_err, 0, 4, c->stream);
    if (e == cudaSuccess) e = cudaMemsetAsync(d_fetch, 0, 4, c->stream);
    if (e != cudaSuccess) {
        cudaFree(tmp);
        return cuda_fail(c, e, "trace batch setup");
    }
    ana::DevScene S = c->ds;
    S.scenes = reinterpret_cast<const ana::DevSceneRec*>(tb);
    S.num_scenes = 1;
    ana::launch_trace_batch(S, 0, d_rays, d_times, n, d_out, occlusion, d_fetch, c->d_err,
                            c->opts.traversal == ANA_TRAVERSAL_PER_RAY ? 0 : 1, c->stream);
    e = cudaGetLastError();
    uint32_t herr = 0;
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(out, d_out, n * sizeof(ana_hit), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(c, e, "trace batch");
    if (herr) return fail(c, ANA_ERR_DEVICE_CHECK, "ana_trace_batch: traversal stack overflow on the device");
    return ANA_OK;
}

int ana_trace_batch(ana_ctx* c, const float* rays, size_t n, ana_hit* out, int occlusion, int on_device) {
    return trace_batch(c, rays, nullptr, n, out, occlusion, on_device);
}

int ana_trace_batch_timed(ana_ctx* c, const float* rays, const float* times, size_t n, ana_hit* out, int occlusion,
                          int on_device) {
    return trace_batch(c, rays, times, n, out, occlusion, on_device);
}

// The same query as ana_trace_batch with host buffers, staged in the fixed
// module scratch (kernels.cu) instead of a per-call cudaMalloc: callers that
// must not allocate (a pick query beside an in-flight frame, where cudaFree
// would wait for the frame; a device already full) use this one. Nothing on
// the success path allocates, on the device or on the host.
int ana_trace_batch_noalloc(ana_ctx* c, const float* rays, size_t n, ana_hit* out, int occlusion) {
    if (!c || (!rays && n) || (!out && n))
        return fail(c, ANA_ERR_INVALID_ARG, "ana_trace_batch_noalloc: NULL argument");
    if (n > ANA_TRACE_NOALLOC_MAX_RAYS)
        return fail(c, ANA_ERR_INVALID_ARG,
                    "ana_trace_batch_noalloc: " + std::to_string(n) + " rays exceed the fixed scratch of " +
                        std::to_string(ANA_TRACE_NOALLOC_MAX_RAYS) +
                        " rays; split the batch or use ana_trace_batch");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_trace_batch_noalloc: no scene uploaded");
    if (n == 0) return ANA_OK;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    unsigned char* base = nullptr;
    cudaError_t e = ana::noalloc_trace_scratch(c->device, &base);
    if (e != cudaSuccess) return cuda_fail(c, e, "ana_trace_batch_noalloc: scratch address (cudaGetSymbolAddress)");
    ana::DevSceneRec R{};
    R.tri_root = c->scenes[0].tri_root;
    R.seg_root = c->scenes[0].seg_root;
    float* d_rays = reinterpret_cast<float*>(base + ana::kNoAllocRays);
    ana_hit* d_out = reinterpret_cast<ana_hit*>(base + ana::kNoAllocHits);
    uint32_t* d_err = reinterpret_cast<uint32_t*>(base + ana::kNoAllocErrOffset);
    uint32_t* d_fetch = d_err + 1;
    e = cudaMemcpyAsync(base, &R, sizeof(R), cudaMemcpyHostToDevice, c->stream);
    // the error word and the persistent schedule's work counter start at zero
    if (e == cudaSuccess) e = cudaMemsetAsync(d_err, 0, 8, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(d_rays, rays, n * 32, cudaMemcpyHostToDevice, c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "ana_trace_batch_noalloc: setup");
    ana::DevScene S = c->ds;
    S.scenes = reinterpret_cast<const ana::DevSceneRec*>(base);
    S.num_scenes = 1;
    ana::launch_trace_batch(S, 0, d_rays, nullptr, n, d_out, occlusion, d_fetch, d_err,
                            c->opts.traversal == ANA_TRAVERSAL_PER_RAY ? 0 : 1, c->stream);
    e = cudaGetLastError();
    uint32_t herr = 0;
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, d_out, n * sizeof(ana_hit), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, d_err, 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (e != cudaSuccess) return cuda_fail(c, e, "ana_trace_batch_noalloc");
    if (herr) return fail(c, ANA_ERR_DEVICE_CHECK, "ana_trace_batch_noalloc: traversal stack overflow on the device");
    return ANA_OK;
}

int ana_bsdf_batch(ana_ctx* c, const ana_material* material, const ana_bsdf_query* q, size_t n,
                   ana_bsdf_result* out) {
    if (!c || !material || (!q && n) || (!out && n))
        return fail(c, ANA_ERR_INVALID_ARG, "ana_bsdf_batch: NULL argument");
    if (n >= (size_t(1) << 31)) return fail(c, ANA_ERR_INVALID_ARG, "ana_bsdf_batch: n >= 2^31");
    ana::DevMaterial m;
    if (const char* why = ana::make_material(*material, m))
        return fail(c, ANA_ERR_INVALID_ARG, std::string("ana_bsdf_batch: ") + why);
    if (n == 0) return ANA_OK;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const size_t qBytes = align_up(n * sizeof(ana_bsdf_query));
    void* tmp = nullptr;
    CK(cudaMalloc(&tmp, qBytes + n * sizeof(ana_bsdf_result)), "cudaMalloc(bsdf query)");
    auto* dq = static_cast<ana_bsdf_query*>(tmp);
    auto* dr = reinterpret_cast<ana_bsdf_result*>(static_cast<unsigned char*>(tmp) + qBytes);
    cudaError_t e = cudaMemcpyAsync(dq, q, n * sizeof(ana_bsdf_query), cudaMemcpyHostToDevice, c->stream);
    if (e == cudaSuccess) {
        ana::launch_bsdf_query(m, dq, uint32_t(n), dr, c->stream);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpyAsync(out, dr, n * sizeof(ana_bsdf_result), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(c, e, "ana_bsdf_batch");
    return ANA_OK;
}

int ana_diff_counts(ana_ctx* c, uint32_t* nm, uint32_t* nl) {
    if (!c || !nm || !nl) return fail(c, ANA_ERR_INVALID_ARG, "ana_diff_counts: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_diff_counts: no scene uploaded");
    *nm = uint32_t(c->h_mats.size());
    *nl = uint32_t(c->h_lights.size());
    return ANA_OK;
}

int ana_diff_get_params(ana_ctx* c, ana_diff_params* out) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_diff_get_params: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_diff_get_params: no scene uploaded");
    for (size_t i = 0; i < c->h_mats.size(); ++i) {
        const ana::DevMaterial& m = c->h_mats[i];
        const bool ss = m.type == ANA_MAT_STANDARD, em = m.type == ANA_MAT_EMISSIVE;
        if (out->albedo) {
            out->albedo[3 * i] = m.albedo.x;
            out->albedo[3 * i + 1] = m.albedo.y;
            out->albedo[3 * i + 2] = m.albedo.z;
        }
        if (out->roughness) out->roughness[i] = ss ? m.rough : 0.f;
        if (out->emission) {
            out->emission[3 * i] = em ? m.emission.x : 0.f;
            out->emission[3 * i + 1] = em ? m.emission.y : 0.f;
            out->emission[3 * i + 2] = em ? m.emission.z : 0.f;
        }
    }
    for (size_t l = 0; l < c->h_lights.size(); ++l) {
        const ana::DevLight& L = c->h_lights[l];
        const bool area = L.type == ANA_LIGHT_AREA;
        if (out->light_le) {
            out->light_le[3 * l] = area ? L.Le.x : 0.f;
            out->light_le[3 * l + 1] = area ? L.Le.y : 0.f;
            out->light_le[3 * l + 2] = area ? L.Le.z : 0.f;
        }
    }
    return ANA_OK;
}

int ana_forward(ana_ctx* c, const ana_render_desc* d, const ana_diff_params* params, float* image) {
    if (!c || !d) return fail(c, ANA_ERR_INVALID_ARG, "ana_forward: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_forward: no scene uploaded");
    if (c->scenes.size() != 1)
        return fail(c, ANA_ERR_UNSUPPORTED, "ana_forward: differentiable rendering takes one uploaded scene");
    if (c->h_mats.size() >= 0xFFFF || c->h_lights.size() >= 0xFFFF)
        return fail(c, ANA_ERR_UNSUPPORTED, "ana_forward: more than 65534 materials or lights");
    for (const ana::DevMaterial& m : c->h_mats)
        if (m.transmission > 0.001f || m.opacity < 1.f || m.tint.x != 0.f || m.tint.y != 0.f || m.tint.z != 0.f)
            return fail(c, ANA_ERR_UNSUPPORTED, "ana_forward: glass and alpha-masked materials are not differentiated");
    if (c->ds.has_motion)
        return fail(c, ANA_ERR_UNSUPPORTED, "ana_forward: motion-blurred meshes are not differentiated");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    c->fwd_valid = false;
    if (params) {
        int rc = apply_params(c, params);
        if (rc) return rc;
    }
    const uint32_t flags = ANA_RENDER_CLEAR_FILM | (d->flags & ANA_RENDER_GRAPH);
    int rc = render_descs(c, d, 1, flags);
    if (rc) return rc;
    c->fwd_desc = *d;
    c->fwd_valid = true;
    if (image) {
        const size_t n = size_t(d->width) * d->height;
        std::vector<ana_film_pixel> px(n);
        CK(cudaMemcpy(px.data(), c->film, n * sizeof(ana_film_pixel), cudaMemcpyDeviceToHost), "film D2H");
        for (size_t i = 0; i < n; ++i) {  // Film::getPixel
            const float w = px[i].w;
            image[3 * i] = w > 0.f ? px[i].r / w : 0.f;
            image[3 * i + 1] = w > 0.f ? px[i].g / w : 0.f;
            image[3 * i + 2] = w > 0.f ? px[i].b / w : 0.f;
        }
    }
    return ANA_OK;
}

int ana_backward(ana_ctx* c, const float* d_image, ana_diff_params* out) {
    if (!c || !d_image || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_backward: NULL argument");
    if (!c->fwd_valid) return fail(c, ANA_ERR_STATE, "ana_backward: no ana_forward since the last scene change");
    const size_t nm = c->h_mats.size(), nl = c->h_lights.size();
    std::vector<float> g(8 * nm + 4 * nl, 0.f);
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    int rc = render_descs(c, &c->fwd_desc, 1, 0, d_image, g.data());
    if (rc) return rc;
    for (size_t i = 0; i < nm; ++i) {
        for (int ch = 0; ch < 3; ++ch) {
            if (out->albedo) out->albedo[3 * i + ch] = g[8 * i + ch];
            if (out->emission) out->emission[3 * i + ch] = g[8 * i + 4 + ch];
        }
        if (out->roughness) out->roughness[i] = g[8 * i + 3];
    }
    for (size_t l = 0; l < nl; ++l)
        for (int ch = 0; ch < 3; ++ch)
            if (out->light_le) out->light_le[3 * l + ch] = g[8 * nm + 4 * l + ch];
    return ANA_OK;
}

int ana_get_stats(ana_ctx* c, ana_stats* out) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_get_stats: NULL argument");
    *out = c->stats;
    return ANA_OK;
}

int ana_last_error(ana_ctx* c, char* buf, size_t len) {
    if (!buf || len == 0) return ANA_ERR_INVALID_ARG;
    std::string m;
    if (c) m = c->err;
    else {
        std::lock_guard<std::mutex> lk(g_err_mu);
        m = g_last_err;
    }
    std::snprintf(buf, len, "%s", m.c_str());
    return ANA_OK;
}

}  // extern "C"
