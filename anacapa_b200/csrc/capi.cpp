// C ABI of the B200 path-tracing hot path (include/anacapa_b200.h).
#include <cuda_runtime.h>

#include <algorithm>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <mutex>
#include <new>
#include <string>
#include <vector>

#include "../../include/anacapa_b200.h"
#include "kernels.h"
#include "prepare.h"

namespace {

std::mutex g_err_mu;
std::string g_last_err;

void set_global_err(const std::string& m) {
    std::lock_guard<std::mutex> lk(g_err_mu);
    g_last_err = m;
}

constexpr size_t kAlign = 256;
inline size_t align_up(size_t x) { return (x + kAlign - 1) & ~(kAlign - 1); }

}  // namespace

// A prepared scene: one contiguous host blob (pinned when CUDA is present)
// holding every device array at 256-byte aligned offsets, so uploading is a
// single host-to-device copy.
struct ana_prepared {
    unsigned char* blob = nullptr;
    size_t size = 0;
    bool pinned = false;
    // offsets into blob
    size_t o_tri_nodes = 0, o_tri_isect = 0, o_tri_shade = 0, o_seg_nodes = 0, o_segs = 0, o_scol = 0,
           o_mats = 0, o_slots = 0, o_lights = 0, o_env_rgb = 0, o_cf = 0, o_cc = 0, o_ci = 0, o_mf = 0,
           o_mc = 0;
    uint32_t n_tri_nodes = 0, n_tris = 0, n_seg_nodes = 0, n_segs = 0, n_mats = 0, n_slots = 0, n_lights = 0;
    bool tri_root_empty = true;
    bool has_emitters = false;
    ana::HostEnv env_meta;  // sizes and scalars only (arrays live in the blob)
    ana_camera camera{};
    ~ana_prepared() {
        if (!blob) return;
        if (pinned) cudaFreeHost(blob);
        else std::free(blob);
    }
};

struct ana_ctx {
    int device = 0;
    cudaStream_t stream = nullptr;
    std::string err;
    ana_device_opts opts{};
    // scene
    unsigned char* d_scene = nullptr;
    size_t d_scene_size = 0;
    ana::DevScene ds{};
    ana_camera camera{};
    bool has_scene = false;
    // film
    ana_film_pixel* film = nullptr;
    uint32_t fw = 0, fh = 0;
    // wavefront buffers
    ana::Queues q{};
    unsigned char* d_queues = nullptr;
    uint32_t cap = 0;
    uint32_t* d_counters = nullptr;
    size_t counters_cap = 0;
    uint32_t* d_err = nullptr;
    unsigned long long* d_work = nullptr;  // 3 work counters (in the error-word allocation)
    std::vector<uint32_t> h_counters;
    std::vector<cudaEvent_t> stage_ev;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    ana_stats stats{};
    int num_sms = 148;
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

#define CK(call, what)                                   \
    do {                                                 \
        cudaError_t e_ = (call);                         \
        if (e_ != cudaSuccess) return cuda_fail(c, e_, what); \
    } while (0)

template <class T>
void put(unsigned char* blob, size_t off, const std::vector<T>& v) {
    if (!v.empty()) std::memcpy(blob + off, v.data(), v.size() * sizeof(T));
}

int build_prepared(const ana::Prepared& P, ana_prepared& out) {
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes);
        return o;
    };
    out.o_tri_nodes = take(P.tri_nodes.size() * sizeof(ana::BvhNode));
    out.o_tri_isect = take(P.tri_isect.size() * 16);
    out.o_tri_shade = take(P.tri_shade.size() * 16);
    out.o_seg_nodes = take(P.seg_nodes.size() * sizeof(ana::BvhNode));
    out.o_segs = take(P.segs.size() * 16);
    out.o_scol = take(P.strand_color.size() * 4);
    out.o_mats = take(P.materials.size() * sizeof(ana::DevMaterial));
    out.o_slots = take(P.slot_material.size() * 4);
    out.o_lights = take(P.lights.size() * sizeof(ana::DevLight));
    out.o_env_rgb = take(P.env.rgb.size() * 4);
    out.o_cf = take(P.env.cond_func.size() * 4);
    out.o_cc = take(P.env.cond_cdf.size() * 4);
    out.o_ci = take(P.env.cond_int.size() * 4);
    out.o_mf = take(P.env.marg_func.size() * 4);
    out.o_mc = take(P.env.marg_cdf.size() * 4);
    out.size = std::max<size_t>(off, kAlign);
    void* mem = nullptr;
    if (cudaHostAlloc(&mem, out.size, cudaHostAllocPortable) == cudaSuccess) {
        out.pinned = true;
    } else {
        cudaGetLastError();
        mem = std::aligned_alloc(kAlign, out.size);
        out.pinned = false;
        if (!mem) return ANA_ERR_OOM;
    }
    out.blob = static_cast<unsigned char*>(mem);
    std::memset(out.blob, 0, out.size);
    put(out.blob, out.o_tri_nodes, P.tri_nodes);
    put(out.blob, out.o_tri_isect, P.tri_isect);
    put(out.blob, out.o_tri_shade, P.tri_shade);
    put(out.blob, out.o_seg_nodes, P.seg_nodes);
    put(out.blob, out.o_segs, P.segs);
    put(out.blob, out.o_scol, P.strand_color);
    put(out.blob, out.o_mats, P.materials);
    put(out.blob, out.o_slots, P.slot_material);
    put(out.blob, out.o_lights, P.lights);
    put(out.blob, out.o_env_rgb, P.env.rgb);
    put(out.blob, out.o_cf, P.env.cond_func);
    put(out.blob, out.o_cc, P.env.cond_cdf);
    put(out.blob, out.o_ci, P.env.cond_int);
    put(out.blob, out.o_mf, P.env.marg_func);
    put(out.blob, out.o_mc, P.env.marg_cdf);
    out.n_tri_nodes = uint32_t(P.tri_nodes.size());
    out.n_tris = P.num_tris;
    out.n_seg_nodes = uint32_t(P.seg_nodes.size());
    out.n_segs = P.num_segs;
    out.n_mats = uint32_t(P.materials.size());
    out.n_slots = uint32_t(P.slot_material.size());
    out.n_lights = uint32_t(P.lights.size());
    out.tri_root_empty = P.tri_root_is_empty;
    out.has_emitters = P.has_emitters;
    out.env_meta.present = P.env.present;
    out.env_meta.width = P.env.width;
    out.env_meta.height = P.env.height;
    out.env_meta.intensity = P.env.intensity;
    out.env_meta.marg_int = P.env.marg_int;
    std::memcpy(out.env_meta.radiance, P.env.radiance, sizeof(P.env.radiance));
    out.camera = P.camera;
    return ANA_OK;
}

// Wavefront buffers for `cap` paths.
int ensure_queues(ana_ctx* c, uint32_t cap) {
    if (c->cap >= cap && c->d_queues) return ANA_OK;
    if (c->d_queues) {
        cudaFree(c->d_queues);
        c->d_queues = nullptr;
        c->cap = 0;
    }
    size_t f4 = size_t(cap) * 16;
    size_t total = 14 * align_up(f4) + align_up(size_t(cap) * 12);
    void* mem = nullptr;
    CK(cudaMalloc(&mem, total), "cudaMalloc(wavefront queues)");
    unsigned char* b = static_cast<unsigned char*>(mem);
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
    c->q.L = reinterpret_cast<float*>(take(size_t(cap) * 12));
    c->q.mis_c = reinterpret_cast<float4*>(take(f4));
    c->d_queues = b;
    c->cap = cap;
    return ANA_OK;
}

int ensure_film(ana_ctx* c, uint32_t w, uint32_t h, bool clear) {
    if (c->film && (c->fw != w || c->fh != h)) {
        cudaFree(c->film);
        c->film = nullptr;
    }
    if (!c->film) {
        void* mem = nullptr;
        CK(cudaMalloc(&mem, size_t(w) * h * sizeof(ana_film_pixel)), "cudaMalloc(film)");
        c->film = static_cast<ana_film_pixel*>(mem);
        c->fw = w;
        c->fh = h;
        clear = true;
    }
    if (clear) CK(cudaMemsetAsync(c->film, 0, size_t(w) * h * sizeof(ana_film_pixel), c->stream), "memset film");
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
    *out = c;
    return ANA_OK;
}

void ana_destroy(ana_ctx* c) {
    if (!c) return;
    cudaSetDevice(c->device);
    if (c->stream) cudaStreamSynchronize(c->stream);
    cudaFree(c->d_scene);
    cudaFree(c->film);
    cudaFree(c->d_queues);
    cudaFree(c->d_counters);
    cudaFree(c->d_err);
    for (cudaEvent_t e : c->stage_ev) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

int ana_prepare_scene(const ana_scene_desc* d, ana_prepared** out) {
    if (!d || !out) return fail(nullptr, ANA_ERR_INVALID_ARG, "ana_prepare_scene: NULL argument");
    *out = nullptr;
    ana::Prepared P;
    std::string err;
    int rc;
    try {
        rc = ana::prepare_scene(*d, P, err);
    } catch (const std::bad_alloc&) {
        return fail(nullptr, ANA_ERR_OOM, "ana_prepare_scene: host allocation failed");
    }
    if (rc != ANA_OK) return fail(nullptr, rc, "ana_prepare_scene: " + err);
    ana_prepared* pp = new (std::nothrow) ana_prepared();
    if (!pp) return fail(nullptr, ANA_ERR_OOM, "ana_prepare_scene: host allocation failed");
    rc = build_prepared(P, *pp);
    if (rc != ANA_OK) {
        delete pp;
        return fail(nullptr, rc, "ana_prepare_scene: blob allocation failed");
    }
    *out = pp;
    return ANA_OK;
}

uint64_t ana_prepared_bytes(const ana_prepared* p) { return p ? p->size : 0; }
void ana_prepared_free(ana_prepared* p) { delete p; }

int ana_upload_prepared(ana_ctx* c, const ana_prepared* p) {
    if (!c || !p) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_prepared: NULL argument");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    if (c->d_scene_size < p->size) {
        CK(cudaStreamSynchronize(c->stream), "sync");
        cudaFree(c->d_scene);
        c->d_scene = nullptr;
        c->d_scene_size = 0;
        void* mem = nullptr;
        CK(cudaMalloc(&mem, p->size), "cudaMalloc(scene)");
        c->d_scene = static_cast<unsigned char*>(mem);
        c->d_scene_size = p->size;
    }
    CK(cudaMemcpyAsync(c->d_scene, p->blob, p->size, cudaMemcpyHostToDevice, c->stream), "scene upload");
    unsigned char* b = c->d_scene;
    ana::DevScene& S = c->ds;
    S = ana::DevScene{};
    S.tri_nodes = reinterpret_cast<const ana::BvhNode*>(b + p->o_tri_nodes);
    S.tri_isect = reinterpret_cast<const float4*>(b + p->o_tri_isect);
    S.tri_shade = reinterpret_cast<const float4*>(b + p->o_tri_shade);
    S.num_tri_nodes = p->n_tri_nodes;
    S.num_tris = p->n_tris;
    S.tri_root_is_empty = p->tri_root_empty ? 1 : 0;
    S.seg_nodes = reinterpret_cast<const ana::BvhNode*>(b + p->o_seg_nodes);
    S.segs = reinterpret_cast<const float4*>(b + p->o_segs);
    S.strand_color = reinterpret_cast<const float*>(b + p->o_scol);
    S.num_seg_nodes = p->n_seg_nodes;
    S.num_segs = p->n_segs;
    S.materials = reinterpret_cast<const ana::DevMaterial*>(b + p->o_mats);
    S.slot_material = reinterpret_cast<const int32_t*>(b + p->o_slots);
    S.num_materials = p->n_mats;
    S.num_slots = p->n_slots;
    S.lights = reinterpret_cast<const ana::DevLight*>(b + p->o_lights);
    S.num_lights = p->n_lights;
    S.has_emitters = p->has_emitters ? 1 : 0;
    ana::DevEnv& E = S.env;
    E.present = p->env_meta.present ? 1 : 0;
    E.rgb = E.present ? reinterpret_cast<const float*>(b + p->o_env_rgb) : nullptr;
    E.cond_func = reinterpret_cast<const float*>(b + p->o_cf);
    E.cond_cdf = reinterpret_cast<const float*>(b + p->o_cc);
    E.cond_int = reinterpret_cast<const float*>(b + p->o_ci);
    E.marg_func = reinterpret_cast<const float*>(b + p->o_mf);
    E.marg_cdf = reinterpret_cast<const float*>(b + p->o_mc);
    E.marg_int = p->env_meta.marg_int;
    E.intensity = p->env_meta.intensity;
    E.width = p->env_meta.width;
    E.height = p->env_meta.height;
    E.radiance = make_float3(p->env_meta.radiance[0], p->env_meta.radiance[1], p->env_meta.radiance[2]);
    c->camera = p->camera;
    c->has_scene = true;
    return ANA_OK;
}

int ana_upload_scene(ana_ctx* c, const ana_scene_desc* d) {
    if (!c || !d) return fail(c, ANA_ERR_INVALID_ARG, "ana_upload_scene: NULL argument");
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
    return rc;
}

int ana_film_clear(ana_ctx* c, uint32_t w, uint32_t h) {
    if (!c || w == 0 || h == 0) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_clear: bad size");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    return ensure_film(c, w, h, true);
}

int ana_film_read(ana_ctx* c, ana_film_pixel* out, size_t count) {
    if (!c || !out) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_read: NULL argument");
    if (!c->film) return fail(c, ANA_ERR_STATE, "ana_film_read: no film");
    if (count != size_t(c->fw) * c->fh) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_read: count != width*height");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    CK(cudaMemcpyAsync(out, c->film, count * sizeof(ana_film_pixel), cudaMemcpyDeviceToHost, c->stream), "film D2H");
    CK(cudaStreamSynchronize(c->stream), "film sync");
    return ANA_OK;
}

int ana_film_device_ptr(ana_ctx* c, void** dptr) {
    if (!c || !dptr) return fail(c, ANA_ERR_INVALID_ARG, "ana_film_device_ptr: NULL argument");
    if (!c->film) return fail(c, ANA_ERR_STATE, "ana_film_device_ptr: no film");
    *dptr = c->film;
    return ANA_OK;
}

int ana_render(ana_ctx* c, const ana_render_desc* r) {
    if (!c || !r) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_render: no scene uploaded");
    if (r->width == 0 || r->height == 0 || r->sample_count == 0)
        return fail(c, ANA_ERR_INVALID_ARG, "ana_render: empty frame or zero samples");
    if (r->max_depth > 255) return fail(c, ANA_ERR_INVALID_ARG, "ana_render: max_depth > 255");
    uint64_t npix = uint64_t(r->width) * r->height;
    if (npix * r->sample_count >= (1ull << 32))
        return fail(c, ANA_ERR_INVALID_ARG, "ana_render: width*height*sample_count must be < 2^32");
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    int rc = ensure_film(c, r->width, r->height, (r->flags & ANA_RENDER_CLEAR_FILM) != 0);
    if (rc) return rc;
    uint32_t want = c->opts.chunk_paths ? c->opts.chunk_paths : (1u << 22);
    if (want < r->sample_count) want = r->sample_count;
    uint32_t chunk_px = want / r->sample_count;
    if (uint64_t(chunk_px) > npix) chunk_px = uint32_t(npix);
    uint32_t cap = chunk_px * r->sample_count;
    rc = ensure_queues(c, cap);
    if (rc) return rc;
    uint32_t nchunks = uint32_t((npix + chunk_px - 1) / chunk_px);
    uint32_t rows = r->max_depth + 2;
    size_t ncount = size_t(nchunks) * rows * ana::kCountersPerBounce;
    if (c->counters_cap < ncount) {
        cudaFree(c->d_counters);
        c->d_counters = nullptr;
        void* mem = nullptr;
        CK(cudaMalloc(&mem, ncount * 4), "cudaMalloc(counters)");
        c->d_counters = static_cast<uint32_t*>(mem);
        c->counters_cap = ncount;
    }
    CK(cudaMemsetAsync(c->d_counters, 0, ncount * 4, c->stream), "memset counters");
    CK(cudaMemsetAsync(c->d_err, 0, 4, c->stream), "memset err");

    ana::Params p{};
    p.S = c->ds;
    p.S.cam = ana::make_camera(c->camera, r->width, r->height);
    p.q = c->q;
    p.film = c->film;
    p.err = c->d_err;
    p.seed = r->seed;
    p.W = r->width;
    p.H = r->height;
    p.spp = r->sample_count;
    p.sample_start = r->sample_start;
    p.max_depth = r->max_depth;
    p.min_depth = r->min_depth;
    ana::LaunchCfg cfg;
    cfg.block = c->opts.block_size ? int(c->opts.block_size) : 256;
    cfg.persistent = c->opts.traversal == ANA_TRAVERSAL_PER_RAY ? 0 : 1;
    long long gcap = ((long long)cap + cfg.block - 1) / cfg.block;
    cfg.grid_cap = int(std::max<long long>(1, std::min<long long>(gcap, 1 << 20)));
    const bool count_work = (r->flags & ANA_RENDER_COUNT_WORK) != 0;
    p.work = c->d_work;
    if (count_work) CK(cudaMemsetAsync(c->d_work, 0, 3 * sizeof(unsigned long long), c->stream), "memset work");
    // Per-stage CUDA events (timing mode): one pair per launch, on this stream.
    const bool timing = c->opts.timing != 0;
    const size_t launches = size_t(nchunks) * (2 + 4 * (r->max_depth + 1));
    if (timing && c->stage_ev.size() < 2 * launches) {
        size_t old = c->stage_ev.size();
        c->stage_ev.resize(2 * launches);
        for (size_t i = old; i < c->stage_ev.size(); ++i) CK(cudaEventCreate(&c->stage_ev[i]), "event create");
    }
    std::vector<int> stage_of;
    if (timing) stage_of.reserve(launches);
    size_t ev_i = 0;
    auto timed = [&](int stage, auto&& launch) {
        if (timing) cudaEventRecord(c->stage_ev[2 * ev_i], c->stream);
        launch();
        if (timing) {
            cudaEventRecord(c->stage_ev[2 * ev_i + 1], c->stream);
            stage_of.push_back(stage);
            ++ev_i;
        }
    };
    CK(cudaEventRecord(c->ev0, c->stream), "event");
    for (uint32_t k = 0; k < nchunks; ++k) {
        p.chunk_first_pixel = k * chunk_px;
        p.chunk_pixels = uint32_t(std::min<uint64_t>(chunk_px, npix - uint64_t(k) * chunk_px));
        p.counters = c->d_counters + size_t(k) * rows * ana::kCountersPerBounce;
        p.bounce = 0;
        timed(4, [&] { ana::launch_generate(p, cfg, c->stream); });
        for (uint32_t b = 0; b <= r->max_depth; ++b) {
            p.bounce = b;
            timed(0, [&] { ana::launch_extend(p, cfg, c->stream, count_work); });
            timed(1, [&] { ana::launch_shade(p, cfg, c->stream); });
            timed(2, [&] { ana::launch_shadow(p, cfg, c->stream); });
            timed(3, [&] { ana::launch_mis(p, cfg, c->stream); });
        }
        timed(4, [&] { ana::launch_film(p, cfg, c->stream); });
    }
    CK(cudaGetLastError(), "kernel launch");
    CK(cudaEventRecord(c->ev1, c->stream), "event");
    unsigned long long hwork[3] = {0, 0, 0};
    if (count_work)
        CK(cudaMemcpyAsync(hwork, c->d_work, sizeof(hwork), cudaMemcpyDeviceToHost, c->stream), "work D2H");
    c->h_counters.resize(ncount);
    CK(cudaMemcpyAsync(c->h_counters.data(), c->d_counters, ncount * 4, cudaMemcpyDeviceToHost, c->stream),
       "counters D2H");
    uint32_t herr = 0;
    CK(cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream), "err D2H");
    CK(cudaStreamSynchronize(c->stream), "render sync");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, c->ev0, c->ev1);
    ana_stats& st = c->stats;
    st = ana_stats{};
    st.paths = npix * r->sample_count;
    for (uint32_t k = 0; k < nchunks; ++k)
        for (uint32_t b = 0; b < rows; ++b) {
            const uint32_t* cc = c->h_counters.data() + (size_t(k) * rows + b) * ana::kCountersPerBounce;
            if (b <= r->max_depth) st.extend_rays += cc[0];
            st.shadow_rays += cc[1];
            st.mis_rays += cc[2];
            if (cc[0]) st.bounces = std::max(st.bounces, b + 1);
        }
    st.render_ms = ms;
    st.chunks = nchunks;
    st.kernel_launches = launches;
    st.extend_launches = size_t(nchunks) * (r->max_depth + 1);
    st.node_fetches = hwork[0];
    st.tri_tests = hwork[1];
    st.seg_tests = hwork[2];
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

int ana_trace_batch(ana_ctx* c, const float* rays, size_t n, ana_hit* out, int occlusion, int on_device) {
    if (!c || (!rays && n) || (!out && n)) return fail(c, ANA_ERR_INVALID_ARG, "ana_trace_batch: NULL argument");
    if (!c->has_scene) return fail(c, ANA_ERR_STATE, "ana_trace_batch: no scene uploaded");
    if (n == 0) return ANA_OK;
    CK(cudaSetDevice(c->device), "cudaSetDevice");
    const float* d_rays = rays;
    ana_hit* d_out = out;
    void* tmp = nullptr;
    if (!on_device) {
        CK(cudaMalloc(&tmp, n * 32 + n * sizeof(ana_hit)), "cudaMalloc(trace batch)");
        d_rays = static_cast<const float*>(tmp);
        d_out = reinterpret_cast<ana_hit*>(static_cast<unsigned char*>(tmp) + n * 32);
        cudaError_t e = cudaMemcpyAsync(tmp, rays, n * 32, cudaMemcpyHostToDevice, c->stream);
        if (e != cudaSuccess) {
            cudaFree(tmp);
            return cuda_fail(c, e, "rays H2D");
        }
    }
    if (n >= (size_t(1) << 32) - 64) return fail(c, ANA_ERR_INVALID_ARG, "ana_trace_batch: n >= 2^32");
    uint32_t* d_fetch = c->d_err + 32;  // fetch counter of the persistent kernel
    CK(cudaMemsetAsync(c->d_err, 0, 4, c->stream), "memset err");
    CK(cudaMemsetAsync(d_fetch, 0, 4, c->stream), "memset fetch");
    ana::launch_trace_batch(c->ds, d_rays, n, d_out, occlusion, d_fetch, c->d_err,
                            c->opts.traversal == ANA_TRAVERSAL_PER_RAY ? 0 : 1, c->stream);
    cudaError_t e = cudaGetLastError();
    uint32_t herr = 0;
    if (e == cudaSuccess && !on_device)
        e = cudaMemcpyAsync(out, d_out, n * sizeof(ana_hit), cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaMemcpyAsync(&herr, c->d_err, 4, cudaMemcpyDeviceToHost, c->stream);
    if (e == cudaSuccess) e = cudaStreamSynchronize(c->stream);
    if (tmp) cudaFree(tmp);
    if (e != cudaSuccess) return cuda_fail(c, e, "trace batch");
    if (herr) return fail(c, ANA_ERR_DEVICE_CHECK, "ana_trace_batch: traversal stack overflow on the device");
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
