/*
 * anacapa_b200 — C ABI of the B200 path-tracing hot path.
 *
 * This is the boundary a host renderer binds. Every entry point returns an
 * int status (ANA_OK = 0); no C++ exception crosses it. All pointers are plain
 * host pointers unless a parameter says otherwise; the library copies what it
 * needs and the caller keeps ownership of every array it passes in.
 *
 * Each declaration names the reference interface it replaces (paths relative
 * to the nhaflinger/anacapa source tree).
 *
 * Threading: one ana_ctx per host thread, one CUDA stream per context; calls
 * on one context are serialised by the caller (the reference calls
 * IIntegrator::renderFrame from its main thread only,
 * src/render/RenderSession.cpp:541).
 */
#ifndef ANACAPA_B200_H
#define ANACAPA_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ------------------------------------------------------ */
enum {
    ANA_OK = 0,
    ANA_ERR_INVALID_ARG = 1,   /* bad pointer, size, index or enum            */
    ANA_ERR_CUDA = 2,          /* a CUDA runtime call failed                   */
    ANA_ERR_OOM = 3,           /* device allocation failed                     */
    ANA_ERR_TIMEOUT = 4,       /* a device-side bounded wait gave up           */
    ANA_ERR_UNSUPPORTED = 5,   /* feature outside the implemented path         */
    ANA_ERR_STATE = 6,         /* call out of order (e.g. render before scene) */
    ANA_ERR_DEVICE_CHECK = 7   /* a device bounds check tripped (stack, index) */
};

/* ---- materials (src/shading/*.h) ----------------------------------------- */
enum {
    ANA_MAT_LAMBERT = 0,   /* LambertianMaterial  src/shading/Lambertian.h:29-82        */
    ANA_MAT_EMISSIVE = 1,  /* EmissiveMaterial    src/shading/Lambertian.h:88-99        */
    ANA_MAT_STANDARD = 2,  /* StandardSurfaceMaterial src/shading/StandardSurface.h:115 */
    ANA_MAT_HAIR = 3       /* MarschnerHairMaterial src/shading/MarschnerHair.h:190     */
};

/* Hair evaluation mode. The reference's MarschnerHairMaterial::evaluate/sample
 * return the Kajiya-Kay lobe before reaching the Marschner code
 * (src/shading/MarschnerHair.h:240, 267-282); KAJIYA_KAY reproduces what the
 * reference executes, MARSCHNER evaluates the R/TT/TRT lobes it defines. */
enum { ANA_HAIR_KAJIYA_KAY = 0, ANA_HAIR_MARSCHNER = 1 };

typedef struct ana_material {
    uint32_t type;
    /* Lambert / Emissive */
    float albedo[3];
    float emission[3];
    /* standard_surface, StandardSurfaceMaterial::Params (StandardSurface.h:117-148);
     * constant values only (evalTOV's non-texture branch, Texture.cpp:126-136) */
    float base_color[3];
    float base;
    float metalness;
    float roughness;
    float specular;
    float specular_color[3];
    float specular_ior;
    float coat;
    float coat_roughness;
    float transmission;    /* > 0.001: dielectric glass (smooth below roughness 0.001, else
                              GGX transmission), StandardSurface.h:245-340, 380-414 */
    float emission_weight; /* Params::emission */
    float emission_color[3];
    uint32_t alpha_mask;   /* Params::alphaMask: opacity below drives alpha testing */
    /* hair, MarschnerHairMaterial::Params (MarschnerHair.h:192-198) */
    float eta;
    float sigma_a[3];
    float beta_m;
    float beta_n;
    float alpha_deg;
    uint32_t hair_mode;    /* ANA_HAIR_* */
    /* standard_surface Params::opacity (constant), read when alpha_mask is set:
     * evalOpacity and the shadow tint 1 - opacity (StandardSurface.h:197-218) */
    float opacity;
} ana_material;

/* ---- lights (include/anacapa/shading/ILight.h) ----------------------------- */
enum {
    ANA_LIGHT_AREA = 0,  /* AreaLight src/shading/lights/AreaLight.h:17-125: quad centre,
                            half-extent axes u and v, radiance Le                     */
    ANA_LIGHT_DOME = 1,  /* DomeLight src/shading/lights/DomeLight.h:205: the scene's
                            equirect environment (ana_scene_desc.env_*)               */
    ANA_LIGHT_DIRECTIONAL = 2 /* DirectionalLight src/shading/lights/DirectionalLight.h:24-160:
                            a delta light at infinity; u = direction toward the light,
                            Le, half_angle_deg = angular radius (0: hard shadows)     */
};

typedef struct ana_light {
    uint32_t type;
    float center[3];
    float u[3];
    float v[3];
    float Le[3];
    float half_angle_deg;
} ana_light;

/* ---- camera (Camera, include/anacapa/integrator/IIntegrator.h:27-144) ------ */
typedef struct ana_camera {
    float from[3];
    float at[3];
    float up[3];
    float vfov_deg;
    float aperture_radius;  /* 0 = pinhole (Camera::makePinhole)                  */
    float focal_distance;   /* thin lens (Camera::makeThinLens) when aperture > 0 */
    float shutter_open;
    float shutter_close;
    /* explicit_basis != 0: use an already built Camera (its origin,
     * lowerLeftCorner, horizontal, vertical, basisU, basisV) instead of
     * from/at/up/vfov; the film size must be the one it was built for. */
    uint32_t explicit_basis;
    float origin[3];
    float lower_left[3];
    float horizontal[3];
    float vertical[3];
    float basis_u[3];
    float basis_v[3];
} ana_camera;

/* A motion key (MotionKey, include/anacapa/accel/GeometryPool.h:16-20): a
 * normalized shutter time and the object-to-world matrix there, row-major
 * (m[row][col]; a point p maps to m * (p, 1) divided by its w). */
typedef struct ana_motion_key {
    float time;
    float object_to_world[16];
} ana_motion_key;

/* ---- scene (GeometryPool + CurvePool + SceneView) ------------------------- */
typedef struct ana_scene_desc {
    /* Triangle meshes (MeshDesc, include/anacapa/accel/GeometryPool.h:28-77),
     * concatenated. Mesh i owns vertices [mesh_vert_offset[i], mesh_vert_offset[i+1])
     * and triangles [mesh_tri_offset[i], mesh_tri_offset[i+1]); indices are local to
     * the mesh's vertex range. meshID = i, primID = triangle index within the mesh. */
    uint32_t num_meshes;
    const uint32_t* mesh_vert_offset;  /* num_meshes + 1 */
    const uint32_t* mesh_tri_offset;   /* num_meshes + 1 */
    const uint8_t* mesh_has_normals;   /* num_meshes; 0 = geometric normal everywhere */
    const float* positions;            /* 3 per vertex, world space (static meshes)   */
    const float* normals;              /* 3 per vertex (read where has_normals)       */
    const uint32_t* indices;           /* 3 per triangle                               */

    /* Hair strands (StrandDesc, include/anacapa/accel/CurvePool.h:27-55). */
    uint32_t num_strands;
    const uint32_t* strand_cp_offset;    /* num_strands + 1 */
    const float* control_points;         /* 3 per CV; segment k uses CVs 3k..3k+3 */
    const uint32_t* strand_width_offset; /* num_strands + 1 */
    const float* widths;                 /* diameters, StrandDesc::widthAt rules */
    const uint32_t* strand_slot;         /* StrandDesc::materialIndex            */
    const float* strand_color;           /* 3 per strand                          */

    /* SceneView::materials: slot -> material (index into materials, -1 = none).
     * Indexed by meshID and by StrandDesc::materialIndex. */
    uint32_t num_materials;
    const ana_material* materials;
    uint32_t num_slots;
    const int32_t* slot_material;

    /* SceneView::lights in order (the integrator picks one uniformly). */
    uint32_t num_lights;
    const ana_light* lights;

    /* SceneView::envLight: equirect RGB float, row 0 = zenith (DomeLight.h:190-201).
     * env_rgb == NULL: constant SceneView::envRadiance. */
    const float* env_rgb;
    uint32_t env_width;
    uint32_t env_height;
    float env_intensity;
    float env_radiance[3];

    ana_camera camera;

    /* BVH build: maximum triangles / curve segments per leaf (reference: 4,
     * BVHBackend.h:67, CurveBrute.cpp:455). 0 = default: 4 triangles, 1 curve
     * segment (the same hits; each segment's box is tested in its node). */
    uint32_t max_leaf_tris;
    uint32_t max_leaf_segments;

    /* Motion blur (MeshDesc::motionKeys): mesh i owns the keys
     * [mesh_motion_offset[i], mesh_motion_offset[i+1]) of motion_keys, sorted
     * by time. A mesh without keys is static (world-space positions); a mesh
     * with keys keeps object-space positions, bounded over all keys, and each
     * ray meets it transformed by the keys interpolated at the ray's time and
     * inverted (BVHBackend.cpp:35-50, 86-95, 356-367, 395-398). A ray's time
     * is the camera's shutter sample (Camera::generateRay). NULL: all static. */
    const uint32_t* mesh_motion_offset;
    const ana_motion_key* motion_keys;
} ana_scene_desc;

/* ---- render ---------------------------------------------------------------- */
typedef struct ana_render_desc {
    uint32_t width;        /* film size (filmWidth, filmHeight)                     */
    uint32_t height;
    uint32_t sample_start; /* first sample index (TileRequest::sampleStart)         */
    uint32_t sample_count; /* samples per pixel this call (TileRequest::sampleCount)*/
    uint32_t max_depth;    /* PathIntegrator(maxDepth), PathIntegrator.h:24          */
    uint32_t min_depth;    /* Russian roulette from this bounce (reference: 2)      */
    uint64_t seed;         /* HaltonSampler seed (RenderSession uses 0)             */
    uint32_t flags;        /* ANA_RENDER_* */
} ana_render_desc;

enum {
    ANA_RENDER_CLEAR_FILM = 1u << 0, /* zero the film before accumulating              */
    ANA_RENDER_COUNT_WORK = 1u << 1, /* count BVH node fetches and primitive tests of the
                                        closest-hit stage (instrumented, slower)        */
    ANA_RENDER_GRAPH = 1u << 2,      /* capture the whole chunk x bounce launch sequence
                                        in a CUDA graph on first use and replay it while
                                        the scenes and descs are unchanged (no per-stage
                                        timing, no work counting)                         */
    ANA_RENDER_AOVS = 1u << 3        /* denoising AOVs (PathIntegrator::renderTile,
                                        PathIntegrator.cpp:31-66): each path's first shaded
                                        surface gives IMaterial::reflectance and the shading
                                        normal; per pixel their averages over the call's
                                        samples (the normal renormalised) are added to the
                                        AOV film with weight 1, as Film::mergeTile does;
                                        honoured by ana_render, ana_render_batch,
                                        ana_render_tiles (per tile) and ana_render_adaptive */
};

/* One device-resident film pixel: the reference's PixelAccumulator
 * (include/anacapa/film/Film.h:24-56): pre-weighted r, g, b, weight, and
 * sum of luminance(sample)^2. */
typedef struct ana_film_pixel {
    float r, g, b, w, sum_lum_sq;
} ana_film_pixel;

/* Closest-hit record of ana_trace_batch (SurfaceInteraction ids,
 * include/anacapa/accel/IAccelerationStructure.h:12-30). */
typedef struct ana_hit {
    int32_t hit;        /* 1 hit, 0 miss (occlusion queries: 1 = occluded)   */
    int32_t mesh_id;    /* meshID, or the strand's material slot for curves   */
    int32_t prim_id;    /* triangle index in its mesh, or curve segment index */
    int32_t strand_id;  /* -1 for triangles                                    */
    float t;
    float u, v;         /* barycentrics (triangles) / strand parameter (curves)*/
    float pad;
} ana_hit;

typedef struct ana_stats {
    uint64_t paths;             /* camera paths traced by the last render     */
    uint64_t extend_rays;       /* closest-hit continuation rays              */
    uint64_t shadow_rays;       /* NEE shadow rays                            */
    uint64_t mis_rays;          /* BSDF-sampled MIS rays toward lights         */
    float render_ms;            /* device time of the last render (CUDA events)*/
    float extend_ms, shade_ms, shadow_ms, mis_ms, film_ms; /* per-stage totals
                                   (device_opts.timing = 1), CUDA events on the
                                   context's stream around every launch           */
    uint32_t bounces;           /* wavefront iterations of the last render      */
    uint32_t chunks;            /* path chunks of the last render               */
    uint64_t kernel_launches;   /* kernels this library launched in the render  */
    uint64_t extend_launches;   /* of which closest-hit (extend) launches       */
    uint64_t node_fetches;      /* ANA_RENDER_COUNT_WORK: 128-byte triangle BVH
                                   node loads (4-wide nodes)                     */
    uint64_t tri_tests;         /*   triangle tests (48 bytes each)              */
    uint64_t seg_tests;         /*   curve segment tests (80 bytes each)         */
    uint64_t curve_node_fetches;/*   128-byte curve BVH node loads (4-wide)      */
    float upload_ms;            /* wall time of the last scene upload call      */
    float build_ms[4];          /* ana_upload_scene_device phases (wall time):
                                   inputs + triangle setup, SAH levels, small
                                   subtrees, 4-wide collapse + layout           */
    uint32_t build_levels;      /* SAH levels run over the large nodes          */
} ana_stats;

typedef struct ana_ctx ana_ctx;

typedef struct ana_device_opts {
    int device;              /* CUDA ordinal                                   */
    uint32_t chunk_paths;    /* wavefront capacity in paths (0 = 2^25)         */
    uint32_t block_size;     /* threads per block of the shading kernel (0 = default 256;
                                larger requests run 256-thread blocks)            */
    uint32_t timing;         /* 1: record per-stage CUDA-event times           */
    uint32_t traversal;      /* ANA_TRAVERSAL_*: schedule of the BVH traversal kernels */
} ana_device_opts;

enum {
    ANA_TRAVERSAL_DEFAULT = 0,     /* the library's choice (persistent)              */
    ANA_TRAVERSAL_PERSISTENT = 1,  /* persistent warps refilling finished lanes      */
    ANA_TRAVERSAL_PER_RAY = 2      /* one thread per ray, grid-stride               */
};

/* Create a context on a device. Replaces CudaPathIntegrator's constructor /
 * CudaContext (src/gpu/cuda/CudaContext.cu:37-58). */
int ana_create(ana_ctx** out, const ana_device_opts* opts);
void ana_destroy(ana_ctx* ctx);

/* Copy a scene to the device and build its BVHs on the host with the
 * reference's algorithms (triangle SAH BVH, BVHBackend::commit,
 * src/accel/BVHBackend.cpp:17-228; curve median-split BVH,
 * src/accel/CurveBrute.cpp:247-396). Replaces IIntegrator::prepare
 * (include/anacapa/integrator/IIntegrator.h:177) + IAccelerationStructure::commit. */
int ana_upload_scene(ana_ctx* ctx, const ana_scene_desc* scene);

/* ana_upload_scene with the triangle setup and SAH BVH build of
 * BVHBackend::commit (src/accel/BVHBackend.cpp:17-228) run on the device:
 * level-synchronous binned SAH over the large nodes, one thread per small
 * subtree, the 4-wide collapse on the device. The uploaded bytes equal
 * ana_upload_scene's (ana_scene_digest). Curves, materials, lights and the
 * dome are prepared on the host as there. */
int ana_upload_scene_device(ana_ctx* ctx, const ana_scene_desc* scene);

/* FNV-1a 64 of the uploaded scene arena (no counterpart in the reference):
 * equals ana_prepared_digest of the same scene prepared on the host. */
int ana_scene_digest(ana_ctx* ctx, uint64_t* out);

/* Host-side scene preparation split from the device copy, so a caller can
 * build once and re-upload: ana_prepare_scene builds the device layout on the
 * host; ana_upload_prepared copies it (host -> device) into the context. */
typedef struct ana_prepared ana_prepared;
int ana_prepare_scene(const ana_scene_desc* scene, ana_prepared** out);
int ana_upload_prepared(ana_ctx* ctx, const ana_prepared* prep);
uint64_t ana_prepared_bytes(const ana_prepared* prep);
/* 64-bit FNV-1a digest of the prepared device layout (a cache key; equal
 * scenes and build options give equal digests). */
uint64_t ana_prepared_digest(const ana_prepared* prep);
void ana_prepared_free(ana_prepared* prep);

/* Render sample_count samples per pixel of the whole frame into the
 * device-resident film (adds, as Film::mergeTile does). Replaces
 * IIntegrator::renderFrame (IIntegrator.h:192-197) for PathIntegrator
 * (src/integrator/PathIntegrator.cpp:8-265). */
int ana_render(ana_ctx* ctx, const ana_render_desc* desc);

/* ---- batches: many scenes, resolutions, spp budgets and depths in one launch
 * sequence. A batch concatenates prepared scenes into one device arena (each
 * scene keeps its own BVHs, materials and lights); ana_render_batch renders
 * item k with descs[k] into its own film. Paths of all items share the
 * wavefront queues, so small items do not leave the GPU idle. There is no
 * reference counterpart: the reference renders one scene per RenderSession
 * (src/render/RenderSession.cpp:402-547); this is the batched form north of
 * it. A batch may hold at most one dome light. */
typedef struct ana_batch ana_batch;
int ana_batch_create(const ana_prepared* const* scenes, uint32_t count, ana_batch** out);
void ana_batch_free(ana_batch* batch);
uint64_t ana_batch_bytes(const ana_batch* batch);
int ana_upload_batch(ana_ctx* ctx, const ana_batch* batch);
int ana_render_batch(ana_ctx* ctx, const ana_render_desc* descs, uint32_t count, uint32_t flags);
/* Film of one item of the last batch render (width*height pixels of that item). */
int ana_batch_film_read(ana_ctx* ctx, uint32_t item, ana_film_pixel* host_out, size_t count);

/* Zero / read back the device film (width*height ana_film_pixel, row 0 = top).
 * After a batch render, ana_film_read returns all items' films back to back. */
int ana_film_clear(ana_ctx* ctx, uint32_t width, uint32_t height);
int ana_film_read(ana_ctx* ctx, ana_film_pixel* host_out, size_t count);
/* Device pointer of the film, for callers that keep the result on the GPU. */
int ana_film_device_ptr(ana_ctx* ctx, void** dptr);

/* The AOV film (Film::m_albedo, m_normals) resolved as PixelAccumulator::resolve
 * does, 3 floats per pixel each (either pointer may be NULL); count = pixels of
 * the last render, which must have accumulated AOVs (ANA_RENDER_AOVS) since the
 * film was last cleared. */
int ana_aov_read(ana_ctx* ctx, float* albedo_rgb, float* normal_xyz, size_t count);

/* Film::writeEXR (src/film/Film.cpp:154-219): R, G, B of the resolved film and,
 * with write_aovs, the albedo.* and normals.* layers; 32-bit float channels, ZIP
 * compression. Film::writePNG (Film.cpp:224-272): 8-bit sRGB of the resolved
 * film scaled by 2^exposure, written to path + ".writing.png" and renamed. The
 * film is the last render's (width * height pixels). */
int ana_film_write_exr(ana_ctx* ctx, uint32_t width, uint32_t height, const char* path, int write_aovs);
int ana_film_write_png(ana_ctx* ctx, uint32_t width, uint32_t height, const char* path, float exposure);

/* The same writers for host images (row 0 = top, 3 floats per pixel; albedo
 * and normal may be NULL). No device needed. */
int ana_image_write_exr(const char* path, uint32_t width, uint32_t height, const float* rgb,
                        const float* albedo, const float* normal);
int ana_image_write_png(const char* path, uint32_t width, uint32_t height, const float* rgb, float exposure);

/* Batched closest-hit / occlusion queries. rays: n x 8 floats
 * (ox, oy, oz, tmin, dx, dy, dz, tmax). Replaces
 * IAccelerationStructure::traceBatch / occludedBatch
 * (include/anacapa/accel/IAccelerationStructure.h:75-87) over CurveBrute
 * (src/accel/CurveBrute.cpp:398-476). rays_on_device != 0: rays and out are
 * device pointers. */
int ana_trace_batch(ana_ctx* ctx, const float* rays, size_t n, ana_hit* out, int occlusion_only,
                    int rays_on_device);

/* ana_trace_batch with each ray's Ray::time (n floats, NULL: 0; on the device
 * with rays_on_device): motion-blurred meshes are met at that time
 * (BVHBackend.cpp:356-367, 420-435). */
int ana_trace_batch_timed(ana_ctx* ctx, const float* rays, const float* times, size_t n, ana_hit* out,
                          int occlusion_only, int rays_on_device);

/* ana_trace_batch without any device allocation (no counterpart in the
 * reference). ana_trace_batch takes a temporary device buffer per call
 * (cudaMalloc / cudaFree); this variant stages the rays, the hits and its
 * counters in a fixed scratch array that lives in the library's module
 * memory, one per device. It is for callers that cannot allocate device
 * memory at the moment they trace: a viewer answering a pick or hover query
 * while a frame renders on another stream (cudaFree waits for all work on
 * the device, so the query would stall until the frame ends), and a process
 * whose device memory is already held by the scene, the films and a caching
 * allocator (an allocation there can fail mid-session).
 *   rays: host array of n x 8 floats as for ana_trace_batch; out: host array
 *   of n hits. n <= ANA_TRACE_NOALLOC_MAX_RAYS, else ANA_ERR_INVALID_ARG and
 *   nothing runs. The call returns after the hits are in `out`.
 * The first call on a device looks up the scratch address
 * (cudaGetSymbolAddress, with the context's device current) and caches it
 * for the device's current CUDA context (after a device reset the next call
 * looks it up again); make that first call before any stream capture begins
 * on the device. Each
 * call zeroes the error word and work counter of the scratch itself; rays
 * and hits need no clearing. The scratch is shared by every context on the
 * device: calls that overlap in time (two threads, two contexts on one
 * device) race on it and must be serialised by the caller. */
#define ANA_TRACE_NOALLOC_MAX_RAYS 65536
int ana_trace_batch_noalloc(ana_ctx* ctx, const float* rays, size_t n, ana_hit* out, int occlusion_only);

/* ---- BSDF queries ------------------------------------------------------------
 * IMaterial::evaluate and IMaterial::sample (include/anacapa/shading/IMaterial.h:
 * 53-80) of one material, run on the device for a batch of shading frames:
 * the device code the renderer shades with, without a scene (material
 * previews, BSDF plots, checks of the lobes). The frame is built as
 * ShadingContext does (include/anacapa/shading/ShadingContext.h:28-50) from a
 * surface interaction with shading and geometric normal n, fiber tangent t
 * (is_curve != 0: hair) and per-strand colour, hit by a ray travelling along
 * -wo. For hair materials hair_mode selects the Kajiya-Kay lobe the reference
 * executes (MarschnerHair.h:240, 267-282) or the R/TT/TRT lobes it defines
 * (MarschnerHair.h:242-257, 284-375). */
typedef struct ana_bsdf_query {
    float n[3];
    float t[3];
    float color[3];
    float wo[3];
    float wi[3];       /* direction evaluate() is asked about                     */
    float u[2];        /* sample(): the 2-D sample and the component sample       */
    float u_comp;
    uint32_t is_curve;
} ana_bsdf_query;

typedef struct ana_bsdf_result {
    float f[3];        /* evaluate(): BSDFEval::f (no cosine) and pdf             */
    float pdf;
    float sample_f[3]; /* sample(): BSDFSample::f (times |cos theta_i|), pdf, wi  */
    float sample_pdf;
    float sample_wi[3];
    uint32_t sample_flags; /* BSDFFlags of the sample (0 when it is invalid)      */
} ana_bsdf_result;

int ana_bsdf_batch(ana_ctx* ctx, const ana_material* material, const ana_bsdf_query* queries, size_t n,
                   ana_bsdf_result* out);

/* ---- tiles and adaptive sampling ------------------------------------------ */
/* A tile of a frame (TileRequest, include/anacapa/integrator/IIntegrator.h):
 * pixels [x0, x0 + width) x [y0, y0 + height), sample indices
 * [sample_start, sample_start + sample_count). */
typedef struct ana_tile {
    uint32_t x0, y0, width, height;
    uint32_t sample_start, sample_count;
} ana_tile;

/* PathIntegrator::renderTile (src/integrator/PathIntegrator.cpp:8-69) over n
 * tiles of one frame, in one launch sequence, each merged into the frame's
 * film as Film::mergeTile does (Film.cpp:34-73). frame gives the film size,
 * depths and seed; its sample_start/sample_count are unused; with
 * ANA_RENDER_CLEAR_FILM the film is cleared first. Tiles must lie inside the
 * frame and must not overlap (ANA_ERR_INVALID_ARG). */
int ana_render_tiles(ana_ctx* ctx, const ana_render_desc* frame, const ana_tile* tiles, uint32_t n);

/* RenderSession::render's adaptive two-pass schedule for a tile-rendering
 * integrator (src/render/RenderSession.cpp:548-653): tiles of tile_size
 * pixels in row-major order (scheduleTiles, RenderSession.cpp:380-397); a base
 * pass of base_spp samples per pixel (0: min(32, max(16, spp / 16)), at most
 * spp); the mean Film::varianceAt (Film.cpp:80-90) of each tile; then every
 * tile gets extra/2 + round(log(1 + var) / sum log(1 + var) * (extra - extra/2)
 * * tiles) more samples (at most extra = spp - base), from sample index base.
 * frame->sample_count is the total spp; the film is cleared first. When
 * extra_out is not NULL it receives the extra samples of each tile
 * (extra_capacity entries at most; the tile count is
 * ceil(W / tile_size) * ceil(H / tile_size)). */
int ana_render_adaptive(ana_ctx* ctx, const ana_render_desc* frame, uint32_t tile_size, uint32_t base_spp,
                        uint32_t* extra_out, uint32_t extra_capacity);

/* ---- differentiable rendering: path-replay adjoint ------------------------
 * A forward/backward pair with autograd-Function semantics over the uploaded
 * scene (one scene, not a batch). Parameters, by uploaded material index i
 * and light index l (NULL arrays are left unchanged / not written):
 *   albedo[i][3]     Lambert and emissive albedo, standard_surface base_color
 *   roughness[i]     standard_surface specular_roughness (others: unused, 0)
 *   emission[i][3]   emissive material Le (others: unused, 0)
 *   light_le[l][3]   area light Le (dome: unused, 0)
 * ana_forward writes the parameters into the scene, renders the frame of
 * `desc` (as ana_render with ANA_RENDER_CLEAR_FILM) and returns the resolved
 * image (width x height x 3 floats, Film::getPixel) when image_out is not
 * NULL. It keeps only the frame description: the sample indices and seed fix
 * every path. ana_backward takes dLoss/d image (same layout) and returns
 * dLoss/d parameters: it replays every path of that frame twice, once for its
 * radiance L and once to propagate the adjoint (Vicini, Speierer, Jakob 2021:
 * sampling decisions, pdfs, MIS weights and roulette are held fixed), and
 * reduces the per-path gradients per warp in FP32 before atomic adds. Hair
 * parameters and the dome are not differentiated. */
typedef struct ana_diff_params {
    float* albedo;
    float* roughness;
    float* emission;
    float* light_le;
} ana_diff_params;

int ana_diff_counts(ana_ctx* ctx, uint32_t* num_materials, uint32_t* num_lights);
/* Current parameter values (as uploaded, or as last set by ana_forward). */
int ana_diff_get_params(ana_ctx* ctx, ana_diff_params* out);
int ana_forward(ana_ctx* ctx, const ana_render_desc* desc, const ana_diff_params* params, float* image_out);
int ana_backward(ana_ctx* ctx, const float* d_image, ana_diff_params* grad_out);

int ana_get_stats(ana_ctx* ctx, ana_stats* out);

/* Copy the last error message of this context (or of the last failed
 * context-less call when ctx is NULL) into buf. */
int ana_last_error(ana_ctx* ctx, char* buf, size_t len);

/* Library/ABI version: major * 10000 + minor * 100 + patch. */
int ana_version(void);

#ifdef __cplusplus
}
#endif
#endif /* ANACAPA_B200_H */
