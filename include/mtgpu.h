/*
 * mtgpu.h - C ABI of the B200 (sm_100a) renderer core for marmel-trace.
 *
 * The library renders marmel-trace scenes on the GPU behind the same entry
 * points the reference exposes to its CLI:
 *
 *   mt_pathtrace_render   <- pathtrace_render   (src/pathtrace.h:78-80)
 *   mt_render_image_ex    <- render_image_ex    (src/render.h:65, src/render.c:1627)
 *   mt_render_image       <- render_image       (src/render.h:29, src/render.c:1522)
 *   mt_pathtrace_radiance <- pathtrace_radiance (src/pathtrace.h:48), batched
 *   mt_intersect          <- scene_intersect    (src/scene.c:767), batched
 *   mt_occluded           <- scene_occluded     (src/scene.c:804), batched
 *   mt_camera_create      <- camera_create      (src/camera.c:24-66)
 *
 * Every signature uses plain C types, pointers and sizes. The reference's
 * own `Scene` / `Camera` structs are converted to the flat descriptors below
 * by a small binding on the reference side (see the integration notes);
 * nothing here depends on the reference headers.
 *
 * Return codes follow the reference exactly for argument errors
 * (src/pathtrace.c:1260-1268, src/render.c:1630-1641):
 *   0 ok, 1 NULL pointer, 2 non-positive dimensions, 3 bad spp / depth,
 * and add codes >= 10 for device-side failures. Unsupported scene content
 * (CSG, SDF, bump maps, starfield / nebula / galaxy sky terms) is rejected
 * with MT_ERR_UNSUPPORTED; there is no CPU fallback. The adjoint also
 * rejects fog, textures, volumetric clouds and marched media.
 *
 * Threading: a scene handle may be used from one host thread at a time.
 * All calls are synchronous unless they take a `stream` argument.
 */
#ifndef MTGPU_H
#define MTGPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------ */
/* Status codes                                                        */
/* ------------------------------------------------------------------ */
#define MT_OK               0
#define MT_ERR_NULL         1   /* NULL pointer (reference code 1)          */
#define MT_ERR_DIMS         2   /* width/height <= 0 (reference code 2)     */
#define MT_ERR_COUNTS       3   /* spp < 1 or depth < 0 (reference code 3)  */
#define MT_ERR_NO_DEVICE    10  /* no usable CUDA device                    */
#define MT_ERR_OOM          11  /* device or host allocation failed         */
#define MT_ERR_LAUNCH       12  /* kernel launch / execution error          */
#define MT_ERR_WATCHDOG     13  /* a bounded device loop hit its cap        */
#define MT_ERR_UNSUPPORTED  14  /* scene feature outside the GPU path       */
#define MT_ERR_INVALID      15  /* malformed descriptor / option            */
#define MT_ERR_OVERFLOW     16  /* a device queue or stack ran out of room  */

/* ------------------------------------------------------------------ */
/* Scene descriptor (mirrors the renderer-visible parts of `Scene`)     */
/* ------------------------------------------------------------------ */

/* Primitive kinds, numbered as the reference's PrimKind (src/geometry.h:32-40). */
#define MT_PRIM_SPHERE   0
#define MT_PRIM_PLANE    1
#define MT_PRIM_BOX      2
#define MT_PRIM_TRIANGLE 3
#define MT_PRIM_CYLINDER 4

/*
 * One primitive, in the reference's `Primitive` order (src/geometry.h:42-66).
 * The array index is the reference `prim_index` used for the equal-t
 * tie-break (src/bvh.c:641-646), so the caller must keep file order.
 *   SPHERE   : v[0..2] center, v[3] radius
 *   PLANE    : v[0..2] point,  v[3..5] unit normal
 *   BOX      : v[0..2] center, v[3..5] half extents
 *   TRIANGLE : v[0..2] a, v[3..5] b, v[6..8] c; when `smooth` is set,
 *              n[0..8] are the vertex normals na, nb, nc (the reference's
 *              prim_triangle_smooth, radius > 0.5 gate, src/geometry.c:506)
 *   CYLINDER : v[0..2] base, v[3..5] top, v[6] r_bottom, v[7] r_top
 * A TRIANGLE with `has_uv` set carries vertex texture coordinates
 * uv = (ua, va, ub, vb, uc, vc) (prim_triangle_uv, src/geometry.c:280-295);
 * its hit (u, v) interpolates them instead of being the barycentrics.
 */
typedef struct {
    int32_t kind;
    int32_t material;
    int32_t smooth;
    int32_t has_uv;
    double  v[9];
    double  n[9];
    double  uv[6];
} mt_prim;

/* Surface material: the `Material` fields the hot path reads (src/material.h). */
typedef struct {
    double  albedo[3];
    double  specular[3];
    double  shininess;
    double  reflectivity;
    double  transparency;
    double  ior;
    double  absorption[3];
    double  deep_color[3];
    double  metallic;
    double  roughness;
    double  emissive[3];
    double  atmosphere_glow[3];
    double  bump_strength;   /* must be <= 1e-6 (bump maps are not on the GPU path) */
    int32_t is_water;
    int32_t beer_lambert;
    int32_t pbr;
    int32_t texture_kind;    /* MT_TEXTURE_* (TextureKind, src/material.h:33-42)   */
    double  texture_scale;   /* world units per cell / UV repeat; <= 0 means 1     */
    double  texture_color_a[3];
    double  texture_color_b[3];
    /* MT_TEXTURE_IMAGE: texture_width x texture_height sRGB bytes, RGB, top row
       first (ImageTexture, src/texture.h); the library copies them at scene
       creation. NULL leaves the albedo untextured, as the reference does. */
    const unsigned char *texture_rgb;
    int32_t texture_width;
    int32_t texture_height;
} mt_material;

/* Material.texture_kind values (TextureKind, src/material.h:33-42). */
#define MT_TEXTURE_NONE         0
#define MT_TEXTURE_CHECKER      1
#define MT_TEXTURE_STRIPES      2
#define MT_TEXTURE_PLANET_EARTH 3
#define MT_TEXTURE_PLANET_MOON  4
#define MT_TEXTURE_NOISE        5
#define MT_TEXTURE_IMAGE        6
#define MT_TEXTURE_UV_CHECKER   7

/* Sky / sun parameters (SkyParams, src/material.h). */
typedef struct {
    double   sun_dir[3];
    double   sun_color[3];
    double   horizon_color[3];
    double   zenith_color[3];
    double   gradient_gamma;
    double   sun_glow_exponent;
    double   sun_glow_strength;
    double   cloud_height;
    double   cloud_scale;
    double   cloud_coverage;
    double   cloud_softness;
    double   cloud_sharpness;
    double   cloud_thickness;   /* > 1e-4: volumetric ray-marched slab   */
    double   sun_radius;        /* degrees; 0 = hard sun                 */
    double   star_intensity;    /* must be 0                             */
    double   nebula_intensity;  /* must be 0                             */
    double   galaxy_intensity;  /* must be 0                             */
    int32_t  cloud_octaves;
    uint32_t seed;
    double   cloud_density;     /* volumetric extinction (<= 0 means 0.08) */
    int32_t  cloud_steps;       /* volumetric march steps                 */
    int32_t  reserved;
} mt_sky;

/* Procedural Gerstner ocean height parameters (SceneOceanParams, src/scene.h:67-77). */
typedef struct {
    int32_t  enabled;
    uint32_t seed;
    double   center[3];
    double   amplitude;
    double   wavelength;
    double   direction[3];
    double   chop;
    double   chop_wavelength;
} mt_ocean;

typedef struct {
    const mt_prim     *prims;
    int32_t            prim_count;
    int32_t            material_count;
    const mt_material *materials;
    mt_sky             sky;
    double             fog_density;     /* FogParams.density (0 = no fog)        */
    double             water_level;     /* Scene.water_level                     */
    int32_t            water_material;  /* Scene.water_material, -1 = none      */
    int32_t            fog_shadow_steps;/* FogParams.shadow_steps (0 = analytic) */
    mt_ocean           ocean;           /* Scene.has_ocean / ocean_params        */
    /* the rest of FogParams (src/material.h:199-209) */
    double             fog_color[3];
    double             fog_height;
    double             fog_height_falloff;
    double             fog_inscatter_strength;
    double             fog_sun_anisotropy;
    double             fog_noise_scale;
    double             fog_noise_amount;
} mt_scene_desc;

/* Pinhole / thin-lens camera (Camera, src/camera.h). */
typedef struct {
    double position[3];
    double lower_left[3];
    double horizontal[3];
    double vertical[3];
    double aperture;
    double focus_distance;
    double dome_radius;
    double anamorphic_squeeze;
} mt_camera;

/* Fixed / adaptive Whitted parameters (RenderParams, src/render.h:49-55). */
typedef struct {
    int32_t samples_per_pixel;
    int32_t max_depth;
    int32_t adaptive;          /* 1 = adaptive refinement (src/render.c:1128-1500) */
    int32_t adaptive_max_spp;
    double  adaptive_tau;
} mt_render_params;

/* ------------------------------------------------------------------ */
/* Build / render options                                              */
/* ------------------------------------------------------------------ */

/* Arithmetic of the device path. FP32 is the production path; FP64 follows
 * the reference's double-precision expression order operation by operation
 * and is the exact-parity mode. */
#define MT_PRECISION_FP32 0
#define MT_PRECISION_FP64 1

/* Integrator for the path tracer. */
#define MT_INTEGRATOR_MEGAKERNEL 0   /* one thread per pixel, full bounce loop    */
#define MT_INTEGRATOR_WAVEFRONT  1   /* per-bounce stage kernels + queues         */

typedef struct {
    int32_t precision;       /* MT_PRECISION_*                                  */
    int32_t integrator;      /* MT_INTEGRATOR_*                                 */
    int32_t block_size;      /* threads per block, 0 = library default          */
    int32_t queue_capacity;  /* wavefront paths in flight, 0 = library default  */
    int32_t bvh_width;       /* 2, 4 or 8; 0 = library default                  */
    int32_t sort_threshold;  /* wavefront: sort a bounce's hits by material and place when
                                it holds at least this many paths (0 = never; default 1 << 18) */
    int32_t use_graph;       /* wavefront: 1 = capture the sample window in a CUDA graph,
                                0 = plain launches, -1 = plain launches timed per stage */
    int32_t device;          /* CUDA device ordinal                             */
    int32_t traversal;       /* wavefront traversal kernels: MT_TRAVERSAL_*     */
    int32_t bvh_builder;     /* MT_BVH_BUILDER_*                                */
    int32_t occluder_cache;  /* wavefront shadow stage: 0 = library default (on
                                for scenes whose materials stop every shadow ray,
                                off for scenes with water or transparency > 0.8),
                                1 = on for every scene, -1 = off (every
                                connection walks the tree)                      */
} mt_options;

/* Where the scene's BVH is built. Both run the reference's binned-SAH
 * algorithm (src/bvh.c:180-422) and give the same tree; the device build
 * orders the primitives inside each node differently (mt_bvh_build_device). */
#define MT_BVH_BUILDER_HOST   0  /* single host thread, the reference's node order */
#define MT_BVH_BUILDER_DEVICE 1  /* breadth-first on the scene's device           */

/* Wavefront traversal kernels (extend and shadow stages). */
#define MT_TRAVERSAL_DEFAULT 0   /* library default (grid-stride)                    */
#define MT_TRAVERSAL_STATIC  1   /* grid-stride loop: one ray per lane per pass      */
#define MT_TRAVERSAL_DYNAMIC 2   /* persistent lanes that refill from the queue as   */
                                 /* their rays finish                                 */

/* Fill `o` with the library defaults (FP32, megakernel, BVH2, device 0). */
void mt_options_default(mt_options *o);

/* ------------------------------------------------------------------ */
/* Scene lifetime                                                      */
/* ------------------------------------------------------------------ */

typedef struct mt_scene mt_scene;

/*
 * Build the acceleration structure on the host (binned SAH, 12 bins, leaf
 * size 4, planes kept out of the tree: src/bvh.c:40-48,180-422), flatten it
 * into the device node layout and upload everything to device memory.
 * `opts` may be NULL (defaults). On success *out owns the device copy and
 * must be released with mt_scene_release.
 */
int  mt_scene_create(const mt_scene_desc *desc, const mt_options *opts, mt_scene **out);
void mt_scene_release(mt_scene *scene);

/* Introspection: tree node count, depth, emissive-light count, device bytes. */
typedef struct {
    int32_t prim_count;
    int32_t plane_count;
    int32_t node_count;       /* binary tree nodes, as bvh_node_count()     */
    int32_t depth;            /* leaf depth, root = 1, as bvh_depth()       */
    int32_t light_count;      /* emissive sphere lights (<= 8)              */
    int32_t light_prims[8];   /* their prim indices, file order             */
    int64_t device_bytes;     /* device memory held by the scene            */
} mt_scene_info;
int mt_scene_get_info(const mt_scene *scene, mt_scene_info *info);

/* Export the host BVH (for parity checks against the reference builder):
 * nodes as {min xyz, max xyz} doubles plus {left, right, first, count} ints
 * in the reference's node order, and the prim permutation `order`. Arrays
 * may be NULL to query sizes only. */
int mt_scene_export_bvh(const mt_scene *scene, double *bounds6, int32_t *links4,
                        int32_t *order, int32_t *node_count, int32_t *order_count);

/* Host-only build of the same BVH (no device needed): nodes, permutation and
 * leaf depth exactly as mt_scene_export_bvh reports them. Call once with NULL
 * arrays to query the sizes. */
int mt_bvh_build_host(const mt_prim *prims, int32_t prim_count, double *bounds6, int32_t *links4,
                      int32_t *order, int32_t *node_count, int32_t *order_count, int32_t *depth);

/* The same build on a CUDA device (bvh_build's algorithm, breadth-first):
 * the nodes, bounds, leaves and preorder numbering of mt_bvh_build_host, with
 * the primitives of each node in a different order (a stable partition
 * replaces the reference's in-place swap partition). The one exception is a
 * median split whose midpoint rounds onto the smallest centroid (centroids
 * one ulp apart): it splits the current order at count / 2, as the reference
 * does, and that order differs. build_ms (optional): device time of the
 * build. Call once with NULL arrays to query the sizes (each call builds). */
int mt_bvh_build_device(const mt_prim *prims, int32_t prim_count, int32_t device, double *bounds6, int32_t *links4,
                        int32_t *order, int32_t *node_count, int32_t *order_count, int32_t *depth, float *build_ms);

/* ------------------------------------------------------------------ */
/* Camera                                                              */
/* ------------------------------------------------------------------ */

/* Restates camera_create (src/camera.c:24-66): look-at basis and viewport. */
void mt_camera_create(const double from[3], const double at[3], const double up[3],
                      double vfov_deg, double aspect, mt_camera *out);

/* ------------------------------------------------------------------ */
/* Renderers (drop-in entry points)                                     */
/* ------------------------------------------------------------------ */

/*
 * Path-traced image into a top-down row-major RGB8 buffer of w*h*3 bytes
 * (src/pathtrace.h:62-80). Per-pixel jitter, lens samples and seeds follow
 * pt_render_pixel (src/pathtrace.c:1047-1096).
 */
int mt_pathtrace_render(mt_scene *scene, const mt_camera *cam, int width, int height,
                        int samples_per_pixel, int max_depth, unsigned char *rgb_out);

/* Whitted renderer, fixed spp (render_image, src/render.c:1522-1625). */
int mt_render_image(mt_scene *scene, const mt_camera *cam, int width, int height,
                    int samples_per_pixel, int max_depth, unsigned char *rgb_out);

/* render_image_ex (src/render.c:1627-1665): fixed or adaptive Whitted. */
int mt_render_image_ex(mt_scene *scene, const mt_camera *cam, int width, int height,
                       const mt_render_params *params, unsigned char *rgb_out);

/*
 * Linear (pre-gamma) per-pixel mean radiance, w*h*3 floats, top-down.
 * mode 0 = path tracer, 1 = Whitted. `out` is host memory. This is the
 * FP32 image the progressive / RMSE measurements read.
 */
#define MT_MODE_PATHTRACE 0
#define MT_MODE_WHITTED   1
int mt_render_linear(mt_scene *scene, const mt_camera *cam, int width, int height,
                     int samples_per_pixel, int max_depth, int mode, float *out);

/*
 * Same as mt_render_linear but for a sample window [spp_begin, spp_end) and
 * with DEVICE output: `accum_dev` (w*h*3 floats) receives the SUM of the
 * window's samples (added to its contents when `accumulate` is 1), so a
 * progressive render is a sequence of windows. Asynchronous on `stream`
 * (a cudaStream_t, NULL = legacy default stream). Used by the benchmark.
 */
int mt_render_accumulate_device(mt_scene *scene, const mt_camera *cam, int width, int height,
                                int spp_begin, int spp_end, int max_depth, int mode,
                                float *accum_dev, int accumulate, void *stream);

/*
 * Same result as mt_render_accumulate_device with the path tracer (the same
 * wavefront stage kernels and random streams), for callers that cannot
 * allocate device memory while they render: for example an application whose
 * own pool allocator owns the whole device budget, or a render loop that must
 * not pay the device-wide synchronisation of cudaMalloc / cudaFree. This
 * entry point has no counterpart in the reference.
 *
 * It allocates nothing. Its queues and path state live in one fixed 12 MiB
 * __device__ array inside the library. A GPU holds the array from the load of
 * the library's module on it until the process exits; modules load lazily by
 * default (CUDA 12.2 and later), so that is the first call of this entry point
 * on the device. A caller whose pool later takes the whole device budget makes
 * one call per device first (a warm-up), or runs with
 * CUDA_MODULE_LOADING=EAGER; if the array cannot be loaded the call returns
 * MT_ERR_OOM. Limits: width * height <= 16384 pixels per call (MT_ERR_INVALID
 * beyond), FP32 scenes only (MT_ERR_UNSUPPORTED). The caller passes the scene,
 * the camera and the device output buffer `accum_dev` (width * height * 3
 * floats). The first call on a device looks up the array's device address;
 * make it before capturing any stream. All calls share the array: calls that
 * overlap on the GPU race and must be serialised by the caller. Renders
 * through this entry point are not counted by mt_set_counting.
 */
int mt_render_accumulate_device_noalloc(mt_scene *scene, const mt_camera *cam, int width, int height,
                                        int spp_begin, int spp_end, int max_depth, float *accum_dev,
                                        int accumulate, void *stream);

/* ------------------------------------------------------------------ */
/* Autotuner                                                           */
/* ------------------------------------------------------------------ */

#define MT_TUNE_MAX_ENTRIES 32

typedef struct {
    mt_options options;   /* a timed configuration                         */
    float ms;             /* its probe window, best of two runs            */
    float pad;
} mt_tune_entry;

typedef struct {
    mt_options chosen;    /* the fastest configuration, now set on the scene */
    float chosen_ms;
    float default_ms;     /* the library defaults on the same probe         */
    int32_t n_entries;
    int32_t pad;
    mt_tune_entry entries[MT_TUNE_MAX_ENTRIES];
} mt_tune_report;

/*
 * Pick the wavefront integrator's configuration for this scene and view by
 * timing probe windows of `probe_spp` samples per pixel on the scene's device
 * (each render takes the next sample window, so that no candidate retraces
 * samples whose blockers the occluder cache already holds). Coordinate
 * descent, each stage keeping the fastest so far (library defaults first):
 *   traversal schedule (grid-stride, dynamic fetch), block size (128, 64),
 *   BVH width (2, 4, 8; wide trees built on first use), sort-by-material
 *   threshold (256K rays, off, always), queue capacity (32M, 8M, 2M), and for
 *   scenes with water or transparency > 0.8 the occluder cache (off, on).
 * Every candidate computes the same image (the tests check this), so the
 * choice only moves time. The scene must be FP32; on return its options are
 * the chosen ones with the wavefront integrator. Allocates probe buffers;
 * synchronous. No counterpart in the reference (a single CPU code path).
 */
int mt_autotune(mt_scene *scene, const mt_camera *cam, int width, int height, int probe_spp, int max_depth,
                mt_tune_report *report);

/* ------------------------------------------------------------------ */
/* Batched rendering: many images in one CUDA-graph launch             */
/* ------------------------------------------------------------------ */

/*
 * A batch context owns `lanes` sets of wavefront queues of `queue_capacity`
 * path slots each (0 = 2M). mt_batch_render spreads the items over the lanes
 * (longest first, by pixels x samples x bounces) and renders all of them with
 * ONE graph launch on `stream`: each lane renders its items in turn, the lanes
 * run concurrently. The graph is captured on the first call and reused while
 * the item list keeps its shape (scenes, sizes, windows, depths); cameras and
 * output pointers may change between calls. Scenes must be FP32 and on the
 * batch's device; their integrator option does not matter (the wavefront
 * stages are used). No counterpart in the reference, whose CLI renders one
 * image per process.
 */
typedef struct mt_batch mt_batch;

typedef struct {
    mt_scene *scene;
    const mt_camera *cam;
    int32_t width, height;
    int32_t s0;           /* first sample of the window                      */
    int32_t spp;          /* samples per pixel [s0, s0 + spp)                */
    int32_t depth;        /* max bounces                                     */
    int32_t pad;
    float *out_dev;       /* device, height x width x 3: mean linear RGB     */
} mt_batch_item;

int mt_batch_create(int32_t lanes, int32_t queue_capacity, int32_t device, mt_batch **out);
void mt_batch_release(mt_batch *batch);

/* item_ms (optional, n floats): each item's completion time after the
 * launch's first node; total_ms (optional): the whole launch. Either one
 * makes the call wait for the launch to finish. */
int mt_batch_render(mt_batch *batch, int32_t n, const mt_batch_item *items, void *stream, float *item_ms,
                    float *total_ms);

/* Per-launch statistics of the last render on this scene. */
typedef struct {
    double  kernel_ms;        /* device time of the render kernels (CUDA events) */
    int64_t primary_rays;     /* camera rays                                     */
    int64_t extension_rays;   /* nearest-hit rays incl. primary                  */
    int64_t shadow_rays;      /* NEE / any-hit rays                              */
    int64_t node_visits;      /* nearest-hit queries: inner nodes whose two child
                                 boxes were tested                               */
    int64_t prim_tests;       /* nearest-hit primitive tests (planes included)   */
    int64_t tri_tests;        /* of which triangle tests                         */
    int64_t any_node_visits;  /* the same three for any-hit (shadow) queries     */
    int64_t any_prim_tests;
    int64_t any_tri_tests;
    int32_t launches;         /* kernels launched                                */
    int32_t error_flags;      /* device error word (0 = clean)                   */
    /* Wavefront stage timing (use_graph < 0 only; reset by mt_set_counting):
     * device ms and launches of extend, shade, shadow and the other kernels. */
    double  stage_ms[4];
    int64_t stage_launches[4];
} mt_stats;
int mt_get_stats(const mt_scene *scene, mt_stats *out);
/* Enable (1) or disable (0) the ray / node counters (off by default: they
 * cost atomics). */
int mt_set_counting(mt_scene *scene, int enable);

/* ------------------------------------------------------------------ */
/* Batched queries (parity harness entry points)                        */
/* ------------------------------------------------------------------ */

/*
 * Batched pathtrace_radiance (src/pathtrace.c:800-1028): n rays (origins and
 * directions as xyz doubles), one seed key each, linear RGB out (doubles).
 */
int mt_pathtrace_radiance(mt_scene *scene, int n, const double *origins, const double *dirs,
                          int max_depth, const uint32_t *seed_keys, double *radiance_out);

/* Batched Whitted trace() at depth 0 (src/render.c:842-863), time 0: n rays
 * (xyz doubles) and seed keys in, linear RGB colour out (doubles). */
int mt_whitted_trace(mt_scene *scene, int n, const double *origins, const double *dirs,
                     int max_depth, const uint32_t *seed_keys, double *color_out);

/*
 * Batched scene_intersect (src/scene.c:767-775 -> src/bvh.c:557-712).
 * Outputs per ray: prim index (-1 = miss), t, u, v, front_face, the unit
 * normal facing the ray (xyz) and the material index. Output pointers may
 * be NULL except prim_out.
 */
int mt_intersect(mt_scene *scene, int n, const double *origins, const double *dirs,
                 double tmin, double tmax, int32_t *prim_out, double *t_out,
                 double *normal_out, int32_t *front_out, int32_t *material_out);

/* Batched any-hit test (scene_occluded, src/scene.c:777-811): 1 = blocked. */
int mt_occluded(mt_scene *scene, int n, const double *origins, const double *dirs,
                double tmin, double tmax, int32_t *occluded_out);

/*
 * Query log of the wavefront integrator (parity harness; no counterpart in the
 * reference, whose traversal calls are plain function calls a test can make
 * itself). While enabled, the FP32 wavefront stages record every traversal
 * query they answer during path-traced renders of this scene: each extension
 * ray with its nearest hit (scene_intersect over [1e-4, 1e30],
 * src/pathtrace.c:829-834) and each shadow connection with its answer
 * (pt_occluded_segment over [1e-3, tmax], src/pathtrace.c:504-532), whether
 * the occluder cache or the tree walk answered it. A test then puts the same
 * queries to the reference.
 *
 * mt_trace_log_enable keeps the first `capacity` records of later renders
 * (capacity 0 turns the log off and frees it); it resets the count.
 * mt_trace_log_read copies min(count, capacity) records of 12 floats:
 *   o.xyz, d.xyz (unit), t, result, kind, bounce, light, 0
 * kind 0 (extension): t = hit distance, result = prim index or -1;
 * kind 1 (shadow): t = tmax, result = 1 when occluded, bounce (-1: not
 * recorded), light = NEE slot (lights 0..7, 8 = the sun).
 * result, kind, bounce and light are int32 bit patterns. *count receives the
 * number of queries seen since the last enable (it may exceed capacity).
 * FP32 scenes only (MT_ERR_UNSUPPORTED otherwise).
 */
int mt_trace_log_enable(mt_scene *scene, int32_t capacity);
int mt_trace_log_read(mt_scene *scene, float *records, int32_t capacity, int64_t *count);

/* Primary rays exactly as pt_render_pixel draws them (src/pathtrace.c:1057-1082):
 * for every (x, y, s), origin + direction (doubles, 6 per ray) in
 * ((y*w + x)*spp + s) order. Computed on the device. */
int mt_primary_rays(mt_scene *scene, const mt_camera *cam, int width, int height, int spp,
                    int mode, double *rays_out);

/* ------------------------------------------------------------------ */
/* Differentiable rendering: path-replay adjoint                        */
/* ------------------------------------------------------------------ */

/*
 * Differentiable parameters, flat: for each material m, albedo rgb at 8m+0..2,
 * roughness 8m+3, metallic 8m+4, emissive rgb 8m+5..7; then the sun radiance
 * (sky sun_color) rgb at 8M+0..2; then for each material m the Beer-Lambert
 * absorption rgb at 8M+3+3m+0..2 (it acts on media and on shadow segments
 * through water / beer_lambert surfaces, src/pathtrace.c:220-233, 504-532).
 * mt_scene_param_count returns 11M + 3.
 * Setting parameters updates the device materials and sun and re-collects the
 * emissive light list (scene_collect_emissive_lights, src/scene.c:1384-1426).
 */
int mt_scene_param_count(const mt_scene *scene);
int mt_scene_get_material_params(const mt_scene *scene, double *params, int n);
int mt_scene_set_material_params(mt_scene *scene, const double *params, int n);

/*
 * Backward of the path-traced linear image I = mt_render_linear(...) with
 * respect to the parameters above, by path replay: each path is traced, then
 * replayed from its own random stream to accumulate
 *     grad[i] = sum_pixels dL_dimage[pixel] . dI[pixel] / dparam[i]
 * with detached sampling (directions, lobe and roulette probabilities held
 * fixed); geometry and visibility derivatives are out of scope. This is the
 * backward half of a torch.autograd.Function whose forward is mt_render_linear.
 * Host buffers: dL_dimage (w*h*3 floats), grad (n doubles).
 */
int mt_adjoint_backward(mt_scene *scene, const mt_camera *cam, int width, int height, int samples_per_pixel,
                        int max_depth, const float *dL_dimage, double *grad, int n);

/* Device-buffer form over the sample window [spp_begin, spp_end), asynchronous
 * on `stream`; grad_dev is overwritten (accumulate = 0) or added to. */
int mt_adjoint_backward_device(mt_scene *scene, const mt_camera *cam, int width, int height, int spp_begin,
                               int spp_end, int max_depth, const float *dL_dimage_dev, double *grad_dev,
                               int accumulate, void *stream);

/*
 * Measured L2 read bandwidth of `device` in GB/s: one launch reads a buffer of
 * `bytes` (a multiple of 16 in [1 MiB, 96 MiB], so that it stays in the 126 MB
 * L2) `reps` times with L2-only 16-byte loads from a grid of 2048 threads per
 * SM; best of three launches after a warm-up one. It is the denominator of
 * the traversal kernels' L2 fractions in the benchmark. Allocates and frees
 * its buffer; synchronous. No counterpart in the reference (a CPU renderer).
 */
int mt_measure_l2_read_gbs(int device, size_t bytes, int reps, double *gbs);

/* Library version and last error text (thread-local, never NULL). */
const char *mt_version(void);
const char *mt_last_error(void);

#ifdef __cplusplus
}
#endif

#endif /* MTGPU_H */
