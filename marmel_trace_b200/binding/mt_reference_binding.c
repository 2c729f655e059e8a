/*
 * mt_reference_binding.c - the reference-side binding of the GPU renderer.
 *
 * This file is compiled INSIDE the reference's build (it includes the
 * reference headers scene.h / camera.h / render.h / pathtrace.h) and links
 * against libmtgpu. It does two things:
 *
 *  1. Converts the reference's runtime `Scene` (src/scene.h:81-106) and
 *     `Camera` (src/camera.h) into the flat C-ABI descriptors of mtgpu.h.
 *     The conversion is a field-by-field copy: primitive order (which is the
 *     reference `prim_index` and thus the equal-t tie-break) is preserved.
 *
 *  2. Provides the link-time wrappers `__wrap_pathtrace_render` and
 *     `__wrap_render_image_ex`. Linking the unchanged reference CLI
 *     (src/main.c) with
 *         -Wl,--wrap=pathtrace_render,--wrap=render_image_ex
 *     routes src/main.c:705-710 to the GPU. `MT_BACKEND=cpu` calls the
 *     original `__real_*` functions (the reference's multithreaded CPU path);
 *     that switch exists for baseline timing and is never taken implicitly.
 *     `MT_PRECISION=fp64` selects the double-precision device path.
 *     Path tracing runs on the wavefront integrator (the fast one);
 *     `MT_INTEGRATOR=megakernel` selects the one-thread-per-pixel kernel.
 *     Both give the same images.
 *
 * Device scenes are cached by (Scene pointer, primitive count); the cache is
 * released at process exit.
 */
#include "scene.h"
#include "camera.h"
#include "render.h"
#include "pathtrace.h"

#include "mtgpu.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>

static void v3(double *dst, Vec3 v)
{
    dst[0] = v.x;
    dst[1] = v.y;
    dst[2] = v.z;
}

/* Convert one reference primitive. Returns 0, or MT_ERR_UNSUPPORTED for
 * CSG / SDF primitives (not on the GPU path). */
static int mtb_prim(const Primitive *p, mt_prim *o)
{
    memset(o, 0, sizeof *o);
    o->material = p->material_index;
    switch (p->kind) {
    case PRIM_SPHERE:
        o->kind = MT_PRIM_SPHERE;
        v3(o->v, p->center);
        o->v[3] = p->radius;
        return 0;
    case PRIM_PLANE:
        o->kind = MT_PRIM_PLANE;
        v3(o->v, p->center);
        v3(o->v + 3, p->axis);
        return 0;
    case PRIM_BOX:
        o->kind = MT_PRIM_BOX;
        v3(o->v, p->center);
        v3(o->v + 3, p->half);
        return 0;
    case PRIM_TRIANGLE:
        o->kind = MT_PRIM_TRIANGLE;
        v3(o->v, p->a);
        v3(o->v + 3, p->b);
        v3(o->v + 6, p->c);
        if (p->radius > 0.5) { /* smooth-normal gate, src/geometry.c:506 */
            o->smooth = 1;
            v3(o->n, p->center);
            v3(o->n + 3, p->axis);
            v3(o->n + 6, p->half);
        }
        if (p->has_uv) { /* vertex texture coordinates, src/geometry.c:527-531 */
            o->has_uv = 1;
            o->uv[0] = p->uva.x;
            o->uv[1] = p->uva.y;
            o->uv[2] = p->uvb.x;
            o->uv[3] = p->uvb.y;
            o->uv[4] = p->uvc.x;
            o->uv[5] = p->uvc.y;
        }
        return 0;
    case PRIM_CYLINDER:
        o->kind = MT_PRIM_CYLINDER;
        v3(o->v, p->a);
        v3(o->v + 3, p->b);
        o->v[6] = p->radius;
        o->v[7] = p->radius2;
        return 0;
    default:
        return MT_ERR_UNSUPPORTED;
    }
}

static void mtb_material(const Material *m, mt_material *o)
{
    memset(o, 0, sizeof *o);
    v3(o->albedo, m->albedo);
    v3(o->specular, m->specular);
    o->shininess = m->shininess;
    o->reflectivity = m->reflectivity;
    o->transparency = m->transparency;
    o->ior = m->ior;
    v3(o->absorption, m->absorption);
    v3(o->deep_color, m->deep_color);
    o->metallic = m->metallic;
    o->roughness = m->roughness;
    v3(o->emissive, m->emissive);
    v3(o->atmosphere_glow, m->atmosphere_glow);
    o->bump_strength = m->bump_strength;
    o->is_water = m->is_water;
    o->beer_lambert = m->beer_lambert;
    o->pbr = m->pbr;
    o->texture_kind = m->texture_kind;
    o->texture_scale = m->texture_scale;
    v3(o->texture_color_a, m->texture_color_a);
    v3(o->texture_color_b, m->texture_color_b);
    if (m->texture_image) {
        const ImageTexture *img = (const ImageTexture *)m->texture_image;
        o->texture_rgb = img->rgb;
        o->texture_width = img->width;
        o->texture_height = img->height;
    }
}

static void mtb_sky(const SkyParams *s, mt_sky *o)
{
    memset(o, 0, sizeof *o);
    v3(o->sun_dir, s->sun_dir);
    v3(o->sun_color, s->sun_color);
    v3(o->horizon_color, s->horizon_color);
    v3(o->zenith_color, s->zenith_color);
    o->gradient_gamma = s->gradient_gamma;
    o->sun_glow_exponent = s->sun_glow_exponent;
    o->sun_glow_strength = s->sun_glow_strength;
    o->cloud_height = s->cloud_height;
    o->cloud_scale = s->cloud_scale;
    o->cloud_coverage = s->cloud_coverage;
    o->cloud_softness = s->cloud_softness;
    o->cloud_sharpness = s->cloud_sharpness;
    o->cloud_thickness = s->cloud_thickness;
    o->sun_radius = s->sun_radius;
    o->star_intensity = s->star_intensity;
    o->nebula_intensity = s->nebula_intensity;
    o->galaxy_intensity = s->galaxy_intensity;
    o->cloud_octaves = s->cloud_octaves;
    o->seed = s->seed;
    o->cloud_density = s->cloud_density;
    o->cloud_steps = s->cloud_steps;
}

/*
 * Fill `d` from `s`. `prims` / `mats` must hold s->geo.count and
 * s->material_count entries. Returns 0 or MT_ERR_UNSUPPORTED.
 */
int mtb_scene_to_desc(const Scene *s, mt_prim *prims, mt_material *mats, mt_scene_desc *d)
{
    int i;
    memset(d, 0, sizeof *d);
    for (i = 0; i < s->geo.count; ++i) {
        if (mtb_prim(&s->geo.prims[i], &prims[i]) != 0) return MT_ERR_UNSUPPORTED;
    }
    for (i = 0; i < s->material_count; ++i) mtb_material(&s->materials[i], &mats[i]);
    d->prims = prims;
    d->prim_count = s->geo.count;
    d->materials = mats;
    d->material_count = s->material_count;
    mtb_sky(&s->sky, &d->sky);
    d->fog_density = s->fog.density;
    d->fog_shadow_steps = s->fog.shadow_steps;
    v3(d->fog_color, s->fog.color);
    d->fog_height = s->fog.height;
    d->fog_height_falloff = s->fog.height_falloff;
    d->fog_inscatter_strength = s->fog.inscatter_strength;
    d->fog_sun_anisotropy = s->fog.sun_anisotropy;
    d->fog_noise_scale = s->fog.noise_scale;
    d->fog_noise_amount = s->fog.noise_amount;
    d->water_level = s->water_level;
    d->water_material = s->water_material;
    d->ocean.enabled = s->has_ocean;
    if (s->has_ocean) {
        d->ocean.seed = s->ocean_params.seed;
        v3(d->ocean.center, s->ocean_params.center);
        d->ocean.amplitude = s->ocean_params.amplitude;
        d->ocean.wavelength = s->ocean_params.wavelength;
        v3(d->ocean.direction, s->ocean_params.direction);
        d->ocean.chop = s->ocean_params.chop;
        d->ocean.chop_wavelength = s->ocean_params.chop_wavelength;
    }
    return 0;
}

void mtb_camera_to_desc(const Camera *c, mt_camera *o)
{
    memset(o, 0, sizeof *o);
    v3(o->position, c->position);
    v3(o->lower_left, c->lower_left);
    v3(o->horizontal, c->horizontal);
    v3(o->vertical, c->vertical);
    o->aperture = c->aperture;
    o->focus_distance = c->focus_distance;
    o->dome_radius = c->dome_radius;
    o->anamorphic_squeeze = c->anamorphic_squeeze;
}

#ifndef MTB_CONVERT_ONLY
/* Build a device scene for `s` with the given options (NULL = defaults). */
int mtb_scene_upload(const Scene *s, const mt_options *opts, mt_scene **out)
{
    mt_scene_desc d;
    mt_prim *prims;
    mt_material *mats;
    int rc;

    prims = (mt_prim *)calloc((size_t)(s->geo.count > 0 ? s->geo.count : 1), sizeof *prims);
    mats = (mt_material *)calloc((size_t)(s->material_count > 0 ? s->material_count : 1), sizeof *mats);
    if (!prims || !mats) {
        free(prims);
        free(mats);
        return MT_ERR_OOM;
    }
    rc = mtb_scene_to_desc(s, prims, mats, &d);
    if (rc == 0) rc = mt_scene_create(&d, opts, out);
    free(prims);
    free(mats);
    return rc;
}

/* ------------------------------------------------------------------ */
/* Link-time wrappers for the reference CLI                             */
/* ------------------------------------------------------------------ */

int __real_pathtrace_render(const Scene *scene, const Camera *cam, int width, int height,
                            int samples_per_pixel, int max_depth, unsigned char *rgb_out);
int __real_render_image_ex(const Scene *scene, const Camera *cam, int width, int height,
                           const RenderParams *params, unsigned char *rgb_out);

static const Scene *g_cached_scene = NULL;
static int g_cached_count = -1;
static mt_scene *g_cached_dev = NULL;

static void mtb_release_cache(void)
{
    if (g_cached_dev) mt_scene_release(g_cached_dev);
    g_cached_dev = NULL;
    g_cached_scene = NULL;
    g_cached_count = -1;
}

static int mtb_want_cpu(void)
{
    const char *b = getenv("MT_BACKEND");
    return b != NULL && strcmp(b, "cpu") == 0;
}

static int mtb_get_scene(const Scene *s, mt_scene **out)
{
    static int registered = 0;
    mt_options o;
    const char *prec, *integ;
    int rc;

    if (g_cached_dev && g_cached_scene == s && g_cached_count == s->geo.count) {
        *out = g_cached_dev;
        return 0;
    }
    mtb_release_cache();
    mt_options_default(&o);
    prec = getenv("MT_PRECISION");
    if (prec != NULL && strcmp(prec, "fp64") == 0) o.precision = MT_PRECISION_FP64;
    integ = getenv("MT_INTEGRATOR");
    o.integrator = (integ != NULL && strcmp(integ, "megakernel") == 0) ? MT_INTEGRATOR_MEGAKERNEL
                                                                      : MT_INTEGRATOR_WAVEFRONT;
    rc = mtb_scene_upload(s, &o, &g_cached_dev);
    if (rc != 0) {
        fprintf(stderr, "mtgpu: scene upload failed (code %d): %s\n", rc, mt_last_error());
        g_cached_dev = NULL;
        return rc;
    }
    g_cached_scene = s;
    g_cached_count = s->geo.count;
    if (!registered) {
        atexit(mtb_release_cache);
        registered = 1;
    }
    *out = g_cached_dev;
    return 0;
}

static double mtb_now(void)
{
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + (double)ts.tv_nsec * 1e-9;
}

int __wrap_pathtrace_render(const Scene *scene, const Camera *cam, int width, int height,
                            int samples_per_pixel, int max_depth, unsigned char *rgb_out)
{
    mt_scene *dev;
    mt_camera c;
    double t0;
    int rc;

    if (mtb_want_cpu()) {
        return __real_pathtrace_render(scene, cam, width, height, samples_per_pixel,
                                       max_depth, rgb_out);
    }
    /* Argument codes first, exactly as src/pathtrace.c:1260-1268. */
    if (scene == NULL || cam == NULL || rgb_out == NULL) return 1;
    if (width <= 0 || height <= 0) return 2;
    if (samples_per_pixel < 1 || max_depth < 0) return 3;

    t0 = mtb_now();
    rc = mtb_get_scene(scene, &dev);
    if (rc != 0) return rc;
    mtb_camera_to_desc(cam, &c);
    rc = mt_pathtrace_render(dev, &c, width, height, samples_per_pixel, max_depth, rgb_out);
    render_set_last_seconds(mtb_now() - t0);
    if (rc != 0) fprintf(stderr, "mtgpu: %s\n", mt_last_error());
    return rc;
}

int __wrap_render_image_ex(const Scene *scene, const Camera *cam, int width, int height,
                           const RenderParams *params, unsigned char *rgb_out)
{
    mt_scene *dev;
    mt_camera c;
    mt_render_params p;
    double t0;
    int rc;

    if (mtb_want_cpu()) {
        return __real_render_image_ex(scene, cam, width, height, params, rgb_out);
    }
    /* Argument codes first, exactly as src/render.c:1630-1641. */
    if (params == NULL) return 1;
    if (scene == NULL || cam == NULL || rgb_out == NULL) return 1;
    if (width <= 0 || height <= 0) return 2;
    if (params->samples_per_pixel < 1 || params->max_depth < 0) return 3;

    t0 = mtb_now();
    rc = mtb_get_scene(scene, &dev);
    if (rc != 0) return rc;
    mtb_camera_to_desc(cam, &c);
    p.samples_per_pixel = params->samples_per_pixel;
    p.max_depth = params->max_depth;
    p.adaptive = params->adaptive;
    p.adaptive_max_spp = params->adaptive_max_spp;
    p.adaptive_tau = params->adaptive_tau;
    rc = mt_render_image_ex(dev, &c, width, height, &p, rgb_out);
    render_set_last_seconds(mtb_now() - t0);
    if (rc != 0) fprintf(stderr, "mtgpu: %s\n", mt_last_error());
    return rc;
}
#endif /* MTB_CONVERT_ONLY */
