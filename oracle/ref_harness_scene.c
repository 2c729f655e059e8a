/*
 * ref_harness_scene.c - oracle harness: scene loading, export and queries.
 *
 * TEST INFRASTRUCTURE ONLY (see ref_harness.h). Includes the reference's
 * src/scene.c so that the file-static scene_collect_emissive_lights
 * (src/scene.c:1384-1426) can be run on scenes assembled directly from a
 * flat descriptor.
 */
#include "scene.c"

#include "ref_harness.h"
#include "mtgpu.h"
#include "scene_desc.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int mtb_scene_to_desc(const Scene *s, mt_prim *prims, mt_material *mats, mt_scene_desc *d);
void mtb_camera_to_desc(const Camera *c, mt_camera *o);

/* Camera exactly as src/main.c:637-668 builds it for a w x h image. */
static void mtref_camera_from_desc(MtRefHandle *h, const SceneDesc *desc, int width, int height)
{
    Vec3 eye, target, up;
    double vfov;
    if (desc->camera.present) {
        eye = desc->camera.eye;
        target = desc->camera.target;
        up = desc->camera.up;
        vfov = desc->camera.vfov_deg;
    } else {
        scene_default_view(&eye, &target, &up, &vfov);
    }
    h->cam = camera_create(eye, target, up, vfov, (double)width / (double)height);
    h->cam.aperture = desc->camera.aperture;
    if (desc->camera.focus_distance > CAMERA_FOCUS_DISTANCE_DERIVED)
        h->cam.focus_distance = desc->camera.focus_distance;
    if (desc->camera.dome_radius > 0.0)
        h->cam.dome_radius = desc->camera.dome_radius;
    if (desc->camera.anamorphic_squeeze > 0.0)
        h->cam.anamorphic_squeeze = desc->camera.anamorphic_squeeze;
    h->cam.flare = desc->camera.flare;
}

static MtRefHandle *mtref_build(SceneDesc *desc, int width, int height)
{
    MtRefHandle *h = (MtRefHandle *)calloc(1, sizeof *h);
    if (!h) return NULL;
    if (scene_build_from_desc(&h->scene, desc) != 0) {
        free(h);
        return NULL;
    }
    mtref_camera_from_desc(h, desc, width, height);
    return h;
}

/* Parse scene text (NULL = the embedded default scene) and build it, as
 * src/main.c:589-668 does. Returns NULL on error (message in err). */
void *mtref_load_text(const char *text, int width, int height, char *err, int errlen)
{
    SceneDesc desc;
    char buf[512];
    MtRefHandle *h;
    scene_desc_init(&desc);
    if (text == NULL) {
        scene_default_desc(&desc);
    } else if (scene_desc_load_string(&desc, text, "<harness>", buf, sizeof buf) != 0) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", buf);
        scene_desc_free(&desc);
        return NULL;
    }
    h = mtref_build(&desc, width, height);
    scene_desc_free(&desc);
    if (!h && err && errlen > 0) snprintf(err, (size_t)errlen, "scene build failed");
    return h;
}

void *mtref_load_file(const char *path, int width, int height, char *err, int errlen)
{
    SceneDesc desc;
    char buf[512];
    MtRefHandle *h;
    scene_desc_init(&desc);
    if (scene_desc_load(&desc, path, buf, sizeof buf) != 0) {
        if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", buf);
        scene_desc_free(&desc);
        return NULL;
    }
    h = mtref_build(&desc, width, height);
    scene_desc_free(&desc);
    return h;
}

static Vec3 dv3(const double *p) { return vec3(p[0], p[1], p[2]); }

/*
 * Assemble a reference Scene directly from a flat descriptor (the inverse of
 * the binding): primitives through the reference constructors, then the
 * emissive-light collector and bvh_build, as scene_build_from_desc ends
 * (src/scene.c:1619-1627). Used for synthetic scenes too large for text.
 */
void *mtref_from_desc(const mt_scene_desc *d, const mt_camera *cam)
{
    MtRefHandle *h = (MtRefHandle *)calloc(1, sizeof *h);
    Scene *s;
    int i;
    if (!h) return NULL;
    s = &h->scene;
    geometry_init(&s->geo);
    s->water_level = d->water_level;
    s->water_material = d->water_material;
    sky_default_params(&s->sky);
    s->sky.sun_dir = dv3(d->sky.sun_dir);
    s->sky.sun_color = dv3(d->sky.sun_color);
    s->sky.horizon_color = dv3(d->sky.horizon_color);
    s->sky.zenith_color = dv3(d->sky.zenith_color);
    s->sky.gradient_gamma = d->sky.gradient_gamma;
    s->sky.sun_glow_exponent = d->sky.sun_glow_exponent;
    s->sky.sun_glow_strength = d->sky.sun_glow_strength;
    s->sky.cloud_height = d->sky.cloud_height;
    s->sky.cloud_scale = d->sky.cloud_scale;
    s->sky.cloud_coverage = d->sky.cloud_coverage;
    s->sky.cloud_softness = d->sky.cloud_softness;
    s->sky.cloud_sharpness = d->sky.cloud_sharpness;
    s->sky.cloud_octaves = d->sky.cloud_octaves;
    s->sky.cloud_thickness = d->sky.cloud_thickness;
    s->sky.seed = d->sky.seed;
    s->sky.sun_radius = d->sky.sun_radius;
    s->sky.star_intensity = d->sky.star_intensity;
    s->sky.nebula_intensity = d->sky.nebula_intensity;
    s->sky.galaxy_intensity = d->sky.galaxy_intensity;
    s->sky.cloud_density = d->sky.cloud_density;
    s->sky.cloud_steps = d->sky.cloud_steps;
    fog_default_params(&s->fog);
    s->fog.density = d->fog_density;
    s->fog.shadow_steps = d->fog_shadow_steps;
    s->fog.color = dv3(d->fog_color);
    s->fog.height = d->fog_height;
    s->fog.height_falloff = d->fog_height_falloff;
    s->fog.inscatter_strength = d->fog_inscatter_strength;
    s->fog.sun_anisotropy = d->fog_sun_anisotropy;
    s->fog.noise_scale = d->fog_noise_scale;
    s->fog.noise_amount = d->fog_noise_amount;
    s->has_ocean = d->ocean.enabled;
    if (d->ocean.enabled) {
        s->ocean_params.enabled = 1;
        s->ocean_params.center = dv3(d->ocean.center);
        s->ocean_params.amplitude = d->ocean.amplitude;
        s->ocean_params.wavelength = d->ocean.wavelength;
        s->ocean_params.direction = dv3(d->ocean.direction);
        s->ocean_params.chop = d->ocean.chop;
        s->ocean_params.chop_wavelength = d->ocean.chop_wavelength;
        s->ocean_params.seed = d->ocean.seed;
    }
    if (d->material_count > 0) {
        s->materials = (Material *)calloc((size_t)d->material_count, sizeof(Material));
        if (!s->materials) goto fail;
        s->material_count = d->material_count;
        for (i = 0; i < d->material_count; ++i) {
            const mt_material *m = &d->materials[i];
            Material *o = &s->materials[i];
            material_texture_defaults(o);
            o->albedo = dv3(m->albedo);
            o->specular = dv3(m->specular);
            o->shininess = m->shininess;
            o->reflectivity = m->reflectivity;
            o->transparency = m->transparency;
            o->ior = m->ior;
            o->is_water = m->is_water;
            o->absorption = dv3(m->absorption);
            o->deep_color = dv3(m->deep_color);
            o->beer_lambert = m->beer_lambert;
            o->metallic = m->metallic;
            o->roughness = m->roughness;
            o->emissive = dv3(m->emissive);
            o->pbr = m->pbr;
            o->texture_kind = m->texture_kind;
            o->texture_scale = m->texture_scale;
            o->texture_color_a = dv3(m->texture_color_a);
            o->texture_color_b = dv3(m->texture_color_b);
            if (m->texture_rgb && m->texture_width > 0 && m->texture_height > 0) {
                /* an image texture, owned by the Scene's texture table */
                ImageTexture *img = texture_image_create(m->texture_width, m->texture_height);
                if (!img) goto fail;
                memcpy(img->rgb, m->texture_rgb, (size_t)m->texture_width * (size_t)m->texture_height * 3u);
                if (s->texture_count == s->texture_capacity) {
                    int cap = s->texture_capacity ? 2 * s->texture_capacity : 4;
                    SceneTexture *t = (SceneTexture *)realloc(s->textures, (size_t)cap * sizeof *t);
                    if (!t) {
                        texture_image_free(img);
                        goto fail;
                    }
                    s->textures = t;
                    s->texture_capacity = cap;
                }
                s->textures[s->texture_count].path = NULL;
                s->textures[s->texture_count].image = img;
                s->texture_count++;
                o->texture_image = img;
            }
            o->bump_strength = m->bump_strength;
            o->bump_scale = 1.0;
            o->atmosphere_glow = dv3(m->atmosphere_glow);
        }
    }
    for (i = 0; i < d->prim_count; ++i) {
        const mt_prim *p = &d->prims[i];
        Primitive q;
        switch (p->kind) {
        case MT_PRIM_SPHERE:
            q = prim_sphere(dv3(p->v), p->v[3], p->material);
            break;
        case MT_PRIM_PLANE:
            q = prim_plane(dv3(p->v), dv3(p->v + 3), p->material);
            q.axis = dv3(p->v + 3); /* keep the caller's unit normal bit-for-bit */
            break;
        case MT_PRIM_BOX:
            q = prim_box(dv3(p->v), dv3(p->v + 3), p->material);
            break;
        case MT_PRIM_TRIANGLE:
            if (p->smooth && p->has_uv)
                q = prim_triangle_smooth_uv(dv3(p->v), dv3(p->v + 3), dv3(p->v + 6), dv3(p->n), dv3(p->n + 3),
                                            dv3(p->n + 6), vec3(p->uv[0], p->uv[1], 0.0),
                                            vec3(p->uv[2], p->uv[3], 0.0), vec3(p->uv[4], p->uv[5], 0.0),
                                            p->material);
            else if (p->smooth)
                q = prim_triangle_smooth(dv3(p->v), dv3(p->v + 3), dv3(p->v + 6),
                                         dv3(p->n), dv3(p->n + 3), dv3(p->n + 6), p->material);
            else if (p->has_uv)
                q = prim_triangle_uv(dv3(p->v), dv3(p->v + 3), dv3(p->v + 6), vec3(p->uv[0], p->uv[1], 0.0),
                                     vec3(p->uv[2], p->uv[3], 0.0), vec3(p->uv[4], p->uv[5], 0.0), p->material);
            else
                q = prim_triangle(dv3(p->v), dv3(p->v + 3), dv3(p->v + 6), p->material);
            break;
        case MT_PRIM_CYLINDER:
            q = prim_cylinder(dv3(p->v), dv3(p->v + 3), p->v[6], p->v[7], p->material);
            break;
        default:
            goto fail;
        }
        if (geometry_add(&s->geo, q) < 0) goto fail;
    }
    scene_collect_emissive_lights(s);
    s->bvh = bvh_build(&s->geo);
    if (!s->bvh && s->geo.count > 0) goto fail;
    if (cam) {
        h->cam.position = dv3(cam->position);
        h->cam.lower_left = dv3(cam->lower_left);
        h->cam.horizontal = dv3(cam->horizontal);
        h->cam.vertical = dv3(cam->vertical);
        h->cam.aperture = cam->aperture;
        h->cam.focus_distance = cam->focus_distance;
        h->cam.dome_radius = cam->dome_radius;
        h->cam.anamorphic_squeeze = cam->anamorphic_squeeze;
    }
    return h;
fail:
    scene_free(s);
    free(h);
    return NULL;
}

void mtref_free(void *hp)
{
    MtRefHandle *h = (MtRefHandle *)hp;
    if (!h) return;
    scene_free(&h->scene);
    free(h);
}

int mtref_prim_count(void *hp) { return ((MtRefHandle *)hp)->scene.geo.count; }
int mtref_material_count(void *hp) { return ((MtRefHandle *)hp)->scene.material_count; }

/* Emissive light list (prim indices, file order); returns the count. */
int mtref_lights(void *hp, int *prim_out)
{
    Scene *s = &((MtRefHandle *)hp)->scene;
    for (int i = 0; i < s->emissive_light_count; ++i)
        if (prim_out) prim_out[i] = s->emissive_lights[i].prim_index;
    return s->emissive_light_count;
}

/* Export through the reference-side binding (flat descriptor + camera). */
int mtref_export(void *hp, mt_prim *prims, mt_material *mats, mt_scene_desc *d, mt_camera *cam)
{
    MtRefHandle *h = (MtRefHandle *)hp;
    int rc = mtb_scene_to_desc(&h->scene, prims, mats, d);
    if (cam) mtb_camera_to_desc(&h->cam, cam);
    return rc;
}

/* Replace the handle's camera (e.g. one built by mt_camera_create). */
void mtref_set_camera(void *hp, const mt_camera *cam)
{
    MtRefHandle *h = (MtRefHandle *)hp;
    h->cam.position = dv3(cam->position);
    h->cam.lower_left = dv3(cam->lower_left);
    h->cam.horizontal = dv3(cam->horizontal);
    h->cam.vertical = dv3(cam->vertical);
    h->cam.aperture = cam->aperture;
    h->cam.focus_distance = cam->focus_distance;
    h->cam.dome_radius = cam->dome_radius;
    h->cam.anamorphic_squeeze = cam->anamorphic_squeeze;
}

/* camera_create (src/camera.c:24-66) for the camera KAT. */
void mtref_camera_create(const double *from, const double *at, const double *up,
                         double vfov, double aspect, mt_camera *out)
{
    Camera c = camera_create(dv3(from), dv3(at), dv3(up), vfov, aspect);
    mtb_camera_to_desc(&c, out);
}

/* Batched scene_intersect (src/scene.c:767-775). */
int mtref_intersect(void *hp, int n, const double *o, const double *dir, double tmin,
                    double tmax, int *prim_out, double *t_out, double *normal_out,
                    int *front_out, int *mat_out)
{
    Scene *s = &((MtRefHandle *)hp)->scene;
    for (int i = 0; i < n; ++i) {
        Ray r;
        Hit h;
        r.origin = dv3(o + 3 * i);
        r.dir = dv3(dir + 3 * i);
        if (scene_intersect(s, r, tmin, tmax, &h)) {
            prim_out[i] = h.prim_index;
            if (t_out) t_out[i] = h.t;
            if (normal_out) {
                normal_out[3 * i] = h.normal.x;
                normal_out[3 * i + 1] = h.normal.y;
                normal_out[3 * i + 2] = h.normal.z;
            }
            if (front_out) front_out[i] = h.front_face;
            if (mat_out) mat_out[i] = h.material_index;
        } else {
            prim_out[i] = -1;
            if (t_out) t_out[i] = 0.0;
            if (front_out) front_out[i] = 0;
            if (mat_out) mat_out[i] = -1;
        }
    }
    return 0;
}

/* Batched linear-scan geometry_intersect (src/geometry.c:1488-1512): the
 * BVH-free ground truth of tests/test_math.c:769-831. */
int mtref_intersect_linear(void *hp, int n, const double *o, const double *dir, double tmin,
                           double tmax, int *prim_out, double *t_out)
{
    Scene *s = &((MtRefHandle *)hp)->scene;
    for (int i = 0; i < n; ++i) {
        Ray r;
        Hit h;
        r.origin = dv3(o + 3 * i);
        r.dir = dv3(dir + 3 * i);
        if (geometry_intersect(&s->geo, r, tmin, tmax, &h)) {
            prim_out[i] = h.prim_index;
            t_out[i] = h.t;
        } else {
            prim_out[i] = -1;
            t_out[i] = 0.0;
        }
    }
    return 0;
}

/* Batched scene_occluded (src/scene.c:804-811). */
int mtref_occluded(void *hp, int n, const double *o, const double *dir, double tmin,
                   double tmax, int *occ_out)
{
    Scene *s = &((MtRefHandle *)hp)->scene;
    for (int i = 0; i < n; ++i) {
        Ray r;
        r.origin = dv3(o + 3 * i);
        r.dir = dv3(dir + 3 * i);
        occ_out[i] = scene_occluded(s, r, tmin, tmax);
    }
    return 0;
}

double mtref_water_height(void *hp, double x, double z)
{
    return scene_water_height(&((MtRefHandle *)hp)->scene, x, z);
}
