// mt_api.cu - implementation of the C ABI declared in include/mtgpu.h.
//
// Host side: validates the scene descriptor, builds the BVH with the
// restated reference builder (mt_bvh.cpp), flattens it, uploads the scene in
// the arithmetic type the options select and dispatches the kernels. Every
// CUDA call is checked and mapped to an MT_ERR_* code; there is no CPU
// fallback anywhere on this path.
#include <cuda_runtime.h>
#include <math.h>
#include <stdarg.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>
#include <cmath>
#include <limits>
#include <string>
#include <vector>

#include "../../include/mtgpu.h"
#include "mt_bvh.h"
#include "mt_launch.h"
#include "mt_layout.h"
#include "mt_wavefront.h"

using namespace mt;

// Adjoint parameter layout (mt_adjoint.cuh): 8 per material, then the sun,
// then 3 absorption coefficients per material.
static constexpr int kParamsPerMaterialApi = 8;
static constexpr int kAdjMaxMaterialsApi = 256;
static inline int param_count(int M) { return kParamsPerMaterialApi * M + 3 + 3 * M; }

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    int code = (e == cudaErrorMemoryAllocation) ? MT_ERR_OOM
               : (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) ? MT_ERR_NO_DEVICE
                                                                               : MT_ERR_LAUNCH;
    return fail(code, "%s: %s", what, cudaGetErrorString(e));
}

#define CK(call, what)                          \
    do {                                        \
        cudaError_t e_ = (call);                \
        if (e_ != cudaSuccess) return cuda_fail(e_, what); \
    } while (0)

// vec3_normalize in host double arithmetic (src/vec3.c:29-37)
void normalize3(const double *a, double *o)
{
    double len_sq = a[0] * a[0] + a[1] * a[1] + a[2] * a[2];
    if (len_sq <= 1e-12) {
        o[0] = o[1] = o[2] = 0.0;
        return;
    }
    double inv = 1.0 / sqrt(len_sq);
    o[0] = a[0] * inv;
    o[1] = a[1] * inv;
    o[2] = a[2] * inv;
}

struct HostSphere {
    int prim;
    int material;
    double center[3];
    double radius;
};

}  // namespace

struct mt_scene {
    mt_options opts;
    HostBvh bvh;
    FlatBvh flat;
    int prim_count = 0;
    int light_count = 0;
    int light_prims[kMaxLights] = {0};
    std::vector<void *> allocs;
    int64_t device_bytes = 0;
    DevScene<float> sf;
    DevScene<double> sd;
    unsigned *d_err = nullptr;
    DevCounters *d_counters = nullptr;
    bool counting = false;
    // wavefront query log (mt_trace_log_enable): records and their count
    float4 *d_trace = nullptr;
    unsigned *d_trace_n = nullptr;
    int trace_cap = 0;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    mt_stats stats;
    WavefrontState *wf = nullptr;
    // host copies used by parameter updates (mt_scene_set_material_params)
    std::vector<mt_material> h_mats;
    std::vector<const unsigned char *> d_tex;  // per material: device copy of its image texture (or NULL)
    mt_sky h_sky;
    std::vector<HostSphere> h_spheres;
    int version = 0;
    // FP32 binary tree on the host (device layout), and the wide trees
    // collapsed from it on first use (index 0: 4 children, 1: 8 children)
    std::vector<float> nodes2;
    const float4 *wide[2] = {nullptr, nullptr};
    int wide_depth[2] = {0, 0};

    template <typename T> int upload(const std::vector<T> &v, const T **dst)
    {
        *dst = nullptr;
        if (v.empty()) return 0;
        void *p = nullptr;
        size_t bytes = v.size() * sizeof(T);
        CK(cudaMalloc(&p, bytes), "cudaMalloc(scene)");
        allocs.push_back(p);
        device_bytes += (int64_t)bytes;
        CK(cudaMemcpy(p, v.data(), bytes, cudaMemcpyHostToDevice), "cudaMemcpy(scene)");
        *dst = (const T *)p;
        return 0;
    }
};

// Outward growth of the FP32 node boxes, in units of 2^-24 times the
// largest coordinate magnitude of the scene (see upload_scene).
#ifndef MT_BOX_PAD
#define MT_BOX_PAD 16
#endif

namespace {

int validate(const mt_scene_desc *d)
{
    if (d->prim_count < 0 || d->material_count < 0) return fail(MT_ERR_INVALID, "negative counts");
    if (d->prim_count > 0 && !d->prims) return fail(MT_ERR_NULL, "prims is NULL");
    if (d->material_count > 0 && !d->materials) return fail(MT_ERR_NULL, "materials is NULL");
    if (d->prim_count >= (1 << 28)) return fail(MT_ERR_UNSUPPORTED, "more than 2^28 primitives");
    const mt_sky &s = d->sky;
    if (s.star_intensity > 0.0 || s.nebula_intensity > 0.0 || s.galaxy_intensity > 0.0)
        return fail(MT_ERR_UNSUPPORTED, "starfield / nebula / galaxy sky terms are not on the GPU path");
    for (int i = 0; i < d->material_count; ++i) {
        const mt_material &m = d->materials[i];
        if (m.texture_kind < MT_TEXTURE_NONE || m.texture_kind > MT_TEXTURE_UV_CHECKER)
            return fail(MT_ERR_INVALID, "material %d: texture kind %d", i, m.texture_kind);
        if (m.texture_rgb && (m.texture_width <= 0 || m.texture_height <= 0))
            return fail(MT_ERR_INVALID, "material %d: image texture of %d x %d", i, m.texture_width, m.texture_height);
        if (m.bump_strength > 1e-6) return fail(MT_ERR_UNSUPPORTED, "material %d: bump maps are not on the GPU path", i);
    }
    for (int i = 0; i < d->prim_count; ++i) {
        int k = d->prims[i].kind;
        if (k < MT_PRIM_SPHERE || k > MT_PRIM_CYLINDER)
            return fail(MT_ERR_UNSUPPORTED, "prim %d: kind %d (CSG / SDF) is not on the GPU path", i, k);
    }
    return 0;
}

// `tex`: the device copy of the material's image texture (or NULL).
template <typename R> void fill_material(const mt_material &m, const unsigned char *tex, DevMaterial<R> *o)
{
    memset(o, 0, sizeof *o);
    o->texture_kind = m.texture_kind;
    o->texture_scale = (R)m.texture_scale;
    for (int k = 0; k < 3; ++k) {
        o->texture_color_a[k] = (R)m.texture_color_a[k];
        o->texture_color_b[k] = (R)m.texture_color_b[k];
    }
    o->texture_rgb = tex;
    o->texture_width = tex ? m.texture_width : 0;
    o->texture_height = tex ? m.texture_height : 0;
    for (int k = 0; k < 3; ++k) {
        o->albedo[k] = (R)m.albedo[k];
        o->specular[k] = (R)m.specular[k];
        o->absorption[k] = (R)m.absorption[k];
        o->deep_color[k] = (R)m.deep_color[k];
        o->emissive[k] = (R)m.emissive[k];
        o->atmosphere_glow[k] = (R)m.atmosphere_glow[k];
    }
    o->shininess = (R)m.shininess;
    o->reflectivity = (R)m.reflectivity;
    o->transparency = (R)m.transparency;
    o->ior = (R)m.ior;
    o->metallic = (R)m.metallic;
    o->roughness = (R)m.roughness;
    o->is_water = m.is_water;
    o->beer_lambert = m.beer_lambert;
    o->pbr = m.pbr;
}

template <typename R> void fill_sky(const mt_sky &s, DevSky<R> *o)
{
    for (int k = 0; k < 3; ++k) {
        o->sun_dir[k] = (R)s.sun_dir[k];
        o->sun_color[k] = (R)s.sun_color[k];
        o->horizon_color[k] = (R)s.horizon_color[k];
        o->zenith_color[k] = (R)s.zenith_color[k];
    }
    o->gradient_gamma = (R)s.gradient_gamma;
    o->sun_glow_exponent = (R)s.sun_glow_exponent;
    o->sun_glow_strength = (R)s.sun_glow_strength;
    o->cloud_height = (R)s.cloud_height;
    o->cloud_scale = (R)s.cloud_scale;
    o->cloud_coverage = (R)s.cloud_coverage;
    o->cloud_softness = (R)s.cloud_softness;
    o->cloud_sharpness = (R)s.cloud_sharpness;
    o->sun_radius = (R)s.sun_radius;
    o->cloud_thickness = (R)s.cloud_thickness;
    o->cloud_density = (R)s.cloud_density;
    o->cloud_steps = s.cloud_steps;
    o->cloud_octaves = s.cloud_octaves;
    o->seed = s.seed;
}

template <typename R> void fill_fog(const mt_scene_desc &d, DevFog<R> *o)
{
    memset(o, 0, sizeof *o);
    o->density = (R)d.fog_density;
    for (int k = 0; k < 3; ++k) o->color[k] = (R)d.fog_color[k];
    o->height = (R)d.fog_height;
    o->height_falloff = (R)d.fog_height_falloff;
    o->inscatter_strength = (R)d.fog_inscatter_strength;
    o->sun_anisotropy = (R)d.fog_sun_anisotropy;
    o->noise_scale = (R)d.fog_noise_scale;
    o->noise_amount = (R)d.fog_noise_amount;
    o->shadow_steps = d.fog_shadow_steps;
}

// scene_collect_emissive_lights (src/scene.c:1384-1426): the first 8 emissive
// PBR spheres with radius > 0, in file order, from the host copies.
template <typename R> void collect_lights(mt_scene *sc, DevScene<R> *S)
{
    S->light_count = 0;
    for (const HostSphere &p : sc->h_spheres) {
        if (S->light_count >= kMaxLights) break;
        if (p.material < 0 || p.material >= (int)sc->h_mats.size()) continue;
        const mt_material &m = sc->h_mats[p.material];
        if (!m.pbr) continue;
        if (m.emissive[0] == 0.0 && m.emissive[1] == 0.0 && m.emissive[2] == 0.0) continue;
        if (!(p.radius > 0.0)) continue;
        DevLight<R> &L = S->lights[S->light_count];
        for (int k = 0; k < 3; ++k) {
            L.center[k] = (R)p.center[k];
            L.emissive[k] = (R)m.emissive[k];
        }
        L.radius = (R)p.radius;
        L.prim = p.prim;
        sc->light_prims[S->light_count] = p.prim;
        S->light_count++;
    }
    sc->light_count = S->light_count;
}

// Upload every array of the scene in arithmetic type R.
template <typename R> int upload_scene(mt_scene *sc, const mt_scene_desc *d, DevScene<R> *S)
{
    const int n = d->prim_count;
    const FlatBvh &fb = sc->flat;
    memset(S, 0, sizeof *S);

    // Slots per kind in leaf order (tree prims), planes in file order.
    std::vector<int2> prim_info(n > 0 ? n : 1, make_int2(0, -1));
    std::vector<int2> refs(fb.ref_prim.size());
    std::vector<float4> tri4;
    std::vector<R> tris, tri_normals, tri_uv, spheres, boxes, cyls, planes;
    std::vector<int> tri_smooth, plane_prims;
    bool any_smooth = false, any_uv = false;
    for (int i = 0; i < n; ++i) {
        if (d->prims[i].kind == MT_PRIM_TRIANGLE && d->prims[i].smooth) any_smooth = true;
        if (d->prims[i].kind == MT_PRIM_TRIANGLE && d->prims[i].has_uv) any_uv = true;
    }

    int ntri = 0, nsph = 0, nbox = 0, ncyl = 0;
    for (size_t k = 0; k < fb.ref_prim.size(); ++k) {
        int pi = fb.ref_prim[k];
        const mt_prim &p = d->prims[pi];
        int code = 0;
        switch (p.kind) {
        case MT_PRIM_SPHERE:
            code = (KIND_SPHERE << 28) | nsph++;
            for (int j = 0; j < 4; ++j) spheres.push_back((R)p.v[j]);
            break;
        case MT_PRIM_BOX:
            code = (KIND_BOX << 28) | nbox++;
            for (int j = 0; j < 6; ++j) boxes.push_back((R)p.v[j]);
            break;
        case MT_PRIM_CYLINDER:
            code = (KIND_CYLINDER << 28) | ncyl++;
            for (int j = 0; j < 8; ++j) cyls.push_back((R)p.v[j]);
            break;
        case MT_PRIM_TRIANGLE: {
            code = (KIND_TRIANGLE << 28) | ntri++;
            if (sizeof(R) == 8) {
                // a, e1 = b - a, e2 = c - a in double (src/geometry.c:229-241)
                for (int j = 0; j < 3; ++j) tris.push_back((R)p.v[j]);
                for (int j = 0; j < 3; ++j) tris.push_back((R)(p.v[3 + j] - p.v[j]));
                for (int j = 0; j < 3; ++j) tris.push_back((R)(p.v[6 + j] - p.v[j]));
                tri_smooth.push_back(p.smooth ? 1 : 0);
            } else {
                float4 a = make_float4((float)p.v[0], (float)p.v[1], (float)p.v[2], 0.0f);
                float4 b = make_float4((float)p.v[3], (float)p.v[4], (float)p.v[5], 0.0f);
                float4 c = make_float4((float)p.v[6], (float)p.v[7], (float)p.v[8], 0.0f);
                int pid = pi, sm = p.smooth ? 1 : 0;
                memcpy(&a.w, &pid, 4);
                memcpy(&b.w, &sm, 4);
                tri4.push_back(a);
                tri4.push_back(b);
                tri4.push_back(c);
            }
            if (any_smooth)
                for (int j = 0; j < 9; ++j) tri_normals.push_back((R)p.n[j]);
            if (any_uv)
                for (int j = 0; j < 6; ++j)
                    tri_uv.push_back(p.has_uv ? (R)p.uv[j] : std::numeric_limits<R>::quiet_NaN());
            break;
        }
        default:
            break;
        }
        refs[k] = make_int2(pi, code);
        prim_info[pi] = make_int2(code, p.material);
    }
    for (size_t k = 0; k < sc->bvh.planes.size(); ++k) {
        int pi = sc->bvh.planes[k];
        const mt_prim &p = d->prims[pi];
        double nrm[3];
        normalize3(p.v + 3, nrm);  // intersect_plane re-normalises the axis (src/geometry.c:375)
        for (int j = 0; j < 3; ++j) planes.push_back((R)p.v[j]);
        for (int j = 0; j < 3; ++j) planes.push_back((R)nrm[j]);
        plane_prims.push_back(pi);
        prim_info[pi] = make_int2((KIND_PLANE << 28) | (int)k, p.material);
    }

    // image textures: one device copy per material, kept for the scene's life
    // (shared by the FP32 and FP64 uploads)
    if (sc->d_tex.size() != (size_t)d->material_count) {
        sc->d_tex.assign(d->material_count, nullptr);
        for (int i = 0; i < d->material_count; ++i) {
            const mt_material &m = d->materials[i];
            if (!m.texture_rgb) continue;
            std::vector<unsigned char> img(m.texture_rgb,
                                           m.texture_rgb + (size_t)m.texture_width * m.texture_height * 3);
            const unsigned char *dp = nullptr;
            int rc = sc->upload(img, &dp);
            if (rc) return rc;
            sc->d_tex[i] = dp;
        }
    }
    std::vector<DevMaterial<R>> mats(d->material_count);
    for (int i = 0; i < d->material_count; ++i) fill_material(d->materials[i], sc->d_tex[i], &mats[i]);

    std::vector<float4> nodes(fb.nodes.size() / 4);
    if (!fb.nodes.empty()) memcpy(nodes.data(), fb.nodes.data(), fb.nodes.size() * sizeof(float));
    // Leaves whose primitives are all triangles point straight at their
    // (consecutive) triangle slots, skipping the reference indirection.
    std::vector<int> tri_prim(ntri > 0 ? ntri : 1, 0);
    for (size_t k = 0; k < refs.size(); ++k)
        if ((refs[k].y >> 28) == KIND_TRIANGLE) tri_prim[refs[k].y & 0x0FFFFFFF] = refs[k].x;
    for (size_t i = 0; i < nodes.size() / 4; ++i) {
        int *q3 = reinterpret_cast<int *>(&nodes[4 * i + 3]);
        for (int side = 0; side < 2; ++side) {
            int c = q3[side];
            if (c >= 0) continue;
            int leaf = ~c;
            int first = leaf >> 4, count = leaf & 7;
            if (count == 0) continue;
            bool all_tri = true;
            for (int j = 0; j < count; ++j) all_tri = all_tri && (refs[first + j].y >> 28) == KIND_TRIANGLE;
            if (all_tri) q3[side] = ~(((refs[first].y & 0x0FFFFFFF) << 4) | (1 << 3) | count);
        }
    }

    // FP32 slab tests (box * inv - o * inv, one fma per plane) round by up to
    // a few units of 2^-24 of the largest coordinate magnitude M of the scene
    // (in world units, whatever the direction), so a hit on or next to a box
    // face could be culled. Every FP32 box is grown outward by MT_BOX_PAD
    // units of 2^-24 * M (and rounded outward): the walks stay conservative,
    // at the cost of a few more node visits. (FP64 keeps the tree as built.)
    double pad = 0.0;
    if (!nodes.empty()) {
        double m = 0.0;
        for (size_t i = 0; i < nodes.size() / 4; ++i) {
            const float *q = reinterpret_cast<const float *>(&nodes[4 * i]);
            for (int k = 0; k < 12; ++k)
                if (std::isfinite(q[k])) m = std::max(m, (double)fabsf(q[k]));
        }
        pad = MT_BOX_PAD * std::ldexp(m, -24);
    }
    auto pad_boxes = [&](size_t first, size_t count) {
        for (size_t i = first; i < first + count; ++i) {
            float *q = reinterpret_cast<float *>(&nodes[4 * i]);
            // lo / hi pairs: x (0, 1), y (2, 3) left; x (4, 5), y (6, 7) right;
            // z (8, 9) left, (10, 11) right
            for (int k = 0; k < 12; k += 2) {
                float lo = (float)((double)q[k] - pad), hi = (float)((double)q[k + 1] + pad);
                if ((double)lo > (double)q[k] - pad) lo = nextafterf(lo, -INFINITY);
                if ((double)hi < (double)q[k + 1] + pad) hi = nextafterf(hi, INFINITY);
                q[k] = lo;
                q[k + 1] = hi;
            }
        }
    };
    if (sizeof(R) == 4) pad_boxes(0, nodes.size() / 4);
    if (sizeof(R) == 4) {
        sc->nodes2.resize(nodes.size() * 4);
        if (!nodes.empty()) memcpy(sc->nodes2.data(), nodes.data(), sc->nodes2.size() * sizeof(float));
    }

    // Pass tree (DevScene::pass_root): the main tree pruned to the tree
    // primitives whose material lets a shadow ray through, appended after the
    // main tree's nodes and references.
    int pass_depth = 0;
    S->pass_root = kNoPassTree;
    {
        std::vector<char> mat_pass(d->material_count > 0 ? d->material_count : 1, 0);
        bool any_pass = false;
        for (int i = 0; i < d->material_count; ++i) {
            mat_pass[i] = d->materials[i].is_water || d->materials[i].transparency > 0.8;
            any_pass = any_pass || mat_pass[i];
        }
        auto passes = [&](int pi) {
            const int m = d->prims[pi].material;
            return m >= 0 && m < d->material_count && mat_pass[m];
        };
        bool plane_pass = false;
        for (int pi : sc->bvh.planes) plane_pass = plane_pass || passes(pi);
        if (any_pass && !plane_pass) {
            std::vector<char> keep(n > 0 ? n : 1, 0);
            for (int pi : sc->bvh.order) keep[pi] = passes(pi);
            HostBvh pb;
            FlatBvh pf;
            prune_bvh(sc->bvh, d->prims, keep, &pb);
            flatten_bvh(pb, &pf);
            if (pf.node_count == 0) {
                S->pass_root = kEmptyPassTree;
            } else {
                const int node_off = (int)(nodes.size() / 4), ref_off = (int)refs.size();
                for (int pi : pf.ref_prim) refs.push_back(make_int2(pi, prim_info[pi].x));
                const size_t base = nodes.size();
                nodes.resize(base + pf.nodes.size() / 4);
                memcpy(&nodes[base], pf.nodes.data(), pf.nodes.size() * sizeof(float));
                for (int i = 0; i < pf.node_count; ++i) {
                    int *q3 = reinterpret_cast<int *>(&nodes[base + 4 * (size_t)i + 3]);
                    for (int side = 0; side < 2; ++side) {
                        const int c = q3[side];
                        if (c >= 0) {
                            q3[side] = c + node_off;
                        } else {
                            const int leaf = ~c, count = leaf & 7;
                            if (count) q3[side] = ~((((leaf >> 4) + ref_off) << 4) | count);
                        }
                    }
                }
                pad_boxes(base / 4, (size_t)pf.node_count);
                S->pass_root = node_off;
                pass_depth = pf.depth;
            }
        }
    }

    int rc = 0;
    if ((rc = sc->upload(nodes, &S->nodes))) return rc;
    if ((rc = sc->upload(refs, &S->refs))) return rc;
    if ((rc = sc->upload(tri4, &S->tri4))) return rc;
    if ((rc = sc->upload(tris, &S->tris))) return rc;
    if ((rc = sc->upload(tri_normals, &S->tri_normals))) return rc;
    if ((rc = sc->upload(tri_uv, &S->tri_uv))) return rc;
    if ((rc = sc->upload(tri_smooth, &S->tri_smooth))) return rc;
    if (sizeof(R) == 8 && ntri > 0)
        if ((rc = sc->upload(tri_prim, &S->tri_prim))) return rc;
    if ((rc = sc->upload(spheres, &S->spheres))) return rc;
    if ((rc = sc->upload(boxes, &S->boxes))) return rc;
    if ((rc = sc->upload(cyls, &S->cyls))) return rc;
    if ((rc = sc->upload(planes, &S->planes))) return rc;
    if ((rc = sc->upload(plane_prims, &S->plane_prims))) return rc;
    if ((rc = sc->upload(prim_info, &S->prim_info))) return rc;
    if ((rc = sc->upload(mats, &S->materials))) return rc;

    S->node_count = fb.node_count;
    // pushes happen only on the way down, in either tree
    S->stack_depth = (fb.depth > pass_depth ? fb.depth : pass_depth) + 1;
    S->bvh_width = 2;
    S->wide_stack_depth = 0;
    S->plane_count = (int)plane_prims.size();
    S->prim_count = n;
    S->material_count = d->material_count;
    S->water_material = d->water_material;
    // pt_occluded_segment passes through water and transparency > 0.8
    // (src/pathtrace.c:516); without such a material it is an any-hit query.
    S->has_passthrough = 0;
    for (int i = 0; i < d->material_count; ++i)
        if (d->materials[i].is_water || d->materials[i].transparency > 0.8) S->has_passthrough = 1;
    S->has_extras = d->fog_density > 0.0 || d->fog_shadow_steps > 0 || d->sky.cloud_thickness > 1e-4;
    for (int i = 0; i < d->material_count; ++i)
        if (d->materials[i].texture_kind != MT_TEXTURE_NONE) S->has_extras = 1;
    // a scene of PBR surfaces only: no path enters a medium or takes the
    // legacy BSDF (the wavefront's specialised shade kernel)
    S->pbr_only = !S->has_extras && !S->has_passthrough && d->water_material < 0;
    for (int i = 0; i < d->material_count; ++i) {
        const mt_material &m = d->materials[i];
        if (!m.pbr || m.is_water || m.beer_lambert || m.atmosphere_glow[0] != 0.0 || m.atmosphere_glow[1] != 0.0 ||
            m.atmosphere_glow[2] != 0.0)
            S->pbr_only = 0;
    }
    S->water_level = (R)d->water_level;
    S->ocean.enabled = d->ocean.enabled;
    S->ocean.seed = d->ocean.seed;
    for (int k = 0; k < 3; ++k) {
        S->ocean.center[k] = (R)d->ocean.center[k];
        S->ocean.direction[k] = (R)d->ocean.direction[k];
    }
    S->ocean.amplitude = (R)d->ocean.amplitude;
    S->ocean.wavelength = (R)d->ocean.wavelength;
    S->ocean.chop = (R)d->ocean.chop;
    S->ocean.chop_wavelength = (R)d->ocean.chop_wavelength;
    fill_sky(d->sky, &S->sky);
    fill_fog(*d, &S->fog);

    // host copies for parameter updates (materials, sun, sphere list); the
    // image pointers are the caller's and are not kept
    sc->h_mats.assign(d->materials, d->materials + d->material_count);
    for (mt_material &m : sc->h_mats) m.texture_rgb = nullptr;
    sc->h_sky = d->sky;
    sc->h_spheres.clear();
    for (int i = 0; i < n; ++i)
        if (d->prims[i].kind == MT_PRIM_SPHERE)
            sc->h_spheres.push_back({i, d->prims[i].material, {d->prims[i].v[0], d->prims[i].v[1], d->prims[i].v[2]},
                                     d->prims[i].v[3]});
    collect_lights(sc, S);
    S->err = sc->d_err;
    S->counters = nullptr;
    S->version = 0;
    return 0;
}

template <typename R> void fill_camera(const mt_camera *c, DevCamera<R> *o)
{
    for (int k = 0; k < 3; ++k) {
        o->position[k] = (R)c->position[k];
        o->lower_left[k] = (R)c->lower_left[k];
        o->horizontal[k] = (R)c->horizontal[k];
        o->vertical[k] = (R)c->vertical[k];
    }
    o->aperture = (R)c->aperture;
    o->focus_distance = (R)c->focus_distance;
    o->dome_radius = (R)c->dome_radius;
    o->anamorphic_squeeze = (R)c->anamorphic_squeeze;
}

int set_device(const mt_scene *sc)
{
    CK(cudaSetDevice(sc->opts.device), "cudaSetDevice");
    return 0;
}

// Check the device error word after a synchronised launch and clear it.
int check_err_word(mt_scene *sc)
{
    unsigned e = 0;
    CK(cudaMemcpy(&e, sc->d_err, sizeof e, cudaMemcpyDeviceToHost), "cudaMemcpy(err)");
    sc->stats.error_flags = (int32_t)e;
    if (e != 0) {
        unsigned z = 0;
        CK(cudaMemcpy(sc->d_err, &z, sizeof z, cudaMemcpyHostToDevice), "cudaMemcpy(err)");
        if (e & ERR_STACK) return fail(MT_ERR_OVERFLOW, "traversal stack overflow");
        if (e & ERR_QUEUE) return fail(MT_ERR_OVERFLOW, "wavefront queue overflow");
        if (e & ERR_WHITTED) return fail(MT_ERR_OVERFLOW, "Whitted frame stack overflow");
        if (e & ERR_ABSORB)
            return fail(MT_ERR_UNSUPPORTED, "adjoint: a shadow segment crossed more than two absorbing materials");
        if (e & ERR_WATCHDOG) return fail(MT_ERR_WATCHDOG, "a bounded device loop reached its cap");
        return fail(MT_ERR_LAUNCH, "device error word 0x%x", e);
    }
    return 0;
}

int read_counters(mt_scene *sc)
{
    if (!sc->counting) return 0;
    DevCounters c;
    CK(cudaMemcpy(&c, sc->d_counters, sizeof c, cudaMemcpyDeviceToHost), "cudaMemcpy(counters)");
    sc->stats.primary_rays = (int64_t)c.primary_rays;
    sc->stats.extension_rays = (int64_t)c.extension_rays;
    sc->stats.shadow_rays = (int64_t)c.shadow_rays;
    sc->stats.node_visits = (int64_t)c.node_visits;
    sc->stats.prim_tests = (int64_t)c.prim_tests;
    sc->stats.tri_tests = (int64_t)c.tri_tests;
    sc->stats.any_node_visits = (int64_t)c.any_node_visits;
    sc->stats.any_prim_tests = (int64_t)c.any_prim_tests;
    sc->stats.any_tri_tests = (int64_t)c.any_tri_tests;
    return 0;
}

int reset_counters(mt_scene *sc)
{
    if (!sc->counting) return 0;
    CK(cudaMemset(sc->d_counters, 0, sizeof(DevCounters)), "cudaMemset(counters)");
    return 0;
}

// The tree the FP32 traversal kernels walk: the binary tree (W = 2) or a
// wide tree collapsed from it (W = 4 or 8), built on first use and kept for
// the scene's lifetime. The FP64 path always walks the binary tree.
int select_bvh_width(mt_scene *sc, int W)
{
    DevScene<float> &S = sc->sf;
    if (sc->opts.precision != MT_PRECISION_FP32 || W == 2 || S.node_count == 0) {
        S.bvh_width = 2;
        S.wnodes = nullptr;
        S.wide_stack_depth = 0;
        return 0;
    }
    if (W != 4 && W != 8) return fail(MT_ERR_INVALID, "bvh_width %d (2, 4 or 8)", W);
    const int k = W == 4 ? 0 : 1;
    if (!sc->wide[k]) {
        std::vector<float> wide;
        int bound = 0;
        if (collapse_bvh(sc->nodes2, S.node_count, W, &wide, &bound)) return fail(MT_ERR_INVALID, "wide BVH collapse");
        std::vector<float4> wn(wide.size() / 4);
        memcpy(wn.data(), wide.data(), wide.size() * sizeof(float));
        int rc = sc->upload(wn, &sc->wide[k]);
        if (rc) return rc;
        sc->wide_depth[k] = bound + 1;
    }
    S.wnodes = sc->wide[k];
    S.bvh_width = W;
    S.wide_stack_depth = sc->wide_depth[k];
    return 0;
}

template <typename R> DevScene<R> &dev_scene(mt_scene *sc);
template <> DevScene<float> &dev_scene<float>(mt_scene *sc) { return sc->sf; }
template <> DevScene<double> &dev_scene<double>(mt_scene *sc) { return sc->sd; }

// Run one per-pixel render kernel over samples [s0, s1) into device memory.
template <typename R>
int render_dev(mt_scene *sc, const mt_camera *cam, int w, int h, int spp_total, int s0, int s1, int depth, int mode,
               int out_kind, void *dout, cudaStream_t stream, bool timed)
{
    DevCamera<R> dc;
    fill_camera(cam, &dc);
    DevScene<R> S = dev_scene<R>(sc);
    S.counters = sc->counting ? sc->d_counters : nullptr;
    if (sc->opts.integrator == MT_INTEGRATOR_WAVEFRONT && mode == RENDER_PT) {
        S.trace_rec = sc->d_trace;
        S.trace_count = sc->d_trace_n;
        S.trace_cap = sc->trace_cap;
        int rc = wavefront_render(sc->wf, S, dc, w, h, s0, s1, depth, out_kind, dout, stream, &sc->opts,
                                     timed ? sc->ev0 : nullptr, timed ? sc->ev1 : nullptr, &sc->stats.launches);
        if (rc) return fail(rc, "wavefront render failed: %s", wavefront_last_error());
        return 0;
    }
    if (timed) CK(cudaEventRecord(sc->ev0, stream), "cudaEventRecord");
    CK(launch_render<R>(S, dc, w, h, spp_total, s0, s1, depth, mode, out_kind, dout, sc->opts.block_size, stream),
       "render kernel launch");
    if (timed) CK(cudaEventRecord(sc->ev1, stream), "cudaEventRecord");
    sc->stats.launches = 1;
    return 0;
}

// The path-replay adjoint with the scene's integrator: the wavefront form
// (primal and replay passes as stage kernels over compacted queues) or one
// thread per pixel running both passes.
template <typename R>
int adjoint_dev(mt_scene *sc, const mt_camera *cam, int w, int h, int s0, int s1, int depth, const float *adj_img,
                double scale, double *grad, int n_params, cudaStream_t stream)
{
    DevCamera<R> dc;
    fill_camera(cam, &dc);
    DevScene<R> S = dev_scene<R>(sc);
    S.counters = sc->counting ? sc->d_counters : nullptr;
    if (sc->opts.integrator == MT_INTEGRATOR_WAVEFRONT) {
        WfAdjointCall a{adj_img, scale, grad, n_params};
        int rc = wavefront_adjoint(sc->wf, S, dc, w, h, s0, s1, depth, a, stream, &sc->opts);
        if (rc) return fail(rc, "wavefront adjoint failed: %s", wavefront_last_error());
        return 0;
    }
    CK(launch_adjoint<R>(S, dc, w, h, s0, s1, depth, adj_img, scale, grad, n_params, stream), "adjoint launch");
    return 0;
}

int render_args(const mt_scene *sc, const mt_camera *cam, const void *out, int w, int h, int spp, int depth)
{
    if (sc == nullptr || cam == nullptr || out == nullptr) return fail(MT_ERR_NULL, "NULL pointer");
    if (w <= 0 || h <= 0) return fail(MT_ERR_DIMS, "non-positive dimensions");
    if (spp < 1 || depth < 0) return fail(MT_ERR_COUNTS, "bad sample / depth counts");
    return 0;
}

// Full-frame render into a host buffer (RGB8 or mean float).
int render_host(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int depth, int mode, int out_kind,
                void *host_out)
{
    int rc = render_args(sc, cam, host_out, w, h, spp, depth);
    if (rc) return rc;
    if (mode == RENDER_WHITTED && depth + 2 > kWhittedFrames)
        return fail(MT_ERR_UNSUPPORTED, "Whitted depth %d exceeds the device frame stack (max %d)", depth,
                    kWhittedFrames - 2);
    if ((rc = set_device(sc))) return rc;
    size_t bytes = (size_t)w * h * 3 * (out_kind == OUT_RGB8 ? 1 : sizeof(float));
    void *dout = nullptr;
    CK(cudaMalloc(&dout, bytes), "cudaMalloc(image)");
    if ((rc = reset_counters(sc))) {
        cudaFree(dout);
        return rc;
    }
    if (sc->opts.precision == MT_PRECISION_FP64)
        rc = render_dev<double>(sc, cam, w, h, spp, 0, spp, depth, mode, out_kind, dout, 0, true);
    else
        rc = render_dev<float>(sc, cam, w, h, spp, 0, spp, depth, mode, out_kind, dout, 0, true);
    cudaError_t e = cudaSuccess;
    if (!rc) {
        e = cudaDeviceSynchronize();
        if (e == cudaSuccess) e = cudaMemcpy(host_out, dout, bytes, cudaMemcpyDeviceToHost);
    }
    cudaFree(dout);
    if (rc) return rc;
    if (e != cudaSuccess) return cuda_fail(e, "render");
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
    sc->stats.kernel_ms = ms;
    if ((rc = read_counters(sc))) return rc;
    return check_err_word(sc);
}

template <typename T> struct DevBuf {
    T *p = nullptr;
    ~DevBuf()
    {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) { return cudaMalloc(&p, (n ? n : 1) * sizeof(T)); }
};

}  // namespace

extern "C" {

void mt_options_default(mt_options *o)
{
    if (!o) return;
    memset(o, 0, sizeof *o);
    o->precision = MT_PRECISION_FP32;
    o->integrator = MT_INTEGRATOR_MEGAKERNEL;
    o->block_size = 128;
    o->queue_capacity = 0;
    o->bvh_width = 2;
    o->sort_threshold = 1 << 18;
    o->use_graph = 1;
    o->device = 0;
    o->traversal = MT_TRAVERSAL_DEFAULT;
    o->bvh_builder = MT_BVH_BUILDER_HOST;
}

const char *mt_version(void) { return "mtgpu 0.1 (sm_100a)"; }
const char *mt_last_error(void) { return g_last_error.c_str(); }

int mt_scene_create(const mt_scene_desc *desc, const mt_options *opts, mt_scene **out)
{
    if (!desc || !out) return fail(MT_ERR_NULL, "NULL pointer");
    *out = nullptr;
    int rc = validate(desc);
    if (rc) return rc;
    int ndev = 0;
    cudaError_t e = cudaGetDeviceCount(&ndev);
    if (e != cudaSuccess || ndev <= 0) return fail(MT_ERR_NO_DEVICE, "no CUDA device (%s)", cudaGetErrorString(e));

    mt_scene *sc = new mt_scene();
    if (opts) sc->opts = *opts;
    else mt_options_default(&sc->opts);
    if (sc->opts.block_size <= 0) sc->opts.block_size = 128;
    if (sc->opts.bvh_width == 0) sc->opts.bvh_width = 2;
    if (sc->opts.bvh_width != 2 && sc->opts.bvh_width != 4 && sc->opts.bvh_width != 8) {
        int wd = sc->opts.bvh_width;
        delete sc;
        return fail(MT_ERR_INVALID, "bvh_width %d (2, 4 or 8)", wd);
    }
    if (sc->opts.device < 0 || sc->opts.device >= ndev) {
        delete sc;
        return fail(MT_ERR_INVALID, "device %d out of range", sc->opts.device);
    }
    sc->prim_count = desc->prim_count;
    memset(&sc->stats, 0, sizeof sc->stats);
    auto bail = [&](int code) {
        mt_scene_release(sc);
        return code;
    };
    if ((rc = set_device(sc))) return bail(rc);

    if (sc->opts.bvh_builder == MT_BVH_BUILDER_DEVICE) {
        std::string err;
        int brc = build_bvh_device(desc->prims, desc->prim_count, &sc->bvh, &err, nullptr);
        if (brc) return bail(fail(brc, "device BVH build: %s", err.c_str()));
    } else {
        build_bvh(desc->prims, desc->prim_count, &sc->bvh);
    }
    flatten_bvh(sc->bvh, &sc->flat);
    if (sc->flat.depth + 1 > kStackSize)
        return bail(fail(MT_ERR_UNSUPPORTED, "BVH depth %d exceeds the traversal stack (%d)", sc->flat.depth,
                         kStackSize));
    if (sc->flat.ref_prim.size() >= (size_t(1) << 26))
        return bail(fail(MT_ERR_UNSUPPORTED, "more than 2^26 tree primitives"));

    void *p = nullptr;
    e = cudaMalloc(&p, sizeof(unsigned));
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(err)"));
    sc->allocs.push_back(p);
    sc->d_err = (unsigned *)p;
    cudaMemset(sc->d_err, 0, sizeof(unsigned));
    e = cudaMalloc(&p, sizeof(DevCounters));
    if (e != cudaSuccess) return bail(cuda_fail(e, "cudaMalloc(counters)"));
    sc->allocs.push_back(p);
    sc->d_counters = (DevCounters *)p;
    cudaMemset(sc->d_counters, 0, sizeof(DevCounters));
    if ((e = cudaEventCreate(&sc->ev0)) != cudaSuccess || (e = cudaEventCreate(&sc->ev1)) != cudaSuccess)
        return bail(cuda_fail(e, "cudaEventCreate"));

    if (sc->opts.precision == MT_PRECISION_FP64) rc = upload_scene<double>(sc, desc, &sc->sd);
    else rc = upload_scene<float>(sc, desc, &sc->sf);
    if (!rc) rc = select_bvh_width(sc, sc->opts.bvh_width);
    if (rc) return bail(rc);
    *out = sc;
    return 0;
}

void mt_scene_release(mt_scene *sc)
{
    if (!sc) return;
    cudaSetDevice(sc->opts.device);
    if (sc->wf) wavefront_destroy(sc->wf);
    for (void *p : sc->allocs) cudaFree(p);
    if (sc->d_trace) cudaFree(sc->d_trace);
    if (sc->d_trace_n) cudaFree(sc->d_trace_n);
    if (sc->ev0) cudaEventDestroy(sc->ev0);
    if (sc->ev1) cudaEventDestroy(sc->ev1);
    delete sc;
}

int mt_scene_get_info(const mt_scene *sc, mt_scene_info *info)
{
    if (!sc || !info) return fail(MT_ERR_NULL, "NULL pointer");
    memset(info, 0, sizeof *info);
    info->prim_count = sc->prim_count;
    info->plane_count = (int32_t)sc->bvh.planes.size();
    info->node_count = (int32_t)sc->bvh.nodes.size();
    info->depth = sc->bvh.depth;
    info->light_count = sc->light_count;
    for (int i = 0; i < sc->light_count; ++i) info->light_prims[i] = sc->light_prims[i];
    info->device_bytes = sc->device_bytes;
    return 0;
}

int mt_scene_export_bvh(const mt_scene *sc, double *bounds6, int32_t *links4, int32_t *order, int32_t *node_count,
                        int32_t *order_count)
{
    if (!sc) return fail(MT_ERR_NULL, "NULL pointer");
    if (node_count) *node_count = (int32_t)sc->bvh.nodes.size();
    if (order_count) *order_count = (int32_t)sc->bvh.order.size();
    for (size_t i = 0; i < sc->bvh.nodes.size(); ++i) {
        const HostNode &n = sc->bvh.nodes[i];
        if (bounds6)
            for (int k = 0; k < 3; ++k) {
                bounds6[6 * i + k] = n.mn[k];
                bounds6[6 * i + 3 + k] = n.mx[k];
            }
        if (links4) {
            links4[4 * i] = n.left;
            links4[4 * i + 1] = n.right;
            links4[4 * i + 2] = n.first;
            links4[4 * i + 3] = n.count;
        }
    }
    if (order)
        for (size_t i = 0; i < sc->bvh.order.size(); ++i) order[i] = sc->bvh.order[i];
    return 0;
}

int mt_bvh_build_host(const mt_prim *prims, int32_t n, double *bounds6, int32_t *links4, int32_t *order,
                      int32_t *node_count, int32_t *order_count, int32_t *depth)
{
    if (n < 0 || (n > 0 && !prims)) return fail(MT_ERR_NULL, "NULL pointer");
    HostBvh b;
    build_bvh(prims, n, &b);
    if (node_count) *node_count = (int32_t)b.nodes.size();
    if (order_count) *order_count = (int32_t)b.order.size();
    if (depth) *depth = b.depth;
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        const HostNode &nd = b.nodes[i];
        if (bounds6)
            for (int k = 0; k < 3; ++k) {
                bounds6[6 * i + k] = nd.mn[k];
                bounds6[6 * i + 3 + k] = nd.mx[k];
            }
        if (links4) {
            links4[4 * i] = nd.left;
            links4[4 * i + 1] = nd.right;
            links4[4 * i + 2] = nd.first;
            links4[4 * i + 3] = nd.count;
        }
    }
    if (order)
        for (size_t i = 0; i < b.order.size(); ++i) order[i] = b.order[i];
    return 0;
}

int mt_bvh_build_device(const mt_prim *prims, int32_t n, int32_t device, double *bounds6, int32_t *links4,
                        int32_t *order, int32_t *node_count, int32_t *order_count, int32_t *depth, float *build_ms)
{
    if (n < 0 || (n > 0 && !prims)) return fail(MT_ERR_NULL, "NULL pointer");
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) return fail(MT_ERR_NO_DEVICE, "no CUDA device");
    if (device < 0 || device >= ndev) return fail(MT_ERR_INVALID, "device %d out of range", device);
    CK(cudaSetDevice(device), "cudaSetDevice");
    HostBvh b;
    std::string err;
    int rc = build_bvh_device(prims, n, &b, &err, build_ms);
    if (rc) return fail(rc, "device BVH build: %s", err.c_str());
    if (node_count) *node_count = (int32_t)b.nodes.size();
    if (order_count) *order_count = (int32_t)b.order.size();
    if (depth) *depth = b.depth;
    for (size_t i = 0; i < b.nodes.size(); ++i) {
        const HostNode &nd = b.nodes[i];
        if (bounds6)
            for (int k = 0; k < 3; ++k) {
                bounds6[6 * i + k] = nd.mn[k];
                bounds6[6 * i + 3 + k] = nd.mx[k];
            }
        if (links4) {
            links4[4 * i] = nd.left;
            links4[4 * i + 1] = nd.right;
            links4[4 * i + 2] = nd.first;
            links4[4 * i + 3] = nd.count;
        }
    }
    if (order)
        for (size_t i = 0; i < b.order.size(); ++i) order[i] = b.order[i];
    return 0;
}

// camera_create (src/camera.c:24-66) in host double arithmetic.
void mt_camera_create(const double from[3], const double at[3], const double up[3], double vfov_deg, double aspect,
                      mt_camera *out)
{
    if (!out) return;
    memset(out, 0, sizeof *out);
    double fwd_raw[3] = {at[0] - from[0], at[1] - from[1], at[2] - from[2]};
    double forward[3];
    normalize3(fwd_raw, forward);
    if (forward[0] * forward[0] + forward[1] * forward[1] + forward[2] * forward[2] <= 1e-12) {
        forward[0] = 0.0;
        forward[1] = 0.0;
        forward[2] = -1.0;
    }
    auto cross3 = [](const double *a, const double *b, double *o) {
        o[0] = a[1] * b[2] - a[2] * b[1];
        o[1] = a[2] * b[0] - a[0] * b[2];
        o[2] = a[0] * b[1] - a[1] * b[0];
    };
    double right[3];
    cross3(forward, up, right);
    if (right[0] * right[0] + right[1] * right[1] + right[2] * right[2] <= 1e-12) {
        double fb[3] = {0.0, 1.0, 0.0};
        if (!(fabs(forward[1]) < 0.99)) {
            fb[0] = 1.0;
            fb[1] = 0.0;
        }
        cross3(forward, fb, right);
    }
    double rn[3];
    normalize3(right, rn);
    double true_up[3];
    cross3(rn, forward, true_up);
    double vfov_rad = vfov_deg * (3.14159265358979323846 / 180.0);
    double half_h = tan(vfov_rad * 0.5);
    double half_w = aspect * half_h;
    for (int k = 0; k < 3; ++k) {
        out->position[k] = from[k];
        out->horizontal[k] = rn[k] * (2.0 * half_w);
        out->vertical[k] = true_up[k] * (2.0 * half_h);
    }
    for (int k = 0; k < 3; ++k) {
        double a = from[k] + forward[k];
        double b = out->horizontal[k] * 0.5 + out->vertical[k] * 0.5;
        out->lower_left[k] = a - b;
    }
    out->aperture = 0.0;
    double dd[3] = {at[0] - from[0], at[1] - from[1], at[2] - from[2]};
    out->focus_distance = sqrt(dd[0] * dd[0] + dd[1] * dd[1] + dd[2] * dd[2]);
    out->dome_radius = 0.0;
    out->anamorphic_squeeze = 1.0;
}

int mt_pathtrace_render(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int depth, unsigned char *rgb)
{
    return render_host(sc, cam, w, h, spp, depth, RENDER_PT, OUT_RGB8, rgb);
}

int mt_render_image(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int depth, unsigned char *rgb)
{
    return render_host(sc, cam, w, h, spp, depth, RENDER_WHITTED, OUT_RGB8, rgb);
}

}  // extern "C"

namespace {

// render_image_adaptive (src/render.c:1382-1500) on the device: pass 0 over
// every pixel, then refinement passes over the pixels the active-set kernel
// flags, until none is flagged or the pass bound is reached; the host reads
// only the flagged count between passes, as the reference's loop does.
template <typename R>
int adaptive_dev(mt_scene *sc, const mt_camera *cam, int w, int h, int n0, int nmax, double tau, int depth,
                 unsigned char *rgb)
{
    DevCamera<R> dc;
    fill_camera(cam, &dc);
    DevScene<R> S = dev_scene<R>(sc);
    S.counters = sc->counting ? sc->d_counters : nullptr;
    const int wh = w * h;
    DevBuf<double> sums;
    DevBuf<int> nsamp, list, count;
    DevBuf<unsigned char> drgb;
    CK(sums.alloc((size_t)wh * 5), "cudaMalloc(adaptive sums)");
    CK(nsamp.alloc((size_t)wh), "cudaMalloc(adaptive counts)");
    CK(list.alloc((size_t)wh), "cudaMalloc(adaptive list)");
    CK(count.alloc(1), "cudaMalloc(adaptive count)");
    CK(drgb.alloc((size_t)wh * 3), "cudaMalloc(rgb)");
    CK(cudaMemset(sums.p, 0, (size_t)wh * 5 * sizeof(double)), "cudaMemset");
    CK(cudaMemset(nsamp.p, 0, (size_t)wh * sizeof(int)), "cudaMemset");
    int max_passes = 1;
    if (nmax > n0 && n0 > 0) max_passes += (nmax - n0 + n0 - 1) / n0;
    CK(cudaEventRecord(sc->ev0, 0), "cudaEventRecord");
    CK(launch_adaptive_pass<R>(S, dc, w, h, n0, nmax, n0, depth, nullptr, nullptr, sums.p, nsamp.p, 0),
       "adaptive pass");
    int passes = 1;
    for (int pass = 1;; ++pass) {
        CK(cudaMemsetAsync(count.p, 0, sizeof(int), 0), "cudaMemsetAsync");
        CK(launch_adaptive_active(wh, nmax, tau, sums.p, nsamp.p, list.p, count.p, 0), "adaptive active set");
        int remaining = 0;
        CK(cudaMemcpy(&remaining, count.p, sizeof(int), cudaMemcpyDeviceToHost), "adaptive count");
        if (remaining == 0 || pass >= max_passes) break;
        CK(launch_adaptive_pass<R>(S, dc, w, h, n0, nmax, n0, depth, list.p, count.p, sums.p, nsamp.p, 0),
           "adaptive pass");
        ++passes;
    }
    CK(launch_adaptive_resolve(wh, sums.p, nsamp.p, drgb.p, 0), "adaptive resolve");
    CK(cudaEventRecord(sc->ev1, 0), "cudaEventRecord");
    CK(cudaMemcpy(rgb, drgb.p, (size_t)wh * 3, cudaMemcpyDeviceToHost), "cudaMemcpy(rgb)");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
    sc->stats.kernel_ms = ms;
    sc->stats.launches = 2 * passes + 1;
    if (sc->counting) {
        int rc = read_counters(sc);
        if (rc) return rc;
    }
    return check_err_word(sc);
}

int render_image_adaptive_dev(mt_scene *sc, const mt_camera *cam, int w, int h, const mt_render_params *p,
                              unsigned char *rgb)
{
    const int n0 = p->samples_per_pixel;
    int nmax = p->adaptive_max_spp > 0 ? p->adaptive_max_spp : 4 * n0;  // default cap (src/render.c:1655-1658)
    if (nmax < n0) nmax = n0;
    const double tau = p->adaptive_tau > 0.0 ? p->adaptive_tau : 0.02;   // default tolerance
    int rc = set_device(sc);
    if (rc) return rc;
    if (sc->opts.precision == MT_PRECISION_FP64)
        return adaptive_dev<double>(sc, cam, w, h, n0, nmax, tau, p->max_depth, rgb);
    return adaptive_dev<float>(sc, cam, w, h, n0, nmax, tau, p->max_depth, rgb);
}

}  // namespace

extern "C" {

int mt_render_image_ex(mt_scene *sc, const mt_camera *cam, int w, int h, const mt_render_params *p,
                       unsigned char *rgb)
{
    if (p == nullptr) return fail(MT_ERR_NULL, "NULL params");
    int rc = render_args(sc, cam, rgb, w, h, p->samples_per_pixel, p->max_depth);
    if (rc) return rc;
    if (p->adaptive) return render_image_adaptive_dev(sc, cam, w, h, p, rgb);
    return render_host(sc, cam, w, h, p->samples_per_pixel, p->max_depth, RENDER_WHITTED, OUT_RGB8, rgb);
}

int mt_render_linear(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int depth, int mode, float *out)
{
    if (mode != MT_MODE_PATHTRACE && mode != MT_MODE_WHITTED) return fail(MT_ERR_INVALID, "bad mode %d", mode);
    return render_host(sc, cam, w, h, spp, depth, mode == MT_MODE_PATHTRACE ? RENDER_PT : RENDER_WHITTED,
                       OUT_MEAN_F32, out);
}

int mt_render_accumulate_device(mt_scene *sc, const mt_camera *cam, int w, int h, int s0, int s1, int depth, int mode,
                                float *accum_dev, int accumulate, void *stream)
{
    int rc = render_args(sc, cam, accum_dev, w, h, s1 - s0, depth);
    if (rc) return rc;
    if (s0 < 0) return fail(MT_ERR_COUNTS, "negative first sample");
    if ((rc = set_device(sc))) return rc;
    int out_kind = accumulate ? OUT_ADD_F32 : OUT_SUM_F32;
    int m = mode == MT_MODE_PATHTRACE ? RENDER_PT : RENDER_WHITTED;
    if (sc->opts.precision == MT_PRECISION_FP64)
        return render_dev<double>(sc, cam, w, h, s1, s0, s1, depth, m, out_kind, accum_dev, (cudaStream_t)stream,
                                  false);
    return render_dev<float>(sc, cam, w, h, s1, s0, s1, depth, m, out_kind, accum_dev, (cudaStream_t)stream, false);
}

int mt_autotune(mt_scene *sc, const mt_camera *cam, int w, int h, int probe_spp, int depth, mt_tune_report *rep)
{
    if (!rep) return fail(MT_ERR_NULL, "NULL report");
    int rc = render_args(sc, cam, rep, w, h, probe_spp, depth);
    if (rc) return rc;
    if (sc->opts.precision != MT_PRECISION_FP32) return fail(MT_ERR_UNSUPPORTED, "mt_autotune: FP32 scenes only");
    if ((rc = set_device(sc))) return rc;
    memset(rep, 0, sizeof *rep);
    DevBuf<float> out;
    CK(out.alloc((size_t)w * h * 3), "cudaMalloc(probe)");
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0), "cudaEventCreate");
    if (cudaEventCreate(&e1) != cudaSuccess) {
        cudaEventDestroy(e0);
        return fail(MT_ERR_LAUNCH, "cudaEventCreate");
    }
    const bool counting = sc->counting;
    sc->counting = false;
    const mt_options saved = sc->opts;
    // Every probe render takes the next sample window, so no candidate sees
    // samples an earlier render already traced (the occluder cache would
    // otherwise hold the very blockers of its rays).
    int window = 0;
    const int s_base = 1 << 20;
    // time one configuration: a warm-up window (captures its graph), then the
    // better of two timed windows
    auto probe = [&](const mt_options &o, float *ms) -> int {
        sc->opts = o;
        int r = select_bvh_width(sc, o.bvh_width);
        if (r) return r;
        float best = 3.0e38f;
        for (int k = 0; k < 3; ++k) {
            if (k) CK(cudaEventRecord(e0, 0), "cudaEventRecord");
            const int s0 = s_base + probe_spp * window++;
            r = render_dev<float>(sc, cam, w, h, s0 + probe_spp, s0, s0 + probe_spp, depth, RENDER_PT, OUT_SUM_F32,
                                  out.p, 0, false);
            if (r) return r;
            if (k) {
                CK(cudaEventRecord(e1, 0), "cudaEventRecord");
                CK(cudaEventSynchronize(e1), "probe");
                float t = 0.f;
                cudaEventElapsedTime(&t, e0, e1);
                best = t < best ? t : best;
            } else {
                CK(cudaDeviceSynchronize(), "probe");
            }
        }
        *ms = best;
        if (rep->n_entries < MT_TUNE_MAX_ENTRIES) {
            rep->entries[rep->n_entries].options = o;
            rep->entries[rep->n_entries].ms = best;
            rep->n_entries++;
        }
        return 0;
    };
    mt_options cur = saved;
    cur.integrator = MT_INTEGRATOR_WAVEFRONT;
    cur.traversal = MT_TRAVERSAL_STATIC;
    cur.block_size = 128;
    cur.bvh_width = 2;
    cur.sort_threshold = 1 << 18;
    cur.queue_capacity = 0;
    cur.use_graph = 1;
    cur.occluder_cache = 0;
    float cur_ms = 0.f;
    rc = probe(cur, &cur_ms);
    rep->default_ms = cur_ms;
    // samples per batch of the probe window for a queue capacity (the largest
    // divisor of probe_spp whose paths fit; 0 = the library default of 2^25)
    auto probe_batch = [&](long long capacity) {
        const long long cap = std::max<long long>(capacity > 0 ? capacity : (1ll << 25), (long long)w * h);
        for (int d = probe_spp; d >= 1; --d)
            if (probe_spp % d == 0 && (long long)w * h * d <= cap) return d;
        return 1;
    };
    // coordinate descent over the knobs, defaults first in each stage
    // (stage 5, scenes with pass-through materials: the occluder cache with
    // the pass tree, off by default there)
    const bool pass_scene = sc->sf.has_passthrough && sc->sf.pass_root != kNoPassTree;
    for (int stage = 0; stage < 6 && !rc; ++stage) {
        int vals[4];
        int nv = 0;
        switch (stage) {
        case 0: vals[nv++] = MT_TRAVERSAL_DYNAMIC; break;
        case 1: vals[nv++] = 64; break;
        case 2: vals[nv++] = 4; vals[nv++] = 8; break;
        case 3: vals[nv++] = 0; vals[nv++] = 1; break;
        case 4: vals[nv++] = 8 << 20; vals[nv++] = 2 << 20; break;
        default:
            if (pass_scene) vals[nv++] = 1;
            break;
        }
        for (int i = 0; i < nv && !rc; ++i) {
            mt_options o = cur;
            if (stage == 0) o.traversal = vals[i];
            else if (stage == 1) o.block_size = vals[i];
            else if (stage == 2) o.bvh_width = vals[i];
            else if (stage == 3) o.sort_threshold = vals[i];
            else if (stage == 4) o.queue_capacity = vals[i];
            else o.occluder_cache = vals[i];
            // a capacity that splits the probe window into the same batches as
            // the current one cannot be told apart by the probe: skip it
            if (stage == 4 && probe_batch(o.queue_capacity) == probe_batch(cur.queue_capacity)) continue;
            float ms = 0.f;
            rc = probe(o, &ms);
            if (!rc && ms < cur_ms) {
                cur = o;
                cur_ms = ms;
            }
        }
    }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    sc->counting = counting;
    if (rc) {
        sc->opts = saved;
        select_bvh_width(sc, saved.bvh_width);
        return rc;
    }
    sc->opts = cur;
    if ((rc = select_bvh_width(sc, cur.bvh_width))) return rc;
    rep->chosen = cur;
    rep->chosen_ms = cur_ms;
    return 0;
}

int mt_get_stats(const mt_scene *csc, mt_stats *out)
{
    if (!csc || !out) return fail(MT_ERR_NULL, "NULL pointer");
    mt_scene *sc = const_cast<mt_scene *>(csc);
    if (sc->counting) {
        // Asynchronous launches (mt_render_accumulate_device) leave the
        // counters on the device: wait for them and read them here.
        int rc = set_device(sc);
        if (rc) return rc;
        CK(cudaDeviceSynchronize(), "mt_get_stats");
        if ((rc = read_counters(sc))) return rc;
    }
    double ms[4];
    long long nl[4];
    wavefront_stage_times(sc->wf, ms, nl);
    for (int i = 0; i < 4; ++i) {
        sc->stats.stage_ms[i] = ms[i];
        sc->stats.stage_launches[i] = nl[i];
    }
    *out = sc->stats;
    return 0;
}

int mt_set_counting(mt_scene *sc, int enable)
{
    if (!sc) return fail(MT_ERR_NULL, "NULL pointer");
    sc->counting = enable != 0;
    sc->sf.counters = nullptr;
    sc->sd.counters = nullptr;
    wavefront_reset_stage_times(sc->wf);
    return reset_counters(sc);
}

int mt_pathtrace_radiance_mode(mt_scene *sc, int n, const double *o, const double *d, int depth,
                               const uint32_t *seeds, double *out, int mode)
{
    if (!sc || !o || !d || !seeds || !out) return fail(MT_ERR_NULL, "NULL pointer");
    if (n <= 0) return 0;
    int rc = set_device(sc);
    if (rc) return rc;
    DevBuf<double> dO, dD, dOut;
    DevBuf<unsigned> dS;
    CK(dO.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dD.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dOut.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dS.alloc((size_t)n), "cudaMalloc");
    CK(cudaMemcpy(dO.p, o, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    CK(cudaMemcpy(dD.p, d, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    CK(cudaMemcpy(dS.p, seeds, n * sizeof(unsigned), cudaMemcpyHostToDevice), "cudaMemcpy");
    if (sc->opts.precision == MT_PRECISION_FP64)
        CK(launch_radiance<double>(sc->sd, n, dO.p, dD.p, depth, dS.p, dOut.p, mode, 0), "radiance launch");
    else
        CK(launch_radiance<float>(sc->sf, n, dO.p, dD.p, depth, dS.p, dOut.p, mode, 0), "radiance launch");
    CK(cudaDeviceSynchronize(), "radiance kernel");
    CK(cudaMemcpy(out, dOut.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return check_err_word(sc);
}

int mt_pathtrace_radiance(mt_scene *sc, int n, const double *o, const double *d, int depth, const uint32_t *seeds,
                          double *out)
{
    return mt_pathtrace_radiance_mode(sc, n, o, d, depth, seeds, out, RENDER_PT);
}

int mt_whitted_trace(mt_scene *sc, int n, const double *o, const double *d, int depth, const uint32_t *seeds,
                     double *out)
{
    if (depth + 2 > kWhittedFrames) return fail(MT_ERR_UNSUPPORTED, "Whitted depth too large");
    return mt_pathtrace_radiance_mode(sc, n, o, d, depth, seeds, out, RENDER_WHITTED);
}

int mt_intersect(mt_scene *sc, int n, const double *o, const double *d, double tmin, double tmax, int32_t *prim,
                 double *t, double *normal, int32_t *front, int32_t *mat)
{
    if (!sc || !o || !d || !prim) return fail(MT_ERR_NULL, "NULL pointer");
    if (n <= 0) return 0;
    int rc = set_device(sc);
    if (rc) return rc;
    DevBuf<double> dO, dD, dT, dN;
    DevBuf<int> dP, dF, dM;
    CK(dO.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dD.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dT.alloc((size_t)n), "cudaMalloc");
    CK(dN.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dP.alloc((size_t)n), "cudaMalloc");
    CK(dF.alloc((size_t)n), "cudaMalloc");
    CK(dM.alloc((size_t)n), "cudaMalloc");
    CK(cudaMemcpy(dO.p, o, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    CK(cudaMemcpy(dD.p, d, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    if (sc->opts.precision == MT_PRECISION_FP64)
        CK(launch_intersect<double>(sc->sd, n, dO.p, dD.p, tmin, tmax, dP.p, dT.p, dN.p, dF.p, dM.p, 0), "launch");
    else
        CK(launch_intersect<float>(sc->sf, n, dO.p, dD.p, tmin, tmax, dP.p, dT.p, dN.p, dF.p, dM.p, 0), "launch");
    CK(cudaDeviceSynchronize(), "intersect kernel");
    CK(cudaMemcpy(prim, dP.p, n * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (t) CK(cudaMemcpy(t, dT.p, n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (normal) CK(cudaMemcpy(normal, dN.p, 3 * n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (front) CK(cudaMemcpy(front, dF.p, n * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    if (mat) CK(cudaMemcpy(mat, dM.p, n * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return check_err_word(sc);
}

int mt_occluded(mt_scene *sc, int n, const double *o, const double *d, double tmin, double tmax, int32_t *occ)
{
    if (!sc || !o || !d || !occ) return fail(MT_ERR_NULL, "NULL pointer");
    if (n <= 0) return 0;
    int rc = set_device(sc);
    if (rc) return rc;
    DevBuf<double> dO, dD;
    DevBuf<int> dOcc;
    CK(dO.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dD.alloc(3 * (size_t)n), "cudaMalloc");
    CK(dOcc.alloc((size_t)n), "cudaMalloc");
    CK(cudaMemcpy(dO.p, o, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    CK(cudaMemcpy(dD.p, d, 3 * n * sizeof(double), cudaMemcpyHostToDevice), "cudaMemcpy");
    if (sc->opts.precision == MT_PRECISION_FP64)
        CK(launch_occluded<double>(sc->sd, n, dO.p, dD.p, tmin, tmax, dOcc.p, 0), "launch");
    else
        CK(launch_occluded<float>(sc->sf, n, dO.p, dD.p, tmin, tmax, dOcc.p, 0), "launch");
    CK(cudaDeviceSynchronize(), "occluded kernel");
    CK(cudaMemcpy(occ, dOcc.p, n * sizeof(int), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return check_err_word(sc);
}

int mt_trace_log_enable(mt_scene *sc, int32_t capacity)
{
    if (!sc) return fail(MT_ERR_NULL, "NULL pointer");
    if (capacity < 0) return fail(MT_ERR_INVALID, "negative capacity");
    if (sc->opts.precision != MT_PRECISION_FP32) return fail(MT_ERR_UNSUPPORTED, "the query log is FP32 only");
    int rc = set_device(sc);
    if (rc) return rc;
    CK(cudaDeviceSynchronize(), "synchronize");
    if (sc->d_trace) cudaFree(sc->d_trace);
    if (sc->d_trace_n) cudaFree(sc->d_trace_n);
    sc->d_trace = nullptr;
    sc->d_trace_n = nullptr;
    sc->trace_cap = 0;
    if (capacity == 0) return 0;
    CK(cudaMalloc((void **)&sc->d_trace, (size_t)capacity * 3 * sizeof(float4)), "cudaMalloc(query log)");
    CK(cudaMalloc((void **)&sc->d_trace_n, sizeof(unsigned)), "cudaMalloc(query log count)");
    CK(cudaMemset(sc->d_trace_n, 0, sizeof(unsigned)), "cudaMemset(query log count)");
    sc->trace_cap = capacity;
    return 0;
}

int mt_trace_log_read(mt_scene *sc, float *records, int32_t capacity, int64_t *count)
{
    if (!sc || !count) return fail(MT_ERR_NULL, "NULL pointer");
    if (!sc->d_trace) return fail(MT_ERR_INVALID, "the query log is not enabled");
    int rc = set_device(sc);
    if (rc) return rc;
    CK(cudaDeviceSynchronize(), "synchronize");
    unsigned n = 0;
    CK(cudaMemcpy(&n, sc->d_trace_n, sizeof n, cudaMemcpyDeviceToHost), "cudaMemcpy(query log count)");
    *count = (int64_t)n;
    int64_t keep = (int64_t)n < (int64_t)sc->trace_cap ? (int64_t)n : (int64_t)sc->trace_cap;
    if (keep > capacity) keep = capacity;
    if (keep > 0 && records)
        CK(cudaMemcpy(records, sc->d_trace, (size_t)keep * 3 * sizeof(float4), cudaMemcpyDeviceToHost),
           "cudaMemcpy(query log)");
    return 0;
}

int mt_primary_rays(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int mode, double *out)
{
    int rc = render_args(sc, cam, out, w, h, spp, 0);
    if (rc) return rc;
    if ((rc = set_device(sc))) return rc;
    size_t n = (size_t)w * h * spp;
    DevBuf<double> dR;
    CK(dR.alloc(6 * n), "cudaMalloc");
    int m = mode == MT_MODE_PATHTRACE ? RENDER_PT : RENDER_WHITTED;
    if (sc->opts.precision == MT_PRECISION_FP64) {
        DevCamera<double> dc;
        fill_camera(cam, &dc);
        CK(launch_primary<double>(sc->sd, dc, w, h, spp, m, dR.p, 0), "launch");
    } else {
        DevCamera<float> dc;
        fill_camera(cam, &dc);
        CK(launch_primary<float>(sc->sf, dc, w, h, spp, m, dR.p, 0), "launch");
    }
    CK(cudaDeviceSynchronize(), "primary kernel");
    CK(cudaMemcpy(out, dR.p, 6 * n * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return 0;
}

int mt_scene_param_count(const mt_scene *sc)
{
    if (!sc) return -fail(MT_ERR_NULL, "NULL pointer");
    return param_count((int)sc->h_mats.size());
}

int mt_scene_get_material_params(const mt_scene *sc, double *params, int n)
{
    if (!sc || !params) return fail(MT_ERR_NULL, "NULL pointer");
    const int M = (int)sc->h_mats.size();
    if (n != param_count(M)) return fail(MT_ERR_INVALID, "expected %d parameters, got %d",
                                                        param_count(M), n);
    for (int m = 0; m < M; ++m) {
        const mt_material &mt = sc->h_mats[m];
        double *p = params + kParamsPerMaterialApi * m;
        for (int k = 0; k < 3; ++k) {
            p[k] = mt.albedo[k];
            p[5 + k] = mt.emissive[k];
        }
        p[3] = mt.roughness;
        p[4] = mt.metallic;
    }
    for (int k = 0; k < 3; ++k) params[kParamsPerMaterialApi * M + k] = sc->h_sky.sun_color[k];
    for (int m = 0; m < M; ++m)
        for (int k = 0; k < 3; ++k) params[kParamsPerMaterialApi * M + 3 + 3 * m + k] = sc->h_mats[m].absorption[k];
    return 0;
}

}  // extern "C"

namespace {
template <typename R> int apply_params(mt_scene *sc, DevScene<R> *S)
{
    std::vector<DevMaterial<R>> mats(sc->h_mats.size());
    for (size_t i = 0; i < mats.size(); ++i) fill_material(sc->h_mats[i], sc->d_tex[i], &mats[i]);
    if (!mats.empty())
        CK(cudaMemcpy((void *)S->materials, mats.data(), mats.size() * sizeof(DevMaterial<R>), cudaMemcpyHostToDevice),
           "cudaMemcpy(materials)");
    for (int k = 0; k < 3; ++k) S->sky.sun_color[k] = (R)sc->h_sky.sun_color[k];
    collect_lights(sc, S);  // a material that gains or loses emission changes the light list
    S->version = sc->version;
    return 0;
}
}  // namespace

extern "C" {

int mt_scene_set_material_params(mt_scene *sc, const double *params, int n)
{
    if (!sc || !params) return fail(MT_ERR_NULL, "NULL pointer");
    const int M = (int)sc->h_mats.size();
    if (n != param_count(M)) return fail(MT_ERR_INVALID, "expected %d parameters, got %d",
                                                        param_count(M), n);
    for (int m = 0; m < M; ++m) {
        mt_material &mt = sc->h_mats[m];
        const double *p = params + kParamsPerMaterialApi * m;
        for (int k = 0; k < 3; ++k) {
            mt.albedo[k] = p[k];
            mt.emissive[k] = p[5 + k];
        }
        mt.roughness = p[3];
        mt.metallic = p[4];
    }
    for (int k = 0; k < 3; ++k) sc->h_sky.sun_color[k] = params[kParamsPerMaterialApi * M + k];
    for (int m = 0; m < M; ++m)
        for (int k = 0; k < 3; ++k) sc->h_mats[m].absorption[k] = params[kParamsPerMaterialApi * M + 3 + 3 * m + k];
    sc->version++;
    int rc = set_device(sc);
    if (rc) return rc;
    if (sc->opts.precision == MT_PRECISION_FP64) return apply_params(sc, &sc->sd);
    return apply_params(sc, &sc->sf);
}

int mt_adjoint_backward_device(mt_scene *sc, const mt_camera *cam, int w, int h, int s0, int s1, int depth,
                               const float *dL_dimage_dev, double *grad_dev, int accumulate, void *stream)
{
    int rc = render_args(sc, cam, dL_dimage_dev, w, h, s1 - s0, depth);
    if (rc) return rc;
    if (!grad_dev) return fail(MT_ERR_NULL, "NULL gradient buffer");
    if (s0 < 0) return fail(MT_ERR_COUNTS, "negative first sample");
    const int M = (int)sc->h_mats.size();
    // the replay's gradient terms cover the scene content of the benchmark
    // configurations; these features change paths in ways it does not model
    if (sc->sf.fog.density > 0 || sc->sd.fog.density > 0)
        return fail(MT_ERR_UNSUPPORTED, "the adjoint does not support fog");
    if (sc->sf.fog.shadow_steps > 0 || sc->sd.fog.shadow_steps > 0)
        return fail(MT_ERR_UNSUPPORTED, "the adjoint does not support marched media (fog shadow_steps > 0)");
    if (sc->h_sky.cloud_thickness > 1e-4) return fail(MT_ERR_UNSUPPORTED, "the adjoint does not support volumetric clouds");
    for (int m = 0; m < M; ++m)
        if (sc->h_mats[m].texture_kind != MT_TEXTURE_NONE)
            return fail(MT_ERR_UNSUPPORTED, "the adjoint does not support textures (material %d)", m);
    if (M > kAdjMaxMaterialsApi) return fail(MT_ERR_UNSUPPORTED, "the adjoint supports at most %d materials",
                                             kAdjMaxMaterialsApi);
    if ((rc = set_device(sc))) return rc;
    const int np = param_count(M);
    cudaStream_t s = (cudaStream_t)stream;
    if (!accumulate) CK(cudaMemsetAsync(grad_dev, 0, np * sizeof(double), s), "cudaMemsetAsync(grad)");
    const double scale = 1.0 / (double)(s1 - s0);
    if (sc->opts.precision == MT_PRECISION_FP64) return adjoint_dev<double>(sc, cam, w, h, s0, s1, depth,
                                                                           dL_dimage_dev, scale, grad_dev, np, s);
    return adjoint_dev<float>(sc, cam, w, h, s0, s1, depth, dL_dimage_dev, scale, grad_dev, np, s);
}

int mt_adjoint_backward(mt_scene *sc, const mt_camera *cam, int w, int h, int spp, int depth, const float *dL_dimage,
                        double *grad, int n)
{
    int rc = render_args(sc, cam, dL_dimage, w, h, spp, depth);
    if (rc) return rc;
    if (!grad) return fail(MT_ERR_NULL, "NULL gradient buffer");
    const int np = param_count((int)sc->h_mats.size());
    if (n != np) return fail(MT_ERR_INVALID, "expected %d parameters, got %d", np, n);
    if ((rc = set_device(sc))) return rc;
    DevBuf<float> dA;
    DevBuf<double> dG;
    size_t npix = (size_t)w * h * 3;
    CK(dA.alloc(npix), "cudaMalloc");
    CK(dG.alloc((size_t)np), "cudaMalloc");
    CK(cudaMemcpy(dA.p, dL_dimage, npix * sizeof(float), cudaMemcpyHostToDevice), "cudaMemcpy");
    CK(cudaEventRecord(sc->ev0, 0), "cudaEventRecord");
    if ((rc = mt_adjoint_backward_device(sc, cam, w, h, 0, spp, depth, dA.p, dG.p, 0, nullptr))) return rc;
    CK(cudaEventRecord(sc->ev1, 0), "cudaEventRecord");
    CK(cudaDeviceSynchronize(), "adjoint kernel");
    float ms = 0.f;
    cudaEventElapsedTime(&ms, sc->ev0, sc->ev1);
    sc->stats.kernel_ms = ms;
    CK(cudaMemcpy(grad, dG.p, np * sizeof(double), cudaMemcpyDeviceToHost), "cudaMemcpy");
    return check_err_word(sc);
}

}  // extern "C"

// Accessors for entry points defined in other translation units.
const mt::DevScene<float> *mt_scene_dev_f32(const mt_scene *sc) { return &sc->sf; }
int mt_scene_precision(const mt_scene *sc) { return sc->opts.precision; }
int mt_scene_device(const mt_scene *sc) { return sc->opts.device; }
void mt_set_last_error_text(const char *msg) { g_last_error = msg; }
