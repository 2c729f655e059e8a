// mt_layout.h - device-resident scene layout (shared by host and device code).
//
// HBM layout (all arrays 16-byte aligned, read through the read-only path):
//   nodes      : BVH2 inner nodes, 64 B each = 4 x 16 B vectors holding BOTH
//                child boxes in FP32 (rounded outward from the double boxes):
//                  q0 = (L.min.x, L.max.x, L.min.y, L.max.y)
//                  q1 = (R.min.x, R.max.x, R.min.y, R.max.y)
//                  q2 = (L.min.z, L.max.z, R.min.z, R.max.z)
//                  q3 = (left, right, left_count, right_count) as int32
//                A child index >= 0 is an inner node; < 0 is a leaf whose
//                primitive references start at ~index (count in q3.z / q3.w).
//                One node load tests two children, the GPU form of the
//                reference's bvh_slab_2way (src/bvh.c:495-533).
//   wnodes     : optional wide tree (bvh_width 4 or 8, FP32 path): 128 / 256 B
//                records of W child boxes as SoA (lo_x, hi_x, lo_y, hi_y, lo_z,
//                hi_z, W floats each) and W child codes, collapsed from `nodes`
//                with the same leaf codes (collapse_bvh, mt_bvh.cpp).
//   refs       : leaf-ordered primitive references, int2 {prim_index, code},
//                code = kind << 28 | slot into the per-kind array.
//   tri4       : FP32 triangles, 48 B = (v0.xyz, prim_index) (e1.xyz, smooth)
//                (e2.xyz, pad), precomputed edges (src/geometry.c:229-241).
//   per-kind R : spheres (cx cy cz r), boxes (center half), cylinders
//                (base top r0 r1), FP64 triangles (a e1 e2), smooth vertex
//                normals (na nb nc); indexed by slot.
//   planes     : kept out of the tree and tested linearly, exactly like the
//                reference's plane side list (src/bvh.c:371-402,579-591).
//   prim_info  : per reference prim_index: {code, material}.
//   materials  : array of DevMaterial<R>.
#pragma once

#include <stdint.h>

namespace mt {

enum : int { KIND_SPHERE = 0, KIND_PLANE = 1, KIND_BOX = 2, KIND_TRIANGLE = 3, KIND_CYLINDER = 4 };

static constexpr int kMaxLights = 8;       // SCENE_MAX_EMISSIVE_LIGHTS, src/scene.h:63
static constexpr int kNeeSlots = kMaxLights + 1;  // NEE connections per path vertex: the lights, then the sun
static constexpr int kStackSize = 64;      // traversal stack entries per ray
static constexpr int kWhittedFrames = 16;  // Whitted recursion frames per sample (max depth 14)

// Error bits of the device error word.
enum : unsigned {
    ERR_STACK = 1u,      // traversal stack would overflow
    ERR_QUEUE = 2u,      // wavefront queue overflow
    ERR_WATCHDOG = 4u,   // bounded loop reached its cap
    ERR_WHITTED = 8u,    // Whitted frame stack overflow
    ERR_ABSORB = 16u,    // adjoint: a shadow segment crossed more than two absorbing materials
};

template <typename R> struct DevMaterial {
    R albedo[3];
    R specular[3];
    R shininess;
    R reflectivity;
    R transparency;
    R ior;
    R absorption[3];
    R deep_color[3];
    R metallic;
    R roughness;
    R emissive[3];
    R atmosphere_glow[3];
    int32_t is_water;
    int32_t beer_lambert;
    int32_t pbr;
    int32_t texture_kind;   // TextureKind (src/material.h:33-42)
    R texture_scale;        // as given; <= 0 means 1 (texture_scale_or_default)
    R texture_color_a[3];
    R texture_color_b[3];
    const unsigned char *texture_rgb;  // image texture: width x height sRGB RGB bytes, top row first
    int32_t texture_width;
    int32_t texture_height;
};

template <typename R> struct DevSky {
    R sun_dir[3];
    R sun_color[3];
    R horizon_color[3];
    R zenith_color[3];
    R gradient_gamma;
    R sun_glow_exponent;
    R sun_glow_strength;
    R cloud_height;
    R cloud_scale;
    R cloud_coverage;
    R cloud_softness;
    R cloud_sharpness;
    R sun_radius;
    R cloud_thickness;   // > 1e-4: volumetric slab (src/material.c:493-557)
    R cloud_density;     // <= 0 means 0.08
    int32_t cloud_steps;
    int32_t cloud_octaves;
    uint32_t seed;
};

// FogParams (src/material.h:199-209).
template <typename R> struct DevFog {
    R density;   // 0: no fog
    R color[3];
    R height;
    R height_falloff;
    R inscatter_strength;
    R sun_anisotropy;
    R noise_scale;
    R noise_amount;
    int32_t shadow_steps;  // > 0: marched at bounce 0 with sun shadow rays
    int32_t pad;
};

template <typename R> struct DevLight {
    R center[3];
    R radius;
    R emissive[3];
    int32_t prim;
    int32_t pad;
};

template <typename R> struct DevOcean {
    R center[3];
    R direction[3];
    R amplitude;
    R wavelength;
    R chop;
    R chop_wavelength;
    uint32_t seed;
    int32_t enabled;
};

// Counters updated by the kernels when counting is enabled.
struct DevCounters {
    unsigned long long primary_rays;
    unsigned long long extension_rays;
    unsigned long long shadow_rays;
    unsigned long long node_visits;
    unsigned long long prim_tests;
    unsigned long long tri_tests;
    unsigned long long any_node_visits;   // the same three for any-hit queries
    unsigned long long any_prim_tests;
    unsigned long long any_tri_tests;
    unsigned long long pad;
};

static constexpr int kNoPassTree = -1;
static constexpr int kEmptyPassTree = -2;

template <typename R> struct DevScene {
    const float4 *nodes;
    const float4 *wnodes;    // wide tree (bvh_width 4 or 8; FP32 path), same leaves as `nodes`
    const int2 *refs;
    const float4 *tri4;      // FP32 triangle records (R = float)
    const R *tris;           // FP64 triangle records a, e1, e2 (R = double)
    const R *tri_normals;    // 9 per triangle slot when smooth
    const int *tri_smooth;   // 1 = smooth (FP64 path)
    const R *spheres;
    const R *boxes;
    const R *cyls;
    const R *planes;         // point, axis
    const int *plane_prims;  // prim_index of each plane
    const int *tri_prim;     // prim_index of each triangle slot (FP64 path)
    const R *tri_uv;         // 6 per triangle slot (ua va ub vb uc vc) when some triangle has UVs; NaN first = none
    const int2 *prim_info;   // {code, material} per prim_index
    const DevMaterial<R> *materials;
    int node_count;
    int plane_count;
    int prim_count;
    int material_count;
    int light_count;
    int water_material;
    int has_passthrough;   // some material lets shadow rays through (water, transparency > 0.8)
    // Pass tree: a second BVH over the tree primitives whose material lets
    // shadow rays through, stored after the main tree in `nodes` / `refs`
    // (mixed leaves, absolute indices). Root index; kNoPassTree when it is
    // not built (no pass-through material, or a pass-through plane);
    // kEmptyPassTree when no tree primitive lets shadow rays through.
    int pass_root;
    int has_extras;        // fog, marched media, volumetric clouds or a textured material
    int pbr_only;          // every material PBR, no water / media / atmosphere glow, no extras
    int stack_depth;       // traversal stack entries per thread (dynamic shared memory)
    int bvh_width;         // 2, or 4 / 8 when `wnodes` is present
    int wide_stack_depth;  // stack entries per thread for the wide tree
    int version;           // bumped whenever material / sun parameters change
    R water_level;
    DevOcean<R> ocean;
    DevSky<R> sky;
    DevFog<R> fog;
    DevLight<R> lights[kMaxLights];
    unsigned *err;               // device error word
    DevCounters *counters;       // NULL when counting is off
    // Query log of the wavefront stages (mt_trace_log_enable; NULL when off):
    // 3 float4 per query, appended at trace_count, the first trace_cap kept.
    float4 *trace_rec;
    unsigned *trace_count;
    int trace_cap;
};

template <typename R> struct DevCamera {
    R position[3];
    R lower_left[3];
    R horizontal[3];
    R vertical[3];
    R aperture;
    R focus_distance;
    R dome_radius;
    R anamorphic_squeeze;
};

}  // namespace mt
