"""Seeded synthetic scenes with the shapes of the benchmark configurations,
plus a writer for the reference's scene text format.

There is no public dataset for this renderer: every workload is generated
here from a fixed seed. Each generator returns a `SceneDesc` whose primitive
order is the reference's prim_index order; `to_scene_text` writes the same
scene in the reference's format (docs/scene_format.md) with every float in
shortest round-trip form, so the reference's parser rebuilds bit-identical
doubles.

    spheres_scene (config "C1"): 320x240, 8 spp, depth 5; ground plane + 64
        spheres (seed 1): 50% Lambert, 25% PBR metal, 25% glass.
    torus_field_scene (config "C2"): 1920x1080, 64 spp, depth 8; 4096
        instances of a 256-triangle torus (1,048,576 triangles, seed 2), PBR
        GGX materials, 8 emissive sphere lights, ground plane, sun and sky.
    batch_workload (config "C3"): 64 mixed scenes (seed 3) of uneven
        triangle count, resolution, spp and depth for one batched launch.
    adjoint_scene (config "C4"): the inverse-rendering scene.
"""
from __future__ import annotations

import math

import numpy as np

from ._capi import MATERIAL_DTYPE, PRIM_DTYPE, PRIM_BOX, PRIM_CYLINDER, PRIM_PLANE, PRIM_SPHERE, PRIM_TRIANGLE
from .api import SceneDesc, default_sky, normalize


def material(albedo=(0.0, 0.0, 0.0), specular=(0.0, 0.0, 0.0), shininess=0.0, reflectivity=0.0, transparency=0.0,
             ior=1.0, absorption=(0.0, 0.0, 0.0), deep_color=(0.0, 0.0, 0.0), metallic=0.0, roughness=0.0,
             emissive=(0.0, 0.0, 0.0), pbr=0, is_water=0, beer_lambert=0, texture_kind=0, texture_scale=1.0,
             texture_color_a=(1.0, 1.0, 1.0), texture_color_b=(0.0, 0.0, 0.0)) -> np.ndarray:
    """One material row; the texture fields default as material_texture_defaults
    does (src/material.h:48-51)."""
    m = np.zeros(1, MATERIAL_DTYPE)
    m["texture_kind"] = texture_kind
    m["texture_scale"] = texture_scale
    m["texture_color_a"] = texture_color_a
    m["texture_color_b"] = texture_color_b
    m["albedo"] = albedo
    m["specular"] = specular
    m["shininess"] = shininess
    m["reflectivity"] = reflectivity
    m["transparency"] = transparency
    m["ior"] = ior
    m["absorption"] = absorption
    m["deep_color"] = deep_color
    m["metallic"] = metallic
    m["roughness"] = roughness
    m["emissive"] = emissive
    m["pbr"] = pbr
    m["is_water"] = is_water
    m["beer_lambert"] = beer_lambert
    return m[0]


def glass_material() -> np.ndarray:
    """`type = glass` preset (sd_glass_preset in the reference's parser)."""
    return material(albedo=(0.02, 0.02, 0.02), specular=(1.0, 1.0, 1.0), shininess=256.0, transparency=1.0, ior=1.5)


def water_material() -> np.ndarray:
    """`type = water` preset (sd_water_preset in the reference's parser)."""
    return material(albedo=(0.05, 0.15, 0.20), specular=(0.9, 0.9, 0.9), shininess=256.0, reflectivity=1.0,
                    transparency=0.85, ior=1.33, is_water=1, absorption=(0.45, 0.12, 0.06),
                    deep_color=(0.02, 0.10, 0.16))


def light_material(color, intensity) -> np.ndarray:
    """Material the reference builds for a `light` block (src/scene.c:1517-1524)."""
    c = tuple(float(x) for x in color)
    return material(albedo=c, emissive=tuple(x * float(intensity) for x in c), roughness=1.0, pbr=1)


def prims_array(n: int) -> np.ndarray:
    return np.zeros(n, PRIM_DTYPE)


def set_sphere(p, center, radius, mat):
    p["kind"] = PRIM_SPHERE
    p["material"] = mat
    p["v"][:3] = center
    p["v"][3] = radius


def set_plane(p, point, normal, mat):
    p["kind"] = PRIM_PLANE
    p["material"] = mat
    p["v"][:3] = point
    p["v"][3:6] = normalize(normal)  # prim_plane normalises the normal once


# ---------------------------------------------------------------------
# C1: ground plane + 64 spheres
# ---------------------------------------------------------------------
def spheres_scene(seed: int = 1, n_spheres: int = 64, metal_reflectivity: float = 0.5) -> SceneDesc:
    rng = np.random.default_rng(seed)
    mats = [material(albedo=(0.5, 0.5, 0.5))]  # ground: Lambert grey
    kinds = np.array([0] * (n_spheres // 2) + [1] * (n_spheres // 4) + [2] * (n_spheres - n_spheres // 2 - n_spheres // 4))
    rng.shuffle(kinds)
    centers = np.stack([rng.uniform(-10, 10, n_spheres), rng.uniform(0.2, 3.0, n_spheres),
                        rng.uniform(-10, 10, n_spheres)], axis=1)
    radii = rng.uniform(0.2, 1.0, n_spheres)
    prims = prims_array(1 + n_spheres)
    set_plane(prims[0], (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0)
    for i in range(n_spheres):
        if kinds[i] == 0:
            mats.append(material(albedo=tuple(rng.uniform(0.1, 0.9, 3))))
        elif kinds[i] == 1:
            mats.append(material(albedo=tuple(rng.uniform(0.5, 0.95, 3)), metallic=1.0,
                                 roughness=float(rng.uniform(0.05, 0.6)), pbr=1, reflectivity=metal_reflectivity))
        else:
            mats.append(glass_material())
        set_sphere(prims[1 + i], centers[i], radii[i], 1 + i)
    sky = default_sky(sun_dir=normalize((0.3, 0.8, 0.5)))
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=sky,
                     camera=dict(eye=(0.0, 2.0, -10.0), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), vfov=45.0))


# ---------------------------------------------------------------------
# C2: 4096 tori (1,048,576 triangles), PBR, 8 emissive sphere lights
# ---------------------------------------------------------------------
def torus_mesh(n_major: int = 16, n_minor: int = 8, R: float = 1.0, r: float = 0.35) -> np.ndarray:
    """Triangles (n_major * n_minor * 2, 3, 3) of a torus around +Y."""
    u = np.arange(n_major) * (2 * math.pi / n_major)
    v = np.arange(n_minor) * (2 * math.pi / n_minor)
    uu, vv = np.meshgrid(u, v, indexing="ij")
    verts = np.stack([(R + r * np.cos(vv)) * np.cos(uu), r * np.sin(vv), (R + r * np.cos(vv)) * np.sin(uu)], axis=-1)
    tris = []
    for i in range(n_major):
        for j in range(n_minor):
            a = verts[i, j]
            b = verts[(i + 1) % n_major, j]
            c = verts[(i + 1) % n_major, (j + 1) % n_minor]
            d = verts[i, (j + 1) % n_minor]
            tris.append((a, b, c))
            tris.append((a, c, d))
    return np.array(tris, np.float64)


def random_rotations(rng, n: int) -> np.ndarray:
    """Uniform random rotation matrices (from unit quaternions)."""
    q = rng.normal(size=(n, 4))
    q /= np.linalg.norm(q, axis=1, keepdims=True)
    w, x, y, z = q.T
    return np.stack([
        np.stack([1 - 2 * (y * y + z * z), 2 * (x * y - z * w), 2 * (x * z + y * w)], -1),
        np.stack([2 * (x * y + z * w), 1 - 2 * (x * x + z * z), 2 * (y * z - x * w)], -1),
        np.stack([2 * (x * z - y * w), 2 * (y * z + x * w), 1 - 2 * (x * x + y * y)], -1),
    ], axis=1)


def torus_field_scene(seed: int = 2, n_instances: int = 4096, n_materials: int = 32, n_lights: int = 8,
                      area: float = 100.0) -> SceneDesc:
    rng = np.random.default_rng(seed)
    mesh = torus_mesh()
    ntri = len(mesh)
    scale = rng.uniform(0.5, 3.0, n_instances)
    rot = random_rotations(rng, n_instances)
    pos = np.stack([rng.uniform(-area / 2, area / 2, n_instances), scale * 0.35 + rng.uniform(0.0, 1.0, n_instances),
                    rng.uniform(-area / 2, area / 2, n_instances)], axis=1)
    mat_of = rng.integers(0, n_materials, n_instances)
    # (inst, tri, vert, xyz) = R @ (s * v) + p
    tv = np.einsum("nij,tkj->ntki", rot, mesh) * scale[:, None, None, None] + pos[:, None, None, :]

    mats = [material(albedo=(0.45, 0.45, 0.42), roughness=0.8, pbr=1)]  # ground: rough PBR dielectric
    for _ in range(n_materials):
        metal = float(rng.uniform() < 0.3)
        mats.append(material(albedo=tuple(rng.uniform(0.2, 0.9, 3)), metallic=metal,
                             roughness=float(rng.uniform(0.02, 0.9)), pbr=1))
    light_pos = np.stack([rng.uniform(-40, 40, n_lights), rng.uniform(2.0, 6.0, n_lights),
                          rng.uniform(-40, 40, n_lights)], axis=1)
    light_int = rng.uniform(5.0, 20.0, n_lights)
    first_light_mat = len(mats)
    for k in range(n_lights):
        mats.append(light_material((1.0, 1.0, 1.0), light_int[k]))

    n = 1 + n_instances * ntri + n_lights
    prims = prims_array(n)
    set_plane(prims[0], (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0)
    tri = prims[1:1 + n_instances * ntri]
    tri["kind"] = PRIM_TRIANGLE
    tri["material"] = np.repeat(1 + mat_of, ntri)
    tri["v"] = tv.reshape(-1, 9)
    for k in range(n_lights):
        set_sphere(prims[1 + n_instances * ntri + k], light_pos[k], 0.5, first_light_mat + k)
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=default_sky(),
                     camera=dict(eye=(0.0, 14.0, -62.0), target=(0.0, 0.0, -5.0), up=(0.0, 1.0, 0.0), vfov=50.0))


# ---------------------------------------------------------------------
# C3: batched uneven workload, 64 scenes (seed 3)
# ---------------------------------------------------------------------
BATCH_RESOLUTIONS = ((256, 256), (512, 512), (768, 432), (1024, 1024))
BATCH_SPP = (16, 64, 256)


def mixed_scene(rng: np.random.Generator, n_triangles: int) -> SceneDesc:
    """A random sphere/triangle mix: ~n_triangles in torus instances (256
    triangles each), 8-40 spheres and a ground plane; Lambert, PBR GGX
    (metal or dielectric), glass and emissive PBR sphere lights."""
    mesh = torus_mesh()
    ntri = len(mesh)
    n_inst = max(2, int(round(n_triangles / ntri)))
    area = 12.0 + 1.6 * math.sqrt(n_inst)
    scale = rng.uniform(0.5, 2.0, n_inst)
    rot = random_rotations(rng, n_inst)
    pos = np.stack([rng.uniform(-area / 2, area / 2, n_inst), scale * 0.35 + rng.uniform(0.0, 1.0, n_inst),
                    rng.uniform(-area / 2, area / 2, n_inst)], axis=1)
    tv = np.einsum("nij,tkj->ntki", rot, mesh) * scale[:, None, None, None] + pos[:, None, None, :]
    mats = [material(albedo=(0.5, 0.5, 0.48))]  # ground: Lambert
    kinds = []
    for _ in range(12):
        k = int(rng.integers(0, 3))
        kinds.append(k)
        if k == 0:
            mats.append(material(albedo=tuple(rng.uniform(0.1, 0.9, 3))))
        elif k == 1:
            mats.append(material(albedo=tuple(rng.uniform(0.2, 0.9, 3)), metallic=float(rng.uniform() < 0.5),
                                 roughness=float(rng.uniform(0.05, 0.8)), pbr=1))
        else:
            mats.append(glass_material())
    n_lights = int(rng.integers(1, 9))
    first_light = len(mats)
    for _ in range(n_lights):
        mats.append(light_material(tuple(rng.uniform(0.6, 1.0, 3)), float(rng.uniform(5.0, 20.0))))
    n_sph = int(rng.integers(8, 41))
    n = 1 + n_inst * ntri + n_sph + n_lights
    prims = prims_array(n)
    set_plane(prims[0], (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), 0)
    tri = prims[1:1 + n_inst * ntri]
    tri["kind"] = PRIM_TRIANGLE
    tri["material"] = np.repeat(rng.integers(1, 13, n_inst), ntri)
    tri["v"] = tv.reshape(-1, 9)
    base = 1 + n_inst * ntri
    for k in range(n_sph):
        r = float(rng.uniform(0.3, 1.2))
        c = (float(rng.uniform(-area / 2, area / 2)), r, float(rng.uniform(-area / 2, area / 2)))
        set_sphere(prims[base + k], c, r, int(rng.integers(1, 13)))
    for k in range(n_lights):
        c = (float(rng.uniform(-area / 3, area / 3)), float(rng.uniform(2.0, 5.0)), float(rng.uniform(-area / 3, area / 3)))
        set_sphere(prims[base + n_sph + k], c, 0.4, first_light + k)
    eye = (0.0, 0.25 * area + 3.0, -0.75 * area - 4.0)
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=default_sky(),
                     camera=dict(eye=eye, target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0), vfov=50.0))


def batch_workload(seed: int = 3, n: int = 64, spp_scale: float = 1.0) -> list:
    """The batched uneven workload: `n` scenes with triangle counts
    log-uniform in [500, 200k], resolution from BATCH_RESOLUTIONS, spp from
    BATCH_SPP (times spp_scale, at least 1), depth 4-10. Returns dicts with
    desc, width, height, spp, depth."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        t = int(round(math.exp(rng.uniform(math.log(500.0), math.log(200_000.0)))))
        w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
        spp = max(1, int(round(BATCH_SPP[int(rng.integers(0, len(BATCH_SPP)))] * spp_scale)))
        depth = int(rng.integers(4, 11))
        out.append(dict(desc=mixed_scene(rng, t), width=w, height=h, spp=spp, depth=depth, triangles=t))
    return out


# ---------------------------------------------------------------------
# C4: inverse-rendering scene, 128 spheres + plane sharing 32 PBR materials
# ---------------------------------------------------------------------
PARAMS_PER_MATERIAL = 8  # albedo rgb, roughness, metallic, emissive rgb


def adjoint_scene(seed: int = 4, n_spheres: int = 128, n_materials: int = 32, n_emissive: int = 4) -> SceneDesc:
    """Spheres and a ground plane sharing `n_materials` PBR materials with the
    hidden true parameters of the inverse-rendering configuration: albedo
    U(0.1, 0.9)^3, roughness U(0.05, 0.8), metallic U(0, 1), emissive 0 except
    for `n_emissive` materials with emissive U(1, 10)^3."""
    rng = np.random.default_rng(seed)
    mats = []
    emissive_ids = set(rng.choice(n_materials, n_emissive, replace=False).tolist())
    for i in range(n_materials):
        em = tuple(rng.uniform(1.0, 10.0, 3)) if i in emissive_ids else (0.0, 0.0, 0.0)
        mats.append(material(albedo=tuple(rng.uniform(0.1, 0.9, 3)), roughness=float(rng.uniform(0.05, 0.8)),
                             metallic=float(rng.uniform(0.0, 1.0)), emissive=em, pbr=1))
    centers = np.stack([rng.uniform(-10, 10, n_spheres), rng.uniform(0.2, 2.5, n_spheres),
                        rng.uniform(-10, 10, n_spheres)], axis=1)
    radii = rng.uniform(0.2, 0.9, n_spheres)
    mat_of = rng.integers(0, n_materials, n_spheres)
    prims = prims_array(1 + n_spheres)
    set_plane(prims[0], (0.0, 0.0, 0.0), (0.0, 1.0, 0.0), int(rng.integers(0, n_materials)))
    for i in range(n_spheres):
        set_sphere(prims[1 + i], centers[i], radii[i], int(mat_of[i]))
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=default_sky(),
                     camera=dict(eye=(0.0, 6.0, -18.0), target=(0.0, 0.5, 0.0), up=(0.0, 1.0, 0.0), vfov=50.0))


def water_scene(seed: int = 6, n_spheres: int = 16) -> SceneDesc:
    """A water surface (two triangles at y = 0, the water preset with
    Beer-Lambert absorption) over a sandy ground at y = -3, spheres above and
    below the surface, one emissive sphere light, sun and sky. Paths refract
    into the water (medium segments) and shadow rays from under water cross
    the surface: both absorption terms of the adjoint are exercised."""
    rng = np.random.default_rng(seed)
    water = water_material()
    mats = [material(albedo=(0.76, 0.70, 0.50)),  # ground: Lambert sand
            water,
            light_material((1.0, 0.9, 0.8), 12.0)]
    for _ in range(6):
        mats.append(material(albedo=tuple(rng.uniform(0.2, 0.9, 3)), roughness=float(rng.uniform(0.1, 0.7)),
                             metallic=float(rng.uniform(0.0, 1.0)), pbr=1))
    S = 12.0
    prims = prims_array(3 + n_spheres + 1)
    set_plane(prims[0], (0.0, -3.0, 0.0), (0.0, 1.0, 0.0), 0)
    for k, tri in enumerate((((-S, 0.0, -S), (S, 0.0, -S), (S, 0.0, S)), ((-S, 0.0, -S), (S, 0.0, S), (-S, 0.0, S)))):
        p = prims[1 + k]
        p["kind"] = PRIM_TRIANGLE
        p["material"] = 1
        p["v"] = np.array(tri, np.float64).ravel()
    for i in range(n_spheres):
        r = float(rng.uniform(0.4, 1.2))
        y = float(rng.uniform(-2.6, 1.5))
        set_sphere(prims[3 + i], (float(rng.uniform(-6, 6)), y, float(rng.uniform(-6, 6))), r, 3 + int(rng.integers(0, 6)))
    set_sphere(prims[3 + n_spheres], (2.0, 4.0, -1.0), 0.6, 2)
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=default_sky(),
                     camera=dict(eye=(0.0, 5.0, -14.0), target=(0.0, -1.5, 0.0), up=(0.0, 1.0, 0.0), vfov=50.0))


# ---------------------------------------------------------------------
# Scene content beyond the benchmark configurations: textures, fog,
# volumetric clouds (the reference's texture_albedo_uv, fog_segment /
# pt_fog_segment and the volumetric sky)
# ---------------------------------------------------------------------
def checker_image(h: int = 6, w: int = 8, seed: int = 9) -> np.ndarray:
    """A small random sRGB image (h, w, 3) uint8 for TEXTURE_IMAGE."""
    return np.random.default_rng(seed).integers(0, 256, (h, w, 3), dtype=np.uint8)


def feature_scene(fog: str | None = None, clouds: bool = False, seed: int = 11) -> SceneDesc:
    """Ground plane (3D checker), spheres with the procedural kinds (stripes,
    earth, moon, noise), UV checker and image textures on a sphere, a box, a
    tapered cylinder, a tilted plane and two UV-mapped triangles, a glass
    sphere and an emissive light, under the default sky.
    fog: None, "analytic" (height fog with noise) or "marched"
    (fog.shadow_steps = 6: sun shadow segments through the medium).
    clouds: a volumetric cloud slab (cloud_thickness 40 at height 60)."""
    rng = np.random.default_rng(seed)
    K = {"checker": 1, "stripes": 2, "earth": 3, "moon": 4, "noise": 5, "image": 6, "uv": 7}
    mats = [material(albedo=(0.8, 0.8, 0.8), texture_kind=K["checker"], texture_scale=1.5,
                     texture_color_a=(0.9, 0.85, 0.8), texture_color_b=(0.2, 0.25, 0.3))]
    kinds = ["stripes", "earth", "moon", "noise", "uv", "image"]
    for k in kinds:
        mats.append(material(albedo=tuple(rng.uniform(0.6, 1.0, 3)), texture_kind=K[k], texture_scale=float(
            rng.uniform(0.6, 2.0)), texture_color_a=tuple(rng.uniform(0.2, 1.0, 3)),
            texture_color_b=tuple(rng.uniform(0.0, 0.6, 3)), roughness=0.6, pbr=int(k in ("earth", "noise"))))
    mats.append(glass_material())
    mats.append(light_material((1.0, 0.9, 0.8), 10.0))
    uv_mat, img_mat = 1 + kinds.index("uv"), 1 + kinds.index("image")
    prims = prims_array(15)
    # the ground lies inside a checker cell (cells of 1.5 from y = 0): on a
    # cell boundary the 3D checker's parity would follow the sign of the hit
    # point's rounding error, in the reference as well
    set_plane(prims[0], (0.0, 0.2, 0.0), (0.0, 1.0, 0.0), 0)
    for i in range(6):
        set_sphere(prims[1 + i], (-6.0 + 2.4 * i, 1.0, 1.0 + 0.8 * (i % 2)), 1.0, 1 + i)
    set_sphere(prims[7], (0.5, 0.7, -2.5), 0.7, 1 + len(kinds))          # glass
    set_sphere(prims[8], (3.0, 5.0, -3.0), 0.5, 2 + len(kinds))          # light
    b = prims[9]
    b["kind"], b["material"] = PRIM_BOX, uv_mat
    b["v"][:6] = (-3.5, 0.8, -2.0, 0.8, 0.8, 0.8)
    c = prims[10]
    c["kind"], c["material"] = PRIM_CYLINDER, img_mat
    c["v"][:8] = (3.5, 0.0, -1.5, 3.2, 2.2, -1.6, 0.9, 0.5)
    for k, (tri, uv) in enumerate(((((-2.0, 0.21, -5.0), (2.0, 0.21, -5.0), (2.0, 3.0, -6.0)), (0, 0, 2, 0, 2, 2)),
                                   (((-2.0, 0.21, -5.0), (2.0, 3.0, -6.0), (-2.0, 3.0, -6.0)), (0, 0, 2, 2, 0, 2)))):
        t = prims[11 + k]
        t["kind"], t["material"], t["has_uv"] = PRIM_TRIANGLE, img_mat, 1
        t["v"] = np.array(tri, np.float64).ravel()
        t["uv"] = uv
    # a tilted plane far below the ground, seen through the glass sphere,
    # carries the UV checker so planes exercise their (u, v) too
    set_plane(prims[13], (0.0, -50.0, 0.0), (0.1, 1.0, 0.05), uv_mat)
    t = prims[14]
    t["kind"], t["material"] = PRIM_TRIANGLE, uv_mat  # barycentric (u, v)
    t["v"] = np.array(((4.0, 0.21, 3.0), (7.0, 0.21, 3.0), (5.5, 2.5, 4.0)), np.float64).ravel()
    sky = default_sky(sun_dir=normalize((0.3, 0.8, 0.5)))
    if clouds:
        sky.update(cloud_thickness=40.0, cloud_height=60.0, cloud_scale=0.02, cloud_coverage=0.45, cloud_steps=16)
    d = SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=sky,
                  camera=dict(eye=(0.0, 4.0, -12.0), target=(0.0, 1.5, 0.0), up=(0.0, 1.0, 0.0), vfov=55.0),
                  images={img_mat: checker_image()})
    if fog == "analytic":
        d.fog_density = 0.04
        d.fog = dict(height=0.5, height_falloff=0.15, noise_scale=0.3, noise_amount=0.4)
    elif fog == "marched":
        d.fog_density = 0.05
        d.fog = dict(height_falloff=0.1, shadow_steps=6)
    return d


# ---------------------------------------------------------------------
# C5: large scene -- water heightfield, trees, spheres (seed 5)
# ---------------------------------------------------------------------
def heightfield_triangles(rng: np.random.Generator, grid: int, half: float) -> np.ndarray:
    """(2 (grid-1)^2, 9) triangles of a grid x grid heightfield over
    [-half, half]^2: a sum of 8 sines with amplitudes U(0.01, 0.1), random
    directions, wavelengths U(2, 30) and phases; normals face +Y."""
    xs = np.linspace(-half, half, grid)
    X, Z = np.meshgrid(xs, xs, indexing="ij")
    Y = np.zeros_like(X)
    for _ in range(8):
        a = rng.uniform(0.01, 0.1)
        th = rng.uniform(0.0, 2 * math.pi)
        k = 2 * math.pi / rng.uniform(2.0, 30.0)
        Y += a * np.sin(k * (math.cos(th) * X + math.sin(th) * Z) + rng.uniform(0.0, 2 * math.pi))
    V = np.stack([X, Y, Z], axis=-1)
    v00, v10, v01, v11 = V[:-1, :-1], V[1:, :-1], V[:-1, 1:], V[1:, 1:]
    t1 = np.concatenate([v00, v01, v11], axis=-1).reshape(-1, 9)
    t2 = np.concatenate([v00, v11, v10], axis=-1).reshape(-1, 9)
    return np.concatenate([t1, t2], axis=0)


def tree_triangles(rng: np.random.Generator, n_trees: int, half: float, generations: int = 7,
                   sides: int = 16) -> np.ndarray:
    """Procedural trees as tapered-cylinder branches (2 * sides triangles
    each, no caps): a trunk, then 3 children per branch per generation with
    length x0.72 and radius x0.62, tilted 25-55 degrees from the parent."""
    base = np.stack([rng.uniform(-half, half, n_trees), np.full(n_trees, -3.0), rng.uniform(-half, half, n_trees)], 1)
    dirs = np.tile([0.0, 1.0, 0.0], (n_trees, 1))
    lens = rng.uniform(6.0, 9.0, n_trees)
    rads = rng.uniform(0.35, 0.55, n_trees)
    segs = []
    for g in range(generations):
        tops = base + dirs * lens[:, None]
        segs.append((base, tops, rads, rads * 0.62))
        if g == generations - 1:
            break
        n = len(base)
        # 3 children: tilt away from the parent direction around a random axis
        up = np.where(np.abs(dirs[:, 1:2]) < 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
        t = np.cross(dirs, up)
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        bvec = np.cross(dirs, t)
        kids_b, kids_d = [], []
        phi0 = rng.uniform(0, 2 * math.pi, n)
        for c in range(3):
            phi = phi0 + c * 2 * math.pi / 3
            tilt = np.radians(rng.uniform(25.0, 55.0, n))
            side = np.cos(phi)[:, None] * t + np.sin(phi)[:, None] * bvec
            nd = np.cos(tilt)[:, None] * dirs + np.sin(tilt)[:, None] * side
            kids_b.append(base + dirs * (lens * rng.uniform(0.6, 1.0, n))[:, None])
            kids_d.append(nd / np.linalg.norm(nd, axis=1, keepdims=True))
        base = np.concatenate(kids_b)
        dirs = np.concatenate(kids_d)
        lens = np.tile(lens * 0.72, 3)
        rads = np.tile(rads * 0.62, 3)
    tris = []
    ang = np.arange(sides + 1) * (2 * math.pi / sides)
    for b0, b1, r0, r1 in segs:
        d = b1 - b0
        d /= np.linalg.norm(d, axis=1, keepdims=True)
        up = np.where(np.abs(d[:, 1:2]) < 0.9, np.array([[0.0, 1.0, 0.0]]), np.array([[1.0, 0.0, 0.0]]))
        t = np.cross(d, up)
        t /= np.linalg.norm(t, axis=1, keepdims=True)
        bb = np.cross(d, t)
        ring = np.cos(ang)[None, :, None] * t[:, None, :] + np.sin(ang)[None, :, None] * bb[:, None, :]
        lo = b0[:, None, :] + ring * r0[:, None, None]
        hi = b1[:, None, :] + ring * r1[:, None, None]
        a0, a1, c0, c1 = lo[:, :-1], lo[:, 1:], hi[:, :-1], hi[:, 1:]
        tris.append(np.concatenate([a0, a1, c1], axis=-1).reshape(-1, 9))
        tris.append(np.concatenate([a0, c1, c0], axis=-1).reshape(-1, 9))
    return np.concatenate(tris, axis=0)


def large_scene(seed: int = 5, grid: int = 2048, n_trees: int = 57, n_spheres: int = 200, n_lights: int = 8,
                half: float = 100.0) -> SceneDesc:
    """Config 5: a grid x grid water heightfield (2 (grid-1)^2 triangles; the
    water preset: IOR 1.33, Beer-Lambert absorption) over a sandy ground
    plane at y = -3, n_trees procedural trees (about 35k triangles each),
    n_spheres glass / metal spheres, n_lights emissive spheres, a soft sun
    (0.5 degree radius). 2048 and 57 give 8.38M + 2.0M triangles."""
    rng = np.random.default_rng(seed)
    water = heightfield_triangles(rng, grid, half)
    tree = tree_triangles(rng, n_trees, 0.8 * half)
    mats = [material(albedo=(0.76, 0.70, 0.50)),          # 0 sand
            water_material(),                              # 1 water
            material(albedo=(0.36, 0.25, 0.16)),           # 2 bark
            glass_material(),                              # 3 glass
            material(albedo=(0.9, 0.8, 0.6), metallic=1.0, roughness=0.2, pbr=1),   # 4 gold-ish metal
            material(albedo=(0.8, 0.8, 0.85), metallic=1.0, roughness=0.05, pbr=1)]  # 5 mirror-like metal
    first_light = len(mats)
    for _ in range(n_lights):
        mats.append(light_material(tuple(rng.uniform(0.7, 1.0, 3)), float(rng.uniform(5.0, 20.0))))
    n = 1 + len(water) + len(tree) + n_spheres + n_lights
    prims = prims_array(n)
    set_plane(prims[0], (0.0, -3.0, 0.0), (0.0, 1.0, 0.0), 0)
    w = prims[1:1 + len(water)]
    w["kind"] = PRIM_TRIANGLE
    w["material"] = 1
    w["v"] = water
    t = prims[1 + len(water):1 + len(water) + len(tree)]
    t["kind"] = PRIM_TRIANGLE
    t["material"] = 2
    t["v"] = tree
    base = 1 + len(water) + len(tree)
    for i in range(n_spheres):
        r = float(rng.uniform(0.5, 2.0))
        c = (float(rng.uniform(-0.8 * half, 0.8 * half)), float(rng.uniform(-2.0, 3.0)),
             float(rng.uniform(-0.8 * half, 0.8 * half)))
        set_sphere(prims[base + i], c, r, 3 + int(rng.integers(0, 3)))
    for k in range(n_lights):
        c = (float(rng.uniform(-0.6 * half, 0.6 * half)), float(rng.uniform(6.0, 12.0)),
             float(rng.uniform(-0.6 * half, 0.6 * half)))
        set_sphere(prims[base + n_spheres + k], c, 0.8, first_light + k)
    return SceneDesc(prims=prims, materials=np.array(mats, MATERIAL_DTYPE), sky=default_sky(sun_radius=0.5),
                     camera=dict(eye=(0.0, 8.0, -0.95 * half), target=(0.0, 0.0, 0.0), up=(0.0, 1.0, 0.0),
                                 vfov=50.0))


def material_params(desc: SceneDesc) -> np.ndarray:
    """Flat parameter vector of the adjoint: per material albedo rgb,
    roughness, metallic, emissive rgb; then the sun radiance rgb; then per
    material the absorption rgb."""
    m = desc.materials
    per = np.concatenate([m["albedo"], m["roughness"][:, None], m["metallic"][:, None], m["emissive"]], axis=1)
    return np.concatenate([per.ravel(), np.asarray(desc.sky["sun_color"], np.float64),
                           np.asarray(m["absorption"], np.float64).ravel()])


def with_params(desc: SceneDesc, params: np.ndarray) -> SceneDesc:
    """A copy of `desc` whose materials and sun radiance take `params`."""
    n = len(desc.materials)
    p = np.asarray(params, np.float64)
    per = p[: PARAMS_PER_MATERIAL * n].reshape(n, PARAMS_PER_MATERIAL)
    mats = desc.materials.copy()
    mats["albedo"] = per[:, 0:3]
    mats["roughness"] = per[:, 3]
    mats["metallic"] = per[:, 4]
    mats["emissive"] = per[:, 5:8]
    base = PARAMS_PER_MATERIAL * n + 3
    if len(p) >= base + 3 * n:
        mats["absorption"] = p[base: base + 3 * n].reshape(n, 3)
    sky = dict(desc.sky)
    sky["sun_color"] = tuple(float(x) for x in p[PARAMS_PER_MATERIAL * n: PARAMS_PER_MATERIAL * n + 3])
    return SceneDesc(prims=desc.prims, materials=mats, sky=sky, water_level=desc.water_level,
                     water_material=desc.water_material, fog_density=desc.fog_density, camera=desc.camera)


# ---------------------------------------------------------------------
# Reference scene text
# ---------------------------------------------------------------------
def _f(x) -> str:
    return repr(float(x))


def _v(v) -> str:
    return " ".join(_f(c) for c in v)


def to_scene_text(desc: SceneDesc) -> str:
    """Write `desc` in the reference's scene format. Primitive and material
    order are preserved, so the reference's prim_index order matches."""
    lines = []
    names = [f"m{i}" for i in range(len(desc.materials))]
    if desc.water_material >= 0:
        lines.append(f"water_level = {_f(desc.water_level)}")
        lines.append(f"water_material = {names[desc.water_material]}")
    if desc.camera:
        c = desc.camera
        lines += ["camera {", f"    eye = {_v(c['eye'])}", f"    target = {_v(c['target'])}", f"    up = {_v(c['up'])}",
                  f"    vfov = {_f(c['vfov'])}", "}"]
    s = desc.sky
    lines.append("sky {")
    for k in ("sun_dir", "sun_color", "horizon_color", "zenith_color"):
        lines.append(f"    {k} = {_v(s[k])}")
    for k in ("gradient_gamma", "sun_glow_exponent", "sun_glow_strength", "cloud_height", "cloud_scale",
              "cloud_coverage", "cloud_softness", "cloud_sharpness"):
        lines.append(f"    {k} = {_f(s[k])}")
    lines.append(f"    cloud_octaves = {int(s['cloud_octaves'])}")
    lines.append(f"    seed = {int(s['seed'])}")
    lines.append(f"    sun_radius = {_f(s['sun_radius'])}")
    lines.append("}")
    for i, m in enumerate(desc.materials):
        lines.append(f"material {names[i]} {{")
        for k in ("albedo", "specular", "absorption", "deep_color", "emissive"):
            lines.append(f"    {k} = {_v(m[k])}")
        for k in ("shininess", "reflectivity", "transparency", "ior", "metallic", "roughness"):
            lines.append(f"    {k} = {_f(m[k])}")
        for k in ("is_water", "beer_lambert", "pbr"):
            lines.append(f"    {k} = {int(m[k])}")
        lines.append("}")
    for p in desc.prims:
        mat = names[p["material"]]
        v = p["v"]
        k = int(p["kind"])
        if k == PRIM_SPHERE:
            lines += ["sphere {", f"    center = {_v(v[:3])}", f"    radius = {_f(v[3])}", f"    material = {mat}", "}"]
        elif k == PRIM_PLANE:
            lines += ["plane {", f"    point = {_v(v[:3])}", f"    normal = {_v(v[3:6])}", f"    material = {mat}", "}"]
        elif k == PRIM_BOX:
            lines += ["box {", f"    center = {_v(v[:3])}", f"    half = {_v(v[3:6])}", f"    material = {mat}", "}"]
        elif k == PRIM_TRIANGLE:
            lines += ["triangle {", f"    a = {_v(v[:3])}", f"    b = {_v(v[3:6])}", f"    c = {_v(v[6:9])}",
                      f"    material = {mat}", "}"]
        elif k == PRIM_CYLINDER:
            lines += ["cylinder {", f"    base = {_v(v[:3])}", f"    top = {_v(v[3:6])}", f"    r_bottom = {_f(v[6])}",
                      f"    r_top = {_f(v[7])}", f"    material = {mat}", "}"]
    return "\n".join(lines) + "\n"
