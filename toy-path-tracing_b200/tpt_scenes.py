"""Seeded synthetic scenes and ray batches for the benchmark workloads.

The reference ships no benchmark assets; these generators build, from a seed,
the scenes its benchmark configurations describe:

* ``sphere_soup``  — traversal microbenchmark: 4,096 UV spheres of exactly 256
  triangles each (16 longitude segments x 8 latitude bands x 2, pole triangles
  kept even though one of each pair is degenerate), radius U[0.1, 1], centres
  uniform in a 100^3 cube, merged into one mesh of 1,048,576 triangles.
* ``coherent_rays`` — pinhole primary rays, 1024x1024 pixels x 16 stratified
  rays per pixel (2^24 rays).
* ``incoherent_rays`` — origins uniform in the cube, directions uniform on S^2.

Matrices use the column-major glam layout of the reference (`Mat4`).
"""
from __future__ import annotations

import numpy as np

IDENTITY4 = np.eye(4, dtype=np.float32).reshape(16)  # symmetric, so layout-agnostic
IDENTITY3 = np.eye(3, dtype=np.float32).reshape(9)


def identity_instance(mesh: int = 0, material: int = 0) -> dict:
    return {
        "mesh": mesh,
        "material": material,
        "local_to_world": IDENTITY4.copy(),
        "world_to_local": IDENTITY4.copy(),
        "normal_to_world": IDENTITY3.copy(),
    }


def uv_sphere(n_phi: int = 16, n_theta: int = 8):
    """Unit UV sphere: (n_theta+1) x (n_phi+1) vertex grid, 2 triangles per cell."""
    th = np.linspace(0.0, np.pi, n_theta + 1)
    ph = np.linspace(0.0, 2.0 * np.pi, n_phi + 1)
    T, P = np.meshgrid(th, ph, indexing="ij")
    pos = np.stack([np.sin(T) * np.cos(P), np.cos(T), np.sin(T) * np.sin(P)], -1).reshape(-1, 3)
    uv = np.stack([P / (2 * np.pi), T / np.pi], -1).reshape(-1, 2)
    idx = []
    w = n_phi + 1
    for i in range(n_theta):
        for j in range(n_phi):
            a, b, c, d = i * w + j, (i + 1) * w + j, (i + 1) * w + j + 1, i * w + j + 1
            idx += [a, b, c, a, c, d]
    return pos, uv, np.asarray(idx, np.uint32)


def sphere_soup(seed: int = 1, n_spheres: int = 4096, cube: float = 100.0):
    """One merged mesh of n_spheres UV spheres (256 triangles each)."""
    rng = np.random.default_rng(seed)
    radius = rng.uniform(0.1, 1.0, n_spheres)
    centre = rng.uniform(0.0, cube, (n_spheres, 3))
    upos, uuv, uidx = uv_sphere()
    nv = upos.shape[0]
    pos = (upos[None, :, :] * radius[:, None, None] + centre[:, None, :]).astype(np.float32).reshape(-1, 3)
    nrm = np.broadcast_to(upos[None], (n_spheres, nv, 3)).astype(np.float32).reshape(-1, 3)
    uv = np.broadcast_to(uuv[None], (n_spheres, nv, 2)).astype(np.float32).reshape(-1, 2)
    idx = (uidx[None, :].astype(np.int64) + (np.arange(n_spheres, dtype=np.int64) * nv)[:, None]).astype(np.uint32)
    return {"positions": pos, "normals": nrm, "uvs": uv, "indices": idx.reshape(-1)}


def coherent_rays(width: int = 1024, height: int = 1024, per_pixel_side: int = 4, seed: int = 2,
                  eye=(50.0, 50.0, -80.0), look_at=(50.0, 50.0, 50.0), fov_y_deg: float = 60.0):
    """Pinhole primary rays, per_pixel_side^2 stratified jittered rays per pixel; float32 [7, n]."""
    rng = np.random.default_rng(seed)
    eye = np.asarray(eye, np.float64)
    fwd = np.asarray(look_at, np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, [0.0, 1.0, 0.0])
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    tan_h = np.tan(0.5 * np.radians(fov_y_deg))
    s = per_pixel_side
    n = width * height * s * s
    k = np.arange(n, dtype=np.int64)
    pix = k // (s * s)
    sub = k % (s * s)
    px = (pix % width).astype(np.float64) + ((sub % s) + rng.random(n)) / s
    py = (pix // width).astype(np.float64) + ((sub // s) + rng.random(n)) / s
    sx = (2.0 * px / width - 1.0) * (width / height) * tan_h
    sy = (1.0 - 2.0 * py / height) * tan_h
    d = fwd[None, :] + sx[:, None] * right[None, :] + sy[:, None] * up[None, :]
    d /= np.linalg.norm(d, axis=1, keepdims=True)
    rays = np.empty((7, n), np.float32)
    rays[0:3] = eye[:, None]
    rays[3:6] = d.T
    rays[6] = np.inf
    return rays


def incoherent_rays(n: int = 1 << 24, seed: int = 3, cube: float = 100.0):
    """Origins uniform in the cube, directions uniform on the sphere; float32 [7, n]."""
    rng = np.random.default_rng(seed)
    rays = np.empty((7, n), np.float32)
    rays[0:3] = rng.uniform(0.0, cube, (3, n))
    d = rng.standard_normal((3, n))
    d /= np.linalg.norm(d, axis=0, keepdims=True)
    rays[3:6] = d
    rays[6] = np.inf
    return rays


# ---------------------------------------------------------------------------
# Cornell-box scene: 5 wall quads, 2 boxes rotated by U[15, 20] degrees about
# +y (one each way), one 0.25 x 0.25 emissive quad just below the ceiling
# (36 triangles).  Materials: one per wall/box with base colour U[0.1, 0.8]^3,
# either NormalizedLambert (rho = colour) or OpenPBR (base_color = colour,
# roughness 1), plus EmissiveMaterial(colour 1, strength 15).

LAMBERT, EMISSIVE, OPENPBR = 0, 1, 2


def _quad(p0, p1, p2, p3, normal):
    pos = np.array([p0, p1, p2, p3], np.float32)
    nrm = np.tile(np.asarray(normal, np.float32), (4, 1))
    uv = np.array([[0, 0], [1, 0], [1, 1], [0, 1]], np.float32)
    idx = np.array([0, 1, 2, 0, 2, 3], np.uint32)
    return {"positions": pos, "normals": nrm, "uvs": uv, "indices": idx}


def _unit_box():
    """Axis-aligned box [-0.5,0.5]x[0,1]x[-0.5,0.5], 4 vertices per face (24), 12 triangles."""
    faces = [
        ((1, 0, 0), [(0.5, 0, -0.5), (0.5, 1, -0.5), (0.5, 1, 0.5), (0.5, 0, 0.5)]),
        ((-1, 0, 0), [(-0.5, 0, 0.5), (-0.5, 1, 0.5), (-0.5, 1, -0.5), (-0.5, 0, -0.5)]),
        ((0, 1, 0), [(-0.5, 1, -0.5), (-0.5, 1, 0.5), (0.5, 1, 0.5), (0.5, 1, -0.5)]),
        ((0, -1, 0), [(-0.5, 0, 0.5), (-0.5, 0, -0.5), (0.5, 0, -0.5), (0.5, 0, 0.5)]),
        ((0, 0, 1), [(0.5, 0, 0.5), (0.5, 1, 0.5), (-0.5, 1, 0.5), (-0.5, 0, 0.5)]),
        ((0, 0, -1), [(-0.5, 0, -0.5), (-0.5, 1, -0.5), (0.5, 1, -0.5), (0.5, 0, -0.5)]),
    ]
    pos, nrm, uv, idx = [], [], [], []
    for f, (n, corners) in enumerate(faces):
        base = 4 * f
        pos += corners
        nrm += [n] * 4
        uv += [(0, 0), (1, 0), (1, 1), (0, 1)]
        idx += [base, base + 1, base + 2, base, base + 2, base + 3]
    return {"positions": np.array(pos, np.float32), "normals": np.array(nrm, np.float32),
            "uvs": np.array(uv, np.float32), "indices": np.array(idx, np.uint32)}


def instance_matrix(mesh, material, l2w64):
    """Instance record from a float64 4x4 local-to-world matrix (math convention)."""
    w2l64 = np.linalg.inv(l2w64)
    n2w = w2l64[:3, :3].T  # glam: Mat3::from_mat4(world_to_local.transpose())
    return {
        "mesh": mesh,
        "material": material,
        "local_to_world": l2w64.T.astype(np.float32).reshape(16),
        "world_to_local": w2l64.T.astype(np.float32).reshape(16),
        "normal_to_world": n2w.T.astype(np.float32).reshape(9),
    }


def _rot_y(deg):
    a = np.radians(deg)
    m = np.eye(4)
    m[0, 0], m[0, 2], m[2, 0], m[2, 2] = np.cos(a), np.sin(a), -np.sin(a), np.cos(a)
    return m


def _trs(t, deg, s):
    m = np.eye(4)
    m[:3, 3] = t
    sc = np.diag([s[0], s[1], s[2], 1.0])
    return m @ _rot_y(deg) @ sc


def cornell_box(seed: int = 1, material: int = OPENPBR, light_strength: float = 15.0):
    rng = np.random.default_rng(seed)
    L, H = 1.5, 3.0
    meshes = [
        _quad((-L, 0, L), (L, 0, L), (L, 0, -L), (-L, 0, -L), (0, 1, 0)),      # floor
        _quad((-L, H, -L), (L, H, -L), (L, H, L), (-L, H, L), (0, -1, 0)),     # ceiling
        _quad((-L, 0, -L), (L, 0, -L), (L, H, -L), (-L, H, -L), (0, 0, 1)),    # back
        _quad((-L, 0, L), (-L, 0, -L), (-L, H, -L), (-L, H, L), (1, 0, 0)),    # left
        _quad((L, 0, -L), (L, 0, L), (L, H, L), (L, H, -L), (-1, 0, 0)),       # right
        _unit_box(),
        _quad((-0.125, H - 0.01, -0.125), (0.125, H - 0.01, -0.125), (0.125, H - 0.01, 0.125),
              (-0.125, H - 0.01, 0.125), (0, -1, 0)),                           # light
    ]
    colors = rng.uniform(0.1, 0.8, (7, 3)).astype(np.float32)
    materials = []
    for c in colors:
        if material == LAMBERT:
            materials.append({"kind": LAMBERT, "rho": c})
        else:
            materials.append({"kind": OPENPBR, "base_color": c, "base_diffuse_roughness": 1.0,
                              "specular_roughness": 1.0})
    materials.append({"kind": EMISSIVE, "color": np.ones(3, np.float32), "strength": np.float32(light_strength)})
    a1, a2 = rng.uniform(15.0, 20.0, 2)
    instances = [identity_instance(k, k) for k in range(5)]
    instances.append(instance_matrix(5, 5, _trs((-0.55, 0.0, -0.45), a1, (0.9, 1.8, 0.9))))
    instances.append(instance_matrix(5, 6, _trs((0.6, 0.0, 0.5), -a2, (0.9, 0.9, 0.9))))
    instances.append(identity_instance(6, 7))
    camera = {"eye": (0.0, 1.5, 6.8), "look_at": (0.0, 1.5, 0.0), "up": (0.0, 1.0, 0.0),
              "fov_y": float(np.float32(np.radians(38.0))), "exposure": 1.0}
    return {"meshes": meshes, "instances": instances, "materials": materials, "camera": camera,
            "angles": (float(a1), float(a2)), "seed": seed}


def lift_boxes(sc: dict, dy: float = 0.002) -> dict:
    """The Cornell box with its two boxes floating dy above the floor.  Where
    rays reach the inside of a box (glass, cut-outs), a box bottom coplanar
    with the floor is a tie between two instances whose winner, and with alpha
    tests the number of AuxRng draws, a last-bit difference in the ray decides;
    lifted boxes make the geometry free of such ties."""
    a1, a2 = sc["angles"]
    sc["instances"][5] = instance_matrix(5, 5, _trs((-0.55, dy, -0.45), a1, (0.9, 1.8, 0.9)))
    sc["instances"][6] = instance_matrix(5, 6, _trs((0.6, dy, 0.5), -a2, (0.9, 0.9, 0.9)))
    return sc


def cornell_glass(seed: int = 1, thin_walled: bool = False, material: int = OPENPBR, dispersion: float = 0.0):
    """The Cornell box with transmissive boxes: the tall box rough (specular
    roughness 0.25) and the short box smooth, both fully transmissive OpenPBR
    (the short one tinted); thin_walled makes both thin-walled sheets;
    dispersion > 0 gives both glasses that transmission_dispersion_scale
    (Abbe number 20 at scale 1).  The walls keep their diffuse materials
    (OpenPBR, or NormalizedLambert)."""
    sc = lift_boxes(cornell_box(seed, material))
    thin = 1 if thin_walled else 0
    sc["materials"][5] = {"kind": OPENPBR, "base_color": np.array([0.8, 0.8, 0.8], np.float32),
                          "specular_roughness": 0.25, "transmission_weight": 1.0, "geometry_thin_walled": thin}
    sc["materials"][6] = {"kind": OPENPBR, "base_color": np.array([0.6, 0.7, 0.5], np.float32),
                          "specular_roughness": 0.0, "transmission_weight": 1.0,
                          "transmission_color": np.array([0.9, 0.75, 0.6], np.float32),
                          "geometry_thin_walled": thin}
    if dispersion > 0.0:
        for k in (5, 6):
            sc["materials"][k]["transmission_dispersion_scale"] = float(dispersion)
    return sc


def cornell_openpbr_emitter(seed: int = 1, coat: float = 0.0, fuzz: float = 0.0, thin_walled: bool = False):
    """The Cornell box lit by OpenPBR emitters (material/open_pbr.rs:351-391):
    the ceiling quad is an OpenPBR surface with emission_luminance 15 and the
    short box glows with luminance 1.5 through its faces.  `coat` and `fuzz`
    put a tinted coat and a fuzz layer over both emitters (their emission leaves
    through the layers); `thin_walled` makes both emit from either face."""
    sc = cornell_box(seed, OPENPBR)
    thin = 1 if thin_walled else 0
    layers = {"coat_weight": coat, "coat_color": np.array([0.6, 0.75, 0.9], np.float32), "coat_roughness": 0.2,
              "fuzz_weight": fuzz, "fuzz_roughness": 0.6, "geometry_thin_walled": thin}
    sc["materials"][7] = {"kind": OPENPBR, "base_color": np.array([0.7, 0.7, 0.7], np.float32),
                          "specular_roughness": 0.5, "emission_luminance": 15.0,
                          "emission_color": np.array([1.0, 0.9, 0.75], np.float32), **layers}
    sc["materials"][6] = {"kind": OPENPBR, "base_color": np.array([0.5, 0.6, 0.4], np.float32),
                          "specular_roughness": 0.4, "emission_luminance": 1.5,
                          "emission_color": np.array([0.3, 0.8, 1.0], np.float32), **layers}
    return sc


def cornell_lights(seed: int = 1, material: int = LAMBERT, area: bool = True):
    """The Cornell box lit by a point light, a spot light and a directional
    light entering through the open front (plus the ceiling quad when `area`).
    Light conventions are the reference's constructors (light/*.rs): point and
    spot `intensity` is the emitted power, spot angles are radians, the
    directional `direction` is the direction of travel and its `intensity` the
    perpendicular irradiance."""
    sc = cornell_box(seed, material)
    if not area:
        sc["meshes"] = sc["meshes"][:-1]
        sc["materials"] = sc["materials"][:-1]
        sc["instances"] = sc["instances"][:-1]
    sc["point_lights"] = [{"position": (0.7, 2.5, 0.4), "color": (1.0, 0.85, 0.6), "intensity": 30.0}]
    sc["spot_lights"] = [{"position": (-0.6, 2.85, 0.6), "direction": (0.25, -1.0, -0.3),
                          "color": (0.6, 0.8, 1.0), "intensity": 60.0,
                          "total_width": float(np.radians(35.0)), "falloff_start": float(np.radians(20.0))}]
    sc["directional_lights"] = [{"direction": (-0.35, -0.45, -1.0), "color": (1.0, 0.95, 0.9), "intensity": 1.5}]
    return sc


def sky_environment(width: int = 64, height: int = 32, sun=(3, 10), sun_radiance: float = 60.0,
                    scale: float = 1.0, rotate_y: float = 0.0) -> dict:
    """A procedural equirectangular sky (row 0 at +y): a blue gradient above
    the horizon, a dark ground below, and a 2 x 2-texel sun."""
    v = (np.arange(height, dtype=np.float32) + 0.5) / height
    zenith = np.array([0.25, 0.45, 0.9], np.float32)
    horizon = np.array([0.9, 0.85, 0.75], np.float32)
    ground = np.array([0.06, 0.05, 0.04], np.float32)
    t = np.clip(v / 0.5, 0.0, 1.0)[:, None]
    rows = np.where((v < 0.5)[:, None], (1.0 - t) * zenith + t * horizon, ground)
    px = np.repeat(rows[:, None, :], width, axis=1).astype(np.float32)
    i, j = sun
    px[j:j + 2, i:i + 2] = sun_radiance
    return {"pixels": px, "scale": scale, "rotate_y": rotate_y}


def cornell_environment(seed: int = 1, material: int = LAMBERT, area: bool = True, **sky):
    """The Cornell box (open at the front) under the procedural sky, rotated so
    that the sun shines in through the opening."""
    sc = cornell_box(seed, material)
    if not area:
        sc["meshes"] = sc["meshes"][:-1]
        sc["materials"] = sc["materials"][:-1]
        sc["instances"] = sc["instances"][:-1]
    sky.setdefault("rotate_y", 0.35)
    sc["environment"] = sky_environment(**sky)
    return sc


# ---------------------------------------------------------------------------
# Differentiable-render scene: the Cornell box with its five walls split into
# 3 x 4 patches each (60 patches, every patch a 4 x 4 grid of quads) and each
# box split into its sides and its caps (4 patches, faces 2 x 2 quads): 64
# OpenPBR materials, one per patch, ~2k triangles, plus the emissive quad.
# Parameters per material: base_color (3), specular_roughness, base_metalness
# (base_diffuse_roughness 1, the other OpenPBR inputs at their defaults).

N_PATCH_MATERIALS = 64


def _grid_quad(p0, du, dv, n_u, n_v, normal):
    """A planar patch p0 + s*du + t*dv, s, t in [0, 1], as an n_u x n_v grid of quads."""
    p0, du, dv = (np.asarray(a, np.float64) for a in (p0, du, dv))
    s = np.linspace(0.0, 1.0, n_u + 1)
    t = np.linspace(0.0, 1.0, n_v + 1)
    S, T = np.meshgrid(s, t, indexing="ij")
    pos = p0[None, None] + S[..., None] * du + T[..., None] * dv
    uv = np.stack([S, T], -1)
    idx = []
    for i in range(n_u):
        for j in range(n_v):
            a, b, c, d = i * (n_v + 1) + j, (i + 1) * (n_v + 1) + j, (i + 1) * (n_v + 1) + j + 1, i * (n_v + 1) + j + 1
            idx += [a, b, c, a, c, d]
    n = pos.reshape(-1, 3).shape[0]
    return {"positions": pos.reshape(-1, 3).astype(np.float32),
            "normals": np.tile(np.asarray(normal, np.float32), (n, 1)),
            "uvs": uv.reshape(-1, 2).astype(np.float32), "indices": np.asarray(idx, np.uint32)}


def _merge(meshes):
    pos, nrm, uv, idx, base = [], [], [], [], 0
    for m in meshes:
        pos.append(m["positions"])
        nrm.append(m["normals"])
        uv.append(m["uvs"])
        idx.append(m["indices"].astype(np.int64) + base)
        base += m["positions"].shape[0]
    return {"positions": np.concatenate(pos), "normals": np.concatenate(nrm), "uvs": np.concatenate(uv),
            "indices": np.concatenate(idx).astype(np.uint32)}


def patch_params(seed: int = 5, start: bool = False, perturb: float = 0.2):
    """float32 [64, 5]: base_color rgb, specular_roughness, base_metalness.  The
    true parameters are base_color U[0.1, 0.9]^3, roughness U[0.1, 1],
    metalness U[0, 1]; start = true + U[-perturb, perturb], clipped."""
    rng = np.random.default_rng(seed)
    p = np.empty((N_PATCH_MATERIALS, 5), np.float64)
    p[:, 0:3] = rng.uniform(0.1, 0.9, (N_PATCH_MATERIALS, 3))
    p[:, 3] = rng.uniform(0.1, 1.0, N_PATCH_MATERIALS)
    p[:, 4] = rng.uniform(0.0, 1.0, N_PATCH_MATERIALS)
    if start:
        p = p + np.random.default_rng(seed + 1).uniform(-perturb, perturb, p.shape)
        p[:, 0:3] = np.clip(p[:, 0:3], 0.02, 0.98)
        p[:, 3] = np.clip(p[:, 3], 0.05, 1.0)
        p[:, 4] = np.clip(p[:, 4], 0.0, 1.0)
    return p.astype(np.float32)


def patch_material(p) -> dict:
    return {"kind": OPENPBR, "base_color": np.asarray(p[0:3], np.float32), "specular_roughness": float(p[3]),
            "base_metalness": float(p[4]), "base_diffuse_roughness": 1.0}


def cornell_patches(seed: int = 5, params=None, light_strength: float = 15.0):
    """The 64-patch Cornell box; `params` [64, 5] (default: the true ones)."""
    if params is None:
        params = patch_params(seed)
    L, H = 1.5, 3.0
    walls = [  # (corner, u edge, v edge, normal)
        ((-L, 0, L), (2 * L, 0, 0), (0, 0, -2 * L), (0, 1, 0)),      # floor
        ((-L, H, -L), (2 * L, 0, 0), (0, 0, 2 * L), (0, -1, 0)),     # ceiling
        ((-L, 0, -L), (2 * L, 0, 0), (0, H, 0), (0, 0, 1)),          # back
        ((-L, 0, L), (0, 0, -2 * L), (0, H, 0), (1, 0, 0)),          # left
        ((L, 0, -L), (0, 0, 2 * L), (0, H, 0), (-1, 0, 0)),          # right
    ]
    meshes, instances = [], []
    for w, (corner, du, dv, n) in enumerate(walls):
        corner, du, dv = (np.asarray(a, np.float64) for a in (corner, du, dv))
        for i in range(3):
            for j in range(4):
                p0 = corner + du * (i / 3.0) + dv * (j / 4.0)
                meshes.append(_grid_quad(p0, du / 3.0, dv / 4.0, 4, 4, n))
                instances.append(identity_instance(len(meshes) - 1, len(instances)))
    # unit box [-0.5, 0.5] x [0, 1] x [-0.5, 0.5]: sides and caps, faces 2 x 2 quads
    sides = _merge([
        _grid_quad((0.5, 0, -0.5), (0, 0, 1), (0, 1, 0), 2, 2, (1, 0, 0)),
        _grid_quad((-0.5, 0, 0.5), (0, 0, -1), (0, 1, 0), 2, 2, (-1, 0, 0)),
        _grid_quad((0.5, 0, 0.5), (-1, 0, 0), (0, 1, 0), 2, 2, (0, 0, 1)),
        _grid_quad((-0.5, 0, -0.5), (1, 0, 0), (0, 1, 0), 2, 2, (0, 0, -1)),
    ])
    caps = _merge([
        _grid_quad((-0.5, 1, -0.5), (0, 0, 1), (1, 0, 0), 2, 2, (0, 1, 0)),
        _grid_quad((-0.5, 0, 0.5), (0, 0, -1), (1, 0, 0), 2, 2, (0, -1, 0)),
    ])
    rng = np.random.default_rng(seed)
    a1, a2 = rng.uniform(15.0, 20.0, 2)
    meshes += [sides, caps]
    ms, mc = len(meshes) - 2, len(meshes) - 1
    for trs in (_trs((-0.55, 0.0, -0.45), a1, (0.9, 1.8, 0.9)), _trs((0.6, 0.0, 0.5), -a2, (0.9, 0.9, 0.9))):
        instances.append(instance_matrix(ms, len(instances), trs))
        instances.append(instance_matrix(mc, len(instances), trs))
    assert len(instances) == N_PATCH_MATERIALS
    meshes.append(_quad((-0.125, H - 0.01, -0.125), (0.125, H - 0.01, -0.125), (0.125, H - 0.01, 0.125),
                        (-0.125, H - 0.01, 0.125), (0, -1, 0)))
    instances.append(identity_instance(len(meshes) - 1, N_PATCH_MATERIALS))
    materials = [patch_material(p) for p in params]
    materials.append({"kind": EMISSIVE, "color": np.ones(3, np.float32), "strength": np.float32(light_strength)})
    camera = {"eye": (0.0, 1.5, 6.8), "look_at": (0.0, 1.5, 0.0), "up": (0.0, 1.0, 0.0),
              "fov_y": float(np.float32(np.radians(38.0))), "exposure": 1.0}
    return {"meshes": meshes, "instances": instances, "materials": materials, "camera": camera,
            "angles": (float(a1), float(a2)), "seed": seed, "params": np.asarray(params, np.float32)}


def pixel_center_rays(camera: dict, width: int, height: int) -> np.ndarray:
    """Pinhole rays through the pixel centres (7 x width*height planes, pixel =
    y * width + x, row 0 at the top), for coverage queries."""
    eye = np.asarray(camera["eye"], np.float64)
    fwd = np.asarray(camera["look_at"], np.float64) - eye
    fwd /= np.linalg.norm(fwd)
    right = np.cross(fwd, np.asarray(camera["up"], np.float64))
    right /= np.linalg.norm(right)
    up = np.cross(right, fwd)
    t = np.tan(0.5 * camera["fov_y"])
    aspect = width / height
    x = (2.0 * (np.arange(width) + 0.5) / width - 1.0) * t * aspect
    y = (1.0 - 2.0 * (np.arange(height) + 0.5) / height) * t
    d = fwd[None, None, :] + x[None, :, None] * right + y[:, None, None] * up
    d /= np.linalg.norm(d, axis=2, keepdims=True)
    rays = np.zeros((7, width * height), np.float32)
    rays[0:3] = eye[:, None]
    rays[3:6] = d.reshape(-1, 3).T
    rays[6] = np.inf
    return rays


def with_patch_params(scene: dict, params) -> dict:
    """The same scene with its 64 patch materials set to `params` [64, 5]."""
    out = dict(scene)
    out["materials"] = [patch_material(p) for p in params] + [scene["materials"][-1]]
    out["params"] = np.asarray(params, np.float32)
    return out


# ---------------------------------------------------------------------------
# Large instanced scene: an n_side x n_side grid of tessellated spheres, boxes
# and tori on a ground plane, lit by small emissive quads.  Each object is an
# instance of one of three prototype meshes (about tris_per_object triangles
# each) with its own scale and rotation, and one of n_materials OpenPBR
# materials (base_color U[0,1]^3, specular_roughness U[0.05,1], metalness
# Bernoulli(0.3), specular_ior 1.5, coat_weight U[0,1], coat_roughness
# U[0,0.3]).  Emitters: n_emissive_tris / 2 downward-facing quads above the
# grid, each with one of 64 emissive materials of strength log-U[1, 100].
# The defaults give ~2.1M triangles, 10,000 emissive triangles and 256
# materials; smaller settings give the batched-render variants.

def _uv_sphere_mesh(n_theta: int):
    n_phi = 2 * n_theta
    pos, uv, idx = uv_sphere(n_phi, n_theta)
    return {"positions": pos.astype(np.float32), "normals": pos.astype(np.float32), "uvs": uv.astype(np.float32),
            "indices": idx}


def _torus_mesh(n_v: int, R: float = 0.7, r: float = 0.3):
    n_u = 2 * n_v
    u = np.linspace(0.0, 2 * np.pi, n_u + 1)
    v = np.linspace(0.0, 2 * np.pi, n_v + 1)
    U, V = np.meshgrid(u, v, indexing="ij")
    pos = np.stack([(R + r * np.cos(V)) * np.cos(U), r * np.sin(V) + r, (R + r * np.cos(V)) * np.sin(U)], -1)
    nrm = np.stack([np.cos(V) * np.cos(U), np.sin(V), np.cos(V) * np.sin(U)], -1)
    uv = np.stack([U / (2 * np.pi), V / (2 * np.pi)], -1)
    idx = []
    w = n_v + 1
    for i in range(n_u):
        for j in range(n_v):
            a, b, c, d = i * w + j, (i + 1) * w + j, (i + 1) * w + j + 1, i * w + j + 1
            idx += [a, c, b, a, d, c]
    return {"positions": pos.reshape(-1, 3).astype(np.float32), "normals": nrm.reshape(-1, 3).astype(np.float32),
            "uvs": uv.reshape(-1, 2).astype(np.float32), "indices": np.asarray(idx, np.uint32)}


def _box_mesh(k: int):
    faces = []
    for axis in range(3):
        for sgn in (1.0, -1.0):
            n = np.zeros(3)
            n[axis] = sgn
            a, b = [(axis + 1) % 3, (axis + 2) % 3]
            du, dv = np.zeros(3), np.zeros(3)
            du[a], dv[b] = 1.0, 1.0
            if sgn < 0:
                du, dv = dv, du
            corner = 0.5 * n - 0.5 * du - 0.5 * dv + np.array([0.0, 0.5, 0.0])
            faces.append(_grid_quad(corner, du, dv, k, k, n))
    return _merge(faces)


def grid_scene(seed: int = 3, n_side: int = 32, tris_per_object: int = 2048, n_materials: int = 256,
               n_emissive_tris: int = 10000, ground: bool = True):
    rng = np.random.default_rng(seed)
    nt = max(2, int(round(np.sqrt(tris_per_object / 4.0))))
    kb = max(1, int(round(np.sqrt(tris_per_object / 12.0))))
    meshes = [_uv_sphere_mesh(nt), _box_mesh(kb), _torus_mesh(nt)]
    spacing = 3.0
    extent = n_side * spacing
    materials = []
    for _ in range(n_materials):
        materials.append({"kind": OPENPBR, "base_color": rng.uniform(0.0, 1.0, 3).astype(np.float32),
                          "specular_roughness": float(rng.uniform(0.05, 1.0)),
                          "base_metalness": float(rng.random() < 0.3), "specular_ior": 1.5,
                          "coat_weight": float(rng.uniform(0.0, 1.0)), "coat_roughness": float(rng.uniform(0.0, 0.3))})
    n_emit_mats = 64
    emit0 = len(materials)
    for _ in range(n_emit_mats):
        materials.append({"kind": EMISSIVE, "color": np.ones(3, np.float32),
                          "strength": np.float32(np.exp(rng.uniform(np.log(1.0), np.log(100.0))))})
    instances = []
    for i in range(n_side):
        for j in range(n_side):
            proto = int(rng.integers(0, 3))
            s = float(rng.uniform(0.8, 1.4))
            c = np.array([(i + 0.5) * spacing - 0.5 * extent, 0.0, (j + 0.5) * spacing - 0.5 * extent])
            if proto == 0:
                c[1] = s  # unit sphere centred at the origin: rest it on the ground
            instances.append(instance_matrix(proto, int(rng.integers(0, n_materials)),
                                             _trs(c, float(rng.uniform(0, 360)), (s, s, s))))
    # emitters: 0.5 x 0.5 quads facing down, 6 to 10 units above the ground
    meshes.append(_quad((-0.25, 0, -0.25), (0.25, 0, -0.25), (0.25, 0, 0.25), (-0.25, 0, 0.25), (0, -1, 0)))
    quad = len(meshes) - 1
    for _ in range(max(1, n_emissive_tris // 2)):
        c = np.array([rng.uniform(-0.5, 0.5) * extent, rng.uniform(6.0, 10.0), rng.uniform(-0.5, 0.5) * extent])
        instances.append(instance_matrix(quad, emit0 + int(rng.integers(0, n_emit_mats)), _trs(c, 0.0, (1, 1, 1))))
    if ground:
        g = 0.5 * extent + 10.0
        meshes.append(_quad((-g, 0, g), (g, 0, g), (g, 0, -g), (-g, 0, -g), (0, 1, 0)))
        instances.append(identity_instance(len(meshes) - 1, int(rng.integers(0, n_materials))))
    tris = sum(meshes[inst["mesh"]]["indices"].size // 3 for inst in instances)
    camera = {"eye": (0.55 * extent, 0.35 * extent + 4.0, 0.75 * extent), "look_at": (0.0, 0.0, 0.0),
              "up": (0.0, 1.0, 0.0), "fov_y": float(np.float32(np.radians(45.0))), "exposure": 1.0}
    return {"meshes": meshes, "instances": instances, "materials": materials, "camera": camera, "triangles": tris,
            "emissive_triangles": 2 * max(1, n_emissive_tris // 2), "seed": seed}


BATCH_RESOLUTIONS = [(128, 128), (256, 192), (512, 384), (640, 480), (1024, 768)]
BATCH_SPP = [16, 64, 256]


def batch_jobs(seed: int = 4, n_jobs: int = 64, spp_scale: float = 1.0, only=None):
    """The batched-render workload: n_jobs seeded grid_scene variants with
    10k-500k triangles (log-uniform), 4-1024 emissive triangles, 8-64
    materials, a resolution from BATCH_RESOLUTIONS, spp from BATCH_SPP (times
    spp_scale, at least 1) and max depth 8-16.  Returns (scene dicts, job specs).
    only: job indices to build (the others' random draws are still made, so job
    k is the same scene and spec either way); each spec then carries "job": k."""
    rng = np.random.default_rng(seed)
    scenes, specs = [], []
    for k in range(n_jobs):
        tris = float(np.exp(rng.uniform(np.log(1e4), np.log(5e5))))
        n_side = int(rng.integers(4, 17))
        per = max(24, int(tris / (n_side * n_side)))
        emis = int(np.exp(rng.uniform(np.log(4), np.log(1024))))
        n_mat = int(rng.integers(8, 65))
        w, h = BATCH_RESOLUTIONS[int(rng.integers(0, len(BATCH_RESOLUTIONS)))]
        spp = max(1, int(round(BATCH_SPP[int(rng.integers(0, len(BATCH_SPP)))] * spp_scale)))
        depth = int(rng.integers(8, 17))
        if only is not None and k not in only:
            continue
        scenes.append(grid_scene(seed=1000 + k, n_side=n_side, tris_per_object=per, n_materials=n_mat,
                                 n_emissive_tris=emis))
        specs.append({"width": w, "height": h, "spp": spp, "max_depth": depth, "job": k})
    return scenes, specs
