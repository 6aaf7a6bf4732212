"""Oracle: CPU restatement of the reference path tracer's per-sample hot path.

Test infrastructure only.  tests/, ``__graft_entry__.smoke()`` and the CPU
baseline leg of ``bench.py`` load it as the checker; the shipped library
(``toy-path-tracing_b200``) never links or calls it.

The C++ sources under ``oracle/src`` restate, function by function, the Rust
reference ``crates/renderer/src`` (file:line cited in each source).  This module
is a thin ctypes binding over ``oracle/_build/liboracle.so``.
"""
from __future__ import annotations

import ctypes as C
import os
import subprocess

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB_PATH = os.path.join(_HERE, "_build", "liboracle.so")
_lib = None

NODE_DTYPE = np.dtype(
    [("b", "<f4", (6, 4)), ("children", "<u4", (4,)), ("valid_mask", "<u4"), ("pad", "<u4", (3,))]
)
assert NODE_DTYPE.itemsize == 128


def build() -> str:
    """Compile the oracle library (make in oracle/)."""
    subprocess.run(["make", "-s", "-C", _HERE], check=True)
    return _LIB_PATH


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB_PATH):
            build()
        _lib = C.CDLL(_LIB_PATH)
        _declare(_lib)
    return _lib


def _p(a):
    return a.ctypes.data_as(C.c_void_p) if a is not None else None


def _declare(L):
    vp, u64, u32, i64, f32, i32 = C.c_void_p, C.c_uint64, C.c_uint32, C.c_int64, C.c_float, C.c_int
    sig = {
        "orc_intersect_triangle": (i32, [vp, f32, vp, vp]),
        "orc_qbvh_build": (vp, [vp, u64]),
        "orc_qbvh_free": (None, [vp]),
        "orc_qbvh_num_nodes": (u64, [vp]),
        "orc_qbvh_num_prims": (u64, [vp]),
        "orc_qbvh_copy": (None, [vp, vp, vp]),
        "orc_qbvh_closest_box": (i64, [vp, vp, vp, vp]),
        "orc_geometry_create": (vp, []),
        "orc_geometry_free": (None, [vp]),
        "orc_geometry_add_mesh": (i64, [vp, vp, u64, vp, vp, vp, u64]),
        "orc_geometry_add_instance": (i64, [vp, u32, u32, vp, vp, vp]),
        "orc_geometry_build": (None, [vp]),
        "orc_geometry_mesh_qbvh_nodes": (u64, [vp, u32]),
        "orc_geometry_mesh_qbvh_copy": (None, [vp, u32, vp, vp]),
        "orc_geometry_tlas_nodes": (u64, [vp]),
        "orc_geometry_tlas_copy": (None, [vp, vp, vp]),
        "orc_geometry_query": (None, [vp, vp, u64, i32, vp, vp, vp, vp, vp, i32]),
        "orc_sampler_vertex_randoms": (None, [u32, u32, u32, u32, u32, u32, u32, vp, vp]),
        "orc_sampler_camera": (None, [u32, u32, u32, u32, u32, u32, vp, vp]),
        "orc_sampler_values": (None, [u32, u32, u32, u64, vp, vp, vp, C.c_int]),
        "orc_brute_force_f64": (None, [vp, vp, u64, vp, u64, vp, vp, vp, C.c_int]),
        "orc_thin_film": (None, [f32, f32, f32, vp, vp, f32, vp]),
        "orc_triangle_f64": (None, [vp, vp, vp, vp, u64, vp, vp, C.c_int]),
        "orc_zsobol_sample_index": (u64, [u32, u32, u32, u32, u32, u32, u32]),
        "orc_shuffled_scrambled_sobol": (None, [u32, u32, i32, vp]),
        "orc_uint_to_float": (f32, [u32]),
        "orc_encode_morton_2": (u64, [u32, u32]),
        "orc_laine_karras": (u32, [u32, u32]),
        "orc_reverse_and_shuffle": (u32, [u32, u32]),
        "orc_pcg_hash": (u32, [u32]),
        "orc_pcg_state_transition": (u32, [u32]),
        "orc_pcg_output": (u32, [u32]),
        "orc_mix_bits": (u64, [u64]),
        "orc_camera_ray": (None, [vp, u32, u32, u32, u32, f32, f32, u32, vp]),
        "orc_render_scene_create": (vp, [vp]),
        "orc_render_scene_free": (None, [vp]),
        "orc_render_scene_set_materials": (None, [vp, vp, vp, vp, vp, u32]),
        "orc_render_scene_set_light_tree": (None, [vp, vp, u64, u32]),
        "orc_render_pixels": (None, [vp, vp, u32, u32, u32, u32, u32, u32, u32, vp, i32, u32]),
        "orc_render_samples": (None, [vp, vp, u32, u32, u32, u32, u32, u64, u64, vp, i32, u32]),
        "orc_render_adjoint": (None, [vp, vp, u32, u32, u32, u32, vp, u32, C.c_float, vp, i32, u32]),
        "orc_geometry_step_sequence": (None, [vp, vp, u64, vp, u32, i32]),
        "orc_render_direct_light": (None, [vp, i32, i32, vp, vp, f32, f32, f32, f32, vp, i32]),
        "orc_render_env_escape": (None, [vp, vp, vp, f32, i32, vp]),
        "orc_render_scene_set_lights": (None, [vp, vp, u32, vp, u32, vp, u32]),
        "orc_render_scene_set_environment": (None, [vp, u32, u32, vp, f32, f32]),
        "orc_env_create": (vp, [u32, u32, vp, f32, f32]),
        "orc_env_free": (None, [vp]),
        "orc_env_total_power": (f32, [vp]),
        "orc_env_radiance": (None, [vp, vp, vp]),
        "orc_env_pdf": (f32, [vp, vp, i32]),
        "orc_env_sample": (i32, [vp, f32, f32, i32, vp]),
        "orc_env_direction_to_uv": (None, [vp, vp]),
        "orc_env_uv_to_direction": (None, [f32, f32, vp]),
        "orc_env_pyramid": (u32, [vp, i32, vp, vp, vp]),
        "orc_render_emitted": (None, [vp, i32, i32, vp, vp, i32, i32, vp, vp, vp, f32, i32, vp]),
        "orc_render_material_pdf": (f32, [vp, i32, i32, vp, vp, vp]),
        "orc_render_scene_set_openpbr": (C.c_char_p, [vp, u32, vp]),
        "orc_lut_dielectric_albedo": (None, [f32, vp]),
        "orc_lut_conductor_ec": (None, [vp, vp]),
        "orc_lut_dielectric_ec": (None, [vp, vp]),
        "orc_lut_conductor_lookup_e": (f32, [f32, f32]),
        "orc_openpbr_params_eval": (None, [vp, i32, f32, f32, vp, vp, i32, vp]),
        "orc_openpbr_params_pdf": (f32, [vp, i32, f32, f32, vp, vp]),
        "orc_openpbr_params_sample": (i32, [vp, i32, f32, f32, vp, f32, f32, f32, i32, vp]),
        "orc_openpbr_params_eval_batch": (None, [vp, i32, f32, f32, vp, vp, u64, i32, vp, vp]),
        "orc_eon_eval_batch": (None, [vp, f32, vp, vp, u64, vp, vp]),
        "orc_eon_sample": (i32, [vp, f32, vp, f32, f32, vp]),
        "orc_openpbr_eval": (None, [vp, i32, vp, vp, i32, vp]),
        "orc_openpbr_pdf": (f32, [vp, i32, vp, vp]),
        "orc_openpbr_sample": (i32, [vp, i32, vp, f32, f32, f32, i32, vp]),
        "orc_render_scene_set_opacity": (None, [vp, vp, u32]),
        "orc_render_scene_closest_alpha": (None, [vp, vp, u64, vp, vp, vp, vp]),
        "orc_openpbr_le": (i32, [vp, i32, vp, vp]),
        "orc_openpbr_eval_ex": (None, [vp, i32, vp, vp, vp, i32, vp]),
        "orc_openpbr_pdf_ex": (f32, [vp, i32, vp, vp, vp]),
        "orc_openpbr_sample_ex": (i32, [vp, i32, vp, f32, f32, f32, vp, vp, i32, vp]),
        "orc_openpbr_params_sample_ex": (i32, [vp, i32, f32, f32, vp, f32, f32, f32, vp, i32, vp]),
        "orc_cauchy_ior": (f32, [f32, f32, f32]),
        "orc_sample_dispersion_wavelength": (f32, [f32, vp, vp]),
        "orc_sample_camera_channel_wavelength": (f32, [i32, f32]),
        "orc_camera_wavelength_sampling_pdf": (f32, [f32, vp]),
        "orc_camera_rgb_basis_at": (None, [f32, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


# --------------------------------------------------------------------------
def intersect_triangle(origin, direction, t_max, v0, v1, v2):
    ray = np.array([*origin, *direction], np.float32)
    v = np.array([*v0, *v1, *v2], np.float32)
    out = np.zeros(4, np.float32)
    ok = lib().orc_intersect_triangle(_p(ray), C.c_float(t_max), _p(v), _p(out))
    return (float(out[0]), out[1:].copy()) if ok else None


class BoxQbvh:
    """QBVH over axis-aligned boxes (the reference's qbvh.rs unit-test harness)."""

    def __init__(self, bounds: np.ndarray):
        self.bounds = np.ascontiguousarray(bounds, np.float32).reshape(-1, 6)
        self.h = lib().orc_qbvh_build(_p(self.bounds), self.bounds.shape[0]) if len(self.bounds) else None

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_qbvh_free(self.h)
        except Exception:
            pass

    def arrays(self):
        n = lib().orc_qbvh_num_nodes(self.h)
        m = lib().orc_qbvh_num_prims(self.h)
        nodes = np.zeros(n, NODE_DTYPE)
        prims = np.zeros(m, np.uint32)
        lib().orc_qbvh_copy(self.h, _p(nodes), _p(prims))
        return nodes, prims

    def closest_box(self, origin, direction):
        ray = np.array([*origin, *direction], np.float32)
        t = np.zeros(1, np.float32)
        idx = lib().orc_qbvh_closest_box(self.h, _p(self.bounds), _p(ray), _p(t))
        return (int(idx), float(t[0])) if idx >= 0 else None


class Geometry:
    """Two-level scene geometry (meshes + instances + TLAS), scene/mod.rs."""

    def __init__(self):
        self.h = lib().orc_geometry_create()
        self._tri_counts = []

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_geometry_free(self.h)
        except Exception:
            pass

    def add_mesh(self, positions, indices, normals=None, uvs=None) -> int:
        pos = np.ascontiguousarray(positions, np.float32).reshape(-1, 3)
        idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
        nrm = None if normals is None else np.ascontiguousarray(normals, np.float32).reshape(-1, 3)
        uv = None if uvs is None else np.ascontiguousarray(uvs, np.float32).reshape(-1, 2)
        self._tri_counts.append(idx.size // 3)
        return lib().orc_geometry_add_mesh(self.h, _p(pos), pos.shape[0], _p(nrm), _p(uv), _p(idx), idx.size)

    def add_instance(self, mesh: int, material: int, local_to_world, world_to_local, normal_to_world) -> int:
        l2w = np.ascontiguousarray(local_to_world, np.float32).reshape(16)
        w2l = np.ascontiguousarray(world_to_local, np.float32).reshape(16)
        n2w = np.ascontiguousarray(normal_to_world, np.float32).reshape(9)
        return lib().orc_geometry_add_instance(self.h, mesh, material, _p(l2w), _p(w2l), _p(n2w))

    def build(self):
        lib().orc_geometry_build(self.h)

    def mesh_qbvh(self, mesh: int):
        n = lib().orc_geometry_mesh_qbvh_nodes(self.h, mesh)
        nodes = np.zeros(n, NODE_DTYPE)
        prims = np.zeros(self._mesh_tris(mesh), np.uint32)
        lib().orc_geometry_mesh_qbvh_copy(self.h, mesh, _p(nodes), _p(prims))
        return nodes, prims

    def _mesh_tris(self, mesh):
        return self._tri_counts[mesh]

    def query(self, rays: np.ndarray, mode: int = 0, stats: bool = False, nthreads: int | None = None):
        """rays: float32 [7, n] planes (ox, oy, oz, dx, dy, dz, tmax)."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[1]
        prim = np.empty(n, np.int32)
        inst = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        bary = np.empty((3, n), np.float32)
        st = np.empty((n, 2), np.uint32) if stats else None
        nthreads = nthreads or os.cpu_count() or 1
        lib().orc_geometry_query(self.h, _p(rays), n, mode, _p(prim), _p(inst), _p(t), _p(bary), _p(st), nthreads)
        out = {"prim": prim, "inst": inst, "t": t, "bary": bary}
        if stats:
            out["nodes"] = st[:, 0]
            out["tris"] = st[:, 1]
        return out


def vertex_randoms(px, py, sample, spp, rx, ry, depth):
    out = np.zeros(12, np.float32)
    seed = np.zeros(1, np.uint32)
    lib().orc_sampler_vertex_randoms(px, py, sample, spp, rx, ry, depth, _p(out), _p(seed))
    return out, int(seed[0])


def brute_force_f64(positions, indices, rays, nthreads=None):
    """FP64 brute force (every ray against every triangle, Moller-Trumbore in
    double): nearest triangle (-1 = miss), its t, and the nearest other t."""
    pos = np.ascontiguousarray(positions, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    r = np.ascontiguousarray(rays, np.float32)
    n = r.shape[1]
    prim = np.empty(n, np.int32)
    t1, t2 = np.empty(n, np.float64), np.empty(n, np.float64)
    lib().orc_brute_force_f64(_p(pos), _p(idx), idx.size // 3, _p(r), n, _p(prim), _p(t1), _p(t2),
                              nthreads or os.cpu_count() or 1)
    return prim, t1, t2


def triangle_f64(positions, indices, tri, rays, nthreads=None):
    """FP64 t (+inf on a miss) and smallest barycentric of triangle tri[i] for ray i."""
    pos = np.ascontiguousarray(positions, np.float32)
    idx = np.ascontiguousarray(indices, np.uint32).reshape(-1)
    r = np.ascontiguousarray(rays, np.float32)
    tr = np.ascontiguousarray(tri, np.int32)
    n = r.shape[1]
    t, mb = np.empty(n, np.float64), np.empty(n, np.float64)
    lib().orc_triangle_f64(_p(pos), _p(idx), _p(tr), _p(r), n, _p(t), _p(mb), nthreads or os.cpu_count() or 1)
    return t, mb


def thin_film_dielectric(cos_i, eta_outside, eta_film, eta_base, thickness_nm):
    """eval_thin_film_dielectric (bsdf/thin_film.rs:11-25)."""
    out = np.zeros(3, np.float32)
    lib().orc_thin_film(float(cos_i), float(eta_outside), float(eta_film), _p(_v3([eta_base] * 3)),
                        _p(_v3([0, 0, 0])), float(thickness_nm), _p(out))
    return out


def thin_film_conductor(cos_i, eta_outside, eta_film, n, k, thickness_nm):
    """eval_thin_film_conductor (bsdf/thin_film.rs:27-45)."""
    out = np.zeros(3, np.float32)
    lib().orc_thin_film(float(cos_i), float(eta_outside), float(eta_film), _p(_v3(n)), _p(_v3(k)),
                        float(thickness_nm), _p(out))
    return out


def sampler_values(width, height, spp, queries, nthreads=None):
    """Per query row (px, py, sample, depth): 16 floats (camera sample, then the
    vertex randoms in dimension order) and 2 seeds (initial aux seed, vertex aux
    seed), the layout of tpt_sampler_values_device."""
    q = np.ascontiguousarray(queries, np.uint32).reshape(-1, 4)
    out = np.zeros((q.shape[0], 16), np.float32)
    seeds = np.zeros((q.shape[0], 2), np.uint32)
    lib().orc_sampler_values(width, height, spp, q.shape[0], _p(q), _p(out), _p(seeds),
                             nthreads or os.cpu_count() or 1)
    return out, seeds


def camera_sample(px, py, sample, spp, rx, ry):
    out = np.zeros(2, np.float32)
    seed = np.zeros(1, np.uint32)
    lib().orc_sampler_camera(px, py, sample, spp, rx, ry, _p(out), _p(seed))
    return out, int(seed[0])


def camera_ray(params, rx, ry, px, py, ux, uy, spp):
    p = np.ascontiguousarray(params, np.float32)
    out = np.zeros(20, np.float32)
    lib().orc_camera_ray(_p(p), rx, ry, px, py, C.c_float(ux), C.c_float(uy), spp, _p(out))
    return out


class Environment:
    """EnvironmentLight (light/environment.rs) on the oracle: pixels [H, W, 3]."""

    def __init__(self, pixels, scale=1.0, rotate_y=0.0):
        px = np.ascontiguousarray(pixels, np.float32)
        self.height, self.width = px.shape[:2]
        self.h = lib().orc_env_create(self.width, self.height, _p(px), float(scale), float(rotate_y))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_env_free(self.h)
        except Exception:
            pass

    def total_power(self):
        return lib().orc_env_total_power(self.h)

    def radiance(self, direction):
        d = np.asarray(direction, np.float32)
        out = np.zeros(3, np.float32)
        lib().orc_env_radiance(self.h, _p(d), _p(out))
        return out

    def pdf(self, direction, compensated=False):
        d = np.asarray(direction, np.float32)
        return lib().orc_env_pdf(self.h, _p(d), int(compensated))

    def sample(self, u, v, compensated=False):
        """dict(direction, radiance, uv, pdf) or None."""
        out = np.zeros(9, np.float32)
        if not lib().orc_env_sample(self.h, float(u), float(v), int(compensated), _p(out)):
            return None
        return {"direction": out[:3].copy(), "radiance": out[3:6].copy(), "uv": out[6:8].copy(),
                "pdf": float(out[8])}

    def pyramid(self, compensated=False):
        """(level dims [(w, h)] coarsest first, total weight, leaf weights [ph, pw])."""
        n = lib().orc_env_pyramid(self.h, int(compensated), None, None, None)
        dims = np.zeros(2 * n, np.uint32)
        total = np.zeros(1, np.float32)
        lib().orc_env_pyramid(self.h, int(compensated), _p(dims), _p(total), None)
        pw, ph = int(dims[-2]), int(dims[-1])
        leaf = np.zeros((ph, pw), np.float32)
        lib().orc_env_pyramid(self.h, int(compensated), None, None, _p(leaf))
        return [tuple(int(x) for x in dims[2 * k:2 * k + 2]) for k in range(n)], float(total[0]), leaf


def env_direction_to_uv(direction):
    d = np.asarray(direction, np.float32)
    uv = np.zeros(2, np.float32)
    lib().orc_env_direction_to_uv(_p(d), _p(uv))
    return uv


def env_uv_to_direction(u, v):
    d = np.zeros(3, np.float32)
    lib().orc_env_uv_to_direction(float(u), float(v), _p(d))
    return d


def light_arrays(scene: dict):
    """Point (n x 7), spot (n x 12) and directional (n x 7) light arrays of a
    scene dict's "point_lights", "spot_lights", "directional_lights" lists."""
    pts = np.array([[*l["position"], *l["color"], l["intensity"]] for l in scene.get("point_lights", [])],
                   np.float32).reshape(-1, 7)
    spots = np.array([[*l["position"], *l["direction"], *l["color"], l["intensity"], l["total_width"],
                       l["falloff_start"]] for l in scene.get("spot_lights", [])], np.float32).reshape(-1, 12)
    dirs = np.array([[*l["direction"], *l["color"], l["intensity"]] for l in scene.get("directional_lights", [])],
                    np.float32).reshape(-1, 7)
    return pts, spots, dirs


class RenderScene:
    """Oracle render scene: geometry + materials + lights + a flattened light tree.

    scene: dict with meshes, instances, materials (tpt_scenes layout);
    light_tree: (nodes, root) in the tpt_light_node layout (the tree the
    library built for the same scene)."""

    def __init__(self, scene: dict, light_tree):
        g = Geometry()
        for m in scene["meshes"]:
            g.add_mesh(m["positions"], m["indices"], m.get("normals"), m.get("uvs"))
        for inst in scene["instances"]:
            g.add_instance(inst["mesh"], inst.get("material", 0), inst["local_to_world"], inst["world_to_local"],
                           inst["normal_to_world"])
        g.build()
        self.g = g
        self.h = lib().orc_render_scene_create(g.h)
        mats = scene["materials"]
        self.n_materials = len(mats)
        kinds = np.array([m["kind"] for m in mats], np.uint32)
        rho = np.array([np.asarray(m.get("rho", (0, 0, 0)), np.float32) for m in mats], np.float32)
        col = np.array([np.asarray(m.get("color", (0, 0, 0)), np.float32) for m in mats], np.float32)
        st = np.array([m.get("strength", 0.0) for m in mats], np.float32)
        lib().orc_render_scene_set_materials(self.h, _p(kinds), _p(rho), _p(col), _p(st), len(mats))
        op = np.array([m.get("opacity", 1.0) for m in mats], np.float32)
        lib().orc_render_scene_set_opacity(self.h, _p(op), len(mats))
        for i, m in enumerate(mats):
            if m["kind"] == 2:
                why = lib().orc_render_scene_set_openpbr(self.h, i, _p(pack_openpbr(m)))
                if why:
                    raise ValueError(why.decode())
        pts, spots, dirs = light_arrays(scene)
        env = scene.get("environment")
        self.non_area_lights = len(pts) + len(spots) + len(dirs) + (env is not None)
        lib().orc_render_scene_set_lights(self.h, _p(pts), len(pts), _p(spots), len(spots), _p(dirs), len(dirs))
        if env is not None:
            px = np.ascontiguousarray(env["pixels"], np.float32)
            h, w = px.shape[:2]
            lib().orc_render_scene_set_environment(self.h, w, h, _p(px), float(env.get("scale", 1.0)),
                                                   float(env.get("rotate_y", 0.0)))
        nodes, root = light_tree
        nodes = np.ascontiguousarray(nodes)
        lib().orc_render_scene_set_light_tree(self.h, nodes.ctypes.data if len(nodes) else None, len(nodes), int(root))

    def __del__(self):
        try:
            if getattr(self, "h", None):
                lib().orc_render_scene_free(self.h)
        except Exception:
            pass

    def closest_alpha(self, rays, aux):
        """Scene::closest_hit with the alpha filter: rays (n, 6) origin +
        direction, aux (n,) uint32 AuxRng states (advanced copy returned).
        Returns (instance, triangle, t, aux)."""
        rays = np.ascontiguousarray(rays, np.float32).reshape(-1, 6)
        n = len(rays)
        a = np.ascontiguousarray(aux, np.uint32).copy()
        inst = np.empty(n, np.int32)
        tri = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        lib().orc_render_scene_closest_alpha(self.h, _p(rays), n, _p(a), _p(inst), _p(tri), _p(t))
        return inst, tri, t, a

    @staticmethod
    def _cam(camera):
        return np.array([*camera["eye"], *camera["look_at"], *camera["up"], camera["fov_y"],
                         camera.get("exposure", 1.0)], np.float32)

    def _check_integrator(self, integrator):
        if integrator not in (0, 1, 2, 3):
            raise ValueError("integrator: 0 MIS, 1 BDPT, 2 NEE, 3 PT")

    def render(self, camera, width, height, spp, max_depth, pixels=None, nthreads=None, integrator=0, seed=0):
        """Image rows [p0, p1) of pixels (flattened y*width+x); returns float32 [n, 3].
        integrator: 0 MIS (integrator/mis.rs), 1 BDPT (integrator/bdpt.rs), 2 NEE
        (integrator/nee.rs), 3 PT (integrator/pt.rs).  seed: the sample streams'
        scramble seed (0: the reference's)."""
        self._check_integrator(integrator)
        p0, p1 = pixels if pixels is not None else (0, width * height)
        out = np.empty((p1 - p0, 3), np.float32)
        cam = self._cam(camera)
        lib().orc_render_pixels(self.h, _p(cam), width, height, spp, max_depth, integrator, p0, p1, _p(out),
                                nthreads or os.cpu_count() or 1, seed)
        return out

    def samples(self, camera, width, height, spp, max_depth, first, count, nthreads=None, integrator=0, seed=0):
        self._check_integrator(integrator)
        out = np.empty((count, 3), np.float32)
        cam = self._cam(camera)
        lib().orc_render_samples(self.h, _p(cam), width, height, spp, max_depth, integrator, first, count, _p(out),
                                 nthreads or os.cpu_count() or 1, seed)
        return out

    def adjoint(self, camera, width, height, spp, max_depth, d_image, mask=31, step=1e-3, nthreads=None, seed=0):
        """Path-replay adjoint (MIS): dLoss/d(OpenPBR parameters) per material,
        float64 [n_materials, 7] = base_color rgb, specular_roughness,
        base_metalness, specular_ior, coat_weight; d_image = dLoss/dimage."""
        d = np.ascontiguousarray(d_image, np.float32).reshape(-1)
        assert d.size == width * height * 3
        out = np.zeros((self.n_materials, 7), np.float64)
        cam = self._cam(camera)
        lib().orc_render_adjoint(self.h, _p(cam), width, height, spp, max_depth, _p(d), mask, float(step), _p(out),
                                 nthreads or os.cpu_count() or 1, seed)
        return out

    # -- unit-level queries (reference integrator unit tests) -------------------
    def direct_light(self, inst, tri, bary, incident, u_tree, us, u_category=0.0, non_area_only=False, nee=False):
        """MIS light sampling (mis.rs:145-210); non_area_only: BDPT's non-area
        light sampling (bdpt.rs:396-464); nee: the NEE integrator's (nee.rs:104-150)."""
        out = np.zeros(3, np.float32)
        b = np.asarray(bary, np.float32)
        d = np.asarray(incident, np.float32)
        mode = 2 if nee else (1 if non_area_only else 0)
        lib().orc_render_direct_light(self.h, inst, tri, _p(b), _p(d), float(u_category), float(u_tree),
                                      float(us[0]), float(us[1]), _p(out), mode)
        return out

    def env_escape(self, direction, throughput, bsdf_pdf, delta=False):
        """Environment radiance for an escaping BSDF sample, MIS-weighted (mis.rs:238-258)."""
        out = np.zeros(3, np.float32)
        d = np.asarray(direction, np.float32)
        t = np.asarray(throughput, np.float32)
        lib().orc_render_env_escape(self.h, _p(d), _p(t), float(bsdf_pdf), int(delta), _p(out))
        return out

    def emitted(self, inst, tri, bary, incident, linst, ltri, lbary, lincident, throughput, bsdf_pdf, delta=False):
        out = np.zeros(3, np.float32)
        arrs = [np.asarray(a, np.float32) for a in (bary, incident, lbary, lincident, throughput)]
        lib().orc_render_emitted(self.h, inst, tri, _p(arrs[0]), _p(arrs[1]), linst, ltri, _p(arrs[2]), _p(arrs[3]),
                                 _p(arrs[4]), float(bsdf_pdf), int(delta), _p(out))
        return out

    def material_pdf(self, inst, tri, bary, incident, wi):
        arrs = [np.asarray(a, np.float32) for a in (bary, incident, wi)]
        return lib().orc_render_material_pdf(self.h, inst, tri, _p(arrs[0]), _p(arrs[1]), _p(arrs[2]))


# --------------------------------------------------------------------------
# OpenPBR (bsdf/open_pbr.rs, material/open_pbr.rs, bsdf/directional_albedo.rs)

# OpenPbrMaterial's untextured parameters in the C ABI's tpt_openpbr_desc
# layout, with the defaults of OpenPbrMaterial::new (material/open_pbr.rs:84-145).
OPENPBR_FIELDS = [
    ("base_weight", 1, 1.0), ("base_color", 3, 0.8), ("base_diffuse_roughness", 1, 0.0),
    ("base_metalness", 1, 0.0), ("specular_weight", 1, 1.0), ("specular_color", 3, 1.0),
    ("specular_roughness", 1, 0.3), ("specular_ior", 1, 1.5), ("specular_roughness_anisotropy", 1, 0.0),
    ("transmission_weight", 1, 0.0), ("transmission_color", 3, 1.0), ("subsurface_weight", 1, 0.0),
    ("subsurface_color", 3, 0.8), ("fuzz_weight", 1, 0.0), ("fuzz_color", 3, 1.0), ("fuzz_roughness", 1, 0.5),
    ("coat_weight", 1, 0.0), ("coat_color", 3, 1.0), ("coat_roughness", 1, 0.0),
    ("coat_roughness_anisotropy", 1, 0.0), ("coat_ior", 1, 1.6), ("coat_darkening", 1, 1.0),
    ("thin_film_weight", 1, 0.0), ("thin_film_thickness", 1, 0.5), ("thin_film_ior", 1, 1.4),
    ("emission_luminance", 1, 0.0), ("emission_color", 3, 1.0), ("geometry_opacity", 1, 1.0),
    ("geometry_thin_walled", 1, 0), ("transmission_dispersion_scale", 1, 0.0),
    ("transmission_dispersion_abbe_number", 1, 20.0),
]
OPENPBR_DTYPE = np.dtype([(n, "<u4" if n == "geometry_thin_walled" else "<f4", (k,) if k > 1 else ())
                          for n, k, _ in OPENPBR_FIELDS])
assert OPENPBR_DTYPE.itemsize == 45 * 4

# OpenPbrBsdfParams as the flat float array of orc_openpbr_params_* (order of
# the oracle's OpenPbrParams; front_face last, as 0/1).
OPENPBR_PARAM_FIELDS = [
    ("base_color", 3), ("base", 1), ("specular", 1), ("specular_color", 3), ("specular_alpha_x", 1),
    ("specular_alpha_y", 1), ("specular_eta", 1), ("transmission_eta", 1), ("metalness", 1), ("coat", 1),
    ("coat_color", 3), ("coat_darkening", 3), ("coat_alpha_x", 1), ("coat_alpha_y", 1), ("coat_eta", 1),
    ("fuzz", 1), ("fuzz_color", 3), ("fuzz_roughness", 1), ("transmission", 1), ("transmission_color", 3),
    ("transmission_alpha_x", 1), ("transmission_alpha_y", 1),
    ("diffuse_roughness", 1), ("subsurface", 1), ("subsurface_color", 3), ("thin_walled", 1),
    ("thin_film_weight", 1), ("thin_film_thickness", 1), ("thin_film_ior", 1), ("metal_n", 3), ("metal_k", 3),
    ("front_face", 1), ("transmission_dispersion_abbe", 1), ("path_throughput", 3), ("has_lock", 1),
    ("wavelength_lock", 1),
]


def pack_openpbr(m: dict) -> np.ndarray:
    """One tpt_openpbr_desc record from a material dict (missing keys: defaults)."""
    rec = np.zeros(1, OPENPBR_DTYPE)
    for name, k, default in OPENPBR_FIELDS:
        rec[name] = m.get(name, default if k == 1 else (default,) * 3)
    return rec


def pack_openpbr_params(p: dict) -> np.ndarray:
    """Flat OpenPbrBsdfParams; the transmission alphas default to the specular
    ones (as make_bsdf sets them) and thin_walled to False."""
    p = dict(p)
    p.setdefault("transmission_alpha_x", p["specular_alpha_x"])
    p.setdefault("transmission_alpha_y", p["specular_alpha_y"])
    p.setdefault("thin_walled", 0.0)
    p.setdefault("thin_film_weight", 0.0)
    p.setdefault("thin_film_thickness", 0.0)
    p.setdefault("thin_film_ior", 1.5)
    p.setdefault("metal_n", 0.0)
    p.setdefault("metal_k", 0.0)
    p.setdefault("transmission_dispersion_abbe", 0.0)
    p.setdefault("path_throughput", 1.0)
    lock = p.get("wavelength_lock")
    p["has_lock"] = 0.0 if lock is None else 1.0
    p["wavelength_lock"] = 0.0 if lock is None else float(lock)
    out = []
    for name, k in OPENPBR_PARAM_FIELDS:
        v = p[name]
        out.extend(np.broadcast_to(np.asarray(v, np.float32), (k,)).tolist() if k > 1 else [float(v)])
    return np.asarray(out, np.float32)


def lut_dielectric_albedo(eta: float) -> np.ndarray:
    out = np.empty(64 * 16 * 64 * 16, np.float32)
    lib().orc_lut_dielectric_albedo(float(eta), _p(out))
    return out


def lut_conductor_ec():
    e, e_avg = np.empty(64 * 64, np.float32), np.empty(64, np.float32)
    lib().orc_lut_conductor_ec(_p(e), _p(e_avg))
    return e, e_avg


def lut_dielectric_ec():
    e, e_avg = np.empty(32 * 32 * 32, np.float32), np.empty(32 * 32, np.float32)
    lib().orc_lut_dielectric_ec(_p(e), _p(e_avg))
    return e, e_avg


def _v3(a):
    return np.ascontiguousarray(np.asarray(a, np.float32).reshape(3))


def _unpack_sample(ok, out):
    if not ok:
        return None
    r = {"weight": out[0:3].copy(), "wi": out[3:6].copy(), "pdf": float(out[6]), "pdf_rev": float(out[7]),
         "flags": int(out[8:9].view(np.uint32)[0])}
    if len(out) > 9:
        r["wavelength_lock"] = None if np.isnan(out[9]) else float(out[9])
    return r


def _state(throughput, lock):
    """Path state of a shading vertex: throughput (3) and lock (NaN = None)."""
    t = np.broadcast_to(np.asarray(throughput, np.float32), (3,))
    return np.ascontiguousarray(np.append(t, np.float32(np.nan if lock is None else lock)), np.float32)


class OpenPbrParamsBsdf:
    """OpenPbrBsdf built from explicit OpenPbrBsdfParams (the reference's unit
    tests construct it this way).  luts: "real" (scene tables for spec_eta /
    coat_eta) or "const" (the tests' constant tables)."""

    def __init__(self, params: dict, luts="real", spec_eta=1.5, coat_eta=1.5):
        self.flat = pack_openpbr_params(params)
        self.mode = 0 if luts == "real" else 1
        self.se, self.ce = float(spec_eta), float(coat_eta)

    def eval(self, wo, wi, mode=0):
        out = np.zeros(3, np.float32)
        lib().orc_openpbr_params_eval(_p(self.flat), self.mode, self.se, self.ce, _p(_v3(wo)), _p(_v3(wi)), mode,
                                      _p(out))
        return out

    def pdf(self, wo, wi):
        return lib().orc_openpbr_params_pdf(_p(self.flat), self.mode, self.se, self.ce, _p(_v3(wo)), _p(_v3(wi)))

    def eval_pdf_batch(self, wo, wis, mode=0):
        wis = np.ascontiguousarray(wis, np.float32).reshape(-1, 3)
        f = np.zeros_like(wis)
        pdf = np.zeros(len(wis), np.float32)
        lib().orc_openpbr_params_eval_batch(_p(self.flat), self.mode, self.se, self.ce, _p(_v3(wo)), _p(wis),
                                            len(wis), mode, _p(f), _p(pdf))
        return f, pdf

    def sample(self, wo, u_lobe, u_dir, mode=0, u_extra=None):
        if u_extra is None:
            out = np.zeros(9, np.float32)
            ok = lib().orc_openpbr_params_sample(_p(self.flat), self.mode, self.se, self.ce, _p(_v3(wo)),
                                                 float(u_lobe), float(u_dir[0]), float(u_dir[1]), mode, _p(out))
            return _unpack_sample(ok, out)
        out = np.zeros(10, np.float32)
        ue = np.ascontiguousarray(u_extra, np.float32).reshape(4)
        ok = lib().orc_openpbr_params_sample_ex(_p(self.flat), self.mode, self.se, self.ce, _p(_v3(wo)),
                                                float(u_lobe), float(u_dir[0]), float(u_dir[1]), _p(ue), mode,
                                                _p(out))
        return _unpack_sample(ok, out)


def eon_eval_pdf_batch(rho, roughness, wo, wis):
    """EonBsdf::eval / pdf (bsdf/eon.rs) over directions wis (n x 3)."""
    wis = np.ascontiguousarray(wis, np.float32).reshape(-1, 3)
    f = np.zeros_like(wis)
    pdf = np.zeros(len(wis), np.float32)
    lib().orc_eon_eval_batch(_p(_v3(rho)), float(roughness), _p(_v3(wo)), _p(wis), len(wis), _p(f), _p(pdf))
    return f, pdf


def eon_sample(rho, roughness, wo, us):
    out = np.zeros(9, np.float32)
    ok = lib().orc_eon_sample(_p(_v3(rho)), float(roughness), _p(_v3(wo)), float(us[0]), float(us[1]), _p(out))
    return _unpack_sample(ok, out)


def hemisphere_grid(n_z: int, n_phi: int):
    """Midpoint grid over the upper hemisphere in (z, phi) with its cell
    measure dz * dphi (bsdf/mod.rs:45-63, eon.rs tests)."""
    dz = np.float32(1.0) / np.float32(n_z)
    dphi = np.float32(2.0 * np.pi) / np.float32(n_phi)
    z = (np.arange(n_z, dtype=np.float32) + np.float32(0.5)) * dz
    phi = (np.arange(n_phi, dtype=np.float32) + np.float32(0.5)) * dphi
    r = np.sqrt(np.maximum(np.float32(1.0) - z * z, np.float32(0.0)))
    zz, pp = np.meshgrid(z, phi, indexing="ij")
    rr = np.broadcast_to(r[:, None], zz.shape)
    wis = np.stack([rr * np.cos(pp), rr * np.sin(pp), zz], -1).reshape(-1, 3).astype(np.float32)
    return wis, float(dz) * float(dphi)


class OpenPbrMaterial:
    """OpenPbrMaterial::make_bsdf of an untextured material, queried in the
    shading frame (local wo / wi)."""

    def __init__(self, m: dict):
        self.rec = pack_openpbr(m)

    def eval(self, wo, wi, front=True, mode=0, throughput=1.0, lock=None):
        out = np.zeros(3, np.float32)
        st = _state(throughput, lock)
        lib().orc_openpbr_eval_ex(_p(self.rec), int(front), _p(_v3(wo)), _p(_v3(wi)), _p(st), mode, _p(out))
        return out

    def pdf(self, wo, wi, front=True, throughput=1.0, lock=None):
        st = _state(throughput, lock)
        return lib().orc_openpbr_pdf_ex(_p(self.rec), int(front), _p(_v3(wo)), _p(_v3(wi)), _p(st))

    def le(self, wo, front=True):
        """Emitted radiance toward the local direction wo, or None."""
        out = np.zeros(3, np.float32)
        ok = lib().orc_openpbr_le(_p(self.rec), int(front), _p(_v3(wo)), _p(out))
        return out if ok else None

    def sample(self, wo, u_lobe, u_dir, front=True, mode=0, u_extra=(0.0, 0.0, 0.0, 0.0), throughput=1.0,
               lock=None):
        """One sample; the result carries the wavelength lock it sets (None: none)."""
        out = np.zeros(10, np.float32)
        ue = np.ascontiguousarray(u_extra, np.float32).reshape(4)
        st = _state(throughput, lock)
        ok = lib().orc_openpbr_sample_ex(_p(self.rec), int(front), _p(_v3(wo)), float(u_lobe), float(u_dir[0]),
                                         float(u_dir[1]), _p(ue), _p(st), mode, _p(out))
        return _unpack_sample(ok, out)


# bsdf/dispersion.rs
def cauchy_ior(lambda_nm, n_d, abbe):
    return lib().orc_cauchy_ior(float(lambda_nm), float(n_d), float(abbe))


def sample_dispersion_wavelength(u, throughput=(1.0, 1.0, 1.0)):
    """(lambda, camera basis / pdf) of sample_dispersion_wavelength_weighted."""
    basis = np.zeros(3, np.float32)
    lam = lib().orc_sample_dispersion_wavelength(float(u), _p(_v3(throughput)), _p(basis))
    return lam, basis


def sample_camera_channel_wavelength(channel, u):
    return lib().orc_sample_camera_channel_wavelength(int(channel), float(u))


def camera_wavelength_sampling_pdf(lambda_nm, throughput=(1.0, 1.0, 1.0)):
    return lib().orc_camera_wavelength_sampling_pdf(float(lambda_nm), _p(_v3(throughput)))


def camera_rgb_basis_at(lambda_nm):
    out = np.zeros(3, np.float32)
    lib().orc_camera_rgb_basis_at(float(lambda_nm), _p(out))
    return out
