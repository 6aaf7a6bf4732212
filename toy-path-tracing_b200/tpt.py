"""Python binding of libtpt_cuda.so (the C ABI declared in include/tpt.h).

This is the host-side mirror of the reference crate's scene/integrator API
(`Scene::add_mesh / add_instance / build_qbvh / closest_hit`,
`IntegratorKind::trace_radiance`) used by the tests and the benchmark.  It is a
thin ctypes layer: every call goes through the C ABI, and there is no CPU
fallback — loading fails loudly when the CUDA library is missing.
"""
from __future__ import annotations

import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(_HERE, "_build", "libtpt_cuda.so")
_lib = None

TPT_OK = 0
STATUS_NAMES = {
    0: "TPT_OK",
    1: "TPT_ERR_INVALID_ARG",
    2: "TPT_ERR_OUT_OF_MEMORY",
    3: "TPT_ERR_CUDA",
    4: "TPT_ERR_CAPACITY",
    5: "TPT_ERR_TIMEOUT",
    6: "TPT_ERR_DEVICE_CHECK",
    7: "TPT_ERR_NOT_BUILT",
}
CLOSEST_HIT = 0
ANY_HIT = 1

NODE_DTYPE = np.dtype(
    [("b", "<f4", (6, 4)), ("children", "<u4", (4,)), ("valid_mask", "<u4"), ("pad", "<u4", (3,))]
)


class TptError(RuntimeError):
    def __init__(self, status: int, message: str):
        super().__init__(f"{STATUS_NAMES.get(status, status)}: {message}")
        self.status = status


class QbvhView(C.Structure):
    _fields_ = [
        ("nodes", C.c_void_p),
        ("num_nodes", C.c_uint64),
        ("primitive_indices", C.c_void_p),
        ("num_primitives", C.c_uint64),
    ]


class MeshDesc(C.Structure):
    _fields_ = [
        ("positions", C.c_void_p),
        ("normals", C.c_void_p),
        ("uvs", C.c_void_p),
        ("num_vertices", C.c_uint64),
        ("indices", C.c_void_p),
        ("num_indices", C.c_uint64),
        ("qbvh", QbvhView),
    ]


class InstanceDesc(C.Structure):
    _fields_ = [
        ("mesh_index", C.c_uint32),
        ("material_index", C.c_uint32),
        ("local_to_world", C.c_float * 16),
        ("world_to_local", C.c_float * 16),
        ("normal_to_world", C.c_float * 9),
    ]


# tpt_openpbr_desc: OpenPbrMaterial's untextured parameters with the defaults of
# OpenPbrMaterial::new (material/open_pbr.rs:84-145; base_color defaults to 0.8).
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


class OpenPbrDesc(C.Structure):
    _fields_ = [(n, C.c_uint32 if n == "geometry_thin_walled" else (C.c_float * 3 if k == 3 else C.c_float))
                for n, k, _ in OPENPBR_FIELDS]


assert C.sizeof(OpenPbrDesc) == 45 * 4


def openpbr_desc(m: dict) -> OpenPbrDesc:
    """A tpt_openpbr_desc from a material dict (missing keys: defaults)."""
    d = OpenPbrDesc()
    for name, k, default in OPENPBR_FIELDS:
        v = m.get(name, default)
        if k == 3:
            getattr(d, name)[:] = [float(np.float32(x)) for x in np.broadcast_to(np.asarray(v, np.float32), (3,))]
        elif name == "geometry_thin_walled":
            setattr(d, name, int(v))
        else:
            setattr(d, name, float(np.float32(v)))
    return d


class MaterialDesc(C.Structure):
    _fields_ = [
        ("kind", C.c_uint32),
        ("rho", C.c_float * 3),
        ("color", C.c_float * 3),
        ("strength", C.c_float),
        ("openpbr", C.c_void_p),
        ("has_opacity", C.c_uint32),
        ("opacity", C.c_float),
    ]


LIGHT_NODE_DTYPE = np.dtype(
    [("flux", "<f4"), ("mu", "<f4", (3,)), ("sigma_s2", "<f4"), ("nu", "<f4", (3,)), ("lambda", "<f4"),
     ("radius", "<f4"), ("left", "<u4"), ("right", "<u4"), ("parent", "<u4"), ("leaf_instance", "<u4"),
     ("leaf_triangle", "<u4"), ("area", "<f4")]
)
assert LIGHT_NODE_DTYPE.itemsize == 64


class LightTreeView(C.Structure):
    _fields_ = [("nodes", C.c_void_p), ("num_nodes", C.c_uint64), ("root", C.c_uint32)]


class PointLightDesc(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("color", C.c_float * 3), ("intensity", C.c_float)]


class SpotLightDesc(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("direction", C.c_float * 3), ("color", C.c_float * 3),
                ("intensity", C.c_float), ("total_width", C.c_float), ("falloff_start", C.c_float)]


class DirectionalLightDesc(C.Structure):
    _fields_ = [("direction", C.c_float * 3), ("color", C.c_float * 3), ("intensity", C.c_float)]


LIGHT_LEAF_POINT, LIGHT_LEAF_SPOT = 0xFFFFFFFE, 0xFFFFFFFD  # tree leaf codes (tpt.h)


class EnvironmentDesc(C.Structure):
    _fields_ = [("width", C.c_uint32), ("height", C.c_uint32), ("pixels", C.c_void_p), ("scale", C.c_float),
                ("rotate_y", C.c_float)]


class SceneDesc(C.Structure):
    _fields_ = [
        ("meshes", C.POINTER(MeshDesc)),
        ("num_meshes", C.c_uint32),
        ("instances", C.POINTER(InstanceDesc)),
        ("num_instances", C.c_uint32),
        ("tlas", QbvhView),
        ("materials", C.POINTER(MaterialDesc)),
        ("num_materials", C.c_uint32),
        ("light_tree", LightTreeView),
        ("point_lights", C.POINTER(PointLightDesc)),
        ("num_point_lights", C.c_uint32),
        ("spot_lights", C.POINTER(SpotLightDesc)),
        ("num_spot_lights", C.c_uint32),
        ("directional_lights", C.POINTER(DirectionalLightDesc)),
        ("num_directional_lights", C.c_uint32),
        ("environment", C.POINTER(EnvironmentDesc)),
    ]


def _f3(v):
    return [float(np.float32(x)) for x in np.asarray(v, np.float32).reshape(3)]


def light_descs(lights: dict):
    """C light arrays from a scene dict's "point_lights", "spot_lights" and
    "directional_lights" lists (dicts: position, direction, color, intensity,
    total_width / falloff_start in radians)."""
    pts = lights.get("point_lights", [])
    spots = lights.get("spot_lights", [])
    dirs = lights.get("directional_lights", [])
    pa = (PointLightDesc * max(1, len(pts)))()
    for i, l in enumerate(pts):
        pa[i] = PointLightDesc(tuple(_f3(l["position"])), tuple(_f3(l["color"])), float(np.float32(l["intensity"])))
    sa = (SpotLightDesc * max(1, len(spots)))()
    for i, l in enumerate(spots):
        sa[i] = SpotLightDesc(tuple(_f3(l["position"])), tuple(_f3(l["direction"])), tuple(_f3(l["color"])),
                              float(np.float32(l["intensity"])), float(np.float32(l["total_width"])),
                              float(np.float32(l["falloff_start"])))
    da = (DirectionalLightDesc * max(1, len(dirs)))()
    for i, l in enumerate(dirs):
        da[i] = DirectionalLightDesc(tuple(_f3(l["direction"])), tuple(_f3(l["color"])),
                                     float(np.float32(l["intensity"])))
    return (pa, len(pts)), (sa, len(spots)), (da, len(dirs))


class CameraDesc(C.Structure):
    _fields_ = [("eye", C.c_float * 3), ("look_at", C.c_float * 3), ("up", C.c_float * 3), ("fov_y", C.c_float),
                ("exposure", C.c_float)]


class RenderJob(C.Structure):
    _fields_ = [("scene", C.c_void_p), ("camera", CameraDesc), ("width", C.c_uint32), ("height", C.c_uint32),
                ("spp", C.c_uint32), ("max_depth", C.c_uint32), ("integrator", C.c_uint32),
                ("execution", C.c_uint32), ("seed", C.c_uint32)]


class AdjointDesc(C.Structure):
    _fields_ = [("param_mask", C.c_uint32), ("fd_step", C.c_float), ("first_pixel", C.c_uint32),
                ("num_pixels", C.c_uint32)]


# gradient layout per material (tpt.h TPT_GRAD_*) and parameter-group bits
GRAD_PARAMS = 7
GRAD_NAMES = ["base_color_r", "base_color_g", "base_color_b", "specular_roughness", "base_metalness",
              "specular_ior", "coat_weight"]
GRAD_MASK_BASE_COLOR, GRAD_MASK_ROUGHNESS, GRAD_MASK_METALNESS, GRAD_MASK_IOR, GRAD_MASK_COAT = 1, 2, 4, 8, 16
GRAD_ALL = 31
# render_function's default backward job: the forward job's seed plus this
ADJOINT_SEED_STEP = 0x9E3779B9

class TuneResult(C.Structure):
    _fields_ = [("execution", C.c_uint32), ("wavefront_capacity", C.c_uint32), ("graphs", C.c_uint32),
                ("shade_block", C.c_uint32), ("ms", C.c_float), ("ms_megakernel", C.c_float), ("ms_wavefront_default", C.c_float),
                ("pilot_paths", C.c_uint64), ("stage", C.c_uint32), ("candidates", C.c_uint32),
                ("batched", C.c_uint32)]


INTEGRATOR_MIS = 0
EXEC_AUTO = 2
EXEC_WAVEFRONT = 0
EXEC_MEGAKERNEL = 1

LAMBERT, EMISSIVE, OPENPBR = 0, 1, 2  # tpt_material_kind
INTEGRATOR_MIS, INTEGRATOR_BDPT, INTEGRATOR_NEE, INTEGRATOR_PT = 0, 1, 2, 3  # tpt_integrator


def lib():
    """Load libtpt_cuda.so; raises when the CUDA build is missing (no fallback)."""
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            raise RuntimeError(
                f"{LIB_PATH} is missing: build it with `make -C toy-path-tracing_b200` "
                "(or __graft_entry__.build()); there is no CPU fallback"
            )
        _lib = C.CDLL(LIB_PATH)
        _declare(_lib)
    return _lib


EXPORTED_SYMBOLS = [
    "tpt_context_create",
    "tpt_context_destroy",
    "tpt_context_check",
    "tpt_last_error",
    "tpt_version",
    "tpt_qbvh_build",
    "tpt_qbvh_build_device",
    "tpt_context_set_gpu_build",
    "tpt_qbvh_view_of",
    "tpt_qbvh_free",
    "tpt_scene_upload",
    "tpt_scene_release",
    "tpt_scene_device_bytes",
    "tpt_traverse",
    "tpt_traverse_device",
    "tpt_traverse_stats_device",
    "tpt_traverse_alpha_device",
    "tpt_scene_light_tree",
    "tpt_render",
    "tpt_render_device",
    "tpt_render_samples_device",
    "tpt_render_pixels_device",
    "tpt_light_tree_build",
    "tpt_light_tree_build_threads",
    "tpt_light_tree_view_of",
    "tpt_light_tree_free",
    "tpt_render_device_noalloc",
    "tpt_sampler_values_device",
    "tpt_openpbr_defaults",
    "tpt_lut_dielectric_albedo",
    "tpt_lut_conductor_ec",
    "tpt_lut_dielectric_ec",
    "tpt_bsdf_eval_device",
    "tpt_bsdf_sample_device",
    "tpt_bsdf_eval_path_device",
    "tpt_bsdf_sample_path_device",
    "tpt_scene_set_openpbr",
    "tpt_render_batch_device",
    "tpt_context_set_wavefront_capacity",
    "tpt_context_wavefront_capacity",
    "tpt_context_set_graphs",
    "tpt_context_set_render_stats",
    "tpt_context_set_shade_block",
    "tpt_autotune",
    "tpt_adjoint_device",
    "tpt_adjoint",
]


def _declare(L):
    vp, u64, i32, cp = C.c_void_p, C.c_uint64, C.c_int, C.c_char_p
    sig = {
        "tpt_context_create": (i32, [i32, C.POINTER(vp)]),
        "tpt_context_destroy": (i32, [vp]),
        "tpt_context_check": (i32, [vp, vp]),
        "tpt_last_error": (cp, [vp]),
        "tpt_version": (cp, []),
        "tpt_qbvh_build": (i32, [vp, u64, i32, C.POINTER(vp)]),
        "tpt_qbvh_build_device": (i32, [vp, vp, u64, vp, C.POINTER(vp)]),
        "tpt_context_set_gpu_build": (i32, [vp, i32]),
        "tpt_qbvh_view_of": (i32, [vp, C.POINTER(QbvhView)]),
        "tpt_qbvh_free": (i32, [vp]),
        "tpt_scene_upload": (i32, [vp, C.POINTER(SceneDesc), C.POINTER(vp)]),
        "tpt_scene_release": (i32, [vp]),
        "tpt_scene_device_bytes": (i32, [vp, C.POINTER(u64)]),
        "tpt_traverse": (i32, [vp, vp, vp, u64, i32, vp, vp, vp, vp]),
        "tpt_traverse_device": (i32, [vp, vp, vp, u64, i32, vp, vp, vp, vp, vp]),
        "tpt_traverse_stats_device": (i32, [vp, vp, vp, u64, i32, vp, vp, vp, vp, vp]),
        "tpt_traverse_alpha_device": (i32, [vp, vp, vp, u64, vp, vp, vp, vp, vp, vp]),
        "tpt_scene_light_tree": (i32, [vp, C.POINTER(LightTreeView)]),
        "tpt_render": (i32, [vp, C.POINTER(RenderJob), i32, C.POINTER(C.c_void_p)]),
        "tpt_render_device": (i32, [vp, C.POINTER(RenderJob), vp, vp]),
        "tpt_render_samples_device": (i32, [vp, C.POINTER(RenderJob), u64, u64, vp, vp]),
        "tpt_render_pixels_device": (i32, [vp, C.POINTER(RenderJob), u64, u64, vp, vp]),
        "tpt_light_tree_build": (i32, [C.POINTER(SceneDesc), C.POINTER(vp)]),
        "tpt_light_tree_build_threads": (i32, [C.POINTER(SceneDesc), C.c_int, C.POINTER(vp)]),
        "tpt_light_tree_view_of": (i32, [vp, C.POINTER(LightTreeView)]),
        "tpt_light_tree_free": (i32, [vp]),
        "tpt_render_device_noalloc": (i32, [vp, C.POINTER(RenderJob), vp, vp]),
        "tpt_sampler_values_device": (i32, [vp, C.c_uint32, C.c_uint32, C.c_uint32, u64, vp, vp, vp, vp]),
        "tpt_openpbr_defaults": (None, [C.POINTER(OpenPbrDesc)]),
        "tpt_lut_dielectric_albedo": (i32, [vp, C.c_float, vp]),
        "tpt_lut_conductor_ec": (i32, [vp, vp, vp]),
        "tpt_lut_dielectric_ec": (i32, [vp, vp, vp]),
        "tpt_bsdf_eval_device": (i32, [vp, vp, C.c_uint32, u64, vp, vp, vp, C.c_uint32, vp, vp, vp]),
        "tpt_bsdf_sample_device": (i32, [vp, vp, C.c_uint32, u64, vp, vp, vp, C.c_uint32, vp, vp]),
        "tpt_bsdf_eval_path_device": (i32, [vp, vp, C.c_uint32, u64, vp, vp, vp, vp, C.c_uint32, vp, vp, vp]),
        "tpt_bsdf_sample_path_device": (i32, [vp, vp, C.c_uint32, u64, vp, vp, vp, vp, C.c_uint32, vp, vp]),
        "tpt_scene_set_openpbr": (i32, [vp, vp, C.c_uint32, vp, vp, vp]),
        "tpt_render_batch_device": (i32, [vp, vp, i32, vp, vp]),
        "tpt_context_set_wavefront_capacity": (i32, [vp, C.c_uint32]),
        "tpt_context_wavefront_capacity": (C.c_uint32, [vp]),
        "tpt_context_set_graphs": (i32, [vp, i32]),
        "tpt_context_set_render_stats": (i32, [vp, vp]),
        "tpt_context_set_shade_block": (i32, [vp, C.c_uint32]),
        "tpt_autotune": (i32, [vp, vp, i32, C.POINTER(TuneResult)]),
        "tpt_adjoint_device": (i32, [vp, C.POINTER(RenderJob), C.POINTER(AdjointDesc), vp, vp, vp]),
        "tpt_adjoint": (i32, [vp, C.POINTER(RenderJob), C.POINTER(AdjointDesc), vp, vp]),
    }
    for name, (res, args) in sig.items():
        fn = getattr(L, name)
        fn.restype = res
        fn.argtypes = args


def _p(a):
    return None if a is None else a.ctypes.data_as(C.c_void_p)


def _stream(handle):
    """cudaStream_t for the C ABI: None = the context's own stream; the legacy
    default stream (handle 0, torch's default) maps to cudaStreamLegacy."""
    if handle is None:
        return None
    return C.c_void_p(1 if handle == 0 else handle)


def _check(status: int, ctx=None):
    if status != TPT_OK:
        msg = lib().tpt_last_error(ctx.h if ctx is not None else None)
        raise TptError(status, (msg or b"").decode())


# --------------------------------------------------------------------------
class Context:
    """`tpt_context`: one CUDA device + stream."""

    def __init__(self, device: int = 0):
        h = C.c_void_p()
        _check(lib().tpt_context_create(device, C.byref(h)))
        self.h = h

    def close(self):
        if getattr(self, "h", None):
            lib().tpt_context_destroy(self.h)
            self.h = None

    def check(self, stream=None):
        """`tpt_context_check`: waits for `stream` and raises TptError when a
        device-side check of work queued by `*_device` calls fired."""
        _check(lib().tpt_context_check(self.h, _stream(stream)), self)

    @property
    def wavefront_capacity(self) -> int:
        return int(lib().tpt_context_wavefront_capacity(self.h))

    @wavefront_capacity.setter
    def wavefront_capacity(self, slots: int):
        _check(lib().tpt_context_set_wavefront_capacity(self.h, int(slots)), self)

    def set_gpu_build(self, enable: bool):
        """`tpt_context_set_gpu_build`: scene uploads build missing QBVHs on the GPU."""
        _check(lib().tpt_context_set_gpu_build(self.h, int(bool(enable))), self)

    def set_graphs(self, enable: bool):
        """`tpt_context_set_graphs`: replay wavefront bounces from CUDA graphs."""
        _check(lib().tpt_context_set_graphs(self.h, int(bool(enable))), self)

    def set_render_stats(self, counters_ptr):
        """`tpt_context_set_render_stats`: device pointer of 8 uint64 counters
        (rays, node tests, triangle tests, hits of path rays, then of shadow
        rays) that wavefront renders add to; None turns counting off."""
        _check(lib().tpt_context_set_render_stats(self.h, None if counters_ptr is None
                                                  else C.c_void_p(counters_ptr)), self)

    def autotune(self, jobs) -> dict:
        """`tpt_autotune`: times candidate settings on a pilot of `jobs` and applies the fastest."""
        arr = (RenderJob * len(jobs))(*jobs)
        r = TuneResult()
        _check(lib().tpt_autotune(self.h, arr, len(jobs), C.byref(r)), self)
        return {k: getattr(r, k) for k, _ in TuneResult._fields_}

    def sampler_values(self, width: int, height: int, spp: int, queries: np.ndarray):
        """`tpt_sampler_values_device`: the device's sample values for query rows
        (px, py, sample, depth) -> (n x 16 floats, n x 2 seeds) on the host."""
        import torch

        q = torch.from_numpy(np.ascontiguousarray(queries, np.uint32).reshape(-1, 4).view(np.int32)).cuda()
        n = q.shape[0]
        out = torch.empty((n, 16), dtype=torch.float32, device="cuda")
        seeds = torch.empty((n, 2), dtype=torch.int32, device="cuda")
        _check(lib().tpt_sampler_values_device(self.h, width, height, spp, n, C.c_void_p(q.data_ptr()),
                                               C.c_void_p(out.data_ptr()), C.c_void_p(seeds.data_ptr()), None),
               self)
        self.check()
        return out.cpu().numpy(), seeds.cpu().numpy().view(np.uint32)

    def set_shade_block(self, threads: int):
        """`tpt_context_set_shade_block`: 128 or 256 threads per shade block."""
        _check(lib().tpt_context_set_shade_block(self.h, int(threads)), self)

    def render_batch_device(self, jobs, out_ptrs, stream=None):
        """`tpt_render_batch_device`: jobs (RenderJob list) into device images."""
        arr = (RenderJob * max(1, len(jobs)))(*jobs)
        outs = (C.c_void_p * max(1, len(jobs)))(*[C.c_void_p(p) for p in out_ptrs])
        _check(lib().tpt_render_batch_device(self.h, arr, len(jobs), outs, _stream(stream)), self)

    # -- OpenPBR tables (built on the GPU on first use) -------------------------
    def lut_dielectric_albedo(self, eta: float) -> np.ndarray:
        out = np.empty(64 * 16 * 64 * 16, np.float32)
        _check(lib().tpt_lut_dielectric_albedo(self.h, float(eta), _p(out)), self)
        return out

    def lut_conductor_ec(self):
        e, e_avg = np.empty(64 * 64, np.float32), np.empty(64, np.float32)
        _check(lib().tpt_lut_conductor_ec(self.h, _p(e), _p(e_avg)), self)
        return e, e_avg

    def lut_dielectric_ec(self):
        e, e_avg = np.empty(32 * 32 * 32, np.float32), np.empty(32 * 32, np.float32)
        _check(lib().tpt_lut_dielectric_ec(self.h, _p(e), _p(e_avg)), self)
        return e, e_avg

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass


def build_qbvh(bounds: np.ndarray, threads: int = 0):
    """Host builder (qbvh.rs `build_qbvh`): returns (nodes[NODE_DTYPE], primitive_indices[u32])."""
    b = np.ascontiguousarray(bounds, np.float32).reshape(-1, 6)
    h = C.c_void_p()
    _check(lib().tpt_qbvh_build(_p(b), b.shape[0], threads, C.byref(h)))
    try:
        v = QbvhView()
        _check(lib().tpt_qbvh_view_of(h, C.byref(v)))
        nodes = np.zeros(v.num_nodes, NODE_DTYPE)
        prims = np.zeros(v.num_primitives, np.uint32)
        if v.num_nodes:
            C.memmove(nodes.ctypes.data, v.nodes, nodes.nbytes)
        C.memmove(prims.ctypes.data, v.primitive_indices, prims.nbytes)
    finally:
        lib().tpt_qbvh_free(h)
    return nodes, prims


def build_qbvh_device(ctx: "Context", bounds_ptr: int, n: int, stream=None):
    """GPU builder (`tpt_qbvh_build_device`) from a device array of n x 6
    floats: returns (nodes[NODE_DTYPE], primitive_indices[u32]), the host
    builder's tree."""
    h = C.c_void_p()
    _check(lib().tpt_qbvh_build_device(ctx.h, C.c_void_p(bounds_ptr), n, _stream(stream), C.byref(h)), ctx)
    try:
        v = QbvhView()
        _check(lib().tpt_qbvh_view_of(h, C.byref(v)))
        nodes = np.zeros(v.num_nodes, NODE_DTYPE)
        prims = np.zeros(v.num_primitives, np.uint32)
        if v.num_nodes:
            C.memmove(nodes.ctypes.data, v.nodes, nodes.nbytes)
        C.memmove(prims.ctypes.data, v.primitive_indices, prims.nbytes)
    finally:
        lib().tpt_qbvh_free(h)
    return nodes, prims


def _view(q):
    if q is None:
        return QbvhView(None, 0, None, 0)
    nodes, prims = q
    return QbvhView(
        nodes.ctypes.data if len(nodes) else None, len(nodes), prims.ctypes.data, len(prims)
    )


def scene_desc(meshes, instances, tlas=None, materials=None, light_tree=None, lights=None):
    """Build a `tpt_scene_desc` (and the list of arrays it points into).
    lights: dict with optional "point_lights", "spot_lights", "directional_lights"."""
    keep = []
    md = (MeshDesc * max(1, len(meshes)))()
    for i, m in enumerate(meshes):
        pos = np.ascontiguousarray(m["positions"], np.float32)
        idx = np.ascontiguousarray(m["indices"], np.uint32).reshape(-1)
        nrm = m.get("normals")
        uv = m.get("uvs")
        nrm = None if nrm is None else np.ascontiguousarray(nrm, np.float32)
        uv = None if uv is None else np.ascontiguousarray(uv, np.float32)
        keep += [pos, idx, nrm, uv]
        q = m.get("qbvh")
        if q is not None:
            q = (np.ascontiguousarray(q[0]), np.ascontiguousarray(q[1], np.uint32))
            keep += list(q)
        md[i] = MeshDesc(
            pos.ctypes.data, None if nrm is None else nrm.ctypes.data, None if uv is None else uv.ctypes.data,
            pos.shape[0], idx.ctypes.data, idx.size, _view(q)
        )
    idesc = (InstanceDesc * max(1, len(instances)))()
    for i, inst in enumerate(instances):
        d = InstanceDesc()
        d.mesh_index = inst["mesh"]
        d.material_index = inst.get("material", 0)
        d.local_to_world[:] = np.asarray(inst["local_to_world"], np.float32).reshape(16).tolist()
        d.world_to_local[:] = np.asarray(inst["world_to_local"], np.float32).reshape(16).tolist()
        d.normal_to_world[:] = np.asarray(inst["normal_to_world"], np.float32).reshape(9).tolist()
        idesc[i] = d
    if tlas is not None:
        tlas = (np.ascontiguousarray(tlas[0]), np.ascontiguousarray(tlas[1], np.uint32))
        keep += list(tlas)
    materials = materials or []
    mdesc = (MaterialDesc * max(1, len(materials)))()
    for i, m in enumerate(materials):
        d = MaterialDesc()
        d.kind = m["kind"]
        d.rho[:] = list(np.asarray(m.get("rho", (0, 0, 0)), np.float32))
        d.color[:] = list(np.asarray(m.get("color", (0, 0, 0)), np.float32))
        d.strength = float(np.float32(m.get("strength", 0.0)))
        if "opacity" in m:
            d.has_opacity = 1
            d.opacity = float(np.float32(m["opacity"]))
        if d.kind == OPENPBR:
            od = openpbr_desc(m)
            keep.append(od)
            d.openpbr = C.addressof(od)
        mdesc[i] = d
    ltv = LightTreeView(None, 0, 0)
    if light_tree is not None:
        nodes, root = np.ascontiguousarray(light_tree[0], LIGHT_NODE_DTYPE), int(light_tree[1])
        keep.append(nodes)
        ltv = LightTreeView(nodes.ctypes.data, len(nodes), root)
    (pa, npts), (sa, nsp), (da, ndir) = light_descs(lights or {})
    keep += [md, idesc, mdesc, pa, sa, da]
    env = (lights or {}).get("environment")
    env_ptr = None
    if env is not None:
        px = np.ascontiguousarray(env["pixels"], np.float32)
        ed = EnvironmentDesc(px.shape[1], px.shape[0], px.ctypes.data, float(np.float32(env.get("scale", 1.0))),
                             float(np.float32(env.get("rotate_y", 0.0))))
        keep += [px, ed]
        env_ptr = C.pointer(ed)
    desc = SceneDesc(md, len(meshes), idesc, len(instances), _view(tlas), mdesc, len(materials), ltv,
                     pa, npts, sa, nsp, da, ndir, env_ptr)
    return desc, keep


def build_light_tree(scene: dict, threads: int = 0):
    """Host light-tree builder (`tpt_light_tree_build_threads`; threads <= 0: all
    hardware threads): (nodes[LIGHT_NODE_DTYPE], root)."""
    desc, keep = scene_desc(scene["meshes"], scene["instances"], materials=scene["materials"], lights=scene)
    h = C.c_void_p()
    _check(lib().tpt_light_tree_build_threads(C.byref(desc), threads, C.byref(h)))
    try:
        v = LightTreeView()
        _check(lib().tpt_light_tree_view_of(h, C.byref(v)))
        nodes = np.zeros(v.num_nodes, LIGHT_NODE_DTYPE)
        C.memmove(nodes.ctypes.data, v.nodes, nodes.nbytes)
        return nodes, v.root
    finally:
        lib().tpt_light_tree_free(h)


class Scene:
    """Device-resident geometry (`tpt_scene`), uploaded from host arrays.

    meshes: list of dicts with positions [V,3], indices [3T], optional normals,
    uvs and a pre-built qbvh (nodes, prims).  instances: list of dicts with
    mesh, material, local_to_world, world_to_local (4x4 column-major) and
    normal_to_world (3x3).  lights: a dict (e.g. the scene dict) with optional
    "point_lights", "spot_lights" and "directional_lights" lists and an
    "environment" dict (pixels [H, W, 3], scale, rotate_y)."""

    def __init__(self, ctx: Context, meshes, instances, tlas=None, materials=None, light_tree=None, lights=None):
        self.ctx = ctx
        desc, keep = scene_desc(meshes, instances, tlas, materials, light_tree, lights)
        h = C.c_void_p()
        _check(lib().tpt_scene_upload(ctx.h, C.byref(desc), C.byref(h)), ctx)
        self.h = h
        self.n_materials = len(materials or [])

    def light_tree(self):
        """(nodes[LIGHT_NODE_DTYPE], root) of the tree the scene uses."""
        v = LightTreeView()
        _check(lib().tpt_scene_light_tree(self.h, C.byref(v)))
        nodes = np.zeros(v.num_nodes, LIGHT_NODE_DTYPE)
        if v.num_nodes:
            C.memmove(nodes.ctypes.data, v.nodes, nodes.nbytes)
        return nodes, v.root

    def job(self, camera: dict, width: int, height: int, spp: int, max_depth: int, integrator: int = 0,
            execution: int = EXEC_WAVEFRONT, seed: int = 0):
        """A `tpt_render_job`; seed 0 gives the reference's sample streams, any
        other value independent ones."""
        cam = CameraDesc()
        cam.eye[:] = [float(np.float32(x)) for x in camera["eye"]]
        cam.look_at[:] = [float(np.float32(x)) for x in camera["look_at"]]
        cam.up[:] = [float(np.float32(x)) for x in camera["up"]]
        cam.fov_y = float(np.float32(camera["fov_y"]))
        cam.exposure = float(np.float32(camera.get("exposure", 1.0)))
        return RenderJob(self.h.value, cam, width, height, spp, max_depth, integrator, execution, seed)

    def render(self, camera: dict, width: int, height: int, spp: int, max_depth: int, integrator: int = 0,
               execution: int = EXEC_WAVEFRONT, seed: int = 0):
        """`tpt_render`: returns float32 [height, width, 3] (host)."""
        j = self.job(camera, width, height, spp, max_depth, integrator, execution, seed)
        out = np.empty((height, width, 3), np.float32)
        ptrs = (C.c_void_p * 1)(out.ctypes.data)
        _check(lib().tpt_render(self.ctx.h, C.byref(j), 1, ptrs), self.ctx)
        return out

    def render_device(self, job, out_ptr: int, stream=None):
        _check(lib().tpt_render_device(self.ctx.h, C.byref(job), C.c_void_p(out_ptr), _stream(stream)), self.ctx)

    def render_pixels_device(self, job, first_pixel: int, num_pixels: int, out_ptr: int, stream=None):
        """`tpt_render_pixels_device`: pixels [first_pixel, first_pixel + num_pixels)
        of the job's image (float32 [num_pixels * 3] at out_ptr)."""
        _check(lib().tpt_render_pixels_device(self.ctx.h, C.byref(job), first_pixel, num_pixels,
                                              C.c_void_p(out_ptr), _stream(stream)), self.ctx)

    def render_samples_device(self, job, first: int, count: int, out_ptr: int, stream=None):
        _check(lib().tpt_render_samples_device(self.ctx.h, C.byref(job), first, count, C.c_void_p(out_ptr),
                                               _stream(stream)), self.ctx)

    def bsdf_eval_device(self, material: int, n: int, wo_ptr: int, wi_ptr: int, front_ptr: int, f_ptr: int,
                         pdf_ptr: int, stream=None, mode: int = 0):
        """`tpt_bsdf_eval_device`: OpenPBR eval + pdf of n direction pairs (device buffers);
        mode 0 radiance, 1 importance transport."""
        _check(lib().tpt_bsdf_eval_device(self.ctx.h, self.h, material, n, C.c_void_p(wo_ptr), C.c_void_p(wi_ptr),
                                          C.c_void_p(front_ptr), mode, C.c_void_p(f_ptr), C.c_void_p(pdf_ptr),
                                          _stream(stream)), self.ctx)

    def bsdf_sample_device(self, material: int, n: int, wo_ptr: int, u_ptr: int, front_ptr: int, out_ptr: int,
                           stream=None, mode: int = 0):
        """`tpt_bsdf_sample_device`: OpenPBR samples (weight, wi, pdf, pdf_rev, flags) for n (wo, u)."""
        _check(lib().tpt_bsdf_sample_device(self.ctx.h, self.h, material, n, C.c_void_p(wo_ptr), C.c_void_p(u_ptr),
                                            C.c_void_p(front_ptr), mode, C.c_void_p(out_ptr), _stream(stream)),
               self.ctx)

    def bsdf_eval_path_device(self, material: int, n: int, wo_ptr: int, wi_ptr: int, front_ptr: int, state_ptr: int,
                              f_ptr: int, pdf_ptr: int, stream=None, mode: int = 0):
        """`tpt_bsdf_eval_path_device`: eval + pdf with a path state per pair
        (n x 4: throughput r, g, b and the wavelength lock, NaN = none)."""
        _check(lib().tpt_bsdf_eval_path_device(self.ctx.h, self.h, material, n, C.c_void_p(wo_ptr),
                                               C.c_void_p(wi_ptr), C.c_void_p(front_ptr), C.c_void_p(state_ptr),
                                               mode, C.c_void_p(f_ptr), C.c_void_p(pdf_ptr), _stream(stream)),
               self.ctx)

    def bsdf_sample_path_device(self, material: int, n: int, wo_ptr: int, u_ptr: int, front_ptr: int,
                                state_ptr: int, out_ptr: int, stream=None, mode: int = 0):
        """`tpt_bsdf_sample_path_device`: samples with a path state; u n x 7
        (u_lobe, u_dir, u_extra0..3), out n x 10 (the sampled lock last, NaN = none)."""
        _check(lib().tpt_bsdf_sample_path_device(self.ctx.h, self.h, material, n, C.c_void_p(wo_ptr),
                                                 C.c_void_p(u_ptr), C.c_void_p(front_ptr), C.c_void_p(state_ptr),
                                                 mode, C.c_void_p(out_ptr), _stream(stream)), self.ctx)

    # -- material updates and the adjoint (no counterpart in the reference) ----
    def set_openpbr(self, material_ids, materials, stream=None):
        """`tpt_scene_set_openpbr`: new parameters (dicts) for OpenPBR materials."""
        ids = np.ascontiguousarray(material_ids, np.uint32)
        descs = (OpenPbrDesc * max(1, len(ids)))()
        for k, m in enumerate(materials):
            descs[k] = openpbr_desc(m)
        _check(lib().tpt_scene_set_openpbr(self.ctx.h, self.h, len(ids), _p(ids), descs, _stream(stream)), self.ctx)

    def adjoint_device(self, job, d_image_ptr: int, grad_ptr: int, mask: int = 0, fd_step: float = 0.0,
                       stream=None, first_pixel: int = 0, num_pixels: int = 0):
        """`tpt_adjoint_device`: dLoss/d(material parameters) (float64 [n_materials, 7]
        at grad_ptr, n_materials = self.n_materials) from dLoss/dimage (float32
        [h*w*3] at d_image_ptr, or [num_pixels*3] for the paths of pixels
        [first_pixel, first_pixel + num_pixels) when num_pixels > 0)."""
        ad = AdjointDesc(mask, fd_step, first_pixel, num_pixels)
        _check(lib().tpt_adjoint_device(self.ctx.h, C.byref(job), C.byref(ad), C.c_void_p(d_image_ptr),
                                        C.c_void_p(grad_ptr), _stream(stream)), self.ctx)

    def adjoint(self, job, d_image: np.ndarray, mask: int = 0, fd_step: float = 0.0, first_pixel: int = 0,
                num_pixels: int = 0):
        """`tpt_adjoint` with host arrays; returns float64 [n_materials, 7]."""
        d = np.ascontiguousarray(d_image, np.float32).reshape(-1)
        assert d.size == (num_pixels or job.width * job.height) * 3
        out = np.zeros((self.n_materials, GRAD_PARAMS), np.float64)
        ad = AdjointDesc(mask, fd_step, first_pixel, num_pixels)
        _check(lib().tpt_adjoint(self.ctx.h, C.byref(job), C.byref(ad), _p(d), _p(out)), self.ctx)
        return out

    def device_bytes(self) -> int:
        v = C.c_uint64()
        _check(lib().tpt_scene_device_bytes(self.h, C.byref(v)))
        return v.value

    def close(self):
        if getattr(self, "h", None):
            lib().tpt_scene_release(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:  # interpreter shutdown: the library may already be gone
            pass

    # -- queries ----------------------------------------------------------
    def closest_hit(self, rays: np.ndarray, mode: int = CLOSEST_HIT, want_instance=False, want_bary=False):
        """Host arrays in/out through `tpt_traverse`. rays: float32 [7, n]."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[1]
        prim = np.empty(n, np.int32)
        t = np.empty(n, np.float32)
        inst = np.empty(n, np.int32) if want_instance else None
        bary = np.empty((3, n), np.float32) if want_bary else None
        _check(
            lib().tpt_traverse(self.ctx.h, self.h, _p(rays), n, mode, _p(prim), _p(t), _p(inst), _p(bary)), self.ctx
        )
        out = {"prim": prim, "t": t}
        if want_instance:
            out["inst"] = inst
        if want_bary:
            out["bary"] = bary
        return out

    def traverse_alpha_device(self, rays_ptr: int, n: int, aux_ptr: int, prim_ptr: int, t_ptr: int, inst_ptr=None,
                              bary_ptr=None, stream=None):
        """`tpt_traverse_alpha_device`: closest hit with the materials' alpha tests,
        drawing from (and advancing) the per-ray AuxRng states at aux_ptr."""
        _check(
            lib().tpt_traverse_alpha_device(
                self.ctx.h, self.h, C.c_void_p(rays_ptr), n, C.c_void_p(aux_ptr), C.c_void_p(prim_ptr),
                C.c_void_p(t_ptr), C.c_void_p(inst_ptr) if inst_ptr else None,
                C.c_void_p(bary_ptr) if bary_ptr else None, _stream(stream),
            ),
            self.ctx,
        )

    def traverse_device(self, rays_ptr: int, n: int, mode: int, prim_ptr: int, t_ptr: int, inst_ptr=None,
                        bary_ptr=None, stream=None):
        """Device pointers (e.g. torch tensor data_ptr()) and a cudaStream_t handle."""
        _check(
            lib().tpt_traverse_device(
                self.ctx.h, self.h, C.c_void_p(rays_ptr), n, mode, C.c_void_p(prim_ptr), C.c_void_p(t_ptr),
                C.c_void_p(inst_ptr) if inst_ptr else None, C.c_void_p(bary_ptr) if bary_ptr else None,
                _stream(stream),
            ),
            self.ctx,
        )

    def traverse_stats_device(self, rays_ptr, n, mode, prim_ptr, t_ptr, nodes_ptr, tris_ptr, stream=None):
        _check(
            lib().tpt_traverse_stats_device(
                self.ctx.h, self.h, C.c_void_p(rays_ptr), n, mode, C.c_void_p(prim_ptr), C.c_void_p(t_ptr),
                C.c_void_p(nodes_ptr), C.c_void_p(tris_ptr), _stream(stream),
            ),
            self.ctx,
        )


# --------------------------------------------------------------------------
def render_function():
    """The forward/backward pair as a torch.autograd.Function (torch is only the
    caller's tensor plumbing here; both passes run through the C ABI):

        image = RenderFunction.apply(params, scene, job, material_ids, materials_of, mask, fd_step, adjoint_job)

    params: float32 [n, k] tensor of material parameters (any layout the caller's
    `materials_of(params_row) -> dict` maps to OpenPBR parameters); forward sets
    the materials and renders; backward runs the path-replay adjoint and returns
    the first k = params.shape[1] columns of the [n_materials, 7] gradient for
    the listed materials (the TPT_GRAD_* order: base_color rgb, roughness,
    metalness, specular_ior, coat_weight), so params rows must follow that
    order up to k.  adjoint_job
    (optional): the job the backward pass replays.  By default it is the
    forward job with another sample-stream seed (ADJOINT_SEED_STEP added), so
    its paths are independent of the forward image's and the gradient of an L2
    loss is not correlated with that image's noise (a same-sample backward is
    biased).  Pass the forward job itself to replay its very paths."""
    import torch

    class RenderFunction(torch.autograd.Function):
        @staticmethod
        def forward(fctx, params, scene, job, material_ids, materials_of, mask=0, fd_step=0.0, adjoint_job=None):
            rows = params.detach().cpu().numpy()
            stream = torch.cuda.current_stream().cuda_stream
            scene.set_openpbr(material_ids, [materials_of(r) for r in rows], stream=stream)
            img = torch.empty(job.height * job.width * 3, dtype=torch.float32, device="cuda")
            scene.render_device(job, img.data_ptr(), stream)
            fctx.scene, fctx.ids, fctx.mask, fctx.step = scene, material_ids, mask, fd_step
            if adjoint_job is None:
                adjoint_job = RenderJob.from_buffer_copy(job)
                adjoint_job.seed = (job.seed + ADJOINT_SEED_STEP) & 0xFFFFFFFF
            fctx.job = adjoint_job
            fctx.k = params.shape[1]
            fctx.device, fctx.dtype = params.device, params.dtype
            return img.view(job.height, job.width, 3)

        @staticmethod
        def backward(fctx, grad_img):
            import torch

            scene, job = fctx.scene, fctx.job
            g = grad_img.contiguous().float().view(-1)
            n_mat = scene.n_materials
            grad = torch.zeros(n_mat * GRAD_PARAMS, dtype=torch.float64, device="cuda")
            scene.adjoint_device(job, g.data_ptr(), grad.data_ptr(), fctx.mask, fctx.step,
                                 stream=torch.cuda.current_stream().cuda_stream)
            grad = grad.view(n_mat, GRAD_PARAMS)[torch.as_tensor(fctx.ids, device="cuda").long()]
            out = grad[:, :fctx.k].to(device=fctx.device, dtype=fctx.dtype)
            return (out, None, None, None, None, None, None, None)

    return RenderFunction
