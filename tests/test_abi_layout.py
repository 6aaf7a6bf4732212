"""The ctypes mirrors in tpt.py against the C header (CPU only): a probe
compiled with the system C compiler from include/tpt.h prints sizeof and
offsetof of every struct the binding passes across the C ABI, and each must
equal the mirror's."""
import ctypes
import os
import shutil
import subprocess
import tempfile

import pytest

import tpt

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [
    ("tpt_qbvh_view", tpt.QbvhView), ("tpt_mesh_desc", tpt.MeshDesc), ("tpt_instance_desc", tpt.InstanceDesc),
    ("tpt_openpbr_desc", tpt.OpenPbrDesc), ("tpt_material_desc", tpt.MaterialDesc),
    ("tpt_light_tree_view", tpt.LightTreeView), ("tpt_point_light_desc", tpt.PointLightDesc),
    ("tpt_spot_light_desc", tpt.SpotLightDesc), ("tpt_directional_light_desc", tpt.DirectionalLightDesc),
    ("tpt_environment_desc", tpt.EnvironmentDesc), ("tpt_scene_desc", tpt.SceneDesc),
    ("tpt_camera_desc", tpt.CameraDesc), ("tpt_render_job", tpt.RenderJob), ("tpt_adjoint_desc", tpt.AdjointDesc),
    ("tpt_tune_result", tpt.TuneResult),
]


@pytest.mark.skipif(shutil.which("cc") is None and shutil.which("gcc") is None, reason="no C compiler")
def test_ctypes_mirrors_match_the_header():
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "tpt.h"', "int main(void) {"]
    for cname, py in PAIRS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in py._fields_:
            lines.append(f'  printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["  return 0;", "}"]
    cc = shutil.which("cc") or shutil.which("gcc")
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "probe.c"), os.path.join(d, "probe")
        with open(src, "w") as f:
            f.write("\n".join(lines) + "\n")
        subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
        out = subprocess.run([exe], check=True, capture_output=True, text=True).stdout
    got = {}
    for ln in out.splitlines():
        cname, field, v = ln.split()
        got[(cname, field)] = int(v)
    for cname, py in PAIRS:
        assert got[(cname, "sizeof")] == ctypes.sizeof(py), cname
        for f in py._fields_:
            assert got[(cname, f[0])] == getattr(py, f[0]).offset, (cname, f[0])

