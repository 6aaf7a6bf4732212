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
