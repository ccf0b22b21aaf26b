"""Scene files in the manifest format that Scene::load reads
(src/scene.rs:11-255) and tools/export_scene.py writes: a version-1
``scene.json`` naming binary files of little-endian 64-byte vertices
(position4, normal4, tangent4, uv4) followed by u32 indices, and x-fastest
f32 SDF samples on the grid nodes of each mesh's SDF bounds.

This module writes such scenes from triangle meshes with analytic signed
distances (boxes, UV spheres, tori), following the exporter's conventions:
SDF bounds padded by two voxels of the vertex-box diagonal and samples
biased by -|bounds diagonal| * 2e-6.  ``Workload.load`` reads them back.
"""
from __future__ import annotations

import hashlib
import json
import math
import os
from dataclasses import dataclass, field

import numpy as np


@dataclass
class MeshSpec:
    id: str
    vertices: np.ndarray            # (N, 16) float32: position4, normal4, tangent4, uv4
    indices: np.ndarray             # (M,) uint32, counter-clockwise fronts
    sdf: object                     # callable p (..., 3) -> signed distance (...,)
    resolution: int = 24


@dataclass
class Scene:
    meshes: list = field(default_factory=list)
    materials: list = field(default_factory=list)
    objects: list = field(default_factory=list)
    lights: list = field(default_factory=list)
    camera: dict = field(default_factory=dict)


def _vertex_rows(p, n, uv):
    p = np.asarray(p, np.float32).reshape(-1, 3)
    n = np.asarray(n, np.float32).reshape(-1, 3)
    uv = np.asarray(uv, np.float32).reshape(-1, 2)
    # any unit tangent orthogonal to n
    a = np.where(np.abs(n[:, 2:3]) > 0.9, np.array([[1, 0, 0]], np.float32), np.array([[0, 0, 1]], np.float32))
    t = np.cross(a, n)
    t /= np.maximum(np.linalg.norm(t, axis=1, keepdims=True), 1e-12)
    rows = np.zeros((len(p), 16), np.float32)
    rows[:, 0:3], rows[:, 3] = p, 1.0
    rows[:, 4:7] = n
    rows[:, 8:11], rows[:, 11] = t, 1.0
    rows[:, 12:14] = uv
    return rows


def box(id: str, lo, hi, resolution: int = 24) -> MeshSpec:
    """Axis-aligned box: 24 vertices (flat faces), 12 triangles."""
    lo = np.asarray(lo, np.float64)
    hi = np.asarray(hi, np.float64)
    P, N, UV, I = [], [], [], []
    for axis in range(3):
        for side in (0, 1):
            nrm = np.zeros(3)
            nrm[axis] = 1.0 if side else -1.0
            u_ax, v_ax = (axis + 1) % 3, (axis + 2) % 3
            corners = []
            for cu, cv in ((0, 0), (1, 0), (1, 1), (0, 1)):
                q = np.empty(3)
                q[axis] = hi[axis] if side else lo[axis]
                q[u_ax] = hi[u_ax] if cu else lo[u_ax]
                q[v_ax] = hi[v_ax] if cv else lo[v_ax]
                corners.append(q)
            base = len(P)
            P += corners
            N += [nrm] * 4
            UV += [(0, 0), (1, 0), (1, 1), (0, 1)]
            quad = [base, base + 1, base + 2, base, base + 2, base + 3]
            # u x v = +axis for the cyclic order; flip the low side
            if not side:
                quad = [base, base + 2, base + 1, base, base + 3, base + 2]
            I += quad

    def sdf(p):
        c = (lo + hi) * 0.5
        h = (hi - lo) * 0.5
        q = np.abs(p - c) - h
        out = np.linalg.norm(np.maximum(q, 0.0), axis=-1)
        return out + np.minimum(q.max(-1), 0.0)

    return MeshSpec(id, _vertex_rows(P, N, UV), np.asarray(I, np.uint32), sdf, resolution)


def uv_sphere(id: str, radius: float, rings: int = 12, segments: int = 24, resolution: int = 24) -> MeshSpec:
    P, N, UV = [], [], []
    for i in range(rings + 1):
        th = math.pi * i / rings
        for j in range(segments + 1):
            ph = 2 * math.pi * j / segments
            n = (math.sin(th) * math.cos(ph), math.sin(th) * math.sin(ph), math.cos(th))
            P.append([radius * c for c in n])
            N.append(n)
            UV.append((j / segments, i / rings))
    I = []
    w = segments + 1
    for i in range(rings):
        for j in range(segments):
            a, b, c, d = i * w + j, i * w + j + 1, (i + 1) * w + j + 1, (i + 1) * w + j
            if i != 0:
                I += [a, d, b]
            if i != rings - 1:
                I += [b, d, c]
    return MeshSpec(id, _vertex_rows(P, N, UV), np.asarray(I, np.uint32),
                    lambda p: np.linalg.norm(p, axis=-1) - radius, resolution)


def torus(id: str, major: float, minor: float, rings: int = 24, sides: int = 12, resolution: int = 24) -> MeshSpec:
    P, N, UV = [], [], []
    for i in range(rings + 1):
        u = 2 * math.pi * i / rings
        for j in range(sides + 1):
            v = 2 * math.pi * j / sides
            n = (math.cos(v) * math.cos(u), math.cos(v) * math.sin(u), math.sin(v))
            P.append(((major + minor * math.cos(v)) * math.cos(u), (major + minor * math.cos(v)) * math.sin(u),
                      minor * math.sin(v)))
            N.append(n)
            UV.append((i / rings, j / sides))
    I = []
    w = sides + 1
    for i in range(rings):
        for j in range(sides):
            a, b, c, d = i * w + j, (i + 1) * w + j, (i + 1) * w + j + 1, i * w + j + 1
            I += [a, b, c, a, c, d]

    def sdf(p):
        q = np.stack([np.linalg.norm(p[..., :2], axis=-1) - major, p[..., 2]], -1)
        return np.linalg.norm(q, axis=-1) - minor

    return MeshSpec(id, _vertex_rows(P, N, UV), np.asarray(I, np.uint32), sdf, resolution)


def sdf_grid(mesh: MeshSpec):
    """Exporter conventions: bounds = vertex box padded by two voxels of its
    diagonal; samples on the res^3 grid nodes (x fastest) minus
    |bounds diagonal| * 2e-6.  Returns (samples f32, lo, hi, error_bound)."""
    res = mesh.resolution
    pos = mesh.vertices[:, :3].astype(np.float64)
    lo, hi = pos.min(0), pos.max(0)
    pad = np.linalg.norm(hi - lo) / (res - 1) * 2
    lo = (lo - pad).astype(np.float32)
    hi = (hi + pad).astype(np.float32)
    ext = float(np.linalg.norm(hi.astype(np.float64) - lo.astype(np.float64)))
    ax = [lo[a] + (np.float64(hi[a]) - lo[a]) * np.arange(res) / (res - 1) for a in range(3)]
    z, y, x = np.meshgrid(ax[2], ax[1], ax[0], indexing="ij")
    p = np.stack([x, y, z], -1)
    samples = (mesh.sdf(p) - ext * 2e-6).astype(np.float32).reshape(-1)
    return samples, lo, hi, ext * 2e-6


def material(id: str, color, roughness=0.5, metallic=0.0, **extra) -> dict:
    m = {"id": id, "base_color": [float(c) for c in color] + ([1.0] if len(color) == 3 else []),
         "roughness": roughness, "metallic": metallic}
    m.update(extra)
    return m


def obj(id: str, mesh: str, mat: str, position=(0, 0, 0), rotation=(0, 0, 0, 1), scale=1.0) -> dict:
    return {"id": id, "mesh": mesh, "material": mat,
            "transform": {"position": [float(v) for v in position], "rotation": [float(v) for v in rotation],
                          "scale": float(scale)}}


def point_light(id: str, position, color=(1, 1, 1), strength=10.0) -> dict:
    return {"id": id, "type": "point", "position": [float(v) for v in position],
            "color": [float(v) for v in color], "strength": float(strength)}


def spot_light(id: str, position, direction, angle, color=(1, 1, 1), strength=50.0) -> dict:
    d = point_light(id, position, color, strength)
    d.update(type="spot", direction=[float(v) for v in direction], angle_radians=float(angle))
    return d


def look_rotation(eye, target) -> list:
    """Quaternion (x, y, z, w) turning the camera's -z toward target with
    +z world up kept on the image's up side."""
    eye, target = np.asarray(eye, np.float64), np.asarray(target, np.float64)
    f = target - eye
    f /= np.linalg.norm(f)
    r = np.cross(f, [0, 0, 1.0])
    r /= np.linalg.norm(r)
    u = np.cross(r, f)
    m = np.stack([r, u, -f], 1)  # columns: camera x, y, z in world
    t = np.trace(m)
    if t > 0:
        s = math.sqrt(t + 1.0) * 2
        q = [(m[2, 1] - m[1, 2]) / s, (m[0, 2] - m[2, 0]) / s, (m[1, 0] - m[0, 1]) / s, 0.25 * s]
    else:
        i = int(np.argmax(np.diag(m)))
        j, k = (i + 1) % 3, (i + 2) % 3
        s = math.sqrt(1.0 + m[i, i] - m[j, j] - m[k, k]) * 2
        q = [0.0] * 4
        q[i] = 0.25 * s
        q[j] = (m[j, i] + m[i, j]) / s
        q[k] = (m[k, i] + m[i, k]) / s
        q[3] = (m[k, j] - m[j, k]) / s
    return [float(v) for v in q]


def write_scene(directory, scene: Scene) -> str:
    """Writes scene.json and its two binary files (geometry, fields) into
    `directory`; returns the manifest path."""
    os.makedirs(directory, exist_ok=True)
    geo, fields, manifest_meshes = bytearray(), bytearray(), []
    entries = []
    for m in scene.meshes:
        samples, lo, hi, err = sdf_grid(m)
        v_off = len(geo)
        geo += np.ascontiguousarray(m.vertices, "<f4").tobytes()
        i_off = len(geo)
        geo += np.ascontiguousarray(m.indices, "<u4").tobytes()
        f_off = len(fields)
        fields += np.ascontiguousarray(samples, "<f4").tobytes()
        entries.append((m, v_off, i_off, f_off, lo, hi, err))
    geo_name = "meshes_" + hashlib.sha256(geo).hexdigest()[:16] + ".bin"
    fld_name = "fields_" + hashlib.sha256(fields).hexdigest()[:16] + ".bin"
    for m, v_off, i_off, f_off, lo, hi, err in entries:
        manifest_meshes.append({
            "id": m.id,
            "geometry": {"path": geo_name, "vertex_offset": v_off, "vertex_count": int(len(m.vertices)),
                         "index_offset": i_off, "index_count": int(len(m.indices))},
            "sdf": {"path": fld_name, "offset": f_off, "resolution": int(m.resolution),
                    "bounds_min": [float(v) for v in lo], "bounds_max": [float(v) for v in hi],
                    "conservative": True, "query": "trilinear_bound", "error_bound": float(err)},
        })
    with open(os.path.join(directory, geo_name), "wb") as f:
        f.write(bytes(geo))
    with open(os.path.join(directory, fld_name), "wb") as f:
        f.write(bytes(fields))
    doc = {"version": 1, "meshes": manifest_meshes, "materials": scene.materials, "objects": scene.objects,
           "lights": scene.lights, "camera": scene.camera}
    path = os.path.join(directory, "scene.json")
    with open(path, "w") as f:
        json.dump(doc, f, indent=2)
    return path


def demo_scene(resolution: int = 24) -> Scene:
    """A small lit room: floor and two walls (boxes), a sphere, a torus and a
    cube on the floor, one point light and one spot light, a camera looking
    into the corner."""
    s = Scene()
    s.meshes = [
        box("floor_box", (-3, -3, -0.2), (3, 3, 0.0), resolution),
        box("wall_box", (-0.1, -3, 0), (0.1, 3, 3), resolution),
        box("cube_box", (-0.4, -0.4, -0.4), (0.4, 0.4, 0.4), resolution),
        uv_sphere("sphere", 0.6, resolution=resolution),
        torus("torus", 0.55, 0.18, resolution=resolution),
    ]
    s.materials = [material("white", (0.8, 0.8, 0.8)), material("red", (0.9, 0.1, 0.1), 0.7),
                   material("green", (0.1, 0.8, 0.2), 0.6), material("metal", (0.9, 0.8, 0.5), 0.3, 1.0),
                   material("blue", (0.2, 0.3, 0.9), 0.4)]
    s.objects = [
        obj("floor", "floor_box", "white"),
        obj("back", "wall_box", "red", (-3.0, 0, 0)),
        obj("side", "wall_box", "green", (0, 3.0, 0), (0, 0, math.sin(math.pi / 4), math.cos(math.pi / 4))),
        obj("cube", "cube_box", "blue", (-1.2, 1.0, 0.4), (0, 0, math.sin(0.3), math.cos(0.3))),
        obj("ball", "sphere", "metal", (0.3, -0.8, 0.6)),
        obj("ring", "torus", "white", (-1.0, -1.2, 0.9), (math.sin(0.5), 0, 0, math.cos(0.5)), 1.2),
    ]
    s.lights = [point_light("lamp", (0.5, 0.5, 2.2), (1.0, 0.9, 0.7), 12.0),
                spot_light("spot", (2.5, -2.5, 2.5), (-1, 1, -1), 0.9, (0.8, 0.9, 1.0), 60.0)]
    eye = (4.5, -3.5, 2.4)
    s.camera = {"position": list(eye), "rotation": look_rotation(eye, (-0.8, 0.4, 0.6)),
                "fov_y_radians": 0.9, "near": 0.1, "far": 100.0}
    return s
