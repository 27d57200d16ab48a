"""Mesh ingest: STL and OBJ files into the triangle arrays the voxelizer takes.

Restates the geometry the reference obtains through three.js (three@0.186.1, not vendored here)
in loadModelFiles (src/voxelize/loaders.ts:41-101) followed by mergeObject (src/voxelize/mesh.ts):

  STL ... STLLoader: binary when 84 + 50 * (face count in bytes 80-83) equals the file size, or when
          the text "solid" is absent from the first five byte offsets; otherwise ASCII, read as
          facets of three "vertex x y z" lines. Up axis 'z' (STL convention), as the reference.
  OBJ ... OBJLoader: "v x y z" positions, "f" faces with 1-based or negative (relative) indices in
          the v, v/vt, v//vn and v/vt/vn forms, polygons triangulated as fans from the first
          vertex; objects, groups and materials merge into one mesh. Up axis 'y'.

Both give non-indexed triangles like three.js's BufferGeometry: positions (3 t, 3) float32 and
indices 0 .. 3 t - 1. glTF / GLB (GLTFLoader with Draco / meshopt decoders) is not restated.
"""
import os
import re

import numpy as np

MODEL_EXTS = ("obj", "stl")


def _is_binary_stl(data: bytes) -> bool:
    if len(data) >= 84:
        n = int.from_bytes(data[80:84], "little")
        if 84 + 50 * n == len(data):
            return True
    solid = b"solid"
    for off in range(5):
        if data[off:off + 5] == solid:
            return False
    return True


def parse_stl(data: bytes):
    """STL bytes -> positions (3 t, 3) float32 (binary or ASCII)."""
    if _is_binary_stl(data):
        n = int.from_bytes(data[80:84], "little")
        rec = np.dtype([("normal", "<f4", 3), ("v", "<f4", (3, 3)), ("attr", "<u2")])
        faces = np.frombuffer(data, rec, count=n, offset=84)
        return np.ascontiguousarray(faces["v"].reshape(-1, 3), np.float32)
    text = data.decode("utf-8", errors="replace")
    num = r"([+\-]?(?:\d+\.?\d*|\.\d+)(?:[eE][+\-]?\d+)?)"
    vert = re.compile(r"vertex\s+" + num + r"\s+" + num + r"\s+" + num)
    out = []
    for facet in re.finditer(r"facet([\s\S]*?)endfacet", text):
        vs = [tuple(float(g) for g in m.groups()) for m in vert.finditer(facet.group(1))]
        if len(vs) == 3:
            out.extend(vs)
    return np.asarray(out, np.float32).reshape(-1, 3)


def parse_obj(text: str):
    """OBJ text -> positions (3 t, 3) float32."""
    verts = []
    tris = []
    for line in text.splitlines():
        line = line.strip()
        if not line or line[0] == "#":
            continue
        parts = line.split()
        if parts[0] == "v" and len(parts) >= 4:
            verts.append((float(parts[1]), float(parts[2]), float(parts[3])))
        elif parts[0] == "f" and len(parts) >= 4:
            idx = []
            for tok in parts[1:]:
                k = int(tok.split("/")[0])
                idx.append(k - 1 if k > 0 else len(verts) + k)
            for j in range(1, len(idx) - 1):
                tris.append((idx[0], idx[j], idx[j + 1]))
    v = np.asarray(verts, np.float32).reshape(-1, 3)
    t = np.asarray(tris, np.int64).reshape(-1, 3)
    if t.size and (t.min() < 0 or t.max() >= len(v)):
        raise ValueError("OBJ face index out of range")
    return np.ascontiguousarray(v[t.reshape(-1)], np.float32) if t.size else np.zeros((0, 3), np.float32)


def load_model(path=None, data=None, name=None):
    """loadModelFile for STL / OBJ: {name, positions, indices, up, triangles}. Give a path, or the
    file's bytes with its name."""
    if path is not None:
        name = name or os.path.basename(path)
        with open(path, "rb") as fh:
            data = fh.read()
    if data is None or not name:
        raise ValueError("need a path, or data with a file name")
    ext = name.rsplit(".", 1)[-1].lower()
    if ext == "stl":
        pos, up = parse_stl(data), "z"
    elif ext == "obj":
        pos, up = parse_obj(data.decode("utf-8", errors="replace")), "y"
    else:
        raise ValueError(f"No model among the files — use {', '.join('.' + e for e in MODEL_EXTS)}")
    if len(pos) == 0:
        raise ValueError("No triangle meshes found in the file")
    idx = np.arange(len(pos), dtype=np.uint32)
    return {"name": name, "positions": pos, "indices": idx, "up": up, "triangles": len(pos) // 3}
