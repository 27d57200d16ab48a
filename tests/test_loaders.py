"""Mesh ingest (STL binary / ASCII, OBJ) into the voxelizer, on the CPU restatement."""
import struct

import numpy as np

from windtunnel_vis_b200 import loaders as Ld
from windtunnel_vis_b200 import mesh as Mh

CUBE_V = np.array([[0, 0, 0], [1, 0, 0], [1, 1, 0], [0, 1, 0], [0, 0, 1], [1, 0, 1], [1, 1, 1], [0, 1, 1]], np.float32)
CUBE_Q = [(0, 3, 2, 1), (4, 5, 6, 7), (0, 1, 5, 4), (2, 3, 7, 6), (1, 2, 6, 5), (0, 4, 7, 3)]


def cube_tris():
    t = []
    for q in CUBE_Q:
        t += [(q[0], q[1], q[2]), (q[0], q[2], q[3])]
    return np.array(t)


def test_binary_stl():
    tris = CUBE_V[cube_tris()]
    data = bytearray(b"solid but binary".ljust(80, b" ")) + struct.pack("<I", len(tris))
    for t in tris:
        data += struct.pack("<3f", 0, 0, 0) + t.astype("<f4").tobytes() + b"\0\0"
    m = Ld.load_model(data=bytes(data), name="cube.stl")
    assert m["up"] == "z" and m["triangles"] == 12
    np.testing.assert_array_equal(m["positions"], tris.reshape(-1, 3))
    np.testing.assert_array_equal(m["indices"], np.arange(36))


def test_ascii_stl():
    tris = CUBE_V[cube_tris()]
    lines = ["solid cube"]
    for t in tris:
        lines += ["  facet normal 0 0 0", "    outer loop"] + [f"      vertex {x:g} {y:g} {z:g}" for x, y, z in t]
        lines += ["    endloop", "  endfacet"]
    lines.append("endsolid cube")
    m = Ld.load_model(data="\n".join(lines).encode(), name="cube.STL")
    np.testing.assert_array_equal(m["positions"], tris.reshape(-1, 3))


def test_obj_quads_and_negative_indices():
    text = "# cube\no cube\n" + "".join(f"v {x} {y} {z}\n" for x, y, z in CUBE_V)
    for k, q in enumerate(CUBE_Q):
        if k % 2:
            text += "f " + " ".join(str(i - 8) for i in q) + "\n"  # relative indices
        else:
            text += "f " + " ".join(f"{i + 1}/{i + 1}/1" for i in q) + "\n"
    m = Ld.load_model(data=text.encode(), name="cube.obj")
    assert m["up"] == "y" and m["triangles"] == 12
    np.testing.assert_array_equal(m["positions"], CUBE_V[cube_tris()].reshape(-1, 3))


def test_loaded_mesh_voxelizes(oracle):
    text = "".join(f"v {x} {y} {z}\n" for x, y, z in CUBE_V) + "".join(
        "f " + " ".join(str(i + 1) for i in q) + "\n" for q in CUBE_Q)
    m = Ld.load_model(data=text.encode(), name="box.obj")
    p, lo, hi, _ = Mh.normalize_mesh(m["positions"], up=m["up"])
    dims = (64, 32, 32)
    M16, _, _ = Mh.placement_matrix(p, lo, hi, dims, dict(mode="ground", lengthFrac=0.25, xFrac=0.4, rideCells=2))
    flags, sdf, info = oracle.voxelize_f32(dims, p, m["indices"], M16)
    # a 16-cell cube standing 2 cells above the floor
    assert abs(info["solidCells"] - 16 ** 3) <= 16 * 16 * 2 and info["frontal"] in (16 * 16, 16 * 17, 17 * 17)
    assert info["min"][1] == 2
