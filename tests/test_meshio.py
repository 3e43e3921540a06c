"""OBJ ingest / egress (pamo_obj_parse / pamo_obj_format through
pamo_b200.meshio) on the host, against a plain-Python reading of the same
statements (the OBJ specification: `v` vertices, `f` polygons as fans, 1-based
and negative indices, `i/t/n` corners)."""
import numpy as np
import pytest

from pamo_b200 import meshgen as mg
from pamo_b200 import meshio


def _plain_obj(text: str):
    """The OBJ statements this reader takes, one line at a time in Python."""
    V, F = [], []
    for line in text.splitlines():
        t = line.split("#", 1)[0].split()
        if not t:
            continue
        if t[0] == "v":
            V.append([float(x) for x in t[1:4]])
        elif t[0] == "f":
            idx = []
            for c in t[1:]:
                i = int(c.split("/")[0])
                idx.append(i - 1 if i > 0 else len(V) + i)
            for k in range(1, len(idx) - 1):
                F.append([idx[0], idx[k], idx[k + 1]])
    return np.array(V, np.float64).reshape(-1, 3), np.array(F, np.int64).reshape(-1, 3)


SAMPLE = """# a comment
mtllib house.mtl
o roof
v 0 0 0
v 1.0 0.0 0.0   # trailing comment
v 1 1 0 1.0
v\t0\t1\t0
vt 0.5 0.5
vn 0 0 1
usemtl tin
s off
f 1 2 3
f 1/1/1 3/1/1 4/1/1
g walls
v -1e-3 2.5E+2 +3.25
v 0.1 0.2 0.3\r
f -2 -1 1 2\r
f 2//1 3//1 5//1 6//1 4//1
l 1 2
"""


def test_statements_fans_and_index_forms():
    got = meshio.parse_obj(SAMPLE.encode())
    V, F = _plain_obj(SAMPLE)
    assert got.vertices.dtype == np.float64 and got.faces.dtype == np.int32
    np.testing.assert_array_equal(got.vertices, V)
    np.testing.assert_array_equal(got.faces, F)
    assert got.faces.tolist() == [[0, 1, 2], [0, 2, 3], [4, 5, 0], [4, 0, 1], [1, 2, 4], [1, 4, 5], [1, 5, 3]]
    f32 = meshio.parse_obj(SAMPLE.encode(), dtype=np.float32)
    np.testing.assert_array_equal(f32.vertices, V.astype(np.float32))  # double, then rounded once


def test_round_trip_is_exact_and_thread_count_free():
    V, F = mg.displaced_icosphere(4, 3)
    rng = np.random.default_rng(0)
    V = (V * rng.uniform(0.1, 1e4, size=(1, 3))).astype(np.float32)
    V[:7] = [[0, -0.0, 1e-38], [3.4e38, -1.5e-45, 1], [0.1, 0.2, 0.3], [1 / 3, 2 / 3, -7], [1e-7, 1e7, 123456.7],
             [np.float32(np.pi), -np.float32(np.e), 2 ** -20], [65504, -65504, 1e-30]]
    text = meshio.format_obj(V, F)
    for threads in (1, 3, 0):
        assert meshio.format_obj(V, F, n_threads=threads) == text
        back = meshio.parse_obj(text, n_threads=threads, dtype=np.float32)
        np.testing.assert_array_equal(back.vertices.view(np.uint32), V.view(np.uint32))
        np.testing.assert_array_equal(back.faces, F.astype(np.int32))
    pv, pf = _plain_obj(text.decode())
    np.testing.assert_array_equal(pv.astype(np.float32), V)
    np.testing.assert_array_equal(pf, F)


def test_large_text_splits_across_threads():
    """A text long enough for many chunks, with negative indices that refer
    back across chunk boundaries."""
    rng = np.random.default_rng(1)
    n = 60_000
    lines = []
    for k in range(n):
        lines.append("v %.9g %.9g %.9g" % tuple(rng.standard_normal(3)))
        if k >= 3:
            lines.append("f -1 -3 -4" if k % 2 else "f %d %d %d" % (k + 1, k, k - 2))
    text = ("\n".join(lines) + "\n").encode()
    assert len(text) > 3 << 20
    V, F = _plain_obj(text.decode())
    for threads in (1, 2, 8):
        got = meshio.parse_obj(text, n_threads=threads)
        np.testing.assert_array_equal(got.vertices, V)
        np.testing.assert_array_equal(got.faces, F)


@pytest.mark.parametrize("bad, line", [
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 4\n", 4),      # index past the vertices
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 0 1 2\n", 4),      # index 0
    ("v 0 0 0\nv 1 0 0\nf -3 1 2\n", 3),              # relative index before the first vertex
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2\n", 4),        # two corners
    ("v 0 0 0\nv 1 x 0\n", 2),                        # malformed coordinate
    ("v 0 0\n", 1),                                   # missing coordinate
    ("v 0 0 0\nv 1 0 0\nv 0 1 0\nf 1 2 3q\n", 4),     # malformed index
])
def test_malformed_statements_raise_with_their_line(bad, line):
    with pytest.raises(ValueError, match=f"OBJ line {line}:"):
        meshio.parse_obj(bad.encode())


def test_empty_and_statement_free_texts():
    for text in (b"", b"# nothing\n\nvn 0 0 1\n"):
        m = meshio.parse_obj(text)
        assert m.vertices.shape == (0, 3) and m.faces.shape == (0, 3)
    assert meshio.format_obj(np.zeros((0, 3)), np.zeros((0, 3))) == b""


def test_format_rejects_bad_indices():
    from pamo_b200._lib import PamoError

    with pytest.raises(PamoError):
        meshio.format_obj(np.zeros((3, 3)), np.array([[0, 1, 3]]))


def test_files(tmp_path):
    V, F = mg.displaced_icosphere(2, 1)
    p = str(tmp_path / "m.obj")
    meshio.save_obj(p, V, F)
    m = meshio.load_obj(p)  # float64: the decimals written, which round back to the float32 values
    np.testing.assert_array_equal(m.vertices.astype(np.float32), V.astype(np.float32))
    np.testing.assert_array_equal(m.faces, F)


def test_cli_passes_the_stage_switches(tmp_path, monkeypatch):
    """The command line mirrors example.py's options: --disable_stage1 /
    --disable_stage3 reach PaMO, the mesh is loaded and the result saved."""
    import sys
    import types

    import pamo_b200
    from pamo_b200 import cli

    seen = {}

    class FakePaMO:
        def __init__(self, mesh, use_stage1=True, use_stage3=True):
            seen["stages"] = (use_stage1, use_stage3)
            self.mesh = mesh

        def run(self, points, triangles, ratio, min_verts):
            seen["ratio"], seen["min_verts"] = ratio, min_verts
            return self.mesh.vertices.astype(np.float32), self.mesh.faces

    fake_torch = types.SimpleNamespace(from_numpy=lambda a: types.SimpleNamespace(
        float=lambda: types.SimpleNamespace(cuda=lambda: a), int=lambda: types.SimpleNamespace(cuda=lambda: a)))
    monkeypatch.setitem(sys.modules, "torch", fake_torch)
    monkeypatch.setattr(pamo_b200, "PaMO", FakePaMO)
    V, F = mg.displaced_icosphere(1, 0)
    src, dst = str(tmp_path / "in.obj"), str(tmp_path / "out.obj")
    meshio.save_obj(src, V, F)
    assert cli.main(["-i", src, "-o", dst, "-r", "0.2", "--disable_stage1"]) == 0
    assert seen == {"stages": (False, True), "ratio": 0.2, "min_verts": 0}
    assert cli.main(["-i", src, "-o", dst, "--disable_stage3", "-mv", "5"]) == 0
    assert seen["stages"] == (True, False) and seen["min_verts"] == 5
    np.testing.assert_array_equal(meshio.load_mesh(dst).faces, F)


def _ply_bytes(V, polys, fmt):
    """A PLY file with extra vertex properties (normal, colour), a face
    property before the index list, and an extra element after the faces."""
    import struct

    head = [
        "ply", f"format {fmt} 1.0", "comment made by the test", f"element vertex {len(V)}",
        "property double x", "property float nx", "property double y", "property double z", "property uchar red",
        f"element face {len(polys)}", "property int flags", "property list uchar uint vertex_indices",
        "element edge 1", "property list int int vertex_index", "end_header",
    ]
    out = ("\n".join(head) + "\n").encode()
    if fmt == "ascii":
        rows = [f"{float(x)!r} 0.5 {float(y)!r} {float(z)!r} 200" for x, y, z in V]
        rows += [" ".join(["7", str(len(p))] + [str(i) for i in p]) for p in polys]
        rows += ["2 0 1"]
        return out + ("\n".join(rows) + "\n").encode()
    e = "<" if fmt == "binary_little_endian" else ">"
    body = b"".join(struct.pack(e + "dfddB", x, 0.5, y, z, 200) for x, y, z in V)
    body += b"".join(struct.pack(e + "iB%dI" % len(p), 7, len(p), *p) for p in polys)
    body += struct.pack(e + "iii", 2, 0, 1)
    return out + body


@pytest.mark.parametrize("fmt", ["ascii", "binary_little_endian", "binary_big_endian"])
def test_ply_formats_properties_and_fans(fmt):
    rng = np.random.default_rng(2)
    V = rng.standard_normal((9, 3))
    polys = [[0, 1, 2], [2, 3, 4, 5], [5, 6, 7, 8, 0]]
    m = meshio.parse_ply(_ply_bytes(V, polys, fmt))
    np.testing.assert_array_equal(m.vertices, V)  # doubles as stored
    assert m.faces.tolist() == [[0, 1, 2], [2, 3, 4], [2, 4, 5], [5, 6, 7], [5, 7, 8], [5, 8, 0]]
    m32 = meshio.parse_ply(_ply_bytes(V, polys, fmt), dtype=np.float32)
    np.testing.assert_array_equal(m32.vertices, V.astype(np.float32))


def test_ply_round_trip_and_errors(tmp_path):
    V, F = mg.displaced_icosphere(3, 2)
    V = V.astype(np.float32)
    p = str(tmp_path / "m.ply")
    meshio.save_mesh(p, V, F)
    m = meshio.load_mesh(p, dtype=np.float32)
    np.testing.assert_array_equal(m.vertices.view(np.uint32), V.view(np.uint32))
    np.testing.assert_array_equal(m.faces, F)
    data = meshio.format_ply(V, F)
    with pytest.raises(ValueError):
        meshio.parse_ply(data[:-5])  # truncated
    with pytest.raises(ValueError):
        meshio.parse_ply(_ply_bytes(np.zeros((3, 3)), [[0, 1, 3]], "ascii"))  # index past the vertices
    with pytest.raises(ValueError):
        meshio.parse_ply(b"ply\nformat ascii 1.0\nelement vertex 1\nproperty float x\nend_header\n1\n")  # no y, z
    with pytest.raises(ValueError):
        meshio.parse_ply(b"solid stl\n")


def test_ply_element_without_properties_is_skipped_at_once():
    """A header element with a huge count and no properties occupies no body
    bytes; the reader must not walk its count."""
    import time

    hdr = (b"ply\nformat binary_little_endian 1.0\nelement empty 9000000000000000000\n"
           b"element vertex 3\nproperty float x\nproperty float y\nproperty float z\n"
           b"element face 1\nproperty list uchar int vertex_indices\nend_header\n")
    body = np.eye(3, dtype=np.float32).tobytes() + bytes([3]) + np.array([0, 1, 2], np.int32).tobytes()
    t0 = time.time()
    m = meshio.parse_ply(hdr + body)
    assert time.time() - t0 < 5.0
    np.testing.assert_array_equal(m.faces, [[0, 1, 2]])
