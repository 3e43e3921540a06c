"""Wavefront OBJ and Stanford PLY in and out, on the host, through
libpamo_b200.so (``pamo_obj_parse`` / ``pamo_obj_format``, ``pamo_ply_parse`` /
``pamo_ply_format``): the mesh loading and saving that the reference's
example.py:24-43 does with trimesh.

    mesh = load_mesh("in.obj")           # Mesh(vertices float64 [n,3], faces int32 [m,3]); .obj or .ply
    save_mesh("out.ply", verts, faces)

``Mesh`` has ``.vertices`` and ``.faces``, so it can be passed to ``PaMO`` as
the input mesh.
"""
from __future__ import annotations

import ctypes
from typing import NamedTuple

import numpy as np

from . import _lib


class Mesh(NamedTuple):
    vertices: np.ndarray  # float64 (or float32) [n, 3]
    faces: np.ndarray  # int32 [m, 3]


def _ptr(a: np.ndarray) -> ctypes.c_void_p:
    return ctypes.c_void_p(a.ctypes.data if a.size else 0)


def parse_obj(text: bytes, n_threads: int = 0, dtype=np.float64) -> Mesh:
    """OBJ text to (vertices [n,3] of `dtype`, float64 as trimesh loads them or
    float32 as `.float()` rounds those, faces int32 [m,3]); polygons are split
    into fans.  Raises ValueError naming the line of a malformed `v` / `f`
    statement or an index outside the vertices."""
    dtype = np.dtype(dtype)
    if dtype not in (np.float32, np.float64):
        raise ValueError("dtype must be float32 or float64")
    buf = np.frombuffer(text, dtype=np.uint8) if len(text) else np.zeros(0, np.uint8)
    L = _lib.lib()
    nv, nt, err = ctypes.c_longlong(), ctypes.c_longlong(), ctypes.c_longlong()
    args = (ctypes.byref(nv), ctypes.byref(nt), ctypes.byref(err))
    rc = L.pamo_obj_parse(_ptr(buf), len(buf), None, None, 0, None, 0, n_threads, *args)
    if rc == 6:  # sized: allocate and parse
        V = np.empty((nv.value, 3), dtype)
        F = np.empty((nt.value, 3), np.int32)
        v32, v64 = (_ptr(V), None) if dtype == np.float32 else (None, _ptr(V))
        rc = L.pamo_obj_parse(_ptr(buf), len(buf), v32, v64, nv.value, _ptr(F), nt.value, n_threads, *args)
    else:
        V = np.zeros((0, 3), dtype)
        F = np.zeros((0, 3), np.int32)
    if rc == 1 and err.value >= 0:
        line = text.count(b"\n", 0, err.value) + 1
        end = text.find(b"\n", err.value)
        raise ValueError(f"OBJ line {line}: {text[err.value:end if end >= 0 else None][:80]!r}")
    _lib.check("pamo_obj_parse", rc)
    return Mesh(V, F)


def load_obj(path: str, n_threads: int = 0, dtype=np.float64) -> Mesh:
    with open(path, "rb") as fh:
        return parse_obj(fh.read(), n_threads, dtype)


def format_obj(vertices, faces, n_threads: int = 0) -> bytes:
    """Vertices and triangles as OBJ text: `v x y z` in the shortest form that
    reads back as the same float32, then `f a b c` (1-based)."""
    V = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32).reshape(-1, 3))
    F = np.ascontiguousarray(np.asarray(faces, dtype=np.int32).reshape(-1, 3))
    L = _lib.lib()
    n = ctypes.c_longlong()
    # longest lines: "v" + 3 x (" " + 15 characters of a float) + "\n", "f" + 3 x (" " + 10 digits) + "\n"
    out = np.empty(len(V) * 50 + len(F) * 35 + 1, np.uint8)
    _lib.check("pamo_obj_format", L.pamo_obj_format(_ptr(V), len(V), _ptr(F), len(F), _ptr(out), out.size, n_threads,
                                                    ctypes.byref(n)))
    return out[:n.value].tobytes()


def save_obj(path: str, vertices, faces, n_threads: int = 0) -> None:
    data = format_obj(vertices, faces, n_threads)
    with open(path, "wb") as fh:
        fh.write(data)


def _sized_parse(fn, data: bytes, dtype, extra=()):
    dtype = np.dtype(dtype)
    if dtype not in (np.float32, np.float64):
        raise ValueError("dtype must be float32 or float64")
    buf = np.frombuffer(data, dtype=np.uint8) if len(data) else np.zeros(0, np.uint8)
    L = _lib.lib()
    nv, nt = ctypes.c_longlong(), ctypes.c_longlong()
    rc = getattr(L, fn)(_ptr(buf), len(buf), None, None, 0, None, 0, *extra, ctypes.byref(nv), ctypes.byref(nt))
    if rc == 6:
        V = np.empty((nv.value, 3), dtype)
        F = np.empty((nt.value, 3), np.int32)
        v32, v64 = (_ptr(V), None) if dtype == np.float32 else (None, _ptr(V))
        rc = getattr(L, fn)(_ptr(buf), len(buf), v32, v64, nv.value, _ptr(F), nt.value, *extra, ctypes.byref(nv),
                            ctypes.byref(nt))
    else:
        V = np.zeros((0, 3), dtype)
        F = np.zeros((0, 3), np.int32)
    if rc == 1:
        raise ValueError(f"{fn}: malformed or truncated mesh data, or a face index outside the vertices")
    _lib.check(fn, rc)
    return Mesh(V, F)


def parse_ply(data: bytes, dtype=np.float64) -> Mesh:
    """PLY (ASCII or binary) to (vertices [n,3] of `dtype`, faces int32 [m,3]);
    polygons are split into fans, other elements and properties skipped."""
    return _sized_parse("pamo_ply_parse", data, dtype)


def format_ply(vertices, faces) -> bytes:
    """Vertices and triangles as binary little-endian PLY."""
    V = np.ascontiguousarray(np.asarray(vertices, dtype=np.float32).reshape(-1, 3))
    F = np.ascontiguousarray(np.asarray(faces, dtype=np.int32).reshape(-1, 3))
    L = _lib.lib()
    n = ctypes.c_longlong()
    rc = L.pamo_ply_format(_ptr(V), len(V), _ptr(F), len(F), None, 0, ctypes.byref(n))
    if rc != 6:
        _lib.check("pamo_ply_format", rc)
    out = np.empty(n.value, np.uint8)
    _lib.check("pamo_ply_format", L.pamo_ply_format(_ptr(V), len(V), _ptr(F), len(F), _ptr(out), n.value,
                                                    ctypes.byref(n)))
    return out.tobytes()


def load_mesh(path: str, dtype=np.float64) -> Mesh:
    """A .obj or .ply file (by its extension)."""
    with open(path, "rb") as fh:
        data = fh.read()
    if path.lower().endswith(".ply"):
        return parse_ply(data, dtype)
    if path.lower().endswith(".obj"):
        return parse_obj(data, 0, dtype)
    raise ValueError(f"{path}: only .obj and .ply are read")


def save_mesh(path: str, vertices, faces) -> None:
    if path.lower().endswith(".ply"):
        data = format_ply(vertices, faces)
    elif path.lower().endswith(".obj"):
        data = format_obj(vertices, faces)
    else:
        raise ValueError(f"{path}: only .obj and .ply are written")
    with open(path, "wb") as fh:
        fh.write(data)
