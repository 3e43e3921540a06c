"""Batched and served stage-2 simplification on one GPU (libpamo_b200.so,
pamo_batch_* entry points).

The reference simplifies one mesh per ``CUDSP_Free`` object and round loop
(simp_cuda/pamo/__init__.py:122-190).  ``BatchEngine`` runs many meshes through
the same collapse rounds: the meshes are packed one after another into one set
of round buffers, every per-element kernel runs once per round for all of them,
and each mesh keeps its own parameters and the state the reference carries
from round to round.  A mesh leaves the batch when its own ``PaMO.run`` loop
would end (target reached, ``tolerance`` rounds without progress, ``iter``
rounds), and its result equals what ``pamo_stage2_run`` gives for it on a fresh
context.  Meshes submitted while others run are admitted between rounds,
whenever the packed capacity, the mesh count and the device-memory budget leave
room for them.

    eng = BatchEngine(max_faces=8_000_000)
    jobs = [eng.submit(V, F, ratio=0.01, min_verts=0) for V, F in meshes]
    eng.run()
    results = [eng.result(j) for j in jobs]
"""
from __future__ import annotations

import ctypes
import time

import numpy as np

from . import _lib
from ._lib import check

JOB_PENDING, JOB_RUNNING, JOB_DONE = 0, 1, 2


def target_faces(n_faces: int, ratio: float, min_verts: int = 10_000_000_000) -> int:
    """PaMO.run's target (simp_cuda/pamo/__init__.py:124)."""
    return max(int(ratio * n_faces), int(min_verts))


class BatchEngine:
    """One pamo_batch on one device and stream."""

    def __init__(self, device: int = 0, max_verts: int | None = None, max_faces: int = 8_000_000,
                 max_meshes: int = 256, memory_budget: int = 0, stream=None):
        import torch

        self.device = device
        if max_verts is None:
            max_verts = max_faces  # closed meshes have about half as many vertices as faces
        self._torch = torch
        self.stream = stream if stream is not None else torch.cuda.current_stream(device)
        h = ctypes.c_void_p()
        check("pamo_batch_create", _lib.lib().pamo_batch_create(
            int(device), int(max_verts), int(max_faces), int(max_meshes), int(memory_budget),
            ctypes.c_void_p(self.stream.cuda_stream), ctypes.byref(h)))
        self.handle = h
        self.max_faces = max_faces
        self.submitted: dict[int, dict] = {}

    def close(self):
        if getattr(self, "handle", None):
            _lib.lib().pamo_batch_destroy(self.handle)
            self.handle = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def submit(self, points, triangles, ratio: float | None = None, tolerance: int = 4, threshold: float = 1e-3,
               iter: int = 1000000, min_verts: int = 10_000_000_000, target: int | None = None) -> int:
        """Queues a mesh: numpy arrays (host) or CUDA tensors (device), points
        [n,3] float32, triangles [m,3] int32.  The target is PaMO.run's
        max(int(ratio * m), min_verts) unless given."""
        torch = self._torch
        if isinstance(points, torch.Tensor):
            if not (points.is_cuda and triangles.is_cuda):
                raise ValueError("tensors must be on the GPU")
            P = points.contiguous().to(torch.float32)
            T = triangles.contiguous().to(torch.int32)
            on_host = 0
            pp, tp = P.data_ptr(), T.data_ptr()
            keep = (P, T)
        else:
            P = np.ascontiguousarray(points, dtype=np.float32)
            T = np.ascontiguousarray(triangles, dtype=np.int32)
            on_host = 1
            pp, tp = P.ctypes.data, T.ctypes.data
            keep = (P, T)
        n, m = int(P.shape[0]), int(T.shape[0])
        if target is None:
            if ratio is None:
                raise ValueError("give ratio or target")
            target = target_faces(m, ratio, min_verts)
        job = ctypes.c_longlong()
        check("pamo_batch_submit", _lib.lib().pamo_batch_submit(
            self.handle, pp, tp, n, m, on_host, int(min(target, 2**62)), int(tolerance), float(threshold),
            int(min(iter, 2**31 - 1)), ctypes.byref(job)))
        del keep  # the engine has its own copy (device inputs are copied in stream order)
        self.submitted[job.value] = {"t_submit": time.perf_counter(), "faces": m}
        return job.value

    def step(self) -> tuple[int, int]:
        """One collapse round for every running mesh; returns (running, pending)."""
        r, p = ctypes.c_int(), ctypes.c_int()
        check("pamo_batch_step", _lib.lib().pamo_batch_step(self.handle, ctypes.byref(r), ctypes.byref(p)))
        return r.value, p.value

    def finished(self) -> list[int]:
        """Jobs that finished (or failed) during the last step()."""
        cap = 256
        while True:
            buf = (ctypes.c_longlong * cap)()
            n = _lib.lib().pamo_batch_finished(self.handle, buf, cap)
            if n < 0:
                raise _lib.PamoError("pamo_batch_finished", -n)
            if n <= cap:
                return list(buf[:n])
            cap = n

    def job(self, job: int) -> dict:
        st, n, m, rounds = ctypes.c_int(), ctypes.c_int(), ctypes.c_int(), ctypes.c_int()
        check("pamo_batch_job", _lib.lib().pamo_batch_job(self.handle, job, ctypes.byref(st), ctypes.byref(n),
                                                          ctypes.byref(m), ctypes.byref(rounds)))
        return {"state": st.value, "n_pts": n.value, "n_tris": m.value, "rounds": rounds.value}

    def done(self, job: int) -> bool:
        st = self.job(job)["state"]
        if st < 0:
            raise _lib.PamoError("pamo_batch job", -st)
        return st == JOB_DONE

    def result(self, job: int, release: bool = True):
        """(points [n,3] float32, faces [m,3] int32) numpy arrays of a finished job."""
        info = self.job(job)
        if info["state"] < 0:
            raise _lib.PamoError("pamo_batch job", -info["state"])
        if info["state"] != JOB_DONE:
            raise RuntimeError(f"job {job} is not finished")
        V = np.empty((info["n_pts"], 3), np.float32)
        F = np.empty((info["n_tris"], 3), np.int32)
        check("pamo_batch_fetch", _lib.lib().pamo_batch_fetch(self.handle, job, V.ctypes.data, F.ctypes.data, 1))
        if release:
            self.release(job)
        return V, F

    def release(self, job: int):
        check("pamo_batch_release", _lib.lib().pamo_batch_release(self.handle, job))
        self.submitted.pop(job, None)

    def stats(self) -> dict:
        a = (ctypes.c_longlong * 8)()
        check("pamo_batch_stats", _lib.lib().pamo_batch_stats(self.handle, a))
        keys = ["running", "pending", "packed_verts", "packed_faces", "bytes_held", "rounds_run", "max_faces",
                "memory_budget"]
        return dict(zip(keys, list(a)))

    def run(self, max_steps: int = 10_000_000):
        """Steps until nothing is running or pending."""
        for _ in range(max_steps):
            r, p = self.step()
            if r == 0 and p == 0:
                return
        raise RuntimeError("batch did not finish")


def simplify_many(meshes, ratio=None, tolerance=4, threshold=1e-3, iter=1000000, min_verts=10_000_000_000,
                  device=0, max_faces=None, max_meshes=256):
    """Stage-2 simplification of a list of (points, triangles) meshes in one
    batch; returns [(points, faces)] in input order.  `ratio` may be one value
    or one per mesh."""
    ratios = ratio if isinstance(ratio, (list, tuple)) else [ratio] * len(meshes)
    if max_faces is None:
        max_faces = max(sum(int(np.asarray(F).shape[0]) for _, F in meshes), 16)
    eng = BatchEngine(device=device, max_faces=max_faces, max_meshes=max_meshes)
    try:
        jobs = [eng.submit(V, F, r, tolerance, threshold, iter, min_verts) for (V, F), r in zip(meshes, ratios)]
        eng.run()
        return [eng.result(j) for j in jobs]
    finally:
        eng.close()
