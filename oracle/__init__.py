"""Test infrastructure only: Python access to the CPU oracle.

The oracle is the FP64 CPU restatement of the reference's
``nextevent_path_tracer`` (``oracle/nee_oracle.cpp``) and, where the
reference's sources are present (``REFERENCE_ROOT``), the reference's own
renderer code compiled from them (``oracle/_ref/wurst_ref``, built by
``oracle/Makefile``).
Only ``tests/``, ``__graft_entry__.smoke()`` and ``bench.py``'s CPU-baseline
leg use this module, always as the checker, never as the measured product.
"""
from __future__ import annotations

import ctypes
import json
import os
import subprocess

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "liboracle_nee.so")
REF_BIN = os.path.join(HERE, "_ref", "wurst_ref")
# where the reference's sources lie (read-only); only the build recipe reads them there
REFERENCE_ROOT = os.environ.get("WURST_REFERENCE_ROOT", "/root/reference")

_lib = None


def build(with_reference: bool = True) -> None:
    """Compiles the oracle (and the reference harness when the reference is present)."""
    subprocess.run(["make", "-s", "-C", HERE, "liboracle_nee.so"], check=True)
    if with_reference and os.path.isdir(REFERENCE_ROOT):
        subprocess.run(["make", "-s", "-C", HERE, "-j8", "ref", "REF=" + REFERENCE_ROOT], check=True)


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(LIB_PATH):
            build(with_reference=False)
        L = ctypes.CDLL(LIB_PATH)
        L.oracle_last_error.restype = ctypes.c_char_p
        L.oracle_scene_load.restype = ctypes.c_void_p
        L.oracle_scene_load.argtypes = [ctypes.c_char_p, ctypes.c_int]
        L.oracle_scene_free.argtypes = [ctypes.c_void_p]
        L.oracle_scene_info.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_set_camera_json.argtypes = [ctypes.c_void_p, ctypes.c_char_p]
        L.oracle_set_camera_json.restype = ctypes.c_int
        L.oracle_render.restype = ctypes.c_double
        L.oracle_render.argtypes = [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_uint,
                                    ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                    ctypes.c_int, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_trace_closest.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                           ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_trace_occluded.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]
        L.oracle_trace_occluded_bracket.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int, ctypes.c_double,
                                                    ctypes.c_void_p, ctypes.c_void_p]
        L.oracle_trace_hits.argtypes = [ctypes.c_void_p, ctypes.c_void_p, ctypes.c_int,
                                        ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p, ctypes.c_void_p]
        _lib = L
    return _lib


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


class OracleScene:
    """A scene JSON loaded by the oracle (FP64 restatement of the reference)."""

    def __init__(self, json_path: str, render_index: int = 0):
        L = lib()
        self._h = L.oracle_scene_load(json_path.encode(), render_index)
        if not self._h:
            raise RuntimeError("oracle: " + L.oracle_last_error().decode())
        info = np.zeros(4, np.int32)
        bbox = np.zeros(6, np.float64)
        counts = np.zeros(3, np.int32)
        L.oracle_scene_info(self._h, _ptr(info), _ptr(bbox), _ptr(counts))
        self.width, self.height, self.spp, self.num_path_vertices = (int(x) for x in info)
        self.bbox_lo, self.bbox_hi = bbox[:3].copy(), bbox[3:].copy()
        self.num_triangles, self.num_meshes, self.num_lights = (int(x) for x in counts)

    def close(self):
        if self._h:
            lib().oracle_scene_free(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_camera(self, camera: dict) -> None:
        if lib().oracle_set_camera_json(self._h, json.dumps(camera).encode()) != 0:
            raise RuntimeError("oracle: " + lib().oracle_last_error().decode())
        info = np.zeros(4, np.int32)
        L = lib()
        L.oracle_scene_info(self._h, _ptr(info), _ptr(np.zeros(6)), _ptr(np.zeros(3, np.int32)))
        self.width, self.height = int(info[0]), int(info[1])

    def render(self, spp=None, num_path_vertices=None, salt=0, crop=None, threads=0):
        """Returns (image HxWx3 float64, seconds, paths)."""
        spp = self.spp if spp is None else spp
        nv = self.num_path_vertices if num_path_vertices is None else num_path_vertices
        out = np.zeros((self.height, self.width, 3), np.float64)
        cx0, cy0, cx1, cy1 = crop if crop is not None else (0, 0, 0, 0)
        paths = ctypes.c_longlong(0)
        sec = lib().oracle_render(self._h, int(spp), int(nv), int(salt) & 0xFFFFFFFF, cx0, cy0, cx1, cy1,
                                  int(threads), _ptr(out), ctypes.byref(paths))
        return out, sec, int(paths.value)

    def trace_closest(self, rays: np.ndarray):
        """rays: (n, 8) float32 [ox, oy, oz, tnear, dx, dy, dz, tfar] -> geom, prim, t, uv."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        g = np.zeros(n, np.int32); p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32); uv = np.zeros((n, 2), np.float32)
        lib().oracle_trace_closest(self._h, _ptr(rays), n, _ptr(g), _ptr(p), _ptr(t), _ptr(uv))
        return g, p, t, uv

    def trace_hits(self, rays: np.ndarray):
        """rays: (n, 8) float32 -> geom, prim, t, Ng (n, 3) as Embree reports them to the reference."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        g = np.zeros(n, np.int32); p = np.zeros(n, np.int32)
        t = np.zeros(n, np.float32); ng = np.zeros((n, 3), np.float32)
        lib().oracle_trace_hits(self._h, _ptr(rays), n, _ptr(g), _ptr(p), _ptr(t), _ptr(ng))
        return g, p, t, ng

    def trace_occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.zeros(rays.shape[0], np.int32)
        lib().oracle_trace_occluded(self._h, _ptr(rays), rays.shape[0], _ptr(occ))
        return occ

    def trace_occluded_bracket(self, rays: np.ndarray, eps: float = 1e-5):
        """Bounds on a correct any-hit answer per ray: (blocked beyond doubt, possibly blocked),
        each (n,) bool. Triangles are tested in FP64 grown / shrunk by eps in barycentric
        coordinates, segment ends moved by eps * max(|t|, 1), grazing rays (|cos| < 1e-4) never
        count as blocked beyond doubt."""
        rays = np.ascontiguousarray(rays, np.float32)
        lo = np.zeros(rays.shape[0], np.int32)
        hi = np.zeros(rays.shape[0], np.int32)
        lib().oracle_trace_occluded_bracket(self._h, _ptr(rays), rays.shape[0], float(eps), _ptr(lo), _ptr(hi))
        return lo.astype(bool), hi.astype(bool)


def reference_available() -> bool:
    return os.path.exists(REF_BIN)


def run_reference(json_path, out_pfm, spp=None, vertices=None, salt=0, crop=None, serial=False,
                  raw=None, camera=None, timeout=None, env=None, threads=None):
    """Runs the reference's own renderer code (oracle/_ref) and returns its JSON report."""
    cmd = [REF_BIN, "render", json_path, out_pfm]
    if spp is not None:
        cmd += ["--spp", str(spp)]
    if vertices is not None:
        cmd += ["--vertices", str(vertices)]
    if salt:
        cmd += ["--salt", str(salt)]
    if crop is not None:
        cmd += ["--crop"] + [str(int(c)) for c in crop]
    if serial:
        cmd += ["--serial"]
    if threads is not None:
        cmd += ["--threads", str(int(threads))]
    if raw is not None:
        cmd += ["--raw", raw]
    if camera is not None:
        cmd += ["--camera", json.dumps(camera)]
    r = subprocess.run(cmd, capture_output=True, text=True, timeout=timeout, env=env)
    if r.returncode != 0:
        raise RuntimeError("wurst_ref failed: " + r.stderr.strip())
    return json.loads(r.stdout.strip().splitlines()[-1])


def run_reference_trace(json_path, rays, work_dir, timeout=None):
    """Closest hits and occlusion of `rays` ((n, 8) float32) through the reference's EmbreeAccel
    scene (``wurst_ref trace2``): geom, prim, t, Ng (n, 3), occluded."""
    rays = np.ascontiguousarray(rays, np.float32)
    rp = os.path.join(work_dir, "trace2_rays.f32")
    hp = os.path.join(work_dir, "trace2_hits.bin")
    rays.tofile(rp)
    r = subprocess.run([REF_BIN, "trace2", json_path, rp, hp], capture_output=True, text=True, timeout=timeout)
    if r.returncode != 0:
        raise RuntimeError("wurst_ref trace2 failed: " + r.stderr.strip())
    out = np.fromfile(hp, np.float32).reshape(-1, 8)
    ids = out[:, :2].copy().view(np.int32)
    return ids[:, 0], ids[:, 1], out[:, 2].copy(), out[:, 3:6].copy(), out[:, 6] > 0.5


def read_pfm(path):
    """Reads a PFM into an HxWx3 float32 array, row 0 = top (floatimage.h:238-277)."""
    with open(path, "rb") as f:
        head = f.readline().strip()
        dims = f.readline().split()
        scale = float(f.readline())
        w, h = int(dims[0]), int(dims[1])
        nc = 3 if head == b"PF" else 1
        data = np.frombuffer(f.read(), dtype="<f4" if scale < 0 else ">f4", count=w * h * nc)
    img = data.reshape(h, w, nc)[::-1]
    if nc == 1:
        img = np.repeat(img, 3, axis=2)
    return np.ascontiguousarray(img, np.float32)
