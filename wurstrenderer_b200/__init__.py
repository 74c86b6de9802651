"""B200-native `nextevent_path_tracer`: Python access to the C ABI.

The product is ``libwurst_b200.so`` (host C++ + sm_100a CUDA, declared in
``include/wurst_b200.h``) and the ``wurst_b200`` CLI, a drop-in for the
reference's ``--simple2parse`` / ``--jsimple2parse`` flow. This module is a
thin ctypes layer over that library for tests, the benchmark and scripting; it
mirrors the reference's entry points:

* :func:`Simple2Parser.Parse` -- ``Simple2Parser::Parse`` (src/sceneio/simple2parser.h:84-223):
  load a scene JSON, render every ``nextevent_path_tracer`` entry, write its PFM;
* :class:`Scene` -- a parsed, uploaded scene (``Simple2Parser::ParseScene`` + BVH build);
* :meth:`Scene.render` -- ``PathNeeRenderer::render`` (src/renderer/pathnextevent.h:152-191)
  returning the film image (base/spp + splat/(spp*W*H)) as an HxWx3 float64 array.

There is no CPU fallback: every call runs the CUDA kernels, and loading fails
loudly when the library has not been built or no GPU is present.
"""
from __future__ import annotations

import ctypes
import os

import numpy as np

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(PKG_DIR, "libwurst_b200.so")
CLI_PATH = os.path.join(PKG_DIR, "wurst_b200")

WR_OK = 0
_STATUS = {1: "invalid argument", 2: "i/o error", 3: "parse error", 4: "unsupported", 5: "cuda error",
           6: "out of memory", 7: "timeout"}


class WurstError(RuntimeError):
    def __init__(self, status, message):
        super().__init__("%s (status %d: %s)" % (message, status, _STATUS.get(status, "?")))
        self.status = status


class RenderDesc(ctypes.Structure):
    _fields_ = [("num_spp", ctypes.c_int), ("num_path_vertices", ctypes.c_int), ("seed", ctypes.c_uint),
                ("render_index", ctypes.c_int), ("queue_capacity", ctypes.c_int), ("grid_trace", ctypes.c_int),
                ("grid_shade", ctypes.c_int), ("use_graph", ctypes.c_int), ("profile", ctypes.c_int),
                ("trace_block", ctypes.c_int), ("integrator", ctypes.c_int), ("guiding", ctypes.c_int),
                ("guide_train_spp", ctypes.c_int), ("guide_pass_spp", ctypes.c_int), ("guide_batch", ctypes.c_int),
                ("guide_steps", ctypes.c_int), ("guide_clamp", ctypes.c_float), ("fetch_threshold", ctypes.c_int),
                ("max_iterations", ctypes.c_int), ("guide_lr", ctypes.c_float), ("reserved", ctypes.c_int * 1)]


class Job(ctypes.Structure):
    _fields_ = [("camera_json", ctypes.c_char_p), ("num_spp", ctypes.c_int), ("num_path_vertices", ctypes.c_int),
                ("seed", ctypes.c_uint), ("reserved", ctypes.c_int * 3)]


class RenderStats(ctypes.Structure):
    _fields_ = [("render_ms", ctypes.c_double), ("paths", ctypes.c_ulonglong), ("iterations", ctypes.c_ulonglong),
                ("max_shadow_queue", ctypes.c_uint), ("queue_capacity", ctypes.c_uint),
                ("grid_trace", ctypes.c_int), ("grid_shade", ctypes.c_int), ("trace_block", ctypes.c_int),
                ("kernel_launches", ctypes.c_ulonglong), ("kernel_ms", ctypes.c_double * 8),
                ("kernel_count", ctypes.c_ulonglong * 8), ("kernel_items", ctypes.c_ulonglong * 8),
                ("extend_node_visits", ctypes.c_ulonglong), ("extend_tri_tests", ctypes.c_ulonglong),
                ("shadow_node_visits", ctypes.c_ulonglong), ("shadow_tri_tests", ctypes.c_ulonglong),
                ("guide_records", ctypes.c_ulonglong), ("guide_steps", ctypes.c_ulonglong),
                ("guide_train_ms", ctypes.c_double), ("guide_loss", ctypes.c_double),
                ("guide_passes", ctypes.c_int), ("reserved_stats", ctypes.c_int)]


KERNELS = ["extend", "shade", "raygen", "shadow", "advance", "resolve", "guide", "train"]
GUIDE_PARAMS = 20480   # 5 layers x 64 x 64 FP32 weights, [layer][out][in]


class SceneInfo(ctypes.Structure):
    _fields_ = [("width", ctypes.c_int), ("height", ctypes.c_int), ("num_spp", ctypes.c_int),
                ("num_path_vertices", ctypes.c_int), ("num_triangles", ctypes.c_ulonglong),
                ("num_meshes", ctypes.c_int), ("num_lights", ctypes.c_int), ("has_envmap", ctypes.c_int),
                ("bvh_nodes", ctypes.c_int), ("bvh_depth", ctypes.c_int), ("bvh_sah_cost", ctypes.c_double),
                ("build_ms", ctypes.c_double), ("num_renders", ctypes.c_int), ("bvh_builder", ctypes.c_int),
                ("bvh_ms", ctypes.c_double)]


class SceneOptions(ctypes.Structure):
    _fields_ = [("bvh_builder", ctypes.c_int), ("max_leaf", ctypes.c_int), ("bvh_width", ctypes.c_int),
                ("sah_trav_cost_milli", ctypes.c_int), ("sah_patch_cost_milli", ctypes.c_int),
                ("reserved", ctypes.c_int * 3)]


BVH_HOST_SAH = 0
BVH_DEVICE_LBVH = 1


# every function the C ABI exports (include/wurst_b200.h)
EXPORTS = ["wr_scene_create", "wr_scene_create_ex", "wr_scene_create_from_json", "wr_scene_destroy", "wr_scene_inspect", "wr_scene_inspect_ex", "wr_scene_get_info",
           "wr_scene_set_camera_json", "wr_render", "wr_render_device", "wr_get_render_stats",
           "wr_trace_closest", "wr_trace_hits", "wr_trace_occluded", "wr_trace_stats", "wr_write_pfm", "wr_read_image", "wr_run_simple2",
           "wr_run_jsimple2", "wr_set_device", "wr_last_error", "wr_abi_version", "wr_render_device_noalloc", "wr_render_batch",
           "wr_render_batch_device", "wr_autotune", "wr_autotune_batch", "wr_guide_reset", "wr_guide_get_params", "wr_guide_set_params",
           "wr_guide_box", "wr_guide_eval", "wr_guide_gradient", "wr_guide_train"]

_lib = None


def load_library(path: str = LIB_PATH):
    """Loads libwurst_b200.so (built by ``wurstrenderer_b200.build``); raises if it is missing."""
    global _lib
    if _lib is not None:
        return _lib
    if not os.path.exists(path):
        raise WurstError(4, "libwurst_b200.so is not built (run python -m wurstrenderer_b200.build)")
    L = ctypes.CDLL(path)
    vp, cp, ip, fp = ctypes.c_void_p, ctypes.c_char_p, ctypes.c_int, ctypes.c_void_p
    L.wr_last_error.restype = ctypes.c_char_p
    L.wr_abi_version.restype = ctypes.c_int
    L.wr_scene_create.argtypes = [cp, ctypes.POINTER(vp)]
    L.wr_scene_create_from_json.argtypes = [cp, cp, ctypes.POINTER(vp)]
    L.wr_scene_create_ex.argtypes = [cp, ctypes.POINTER(SceneOptions), ctypes.POINTER(vp)]
    L.wr_scene_destroy.argtypes = [vp]
    L.wr_scene_destroy.restype = None
    L.wr_scene_get_info.argtypes = [vp, ctypes.POINTER(SceneInfo)]
    L.wr_scene_inspect.argtypes = [cp, ctypes.POINTER(SceneInfo)]
    L.wr_scene_inspect_ex.argtypes = [cp, ctypes.POINTER(SceneOptions), ctypes.POINTER(SceneInfo)]
    L.wr_scene_set_camera_json.argtypes = [vp, cp]
    L.wr_render.argtypes = [vp, ctypes.POINTER(RenderDesc), fp]
    L.wr_render_device.argtypes = [vp, ctypes.POINTER(RenderDesc), fp]
    L.wr_render_device_noalloc.argtypes = [vp, ctypes.POINTER(RenderDesc), fp]
    L.wr_render_batch.argtypes = [vp, ctypes.POINTER(Job), ip, ctypes.POINTER(RenderDesc), fp]
    L.wr_autotune.argtypes = [vp, ctypes.POINTER(RenderDesc), ip, ctypes.POINTER(RenderDesc),
                              ctypes.POINTER(ctypes.c_double)]
    L.wr_render_batch_device.argtypes = [vp, ctypes.POINTER(Job), ip, ctypes.POINTER(RenderDesc), fp]
    L.wr_autotune_batch.argtypes = [vp, ctypes.POINTER(Job), ip, ctypes.POINTER(RenderDesc), ctypes.POINTER(RenderDesc),
                                    ctypes.POINTER(ctypes.c_double)]
    L.wr_get_render_stats.argtypes = [vp, ctypes.POINTER(RenderStats)]
    L.wr_trace_closest.argtypes = [vp, fp, ip, fp, fp, fp, fp]
    L.wr_trace_hits.argtypes = [vp, fp, ip, fp, fp, fp, fp]
    L.wr_trace_occluded.argtypes = [vp, fp, ip, fp]
    L.wr_trace_stats.argtypes = [vp, fp, ip, ip, ctypes.POINTER(ctypes.c_ulonglong), ctypes.POINTER(ctypes.c_ulonglong)]
    L.wr_write_pfm.argtypes = [cp, fp, ip, ip]
    L.wr_read_image.argtypes = [cp, ctypes.POINTER(ctypes.c_int), ctypes.POINTER(ctypes.c_int), fp]
    L.wr_run_simple2.argtypes = [cp]
    L.wr_run_jsimple2.argtypes = [cp]
    L.wr_set_device.argtypes = [ip]
    L.wr_guide_reset.argtypes = [vp, ctypes.c_uint]
    L.wr_guide_get_params.argtypes = [vp, fp]
    L.wr_guide_set_params.argtypes = [vp, fp]
    L.wr_guide_box.argtypes = [vp, fp, fp]
    L.wr_guide_eval.argtypes = [vp, fp, ip, fp]
    L.wr_guide_gradient.argtypes = [vp, fp, ip, ctypes.c_float, fp, ctypes.POINTER(ctypes.c_double)]
    L.wr_guide_train.argtypes = [vp, fp, ip, ip, ip, ctypes.c_float, fp]
    _lib = L
    return L


def _check(rc):
    if rc != WR_OK:
        raise WurstError(rc, load_library().wr_last_error().decode(errors="replace"))


def _ptr(a):
    return ctypes.c_void_p(a.ctypes.data) if isinstance(a, np.ndarray) else ctypes.c_void_p(int(a))


class Scene:
    """A simple2 scene parsed, BVH-built and uploaded to the current CUDA device."""

    def __init__(self, handle):
        self._h = handle

    @classmethod
    def from_file(cls, json_path: str, bvh_builder: int = BVH_HOST_SAH, max_leaf: int = 0,
                  bvh_width: int = 0, sah_trav_cost: float = 0.0, sah_patch_cost: float = 0.0) -> "Scene":
        """bvh_width: 2 binary BVH, 8 compressed 8-wide BVH, 0 the library default.
        sah_trav_cost / sah_patch_cost: host SAH cost of a traversal step / of a Phong patch test,
        relative to a triangle test (0: the library defaults, 1 and 16)."""
        L = load_library()
        h = ctypes.c_void_p()
        opts = SceneOptions()
        opts.bvh_builder = int(bvh_builder)
        opts.max_leaf = int(max_leaf)
        opts.bvh_width = int(bvh_width)
        opts.sah_trav_cost_milli = int(round(float(sah_trav_cost) * 1000))
        opts.sah_patch_cost_milli = int(round(float(sah_patch_cost) * 1000))
        _check(L.wr_scene_create_ex(os.fspath(json_path).encode(), ctypes.byref(opts), ctypes.byref(h)))
        return cls(h)

    @classmethod
    def from_json(cls, json_text: str, base_dir: str = ".") -> "Scene":
        L = load_library()
        h = ctypes.c_void_p()
        _check(L.wr_scene_create_from_json(json_text.encode(), base_dir.encode(), ctypes.byref(h)))
        return cls(h)

    def close(self):
        if self._h:
            load_library().wr_scene_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def info(self) -> dict:
        inf = SceneInfo()
        _check(load_library().wr_scene_get_info(self._h, ctypes.byref(inf)))
        return {k: getattr(inf, k) for k, _ in SceneInfo._fields_}

    def set_camera(self, camera_json: str) -> None:
        _check(load_library().wr_scene_set_camera_json(self._h, camera_json.encode()))

    @staticmethod
    def _desc(spp, num_path_vertices, seed, render_index, queue_capacity, grid_trace, grid_shade, use_graph,
              profile=0, trace_block=None, integrator=None, guiding=0, guide_train_spp=None, guide_pass_spp=None,
              guide_batch=None, guide_steps=None, guide_clamp=None, fetch_threshold=None, max_iterations=None,
              guide_lr=None):
        d = RenderDesc()
        d.num_spp = int(spp or 0)
        d.num_path_vertices = int(num_path_vertices or 0)
        d.seed = int(seed) & 0xFFFFFFFF
        d.render_index = int(render_index)
        d.queue_capacity = int(queue_capacity or 0)
        d.grid_trace = int(grid_trace or 0)
        d.grid_shade = int(grid_shade or 0)
        d.use_graph = 1 if use_graph else 0
        d.profile = int(profile)
        d.trace_block = int(trace_block or 0)
        d.integrator = {None: 0, "nextevent_path_tracer": 1, "primitive_path_tracer": 2,
                        "light_splatting": 3}[integrator]
        d.guiding = {False: 0, True: 1, 0: 0, 1: 1, 2: 2, "off": 0, "train": 1, "frozen": 2}[guiding]
        d.guide_train_spp = int(guide_train_spp or 0)
        d.guide_pass_spp = int(guide_pass_spp or 0)
        d.guide_batch = int(guide_batch or 0)
        d.guide_steps = int(guide_steps or 0)
        d.guide_clamp = float(guide_clamp or 0.0)
        d.fetch_threshold = int(fetch_threshold or 0)
        d.max_iterations = int(max_iterations or 0)
        d.guide_lr = float(guide_lr or 0.0)
        return d

    def render(self, spp=None, num_path_vertices=None, seed=0, render_index=0, queue_capacity=None,
               grid_trace=None, grid_shade=None, use_graph=True, out=None, profile=0, trace_block=None,
               integrator=None, guiding=0, guide_train_spp=None, guide_pass_spp=None,
               guide_batch=None, guide_steps=None, guide_clamp=None, fetch_threshold=None,
               max_iterations=None, guide_lr=None) -> np.ndarray:
        """Renders into host memory; returns an (H, W, 3) float64 image (row 0 = top).
        integrator: None (the render entry's), "nextevent_path_tracer", "primitive_path_tracer" or
        "light_splatting".
        guiding: 0 / "off" (plain NEE+MIS), 1 / "train" (learned proposal trained online on the first
        guide_train_spp samples, default 32), 2 / "frozen" (the scene's current network, no training);
        guide_lr: the Adam learning rate of the training (default 1e-3).
        max_iterations: lowers the wavefront's iteration bound (debugging; a render that needs more
        raises WurstError with status WR_ERR_TIMEOUT)."""
        inf = self.info
        if out is None:
            out = np.empty((inf["height"], inf["width"], 3), np.float64)
        d = self._desc(spp, num_path_vertices, seed, render_index, queue_capacity, grid_trace, grid_shade, use_graph,
                       profile, trace_block, integrator, guiding, guide_train_spp, guide_pass_spp, guide_batch,
                       guide_steps, guide_clamp, fetch_threshold, max_iterations, guide_lr)
        _check(load_library().wr_render(self._h, ctypes.byref(d), _ptr(out)))
        return out

    def render_device(self, out_device_ptr: int, spp=None, num_path_vertices=None, seed=0, render_index=0,
                      queue_capacity=None, grid_trace=None, grid_shade=None, use_graph=True, profile=0,
                      trace_block=None, guiding=0, guide_steps=None, fetch_threshold=None) -> None:
        """Renders into device memory at `out_device_ptr` (W*H*3 doubles)."""
        d = self._desc(spp, num_path_vertices, seed, render_index, queue_capacity, grid_trace, grid_shade, use_graph,
                       profile, trace_block, None, guiding, None, None, None, guide_steps, None, fetch_threshold)
        _check(load_library().wr_render_device(self._h, ctypes.byref(d), ctypes.c_void_p(int(out_device_ptr))))

    def autotune(self, probe_spp=4, **base):
        """Runs the library's autotuner; returns (settings dict, ms per probe render)."""
        d0 = self._desc(None, None, 0, 0, base.get("queue_capacity"), base.get("grid_trace"), base.get("grid_shade"),
                        base.get("use_graph", True), 0, base.get("trace_block"))
        best = RenderDesc()
        ms = ctypes.c_double(0.0)
        _check(load_library().wr_autotune(self._h, ctypes.byref(d0), int(probe_spp), ctypes.byref(best), ctypes.byref(ms)))
        keys = ("queue_capacity", "grid_trace", "grid_shade", "trace_block", "use_graph", "fetch_threshold")
        return {k: getattr(best, k) for k in keys}, ms.value

    def _job_array(self, jobs):
        import json as _json
        n = len(jobs)
        arr = (Job * n)()
        keep = []
        shapes = []
        for i, j in enumerate(jobs):
            cam = j.get("camera")
            if isinstance(cam, dict):
                cam = _json.dumps(cam)
            if cam is not None:
                keep.append(cam.encode())
                arr[i].camera_json = keep[-1]
                c = _json.loads(cam)
                shapes.append((int(c["resolution"][1]), int(c["resolution"][0])))
            else:
                inf = self.info
                shapes.append((inf["height"], inf["width"]))
            arr[i].num_spp = int(j.get("num_spp", 0))
            arr[i].num_path_vertices = int(j.get("num_path_vertices", 0))
            arr[i].seed = int(j.get("seed", 0)) & 0xFFFFFFFF
        return arr, keep, shapes

    def autotune_batch(self, jobs, **base):
        """The autotuner timed on render_batch over `jobs` (a probe subset of a batch); returns
        (settings dict, ms per probe batch)."""
        arr, keep, _ = self._job_array(jobs)
        d0 = self._desc(None, None, 0, 0, base.get("queue_capacity"), base.get("grid_trace"), base.get("grid_shade"),
                        base.get("use_graph", True), 0, base.get("trace_block"))
        best = RenderDesc()
        ms = ctypes.c_double(0.0)
        _check(load_library().wr_autotune_batch(self._h, arr, len(jobs), ctypes.byref(d0), ctypes.byref(best),
                                                ctypes.byref(ms)))
        del keep
        keys = ("queue_capacity", "grid_trace", "grid_shade", "trace_block", "use_graph", "fetch_threshold")
        return {k: getattr(best, k) for k in keys}, ms.value

    def render_batch(self, jobs, queue_capacity=None, grid_trace=None, grid_shade=None, use_graph=True, profile=0,
                     trace_block=None, fetch_threshold=None):
        """jobs: list of dicts {camera (dict or JSON text), num_spp, num_path_vertices, seed}.
        Returns one (H, W, 3) float64 image per job, rendered in one wavefront."""
        n = len(jobs)
        arr, keep, shapes = self._job_array(jobs)
        total = sum(h * w for h, w in shapes)
        out = np.empty(total * 3, np.float64)
        d = self._desc(None, None, 0, 0, queue_capacity, grid_trace, grid_shade, use_graph, profile, trace_block,
                       fetch_threshold=fetch_threshold)
        _check(load_library().wr_render_batch(self._h, arr, n, ctypes.byref(d), _ptr(out)))
        imgs, off = [], 0
        for h, w in shapes:
            imgs.append(out[off * 3:(off + h * w) * 3].reshape(h, w, 3))
            off += h * w
        return imgs

    @property
    def stats(self) -> dict:
        st = RenderStats()
        _check(load_library().wr_get_render_stats(self._h, ctypes.byref(st)))
        out = {}
        for k, _ in RenderStats._fields_:
            v = getattr(st, k)
            out[k] = list(v) if isinstance(v, ctypes.Array) else v
        return out

    # ---- learned guiding proposal ----
    def guide_reset(self, seed=0) -> None:
        _check(load_library().wr_guide_reset(self._h, int(seed) & 0xFFFFFFFF))

    def guide_params(self) -> np.ndarray:
        """FP32 master weights, shape (5, 64, 64) [layer][out][in]."""
        w = np.empty(GUIDE_PARAMS, np.float32)
        _check(load_library().wr_guide_get_params(self._h, _ptr(w)))
        return w.reshape(5, 64, 64)

    def guide_set_params(self, w) -> None:
        w = np.ascontiguousarray(w, np.float32).reshape(-1)
        if w.size != GUIDE_PARAMS:
            raise ValueError("expected %d weights" % GUIDE_PARAMS)
        _check(load_library().wr_guide_set_params(self._h, _ptr(w)))

    def guide_box(self):
        lo = np.empty(3, np.float32)
        inv = np.empty(3, np.float32)
        _check(load_library().wr_guide_box(self._h, _ptr(lo), _ptr(inv)))
        return lo, inv

    def guide_eval(self, rows):
        """rows (n, 9) [position, normal, outgoing] -> (axis (n, 8, 3), sharpness (n, 8), weight (n, 8))."""
        rows = np.ascontiguousarray(rows, np.float32)
        n = rows.shape[0]
        out = np.empty((n, 40), np.float32)
        _check(load_library().wr_guide_eval(self._h, _ptr(rows), n, _ptr(out)))
        lob = out[:, :32].reshape(n, 8, 4)
        return lob[..., :3], lob[..., 3], out[:, 32:]

    def guide_gradient(self, records, c_max=100.0):
        """records (n, 20) -> (gradient (5, 64, 64), summed loss)."""
        records = np.ascontiguousarray(records, np.float32)
        g = np.empty(GUIDE_PARAMS, np.float32)
        loss = ctypes.c_double(0.0)
        _check(load_library().wr_guide_gradient(self._h, _ptr(records), records.shape[0], float(c_max), _ptr(g),
                                                ctypes.byref(loss)))
        return g.reshape(5, 64, 64), loss.value

    def guide_train(self, records, steps, batch=65536, lr=1e-3):
        """Adam steps on the records; returns each step's mean loss."""
        records = np.ascontiguousarray(records, np.float32)
        losses = np.zeros(int(steps), np.float64)
        _check(load_library().wr_guide_train(self._h, _ptr(records), records.shape[0], int(steps), int(batch),
                                             float(lr), _ptr(losses)))
        return losses

    def trace_closest(self, rays: np.ndarray):
        """rays (n, 8) float32 [ox, oy, oz, tnear, dx, dy, dz, tfar] -> (geom_id, prim_id, t, uv)."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        g = np.empty(n, np.int32); p = np.empty(n, np.int32)
        t = np.empty(n, np.float32); uv = np.empty((n, 2), np.float32)
        _check(load_library().wr_trace_closest(self._h, _ptr(rays), n, _ptr(g), _ptr(p), _ptr(t), _ptr(uv)))
        return g, p, t, uv

    def trace_hits(self, rays: np.ndarray):
        """Closest hits with the unit geometry normal: (geom_id, prim_id, t, normal (n, 3))."""
        rays = np.ascontiguousarray(rays, np.float32)
        n = rays.shape[0]
        g = np.empty(n, np.int32); p = np.empty(n, np.int32)
        t = np.empty(n, np.float32); nrm = np.empty((n, 3), np.float32)
        _check(load_library().wr_trace_hits(self._h, _ptr(rays), n, _ptr(g), _ptr(p), _ptr(t), _ptr(nrm)))
        return g, p, t, nrm

    def trace_occluded(self, rays: np.ndarray):
        rays = np.ascontiguousarray(rays, np.float32)
        occ = np.empty(rays.shape[0], np.int32)
        _check(load_library().wr_trace_occluded(self._h, _ptr(rays), rays.shape[0], _ptr(occ)))
        return occ

    def trace_stats(self, rays: np.ndarray, any_hit=False):
        """Total inner-node visits and triangle tests for a ray batch."""
        rays = np.ascontiguousarray(rays, np.float32)
        nv, nt = ctypes.c_ulonglong(0), ctypes.c_ulonglong(0)
        _check(load_library().wr_trace_stats(self._h, _ptr(rays), rays.shape[0], 1 if any_hit else 0,
                                             ctypes.byref(nv), ctypes.byref(nt)))
        return int(nv.value), int(nt.value)


def set_device(device: int) -> None:
    """Selects the CUDA device the library uses on this thread."""
    _check(load_library().wr_set_device(int(device)))


def inspect_scene(json_path: str, max_leaf: int = 0, bvh_width: int = 0, sah_trav_cost: float = 0.0) -> dict:
    """Host-only scene validation (parse + host SAH BVH build, no GPU): returns the scene info.
    The build options mean what they mean for Scene.from_file."""
    inf = SceneInfo()
    opts = SceneOptions()
    opts.bvh_builder = BVH_HOST_SAH
    opts.max_leaf = int(max_leaf)
    opts.bvh_width = int(bvh_width)
    opts.sah_trav_cost_milli = int(round(float(sah_trav_cost) * 1000))
    _check(load_library().wr_scene_inspect_ex(os.fspath(json_path).encode(), ctypes.byref(opts), ctypes.byref(inf)))
    return {k: getattr(inf, k) for k, _ in SceneInfo._fields_}


class Simple2Parser:
    """The reference's scene-JSON entry point (src/sceneio/simple2parser.h)."""

    @staticmethod
    def Parse(scene_json_path: str) -> None:
        _check(load_library().wr_run_simple2(os.fspath(scene_json_path).encode()))

    @staticmethod
    def ParseJson(json_text: str) -> None:
        _check(load_library().wr_run_jsimple2(json_text.encode()))


def write_pfm(path: str, image: np.ndarray) -> None:
    """PFM in the reference's layout (rows bottom-to-top, little-endian float RGB)."""
    img = np.ascontiguousarray(image, np.float64)
    _check(load_library().wr_write_pfm(os.fspath(path).encode(), _ptr(img), img.shape[1], img.shape[0]))


def read_image(path: str) -> np.ndarray:
    """Reads a .pfm / .hdr / .exr image as the scene loader reads environment maps:
    (H, W, 3) float32, row 0 = top (FimageIo::Load, src/common/floatimage.h:379-404)."""
    L = load_library()
    w, h = ctypes.c_int(0), ctypes.c_int(0)
    _check(L.wr_read_image(os.fspath(path).encode(), ctypes.byref(w), ctypes.byref(h), None))
    out = np.empty((h.value, w.value, 3), np.float32)
    _check(L.wr_read_image(os.fspath(path).encode(), ctypes.byref(w), ctypes.byref(h), _ptr(out)))
    return out


def read_pfm(path: str) -> np.ndarray:
    """Reads a PFM into an (H, W, 3) float32 array, row 0 = top."""
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
