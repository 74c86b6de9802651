"""wr_render_device_noalloc: the render entry point that allocates nothing.

Some callers may not allocate device memory once they are running -- an
application with a fixed device-memory budget (its own caching allocator owns
the rest of the GPU) or a latency-bound service that cannot accept the implicit
synchronisation cudaMalloc/cudaFree can cause. For them the wavefront and film
scratch live in one fixed 10 MiB static device array. This file runs last
(pytest collects it after the others) and checks, through the C ABI, that two
calls in a row give the image of the allocating entry point wr_render_device,
within the tolerance the other render tests use, and that films above the
fixed limit are rejected.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_scene

pytestmark = pytest.mark.gpu


def _render(lib, scene, fn, spp, seed, out):
    d = lib.RenderDesc()
    d.num_spp = spp
    d.seed = seed
    rc = fn(scene._h, ctypes.byref(d), ctypes.c_void_p(out.data_ptr()))
    assert rc == 0, lib.load_library().wr_last_error().decode()


def test_noalloc_matches_allocating_entry_point(wr_lib):
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("zoo")
    with wr_lib.Scene.from_file(path) as sc:
        inf = sc.info
        shape = (inf["height"], inf["width"], 3)
        ref = torch.empty(shape, dtype=torch.float64, device="cuda")
        _render(wr_lib, sc, L.wr_render_device, 64, 21, ref)
        outs = []
        for _ in range(2):   # the second call must not see the first call's leftovers
            o = torch.full(shape, -1.0, dtype=torch.float64, device="cuda")
            _render(wr_lib, sc, L.wr_render_device_noalloc, 64, 21, o)
            outs.append(o.cpu().numpy())
        assert sc.stats["queue_capacity"] == 32768
    ref = ref.cpu().numpy()
    assert np.isfinite(ref).all() and ref.mean() > 0
    for o in outs:
        assert np.allclose(o, ref, rtol=1e-9, atol=1e-12), np.abs(o - ref).max()


def test_noalloc_rejects_films_above_the_limit(wr_lib):
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        sc.set_camera('{"pos": [0,1,3.6], "lookat": [0,1,0], "up": [0,1,0], "fovy": 40, "resolution": [300, 300]}')
        out = torch.empty((300, 300, 3), dtype=torch.float64, device="cuda")
        d = wr_lib.RenderDesc()
        d.num_spp = 1
        rc = L.wr_render_device_noalloc(sc._h, ctypes.byref(d), ctypes.c_void_p(out.data_ptr()))
        assert rc == 1
        assert b"65536" in L.wr_last_error()
