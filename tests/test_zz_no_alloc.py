"""wr_render_device_noalloc: the render entry point that allocates nothing.

Some callers may not allocate device memory once they are running -- an
application with a fixed device-memory budget (its own caching allocator owns
the rest of the GPU) or a latency-bound service that cannot accept the implicit
synchronisation cudaMalloc/cudaFree can cause. For them the wavefront and film
scratch live in one fixed 10 MiB static device array. This file runs last
(pytest collects it after the others) and checks, through the C ABI, that two
calls in a row give the image of the allocating entry point wr_render_device,
within the tolerance the other render tests use, for all three integrators
(chosen by the scene's render entry or by the request), that films above the
fixed limit and guided requests are rejected, and that a render stopped by its
iteration bound reports WR_ERR_TIMEOUT and leaves the array usable.
"""
import ctypes

import numpy as np
import pytest

from conftest import golden_scene

pytestmark = pytest.mark.gpu


def _desc(lib, spp, seed, integrator=0, guiding=0, max_iterations=0):
    d = lib.RenderDesc()
    d.num_spp = spp
    d.seed = seed
    d.integrator = integrator
    d.guiding = guiding
    d.max_iterations = max_iterations
    return d


def _render(lib, scene, fn, out, **kw):
    rc = fn(scene._h, ctypes.byref(_desc(lib, **kw)), ctypes.c_void_p(out.data_ptr()))
    assert rc == 0, lib.load_library().wr_last_error().decode()


def _stats(lib, scene):
    st = lib.RenderStats()
    assert lib.load_library().wr_get_render_stats(scene._h, ctypes.byref(st)) == 0
    return st


# (fixture, desc.integrator): 0 takes the render entry's "integrator"; 2 asks for
# primitive_path_tracer on a scene whose entry names nextevent_path_tracer
CASES = [("zoo", 0), ("cornell_pt", 0), ("cornell_ls", 0), ("cornell", 2)]


@pytest.mark.parametrize("name,integrator", CASES)
def test_noalloc_matches_allocating_entry_point(wr_lib, name, integrator):
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene(name)
    with wr_lib.Scene.from_file(path) as sc:
        inf = sc.info
        shape = (inf["height"], inf["width"], 3)
        ref = torch.empty(shape, dtype=torch.float64, device="cuda")
        _render(wr_lib, sc, L.wr_render_device, ref, spp=64, seed=21, integrator=integrator)
        ref_iters = _stats(wr_lib, sc).iterations
        outs = []
        for _ in range(2):   # the second call must not see the first call's leftovers
            o = torch.full(shape, -1.0, dtype=torch.float64, device="cuda")
            _render(wr_lib, sc, L.wr_render_device_noalloc, o, spp=64, seed=21, integrator=integrator)
            outs.append(o.cpu().numpy())
            st = _stats(wr_lib, sc)
            assert st.queue_capacity == 32768
            # bounce iterations + 1 (the longest path decides; a smaller wavefront needs more waves)
            assert st.iterations >= ref_iters > 0
    ref = ref.cpu().numpy()
    assert np.isfinite(ref).all() and ref.mean() > 0
    for o in outs:
        assert np.allclose(o, ref, rtol=1e-9, atol=1e-12), np.abs(o - ref).max()


def test_noalloc_integrators_differ(wr_lib):
    """The request's integrator reaches the kernels: primitive_path_tracer and
    nextevent_path_tracer renders of the same scene and seed are different images."""
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        inf = sc.info
        shape = (inf["height"], inf["width"], 3)
        a = torch.empty(shape, dtype=torch.float64, device="cuda")
        b = torch.empty(shape, dtype=torch.float64, device="cuda")
        _render(wr_lib, sc, L.wr_render_device_noalloc, a, spp=16, seed=3, integrator=1)
        _render(wr_lib, sc, L.wr_render_device_noalloc, b, spp=16, seed=3, integrator=2)
    assert not np.allclose(a.cpu().numpy(), b.cpu().numpy())


def test_noalloc_rejects_films_above_the_limit(wr_lib):
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        sc.set_camera('{"pos": [0,1,3.6], "lookat": [0,1,0], "up": [0,1,0], "fovy": 40, "resolution": [300, 300]}')
        out = torch.empty((300, 300, 3), dtype=torch.float64, device="cuda")
        rc = L.wr_render_device_noalloc(sc._h, ctypes.byref(_desc(wr_lib, 1, 0)), ctypes.c_void_p(out.data_ptr()))
        assert rc == 1
        assert b"65536" in L.wr_last_error()


def test_noalloc_rejects_guiding_and_bad_integrators(wr_lib):
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("cornell")
    with wr_lib.Scene.from_file(path) as sc:
        inf = sc.info
        out = torch.empty((inf["height"], inf["width"], 3), dtype=torch.float64, device="cuda")
        for g in (1, 2):
            rc = L.wr_render_device_noalloc(sc._h, ctypes.byref(_desc(wr_lib, 4, 0, guiding=g)),
                                            ctypes.c_void_p(out.data_ptr()))
            assert rc == 4, L.wr_last_error()   # WR_ERR_UNSUPPORTED
            assert b"guiding" in L.wr_last_error()
        rc = L.wr_render_device_noalloc(sc._h, ctypes.byref(_desc(wr_lib, 4, 0, max_iterations=-1)),
                                        ctypes.c_void_p(out.data_ptr()))
        assert rc == 1


def test_noalloc_timeout_then_next_call_is_correct(wr_lib):
    """An iteration bound too small for the paths stops the render with WR_ERR_TIMEOUT; the
    caller's device stays current and the next call renders the right image."""
    import torch
    L = wr_lib.load_library()
    path, _ = golden_scene("zoo")
    with wr_lib.Scene.from_file(path) as sc:
        inf = sc.info
        shape = (inf["height"], inf["width"], 3)
        ref = torch.empty(shape, dtype=torch.float64, device="cuda")
        _render(wr_lib, sc, L.wr_render_device, ref, spp=32, seed=5)
        out = torch.full(shape, -1.0, dtype=torch.float64, device="cuda")
        dev_before = torch.cuda.current_device()
        rc = L.wr_render_device_noalloc(sc._h, ctypes.byref(_desc(wr_lib, 32, 5, max_iterations=3)),
                                        ctypes.c_void_p(out.data_ptr()))
        assert rc == 7, L.wr_last_error()   # WR_ERR_TIMEOUT
        assert torch.cuda.current_device() == dev_before
        _render(wr_lib, sc, L.wr_render_device_noalloc, out, spp=32, seed=5)
    assert np.allclose(out.cpu().numpy(), ref.cpu().numpy(), rtol=1e-9, atol=1e-12)
