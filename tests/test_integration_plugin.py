"""The reference-side plugin of INTEGRATION.md compiles against the reference's headers.

INTEGRATION.md section 2 shows the Renderer a maintainer adds to the reference
(`PathNeeB200Renderer`, a SingleCameraRenderer that forwards render() to wr_render). This test
cuts that C++ block out of INTEGRATION.md and compiles it to an object file against the
reference's own src/ headers (common/renderer.h, Film, Camera, Util::Json) and
include/wurst_b200.h, with the reference's compiler flags, so that a stale signature on either
side fails here. Needs the reference sources (WURST_REFERENCE_ROOT); skipped where they are absent.
"""
import os
import re
import subprocess

import pytest

from conftest import ROOT


def _reference_root():
    import oracle
    return oracle.REFERENCE_ROOT


def _plugin_source():
    text = open(os.path.join(ROOT, "INTEGRATION.md")).read()
    section = text[text.index("## 2."):]
    m = re.search(r"```cpp\n(.*?)```", section, re.S)
    assert m, "INTEGRATION.md section 2 has no C++ block"
    return m.group(1)


def test_plugin_block_names_the_c_abi():
    src = _plugin_source()
    for sym in ("wr_scene_create", "wr_render", "wr_scene_destroy", "wr_last_error", "wr_render_desc"):
        assert sym in src
    header = open(os.path.join(ROOT, "include", "wurst_b200.h")).read()
    for sym in ("wr_scene_create", "wr_render", "wr_scene_destroy", "wr_last_error"):
        assert re.search(r"\b%s\s*\(" % sym, header), sym


def test_plugin_compiles_against_reference_headers(tmp_path):
    ref = _reference_root()
    if not os.path.isdir(os.path.join(ref, "src", "common")):
        pytest.skip("reference sources not present")
    (tmp_path / "pathnextevent_b200.h").write_text(_plugin_source())
    (tmp_path / "plugin_tu.cpp").write_text(
        '#include "common/wurst.h"\n'
        '#include "pathnextevent_b200.h"\n'
        "// take the factory's address so that the class and its members are instantiated\n"
        "auto *g_factory = &PathNeeB200Renderer::FromSimple2Json;\n")
    cmd = ["g++", "-std=c++17", "-O0", "-mavx2", "-DAVX2", "-DNDEBUG", "-w",
           "-I", os.path.join(ref, "src"),
           "-I", os.path.join(ref, "dependencies", "embree", "include"),
           "-I", os.path.join(ref, "dependencies", "pbrt-parser", "pbrtParser", "include"),
           "-I", os.path.join(ROOT, "include"), "-I", str(tmp_path),
           "-c", str(tmp_path / "plugin_tu.cpp"), "-o", str(tmp_path / "plugin_tu.o")]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-4000:]
    # the object refers to the C ABI the library exports
    nm = subprocess.run(["nm", "-u", str(tmp_path / "plugin_tu.o")], capture_output=True, text=True).stdout
    for sym in ("wr_scene_create", "wr_render", "wr_scene_destroy", "wr_last_error"):
        assert re.search(r"\b%s\b" % sym, nm), sym
