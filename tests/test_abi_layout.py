"""The Python ctypes mirrors of the C ABI's structs (wurstrenderer_b200/__init__.py) against the
layout the C compiler gives the public header (include/wurst_b200.h): every struct's size and
every field's offset agree, so a field added to the header cannot shift the ones the Python side
(or a binding written from the header) reads."""
import ctypes
import os
import subprocess

import pytest

import wurstrenderer_b200 as wr

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

STRUCTS = {"wr_render_desc": wr.RenderDesc, "wr_render_stats": wr.RenderStats, "wr_scene_info": wr.SceneInfo,
           "wr_scene_options": wr.SceneOptions, "wr_job": wr.Job}


def _c_layout(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "wurst_b200.h"', 'int main(void) {']
    for cname, py in STRUCTS.items():
        lines.append('printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for field, _ in py._fields_:
            lines.append('printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, field, cname, field))
    lines += ['return 0;', '}']
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    return {tuple(l.split()[:2]): int(l.split()[2]) for l in out.splitlines()}


@pytest.mark.parametrize("cname", sorted(STRUCTS))
def test_ctypes_mirror_matches_header(tmp_path, cname):
    c = _c_layout(tmp_path)
    py = STRUCTS[cname]
    assert c[(cname, "size")] == ctypes.sizeof(py), cname
    for field, _ in py._fields_:
        assert c[(cname, field)] == getattr(py, field).offset, (cname, field)
