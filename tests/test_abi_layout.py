"""The ctypes mirrors of the C ABI's structs (cudaraytracer_b200._lib) have
the sizes and field offsets that include/crt.h gives them: a small C program
compiled with the host compiler prints sizeof and offsetof for every field,
and the test compares them with ctypes (no GPU needed)."""
import ctypes
import os
import shutil
import subprocess

import pytest
from conftest import ROOT

from cudaraytracer_b200 import _lib

PAIRS = [  # ctypes mirror -> C type
    (_lib.SceneInfo, "crt_scene_info_t"),
    (_lib.RenderParams, "crt_render_params"),
    (_lib.Camera, "crt_camera"),
    (_lib.GBuffer, "crt_gbuffer"),
    (_lib.DenoiseParams, "crt_denoise_params"),
    (_lib.MaterialDesc, "crt_material_desc"),
    (_lib.TextureDesc, "crt_texture_desc"),
    (_lib.MeshDesc, "crt_mesh_desc"),
    (_lib.LightDesc, "crt_light_desc"),
    (_lib.SceneDesc, "crt_scene_desc"),
    (_lib.ServerConfig, "crt_server_config"),
    (_lib.Request, "crt_request"),
    (_lib.ServerStats, "crt_server_stats"),
]


@pytest.fixture(scope="module")
def c_layout(tmp_path_factory):
    cc = shutil.which("gcc") or shutil.which("cc")
    if cc is None:
        pytest.skip("no host C compiler")
    lines = ['#include <stddef.h>', '#include <stdio.h>', '#include "crt.h"', "int main(void) {"]
    for cls, cname in PAIRS:
        lines.append(f'    printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for f in cls._fields_:
            lines.append(f'    printf("{cname} {f[0]} %zu\\n", offsetof({cname}, {f[0]}));')
    lines += ["    return 0;", "}"]
    d = tmp_path_factory.mktemp("abi")
    src, exe = d / "layout.c", d / "layout"
    src.write_text("\n".join(lines) + "\n")
    r = subprocess.run([cc, "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                       capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-2000:]
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout
    table = {}
    for line in out.splitlines():
        cname, field, value = line.split()
        table[(cname, field)] = int(value)
    return table


@pytest.mark.parametrize("cls,cname", PAIRS, ids=[c for _, c in PAIRS])
def test_struct_layout_matches_header(c_layout, cls, cname):
    assert ctypes.sizeof(cls) == c_layout[(cname, "sizeof")], cname
    for f in cls._fields_:
        assert getattr(cls, f[0]).offset == c_layout[(cname, f[0])], (cname, f[0])
