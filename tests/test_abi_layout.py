"""Every ctypes mirror of a C-ABI struct (spacetime-optics_b200/abi.py) against include/so_tracer.h:
a C program compiled here prints sizeof and offsetof of each field, and they must equal the ctypes
layout, field by field.  A field added on one side only would shift every later field the binding
reads (statistics, options), so this runs on the CPU with every build."""
import ctypes as C
import os
import subprocess
import tempfile

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# ctypes class -> C typedef
STRUCTS = {
    "Vec3": "so_vec3", "Mat3": "so_mat3", "KerrPoint": "so_kerr_point", "Scene": "so_scene", "Frame": "so_frame",
    "Tables": "so_tables", "Settings": "so_settings", "Post": "so_post", "HdrFrame": "so_hdr_frame",
    "Stats": "so_stats", "RaysOut": "so_rays_out", "Plasma": "so_plasma", "Mode": "so_mode",
    "MixedOpts": "so_mixed_opts", "Tune": "so_tune", "SurRay": "so_sur_ray", "SurTarget": "so_sur_target",
    "SurOpts": "so_sur_opts", "SurLoss": "so_sur_loss", "SurRanges": "so_sur_ranges",
    "SurFrameOpts": "so_sur_frame_opts", "SurReport": "so_sur_report", "SceneInfo": "so_scene_info",
}


def _fields(cls):
    out = []
    for f in cls._fields_:
        name = f[0]
        out.append((name, getattr(cls, name).offset))
    return out


def test_ctypes_mirrors_match_the_header(so):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "so_tracer.h"', "int main(void) {"]
    expect = []
    for py, cname in STRUCTS.items():
        cls = getattr(so.abi, py)
        lines.append(f'  printf("{py} size %zu\\n", sizeof({cname}));')
        expect.append(f"{py} size {C.sizeof(cls)}")
        for name, off in _fields(cls):
            lines.append(f'  printf("{py}.{name} %zu\\n", offsetof({cname}, {name}));')
            expect.append(f"{py}.{name} {off}")
    lines += ["  return 0;", "}"]
    with tempfile.TemporaryDirectory() as d:
        src, exe = os.path.join(d, "layout.c"), os.path.join(d, "layout")
        with open(src, "w") as fh:
            fh.write("\n".join(lines) + "\n")
        cc = subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), src, "-o", exe],
                            capture_output=True, text=True)
        if cc.returncode != 0:
            pytest.fail("layout program does not compile:\n" + cc.stderr[-2000:])
        got = subprocess.run([exe], capture_output=True, text=True, check=True).stdout.split("\n")
    got = [g for g in got if g]
    mismatch = [(e, g) for e, g in zip(expect, got) if e != g]
    assert len(got) == len(expect) and not mismatch, mismatch[:10]
