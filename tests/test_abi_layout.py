"""The C structs of include/lenia_b200.h against their ctypes mirrors in the
Python binding: a small C program compiled with gcc against the header prints
every struct's size and the offset and size of every member the binding
names, and all must equal the ctypes layout (a member appended on one side
only, or a type that differs in width, would otherwise shift or truncate
fields silently). No GPU and no library load needed."""
import os
import shutil
import subprocess

import ctypes
import pytest

import life_simulation_b200 as lb

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PAIRS = [
    (lb.KernelDef, "lenia_kernel_def"),
    (lb.Config, "lenia_config"),
    (lb.FrameParams, "lenia_frame_params"),
    (lb.Info, "lenia_info"),
    (lb.ColorMap, "lenia_colormap"),
    (lb.Mapping, "lenia_mapping"),
    (lb.SceneInfo, "lenia_scene_info"),
    (lb.AdjointConfig, "lenia_adjoint_config"),
    (lb.World, "lenia_world"),
    (lb.ProfileData, "lenia_profile_data"),
]


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_structs_match_the_c_header(tmp_path):
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "lenia_b200.h"', "int main(void) {"]
    expect = []
    for cls, cname in PAIRS:
        lines.append(f'  printf("%zu\\n", sizeof({cname}));')
        expect.append((f"sizeof({cname})", ctypes.sizeof(cls)))
        for fname, _ in cls._fields_:
            lines.append(f'  printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append((f"offsetof({cname}, {fname})", getattr(cls, fname).offset))
            lines.append(f'  printf("%zu\\n", sizeof((({cname} *)0)->{fname}));')
            expect.append((f"sizeof({cname}.{fname})", getattr(cls, fname).size))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert len(got) == len(expect)
    bad = [(what, c, py) for (what, py), c in zip(expect, got) if c != py]
    assert not bad, bad
