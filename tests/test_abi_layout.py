"""The ctypes mirrors in efem_b200/api.py against the C structs of
include/efem_gpu.h: a small C program built with the host compiler prints
sizeof and offsetof of every field, and each must equal ctypes' layout (a
mismatch would make the library read or write the wrong bytes)."""
import ctypes
import os
import shutil
import subprocess

import pytest

from efem_b200 import api

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
STRUCTS = {
    "efem_material": api.Material,
    "efem_element_block": api.ElementBlock,
    "efem_mesh_desc": api.MeshDesc,
    "efem_load_desc": api.LoadDesc,
    "efem_options": api.Options,
    "efem_solve_info": api.SolveInfo,
    "efem_model_info": api.ModelInfo,
    "efem_adjoint_info": api.AdjointInfo,
}


@pytest.mark.skipif(shutil.which("gcc") is None, reason="no host C compiler")
def test_ctypes_structs_match_header(tmp_path):
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "efem_gpu.h"', "int main(void) {"]
    expect = []
    for cname, cls in STRUCTS.items():
        lines.append(f'    printf("%zu\\n", sizeof({cname}));')
        expect.append((f"sizeof({cname})", ctypes.sizeof(cls)))
        for fname, _ in cls._fields_:
            lines.append(f'    printf("%zu\\n", offsetof({cname}, {fname}));')
            expect.append((f"{cname}.{fname}", getattr(cls, fname).offset))
    lines += ["    return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)], check=True)
    got = [int(x) for x in subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()]
    assert len(got) == len(expect)
    bad = [(name, want, g) for (name, want), g in zip(expect, got) if want != g]
    assert not bad, f"ctypes layout differs from the C header (name, ctypes, C): {bad}"
