"""The C-ABI library builds for sm_100a, loads and exports every declared symbol.

These checks need no GPU: they load libahop_b200.so without calling into CUDA.
"""
import ctypes
import os
import re
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


def declared(header):
    src = open(os.path.join(REPO, "include", header)).read()
    src = re.sub(r"/\*.*?\*/", "", src, flags=re.S)
    return sorted(set(re.findall(r"\b(ahop_\w+|halo_\w+)\s*\(", src)))


@pytest.fixture(scope="module")
def libpath():
    from ahop_b200 import build
    return build.build()


def test_library_exports_every_declared_symbol(libpath):
    syms = subprocess.run(["nm", "-D", "--defined-only", libpath], capture_output=True, text=True).stdout
    exported = set(re.findall(r" T (\w+)", syms))
    for h in os.listdir(os.path.join(REPO, "include")):
        for name in declared(h):
            assert name in exported, f"{name} declared in include/{h} but not exported"


def test_library_loads_and_reports_errors(libpath):
    lib = ctypes.CDLL(libpath)
    lib.ahop_last_error.restype = ctypes.c_char_p
    # argument validation happens before any CUDA call
    assert lib.ahop_sync_others(None) == 1
    assert b"null" in lib.ahop_last_error()


def test_built_for_sm100a():
    from ahop_b200 import build
    assert build.ARCH == ["-gencode", "arch=compute_100a,code=sm_100a"]


def test_dropin_module_surface():
    from compute_adaptahop import neikdtree
    for name in ("compute_adaptahop", "sync_from_change_pos", "sync_from_init_adaptahop", "sync_others", "close"):
        assert callable(getattr(neikdtree, name))
    for name in ("liste_parts", "density", "nnodes", "real_table", "integer_table"):
        assert hasattr(neikdtree, name)


STRUCTS = {
    "AhopInit": ("ahop_b200._lib", "AhopInit"),
    "AhopOthers": ("ahop_b200._lib", "AhopOthers"),
    "AhopOutputs": ("ahop_b200._lib", "AhopOutputs"),
    "AhopTimings": ("ahop_b200._lib", "AhopTimings"),
    "AhopStructs": ("ahop_b200.msm", "AhopStructs"),
    "AhopRamsesParams": ("ahop_b200.ramses", "AhopRamsesParams"),
    "AhopRamsesCounts": ("ahop_b200.ramses", "AhopRamsesCounts"),
    "AhopHaloParams": ("ahop_b200.halo_props", "AhopHaloParams"),
    "AhopHaloTimings": ("ahop_b200.halo_props", "AhopHaloTimings"),
    "AhopVirialParams": ("ahop_b200.halo_props", "AhopVirialParams"),
    "AhopAdjParams": ("ahop_b200.autograd", "AhopAdjParams"),
}


def test_python_structs_match_the_header(tmp_path):
    """Every ctypes mirror has the C struct's size and field offsets (a C
    program compiled against include/ahop_b200.h prints them)."""
    import importlib
    mirrors = {k: getattr(importlib.import_module(m), c) for k, (m, c) in STRUCTS.items()}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "ahop_b200.h"', "int main(void) {"]
    for name, cls in mirrors.items():
        lines.append(f'  printf("{name} size %zu\\n", sizeof({name}));')
        for fname, _ in cls._fields_:
            lines.append(f'  printf("{name} {fname} %zu\\n", offsetof({name}, {fname}));')
    lines.append("  return 0;\n}")
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines))
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, check=True).stdout.split("\n")
    seen = 0
    for line in out:
        if not line:
            continue
        name, what, val = line.split()
        cls = mirrors[name]
        got = ctypes.sizeof(cls) if what == "size" else getattr(cls, what).offset
        assert got == int(val), f"{name}.{what}: ctypes {got}, C {val}"
        seen += 1
    assert seen == sum(1 + len(c._fields_) for c in mirrors.values())
