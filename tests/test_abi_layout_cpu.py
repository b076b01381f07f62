"""The ctypes mirrors of include/qsgpu.h's structs have the C layout: a small
C program compiled against the header prints every struct's size and field
offsets, which must equal ctypes' (no GPU needed)."""
import ctypes
import importlib
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_struct_layouts_match_header(qs, tmp_path):
    abi = importlib.import_module(qs.__name__ + "._abi")
    structs = {name: getattr(abi, name) for name in
               ("qs_view", "qs_plan_options", "qs_plan_info", "qs_group_info", "qs_allocator")}
    lines = ['#include <stdio.h>', '#include <stddef.h>', '#include "qsgpu.h"', "int main(void) {"]
    for name, cls in structs.items():
        lines.append(f'  printf("{name} %zu\\n", sizeof({name}));')
        for field, _ in cls._fields_:
            lines.append(f'  printf("{name}.{field} %zu\\n", offsetof({name}, {field}));')
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / "layout"
    subprocess.run(["gcc", "-std=c11", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    c = dict(line.rsplit(" ", 1) for line in out.strip().splitlines())
    for name, cls in structs.items():
        assert int(c[name]) == ctypes.sizeof(cls), name
        for field, _ in cls._fields_:
            assert int(c[f"{name}.{field}"]) == getattr(cls, field).offset, f"{name}.{field}"


def test_allocator_arguments_validated(qs):
    assert qs.allocator_checkpoint(None) is None
    qs.allocator_reset(None, None)          # DefaultAllocator: nothing to reset
    with pytest.raises(qs.ArgumentError, match="unsupported allocator"):
        qs.allocators.allocator_handle(object())
