"""The ctypes structures of the Python binding (racon_b200/__init__.py) have
the sizes and field offsets of the C ABI's structs (include/racon_b200.h),
as gcc lays them out for this platform. No GPU: a small C program built
against the header prints sizeof / offsetof for every struct the binding
passes across the boundary."""
import ctypes
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

# C struct name -> name of the ctypes class in racon_b200
STRUCTS = {
    "rb_params": "_Params",
    "rb_pair": "_Pair",
    "rb_aln_result": "_AlnResult",
    "rb_cigar_overlap": "_CigarOverlap",
    "rb_window": "_Window",
    "rb_sequence": "_Sequence",
    "rb_layer_overlap": "_LayerOverlap",
    "rb_store_pair": "_StorePair",
    "rb_poa_result": "_PoaResult",
    "rb_server_params": "_ServerParams",
    "rb_server_job": "_ServerJob",
    "rb_server_times": "ServerTimes",
    "rb_stats": "Stats",
    "rb_tuning": "Tuning",
}


def _layouts(tmp_path, binding):
    lines = ["#include <stdio.h>", "#include <stddef.h>", '#include "racon_b200.h"', "int main(void) {"]
    for cname, pyname in STRUCTS.items():
        cls = getattr(binding, pyname)
        lines.append('  printf("%s size %%zu\\n", sizeof(%s));' % (cname, cname))
        for field in cls._fields_:
            fname = field[0]
            lines.append('  printf("%s %s %%zu\\n", offsetof(%s, %s));' % (cname, fname, cname, fname))
    lines += ["  return 0;", "}"]
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text("\n".join(lines) + "\n")
    subprocess.run(["gcc", "-std=c99", "-I", os.path.join(ROOT, "include"), str(src), "-o", str(exe)],
                   check=True, capture_output=True, text=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout
    got = {}
    for line in out.splitlines():
        name, field, value = line.split()
        got[(name, field)] = int(value)
    return got


@pytest.mark.skipif(shutil.which("gcc") is None, reason="gcc is needed to lay out the header's structs")
def test_binding_structs_match_the_header(tmp_path):
    import racon_b200

    got = _layouts(tmp_path, racon_b200)
    for cname, pyname in STRUCTS.items():
        cls = getattr(racon_b200, pyname)
        assert ctypes.sizeof(cls) == got[(cname, "size")], (cname, "size")
        for field in cls._fields_:
            fname = field[0]
            assert getattr(cls, fname).offset == got[(cname, fname)], (cname, fname)
