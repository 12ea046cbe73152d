"""The ctypes mirrors of the C ABI's structs (vlasov.jl_b200/_lib.py) against
the header itself: a small C program built with gcc from
include/vlasov_b200.h prints sizeof and the offset of every field, and each
must equal the mirror's.  A binding in another host language (a Julia
ccall binding, for one) has to match the same numbers."""
import ctypes as C
import shutil
import subprocess

import pytest

from conftest import ROOT, load_package

vb = load_package()
L = vb._lib

PAIRS = [
    ("vlb_level_desc", L.LevelDesc),
    ("vlb_smoothing_desc", L.SmoothingDesc),
    ("vlb_config", L.Config),
    ("vlb_projectile", L.ProjectileDesc),
    ("vlb_step_params", L.StepParams),
    ("vlb_step_result", L.StepResult),
    ("vlb_exchange", L.Exchange),
    ("vlb_tuning", L.Tuning),
]


def _program():
    lines = ["#include <stddef.h>", "#include <stdio.h>", '#include "vlasov_b200.h"', "int main(void) {"]
    for cname, mirror in PAIRS:
        lines.append(f'  printf("{cname} sizeof %zu\\n", sizeof({cname}));')
        for field, _ in mirror._fields_:
            lines.append(f'  printf("{cname} {field} %zu\\n", offsetof({cname}, {field}));')
    lines += ["  return 0;", "}"]
    return "\n".join(lines) + "\n"


@pytest.mark.skipif(shutil.which("gcc") is None, reason="needs gcc")
def test_ctypes_mirrors_match_the_header(tmp_path):
    src = tmp_path / "layout.c"
    exe = tmp_path / "layout"
    src.write_text(_program())
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split("\n")
    seen = {}
    for line in filter(None, out):
        cname, what, value = line.split()
        seen[(cname, what)] = int(value)
    for cname, mirror in PAIRS:
        assert seen[(cname, "sizeof")] == C.sizeof(mirror), cname
        for field, _ in mirror._fields_:
            assert seen[(cname, field)] == getattr(mirror, field).offset, (cname, field)
