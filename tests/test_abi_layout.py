"""The ctypes mirrors of the C-ABI structures have the C layout: every field's offset
and each structure's size, as gcc lays out the declarations of include/hawassi_b200.h
(and of the oracle's headers for the test harness's mirrors).  A drifted mirror would
hand the library shifted tables without any error."""
import ctypes
import os
import subprocess

import pytest

import oracle_lib as ol
from hawassi_c_b200.engine import HwJonswap, HwOpts
from hawassi_c_b200.engine2d import Hw2dOutputs, Hw2dTables

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

CASES = [
    ("include/hawassi_b200.h", "hw_opts", HwOpts),
    ("include/hawassi_b200.h", "hw_jonswap", HwJonswap),
    ("include/hawassi_b200.h", "hw2d_tables", Hw2dTables),
    ("include/hawassi_b200.h", "hw2d_outputs", Hw2dOutputs),
    ("oracle/hw_oracle.h", "or_opts", ol.OrOpts),
    ("oracle/hw_oracle2d.h", "or2d_tables", ol.Or2dTables),
    ("oracle/hw_oracle2d.h", "or2d_outputs", ol.Or2dOutputs),
]


def c_layout(tmp_path, header, name, fields):
    src = tmp_path / f"{name}.c"
    lines = [f'#include "{os.path.join(ROOT, header)}"', "#include <stddef.h>", "#include <stdio.h>",
             "int main(void) {", f'  printf("%zu\\n", sizeof({name}));']
    lines += [f'  printf("%zu\\n", offsetof({name}, {f}));' for f in fields]
    lines += ["  return 0;", "}"]
    src.write_text("\n".join(lines) + "\n")
    exe = tmp_path / name
    subprocess.run(["gcc", "-std=c11", "-o", str(exe), str(src)], check=True)
    out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
    return int(out[0]), [int(v) for v in out[1:]]


@pytest.mark.parametrize("header,name,mirror", CASES, ids=[c[1] for c in CASES])
def test_ctypes_mirror_matches_c_layout(tmp_path, header, name, mirror):
    fields = [f[0] for f in mirror._fields_]
    size, offsets = c_layout(tmp_path, header, name, fields)
    assert ctypes.sizeof(mirror) == size
    assert [getattr(mirror, f).offset for f in fields] == offsets
