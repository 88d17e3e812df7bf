"""The C-ABI boundary as a C caller uses it (tests/c_boundary/gsl_driver.c).

The driver registers hw_gsl_rhs in a gsl_odeiv_system-shaped struct
(1d/functions.c:71-89) and runs the evolve loop of ode_solver_Ham
(1d/functions.c:546-553) with hw_evolve_apply, compiled against
include/hawassi_b200.h alone.  On the CPU the driver must compile and link
against the built library; on the GPU its run on the reference's 1dFBr005Bor deck
(HS2, breaking, reference tolerances) through the breaking onset must match the
oracle driven by the same loop: time, step counts, state (relative L2 1e-9), the
RHS through the struct at the end, and the breaking.dat records.
"""
import os
import subprocess

import numpy as np
import pytest

import oracle_lib as ol
from decks_util import rel_l2

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
SRC = os.path.join(ROOT, "tests", "c_boundary", "gsl_driver.c")
LIBDIR = os.path.join(ROOT, "hawassi_c_b200", "lib")


def _compile(out):
    if not os.path.exists(os.path.join(LIBDIR, "libhawassi_b200.so")):
        pytest.skip("engine not built")
    cmd = ["gcc", "-std=c11", "-Wall", "-Wextra", "-Werror", "-O2", "-I", os.path.join(ROOT, "include"), SRC,
           "-L", LIBDIR, "-lhawassi_b200", f"-Wl,-rpath,{LIBDIR}", "-o", out]
    r = subprocess.run(cmd, capture_output=True, text=True)
    assert r.returncode == 0, r.stderr
    return out


def test_driver_compiles_against_header(tmp_path):
    _compile(str(tmp_path / "gsl_driver"))


def _read(path):
    a = np.fromfile(path, dtype=np.float64)
    nx = int(a[0])
    t, h, rhs, acc, rej = a[1], a[2], int(a[3]), int(a[4]), int(a[5])
    y = a[6:6 + 4 * nx]
    dydt = a[6 + 4 * nx:6 + 8 * nx]
    n = int(a[6 + 8 * nx])
    log = a[7 + 8 * nx:7 + 8 * nx + n]
    return dict(nx=nx, t=t, h=h, stats=(rhs, acc, rej), y=y, dydt=dydt, log=log)


def _log_records(flat):
    out, i = [], 0
    while i < flat.size:
        cnt = int(flat[i + 1])
        out.append((f"{flat[i]:f}", [int(v) for v in flat[i + 2:i + 2 + cnt]]))
        i += 2 + cnt
    return out


@pytest.mark.gpu
def test_driver_matches_oracle(tmp_path, golden_dir):
    exe = _compile(str(tmp_path / "gsl_driver"))
    deck = os.path.join(golden_dir, "fbr005")
    t_stop = 13.0
    out = str(tmp_path / "gpu.bin")
    r = subprocess.run([exe, deck, str(t_stop), "2", out], capture_output=True, text=True, timeout=600)
    assert r.returncode == 0, r.stderr
    g = _read(out)
    # the same loop on the oracle, then the same RHS call at the end
    o = ol.Oracle(deck)
    tt = o.table("ttrace")
    y = o.initial_state()
    t, h = float(tt[0]), 1e-4
    for ti in tt[1:]:
        if ti > t_stop:
            break
        while t < ti:
            t, h = o.evolve_apply(t, ti, h, y)
    dydt = o.rhs(t, y)
    assert g["t"] == pytest.approx(t, rel=1e-13)
    assert g["h"] == pytest.approx(h, rel=1e-6)
    assert g["stats"] == tuple(o.stats())
    assert rel_l2(g["y"], y) < 1e-9
    assert rel_l2(g["dydt"], dydt) < 1e-8
    mine = _log_records(g["log"])
    ref = [(l.split()[0], [int(v) for v in l.split()[2:]]) for l in o.breaking_log().splitlines()]
    assert len(ref) >= 5 and mine == ref
