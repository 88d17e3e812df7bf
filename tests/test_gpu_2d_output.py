"""The 2D output stage on the device (hw2d_fields, hw2d_run_outputs) against the
oracle's restatement of ode_solver_uv's loop and files (2d/fun_odesolver.c:2565-2843).

Field files are FP32 images of FP64 fields that agree to ~1e-12, so they are
compared to a few FP32 ulps; Constant_01.dat (tables only) must be byte-identical,
gauge files agree to the last printed digit and breaking.dat record by record."""
import os

import numpy as np
import pytest

from breaking2d_case import steep_crest_case
from hawassi_c_b200 import decks2d
from hawassi_c_b200.engine2d import Engine2D
from oracle_lib import Oracle2D, fields2d, run_outputs2d
from test_oracle2d_output import smooth_fields, state_of

pytestmark = pytest.mark.gpu


def flat_tables(nx, ny):
    return decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                          t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=3)


@pytest.mark.parametrize("nx,ny", [(64, 64), (128, 64), (64, 256), (1024, 64)])
def test_fields_parity(nx, ny):
    """Every wavenumber excited and no Hermitian symmetry: the symmetrisation decides."""
    tb = flat_tables(nx, ny)
    rng = np.random.default_rng(nx + ny)
    z = rng.standard_normal(6 * nx * ny)
    eng = Engine2D(tb)
    eng.set_state(0.0, 0.01, z)
    for got, want in zip(eng.fields(), fields2d(nx, ny, z)):
        assert np.abs(got - want).max() < 1e-13 * max(1.0, np.abs(want).max())


def compare_dirs(da, db, n):
    na, nb = sorted(os.listdir(da)), sorted(os.listdir(db))
    assert na == nb
    for name in na:
        a, b = os.path.join(da, name), os.path.join(db, name)
        if name.startswith("Constant"):
            assert open(a, "rb").read() == open(b, "rb").read()
        elif name.endswith("_gauge.dat"):
            ra = [ln.split() for ln in open(a).read().splitlines()]
            rb = [ln.split() for ln in open(b).read().splitlines()]
            assert len(ra) == len(rb) and ra[:2] == rb[:2]
            assert np.allclose(np.array(ra[2:], float), np.array(rb[2:], float), rtol=0, atol=2.01e-6)
        elif name.startswith("Hawassi_"):
            fa, fb = np.fromfile(a, dtype=np.float32), np.fromfile(b, dtype=np.float32)
            assert fa.size == fb.size and fa.size % n == 0
            scale = max(float(np.abs(fb).max()), 1e-30)
            assert np.abs(fa.astype(np.float64) - fb).max() <= 1e-6 * scale
    return na


@pytest.mark.parametrize("uv_every", [False, True])
def test_run_outputs_parity(tmp_path, uv_every):
    tb = flat_tables(64, 64)
    nx, ny = tb["nx"], tb["ny"]
    z0 = state_of(*smooth_fields(tb, 5))
    tout = np.round(np.arange(7) * 0.1, 12)
    args = decks2d.outputs(tb, tout, npartition=3, gauges=[(tb["x"][5], tb["y"][3]), (tb["x"][40], tb["y"][20])],
                           uv_every_sample=uv_every, chiadjphi=np.ones((ny, nx)))
    eng = Engine2D(tb, 1e-8, 1e-6)
    eng.set_state(0.0, 0.02, z0)
    (tmp_path / "gpu").mkdir()
    (tmp_path / "cpu").mkdir()
    assert eng.run_outputs(tmp_path / "gpu", **args) == 7
    r, t, _ = run_outputs2d(Oracle2D(tb, 1e-8, 1e-6), 0.0, 0.02, z0.copy(), tmp_path / "cpu", **args)
    assert r == 7
    names = compare_dirs(tmp_path / "gpu", tmp_path / "cpu", nx * ny)
    assert "Hawassi_eta_04.dat" in names and "Constant_01.dat" in names
    te, _, _ = eng.state(with_y=False)
    assert te == t


def test_run_outputs_breaking_parity(tmp_path):
    """Two-depth bottom with kinematic breaking: the same files and breaking.dat."""
    tb, z = steep_crest_case(64, 64)
    tout = 0.3 + 0.02 * np.arange(6)
    args = decks2d.outputs(tb, tout, npartition=2, gauges=[(tb["x"][40], tb["y"][30])])
    eng = Engine2D(tb, 1e-6, 1e-4)
    eng.set_state(0.3, 0.005, z)
    (tmp_path / "gpu").mkdir()
    (tmp_path / "cpu").mkdir()
    assert eng.run_outputs(tmp_path / "gpu", **args) == 6
    ora = Oracle2D(tb, 1e-6, 1e-4)
    ora.set_tprev(0.3)
    run_outputs2d(ora, 0.3, 0.005, z.copy(), tmp_path / "cpu", **args)
    names = compare_dirs(tmp_path / "gpu", tmp_path / "cpu", 64 * 64)
    assert "breaking.dat" in names
    la = open(tmp_path / "gpu" / "breaking.dat").read().splitlines()
    lb = open(tmp_path / "cpu" / "breaking.dat").read().splitlines()
    assert len(la) == len(lb) and len(lb) > 0
    for a, b in zip(la, lb):
        a, b = a.split(), b.split()
        assert abs(float(a[0]) - float(b[0])) <= 1.01e-6 and a[1:] == b[1:]
