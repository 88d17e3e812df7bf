"""CPU checks of the 2D oracle's output stage: ifftw_2d_c2r of the state and the
files ode_solver_uv writes (Constant_01.dat, Hawassi_{eta,u,v}_NN.dat, the gauge
files), on a small flat deck (no GPU needed)."""
import os

import numpy as np
import pytest

from hawassi_c_b200 import decks2d
from oracle_lib import Oracle2D, fields2d, run_outputs2d, sym2


def small_tables(nx=64, ny=32):
    return decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                          t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=3)


def state_of(eta, u, v):
    ny, nx = eta.shape
    n = nx * ny
    z = np.zeros(6 * n)
    for f, a in enumerate((eta, u, v)):
        A = np.fft.fft2(a)
        z[2 * f * n:(2 * f + 1) * n] = A.real.ravel()
        z[(2 * f + 1) * n:(2 * f + 2) * n] = A.imag.ravel()
    return z


def smooth_fields(tb, seed):
    rng = np.random.default_rng(seed)
    X, Y = np.meshgrid(tb["x"], tb["y"])
    out = []
    for _ in range(3):
        a = np.zeros_like(X)
        for _ in range(4):
            kx, ky = rng.integers(1, 4), rng.integers(0, 3)
            a += 0.02 * rng.standard_normal() * np.cos(2 * np.pi * (kx * X / tb["x"][-1] + ky * Y / tb["y"][-1])
                                                         + rng.uniform(0, 2 * np.pi))
        out.append(a)
    return out


def test_fields_invert_the_forward_transform():
    tb = small_tables()
    rng = np.random.default_rng(1)
    eta, u, v = (rng.standard_normal((32, 64)) for _ in range(3))
    for got, want in zip(fields2d(64, 32, state_of(eta, u, v)), (eta, u, v)):
        assert np.abs(got - want).max() < 1e-13 * np.abs(want).max() * 64


def test_fields_symmetrise_before_the_transform():
    """A spectrum that is not Hermitian: the real part of the inverse transform of its
    fftwcomplex_2d_sym image, divided by Nx Ny (ifftw_2d_c2r)."""
    rng = np.random.default_rng(2)
    ny, nx = 32, 64
    n = nx * ny
    z = rng.standard_normal(6 * n)
    got = fields2d(nx, ny, z)
    for f in range(3):
        A = (z[2 * f * n:(2 * f + 1) * n] + 1j * z[(2 * f + 1) * n:(2 * f + 2) * n]).reshape(ny, nx)
        want = np.fft.ifft2(sym2(A)).real
        assert np.abs(got[f] - want).max() < 1e-14 * max(1.0, np.abs(want).max()) * 64


def read_constant(path, nx, ny, with_chi):
    a = np.fromfile(path, dtype=np.float64)
    o = 0
    out = {}
    for key, size in (("NX", 1), ("x", nx), ("NY", 1), ("y", ny), ("NT", 1)):
        out[key] = a[o:o + size]
        o += size
    nt = int(out["NT"][0])
    for key, size in (("th", nt), ("hs", 1), ("kp", 1), ("wp", 1), ("kx", nx), ("ky", ny), ("bathy", nx * ny),
                      ("cfsa", nx * ny)) + ((("chi", nx * ny),) if with_chi else ()):
        out[key] = a[o:o + size]
        o += size
    assert o == a.size
    return out


@pytest.mark.parametrize("uv_every", [False, True])
def test_output_files(tmp_path, uv_every):
    tb = small_tables()
    nx, ny = tb["nx"], tb["ny"]
    n = nx * ny
    z0 = state_of(*smooth_fields(tb, 5))
    tout = np.round(np.arange(7) * 0.1, 12)
    chi = np.linspace(0.5, 1.0, n).reshape(ny, nx)
    gauges = [(tb["x"][5] + 0.2, tb["y"][3] - 0.1), (tb["x"][40], tb["y"][20])]
    args = decks2d.outputs(tb, tout, npartition=3, gauges=gauges, uv_every_sample=uv_every, chiadjphi=chi)
    ora = Oracle2D(tb, 1e-8, 1e-6)
    z = z0.copy()
    r, t, h = run_outputs2d(ora, 0.0, 0.02, z, tmp_path, **args)
    assert r == 7 and t == tout[-1]
    # ntpart = 7 // 3 = 2: partitions start at samples 0, 2, 4, 6
    names = sorted(os.listdir(tmp_path))
    assert names == sorted(["Constant_01.dat", "Hawassi_eta_gauge.dat", "Hawassi_u_gauge.dat", "Hawassi_v_gauge.dat"]
                           + [f"Hawassi_{f}_{p:02d}.dat" for f in ("eta", "u", "v") for p in (1, 2, 3, 4)])
    for p, ns in ((1, 2), (2, 2), (3, 2), (4, 1)):
        assert os.path.getsize(tmp_path / f"Hawassi_eta_{p:02d}.dat") == 4 * n * ns
        assert os.path.getsize(tmp_path / f"Hawassi_u_{p:02d}.dat") == 4 * n * (ns if uv_every else 1)
    c = read_constant(tmp_path / "Constant_01.dat", nx, ny, True)
    assert c["NX"][0] == nx and c["NY"][0] == ny and c["NT"][0] == 2
    assert np.array_equal(c["th"], np.arange(2) * (tout[1] - tout[0]))
    for key, want in (("x", tb["x"]), ("y", tb["y"]), ("kx", tb["kx"]), ("ky", tb["ky"]), ("bathy", tb["bathy"]),
                      ("cfsa", tb["cfsa"]), ("chi", chi)):
        assert np.array_equal(c[key], np.ravel(want))
    assert (c["hs"][0], c["kp"][0], c["wp"][0]) == (tb["hs"], tb["kp"], tb["wp"])
    # sample 0 is the initial state; sample 3 (second of partition 2) the state at 0.3
    e1 = np.fromfile(tmp_path / "Hawassi_eta_01.dat", dtype=np.float32).reshape(2, ny, nx)
    eta0, u0, v0 = fields2d(nx, ny, z0)
    assert np.array_equal(e1[0], eta0.astype(np.float32))
    u1 = np.fromfile(tmp_path / "Hawassi_u_01.dat", dtype=np.float32).reshape(-1, ny, nx)
    assert np.array_equal(u1[0], u0.astype(np.float32))
    ora2 = Oracle2D(tb, 1e-8, 1e-6)
    z3, t3, h3 = z0.copy(), 0.0, 0.02
    for ti in tout[1:4]:   # the loop stops at every output time
        t3, h3 = ora2.run_to(t3, ti, h3, z3)
    e2 = np.fromfile(tmp_path / "Hawassi_eta_02.dat", dtype=np.float32).reshape(2, ny, nx)
    eta3, u3, v3 = fields2d(nx, ny, z3)
    assert np.array_equal(e2[1], eta3.astype(np.float32))
    # gauges: two header rows (x, y of the nearest grid points), then t and the values
    rows = [ln.split() for ln in open(tmp_path / "Hawassi_v_gauge.dat").read().splitlines()]
    assert len(rows) == 2 + 7
    assert rows[0] == ["0", "%f" % tb["x"][5], "%f" % tb["x"][40]]
    assert rows[1] == ["0", "%f" % tb["y"][3], "%f" % tb["y"][20]]
    assert rows[2] == ["%f" % 0.0, "%f" % v0[3, 5], "%f" % v0[20, 40]]
    assert rows[5] == ["%f" % 0.3, "%f" % v3[3, 5], "%f" % v3[20, 40]]


def test_gauge_outside_the_domain(tmp_path):
    tb = small_tables()
    args = decks2d.outputs(tb, [0.0, 0.1], gauges=[(tb["x"][-1] + 5.0, 0.0)])
    with pytest.raises(RuntimeError, match="outside of the domain"):
        run_outputs2d(Oracle2D(tb), 0.0, 0.02, np.zeros(6 * tb["nx"] * tb["ny"]), tmp_path, **args)
