"""2D flat-bottom engine (hw2d_*) against the 2D oracle restatement."""
import numpy as np
import pytest

from hawassi_c_b200 import decks2d
from hawassi_c_b200.engine2d import Engine2D
from oracle_lib import Oracle2D

pytestmark = pytest.mark.gpu


def tables(nx, ny, nadj=1.0, propagation=0, seed=1, source=True, bathymetry="flat", walls=(), model=2):
    tb = decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=24,
                        n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=nadj, propagation=propagation,
                        seed=seed, bathymetry=bathymetry, walls=walls, model=model)
    if not source:
        for k in ("newgam", "skewgam", "tsig", "sig", "sigskew"):
            tb[k] = None
        tb["nt"] = 0
    return tb


def band_limited_state(tb, amp, seed):
    """Random spectral state inside the aliasing mask (what the stepper keeps)."""
    rng = np.random.default_rng(seed)
    n = tb["nx"] * tb["ny"]
    a = np.tile(tb["aal"].ravel(), 6)
    return amp * rng.standard_normal(6 * n) * a * np.sqrt(n)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("nx,ny,nadj,prop", [
    (64, 64, 1.0, 0), (128, 64, 1.0, 1), (64, 128, 0.0, 2), (256, 256, 1.0, 0), (1024, 64, 1.0, 0),
    (64, 1024, 1.0, 0),
])
def test_rhs_parity(nx, ny, nadj, prop):
    tb = tables(nx, ny, nadj=nadj, propagation=prop)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed, t in ((1, 0.7), (2, 3.3)):
        y = band_limited_state(tb, 0.02, seed)
        assert rel(eng.rhs(t, y), ora.rhs(t, y)) < 1e-11


def test_rhs_parity_unfiltered_state():
    """Every wavenumber excited (the Nyquist lines and the symmetrisation edges too)."""
    tb = tables(128, 64)
    eng, ora = Engine2D(tb), Oracle2D(tb)
    rng = np.random.default_rng(9)
    y = 0.01 * rng.standard_normal(6 * tb["nx"] * tb["ny"]) * 90
    assert rel(eng.rhs(1.0, y), ora.rhs(1.0, y)) < 1e-11


def test_rhs_without_source():
    tb = tables(128, 128, source=False)
    eng, ora = Engine2D(tb), Oracle2D(tb)
    y = band_limited_state(tb, 0.02, 4)
    assert rel(eng.rhs(0.0, y), ora.rhs(0.0, y)) < 1e-11


def test_evolve_apply_replay():
    """One gsl_odeiv2_evolve_apply call from the same state, on both sides."""
    tb = tables(64, 64)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y0 = band_limited_state(tb, 0.01, 5)
    for t0, h0 in ((0.5, 0.01), (1.0, 0.2), (2.0, 1e-3)):
        yg, yo = y0.copy(), y0.copy()
        tg, hg = eng.evolve_apply(t0, t0 + 0.5, h0, yg)
        to, ho = ora.evolve_apply(t0, t0 + 0.5, h0, yo)
        assert abs(tg - to) <= 1e-13 * max(1.0, abs(to))
        assert abs(hg - ho) <= 1e-6 * abs(ho)
        assert rel(yg, yo) < 1e-12


def test_run_to_time_parity():
    tb = tables(64, 64)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    n6 = 6 * tb["nx"] * tb["ny"]
    y = np.zeros(n6)
    eng.set_state(0.0, 0.02, y)
    to, ho = 0.0, 0.02
    for T in (1.0, 2.5, 4.0):
        eng.run_to_time(T)
        to, ho = ora.run_to(to, T, ho, y)
        tg, hg, yg = eng.state()
        assert tg == T
        assert rel(yg, y) < 1e-9
    sg, so = eng.stats(), ora.stats()
    assert sg["accepted"] == so["accepted"] and sg["rejected"] == so["rejected"]


def test_gsl_rhs_entry_matches_rhs():
    import ctypes
    tb = tables(64, 64)
    eng = Engine2D(tb)
    y = band_limited_state(tb, 0.02, 7)
    a = eng.rhs(1.5, y)
    out = np.empty_like(y)
    dp = ctypes.POINTER(ctypes.c_double)
    rc = eng._L.hw2d_gsl_rhs(1.5, y.ctypes.data_as(dp), out.ctypes.data_as(dp), ctypes.c_void_p(eng._h))
    assert rc == 0
    assert np.array_equal(a, out)


def test_bad_tables_rejected():
    tb = tables(64, 64)
    tb["nx"] = 96
    with pytest.raises(Exception):
        Engine2D(tb)


# --- varying bottom, two reference depths (rhs_AB2_2DB_uv) -------------------
@pytest.mark.parametrize("nx,ny,nadj", [(64, 64, 1.0), (128, 64, 0.0), (64, 128, 1.0), (256, 256, 1.0)])
def test_rhs_parity_varying_depth(nx, ny, nadj):
    tb = tables(nx, ny, nadj=nadj, bathymetry="shoal")
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed, t in ((1, 0.7), (2, 3.3)):
        y = band_limited_state(tb, 0.02, seed)
        assert rel(eng.rhs(t, y), ora.rhs(t, y)) < 1e-11


def test_rhs_parity_varying_depth_unfiltered():
    tb = tables(128, 64, bathymetry="shoal")
    eng, ora = Engine2D(tb), Oracle2D(tb)
    rng = np.random.default_rng(11)
    y = 0.01 * rng.standard_normal(6 * tb["nx"] * tb["ny"]) * 90
    assert rel(eng.rhs(1.0, y), ora.rhs(1.0, y)) < 1e-11


def test_run_to_time_parity_varying_depth():
    tb = tables(64, 64, bathymetry="shoal")
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = np.zeros(6 * tb["nx"] * tb["ny"])
    eng.set_state(0.0, 0.02, y)
    to, ho = 0.0, 0.02
    for T in (1.0, 2.5):
        eng.run_to_time(T)
        to, ho = ora.run_to(to, T, ho, y)
        tg, hg, yg = eng.state()
        assert tg == T
        assert rel(yg, y) < 1e-9
    sg, so = eng.stats(), ora.stats()
    assert sg["accepted"] == so["accepted"] and sg["rejected"] == so["rejected"]


# --- harbour wall (dominfo.wallchar in the H2 products, damping inside the wall) --
def _wall(nx, ny):
    Lx, Ly = 0.9 * nx, 0.9 * ny
    return ((0.6 * Lx, 0.3 * Ly, 0.63 * Lx, 0.7 * Ly),)


@pytest.mark.parametrize("nx,ny,bottom", [(64, 64, "shoal"), (128, 128, "shoal"), (64, 64, "flat"), (128, 64, "flat")])
def test_rhs_parity_wall(nx, ny, bottom):
    """Walls: wallchar in the H2 products on both bottoms, and on the flat bottom
    fun_delphiH1hat's round trip of (C u^, C v^) through the wall mask."""
    tb = tables(nx, ny, bathymetry=bottom, walls=_wall(nx, ny))
    assert (tb["wallchar"] < 1).any()
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = band_limited_state(tb, 0.02, 3)
    assert rel(eng.rhs(1.1, y), ora.rhs(1.1, y)) < 1e-11


@pytest.mark.parametrize("bottom", ["shoal", "flat"])
def test_run_to_time_parity_wall(bottom):
    tb = tables(64, 64, bathymetry=bottom, walls=_wall(64, 64))
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = np.zeros(6 * tb["nx"] * tb["ny"])
    eng.set_state(0.0, 0.02, y)
    to, ho = ora.run_to(0.0, 2.0, 0.02, y)
    eng.run_to_time(2.0)
    tg, hg, yg = eng.state()
    assert tg == to and rel(yg, y) < 1e-9


@pytest.mark.parametrize("nx,ny", [(64, 64), (128, 64)])
def test_fully_reflecting_wall_flat_bottom(nx, ny):
    """refl_coef = 1: fun_delphiH1hat's flux branch (divergence through the mask,
    fluxes through its gradient)."""
    tb = decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                        t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=1, walls=_wall(nx, ny), refl=1.0)
    assert tb["refl_coef"] == 1.0 and (tb["wallchar"] == 0).any()
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = band_limited_state(tb, 0.02, 5)
    assert rel(eng.rhs(0.9, y), ora.rhs(0.9, y)) < 1e-11
    if nx == 64:
        y = np.zeros(6 * nx * ny)
        eng.set_state(0.0, 0.02, y)
        to, ho = ora.run_to(0.0, 2.0, 0.02, y)
        eng.run_to_time(2.0)
        tg, hg, yg = eng.state()
        assert tg == to and rel(yg, y) < 1e-9


@pytest.mark.parametrize("nx,ny,prop,bottom", [(64, 64, 0, "flat"), (128, 64, 2, "flat"), (64, 128, 0, "shoal")])
def test_rhs_parity_hs1(nx, ny, prop, bottom):
    """HS1 (rhs_AB1_2DF_uv / rhs_AB1_2DB_uv): the linear model with damping and source."""
    tb = tables(nx, ny, propagation=prop, model=1, bathymetry=bottom)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = band_limited_state(tb, 0.02, 3)
    assert rel(eng.rhs(0.8, y), ora.rhs(0.8, y)) < 1e-11


@pytest.mark.parametrize("bottom,refl", [("flat", 0.5), ("flat", 1.0), ("shoal", 0.5)])
def test_rhs_parity_hs1_wall(bottom, refl):
    """HS1 with walls: on the flat bottom fun_delphiH1hat's wall branches (both), on the
    two-depth bottom the walls enter through the tables only (HS1's cutoff
    coefficients, no x10 damping)."""
    tb = decks2d.tables(nx=64, ny=64, Lx=57.6, Ly=57.6, depth=2.0, shallow=0.6, Hs=0.1, Tp=3.0, n_freq=24,
                        n_dir=6, t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, seed=1, walls=_wall(64, 64), refl=refl,
                        model=1, bathymetry=bottom)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed in (3, 4):
        y = band_limited_state(tb, 0.02, seed)
        assert rel(eng.rhs(0.8, y), ora.rhs(0.8, y)) < 1e-11


def test_run_to_time_parity_hs1():
    tb = tables(64, 64, model=1)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = np.zeros(6 * tb["nx"] * tb["ny"])
    eng.set_state(0.0, 0.02, y)
    to, ho = ora.run_to(0.0, 3.0, 0.02, y)
    eng.run_to_time(3.0)
    tg, hg, yg = eng.state()
    assert tg == 3.0 and rel(yg, y) < 1e-9
    sg, so = eng.stats(), ora.stats()
    # a step whose error ratio sits on the 1.1 rejection threshold to rounding can be
    # decided either way (measured once in 16 rejections): allow one such decision
    assert abs(sg["accepted"] - so["accepted"]) <= 1 and abs(sg["rejected"] - so["rejected"]) <= 1

