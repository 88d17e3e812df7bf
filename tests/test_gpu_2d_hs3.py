"""HS3 on the flat bottom (rhs_AB3_2DF_uv) on the device against the 2D oracle
restatement: the RHS (every grid shape, ChiAdj on and off, walls of both branches),
the stepping, and kinematic breaking with the HS3 RHS."""
import numpy as np
import pytest

from breaking2d_case import steep_crest_case
from hawassi_c_b200 import decks2d
from hawassi_c_b200.engine2d import Engine2D
from oracle_lib import Oracle2D
from test_oracle2d_output import smooth_fields, state_of

pytestmark = pytest.mark.gpu


def tables(nx, ny, nadj=1.0, propagation=0, walls=(), refl=0.5, seed=1):
    return decks2d.tables(nx=nx, ny=ny, Lx=0.9 * nx, Ly=0.9 * ny, depth=2.0, Hs=0.1, Tp=3.0, n_freq=24, n_dir=6,
                          t_end=6.0, dt=0.1, damp=6.0, x_line=10.0, nadj=nadj, propagation=propagation, seed=seed,
                          walls=walls, refl=refl, model=3)


def band_limited_state(tb, amp, seed):
    rng = np.random.default_rng(seed)
    n = tb["nx"] * tb["ny"]
    return amp * rng.standard_normal(6 * n) * np.tile(tb["aal"].ravel(), 6) * np.sqrt(n)


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


@pytest.mark.parametrize("nx,ny,nadj,prop", [
    (64, 64, 1.0, 0), (128, 64, 1.0, 1), (64, 128, 0.0, 2), (256, 256, 1.0, 0), (1024, 64, 1.0, 0),
    (64, 1024, 0.0, 0),
])
def test_rhs_parity_hs3(nx, ny, nadj, prop):
    tb = tables(nx, ny, nadj=nadj, propagation=prop)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    for seed, t in ((1, 0.7), (2, 3.3)):
        y = band_limited_state(tb, 0.03, seed)
        assert rel(eng.rhs(t, y), ora.rhs(t, y)) < 1e-11


def test_rhs_parity_hs3_unfiltered_state():
    """Every wavenumber excited: the symmetrisation edges of the cubic terms too."""
    tb = tables(128, 64)
    eng, ora = Engine2D(tb), Oracle2D(tb)
    rng = np.random.default_rng(9)
    y = 0.01 * rng.standard_normal(6 * tb["nx"] * tb["ny"]) * 90
    assert rel(eng.rhs(1.0, y), ora.rhs(1.0, y)) < 1e-11


@pytest.mark.parametrize("refl", [0.5, 1.0])
def test_rhs_parity_hs3_wall(refl):
    tb = tables(128, 128, walls=((60.0, 30.0, 66.0, 90.0),), refl=refl)
    eng, ora = Engine2D(tb), Oracle2D(tb)
    for seed in (3, 4):
        y = band_limited_state(tb, 0.03, seed)
        assert rel(eng.rhs(0.9, y), ora.rhs(0.9, y)) < 1e-11


def test_run_to_time_parity_hs3():
    tb = tables(64, 64)
    eng, ora = Engine2D(tb, 1e-8, 1e-6), Oracle2D(tb, 1e-8, 1e-6)
    y = state_of(*[2.5 * a for a in smooth_fields(tb, 5)])
    eng.set_state(0.0, 0.02, y)
    to, ho = 0.0, 0.02
    for T in (0.6, 1.2):
        eng.run_to_time(T)
        to, ho = ora.run_to(to, T, ho, y)
        tg, hg, yg = eng.state()
        assert tg == T
        assert rel(yg, y) < 1e-9
    sg, so = eng.stats(), ora.stats()
    assert sg["accepted"] == so["accepted"] and sg["rejected"] == so["rejected"]


def test_breaking_evolve_parity_hs3():
    tb, z = steep_crest_case(64, 64, bathymetry="flat", model=3)
    eng, ora = Engine2D(tb, 1e-6, 1e-4), Oracle2D(tb, 1e-6, 1e-4)
    t0, h0 = 0.3, 0.005
    eng.set_state(t0, h0, z)
    ora.set_tprev(t0)
    ya, yb = z.copy(), z.copy()
    ta, ha, tb_, hb = t0, h0, t0, h0
    for _ in range(6):
        ta, ha = ora.evolve_apply(ta, 0.6, ha, ya)
        tb_, hb = eng.evolve_apply(tb_, 0.6, hb, yb)
        assert abs(ta - tb_) < 1e-11 and abs(ha - hb) <= 1e-6 * abs(ha)
        assert rel(yb, ya) < 1e-9
    assert eng.stats()["accepted"] == ora.stats()["accepted"]
    la, lb = eng.breaking_log(), ora.breaking_log()
    assert len(la) == len(lb) and all(a[1] == b[1] for a, b in zip(la, lb))
