"""2D kinematic breaking on the device (breaking_process and fun_sbreaking as called
by rhs_AB2_2DB_uv) against the 2D oracle restatement, on the steep-crest deck.

The breaking state advances on every RHS past tprev, rejected attempts included,
so parity is checked on the same sequence of calls: the step sizes, the accepted
and rejected counts, the crest flags, the break nodes of breaking.dat (identical
lists), B and the eddy-viscosity force Sb, and the state."""
import numpy as np
import pytest

from breaking2d_case import steep_crest_case
from hawassi_c_b200.engine2d import Engine2D
from oracle_lib import Oracle2D

pytestmark = pytest.mark.gpu

EPS_ABS, EPS_REL = 1e-6, 1e-4


def rel(a, b):
    return np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300)


def same_logs(a, b):
    assert len(a) == len(b)
    for (ta, na), (tb_, nb) in zip(a, b):
        assert abs(ta - tb_) <= 1e-12 * max(1.0, abs(tb_))
        assert na == nb


def check_fields(eng, ora, tol=1e-8):
    Be, sxe, sye, fe, ne = eng.breaking_fields()
    Bo, sxo, syo, fo, no = ora.breaking_fields()
    assert (fe, ne) == (fo, no)
    assert np.array_equal(Be > 0, Bo > 0)
    assert np.abs(Be - Bo).max() < 1e-9
    if np.abs(sxo).max() > 0:
        assert rel(sxe, sxo) < tol and rel(sye, syo) < tol
    else:
        assert np.abs(sxe).max() == 0
    return fo


@pytest.mark.parametrize("nx,ny,bottom", [(64, 64, "shoal"), (128, 64, "shoal"), (64, 128, "flat")])
def test_breaking_evolve_parity(nx, ny, bottom):
    tb, z = steep_crest_case(nx, ny, bathymetry=bottom)
    eng, ora = Engine2D(tb, EPS_ABS, EPS_REL), Oracle2D(tb, EPS_ABS, EPS_REL)
    t0, h0 = 0.3, 0.005
    eng.set_state(t0, h0, z)
    ora.set_tprev(t0)
    ya, yb = z.copy(), z.copy()
    ta, ha, tb_, hb = t0, h0, t0, h0
    flags = []
    for _ in range(8):
        ta, ha = ora.evolve_apply(ta, 0.6, ha, ya)
        tb_, hb = eng.evolve_apply(tb_, 0.6, hb, yb)
        # t and h derive from the embedded error estimate: they agree to ~1e-12 relative
        assert abs(ta - tb_) < 1e-11 and abs(ha - hb) <= 1e-6 * abs(ha)
        assert rel(yb, ya) < 1e-9
        assert eng.stats()["accepted"] == ora.stats()["accepted"]
        assert eng.stats()["rejected"] == ora.stats()["rejected"]
        flags.append(check_fields(eng, ora))
    assert 2 in flags                      # crests were tracked with break nodes
    same_logs(eng.breaking_log(), ora.breaking_log())


def test_breaking_direct_rhs_update():
    """One RHS past tprev: the criterion runs, dt eta^ takes the symmetrised delphiH^."""
    tb, z = steep_crest_case(64, 64)
    eng, ora = Engine2D(tb, EPS_ABS, EPS_REL), Oracle2D(tb, EPS_ABS, EPS_REL)
    eng.set_state(0.3, 0.005, z)
    ora.set_tprev(0.3)
    t = 0.3 + 0.004
    assert rel(eng.rhs(t, z), ora.rhs(t, z)) < 1e-11
    check_fields(eng, ora)
    same_logs(eng.breaking_log(), ora.breaking_log())
    # at t == tprev no update runs
    assert rel(eng.rhs(0.3, z), ora.rhs(0.3, z)) < 1e-11


def test_breaking_run_to_time_parity():
    """The device loop (graph-captured attempts replayed in batches) to t = 0.33."""
    tb, z = steep_crest_case(64, 64)
    eng, ora = Engine2D(tb, EPS_ABS, EPS_REL), Oracle2D(tb, EPS_ABS, EPS_REL)
    eng.set_state(0.3, 0.005, z)
    ora.set_tprev(0.3)
    y = z.copy()
    t, h = ora.run_to(0.3, 0.33, 0.005, y)
    eng.run_to_time(0.33)
    te, he, ye = eng.state()
    assert abs(te - t) < 1e-11 and abs(he - h) <= 1e-6 * abs(h)
    assert rel(ye, y) < 1e-9
    so, se = ora.stats(), eng.stats()
    assert (se["accepted"], se["rejected"]) == (so["accepted"], so["rejected"])
    check_fields(eng, ora)
    log = ora.breaking_log()
    assert len(log) > 0
    same_logs(eng.breaking_log(), log)
