"""The 2D set-up's directional JONSWAP line signal (jonswap_influx,
2d/functions.c:2310-2446) on the device (hw2d_directional_influx) against the
oracle's direct sum, and a 2D deck built on it running in parity."""
import math

import numpy as np
import pytest

import oracle_lib as ol
from hawassi_c_b200 import decks2d

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("nt,nlines,s_spread,mdir", [(401, 64, 10.0, 0.0), (1000, 37, 4.0, 0.3), (257, 16, None, 0.0)])
def test_directional_signal_matches_direct_sum(nt, nlines, s_spread, mdir):
    from hawassi_c_b200.engine2d import directional_signal
    dt = 0.1
    t = np.arange(nt) * dt
    y = np.linspace(0.0, 60.0, nlines)
    comps = decks2d.reference_directional_components(t, 0.5, 6.0, 3.3, s_spread, 4.0, seed=3)
    r = np.clip(t / 2.0, 0, 1)
    ramp_t, ramp_y = 0.5 * (1 - np.cos(math.pi * r)), np.linspace(0.5, 1.0, nlines)
    eta, skew = directional_signal(0.0, dt, nt, y, y[0], comps, mdir=mdir, ramp_t=ramp_t, ramp_y=ramp_y)
    e_o, s_o = ol.directional_signal_2d(t, y, y[0], comps, mdir=mdir, ramp_t=ramp_t, ramp_y=ramp_y)
    scale = np.abs(e_o).max()
    assert scale > 0.01
    assert np.abs(eta - e_o).max() < 1e-11 * scale and np.abs(skew - s_o).max() < 1e-11 * scale


def test_deck_on_reference_influx_runs_in_parity():
    """A 2D deck whose line signals come from the reference's influx model: one RHS
    against the oracle, then a short run with the same step counts."""
    from hawassi_c_b200.engine2d import Engine2D
    tb = decks2d.tables(nx=64, ny=64, Lx=57.6, Ly=57.6, depth=2.0, Hs=0.1, Tp=3.0, t_end=6.0, dt=0.1, damp=6.0,
                        x_line=10.0, seed=2, influx_model="reference")
    eng, ora = Engine2D(tb, 1e-8, 1e-6), ol.Oracle2D(tb, 1e-8, 1e-6)
    n = tb["nx"] * tb["ny"]
    y = np.zeros(6 * n)
    eng.set_state(0.0, 0.02, y)
    t, h = ora.run_to(0.0, 3.0, 0.02, y)
    eng.run_to_time(3.0)
    te, he, ye = eng.state()
    assert abs(te - t) < 1e-12
    so, se = ora.stats(), eng.stats()
    assert (se["accepted"], se["rejected"]) == (so["accepted"], so["rejected"])
    assert np.abs(y).max() > 0 and np.linalg.norm(ye - y) / np.linalg.norm(y) < 1e-9
