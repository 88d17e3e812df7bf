"""Kinematics on the device (hw_kinematics: kinematic_modul, 1d/kinematic_modul.c)
against the oracle's restatement, from the same state and RHS (the engine's own
after a step), flat and sloping bottoms."""
import numpy as np
import pytest

import hawassi_c_b200 as hw
import oracle_lib as ol
from decks_util import random_state, small_deck

pytestmark = pytest.mark.gpu

FIELDS = ("P", "dxphi", "dzphi", "dtdxphi", "dtdzphi")


@pytest.mark.parametrize("nx,varying", [(1024, False), (1024, True), (4096, True)])
def test_kinematics_parity(tmp_path, nx, varying):
    deck = small_deck(tmp_path, "kin", nx=nx, varying=varying, kinematic=True,
                      kin_window=(0.35 * 0.05 * nx, 0.65 * 0.05 * nx), nsurf=20, ndeep=15, T_end=4.0)
    o = ol.Oracle(deck, eps_abs=1e-8, eps_rel=1e-6)
    e = hw.Engine(deck, eps_abs=1e-8, eps_rel=1e-6, device=0)
    y = random_state(nx, 5, scale=3e-3)
    t, h = e.evolve_apply(1.0, 1.5, 1e-3, y)           # state and last RHS on the device
    dy = e.last_dydt()
    tprev = 1.0
    got = e.kinematics(tprev)
    ref = o.kinematics(t, tprev, y, dy)
    assert np.array_equal(got["x_out"], ref["x_out"]) and np.allclose(got["z_out"], ref["z_out"], rtol=0, atol=1e-13)
    assert np.abs(got["eta_cut"] - ref["eta_cut"]).max() <= 1e-12 * np.abs(ref["eta_cut"]).max()
    for f in FIELDS:
        a, b = got[f], ref[f]
        assert np.array_equal(np.isnan(a), np.isnan(b)), f
        fin = ~np.isnan(b)
        assert fin.any()
        err = np.abs(a[fin] - b[fin]).max() / np.abs(b[fin]).max()
        assert err < 1e-10, (f, err)
    e.close()
    o.close()


def test_kinematics_rejects_plain_deck(tmp_path):
    deck = small_deck(tmp_path, "plain", nx=1024)
    e = hw.Engine(deck, device=0)
    with pytest.raises(hw.EngineError):
        e.kinematics(0.0)
    e.close()
