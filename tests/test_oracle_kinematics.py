"""Kinematics restatement (kinematic_modul, 1d/kinematic_modul.c; read_kinematics,
1d/functions.c:3555-3669) in the oracle: the output grid and the properties the
reference's formulas fix."""
import numpy as np

import oracle_lib as ol
from decks_util import random_state, small_deck

G = 9.80665


def _deck(tmp, varying=False, nx=1024):
    return small_deck(tmp, f"kin{int(varying)}{nx}", nx=nx, varying=varying, kinematic=True,
                      kin_window=(0.4 * 0.05 * nx, 0.6 * 0.05 * nx), nsurf=20, ndeep=15, T_end=4.0)


def test_kinematics_grid(tmp_path):
    o = ol.Oracle(_deck(tmp_path), eps_abs=1e-8, eps_rel=1e-6)
    r = o.kinematics(1.0, 0.5, np.zeros(4 * 1024), np.zeros(4 * 1024))
    z, x = r["z_out"], r["x_out"]
    assert z.size == 35 and np.all(np.diff(z) > 0)
    hs = o.scalar("Hs_in")
    # surface layer: 20 equal steps between -2.5 Hs and 2.5 Hs (initial zero)
    surf = z[z >= -2.5 * hs - 1e-12]
    assert surf.size >= 20 and abs(z.max() - 2.5 * hs) < 1e-12
    assert abs(x[0] - 0.4 * 0.05 * 1024) < 0.06 and abs(x[-1] - 0.6 * 0.05 * 1024) < 0.06


def test_kinematics_still_water_is_hydrostatic(tmp_path):
    """Zero state: no motion, P = -g z in the water, NaN above the surface."""
    o = ol.Oracle(_deck(tmp_path, varying=True), eps_abs=1e-8, eps_rel=1e-6)
    r = o.kinematics(1.0, 0.5, np.zeros(4 * 1024), np.zeros(4 * 1024))
    z = r["z_out"]
    wet = ~np.isnan(r["P"])
    assert np.array_equal(wet, np.broadcast_to(z[None, :] <= 0, wet.shape) & wet)
    assert wet.any() and np.all(np.isnan(r["P"][:, z > 0]))
    zz = np.broadcast_to(z[None, :], r["P"].shape)
    assert np.abs(r["P"][wet] + G * zz[wet]).max() < 1e-12
    assert np.abs(r["dxphi"][wet]).max() == 0 and np.abs(r["dzphi"][wet]).max() == 0


def test_kinematics_masks_follow_surface_and_bed(tmp_path):
    o = ol.Oracle(_deck(tmp_path, varying=True), eps_abs=1e-8, eps_rel=1e-6)
    y = random_state(1024, 11, scale=4e-3)
    dy = o.rhs(1.0, y)
    r = o.kinematics(1.0, 0.98, y, dy)
    eta = r["eta_cut"]
    z = r["z_out"]
    nan = np.isnan(r["dxphi"])
    assert np.array_equal(nan[:, :], (z[None, :] > eta[:, None]) | nan)
    assert np.all(nan[z[None, :].repeat(eta.size, 0) > eta[:, None]])
    # accelerations are the velocities over (t - tprev), as the reference divides them
    fin = ~nan
    assert np.allclose(r["dtdxphi"][fin], r["dxphi"][fin] / 0.02, rtol=1e-12, atol=0)
