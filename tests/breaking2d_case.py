"""A 2D deck whose waves break within a few steps: the two-depth shoal tables with
kinematic breaking, and a steep crest laid across the shoal whose particle speed
exceeds the phase speed (u ahead of the crest, so that break nodes appear once
the crest is tracked).  Seeded and small enough for the oracle."""
import numpy as np

from hawassi_c_b200 import decks2d

GRAV = 9.80665


def steep_crest_case(nx=64, ny=64, dt_out=0.002, x_crest=40.0, seed=1, bathymetry="shoal", model=2, ninterp=2,
                     walls=()):
    tb = decks2d.tables(nx=nx, ny=ny, Lx=float(nx), Ly=float(ny), depth=3.0 if bathymetry != "flat" else 1.5,
                        shallow=0.5, Hs=0.6, Tp=4.0, n_freq=16, n_dir=4, t_end=10.0, dt=0.1, damp=6.0, x_line=8.0,
                        seed=seed, bathymetry=bathymetry, breaking=True, model=model, ninterp=ninterp, walls=walls)
    tb["dt_out"] = dt_out
    d = -tb["bathy"]
    X, Y = np.meshgrid(tb["x"], tb["y"])
    eta = 0.7 * np.exp(-((X - x_crest) / 3.0) ** 2) * (0.8 + 0.2 * np.cos(2 * np.pi * Y / tb["y"][-1]))
    u = 1.05 * np.sqrt(GRAV * (d + eta)) * np.exp(-((X - x_crest - 1.5) / 3.0) ** 2)
    v = 0.1 * u * np.sin(2 * np.pi * Y / tb["y"][-1])
    n = nx * ny
    z = np.zeros(6 * n)
    for f, a in enumerate((eta, u, v)):
        A = np.fft.fft2(a)
        z[2 * f * n:(2 * f + 1) * n] = A.real.ravel()
        z[(2 * f + 1) * n:(2 * f + 2) * n] = A.imag.ravel()
    return tb, z
