"""Small seeded decks shared by the parity tests."""
import os

import numpy as np

from hawassi_c_b200 import decks


def small_deck(root, name, nx=1024, model="HS2", varying=False, breaking=False, T_end=8.0, seed=3,
               Hs=0.08, Tp=1.2, length=None, n_samples=400, n_lines=150, **kw):
    path = os.path.join(str(root), name)
    length = length if length is not None else 0.05 * nx
    bath = None
    if varying:
        bath = decks.slope_bathymetry(nx, length, h0=1.0, x_toe=0.45 * length, slope=1.0 / 30.0, h_min=0.3)
    decks.write_deck(path, nx=nx, length=length, xinflux=0.15 * length, depth=1.0, bath=bath, model=model,
                     breaking=breaking, T_end=T_end, n_samples=n_samples, n_lines=n_lines, Hs=Hs, Tp=Tp,
                     gamma=3.3, seed=seed, damp=(0.08 * length, 0.08 * length), adjcoef=0.5, **kw)
    return path


def random_state(nx, seed, scale=1e-3):
    """A smooth random spectral state (Hermitian-ish) for single-RHS checks."""
    rng = np.random.default_rng(seed)
    eta = np.convolve(rng.standard_normal(nx), np.ones(16) / 16, mode="same") * scale * 20
    u = np.convolve(rng.standard_normal(nx), np.ones(16) / 16, mode="same") * scale * 40
    eh = np.fft.fft(eta)
    uh = np.fft.fft(u)
    # break exact Hermitian symmetry slightly, as the reference state drifts off it
    eh = eh + 1e-6 * (rng.standard_normal(nx) + 1j * rng.standard_normal(nx)) * np.abs(eh).max()
    return np.concatenate([eh.real, eh.imag, uh.real, uh.imag])


def rel_l2(a, b):
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))
