"""Generate the oracle fixtures of the long configuration runs (CPU only).

    python tests/golden/make_oracle_fixtures.py [c2]

These runs take the CPU oracle tens of minutes, far too long for a test, so
their outcome is committed here and the GPU tests compare against it.

c2_k3_onset.npz -- the 1D varying-bathymetry breaking configuration (L = 400 m,
  Nx = 16384, 1.0 m flat to x = 150 m then a 1:30 slope to 0.05 m, HS3,
  kinematic breaking KBC 0.8 / TC 0.2 / Tchar 0.5, JONSWAP Hs 0.15 m, Tp 2.5 s,
  gamma 3.3, seed 0, rtol 1e-6 / atol 1e-8) with the reference's own operator:
  three reference depths (Up3IP).  The oracle is stepped output sample by output
  sample (the loop of ode_solver_Ham, 1d/functions.c:546-553) until the first
  breaking.dat record appears (sample index i_onset), and then EXTRA more
  samples.  Stored: the influx file's digest (the GPU side rebuilds the deck
  from the same seed and checks it), i_onset, the step counters at i_onset and
  at the end, the breaking log at both, the quadratic energy of the state at
  both, and eta, u in physical space at every 16th grid point at the end.
"""
import hashlib
import os
import sys
import tempfile
import time

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path.insert(0, ROOT)
sys.path.insert(0, os.path.join(ROOT, "tests"))

import oracle_lib as ol  # noqa: E402
from hawassi_c_b200 import decks  # noqa: E402

G = 9.80665
EXTRA = 10


def file_digest(path):
    with open(path, "rb") as f:
        return hashlib.sha256(f.read()).hexdigest()


def energy(y, csqr, dx):
    """1/2 int (g eta^2 + u (C^2/g) u) dx by Parseval, C^2 of the influx depth (the
    definition of hw_energy)."""
    n = csqr.size
    e2 = y[:n] ** 2 + y[n:2 * n] ** 2
    u2 = y[2 * n:3 * n] ** 2 + y[3 * n:] ** 2
    return 0.5 * float(np.sum(G * e2 + csqr / G * u2)) * dx / n


def physical(y):
    n = y.size // 4
    eta = np.fft.ifft(y[:n] + 1j * y[n:2 * n]).real
    u = np.fft.ifft(y[2 * n:3 * n] + 1j * y[3 * n:]).real
    return eta, u


def make_c2(out_path):
    with tempfile.TemporaryDirectory() as tmp:
        deck = decks.config2_deck(os.path.join(tmp, "c2"), seed=0)
        digest = file_digest(os.path.join(deck, "influx.dat"))
        o = ol.Oracle(deck, eps_abs=1e-8, eps_rel=1e-6)
        csqr, dx = o.table("Csqr"), o.scalar("dx")
        tt = o.table("ttrace")
        y = o.initial_state()
        t, h = float(tt[0]), 1e-4
        i_onset, rec = -1, {}
        t_wall = time.time()
        for i in range(1, tt.size):
            while t < tt[i]:
                t, h = o.evolve_apply(t, tt[i], h, y)
            if i_onset < 0 and o.breaking_log():
                i_onset = i
                rec["onset_stats"] = np.array(o.stats(), dtype=np.int64)
                rec["onset_t"] = t
                rec["onset_log"] = o.breaking_log()
                rec["onset_energy"] = energy(y, csqr, dx)
                print(f"onset at sample {i}, t = {t:.6f} ({time.time() - t_wall:.0f} s)", flush=True)
            if i % 100 == 0:
                print(f"sample {i} t {t:.3f} stats {o.stats()} ({time.time() - t_wall:.0f} s)", flush=True)
            if i_onset > 0 and i == i_onset + EXTRA:
                break
        if i_onset < 0:
            raise RuntimeError("no breaking record before t_end")
        eta, u = physical(y)
        np.savez_compressed(
            out_path, influx_sha256=digest, i_onset=i_onset, i_end=i_onset + EXTRA, t_end=t, h_end=h,
            end_stats=np.array(o.stats(), dtype=np.int64), end_log=o.breaking_log(), end_energy=energy(y, csqr, dx),
            eta16=eta[::16], u16=u[::16], **rec)
        o.close()


if __name__ == "__main__":
    which = sys.argv[1:] or ["c2"]
    if "c2" in which:
        make_c2(os.path.join(HERE, "c2_k3_onset.npz"))
