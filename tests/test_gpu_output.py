"""Output stage on the device (1d/functions.c:700-760): gauge series of eta and
d eta/dt computed inside the evolve kernel at every output sample, against the
oracle's output loop (or_run) and the reference's golden gauge file."""
import os

import numpy as np
import pytest

import oracle_lib as ol
from decks_util import small_deck

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


def test_gauges_match_golden_and_oracle(golden_dir):
    deck = os.path.join(golden_dir, "fbr005")          # breaking: the exact RHS sequence
    e = hw.Engine(deck, cluster=2)
    e.run_to_time(4.0)
    tim, eta, deta = e.gauges()
    assert len(tim) >= 150 and eta.shape[1] == 1
    o = ol.Oracle(deck, t_stop=4.0)
    to, eo, do = o.run()
    rows = min(len(tim), len(to))
    assert np.allclose(tim[:rows], to[:rows], rtol=1e-12, atol=0)
    scale = np.abs(eo[:rows]).max()
    assert np.abs(eta[:rows] - eo[:rows]).max() <= 1e-9 * scale
    assert np.abs(deta[:rows] - do[:rows]).max() <= 1e-9 * np.abs(do[:rows]).max()
    # the reference's own Hawassi_eta_gauge output, printed with %f
    gold = np.loadtxt(os.path.join(golden_dir, "fbr005_gauge_head.txt"), skiprows=1)
    k = min(rows, len(gold))
    assert np.allclose(tim[:k], gold[:k, 0], atol=5e-7)
    assert np.abs(eta[:k, 0] - gold[:k, 1]).max() <= 5e-7


@pytest.mark.parametrize("nx,cluster", [(1024, 1), (2048, 2), (4096, 4)])
def test_gauges_pure_rhs(tmp_path, nx, cluster):
    length = 0.05 * nx
    gauges = (0.0, 0.3 * length, 0.5 * length + 0.013, 0.9 * length, 0.999 * length)
    deck = small_deck(tmp_path, f"g{nx}", nx=nx, T_end=3.0, gauges=gauges)
    e = hw.Engine(deck, cluster=cluster, eps_abs=1e-8, eps_rel=1e-6)
    e.run()
    tim, eta, deta = e.gauges()
    o = ol.Oracle(deck, eps_abs=1e-8, eps_rel=1e-6)
    to, eo, do = o.run()
    assert len(tim) == len(to) and eta.shape == eo.shape
    assert np.array_equal(tim, to) or np.allclose(tim, to, rtol=1e-13, atol=0)
    assert np.abs(eta - eo).max() <= 1e-9 * np.abs(eo).max()
    assert np.abs(deta - do).max() <= 1e-8 * np.abs(do).max()
