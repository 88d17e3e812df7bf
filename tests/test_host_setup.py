"""CPU tests of the product's host side (no GPU): the C++ deck parser and table
set-up against the oracle, the deck writer, and the C ABI's exported symbols."""
import ctypes
import os
import re

import numpy as np
import pytest

import oracle_lib as ol
from decks_util import small_deck
from hawassi_c_b200 import decks, engine

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

TABLES = ["x", "k", "depth", "dampchar", "dampcoef", "aal", "ChiAdj", "Csqr", "gamX", "gamX_skew", "insig",
          "insig_skew", "ttrace"]
SCALARS = ["Nx", "n", "dx", "nu_peak", "kp", "lambda_p", "Hs_in", "MaxEtaInit"]


def _compare(deck, nref=0):
    o = ol.Oracle(deck, nref=nref)
    for nm in TABLES:
        a, b = o.table(nm), engine.deck_table(deck, nm, nref=nref)
        assert a.size == b.size, nm
        np.testing.assert_allclose(b, a, rtol=0, atol=1e-13 * max(1.0, np.abs(a).max()), err_msg=nm)
    for nm in SCALARS:
        assert engine.deck_table(deck, nm, nref=nref)[0] == pytest.approx(o.scalar(nm), rel=1e-14), nm
    np.testing.assert_allclose(engine.deck_table(deck, "y0", nref=nref), o.initial_state(), rtol=0, atol=1e-12)
    return o


def test_golden_deck_setup(golden_dir):
    o = _compare(os.path.join(golden_dir, "fbr005"))
    assert o.scalar("breaking") == 1


@pytest.mark.parametrize("model,varying,nref", [("HS2", False, 0), ("HS3", True, 0), ("HS3", True, 2),
                                                ("HS2", True, 16), ("HS1", False, 0)])
def test_synthetic_deck_setup(tmp_path, model, varying, nref):
    deck = small_deck(tmp_path, f"d_{model}_{nref}", nx=1024, model=model, varying=varying)
    o = _compare(deck, nref)
    if varying:
        if nref > 3:
            np.testing.assert_array_equal(engine.deck_table(deck, "gamK", nref=nref), o.table("gamK"))
        else:
            for nm in ("gam_min", "gam_plus", "Csq_min", "Csq_plus"):
                np.testing.assert_array_equal(engine.deck_table(deck, nm, nref=nref), o.table(nm))


def test_config_decks_parse(tmp_path):
    d1 = decks.config1_deck(str(tmp_path / "c1"), seed=2)
    assert engine.deck_table(d1, "Nx")[0] == 4096
    assert engine.deck_table(d1, "n")[0] == 2048
    d2 = decks.config2_deck(str(tmp_path / "c2"), seed=2)
    assert engine.deck_table(d2, "Nx")[0] == 16384
    assert engine.deck_table(d2, "depth").min() == pytest.approx(0.05)


def test_bad_deck_reports_error(tmp_path):
    p = tmp_path / "bad"
    p.mkdir()
    (p / "input.txt").write_text("&INFLUX_SIGNAL\nwavename = zero\n")
    with pytest.raises(engine.EngineError):
        engine.deck_table(str(p), "Nx")


def test_seeded_influx_reproducible(tmp_path):
    t1, e1 = decks.jonswap_signal(100.0, 2048, 1024, 0.1, 2.0, 3.3, seed=5)
    t2, e2 = decks.jonswap_signal(100.0, 2048, 1024, 0.1, 2.0, 3.3, seed=5)
    _, e3 = decks.jonswap_signal(100.0, 2048, 1024, 0.1, 2.0, 3.3, seed=6)
    assert np.array_equal(e1, e2) and not np.array_equal(e1, e3)
    assert 4 * e1.std() == pytest.approx(0.1, rel=1e-12)


def test_library_exports_every_declared_symbol():
    header = open(os.path.join(ROOT, "include", "hawassi_b200.h")).read()
    declared = set(re.findall(r"\b(hw2?d?_[a-z_0-9]+)\s*\(", header))
    lib = ctypes.CDLL(engine.library_path())
    missing = [s for s in sorted(declared) if not hasattr(lib, s)]
    assert not missing, missing
    assert set(engine.EXPORTS) <= declared


def test_reference_decks_setup(tmp_path):
    """Every packed reference deck: the host set-up's tables equal the oracle's
    (AreaShort and Area influx, user-defined bars, an initial-value bore)."""
    from reference_decks import WINDOW, unpack
    decks_ = unpack(tmp_path)
    assert set(decks_) == set(WINDOW)
    for name, deck in decks_.items():
        _compare(deck)


def test_k_reference_weights_reproduce_the_peak_dispersion(tmp_path):
    """The K-reference operator's defining property, checked independently of both
    restatements: at every point the two non-zero weights are those of the bracketing
    pair of log-spaced reference depths, and the blend of the pair's squared phase
    speeds and frequencies at the point's peak wavenumber gives the point's own
    (measured 1.4e-10 and 6.5e-11 relative)."""
    from hawassi_c_b200.learned import kappa_linear, reference_depths
    deck = small_deck(tmp_path, "kref", nx=1024, model="HS2", varying=True)
    K = 16
    g = engine.deck_table(deck, "gamK", nref=K).reshape(K, -1)
    h = engine.deck_table(deck, "depth")
    nu = float(engine.deck_table(deck, "nu_peak")[0])
    D = reference_depths(h, K)
    nz = (g != 0).sum(axis=0)
    assert nz.max() <= 2
    j = np.clip(np.searchsorted(D, h, side="right") - 1, 0, K - 2)
    assert np.all((g[j, np.arange(h.size)] != 0) | (h == D[j + 1]))
    kap = kappa_linear(nu, h)
    G = 9.80665
    cp2 = lambda k, d: G * np.tanh(k * d) / k
    om = lambda k, d: np.sqrt(G * k * np.tanh(k * d))
    blend_c = sum(g[q] * cp2(kap, D[q]) for q in range(K))
    blend_o = sum(g[q] * om(kap, D[q]) for q in range(K))
    assert np.max(np.abs(blend_c / cp2(kap, h) - 1)) < 1e-8
    assert np.max(np.abs(blend_o / om(kap, h) - 1)) < 1e-8


def test_up3ip_weights_solve_the_three_depth_system(golden_dir, tmp_path):
    """Up3IP's weights (1d/functions.c:2247-2340), checked independently of both
    restatements: at every point the blend of the three reference depths' long-wave
    speed, frequency and squared phase speed at the point's peak wavenumber gives the
    point's own -- exactly at the 101 depth samples the reference solves at, to the
    natural spline's interpolation error between them (measured below 3e-5)."""
    from hawassi_c_b200.learned import kappa_linear
    G = 9.80665
    cp2 = lambda k, d: G * np.tanh(k * d) / k
    om = lambda k, d: np.sqrt(G * k * np.tanh(k * d))
    c0 = lambda d: np.sqrt(G * d)
    for deck in (os.path.join(golden_dir, "harmbar"), small_deck(tmp_path, "v3", nx=1024, varying=True)):
        h = engine.deck_table(deck, "depth")
        nu = float(engine.deck_table(deck, "nu_peak")[0])
        g = [engine.deck_table(deck, n) for n in ("gam_min", "gam_mid", "gam_plus")]
        D = (h.min(), (h.min() + h.max()) / 2, h.max())
        kap = kappa_linear(nu, h)
        for f in (lambda d: c0(d), lambda d: om(kap, d), lambda d: cp2(kap, d)):
            blend = sum(gj * f(Dj) for gj, Dj in zip(g, D))
            assert np.max(np.abs(blend / f(h) - 1)) < 1e-4
