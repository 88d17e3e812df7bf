"""Pins the CPU oracle against the reference's own shipped golden outputs.

Deck 1d/Testcases/1dFBr005Bor (HS2, flat 1 m, Nx=4096, IVP from initial.dat,
kinematic breaking on, reference tolerances eps_abs=1e-5 / eps_rel=1e-4):
  * Constants_01.dat grids (x, t, depth, k from freqspace, nu_peak) bit-exact;
  * Hawassi_eta_gauge.txt (printed %f) within print precision;
  * breaking.dat: every onset line up to t=12.7 s identical (time printed %lf
    and the node indices), which pins RHS, breaking state machine and the
    GSL rkf45/control_y/evolve_apply step sequence together.
Deck 1dB001IrSlope: Constants_01.dat (x, k, depth, nu_peak of a user-defined
influx and bathymetry) when the reference checkout is named by $HAWASSI_REFERENCE.
Deck 1dB002HarmBar (HS2 over a submerged bar: varying bathymetry through the
three-reference-depth operator Up3IP / HSS, Area influx of a user-defined
signal through define_forcing, nonlinear adjustment adjcoef 0.3 (ChiAdj);
reference tolerances, Nx = 2048):
  * Constants_01.dat grids bit-exact;
  * Hawassi_eta_gauge.txt and Hawassi_dteta_gauge.txt within print precision
    over the first 30 s here, and over the whole 196.52 s run in the slow test.
"""
import os

import numpy as np
import pytest

import oracle_lib as ol

_REF_ROOT = os.environ.get("HAWASSI_REFERENCE", "")
REF = os.path.join(_REF_ROOT, "1d", "Testcases", "1dB001IrSlope", "Input") if _REF_ROOT else ""
PRINT = 5.01e-7   # half a unit of %f


def test_fbr005_constants(golden_dir):
    o = ol.Oracle(os.path.join(golden_dir, "fbr005"))
    c = np.load(os.path.join(golden_dir, "fbr005_constants.npz"))
    assert o.nx == 4096
    assert np.array_equal(o.table("x"), c["x"])
    assert np.array_equal(o.table("k"), c["k"])
    assert np.array_equal(o.table("depth"), c["depth"])
    assert np.array_equal(o.table("ttrace")[: c["t"].size], c["t"])
    assert o.scalar("nu_peak") == c["nu_peak"][0]


@pytest.mark.skipif(not (REF and os.path.isdir(REF)), reason="HAWASSI_REFERENCE does not name a reference checkout")
def test_irslope_constants(golden_dir):
    o = ol.Oracle(REF)
    c = np.load(os.path.join(golden_dir, "irslope_constants.npz"))
    assert o.nx == c["x"].size
    assert np.array_equal(o.table("x"), c["x"])
    assert np.array_equal(o.table("k"), c["k"])
    assert np.array_equal(o.table("depth"), c["depth"])
    assert o.scalar("nu_peak") == c["nu_peak"][0]


@pytest.fixture(scope="module")
def fbr_run(golden_dir):
    o = ol.Oracle(os.path.join(golden_dir, "fbr005"), t_stop=12.7)
    tim, ge, gd = o.run()
    return o, tim, ge, gd


def test_fbr005_gauge(golden_dir, fbr_run):
    o, tim, ge, _ = fbr_run
    gold = np.loadtxt(os.path.join(golden_dir, "fbr005_gauge_head.txt"), skiprows=1)
    m = min(len(tim), gold.shape[0])
    assert m > 600
    assert np.abs(gold[:m, 0] - tim[:m]).max() < 1e-9
    assert np.abs(gold[:m, 1] - ge[:m, 0]).max() <= 5.01e-7   # %f print precision


def test_fbr005_breaking_onset(golden_dir, fbr_run):
    o, tim, _, _ = fbr_run
    mine = [l.split() for l in o.breaking_log().splitlines()]
    gold = [l.split() for l in open(os.path.join(golden_dir, "fbr005_breaking_head.txt"))]
    gold = [g for g in gold if float(g[0]) <= tim[-1]]
    assert len(gold) >= 5
    assert len(mine) >= len(gold)
    for a, b in zip(mine, gold):
        assert a == b


def _harmbar_gold(golden_dir):
    z = np.load(os.path.join(golden_dir, "harmbar_gauges.npz"))
    return z["micro_t"] / 1e6, z["micro_eta"] / 1e6, z["micro_dteta"] / 1e6, z["xgauge"]


def test_harmbar_constants(golden_dir):
    o = ol.Oracle(os.path.join(golden_dir, "harmbar"))
    c = np.load(os.path.join(golden_dir, "harmbar_constants.npz"))
    assert o.nx == 2048
    for name in ("x", "k", "depth"):
        assert np.array_equal(o.table(name), c[name]), name
    assert np.array_equal(o.table("ttrace")[: c["t"].size], c["t"])
    # nu_peak is printed from the spectrum of the user-defined signal
    assert o.scalar("nu_peak") == c["nu_peak"][0]


def _harmbar_check(o, tim, ge, gd, golden_dir, t_max):
    t, eta, dteta, _ = _harmbar_gold(golden_dir)
    m = min(len(tim), t.size)
    assert tim[m - 1] >= t_max - 0.05
    assert np.abs(t[:m] - tim[:m]).max() <= PRINT
    assert np.abs(eta[:m] - ge[:m]).max() <= PRINT
    assert np.abs(dteta[:m] - gd[:m]).max() <= PRINT
    # waves reached the gauges: the comparison is not of zeros
    assert np.abs(eta[:m]).max() > 0.01


def test_harmbar_gauges_30s(golden_dir):
    o = ol.Oracle(os.path.join(golden_dir, "harmbar"), t_stop=30.0)
    tim, ge, gd = o.run()
    _harmbar_check(o, tim, ge, gd, golden_dir, 30.0)


@pytest.mark.slow
def test_harmbar_gauges_full_run(golden_dir):
    o = ol.Oracle(os.path.join(golden_dir, "harmbar"))
    tim, ge, gd = o.run()
    assert len(tim) == 5000
    _harmbar_check(o, tim, ge, gd, golden_dir, 196.52)
