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


def _read_constants(path):
    a = np.fromfile(path, dtype=np.float64)
    nx = int(a[0])
    nt = int(a[1 + nx])
    rest = a[2 + nx + nt:]
    return dict(x=a[1:1 + nx], t=a[2 + nx:2 + nx + nt], depth=rest[:nx], k=rest[nx:2 * nx],
                nu_peak=rest[2 * nx:2 * nx + 1])


def test_output_files_match_golden_constants_and_oracle(golden_dir, tmp_path):
    deck = os.path.join(golden_dir, "fbr005")
    e = hw.Engine(deck, cluster=2)
    e.enable_fields()
    e.run_to_time(2.0)
    rows = e.write_outputs(str(tmp_path / "gpu"))
    assert rows >= 90
    # Constants_01.dat: the reference's own output, array for array
    gold = np.load(os.path.join(golden_dir, "fbr005_constants.npz"))
    mine = _read_constants(str(tmp_path / "gpu" / "Constants_01.dat"))
    for key in ("x", "t", "depth", "k", "nu_peak"):
        assert np.array_equal(mine[key], gold[key]), key
    # fields and gauge text against the oracle's output loop
    os.makedirs(tmp_path / "ora", exist_ok=True)
    o = ol.Oracle(deck, t_stop=2.0, write_fields=1, outdir=str(tmp_path / "ora"))
    o.run()
    o.close()
    nx = e.nx[0]
    for name in ("eta", "u", "phi"):
        a = np.fromfile(str(tmp_path / "gpu" / f"Hawassi_{name}_01.dat")).reshape(-1, nx)
        b = np.fromfile(str(tmp_path / "ora" / f"Hawassi_{name}_01.dat")).reshape(-1, nx)
        r = min(len(a), len(b))
        assert r >= 90
        assert np.abs(a[:r] - b[:r]).max() <= 1e-9 * np.abs(b[:r]).max(), name
    assert open(tmp_path / "gpu" / "Hawassi_eta_gauge.txt").readline().split() == ["0", "20.000000"]


def test_output_partitions(tmp_path):
    deck = small_deck(tmp_path, "part", nx=1024, T_end=2.0, n_samples=101, npartition=3,
                      gauges=(10.0, 25.0))
    e = hw.Engine(deck, eps_abs=1e-8, eps_rel=1e-6)
    e.enable_fields()
    e.run()
    assert e.write_outputs(str(tmp_path / "gpu")) == 101
    os.makedirs(tmp_path / "ora", exist_ok=True)
    o = ol.Oracle(deck, eps_abs=1e-8, eps_rel=1e-6, write_fields=1, outdir=str(tmp_path / "ora"))
    o.run()
    o.close()
    # 101 samples in 3 partitions of 33 and a rest of 2: files 01..04
    for ip in range(1, 5):
        sfx = f"{ip:02d}.dat"
        a = open(tmp_path / "gpu" / f"Constants_{sfx}", "rb").read()
        b = open(tmp_path / "ora" / f"Constants_{sfx}", "rb").read()
        assert a == b, sfx
        fa = np.fromfile(str(tmp_path / "gpu" / f"Hawassi_eta_{sfx}"))
        fb = np.fromfile(str(tmp_path / "ora" / f"Hawassi_eta_{sfx}"))
        assert fa.size == fb.size and fa.size == (33 if ip <= 3 else 2) * 1024
        assert np.abs(fa - fb).max() <= 1e-9 * max(np.abs(fb).max(), 1e-300)
