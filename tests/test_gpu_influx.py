"""Device synthesis of seeded JONSWAP influx signals for an ensemble
(hw_jonswap_influx: jonswap_influx, 1d/influx_lib.c:137-255) against the oracle's
restatement, members of even and odd sample counts in one launch."""
import numpy as np
import pytest

from hawassi_c_b200.engine import jonswap_influx
import oracle_lib as ol

pytestmark = pytest.mark.gpu


def test_jonswap_influx_matches_oracle():
    rng = np.random.default_rng(4)
    specs = []
    grids = [(60.0, 0.05), (63.9375, 0.0625), (100.0, 0.04), (127.9375, 0.0625)]   # 1201, 1024, 2501, 2048 samples
    for m in range(12):
        Tend, dt = grids[m % 4]
        specs.append(dict(T0=0.0, Tend=Tend, dt=dt,
                          Tp=float(rng.uniform(1.5, 3.0)), Hs=float(rng.uniform(0.05, 0.2)),
                          gamma=float(rng.uniform(1.0, 5.0)), nTramp=4.0 if m % 3 else 2.0, seed=1000 + m))
    got = jonswap_influx(specs)
    sizes = set()
    for sp, g in zip(specs, got):
        ref = ol.jonswap_signal(sp["T0"], sp["Tend"], sp["dt"], sp["Tp"], sp["Hs"], sp["gamma"], sp["nTramp"],
                                sp["seed"])
        assert g.size == ref.size
        sizes.add(ref.size % 2)
        assert np.abs(g - ref).max() <= 1e-11 * np.abs(ref).max()
        # normalised to Hs = 4 std
        assert abs(4 * g.std() - sp["Hs"]) < 1e-12
    assert sizes == {0, 1}


def test_ensemble_jonswap_decks_use_device_signals(tmp_path):
    """An ensemble of jonswap decks: member m's signal comes from the device synthesis
    with seed + m; its RHS during the influx equals the oracle's built with that seed."""
    import hawassi_c_b200 as hw
    from hawassi_c_b200 import decks
    from decks_util import random_state, rel_l2
    paths = []
    for m in range(3):
        paths.append(decks.write_deck(str(tmp_path / f"js{m}"), nx=1024, length=51.2, xinflux=8.0, depth=1.0,
                                      model="HS2", T_end=20.0, Hs=0.08, Tp=1.3 + 0.2 * m, gamma=3.3,
                                      wavename="jonswap", damp=(4.0, 4.0), dt=0.02))
    base = 77
    e = hw.Engine(paths, eps_abs=1e-8, eps_rel=1e-6, seed=base, device=0)
    y = random_state(1024, 3)
    for m, p in enumerate(paths):
        o = ol.Oracle(p, eps_abs=1e-8, eps_rel=1e-6, seed=base + m)
        ref = o.rhs(9.7, y)
        assert rel_l2(e.rhs(9.7, y, member=m), ref) < 1e-11
        o.close()
    e.close()
