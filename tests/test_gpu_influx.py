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
