"""The autotuner of the batched runner: it times the candidate slice sizes per grid
size on the device, and the tuned ensemble computes what the default one does."""
import numpy as np
import pytest

from decks_util import rel_l2, small_deck

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


def test_autotune_picks_valid_slices_and_keeps_results(tmp_path):
    from hawassi_c_b200.autotune import autotune_slices
    decks = [small_deck(tmp_path, f"a{i}", nx=nx, T_end=2.0, seed=20 + i)
             for i, nx in enumerate((2048, 2048, 4096, 4096))]
    best, trials = autotune_slices(decks, candidates=(2048, 1024, 512), window=3, warm=1)
    assert set(best) == {2048, 4096}
    assert all(nx % s == 0 for nx, s in best.items())
    assert len(trials) >= 5                             # start + two alternatives per class
    rates = {tuple(sorted(t.items())): v for t, v in trials}
    assert rates[tuple(sorted(best.items()))] == max(v for _, v in trials)
    a = hw.Engine(decks, eps_abs=1e-8, eps_rel=1e-6)
    b = hw.Engine(decks, eps_abs=1e-8, eps_rel=1e-6, slices={2048: 512, 4096: 1024})
    a.run(30)
    b.run(30)
    for m in range(4):
        ta, _, ya = a.state(m)
        tb, _, yb = b.state(m)
        assert ta == tb
        assert rel_l2(yb, ya) < 1e-9
