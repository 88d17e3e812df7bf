"""Batched state transfers of a ragged ensemble (hw_set_states / hw_get_states):
one host copy and one layout kernel for every member, against the per-member
read-back and a per-member restart."""
import numpy as np
import pytest

from decks_util import small_deck

pytestmark = pytest.mark.gpu

hw = pytest.importorskip("hawassi_c_b200")


def test_batched_states_round_trip_and_restart(tmp_path):
    decks = [small_deck(tmp_path, f"s{i}", nx=nx, T_end=3.0, seed=10 + i)
             for i, nx in enumerate((1024, 4096, 2048))]
    e = hw.Engine(decks, eps_abs=1e-8, eps_rel=1e-6)
    e.run(20)                                              # move every member off its initial state
    tot = sum(4 * n for n in e.nx)
    got = e.get_states(np.empty(tot))
    per = np.concatenate([e.state(m)[2] for m in range(e.members)])
    assert np.array_equal(got, per)
    # a modified ensemble state goes in and comes back unchanged
    mod = got * 0.5
    e.set_states(mod)
    back = e.get_states(np.empty(tot))
    assert np.array_equal(back, mod)
    # continuing from the batched state equals continuing from per-member sets
    e.run(40)
    a = e.get_states(np.empty(tot))
    f = hw.Engine(decks, eps_abs=1e-8, eps_rel=1e-6)
    f.run(20)
    off = 0
    for m in range(f.members):
        t, h, _ = f.state(m)
        f.set_state(t, h, mod[off:off + 4 * f.nx[m]], member=m, i_out=20)
        off += 4 * f.nx[m]
    f.run(40)
    b = f.get_states(np.empty(tot))
    assert np.array_equal(a, b)


@pytest.mark.parametrize("resident", [-1, 2])
def test_persistent_grid_matches_one_cluster_per_member(tmp_path, resident):
    """The persistent evolve grid (clusters pulling members from the class's work
    queue; resident -1 sizes it to the class's share of the GPU, 2 allows two clusters
    per class so each cluster runs several members in turn) gives every member the
    bit-identical state, step counts and breaking log of one cluster per member."""
    decks = [small_deck(tmp_path, f"q{i}", nx=nx, T_end=3.0, seed=20 + i, breaking=bool(i % 2))
             for i, nx in enumerate((1024, 4096, 2048, 4096, 1024, 4096, 2048))]
    runs = []
    for r in (0, resident):
        e = hw.Engine(decks, eps_abs=1e-8, eps_rel=1e-6, resident=r)
        e.run(30)
        tot = sum(4 * n for n in e.nx)
        runs.append((e.get_states(np.empty(tot)), [e.stats(m) for m in range(e.members)],
                     [e.breaking_log(m) for m in range(e.members)]))
        e.close()
    assert np.array_equal(runs[0][0], runs[1][0])
    assert runs[0][1] == runs[1][1]
    assert runs[0][2] == runs[1][2]
